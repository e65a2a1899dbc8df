"""The CPU restatement of the learned refinement predictor (oracle/learn_net.py)
checked on its own: exact FP64 gradients against central differences, the
im2col / col2im pair adjoint, BF16 rounding to nearest even."""
import numpy as np
import pytest

from oracle import learn_net as ln


def _case(dim, n, seed):
    rng = np.random.default_rng(seed)
    P = ln.geometry(dim)[0]
    X = rng.standard_normal((n * P, ln.C0))
    X[:, 7] = 1.0
    Y = (rng.random((n, 2)) < 0.4).astype(np.float64)
    Wt = np.ones(n)
    Wt[0] = 0.0                      # a block that no longer exists carries no weight
    return X, Y, Wt


@pytest.mark.parametrize("dim,pw", [(2, (1.0, 1.0)), (3, (1.0, 1.0)), (2, (7.5, 3.0))])
def test_exact_gradient_matches_finite_differences(dim, pw):
    X, Y, Wt = _case(dim, 3 if dim == 2 else 2, 7 + dim)
    w = ln.init_params(dim, seed=dim)
    w[ln.split(np.arange(len(w)), dim)["b1"]] = 0.05
    _, loss, g = ln.forward_backward(w, X, dim, Y, Wt, bf16_emulation=False, pos_weight=pw)
    assert np.isfinite(loss)
    parts = ln.split(np.arange(len(w)), dim)
    rng = np.random.default_rng(dim)
    K1 = ln.geometry(dim)[2]
    idx = np.concatenate([rng.choice(parts["W1"][:, :K1].ravel(), 6), rng.choice(parts["W2"].ravel(), 6),
                          rng.choice(parts["W3"].ravel(), 6), parts["b1"][:3], parts["b2"][:3], parts["b3"]])
    fd = ln.finite_difference(w, X, dim, Y, Wt, idx, pos_weight=pw)
    assert np.abs(fd - g[idx]).max() <= 1e-6 * max(1.0, np.abs(g[idx]).max())
    assert (g[parts["W1"][:, K1:].ravel()] == 0).all()     # padding columns get no gradient


@pytest.mark.parametrize("dim", [2, 3])
def test_im2col_col2im_adjoint(dim):
    rng = np.random.default_rng(dim)
    n, C = 3, 5
    P, T = ln.geometry(dim)[:2]
    H = rng.standard_normal((n * P, C))
    D = rng.standard_normal((n * P, T * C))
    assert np.isclose((ln.im2col(H, dim, n) * D).sum(), (H * ln.col2im(D, dim, n, C)).sum(), rtol=1e-12)
    # centre tap is the cell itself; a corner cell sees 2^d of the 3^d taps
    X = ln.im2col(H, dim, n)
    centre = T // 2
    assert np.array_equal(X[:, centre * C:(centre + 1) * C], H)
    assert (np.abs(X[0].reshape(T, C)).sum(axis=1) > 0).sum() == 2 ** dim


def test_bf16_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 1.0 + 2.0 ** -9, -2.5, 0.0, 3.0e38], np.float32)
    r = ln.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0                    # tie to even
    assert r[2] == np.float32(1.0 + 4 * 2.0 ** -8)        # tie to even, upwards
    assert r[3] == 1.0 and r[4] == -2.5 and r[5] == 0.0
    assert (r.view(np.uint32) & 0xFFFF == 0).all()


@pytest.mark.parametrize("dim", [2, 3])
def test_bf16_emulation_close_to_exact(dim):
    """The BF16 network is the exact one within BF16 resolution (a few 1e-3)."""
    X, Y, Wt = _case(dim, 4, 11 + dim)
    w = ln.init_params(dim, seed=3)
    z64, l64, g64 = ln.forward_backward(w, X, dim, Y, Wt, bf16_emulation=False)
    z16, l16, g16 = ln.forward_backward(w, X, dim, Y, Wt, bf16_emulation=True)
    assert abs(l16 - l64) <= 2e-2 * abs(l64)
    assert np.linalg.norm(g16 - g64) <= 5e-2 * np.linalg.norm(g64)
