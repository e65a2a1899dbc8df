"""Learned refinement predictor on the GPU: the tcgen05 GEMM behind its
layers, the per-block features, the loss and gradients of the CUDA forward /
backward pass against the numpy restatement (oracle/learn_net.py, BF16
rounding at the same points), training on snapshots the plain percentile
criterion labels, and the predictor driving a case's refinement with the
plain criterion as judge."""
import ctypes as C

import numpy as np
import pytest

from helpers import lattice, macros_from_F
from oracle import learn_net as ln
from test_gpu_amr import amr_params
from test_oracle import run_like_reference

import agal_b200 as ag
from agal_b200 import _lib

pytestmark = pytest.mark.gpu


def bf16_bits(x):
    """Round-to-nearest-even FP32 -> BF16 bit patterns, and the rounded values."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    return r, (r.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.parametrize("M,N,K", [(128, 32, 16), (300, 32, 288), (1000, 17, 864), (64, 8, 80)])
def test_tcgen05_gemm_matches_numpy(M, N, K):
    rng = np.random.default_rng(M + N + K)
    a_bits, a = bf16_bits(rng.standard_normal((M, K)))
    b_bits, b = bf16_bits(rng.standard_normal((N, K)))
    d = np.zeros((M, N), np.float32)
    rc = _lib.lib().agal_learn_gemm_bf16(a_bits.ctypes.data_as(C.c_void_p), b_bits.ctypes.data_as(C.c_void_p),
                                        d.ctypes.data_as(C.c_void_p), M, N, K)
    assert rc == 0
    ref = a.astype(np.float64) @ b.astype(np.float64).T
    # products of BF16 values are exact in FP32; only the FP32 accumulation rounds
    assert np.abs(d - ref).max() <= 1e-5 * np.abs(ref).max() + 1e-5


# ---- cases ------------------------------------------------------------------
def learn_params(Q, N, **kw):
    base = dict(S_CRITERION=_lib.CRITERION_PERCENTILE, P_REFINE=8,
                MAX_LEVELS_INTERIOR=3 if Q == 9 else 2, v0=5e-4 if Q == 9 else 2.5e-4)
    base.update(kw)
    return amr_params(Q, N, **base)


def collect(Q, N, steps, seed=1, horizon=None, **kw):
    """A learner in collect mode over a plain percentile-criterion run
    (horizon None: the one-regrid-delayed mode)."""
    p = learn_params(Q, N, **kw)
    c = ag.Case(p)
    m = ag.Learner(2 if Q == 9 else 3, seed=seed)
    if horizon is not None:
        m.set_horizon(horizon)
    m.attach(c, 1)
    run_like_reference(c, p, steps)
    c.sync()
    return p, c, m


def active_ids(c):
    cnt = c.counts()
    ids = c.dump(_lib.ARR_ID_SET).reshape(cnt["max_levels"], cnt["n_maxcblocks"])
    return np.concatenate([ids[L, :cnt["n_ids"][L]] for L in range(cnt["max_levels"])]).astype(np.int64)


def features_numpy(c, p):
    """The 8 input channels of every active block from the dumped populations."""
    Q, dim, MC = c.Q, c.dim, c.M_CBLOCK
    ids = active_ids(c)
    nmb = c.counts()["n_maxcblocks"]
    F = c.dump(_lib.ARR_F).reshape(Q, nmb, MC)[:, ids, :].reshape(Q, -1)
    pb, cv, _ = lattice(Q)
    rho, u = macros_from_F(F, dim, Q, pb, cv)
    U = np.float32(p.u_ref)
    su = np.stack([(u[a].astype(np.float32) / U).reshape(-1, MC) for a in range(dim)]
                  + ([] if dim == 3 else [np.zeros((len(ids), MC), np.float32)]))
    cell = np.arange(MC)
    pos = [cell & 3, (cell >> 2) & 3, cell >> 4]

    def d(comp, axis):
        step = (1, 4, 16)[axis]
        lo = np.where(pos[axis] > 0, cell - step, cell)
        hi = np.where(pos[axis] < 3, cell + step, cell)
        den = ((pos[axis] > 0).astype(np.float32) + (pos[axis] < 3).astype(np.float32))
        return (su[comp][:, hi] - su[comp][:, lo]) / den

    if dim == 2:
        om = np.abs(d(1, 0) - d(0, 1))
    else:
        om = np.sqrt((d(2, 1) - d(1, 2)) ** 2 + (d(0, 2) - d(2, 0)) ** 2 + (d(1, 0) - d(0, 1)) ** 2)
    lev = c.dump(_lib.ARR_CBLOCK_LEVEL)[ids]
    ref = c.dump(_lib.ARR_CBLOCK_ID_REF)[ids]
    ml = c.counts()["max_levels"]
    X = np.zeros((len(ids), MC, 8), np.float32)
    X[..., 0] = ((rho - 1.0).astype(np.float32) / (U * U)).reshape(-1, MC)
    for a in range(3):
        X[..., 1 + a] = su[a]
    X[..., 4] = om * (2.0 ** lev).astype(np.float32)[:, None]
    X[..., 5] = (lev / max(ml - 1, 1)).astype(np.float32)[:, None]
    X[..., 6] = np.isin(ref, (1, 2)).astype(np.float32)[:, None]
    X[..., 7] = 1.0
    return X.reshape(-1, 8)


@pytest.mark.parametrize("Q,N", [(9, 32), (19, 16)])
def test_features_match_populations(Q, N):
    p = learn_params(Q, N)
    with ag.Case(p) as c, ag.Learner(2 if Q == 9 else 3, seed=1) as m:
        run_like_reference(c, p, 24)
        c.sync()
        assert c.counts()["n_ids"][1] > 0
        m.record(c)
        X, _, _ = m.snapshot(0)
        Xr = features_numpy(c, p)
        assert X.shape == Xr.shape
        assert np.allclose(X, Xr, rtol=1e-5, atol=2e-6)


def labelled_with_marks(m):
    """Labelled snapshots holding refinement or coarsening marks, most recent last."""
    out = []
    for k in range(m.counts()["labelled"]):
        _, Y, W = m.snapshot(k)
        if W.sum() > 0 and (Y * W[:, None]).sum() > 0:
            out.append(k)
    return out


@pytest.mark.parametrize("Q,N,steps,mli", [(9, 32, 48, 3), (19, 16, 48, 3)])
def test_gradients_match_numpy(Q, N, steps, mli):
    """Loss and gradient of the CUDA pass against the numpy network with the
    same BF16 rounding: loss within 1e-4, every parameter block within 5e-3
    relative L2; and within 5e-2 of the exact FP64 gradient."""
    p, c, m = collect(Q, N, steps, MAX_LEVELS_INTERIOR=mli)
    try:
        ks = labelled_with_marks(m)
        assert ks, m.counts()
        k = ks[-1]
        pw = m.balance_classes(0, k + 1)
        # move off the initial weights so that every ReLU pattern is exercised
        m.train(0, k, 2, lr=1e-3, seed=3)
        w = m.get_params()
        X, Y, W = m.snapshot(k)
        loss, g = m.gradients(k)
        z_np, l_np, g_np = ln.forward_backward(w, X, m.dim, Y, W, pos_weight=pw)
        assert abs(loss - l_np) <= 1e-4 * abs(l_np)
        parts = ln.split(np.arange(m.num_params), m.dim)
        for name, idx in parts.items():
            a, b = g[idx.ravel()], g_np[idx.ravel()]
            assert np.linalg.norm(a - b) <= 5e-3 * np.linalg.norm(b) + 1e-9, name
        _, _, g64 = ln.forward_backward(w, X, m.dim, Y, W, bf16_emulation=False, pos_weight=pw)
        assert np.linalg.norm(g - g64) <= 5e-2 * np.linalg.norm(g64)
        z = m.predict(k)
        assert np.abs(z - z_np).max() <= 1e-3 * max(1.0, np.abs(z_np).max())
    finally:
        m.attach(c, 0)
        m.close()
        c.close()


@pytest.mark.parametrize("Q,N", [(9, 32), (19, 16)])
def test_implicit_gemm_logits_equal_im2col(Q, N):
    """Inference convolutions as implicit GEMMs (columns gathered into the
    tensor-core GEMM's shared memory) give the logits of the im2col path bit
    for bit, on every snapshot of a run, after some training."""
    p, c, m = collect(Q, N, 48 if Q == 9 else 24, MAX_LEVELS_INTERIOR=3 if Q == 9 else 2)
    try:
        n, nl = m.counts()["snapshots"], m.counts()["labelled"]
        assert n > 0 and nl > 0
        m.train(0, nl, 1, lr=1e-3, seed=5)
        for k in range(n):
            m.set_implicit(True)
            a = m.predict(k)
            m.set_implicit(False)
            b = m.predict(k)
            assert a.shape == b.shape and len(a) > 0
            assert np.array_equal(a, b), k
    finally:
        m.attach(c, 0)
        m.close()
        c.close()


def f1(pred, true):
    tp = (pred & true).sum()
    return 2.0 * tp / max(pred.sum() + true.sum(), 1)


CHANNEL = dict(bc_preset=_lib.BC_FPSC2D, ic_preset=_lib.IC_UNIFORM, ic_noise=0.3, v0=1e-4,
               storage=_lib.STORE_FP32, MAX_LEVELS_INTERIOR=3)


def test_training_gain_over_untrained_and_persistence():
    """Channel flow carrying seeded perturbations downstream, a regrid every
    8 steps.  Trained on the earlier snapshots, the network predicts the
    percentile rule's refinement decisions at the next regrid on the later
    (held-out) snapshots far better than before training, and at least as
    well as the rule itself applied to the same (8 steps older) state - the
    marks a solver that adapts from its last criterion run would use."""
    p, c, m = collect(9, 64, 480, **CHANNEL)
    try:
        nl = m.counts()["labelled"]
        assert nl >= 50
        split = int(nl * 0.7)
        snaps = [m.snapshot(k) for k in range(nl)]
        test_ks = range(split, nl)

        def score(pred_fn, out=0):
            P_, T_ = [], []
            for k in test_ks:
                X, Y, W = snaps[k]
                v = W > 0
                P_.append(pred_fn(k)[v, out] > 0)
                T_.append(Y[v, out] > 0.5)
            return f1(np.concatenate(P_), np.concatenate(T_))

        pw = m.balance_classes(0, split)
        f1_untrained = score(m.predict)
        loss0 = np.mean([m.gradients(k)[0] for k in test_ks])
        m.train(0, split, 40, lr=2e-3, seed=11)
        loss1 = np.mean([m.gradients(k)[0] for k in test_ks])
        f1_trained, f1c_trained = score(m.predict), score(m.predict, 1)
        f1_persist = score(lambda k: m.decisions(k) - 0.5)
        f1c_persist = score(lambda k: m.decisions(k) - 0.5, 1)
        print(f"class weights ({pw[0]:.2f}, {pw[1]:.2f}); held-out F1 of the refinement decision: untrained "
              f"{f1_untrained:.3f}, trained {f1_trained:.3f}, rule on the older state {f1_persist:.3f}; "
              f"coarsening decision: trained {f1c_trained:.3f}, rule on the older state {f1c_persist:.3f}; "
              f"loss {loss0:.4f} -> {loss1:.4f}")
        assert loss1 < 0.7 * loss0
        assert f1_trained > f1_untrained + 0.1
        assert f1_trained >= f1_persist - 0.02
    finally:
        m.attach(c, 0)
        m.close()
        c.close()


def test_predict_mode_judged_refinement():
    """A trained network drives the refinement of a fresh run; the plain
    criterion judges every 4th regrid, counting and applying the refinement
    marks the network did not predict.  The mesh stays within a factor 2 of
    the plain run's and the flow stays bounded.  (The missed fraction is
    printed, not bounded: the marks of a regrid are the few blocks crossing the
    rule's quantile, which the network predicts poorly.)"""
    p, c, m = collect(9, 64, 320, **CHANNEL)
    try:
        nl = m.counts()["labelled"]
        plain_ids = c.counts()["n_ids"]
        m.balance_classes(0, nl)
        m.train(0, nl, 30, lr=2e-3, seed=5)
        thr = m.calibrate_thresholds(0, nl)
        m.attach(c, 0)
        c.close()
        with ag.Case(p) as c2:
            m.attach(c2, 2, judge_every=4)
            m.set_thresholds(*thr)
            run_like_reference(c2, p, 320)
            c2.sync()
            cnt = m.counts()
            ids = c2.counts()["n_ids"]
            print(f"thresholds {thr}; judged {cnt['judged']} of {cnt['regrids']} regrids, missed {cnt['missed']} of "
                  f"{cnt['plain_refine']} plain refinement marks; blocks per level {ids} (plain run {plain_ids})")
            assert cnt["regrids"] == 320 // p.P_REFINE
            assert cnt["judged"] >= cnt["regrids"] // 4
            assert 0 <= cnt["missed"] <= cnt["plain_refine"]
            assert 0.5 * sum(plain_ids[1:]) <= sum(ids[1:]) <= 2.0 * sum(plain_ids[1:])
            mm = c2.mass_momentum()
            assert np.isfinite(mm).all()
            m.attach(c2, 0)
    finally:
        m.close()


def test_horizon_labels_cover_later_regrids():
    """Look-ahead labels over 3 regrids against the same (deterministic) run
    labelled over 1: a block the rule refines at the snapshot's regrid is
    labelled for refinement, one it does not coarsen there is not labelled
    for coarsening, and a block that changes level within the horizon carries
    no weight; the last 2 snapshots stay unlabelled."""
    out = {}
    for h in (1, 3):
        p, c, m = collect(9, 64, 160, horizon=h, **CHANNEL)
        try:
            cnt = m.counts()
            out[h] = (cnt, [m.snapshot(k) for k in range(cnt["labelled"])])
        finally:
            m.attach(c, 0)
            m.close()
            c.close()
    (c1, s1), (c3, s3) = out[1], out[3]
    assert c1["snapshots"] == c3["snapshots"] == 160 // 8
    assert c1["labelled"] == c1["snapshots"] and c3["labelled"] == c3["snapshots"] - 2
    wider = 0
    for (X1, Y1, W1), (X3, Y3, W3) in zip(s1, s3):
        assert np.array_equal(X1, X3)                      # the same states
        assert np.all(W3 <= W1)
        v = W3 > 0
        assert np.all(Y3[v, 0] >= Y1[v, 0])               # refine: any of the regrids
        assert np.all(Y3[v, 1] <= Y1[v, 1])               # coarsen: all of them
        wider += int((Y3[v, 0] > Y1[v, 0]).sum())
    assert wider > 0                                       # the horizon adds refinement labels


def test_predict_ahead_regrids_less_often():
    """A network trained on labels covering 4 regrids drives a run that
    regrids 4 times less often (P_REFINE x 4), predicting at each regrid for
    that regrid, the rule judging every regrid: the regrid count drops 4x, the
    missed fraction is reported, the mesh stays within a factor 2 of the plain
    run's and the flow stays bounded."""
    p, c, m = collect(9, 64, 320, horizon=4, **CHANNEL)
    try:
        nl = m.counts()["labelled"]
        plain_ids = c.counts()["n_ids"]
        m.balance_classes(0, nl)
        m.train(0, nl, 30, lr=2e-3, seed=5)
        thr = m.calibrate_thresholds(0, nl)
        m.attach(c, 0)
        c.close()
        p.P_REFINE *= 4
        with ag.Case(p) as c2:
            m.attach(c2, 2, judge_every=1)
            m.set_thresholds(*thr)
            run_like_reference(c2, p, 320)
            c2.sync()
            cnt = m.counts()
            ids = c2.counts()["n_ids"]
            frac = cnt["missed"] / max(cnt["plain_refine"], 1)
            print(f"horizon 4: {cnt['regrids']} regrids (plain run 40), missed {cnt['missed']} of "
                  f"{cnt['plain_refine']} plain refinement marks ({frac:.2f}); blocks {ids} (plain {plain_ids})")
            assert cnt["regrids"] == 320 // p.P_REFINE == 10
            assert cnt["judged"] == cnt["regrids"]
            assert 0 <= cnt["missed"] <= cnt["plain_refine"]
            assert 0.5 * sum(plain_ids[1:]) <= sum(ids[1:]) <= 2.0 * sum(plain_ids[1:])
            assert np.isfinite(c2.mass_momentum()).all()
            m.attach(c2, 0)
    finally:
        m.close()


def test_attach_rejects_mismatch():
    p = learn_params(9, 32)
    with ag.Case(p) as c, ag.Learner(3, seed=0) as m:
        with pytest.raises(ag.AgalError):
            m.attach(c, 2)
        with ag.Learner(2, seed=0) as m2:
            with pytest.raises(ag.AgalError):
                m2.attach(c, 3)
            w = m2.get_params()
            with pytest.raises(ag.AgalError):
                m2.set_params(w[:-1])
