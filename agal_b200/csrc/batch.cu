// Batched execution of independent cases.
//
// A batch advances many contexts (cases of any size, level count, velocity
// set, precision and boundary) together: one CUDA graph per coarse step holds
// every case's launches as its own branch (fork from a master stream, each
// case recorded on its own stream, join back), so the GPU runs the small,
// latency-bound kernels of different cases concurrently instead of one case
// after another.  Each case keeps its own mesh, buffers and parity; results
// are identical to advancing the cases one at a time (the same launches in
// the same per-case order).  The solution-based refinement of a multi-level
// case runs between graph replays on its own stream, every P_REFINE coarse
// steps as in M_AdvanceLoop (mesh_advance.cu:421-463); a regrid invalidates
// the batch graphs.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "ctx.h"

struct agal_batch {
    std::vector<agal_ctx *> cases;
    cudaStream_t master = nullptr;
    cudaEvent_t fork = nullptr, done = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    std::vector<std::vector<int>> graph_cur[2];   // every case's cur[] at capture
    std::string err;
};

namespace {

int berr(agal_batch *b, int code, const std::string &m)
{
    if (b) b->err = m;
    return code;
}

int bcuda(agal_batch *b, cudaError_t e, const char *what)
{
    return berr(b, e == cudaErrorMemoryAllocation ? AGAL_ERR_OOM : AGAL_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

#define BCUDA(b, call)                                   \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return bcuda((b), e_, #call); \
    } while (0)

void drop(agal_batch *b)
{
    for (int k = 0; k < 2; k++) {
        if (b->graph[k]) cudaGraphExecDestroy(b->graph[k]);
        b->graph[k] = nullptr;
        b->graph_cur[k].clear();
    }
}

std::vector<std::vector<int>> curs(const agal_batch *b)
{
    std::vector<std::vector<int>> v;
    v.reserve(b->cases.size());
    for (const agal_ctx *c : b->cases) v.push_back(c->cur);
    return v;
}

bool multi_level(const agal_ctx *c) { return c->max_levels > 1 && c->max_levels != c->L0 + 1; }

// One coarse step of every case, each on its own stream, joined on the master.
int record_step(agal_batch *b)
{
    BCUDA(b, cudaEventRecord(b->fork, b->master));
    for (size_t i = 0; i < b->cases.size(); i++) {
        agal_ctx *c = b->cases[i];
        BCUDA(b, cudaStreamWaitEvent(c->stream, b->fork, 0));
        const int rc = agal_record_coarse_step(c);
        if (rc) return berr(b, rc, "case " + std::to_string(i) + ": " + c->err);
        BCUDA(b, cudaEventRecord(b->join[i], c->stream));
        BCUDA(b, cudaStreamWaitEvent(b->master, b->join[i], 0));
    }
    return AGAL_OK;
}

int capture(agal_batch *b, cudaGraphExec_t *out)
{
    std::vector<std::vector<int>> cur0 = curs(b);
    cudaGraph_t g = nullptr;
    BCUDA(b, cudaStreamBeginCapture(b->master, cudaStreamCaptureModeThreadLocal));
    int rc = record_step(b);
    cudaError_t e = cudaStreamEndCapture(b->master, &g);
    for (size_t i = 0; i < b->cases.size(); i++) b->cases[i]->cur = cur0[i];   // only recorded
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return bcuda(b, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return bcuda(b, e, "cudaGraphInstantiate");
    return AGAL_OK;
}

}  // namespace

extern "C" int agal_batch_create(agal_ctx *const *cases, int n_cases, agal_batch **out)
{
    if (!cases || !out || n_cases <= 0) return AGAL_ERR_PARAM;
    *out = nullptr;
    int dev = -1;
    for (int i = 0; i < n_cases; i++) {
        if (!cases[i]) return AGAL_ERR_PARAM;
        if (dev < 0) dev = cases[i]->device;
        if (cases[i]->device != dev) return AGAL_ERR_PARAM;   // one device per batch
        for (int j = 0; j < i; j++)
            if (cases[j] == cases[i]) return AGAL_ERR_PARAM;
    }
    agal_batch *b = new agal_batch();
    b->cases.assign(cases, cases + n_cases);
    cudaSetDevice(dev);
    bool ok = cudaStreamCreateWithFlags(&b->master, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) == cudaSuccess;
    b->join.assign(n_cases, nullptr);
    for (int i = 0; ok && i < n_cases; i++) ok = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        agal_batch_destroy(b);
        return AGAL_ERR_CUDA;
    }
    *out = b;
    return AGAL_OK;
}

extern "C" int agal_batch_destroy(agal_batch *b)
{
    if (!b) return AGAL_ERR_PARAM;
    if (b->master) cudaStreamSynchronize(b->master);
    drop(b);
    for (cudaEvent_t e : b->join)
        if (e) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->done) cudaEventDestroy(b->done);
    if (b->master) cudaStreamDestroy(b->master);
    delete b;
    return AGAL_OK;
}

extern "C" const char *agal_batch_last_error(const agal_batch *b) { return b ? b->err.c_str() : ""; }

// n coarse steps of every case.  use_graph replays one captured step of the
// whole batch (two cached, for the alternating buffer parities).
extern "C" int agal_batch_advance_n(agal_batch *b, int n, int use_graph)
{
    if (!b || n < 0) return AGAL_ERR_PARAM;
    int rc;
    // Work already queued on the case streams precedes the batch.
    for (size_t i = 0; i < b->cases.size(); i++) {
        BCUDA(b, cudaEventRecord(b->join[i], b->cases[i]->stream));
        BCUDA(b, cudaStreamWaitEvent(b->master, b->join[i], 0));
    }
    for (int s = 0; s < n; s++) {
        if (use_graph) {
            const std::vector<std::vector<int>> now = curs(b);
            int k = (b->graph[0] && b->graph_cur[0] == now) ? 0 : (b->graph[1] && b->graph_cur[1] == now) ? 1 : -1;
            if (k < 0) {
                k = b->graph[0] ? 1 : 0;
                if (b->graph[k]) { cudaGraphExecDestroy(b->graph[k]); b->graph[k] = nullptr; }
                if ((rc = capture(b, &b->graph[k]))) return rc;
                b->graph_cur[k] = now;
            }
            BCUDA(b, cudaGraphLaunch(b->graph[k], b->master));
            for (agal_ctx *c : b->cases) agal_advance_parity(c, 1);
        } else {
            if ((rc = record_step(b))) return rc;
        }
        // Solution-based refinement of the cases that are due, on their own
        // streams after this step.
        bool regrid = false;
        BCUDA(b, cudaEventRecord(b->done, b->master));
        for (size_t i = 0; i < b->cases.size(); i++) {
            agal_ctx *c = b->cases[i];
            const long long it = c->iter;
            if (multi_level(c) && c->P.P_REFINE > 0 && (it + 1) % c->P.P_REFINE == 0 && it > 0) {
                BCUDA(b, cudaStreamWaitEvent(c->stream, b->done, 0));
                if ((rc = agal_refine_with_solution(c))) return berr(b, rc, "case " + std::to_string(i) + ": " + c->err);
                BCUDA(b, cudaEventRecord(b->join[i], c->stream));
                BCUDA(b, cudaStreamWaitEvent(b->master, b->join[i], 0));
                regrid = true;
            }
            c->iter++;
        }
        if (regrid) drop(b);
    }
    // Later work on a case stream follows the batch.
    BCUDA(b, cudaEventRecord(b->done, b->master));
    for (agal_ctx *c : b->cases) BCUDA(b, cudaStreamWaitEvent(c->stream, b->done, 0));
    return AGAL_OK;
}

extern "C" int agal_batch_sync(agal_batch *b)
{
    if (!b) return AGAL_ERR_PARAM;
    BCUDA(b, cudaStreamSynchronize(b->master));
    for (size_t i = 0; i < b->cases.size(); i++) {
        const int rc = agal_sync(b->cases[i]);
        if (rc) return berr(b, rc, "case " + std::to_string(i) + ": " + b->cases[i]->err);
    }
    return AGAL_OK;
}

extern "C" int agal_batch_get_stream(const agal_batch *b, void **stream)
{
    if (!b || !stream) return AGAL_ERR_PARAM;
    *stream = (void *)b->master;
    return AGAL_OK;
}
