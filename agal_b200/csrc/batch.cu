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
//
// Work-list mode (the default when every case allows it): the fused steps of
// all cases are one launch per phase.  A coarse step of every case is first
// recorded, not launched (agal_ctx::rec): each launcher appends its launch to
// the case's list.  The lists are merged into one sequence of phases that
// keeps every case's own order (a phase is one launch kind at one level, e.g.
// the second sub-step of level 1); a step phase is one persistent kernel over
// the chunks of every case stepping in it (k_step_batch, a global work list
// of (case, chunk) with each case's arguments in a device table), then the
// wall steps of the cases that have walls, then one batched fix-up launch;
// an interpolation or averaging phase is one launch over (case, parent block)
// items; the other phases (forces, the rounding counter) run each case's
// launch on its own stream.  Every case's kernels and their
// order are those of advancing it alone, so the results are identical.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "ctx.h"
#include "step_common.cuh"

// A launch recorded for the batch: a fused step (kind 0) or a closure.
struct agal_op {
    int kind = 0;              // 0: fused step; else AGAL_OP_*
    int L = 0;
    int key = 0;               // fused step: batched-kernel key
    int n_blocks = 0;          // fused step: blocks of the level
    agal::StepArgs step{};
    std::vector<unsigned char> args;   // transfers: the argument structure
    int n_items = 0;                   // transfers: blocks of the launch
    const void *fin = nullptr;
    void *fout = nullptr;
    std::function<int(agal_ctx *)> fn;
    // the case's launch state when the launch was recorded (launchers read
    // the buffer parities and the rounding salt when they launch)
    std::vector<int> cur;
    int sr_salt = 0, liter = 0;
};

// Issue a recorded closure (or a step's wall step) in the launch state it was
// recorded in.
static int run_in_state(agal_ctx *c, const agal_op &op, const std::function<int(agal_ctx *)> &fn)
{
    const std::vector<int> cur = c->cur;
    const int salt = c->sr_salt, liter = c->liter;
    c->cur = op.cur;
    c->sr_salt = op.sr_salt;
    c->liter = op.liter;
    const int rc = fn(c);
    c->cur = cur;
    c->sr_salt = salt;
    c->liter = liter;
    return rc;
}
struct agal_oplist {
    std::vector<agal_op> ops;
};

int agal_record_step(agal_ctx *c, int L, const void *args, size_t bytes, int key, int n_blocks, const void *fin,
                     void *fout)
{
    if (bytes != sizeof(agal::StepArgs)) return agal_set_err(c, AGAL_ERR_PARAM, "batch: step arguments size");
    agal_op op;
    op.L = L;
    op.key = key;
    op.n_blocks = n_blocks;
    std::memcpy(&op.step, args, bytes);
    op.fin = fin;
    op.fout = fout;
    op.cur = c->cur;
    op.sr_salt = c->sr_salt;
    op.liter = c->liter;
    c->rec->ops.push_back(std::move(op));
    return AGAL_OK;
}

int agal_record_args(agal_ctx *c, int kind, int L, const void *args, size_t bytes, int key, int n_items)
{
    if (bytes != agal_transfer_args_size(kind)) return agal_set_err(c, AGAL_ERR_PARAM, "batch: transfer arguments size");
    agal_op op;
    op.kind = kind;
    op.L = L;
    op.key = key;
    op.n_items = n_items;
    op.args.assign(static_cast<const unsigned char *>(args), static_cast<const unsigned char *>(args) + bytes);
    op.cur = c->cur;
    op.sr_salt = c->sr_salt;
    op.liter = c->liter;
    c->rec->ops.push_back(std::move(op));
    return AGAL_OK;
}

int agal_record_other(agal_ctx *c, int tag, int L, std::function<int(agal_ctx *)> fn)
{
    agal_op op;
    op.kind = tag;
    op.L = L;
    op.fn = std::move(fn);
    op.cur = c->cur;
    op.sr_salt = c->sr_salt;
    op.liter = c->liter;
    c->rec->ops.push_back(std::move(op));
    return AGAL_OK;
}

struct agal_batch {
    std::vector<agal_ctx *> cases;
    cudaStream_t master = nullptr;
    cudaEvent_t fork = nullptr, done = nullptr;
    std::vector<cudaEvent_t> join;
    std::vector<cudaStream_t> gstream;            // one stream per phase group (work-list mode)
    std::vector<cudaEvent_t> gjoin;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    std::vector<std::vector<int>> graph_cur[2];   // every case's cur[] at capture
    bool worklist = false;                        // work-list mode in force
    char *tables[3] = {nullptr, nullptr, nullptr};   // step tables of graph 0, 1 and of direct launches
    size_t tables_cap[3] = {0, 0, 0};
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

// One phase of a merged coarse step: launch kind, level, occurrence, and the
// (case, op) pairs in it.
struct Phase {
    int kind, L, occ;
    std::vector<std::pair<int, int>> items;
    int group = 0;   // cases of one level count share a phase sequence
};

// Record one coarse step of every case (nothing launched; the cases' buffer
// parities advance as if it ran) and merge the lists into phases.
int plan_step(agal_batch *b, std::vector<agal_oplist> &lists, std::vector<Phase> &phases)
{
    const int n = (int)b->cases.size();
    lists.assign(n, agal_oplist{});
    for (int i = 0; i < n; i++) {
        agal_ctx *c = b->cases[i];
        c->rec = &lists[i];
        const int rc = agal_record_coarse_step(c);
        c->rec = nullptr;
        if (rc) return berr(b, rc, "case " + std::to_string(i) + ": " + c->err);
    }
    // Cases with the same number of levels run the same sequence: each such
    // group gets its own merged phases (issued on its own stream, so light
    // phases of one group overlap the others).
    std::map<int, std::vector<int>> groups;
    for (int i = 0; i < n; i++) groups[b->cases[i]->max_levels].push_back(i);
    phases.clear();
    int gi = 0;
    for (auto &gv : groups) {
        std::vector<int> order = gv.second;
        std::stable_sort(order.begin(), order.end(),
                         [&](int x, int y) { return lists[x].ops.size() > lists[y].ops.size(); });
        std::vector<Phase> ph;
        for (int i : order) {
            std::map<std::pair<int, int>, int> occ;
            int pos = -1;
            for (int j = 0; j < (int)lists[i].ops.size(); j++) {
                const agal_op &op = lists[i].ops[j];
                const int k = occ[{op.kind, op.L}]++;
                int at = -1;
                for (int p = pos + 1; p < (int)ph.size(); p++)
                    if (ph[p].kind == op.kind && ph[p].L == op.L && ph[p].occ == k) {
                        at = p;
                        break;
                    }
                if (at < 0) {
                    at = pos + 1;
                    ph.insert(ph.begin() + at, Phase{op.kind, op.L, k, {}, gi});
                }
                ph[at].items.push_back({i, j});
                pos = at;
            }
        }
        phases.insert(phases.end(), ph.begin(), ph.end());
        gi++;
    }
    return AGAL_OK;
}

// Launch kinds run as one batched kernel per phase: fused steps and transfers.
static bool batched_kind(int kind) { return kind == 0 || kind == AGAL_OP_INTERP || kind == AGAL_OP_AVERAGE; }

// Device tables of the batched phases: per phase and kernel key, the cases'
// argument structures then the work prefix (n + 1 ints: chunks of a step,
// blocks of a transfer).  Written to tables[slot] before the launches that
// read them are issued.
struct StepGroup {
    int phase, key, n, total;
    size_t off_args, off_start;
    std::vector<int> items;   // indices into the phase's items
};

int build_tables(agal_batch *b, int slot, const std::vector<agal_oplist> &lists, const std::vector<Phase> &phases,
                 std::vector<StepGroup> &groups)
{
    groups.clear();
    std::vector<char> host;
    auto align = [&](size_t a) { host.resize((host.size() + a - 1) / a * a); };
    for (int p = 0; p < (int)phases.size(); p++) {
        const int kind = phases[p].kind;
        if (!batched_kind(kind)) continue;
        std::map<int, std::vector<int>> by_key;
        for (int t = 0; t < (int)phases[p].items.size(); t++) {
            const auto &it = phases[p].items[t];
            by_key[lists[it.first].ops[it.second].key].push_back(t);
        }
        for (auto &kv : by_key) {
            StepGroup g{p, kv.first, (int)kv.second.size(), 0, 0, 0, kv.second};
            const size_t asz = kind == 0 ? sizeof(agal::StepArgs) : agal_transfer_args_size(kind);
            align(16);
            g.off_args = host.size();
            host.resize(host.size() + asz * g.n);
            align(16);
            g.off_start = host.size();
            host.resize(host.size() + sizeof(int) * (g.n + 1));
            int acc = 0;
            for (int q = 0; q < g.n; q++) {
                const auto &it = phases[p].items[g.items[q]];
                const agal_op &op = lists[it.first].ops[it.second];
                const int mc = b->cases[it.first]->MC;
                std::memcpy(host.data() + g.off_args + asz * q, kind == 0 ? (const void *)&op.step : op.args.data(), asz);
                reinterpret_cast<int *>(host.data() + g.off_start)[q] = acc;
                acc += kind == 0 ? (op.n_blocks + 256 / mc - 1) / (256 / mc) : op.n_items;
            }
            reinterpret_cast<int *>(host.data() + g.off_start)[g.n] = acc;
            g.total = acc;
            groups.push_back(std::move(g));
        }
    }
    if (host.empty()) return AGAL_OK;
    if (host.size() > b->tables_cap[slot]) {
        if (b->tables[slot]) cudaFree(b->tables[slot]);
        b->tables[slot] = nullptr;
        b->tables_cap[slot] = 0;
        BCUDA(b, cudaMalloc(&b->tables[slot], host.size()));
        b->tables_cap[slot] = host.size();
    }
    BCUDA(b, cudaStreamSynchronize(b->master));   // earlier launches may still read the slot
    BCUDA(b, cudaMemcpy(b->tables[slot], host.data(), host.size(), cudaMemcpyHostToDevice));
    return AGAL_OK;
}

// Run fn(case) for the listed cases, each on its own stream, between a fork
// from and a join back to the master stream.
template <class F>
int fan_out(agal_batch *b, cudaStream_t s, const std::vector<int> &cases, F fn)
{
    if (cases.empty()) return AGAL_OK;
    BCUDA(b, cudaEventRecord(b->fork, s));
    for (int i : cases) {
        agal_ctx *c = b->cases[i];
        BCUDA(b, cudaStreamWaitEvent(c->stream, b->fork, 0));
        const int rc = fn(c);
        if (rc) return berr(b, rc, "case " + std::to_string(i) + ": " + c->err);
        BCUDA(b, cudaEventRecord(b->join[i], c->stream));
        BCUDA(b, cudaStreamWaitEvent(s, b->join[i], 0));
    }
    return AGAL_OK;
}

// Stream of phase group g (created on first use), forked from the master.
int group_stream(agal_batch *b, int g, cudaStream_t *out)
{
    while ((int)b->gstream.size() <= g) {
        cudaStream_t st = nullptr;
        cudaEvent_t ev = nullptr;
        BCUDA(b, cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        BCUDA(b, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        b->gstream.push_back(st);
        b->gjoin.push_back(ev);
    }
    *out = b->gstream[g];
    return AGAL_OK;
}

// Issue the planned phases (under capture or not): each phase group on its
// own stream, forked from the master and joined back into it.
int issue_step(agal_batch *b, int slot, const std::vector<agal_oplist> &lists, const std::vector<Phase> &phases,
               const std::vector<StepGroup> &groups)
{
    size_t g = 0;
    int cur_group = -1;
    cudaStream_t s = b->master;
    BCUDA(b, cudaEventRecord(b->done, b->master));   // every group starts after the master's work
    auto end_group = [&]() -> int {
        if (cur_group < 0) return AGAL_OK;
        BCUDA(b, cudaEventRecord(b->gjoin[cur_group], s));
        BCUDA(b, cudaStreamWaitEvent(b->master, b->gjoin[cur_group], 0));
        return AGAL_OK;
    };
    for (int p = 0; p < (int)phases.size(); p++) {
        const Phase &ph = phases[p];
        if (ph.group != cur_group) {
            int rc = end_group();
            if (!rc) rc = group_stream(b, ph.group, &s);
            if (rc) return rc;
            cur_group = ph.group;
            BCUDA(b, cudaStreamWaitEvent(s, b->done, 0));
        }
        if (ph.kind == AGAL_OP_INTERP || ph.kind == AGAL_OP_AVERAGE) {
            for (; g < groups.size() && groups[g].phase == p; g++) {
                const StepGroup &sg = groups[g];
                const char *base = b->tables[slot];
                const int rc = agal_launch_transfer_batch(ph.kind, sg.key, s, base + sg.off_args,
                                                          reinterpret_cast<const int *>(base + sg.off_start), sg.n,
                                                          sg.total);
                if (rc) return berr(b, rc, "batched transfer launch failed");
            }
            continue;
        }
        if (ph.kind != 0) {
            std::vector<int> cs;
            for (const auto &it : ph.items) cs.push_back(it.first);
            size_t q = 0;
            const int rc = fan_out(b, s, cs, [&](agal_ctx *c) {
                const auto &it = ph.items[q++];
                const agal_op &op = lists[it.first].ops[it.second];
                return run_in_state(c, op, op.fn);
            });
            if (rc) return rc;
            continue;
        }
        for (; g < groups.size() && groups[g].phase == p; g++) {
            const StepGroup &sg = groups[g];
            const char *base = b->tables[slot];
            int rc = agal_launch_step_batch(sg.key, s, base + sg.off_args,
                                            reinterpret_cast<const int *>(base + sg.off_start), sg.n, sg.total, 0);
            if (rc) return berr(b, rc, "batched step launch failed");
            // the wall steps of cases with walls, then the fix-ups of all
            std::vector<int> cs;
            std::vector<const agal_op *> ops;
            for (int t : sg.items) {
                const auto &it = ph.items[t];
                const agal_op &op = lists[it.first].ops[it.second];
                if (agal_wall_active(b->cases[it.first])) {
                    cs.push_back(it.first);
                    ops.push_back(&op);
                }
            }
            size_t q = 0;
            rc = fan_out(b, s, cs, [&](agal_ctx *c) {
                const agal_op *op = ops[q++];
                return run_in_state(c, *op, [op](agal_ctx *x) { return agal_launch_wall_step(x, op->L, op->fin, op->fout); });
            });
            if (rc) return rc;
            rc = agal_launch_step_batch(sg.key, s, base + sg.off_args,
                                        reinterpret_cast<const int *>(base + sg.off_start), sg.n, 0, 1);
            if (rc) return berr(b, rc, "batched fix-up launch failed");
        }
    }
    return end_group();
}

// Work-list mode needs every case on one launch path: no LES, no control-volume
// forces (their launch sequence interleaves levels differently).
bool worklist_ok(const agal_batch *b)
{
    for (const agal_ctx *c : b->cases)
        if (c->nu_sgs || c->P.S_FORCE_TYPE == 1) return false;
    return true;
}

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

int capture(agal_batch *b, int slot, cudaGraphExec_t *out)
{
    std::vector<std::vector<int>> cur0 = curs(b);
    std::vector<agal_oplist> lists;
    std::vector<Phase> phases;
    std::vector<StepGroup> groups;
    if (b->worklist) {
        // plan and upload the step tables before the capture begins
        int rc = plan_step(b, lists, phases);
        if (!rc) rc = build_tables(b, slot, lists, phases, groups);
        if (rc) {
            for (size_t i = 0; i < b->cases.size(); i++) b->cases[i]->cur = cur0[i];
            return rc;
        }
    }
    cudaGraph_t g = nullptr;
    BCUDA(b, cudaStreamBeginCapture(b->master, cudaStreamCaptureModeThreadLocal));
    int rc = b->worklist ? issue_step(b, slot, lists, phases, groups) : record_step(b);
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
    b->worklist = worklist_ok(b);
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
    for (cudaEvent_t e : b->gjoin)
        if (e) cudaEventDestroy(e);
    for (cudaStream_t st : b->gstream)
        if (st) cudaStreamDestroy(st);
    if (b->master) cudaStreamDestroy(b->master);
    for (char *t : b->tables)
        if (t) cudaFree(t);
    delete b;
    return AGAL_OK;
}

extern "C" const char *agal_batch_last_error(const agal_batch *b) { return b ? b->err.c_str() : ""; }

// Work-list mode on (1, where every case allows it) or off (0: one graph
// branch per case); returns AGAL_ERR_UNSUPPORTED for 1 when a case does not
// allow it (LES, control-volume forces).
extern "C" int agal_batch_set_worklist(agal_batch *b, int on)
{
    if (!b) return AGAL_ERR_PARAM;
    if (on && !worklist_ok(b)) return berr(b, AGAL_ERR_UNSUPPORTED, "work-list mode: a case has LES or CV forces");
    if ((on != 0) != b->worklist) drop(b);
    b->worklist = on != 0;
    return AGAL_OK;
}

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
                if ((rc = capture(b, k, &b->graph[k]))) return rc;
                b->graph_cur[k] = now;
            }
            BCUDA(b, cudaGraphLaunch(b->graph[k], b->master));
            for (agal_ctx *c : b->cases) agal_advance_parity(c, 1);
        } else if (b->worklist) {
            std::vector<agal_oplist> lists;
            std::vector<Phase> phases;
            std::vector<StepGroup> groups;
            if ((rc = plan_step(b, lists, phases))) return rc;
            if ((rc = build_tables(b, 2, lists, phases, groups))) return rc;
            if ((rc = issue_step(b, 2, lists, phases, groups))) return rc;
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

// Time `steps` graph-replayed coarse steps in each launch mode (work list,
// where allowed, and one branch per case) after a warm-up of two steps each,
// and keep the faster.  The cases advance by 2 x (steps + 2) coarse steps,
// with their regrids as usual; both modes give identical results.
extern "C" int agal_batch_autotune(agal_batch *b, int steps, float *ms, int *mode)
{
    if (!b || steps < 1) return AGAL_ERR_PARAM;
    float t[2] = {-1.f, -1.f};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    BCUDA(b, cudaEventCreate(&e0));
    BCUDA(b, cudaEventCreate(&e1));
    int rc = AGAL_OK;
    for (int on = 1; on >= 0 && rc == AGAL_OK; on--) {
        if (on && !worklist_ok(b)) continue;
        if ((rc = agal_batch_set_worklist(b, on))) break;
        if ((rc = agal_batch_advance_n(b, 2, 1))) break;
        if ((rc = agal_batch_sync(b))) break;
        if (cudaEventRecord(e0, b->master) != cudaSuccess) { rc = AGAL_ERR_CUDA; break; }
        if ((rc = agal_batch_advance_n(b, steps, 1))) break;
        if (cudaEventRecord(e1, b->master) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&t[on], e0, e1) != cudaSuccess)
            rc = AGAL_ERR_CUDA;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc == AGAL_ERR_CUDA ? berr(b, rc, "batch autotune timing failed") : rc;
    const int best = (t[1] >= 0.f && t[1] <= t[0]) ? 1 : 0;
    if ((rc = agal_batch_set_worklist(b, best))) return rc;
    if (ms) { ms[0] = t[0] / steps; ms[1] = t[1] >= 0.f ? t[1] / steps : -1.f; }
    if (mode) *mode = best;
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
