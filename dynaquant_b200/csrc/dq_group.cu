// dq_group.cu — several ensembles ("aggregates": their own Hamiltonian,
// size and trajectory count) advanced together.  The reference runs one
// system per process; uneven aggregates are this build's addition.  Each
// group step is one CUDA graph with one branch per member: a fork event on
// the group's stream, every member's whole ensemble step on its own stream,
// and a join back, so the small aggregates' kernels run beside the large
// ones instead of after them.  The graph is recaptured on every
// dq_group_run call, so a member's tiling or couplings may change between
// calls.
#include <vector>

#include "dq_internal.h"

struct dq_group {
    std::vector<dq_ctx*> members;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<cudaEvent_t> events;   // fork + one join per member
    std::string err;
};

namespace {
dq_status gfail(dq_group* g, int code, const std::string& msg) {
    if (g) g->err = msg;
    return code;
}
dq_status gcuda(dq_group* g, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return DQ_OK;
    return gfail(g, DQ_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define DQ_GCU(call)                                        \
    do {                                                    \
        dq_status _s = gcuda(g, (call), #call);             \
        if (_s != DQ_OK) return _s;                         \
    } while (0)
}  // namespace

extern "C" {

dq_status dq_group_create(dq_ctx* const* members, int n_members, dq_group** out) {
    if (!members || n_members < 1 || !out) return DQ_ERR_ARG;
    *out = nullptr;
    for (int i = 0; i < n_members; ++i) {
        if (!members[i]) return DQ_ERR_ARG;
        for (int k = 0; k < i; ++k)
            if (members[k] == members[i]) return DQ_ERR_ARG;
        if (members[i]->cfg.device != members[0]->cfg.device) return DQ_ERR_ARG;
    }
    dq_group* g = new dq_group();
    g->members.assign(members, members + n_members);
    g->device = members[0]->cfg.device;
    dq::DeviceScope dev_scope(g->device);
    cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
    g->events.assign(n_members + 1, nullptr);
    for (int i = 0; e == cudaSuccess && i <= n_members; ++i)
        e = cudaEventCreateWithFlags(&g->events[i], cudaEventDisableTiming);
    if (e != cudaSuccess) {
        dq_group_destroy(g);
        return DQ_ERR_CUDA;
    }
    *out = g;
    return DQ_OK;
}

void dq_group_destroy(dq_group* g) {
    if (!g) return;
    dq::DeviceScope dev_scope(g->device);
    if (g->stream) cudaStreamSynchronize(g->stream);
    for (auto ev : g->events)
        if (ev) cudaEventDestroy(ev);
    if (g->stream) cudaStreamDestroy(g->stream);
    delete g;
}

const char* dq_group_last_error(const dq_group* g) { return g ? g->err.c_str() : "null group"; }

dq_status dq_group_run(dq_group* g, int n_steps) { return dq_group_run_timed(g, n_steps, nullptr); }

dq_status dq_group_run_timed(dq_group* g, int n_steps, double* device_ms) {
    if (!g) return DQ_ERR_ARG;
    if (device_ms) *device_ms = 0.0;
    if (n_steps < 0) return gfail(g, DQ_ERR_ARG, "group run: negative step count");
    if (n_steps == 0) return DQ_OK;
    dq::DeviceScope dev_scope(g->device);
    // every member's ensemble exists and is ready, as dq_run would make it
    for (dq_ctx* c : g->members) {
        if (c->steps_done + n_steps > c->cfg.max_steps)
            return gfail(g, DQ_ERR_ARG, "group run: a member's steps exceed its max_steps");
        dq_status st = DQ_OK;
        if (c->tk_p > 0) return gfail(g, DQ_ERR_STATE, "group run: Taylor-Krylov members run on their own");
        if (!c->bat) {
            if ((st = dq::batched_alloc(c))) return gfail(g, st, c->err);
            c->ready = false;
        }
        if (!c->ready && (st = dq_reset(c))) return gfail(g, st, c->err);
        DQ_GCU(cudaStreamSynchronize(c->stream));
    }
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    DQ_GCU(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
    dq_status st = DQ_OK;
    cudaError_t e = cudaEventRecord(g->events[0], g->stream);
    for (size_t i = 0; e == cudaSuccess && st == DQ_OK && i < g->members.size(); ++i) {
        dq_ctx* c = g->members[i];
        e = cudaStreamWaitEvent(c->stream, g->events[0], 0);
        if (e == cudaSuccess) st = dq::batched_enqueue_step(c);
        if (e == cudaSuccess && st == DQ_OK) e = cudaEventRecord(g->events[i + 1], c->stream);
        if (e == cudaSuccess && st == DQ_OK) e = cudaStreamWaitEvent(g->stream, g->events[i + 1], 0);
    }
    cudaError_t e2 = cudaStreamEndCapture(g->stream, &graph);
    if (st) {
        if (graph) cudaGraphDestroy(graph);
        return gfail(g, st, "group run: a member's step failed to enqueue");
    }
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return gcuda(g, e != cudaSuccess ? e : e2, "group graph capture");
    }
    e = cudaGraphInstantiate(&exec, graph, 0);
    // device time of the launches alone (capture and instantiation excluded)
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (e == cudaSuccess && device_ms) {
        e = cudaEventCreate(&t0);
        if (e == cudaSuccess) e = cudaEventCreate(&t1);
        if (e == cudaSuccess) e = cudaEventRecord(t0, g->stream);
    }
    for (int k = 0; e == cudaSuccess && k < n_steps; ++k) e = cudaGraphLaunch(exec, g->stream);
    if (e == cudaSuccess && device_ms) e = cudaEventRecord(t1, g->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
    if (e == cudaSuccess && device_ms) {
        float ms = 0.f;
        e = cudaEventElapsedTime(&ms, t0, t1);
        *device_ms = ms;
    }
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    if (exec) cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return gcuda(g, e, "group graph launch");
    for (dq_ctx* c : g->members) {
        c->steps_done += n_steps;
        c->last_path = 1;
        if ((st = dq::batched_read_status(c))) return gfail(g, st, c->err);
    }
    return DQ_OK;
}

}  // extern "C"
