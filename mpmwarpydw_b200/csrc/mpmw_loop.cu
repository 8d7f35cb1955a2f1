// mpmw_loop.cu -- the driver's loops with their stop tests on the device, each
// one CUDA graph with a while node:
//   mpmw_loop_*        phase 1, MPM substeps only (runMPMYDW.py:656-727);
//   mpmw_phase_loop_*  phase 1 with the XPBD steps and the gravity pulse inside
//                      the graph (IF nodes choose the branch per chunk,
//                      runMPMYDW.py:646-682);
//   mpmw_xpbd_loop_*   phase 2, XPBD-only steps with the sleep-ratio stop
//                      (runMPMYDW.py:780-844).
#include <cstring>
#include <new>
#include <vector>

#include "mpmw_common.cuh"
#include "mpmw_internal.cuh"

struct mpmw_loop {
    cudaGraph_t graph;
    cudaGraphExec_t exec;
};

namespace mpmw {

// One check of the phase-1 loop after `chunk` substeps (the package driver's
// PhaseOneMonitor.update with k = chunk), and the while node's condition.
__global__ void k_loop_decide(mpmw_loop_state_t *st, const mpmw_loop_params_t lp, cudaGraphConditionalHandle h)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    st->counter += lp.chunk;
    const double active = st->stats[1];
    const double residual = active > 0.0 ? st->stats[0] / active : 0.0;
    const double mean_damage = active > 0.0 ? st->stats[2] / active : 0.0;
    const double change = mean_damage - st->prev_damage;
    if (change < lp.stall_threshold * (double)lp.chunk && st->counter > lp.min_steps) st->stall += lp.chunk;
    else st->stall = 0;
    st->prev_damage = mean_damage;
    st->residual = residual;
    st->segment_left -= lp.chunk;
    unsigned go = 0;
    if (st->stall >= lp.stall_steps && st->counter > lp.min_steps) {
        st->stopped_early = 1;
    } else {
        const bool running = st->counter < lp.n_steps && (st->counter < lp.min_steps || residual > lp.residual_threshold);
        go = running && st->segment_left >= lp.chunk ? 1u : 0u;
    }
    cudaGraphSetConditional(h, go);
}

// The branch conditions of one iteration of the phase loop (counter c before
// the chunk of substeps c .. c + chunk - 1): the whole chunk in the gravity
// pulse (c + chunk <= P), none of it (c >= P), or the chunk the pulse ends in;
// an XPBD step after it when its last substep index j = c + chunk - 1 is a
// positive multiple of the XPBD ratio, with the pulse's or the plain XPBD
// parameters as the driver's gravity is at that substep (runMPMYDW.py:646-682).
struct PhaseHandles {
    cudaGraphConditionalHandle pulse, normal, split, xpbd_pulse, xpbd_normal;
};

__global__ void k_phase_flags(const mpmw_loop_state_t *st, const mpmw_phase_params_t pp, PhaseHandles h,
                              unsigned mask)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const long long c = st->counter, k = pp.loop.chunk, P = pp.pulse_steps, j = c + k - 1;
    const bool full_pulse = P > 0 && c + k <= P, no_pulse = c >= P, split = !full_pulse && !no_pulse;
    const bool xp = pp.xpbd_ratio > 0 && j >= pp.xpbd_ratio && j % pp.xpbd_ratio == 0;
    if (mask & 1u) cudaGraphSetConditional(h.pulse, full_pulse ? 1u : 0u);
    if (mask & 2u) cudaGraphSetConditional(h.normal, no_pulse ? 1u : 0u);
    if (mask & 4u) cudaGraphSetConditional(h.split, split ? 1u : 0u);
    if (mask & 8u) cudaGraphSetConditional(h.xpbd_pulse, xp && j < P ? 1u : 0u);
    if (mask & 16u) cudaGraphSetConditional(h.xpbd_normal, xp && j >= P ? 1u : 0u);
}

// one check of the XPBD-only phase (runMPMYDW.py:780-844): a step done, stop
// when the sleeping fraction of XPBD particles reaches the ratio, or when the
// steps or the segment run out
__global__ void k_xpbd_phase_decide(mpmw_loop_state_t *st, const int32_t *counts, int max_steps, double sleep_ratio,
                                    cudaGraphConditionalHandle h)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    st->counter += 1;
    st->segment_left -= 1;
    const int tot = counts[0], slp = counts[1];
    st->stats[0] = (double)tot;
    st->stats[1] = (double)slp;
    unsigned go = 1u;
    if (sleep_ratio < 1.0 && tot > 0 && (double)slp / (double)tot >= sleep_ratio) {
        st->stopped_early = 1;
        go = 0u;
    }
    if (st->counter >= max_steps || st->segment_left < 1) go = 0u;
    cudaGraphSetConditional(h, go);
}

namespace {

// adds an IF node after `dep` into `graph` and captures `fill` into its body
template <class Fill>
int add_if(cudaGraph_t graph, cudaGraphNode_t dep, cudaGraphConditionalHandle h, cudaStream_t s, Fill fill,
           cudaGraphNode_t *node_out)
{
    alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
    memset(raw, 0, sizeof(raw));
    cudaGraphNodeParams &np = *reinterpret_cast<cudaGraphNodeParams *>(raw);
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeIf;
    np.conditional.size = 1;
    if (cudaGraphAddNode(node_out, graph, &dep, 1, &np) != cudaSuccess) {
        set_error("loop: cannot add a conditional node");
        return MPMW_E_DEVICE;
    }
    cudaGraph_t body = np.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        set_error("loop: cannot capture on this stream");
        return MPMW_E_DEVICE;
    }
    int rc = fill();
    cudaGraph_t captured = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(s, &captured);
    if (rc == MPMW_OK && ec != cudaSuccess) {
        set_error("loop: capture failed: %s", cudaGetErrorString(ec));
        rc = MPMW_E_DEVICE;
    }
    return rc;
}

// captures `fill` into `graph` after the node `dep` (as a root when dep is null)
template <class Fill>
int capture_into(cudaGraph_t graph, const cudaGraphNode_t *dep, cudaStream_t s, Fill fill)
{
    if (cudaStreamBeginCaptureToGraph(s, graph, dep, nullptr, dep ? 1 : 0, cudaStreamCaptureModeThreadLocal) !=
        cudaSuccess) {
        set_error("loop: cannot capture on this stream");
        return MPMW_E_DEVICE;
    }
    int rc = fill();
    cudaGraph_t captured = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(s, &captured);
    if (rc == MPMW_OK && ec != cudaSuccess) {
        set_error("loop: capture failed: %s", cudaGetErrorString(ec));
        rc = MPMW_E_DEVICE;
    }
    return rc;
}

// the graph's single node without successors (after a linear capture)
cudaGraphNode_t sink_node(cudaGraph_t graph)
{
    size_t n = 0;
    if (cudaGraphGetNodes(graph, nullptr, &n) != cudaSuccess || n == 0) return nullptr;
    std::vector<cudaGraphNode_t> nodes(n);
    if (cudaGraphGetNodes(graph, nodes.data(), &n) != cudaSuccess) return nullptr;
    cudaGraphNode_t sink = nullptr;
    for (cudaGraphNode_t nd : nodes) {
        size_t out = 0;
        if (cudaGraphNodeGetDependentNodes(nd, nullptr, &out) != cudaSuccess) return nullptr;
        if (out == 0) {
            if (sink) return nullptr;  // more than one sink: not a chain
            sink = nd;
        }
    }
    return sink;
}

// a graph whose root is a while node; *body receives its body graph
int make_while_graph(cudaGraph_t *graph, cudaGraph_t *body, cudaGraphConditionalHandle *h)
{
    *graph = nullptr;
    cudaGraphNode_t node;
    alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
    memset(raw, 0, sizeof(raw));
    cudaGraphNodeParams &np = *reinterpret_cast<cudaGraphNodeParams *>(raw);
    if (cudaGraphCreate(graph, 0) != cudaSuccess ||
        cudaGraphConditionalHandleCreate(h, *graph, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
        set_error("loop: cannot create the graph");
        if (*graph) cudaGraphDestroy(*graph);
        *graph = nullptr;
        return MPMW_E_DEVICE;
    }
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = *h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    if (cudaGraphAddNode(&node, *graph, nullptr, 0, &np) != cudaSuccess) {
        cudaGraphDestroy(*graph);
        *graph = nullptr;
        set_error("loop: cannot add the while node");
        return MPMW_E_DEVICE;
    }
    *body = np.conditional.phGraph_out[0];
    return MPMW_OK;
}

int finish_loop(cudaGraph_t graph, int rc, mpmw_loop_t **out)
{
    cudaGraphExec_t exec = nullptr;
    if (rc == MPMW_OK && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
        set_error("loop: cannot instantiate the graph");
        rc = MPMW_E_DEVICE;
    }
    mpmw_loop *L = rc == MPMW_OK ? new (std::nothrow) mpmw_loop : nullptr;
    if (rc == MPMW_OK && !L) {
        set_error("loop: out of host memory");
        rc = MPMW_E_DEVICE;
    }
    if (rc != MPMW_OK) {
        if (exec) cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        return rc;
    }
    L->graph = graph;
    L->exec = exec;
    *out = L;
    return MPMW_OK;
}

}  // namespace

}  // namespace mpmw

using namespace mpmw;

extern "C" {

int mpmw_loop_create(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm,
                     const mpmw_loop_params_t *lp, mpmw_loop_state_t *state, uint32_t *status, void *workspace,
                     size_t ws_bytes, mpmw_loop_t **out, mpmw_stream_t stream)
{
    if (!out) { set_error("loop: out is NULL"); return MPMW_E_ARG; }
    *out = nullptr;
    if (!p || !g || !prm || !lp || !state) { set_error("loop: NULL argument"); return MPMW_E_ARG; }
    if (lp->chunk < 1) { set_error("loop: chunk must be >= 1"); return MPMW_E_ARG; }
    if (reinterpret_cast<uintptr_t>(state) & 7u) { set_error("loop: state must be 8-byte aligned"); return MPMW_E_ARG; }
    if (!workspace) { set_error("loop: a workspace is required (the fused substeps)"); return MPMW_E_WORKSPACE; }
    cudaStream_t s = as_stream(stream);
    if (!s) { set_error("loop: a non-default stream is required for capture"); return MPMW_E_ARG; }
    if (const int rc0 = reserve_fused_smem()) return rc0;  // no attribute call inside the capture
    cudaGraph_t graph = nullptr, body = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphConditionalHandle h;
    cudaGraphNode_t node;
    // zero-filled node parameters (the struct's unused bytes must be zero; its
    // default constructor is deleted)
    alignas(cudaGraphNodeParams) unsigned char np_raw[sizeof(cudaGraphNodeParams)];
    memset(np_raw, 0, sizeof(np_raw));
    cudaGraphNodeParams &np = *reinterpret_cast<cudaGraphNodeParams *>(np_raw);
    if (cudaGraphCreate(&graph, 0) != cudaSuccess ||
        cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
        set_error("loop: cannot create the graph");
        if (graph) cudaGraphDestroy(graph);
        return MPMW_E_DEVICE;
    }
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    if (cudaGraphAddNode(&node, graph, nullptr, 0, &np) != cudaSuccess) {
        cudaGraphDestroy(graph);
        set_error("loop: cannot add the while node");
        return MPMW_E_DEVICE;
    }
    body = np.conditional.phGraph_out[0];
    // the body: capture the chunk of substeps, the statistics and the decision
    if (cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGraphDestroy(graph);
        set_error("loop: cannot capture on this stream");
        return MPMW_E_DEVICE;
    }
    int rc = mpmw_run_substeps(p, g, prm, lp->chunk, status, workspace, ws_bytes, stream);
    if (rc == MPMW_OK) rc = mpmw_stats(p, state->stats, stream);
    if (rc == MPMW_OK) {
        k_loop_decide<<<1, 32, 0, s>>>(state, *lp, h);
        rc = check_launch("k_loop_decide");
    }
    cudaGraph_t captured = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(s, &captured);
    if (rc != MPMW_OK || ec != cudaSuccess) {
        cudaGraphDestroy(graph);
        if (rc == MPMW_OK) set_error("loop: capture failed: %s", cudaGetErrorString(ec));
        return rc != MPMW_OK ? rc : MPMW_E_DEVICE;
    }
    if (cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
        cudaGraphDestroy(graph);
        set_error("loop: cannot instantiate the graph");
        return MPMW_E_DEVICE;
    }
    mpmw_loop *L = new (std::nothrow) mpmw_loop;
    if (!L) {
        cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        set_error("loop: out of host memory");
        return MPMW_E_DEVICE;
    }
    L->graph = graph;
    L->exec = exec;
    *out = L;
    return MPMW_OK;
}

int mpmw_phase_loop_create(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm,
                           const mpmw_params_t *prm_pulse, const mpmw_xpbd_t *x, const mpmw_hash_t *h,
                           const mpmw_xpbd_params_t *q, const mpmw_xpbd_params_t *q_pulse,
                           const mpmw_phase_params_t *pp, mpmw_loop_state_t *state, uint32_t *status,
                           void *workspace, size_t ws_bytes, void *xpbd_workspace, size_t xpbd_ws_bytes,
                           mpmw_loop_t **out, mpmw_stream_t stream)
{
    if (!out) { set_error("phase loop: out is NULL"); return MPMW_E_ARG; }
    *out = nullptr;
    if (!p || !g || !prm || !pp || !state) { set_error("phase loop: NULL argument"); return MPMW_E_ARG; }
    const int k = pp->loop.chunk, P = pp->pulse_steps, R = pp->xpbd_ratio;
    if (k < 1 || P < 0 || R < 0) { set_error("phase loop: chunk >= 1, pulse_steps >= 0, xpbd_ratio >= 0"); return MPMW_E_ARG; }
    if (pp->phase < 0 || pp->phase >= k) { set_error("phase loop: phase must be in [0, chunk)"); return MPMW_E_ARG; }
    if (R > 0) {
        if (R % k != 0) { set_error("phase loop: chunk %d must divide the XPBD ratio %d", k, R); return MPMW_E_ARG; }
        if (pp->phase != 1 % k) { set_error("phase loop: with XPBD steps the chunks start at counters = 1 mod chunk"); return MPMW_E_ARG; }
        if (!x || !h || !q || !xpbd_workspace) { set_error("phase loop: the XPBD arrays, hash, parameters and workspace are required"); return MPMW_E_ARG; }
    }
    if (P > 0 && (!prm_pulse || (R > 0 && !q_pulse))) { set_error("phase loop: the pulse parameters are required"); return MPMW_E_ARG; }
    if (reinterpret_cast<uintptr_t>(state) & 7u) { set_error("phase loop: state must be 8-byte aligned"); return MPMW_E_ARG; }
    if (!workspace) { set_error("phase loop: a workspace is required (the fused substeps)"); return MPMW_E_WORKSPACE; }
    cudaStream_t s = as_stream(stream);
    if (!s) { set_error("phase loop: a non-default stream is required for capture"); return MPMW_E_ARG; }
    if (const int rc0 = reserve_fused_smem()) return rc0;
    cudaGraph_t graph = nullptr, body = nullptr;
    cudaGraphConditionalHandle hw;
    int rc = make_while_graph(&graph, &body, &hw);
    if (rc != MPMW_OK) return rc;
    PhaseHandles hs{};
    unsigned mask = 0;
    // chunks that start at counters = phase (mod chunk) and contain the pulse's end split after r substeps
    const int r = P > 0 ? (int)(((long long)P - pp->phase) % k + k) % k : 0;
    const bool want[5] = {P > 0, true, P > 0 && r != 0, R > 0 && P > 0, R > 0};
    cudaGraphConditionalHandle *hp[5] = {&hs.pulse, &hs.normal, &hs.split, &hs.xpbd_pulse, &hs.xpbd_normal};
    for (int i = 0; i < 5 && rc == MPMW_OK; ++i) {
        if (!want[i]) continue;
        if (cudaGraphConditionalHandleCreate(hp[i], body, 0, 0) != cudaSuccess) {
            set_error("phase loop: cannot create a branch condition");
            rc = MPMW_E_DEVICE;
        }
        mask |= 1u << i;
    }
    // the branch flags, the substep branches, the XPBD branches, then statistics and decision
    if (rc == MPMW_OK)
        rc = capture_into(body, nullptr, s, [&]() {
            k_phase_flags<<<1, 32, 0, s>>>(state, *pp, hs, mask);
            return check_launch("k_phase_flags");
        });
    cudaGraphNode_t last = rc == MPMW_OK ? sink_node(body) : nullptr;
    if (rc == MPMW_OK && !last) { set_error("phase loop: the flag kernel node is missing"); rc = MPMW_E_DEVICE; }
    auto branch = [&](int i, auto fill) {
        if (rc != MPMW_OK || !want[i]) return;
        cudaGraphNode_t nd = nullptr;
        rc = add_if(body, last, *hp[i], s, fill, &nd);
        if (rc == MPMW_OK) last = nd;
    };
    branch(0, [&]() { return mpmw_run_substeps(p, g, prm_pulse, k, status, workspace, ws_bytes, stream); });
    branch(1, [&]() { return mpmw_run_substeps(p, g, prm, k, status, workspace, ws_bytes, stream); });
    branch(2, [&]() {
        int e = mpmw_run_substeps(p, g, prm_pulse, r, status, workspace, ws_bytes, stream);
        return e == MPMW_OK ? mpmw_run_substeps(p, g, prm, k - r, status, workspace, ws_bytes, stream) : e;
    });
    branch(3, [&]() { return mpmw_xpbd_step(p, x, h, q_pulse, status, xpbd_workspace, xpbd_ws_bytes, stream); });
    branch(4, [&]() { return mpmw_xpbd_step(p, x, h, q, status, xpbd_workspace, xpbd_ws_bytes, stream); });
    if (rc == MPMW_OK)
        rc = capture_into(body, &last, s, [&]() {
            int e = mpmw_stats(p, state->stats, stream);
            if (e != MPMW_OK) return e;
            k_loop_decide<<<1, 32, 0, s>>>(state, pp->loop, hw);
            return check_launch("k_loop_decide");
        });
    return finish_loop(graph, rc, out);
}

int mpmw_xpbd_loop_create(const mpmw_particles_t *p, const mpmw_xpbd_t *x, const mpmw_hash_t *h,
                          const mpmw_xpbd_params_t *q, int max_steps, double sleep_ratio, mpmw_loop_state_t *state,
                          uint32_t *status, void *xpbd_workspace, size_t xpbd_ws_bytes, mpmw_loop_t **out,
                          mpmw_stream_t stream)
{
    if (!out) { set_error("xpbd loop: out is NULL"); return MPMW_E_ARG; }
    *out = nullptr;
    if (!p || !x || !h || !q || !state || !xpbd_workspace) { set_error("xpbd loop: NULL argument"); return MPMW_E_ARG; }
    if (!x->counts) { set_error("xpbd loop: the XPBD counts array is required (the sleep-ratio stop)"); return MPMW_E_ARG; }
    if (max_steps < 1) { set_error("xpbd loop: max_steps must be >= 1"); return MPMW_E_ARG; }
    if (reinterpret_cast<uintptr_t>(state) & 7u) { set_error("xpbd loop: state must be 8-byte aligned"); return MPMW_E_ARG; }
    cudaStream_t s = as_stream(stream);
    if (!s) { set_error("xpbd loop: a non-default stream is required for capture"); return MPMW_E_ARG; }
    cudaGraph_t graph = nullptr, body = nullptr;
    cudaGraphConditionalHandle hw;
    int rc = make_while_graph(&graph, &body, &hw);
    if (rc != MPMW_OK) return rc;
    rc = capture_into(body, nullptr, s, [&]() {
        int e = mpmw_xpbd_step(p, x, h, q, status, xpbd_workspace, xpbd_ws_bytes, stream);
        if (e != MPMW_OK) return e;
        k_xpbd_phase_decide<<<1, 32, 0, s>>>(state, x->counts, max_steps, sleep_ratio, hw);
        return check_launch("k_xpbd_phase_decide");
    });
    return finish_loop(graph, rc, out);
}

int mpmw_loop_launch(mpmw_loop_t *loop, mpmw_stream_t stream)
{
    if (!loop) { set_error("loop is NULL"); return MPMW_E_ARG; }
    if (cudaGraphLaunch(loop->exec, as_stream(stream)) != cudaSuccess) {
        set_error("loop: launch failed");
        return MPMW_E_LAUNCH;
    }
    return MPMW_OK;
}

void mpmw_loop_destroy(mpmw_loop_t *loop)
{
    if (!loop) return;
    cudaGraphExecDestroy(loop->exec);
    cudaGraphDestroy(loop->graph);
    delete loop;
}

}  // extern "C"
