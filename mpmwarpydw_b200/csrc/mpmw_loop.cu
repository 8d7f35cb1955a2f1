// mpmw_loop.cu -- the driver's phase-1 loop with its stop test on the device
// (reference: runMPMYDW.py:656-727), as one CUDA graph with a while node.
#include <new>

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
