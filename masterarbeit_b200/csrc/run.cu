// run.cu -- the update/measure loop of one lattice, captured once as a CUDA graph and replayed.
//
// Reference: the driver loop of LGT_Code/main/qcd.c:55-60, gaugefieldUpdate (update.c:102-175)
// followed by plaquette() (plaquette.c:67-100) after every sweep.  One block is `meas_every`
// sweeps of (n_hb heatbath + n_or overrelaxation) and the plaquette, summed inside the last
// sweep's update passes.  The heatbath sweep index that keys the Philox stream and the trace row
// are device counters that the graph advances itself, so a replayed block draws exactly the randoms
// su2g_sweep draws for the same sweeps and the trace equals the one of the plain
// su2g_sweep_plaquette sequence bit for bit.
#include <algorithm>
#include <vector>

#include "internal.cuh"

using namespace su2g;

namespace {

constexpr int kSlotAcc = kOutSlots - 2;    // heatbath acceptance accumulator of the running block
constexpr int kSlotPlaq = kOutSlots - 1;   // plaquette of the running block

// Close one block: record (plaquette, acceptance) in its trace row, advance the counters,
// clear the acceptance accumulator.
__global__ void k_run_record(const double* __restrict__ plaq, double* __restrict__ acc, uint32_t* __restrict__ ctr,
                             double* __restrict__ trace, uint32_t rows, double acc_scale, uint32_t hb_per_block)
{
    const uint32_t row = ctr[1];
    if (row < rows) {
        trace[2 * (size_t)row] = *plaq;
        trace[2 * (size_t)row + 1] = *acc * acc_scale;
    }
    ctr[1] = row + 1;
    ctr[0] += hb_per_block;
    *acc = 0.0;
}

bool graph_matches(const su2g_lattice* h, int meas_every, int n_hb, int n_or)
{
    const auto& r = h->run;
    if (!r.exec || r.meas_every != meas_every || r.n_hb != n_hb || r.n_or != n_or || r.beta != h->beta ||
        r.seed != h->seed || r.partials != h->partials || r.trace != h->d_trace)
        return false;
    for (int mu = 0; mu < 4; ++mu)
        if (r.dirp[mu] != h->dirp[mu]) return false;
    return true;
}

// Enqueue one block on the handle's stream (used under stream capture).
int enqueue_block(su2g_lattice* h, int meas_every, int n_hb, int n_or)
{
    double* acc = h->d_out + kSlotAcc;
    // the plaquette is summed inside the last sub-sweep's update passes (su2g_sweep_plaquette)
    int rc = sweep_enqueue(h, meas_every, n_hb, n_or, 0u, h->d_run_ctr, acc, kSlotPlaq);
    if (rc) return rc;
    const double nupd = (double)meas_every * n_hb * 4.0 * (double)h->g.V;
    k_run_record<<<1, 1, 0, h->stream>>>(h->d_out + kSlotPlaq, acc, h->d_run_ctr, h->d_trace, (uint32_t)h->trace_rows,
                                         nupd > 0 ? 1.0 / nupd : 0.0, (uint32_t)(meas_every * n_hb));
    return check_cuda(h, cudaGetLastError(), "trace record");
}

int capture(su2g_lattice* h, int meas_every, int n_hb, int n_or)
{
    release_run_graph(h);
    // everything the block allocates is allocated before the capture starts
    int rc = ensure_partial_entries(h, std::max(2 * (size_t)((h->g.Vh + kBlock - 1) / kBlock), 3 * (size_t)update_plaq_parts(h)));
    if (rc) return rc;
    const bool prof = h->profiling;
    h->profiling = false;   // no per-launch events inside the graph
    rc = check_cuda(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "beginning graph capture");
    if (rc) {
        h->profiling = prof;
        return rc;
    }
    rc = enqueue_block(h, meas_every, n_hb, n_or);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
    h->profiling = prof;
    if (!rc) rc = check_cuda(h, e, "ending graph capture");
    if (!rc) rc = check_cuda(h, cudaGraphInstantiate(&h->run.exec, graph, 0), "instantiating the update graph");
    if (graph) cudaGraphDestroy(graph);
    if (rc) {
        h->run.exec = nullptr;
        cudaGetLastError();
        return rc;
    }
    auto& r = h->run;
    r.meas_every = meas_every;
    r.n_hb = n_hb;
    r.n_or = n_or;
    r.beta = h->beta;
    r.seed = h->seed;
    r.partials = h->partials;
    r.trace = h->d_trace;
    for (int mu = 0; mu < 4; ++mu) r.dirp[mu] = h->dirp[mu];
    return SU2G_OK;
}

}  // namespace

void su2g::release_run_graph(su2g_lattice* h)
{
    if (h->run.exec) cudaGraphExecDestroy(h->run.exec);
    h->run.exec = nullptr;
}

extern "C" int su2g_graph_run(su2g_lattice* h, int32_t n_blocks, int32_t meas_every, int32_t n_hb, int32_t n_or,
                              double* plaq, double* acc)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_graph_run: null handle");
    if (n_blocks < 0 || meas_every < 1 || n_hb < 0 || n_or < 0)
        return set_error(h, SU2G_EINVAL, "su2g_graph_run: bad counts (blocks %d, every %d, hb %d, or %d)", n_blocks,
                         meas_every, n_hb, n_or);
    if (n_blocks == 0) return SU2G_OK;
    cudaSetDevice(h->device);
    int rc = SU2G_OK;
    if (!h->d_run_ctr && (rc = check_cuda(h, cudaMalloc(&h->d_run_ctr, 2 * sizeof(uint32_t)), "allocating counters")))
        return rc;
    if ((size_t)n_blocks > h->trace_rows) {
        cudaStreamSynchronize(h->stream);
        release_run_graph(h);   // the new buffer may reuse the old address, so the key cannot tell
        cudaFree(h->d_trace);
        h->d_trace = nullptr;
        h->trace_rows = 0;
        if ((rc = check_cuda(h, cudaMalloc(&h->d_trace, 2 * sizeof(double) * (size_t)n_blocks), "allocating the trace")))
            return rc;
        h->trace_rows = (size_t)n_blocks;
    }
    if (!graph_matches(h, meas_every, n_hb, n_or) && (rc = capture(h, meas_every, n_hb, n_or))) return rc;
    const uint32_t ctr[2] = {h->hb_sweeps, 0u};
    rc = check_cuda(h, cudaMemcpyAsync(h->d_run_ctr, ctr, sizeof(ctr), cudaMemcpyHostToDevice, h->stream),
                    "setting counters");
    if (!rc) rc = check_cuda(h, cudaMemsetAsync(h->d_out + kSlotAcc, 0, sizeof(double), h->stream), "clearing acceptance");
    for (int b = 0; b < n_blocks && !rc; ++b)
        rc = check_cuda(h, cudaGraphLaunch(h->run.exec, h->stream), "replaying the update graph");
    if (rc) return rc;
    h->hb_sweeps += (uint32_t)(n_blocks * meas_every * n_hb);
    std::vector<double> tr(2 * (size_t)n_blocks);
    rc = check_cuda(h, cudaMemcpyAsync(tr.data(), h->d_trace, tr.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
                    "copying the trace");
    if (!rc) rc = fetch_results(h, 0, 0);   // synchronises and checks the status word
    if (rc) return rc;
    for (int b = 0; b < n_blocks; ++b) {
        if (plaq) plaq[b] = tr[2 * (size_t)b];
        if (acc) acc[b] = tr[2 * (size_t)b + 1];
    }
    return SU2G_OK;
}

extern "C" int su2g_graph_release(su2g_lattice* h)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_graph_release: null handle");
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    release_run_graph(h);
    return SU2G_OK;
}
