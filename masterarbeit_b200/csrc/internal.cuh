// internal.cuh -- handle state, launch/profiling helpers and compensated FP64 reductions.
#pragma once
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>

#include "su2g.h"
#include "su2.cuh"

namespace su2g {

constexpr int kBlock = 256;            // threads per CTA for the stencil kernels
constexpr int kMaxPartials = 8192;     // per-CTA partial sums a reduction may write
constexpr int kFinBlocks = 128;        // CTAs of the wide final reduction (one slot, many partials)
constexpr int kOutSlots = 16384;       // device result doubles per handle
constexpr uint32_t kMaxTrials = 1u << 20;   // Kennedy-Pendleton trials before a link gives up

// Status bits a kernel may raise in the handle's status word.
enum : unsigned { kStatusKpTrials = 1u, kStatusNonFinite = 2u, kStatusTmaTimeout = 4u, kStatusGridTimeout = 8u };

// Compensated sum: value s plus running error e (TwoSum, Knuth TAOCP vol. 2, 4.2.2).
struct DD {
    double s, e;
};

__device__ __forceinline__ DD dd_add(DD a, DD b)
{
    double s = a.s + b.s;
    double bb = s - a.s;
    double err = (a.s - (s - bb)) + (b.s - bb);
    DD r;
    r.s = s;
    r.e = err + a.e + b.e;
    return r;
}

__device__ __forceinline__ DD dd_add(DD a, double b)
{
    DD t;
    t.s = b;
    t.e = 0.0;
    return dd_add(a, t);
}

__device__ __forceinline__ DD dd_shfl_xor(DD v, int lane_mask)
{
    DD r;
    r.s = __shfl_xor_sync(0xffffffffu, v.s, lane_mask);
    r.e = __shfl_xor_sync(0xffffffffu, v.e, lane_mask);
    return r;
}

__device__ __forceinline__ DD dd_warp_sum(DD v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = dd_add(v, dd_shfl_xor(v, o));
    return v;
}

// Block-wide sum of one double per thread: plain FP64 within each warp (32 terms, relative error
// <= 32 ulp of the warp's partial, far below the compensated sum across warps and CTAs that
// follows), then compensated across the warps.  Result valid in thread 0; fixed order.
template <int NT>
__device__ __forceinline__ DD dd_block_sum_d(double x)
{
    __shared__ double warp_part[NT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) warp_part[warp] = x;
    __syncthreads();
    DD v = {0.0, 0.0};
    if (threadIdx.x == 0)
        for (int w = 0; w < NT / 32; ++w) v = dd_add(v, warp_part[w]);
    __syncthreads();
    return v;
}

// Block-wide compensated sum; the result is valid in thread 0.  Fixed order -> deterministic.
template <int NT>
__device__ __forceinline__ DD dd_block_sum(DD v)
{
    __shared__ DD warp_part[NT / 32];
    v = dd_warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) warp_part[warp] = v;
    __syncthreads();
    if (warp == 0) {
        DD w;
        w.s = lane < NT / 32 ? warp_part[lane].s : 0.0;
        w.e = lane < NT / 32 ? warp_part[lane].e : 0.0;
        v = dd_warp_sum(w);
    }
    __syncthreads();
    return v;
}

// Sums `nparts` per-CTA partials for `nslots` independent slots (partials[slot*stride + part])
// into out[slot] = scale * sum.  One CTA per slot, fixed order.
__global__ void k_finalize(const DD* __restrict__ partials, int nparts, int stride, double scale,
                           double* __restrict__ out);

}  // namespace su2g

struct su2g_meas_graph;   // measure.cu

struct su2g_lattice {
    su2g::Geom g;
    int prec = SU2G_FP32;
    double beta = 0.0;
    uint64_t seed = 0;
    uint32_t replica = 0;
    uint32_t hb_sweeps = 0;
    int device = 0;
    int num_sms = 148;
    size_t link_bytes = 16;
    void* field = nullptr;       // 4V links, layout of su2.cuh
    void* field_alt = nullptr;   // second field for Jacobi smearing (allocated on first use)
    void* dirp[4] = {nullptr, nullptr, nullptr, nullptr};   // current base of each direction
    void* altp[4] = {nullptr, nullptr, nullptr, nullptr};   // ping-pong partner of each direction
    su2g::DD* partials = nullptr;   // kMaxPartials x kPartialSlots compensated partial sums
    size_t partial_slots = 0;
    double* d_out = nullptr;     // device result slots
    double* h_out = nullptr;     // pinned host mirror of d_out
    unsigned* d_status = nullptr;
    su2g::DD* fin_blocks = nullptr;   // per-CTA sums of the wide final reduction (kFinBlocks)
    unsigned* fin_ticket = nullptr;   // its arrival counter (zero between launches)
    double* d_aos = nullptr;     // device staging for AoS FP64 transfers
    size_t aos_sites = 0;        // sites the staging buffer holds
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_begin = nullptr, ev_end = nullptr;
    int max_smem = 0;            // opt-in shared memory per CTA
    int ape_variant = 0;         // 0: per-site APE kernel, 1: TMA-tiled FP32 APE_all where it applies
    // Graph of one measurement block of su2g_run (recaptured when its key changes).
    struct RunGraph {
        cudaGraphExec_t exec = nullptr;
        int meas_every = 0, n_hb = 0, n_or = 0;
        double beta = 0.0;
        uint64_t seed = 0;
        const void* partials = nullptr;
        const double* trace = nullptr;
        void* dirp[4] = {nullptr, nullptr, nullptr, nullptr};
    } run;
    cudaMemPool_t pool = nullptr;      // scratch of the adjoint; keeps its memory until destroy
    su2g_meas_graph* meas = nullptr;   // graph of one su2g_measure spec
    void* lines = nullptr;             // 2- and 3-link line products of the field Q is measured on
    void* meas_work = nullptr;         // measurement copy of the field and its ping-pong partner
    void* meas_alt = nullptr;
    uint32_t* d_run_ctr = nullptr;   // [0] heatbath sweep index, [1] trace row (advanced by the graph)
    double* d_trace = nullptr;       // per block: plaquette, acceptance
    size_t trace_rows = 0;
    bool profiling = false;
    struct Prof {
        cudaEvent_t a, b;
        int cls;
    };
    std::vector<Prof> prof_pending;
    std::vector<cudaEvent_t> event_pool;
    long long prof_launches[SU2G_K_COUNT] = {0};
    double prof_ms[SU2G_K_COUNT] = {0};
    char err[512] = {0};
};

namespace su2g {

int set_error(su2g_lattice* h, int code, const char* fmt, ...);
int check_cuda(su2g_lattice* h, cudaError_t e, const char* what);

// Number of CTAs for a grid-stride kernel over `work` items: at most `per_sm` resident CTAs
// on every SM, never more than needed, never more than kMaxPartials.
int grid_for(const su2g_lattice* h, long long work, int per_sm);

// Grid for a grid-stride kernel whose CTAs must all be resident at once (so that the CTAs in
// flight sweep one contiguous window of the lattice): SMs x resident CTAs of `kernel` per SM.
int resident_grid(const su2g_lattice* h, const void* kernel, long long work, size_t smem = 0);

// Bracket a launch with profiling events when profiling is on; check the launch.
int launch_begin(su2g_lattice* h, int cls);
int launch_end(su2g_lattice* h, int cls, const char* what);

// Make sure the partial-sum scratch holds `slots` x kMaxPartials entries (or at least n entries).
int ensure_partials(su2g_lattice* h, size_t slots);
int ensure_partial_entries(su2g_lattice* h, size_t n);
// Launch k_finalize over `nslots` slots of `nparts` partials (slot k at partials[k * stride],
// stride 0 = kMaxPartials) into d_out[out_off ...].
int finalize(su2g_lattice* h, int nparts, int nslots, double scale, int out_off, int stride = 0);
// Copy n result doubles from d_out[off] to h_out and synchronise; then check the status word.
int fetch_results(su2g_lattice* h, int off, int n);

}  // namespace su2g

namespace su2g {
// Enqueue `ns` smearing steps on the handle's stream (no synchronisation).
int ape_enqueue(su2g_lattice* h, int ns, double alpha, int mode);
// One smearing step from the field at in_dirs into out_dirs (only the smeared directions are written).
int ape_step(su2g_lattice* h, void* const in_dirs[4], void* const out_dirs[4], int mode, double alpha);
// `steps` smearing steps on (cur, alt); the smeared directions swap buffers after every step, so
// the result is at cur.
int ape_run(su2g_lattice* h, void* cur[4], void* alt[4], int steps, int mode, double alpha);
// TMA-tiled APE_all (FP32): rows per CTA if it applies to the geometry, else 0; and its launch.
int ape_tma_rows(const Geom& g, int max_smem);
int ape_tma_launch(su2g_lattice* h, void* const in_dirs[4], void* const out_dirs[4], double alpha, int yb);
// Scratch of the charge kernel (two fields of line products); allocate before any capture.
int ensure_lines(su2g_lattice* h);
// Enqueue Q of the field at dirs (ensure_lines first); Q and sum|q| land in d_out[out_off], d_out[out_off + 1].
int qtop_enqueue(su2g_lattice* h, void* const dirs[4], int out_off);
// FP64 AoS staging (the reference's pu layout) and the conversions of sites [n0, n0 + count)
// between a device AoS buffer and the handle's field.
int ensure_aos(su2g_lattice* h);
int aos_to_field(su2g_lattice* h, const double* d_src, size_t n0, int count);
int field_to_aos(su2g_lattice* h, double* d_dst, size_t n0, int count);
// t_int.c on n_series device series (element i of series s at d_x[i*si + s*ss]); d_out gets
// {mean, tau_int, naive error, error} per series, d_resolved 100 tau <= n (stats.cu).
int tau_int_enqueue(const double* d_x, long long n, long long si, long long ss, int n_series, cudaStream_t stream,
                    double* d_out, int* d_resolved);
// Destroy the captured su2g_measure graph, if any.
void release_meas_graph(su2g_lattice* h);
// Destroy the captured su2g_graph_run block, if any.
void release_run_graph(su2g_lattice* h);
// Enqueue W(R[i], T[i]) of the field at dirs.  Loops are measured in chunks of R and T; each
// chunk's results land in consecutive d_out slots from out_off on, and slot[i] receives the d_out
// index of pair i.  Fails (nothing enqueued) if the pairs need more than `max_slots` slots.
int wilson_enqueue(su2g_lattice* h, void* const dirs[4], const int32_t* R, const int32_t* T, int n, int out_off,
                   int max_slots, int* slot);
// Raise the dynamic shared memory limit of the Wilson loop kernels (once per handle, at creation).
void wilson_prepare(su2g_lattice* h);
// Check R, T >= 1 and T <= L_t - 1 (measureWilsonLoop, wilson.c:290-291).
int wilson_check(su2g_lattice* h, const int32_t* R, const int32_t* T, int n, const char* who);
// Enqueue the plaquette of the current field into d_out[out_off].
int plaquette_enqueue(su2g_lattice* h, int out_off);
// One (mu, parity) update pass.  The heatbath sweep index is `sweep`, plus *sweep_base when
// sweep_base is given (a device counter, so that a captured graph advances it by itself).  With
// plaq_part (parity-1 passes of mu >= 1 only) the pass also writes one plaquette partial per CTA.
int launch_update(su2g_lattice* h, int kind, int mu, int par, uint32_t sweep, double* acc_sum,
                  const uint32_t* sweep_base = nullptr, DD* plaq_part = nullptr);
// CTAs of an update pass (one link per thread), and the plaquette partials of a fused pass.
int update_grid(const su2g_lattice* h);
int update_plaq_parts(const su2g_lattice* h);
// Enqueue n_sweeps x (n_hb heatbath + n_or overrelaxation sweeps); heatbath sub-sweep j (counted
// from 0 within the call) has index sweep0 + j (+ *base).  With plaq_off >= 0 the last sub-sweep
// also sums the plaquette of the final field into d_out[plaq_off] (the plaquette kernel runs
// instead when there is no sub-sweep); partials[0 .. 3 * update_plaq_parts) are used.
int sweep_enqueue(su2g_lattice* h, int n_sweeps, int n_hb, int n_or, uint32_t sweep0, const uint32_t* base,
                  double* acc_dev, int plaq_off);
}  // namespace su2g
