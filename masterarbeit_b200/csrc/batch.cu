// batch.cu -- many independent lattices (replicas) updated and measured together.
//
// The reference runs one lattice per process (its thesis runs were separate processes, one per
// hot/cold start and id).  Here a batch holds R replicas of possibly different extents, beta,
// seed and start in one device pool.  A replica-offset table maps every CTA of a launch to its
// replica, so one launch per checkerboard pass (mu, parity) updates all replicas, and one launch
// measures every replica's plaquette.  A whole measurement block (meas_every sweeps of n_hb
// heatbath + n_or overrelaxation passes, then the plaquettes) is captured once in a CUDA graph and
// replayed; the Philox sweep index and the measurement slot live in device counters that the graph
// advances itself.  Each replica draws the same Philox streams as a single-lattice handle with the
// same (seed, replica id), so a batch and a set of single handles give identical fields.
//
// Persistent form.  Alternatively one cooperative launch runs every measurement block of a
// su2g_batch_run: its CTAs (all resident) walk the links of each pass as one global index over all
// replicas, in tiles of one CTA's width, so small replicas share a CTA, and meet at a grid-wide
// barrier between passes.  The barrier's wait is bounded: a CTA that waits too long raises
// kStatusGridTimeout and every CTA leaves at its next barrier.  su2g_batch_autotune times both
// forms over CTA widths and keeps the fastest.
#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "internal.cuh"
#include "philox.cuh"
#include "update.cuh"

using namespace su2g;

namespace {

struct Replica {
    Geom g;
    double beta;
    uint64_t seed;
    uint32_t id;
    int start;
    void* dirs[4];
};

enum { kCtrSweep = 0, kCtrMeas = 1 };

// Grid-wide barrier state of the persistent form (zeroed before every launch).
struct GridBarrier {
    unsigned count, gen, abort, pad;
};

}  // namespace

struct su2g_batch {
    int n = 0, prec = SU2G_FP32, device = 0, num_sms = 148, block = 256;
    size_t link_bytes = 16;
    std::vector<Replica> reps;
    Replica* d_reps = nullptr;
    int *d_umap = nullptr, *d_smap = nullptr;     // CTA -> replica for link / site launches
    std::vector<int> ublk, sblk;                   // first CTA of each replica (+ total)
    void* pool = nullptr;
    size_t pool_bytes = 0;
    DD* partials = nullptr;
    uint32_t* d_ctr = nullptr;                     // [sweep index, measurement slot]
    unsigned* d_status = nullptr;
    double* d_trace = nullptr;
    size_t trace_cap = 0;
    int trace_rows = 0;                            // measurements in the trace of the last run
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    int g_hb = -1, g_or = -1, g_meas = -1, g_every = -1, g_block = -1;
    int mode = SU2G_BATCH_GRAPH;                   // su2g_batch_mode
    int* d_upre = nullptr;                         // first global link index of each replica in a pass (n+1)
    GridBarrier* d_gb = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    char err[512] = {0};
};

namespace {

int berr(su2g_batch* b, int code, const char* fmt, ...)
{
    char* dst = b->err;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(dst, sizeof(b->err), fmt, ap);
    va_end(ap);
    return code;
}

int bcuda(su2g_batch* b, cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return SU2G_OK;
    return berr(b, e == cudaErrorMemoryAllocation ? SU2G_ENOMEM : SU2G_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

template <typename R>
__device__ __forceinline__ Field<R> rep_field(const Replica& r)
{
    Field<R> f;
    for (int mu = 0; mu < 4; ++mu) f.p[mu] = reinterpret_cast<typename Field<R>::ptr_t>(r.dirs[mu]);
    f.Vh = r.g.Vh;
    return f;
}

template <typename R, int MU, int KIND>
__global__ void __launch_bounds__(256, 4) k_batch_update(const Replica* __restrict__ reps, const int* __restrict__ map,
                                                      const int* __restrict__ blk0, int par, int sub,
                                                      const uint32_t* __restrict__ ctr, unsigned* __restrict__ status)
{
    const int r = map[blockIdx.x];
    const Replica& rp = reps[r];
    const Geom g = rp.g;
    const int h = (blockIdx.x - blk0[r]) * blockDim.x + threadIdx.x;
    if (h >= g.Vh) return;
    const Field<R> U = rep_field<R>(rp);
    const Site s = site_of(g, par, h);
    const Q<R> A = staple_update<R, MU>(U, g, s, par);
    if (KIND == SU2G_HEATBATH) {
        Q<R> out;
        uint32_t trials = 0;
        if (heatbath_link<R>(A, (R)rp.beta, rp.seed, (uint32_t)s.n, ctr[kCtrSweep] + sub, (uint32_t)MU, rp.id, trials,
                             out, status))
            U.sth(MU, par, h, hb_store(out));
    } else {
        U.sth(MU, par, h, q_project(overrelax_link<R>(A, U.ldh(MU, par, h))));
    }
}

template <typename R>
__global__ void __launch_bounds__(256) k_batch_plaquette(const Replica* __restrict__ reps, const int* __restrict__ map,
                                                         const int* __restrict__ blk0, DD* __restrict__ partials)
{
    const int r = map[blockIdx.x];
    const Replica& rp = reps[r];
    const Geom g = rp.g;
    const int i = (blockIdx.x - blk0[r]) * blockDim.x + threadIdx.x;
    double site = 0.0;
    if (i < g.V) {
        const Field<R> U = rep_field<R>(rp);
        int par;
        const Site s = site_lex(g, i, par);
        const int h = i >> 1, q = par ^ 1;
#pragma unroll
        for (int mu = 0; mu < 3; ++mu)
#pragma unroll
            for (int nu = mu + 1; nu < 4; ++nu) {
                const Q<R> a = q_mul(U.ldh(mu, par, h), U.ld(nu, q, s.n + up_off_rt(g, s.c, mu)));
                const Q<R> b = q_mul(U.ldh(nu, par, h), U.ld(mu, q, s.n + up_off_rt(g, s.c, nu)));
                site += (double)q_dot(a, b);
            }
    }
    // block sums with 256 threads at most; inactive threads contribute 0
    __shared__ DD part[8];
    DD v = dd_warp_sum(DD{site, 0.0});
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        DD w = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : DD{0.0, 0.0};
        w = dd_warp_sum(w);
        if (threadIdx.x == 0) partials[blockIdx.x] = w;
    }
}

// One CTA per replica: fixed-order sum of its CTAs' partials into trace[slot][r].
__global__ void __launch_bounds__(kBlock) k_batch_plaq_final(const Replica* __restrict__ reps,
                                                             const int* __restrict__ blk0, const DD* __restrict__ partials,
                                                             int nrep, double* __restrict__ trace,
                                                             const uint32_t* __restrict__ ctr)
{
    const int r = blockIdx.x;
    DD acc = {0.0, 0.0};
    for (int b = blk0[r] + threadIdx.x; b < blk0[r + 1]; b += blockDim.x) acc = dd_add(acc, partials[b]);
    acc = dd_block_sum<kBlock>(acc);
    if (threadIdx.x == 0) trace[(size_t)ctr[kCtrMeas] * nrep + r] = (acc.s + acc.e) / (6.0 * (double)reps[r].g.V);
}

__global__ void k_batch_tick(uint32_t* ctr, int n_hb, int meas)
{
    ctr[kCtrSweep] += (uint32_t)n_hb;
    ctr[kCtrMeas] += (uint32_t)meas;
}

template <typename R>
__global__ void __launch_bounds__(256) k_batch_start(const Replica* __restrict__ reps, const int* __restrict__ map,
                                                     const int* __restrict__ blk0)
{
    const int r = map[blockIdx.x];
    const Replica& rp = reps[r];
    const Geom g = rp.g;
    const int i = (blockIdx.x - blk0[r]) * blockDim.x + threadIdx.x;
    if (i >= g.V) return;
    const Field<R> U = rep_field<R>(rp);
    int par;
    const Site s = site_lex(g, i, par);
    const int h = i >> 1;
    for (int mu = 0; mu < 4; ++mu) {
        Q<R> u = q_one<R>();
        if (rp.start != SU2G_START_COLD) {
            U4 w = link_random(rp.seed, (uint32_t)s.n, 0u, (uint32_t)mu, 0u, 0u, kStreamStart, rp.id);
            const R r0 = u01(w.x, R(0)), r1 = u01(w.y, R(0)), r2 = u01(w.z, R(0)), r3 = u01(w.w, R(0));
            if (rp.start == SU2G_START_REF) {
                u = fallback_link<R>(r0, r1, r2);
            } else {
                const R ra = sqrt_r(R(-2) * log(r0)), rb = sqrt_r(R(-2) * log(r2));
                R sa, ca, sb, cb;
                sincospi(R(2) * r1, &sa, &ca);
                sincospi(R(2) * r3, &sb, &cb);
                u = q_project(q_make<R>(ra * ca, ra * sa, rb * cb, rb * sb));
            }
        }
        U.sth(mu, par, h, u);
    }
}

template <typename R>
__global__ void __launch_bounds__(256) k_batch_aos(const Replica* __restrict__ reps, int r, double2* __restrict__ aos,
                                                   int to_host)
{
    const Replica& rp = reps[r];
    const Geom g = rp.g;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.V) return;
    const Field<R> U = rep_field<R>(rp);
    uint32_t t = fdiv((uint32_t)n, g.dS0), rr = (uint32_t)n - t * (uint32_t)g.S[0];
    uint32_t x = fdiv(rr, g.dS1);
    rr -= x * (uint32_t)g.S[1];
    uint32_t y = fdiv(rr, g.dS2), z = rr - y * (uint32_t)g.S[2];
    const int par = (int)((t + x + y + z) & 1u);
    for (int mu = 0; mu < 4; ++mu) {
        double2* a = aos + (size_t)n * 8 + 2 * mu;
        if (to_host) {
            const Q<R> q = U.ldh(mu, par, n >> 1);
            a[0] = make_double2((double)q.c0, (double)q.c1);
            a[1] = make_double2((double)q.c2, (double)q.c3);
        } else {
            U.sth(mu, par, n >> 1, q_make<R>((R)a[0].x, (R)a[0].y, (R)a[1].x, (R)a[1].y));
        }
    }
}

// ---------------------------------------------------------------- persistent form ---

constexpr long long kGridWaitCycles = 4000000000ll;   // about 2 s at the B200's clock

// Grid-wide barrier of a cooperative launch (every CTA resident).  Thread 0 of each CTA arrives on
// a counter; the last of `arrivals` (default: every CTA) resets it and advances the generation the
// others poll.  The poll gives up
// after kGridWaitCycles or when another CTA has given up; then the CTA raises kStatusGridTimeout and
// every CTA returns false here, now or at its next barrier, so none is left waiting.  The fences
// make the field writes of the pass before the barrier visible to the loads after it.
__device__ __forceinline__ bool grid_sync(GridBarrier* gb, unsigned* status, unsigned arrivals = 0u,
                                          long long wait_cycles = kGridWaitCycles)
{
    if (arrivals == 0u) arrivals = gridDim.x;
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = &gb->gen;
        volatile unsigned* vabort = &gb->abort;
        const unsigned g0 = *vgen;
        int ok = 1;
        __threadfence();
        if (atomicAdd(&gb->count, 1u) == arrivals - 1) {
            atomicExch(&gb->count, 0u);
            __threadfence();
            atomicAdd(&gb->gen, 1u);
        } else {
            const long long t0 = clock64();
            while (*vgen == g0) {
                if (*vabort || clock64() - t0 > wait_cycles) {
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        if (!ok) {
            atomicExch(&gb->abort, 1u);
            atomicOr(status, kStatusGridTimeout);
        }
        __threadfence();
        s_ok = ok && !*vabort;
    }
    __syncthreads();
    return s_ok != 0;
}

struct PersistArgs {
    const Replica* reps;
    const int* upre;     // n+1 first global link index of each replica in a pass
    const int* smap;     // site chunk -> replica, chunks of blockDim sites (the plaquette)
    const int* sblk;     // n+1 first site chunk of each replica
    int n, nblocks, every, n_hb, n_or, meas;
    uint32_t* ctr;
    double* trace;
    DD* partials;
    GridBarrier* gb;
    unsigned* status;
};

template <typename R>
__device__ __forceinline__ FieldCG<R> rep_field_cg(const Replica& r)
{
    FieldCG<R> f;
    for (int mu = 0; mu < 4; ++mu) f.p[mu] = reinterpret_cast<typename Field<R>::ptr_t>(r.dirs[mu]);
    f.Vh = r.g.Vh;
    return f;
}

// One checkerboard pass (mu, par) over every replica: global link index gi over all replicas, tiles
// of one CTA's width, tile k handled by CTA k mod gridDim (in order, so the CTAs in flight cover a
// contiguous window of the pool).  The link of gi is h = gi - upre[r] of the replica r with
// upre[r] <= gi < upre[r+1] (binary search in shared memory).
template <typename R, int MU, int KIND>
__device__ __forceinline__ void persist_pass(const PersistArgs& a, const int* __restrict__ s_pre, int par,
                                             uint32_t sweep)
{
    const int total = s_pre[a.n];
    for (int gi = blockIdx.x * blockDim.x + threadIdx.x; gi < total; gi += gridDim.x * blockDim.x) {
        int lo = 0, hi = a.n;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_pre[mid] <= gi) lo = mid;
            else hi = mid;
        }
        const Replica& rp = a.reps[lo];
        const Geom g = rp.g;
        const int h = gi - s_pre[lo];
        const FieldCG<R> U = rep_field_cg<R>(rp);
        const Site s = site_of(g, par, h);
        const Q<R> A = staple_update<R, MU, 0, FieldCG<R>>(U, g, s, par);
        if (KIND == SU2G_HEATBATH) {
            Q<R> out;
            uint32_t trials = 0;
            if (heatbath_link<R>(A, (R)rp.beta, rp.seed, (uint32_t)s.n, sweep, (uint32_t)MU, rp.id, trials, out,
                                 a.status))
                U.sth(MU, par, h, hb_store(out));
        } else {
            U.sth(MU, par, h, q_project(overrelax_link<R>(A, U.ldh(MU, par, h))));
        }
    }
}

template <typename R, int KIND>
__device__ __forceinline__ void persist_pass_mu(const PersistArgs& a, const int* s_pre, int mu, int par, uint32_t sweep)
{
    switch (mu) {
        case 0: persist_pass<R, 0, KIND>(a, s_pre, par, sweep); break;
        case 1: persist_pass<R, 1, KIND>(a, s_pre, par, sweep); break;
        case 2: persist_pass<R, 2, KIND>(a, s_pre, par, sweep); break;
        default: persist_pass<R, 3, KIND>(a, s_pre, par, sweep); break;
    }
}

// Every measurement block of a run in one launch: `every` sweeps of n_hb heatbath and n_or
// overrelaxation passes, then (if meas) each replica's plaquette into its trace slot, exactly the
// work and the Philox streams of the replayed graph of launches.
template <typename R, int NT>
__global__ void __launch_bounds__(NT, (sizeof(R) == 8 ? 512 : 1024) / NT) k_batch_persist(PersistArgs a)
{
    extern __shared__ int s_pre[];
    for (int i = threadIdx.x; i <= a.n; i += NT) s_pre[i] = a.upre[i];
    __syncthreads();
    // every CTA reads the counters here; CTA 0 writes them back only after the last barrier
    uint32_t sweep = a.ctr[kCtrSweep], slot = a.ctr[kCtrMeas];
    const int nchunks = a.sblk[a.n];
    for (int blk = 0; blk < a.nblocks; ++blk) {
        for (int s = 0; s < a.every; ++s) {
            for (int i = 0; i < a.n_hb; ++i, ++sweep)
                for (int mu = 0; mu < 4; ++mu)
                    for (int par = 0; par < 2; ++par) {
                        persist_pass_mu<R, SU2G_HEATBATH>(a, s_pre, mu, par, sweep);
                        if (!grid_sync(a.gb, a.status)) return;
                    }
            for (int i = 0; i < a.n_or; ++i)
                for (int mu = 0; mu < 4; ++mu)
                    for (int par = 0; par < 2; ++par) {
                        persist_pass_mu<R, SU2G_OVERRELAX>(a, s_pre, mu, par, 0u);
                        if (!grid_sync(a.gb, a.status)) return;
                    }
        }
        if (!a.meas) continue;
        // plaquette partials: site chunk c of replica r covers sites (c - sblk[r]) NT .. + NT - 1
        for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
            const int r = a.smap[c];
            const Replica& rp = a.reps[r];
            const Geom g = rp.g;
            const int i = (c - a.sblk[r]) * NT + threadIdx.x;
            double site = 0.0;
            if (i < g.V) {
                const FieldCG<R> U = rep_field_cg<R>(rp);
                int par;
                const Site st = site_lex(g, i, par);
                const int h = i >> 1, q = par ^ 1;
#pragma unroll
                for (int mu = 0; mu < 3; ++mu)
#pragma unroll
                    for (int nu = mu + 1; nu < 4; ++nu) {
                        const Q<R> x = q_mul(U.ldh(mu, par, h), U.ld(nu, q, st.n + up_off_rt(g, st.c, mu)));
                        const Q<R> y = q_mul(U.ldh(nu, par, h), U.ld(mu, q, st.n + up_off_rt(g, st.c, nu)));
                        site += (double)q_dot(x, y);
                    }
            }
            const DD v = dd_block_sum<NT>(DD{site, 0.0});
            if (threadIdx.x == 0) a.partials[c] = v;
        }
        if (!grid_sync(a.gb, a.status)) return;
        // one CTA per replica: fixed-order sum of its chunks' partials
        for (int r = blockIdx.x; r < a.n; r += gridDim.x) {
            DD acc = {0.0, 0.0};
            for (int c = a.sblk[r] + threadIdx.x; c < a.sblk[r + 1]; c += NT)
                acc = dd_add(acc, DD{__ldcg(&a.partials[c].s), __ldcg(&a.partials[c].e)});
            acc = dd_block_sum<NT>(acc);
            if (threadIdx.x == 0) a.trace[(size_t)slot * a.n + r] = (acc.s + acc.e) / (6.0 * (double)a.reps[r].g.V);
        }
        ++slot;
        if (!grid_sync(a.gb, a.status)) return;   // the partials are written again by the next block
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.ctr[kCtrSweep] = sweep;
        a.ctr[kCtrMeas] = slot;
    }
}

// CTA maps for a block size: CTAs of replica r are [blk[r], blk[r+1]).
int build_maps(su2g_batch* b, int block)
{
    std::vector<int> umap, smap;
    b->ublk.assign(b->n + 1, 0);
    b->sblk.assign(b->n + 1, 0);
    for (int r = 0; r < b->n; ++r) {
        const int nu = (b->reps[r].g.Vh + block - 1) / block, ns = (b->reps[r].g.V + block - 1) / block;
        b->ublk[r + 1] = b->ublk[r] + nu;
        b->sblk[r + 1] = b->sblk[r] + ns;
        umap.insert(umap.end(), nu, r);
        smap.insert(smap.end(), ns, r);
    }
    if (b->graph) cudaGraphExecDestroy(b->graph);   // a captured graph holds the old maps
    b->graph = nullptr;
    cudaFree(b->d_umap);
    cudaFree(b->d_smap);
    b->d_umap = b->d_smap = nullptr;
    // each map is followed by the n+1 first-CTA table
    int rc = bcuda(b, cudaMalloc(&b->d_umap, (umap.size() + b->n + 1) * sizeof(int)), "allocating CTA maps");
    if (!rc) rc = bcuda(b, cudaMalloc(&b->d_smap, (smap.size() + b->n + 1) * sizeof(int)), "allocating CTA maps");
    if (!rc) rc = bcuda(b, cudaMemcpy(b->d_umap, umap.data(), umap.size() * sizeof(int), cudaMemcpyHostToDevice), "maps");
    if (!rc)
        rc = bcuda(b, cudaMemcpy(b->d_umap + umap.size(), b->ublk.data(), (b->n + 1) * sizeof(int), cudaMemcpyHostToDevice),
                   "maps");
    if (!rc) rc = bcuda(b, cudaMemcpy(b->d_smap, smap.data(), smap.size() * sizeof(int), cudaMemcpyHostToDevice), "maps");
    if (!rc)
        rc = bcuda(b, cudaMemcpy(b->d_smap + smap.size(), b->sblk.data(), (b->n + 1) * sizeof(int), cudaMemcpyHostToDevice),
                   "maps");
    cudaFree(b->partials);
    b->partials = nullptr;
    if (!rc) rc = bcuda(b, cudaMalloc(&b->partials, smap.size() * sizeof(DD)), "allocating partial sums");
    b->block = block;
    return rc;
}

const int* ublk0(const su2g_batch* b) { return b->d_umap + b->ublk[b->n]; }
const int* sblk0(const su2g_batch* b) { return b->d_smap + b->sblk[b->n]; }

template <typename R, int KIND>
void launch_pass(su2g_batch* b, int mu, int par, int sub)
{
    const int grid = b->ublk[b->n];
    switch (mu) {
        case 0: k_batch_update<R, 0, KIND><<<grid, b->block, 0, b->stream>>>(b->d_reps, b->d_umap, ublk0(b), par, sub, b->d_ctr, b->d_status); break;
        case 1: k_batch_update<R, 1, KIND><<<grid, b->block, 0, b->stream>>>(b->d_reps, b->d_umap, ublk0(b), par, sub, b->d_ctr, b->d_status); break;
        case 2: k_batch_update<R, 2, KIND><<<grid, b->block, 0, b->stream>>>(b->d_reps, b->d_umap, ublk0(b), par, sub, b->d_ctr, b->d_status); break;
        default: k_batch_update<R, 3, KIND><<<grid, b->block, 0, b->stream>>>(b->d_reps, b->d_umap, ublk0(b), par, sub, b->d_ctr, b->d_status); break;
    }
}

// The launches of one measurement block: `every` sweeps, then (if meas) the plaquettes.
template <typename R>
void enqueue_block(su2g_batch* b, int n_hb, int n_or, int every, int meas)
{
    for (int s = 0; s < every; ++s) {
        for (int i = 0; i < n_hb; ++i)
            for (int mu = 0; mu < 4; ++mu)
                for (int par = 0; par < 2; ++par) launch_pass<R, SU2G_HEATBATH>(b, mu, par, s * n_hb + i);
        for (int i = 0; i < n_or; ++i)
            for (int mu = 0; mu < 4; ++mu)
                for (int par = 0; par < 2; ++par) launch_pass<R, SU2G_OVERRELAX>(b, mu, par, 0);
    }
    if (meas) {
        k_batch_plaquette<R><<<b->sblk[b->n], b->block, 0, b->stream>>>(b->d_reps, b->d_smap, sblk0(b), b->partials);
        k_batch_plaq_final<<<b->n, kBlock, 0, b->stream>>>(b->d_reps, sblk0(b), b->partials, b->n, b->d_trace, b->d_ctr);
    }
    k_batch_tick<<<1, 1, 0, b->stream>>>(b->d_ctr, n_hb * every, meas);
}

int ensure_graph(su2g_batch* b, int n_hb, int n_or, int every, int meas)
{
    if (b->graph && b->g_hb == n_hb && b->g_or == n_or && b->g_every == every && b->g_meas == meas &&
        b->g_block == b->block)
        return SU2G_OK;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    cudaGraph_t gr = nullptr;
    int rc = bcuda(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "beginning graph capture");
    if (rc) return rc;
    if (b->prec == SU2G_FP32) enqueue_block<float>(b, n_hb, n_or, every, meas);
    else enqueue_block<double>(b, n_hb, n_or, every, meas);
    cudaError_t launch_err = cudaGetLastError();
    rc = bcuda(b, cudaStreamEndCapture(b->stream, &gr), "ending graph capture");
    if (!rc) rc = bcuda(b, launch_err, "capturing the sweep");
    if (!rc) rc = bcuda(b, cudaGraphInstantiate(&b->graph, gr, 0), "instantiating the sweep graph");
    if (gr) cudaGraphDestroy(gr);
    if (rc) return rc;
    b->g_hb = n_hb;
    b->g_or = n_or;
    b->g_every = every;
    b->g_meas = meas;
    b->g_block = b->block;
    return SU2G_OK;
}

// Diagnostic of the bounded barrier: two barriers that wait for `arrivals` CTAs.  With one arrival
// more than the grid has, nobody is last, every CTA gives up after wait_cycles and the status word
// says so; nothing faults and no CTA is left waiting.
__global__ void __launch_bounds__(128) k_grid_selftest(GridBarrier* gb, unsigned* status, unsigned arrivals,
                                                       long long wait_cycles)
{
    if (!grid_sync(gb, status, arrivals, wait_cycles)) return;
    grid_sync(gb, status, arrivals, wait_cycles);
}

template <typename R, int NT>
int launch_persist_t(su2g_batch* b, const PersistArgs& a)
{
    const size_t smem = (size_t)(b->n + 1) * sizeof(int);
    int per_sm = 0;
    int rc = bcuda(b, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_persist<R, NT>, NT, smem),
                   "occupancy of the persistent sweep");
    if (rc) return rc;
    if (per_sm < 1) return berr(b, SU2G_ECUDA, "the persistent sweep kernel does not fit on an SM");
    const int grid = b->num_sms * per_sm;   // all resident: the cooperative launch checks it
    PersistArgs args = a;
    void* params[] = {&args};
    return bcuda(b, cudaLaunchCooperativeKernel((const void*)k_batch_persist<R, NT>, dim3(grid), dim3(NT), params, smem,
                                                b->stream),
                 "launching the persistent sweep");
}

// Every block of a run as one cooperative launch (the persistent form).
int launch_persist(su2g_batch* b, int nblocks, int n_hb, int n_or, int every, int meas)
{
    PersistArgs a;
    a.reps = b->d_reps;
    a.upre = b->d_upre;
    a.smap = b->d_smap;
    a.sblk = sblk0(b);
    a.n = b->n;
    a.nblocks = nblocks;
    a.every = every;
    a.n_hb = n_hb;
    a.n_or = n_or;
    a.meas = meas;
    a.ctr = b->d_ctr;
    a.trace = b->d_trace;
    a.partials = b->partials;
    a.gb = b->d_gb;
    a.status = b->d_status;
    int rc = bcuda(b, cudaMemsetAsync(b->d_gb, 0, sizeof(GridBarrier), b->stream), "clearing the grid barrier");
    if (rc) return rc;
    if (b->block == 128)
        return b->prec == SU2G_FP32 ? launch_persist_t<float, 128>(b, a) : launch_persist_t<double, 128>(b, a);
    return b->prec == SU2G_FP32 ? launch_persist_t<float, 256>(b, a) : launch_persist_t<double, 256>(b, a);
}

int check_status(su2g_batch* b)
{
    unsigned st = 0;
    int rc = bcuda(b, cudaMemcpy(&st, b->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost), "reading status");
    if (rc) return rc;
    if (st) cudaMemset(b->d_status, 0, sizeof(unsigned));   // reported once; the batch stays usable
    if (st & kStatusKpTrials) return berr(b, SU2G_EDEVICE, "a heatbath link exceeded %u Kennedy-Pendleton trials", kMaxTrials);
    if (st & kStatusGridTimeout)
        return berr(b, SU2G_EDEVICE, "the persistent sweep gave up waiting at a grid-wide barrier (the fields are not valid)");
    if (st) return berr(b, SU2G_EDEVICE, "device status word 0x%x", st);
    return SU2G_OK;
}

}  // namespace

extern "C" const char* su2g_batch_last_error(const su2g_batch* b) { return b ? b->err : su2g_last_error(nullptr); }

extern "C" int su2g_batch_destroy(su2g_batch* b)
{
    if (!b) return SU2G_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    cudaFree(b->d_reps);
    cudaFree(b->d_umap);
    cudaFree(b->d_smap);
    cudaFree(b->pool);
    cudaFree(b->partials);
    cudaFree(b->d_ctr);
    cudaFree(b->d_status);
    cudaFree(b->d_trace);
    cudaFree(b->d_upre);
    cudaFree(b->d_gb);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return SU2G_OK;
}

extern "C" int su2g_batch_create(const su2g_replica* reps, int32_t n, int32_t precision, int32_t device,
                                 su2g_batch** out)
{
    if (!reps || !out || n <= 0) return set_error(nullptr, SU2G_EINVAL, "su2g_batch_create: bad argument");
    *out = nullptr;
    if (precision != SU2G_FP32 && precision != SU2G_FP64)
        return set_error(nullptr, SU2G_EINVAL, "su2g_batch_create: unknown precision %d", precision);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
        return set_error(nullptr, SU2G_ENODEV, "su2g_batch_create: no CUDA device visible");
    if (device < 0 || device >= ndev) return set_error(nullptr, SU2G_EINVAL, "su2g_batch_create: bad device %d", device);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10)
        return set_error(nullptr, SU2G_ENODEV, "su2g_batch_create: device %d is not sm_100 class", device);
    cudaSetDevice(device);
    su2g_batch* b = new (std::nothrow) su2g_batch();
    if (!b) return set_error(nullptr, SU2G_ENOMEM, "su2g_batch_create: out of host memory");
    b->n = n;
    b->prec = precision;
    b->device = device;
    b->num_sms = prop.multiProcessorCount;
    b->link_bytes = precision == SU2G_FP32 ? 16 : 32;
    size_t total = 0;
    std::vector<size_t> off(n);
    for (int r = 0; r < n; ++r) {
        long long V = 1;
        for (int d = 0; d < 4; ++d) {
            if (reps[r].dims[d] < 2 || (reps[r].dims[d] & 1)) {
                set_error(nullptr, SU2G_EINVAL, "su2g_batch_create: replica %d: extent %d must be even and >= 2", r,
                          reps[r].dims[d]);
                su2g_batch_destroy(b);
                return SU2G_EINVAL;
            }
            V *= reps[r].dims[d];
        }
        if (V > (1ll << 30) || reps[r].start < SU2G_START_COLD || reps[r].start > SU2G_START_REF) {
            set_error(nullptr, SU2G_EINVAL, "su2g_batch_create: replica %d: bad volume or start mode", r);
            su2g_batch_destroy(b);
            return SU2G_EINVAL;
        }
        Replica rp;
        rp.g = make_geom(reps[r].dims);
        rp.beta = reps[r].beta;
        rp.seed = reps[r].seed;
        rp.id = reps[r].replica;
        rp.start = reps[r].start;
        off[r] = total;
        total += ((4ull * V * b->link_bytes) + 255) / 256 * 256;
        b->reps.push_back(rp);
    }
    b->pool_bytes = total;
    int rc = bcuda(b, cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "creating stream");
    if (!rc) rc = bcuda(b, cudaMalloc(&b->pool, total), "allocating the replica pool");
    if (!rc)
        for (int r = 0; r < n; ++r)
            for (int mu = 0; mu < 4; ++mu)
                b->reps[r].dirs[mu] = (char*)b->pool + off[r] + (size_t)mu * 2 * b->reps[r].g.Vh * b->link_bytes;
    if (!rc) rc = bcuda(b, cudaMalloc(&b->d_reps, n * sizeof(Replica)), "allocating the replica table");
    if (!rc) rc = bcuda(b, cudaMemcpy(b->d_reps, b->reps.data(), n * sizeof(Replica), cudaMemcpyHostToDevice), "table");
    if (!rc) {
        std::vector<int> upre(n + 1, 0);
        long long tot = 0;
        for (int r = 0; r < n; ++r) {
            upre[r] = (int)tot;
            tot += b->reps[r].g.Vh;
        }
        if (tot > (1ll << 30)) rc = berr(b, SU2G_EINVAL, "the replicas hold more than 2^31 links");
        upre[n] = (int)tot;
        if (!rc) rc = bcuda(b, cudaMalloc(&b->d_upre, (n + 1) * sizeof(int)), "allocating the link prefix table");
        if (!rc) rc = bcuda(b, cudaMemcpy(b->d_upre, upre.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice), "table");
        if (!rc) rc = bcuda(b, cudaMalloc(&b->d_gb, sizeof(GridBarrier)), "allocating the grid barrier");
    }
    if (!rc) rc = bcuda(b, cudaMalloc(&b->d_ctr, 2 * sizeof(uint32_t)), "allocating counters");
    if (!rc) rc = bcuda(b, cudaMemset(b->d_ctr, 0, 2 * sizeof(uint32_t)), "clearing counters");
    if (!rc) rc = bcuda(b, cudaMalloc(&b->d_status, sizeof(unsigned)), "allocating status");
    if (!rc) rc = bcuda(b, cudaMemset(b->d_status, 0, sizeof(unsigned)), "clearing status");
    if (!rc) rc = bcuda(b, cudaEventCreate(&b->ev0), "events");
    if (!rc) rc = bcuda(b, cudaEventCreate(&b->ev1), "events");
    if (!rc) rc = build_maps(b, 256);
    if (!rc) {
        if (precision == SU2G_FP32) k_batch_start<float><<<b->sblk[n], b->block, 0, b->stream>>>(b->d_reps, b->d_smap, sblk0(b));
        else k_batch_start<double><<<b->sblk[n], b->block, 0, b->stream>>>(b->d_reps, b->d_smap, sblk0(b));
        rc = bcuda(b, cudaGetLastError(), "start kernel");
    }
    if (!rc) rc = bcuda(b, cudaStreamSynchronize(b->stream), "initialising replicas");
    if (rc) {
        set_error(nullptr, rc, "su2g_batch_create: %s", b->err);
        su2g_batch_destroy(b);
        return rc;
    }
    *out = b;
    return SU2G_OK;
}

extern "C" int su2g_batch_run(su2g_batch* b, int32_t n_sweeps, int32_t n_hb, int32_t n_or, int32_t meas_every,
                              double* plaq_trace, double* ms)
{
    if (!b) return set_error(nullptr, SU2G_EINVAL, "su2g_batch_run: null batch");
    if (n_sweeps < 0 || n_hb < 0 || n_or < 0 || meas_every < 0 || (meas_every > 0 && n_sweeps % meas_every))
        return berr(b, SU2G_EINVAL, "su2g_batch_run: bad counts (n_sweeps must be a multiple of meas_every)");
    cudaSetDevice(b->device);
    const int every = meas_every > 0 ? meas_every : 1;
    const int meas = meas_every > 0;
    const int nblocks = n_sweeps / every;
    int rc = SU2G_OK;
    if (meas && (size_t)nblocks * b->n > b->trace_cap) {
        cudaFree(b->d_trace);
        b->d_trace = nullptr;
        b->trace_cap = 0;
        if ((rc = bcuda(b, cudaMalloc(&b->d_trace, (size_t)nblocks * b->n * sizeof(double)), "allocating the trace")))
            return rc;
        b->trace_cap = (size_t)nblocks * b->n;
        if (b->graph) cudaGraphExecDestroy(b->graph);   // the graph holds the old trace pointer
        b->graph = nullptr;
    }
    if (!b->d_trace) {
        if ((rc = bcuda(b, cudaMalloc(&b->d_trace, b->n * sizeof(double)), "allocating the trace"))) return rc;
        b->trace_cap = b->n;
    }
    const bool persist = b->mode == SU2G_BATCH_PERSISTENT;
    if (!persist && (rc = ensure_graph(b, n_hb, n_or, every, meas))) return rc;
    // measurement slots restart at 0 for every run
    uint32_t zero = 0;
    if ((rc = bcuda(b, cudaMemcpyAsync(b->d_ctr + kCtrMeas, &zero, sizeof(zero), cudaMemcpyHostToDevice, b->stream),
                    "resetting the slot counter")))
        return rc;
    cudaEventRecord(b->ev0, b->stream);
    if (persist) {
        if (nblocks > 0 && (rc = launch_persist(b, nblocks, n_hb, n_or, every, meas))) return rc;
    } else {
        for (int i = 0; i < nblocks; ++i)
            if ((rc = bcuda(b, cudaGraphLaunch(b->graph, b->stream), "launching the sweep graph"))) return rc;
    }
    cudaEventRecord(b->ev1, b->stream);
    if ((rc = bcuda(b, cudaStreamSynchronize(b->stream), "running sweeps"))) return rc;
    if (ms) {
        float f = 0.f;
        cudaEventElapsedTime(&f, b->ev0, b->ev1);
        *ms = f;
    }
    if ((rc = check_status(b))) return rc;
    b->trace_rows = meas ? nblocks : 0;
    if (meas && plaq_trace && nblocks > 0)
        rc = bcuda(b, cudaMemcpy(plaq_trace, b->d_trace, (size_t)nblocks * b->n * sizeof(double), cudaMemcpyDeviceToHost),
                   "copying the trace");
    return rc;
}

extern "C" int su2g_batch_tau_int(su2g_batch* b, int32_t skip, double* out, int32_t* resolved)
{
    if (!b) return set_error(nullptr, SU2G_EINVAL, "su2g_batch_tau_int: null batch");
    if (!out || skip < 0 || b->trace_rows - skip < 2)
        return berr(b, SU2G_EINVAL, "su2g_batch_tau_int: needs an output and at least 2 measurements after skip "
                                    "(trace has %d)", b->trace_rows);
    cudaSetDevice(b->device);
    double* d_out = nullptr;
    int* d_res = nullptr;
    int rc = bcuda(b, cudaMalloc(&d_out, 4 * (size_t)b->n * sizeof(double)), "allocating results");
    if (!rc) rc = bcuda(b, cudaMalloc(&d_res, (size_t)b->n * sizeof(int)), "allocating results");
    // trace[meas][replica]: series r has stride n and starts at row `skip`
    if (!rc && tau_int_enqueue(b->d_trace + (size_t)skip * b->n, b->trace_rows - skip, b->n, 1, b->n, b->stream, d_out,
                               d_res))
        rc = berr(b, SU2G_ECUDA, "su2g_batch_tau_int: %s", su2g_last_error(nullptr));
    if (!rc)
        rc = bcuda(b, cudaMemcpyAsync(out, d_out, 4 * (size_t)b->n * sizeof(double), cudaMemcpyDeviceToHost, b->stream),
                   "copying results");
    if (!rc && resolved)
        rc = bcuda(b, cudaMemcpyAsync(resolved, d_res, (size_t)b->n * sizeof(int), cudaMemcpyDeviceToHost, b->stream),
                   "copying results");
    if (!rc) rc = bcuda(b, cudaStreamSynchronize(b->stream), "analysing the trace");
    cudaFree(d_out);
    cudaFree(d_res);
    return rc;
}

extern "C" int su2g_batch_autotune(su2g_batch* b, int32_t n_hb, int32_t n_or, int32_t* block_out)
{
    if (!b) return set_error(nullptr, SU2G_EINVAL, "su2g_batch_autotune: null batch");
    cudaSetDevice(b->device);
    // the trial sweeps must not move the chains: save and restore the pool and the counters
    const size_t pool_bytes = b->pool_bytes;
    void* save = nullptr;
    uint32_t ctr[2];
    int rc = bcuda(b, cudaMalloc(&save, pool_bytes), "allocating the autotune copy");
    if (!rc) rc = bcuda(b, cudaMemcpy(save, b->pool, pool_bytes, cudaMemcpyDeviceToDevice), "saving replicas");
    if (!rc) rc = bcuda(b, cudaMemcpy(ctr, b->d_ctr, sizeof(ctr), cudaMemcpyDeviceToHost), "saving counters");
    // the two forms (replayed graph of per-pass launches; one persistent launch) over CTA widths,
    // each timed on 4 sweeps with a plaquette after every sweep, after 2 warm-up sweeps
    const int candidates[][2] = {{SU2G_BATCH_GRAPH, 64},       {SU2G_BATCH_GRAPH, 128}, {SU2G_BATCH_GRAPH, 256},
                                 {SU2G_BATCH_PERSISTENT, 128}, {SU2G_BATCH_PERSISTENT, 256}};
    double best = 1e30;
    int best_block = b->block, best_mode = b->mode;
    for (const auto& c : candidates) {
        if (rc) break;
        if ((rc = build_maps(b, c[1]))) break;
        b->mode = c[0];
        double ms = 0;
        if ((rc = su2g_batch_run(b, 2, n_hb, n_or, 1, nullptr, &ms))) break;   // warm-up + graph build
        if ((rc = su2g_batch_run(b, 4, n_hb, n_or, 1, nullptr, &ms))) break;
        if (ms < best) {
            best = ms;
            best_block = c[1];
            best_mode = c[0];
        }
    }
    b->mode = best_mode;
    if (!rc) rc = build_maps(b, best_block);
    if (!rc) rc = bcuda(b, cudaMemcpy(b->pool, save, pool_bytes, cudaMemcpyDeviceToDevice), "restoring replicas");
    if (!rc) rc = bcuda(b, cudaMemcpy(b->d_ctr, ctr, sizeof(ctr), cudaMemcpyHostToDevice), "restoring counters");
    cudaFree(save);
    if (block_out) *block_out = b->block;
    return rc;
}

extern "C" int su2g_batch_download(su2g_batch* b, int32_t r, double* links)
{
    if (!b || !links || r < 0 || r >= b->n) return set_error(nullptr, SU2G_EINVAL, "su2g_batch_download: bad argument");
    cudaSetDevice(b->device);
    const Geom& g = b->reps[r].g;
    double* d = nullptr;
    int rc = bcuda(b, cudaMalloc(&d, (size_t)g.V * 16 * sizeof(double)), "allocating staging");
    if (rc) return rc;
    if (b->prec == SU2G_FP32) k_batch_aos<float><<<(g.V + 255) / 256, 256, 0, b->stream>>>(b->d_reps, r, (double2*)d, 1);
    else k_batch_aos<double><<<(g.V + 255) / 256, 256, 0, b->stream>>>(b->d_reps, r, (double2*)d, 1);
    rc = bcuda(b, cudaGetLastError(), "layout conversion");
    if (!rc) rc = bcuda(b, cudaMemcpyAsync(links, d, (size_t)g.V * 16 * sizeof(double), cudaMemcpyDeviceToHost, b->stream),
                        "downloading");
    if (!rc) rc = bcuda(b, cudaStreamSynchronize(b->stream), "downloading");
    cudaFree(d);
    return rc;
}

extern "C" int su2g_batch_upload(su2g_batch* b, int32_t r, const double* links)
{
    if (!b || !links || r < 0 || r >= b->n) return set_error(nullptr, SU2G_EINVAL, "su2g_batch_upload: bad argument");
    cudaSetDevice(b->device);
    const Geom& g = b->reps[r].g;
    double* d = nullptr;
    int rc = bcuda(b, cudaMalloc(&d, (size_t)g.V * 16 * sizeof(double)), "allocating staging");
    if (rc) return rc;
    rc = bcuda(b, cudaMemcpyAsync(d, links, (size_t)g.V * 16 * sizeof(double), cudaMemcpyHostToDevice, b->stream), "uploading");
    if (!rc) {
        if (b->prec == SU2G_FP32) k_batch_aos<float><<<(g.V + 255) / 256, 256, 0, b->stream>>>(b->d_reps, r, (double2*)d, 0);
        else k_batch_aos<double><<<(g.V + 255) / 256, 256, 0, b->stream>>>(b->d_reps, r, (double2*)d, 0);
        rc = bcuda(b, cudaGetLastError(), "layout conversion");
    }
    if (!rc) rc = bcuda(b, cudaStreamSynchronize(b->stream), "uploading");
    cudaFree(d);
    return rc;
}

extern "C" int su2g_batch_configure(su2g_batch* b, int32_t mode, int32_t block)
{
    if (!b) return set_error(nullptr, SU2G_EINVAL, "su2g_batch_configure: null batch");
    if (mode != SU2G_BATCH_GRAPH && mode != SU2G_BATCH_PERSISTENT)
        return berr(b, SU2G_EINVAL, "su2g_batch_configure: unknown mode %d", mode);
    if (block != 64 && block != 128 && block != 256)
        return berr(b, SU2G_EINVAL, "su2g_batch_configure: CTA width %d (64, 128 or 256)", block);
    if (mode == SU2G_BATCH_PERSISTENT && block == 64)
        return berr(b, SU2G_EINVAL, "su2g_batch_configure: the persistent form runs 128 or 256 threads a CTA");
    cudaSetDevice(b->device);
    b->mode = mode;
    return block == b->block ? SU2G_OK : build_maps(b, block);
}

extern "C" int su2g_batch_config(const su2g_batch* b, int32_t* mode, int32_t* block)
{
    if (!b) return set_error(nullptr, SU2G_EINVAL, "su2g_batch_config: null batch");
    if (mode) *mode = b->mode;
    if (block) *block = b->block;
    return SU2G_OK;
}

extern "C" int su2g_batch_selftest_grid_barrier(su2g_batch* b, int32_t missing, int64_t wait_cycles)
{
    if (!b) return set_error(nullptr, SU2G_EINVAL, "su2g_batch_selftest_grid_barrier: null batch");
    if (missing < 0 || wait_cycles <= 0 || wait_cycles > kGridWaitCycles)
        return berr(b, SU2G_EINVAL, "su2g_batch_selftest_grid_barrier: bad argument");
    cudaSetDevice(b->device);
    GridBarrier* gb = b->d_gb;
    unsigned* st = b->d_status;
    unsigned arrivals = (unsigned)(b->num_sms + missing);
    long long wc = (long long)wait_cycles;
    void* params[] = {&gb, &st, &arrivals, &wc};
    int rc = bcuda(b, cudaMemsetAsync(b->d_gb, 0, sizeof(GridBarrier), b->stream), "clearing the grid barrier");
    if (!rc)
        rc = bcuda(b, cudaLaunchCooperativeKernel((const void*)k_grid_selftest, dim3(b->num_sms), dim3(128), params, 0,
                                                  b->stream),
                   "launching the barrier self-test");
    if (!rc) rc = bcuda(b, cudaStreamSynchronize(b->stream), "barrier self-test");
    if (!rc) rc = check_status(b);
    return rc;
}
