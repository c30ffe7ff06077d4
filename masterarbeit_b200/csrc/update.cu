// update.cu -- checkerboard heatbath and overrelaxation passes.
//
// Reference: gaugefieldUpdate (LGT_Code/modules/update/update.c:102-175) sweeps sites in
// lexicographic order and calls localHeatbathUpdate (LGT_Code/modules/update/heatbath.c:124-149)
// with the staple sum of staples() (LGT_Code/modules/update/metro.c:34-63) and the
// Kennedy-Pendleton sampler generateSU2InHeatbath_Improved (heatbath.c:76-121).  Here a sweep is
// eight passes (mu = 0..3, site parity 0 then 1); all links of one (mu, parity) are independent
// and are updated by one kernel launch, one thread per link.  Overrelaxation has no reference
// counterpart: U' = W^dag U^dag W^dag with W = A/|A|.
//
// Every updated link is reprojected before its store (in place of project_gfield_to_sun after
// the sweep, update.c:166), except an FP64 heatbath draw, which is unit to rounding (hb_store).
// Randoms come from Philox keyed by (seed, site, sweep, dir, draw,
// replica), so the result does not depend on grid shape or on which thread takes which link.
#include <cfloat>
#include <cmath>

#include "internal.cuh"
#include "philox.cuh"
#include "update.cuh"

using namespace su2g;

namespace {

// 32 resident warps per SM (at most 64 registers a thread): measured at 48^4 on B200 against 8, 16,
// 24 and 48, it is the fastest for both kinds and precisions (OR FP32 64 us against 79 us unbounded).
// Both kinds run them as eight 128-thread CTAs: finer CTAs shorten the pass's tail (OR 65.8 against
// 66.7 us, HB 86.7 against 88.1 us with four CTAs of 256).
template <int KIND>
constexpr int update_block() { return 128; }

// PLQ: the pass also sums the plaquettes of the planes (MU, nu < MU) of the configuration it leaves
// (one partial per warp into plaq_part).  Run in the parity-1 passes of MU = 1, 2, 3 of a
// sweep's last sub-sweep, these are all 6V plaquettes of the final field, each once: when U_MU(x)
// at the odd sites is updated, every other link of the plaquettes of the planes (MU, nu < MU) is
// final (directions nu < MU and U_MU at the even sites were updated by earlier passes), and each
// such plaquette holds exactly one odd-site U_MU link.  So with A_low the staple terms nu < MU,
// (1/2) Re tr of those plaquettes summed is (U'_MU(x) A_low(x)).c0, for the staple convention of
// staple_update (U A = the sum of the plaquettes through U); the separate plaquette kernel
// (plaquette.c:67-100) then need not run.
template <typename R, int MU, int KIND, bool PLQ = false>
__global__ void __launch_bounds__(update_block<KIND>(), 1024 / update_block<KIND>()) k_update(Field<R> U, Geom g, int par, R beta, PhiloxKeys seed, uint32_t sweep,
                                                   const uint32_t* __restrict__ sweep_base, uint32_t replica,
                                                   double* __restrict__ acc_sum, unsigned* __restrict__ status,
                                                   DD* __restrict__ plaq_part = nullptr)
{
    // one link per thread; CTAs are dispatched in index order, so the CTAs in flight cover a
    // contiguous window of the lattice and neighbours one t-slice away are still in L2
    double acc_thread = 0.0, plaq_thread = 0.0;
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h < g.Vh) {
        const Site s = site_of(g, par, h);
        Q<R> low;
        const Q<R> A = staple_update<R, MU, PLQ ? MU : 0>(U, g, s, par, PLQ ? &low : nullptr);
        if (KIND == SU2G_HEATBATH) {
            if (sweep_base) sweep += *sweep_base;
            Q<R> out;
            uint32_t trials = 0;
            if (heatbath_link<R>(A, beta, seed, (uint32_t)s.n, sweep, (uint32_t)MU, replica, trials, out, status))
                U.sth(MU, par, h, hb_store(out));
            if (acc_sum && trials) acc_thread = 1.0 / (double)trials;
        } else {
            U.sth(MU, par, h, q_project(overrelax_link<R>(A, U.ldh(MU, par, h))));
        }
        if constexpr (PLQ) {
            // the link as stored (or kept, if the trial bound was hit), read back through L2, which
            // sees this thread's own store; the update above is the same code as without PLQ, so
            // both kernels compile it alike and leave the same field
            FieldCG<R> Uc;
            for (int d = 0; d < 4; ++d) Uc.p[d] = U.p[d];
            Uc.Vh = U.Vh;
            plaq_thread = (double)q_mul(Uc.ldh(MU, par, h), low).c0;
        }
    }
    if (KIND == SU2G_HEATBATH && acc_sum) {
        DD v = {acc_thread, 0.0};
        v = dd_block_sum<update_block<KIND>()>(v);
        if (threadIdx.x == 0) atomicAdd(acc_sum, v.s + v.e);
    }
    if (PLQ) {
        // one partial per warp (plain FP64 over its 32 terms), no CTA barrier: a barrier would
        // hold the CTA's warps until its slowest Kennedy-Pendleton lane is done
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) plaq_thread += __shfl_xor_sync(0xffffffffu, plaq_thread, o);
        if ((threadIdx.x & 31) == 0)
            plaq_part[blockIdx.x * (update_block<KIND>() / 32) + (threadIdx.x >> 5)] = DD{plaq_thread, 0.0};
    }
}

// The reference's other update algorithm and sweep order (gaugefieldUpdate's utype 0 and
// stype 1, update.c:121-163): one link per thread as above, with
//  - KIND = Metropolis: `hits` Metropolis hits per visit (metropolis_link);
//  - ORDER = 1: a Binomial(V, 1/V) number of visits per site and sweep (visit_count, the same
//    count for the site's four links), heatbath or Metropolis once per visit.
// The acceptance sum counts 1/trials per heatbath visit and accepted/hits per Metropolis visit.
struct VisitArgs {
    double beta, eps;
    int hits;
    double p0;   // (1 - 1/V)^V
    uint64_t seed;
    uint32_t sweep, replica;
};

// Two resident CTAs per SM: the visit loop and the Metropolis state spill at 64 registers.
template <typename R, int MU, int KIND, int ORDER>
__global__ void __launch_bounds__(kBlock, 2) k_visit(Field<R> U, Geom g, int par, VisitArgs a,
                                                  double* __restrict__ acc_sum, unsigned* __restrict__ status)
{
    double acc_thread = 0.0;
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h < g.Vh) {
        const Site s = site_of(g, par, h);
        int visits = 1;
        if (ORDER == 1)
            visits = visit_count(link_random(a.seed, (uint32_t)s.n, a.sweep, 0u, 0u, 0u, kStreamVisit, a.replica).x,
                                 a.p0, (double)g.V);
        if (visits > 0) {
            const Q<R> A = staple_update<R, MU>(U, g, s, par);
            if (KIND == SU2G_HEATBATH) {
                Q<R> cur, out;
                bool changed = false;
                for (int v = 0; v < visits; ++v) {
                    uint32_t trials = 0;
                    if (heatbath_link<R>(A, (R)a.beta, a.seed, (uint32_t)s.n, a.sweep, (uint32_t)MU, a.replica, trials,
                                         out, status, (uint32_t)v << kVisitShift)) {
                        cur = out;
                        changed = true;
                    }
                    if (trials) acc_thread += 1.0 / (double)trials;
                }
                if (changed) U.sth(MU, par, h, hb_store(cur));
            } else {
                uint32_t accepted = 0;
                const Q<R> u = metropolis_link<R>(A, U.ldh(MU, par, h), (R)a.beta, (R)a.eps, visits * a.hits, a.seed,
                                                  (uint32_t)s.n, a.sweep, (uint32_t)MU, a.replica, accepted);
                U.sth(MU, par, h, q_project(u));
                acc_thread = (double)accepted / (double)a.hits;
            }
        }
    }
    if (acc_sum) {
        DD v = {acc_thread, 0.0};
        v = dd_block_sum<kBlock>(v);
        if (threadIdx.x == 0) atomicAdd(acc_sum, v.s + v.e);
    }
}

template <typename R, int KIND, int ORDER>
void launch_visit_t(su2g_lattice* h, int mu, int par, const VisitArgs& a, double* acc_sum, int grid)
{
    Field<R> U = make_field<R>(h->dirp, h->g.Vh);
    switch (mu) {
        case 0: k_visit<R, 0, KIND, ORDER><<<grid, kBlock, 0, h->stream>>>(U, h->g, par, a, acc_sum, h->d_status); break;
        case 1: k_visit<R, 1, KIND, ORDER><<<grid, kBlock, 0, h->stream>>>(U, h->g, par, a, acc_sum, h->d_status); break;
        case 2: k_visit<R, 2, KIND, ORDER><<<grid, kBlock, 0, h->stream>>>(U, h->g, par, a, acc_sum, h->d_status); break;
        default: k_visit<R, 3, KIND, ORDER><<<grid, kBlock, 0, h->stream>>>(U, h->g, par, a, acc_sum, h->d_status); break;
    }
}

template <typename R>
void launch_visit_r(su2g_lattice* h, int kind, int order, int mu, int par, const VisitArgs& a, double* acc_sum, int grid)
{
    if (kind == SU2G_HEATBATH) launch_visit_t<R, SU2G_HEATBATH, 1>(h, mu, par, a, acc_sum, grid);   // order 1 only
    else if (order) launch_visit_t<R, SU2G_METROPOLIS, 1>(h, mu, par, a, acc_sum, grid);
    else launch_visit_t<R, SU2G_METROPOLIS, 0>(h, mu, par, a, acc_sum, grid);
}

template <typename R, int KIND>
void launch_update_t(su2g_lattice* h, int mu, int par, uint32_t sweep, const uint32_t* base, double* acc_sum, int grid,
                     DD* plaq_part)
{
    Field<R> U = make_field<R>(h->dirp, h->g.Vh);
    const R beta = (R)h->beta;
    const int nt = update_block<KIND>();
    cudaStream_t st = h->stream;
    const PhiloxKeys keys = philox_keys(h->seed);
    if (plaq_part) {   // parity-1 passes of MU >= 1 only
        switch (mu) {
            case 1: k_update<R, 1, KIND, true><<<grid, nt, 0, st>>>(U, h->g, par, beta, keys, sweep, base, h->replica, acc_sum, h->d_status, plaq_part); break;
            case 2: k_update<R, 2, KIND, true><<<grid, nt, 0, st>>>(U, h->g, par, beta, keys, sweep, base, h->replica, acc_sum, h->d_status, plaq_part); break;
            default: k_update<R, 3, KIND, true><<<grid, nt, 0, st>>>(U, h->g, par, beta, keys, sweep, base, h->replica, acc_sum, h->d_status, plaq_part); break;
        }
        return;
    }
    switch (mu) {
        case 0: k_update<R, 0, KIND><<<grid, nt, 0, st>>>(U, h->g, par, beta, keys, sweep, base, h->replica, acc_sum, h->d_status); break;
        case 1: k_update<R, 1, KIND><<<grid, nt, 0, st>>>(U, h->g, par, beta, keys, sweep, base, h->replica, acc_sum, h->d_status); break;
        case 2: k_update<R, 2, KIND><<<grid, nt, 0, st>>>(U, h->g, par, beta, keys, sweep, base, h->replica, acc_sum, h->d_status); break;
        default: k_update<R, 3, KIND><<<grid, nt, 0, st>>>(U, h->g, par, beta, keys, sweep, base, h->replica, acc_sum, h->d_status); break;
    }
}

}  // namespace

int su2g::update_grid(const su2g_lattice* h)
{
    return (int)((h->g.Vh + update_block<SU2G_HEATBATH>() - 1) / update_block<SU2G_HEATBATH>());
}

int su2g::update_plaq_parts(const su2g_lattice* h)
{
    return update_grid(h) * (update_block<SU2G_HEATBATH>() / 32);
}

int su2g::launch_update(su2g_lattice* h, int kind, int mu, int par, uint32_t sweep, double* acc_sum,
                        const uint32_t* base, DD* plaq_part)
{
    static_assert(update_block<SU2G_HEATBATH>() == update_block<SU2G_OVERRELAX>(), "one grid for both kinds");
    const int cls = kind == SU2G_HEATBATH ? SU2G_K_HEATBATH : SU2G_K_OVERRELAX;
    const int grid = update_grid(h);
    if (plaq_part && (mu < 1 || par != 1))
        return set_error(h, SU2G_EINVAL, "fused plaquette: only the parity-1 passes of mu >= 1 sum plaquettes");
    launch_begin(h, cls);
    if (h->prec == SU2G_FP32) {
        if (kind == SU2G_HEATBATH) launch_update_t<float, SU2G_HEATBATH>(h, mu, par, sweep, base, acc_sum, grid, plaq_part);
        else launch_update_t<float, SU2G_OVERRELAX>(h, mu, par, sweep, base, acc_sum, grid, plaq_part);
    } else {
        if (kind == SU2G_HEATBATH) launch_update_t<double, SU2G_HEATBATH>(h, mu, par, sweep, base, acc_sum, grid, plaq_part);
        else launch_update_t<double, SU2G_OVERRELAX>(h, mu, par, sweep, base, acc_sum, grid, plaq_part);
    }
    return launch_end(h, cls, kind == SU2G_HEATBATH ? "heatbath pass" : "overrelaxation pass");
}

namespace {

// ----------------------------------------------------------- sampler test ---

// x0 histogram of the Kennedy-Pendleton sampler at fixed alpha (LGT_Code/main_test/test.c:115-166),
// drawn by the production sampler heatbath_link<R> of the sweeps in the handle's precision: with the
// staple A = 1 and beta = alpha it samples at alpha = |A| beta and returns X itself (A/|A| = 1), so
// the FP32 histogram exercises the FP32 sampler's fast logarithm, sine/cosine, approximate square
// roots and delta clamp.  Draw i uses the Philox stream of site i (sweep i >> 32, direction 0).
template <typename R>
__global__ void __launch_bounds__(kBlock) k_kp_histogram(double alpha, uint64_t seed, long long n, int nbins,
                                                         unsigned long long* __restrict__ counts,
                                                         unsigned* __restrict__ status)
{
    extern __shared__ unsigned int sh_hist[];
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) sh_hist[b] = 0;
    __syncthreads();
    const Q<R> A = q_one<R>();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        Q<R> X;
        uint32_t trials = 0;
        if (!heatbath_link<R>(A, (R)alpha, seed, (uint32_t)i, (uint32_t)(i >> 32), 0u, 0u, trials, X, status))
            continue;   // trial bound hit: the status word tells the host
        int b = (int)(((double)X.c0 + 1.0) * 0.5 * nbins);   // bin of x0 on [-1, 1]
        b = b < 0 ? 0 : (b >= nbins ? nbins - 1 : b);
        atomicAdd(&sh_hist[b], 1u);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nbins; b += blockDim.x)
        if (sh_hist[b]) atomicAdd(&counts[b], (unsigned long long)sh_hist[b]);
}

}  // namespace

extern "C" int su2g_update_pass(su2g_lattice* h, int32_t kind, int32_t mu, int32_t parity, uint32_t sweep)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_update_pass: null handle");
    if ((kind != SU2G_HEATBATH && kind != SU2G_OVERRELAX) || mu < 0 || mu > 3 || (parity != 0 && parity != 1))
        return set_error(h, SU2G_EINVAL, "su2g_update_pass: bad kind/mu/parity (%d, %d, %d)", kind, mu, parity);
    cudaSetDevice(h->device);
    return launch_update(h, kind, mu, parity, sweep, nullptr);
}

int su2g::sweep_enqueue(su2g_lattice* h, int n_sweeps, int n_hb, int n_or, uint32_t sweep0, const uint32_t* base,
                        double* acc_dev, int plaq_off)
{
    const int parts = update_plaq_parts(h);   // per fused pass
    const int subs = n_sweeps * (n_hb + n_or);
    int rc = SU2G_OK;
    if (plaq_off >= 0 && subs > 0 && (rc = ensure_partial_entries(h, 3 * (size_t)parts))) return rc;
    int sub = 0;
    for (int s = 0; s < n_sweeps; ++s)
        for (int i = 0; i < n_hb + n_or; ++i) {
            const bool hb = i < n_hb;
            const bool last = ++sub == subs && plaq_off >= 0;
            for (int mu = 0; mu < 4; ++mu)
                for (int par = 0; par < 2; ++par) {
                    DD* part = last && mu >= 1 && par == 1 ? h->partials + (size_t)(mu - 1) * parts : nullptr;
                    rc = hb ? launch_update(h, SU2G_HEATBATH, mu, par, sweep0 + (uint32_t)(s * n_hb + i), acc_dev, base, part)
                            : launch_update(h, SU2G_OVERRELAX, mu, par, 0u, nullptr, nullptr, part);
                    if (rc) return rc;
                }
        }
    if (plaq_off < 0) return SU2G_OK;
    if (subs == 0) return plaquette_enqueue(h, plaq_off);
    // the partials of the passes (1, 1), (2, 1), (3, 1): 6V plaquettes, (1/2) Re tr each
    return finalize(h, 3 * parts, 1, 1.0 / (6.0 * (double)h->g.V), plaq_off);
}

namespace {

int sweep_call(su2g_lattice* h, int32_t n_sweeps, int32_t n_hb, int32_t n_or, double* plaq_out, double* acc_out,
               const char* who)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "%s: null handle", who);
    if (n_sweeps < 0 || n_hb < 0 || n_or < 0) return set_error(h, SU2G_EINVAL, "%s: negative count", who);
    cudaSetDevice(h->device);
    double* acc_dev = nullptr;
    const int slot_acc = 0, slot_plaq = 1;
    int rc = SU2G_OK;
    if (acc_out) {
        acc_dev = h->d_out + slot_acc;
        if ((rc = check_cuda(h, cudaMemsetAsync(acc_dev, 0, sizeof(double), h->stream), "clearing acceptance")))
            return rc;
    }
    rc = sweep_enqueue(h, n_sweeps, n_hb, n_or, h->hb_sweeps, nullptr, acc_dev, plaq_out ? slot_plaq : -1);
    if (rc) return rc;
    h->hb_sweeps += (uint32_t)(n_sweeps * n_hb);
    if (acc_out || plaq_out) {
        if ((rc = fetch_results(h, slot_acc, 2))) return rc;
        const double nupd = (double)n_sweeps * n_hb * 4.0 * (double)h->g.V;
        if (acc_out) *acc_out = nupd > 0 ? h->h_out[slot_acc] / nupd : 0.0;
        if (plaq_out) *plaq_out = h->h_out[slot_plaq];
    }
    return SU2G_OK;
}

}  // namespace

extern "C" int su2g_sweep(su2g_lattice* h, int32_t n_sweeps, int32_t n_hb, int32_t n_or, double* acc_out)
{
    return sweep_call(h, n_sweeps, n_hb, n_or, nullptr, acc_out, "su2g_sweep");
}

extern "C" int su2g_sweep_plaquette(su2g_lattice* h, int32_t n_sweeps, int32_t n_hb, int32_t n_or, double* plaq,
                                    double* acc_out)
{
    if (h && !plaq) return set_error(h, SU2G_EINVAL, "su2g_sweep_plaquette: null plaquette output");
    return sweep_call(h, n_sweeps, n_hb, n_or, plaq, acc_out, "su2g_sweep_plaquette");
}

extern "C" int su2g_gauge_update(su2g_lattice* h, int32_t nup, int32_t utype, int32_t stype, double eps, int32_t hits,
                                 double* acc_out)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_gauge_update: null handle");
    // the reference's checks and messages (update.c:109-113)
    if (utype != 0 && utype != 1)
        return set_error(h, SU2G_EINVAL, "su2g_gauge_update: unknown update type %d (Metropolis 0 and heatbath 1)", utype);
    if (stype != 0 && stype != 1)
        return set_error(h, SU2G_EINVAL, "su2g_gauge_update: unknown sweep type %d (sequential 0 and random 1)", stype);
    if (nup < 0) return set_error(h, SU2G_EINVAL, "su2g_gauge_update: negative sweep count");
    if (utype == 0 && (hits < 1 || !std::isfinite(eps)))
        return set_error(h, SU2G_EINVAL, "su2g_gauge_update: Metropolis needs hits >= 1 and a finite step size");
    if (utype == 1 && stype == 0) return su2g_sweep(h, nup, 1, 0, acc_out);
    cudaSetDevice(h->device);
    double* acc_dev = nullptr;
    int rc = SU2G_OK;
    if (acc_out) {
        acc_dev = h->d_out;
        if ((rc = check_cuda(h, cudaMemsetAsync(acc_dev, 0, sizeof(double), h->stream), "clearing acceptance")))
            return rc;
    }
    VisitArgs a;
    a.beta = h->beta;
    a.eps = eps;
    a.hits = utype == 0 ? hits : 1;
    a.p0 = std::exp((double)h->g.V * std::log1p(-1.0 / (double)h->g.V));
    a.seed = h->seed;
    a.replica = h->replica;
    const int kind = utype == 0 ? SU2G_METROPOLIS : SU2G_HEATBATH;
    const int cls = kind == SU2G_HEATBATH ? SU2G_K_HEATBATH : SU2G_K_METROPOLIS;
    const int grid = (int)((h->g.Vh + kBlock - 1) / kBlock);
    for (int s = 0; s < nup; ++s) {
        a.sweep = h->hb_sweeps;
        for (int mu = 0; mu < 4; ++mu)
            for (int par = 0; par < 2; ++par) {
                launch_begin(h, cls);
                if (h->prec == SU2G_FP32) launch_visit_r<float>(h, kind, stype, mu, par, a, acc_dev, grid);
                else launch_visit_r<double>(h, kind, stype, mu, par, a, acc_dev, grid);
                if ((rc = launch_end(h, cls, "update pass"))) return rc;
            }
        h->hb_sweeps++;
    }
    if (acc_out) {
        if ((rc = fetch_results(h, 0, 1))) return rc;
        const double nvis = (double)nup * 4.0 * (double)h->g.V;
        *acc_out = nvis > 0 ? h->h_out[0] / nvis : 0.0;
    }
    return SU2G_OK;
}

extern "C" int su2g_kp_histogram(su2g_lattice* h, double alpha, uint64_t seed, int64_t n, int32_t nbins,
                                 int64_t* counts)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_kp_histogram: null handle");
    if (!counts || nbins <= 0 || nbins > 8192 || n < 0 || !(alpha > 0.0))
        return set_error(h, SU2G_EINVAL, "su2g_kp_histogram: bad argument");
    cudaSetDevice(h->device);
    unsigned long long* d_counts = nullptr;
    int rc = check_cuda(h, cudaMallocAsync(&d_counts, nbins * sizeof(unsigned long long), h->stream),
                        "allocating histogram");
    if (rc) return rc;
    rc = check_cuda(h, cudaMemsetAsync(d_counts, 0, nbins * sizeof(unsigned long long), h->stream), "clearing histogram");
    if (!rc) {
        const int grid = grid_for(h, n, 8);
        launch_begin(h, SU2G_K_OTHER);
        if (h->prec == SU2G_FP32)
            k_kp_histogram<float><<<grid, kBlock, nbins * sizeof(unsigned int), h->stream>>>(alpha, seed, n, nbins,
                                                                                            d_counts, h->d_status);
        else
            k_kp_histogram<double><<<grid, kBlock, nbins * sizeof(unsigned int), h->stream>>>(alpha, seed, n, nbins,
                                                                                             d_counts, h->d_status);
        rc = launch_end(h, SU2G_K_OTHER, "sampler histogram");
    }
    if (!rc)
        rc = check_cuda(h, cudaMemcpyAsync(counts, d_counts, nbins * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                           h->stream),
                        "copying histogram");
    cudaFreeAsync(d_counts, h->stream);
    if (!rc) rc = fetch_results(h, 0, 0);
    return rc;
}
