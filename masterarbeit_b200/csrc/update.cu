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
// the sweep, update.c:166).  Randoms come from Philox keyed by (seed, site, sweep, dir, draw,
// replica), so the result does not depend on grid shape or on which thread takes which link.
#include <cfloat>

#include "internal.cuh"
#include "philox.cuh"

using namespace su2g;

namespace {

template <typename R>
__device__ __forceinline__ R eps_r();
template <>
__device__ __forceinline__ float eps_r<float>() { return FLT_EPSILON; }
template <>
__device__ __forceinline__ double eps_r<double>() { return DBL_EPSILON; }

// Sampler math.  FP64 uses the accurate library functions.  FP32 uses the hardware approximations
// (__logf: absolute error ~2^-21 on (0,1]; __sincosf on [-pi, pi]: ~2^-21), which are below the
// 2^-23 resolution of the FP32 uniforms' effect on delta and the angles.
__device__ __forceinline__ float kp_log(float x) { return __logf(x); }
__device__ __forceinline__ double kp_log(double x) { return log(x); }
// cos and sin of 2 pi u for u in (0,1)
__device__ __forceinline__ void kp_sincos2pi(float u, float* s, float* c)
{
    float ss, cc;
    __sincosf(6.28318530717958647692f * (u - 0.5f), &ss, &cc);   // 2 pi (u - 1/2) in [-pi, pi]
    *s = -ss;
    *c = -cc;
}
__device__ __forceinline__ void kp_sincos2pi(double u, double* s, double* c) { sincospi(2.0 * u, s, c); }
__device__ __forceinline__ float kp_cos2pi(float u) { return -__cosf(6.28318530717958647692f * (u - 0.5f)); }
__device__ __forceinline__ double kp_cos2pi(double u) { return cospi(2.0 * u); }

// Staple sum A with U_mu(x) A = sum of the six plaquettes containing U_mu(x)  (metro.c:34-63):
//   A = sum_{nu != mu} U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag + U_nu(x-nu+mu)^dag U_mu(x-nu)^dag U_nu(x-nu)
// All 18 links are loaded before the first product, so that a thread keeps every load of its
// staple in flight at once (the pass is bound by memory latency x parallelism, not by ALU).
template <typename R, int MU>
__device__ __forceinline__ Q<R> staple_update(const Field<R>& U, const Geom& g, const Site& s, int par)
{
    const int q = par ^ 1;
    const int dmu = up_off<MU>(g, s);
    const int xmu = s.n + dmu;
    Q<R> a[3], b[3], c[3], d[3], e[3], f[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int nu = k < MU ? k : k + 1;
        const int xnu = s.n + up_off_rt(g, s.c, nu);
        const int xmn = s.n + dn_off_rt(g, s.c, nu);
        a[k] = U.ld(nu, q, xmu);           // U_nu(x+mu)
        b[k] = U.ld(MU, q, xnu);           // U_mu(x+nu)
        c[k] = U.ld(nu, par, s.n);         // U_nu(x)
        d[k] = U.ld(nu, par, xmn + dmu);   // U_nu(x-nu+mu)
        e[k] = U.ld(MU, q, xmn);           // U_mu(x-nu)
        f[k] = U.ld(nu, q, xmn);           // U_nu(x-nu)
    }
    Q<R> A = q_zero<R>();
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        A = q_add(A, q_mul_nd(q_mul_nd(a[k], b[k]), c[k]));
        A = q_add(A, q_mul_dn(q_mul(e[k], d[k]), f[k]));
    }
    return A;
}

// su2RandomMatrix (LGT_Code/modules/random/random_su3.c:141-155) for the zero-staple fallback.
template <typename R>
__device__ __forceinline__ Q<R> fallback_link(R r0, R r1, R r2)
{
    Q<R> u;
    u.c0 = R(1) - R(2) * r0;
    u.c1 = R(1) - R(2) * r1;
    R zw = sqrt_r(R(1) - u.c1 * u.c1);
    R s, c;
    sincospi(R(2) * r2, &s, &c);
    u.c2 = zw * c;
    u.c3 = zw * s;
    zw = sqrt_r(R(1) - u.c0 * u.c0);
    u.c1 *= zw;
    u.c2 *= zw;
    u.c3 *= zw;
    return u;
}

// Kennedy-Pendleton heatbath of one link given its staple sum (heatbath.c:76-149).
// Writes the new link to `out` and the number of trials to `trials` (0 for the zero-staple
// fallback; the reference counts 1/trials into its acceptance, heatbath.c:137, :148).  Returns
// false only if the trial bound is hit (the link then keeps its old value).
template <typename R>
__device__ __forceinline__ bool heatbath_link(const Q<R>& A, R beta, uint64_t seed, uint32_t site, uint32_t sweep,
                                              uint32_t mu, uint32_t replica, uint32_t& trials, Q<R>& out,
                                              unsigned* status)
{
    const R k = sqrt_r(q_norm2(A));
    if (!(k > eps_r<R>())) {
        U4 w = link_random(seed, site, sweep, mu, 1u, 1u, kStreamUpdate, replica);
        trials = 0;
        out = fallback_link<R>(u01(w.x, R(0)), u01(w.y, R(0)), u01(w.z, R(0)));
        return true;
    }
    const R ik = R(1) / k;
    const R ia = R(1) / (k * beta);          // 1/alpha, alpha = k*beta (heatbath.c:142)
    R delta;
    uint32_t trial = 0;
    for (;;) {
        U4 w = link_random(seed, site, sweep, mu, trial, 0u, kStreamUpdate, replica);
        ++trial;
        const R u0 = u01(w.x, R(0)), u1 = u01(w.y, R(0)), u2 = u01(w.z, R(0)), u3 = u01(w.w, R(0));
        const R c = kp_cos2pi(u2);
        // X1 = -ln(u0)/alpha, X2 = -ln(u1)/alpha, delta = X2 + X1 cos^2(2 pi u2)  (heatbath.c:86-90)
        delta = -(kp_log(u1) + kp_log(u0) * (c * c)) * ia;
        if (u3 * u3 <= R(1) - R(0.5) * delta) break;   // heatbath.c:94
        if (trial >= kMaxTrials) {   // the link keeps its value and the host sees the status bit
            atomicOr(status, kStatusKpTrials);
            trials = 0;
            return false;
        }
    }
    trials = trial;
    // x0 = 1 - delta; (x1,x2,x3) = sqrt(1-x0^2) (sin th cos ph, sin th sin ph, cos th)  (heatbath.c:96-107)
    U4 w = link_random(seed, site, sweep, mu, 0u, 1u, kStreamUpdate, replica);
    const R a0 = u01(w.x, R(0)), a1 = u01(w.y, R(0));
    const R cth = R(1) - R(2) * a1;
    const R sth = R(2) * sqrt_r(a1 * (R(1) - a1));       // sin(acos(1 - 2 a1))
    R sph, cph;
    kp_sincos2pi(a0, &sph, &cph);
    const R len = sqrt_r(delta * (R(2) - delta));          // sqrt(1 - (1-delta)^2)
    Q<R> X = q_make<R>(R(1) - delta, len * sth * cph, len * sth * sph, len * cth);
    // U = X V^dag, V = A/k  (heatbath.c:140-146)
    out = q_mul_nd(X, q_scale(A, ik));
    return true;
}

// Overrelaxation U' = (W U W)^dag with W = A/|A|: keeps Re tr(U A), and applied twice is the identity.
template <typename R>
__device__ __forceinline__ Q<R> overrelax_link(const Q<R>& A, const Q<R>& U)
{
    const R k2 = q_norm2(A);
    if (!(k2 > eps_r<R>() * eps_r<R>())) return U;
    const Q<R> W = q_scale(A, rsqrt_r(k2));
    return q_dag(q_mul(q_mul(W, U), W));
}

template <typename R, int MU, int KIND>
__global__ void __launch_bounds__(kBlock) k_update(Field<R> U, Geom g, int par, R beta, uint64_t seed, uint32_t sweep,
                                                   uint32_t replica, double* __restrict__ acc_sum,
                                                   unsigned* __restrict__ status)
{
    // one link per thread; CTAs are dispatched in index order, so the CTAs in flight cover a
    // contiguous window of the lattice and neighbours one t-slice away are still in L2
    double acc_thread = 0.0;
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h < g.Vh) {
        const Site s = site_of(g, par, h);
        const Q<R> A = staple_update<R, MU>(U, g, s, par);
        if (KIND == SU2G_HEATBATH) {
            Q<R> out;
            uint32_t trials = 0;
            if (heatbath_link<R>(A, beta, seed, (uint32_t)s.n, sweep, (uint32_t)MU, replica, trials, out, status))
                U.sth(MU, par, h, q_project(out));
            if (acc_sum && trials) acc_thread = 1.0 / (double)trials;
        } else {
            U.sth(MU, par, h, q_project(overrelax_link<R>(A, U.ldh(MU, par, h))));
        }
    }
    if (KIND == SU2G_HEATBATH && acc_sum) {
        DD v = {acc_thread, 0.0};
        v = dd_block_sum<kBlock>(v);
        if (threadIdx.x == 0) atomicAdd(acc_sum, v.s + v.e);
    }
}

template <typename R, int KIND>
void launch_update_t(su2g_lattice* h, int mu, int par, uint32_t sweep, double* acc_sum, int grid)
{
    Field<R> U = make_field<R>(h->dirp, h->g.Vh);
    const R beta = (R)h->beta;
    switch (mu) {
        case 0: k_update<R, 0, KIND><<<grid, kBlock, 0, h->stream>>>(U, h->g, par, beta, h->seed, sweep, h->replica, acc_sum, h->d_status); break;
        case 1: k_update<R, 1, KIND><<<grid, kBlock, 0, h->stream>>>(U, h->g, par, beta, h->seed, sweep, h->replica, acc_sum, h->d_status); break;
        case 2: k_update<R, 2, KIND><<<grid, kBlock, 0, h->stream>>>(U, h->g, par, beta, h->seed, sweep, h->replica, acc_sum, h->d_status); break;
        default: k_update<R, 3, KIND><<<grid, kBlock, 0, h->stream>>>(U, h->g, par, beta, h->seed, sweep, h->replica, acc_sum, h->d_status); break;
    }
}

int launch_update(su2g_lattice* h, int kind, int mu, int par, uint32_t sweep, double* acc_sum)
{
    const int cls = kind == SU2G_HEATBATH ? SU2G_K_HEATBATH : SU2G_K_OVERRELAX;
    const int grid = (int)((h->g.Vh + kBlock - 1) / kBlock);
    launch_begin(h, cls);
    if (h->prec == SU2G_FP32) {
        if (kind == SU2G_HEATBATH) launch_update_t<float, SU2G_HEATBATH>(h, mu, par, sweep, acc_sum, grid);
        else launch_update_t<float, SU2G_OVERRELAX>(h, mu, par, sweep, acc_sum, grid);
    } else {
        if (kind == SU2G_HEATBATH) launch_update_t<double, SU2G_HEATBATH>(h, mu, par, sweep, acc_sum, grid);
        else launch_update_t<double, SU2G_OVERRELAX>(h, mu, par, sweep, acc_sum, grid);
    }
    return launch_end(h, cls, kind == SU2G_HEATBATH ? "heatbath pass" : "overrelaxation pass");
}

// ----------------------------------------------------------- sampler test ---

// x0 histogram of the Kennedy-Pendleton sampler at fixed alpha (LGT_Code/main_test/test.c:115-166).
__global__ void __launch_bounds__(kBlock) k_kp_histogram(double alpha, uint64_t seed, long long n, int nbins,
                                                         unsigned long long* __restrict__ counts,
                                                         unsigned* __restrict__ status)
{
    extern __shared__ unsigned int sh_hist[];
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) sh_hist[b] = 0;
    __syncthreads();
    const double ia = 1.0 / alpha;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double delta = 0.0;
        uint32_t trial = 0;
        bool ok = false;
        while (trial < kMaxTrials) {
            U4 w = link_random(seed, (uint32_t)i, (uint32_t)(i >> 32), 0u, trial, 0u, kStreamUpdate, 0u);
            ++trial;
            const double c = cospi(2.0 * u01(w.z, 0.0));
            delta = -(log(u01(w.y, 0.0)) + log(u01(w.x, 0.0)) * (c * c)) * ia;
            const double u3 = u01(w.w, 0.0);
            if (u3 * u3 <= 1.0 - 0.5 * delta) {
                ok = true;
                break;
            }
        }
        if (!ok) {
            atomicOr(status, kStatusKpTrials);
            continue;
        }
        int b = (int)((2.0 - delta) * 0.5 * nbins);   // bin of x0 = 1 - delta on [-1, 1]
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

extern "C" int su2g_sweep(su2g_lattice* h, int32_t n_sweeps, int32_t n_hb, int32_t n_or, double* acc_out)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_sweep: null handle");
    if (n_sweeps < 0 || n_hb < 0 || n_or < 0) return set_error(h, SU2G_EINVAL, "su2g_sweep: negative count");
    cudaSetDevice(h->device);
    double* acc_dev = nullptr;
    const int slot = 0;
    int rc = SU2G_OK;
    if (acc_out) {
        acc_dev = h->d_out + slot;
        if ((rc = check_cuda(h, cudaMemsetAsync(acc_dev, 0, sizeof(double), h->stream), "clearing acceptance")))
            return rc;
    }
    for (int s = 0; s < n_sweeps; ++s) {
        for (int i = 0; i < n_hb; ++i) {
            for (int mu = 0; mu < 4; ++mu)
                for (int par = 0; par < 2; ++par)
                    if ((rc = launch_update(h, SU2G_HEATBATH, mu, par, h->hb_sweeps, acc_dev))) return rc;
            h->hb_sweeps++;
        }
        for (int i = 0; i < n_or; ++i)
            for (int mu = 0; mu < 4; ++mu)
                for (int par = 0; par < 2; ++par)
                    if ((rc = launch_update(h, SU2G_OVERRELAX, mu, par, 0u, nullptr))) return rc;
    }
    if (acc_out) {
        if ((rc = fetch_results(h, slot, 1))) return rc;
        const double nupd = (double)n_sweeps * n_hb * 4.0 * (double)h->g.V;
        *acc_out = nupd > 0 ? h->h_out[slot] / nupd : 0.0;
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
        k_kp_histogram<<<grid, kBlock, nbins * sizeof(unsigned int), h->stream>>>(alpha, seed, n, nbins, d_counts,
                                                                                 h->d_status);
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
