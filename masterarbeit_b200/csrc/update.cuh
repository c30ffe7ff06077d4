// update.cuh -- per-link heatbath and overrelaxation (shared by the single-lattice and the
// batched sweeps).  Reference: staples (LGT_Code/modules/update/metro.c:34-63),
// generateSU2InHeatbath_Improved / localHeatbathUpdate (LGT_Code/modules/update/heatbath.c:76-149).
#pragma once
#include <cfloat>

#include "internal.cuh"
#include "philox.cuh"

namespace su2g {

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
// Square root of x >= 0: FP32 uses the hardware approximation (sqrt.approx.f32, relative error
// ~2^-23), FP64 the correctly rounded one.
__device__ __forceinline__ float kp_sqrt(float x)
{
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ double kp_sqrt(double x) { return sqrt(x); }
// 1/|A| and 1/(beta |A|) from |A|^2, from one reciprocal square root (FP32: the hardware
// approximation; FP64: rsqrt, within an ulp, in place of a square root and two divisions: the FP64
// heatbath pass 152.9 -> 152.1 us at 48^4).  |A| = 0 gives k = NaN (0 * inf), which fails the
// k > eps test like k = 0 does.
__device__ __forceinline__ void kp_norms(float n2, float beta, float& k, float& ik, float& ia)
{
    ik = rsqrtf(n2);
    k = n2 * ik;
    ia = __fdividef(ik, beta);
}
__device__ __forceinline__ void kp_norms(double n2, double beta, double& k, double& ik, double& ia)
{
    ik = rsqrt(n2);
    k = n2 * ik;
    ia = ik / beta;
}
// The FP32 logs of uniforms just below 1 may come out positive by their absolute error (~2^-21);
// delta is clamped at 0 so that sqrt(delta (2 - delta)) stays real.  FP64 logs are exact in sign.
__device__ __forceinline__ float kp_clamp(float d) { return fmaxf(d, 0.0f); }
__device__ __forceinline__ double kp_clamp(double d) { return d; }

// Staple sum A with U_mu(x) A = sum of the six plaquettes containing U_mu(x)  (metro.c:34-63):
//   A = sum_{nu != mu} U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag + U_nu(x-nu+mu)^dag U_mu(x-nu)^dag U_nu(x-nu)
// All 18 links are loaded before the first product, so that a thread keeps every load of its
// staple in flight at once (the pass is bound by memory latency x parallelism, not by ALU).  Each
// term's last product accumulates into A inside its multiply-adds (24 fewer additions a link: the
// FP64 heatbath pass 169 -> 155 us at 48^4 on B200).  With NLOW > 0, *low receives the partial sum
// of the first NLOW terms (nu = 0 .. NLOW-1 for NLOW <= MU), taken from the same accumulation, so A
// is the same either way.
template <typename R, int MU, int NLOW = 0, typename F = Field<R>>
__device__ __forceinline__ Q<R> staple_update(const F& U, const Geom& g, const Site& s, int par, Q<R>* low = nullptr)
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
        A = q_mul_nd_add(A, q_mul_nd(a[k], b[k]), c[k]);
        A = q_mul_dn_add(A, q_mul(e[k], d[k]), f[k]);
        if (k + 1 == NLOW) *low = A;
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
// `draw_base` (visit << kVisitShift) separates the draws of repeated visits in a random-order sweep.
constexpr int kVisitShift = 21;   // above every trial index (kMaxTrials = 2^20)

// `seed` is the 64-bit seed or its precomputed round keys (PhiloxKeys): the same draws either way.
template <typename R, typename Seed>
__device__ __forceinline__ bool heatbath_link(const Q<R>& A, R beta, const Seed& seed, uint32_t site, uint32_t sweep,
                                              uint32_t mu, uint32_t replica, uint32_t& trials, Q<R>& out,
                                              unsigned* status, uint32_t draw_base = 0u)
{
    R k, ik, ia;   // |A|, 1/|A|, 1/alpha with alpha = |A| beta (heatbath.c:142)
    kp_norms(q_norm2(A), beta, k, ik, ia);
    if (!(k > eps_r<R>())) {
        U4 w = link_random(seed, site, sweep, mu, draw_base | 1u, 1u, kStreamUpdate, replica);
        trials = 0;
        out = fallback_link<R>(u01(w.x, R(0)), u01(w.y, R(0)), u01(w.z, R(0)));
        return true;
    }
    R delta;
    uint32_t trial = 0;
    for (;;) {
        U4 w = link_random(seed, site, sweep, mu, draw_base | trial, 0u, kStreamUpdate, replica);
        ++trial;
        const R u0 = u01(w.x, R(0)), u1 = u01(w.y, R(0)), u2 = u01(w.z, R(0)), u3 = u01(w.w, R(0));
        const R c = kp_cos2pi(u2);
        // X1 = -ln(u0)/alpha, X2 = -ln(u1)/alpha, delta = X2 + X1 cos^2(2 pi u2)  (heatbath.c:86-90)
        delta = kp_clamp(-(kp_log(u1) + kp_log(u0) * (c * c)) * ia);
        if (u3 * u3 <= R(1) - R(0.5) * delta) break;   // heatbath.c:94
        if (trial >= kMaxTrials) {   // the link keeps its value and the host sees the status bit
            atomicOr(status, kStatusKpTrials);
            trials = 0;
            return false;
        }
    }
    trials = trial;
    // x0 = 1 - delta; (x1,x2,x3) = sqrt(1-x0^2) (sin th cos ph, sin th sin ph, cos th)  (heatbath.c:96-107)
    U4 w = link_random(seed, site, sweep, mu, draw_base, 1u, kStreamUpdate, replica);
    const R a0 = u01(w.x, R(0)), a1 = u01(w.y, R(0));
    const R cth = R(1) - R(2) * a1;
    const R sth = R(2) * kp_sqrt(a1 * (R(1) - a1));       // sin(acos(1 - 2 a1))
    R sph, cph;
    kp_sincos2pi(a0, &sph, &cph);
    const R len = kp_sqrt(delta * (R(2) - delta));          // sqrt(1 - (1-delta)^2)
    Q<R> X = q_make<R>(R(1) - delta, len * sth * cph, len * sth * sph, len * cth);
    // U = X V^dag, V = A/k  (heatbath.c:140-146)
    out = q_mul_nd(X, q_scale(A, ik));
    return true;
}

// The value a heatbath pass stores: X (A/|A|)^dag is unit to rounding (|X| = 1 by construction and
// A/|A| is normalised), and a heatbath link is drawn afresh, not compounded from its old value, so
// FP64 stores it as drawn (reprojecting cost 7 % of the FP64 pass: norm, reciprocal square root,
// scale); FP32 reprojects every store.
template <typename R>
__device__ __forceinline__ Q<R> hb_store(const Q<R>& q)
{
    return sizeof(R) == 8 ? q : q_project(q);
}

__device__ __forceinline__ float metro_exp(float x) { return __expf(x); }
__device__ __forceinline__ double metro_exp(double x) { return exp(x); }

// Metropolis hits on one link (localMetropolisUpdate, metro.c:78-109).  Hit i draws one Philox
// block: X = (1 - 2 r0, 1 - 2 r1, 1 - 2 r2) (proposeNewLink, metro.c:65-76), the proposal is
// exp(eps X) U with the O(X^2)-exact SU(2) exponential of expx (exp_fct.c:137-151), and it is
// accepted when r3 <= exp(beta (Re tr(U' A) - Re tr(U A)) / 2).  Returns the new link; `accepted`
// counts accepted hits.
template <typename R>
__device__ __forceinline__ Q<R> metropolis_link(const Q<R>& A, Q<R> U, R beta, R eps, int hits, uint64_t seed,
                                                uint32_t site, uint32_t sweep, uint32_t mu, uint32_t replica,
                                                uint32_t& accepted)
{
    R s_old = R(2) * q_mul(U, A).c0;   // Re tr(U A)
    for (int i = 0; i < hits; ++i) {
        U4 w = link_random(seed, site, sweep, mu, (uint32_t)i, 0u, kStreamMetro, replica);
        const R x1 = R(1) - R(2) * u01(w.x, R(0)), x2 = R(1) - R(2) * u01(w.y, R(0)), x3 = R(1) - R(2) * u01(w.z, R(0));
        R z = eps * eps * (x1 * x1 + x2 * x2 + x3 * x3) / R(4);
        const R e0 = R(1) - z;
        z = R(1) / (R(1) + z);
        const R ze = z * eps;
        const Q<R> P = q_mul(q_make<R>(e0 * z, ze * x1, ze * x2, ze * x3), U);
        const R s_new = R(2) * q_mul(P, A).c0;
        if (u01(w.w, R(0)) <= metro_exp(beta * (s_new - s_old) / R(2))) {
            U = P;
            s_old = s_new;
            ++accepted;
        }
    }
    return U;
}

// Times a site is drawn when V sites are drawn with replacement, as in gaugefieldUpdate's random
// sweep (update.c:126-136): Binomial(V, 1/V), by inverting its CDF on one 32-bit uniform
// (p0 = (1 - 1/V)^V, p_{k+1} = p_k (V - k) / ((k + 1)(V - 1))).  Computed in FP64 in both precision
// modes, so FP32 and FP64 chains make the same visit decisions.
__device__ __forceinline__ int visit_count(uint32_t w, double p0, double V)
{
    const double u = ((double)w + 0.5) * (1.0 / 4294967296.0);
    double p = p0, c = p0;
    int k = 0;
    while (u > c && k < 32) {
        p *= (V - k) / ((k + 1) * (V - 1.0));
        c += p;
        ++k;
    }
    return k;
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

}  // namespace su2g
