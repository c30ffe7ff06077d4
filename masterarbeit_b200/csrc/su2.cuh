// su2.cuh -- quaternion SU(2) algebra, lattice geometry and link-field access for sm_100a.
//
// Quaternion convention follows the reference (LGT_Code/include/gauge.h:21-24, :190-198):
// U = c0*1 + i(c1 s1 + c2 s2 + c3 s3); product gauge.h:83-91, product with dagger :94-102,
// Re tr U = 2 c0 (:177-178).
//
// Device link layout (structure of arrays, checkerboarded): every direction mu has its own
// array of 2*Vh links, link(mu, parity, h) at element (parity*Vh + h) of it, h = n >> 1,
// where n = ((t*L1 + x)*L2 + y)*L3 + z is the reference's lexicographic site index
// (LGT_Code/modules/admin/init.c:741-829) and parity = (t+x+y+z) & 1.  Because L3 is even,
// the two sites n = 2h and 2h+1 have opposite parity, so h enumerates each parity exactly once.
// One link is 16 B in FP32 (one float4, one 128-bit load) and 32 B in FP64 (two double2).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace su2g {

template <typename R>
struct Q {
    R c0, c1, c2, c3;
};

template <typename R>
__host__ __device__ __forceinline__ Q<R> q_make(R a, R b, R c, R d)
{
    Q<R> q;
    q.c0 = a; q.c1 = b; q.c2 = c; q.c3 = d;
    return q;
}

template <typename R>
__host__ __device__ __forceinline__ Q<R> q_one() { return q_make<R>(R(1), R(0), R(0), R(0)); }
template <typename R>
__host__ __device__ __forceinline__ Q<R> q_zero() { return q_make<R>(R(0), R(0), R(0), R(0)); }

// a * b
template <typename R>
__host__ __device__ __forceinline__ Q<R> q_mul(const Q<R>& a, const Q<R>& b)
{
    Q<R> r;
    r.c0 = a.c0 * b.c0 - a.c1 * b.c1 - a.c2 * b.c2 - a.c3 * b.c3;
    r.c1 = a.c0 * b.c1 + a.c1 * b.c0 - a.c2 * b.c3 + a.c3 * b.c2;
    r.c2 = a.c0 * b.c2 + a.c1 * b.c3 + a.c2 * b.c0 - a.c3 * b.c1;
    r.c3 = a.c0 * b.c3 - a.c1 * b.c2 + a.c2 * b.c1 + a.c3 * b.c0;
    return r;
}

// a * b^dag
template <typename R>
__host__ __device__ __forceinline__ Q<R> q_mul_nd(const Q<R>& a, const Q<R>& b)
{
    Q<R> r;
    r.c0 = a.c0 * b.c0 + a.c1 * b.c1 + a.c2 * b.c2 + a.c3 * b.c3;
    r.c1 = -a.c0 * b.c1 + a.c1 * b.c0 + a.c2 * b.c3 - a.c3 * b.c2;
    r.c2 = -a.c0 * b.c2 - a.c1 * b.c3 + a.c2 * b.c0 + a.c3 * b.c1;
    r.c3 = -a.c0 * b.c3 + a.c1 * b.c2 - a.c2 * b.c1 + a.c3 * b.c0;
    return r;
}

// a^dag * b
template <typename R>
__host__ __device__ __forceinline__ Q<R> q_mul_dn(const Q<R>& a, const Q<R>& b)
{
    Q<R> r;
    r.c0 = a.c0 * b.c0 + a.c1 * b.c1 + a.c2 * b.c2 + a.c3 * b.c3;
    r.c1 = a.c0 * b.c1 - a.c1 * b.c0 + a.c2 * b.c3 - a.c3 * b.c2;
    r.c2 = a.c0 * b.c2 - a.c1 * b.c3 - a.c2 * b.c0 + a.c3 * b.c1;
    r.c3 = a.c0 * b.c3 + a.c1 * b.c2 - a.c2 * b.c1 - a.c3 * b.c0;
    return r;
}

// s + a*b and s + a*b^dag, written so that the accumulation folds into the multiply-adds
template <typename R>
__host__ __device__ __forceinline__ Q<R> q_mul_add(const Q<R>& s, const Q<R>& a, const Q<R>& b)
{
    Q<R> r;
    r.c0 = s.c0 + a.c0 * b.c0 - a.c1 * b.c1 - a.c2 * b.c2 - a.c3 * b.c3;
    r.c1 = s.c1 + a.c0 * b.c1 + a.c1 * b.c0 - a.c2 * b.c3 + a.c3 * b.c2;
    r.c2 = s.c2 + a.c0 * b.c2 + a.c1 * b.c3 + a.c2 * b.c0 - a.c3 * b.c1;
    r.c3 = s.c3 + a.c0 * b.c3 - a.c1 * b.c2 + a.c2 * b.c1 + a.c3 * b.c0;
    return r;
}

template <typename R>
__host__ __device__ __forceinline__ Q<R> q_mul_nd_add(const Q<R>& s, const Q<R>& a, const Q<R>& b)
{
    Q<R> r;
    r.c0 = s.c0 + a.c0 * b.c0 + a.c1 * b.c1 + a.c2 * b.c2 + a.c3 * b.c3;
    r.c1 = s.c1 - a.c0 * b.c1 + a.c1 * b.c0 + a.c2 * b.c3 - a.c3 * b.c2;
    r.c2 = s.c2 - a.c0 * b.c2 - a.c1 * b.c3 + a.c2 * b.c0 + a.c3 * b.c1;
    r.c3 = s.c3 - a.c0 * b.c3 + a.c1 * b.c2 - a.c2 * b.c1 + a.c3 * b.c0;
    return r;
}

template <typename R>
__host__ __device__ __forceinline__ Q<R> q_mul_dn_add(const Q<R>& s, const Q<R>& a, const Q<R>& b)
{
    Q<R> r;
    r.c0 = s.c0 + a.c0 * b.c0 + a.c1 * b.c1 + a.c2 * b.c2 + a.c3 * b.c3;
    r.c1 = s.c1 + a.c0 * b.c1 - a.c1 * b.c0 + a.c2 * b.c3 - a.c3 * b.c2;
    r.c2 = s.c2 + a.c0 * b.c2 - a.c1 * b.c3 - a.c2 * b.c0 + a.c3 * b.c1;
    r.c3 = s.c3 + a.c0 * b.c3 + a.c1 * b.c2 - a.c2 * b.c1 - a.c3 * b.c0;
    return r;
}

template <typename R>
__host__ __device__ __forceinline__ Q<R> q_dag(const Q<R>& a) { return q_make<R>(a.c0, -a.c1, -a.c2, -a.c3); }

template <typename R>
__host__ __device__ __forceinline__ Q<R> q_add(const Q<R>& a, const Q<R>& b)
{
    return q_make<R>(a.c0 + b.c0, a.c1 + b.c1, a.c2 + b.c2, a.c3 + b.c3);
}

template <typename R>
__host__ __device__ __forceinline__ Q<R> q_sub(const Q<R>& a, const Q<R>& b)
{
    return q_make<R>(a.c0 - b.c0, a.c1 - b.c1, a.c2 - b.c2, a.c3 - b.c3);
}

template <typename R>
__host__ __device__ __forceinline__ Q<R> q_scale(const Q<R>& a, R s)
{
    return q_make<R>(a.c0 * s, a.c1 * s, a.c2 * s, a.c3 * s);
}

// a + s*b
template <typename R>
__host__ __device__ __forceinline__ Q<R> q_axpy(R s, const Q<R>& b, const Q<R>& a)
{
    return q_make<R>(a.c0 + s * b.c0, a.c1 + s * b.c1, a.c2 + s * b.c2, a.c3 + s * b.c3);
}

// 4-vector dot = (1/2) Re tr(a b^dag)
template <typename R>
__host__ __device__ __forceinline__ R q_dot(const Q<R>& a, const Q<R>& b)
{
    return a.c0 * b.c0 + a.c1 * b.c1 + a.c2 * b.c2 + a.c3 * b.c3;
}

template <typename R>
__host__ __device__ __forceinline__ R q_norm2(const Q<R>& a) { return q_dot(a, a); }

__device__ __forceinline__ float rsqrt_r(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrt_r(double x) { return rsqrt(x); }
__device__ __forceinline__ float sqrt_r(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrt_r(double x) { return sqrt(x); }

// Reprojection onto SU(2): U / |U| (project_to_su2, LGT_Code/modules/admin/sun_vfunc.c:69-79).
template <typename R>
__device__ __forceinline__ Q<R> q_project(const Q<R>& a)
{
    return q_scale(a, rsqrt_r(q_norm2(a)));
}

// ---------------------------------------------------------------- geometry ---

// Division by a run-time constant via a multiply-high (Granlund & Montgomery, PLDI'94):
// for d >= 1, l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1,
// q = (t + ((n - t) >> 1)) >> (l - 1) with t = mulhi(m, n), exact for all 32-bit n.
struct FastDiv {
    uint32_t d, m, s1, s2;
};

inline FastDiv make_fastdiv(uint32_t d)
{
    FastDiv f;
    f.d = d;
    uint32_t l = 0;
    while ((1ull << l) < d) ++l;
    f.m = (uint32_t)((((1ull << l) - d) << 32) / d + 1);
    f.s1 = l > 0 ? 1u : 0u;
    f.s2 = l > 0 ? l - 1 : 0u;
    return f;
}

__host__ __device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv& f)
{
#ifdef __CUDA_ARCH__
    uint32_t t = __umulhi(f.m, n);
#else
    uint32_t t = (uint32_t)(((uint64_t)f.m * n) >> 32);
#endif
    return (t + ((n - t) >> f.s1)) >> f.s2;
}

struct Geom {
    int L[4];       // extents t, x, y, z
    int S[4];       // lexicographic strides: S[3] = 1, S[2] = L3, S[1] = L2 L3, S[0] = L1 L2 L3
    int V, Vh;      // volume, half volume
    FastDiv dS0, dS1, dS2;
};

inline Geom make_geom(const int L[4])
{
    Geom g;
    for (int d = 0; d < 4; ++d) g.L[d] = L[d];
    g.S[3] = 1;
    g.S[2] = L[3];
    g.S[1] = L[2] * L[3];
    g.S[0] = L[1] * L[2] * L[3];
    g.V = g.S[0] * L[0];
    g.Vh = g.V / 2;
    g.dS0 = make_fastdiv((uint32_t)g.S[0]);
    g.dS1 = make_fastdiv((uint32_t)g.S[1]);
    g.dS2 = make_fastdiv((uint32_t)g.S[2]);
    return g;
}

// A site with its coordinates and lexicographic index.
struct Site {
    int c[4];
    int n;
};

// Site of the given parity with half-index h.
__device__ __forceinline__ Site site_of(const Geom& g, int parity, int h)
{
    Site s;
    uint32_t n0 = 2u * (uint32_t)h;
    uint32_t t = fdiv(n0, g.dS0);
    uint32_t r = n0 - t * (uint32_t)g.S[0];
    uint32_t x = fdiv(r, g.dS1);
    r -= x * (uint32_t)g.S[1];
    uint32_t y = fdiv(r, g.dS2);
    uint32_t z = r - y * (uint32_t)g.S[2];
    uint32_t odd = ((t + x + y + z) ^ (uint32_t)parity) & 1u;   // z is even here
    s.c[0] = (int)t; s.c[1] = (int)x; s.c[2] = (int)y; s.c[3] = (int)(z + odd);
    s.n = (int)(n0 + odd);
    return s;
}

// Site with lexicographic index n; par receives its parity (t+x+y+z) & 1.  Kernels that visit every
// site enumerate n in order, so that both parities of a region of the lattice are in flight
// together (each link array is then streamed from DRAM once, not once per parity half).
__device__ __forceinline__ Site site_lex(const Geom& g, int n, int& par)
{
    Site s;
    uint32_t t = fdiv((uint32_t)n, g.dS0);
    uint32_t r = (uint32_t)n - t * (uint32_t)g.S[0];
    uint32_t x = fdiv(r, g.dS1);
    r -= x * (uint32_t)g.S[1];
    uint32_t y = fdiv(r, g.dS2);
    uint32_t z = r - y * (uint32_t)g.S[2];
    s.c[0] = (int)t; s.c[1] = (int)x; s.c[2] = (int)y; s.c[3] = (int)z;
    s.n = n;
    par = (int)((t + x + y + z) & 1u);
    return s;
}

// Site visited by thread `tid` of CTA `cta` when CTAs alternate parity over the same run of h:
// CTA 2k takes parity 0 and CTA 2k+1 parity 1 of h = k*ntid .. k*ntid+ntid-1.  A warp still reads
// consecutive links of one array (full 128-bit coalescing), while the CTAs in flight cover both
// parities of one region, so each array is streamed from DRAM once.  Grid: 2 * ceil(Vh / ntid).
__device__ __forceinline__ bool site_cta_pair(const Geom& g, int cta, int tid, int ntid, Site& s, int& par, int& h)
{
    par = cta & 1;
    h = (cta >> 1) * ntid + tid;
    if (h >= g.Vh) return false;
    s = site_of(g, par, h);
    return true;
}

// Site visited by thread `tid` of CTA `cta` when the warps of a CTA alternate parity over the same
// run of h: warp 2k takes parity 0 and warp 2k+1 parity 1 of h = cta ntid/2 + 32k .. + 31.  Every warp
// still reads consecutive links of one parity array, and both parities of a region are loaded by
// the same SM, so a site's neighbours of the other parity are often in its L1.
// Grid: ceil(Vh / (ntid / 2)); ntid a multiple of 64.
__device__ __forceinline__ bool site_warp_pair(const Geom& g, int cta, int tid, int ntid, Site& s, int& par, int& h)
{
    const int w = tid >> 5;
    par = w & 1;
    h = cta * (ntid >> 1) + (w >> 1) * 32 + (tid & 31);
    if (h >= g.Vh) return false;
    s = site_of(g, par, h);
    return true;
}

// Lexicographic index offset of the +mu / -mu neighbour of a site (periodic).
template <int MU>
__device__ __forceinline__ int up_off(const Geom& g, const Site& s)
{
    return s.c[MU] == g.L[MU] - 1 ? -(g.L[MU] - 1) * g.S[MU] : g.S[MU];
}
template <int MU>
__device__ __forceinline__ int dn_off(const Geom& g, const Site& s)
{
    return s.c[MU] == 0 ? (g.L[MU] - 1) * g.S[MU] : -g.S[MU];
}

// Run-time direction variants (for loops whose direction is not a template parameter).
__device__ __forceinline__ int up_off_rt(const Geom& g, const int c[4], int mu)
{
    return c[mu] == g.L[mu] - 1 ? -(g.L[mu] - 1) * g.S[mu] : g.S[mu];
}
__device__ __forceinline__ int dn_off_rt(const Geom& g, const int c[4], int mu)
{
    return c[mu] == 0 ? (g.L[mu] - 1) * g.S[mu] : -g.S[mu];
}

// ------------------------------------------------------------------ fields ---

// View of one link field on the device: one base pointer per direction, so that a smearing
// step can replace some directions (ping-pong) while others stay where they are.  Within a
// direction the element index is parity*Vh + h.
template <typename R>
struct Field;

template <>
struct Field<float> {
    using ptr_t = float4*;
    float4* p[4];
    int Vh;
    // Link at lexicographic site index n of parity par -- h = n >> 1.  Element indices are 32-bit
    // (V <= 2^30 sites), so that an address is one wide multiply-add on the direction's base.
    __device__ __forceinline__ Q<float> ld(int mu, int par, int n) const { return ldh(mu, par, (int)((unsigned)n >> 1)); }
    __device__ __forceinline__ Q<float> ldh(int mu, int par, int h) const
    {
        float4 v = __ldg(p[mu] + (unsigned)(par * Vh + h));
        return q_make<float>(v.x, v.y, v.z, v.w);
    }
    __device__ __forceinline__ void sth(int mu, int par, int h, const Q<float>& q) const
    {
        p[mu][(unsigned)(par * Vh + h)] = make_float4(q.c0, q.c1, q.c2, q.c3);
    }
};

template <>
struct Field<double> {
    using ptr_t = double2*;
    double2* p[4];   // two double2 per link
    int Vh;
    __device__ __forceinline__ Q<double> ld(int mu, int par, int n) const { return ldh(mu, par, (int)((unsigned)n >> 1)); }
    __device__ __forceinline__ Q<double> ldh(int mu, int par, int h) const
    {
        const double2* a = p[mu] + 2u * (unsigned)(par * Vh + h);
        double2 x = __ldg(a), y = __ldg(a + 1);
        return q_make<double>(x.x, x.y, y.x, y.y);
    }
    __device__ __forceinline__ void sth(int mu, int par, int h, const Q<double>& q) const
    {
        double2* a = p[mu] + 2u * (unsigned)(par * Vh + h);
        a[0] = make_double2(q.c0, q.c1);
        a[1] = make_double2(q.c2, q.c3);
    }
};

// The same views with loads through L2 only (ld.global.cg), for a kernel that reads links other
// CTAs of the same launch have written (a persistent kernel, after a grid-wide barrier): the
// read-only path of __ldg may serve such a link from a stale line.
template <typename R>
struct FieldCG;

template <>
struct FieldCG<float> : Field<float> {
    __device__ __forceinline__ Q<float> ld(int mu, int par, int n) const { return ldh(mu, par, (int)((unsigned)n >> 1)); }
    __device__ __forceinline__ Q<float> ldh(int mu, int par, int h) const
    {
        float4 v = __ldcg(p[mu] + (unsigned)(par * Vh + h));
        return q_make<float>(v.x, v.y, v.z, v.w);
    }
};

template <>
struct FieldCG<double> : Field<double> {
    __device__ __forceinline__ Q<double> ld(int mu, int par, int n) const { return ldh(mu, par, (int)((unsigned)n >> 1)); }
    __device__ __forceinline__ Q<double> ldh(int mu, int par, int h) const
    {
        const double2* a = p[mu] + 2u * (unsigned)(par * Vh + h);
        double2 x = __ldcg(a), y = __ldcg(a + 1);
        return q_make<double>(x.x, x.y, y.x, y.y);
    }
};

// Field view over four direction base pointers (each 2*Vh links long).
template <typename R>
inline Field<R> make_field(void* const dirs[4], int Vh)
{
    Field<R> f;
    for (int mu = 0; mu < 4; ++mu) f.p[mu] = reinterpret_cast<typename Field<R>::ptr_t>(dirs[mu]);
    f.Vh = Vh;
    return f;
}

}  // namespace su2g
