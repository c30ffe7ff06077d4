// observables.cu -- plaquette, APE smearing, planar Wilson loops and the improved-clover charge.
//
// Reference routines: plaquette() (LGT_Code/modules/obs/plaquette.c:67-100), smearing_APE_*
// (LGT_Code/modules/obs/smearing.c:42-168), compute_wloop / measureWilsonLoop
// (LGT_Code/modules/obs/wilson.c:21-56, :268-324), topologicalCharge and helpers
// (LGT_Code/modules/obs/topologicalcharge.c:18-199).
//
// Global sums are compensated FP64 (TwoSum) in every precision mode: per-thread sums, warp and
// CTA trees, then a fixed-order pass over the per-CTA partials, so results are bit-reproducible
// for a given lattice and grid.
#include <algorithm>
#include <cmath>

#include "internal.cuh"
#include "clover.cuh"
#include "ape.cuh"

using namespace su2g;

namespace {

constexpr double kPi = 3.14159265358979323846;

// ------------------------------------------------------------ plaquette ---

// One site per thread, CTAs dispatched in order; each CTA leaves one compensated partial sum.
// Eight 128-thread CTAs per SM: at 48^4 on B200, 182 against 189 us (FP64) and 103 against 106.5 us
// (FP32) with four CTAs of 256 threads.
template <typename R>
__global__ void __launch_bounds__(128, 8) k_plaquette(Field<R> U, Geom g, DD* __restrict__ partials)
{
    double site = 0.0;
    Site s;
    int par, h;
    if (site_cta_pair(g, blockIdx.x, threadIdx.x, blockDim.x, s, par, h)) {
        const int q = par ^ 1;
        Q<R> u[4];
        int xp[4];
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) {
            u[mu] = U.ldh(mu, par, h);
            xp[mu] = s.n + up_off_rt(g, s.c, mu);
        }
#pragma unroll
        for (int mu = 0; mu < 3; ++mu)
#pragma unroll
            for (int nu = mu + 1; nu < 4; ++nu) {
                // Re tr U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag = 2 <U_mu(x)U_nu(x+mu), U_nu(x)U_mu(x+nu)>
                Q<R> a = q_mul(u[mu], U.ld(nu, q, xp[mu]));
                Q<R> b = q_mul(u[nu], U.ld(mu, q, xp[nu]));
                site += (double)q_dot(a, b);
            }
    }
    DD acc = dd_block_sum_d<128>(site);
    if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

// ------------------------------------------------------------------- APE ---

// One Jacobi step U'_mu(x) = Proj(U_mu(x) + alpha S_mu(x)) (smearing.c:74-168) with the staple
// sums of ape_staples (ape.cuh).  Reads `in`, writes only the updated directions of `out`.
// 128-thread CTAs; resident CTAs per SM, measured at 48^4 on B200: FP32 APE_all four (at most 128
// registers; 235.5 us against 238.8 us with five, 243 us with six, 254 us with two 256-thread
// CTAs); FP32 spatial and temporal eight (131.4 us spatial against 132.6 us with four of 256, 136 us
// with six, 164 us with two). FP64
// APE_all three (619 us against 626 us with four, 655 us with two of 256), spatial four (337 us
// against 359 us with three, 357 us with two of 256), temporal eight (212 against 216 us with four
// of 256).
template <typename R, int MODE>
constexpr int ape_min_blocks()
{
    return MODE == SU2G_APE_ALL ? (sizeof(R) == 4 ? 4 : 3) : (sizeof(R) == 4 || MODE == SU2G_APE_TEMPORAL ? 8 : 4);
}
template <typename R, int MODE>
constexpr int ape_block()
{
    return 128;
}

template <typename R, int MODE>
__global__ void __launch_bounds__(ape_block<R, MODE>(), ape_min_blocks<R, MODE>()) k_ape(Field<R> in, Field<R> out,
                                                                                        Geom g, R alpha)
{
    // one site per thread; CTAs dispatched in order, warps alternating parity over the same h run
    // (so that both parities of a region share an L1: FP32 APE_all 237.8 against 240.7 us, spatial
    // 129.1 against 131.6 us, FP64 spatial 355 against 367 us with parity-alternating CTAs)
    Site s;
    int par, h;
    if (site_warp_pair(g, blockIdx.x, threadIdx.x, blockDim.x, s, par, h)) {
        ape_staples<R, MODE>(in, g, s, par, h, [&](int mu, const Q<R>& u, const Q<R>& S) {
            out.sth(mu, par, h, q_project(q_axpy(alpha, S, u)));
        });
    }
}

// ---------------------------------------------------------- Wilson loops ---

constexpr int kWilsonTChunk = 32;   // T values one launch records
constexpr int kWilsonWarps = kBlock / 32;

template <int K>
__device__ __forceinline__ int shift_k(const Geom& g, int ck, int j)
{
    int c = ck + j;
    c -= c >= g.L[K] ? g.L[K] : 0;
    if (c >= g.L[K]) c %= g.L[K];   // j >= L_K: a loop longer than the lattice
    return (c - ck) * g.S[K];
}

__device__ __forceinline__ int shift_t(const Geom& g, int ct, int T)
{
    int c = ct + T;
    c -= c >= g.L[0] ? g.L[0] : 0;
    if (c >= g.L[0]) c %= g.L[0];   // T >= L_t does not occur (T <= L_t - 1 is checked)
    return (c - ct) * g.S[0];
}

// For one site x and spatial direction K: all loops W(R, T) with R in [r0, r0+RC) and T in
// [tlo, thi], by line products (compute_wloop, wilson.c:21-56, factored):
//   W = (1/2) Re tr [T_T(x) S_R(x+T t) T_T(x+R k)^dag S_R(x)^dag] = <T_T(x) S_R(x+T t), S_R(x) T_T(x+R k)>
// with T_T(y) = U_0(y) U_0(y+t) ... (T links) and S_R(y) = U_K(y) ... U_K(y+(R-1)k) (R links).
// Temporal lines grow by one link per T; spatial lines at x+T t are rebuilt per T.
template <typename R, int K, int RC>
__device__ __forceinline__ void wilson_site(const Field<R>& U, const Geom& g, const Site& s, int par, int r0, int tlo,
                                            int thi, DD* __restrict__ wacc)
{
    const int lane = threadIdx.x & 31;
    Q<R> SX[RC], TR[RC];
    int xr[RC];   // lexicographic index of x + (r0 + r) k
    // spatial lines at x
    Q<R> S = q_one<R>();
    for (int j = 0; j < r0 - 1; ++j) S = q_mul(S, U.ld(K, par ^ (j & 1), s.n + shift_k<K>(g, s.c[K], j)));
#pragma unroll
    for (int r = 0; r < RC; ++r) {
        const int j = r0 - 1 + r;
        S = q_mul(S, U.ld(K, par ^ (j & 1), s.n + shift_k<K>(g, s.c[K], j)));
        SX[r] = S;
        xr[r] = s.n + shift_k<K>(g, s.c[K], j + 1);
        TR[r] = q_one<R>();
    }
    Q<R> TX = q_one<R>();
    for (int T = 1; T <= thi; ++T) {
        const int tprev = shift_t(g, s.c[0], T - 1), tcur = shift_t(g, s.c[0], T);
        const int pprev = par ^ ((T - 1) & 1);
        TX = q_mul(TX, U.ld(0, pprev, s.n + tprev));
#pragma unroll
        for (int r = 0; r < RC; ++r) TR[r] = q_mul(TR[r], U.ld(0, pprev ^ ((r0 + r) & 1), xr[r] + tprev));
        // spatial lines at x + T t
        const int pT = par ^ (T & 1);
        Q<R> ST = q_one<R>();
        for (int j = 0; j < r0 - 1; ++j)
            ST = q_mul(ST, U.ld(K, pT ^ (j & 1), s.n + tcur + shift_k<K>(g, s.c[K], j)));
#pragma unroll
        for (int r = 0; r < RC; ++r) {
            const int j = r0 - 1 + r;
            ST = q_mul(ST, U.ld(K, pT ^ (j & 1), s.n + tcur + shift_k<K>(g, s.c[K], j)));
            double w = 0.0;
            if (T >= tlo) w = (double)q_dot(q_mul(TX, ST), q_mul(SX[r], TR[r]));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
            if (T >= tlo && lane == 0) {
                DD* slot = wacc + r * kWilsonTChunk + (T - tlo);
                *slot = dd_add(*slot, w);
            }
        }
    }
}

template <typename R, int RC>
__global__ void __launch_bounds__(kBlock) k_wilson(Field<R> U, Geom g, int r0, int tlo, int thi,
                                                   DD* __restrict__ partials)
{
    __shared__ DD wacc[kWilsonWarps][RC * kWilsonTChunk];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int j = lane; j < RC * kWilsonTChunk; j += 32) wacc[warp][j] = DD{0.0, 0.0};
    __syncwarp();
    // every lane of a warp runs the same number of iterations (shuffles inside)
    const int stride = gridDim.x * blockDim.x;
    const int base = blockIdx.x * blockDim.x + warp * 32;
    for (int i0 = base; i0 < g.V; i0 += stride) {
        const int i = i0 + lane;
        const bool valid = i < g.V;
        const int ii = valid ? i : i0;   // inactive lanes recompute a valid site and contribute 0
        int par;
        const Site s = site_lex(g, ii, par);
        DD* acc = &wacc[warp][0];
        // Lanes past the end recompute a valid site with an empty record window (tlo > thi).  Every
        // lane makes the same calls, so each full-mask shuffle inside is one instruction executed
        // by the whole warp.
        const int tlo_lane = valid ? tlo : thi + 1;
        wilson_site<R, 1, RC>(U, g, s, par, r0, tlo_lane, thi, acc);
        wilson_site<R, 2, RC>(U, g, s, par, r0, tlo_lane, thi, acc);
        wilson_site<R, 3, RC>(U, g, s, par, r0, tlo_lane, thi, acc);
    }
    __syncthreads();
    // fixed-order sum over warps, one partial per slot
    for (int j = threadIdx.x; j < RC * kWilsonTChunk; j += blockDim.x) {
        DD v = {0.0, 0.0};
        for (int w = 0; w < kWilsonWarps; ++w) v = dd_add(v, wacc[w][j]);
        partials[(size_t)j * kMaxPartials + blockIdx.x] = v;
    }
}

// Column form of the same sums.  A CTA owns `sw` consecutive spatial sites s (the lexicographic
// index within a time slice) in every time slice; thread t * sw + j takes site t S0 + s0 + j.  Per
// spatial direction K each thread stores its spatial lines S_{r0+r}(x) in shared memory, so the
// line at x + T t that the loop needs for every T is the one the thread of slice t + T stored:
// it is read, not rebuilt, which removes the longest product chain of the per-site form.
constexpr int kWilsonColMaxThreads = 512;
constexpr int kWilsonRc8MaxThreads = 192;   // the column kernel with eight (FP32) / four (FP64) loops

// Accumulation of the column kernel's loop terms in shared memory.  FP32: the 32 lanes' terms are
// summed in the link precision (one shuffle per step; its rounding, ~1e-7 of a warp sum, is far
// below the FP32 links' own) and lane 0 adds the warp sum to the warp's slot.  FP64: every thread
// adds its own term to its own slot (no shuffles; the FP64 shuffle pairs cost more than the larger
// slot array).  A slot adds a few hundred terms (3 directions x the CTA's tiles) in plain FP64; the
// slots of all warps or threads and of all CTAs are then summed compensated, in a fixed order.
// Slot layout: [r][T - tlo][owner], owner = warp (FP32) or thread (FP64).
template <typename R>
__host__ __device__ constexpr bool wilson_thread_slots() { return sizeof(R) == 8; }

template <typename R>
__device__ __forceinline__ size_t wilson_slot(int r, int ti, int nT, int warp)
{
    return wilson_thread_slots<R>() ? ((size_t)r * nT + ti) * blockDim.x + threadIdx.x
                                    : ((size_t)r * nT + ti) * (blockDim.x >> 5) + warp;
}

// The RC terms w[r] of one T into their slots.  FP64: each thread into its own slots.  FP32: the
// warp sums of all RC terms by one transposing reduction (RC a power of two <= 32): at each of the
// first log2(RC) shuffle levels a lane keeps one half of its values and sends the other half to its
// partner, which keeps the opposite half, so the value count halves with the distance; a plain
// butterfly over the remaining lane bits follows.  Lane r * (32 / RC) then holds the warp sum of
// term r, after RC - 1 + 5 - log2(RC) shuffles and adds (6 for RC = 4; one butterfly per term took
// 5 RC = 20).
template <typename R, int RC>
__device__ __forceinline__ void wilson_acc(double* __restrict__ wacc, R (&w)[RC], int ti, int nT, int warp, int lane)
{
    if (wilson_thread_slots<R>()) {
#pragma unroll
        for (int r = 0; r < RC; ++r) wacc[wilson_slot<R>(r, ti, nT, warp)] += (double)w[r];
    } else {
        static_assert(RC >= 1 && RC <= 32 && (RC & (RC - 1)) == 0, "RC must be a power of two <= 32");
#pragma unroll
        for (int n = RC, width = 16; n > 1; n >>= 1, width >>= 1) {
            const bool upper = (lane & width) != 0;
#pragma unroll
            for (int i = 0; i < n / 2; ++i) {
                const R keep = upper ? w[i + n / 2] : w[i];
                const R send = upper ? w[i] : w[i + n / 2];
                w[i] = keep + __shfl_xor_sync(0xffffffffu, send, width);
            }
        }
        R x = w[0];
#pragma unroll
        for (int width = 16 / RC; width > 0; width >>= 1) x += __shfl_xor_sync(0xffffffffu, x, width);
        constexpr int group = 32 / RC;
        if ((lane & (group - 1)) == 0) wacc[wilson_slot<R>(lane / group, ti, nT, warp)] += (double)x;
    }
}

// The loops of one spatial direction K for a CTA's column, transported up in time:
//   Y_R^T(x) = T_T(x) S_R(x + T t) T_T(x + R k)^dag = U_t(x) Y_R^{T-1}(x + t) U_t(x + R k)^dag,
//   Y_R^0 = S_R,   W(R, T) at x = <Y_R^T(x), S_R(x)>  (compute_wloop, wilson.c:21-56, factored).
// U_t(x + R k) does not depend on T, so the T loop loads nothing from global memory: Y^{T-1}(x + t)
// is the value the thread one time slice up (thread (t+1) sw + j, periodic) wrote into a
// double-buffered shared array, one barrier per T; two products per (R, T) and site.
template <typename R, int K, int RC>
__device__ __forceinline__ void wilson_col_dir(const Field<R>& U, const Geom& g, Q<R>* __restrict__ ybuf,
                                               double* __restrict__ wacc, int sw, int t, int j, int s, bool valid,
                                               int r0, int tlo, int thi)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nT = thi - tlo + 1;
    int par;
    const int n = t * g.S[0] + s;
    const Site st = site_lex(g, n, par);
    Q<R> SX[RC], UR[RC], Y[RC];   // S_{r0+r}(x); U_t(x + (r0+r) k); the transported loop
    Q<R> S = q_one<R>();
    for (int jj = 0; jj < r0 - 1; ++jj) S = q_mul(S, U.ld(K, par ^ (jj & 1), n + shift_k<K>(g, st.c[K], jj)));
#pragma unroll
    for (int r = 0; r < RC; ++r) {
        const int jj = r0 - 1 + r;
        S = q_mul(S, U.ld(K, par ^ (jj & 1), n + shift_k<K>(g, st.c[K], jj)));
        SX[r] = S;
        Y[r] = S;
        UR[r] = U.ld(0, par ^ ((jj + 1) & 1), n + shift_k<K>(g, st.c[K], jj + 1));
    }
    const Q<R> UT = U.ld(0, par, n);
    int tn = t + 1;
    tn -= tn >= g.L[0] ? g.L[0] : 0;
    // buffer layout [T & 1][r][thread]: a warp's 16-byte accesses to one r are consecutive, so they
    // are free of bank conflicts (a per-thread block of RC loops put lanes RC * 16 bytes apart)
    const int up = tn * sw + j, nt = blockDim.x;
    for (int T = 1; T <= thi; ++T) {
        Q<R>* buf = ybuf + (size_t)(T & 1) * nt * RC;
#pragma unroll
        for (int r = 0; r < RC; ++r) buf[(size_t)r * nt + threadIdx.x] = Y[r];
        __syncthreads();   // the other buffer was last read before the previous barrier
#pragma unroll
        for (int r = 0; r < RC; ++r) Y[r] = q_mul_nd(q_mul(UT, buf[(size_t)r * nt + up]), UR[r]);
        if (T < tlo) continue;
        R w[RC];
#pragma unroll
        for (int r = 0; r < RC; ++r) w[r] = valid ? q_dot(Y[r], SX[r]) : R(0);
        wilson_acc<R, RC>(wacc, w, T - tlo, nT, warp, lane);
    }
    __syncthreads();   // the buffers are written again by the next direction
}

// FP32 with eight loops a thread (167 registers) and FP64 with four (162) are capped at
// kWilsonRc8MaxThreads threads (96-thread CTAs at 48^4) so that they need not spill: the R <= 9 set
// took 3.95 ms against 4.25 ms with four loops (FP32) and 9.87 against 10.10 ms with two loops in
// 288-thread CTAs (FP64).  These widths are chosen only where a column fits the cap.
template <typename R, int RC>
__global__ void __launch_bounds__((sizeof(R) == 4 && RC >= 8) || (sizeof(R) == 8 && RC >= 4) ? kWilsonRc8MaxThreads : kWilsonColMaxThreads, 1) k_wilson_col(Field<R> U, Geom g, int sw, int r0, int tlo,
                                                                        int thi, DD* __restrict__ partials)
{
    extern __shared__ __align__(16) unsigned char wsm[];
    Q<R>* ybuf = (Q<R>*)wsm;   // two buffers of RC loops per thread
    const int nwarps = blockDim.x >> 5, nT = thi - tlo + 1;
    double* wacc = (double*)(wsm + (size_t)2 * blockDim.x * RC * sizeof(Q<R>));
    const int owners = wilson_thread_slots<R>() ? (int)blockDim.x : nwarps;
    for (int i = threadIdx.x; i < owners * RC * nT; i += blockDim.x) wacc[i] = 0.0;
    __syncthreads();
    const int t = threadIdx.x / sw, j = threadIdx.x % sw;
    const int stot = g.S[0], ntiles = (stot + sw - 1) / sw;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int s_req = tile * sw + j;
        const bool valid = s_req < stot;
        const int s = valid ? s_req : stot - 1;   // threads past the end read a valid site and add 0
        wilson_col_dir<R, 1, RC>(U, g, ybuf, wacc, sw, t, j, s, valid, r0, tlo, thi);
        wilson_col_dir<R, 2, RC>(U, g, ybuf, wacc, sw, t, j, s, valid, r0, tlo, thi);
        wilson_col_dir<R, 3, RC>(U, g, ybuf, wacc, sw, t, j, s, valid, r0, tlo, thi);
    }
    // fixed-order sum over warps; slot r * kWilsonTChunk + (T - tlo) as in k_wilson
    for (int i = threadIdx.x; i < RC * nT; i += blockDim.x) {
        const int r = i / nT, ti = i % nT;
        DD v = {0.0, 0.0};
        for (int w = 0; w < owners; ++w) v = dd_add(v, wacc[((size_t)r * nT + ti) * owners + w]);
        partials[(size_t)(r * kWilsonTChunk + ti) * kMaxPartials + blockIdx.x] = v;
    }
}

// Spatial sites per CTA for the column kernel: the smallest sw with L_t sw a multiple of 32 and at
// least `min_threads` threads; 0 if that exceeds kWilsonColMaxThreads (the per-site kernel then
// runs).  Wide CTAs read longer runs of consecutive sites; small ones pack the SM's four schedulers
// evenly.  Measured at 24^4 and 48^4 on B200: the FP32 R-chunk-4 kernel (106 registers, 4 warps per
// scheduler) is fastest with ~96 threads (a 288-thread CTA left room for one CTA per SM), every
// other instance with >= 256 threads (FP64 chunk 4: 23.4 ms against 26.7 ms at 96 threads).
int wilson_col_width(const Geom& g, int min_threads = 256)
{
    int a = g.L[0], b = 32;
    while (b) {
        const int r = a % b;
        a = b;
        b = r;
    }
    const int m = 32 / a;
    if (g.L[0] * m > kWilsonColMaxThreads) return 0;
    int sw = m;
    while (g.L[0] * (sw + m) <= kWilsonColMaxThreads && g.L[0] * sw < min_threads) sw += m;
    return sw;
}

template <typename R, int RC>
size_t wilson_col_smem(int threads, int nT)
{
    const int owners = wilson_thread_slots<R>() ? threads : threads / 32;
    return (size_t)2 * threads * RC * sizeof(Q<R>) + (size_t)owners * RC * nT * sizeof(double);
}

// --------------------------------------------------- topological charge ---

// Line products for the charge: L^e_D(x) = U_D(x) U_D(x+D) ... U_D(x+(e-1)D) for e = 2, 3 and every
// direction D, stored in the field's layout (L2 and L3 are two four-direction fields).  The clover
// leaves of size e are then products of four e-link segments, each one line (computeLine,
// topologicalcharge.c:18-44, evaluated once per segment and site instead of once per leaf).
template <typename R>
__global__ void __launch_bounds__(kBlock) k_lines(Field<R> U, Field<R> L2, Field<R> L3, Geom g)
{
    Site s;
    int par, h;
    if (!site_cta_pair(g, blockIdx.x, threadIdx.x, blockDim.x, s, par, h)) return;
#pragma unroll
    for (int D = 0; D < 4; ++D) {
        int c = s.c[D] + 1;
        c -= c >= g.L[D] ? g.L[D] : 0;
        const int n1 = s.n + (c - s.c[D]) * g.S[D];
        int c2 = c + 1;
        c2 -= c2 >= g.L[D] ? g.L[D] : 0;
        const int n2 = s.n + (c2 - s.c[D]) * g.S[D];
        const Q<R> l2 = q_mul(U.ldh(D, par, h), U.ld(D, par ^ 1, n1));
        L2.sth(D, par, h, l2);
        L3.sth(D, par, h, q_mul(l2, U.ld(D, par, n2)));
    }
}

// Offset of the lexicographic index for k steps (|k| <= 3) along direction d from coordinate c.
__device__ __forceinline__ int shift_by(const Geom& g, int d, int c, int k)
{
    const int L = g.L[d];
    int cc = c + k;
#pragma unroll
    for (int i = 0; i < 2; ++i) {   // |k| <= 3 <= 2 L - 1 for L >= 2: two wraps at most
        cc += cc < 0 ? L : 0;
        cc -= cc >= L ? L : 0;
    }
    return (cc - c) * g.S[d];
}

// Improved clover field strength in plane (A, B) at site s from line products (the same
// F = [(k1 C1 + k2 C2 + k3 C3) - h.c.]/2, C_e = (1/4) sum of the four e x e leaves, (k1, k2, k3) =
// (1.5, -0.15, 1/90), as clover_F in clover.cuh; topologicalcharge.c:46-162).  With a = eA, b = eB
// and L the e-link lines of the two directions, the leaves starting and ending at x are
//   +A +B -A -B:  LA(x) LB(x+a) LA(x+b)^dag LB(x)^dag
//   -B +A +B -A:  LB(x-b)^dag LA(x-b) LB(x+a-b) LA(x)^dag
//   +B -A -B +A:  LB(x) LA(x-a+b)^dag LB(x-a)^dag LA(x-a)
//   -A -B +A +B:  LA(x-a)^dag LB(x-a-b)^dag LA(x-a-b) LB(x-b)
// : twelve loads and twelve products per size.
template <typename R, int A, int B>
__device__ __forceinline__ Q<R> clover_F_lines(const Field<R>& U, const Field<R>& L2, const Field<R>& L3,
                                               const Geom& g, const Site& s, int par)
{
    Q<R> F = q_zero<R>();
#pragma unroll 1
    for (int e = 1; e <= 3; ++e) {
        // the two directions' e-link lines (pointers selected in registers, not a field by reference)
        Field<R> L;
        L.Vh = U.Vh;
        L.p[A] = e == 1 ? U.p[A] : (e == 2 ? L2.p[A] : L3.p[A]);
        L.p[B] = e == 1 ? U.p[B] : (e == 2 ? L2.p[B] : L3.p[B]);
        const R kcoef = e == 1 ? R(1.5) : (e == 2 ? R(-0.15) : R(1.0 / 90.0));
        const int pa = A, pb = B;
        const int oa = shift_by(g, pa, s.c[pa], e), ma = shift_by(g, pa, s.c[pa], -e);
        const int ob = shift_by(g, pb, s.c[pb], e), mb = shift_by(g, pb, s.c[pb], -e);
        const int q1 = par ^ (e & 1);   // parity one segment away
        const int n = s.n;
        const Q<R> LAx = L.ld(A, par, n), LBx = L.ld(B, par, n);
        const Q<R> LBxa = L.ld(B, q1, n + oa), LAxb = L.ld(A, q1, n + ob);
        const Q<R> LBxmb = L.ld(B, q1, n + mb), LAxmb = L.ld(A, q1, n + mb);
        const Q<R> LBxamb = L.ld(B, par, n + oa + mb), LAxmab = L.ld(A, par, n + ma + ob);
        const Q<R> LBxma = L.ld(B, q1, n + ma), LAxma = L.ld(A, q1, n + ma);
        const Q<R> LBxmamb = L.ld(B, par, n + ma + mb), LAxmamb = L.ld(A, par, n + ma + mb);
        const Q<R> l0 = q_mul_nd(q_mul_nd(q_mul(LAx, LBxa), LAxb), LBx);
        const Q<R> l1 = q_mul_nd(q_mul(q_mul_dn(LBxmb, LAxmb), LBxamb), LAx);
        const Q<R> l2 = q_mul(q_mul_nd(q_mul_nd(LBx, LAxmab), LBxma), LAxma);
        const Q<R> l3 = q_mul(q_mul(q_dag(q_mul(LBxmamb, LAxma)), LAxmamb), LBxmb);
        F = q_axpy(kcoef * R(0.25), q_add(q_add(l0, l1), q_add(l2, l3)), F);
    }
    F.c0 = R(0);   // (F - F^dag)/2 keeps the su(2) part
    return F;
}

// q(x) = 8 [tr F01 F23 + tr F02 F31 + tr F03 F12], tr = 2 c0 (topologicalcharge.c:175-178)
template <typename R>
__device__ __forceinline__ double qtop_density(const Field<R>& U, const Field<R>& L2, const Field<R>& L3,
                                               const Geom& g, const Site& s, int par)
{
    double d = 0.0;
    d += 16.0 * (double)q_mul(clover_F_lines<R, 0, 1>(U, L2, L3, g, s, par), clover_F_lines<R, 2, 3>(U, L2, L3, g, s, par)).c0;
    d += 16.0 * (double)q_mul(clover_F_lines<R, 0, 2>(U, L2, L3, g, s, par), clover_F_lines<R, 3, 1>(U, L2, L3, g, s, par)).c0;
    d += 16.0 * (double)q_mul(clover_F_lines<R, 0, 3>(U, L2, L3, g, s, par), clover_F_lines<R, 1, 2>(U, L2, L3, g, s, par)).c0;
    return d;
}

// One site per thread; CTA partials of q and |q| at partials[b] and partials[gridDim.x + b].
// Resident CTAs per SM: three in FP32 and two in FP64.
template <typename R>
__global__ void __launch_bounds__(kBlock, sizeof(R) == 4 ? 3 : 2) k_qtop(Field<R> U, Field<R> L2, Field<R> L3, Geom g,
                                                                        DD* __restrict__ partials)
{
    // parities paired per warp (site_warp_pair); grid ceil(V / kBlock)
    Site s;
    int par, h;
    double d = 0.0;
    if (site_warp_pair(g, blockIdx.x, threadIdx.x, blockDim.x, s, par, h)) d = qtop_density<R>(U, L2, L3, g, s, par);
    DD acc = dd_block_sum_d<kBlock>(d);
    DD aabs = dd_block_sum_d<kBlock>(fabs(d));
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = acc;
        partials[gridDim.x + blockIdx.x] = aabs;
    }
}

int ensure_alt(su2g_lattice* h)
{
    if (h->field_alt) return SU2G_OK;
    cudaError_t e = cudaMalloc(&h->field_alt, 4ull * h->g.V * h->link_bytes);
    if (e != cudaSuccess) return check_cuda(h, e, "allocating the smearing field");
    // the partner of each direction is the slot in the other allocation not currently used
    for (int mu = 0; mu < 4; ++mu) {
        size_t off = (size_t)mu * 2 * h->g.Vh * h->link_bytes;
        h->altp[mu] = (char*)h->field_alt + off;
    }
    return SU2G_OK;
}

template <typename R, int MODE>
void launch_ape_t(su2g_lattice* h, const Field<R>& in, const Field<R>& out, R alpha)
{
    constexpr int block = ape_block<R, MODE>();
    const int grid = (int)((2 * (long long)h->g.Vh + block - 1) / block);   // warp pairs over the same h run
    k_ape<R, MODE><<<grid, block, 0, h->stream>>>(in, out, h->g, alpha);
}

template <typename R>
void launch_ape(su2g_lattice* h, void* const in_dirs[4], void* const out_dirs[4], int mode, R alpha)
{
    Field<R> in = make_field<R>(in_dirs, h->g.Vh), out = make_field<R>(out_dirs, h->g.Vh);
    if (mode == SU2G_APE_ALL) launch_ape_t<R, SU2G_APE_ALL>(h, in, out, alpha);
    else if (mode == SU2G_APE_SPATIAL) launch_ape_t<R, SU2G_APE_SPATIAL>(h, in, out, alpha);
    else launch_ape_t<R, SU2G_APE_TEMPORAL>(h, in, out, alpha);
}

// Launch one chunk of loops; returns the number of CTAs (= partials per slot), 0 on a launch error.
template <typename R, int RC>
int launch_wilson_t(su2g_lattice* h, void* const dirs[4], int r0, int tlo, int thi)
{
    const Field<R> U = make_field<R>(dirs, h->g.Vh);
    const int sw = wilson_col_width(h->g, (sizeof(R) == 4 && RC >= 4) || (sizeof(R) == 8 && RC >= 4) ? 64 : 256);
    if (sw > 0) {
        const int threads = sw * h->g.L[0];
        const size_t smem = wilson_col_smem<R, RC>(threads, thi - tlo + 1);
        int per_sm = 0;
        if (smem <= (size_t)h->max_smem &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wilson_col<R, RC>, threads, smem) == cudaSuccess &&
            per_sm > 0) {
            const int ntiles = (h->g.S[0] + sw - 1) / sw;
            const int grid = std::max(1, std::min(std::min(ntiles, h->num_sms * per_sm), kMaxPartials));
            k_wilson_col<R, RC><<<grid, threads, smem, h->stream>>>(U, h->g, sw, r0, tlo, thi, h->partials);
            return grid;
        }
        cudaGetLastError();
    }
    const int grid = resident_grid(h, (const void*)k_wilson<R, RC>, h->g.V);
    k_wilson<R, RC><<<grid, kBlock, 0, h->stream>>>(U, h->g, r0, tlo, thi, h->partials);
    return grid;
}

template <typename R>
int launch_wilson(su2g_lattice* h, void* const dirs[4], int rc, int r0, int tlo, int thi)
{
    switch (rc) {
        case 1: return launch_wilson_t<R, 1>(h, dirs, r0, tlo, thi);
        case 2: return launch_wilson_t<R, 2>(h, dirs, r0, tlo, thi);
        case 4: return launch_wilson_t<R, 4>(h, dirs, r0, tlo, thi);
        default: return launch_wilson_t<R, 8>(h, dirs, r0, tlo, thi);
    }
}

template <typename R, int RC>
void wilson_smem_attr(int bytes)
{
    cudaFuncSetAttribute(k_wilson_col<R, RC>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    // the small FP32 CTAs (96 threads, two buffers of RC loops, ~13 KB) fit six per SM by their
    // registers and need ~80 KB of shared memory for that; without a preference the driver picked a
    // 32 KB carveout.  The FP64 instances keep the default, which leaves L1 its room (a maximal
    // carveout cost FP64 5 %).
    if (sizeof(R) == 4 && RC >= 4)
        cudaFuncSetAttribute(k_wilson_col<R, RC>, cudaFuncAttributePreferredSharedMemoryCarveout, 50);
}

}  // namespace

extern "C" int su2g_plaquette(su2g_lattice* h, double* p)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_plaquette: null handle");
    if (!p) return set_error(h, SU2G_EINVAL, "su2g_plaquette: null output");
    cudaSetDevice(h->device);
    int rc = plaquette_enqueue(h, 0);
    if (!rc) rc = fetch_results(h, 0, 1);
    if (!rc) *p = h->h_out[0];
    return rc;
}

int su2g::plaquette_enqueue(su2g_lattice* h, int out_off)
{
    const int grid = 2 * (int)((h->g.Vh + 127) / 128);
    int rc = ensure_partial_entries(h, grid);
    if (rc) return rc;
    launch_begin(h, SU2G_K_PLAQUETTE);
    if (h->prec == SU2G_FP32)
        k_plaquette<float><<<grid, 128, 0, h->stream>>>(make_field<float>(h->dirp, h->g.Vh), h->g, h->partials);
    else
        k_plaquette<double><<<grid, 128, 0, h->stream>>>(make_field<double>(h->dirp, h->g.Vh), h->g, h->partials);
    rc = launch_end(h, SU2G_K_PLAQUETTE, "plaquette kernel");
    // plaq = sum 2 c0 / (2 * 6 * V)  (plaquette.c:97); the kernel sums c0 = (1/2) Re tr
    if (!rc) rc = finalize(h, grid, 1, 1.0 / (6.0 * (double)h->g.V), out_off, grid);
    return rc;
}

// Enqueue `ns` smearing steps without synchronising (used by su2g_ape and the adjoint).
int su2g::ape_step(su2g_lattice* h, void* const in_dirs[4], void* const out_dirs[4], int mode, double alpha)
{
    if (h->prec == SU2G_FP32 && mode == SU2G_APE_ALL && h->ape_variant == 1) {
        const int yb = ape_tma_rows(h->g, h->max_smem);
        if (yb > 0) return ape_tma_launch(h, in_dirs, out_dirs, alpha, yb);
    }
    launch_begin(h, SU2G_K_APE);
    if (h->prec == SU2G_FP32) launch_ape<float>(h, in_dirs, out_dirs, mode, (float)alpha);
    else launch_ape<double>(h, in_dirs, out_dirs, mode, alpha);
    return launch_end(h, SU2G_K_APE, "APE kernel");
}

int su2g::ape_run(su2g_lattice* h, void* cur[4], void* alt[4], int steps, int mode, double alpha)
{
    for (int step = 0; step < steps; ++step) {
        const int rc = ape_step(h, cur, alt, mode, alpha);
        if (rc) return rc;
        for (int mu = 0; mu < 4; ++mu)
            if (ape_updates(mode, mu)) std::swap(cur[mu], alt[mu]);
    }
    return SU2G_OK;
}

int su2g::ape_enqueue(su2g_lattice* h, int ns, double alpha, int mode)
{
    const int rc = ensure_alt(h);
    return rc ? rc : ape_run(h, h->dirp, h->altp, ns, mode, alpha);
}

int su2g::ensure_lines(su2g_lattice* h)
{
    if (h->lines) return SU2G_OK;
    const cudaError_t e = cudaMalloc(&h->lines, 8ull * h->g.V * h->link_bytes);
    if (e != cudaSuccess) return check_cuda(h, e, "allocating the charge's line products");
    return SU2G_OK;
}

int su2g::qtop_enqueue(su2g_lattice* h, void* const dirs[4], int out_off)
{
    if (!h->lines) return set_error(h, SU2G_EINVAL, "topological charge: line scratch not allocated");
    const int grid = (int)((h->g.V + kBlock - 1) / kBlock);
    int rc0 = ensure_partial_entries(h, 2ull * grid);
    if (rc0) return rc0;
    void* l2[4];
    void* l3[4];
    for (int mu = 0; mu < 4; ++mu) {
        l2[mu] = (char*)h->lines + (size_t)mu * h->g.V * h->link_bytes;
        l3[mu] = (char*)h->lines + (size_t)(4 + mu) * h->g.V * h->link_bytes;
    }
    const int lgrid = 2 * (int)((h->g.Vh + kBlock - 1) / kBlock);
    launch_begin(h, SU2G_K_QTOP);
    if (h->prec == SU2G_FP32) {
        const Field<float> U = make_field<float>(dirs, h->g.Vh), L2 = make_field<float>(l2, h->g.Vh),
                           L3 = make_field<float>(l3, h->g.Vh);
        k_lines<float><<<lgrid, kBlock, 0, h->stream>>>(U, L2, L3, h->g);
        k_qtop<float><<<grid, kBlock, 0, h->stream>>>(U, L2, L3, h->g, h->partials);
    } else {
        const Field<double> U = make_field<double>(dirs, h->g.Vh), L2 = make_field<double>(l2, h->g.Vh),
                            L3 = make_field<double>(l3, h->g.Vh);
        k_lines<double><<<lgrid, kBlock, 0, h->stream>>>(U, L2, L3, h->g);
        k_qtop<double><<<grid, kBlock, 0, h->stream>>>(U, L2, L3, h->g, h->partials);
    }
    int rc = launch_end(h, SU2G_K_QTOP, "topological charge kernel");
    // Q = sum_x q(x) / (32 pi^2)  (topologicalcharge.c:194)
    if (!rc) rc = finalize(h, grid, 2, 1.0 / (32.0 * kPi * kPi), out_off, grid);
    return rc;
}

extern "C" int su2g_ape(su2g_lattice* h, int32_t ns, double alpha, int32_t mode)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_ape: null handle");
    if (ns < 0 || mode < SU2G_APE_ALL || mode > SU2G_APE_TEMPORAL || !std::isfinite(alpha))
        return set_error(h, SU2G_EINVAL, "su2g_ape: bad argument (ns=%d, mode=%d)", ns, mode);
    cudaSetDevice(h->device);
    return ape_enqueue(h, ns, alpha, mode);
}

void su2g::wilson_prepare(su2g_lattice* h)
{
    // the column kernel's dynamic shared memory can exceed the 48 KB default; allowed once per handle
    wilson_smem_attr<float, 1>(h->max_smem);
    wilson_smem_attr<float, 2>(h->max_smem);
    wilson_smem_attr<float, 4>(h->max_smem);
    wilson_smem_attr<float, 8>(h->max_smem);
    wilson_smem_attr<double, 1>(h->max_smem);
    wilson_smem_attr<double, 2>(h->max_smem);
    wilson_smem_attr<double, 4>(h->max_smem);
    wilson_smem_attr<double, 8>(h->max_smem);
    cudaGetLastError();
}

int su2g::wilson_check(su2g_lattice* h, const int32_t* R, const int32_t* T, int n, const char* who)
{
    int tmax = 0;
    for (int i = 0; i < n; ++i) {
        if (R[i] < 1 || T[i] < 1) return set_error(h, SU2G_EINVAL, "%s: R and T must be >= 1", who);
        tmax = std::max(tmax, (int)T[i]);
    }
    // measureWilsonLoop refuses T > L_t - 1 (wilson.c:290-291)
    if (tmax > h->g.L[0] - 1)
        return set_error(h, SU2G_EINVAL, "%s: lattice too small to measure loops (T=%d, L_t=%d)", who, tmax, h->g.L[0]);
    return SU2G_OK;
}

int su2g::wilson_enqueue(su2g_lattice* h, void* const dirs[4], const int32_t* R, const int32_t* T, int n, int out_off,
                         int max_slots, int* slot)
{
    int rmax = 0, tmax = 0;
    for (int i = 0; i < n; ++i) {
        rmax = std::max(rmax, (int)R[i]);
        tmax = std::max(tmax, (int)T[i]);
    }
    std::vector<char> want((size_t)rmax * tmax, 0);
    for (int i = 0; i < n; ++i) want[(size_t)(R[i] - 1) * tmax + (T[i] - 1)] = 1;
    // R in chunks of 8/4/2/1, T in chunks of kWilsonTChunk; a chunk with no wanted pair is skipped
    struct Chunk {
        int rc_n, r0, tlo, thi, base;
    };
    std::vector<Chunk> plan;
    std::vector<int> slot_rt((size_t)rmax * tmax, -1);
    int used = 0;
    // the column kernel transports its loops in time, so a narrow R chunk costs it only the rebuild
    // of its spatial lines: FP32 runs chunks of 4 loops per thread, FP64 of 2 (4 spills in FP64:
    // 22.5 ms against 11.2 ms for W(R, T <= 9) at 48^4); the per-site kernel prefers 8
    const int sw8 = wilson_col_width(h->g, 64);
    const bool rc8 = sw8 > 0 && sw8 * h->g.L[0] <= kWilsonRc8MaxThreads;
    const int rc_max = wilson_col_width(h->g) > 0 ? (h->prec == SU2G_FP32 ? (rc8 ? 8 : 4) : (rc8 ? 4 : 2)) : 8;
    for (int r0 = 1; r0 <= rmax;) {
        const int left = rmax - r0 + 1;
        const int rc_n = left >= 8 && rc_max >= 8 ? 8 : (left >= 4 ? 4 : (left >= 2 ? 2 : 1));
        for (int tlo = 1; tlo <= tmax; tlo += kWilsonTChunk) {
            const int thi = std::min(tmax, tlo + kWilsonTChunk - 1);
            bool any = false;
            for (int r = r0; r < r0 + rc_n; ++r)
                for (int t = tlo; t <= thi; ++t) any = any || want[(size_t)(r - 1) * tmax + (t - 1)];
            if (!any) continue;
            plan.push_back({rc_n, r0, tlo, thi, out_off + used});
            for (int r = 0; r < rc_n; ++r)
                for (int t = tlo; t <= thi; ++t)
                    slot_rt[(size_t)(r0 + r - 1) * tmax + (t - 1)] = out_off + used + r * kWilsonTChunk + (t - tlo);
            used += rc_n * kWilsonTChunk;
        }
        r0 += rc_n;
    }
    if (used > max_slots)
        return set_error(h, SU2G_EINVAL, "Wilson loops: %d result slots needed, %d available", used, max_slots);
    int rc = ensure_partials(h, 8 * kWilsonTChunk);
    if (rc) return rc;
    for (const Chunk& c : plan) {
        launch_begin(h, SU2G_K_WILSON);
        const int grid = h->prec == SU2G_FP32 ? launch_wilson<float>(h, dirs, c.rc_n, c.r0, c.tlo, c.thi)
                                              : launch_wilson<double>(h, dirs, c.rc_n, c.r0, c.tlo, c.thi);
        if ((rc = launch_end(h, SU2G_K_WILSON, "Wilson loop kernel"))) return rc;
        // W = sum_x,k c0 / (3 V)  (wilson.c:322: sum of Re tr / (3 V 2))
        if ((rc = finalize(h, grid, c.rc_n * kWilsonTChunk, 1.0 / (3.0 * (double)h->g.V), c.base))) return rc;
    }
    for (int i = 0; i < n; ++i) slot[i] = slot_rt[(size_t)(R[i] - 1) * tmax + (T[i] - 1)];
    return SU2G_OK;
}

extern "C" int su2g_wilson(su2g_lattice* h, const int32_t* R, const int32_t* T, int32_t n, double* w)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_wilson: null handle");
    if (n < 0 || (n > 0 && (!R || !T || !w))) return set_error(h, SU2G_EINVAL, "su2g_wilson: bad argument");
    if (n == 0) return SU2G_OK;
    int rc = wilson_check(h, R, T, n, "su2g_wilson");
    if (rc) return rc;
    cudaSetDevice(h->device);
    // pairs are measured in groups whose chunks fit the result slots
    std::vector<int> slot(n);
    for (int i0 = 0; i0 < n;) {
        int i1 = n;
        while ((rc = wilson_enqueue(h, h->dirp, R + i0, T + i0, i1 - i0, 0, kOutSlots - 2, slot.data() + i0)) ==
                   SU2G_EINVAL &&
               i1 - i0 > 1)
            i1 = i0 + (i1 - i0) / 2;
        if (rc) return rc;
        const int nres = 1 + *std::max_element(slot.begin() + i0, slot.begin() + i1);
        if ((rc = fetch_results(h, 0, nres))) return rc;
        for (int i = i0; i < i1; ++i) w[i] = h->h_out[slot[i]];
        i0 = i1;
    }
    return SU2G_OK;
}

extern "C" int su2g_qtop(su2g_lattice* h, double* q, double* sum_abs)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_qtop: null handle");
    if (!q) return set_error(h, SU2G_EINVAL, "su2g_qtop: null output");
    cudaSetDevice(h->device);
    int rc = ensure_lines(h);
    if (!rc) rc = qtop_enqueue(h, h->dirp, 0);
    if (!rc) rc = fetch_results(h, 0, 2);
    if (!rc) {
        *q = h->h_out[0];
        if (sum_abs) *sum_abs = h->h_out[1];
    }
    return rc;
}
