// adjoint.cu -- vector-Jacobian product of N APE_all steps followed by the clover charge.
//
// Forward map (the reference's qtop flow, LGT_Code/main_qtop/qtop.c:76-91):
//   U_{k+1} = Proj(U_k + alpha S[U_k])   (smearing_APE_all, LGT_Code/modules/obs/smearing.c:74-105)
//   Q = sum_x q(x) / (32 pi^2)           (topologicalCharge, LGT_Code/modules/obs/topologicalcharge.c:164-199)
// The reference has no derivative code; this file is new.
//
// Conventions.  A link is a quaternion in R^4 with the inner product <a, b> = (1/2) Re tr(a b^dag),
// the 4-vector dot product.  For a product P = a b: dP/da contracts as  p b^dag,  dP/db as  a^dag p.
// G_k denotes dQ/dU_k in that sense.  The output for a link U of U_0 is the su(2) gradient under
// U -> exp(eps X) U with X = i x.sigma, i.e. g = vec(G_0 U^dag) (three coefficients).
//
// Passes.
//  1. Forward with sqrt(N) checkpointing: U_0 and every c-th level are kept (c = ckpt or ceil(sqrt N)).
//  2. G_N = dQ/dU_N: F-bar per site and plane (k_qgrad_fbar), then every link of every clover leaf
//     receives prefix^dag F-bar suffix^dag (k_qgrad_scatter, atomic adds).
//  3. Per segment, recompute its levels from the checkpoint; per level, backwards:
//     v-bar = (G_{k+1} - u' <u', G_{k+1}>) / |v|, the Jacobian of u' = v/|v| (k_ape_vbar), then
//     G_k = v-bar + alpha * (the 18 staple terms in which a link appears) (k_ape_gather).
#include <algorithm>
#include <cmath>
#include <vector>

#include "ape.cuh"
#include "clover.cuh"
#include "internal.cuh"

using namespace su2g;

namespace {

constexpr double kPi = 3.14159265358979323846;

// Plain quaternion arrays (F-bar per plane and site).
__device__ __forceinline__ Q<float> ldq(const float* p, size_t i)
{
    float4 v = reinterpret_cast<const float4*>(p)[i];
    return q_make<float>(v.x, v.y, v.z, v.w);
}
__device__ __forceinline__ Q<double> ldq(const double* p, size_t i)
{
    const double2* a = reinterpret_cast<const double2*>(p) + 2 * i;
    double2 x = a[0], y = a[1];
    return q_make<double>(x.x, x.y, y.x, y.y);
}
__device__ __forceinline__ void stq(float* p, size_t i, const Q<float>& q)
{
    reinterpret_cast<float4*>(p)[i] = make_float4(q.c0, q.c1, q.c2, q.c3);
}
__device__ __forceinline__ void stq(double* p, size_t i, const Q<double>& q)
{
    double2* a = reinterpret_cast<double2*>(p) + 2 * i;
    a[0] = make_double2(q.c0, q.c1);
    a[1] = make_double2(q.c2, q.c3);
}

// Atomic accumulation into a link of a gradient field.
__device__ __forceinline__ void atomic_add_link(const Field<float>& G, int mu, int par, int n, const Q<float>& v)
{
    // one 16-byte vector atomic per link
    atomicAdd(G.p[mu] + (unsigned)(par * G.Vh + (int)((unsigned)n >> 1)), make_float4(v.c0, v.c1, v.c2, v.c3));
}
__device__ __forceinline__ void atomic_add_link(const Field<double>& G, int mu, int par, int n, const Q<double>& v)
{
    double* a = reinterpret_cast<double*>(G.p[mu] + 2u * (unsigned)(par * G.Vh + (int)((unsigned)n >> 1)));
    atomicAdd(a + 0, v.c0);
    atomicAdd(a + 1, v.c1);
    atomicAdd(a + 2, v.c2);
    atomicAdd(a + 3, v.c3);
}

// ----------------------------------------------------------- dQ / dU_N ---

// Planes in the order of the charge's three products: (01)(23), (02)(31), (03)(12).
__host__ __device__ constexpr int plane_a(int p) { return p == 0 ? 0 : p == 1 ? 2 : p == 2 ? 0 : p == 3 ? 3 : p == 4 ? 0 : 1; }
__host__ __device__ constexpr int plane_b(int p) { return p == 0 ? 1 : p == 1 ? 3 : p == 2 ? 2 : p == 3 ? 1 : p == 4 ? 3 : 2; }

// F-bar(x, plane) = dQ/dF(x, plane).  With F pure, c0(F_a F_b) = -<F_a, F_b>, and
// q = 16 sum_pairs c0(F_a F_b)  =>  dQ/dF_a = -16 s F_b, dQ/dF_b = -16 s F_a, s = 1/(32 pi^2).
template <typename R>
__global__ void __launch_bounds__(kBlock) k_qgrad_fbar(Field<R> U, Geom g, R* __restrict__ fbar, R scale)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.V) return;
    int par;
    const Site s = site_lex(g, i, par);
    const size_t V = (size_t)g.V, n = (size_t)s.n;
    Q<R> f0 = clover_F<R, 0, 1>(U, g, s, par), f1 = clover_F<R, 2, 3>(U, g, s, par);
    stq(fbar, 0 * V + n, q_scale(f1, -scale));
    stq(fbar, 1 * V + n, q_scale(f0, -scale));
    f0 = clover_F<R, 0, 2>(U, g, s, par);
    f1 = clover_F<R, 3, 1>(U, g, s, par);
    stq(fbar, 2 * V + n, q_scale(f1, -scale));
    stq(fbar, 3 * V + n, q_scale(f0, -scale));
    f0 = clover_F<R, 0, 3>(U, g, s, par);
    f1 = clover_F<R, 1, 2>(U, g, s, par);
    stq(fbar, 4 * V + n, q_scale(f1, -scale));
    stq(fbar, 5 * V + n, q_scale(f0, -scale));
}

// Leaf step tables: leaf l, segment k -> (direction A or B, sign); the four leaves of
// computeCloverAverages (topologicalcharge.c:70-100): +A+B-A-B, -B+A+B-A, +B-A-B+A, -A-B+A+B.
__host__ __device__ constexpr bool leaf_on_a(int l, int k)
{
    return (l == 0 || l == 3) ? (k == 0 || k == 2) : (k == 1 || k == 3);
}
__host__ __device__ constexpr int leaf_sign(int l, int k)
{
    return l == 0 ? (k < 2 ? 1 : -1) : l == 1 ? (k == 0 || k == 3 ? -1 : 1) : l == 2 ? (k == 0 || k == 3 ? 1 : -1)
                                                                                    : (k < 2 ? -1 : 1);
}

// For one leaf (an E x E loop from x) with adjoint Gbar: every link P_i of the ordered product
// L = P_0 ... P_{M-1} gets  (P_0..P_{i-1})^dag Gbar (P_{i+1}..P_{M-1})^dag, daggered when P_i = U^dag.
template <typename R, int A, int B, int E, int LEAF>
__device__ __forceinline__ void leaf_adjoint(const Field<R>& U, const Field<R>& G, const Geom& g, const Site& s,
                                             int par, const Q<R>& Gbar)
{
    constexpr int M = 4 * E;
    Q<R> pre[M];
    int pos[M];
    int n = s.n, ca = s.c[A], cb = s.c[B], p = par;
    Q<R> acc = q_one<R>();
#pragma unroll
    for (int i = 0; i < M; ++i) {
        const int k = i / E;
        const bool on_a = leaf_on_a(LEAF, k);
        const int D = on_a ? A : B;
        int& c = on_a ? ca : cb;
        if (leaf_sign(LEAF, k) > 0) {
            pos[i] = n;
            acc = q_mul(acc, U.ld(D, p, n));
            if (c == g.L[D] - 1) { n -= (g.L[D] - 1) * g.S[D]; c = 0; }
            else { n += g.S[D]; ++c; }
        } else {
            if (c == 0) { n += (g.L[D] - 1) * g.S[D]; c = g.L[D] - 1; }
            else { n -= g.S[D]; --c; }
            pos[i] = n;
            acc = q_mul_nd(acc, U.ld(D, p ^ 1, n));
        }
        p ^= 1;
        pre[i] = acc;
    }
    Q<R> S = q_one<R>();
#pragma unroll
    for (int i = M - 1; i >= 0; --i) {
        const int k = i / E;
        const int D = leaf_on_a(LEAF, k) ? A : B;
        const bool fwd = leaf_sign(LEAF, k) > 0;
        // parity of the link's site: the walk's parity before a forward step, after a backward one
        const int lp = par ^ ((fwd ? i : i + 1) & 1);
        const Q<R> link = U.ld(D, lp, pos[i]);
        const Q<R> left = i > 0 ? pre[i > 0 ? i - 1 : 0] : q_one<R>();
        const Q<R> gi = q_mul_nd(q_mul_dn(left, Gbar), S);
        if (fwd) {
            atomic_add_link(G, D, lp, pos[i], gi);
            S = q_mul(link, S);
        } else {
            atomic_add_link(G, D, lp, pos[i], q_dag(gi));
            S = q_mul_dn(link, S);
        }
    }
}

template <typename R, int A, int B, int E>
__device__ __forceinline__ void clover_adjoint_e(const Field<R>& U, const Field<R>& G, const Geom& g, const Site& s,
                                                 int par, const Q<R>& Fbar)
{
    const R kcoef = E == 1 ? R(1.5) : E == 2 ? R(-0.15) : R(1.0 / 90.0);
    const Q<R> Gbar = q_scale(Fbar, kcoef * R(0.25));
    leaf_adjoint<R, A, B, E, 0>(U, G, g, s, par, Gbar);
    leaf_adjoint<R, A, B, E, 1>(U, G, g, s, par, Gbar);
    leaf_adjoint<R, A, B, E, 2>(U, G, g, s, par, Gbar);
    leaf_adjoint<R, A, B, E, 3>(U, G, g, s, par, Gbar);
}

template <typename R, int PLANE>
__global__ void __launch_bounds__(kBlock) k_qgrad_scatter(Field<R> U, Field<R> G, Geom g, const R* __restrict__ fbar)
{
    constexpr int A = plane_a(PLANE), B = plane_b(PLANE);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.V) return;
    int par;
    const Site s = site_lex(g, i, par);
    const Q<R> Fbar = ldq(fbar, (size_t)PLANE * g.V + (size_t)s.n);
    clover_adjoint_e<R, A, B, 1>(U, G, g, s, par, Fbar);
    clover_adjoint_e<R, A, B, 2>(U, G, g, s, par, Fbar);
    clover_adjoint_e<R, A, B, 3>(U, G, g, s, par, Fbar);
}

// ------------------------------------------------------ one APE step back ---

// v-bar(x, mu) = (Gn - u' <u', Gn>) / |v|,  v = U + alpha S,  u' = v / |v|  (all four directions).
// The staple sums are the forward step's own (ape_staples), so v is exactly the forward's
// pre-projection link; same site order and occupancy as the forward kernel.
template <typename R>
__global__ void __launch_bounds__(kBlock, 2) k_ape_vbar(Field<R> U, Field<R> Gn, Field<R> Vbar, Geom g, R alpha)
{
    Site s;
    int par, h;
    if (!site_warp_pair(g, blockIdx.x, threadIdx.x, blockDim.x, s, par, h)) return;
    ape_staples<R, SU2G_APE_ALL>(U, g, s, par, h, [&](int mu, const Q<R>& u, const Q<R>& S) {
        const Q<R> v = q_axpy(alpha, S, u);
        const R inv = rsqrt_r(q_norm2(v));
        const Q<R> up = q_scale(v, inv);
        const Q<R> gn = Gn.ldh(mu, par, h);
        Vbar.sth(mu, par, h, q_scale(q_axpy(-q_dot(up, gn), up, gn), inv));
    });
}

// G_k(y, l) = vbar(y, l) + alpha * sum of the 18 staple terms containing U_l(y) (derivation in the
// file header's conventions; smearing.c:42-71 for the staples):
//  for mu != l:  vbar(y,mu) U_l(y+mu) U_mu(y+l)^dag          (first factor of the upper staple of (y, mu))
//                vbar(y-mu,mu)^dag U_l(y-mu) U_mu(y-mu+l)    (third factor, upper staple of (y-mu, mu))
//                U_mu(y) U_l(y+mu) vbar(y+l,mu)^dag          (first factor, lower staple of (y+l, mu))
//                U_mu(y-mu)^dag U_l(y-mu) vbar(y+l-mu,mu)    (third factor, lower staple of (y+l-mu, mu))
//  for nu != l:  U_nu(y-nu)^dag vbar(y-nu,l) U_nu(y-nu+l)    (middle, upper staple of (y-nu, l))
//                U_nu(y) vbar(y+nu,l) U_nu(y+l)^dag          (middle, lower staple of (y+nu, l))
template <typename R, int L>
__device__ __forceinline__ void gather_link(const Field<R>& U, const Field<R>& Vb, const Field<R>& G, const Geom& g,
                                            const Site& s, int par, int h, R alpha)
{
    const int q = par ^ 1;
    const int dl = up_off<L>(g, s);
    Q<R> acc = q_zero<R>();
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        if (m == L) continue;
        const int ym = s.n + dn_off_rt(g, s.c, m);   // y - m
        const int yp = s.n + up_off_rt(g, s.c, m);   // y + m
        const int yl = s.n + dl;                     // y + l
        const int yml = ym + dl;                     // y - m + l
        // The six terms with a common plane share factors: with A = U_m(y), X = U_l(y+m),
        // Xv = vbar(y+m, l), B = U_m(y+l), Vm = vbar(y, m), Vn = vbar(y+l, m)
        //   Vm X B^dag + A Xv B^dag + A X Vn^dag = (Vm X + A Xv) B^dag + (A X) Vn^dag,
        // and with C = U_m(y-m), Y = U_l(y-m), Yv = vbar(y-m, l), D = U_m(y-m+l),
        // Wm = vbar(y-m, m), Wd = vbar(y-m+l, m)
        //   Wm^dag Y D + C^dag Yv D + C^dag Y Wd = (Wm^dag Y + C^dag Yv) D + (C^dag Y) Wd:
        // 10 products and 12 loads instead of 12 and 18.
        {
            const Q<R> A = U.ld(m, par, s.n), X = U.ld(L, q, yp), Xv = Vb.ld(L, q, yp);
            const Q<R> B = U.ld(m, q, yl), Vm = Vb.ld(m, par, s.n), Vn = Vb.ld(m, q, yl);
            const Q<R> AX = q_mul(A, X);
            acc = q_add(acc, q_mul_nd(q_add(q_mul(Vm, X), q_mul(A, Xv)), B));
            acc = q_add(acc, q_mul_nd(AX, Vn));
        }
        {
            const Q<R> C = U.ld(m, q, ym), Y = U.ld(L, q, ym), Yv = Vb.ld(L, q, ym);
            const Q<R> D = U.ld(m, par, yml), Wm = Vb.ld(m, q, ym), Wd = Vb.ld(m, par, yml);
            acc = q_add(acc, q_mul(q_add(q_mul_dn(Wm, Y), q_mul_dn(C, Yv)), D));
            acc = q_add(acc, q_mul(q_mul_dn(C, Y), Wd));
        }
    }
    G.sth(L, par, h, q_axpy(alpha, acc, Vb.ldh(L, par, h)));
}

// One link per thread, blockIdx.y = its direction.  Warp 2k takes parity 0 and warp 2k+1 parity 1
// of the same 32 half-volume indices (site_warp_pair): every warp reads consecutive links of one
// parity array, and both parities of a region are loaded by the same SM.
template <typename R>
__global__ void __launch_bounds__(kBlock) k_ape_gather(Field<R> U, Field<R> Vb, Field<R> G, Geom g, R alpha)
{
    Site s;
    int par, h;
    if (!site_warp_pair(g, blockIdx.x, threadIdx.x, blockDim.x, s, par, h)) return;
    switch (blockIdx.y) {
        case 0: gather_link<R, 0>(U, Vb, G, g, s, par, h, alpha); break;
        case 1: gather_link<R, 1>(U, Vb, G, g, s, par, h, alpha); break;
        case 2: gather_link<R, 2>(U, Vb, G, g, s, par, h, alpha); break;
        default: gather_link<R, 3>(U, Vb, G, g, s, par, h, alpha); break;
    }
}

// su(2) gradient g = vec(G U^dag) per link, written in the reference's site-major order [n][mu][3].
template <typename R>
__global__ void __launch_bounds__(kBlock) k_grad_out(Field<R> G, Field<R> U, Geom g, double* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.V) return;
    int par;
    const Site s = site_lex(g, i, par);
    const int h = i >> 1;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        const Q<R> v = q_mul_nd(G.ldh(mu, par, h), U.ldh(mu, par, h));
        double* o = out + ((size_t)s.n * 4 + mu) * 3;
        o[0] = (double)v.c1;
        o[1] = (double)v.c2;
        o[2] = (double)v.c3;
    }
}

// ------------------------------------------------------------- driver ---

struct FieldBuf {
    void* base = nullptr;
    void* dirs[4] = {nullptr, nullptr, nullptr, nullptr};
};

// Scratch of one VJP from the handle's own stream-ordered pool.  The pool keeps its memory between
// calls (release threshold: unlimited), so repeated calls do not map gigabytes of pages again; the
// memory goes back when the handle is destroyed.
int ensure_pool(su2g_lattice* h)
{
    if (h->pool) return SU2G_OK;
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = h->device;
    int rc = check_cuda(h, cudaMemPoolCreate(&h->pool, &props), "creating the scratch pool");
    if (rc) return rc;
    uint64_t keep = ~0ull;
    return check_cuda(h, cudaMemPoolSetAttribute(h->pool, cudaMemPoolAttrReleaseThreshold, &keep),
                      "configuring the scratch pool");
}

struct Arena {
    su2g_lattice* h;
    std::vector<void*> ptrs;
    int rc = SU2G_OK;
    explicit Arena(su2g_lattice* hh) : h(hh) { rc = ensure_pool(hh); }
    void* get(size_t bytes)
    {
        if (rc) return nullptr;
        void* p = nullptr;
        cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, h->pool, h->stream);
        if (e != cudaSuccess) {
            rc = check_cuda(h, e, "allocating adjoint buffers");
            return nullptr;
        }
        ptrs.push_back(p);
        return p;
    }
    FieldBuf field()
    {
        FieldBuf f;
        const size_t dir_bytes = 2ull * h->g.Vh * h->link_bytes;
        f.base = get(4 * dir_bytes);
        if (f.base)
            for (int mu = 0; mu < 4; ++mu) f.dirs[mu] = (char*)f.base + mu * dir_bytes;
        return f;
    }
    ~Arena()
    {
        for (void* p : ptrs) cudaFreeAsync(p, h->stream);
    }
};

template <typename R>
int vjp_t(su2g_lattice* h, int n_ape, double alpha, int c, double* q_out, double* grad_host)
{
    const Geom& g = h->g;
    const int nseg = n_ape > 0 ? (n_ape + c - 1) / c : 1;
    const int grid = (int)((g.V + kBlock - 1) / kBlock);
    const size_t dir_bytes = 2ull * g.Vh * h->link_bytes;
    Arena ar(h);
    std::vector<FieldBuf> ck(nseg), lev(std::max(c - 1, 0));
    for (auto& f : ck) f = ar.field();
    for (auto& f : lev) f = ar.field();
    FieldBuf tmp[2] = {ar.field(), ar.field()};
    FieldBuf G[2] = {ar.field(), ar.field()};
    FieldBuf Vb = ar.field();
    R* fbar = (R*)ar.get((size_t)6 * g.V * 4 * sizeof(R));
    double* gout = grad_host ? (double*)ar.get((size_t)g.V * 12 * sizeof(double)) : nullptr;
    if (ar.rc) return ar.rc;
    int rc = SU2G_OK;
    // U_0: the handle's field (directions may live in either of its allocations)
    for (int mu = 0; mu < 4; ++mu)
        if ((rc = check_cuda(h, cudaMemcpyAsync(ck[0].dirs[mu], h->dirp[mu], dir_bytes, cudaMemcpyDeviceToDevice,
                                                h->stream), "copying U_0")))
            return rc;
    // forward: keep U_{j c}; the other levels go through two scratch fields
    void* const* cur = ck[0].dirs;
    for (int k = 0; k < n_ape; ++k) {
        void* const* dst = ((k + 1) % c == 0 && (k + 1) / c < nseg) ? ck[(k + 1) / c].dirs : tmp[k & 1].dirs;
        if ((rc = ape_step(h, cur, dst, SU2G_APE_ALL, alpha))) return rc;
        cur = dst;
    }
    if ((rc = ensure_lines(h)) || (rc = qtop_enqueue(h, cur, 0))) return rc;
    // G_N = dQ/dU_N
    const R scale = R(16.0 / (32.0 * kPi * kPi));
    Field<R> UN = make_field<R>(cur, g.Vh);
    Field<R> Gc = make_field<R>(G[0].dirs, g.Vh);
    if ((rc = check_cuda(h, cudaMemsetAsync(G[0].base, 0, 4 * dir_bytes, h->stream), "clearing the gradient")))
        return rc;
    launch_begin(h, SU2G_K_OTHER);
    k_qgrad_fbar<R><<<grid, kBlock, 0, h->stream>>>(UN, g, fbar, scale);
    k_qgrad_scatter<R, 0><<<grid, kBlock, 0, h->stream>>>(UN, Gc, g, fbar);
    k_qgrad_scatter<R, 1><<<grid, kBlock, 0, h->stream>>>(UN, Gc, g, fbar);
    k_qgrad_scatter<R, 2><<<grid, kBlock, 0, h->stream>>>(UN, Gc, g, fbar);
    k_qgrad_scatter<R, 3><<<grid, kBlock, 0, h->stream>>>(UN, Gc, g, fbar);
    k_qgrad_scatter<R, 4><<<grid, kBlock, 0, h->stream>>>(UN, Gc, g, fbar);
    k_qgrad_scatter<R, 5><<<grid, kBlock, 0, h->stream>>>(UN, Gc, g, fbar);
    if ((rc = launch_end(h, SU2G_K_OTHER, "charge adjoint kernels"))) return rc;
    // backwards through the smearing, one checkpoint segment at a time
    int gi = 0;
    for (int j = nseg - 1; j >= 0; --j) {
        const int k0 = j * c, m = std::min(c, n_ape - k0);
        std::vector<void* const*> L(m > 0 ? m : 1);
        L[0] = ck[j].dirs;
        for (int i = 1; i < m; ++i) {
            if ((rc = ape_step(h, L[i - 1], lev[i - 1].dirs, SU2G_APE_ALL, alpha))) return rc;
            L[i] = lev[i - 1].dirs;
        }
        for (int i = m - 1; i >= 0; --i) {
            Field<R> Uk = make_field<R>(L[i], g.Vh);
            Field<R> Gn = make_field<R>(G[gi].dirs, g.Vh), Gk = make_field<R>(G[gi ^ 1].dirs, g.Vh);
            Field<R> Vbf = make_field<R>(Vb.dirs, g.Vh);
            launch_begin(h, SU2G_K_OTHER);
            k_ape_vbar<R><<<2 * (int)((g.Vh + kBlock - 1) / kBlock), kBlock, 0, h->stream>>>(Uk, Gn, Vbf, g, (R)alpha);
            k_ape_gather<R><<<dim3(2 * (int)((g.Vh + kBlock - 1) / kBlock), 4), kBlock, 0, h->stream>>>(Uk, Vbf, Gk, g,
                                                                                                      (R)alpha);
            if ((rc = launch_end(h, SU2G_K_OTHER, "smearing adjoint kernels"))) return rc;
            gi ^= 1;
        }
    }
    if (grad_host) {
        launch_begin(h, SU2G_K_OTHER);
        k_grad_out<R><<<grid, kBlock, 0, h->stream>>>(make_field<R>(G[gi].dirs, g.Vh), make_field<R>(ck[0].dirs, g.Vh),
                                                      g, gout);
        if ((rc = launch_end(h, SU2G_K_OTHER, "gradient output"))) return rc;
        if ((rc = check_cuda(h, cudaMemcpyAsync(grad_host, gout, (size_t)g.V * 12 * sizeof(double),
                                                cudaMemcpyDeviceToHost, h->stream), "copying the gradient")))
            return rc;
    }
    if ((rc = fetch_results(h, 0, 2))) return rc;
    if (q_out) *q_out = h->h_out[0];
    return SU2G_OK;
}

int segment_length(int n_ape, int ckpt)
{
    if (ckpt > 0) return std::min(ckpt, std::max(n_ape, 1));
    int c = (int)std::ceil(std::sqrt((double)std::max(n_ape, 1)));
    return std::max(c, 1);
}

// One step along su(2) coefficients x (per site and direction, the layout of the VJP's gradient):
// U_mu(n) <- exp(eps X) U_mu(n), X = i x.sigma, exp(eps X) = (cos(eps|x|), sin(eps|x|) x/|x|), for
// the sites [n0, n0 + count) whose coefficients are in `xs` (12 doubles per site).
template <typename R>
__global__ void __launch_bounds__(kBlock) k_tangent_step(const double* __restrict__ xs, Field<R> U, Geom g, int n0,
                                                         int count, double eps)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const int n = n0 + i;
        int par;
        const Site s = site_lex(g, n, par);
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) {
            const double* x = xs + (size_t)i * 12 + 3 * mu;
            const double nx = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
            double sn, cs;
            sincos(eps * nx, &sn, &cs);
            const double f = nx > 0.0 ? sn / nx : 0.0;
            const Q<R> E = q_make<R>((R)cs, (R)(f * x[0]), (R)(f * x[1]), (R)(f * x[2]));
            U.sth(mu, par, n >> 1, q_mul(E, U.ld(mu, par, s.n)));
        }
    }
}

}  // namespace

extern "C" int su2g_ape_qtop_vjp(su2g_lattice* h, int32_t n_ape, double alpha, int32_t ckpt, double* q, double* grad)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_ape_qtop_vjp: null handle");
    if (n_ape < 0 || ckpt < 0 || !std::isfinite(alpha))
        return set_error(h, SU2G_EINVAL, "su2g_ape_qtop_vjp: bad argument (n_ape=%d, ckpt=%d)", n_ape, ckpt);
    cudaSetDevice(h->device);
    const int c = segment_length(n_ape, ckpt);
    return h->prec == SU2G_FP32 ? vjp_t<float>(h, n_ape, alpha, c, q, grad) : vjp_t<double>(h, n_ape, alpha, c, q, grad);
}

extern "C" int su2g_vjp_plan(const su2g_lattice* h, int32_t n_ape, int32_t ckpt, int32_t* levels_stored,
                             int64_t* device_bytes)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_vjp_plan: null handle");
    if (n_ape < 0 || ckpt < 0) return set_error(nullptr, SU2G_EINVAL, "su2g_vjp_plan: bad argument");
    const int c = segment_length(n_ape, ckpt);
    const int nseg = n_ape > 0 ? (n_ape + c - 1) / c : 1;
    const int levels = nseg + std::max(c - 1, 0);   // checkpoints + one recomputed segment
    const int64_t field = 4ll * h->g.V * (int64_t)h->link_bytes;
    if (levels_stored) *levels_stored = levels;
    // levels + 2 forward scratch + 2 gradients + v-bar + F-bar (6 quaternions per site) + output staging
    if (device_bytes)
        *device_bytes = (int64_t)(levels + 5) * field + 6ll * h->g.V * (int64_t)h->link_bytes + 96ll * h->g.V;
    return SU2G_OK;
}

extern "C" int su2g_tangent_step(su2g_lattice* h, const double* x, double eps)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_tangent_step: null handle");
    if (!x || !std::isfinite(eps)) return set_error(h, SU2G_EINVAL, "su2g_tangent_step: bad argument");
    cudaSetDevice(h->device);
    int rc = ensure_aos(h);   // the coefficients stream through the transfer staging, 12 of its 16 doubles a site
    if (rc) return rc;
    for (size_t n0 = 0; n0 < (size_t)h->g.V; n0 += h->aos_sites) {
        const int cnt = (int)std::min(h->aos_sites, (size_t)h->g.V - n0);
        rc = check_cuda(h, cudaMemcpyAsync(h->d_aos, x + n0 * 12, (size_t)cnt * 12 * sizeof(double),
                                           cudaMemcpyHostToDevice, h->stream),
                        "uploading tangent coefficients");
        if (rc) return rc;
        const int grid = grid_for(h, cnt, 8);
        launch_begin(h, SU2G_K_OTHER);
        if (h->prec == SU2G_FP32)
            k_tangent_step<float><<<grid, kBlock, 0, h->stream>>>(h->d_aos, make_field<float>(h->dirp, h->g.Vh), h->g,
                                                                 (int)n0, cnt, eps);
        else
            k_tangent_step<double><<<grid, kBlock, 0, h->stream>>>(h->d_aos, make_field<double>(h->dirp, h->g.Vh), h->g,
                                                                  (int)n0, cnt, eps);
        if ((rc = launch_end(h, SU2G_K_OTHER, "tangent step"))) return rc;
    }
    return check_cuda(h, cudaStreamSynchronize(h->stream), "tangent step");
}
