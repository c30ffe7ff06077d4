// clover.cuh -- path products and the improved clover field strength (shared by the charge and
// its adjoint).  Reference: computeLine / computeCloverAverages / hermitianTraceless /
// computeCloverProducts, LGT_Code/modules/obs/topologicalcharge.c:18-162.
#pragma once
#include "su2.cuh"

namespace su2g {

// Walk `steps` links along direction D (negative: backwards), multiplying the path product.
// Forward: acc *= U_D(y), y += D.  Backward: y -= D, acc *= U_D(y)^dag  (computeLine,
// topologicalcharge.c:18-44).
template <typename R, int D>
__device__ __forceinline__ void walk(const Field<R>& U, const Geom& g, int& n, int& c, int& par, int steps, Q<R>& acc)
{
    if (steps > 0) {
        for (int i = 0; i < steps; ++i) {
            acc = q_mul(acc, U.ld(D, par, n));
            if (c == g.L[D] - 1) { n -= (g.L[D] - 1) * g.S[D]; c = 0; }
            else { n += g.S[D]; ++c; }
            par ^= 1;
        }
    } else {
        for (int i = 0; i < -steps; ++i) {
            if (c == 0) { n += (g.L[D] - 1) * g.S[D]; c = g.L[D] - 1; }
            else { n -= g.S[D]; --c; }
            par ^= 1;
            acc = q_mul_nd(acc, U.ld(D, par, n));
        }
    }
}

// Improved clover field strength in plane (A, B) at site s:
// F = [(k1 C1 + k2 C2 + k3 C3) - h.c.]/2 with C_e = (1/4) sum of the four e x e leaves and
// (k1, k2, k3) = (1.5, -0.15, 1/90)  (computeCloverAverages / computeCloverProducts /
// hermitianTraceless, topologicalcharge.c:46-162).  The leaves, all starting and ending at x:
//   +A +B -A -B,   -B +A +B -A,   +B -A -B +A,   -A -B +A +B.
template <typename R, int A, int B>
__device__ __forceinline__ Q<R> clover_F(const Field<R>& U, const Geom& g, const Site& s, int par)
{
    const R kcoef[3] = {R(1.5), R(-0.15), R(1.0 / 90.0)};
    Q<R> F = q_zero<R>();
#pragma unroll
    for (int e = 1; e <= 3; ++e) {
        Q<R> C = q_zero<R>();
        int n = s.n, ca = s.c[A], cb = s.c[B], p = par;
        Q<R> l = q_one<R>();
        walk<R, A>(U, g, n, ca, p, e, l); walk<R, B>(U, g, n, cb, p, e, l);
        walk<R, A>(U, g, n, ca, p, -e, l); walk<R, B>(U, g, n, cb, p, -e, l);
        C = q_add(C, l);
        l = q_one<R>();
        walk<R, B>(U, g, n, cb, p, -e, l); walk<R, A>(U, g, n, ca, p, e, l);
        walk<R, B>(U, g, n, cb, p, e, l); walk<R, A>(U, g, n, ca, p, -e, l);
        C = q_add(C, l);
        l = q_one<R>();
        walk<R, B>(U, g, n, cb, p, e, l); walk<R, A>(U, g, n, ca, p, -e, l);
        walk<R, B>(U, g, n, cb, p, -e, l); walk<R, A>(U, g, n, ca, p, e, l);
        C = q_add(C, l);
        l = q_one<R>();
        walk<R, A>(U, g, n, ca, p, -e, l); walk<R, B>(U, g, n, cb, p, -e, l);
        walk<R, A>(U, g, n, ca, p, e, l); walk<R, B>(U, g, n, cb, p, e, l);
        C = q_add(C, l);
        F = q_axpy(kcoef[e - 1] * R(0.25), C, F);
    }
    F.c0 = R(0);   // (F - F^dag)/2 keeps the su(2) part
    return F;
}

}  // namespace su2g
