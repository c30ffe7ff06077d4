// clover.cuh -- path products and the improved clover field strength (shared by the charge and
// its adjoint).  Reference: computeLine / computeCloverAverages / hermitianTraceless /
// computeCloverProducts, LGT_Code/modules/obs/topologicalcharge.c:18-162.
#pragma once
#include "su2.cuh"

namespace su2g {

// A path walker: its product and position (lexicographic index, coordinates along A and B, parity).
template <typename R>
struct Walker {
    Q<R> acc;
    int n, ca, cb, p;
};

// One step of a walker along +D or -D (D = A or B of the plane; the coordinate tracked is ca or cb).
// Forward: acc *= U_D(y), y += D.  Backward: y -= D, acc *= U_D(y)^dag  (computeLine,
// topologicalcharge.c:18-44).
template <typename R, int D, bool FWD, bool ISA>
__device__ __forceinline__ void wstep(const Field<R>& U, const Geom& g, Walker<R>& w)
{
    int& c = ISA ? w.ca : w.cb;
    if (FWD) {
        w.acc = q_mul(w.acc, U.ld(D, w.p, w.n));
        if (c == g.L[D] - 1) { w.n -= (g.L[D] - 1) * g.S[D]; c = 0; }
        else { w.n += g.S[D]; ++c; }
        w.p ^= 1;
    } else {
        if (c == 0) { w.n += (g.L[D] - 1) * g.S[D]; c = g.L[D] - 1; }
        else { w.n -= g.S[D]; --c; }
        w.p ^= 1;
        w.acc = q_mul_nd(w.acc, U.ld(D, w.p, w.n));
    }
}

// Improved clover field strength in plane (A, B) at site s:
// F = [(k1 C1 + k2 C2 + k3 C3) - h.c.]/2 with C_e = (1/4) sum of the four e x e leaves and
// (k1, k2, k3) = (1.5, -0.15, 1/90)  (computeCloverAverages / computeCloverProducts /
// hermitianTraceless, topologicalcharge.c:46-162).  The leaves, all starting and ending at x:
//   +A +B -A -B,   -B +A +B -A,   +B -A -B +A,   -A -B +A +B
// (each segment e links long).  The four leaves walk in lockstep, one step each per iteration, so
// a thread keeps four independent product chains in flight.  The clover sizes run as a loop, not
// unrolled, which keeps the register count low enough for two CTAs per SM.
template <typename R, int A, int B>
__device__ __forceinline__ Q<R> clover_F(const Field<R>& U, const Geom& g, const Site& s, int par)
{
    Q<R> F = q_zero<R>();
#pragma unroll 1
    for (int e = 1; e <= 3; ++e) {
        const R kcoef = e == 1 ? R(1.5) : (e == 2 ? R(-0.15) : R(1.0 / 90.0));
        Walker<R> w[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) w[i] = Walker<R>{q_one<R>(), s.n, s.c[A], s.c[B], par};
        for (int i = 0; i < e; ++i) {   // segment 1: +A, -B, +B, -A
            wstep<R, A, true, true>(U, g, w[0]);
            wstep<R, B, false, false>(U, g, w[1]);
            wstep<R, B, true, false>(U, g, w[2]);
            wstep<R, A, false, true>(U, g, w[3]);
        }
        for (int i = 0; i < e; ++i) {   // segment 2: +B, +A, -A, -B
            wstep<R, B, true, false>(U, g, w[0]);
            wstep<R, A, true, true>(U, g, w[1]);
            wstep<R, A, false, true>(U, g, w[2]);
            wstep<R, B, false, false>(U, g, w[3]);
        }
        for (int i = 0; i < e; ++i) {   // segment 3: -A, +B, -B, +A
            wstep<R, A, false, true>(U, g, w[0]);
            wstep<R, B, true, false>(U, g, w[1]);
            wstep<R, B, false, false>(U, g, w[2]);
            wstep<R, A, true, true>(U, g, w[3]);
        }
        for (int i = 0; i < e; ++i) {   // segment 4: -B, -A, +A, +B
            wstep<R, B, false, false>(U, g, w[0]);
            wstep<R, A, false, true>(U, g, w[1]);
            wstep<R, A, true, true>(U, g, w[2]);
            wstep<R, B, true, false>(U, g, w[3]);
        }
        const Q<R> C = q_add(q_add(w[0].acc, w[1].acc), q_add(w[2].acc, w[3].acc));
        F = q_axpy(kcoef * R(0.25), C, F);
    }
    F.c0 = R(0);   // (F - F^dag)/2 keeps the su(2) part
    return F;
}

}  // namespace su2g
