// ape.cuh -- the APE staple sums of one site, shared by the smearing step and its adjoint.
// Reference: staples_smearing / smearing_APE_all, _spatial, _temporal
// (LGT_Code/modules/obs/smearing.c:42-168).
#pragma once
#include "internal.cuh"

namespace su2g {

__host__ __device__ constexpr bool ape_updates(int mode, int mu)
{
    return mode == SU2G_APE_ALL ? true : (mode == SU2G_APE_SPATIAL ? mu != 0 : mu == 0);
}
// Is nu a staple direction for link mu?  staples_smearing(n, dir, dt) skips kk == dir and kk == dt
// with dt = dir (all), 0 (spatial, temporal)  (smearing.c:51, :89, :122, :155).
__host__ __device__ constexpr bool ape_staple(int mode, int mu, int nu)
{
    return nu != mu && (mode == SU2G_APE_ALL ? true : nu != 0);
}

// Staple sums S_mu(x) of the links the mode updates, and the links u_mu(x) they need, with the
// staples of smearing.c:42-71:
//   S_mu(x) = sum_nu U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag + U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu).
// The middle product P = U_mu(x+nu) U_nu(x+mu)^dag of the forward staple of mu in plane nu is
// also the dagger of the middle product of the forward staple of nu in plane mu, so each plane's
// P is formed once.  emit(mu, u_mu, S_mu) is called for each updated link as soon as its sum is
// complete (the caller stores or differentiates it; one link's state at a time stays live).
template <typename R, int MODE, typename Emit>
__device__ __forceinline__ void ape_staples(const Field<R>& in, const Geom& g, const Site& s, int par, int h,
                                            Emit&& emit)
{
    const int q = par ^ 1;
    int xp[4], xm[4];
    Q<R> u[4], S[4];
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        xp[mu] = s.n + up_off_rt(g, s.c, mu);
        xm[mu] = s.n + dn_off_rt(g, s.c, mu);
        S[mu] = q_zero<R>();
        bool need = ape_updates(MODE, mu);
#pragma unroll
        for (int nu = 0; nu < 4; ++nu) need = need || (ape_updates(MODE, nu) && ape_staple(MODE, nu, mu));
        if (need) u[mu] = in.ldh(mu, par, h);
    }
#pragma unroll
    for (int mu = 0; mu < 4; ++mu)
#pragma unroll
        for (int nu = mu + 1; nu < 4; ++nu) {
            const bool a = ape_updates(MODE, mu) && ape_staple(MODE, mu, nu);
            const bool b = ape_updates(MODE, nu) && ape_staple(MODE, nu, mu);
            if (!a && !b) continue;
            const Q<R> P = q_mul_nd(in.ld(mu, q, xp[nu]), in.ld(nu, q, xp[mu]));
            if (a) S[mu] = q_mul_add(S[mu], u[nu], P);      // U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag
            if (b) S[nu] = q_mul_nd_add(S[nu], u[mu], P);   // U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag
        }
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        if (!ape_updates(MODE, mu)) continue;
        const int dmu = xp[mu] - s.n;
#pragma unroll
        for (int nu = 0; nu < 4; ++nu) {
            if (!ape_staple(MODE, mu, nu)) continue;
            const Q<R> a = in.ld(nu, q, xm[nu]);          // U_nu(x-nu)
            const Q<R> b = in.ld(mu, q, xm[nu]);          // U_mu(x-nu)
            const Q<R> c = in.ld(nu, par, xm[nu] + dmu);  // U_nu(x-nu+mu)
            S[mu] = q_mul_add(S[mu], q_mul_dn(a, b), c);
        }
        emit(mu, u[mu], S[mu]);
    }
}

}  // namespace su2g
