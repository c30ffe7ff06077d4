/*
 * su2_oracle.c -- CPU restatement of the reference's SU(2) pure-gauge hot path.
 *
 * ORACLE / TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load this library, and only as the checker.
 * The product path (masterarbeit_b200/, libsu2g.so) never links or calls it.
 *
 * Parity is pinned: tests/test_oracle_cpu.py checks every routine here against
 * outputs of the reference's own C code (compiled from source by
 * oracle/build_ref.sh, run through oracle/ref_harness.c) committed as golden
 * fixtures under tests/golden/.
 *
 * Field layout is the reference's host layout (`pu[0][0]` block,
 * LGT_Code/modules/admin/init.c:842-858): double U[V][4][4], site-major, then
 * direction, then quaternion components c0..c3, with the lexicographic site
 * index n = ((t*L1 + x)*L2 + y)*L3 + z (LGT_Code/README.txt:129-133,
 * init.c:741-829).  Extents are run-time parameters here.
 *
 * Quaternion convention (LGT_Code/include/gauge.h:21-24, :190-198):
 *   U = c0*1 + i(c1 s1 + c2 s2 + c3 s3),  products as gauge.h:83-102.
 */
#include <math.h>
#include <float.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "philox.h"

typedef struct { double c[4]; } qd;

static const double kPi = 3.14159265358979323846;

/* ---------------------------------------------------------------- algebra --- */

/* a*b, gauge.h:83-91 */
static inline qd q_mul(qd a, qd b)
{
    qd r;
    r.c[0] = a.c[0] * b.c[0] - a.c[1] * b.c[1] - a.c[2] * b.c[2] - a.c[3] * b.c[3];
    r.c[1] = a.c[0] * b.c[1] + a.c[1] * b.c[0] - a.c[2] * b.c[3] + a.c[3] * b.c[2];
    r.c[2] = a.c[0] * b.c[2] + a.c[1] * b.c[3] + a.c[2] * b.c[0] - a.c[3] * b.c[1];
    r.c[3] = a.c[0] * b.c[3] - a.c[1] * b.c[2] + a.c[2] * b.c[1] + a.c[3] * b.c[0];
    return r;
}

static inline qd q_dag(qd a)
{
    qd r = {{a.c[0], -a.c[1], -a.c[2], -a.c[3]}};
    return r;
}

/* a*b^dag, gauge.h:94-102 */
static inline qd q_mul_nd(qd a, qd b) { return q_mul(a, q_dag(b)); }
/* a^dag*b */
static inline qd q_mul_dn(qd a, qd b) { return q_mul(q_dag(a), b); }

static inline qd q_add(qd a, qd b)
{
    qd r;
    for (int i = 0; i < 4; ++i) r.c[i] = a.c[i] + b.c[i];
    return r;
}

static inline qd q_scale(qd a, double s)
{
    qd r;
    for (int i = 0; i < 4; ++i) r.c[i] = a.c[i] * s;
    return r;
}

static inline double q_norm(qd a)
{
    return sqrt(fabs(a.c[0] * a.c[0] + a.c[1] * a.c[1] + a.c[2] * a.c[2] + a.c[3] * a.c[3]));
}

/* project_to_su2, LGT_Code/modules/admin/sun_vfunc.c:69-79 */
static inline qd q_project(qd a)
{
    double n = q_norm(a);
    qd r;
    for (int i = 0; i < 4; ++i) r.c[i] = a.c[i] / n;
    return r;
}

static inline qd q_zero(void)
{
    qd r = {{0, 0, 0, 0}};
    return r;
}

static inline qd q_one(void)
{
    qd r = {{1, 0, 0, 0}};
    return r;
}

/* ---------------------------------------------------------------- lattice --- */

typedef struct {
    int L[4];
    uint64_t stride[4];
    uint64_t V;
} lat_t;

static int lat_init(lat_t *g, const int dims[4])
{
    for (int d = 0; d < 4; ++d) {
        if (dims[d] < 2 || (dims[d] & 1)) return -1;
        g->L[d] = dims[d];
    }
    g->stride[3] = 1;
    g->stride[2] = (uint64_t)dims[3];
    g->stride[1] = (uint64_t)dims[2] * dims[3];
    g->stride[0] = (uint64_t)dims[1] * dims[2] * dims[3];
    g->V = g->stride[0] * (uint64_t)dims[0];
    return 0;
}

static inline int coord(const lat_t *g, uint64_t n, int mu)
{
    return (int)((n / g->stride[mu]) % (uint64_t)g->L[mu]);
}

static inline uint64_t up(const lat_t *g, uint64_t n, int mu)
{
    return coord(g, n, mu) == g->L[mu] - 1 ? n - (uint64_t)(g->L[mu] - 1) * g->stride[mu] : n + g->stride[mu];
}

static inline uint64_t dn(const lat_t *g, uint64_t n, int mu)
{
    return coord(g, n, mu) == 0 ? n + (uint64_t)(g->L[mu] - 1) * g->stride[mu] : n - g->stride[mu];
}

static inline int parity(const lat_t *g, uint64_t n)
{
    return (coord(g, n, 0) + coord(g, n, 1) + coord(g, n, 2) + coord(g, n, 3)) & 1;
}

static inline qd ld(const double *U, uint64_t n, int mu)
{
    qd r;
    memcpy(r.c, U + (n * 4 + (uint64_t)mu) * 4, sizeof(r.c));
    return r;
}

static inline void st(double *U, uint64_t n, int mu, qd v)
{
    memcpy(U + (n * 4 + (uint64_t)mu) * 4, v.c, sizeof(v.c));
}

/* ------------------------------------------------------------- observables --- */

/* plaquette(), LGT_Code/modules/obs/plaquette.c:67-100: mean of (1/2) Re tr U_p over 6V plaquettes */
int su2o_plaquette(const int dims[4], const double *U, double *out)
{
    lat_t g;
    if (lat_init(&g, dims)) return -1;
    double sum = 0.0;
    for (uint64_t n = 0; n < g.V; ++n)
        for (int mu = 0; mu < 3; ++mu)
            for (int nu = mu + 1; nu < 4; ++nu) {
                qd p = q_mul(ld(U, n, mu), ld(U, up(&g, n, mu), nu));
                p = q_mul_nd(p, ld(U, up(&g, n, nu), mu));
                p = q_mul_nd(p, ld(U, n, nu));
                sum += 2.0 * p.c[0];
            }
    *out = sum / (2.0 * 6.0 * (double)g.V);
    return 0;
}

/* Sum of the staples closing U_mu(n) into plaquettes, U_mu(n)*A = sum of plaquettes:
 * staples(), LGT_Code/modules/update/metro.c:34-63. */
static qd staple_update(const lat_t *g, const double *U, uint64_t n, int mu)
{
    qd a = q_zero();
    uint64_t nmu = up(g, n, mu);
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu) continue;
        /* U_nu(n+mu) U_mu(n+nu)^dag U_nu(n)^dag */
        qd s = q_mul_nd(ld(U, nmu, nu), ld(U, up(g, n, nu), mu));
        a = q_add(a, q_mul_nd(s, ld(U, n, nu)));
        /* U_nu(n-nu+mu)^dag U_mu(n-nu)^dag U_nu(n-nu) */
        uint64_t m = dn(g, n, nu);
        qd t = q_mul_nd(q_dag(ld(U, up(g, m, mu), nu)), ld(U, m, mu));
        a = q_add(a, q_mul(t, ld(U, m, nu)));
    }
    return a;
}

/* Staples of the smearing step, staples_smearing(), LGT_Code/modules/obs/smearing.c:42-71:
 * orientation is the dagger of staple_update(); directions equal to mu or to `skip` excluded. */
static qd staple_ape(const lat_t *g, const double *U, uint64_t n, int mu, int skip)
{
    qd a = q_zero();
    uint64_t nmu = up(g, n, mu);
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu || nu == skip) continue;
        /* U_nu(n) U_mu(n+nu) U_nu(n+mu)^dag */
        qd s = q_mul(ld(U, n, nu), ld(U, up(g, n, nu), mu));
        a = q_add(a, q_mul_nd(s, ld(U, nmu, nu)));
        /* U_nu(n-nu)^dag U_mu(n-nu) U_nu(n-nu+mu) */
        uint64_t m = dn(g, n, nu);
        qd t = q_mul_dn(ld(U, m, nu), ld(U, m, mu));
        a = q_add(a, q_mul(t, ld(U, up(g, m, mu), nu)));
    }
    return a;
}

/* APE smearing, smearing_APE_all/spatial/temporal, LGT_Code/modules/obs/smearing.c:74-168:
 * ns Jacobi steps U <- Proj(U + alpha*S[U_old]), staples from a copy of the field.
 * mode 0 = all (4 links, 6 staples), 1 = spatial (links 1..3, 4 spatial staples),
 * 2 = temporal (link 0, 6 staples). */
int su2o_ape(const int dims[4], double *U, int ns, double alpha, int mode)
{
    lat_t g;
    if (lat_init(&g, dims) || mode < 0 || mode > 2 || ns < 0) return -1;
    size_t bytes = (size_t)g.V * 16 * sizeof(double);
    double *old = (double *)malloc(bytes);
    if (!old) return -2;
    int mu0 = mode == 1 ? 1 : 0, mu1 = mode == 2 ? 0 : 3;
    for (int s = 0; s < ns; ++s) {
        memcpy(old, U, bytes);
        for (uint64_t n = 0; n < g.V; ++n)
            for (int mu = mu0; mu <= mu1; ++mu) {
                int skip = mode == 0 ? mu : 0;
                qd S = staple_ape(&g, old, n, mu, skip);
                st(U, n, mu, q_project(q_add(ld(old, n, mu), q_scale(S, alpha))));
            }
    }
    free(old);
    return 0;
}

/* Product of links along a rectilinear path from n; steps (dir, +-len). */
static qd path_product(const lat_t *g, const double *U, uint64_t *n, const int *dirs, const int *lens, int nseg, qd acc)
{
    for (int s = 0; s < nseg; ++s) {
        int mu = dirs[s], l = lens[s];
        if (l > 0) {
            for (int i = 0; i < l; ++i) {
                acc = q_mul(acc, ld(U, *n, mu));
                *n = up(g, *n, mu);
            }
        } else {
            for (int i = 0; i < -l; ++i) {
                *n = dn(g, *n, mu);
                acc = q_mul_nd(acc, ld(U, *n, mu));
            }
        }
    }
    return acc;
}

/* measureWilsonLoop (explicit-list mode), LGT_Code/modules/obs/wilson.c:21-56, :268-324:
 * W(R,T) = sum over sites and spatial k of Re tr [T links +t, R links +k, T links -t, R links -k]
 * divided by 3*V*2. */
int su2o_wilson(const int dims[4], const double *U, const int *R, const int *T, int nloop, double *w)
{
    lat_t g;
    if (lat_init(&g, dims)) return -1;
    for (int i = 0; i < nloop; ++i) {
        if (R[i] < 0 || T[i] < 0) return -1;
        double sum = 0.0;
        for (uint64_t n = 0; n < g.V; ++n)
            for (int k = 1; k < 4; ++k) {
                int dirs[4] = {0, k, 0, k}, lens[4] = {T[i], R[i], -T[i], -R[i]};
                uint64_t m = n;
                qd p = path_product(&g, U, &m, dirs, lens, 4, q_one());
                sum += 2.0 * p.c[0];
            }
        w[i] = sum / (3.0 * (double)g.V * 2.0);
    }
    return 0;
}

/* Square e x e clover average in plane (a,b), four leaves, computeCloverAverages()
 * LGT_Code/modules/obs/topologicalcharge.c:46-110 (e1 == e2 branch). */
static qd clover_avg(const lat_t *g, const double *U, uint64_t n, int a, int b, int e)
{
    static const int sgn[4][4] = {{+1, +1, -1, -1}, {-1, +1, +1, -1}, {+1, -1, -1, +1}, {-1, -1, +1, +1}};
    qd sum = q_zero();
    for (int leaf = 0; leaf < 4; ++leaf) {
        int dirs[4], lens[4];
        /* leaf 0: +a +b -a -b ; leaf 1: -b +a +b -a ; leaf 2: +b -a -b +a ; leaf 3: -a -b +a +b */
        static const int order[4][4] = {{0, 1, 0, 1}, {1, 0, 1, 0}, {1, 0, 1, 0}, {0, 1, 0, 1}};
        for (int s = 0; s < 4; ++s) {
            dirs[s] = order[leaf][s] == 0 ? a : b;
            lens[s] = sgn[leaf][s] * e;
        }
        uint64_t m = n;
        sum = q_add(sum, path_product(g, U, &m, dirs, lens, 4, q_one()));
    }
    return q_scale(sum, 0.25);
}

/* F_ab: improved clover combination k1 C1 + k2 C2 + k3 C3 (topologicalcharge.c:127),
 * then (F - F^dag)/2 (hermitianTraceless, :112-121). */
static qd field_strength(const lat_t *g, const double *U, uint64_t n, int a, int b)
{
    const double k[3] = {1.5, -0.15, 1.0 / 90.0};
    qd f = q_zero();
    for (int e = 1; e <= 3; ++e) f = q_add(f, q_scale(clover_avg(g, U, n, a, b, e), k[e - 1]));
    f.c[0] = 0.0;
    return f;
}

/* Per-site density 8*[tr F01 F23 + tr F02 F31 + tr F03 F12] (topologicalcharge.c:175-178). */
static double qtop_density(const lat_t *g, const double *U, uint64_t n)
{
    static const int pairs[3][4] = {{0, 1, 2, 3}, {0, 2, 3, 1}, {0, 3, 1, 2}};
    double s = 0.0;
    for (int p = 0; p < 3; ++p) {
        qd f1 = field_strength(g, U, n, pairs[p][0], pairs[p][1]);
        qd f2 = field_strength(g, U, n, pairs[p][2], pairs[p][3]);
        s += 8.0 * (2.0 * q_mul(f1, f2).c[0]);
    }
    return s;
}

/* topologicalCharge(), topologicalcharge.c:164-199: Q = sum_n density / (32 pi^2).
 * sum_abs (optional) returns sum_n |density| / (32 pi^2), the condition scale of Q. */
int su2o_qtop(const int dims[4], const double *U, double *q, double *sum_abs)
{
    lat_t g;
    if (lat_init(&g, dims)) return -1;
    double s = 0.0, sa = 0.0;
    for (uint64_t n = 0; n < g.V; ++n) {
        double d = qtop_density(&g, U, n);
        s += d;
        sa += fabs(d);
    }
    *q = s / (32.0 * kPi * kPi);
    if (sum_abs) *sum_abs = sa / (32.0 * kPi * kPi);
    return 0;
}

/* Q after ns APE_all steps of parameter alpha, on a copy of U (the adjoint's forward map). */
int su2o_ape_qtop(const int dims[4], const double *U, int ns, double alpha, double *q)
{
    lat_t g;
    if (lat_init(&g, dims)) return -1;
    size_t bytes = (size_t)g.V * 16 * sizeof(double);
    double *W = (double *)malloc(bytes);
    if (!W) return -2;
    memcpy(W, U, bytes);
    int rc = su2o_ape(dims, W, ns, alpha, 0);
    if (!rc) rc = su2o_qtop(dims, W, q, NULL);
    free(W);
    return rc;
}

/* --------------------------------------------------------------- updates --- */

void su2o_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    philox4x32_10(ctr, key, out);
}

/* su2RandomMatrix formula (LGT_Code/modules/random/random_su3.c:141-155) on uniforms r[3]. */
static qd ref_random_link(const double r[3])
{
    qd u;
    double twopi = 2.0 * kPi;
    u.c[0] = 1 - 2. * r[0];
    u.c[1] = 1 - 2. * r[1];
    double zw = sqrt(1. - u.c[1] * u.c[1]);
    u.c[2] = zw * cos(twopi * r[2]);
    u.c[3] = zw * sin(twopi * r[2]);
    zw = sqrt(1. - u.c[0] * u.c[0]);
    u.c[1] *= zw;
    u.c[2] *= zw;
    u.c[3] *= zw;
    return u;
}

/* Start configurations (initGaugeField, LGT_Code/modules/admin/init.c:831-869):
 * mode 0 cold (unit links), 1 haar (4 Box-Muller normals, normalised), 2 ref (su2RandomMatrix). */
int su2o_start(const int dims[4], double *U, int mode, uint64_t seed, uint32_t replica)
{
    lat_t g;
    if (lat_init(&g, dims) || mode < 0 || mode > 2) return -1;
    for (uint64_t n = 0; n < g.V; ++n)
        for (int mu = 0; mu < 4; ++mu) {
            qd u = q_one();
            if (mode != 0) {
                uint32_t w[4];
                su2_philox_link(seed, (uint32_t)n, 0, (uint32_t)mu, 0, 0, SU2_STREAM_INIT, replica, w);
                double r[4];
                for (int i = 0; i < 4; ++i) r[i] = philox_u01_f64(w[i]);
                if (mode == 2) {
                    u = ref_random_link(r);
                } else {
                    double twopi = 2.0 * kPi;
                    double ra = sqrt(-2.0 * log(r[0])), rb = sqrt(-2.0 * log(r[2]));
                    u.c[0] = ra * cos(twopi * r[1]);
                    u.c[1] = ra * sin(twopi * r[1]);
                    u.c[2] = rb * cos(twopi * r[3]);
                    u.c[3] = rb * sin(twopi * r[3]);
                    u = q_project(u);
                }
            }
            st(U, n, mu, u);
        }
    return 0;
}

/* One link of the Kennedy-Pendleton heatbath: localHeatbathUpdate() and
 * generateSU2InHeatbath_Improved(), LGT_Code/modules/update/heatbath.c:76-149,
 * with the uniforms drawn from the Philox stream of this link.  Returns 1/trials
 * (0 for the zero-staple fallback), as the reference does. */
static double hb_link_v(const lat_t *g, double *U, uint64_t n, int mu, double beta, uint64_t seed, uint32_t sweep,
                        uint32_t replica, uint32_t draw_base)
{
    qd A = staple_update(g, U, n, mu);
    double k = q_norm(A);
    uint32_t w[4];
    if (k <= DBL_EPSILON) {
        su2_philox_link(seed, (uint32_t)n, sweep, (uint32_t)mu, draw_base | 1u, 1, SU2_STREAM_UPDATE, replica, w);
        double r[3] = {philox_u01_f64(w[0]), philox_u01_f64(w[1]), philox_u01_f64(w[2])};
        st(U, n, mu, q_project(ref_random_link(r)));
        return 0.0;
    }
    qd V;
    for (int i = 0; i < 4; ++i) V.c[i] = A.c[i] / k; /* su2_dble_div, heatbath.c:140 */
    double alpha = k * beta, delta;
    uint32_t trial = 0;
    for (;;) {
        su2_philox_link(seed, (uint32_t)n, sweep, (uint32_t)mu, draw_base | trial, 0, SU2_STREAM_UPDATE, replica, w);
        trial++;
        double u0 = philox_u01_f64(w[0]), u1 = philox_u01_f64(w[1]);
        double u2 = philox_u01_f64(w[2]), u3 = philox_u01_f64(w[3]);
        double X1 = -log(u0) / alpha, X2 = -log(u1) / alpha;
        double c = cos(2.0 * kPi * u2);
        delta = X2 + X1 * (c * c);
        if (u3 * u3 <= 1.0 - 0.5 * delta) break;
    }
    su2_philox_link(seed, (uint32_t)n, sweep, (uint32_t)mu, draw_base, 1, SU2_STREAM_UPDATE, replica, w);
    double phi = 2.0 * kPi * philox_u01_f64(w[0]);
    double theta = acos(1.0 - 2.0 * philox_u01_f64(w[1]));
    qd X;
    X.c[0] = 1.0 - delta;
    double len = sqrt(1.0 - X.c[0] * X.c[0]);
    X.c[1] = len * sin(theta) * cos(phi);
    X.c[2] = len * sin(theta) * sin(phi);
    X.c[3] = len * cos(theta);
    st(U, n, mu, q_project(q_mul_nd(X, V)));
    return 1.0 / (double)trial;
}

static double hb_link(const lat_t *g, double *U, uint64_t n, int mu, double beta, uint64_t seed, uint32_t sweep,
                      uint32_t replica)
{
    return hb_link_v(g, U, n, mu, beta, seed, sweep, replica, 0u);
}

/* localMetropolisUpdate(n, dir, m) (LGT_Code/modules/update/metro.c:78-109) on Philox draws: hit i
 * takes one block w of stream SU2_STREAM_METRO with draw index i; w[0..2] are the three uniforms of
 * proposeNewLink (X_j = 1 - 2 r_j, metro.c:65-76), w[3] the acceptance uniform.  The proposal is
 * expx(eps, X, u) (exp_fct.c:137-151): U' = E U with E = ((1 - z), eps X) / (1 + z),
 * z = eps^2 |X|^2 / 4.  Returns the number of accepted hits. */
static int metro_link(const lat_t *g, double *U, uint64_t n, int mu, double beta, double eps, int hits,
                      uint64_t seed, uint32_t sweep, uint32_t replica)
{
    const qd stap = staple_update(g, U, n, mu);
    qd u = ld(U, n, mu);
    int iac = 0;
    for (int i = 0; i < hits; ++i) {
        const double lpl_old = 2.0 * q_mul(u, stap).c[0];
        uint32_t w[4];
        su2_philox_link(seed, (uint32_t)n, sweep, (uint32_t)mu, (uint32_t)i, 0, SU2_STREAM_METRO, replica, w);
        double X[3];
        for (int j = 0; j < 3; ++j) X[j] = 1.0 - 2.0 * philox_u01_f64(w[j]);
        double zw = eps * eps * (X[0] * X[0] + X[1] * X[1] + X[2] * X[2]) / 4.0;
        qd e;
        e.c[0] = 1.0 - zw;
        zw = 1.0 / (1.0 + zw);
        e.c[0] *= zw;
        for (int j = 0; j < 3; ++j) e.c[j + 1] = zw * eps * X[j];
        const qd prop = q_mul(e, u);
        const double lpl = 2.0 * q_mul(prop, stap).c[0];
        if (philox_u01_f64(w[3]) <= exp(beta * (lpl - lpl_old) / 2.0)) {
            u = prop;
            iac++;
        }
    }
    st(U, n, mu, q_project(u));
    return iac;
}

/* Times a site is drawn when V sites are drawn with replacement (the random sweep of
 * gaugefieldUpdate, update.c:126-136): Binomial(V, 1/V) by inverse CDF on one uniform. */
static int visit_count(uint32_t w, uint64_t V)
{
    const double u = philox_u01_f64(w), v = (double)V;
    const double p0 = exp(v * log1p(-1.0 / v));
    double p = p0, c = p0;
    int k = 0;
    while (u > c && k < 32) {
        p *= (v - k) / ((k + 1) * (v - 1.0));
        c += p;
        ++k;
    }
    return k;
}

/* Overrelaxation (no reference counterpart): U' = W^dag U^dag W^dag with W = A/|A|,
 * which keeps Re tr(U A) and is an involution. */
static void or_link(const lat_t *g, double *U, uint64_t n, int mu)
{
    qd A = staple_update(g, U, n, mu);
    double k = q_norm(A);
    if (k <= DBL_EPSILON) return;
    qd W = q_scale(A, 1.0 / k);
    qd Wd = q_dag(W);
    qd u = q_mul(q_mul(Wd, q_dag(ld(U, n, mu))), Wd);
    st(U, n, mu, q_project(u));
}

/* One checkerboard sweep: for mu = 0..3, parity 0 then 1, every link U_mu(n) of that parity.
 * kind 0 = heatbath with sweep index `sweep`, kind 1 = overrelaxation. acc gets mean 1/trials. */
int su2o_sweep(const int dims[4], double *U, int kind, double beta, uint64_t seed, uint32_t sweep, uint32_t replica,
               double *acc)
{
    lat_t g;
    if (lat_init(&g, dims)) return -1;
    double a = 0.0;
    for (int mu = 0; mu < 4; ++mu)
        for (int p = 0; p < 2; ++p)
            for (uint64_t n = 0; n < g.V; ++n) {
                if (parity(&g, n) != p) continue;
                if (kind == 0)
                    a += hb_link(&g, U, n, mu, beta, seed, sweep, replica);
                else
                    or_link(&g, U, n, mu);
            }
    if (acc) *acc = a / (4.0 * (double)g.V);
    return 0;
}

/* Heatbath of the links of sites [n0, n0 + count), all four directions, site-major: the loop body
 * of gaugefieldUpdate (LGT_Code/modules/update/update.c:118-163) on a bounded slice, used to time
 * the CPU port.  acc gets the sum of 1/trials. */
int su2o_hb_slice(const int dims[4], double *U, double beta, uint64_t seed, uint32_t sweep, uint64_t n0,
                  uint64_t count, double *acc)
{
    lat_t g;
    if (lat_init(&g, dims) || n0 + count > g.V) return -1;
    double a = 0.0;
    for (uint64_t n = n0; n < n0 + count; ++n)
        for (int mu = 0; mu < 4; ++mu) a += hb_link(&g, U, n, mu, beta, seed, sweep, 0);
    if (acc) *acc = a;
    return 0;
}

/* Re tr(U_mu(n) A_mu(n)) summed over all links: the local action kept by overrelaxation. */
int su2o_link_action(const int dims[4], const double *U, double *out)
{
    lat_t g;
    if (lat_init(&g, dims)) return -1;
    double s = 0.0;
    for (uint64_t n = 0; n < g.V; ++n)
        for (int mu = 0; mu < 4; ++mu) s += 2.0 * q_mul(ld(U, n, mu), staple_update(&g, U, n, mu)).c[0];
    *out = s;
    return 0;
}

/* Kennedy-Pendleton sampler alone: x0 of n draws at fixed alpha with Philox stream (seed, draw index). */
int su2o_kp_samples(double alpha, uint64_t seed, uint64_t n, double *x0)
{
    for (uint64_t i = 0; i < n; ++i) {
        uint32_t trial = 0, w[4];
        double delta;
        for (;;) {
            su2_philox_link(seed, (uint32_t)i, (uint32_t)(i >> 32), 0, trial, 0, SU2_STREAM_UPDATE, 0, w);
            trial++;
            double X1 = -log(philox_u01_f64(w[0])) / alpha, X2 = -log(philox_u01_f64(w[1])) / alpha;
            double c = cos(2.0 * kPi * philox_u01_f64(w[2]));
            delta = X2 + X1 * (c * c);
            double u3 = philox_u01_f64(w[3]);
            if (u3 * u3 <= 1.0 - 0.5 * delta) break;
        }
        x0[i] = 1.0 - delta;
    }
    return 0;
}

/* ------------------------------------------------------------- reflection --- */

/* readConfigForThermalisation (LGT_Code/modules/io/config_IO.c:348-535): the field of extents
 * dims is filled from one of extents dims/2 (`small`, same host layout) by 2^4 mirror images.
 * Image k mirrors direction j when bit j of k is set (config_IO.c:448-456).  For small site c,
 * link direction mu and image k the target coordinate along j is (config_IO.c:488-507)
 *   L_j - c_j - 1                     mirrored, j == mu,
 *   c_j == 0 ? L_j / 2 : L_j - c_j    mirrored, j != mu,
 *   c_j                               not mirrored,
 * and the stored link is U^dag when mu is mirrored (config_IO.c:510-517). */
int su2o_reflect(const int dims[4], const double *small, double *U)
{
    lat_t g;
    if (lat_init(&g, dims)) return -1;
    int hl[4];
    for (int j = 0; j < 4; ++j) {
        if (dims[j] % 2) return -1;
        hl[j] = dims[j] / 2;
    }
    const uint64_t vsmall = g.V / 16;
    for (uint64_t in = 0; in < vsmall; ++in) {
        int c[4];
        uint64_t rem = in;
        for (int j = 3; j >= 0; --j) {
            c[j] = (int)(rem % (uint64_t)hl[j]);
            rem /= (uint64_t)hl[j];
        }
        for (int mu = 0; mu < 4; ++mu) {
            const qd u = ld(small, in, mu), ud = q_dag(u);
            for (int k = 0; k < 16; ++k) {
                uint64_t n = 0;
                for (int j = 0; j < 4; ++j) {
                    int x = c[j];
                    if ((k >> j) & 1) x = (j == mu) ? dims[j] - c[j] - 1 : (c[j] == 0 ? hl[j] : dims[j] - c[j]);
                    n = n * (uint64_t)dims[j] + (uint64_t)x;
                }
                st(U, n, mu, ((k >> mu) & 1) ? ud : u);
            }
        }
    }
    return 0;
}

/* One sweep of gaugefieldUpdate(iup, 1, utype, stype) (update.c:102-175) in checkerboard order,
 * as the library runs it: utype 1 heatbath / 0 Metropolis (`hits` hits per visit, step eps);
 * stype 0 every link once / 1 a Binomial(V, 1/V) number of visits per site (stream
 * SU2_STREAM_VISIT, one count per site and sweep).  acc gets the mean acceptance per link visit
 * over 4 V expected visits. */
int su2o_visit_sweep(const int dims[4], double *U, int utype, int stype, double beta, double eps, int hits,
                     uint64_t seed, uint32_t sweep, uint32_t replica, double *acc)
{
    lat_t g;
    if (lat_init(&g, dims)) return -1;
    double a = 0.0;
    for (int mu = 0; mu < 4; ++mu)
        for (int p = 0; p < 2; ++p)
            for (uint64_t n = 0; n < g.V; ++n) {
                if (parity(&g, n) != p) continue;
                int visits = 1;
                if (stype == 1) {
                    uint32_t w[4];
                    su2_philox_link(seed, (uint32_t)n, sweep, 0, 0, 0, SU2_STREAM_VISIT, replica, w);
                    visits = visit_count(w[0], g.V);
                }
                if (utype == 1) {
                    for (int v = 0; v < visits; ++v)
                        a += hb_link_v(&g, U, n, mu, beta, seed, sweep, replica, (uint32_t)v << SU2_VISIT_SHIFT);
                } else if (visits > 0) {
                    a += (double)metro_link(&g, U, n, mu, beta, eps, visits * hits, seed, sweep, replica) / hits;
                }
            }
    if (acc) *acc = a / (4.0 * (double)g.V);
    return 0;
}

/* ------------------------------------------------------------- statistics --- */

/* LGT_Code/Autocorrelation/t_int.c:24-74 for one series x[i * stride], i < n: out = {mean,
 * integrated autocorrelation time (integratedAutocorrelationTime, :44-55), naive error (:58-60),
 * error = sqrt(2 tau) naive (:71)}; returns 1 when ceil(100 tau) <= n (:65-69), else 0.  The sums
 * run in the reference's order. */
static double ts_avg(const double *x, int64_t stride, int64_t a, int64_t b)
{
    double s = 0.0;
    for (int64_t i = a; i < b; ++i) s += x[i * stride];
    return s / (double)(b - a);
}

static double ts_gamma(const double *x, int64_t stride, int64_t n, int64_t k)
{
    const double a0 = ts_avg(x, stride, 0, n - k), ak = ts_avg(x, stride, k, n);
    double c = 0.0;
    for (int64_t i = 0; i < n - k; ++i) c += (x[i * stride] - a0) * (x[(i + k) * stride] - ak);
    return c / (double)(n - k);
}

int su2o_tau_int(const double *x, int64_t n, int64_t stride, double out[4])
{
    const double g0 = ts_gamma(x, stride, n, 0);
    double t = 0.5 * g0;
    for (int64_t k = 1; k < n; ++k) {
        const double gk = ts_gamma(x, stride, n, k);
        if (gk < 0.0) break;
        t += gk;
    }
    const double tau = t / g0, naive = sqrt(g0 / (double)(n - 1));
    out[0] = ts_avg(x, stride, 0, n);
    out[1] = tau;
    out[2] = naive;
    out[3] = sqrt(2.0 * tau) * naive;
    return (int64_t)ceil(100.0 * tau) <= n;
}

/* The jackknife effective potential of Analysis/static potential/static_potential.py:80-146.
 * w[c][r][t] (n_conf x n_r x n_t) are W(R_r, T_t) per configuration.  With B = n_bins blocks of
 * L = n_conf / B configurations (block k = [kL, (k+1)L); the n_conf - B L last ones are never
 * left out):
 *   Wbar, Wbar_k       means over all configurations and over all but block k (:80-86);
 *   V_eff(r,t)         log(Wbar(t) / Wbar(t+1)) and V_eff_k likewise (:90-97);
 *   err(r,t)           sqrt((B-1)/B sum_k (V_eff_k - V_eff)^2) (:100-107);
 *   veff(r,t)          V_eff - (B-1)(mean_k V_eff_k - V_eff) (bias corrected, :110-113);
 *   fit_k(r)           sum_t V_eff_k / err^2 / sum_t 1/err^2 over t in [t0(r), t1(r)) (:28-42, :117-127);
 *   v(r)               the same fit of the corrected veff (:129-132);
 *   v_err(r)           sqrt((B-1)/B sum_k (fit_k - v)^2) (:135-141);
 *   v(r)               corrected: v - (B-1)(mean_k fit_k - v) (:143-145).
 * veff, veff_err: n_r x (n_t - 1).  Sums run in index order. */
int su2o_veff(const double *w, int n_conf, int n_r, int n_t, int n_bins, const int *t0, const int *t1, double *veff,
              double *veff_err, double *v, double *v_err)
{
    const int B = n_bins, L = n_conf / B, nt1 = n_t - 1;
    if (B < 2 || L < 1 || n_t < 2) return -1;
    double *wbar = malloc(sizeof(double) * n_r * n_t * (B + 1));
    double *vj = malloc(sizeof(double) * n_r * nt1 * B);
    if (!wbar || !vj) return -1;
    for (int r = 0; r < n_r; ++r)
        for (int t = 0; t < n_t; ++t) {
            double all = 0.0;
            for (int c = 0; c < n_conf; ++c) all += w[((size_t)c * n_r + r) * n_t + t];
            double *wb = wbar + ((size_t)r * n_t + t) * (B + 1);
            wb[0] = all / n_conf;
            for (int k = 0; k < B; ++k) {
                double blk = 0.0;
                for (int c = k * L; c < (k + 1) * L; ++c) blk += w[((size_t)c * n_r + r) * n_t + t];
                wb[1 + k] = (all - blk) / (n_conf - L);
            }
        }
    for (int r = 0; r < n_r; ++r)
        for (int t = 0; t < nt1; ++t) {
            const double *a = wbar + ((size_t)r * n_t + t) * (B + 1), *b = a + (B + 1);
            const double full = log(a[0] / b[0]);
            double s2 = 0.0, sm = 0.0;
            for (int k = 0; k < B; ++k) {
                const double e = log(a[1 + k] / b[1 + k]);
                vj[((size_t)r * nt1 + t) * B + k] = e;
                s2 += (e - full) * (e - full);
                sm += e;
            }
            veff_err[(size_t)r * nt1 + t] = sqrt((double)(B - 1) / B * s2);
            veff[(size_t)r * nt1 + t] = full - (B - 1) * (sm / B - full);
        }
    for (int r = 0; r < n_r; ++r) {
        const double *ve = veff + (size_t)r * nt1, *er = veff_err + (size_t)r * nt1;
        double sig = 0.0;
        for (int t = t0[r]; t < t1[r]; ++t) sig += 1.0 / (er[t] * er[t]);
        double a = 0.0;
        for (int t = t0[r]; t < t1[r]; ++t) a += ve[t] / (sig * er[t] * er[t]);
        double s2 = 0.0, sm = 0.0;
        for (int k = 0; k < B; ++k) {
            double f = 0.0;
            for (int t = t0[r]; t < t1[r]; ++t) f += vj[((size_t)r * nt1 + t) * B + k] / (sig * er[t] * er[t]);
            s2 += (f - a) * (f - a);
            sm += f;
        }
        v_err[r] = sqrt((double)(B - 1) / B * s2);
        v[r] = a - (B - 1) * (sm / B - a);
    }
    free(wbar);
    free(vj);
    return 0;
}
