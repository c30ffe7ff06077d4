/*
 * ref_harness.c -- command-line harness around the reference's own C routines.
 *
 * ORACLE / TEST INFRASTRUCTURE ONLY.  It is compiled by oracle/build_ref.sh
 * together with the reference's module sources, read in place from the
 * reference tree (LGT_Code/modules/...), into oracle/_ref/<dims>/.  Nothing of
 * the product links it; tests, the golden-fixture generator and bench.py's
 * CPU-baseline leg run it as a checker / baseline.
 *
 * It replaces the reference's drivers (LGT_Code/main/qcd.c, main_meas/meas.c,
 * main_qtop/qtop.c) by one binary whose sub-commands call the same library
 * functions with explicit parameters, and prints results as
 *     RESULT <key> <values...>      with %.17g
 * so that a Python test can parse them.  Two binaries are built per lattice
 * size: `harness` (real RANLUX, LGT_Code/modules/random/ranlxd.c) and
 * `harness_inj` (oracle/inject_ranlxd.c: Philox uniforms keyed by link).
 *
 * Set-up the reference's drivers do and that is mirrored here:
 *  - PI = 2 asin(1) and initTwoPi()  (LGT_Code/modules/admin/init.c:56-66;
 *    initProgram itself is not called because it validates run parameters
 *    this harness does not use),
 *  - LOG_FILE set (logging() has no NULL check, LGT_Code/modules/io/IO_utils.c:47-58),
 *  - initArrayOfNeighbours() + initGaugeField() (init.c:741-869).
 */
#define MAIN_C

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "ranlxd.h"
#include "headers.h"
#include "modules.h"

extern void initTwoPi(void);
extern double getTime(void);
extern void project_gfield_to_sun(sun_mat *u[VOL][DIM]);

#ifdef SU2_INJECT
extern void inject_set_seed(uint64_t seed);
extern void inject_set_link(uint32_t site, uint32_t dir, uint32_t sweep);
extern void inject_begin_init(void);
extern void inject_end_init(void);
extern void inject_set_metro(int on);
#endif

static void die(const char *msg)
{
    fprintf(stderr, "ref_harness: %s\n", msg);
    exit(2);
}

static void setup(int start)
{
    const char *log = getenv("SU2_HARNESS_LOG");
    snprintf(LOG_FILE, sizeof(LOG_FILE), "%s", log ? log : "/dev/null");
    PI = 2.0 * asin(1.0);
    initTwoPi();
    initArrayOfNeighbours();
    initGaugeField(start);
}

static void print_dims(void)
{
    printf("RESULT dims %lu %lu %lu %lu\n", (unsigned long)LENGT, (unsigned long)LENGS1,
           (unsigned long)LENGS2, (unsigned long)LENGS3);
}

static int site_parity(uint64_t n)
{
    int s = 0;
    for (int d = 0; d < DIM; d++) {
        s += (int)(n / (uint64_t)latParams.volumeFactor[d]);
        n %= (uint64_t)latParams.volumeFactor[d];
    }
    return s & 1;
}

static int parse_list(const char *s, int *out, int maxn)
{
    int n = 0;
    char *buf = strdup(s), *tok, *save = NULL;
    for (tok = strtok_r(buf, ",", &save); tok && n < maxn; tok = strtok_r(NULL, ",", &save))
        out[n++] = atoi(tok);
    free(buf);
    return n;
}

static void load_or_start(const char *what)
{
    if (strcmp(what, "cold") == 0)
        setup(0);
    else if (strcmp(what, "hot") == 0)
        setup(1);
    else {
        setup(0);
        readConfig((char *)what);
    }
}

int main(int argc, char *argv[])
{
    if (argc < 2) die("usage: harness <cmd> ...");
    const char *cmd = argv[1];

    if (strcmp(cmd, "dims") == 0) {
        print_dims();
        return 0;
    }

    /* gen <start 0|1> <seed> <beta> <nsweeps> <out.cfg>: qcd.c:54-74 without the file cadence */
    if (strcmp(cmd, "gen") == 0) {
        if (argc != 7) die("gen <start> <seed> <beta> <nsweeps> <out>");
        int start = atoi(argv[2]), seed = atoi(argv[3]), nsw = atoi(argv[5]);
        runParams.beta = atof(argv[4]);
        rlxd_init(2, seed);
        setup(start);
        for (int n = 0; n < nsw; n++) {
            gaugefieldUpdate(n + 1, 1, SIM_TYPE, SWEEP_TYPE);
            printf("RESULT plaq %d %.17g\n", n + 1, plaquette());
        }
        writeConfig(argv[6]);
        return 0;
    }

    /* genm <start> <seed> <beta> <eps> <utype> <stype> <nsweeps>: the qcd.c loop with any of the
     * reference's update algorithms (utype 0 Metropolis, 1 heatbath) and sweep orders (stype 0
     * sequential, 1 random sites), update.c:102-175, plaquette after every sweep */
    if (strcmp(cmd, "genm") == 0) {
        if (argc != 9) die("genm <start> <seed> <beta> <eps> <utype> <stype> <nsweeps>");
        int start = atoi(argv[2]), seed = atoi(argv[3]), utype = atoi(argv[6]), stype = atoi(argv[7]);
        int nsw = atoi(argv[8]);
        runParams.beta = atof(argv[4]);
        runParams.eps = atof(argv[5]);
        rlxd_init(2, seed);
        setup(start);
        for (int n = 0; n < nsw; n++) {
            gaugefieldUpdate(n + 1, 1, utype, stype);
            printf("RESULT plaq %d %.17g\n", n + 1, plaquette());
        }
        return 0;
    }

    /* genw <start> <seed> <beta> <nsweeps> <every> <R,..> <T,..>: the qcd.c loop (heatbath sweep +
     * plaquette per sweep) with measureWilsonLoop every `every` sweeps (the meas.c measurement) */
    if (strcmp(cmd, "genw") == 0) {
        if (argc != 9) die("genw <start> <seed> <beta> <nsweeps> <every> <R,..> <T,..>");
        int start = atoi(argv[2]), seed = atoi(argv[3]), nsw = atoi(argv[5]), every = atoi(argv[6]);
        static int R[256], T[256];
        int nr = parse_list(argv[7], R, 256), nt = parse_list(argv[8], T, 256), tmax = 0;
        if (nr != nt || every <= 0) die("bad W list or cadence");
        for (int i = 0; i < nt; i++) tmax = T[i] > tmax ? T[i] : tmax;
        measParams.mwil_mode = nr;
        measParams.rExtents = R;
        measParams.tExtents = T;
        measParams.tf = tmax;
        runParams.beta = atof(argv[4]);
        rlxd_init(2, seed);
        setup(start);
        double w[256];
        for (int n = 0; n < nsw; n++) {
            gaugefieldUpdate(n + 1, 1, SIM_TYPE, SWEEP_TYPE);
            printf("RESULT plaq %d %.17g\n", n + 1, plaquette());
            if ((n + 1) % every == 0) {
                measureWilsonLoop(w);
                for (int i = 0; i < nr; i++) printf("RESULT wil %d %d %d %.17g\n", n + 1, R[i], T[i], w[i]);
            }
        }
        return 0;
    }

    /* plaq <cfg> */
    if (strcmp(cmd, "plaq") == 0) {
        if (argc != 3) die("plaq <cfg>");
        load_or_start(argv[2]);
        printf("RESULT plaq %.17g\n", plaquette());
        return 0;
    }

    /* ape <cfg> <all|spatial|temporal> <ns> <alpha> <out.cfg> */
    if (strcmp(cmd, "ape") == 0) {
        if (argc != 7) die("ape <cfg> <mode> <ns> <alpha> <out>");
        load_or_start(argv[2]);
        int ns = atoi(argv[4]);
        double alpha = atof(argv[5]);
        if (strcmp(argv[3], "all") == 0)
            smearing_APE_all(ns, alpha, pu);
        else if (strcmp(argv[3], "spatial") == 0)
            smearing_APE_spatial(ns, alpha, pu);
        else if (strcmp(argv[3], "temporal") == 0)
            smearing_APE_temporal(ns, alpha, pu);
        else
            die("unknown APE mode");
        printf("RESULT plaq %.17g\n", plaquette());
        writeConfig(argv[6]);
        return 0;
    }

    /* wil <cfg> <R list> <T list>: explicit-list mode of measureWilsonLoop (wilson.c:268-324) */
    if (strcmp(cmd, "wil") == 0) {
        if (argc != 5) die("wil <cfg> <R,..> <T,..>");
        load_or_start(argv[2]);
        static int R[4096], T[4096];
        int nr = parse_list(argv[3], R, 4096), nt = parse_list(argv[4], T, 4096);
        if (nr != nt) die("R and T lists differ in length");
        int tmax = 0;
        for (int i = 0; i < nt; i++) tmax = T[i] > tmax ? T[i] : tmax;
        measParams.mwil_mode = nr;
        measParams.rExtents = R;
        measParams.tExtents = T;
        measParams.tf = tmax;
        double *w = malloc(sizeof(double) * nr);
        measureWilsonLoop(w);
        for (int i = 0; i < nr; i++) printf("RESULT wil %d %d %.17g\n", R[i], T[i], w[i]);
        free(w);
        return 0;
    }

    /* qtop <cfg> <alpha> <N1,N2,...>: qtop.c:76-91 -- Q after cumulative APE_all steps */
    if (strcmp(cmd, "qtop") == 0) {
        if (argc != 5) die("qtop <cfg> <alpha> <N,..>");
        load_or_start(argv[2]);
        double alpha = atof(argv[3]);
        static int N[1024];
        int nn = parse_list(argv[4], N, 1024), done = 0;
        for (int i = 0; i < nn; i++) {
            if (N[i] < done) die("qtop N list must be non-decreasing");
            smearing_APE_all(N[i] - done, alpha, pu);
            done = N[i];
            printf("RESULT qtop %d %.17g\n", N[i], topologicalCharge());
        }
        return 0;
    }

    /* bench_sweep <start> <seed> <beta> <nsweeps>: gaugefieldUpdate timed by getTime (update.c:117, :168) */
    if (strcmp(cmd, "bench_sweep") == 0) {
        if (argc != 6) die("bench_sweep <start> <seed> <beta> <nsweeps>");
        int start = atoi(argv[2]), seed = atoi(argv[3]), nsw = atoi(argv[5]);
        runParams.beta = atof(argv[4]);
        rlxd_init(2, seed);
        setup(start);
        print_dims();
        getTime();
        for (int n = 0; n < nsw; n++) {
            double t1 = getTime();
            gaugefieldUpdate(n + 1, 1, SIM_TYPE, SWEEP_TYPE);
            double t2 = getTime();
            printf("RESULT sweep_s %d %.9f\n", n + 1, t2 - t1);
            fflush(stdout);
        }
        return 0;
    }

    /* bench_hb <start> <seed> <beta> <nsites> <reps>: heatbath of the first nsites sites x 4 dirs,
     * the loop body of gaugefieldUpdate (update.c:118-163) on a bounded slice of the lattice */
    if (strcmp(cmd, "bench_hb") == 0) {
        if (argc != 7) die("bench_hb <start> <seed> <beta> <nsites> <reps>");
        int start = atoi(argv[2]), seed = atoi(argv[3]), reps = atoi(argv[6]);
        uint64_t ns = (uint64_t)atoll(argv[5]);
        if (ns > VOL) ns = VOL;
        runParams.beta = atof(argv[4]);
        rlxd_init(2, seed);
        setup(start);
        print_dims();
        getTime();
        for (int r = 0; r < reps; r++) {
            double acc = 0.0;
            double t1 = getTime();
            for (uint64_t n = 0; n < ns; n++)
                for (int dir = 0; dir < DIM; dir++) acc += localHeatbathUpdate(n, dir, 1);
            double t2 = getTime();
            printf("RESULT hb_s %d %lu %.9f %.6f\n", r, (unsigned long)(ns * DIM), t2 - t1,
                   acc / (double)(ns * DIM));
            fflush(stdout);
        }
        return 0;
    }

    /* bench_ape <all|spatial> <alpha> <reps>: one smearing step per rep, hot start */
    if (strcmp(cmd, "bench_ape") == 0) {
        if (argc != 5) die("bench_ape <mode> <alpha> <reps>");
        rlxd_init(2, 1);
        setup(1);
        print_dims();
        double alpha = atof(argv[3]);
        int reps = atoi(argv[4]);
        getTime();
        for (int r = 0; r < reps; r++) {
            double t1 = getTime();
            if (strcmp(argv[2], "all") == 0)
                smearing_APE_all(1, alpha, pu);
            else
                smearing_APE_spatial(1, alpha, pu);
            double t2 = getTime();
            printf("RESULT ape_s %d %.9f\n", r, t2 - t1);
            fflush(stdout);
        }
        return 0;
    }

    /* bench_wil <rmax> <tmax> <reps>: measureWilsonLoop (wilson.c:268-324) over the grid R <= rmax,
     * T <= tmax on a hot start, timed per rep */
    if (strcmp(cmd, "bench_wil") == 0) {
        if (argc != 5) die("bench_wil <rmax> <tmax> <reps>");
        int rmax = atoi(argv[2]), tmax = atoi(argv[3]), reps = atoi(argv[4]), nl = 0;
        static int R[1024], T[1024];
        static double w[1024];
        if (rmax * tmax > 1024) die("too many loops");
        for (int r = 1; r <= rmax; r++)
            for (int t = 1; t <= tmax; t++) {
                R[nl] = r;
                T[nl++] = t;
            }
        measParams.mwil_mode = nl;
        measParams.rExtents = R;
        measParams.tExtents = T;
        measParams.tf = tmax;
        rlxd_init(2, 1);
        setup(1);
        print_dims();
        getTime();
        for (int rp = 0; rp < reps; rp++) {
            double t1 = getTime();
            measureWilsonLoop(w);
            double t2 = getTime();
            printf("RESULT wil_s %d %.9f %.17g\n", rp, t2 - t1, w[0]);
            fflush(stdout);
        }
        return 0;
    }

    /* bench_qtop <reps>: topologicalCharge (topologicalcharge.c:164-199) on a hot start */
    if (strcmp(cmd, "bench_qtop") == 0) {
        if (argc != 3) die("bench_qtop <reps>");
        int reps = atoi(argv[2]);
        rlxd_init(2, 1);
        setup(1);
        print_dims();
        getTime();
        for (int rp = 0; rp < reps; rp++) {
            double t1 = getTime();
            double q = topologicalCharge();
            double t2 = getTime();
            printf("RESULT qtop_s %d %.9f %.17g\n", rp, t2 - t1, q);
            fflush(stdout);
        }
        return 0;
    }

    /* reflect <small.cfg> <out.cfg>: readConfigForThermalisation (config_IO.c:348-535) of a
     * configuration with half this build's extents, then writeConfig of the full lattice */
    if (strcmp(cmd, "reflect") == 0) {
        if (argc != 4) die("reflect <small.cfg> <out>");
        setup(0);
        readConfigForThermalisation(argv[2]);
        printf("RESULT plaq %.17g\n", plaquette());
        writeConfig(argv[3]);
        return 0;
    }

#ifdef SU2_INJECT
    /* hotinj <seed> <out.cfg>: initGaugeField(1) on Philox uniforms (init.c:831-869) */
    if (strcmp(cmd, "hotinj") == 0) {
        if (argc != 4) die("hotinj <seed> <out>");
        inject_set_seed((uint64_t)strtoull(argv[2], NULL, 0));
        inject_begin_init();
        setup(1);
        inject_end_init();
        printf("RESULT plaq %.17g\n", plaquette());
        writeConfig(argv[3]);
        return 0;
    }

    /* hbinj <cfg|cold|hot> <seed> <beta> <sweep0> <nsweeps> <out.cfg>:
     * checkerboard sweeps (dir-major, even then odd parity) of the reference's own
     * localHeatbathUpdate (heatbath.c:124-149) on Philox uniforms, followed by the
     * reference's whole-field reprojection after every sweep (update.c:166). */
    if (strcmp(cmd, "hbinj") == 0) {
        if (argc != 8) die("hbinj <cfg> <seed> <beta> <sweep0> <nsweeps> <out>");
        load_or_start(argv[2]);
        inject_set_seed((uint64_t)strtoull(argv[3], NULL, 0));
        runParams.beta = atof(argv[4]);
        uint32_t sweep0 = (uint32_t)strtoul(argv[5], NULL, 0);
        int nsw = atoi(argv[6]);
        for (int s = 0; s < nsw; s++) {
            double acc = 0.0;
            for (int dir = 0; dir < DIM; dir++)
                for (int p = 0; p < 2; p++)
                    for (uint64_t n = 0; n < VOL; n++) {
                        if (site_parity(n) != p) continue;
                        inject_set_link((uint32_t)n, (uint32_t)dir, sweep0 + (uint32_t)s);
                        acc += localHeatbathUpdate(n, dir, 1);
                    }
            project_gfield_to_sun(pu);
            printf("RESULT hb %d %.17g %.17g\n", s, acc / (double)(VOL * DIM), plaquette());
        }
        writeConfig(argv[7]);
        return 0;
    }
#endif

#ifdef SU2_INJECT
    /* metroinj <cfg|cold|hot> <seed> <beta> <eps> <sweep0> <nsweeps> <out.cfg>: checkerboard sweeps
     * (dir-major, even then odd parity) of the reference's own localMetropolisUpdate(n, dir, 1)
     * (metro.c:78-109) on Philox uniforms, then the whole-field reprojection (update.c:166) */
    if (strcmp(cmd, "metroinj") == 0) {
        if (argc != 9) die("metroinj <cfg> <seed> <beta> <eps> <sweep0> <nsweeps> <out>");
        load_or_start(argv[2]);
        inject_set_seed((uint64_t)strtoull(argv[3], NULL, 0));
        inject_set_metro(1);
        runParams.beta = atof(argv[4]);
        runParams.eps = atof(argv[5]);
        uint32_t sweep0 = (uint32_t)strtoul(argv[6], NULL, 0);
        int nsw = atoi(argv[7]);
        for (int s = 0; s < nsw; s++) {
            double acc = 0.0;
            for (int dir = 0; dir < DIM; dir++)
                for (int p = 0; p < 2; p++)
                    for (uint64_t n = 0; n < VOL; n++) {
                        if (site_parity(n) != p) continue;
                        inject_set_link((uint32_t)n, (uint32_t)dir, sweep0 + (uint32_t)s);
                        acc += localMetropolisUpdate(n, dir, 1);
                    }
            project_gfield_to_sun(pu);
            printf("RESULT metro %d %.17g %.17g\n", s, acc / (double)(VOL * DIM), plaquette());
        }
        writeConfig(argv[8]);
        return 0;
    }
#endif

    die("unknown command");
    return 2;
}
