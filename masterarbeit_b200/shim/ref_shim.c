/*
 * ref_shim.c -- the reference's update and measurement routines, implemented on libsu2g.
 *
 * The reference (LGT_Code) has no plugin interface: its drivers call global C functions over the
 * global field `pu` (include/headers.h:402).  This file defines those functions with the
 * reference's own signatures (include/modules.h:27-42, :99, :121-123) on top of the C ABI in
 * include/su2g.h.  build_dropin.sh compiles it against the reference's headers (the lattice size
 * is fixed there, include/headers.h:22-25) and links it into the reference's unmodified drivers
 * (main/qcd.c, main_meas/meas.c, main_qtop/qtop.c) in place of the modules update, heatbath,
 * metro, exp_fct, plaquette, smearing, wilson and topologicalcharge.
 *
 * Field residency.  The GPU handle is created on first use with the extents of headers.h and
 * runParams.beta; its Philox key is drawn from the reference's own RANLUX stream (two ranlxd
 * draws after rlxd_init), so a run is a deterministic function of the input file's seed.  The
 * field stays on the device between calls.  `pu` is brought up to date only when reference code
 * reads it directly: readConfig/writeConfig/readConfigForThermalisation and measure2ptFunctions
 * are wrapped (their originals are renamed to ref_* at link time), and everything the reference
 * writes into `pu` through them is uploaded before the next GPU call.
 *
 * Environment: SU2G_PRECISION = fp64 (default) | fp32;  SU2G_OR = overrelaxation sweeps after
 * each heatbath sweep (default 0, as the reference has none);  SU2G_DEVICE = CUDA device.
 *
 * Errors use the reference's convention: error() logs to LOG_FILE and exits
 * (modules/io/IO_utils.c:61-80).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "ranlxd.h"
#include "headers.h"
#include "modules.h"
#include "su2g.h"

extern double getTime(void);
/* the reference's own routines, renamed at link time by build_dropin.sh (objcopy --redefine-sym) */
extern void ref_readConfig(char *);
extern void ref_writeConfig(char *);
extern void ref_readConfigForThermalisation(char *);
extern void ref_measure2ptFunctions(int *, int, int, int *, int *) __attribute__((weak));

enum { HOST_NEWER = 0, DEVICE_NEWER = 1, IN_SYNC = 2 };

static su2g_lattice *g_h = NULL;     /* the field's device copy */
static su2g_lattice *g_chk = NULL;   /* FP64 handle for the I/O plaquette checks in FP32 mode */
static int g_state = HOST_NEWER;
static int g_prec = SU2G_FP64;
static int g_nor = 0;
static int g_io = 0;                 /* > 0 inside a wrapped readConfig / writeConfig */
static double g_plaq = 0.0;          /* plaquette of the device field summed by the last sweep */
static int g_plaq_ok = 0;            /* g_plaq is the current field's (no change since that sweep) */

static void check(int rc, su2g_lattice *h, const char *where)
{
    error(rc != 0, (char *)where, "%s", su2g_last_error(h));
}

static void release(void)
{
    su2g_destroy(g_h);
    su2g_destroy(g_chk);
    g_h = g_chk = NULL;
}

static su2g_params params(int precision)
{
    su2g_params p;
    memset(&p, 0, sizeof(p));
    p.dims[0] = (int32_t)LENGT;
    p.dims[1] = (int32_t)LENGS1;
    p.dims[2] = (int32_t)LENGS2;
    p.dims[3] = (int32_t)LENGS3;
    p.precision = precision;
    p.start = SU2G_START_COLD;
    p.beta = runParams.beta;
    p.device = getenv("SU2G_DEVICE") ? atoi(getenv("SU2G_DEVICE")) : 0;
    return p;
}

static void configure(void)
{
    static int done = 0;
    if (done) return;
    const char *prec = getenv("SU2G_PRECISION");
    g_prec = (prec && strcmp(prec, "fp32") == 0) ? SU2G_FP32 : SU2G_FP64;
    g_nor = getenv("SU2G_OR") ? atoi(getenv("SU2G_OR")) : 0;
    done = 1;
}

static su2g_lattice *handle(void)
{
    if (g_h) return g_h;
    configure();
    su2g_params p = params(g_prec);
    double r[2];
    ranlxd(r, 2);
    p.seed = ((uint64_t)(r[0] * 4294967296.0) << 32) | (uint64_t)(r[1] * 4294967296.0);
    check(su2g_create(&p, &g_h), NULL, "su2g_create [ref_shim.c]");
    atexit(release);
    g_state = HOST_NEWER;
    return g_h;
}

static void to_device(void)
{
    handle();
    if (g_state == HOST_NEWER) {
        check(su2g_upload_aos_f64(g_h, (const double *)pu[0][0]), g_h, "su2g_upload_aos_f64 [ref_shim.c]");
        g_state = IN_SYNC;
        g_plaq_ok = 0;
    }
}

static void to_host(void)
{
    if (g_h && g_state == DEVICE_NEWER) {
        check(su2g_download_aos_f64(g_h, (double *)pu[0][0]), g_h, "su2g_download_aos_f64 [ref_shim.c]");
        g_state = IN_SYNC;
    }
}

/* gaugefieldUpdate, modules/update/update.c:102-175: nup sweeps of the heatbath (utype 1) or of
 * Metropolis with step runParams.eps (utype 0), every link once (stype 0) or random site
 * selection (stype 1); heatbath sequential sweeps are followed by SU2G_OR overrelaxation sweeps
 * each.  Reprojection on every store, the same log lines.  Heatbath sequential sweeps run as
 * su2g_sweep_plaquette, which also sums the plaquette of the new field inside its update passes:
 * the plaquette() that main/qcd.c calls next (qcd.c:55-60) returns it without another kernel. */
void gaugefieldUpdate(int iup, int nup, int utype, int stype)
{
    double acc = 0.0, t1, t2;

    error(utype != 0 && utype != 1, "update [update.c]", "Unknown update type! Only "
          "Metropolis (SIM_TYPE=0) and heatbath (SIM_TYPE=1) implemented!");
    error(stype != 0 && stype != 1, "update [update.c]", "Unknown sweep type! "
          "Only sequential (SWEEP_TYPE=0) and random (SWEEP_TYPE=1) sweeps implemented!");

    to_device();
    check(su2g_set_beta(g_h, runParams.beta), g_h, "su2g_set_beta [ref_shim.c]");
    t1 = getTime();
    g_plaq_ok = 0;
    if (utype == 1 && stype == 0) {
        check(su2g_sweep_plaquette(g_h, nup, 1, g_nor, &g_plaq, &acc), g_h, "su2g_sweep_plaquette [ref_shim.c]");
        g_plaq_ok = 1;
    } else {
        check(su2g_gauge_update(g_h, nup, utype, stype, runParams.eps, 1, &acc), g_h,
              "su2g_gauge_update [ref_shim.c]");
    }
    t2 = getTime();
    g_state = DEVICE_NEWER;

    logging("\nUpdate %d done:\n"
            "(algorithm %d; sweep %d; acc=%.3f)\n"
            "update took %.9f seconds\n",
            iup, utype, stype, acc, t2 - t1);
}

/* plaquette(), modules/obs/plaquette.c:67-100.  Inside readConfig/writeConfig the value is taken
 * in FP64 from the host field, as the file's plaquette check (config_IO.c:611-614) needs. */
double plaquette(void)
{
    double p = 0.0;
    configure();
    if (g_io && g_prec != SU2G_FP64) {
        if (!g_chk) {
            su2g_params q = params(SU2G_FP64);
            check(su2g_create(&q, &g_chk), NULL, "su2g_create [ref_shim.c]");
        }
        check(su2g_upload_aos_f64(g_chk, (const double *)pu[0][0]), g_chk, "su2g_upload_aos_f64 [ref_shim.c]");
        check(su2g_plaquette(g_chk, &p), g_chk, "su2g_plaquette [ref_shim.c]");
        return p;
    }
    if (g_plaq_ok && g_h && g_state == DEVICE_NEWER) return g_plaq;
    to_device();
    check(su2g_plaquette(g_h, &p), g_h, "su2g_plaquette [ref_shim.c]");
    return p;
}

/* gaugeAction, modules/obs/plaquette.c:104-110 */
double gaugeAction(void)
{
    return runParams.beta * NPLAQ * VOL * (1. - plaquette());
}

static void smear(int ns, double sp, sun_mat *u[VOL][DIM], int mode)
{
    error(u != pu, "smearing_APE [ref_shim.c]", "The GPU path smears the global field pu only");
    to_device();
    check(su2g_ape(g_h, ns, sp, mode), g_h, "su2g_ape [ref_shim.c]");
    g_state = DEVICE_NEWER;
    g_plaq_ok = 0;
}

/* smearing_APE_all / _spatial / _temporal, modules/obs/smearing.c:74-168 */
void smearing_APE_all(int ns, double sp, sun_mat *u[VOL][DIM]) { smear(ns, sp, u, SU2G_APE_ALL); }
void smearing_APE_spatial(int ns, double sp, sun_mat *u[VOL][DIM]) { smear(ns, sp, u, SU2G_APE_SPATIAL); }
void smearing_APE_temporal(int ns, double sp, sun_mat *u[VOL][DIM]) { smear(ns, sp, u, SU2G_APE_TEMPORAL); }

/* measureWilsonLoop, modules/obs/wilson.c:268-324: the pair list of measParams, same order. */
void measureWilsonLoop(double *w)
{
    int nloop;
    if (measParams.mwil_mode <= 0) {
        int nt = ((measParams.tf - measParams.ts) / measParams.dt) + 1;
        int nr = ((measParams.rf - measParams.rs) / measParams.dr) + 1;
        nloop = nt * nr;
    } else {
        nloop = measParams.mwil_mode;
    }
    error((uint64_t)(latParams.linearExtent[0] - 1) < (uint64_t)measParams.tf, "meas_wilson",
          "Lattice too small to measure loops!");
    to_device();
    check(su2g_wilson(g_h, measParams.rExtents, measParams.tExtents, nloop, w), g_h, "su2g_wilson [ref_shim.c]");
}

/* topologicalCharge, modules/obs/topologicalcharge.c:164-199 (same log lines).  The normalisation
 * 1/(32 pi^2) uses pi itself, so Q is finite even in drivers that never set the global PI. */
double topologicalCharge(void)
{
    double q = 0.0, t1, t2;
    t1 = getTime();
    logging("calculating topological charge ..\n");
    to_device();
    check(su2g_qtop(g_h, &q, NULL), g_h, "su2g_qtop [ref_shim.c]");
    t2 = getTime();
    logging("measurement done (took %.3e sec)\n", t2 - t1);
    return q;
}

/* readConfig / readConfigForThermalisation / writeConfig (modules/io/config_IO.c): the reference's
 * own code on the host field, with `pu` synchronised around it. */
void readConfig(char *infile)
{
    g_state = HOST_NEWER;
    g_plaq_ok = 0;
    g_io++;
    ref_readConfig(infile);   /* its plaquette check uploads the new field in FP64 mode */
    g_io--;
    if (g_prec != SU2G_FP64 || !g_h) g_state = HOST_NEWER;
}

void readConfigForThermalisation(char *infile)
{
    g_state = HOST_NEWER;
    g_plaq_ok = 0;
    g_io++;
    ref_readConfigForThermalisation(infile);
    g_io--;
    g_state = HOST_NEWER;
}

void writeConfig(char *outfile)
{
    to_host();
    g_io++;
    ref_writeConfig(outfile);
    g_io--;
}

/* The fermion measurements read pu directly (modules/obs/2pt.c:140). */
void measure2ptFunctions(int *source, int stype, int n2pt, int *g1, int *g2)
{
    error(ref_measure2ptFunctions == NULL, "measure2ptFunctions [ref_shim.c]", "2pt module not linked");
    to_host();
    ref_measure2ptFunctions(source, stype, n2pt, g1, g2);
}
