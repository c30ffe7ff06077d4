/*
 * inject_ranlxd.c -- a drop-in replacement for the reference's RANLUX entry points
 * (LGT_Code/include/ranlxd.h:12-18) that serves Philox uniforms keyed by the link
 * being updated.
 *
 * ORACLE / TEST INFRASTRUCTURE ONLY.  It is linked, instead of
 * LGT_Code/modules/random/ranlxd.c, into the harness binary `harness_inj`, so
 * that the reference's own `localHeatbathUpdate` (LGT_Code/modules/update/
 * heatbath.c:124-149) and `initGaugeField` / `su2RandomMatrix`
 * (LGT_Code/modules/admin/init.c:831-869, LGT_Code/modules/random/
 * random_su3.c:141-155) run on exactly the uniforms the GPU kernels draw.
 *
 * Draw protocol of the reference, per link:
 *   heatbath.c:84    ranlxd(ud, 4)      once per Kennedy-Pendleton trial
 *   heatbath.c:97    ranlxd(angles, 2)  once after acceptance
 *   random_su3.c:145 ranlxd(r, 3)       zero-staple fallback / hot start
 * and, in Metropolis mode (inject_set_metro), per hit of localMetropolisUpdate:
 *   metro.c:71       ranlxd(r, 3)       the proposal: words 0..2 of block (stream METRO, draw = hit)
 *   metro.c:98       ranlxd(r, 1)       the acceptance uniform: word 3 of the same block
 * The reference consumes ud[0], ud[1] as log(1 - ud); the GPU consumes log(u)
 * with u in (0,1).  We therefore hand out 1 - u for those two slots; for
 * u = (w + 0.5) 2^-32 both 1 - u and 1 - (1 - u) are exact in double, so the
 * reference sees bit-identical arguments to log.
 */
#include <stdio.h>
#include <stdlib.h>
#include <stdint.h>
#include "philox.h"

static uint64_t g_seed = 0;
static uint32_t g_site = 0, g_sweep = 0, g_dir = 0, g_replica = 0;
static uint32_t g_trial = 0;
static int g_init_mode = 0;
static int g_metro = 0;
static uint32_t g_metro_word = 0;
static uint64_t g_init_link = 0;

void inject_set_seed(uint64_t seed) { g_seed = seed; }

void inject_set_link(uint32_t site, uint32_t dir, uint32_t sweep)
{
    g_site = site;
    g_dir = dir;
    g_sweep = sweep;
    g_trial = 0;
}

/* Hot start: initGaugeField calls su2RandomMatrix once per link in (site, dir) order. */
void inject_begin_init(void)
{
    g_init_mode = 1;
    g_init_link = 0;
}

void inject_end_init(void) { g_init_mode = 0; }

void inject_set_metro(int on) { g_metro = on; }

void ranlxd(double r[], int n)
{
    uint32_t w[4];
    if (g_init_mode) {
        if (n != 3) {
            fprintf(stderr, "inject_ranlxd: unexpected draw of %d during init\n", n);
            exit(3);
        }
        uint32_t site = (uint32_t)(g_init_link / 4), dir = (uint32_t)(g_init_link % 4);
        su2_philox_link(g_seed, site, 0, dir, 0, 0, SU2_STREAM_INIT, g_replica, w);
        for (int i = 0; i < 3; ++i) r[i] = philox_u01_f64(w[i]);
        g_init_link++;
        return;
    }
    if (g_metro) {
        if (n == 3) {
            su2_philox_link(g_seed, g_site, g_sweep, g_dir, g_trial, 0, SU2_STREAM_METRO, g_replica, w);
            for (int i = 0; i < 3; ++i) r[i] = philox_u01_f64(w[i]);
            g_metro_word = w[3];
        } else if (n == 1) {
            r[0] = philox_u01_f64(g_metro_word);
            g_trial++;
        } else {
            fprintf(stderr, "inject_ranlxd: unexpected draw of %d in Metropolis mode\n", n);
            exit(3);
        }
        return;
    }
    if (n == 4) {
        su2_philox_link(g_seed, g_site, g_sweep, g_dir, g_trial, 0, SU2_STREAM_UPDATE, g_replica, w);
        g_trial++;
        r[0] = 1.0 - philox_u01_f64(w[0]);
        r[1] = 1.0 - philox_u01_f64(w[1]);
        r[2] = philox_u01_f64(w[2]);
        r[3] = philox_u01_f64(w[3]);
    } else if (n == 2) {
        su2_philox_link(g_seed, g_site, g_sweep, g_dir, 0, 1, SU2_STREAM_UPDATE, g_replica, w);
        r[0] = philox_u01_f64(w[0]);
        r[1] = philox_u01_f64(w[1]);
    } else if (n == 3) {
        su2_philox_link(g_seed, g_site, g_sweep, g_dir, 1, 1, SU2_STREAM_UPDATE, g_replica, w);
        for (int i = 0; i < 3; ++i) r[i] = philox_u01_f64(w[i]);
    } else {
        fprintf(stderr, "inject_ranlxd: unexpected draw of %d\n", n);
        exit(3);
    }
}

void rlxd_init(int level, int seed)
{
    (void)level;
    g_seed = (uint64_t)(uint32_t)seed;
}

int rlxd_size(void) { return 0; }
void rlxd_get(int state[]) { (void)state; }
void rlxd_reset(int state[]) { (void)state; }
