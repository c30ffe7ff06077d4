/*
 * su2g.h -- C ABI of the B200 (sm_100a) SU(2) pure-gauge lattice library (libsu2g.so).
 *
 * The reference (daggerfall247/Masterarbeit, LGT_Code) has no plugin or FFI layer: its
 * update and measurement routines are plain C functions over a global field `pu`
 * (LGT_Code/include/modules.h, LGT_Code/include/headers.h:402).  Each entry point below
 * replaces one of those routines; the comment names the reference interface it stands in
 * for.  The shim masterarbeit_b200/shim/ref_shim.c defines the reference's own symbols on
 * top of these calls, so the reference's drivers (LGT_Code/main/qcd.c, main_meas/meas.c,
 * main_qtop/qtop.c) link against it unchanged.
 *
 * Conventions
 *  - Every call returns an int status: 0 = OK, negative = error (SU2G_E*).  The message of
 *    the last failure on a handle is su2g_last_error(h); failures before a handle exists
 *    (su2g_create) are reported by su2g_last_error(NULL).
 *  - Host arrays are plain C arrays owned by the caller.  The gauge field itself lives in
 *    device memory owned by the handle and stays resident between calls.
 *  - A handle owns one CUDA stream; calls on one handle are ordered on that stream.
 *    Calls that return values to host memory synchronise that stream.  A handle is not
 *    thread-safe; distinct handles may be used from distinct threads.
 *  - Lattice extents dims[4] = (L_t, L_x, L_y, L_z), each even and >= 2 (the reference's
 *    compile-time checks, LGT_Code/include/headers.h:58-69, with L_x,y,z >= 4 there).
 *    Site index n = ((t*L_x + x)*L_y + y)*L_z + z (LGT_Code/modules/admin/init.c:741-829).
 *  - Host field arrays use the reference's layout exactly: the block behind pu[0][0],
 *    double[V][4][4] = site, direction (0 = t), quaternion c0..c3
 *    (LGT_Code/modules/admin/init.c:842-858; file body of config_IO.c:95-105).
 */
#ifndef SU2G_H
#define SU2G_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct su2g_lattice su2g_lattice;

enum su2g_status {
    SU2G_OK = 0,
    SU2G_EINVAL = -1,   /* bad argument */
    SU2G_ENOMEM = -2,   /* device or pinned host allocation failed */
    SU2G_ECUDA = -3,    /* CUDA runtime error */
    SU2G_EDEVICE = -4,  /* a kernel reported a failure through its status word */
    SU2G_ENODEV = -5,   /* no usable sm_100 device */
    SU2G_EFILE = -6     /* a configuration file could not be opened, read or written, or failed a check */
};

enum su2g_precision { SU2G_FP32 = 0, SU2G_FP64 = 1 };

/* Start configurations, initGaugeField (LGT_Code/modules/admin/init.c:831-869):
 * cold = unit links; haar = four normalised N(0,1) draws per link;
 * ref = the reference's su2RandomMatrix formula (LGT_Code/modules/random/random_su3.c:141-155). */
enum su2g_start { SU2G_START_COLD = 0, SU2G_START_HAAR = 1, SU2G_START_REF = 2 };

/* APE variants, smearing_APE_all / _spatial / _temporal (LGT_Code/modules/obs/smearing.c:74-168). */
enum su2g_ape_mode { SU2G_APE_ALL = 0, SU2G_APE_SPATIAL = 1, SU2G_APE_TEMPORAL = 2 };

/* Update kinds for su2g_update_pass. */
enum su2g_update_kind { SU2G_HEATBATH = 0, SU2G_OVERRELAX = 1, SU2G_METROPOLIS = 2 };

typedef struct su2g_params {
    int32_t dims[4];     /* L_t, L_x, L_y, L_z (headers.h:22-25 LENGT, LENGS1-3) */
    int32_t precision;   /* su2g_precision */
    int32_t start;       /* su2g_start */
    double beta;         /* runParams.beta (headers.h:347) */
    uint64_t seed;       /* Philox key (replaces rlxd_init(2, seed), LGT_Code/main/qcd.c:36) */
    uint32_t replica;    /* stream id mixed into every Philox counter (0 for a single lattice) */
    int32_t device;      /* CUDA device ordinal */
} su2g_params;

/* ---- handle lifetime: initArrayOfNeighbours + initGaugeField + releaseGaugeField
 *      (LGT_Code/modules/admin/init.c:741-869, :922-925) */
int su2g_create(const su2g_params *params, su2g_lattice **out);
int su2g_destroy(su2g_lattice *h);
const char *su2g_last_error(const su2g_lattice *h);

/* Re-initialise the field (initGaugeField, init.c:831-869) with a start mode and seed. */
int su2g_start(su2g_lattice *h, int32_t start, uint64_t seed);

/* Lattice facts: dims, precision, volume, heatbath sweeps done (the Philox sweep counter). */
int su2g_info(const su2g_lattice *h, int32_t dims[4], int32_t *precision, int64_t *volume,
              uint32_t *hb_sweeps);
int su2g_set_beta(su2g_lattice *h, double beta);
/* The heatbath sweep counter keys the Philox stream; setting it makes a resume bit-exact. */
int su2g_set_sweep_counter(su2g_lattice *h, uint32_t hb_sweeps);

/* ---- host <-> device field transfer: the pu[0][0] block (readConfig / writeConfig body,
 *      LGT_Code/modules/io/config_IO.c:537-621, :40-117).  links = double[V*16]. */
int su2g_upload_aos_f64(su2g_lattice *h, const double *links);
int su2g_download_aos_f64(su2g_lattice *h, double *links);

/* ---- updates: gaugefieldUpdate(iup, nup, utype=1, stype=0) (LGT_Code/modules/update/update.c:102-175)
 * n_sweeps times: n_hb checkerboard heatbath sweeps (localHeatbathUpdate, heatbath.c:124-149)
 * followed by n_or overrelaxation sweeps (new, no reference counterpart).  Every store is
 * reprojected (replaces project_gfield_to_sun, update.c:166).  If acc_out is not NULL it
 * receives the mean of 1/trials over all heatbath link updates (the `acc=` log value,
 * update.c:169-173) and the call synchronises; otherwise the call only enqueues. */
int su2g_sweep(su2g_lattice *h, int32_t n_sweeps, int32_t n_hb, int32_t n_or, double *acc_out);
/* su2g_sweep followed by plaquette() (plaquette.c:67-100) -- the qcd.c:55-60 loop body -- with the
 * plaquette summed inside the update passes: in the parity-1 passes of mu = 1, 2, 3 of the last
 * sub-sweep, (U'_mu(x) A_low(x)).c0 over the odd sites, A_low the staple terms of the planes
 * (mu, nu < mu), covers all 6V plaquettes of the final field once (each holds one odd-site link of
 * its higher direction, and the plaquette's other links are final by then).  *plaq equals
 * su2g_plaquette of the resulting field to rounding (the terms are summed in another order).  The
 * field and the acceptance equal su2g_sweep's to rounding: the fused passes are separately compiled
 * kernels whose multiply-adds may round differently in the last bit.  Synchronises.  With no
 * sub-sweep, *plaq is su2g_plaquette. */
int su2g_sweep_plaquette(su2g_lattice *h, int32_t n_sweeps, int32_t n_hb, int32_t n_or, double *plaq,
                         double *acc_out);

/* gaugefieldUpdate(iup, nup, utype, stype) with both of the reference's update algorithms and
 * sweep orders (update.c:102-175).  utype 1 = heatbath, 0 = Metropolis: localMetropolisUpdate
 * (metro.c:78-109) with the proposal exp(eps X) U of proposeNewLink / expx (metro.c:65-76,
 * exp_fct.c:137-151), step size eps (runParams.eps) and `hits` hits per visit (the reference's
 * m = 1).  stype 0 = every link once per sweep; stype 1 = random site selection: V sites drawn
 * with replacement (update.c:126-136), i.e. each site visited a Binomial(V, 1/V) number of times,
 * a visit updating the site's four links.  Sweeps run as checkerboard passes, as su2g_sweep; a
 * site's visits follow one another in its links' passes.  If acc_out is not NULL it receives the
 * mean acceptance per link visit (update.c:164-171) and the call synchronises.  utype 1 with
 * stype 0 is su2g_sweep(h, nup, 1, 0, acc_out). */
int su2g_gauge_update(su2g_lattice *h, int32_t nup, int32_t utype, int32_t stype, double eps, int32_t hits,
                      double *acc_out);

/* One checkerboard pass: links of direction mu and site parity `parity`, heatbath or
 * overrelaxation.  For a heatbath pass, `sweep` is the Philox sweep index. */
int su2g_update_pass(su2g_lattice *h, int32_t kind, int32_t mu, int32_t parity, uint32_t sweep);

/* ---- configuration files in the reference's binary format (writeConfig / readConfig,
 * LGT_Code/modules/io/config_IO.c:40-117, :537-621): int32 {4, 2}, int32 {L_t, L_x, L_y, L_z},
 * the double plaquette, then for every site in lexicographic order and every direction the four
 * doubles of the link; little-endian.  The links stream between the file and the device field
 * through pinned double buffers, file I/O overlapping the copies and the layout conversion.
 * su2g_read_config checks the header (dimension 4, SU(2), the handle's extents) and then the
 * plaquette against the file's, |P - P_file| <= sqrt(6 V) DBL_EPSILON as readConfig does (for an
 * FP32 handle, whose links are rounded on the way in, the bound is 1e-5).  plaq_file and plaq
 * (either may be NULL) receive the file's and the computed plaquette.  On SU2G_EFILE the
 * field may hold part of the file. */
int su2g_read_config(su2g_lattice *h, const char *path, double *plaq_file, double *plaq);
/* Writes the field with its plaquette (returned in plaq if not NULL) in the header. */
int su2g_write_config(su2g_lattice *h, const char *path, double *plaq);
/* readConfigForThermalisation (config_IO.c:348-535): the file holds a lattice of half the
 * handle's extents in every direction; the field becomes its 16 mirror images, with the links
 * along a mirrored direction daggered.  Same checks as su2g_read_config (the plaquette of the
 * mirrored lattice equals the file's). */
int su2g_read_config_reflect(su2g_lattice *h, const char *path, double *plaq_file, double *plaq);

/* ---- one configuration's measurement in the meas and qtop drivers
 * (LGT_Code/main_meas/meas.c:93-126, LGT_Code/main_qtop/qtop.c:76-91) as one replayed CUDA graph.
 * Both branches start from a device copy of the handle's field, which is left unchanged:
 *  - charges: q[i] = Q after q_ape[i] APE_all steps of parameter alpha_q (cumulative counts,
 *    ascending; meas.c records one charge after smear_tc steps, qtop.c one per step count);
 *  - loops: w[i] = W(R[i], T[i]) after ns_t temporal steps (alpha_t) and then ns_s spatial steps
 *    (alpha_s), the tSmear / rSmear order of meas.c:106-109.
 * The graph is captured on the first call with a given spec and replayed by later calls with the
 * same spec (a new field read into the handle needs no new capture). */
typedef struct su2g_meas_spec {
    int32_t n_q;            /* charges to record (0: none) */
    const int32_t *q_ape;   /* APE_all step count before each charge */
    double alpha_q;
    int32_t n_w;            /* Wilson loops to record (0: none) */
    const int32_t *R;       /* spatial extents (measParams.rExtents) */
    const int32_t *T;       /* temporal extents (measParams.tExtents), each <= L_t - 1 */
    int32_t ns_t;           /* temporal APE steps before the loops (measParams.ismt) */
    double alpha_t;         /* measParams.smpart */
    int32_t ns_s;           /* spatial APE steps before the loops (measParams.isms) */
    double alpha_s;         /* measParams.smpars */
} su2g_meas_spec;
int su2g_measure(su2g_lattice *h, const su2g_meas_spec *spec, double *q, double *w);
/* Free the measurement graph and its two field copies (also freed by su2g_destroy). */
int su2g_measure_release(su2g_lattice *h);

/* ---- the reference's analysis tools on the device.  Inputs may be host or device memory;
 * outputs are host memory; the calls synchronise `device` and report failures through
 * su2g_last_error(NULL).
 * su2g_stats_tau_int: LGT_Code/Autocorrelation/t_int.c:24-74 for n_series series of length n,
 * element i of series s at data[i * stride_i + s * stride_s]: out[4 s + {0,1,2,3}] = mean,
 * integrated autocorrelation time tau (Gamma(k) with separate window means, summed up to the
 * first negative lag), naive error sqrt(Gamma(0)/(n-1)) and error sqrt(2 tau) x naive; resolved[s]
 * (may be NULL) = 1 when ceil(100 tau) <= n, the tool's condition for a trustworthy tau (t_int.c:65-69).
 * The sums run in the tool's order, so the results equal its arithmetic. */
int su2g_stats_tau_int(const double *data, int64_t n, int32_t n_series, int64_t stride_i, int64_t stride_s,
                       int32_t device, double *out, int32_t *resolved);
/* su2g_stats_veff: the block jackknife of Analysis/static potential/static_potential.py:28-146
 * on w[c][r][t] = W(R_r, T_t) of configuration c (n_conf x n_r x n_t): n_bins blocks of
 * n_conf / n_bins configurations, veff[r][t] = log(W(T_t)/W(T_t+1)) bias corrected and its
 * jackknife error veff_err (n_r x (n_t - 1)), v[r] = the weighted constant fit of veff over
 * t in [t_fit_start[r], t_fit_end[r]) (indices into veff), bias corrected, and its jackknife error. */
int su2g_stats_veff(const double *w, int32_t n_conf, int32_t n_r, int32_t n_t, int32_t n_bins,
                    const int32_t *t_fit_start, const int32_t *t_fit_end, int32_t device, double *veff,
                    double *veff_err, double *v, double *v_err);

/* ---- the driver loop of LGT_Code/main/qcd.c:55-60 (gaugefieldUpdate, then plaquette) as one
 * replayed CUDA graph.  Runs n_blocks blocks of [meas_every x (n_hb heatbath + n_or overrelaxation
 * sweeps), plaquette].  The block is captured on first use and replayed; it is captured again
 * when the block shape, beta, the seed or the field's buffers have changed.  The results equal
 * those of the same su2g_sweep_plaquette sequence bit for bit.  plaq[b] and acc[b] (either
 * may be NULL) receive the plaquette after block b and block b's mean heatbath acceptance. */
int su2g_graph_run(su2g_lattice *h, int32_t n_blocks, int32_t meas_every, int32_t n_hb, int32_t n_or,
                   double *plaq, double *acc);
/* Free the captured block (it is also freed by su2g_destroy). */
int su2g_graph_release(su2g_lattice *h);

/* ---- observables */
/* plaquette() (LGT_Code/modules/obs/plaquette.c:67-100): <(1/2) Re tr U_p> over 6V plaquettes. */
int su2g_plaquette(su2g_lattice *h, double *p);
/* smearing_APE_* (LGT_Code/modules/obs/smearing.c:74-168), in place on the handle's field. */
int su2g_ape(su2g_lattice *h, int32_t ns, double alpha, int32_t mode);
/* measureWilsonLoop (LGT_Code/modules/obs/wilson.c:268-324), explicit pair list:
 * w[i] = W(R[i], T[i]); pairs in any order; the T <= L_t - 1 check of wilson.c:290-291. */
int su2g_wilson(su2g_lattice *h, const int32_t *R, const int32_t *T, int32_t n, double *w);
/* topologicalCharge() (LGT_Code/modules/obs/topologicalcharge.c:164-199); sum_abs (may be NULL)
 * receives sum_x |q(x)|, the scale against which the cancellation in Q is judged. */
int su2g_qtop(su2g_lattice *h, double *q, double *sum_abs);

/* ---- adjoint of the smeared charge (no counterpart in the reference, which has no derivative code):
 * Q(U_N) after n_ape APE_all steps of parameter alpha (smearing_APE_all + topologicalCharge, the
 * qtop.c:76-91 flow), and its vector-Jacobian product with respect to the handle's (unsmeared)
 * field.  grad (may be NULL) receives, per link in the host order double[V][4][3], the su(2)
 * coefficients g of dQ under U -> exp(eps X) U, X = i x.sigma:  dQ = eps * sum g.x + O(eps^2).
 * The smeared levels are kept every `ckpt` steps (0 = ceil(sqrt(n_ape))) and recomputed in
 * between.  The handle's field is not modified.  The scratch (su2g_vjp_plan) comes from a memory
 * pool of the handle that keeps it for later calls until su2g_destroy. */
int su2g_ape_qtop_vjp(su2g_lattice *h, int32_t n_ape, double alpha, int32_t ckpt, double *q, double *grad);
/* One step along su(2) coefficients, the step an optimiser takes along the VJP's gradient (no
 * counterpart in the reference): every link U -> exp(eps X) U with X = i x.sigma, x = three
 * doubles per link in the gradient's layout double[V][4][3] (host memory), exp computed exactly
 * (cos(eps|x|), sin(eps|x|) x/|x|).  With eps = +-e it is the perturbation of a central finite
 * difference along x.  Synchronises. */
int su2g_tangent_step(su2g_lattice *h, const double *x, double eps);
/* Levels the VJP keeps on the device and its device memory, for a given n_ape and ckpt. */
int su2g_vjp_plan(const su2g_lattice *h, int32_t n_ape, int32_t ckpt, int32_t *levels_stored,
                  int64_t *device_bytes);

/* ---- batched replicas: many independent lattices in one device pool, updated by one launch per
 * checkerboard pass (no counterpart in the reference, whose thesis runs were one process per
 * lattice).  Each replica draws the Philox streams of a single handle with the same seed and
 * replica id, so results equal those of separate handles. */
typedef struct su2g_batch su2g_batch;
typedef struct su2g_replica {
    int32_t dims[4];
    double beta;
    uint64_t seed;
    uint32_t replica;    /* Philox stream id */
    int32_t start;       /* su2g_start */
} su2g_replica;
int su2g_batch_create(const su2g_replica *reps, int32_t n, int32_t precision, int32_t device, su2g_batch **out);
int su2g_batch_destroy(su2g_batch *b);
const char *su2g_batch_last_error(const su2g_batch *b);
/* n_sweeps sweeps of (n_hb heatbath + n_or overrelaxation); every meas_every sweeps the plaquette
 * of every replica goes to plaq_trace[k * n + r] (k-th measurement; may be NULL; 0 = no
 * measurement).  The block of meas_every sweeps plus measurement is one CUDA graph, replayed.
 * ms (may be NULL) receives the device time of the replays. */
int su2g_batch_run(su2g_batch *b, int32_t n_sweeps, int32_t n_hb, int32_t n_or, int32_t meas_every,
                   double *plaq_trace, double *ms);
/* How a batch runs its sweeps.  SU2G_BATCH_GRAPH: one launch per checkerboard pass for all replicas
 * (CTAs mapped to replicas by the replica-offset table), a measurement block captured once in a CUDA
 * graph and replayed.  SU2G_BATCH_PERSISTENT: the whole su2g_batch_run as one cooperative launch
 * whose resident CTAs walk every pass as one global link index over all replicas (small replicas
 * share a CTA) and meet at a bounded grid-wide barrier between passes; a barrier that waits too
 * long makes the run return SU2G_EDEVICE.  Both draw the same Philox streams; the persistent
 * kernel's multiply-adds may round differently in the last bit, so its fields agree with the
 * graph form's to rounding, not bit for bit. */
enum su2g_batch_mode { SU2G_BATCH_GRAPH = 0, SU2G_BATCH_PERSISTENT = 1 };
/* Choose the form and the CTA width (64, 128 or 256 threads; 128 or 256 for the persistent form). */
int su2g_batch_configure(su2g_batch *b, int32_t mode, int32_t block);
int su2g_batch_config(const su2g_batch *b, int32_t *mode, int32_t *block);
/* Diagnostic of the persistent form's bounded grid-wide barrier (no counterpart in the reference):
 * one cooperative launch of one CTA per SM passes two barriers that wait for `missing` more CTAs
 * than the grid holds.  missing = 0 returns SU2G_OK; missing > 0 lets every CTA give up after
 * wait_cycles SM clock cycles, and the call returns SU2G_EDEVICE with the reason -- without a fault,
 * the batch staying usable. */
int su2g_batch_selftest_grid_barrier(su2g_batch *b, int32_t missing, int64_t wait_cycles);
/* Times both forms over their CTA widths (sweeps of n_hb + n_or with a plaquette after each) and
 * keeps the fastest, returning its CTA width in block_out (su2g_batch_config gives the form); the
 * fields and counters are restored. */
int su2g_batch_autotune(su2g_batch *b, int32_t n_hb, int32_t n_or, int32_t *block_out);
/* The integrated autocorrelation analysis of LGT_Code/Autocorrelation/t_int.c (see
 * su2g_stats_tau_int) of every replica's plaquette trace from the last su2g_batch_run, on the
 * device, the first `skip` measurements left out: out[4 r + {0,1,2,3}] = mean, tau_int, naive
 * error, error of replica r; resolved[r] (may be NULL) = 1 when 100 tau_int <= the series length. */
int su2g_batch_tau_int(su2g_batch *b, int32_t skip, double *out, int32_t *resolved);
int su2g_batch_download(su2g_batch *b, int32_t r, double *links);
int su2g_batch_upload(su2g_batch *b, int32_t r, const double *links);

/* ---- Kennedy-Pendleton sampler alone (generateSU2InHeatbath_Improved, heatbath.c:76-121;
 * the reference's sampler test LGT_Code/main_test/test.c:115-166): counts of x0 in nbins
 * equal bins on [-1,1] for n draws at fixed alpha, drawn by the same per-link sampler the
 * heatbath sweeps run, in the handle's precision (FP32: fast logarithm and sine/cosine,
 * approximate square roots, delta clamped at 0). */
int su2g_kp_histogram(su2g_lattice *h, double alpha, uint64_t seed, int64_t n, int32_t nbins,
                      int64_t *counts);

/* ---- APE smearing without any allocation.  No counterpart in the reference.
 * For callers that keep their field in device memory they obtained elsewhere and may not call
 * cudaMalloc themselves (memory handed out by another component or a fixed budget, or loops that
 * must not pay cudaMalloc's device-wide synchronisation), so they cannot create a handle.
 * links: device pointer to the field in the reference's layout, double[V][4][4]; smeared in place,
 * ns steps of `mode` with parameter alpha, enqueued on cuda_stream (NULL = default stream); the
 * call does not synchronise.  The intermediate level lives in a static device array of 48 MiB
 * that every GPU loading the library keeps until exit; lattices above 393216 sites are rejected
 * with SU2G_EINVAL, and so is a field pointer that is not 16-byte aligned device (or managed)
 * memory of the current device.  The first call on a device looks up that array's address (issue
 * it before any stream capture); the address is cached for the life of the process, so after
 * cudaDeviceReset this entry point must not be called again in that process.  All calls share the
 * array: calls that overlap on the GPU race.  Errors are reported by su2g_last_error(NULL). */
int su2g_ape_inplace_noalloc(double *links, const int32_t dims[4], int32_t ns, double alpha, int32_t mode,
                             void *cuda_stream);

/* ---- pinned (page-locked) host memory for field arrays, so that transfers run at full link
 * speed; the reference's pu block (init.c:842-858) can live in it. */
int su2g_host_alloc(size_t bytes, void **ptr);
int su2g_host_free(void *ptr);

/* ---- timing and profiling on the handle's stream (CUDA events). */
int su2g_stream(su2g_lattice *h, void **cuda_stream);
int su2g_synchronize(su2g_lattice *h);
int su2g_timer_begin(su2g_lattice *h);
int su2g_timer_end(su2g_lattice *h, double *ms);
/* When enabled, every kernel launch is bracketed by events; su2g_profile_read returns, for a
 * kernel class, the launch count and summed device time since the last reset. */
enum su2g_kernel_class {
    SU2G_K_HEATBATH = 0, SU2G_K_OVERRELAX = 1, SU2G_K_PLAQUETTE = 2, SU2G_K_APE = 3,
    SU2G_K_WILSON = 4, SU2G_K_QTOP = 5, SU2G_K_REDUCE = 6, SU2G_K_OTHER = 7, SU2G_K_METROPOLIS = 8,
    SU2G_K_COUNT = 9
};
int su2g_profile_enable(su2g_lattice *h, int32_t enable);
/* Kernel choice for a class (no reference counterpart).  SU2G_K_APE: 0 = the per-site kernel
 * (default), 1 = the TMA-tiled FP32 APE_all kernel where the geometry allows it (plane tiles staged
 * by cp.async.bulk; slower on B200 at 48^4 because its shared memory admits one CTA per SM). */
int su2g_set_kernel_variant(su2g_lattice *h, int32_t kernel_class, int32_t variant);
/* The variant an APE_all step of this handle runs (0 = per-site, 1 = TMA-tiled). */
int su2g_kernel_variant(const su2g_lattice *h, int32_t kernel_class, int32_t *active);
int su2g_profile_read(su2g_lattice *h, int32_t kernel_class, int64_t *launches, double *ms);

/* ---- failure detection without a GPU fault (no counterpart in the reference).  Device-side
 * failures (a heatbath link past the Kennedy-Pendleton trial bound, a bulk copy whose wait ran out)
 * set bits of the handle's status word; the next synchronising call returns SU2G_EDEVICE with the
 * reason and clears the word, and the handle stays usable.  This diagnostic runs one CTA that arms
 * an mbarrier for a bulk copy that is never issued and waits with the library's bounded wait (at
 * most poll_limit polls, 1 ... 2^22): it returns SU2G_EDEVICE with the timeout message. */
int su2g_selftest_bounded_wait(su2g_lattice *h, uint32_t poll_limit);

#ifdef __cplusplus
}
#endif

#endif /* SU2G_H */
