/*
 * philox.h -- Philox4x32-10 counter-based generator, plain C (test infrastructure).
 *
 * ORACLE / TEST INFRASTRUCTURE ONLY.  This header is used by the CPU oracle
 * (oracle/su2_oracle.c) and by the reference harness's injected-uniform RNG
 * (oracle/inject_ranlxd.c).  The product path has its own device version in
 * masterarbeit_b200/csrc/philox.cuh; the tests check that both agree with the
 * published known-answer vectors.
 *
 * Algorithm: J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw,
 * "Parallel random numbers: as easy as 1, 2, 3", SC'11, section 4 (Philox):
 * ten rounds of two 32x32->64 multiplies with the round multipliers
 * 0xD2511F53 / 0xCD9E8D57 and a Weyl key schedule with increments
 * 0x9E3779B9 / 0xBB67AE85.
 *
 * The reference draws its randoms from RANLUX (LGT_Code/modules/random/ranlxd.c);
 * this build replaces it by Philox keyed by lattice coordinates, so the stream
 * layout below (which counter word carries what) is this project's own choice:
 *   key  = (seed & 0xffffffff, seed >> 32)
 *   ctr0 = lexicographic site index n  (n = ((t*L1 + x)*L2 + y)*L3 + z)
 *   ctr1 = heatbath sweep index (init streams: 0)
 *   ctr2 = (draw << 3) | (dir << 1) | tag      tag 0: KP trial 'draw'
 *                                               tag 1, draw 0: the two angles
 *                                               tag 1, draw 1: zero-staple fallback
 *   ctr3 = (kind << 24) | replica              kind 0: update, 1: hot start
 */
#ifndef SU2_ORACLE_PHILOX_H
#define SU2_ORACLE_PHILOX_H

#include <stdint.h>

#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

static inline void philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t x0 = ctr[0], x1 = ctr[1], x2 = ctr[2], x3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)PHILOX_M0 * x0;
        uint64_t p1 = (uint64_t)PHILOX_M1 * x2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ x1 ^ k0;
        uint32_t n2 = hi0 ^ x3 ^ k1;
        x0 = n0; x1 = lo1; x2 = n2; x3 = lo0;
        k0 += PHILOX_W0; k1 += PHILOX_W1;
    }
    out[0] = x0; out[1] = x1; out[2] = x2; out[3] = x3;
}

/* 32-bit word -> double uniform in the open interval (0,1), exact. */
static inline double philox_u01_f64(uint32_t w)
{
    return ((double)w + 0.5) * (1.0 / 4294967296.0);
}

/* 32-bit word -> float uniform in (0,1): top 23 bits plus half a step, exact in float. */
static inline float philox_u01_f32(uint32_t w)
{
    return ((float)(w >> 9) + 0.5f) * (1.0f / 8388608.0f);
}

#define SU2_STREAM_UPDATE 0u
#define SU2_STREAM_INIT 1u
#define SU2_STREAM_METRO 2u
#define SU2_STREAM_VISIT 3u
#define SU2_VISIT_SHIFT 21   /* draw index of visit v's heatbath draws: (v << SU2_VISIT_SHIFT) | trial */

static inline void su2_philox_link(uint64_t seed, uint32_t site, uint32_t sweep, uint32_t dir,
                                   uint32_t draw, uint32_t tag, uint32_t kind, uint32_t replica,
                                   uint32_t out[4])
{
    uint32_t key[2] = {(uint32_t)(seed & 0xffffffffu), (uint32_t)(seed >> 32)};
    uint32_t ctr[4] = {site, sweep, (draw << 3) | (dir << 1) | tag, (kind << 24) | replica};
    philox4x32_10(ctr, key, out);
}

#endif
