// philox.cuh -- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11) for device code, keyed by lattice coordinates.
//
// The reference draws from a sequential RANLUX stream (LGT_Code/modules/random/ranlxd.c);
// a counter-based generator keyed by (site, sweep, dir, draw, replica) makes every link
// update independent of launch shape and update order inside a checkerboard pass.
// Counter layout (shared with the test oracle):
//   key  = (seed lo, seed hi)
//   ctr0 = lexicographic site index n
//   ctr1 = heatbath sweep index (0 for start-up streams)
//   ctr2 = (draw << 3) | (dir << 1) | tag     tag 0: Kennedy-Pendleton trial `draw`
//                                             tag 1, draw 0: the two angles
//                                             tag 1, draw 1: zero-staple fallback link
//   ctr3 = (kind << 24) | replica             kind 0: update, 1: start-up
#pragma once
#include <cstdint>

namespace su2g {

struct U4 {
    uint32_t x, y, z, w;
};

__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        U4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// The ten round keys of a seed, computed once on the host: a kernel that takes them as a parameter
// reads them from the constant bank inside each round instead of adding the Weyl increments per
// block (the same words, so the same draws).
struct PhiloxKeys {
    uint32_t k0[10], k1[10];
};

inline PhiloxKeys philox_keys(uint64_t seed)
{
    PhiloxKeys K;
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    for (int r = 0; r < 10; ++r) {
        K.k0[r] = k0;
        K.k1[r] = k1;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return K;
}

__device__ __forceinline__ U4 philox4x32_10(U4 c, const PhiloxKeys& K)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        U4 n;
        n.x = hi1 ^ c.y ^ K.k0[r];
        n.y = lo1;
        n.z = hi0 ^ c.w ^ K.k1[r];
        n.w = lo0;
        c = n;
    }
    return c;
}

// Stream kinds: heatbath/fallback draws, starts, Metropolis hits, random-order visit counts.
enum : uint32_t { kStreamUpdate = 0u, kStreamStart = 1u, kStreamMetro = 2u, kStreamVisit = 3u };

__device__ __forceinline__ U4 link_random(uint64_t seed, uint32_t site, uint32_t sweep, uint32_t dir,
                                          uint32_t draw, uint32_t tag, uint32_t kind, uint32_t replica)
{
    U4 c;
    c.x = site;
    c.y = sweep;
    c.z = (draw << 3) | (dir << 1) | tag;
    c.w = (kind << 24) | replica;
    return philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
}

__device__ __forceinline__ U4 link_random(const PhiloxKeys& K, uint32_t site, uint32_t sweep, uint32_t dir,
                                          uint32_t draw, uint32_t tag, uint32_t kind, uint32_t replica)
{
    U4 c;
    c.x = site;
    c.y = sweep;
    c.z = (draw << 3) | (dir << 1) | tag;
    c.w = (kind << 24) | replica;
    return philox4x32_10(c, K);
}

// Uniforms in the open interval (0,1).  FP64 keeps all 32 bits; FP32 keeps the top 23 bits, so the
// FP32 and FP64 chains consume identical Philox words and differ only by the conversion.
// FP64: (w + 1/2) / 2^32 as one multiply-add; w 2^-32 and the sum are exact, so the value is the same
__device__ __forceinline__ double u01(uint32_t w, double) { return fma((double)w, 1.0 / 4294967296.0, 0.5 / 4294967296.0); }
__device__ __forceinline__ float u01(uint32_t w, float)
{
    // ((w >> 9) + 1/2) / 2^23 as one multiply-add: both forms are exact, so the value is the same
    return fmaf((float)(w >> 9), 1.0f / 8388608.0f, 0.5f / 8388608.0f);
}

}  // namespace su2g
