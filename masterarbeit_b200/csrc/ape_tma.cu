// ape_tma.cu -- APE_all smearing step (FP32) with TMA-staged plane tiles marching along t.
//
// Same step as k_ape<float, ALL> (smearing_APE_all, LGT_Code/modules/obs/smearing.c:74-105):
//   U'_mu(x) = Proj(U_mu(x) + alpha S_mu(x)),
//   S_mu(x) = sum_nu U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag + U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu).
//
// Data movement.  A CTA owns one column (x, rows y0 .. y0+YB-1, all z) and marches over t.  The
// links a plane (t, x) needs live in seven plane tiles: (t-1|t|t+1, x), (t-1|t, x+1), (t|t+1, x-1),
// each holding rows y0-1 .. y0+YB (one halo row each side) of all four directions and both
// parities.  Tiles are copied by cp.async.bulk (the Blackwell bulk-copy engine) into a ring of ten
// shared-memory slots; at step t the three tiles that step t+1 adds, (t+2, x), (t+1, x+1) and
// (t+2, x-1), are fetched while plane t is computed from shared memory.  A tile is a set of
// contiguous runs of the checkerboarded field (one run per direction and parity, split in two
// where the y halo wraps), so no tensor map is needed.  Every tile of the field is read from L2
// or HBM by three CTAs at most, and every link of the output is written once.
//
// Waits.  Each slot has an mbarrier that completes when its tile's bytes have landed; waits are
// bounded (kWaitLimit polls) and a CTA that gives up raises kStatusTmaTimeout and stops.
#include <cstdint>

#include "internal.cuh"
#include "mbarrier.cuh"

using namespace su2g;

namespace {

constexpr int kSlots = 10;                 // 4 centre-column slots, 3 for x+1, 3 for x-1
constexpr uint32_t kWaitLimit = 1u << 22;  // bounded mbarrier polling

__device__ __forceinline__ void bulk_copy(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

struct TileGeom {
    int rows;        // YB + 2
    int hl;          // links per row and parity = L3 / 2
    int chunk;       // float4 per (direction, parity) chunk = rows * hl
    int tile;        // float4 per tile = 8 * chunk
};

// Issue the copies of tile (tp, xp) into slot s (one thread).  Rows y0-1 .. y0+YB, wrapped in y.
__device__ __forceinline__ void issue_tile(const Field<float>& in, const Geom& g, const TileGeom& tg, float4* slots,
                                           uint32_t bars, int s, int tp, int xp, int y0)
{
    const uint32_t bar = bars + 8u * (uint32_t)s;
    mbar_expect_tx(bar, (uint32_t)tg.tile * 16u);
    float4* tile = slots + (size_t)s * tg.tile;
    // runs of consecutive rows that are consecutive in memory
    int r = 0;
    while (r < tg.rows) {
        int y = y0 - 1 + r;
        y += (y < 0) ? g.L[2] : 0;
        y -= (y >= g.L[2]) ? g.L[2] : 0;
        int len = min(tg.rows - r, g.L[2] - y);
        const int hrow = (((tp * g.L[1] + xp) * g.L[2] + y) * g.L[3]) >> 1;
        for (int dp = 0; dp < 8; ++dp) {
            const int dir = dp >> 1, par = dp & 1;
            const float4* src = in.p[dir] + (size_t)par * g.Vh + hrow;
            bulk_copy(smem_addr(tile + dp * tg.chunk + r * tg.hl), src, (uint32_t)(len * tg.hl) * 16u, bar);
        }
        r += len;
    }
}

__device__ __forceinline__ int wrap(int v, int L) { return v < 0 ? v + L : (v >= L ? v - L : v); }

__global__ void __launch_bounds__(256, 1)
    k_ape_all_tma(Field<float> in, Field<float> out, Geom g, float alpha, int yb, unsigned* __restrict__ status)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    TileGeom tg;
    tg.rows = yb + 2;
    tg.hl = g.L[3] >> 1;
    tg.chunk = tg.rows * tg.hl;
    tg.tile = 8 * tg.chunk;
    float4* slots = reinterpret_cast<float4*>(smem_raw);
    uint64_t* bar_mem = reinterpret_cast<uint64_t*>(smem_raw + (size_t)kSlots * tg.tile * 16);
    const uint32_t bars = smem_addr(bar_mem);

    const int nyb = g.L[2] / yb;
    const int x = blockIdx.x / nyb, y0 = (blockIdx.x % nyb) * yb;
    const int xpl = wrap(x + 1, g.L[1]), xmn = wrap(x - 1, g.L[1]);
    const int LT = g.L[0];
    // slots: centre column C(t) in t%4, x+1 column P(t) in 4 + t%3, x-1 column M(t) in 7 + t%3
    auto sC = [](int t) { return t & 3; };
    auto sP = [](int t) { return 4 + t % 3; };
    auto sM = [](int t) { return 7 + t % 3; };

    if (threadIdx.x == 0) {
        for (int s = 0; s < kSlots; ++s) mbar_init(bars + 8u * s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // tiles in time order; slot phases flip per completed tile
    uint32_t phase = 0;     // bit s = parity of slot s's next completion
    uint32_t pending = 0;   // thread 0: slots whose copies have been issued and not yet seen complete
    if (threadIdx.x == 0) {
        // t = -1 is plane LT-1; ring slots are indexed with t + 4*LT (>= 0)
        issue_tile(in, g, tg, slots, bars, sC(4 * LT - 1), LT - 1, x, y0);
        issue_tile(in, g, tg, slots, bars, sC(4 * LT + 0), 0, x, y0);
        issue_tile(in, g, tg, slots, bars, sC(4 * LT + 1), wrap(1, LT), x, y0);
        issue_tile(in, g, tg, slots, bars, sP(3 * LT - 1), LT - 1, xpl, y0);
        issue_tile(in, g, tg, slots, bars, sP(3 * LT + 0), 0, xpl, y0);
        issue_tile(in, g, tg, slots, bars, sM(3 * LT + 0), 0, xmn, y0);
        issue_tile(in, g, tg, slots, bars, sM(3 * LT + 1), wrap(1, LT), xmn, y0);
        pending = (1u << sC(4 * LT - 1)) | (1u << sC(4 * LT)) | (1u << sC(4 * LT + 1)) | (1u << sP(3 * LT - 1)) |
                  (1u << sP(3 * LT)) | (1u << sM(3 * LT)) | (1u << sM(3 * LT + 1));
    }
    // thread -> output site (row yl, z) of the current plane
    const int L3 = g.L[3];
    const int yl = threadIdx.x / L3, z = threadIdx.x - yl * L3;
    const bool active = yl < yb;
    const int y = y0 + yl;
    const int zp = z == L3 - 1 ? 0 : z + 1, zm = z == 0 ? L3 - 1 : z - 1;

    // Bounded wait for slot s; every thread polls, and the decision to give up is taken by the
    // whole CTA (__syncthreads_or) so that no thread is left waiting at a barrier.
    bool ok = true;
    auto wait_slot = [&](int s) {
        const uint32_t bar = bars + 8u * (uint32_t)s;
        const uint32_t ph = (phase >> s) & 1u;
        if (ok) ok = mbar_wait_bounded(bar, ph, kWaitLimit);
        if (ok) pending &= ~(1u << s);
        phase ^= 1u << s;
    };
    // On a timeout the CTA stops; before it exits, thread 0 waits (again bounded) for the copies it
    // issued that have not been seen to complete, so that no bulk copy into this CTA's shared memory
    // is left in flight.  Every issued slot has had exactly one wait_slot since its issue, which
    // flipped its phase bit, so the phase still owed is the flipped-back one.
    auto give_up = [&]() {
        if (threadIdx.x == 0) {
            for (int s = 0; s < kSlots; ++s)
                if (pending & (1u << s)) mbar_wait_bounded(bars + 8u * (uint32_t)s, ((phase >> s) & 1u) ^ 1u, kWaitLimit);
            atomicOr(status, kStatusTmaTimeout);
        }
    };
    // first step needs all seven tiles
    wait_slot(sC(4 * LT - 1));
    wait_slot(sC(4 * LT));
    wait_slot(sC(4 * LT + 1));
    wait_slot(sP(3 * LT - 1));
    wait_slot(sP(3 * LT));
    wait_slot(sM(3 * LT));
    wait_slot(sM(3 * LT + 1));
    if (__syncthreads_or(!ok)) {
        give_up();
        return;
    }

    for (int t = 0; t < LT; ++t) {
        const int tt = t + 4 * LT;   // non-negative ring index for t-1
        const int t3 = t + 3 * LT;
        if (t + 1 < LT && threadIdx.x == 0) {
            issue_tile(in, g, tg, slots, bars, sC(tt + 2), wrap(t + 2, LT), x, y0);
            issue_tile(in, g, tg, slots, bars, sP(t3 + 1), wrap(t + 1, LT), xpl, y0);
            issue_tile(in, g, tg, slots, bars, sM(t3 + 2), wrap(t + 2, LT), xmn, y0);
            pending |= (1u << sC(tt + 2)) | (1u << sP(t3 + 1)) | (1u << sM(t3 + 2));
        }
        if (active) {
            // link loader: tile (dt, dx) relative to (t, x), row offset dy, z offset dz
            const int pbase = (t + x + y0 - 1 + z) & 1;   // parity of (t, x, row 0, z)
            auto tile_of = [&](int dt, int dx) -> const float4* {
                int s = dx == 0 ? sC(tt + dt) : (dx > 0 ? sP(t3 + dt) : sM(t3 + dt));
                return slots + (size_t)s * tg.tile;
            };
            auto L = [&](int dir, int dt, int dx, int dy, int dz) -> Q<float> {
                const int r = yl + 1 + dy;
                const int zz = dz == 0 ? z : (dz > 0 ? zp : zm);
                const int par = (pbase + dt + dx + 1 + yl + dy + dz) & 1;   // row r = yl+1+dy, z + dz
                const float4 v = tile_of(dt, dx)[(dir * 2 + par) * tg.chunk + r * tg.hl + (zz >> 1)];
                return q_make<float>(v.x, v.y, v.z, v.w);
            };
            // offsets of +-mu as (dt, dx, dy, dz)
            Q<float> u[4], S[4];
#pragma unroll
            for (int mu = 0; mu < 4; ++mu) {
                u[mu] = L(mu, 0, 0, 0, 0);
                S[mu] = q_zero<float>();
            }
#define OFF(m, s) ((m) == 0 ? (s) : 0), ((m) == 1 ? (s) : 0), ((m) == 2 ? (s) : 0), ((m) == 3 ? (s) : 0)
#pragma unroll
            for (int mu = 0; mu < 4; ++mu)
#pragma unroll
                for (int nu = mu + 1; nu < 4; ++nu) {
                    // P = U_mu(x+nu) U_nu(x+mu)^dag, shared by the forward staples of mu (plane nu) and nu (plane mu)
                    const Q<float> P = q_mul_nd(L(mu, OFF(nu, 1)), L(nu, OFF(mu, 1)));
                    S[mu] = q_mul_add(S[mu], u[nu], P);
                    S[nu] = q_mul_nd_add(S[nu], u[mu], P);
                }
#pragma unroll
            for (int mu = 0; mu < 4; ++mu)
#pragma unroll
                for (int nu = 0; nu < 4; ++nu) {
                    if (nu == mu) continue;
                    // U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu)
                    const int dt = (nu == 0 ? -1 : 0) + (mu == 0 ? 1 : 0);
                    const int dx = (nu == 1 ? -1 : 0) + (mu == 1 ? 1 : 0);
                    const int dy = (nu == 2 ? -1 : 0) + (mu == 2 ? 1 : 0);
                    const int dz = (nu == 3 ? -1 : 0) + (mu == 3 ? 1 : 0);
                    S[mu] = q_mul_add(S[mu], q_mul_dn(L(nu, OFF(nu, -1)), L(mu, OFF(nu, -1))), L(nu, dt, dx, dy, dz));
                }
#undef OFF
            const int n = ((t * g.L[1] + x) * g.L[2] + y) * L3 + z;
            const int par = (t + x + y + z) & 1;
#pragma unroll
            for (int mu = 0; mu < 4; ++mu) out.sth(mu, par, n >> 1, q_project(q_axpy(alpha, S[mu], u[mu])));
        }
        __syncthreads();   // every read of this step's slots is done before step t+1 refills them
        if (t + 1 < LT) {
            wait_slot(sC(tt + 2));
            wait_slot(sP(t3 + 1));
            wait_slot(sM(t3 + 2));
            if (__syncthreads_or(!ok)) {
                give_up();
                return;
            }
        }
    }
}

}  // namespace

namespace su2g {

// Rows per CTA for which the ten tile slots fit in shared memory; 0 if this kernel does not apply.
int ape_tma_rows(const Geom& g, int max_smem)
{
    if (g.L[3] > 256 || (g.L[3] & 1)) return 0;
    for (int yb : {4, 2}) {
        if (g.L[2] % yb) continue;
        const long long threads = (long long)yb * g.L[3];
        const long long tile = 8ll * (yb + 2) * (g.L[3] / 2) * 16;
        const long long smem = kSlots * tile + 8 * kSlots;
        if (threads >= 64 && threads <= 256 && smem <= max_smem) return yb;
    }
    return 0;
}

int ape_tma_launch(su2g_lattice* h, void* const in_dirs[4], void* const out_dirs[4], double alpha, int yb)
{
    const Geom& g = h->g;
    const int threads = yb * g.L[3];
    const size_t smem = (size_t)kSlots * 8 * (yb + 2) * (g.L[3] / 2) * 16 + 8 * kSlots;
    cudaFuncSetAttribute(k_ape_all_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int grid = g.L[1] * (g.L[2] / yb);
    launch_begin(h, SU2G_K_APE);
    k_ape_all_tma<<<grid, threads, smem, h->stream>>>(make_field<float>(in_dirs, g.Vh), make_field<float>(out_dirs, g.Vh),
                                                       g, (float)alpha, yb, h->d_status);
    return launch_end(h, SU2G_K_APE, "APE kernel (TMA tiles)");
}

}  // namespace su2g
