// capi.cu -- handle lifetime, field transfer and start-up kernels, timing/profiling, shared helpers.
//
// Reference counterparts: initArrayOfNeighbours / initGaugeField / allocateGaugeField /
// releaseGaugeField (LGT_Code/modules/admin/init.c:741-925) and the body of
// readConfig / writeConfig (LGT_Code/modules/io/config_IO.c:537-621, :40-117).  The
// neighbour table disappears: sites are decoded arithmetically (su2.cuh).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <new>

#include "internal.cuh"
#include "philox.cuh"

using namespace su2g;

static thread_local char g_create_err[512] = "no error";

namespace su2g {

int set_error(su2g_lattice* h, int code, const char* fmt, ...)
{
    char* dst = h ? h->err : g_create_err;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(dst, 512, fmt, ap);
    va_end(ap);
    return code;
}

int check_cuda(su2g_lattice* h, cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return SU2G_OK;
    return set_error(h, e == cudaErrorMemoryAllocation ? SU2G_ENOMEM : SU2G_ECUDA, "%s: %s", what,
                     cudaGetErrorString(e));
}

int grid_for(const su2g_lattice* h, long long work, int per_sm)
{
    long long need = (work + kBlock - 1) / kBlock;
    long long cap = (long long)h->num_sms * per_sm;
    long long g = std::min(need, cap);
    g = std::min<long long>(g, kMaxPartials);
    return (int)std::max<long long>(g, 1);
}

int resident_grid(const su2g_lattice* h, const void* kernel, long long work, size_t smem)
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return grid_for(h, work, per_sm);
}

static cudaEvent_t pool_event(su2g_lattice* h)
{
    if (!h->event_pool.empty()) {
        cudaEvent_t e = h->event_pool.back();
        h->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

static void drain_profile(su2g_lattice* h)
{
    if (h->prof_pending.empty()) return;
    cudaStreamSynchronize(h->stream);
    for (auto& p : h->prof_pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            h->prof_ms[p.cls] += ms;
            h->prof_launches[p.cls] += 1;
        }
        h->event_pool.push_back(p.a);
        h->event_pool.push_back(p.b);
    }
    h->prof_pending.clear();
}

int launch_begin(su2g_lattice* h, int cls)
{
    if (!h->profiling) return SU2G_OK;
    if (h->prof_pending.size() > 4096) drain_profile(h);
    su2g_lattice::Prof p;
    p.a = pool_event(h);
    p.b = pool_event(h);
    p.cls = cls;
    cudaEventRecord(p.a, h->stream);
    h->prof_pending.push_back(p);
    return SU2G_OK;
}

int launch_end(su2g_lattice* h, int cls, const char* what)
{
    (void)cls;
    if (h->profiling && !h->prof_pending.empty()) cudaEventRecord(h->prof_pending.back().b, h->stream);
    return check_cuda(h, cudaGetLastError(), what);
}

int ensure_partials(su2g_lattice* h, size_t slots)
{
    if (slots <= h->partial_slots) return SU2G_OK;
    if (h->partials) cudaFree(h->partials);
    h->partials = nullptr;
    h->partial_slots = 0;
    cudaError_t e = cudaMalloc(&h->partials, slots * kMaxPartials * sizeof(DD));
    if (e != cudaSuccess) return check_cuda(h, e, "allocating reduction scratch");
    h->partial_slots = slots;
    return SU2G_OK;
}

int ensure_partial_entries(su2g_lattice* h, size_t n)
{
    return ensure_partials(h, (n + kMaxPartials - 1) / kMaxPartials);
}

// One CTA of kFinalizeBlock threads per slot.  Thread t sums partials t, t + NT, t + 2 NT, ... into
// four compensated accumulators in turn (four independent load/add chains in flight), combines them
// in a fixed order, and the CTA tree follows: the order is fixed, so the result is deterministic.
// (The plaquette's 20736 partials at 48^4 took 42 us with one chain per thread of 256.)
constexpr int kFinalizeBlock = 1024;

__global__ void __launch_bounds__(kFinalizeBlock) k_finalize(const DD* __restrict__ partials, int nparts, int stride,
                                                             double scale, double* __restrict__ out)
{
    const DD* p = partials + (size_t)blockIdx.x * stride;
    DD acc[4] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    int i = threadIdx.x;
    for (; i + 3 * kFinalizeBlock < nparts; i += 4 * kFinalizeBlock) {
        const DD a = p[i], b = p[i + kFinalizeBlock], c = p[i + 2 * kFinalizeBlock], d = p[i + 3 * kFinalizeBlock];
        acc[0] = dd_add(acc[0], a);
        acc[1] = dd_add(acc[1], b);
        acc[2] = dd_add(acc[2], c);
        acc[3] = dd_add(acc[3], d);
    }
    if (i < nparts) acc[0] = dd_add(acc[0], p[i]);   // at most three left for this thread
    if (i + kFinalizeBlock < nparts) acc[1] = dd_add(acc[1], p[i + kFinalizeBlock]);
    if (i + 2 * kFinalizeBlock < nparts) acc[2] = dd_add(acc[2], p[i + 2 * kFinalizeBlock]);
    DD v = dd_add(dd_add(acc[0], acc[1]), dd_add(acc[2], acc[3]));
    v = dd_block_sum<kFinalizeBlock>(v);
    if (threadIdx.x == 0) out[blockIdx.x] = (v.s + v.e) * scale;
}

// One slot of many partials: CTA b sums the contiguous chunk b (fixed assignment), and the CTA
// that arrives last on the counter sums the CTA results in index order and clears the counter, so
// the result does not depend on which CTA finished when.  (The fused plaquette's 249k partials
// at 48^4 took 17 us in one CTA of k_finalize.)
constexpr int kFinWideThreads = 256;
static_assert(kFinBlocks <= kFinWideThreads, "the last CTA sums one CTA result per thread");

__global__ void __launch_bounds__(kFinWideThreads) k_finalize_wide(const DD* __restrict__ partials, int nparts,
                                                                   double scale, double* __restrict__ out,
                                                                   DD* __restrict__ blocks, unsigned* ticket)
{
    const int nb = gridDim.x;
    const int chunk = (nparts + nb - 1) / nb;
    const int lo = blockIdx.x * chunk, hi = min(nparts, lo + chunk);
    DD acc[2] = {{0.0, 0.0}, {0.0, 0.0}};
    int i = lo + threadIdx.x;
    for (; i + kFinWideThreads < hi; i += 2 * kFinWideThreads) {
        acc[0] = dd_add(acc[0], partials[i]);
        acc[1] = dd_add(acc[1], partials[i + kFinWideThreads]);
    }
    if (i < hi) acc[0] = dd_add(acc[0], partials[i]);
    const DD v = dd_block_sum<kFinWideThreads>(dd_add(acc[0], acc[1]));
    __shared__ bool last;
    if (threadIdx.x == 0) {
        blocks[blockIdx.x] = v;
        __threadfence();
        last = atomicAdd(ticket, 1u) == (unsigned)nb - 1u;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    DD w = {0.0, 0.0};
    if (threadIdx.x < nb) {
        const double2 b = __ldcg(reinterpret_cast<const double2*>(blocks) + threadIdx.x);
        w.s = b.x;
        w.e = b.y;
    }
    w = dd_block_sum<kFinWideThreads>(w);
    if (threadIdx.x == 0) {
        *out = (w.s + w.e) * scale;
        *ticket = 0u;
    }
}

int finalize(su2g_lattice* h, int nparts, int nslots, double scale, int out_off, int stride)
{
    if (out_off + nslots > kOutSlots) return set_error(h, SU2G_EINVAL, "too many result slots");
    launch_begin(h, SU2G_K_REDUCE);
    if (nslots == 1 && nparts > 4 * kFinalizeBlock) {
        const int nb = std::min(kFinBlocks, (nparts + 2 * kFinWideThreads - 1) / (2 * kFinWideThreads));
        k_finalize_wide<<<nb, kFinWideThreads, 0, h->stream>>>(h->partials, nparts, scale, h->d_out + out_off,
                                                              h->fin_blocks, h->fin_ticket);
    } else {
        k_finalize<<<nslots, kFinalizeBlock, 0, h->stream>>>(h->partials, nparts, stride > 0 ? stride : kMaxPartials,
                                                              scale, h->d_out + out_off);
    }
    return launch_end(h, SU2G_K_REDUCE, "finalize reduction");
}

int fetch_results(su2g_lattice* h, int off, int n)
{
    int rc = check_cuda(h, cudaMemcpyAsync(h->h_out + off, h->d_out + off, n * sizeof(double),
                                           cudaMemcpyDeviceToHost, h->stream),
                        "copying results");
    if (rc) return rc;
    unsigned status = 0;
    rc = check_cuda(h, cudaMemcpyAsync(&status, h->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream),
                    "reading status word");
    if (rc) return rc;
    rc = check_cuda(h, cudaStreamSynchronize(h->stream), "synchronising");
    if (rc) return rc;
    // a reported failure is reported once: the word is cleared and the handle stays usable
    if (status && (rc = check_cuda(h, cudaMemsetAsync(h->d_status, 0, sizeof(unsigned), h->stream), "clearing status")))
        return rc;
    if (status & kStatusKpTrials)
        return set_error(h, SU2G_EDEVICE, "a heatbath link exceeded %u Kennedy-Pendleton trials", kMaxTrials);
    if (status & kStatusTmaTimeout)
        return set_error(h, SU2G_EDEVICE, "a bulk copy into shared memory did not complete in time");
    if (status) return set_error(h, SU2G_EDEVICE, "device status word 0x%x", status);
    return SU2G_OK;
}

}  // namespace su2g

// ----------------------------------------------------------------- kernels ---

namespace {

// su2RandomMatrix (LGT_Code/modules/random/random_su3.c:141-155) on three uniforms.
template <typename R>
__device__ __forceinline__ Q<R> ref_random_link(R r0, R r1, R r2)
{
    Q<R> u;
    u.c0 = R(1) - R(2) * r0;
    u.c1 = R(1) - R(2) * r1;
    R zw = sqrt_r(R(1) - u.c1 * u.c1);
    R s, c;
    sincospi(R(2) * r2, &s, &c);
    u.c2 = zw * c;
    u.c3 = zw * s;
    zw = sqrt_r(R(1) - u.c0 * u.c0);
    u.c1 *= zw;
    u.c2 *= zw;
    u.c3 *= zw;
    return u;
}

__device__ __forceinline__ float log_r(float x) { return logf(x); }
__device__ __forceinline__ double log_r(double x) { return log(x); }

template <typename R>
__global__ void __launch_bounds__(kBlock) k_start(Field<R> U, Geom g, int mode, uint64_t seed, uint32_t replica)
{
    const long long nlinks = 4ll * g.V;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nlinks;
         i += (long long)gridDim.x * blockDim.x) {
        int mu = (int)(i / g.V);
        int rem = (int)(i - (long long)mu * g.V);
        int par = rem >= g.Vh;
        int h = rem - par * g.Vh;
        Q<R> u = q_one<R>();
        if (mode != SU2G_START_COLD) {
            Site s = site_of(g, par, h);
            U4 w = link_random(seed, (uint32_t)s.n, 0u, (uint32_t)mu, 0u, 0u, kStreamStart, replica);
            R r0 = u01(w.x, R(0)), r1 = u01(w.y, R(0)), r2 = u01(w.z, R(0)), r3 = u01(w.w, R(0));
            if (mode == SU2G_START_REF) {
                u = ref_random_link<R>(r0, r1, r2);
            } else {
                // Box-Muller: two pairs of N(0,1) draws, normalised -> Haar-uniform on S^3.
                R ra = sqrt_r(R(-2) * log_r(r0)), rb = sqrt_r(R(-2) * log_r(r2));
                R sa, ca, sb, cb;
                sincospi(R(2) * r1, &sa, &ca);
                sincospi(R(2) * r3, &sb, &cb);
                u = q_project(q_make<R>(ra * ca, ra * sa, rb * cb, rb * sb));
            }
        }
        U.sth(mu, par, h, u);
    }
}

// AoS FP64 (reference host layout) -> device layout, for sites [n0, n0 + count).
template <typename R>
__global__ void __launch_bounds__(kBlock) k_aos_in(const double2* __restrict__ aos, Field<R> U, Geom g, int n0,
                                                   int count)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        int n = n0 + i;
        uint32_t t = fdiv((uint32_t)n, g.dS0);
        uint32_t r = (uint32_t)n - t * (uint32_t)g.S[0];
        uint32_t x = fdiv(r, g.dS1);
        r -= x * (uint32_t)g.S[1];
        uint32_t y = fdiv(r, g.dS2);
        uint32_t z = r - y * (uint32_t)g.S[2];
        int par = (int)((t + x + y + z) & 1u);
        const double2* src = aos + (size_t)i * 8;
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) {
            double2 a = src[2 * mu], b = src[2 * mu + 1];
            U.sth(mu, par, n >> 1, q_make<R>((R)a.x, (R)a.y, (R)b.x, (R)b.y));
        }
    }
}

template <typename R>
__global__ void __launch_bounds__(kBlock) k_aos_out(double2* __restrict__ aos, Field<R> U, Geom g, int n0, int count)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        int n = n0 + i;
        uint32_t t = fdiv((uint32_t)n, g.dS0);
        uint32_t r = (uint32_t)n - t * (uint32_t)g.S[0];
        uint32_t x = fdiv(r, g.dS1);
        r -= x * (uint32_t)g.S[1];
        uint32_t y = fdiv(r, g.dS2);
        uint32_t z = r - y * (uint32_t)g.S[2];
        int par = (int)((t + x + y + z) & 1u);
        double2* dst = aos + (size_t)i * 8;
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) {
            Q<R> q = U.ldh(mu, par, n >> 1);
            dst[2 * mu] = make_double2((double)q.c0, (double)q.c1);
            dst[2 * mu + 1] = make_double2((double)q.c2, (double)q.c3);
        }
    }
}

constexpr size_t kAosChunkSites = 1u << 20;   // 128 MB of FP64 AoS staging

}  // namespace

int su2g::ensure_aos(su2g_lattice* h)
{
    if (h->d_aos) return SU2G_OK;
    size_t sites = std::min<size_t>((size_t)h->g.V, kAosChunkSites);
    cudaError_t e = cudaMalloc(&h->d_aos, sites * 16 * sizeof(double));
    if (e != cudaSuccess) return check_cuda(h, e, "allocating transfer staging");
    h->aos_sites = sites;
    return SU2G_OK;
}

int su2g::aos_to_field(su2g_lattice* h, const double* d_src, size_t n0, int count)
{
    const int grid = grid_for(h, count, 8);
    launch_begin(h, SU2G_K_OTHER);
    if (h->prec == SU2G_FP32)
        k_aos_in<float><<<grid, kBlock, 0, h->stream>>>((const double2*)d_src, make_field<float>(h->dirp, h->g.Vh), h->g,
                                                       (int)n0, count);
    else
        k_aos_in<double><<<grid, kBlock, 0, h->stream>>>((const double2*)d_src, make_field<double>(h->dirp, h->g.Vh),
                                                        h->g, (int)n0, count);
    return launch_end(h, SU2G_K_OTHER, "layout conversion");
}

int su2g::field_to_aos(su2g_lattice* h, double* d_dst, size_t n0, int count)
{
    const int grid = grid_for(h, count, 8);
    launch_begin(h, SU2G_K_OTHER);
    if (h->prec == SU2G_FP32)
        k_aos_out<float><<<grid, kBlock, 0, h->stream>>>((double2*)d_dst, make_field<float>(h->dirp, h->g.Vh), h->g,
                                                        (int)n0, count);
    else
        k_aos_out<double><<<grid, kBlock, 0, h->stream>>>((double2*)d_dst, make_field<double>(h->dirp, h->g.Vh), h->g,
                                                         (int)n0, count);
    return launch_end(h, SU2G_K_OTHER, "layout conversion");
}

// ------------------------------------------------------------------- C ABI ---

extern "C" const char* su2g_last_error(const su2g_lattice* h) { return h ? h->err : g_create_err; }

extern "C" int su2g_create(const su2g_params* p, su2g_lattice** out)
{
    if (!p || !out) return set_error(nullptr, SU2G_EINVAL, "su2g_create: null argument");
    *out = nullptr;
    long long V = 1;
    for (int d = 0; d < 4; ++d) {
        if (p->dims[d] < 2 || (p->dims[d] & 1))
            return set_error(nullptr, SU2G_EINVAL, "su2g_create: extent %d of direction %d must be even and >= 2",
                             p->dims[d], d);
        V *= p->dims[d];
    }
    if (V > (1ll << 30)) return set_error(nullptr, SU2G_EINVAL, "su2g_create: volume %lld exceeds 2^30 sites", V);
    if (p->precision != SU2G_FP32 && p->precision != SU2G_FP64)
        return set_error(nullptr, SU2G_EINVAL, "su2g_create: unknown precision %d", p->precision);
    if (p->start < SU2G_START_COLD || p->start > SU2G_START_REF)
        return set_error(nullptr, SU2G_EINVAL, "su2g_create: unknown start mode %d", p->start);
    if (p->replica >= (1u << 24)) return set_error(nullptr, SU2G_EINVAL, "su2g_create: replica id >= 2^24");

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
        return set_error(nullptr, SU2G_ENODEV, "su2g_create: no CUDA device visible");
    if (p->device < 0 || p->device >= ndev)
        return set_error(nullptr, SU2G_EINVAL, "su2g_create: device %d out of range (%d devices)", p->device, ndev);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, p->device) != cudaSuccess || prop.major < 10)
        return set_error(nullptr, SU2G_ENODEV, "su2g_create: device %d is not sm_100 class", p->device);
    if (cudaSetDevice(p->device) != cudaSuccess)
        return set_error(nullptr, SU2G_ECUDA, "su2g_create: cudaSetDevice(%d) failed", p->device);

    su2g_lattice* h = new (std::nothrow) su2g_lattice();
    if (!h) return set_error(nullptr, SU2G_ENOMEM, "su2g_create: out of host memory");
    h->g = make_geom(p->dims);
    h->prec = p->precision;
    h->beta = p->beta;
    h->seed = p->seed;
    h->replica = p->replica;
    h->device = p->device;
    h->num_sms = prop.multiProcessorCount;
    h->max_smem = (int)prop.sharedMemPerBlockOptin;
    h->link_bytes = p->precision == SU2G_FP32 ? 16 : 32;

    int rc = SU2G_OK;
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess)
        rc = check_cuda(h, e, "creating stream");
    if (!rc && (e = cudaMalloc(&h->field, 4ull * V * h->link_bytes)) != cudaSuccess)
        rc = check_cuda(h, e, "allocating the gauge field");
    if (!rc)
        for (int mu = 0; mu < 4; ++mu) h->dirp[mu] = (char*)h->field + (size_t)mu * 2 * h->g.Vh * h->link_bytes;
    if (!rc && (e = cudaMalloc(&h->d_out, kOutSlots * sizeof(double))) != cudaSuccess)
        rc = check_cuda(h, e, "allocating result slots");
    if (!rc && (e = cudaMallocHost(&h->h_out, kOutSlots * sizeof(double))) != cudaSuccess)
        rc = check_cuda(h, e, "allocating pinned result slots");
    if (!rc && (e = cudaMalloc(&h->d_status, sizeof(unsigned))) != cudaSuccess)
        rc = check_cuda(h, e, "allocating status word");
    if (!rc) rc = check_cuda(h, cudaMemsetAsync(h->d_status, 0, sizeof(unsigned), h->stream), "clearing status");
    if (!rc && (e = cudaMalloc(&h->fin_blocks, kFinBlocks * sizeof(DD))) != cudaSuccess)
        rc = check_cuda(h, e, "allocating reduction scratch");
    if (!rc && (e = cudaMalloc(&h->fin_ticket, sizeof(unsigned))) != cudaSuccess)
        rc = check_cuda(h, e, "allocating reduction scratch");
    if (!rc) rc = check_cuda(h, cudaMemsetAsync(h->fin_ticket, 0, sizeof(unsigned), h->stream), "clearing reduction counter");
    if (!rc) rc = ensure_partials(h, 2);
    if (!rc) wilson_prepare(h);
    if (!rc) rc = check_cuda(h, cudaEventCreate(&h->ev_begin), "creating events");
    if (!rc) rc = check_cuda(h, cudaEventCreate(&h->ev_end), "creating events");
    if (!rc) rc = su2g_start(h, p->start, p->seed);
    if (!rc) rc = check_cuda(h, cudaStreamSynchronize(h->stream), "initialising the field");
    if (rc) {
        set_error(nullptr, rc, "su2g_create: %s", h->err);
        su2g_destroy(h);
        return rc;
    }
    *out = h;
    return SU2G_OK;
}

extern "C" int su2g_destroy(su2g_lattice* h)
{
    if (!h) return SU2G_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (auto& pe : h->prof_pending) {
        cudaEventDestroy(pe.a);
        cudaEventDestroy(pe.b);
    }
    for (auto e : h->event_pool) cudaEventDestroy(e);
    if (h->ev_begin) cudaEventDestroy(h->ev_begin);
    if (h->ev_end) cudaEventDestroy(h->ev_end);
    release_run_graph(h);
    release_meas_graph(h);
    if (h->pool) cudaMemPoolDestroy(h->pool);
    cudaFree(h->lines);
    cudaFree(h->meas_work);
    cudaFree(h->meas_alt);
    cudaFree(h->d_run_ctr);
    cudaFree(h->d_trace);
    cudaFree(h->field);
    cudaFree(h->field_alt);
    cudaFree(h->partials);
    cudaFree(h->d_out);
    cudaFree(h->d_status);
    cudaFree(h->fin_blocks);
    cudaFree(h->fin_ticket);
    cudaFree(h->d_aos);
    if (h->h_out) cudaFreeHost(h->h_out);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return SU2G_OK;
}

extern "C" int su2g_start(su2g_lattice* h, int32_t start, uint64_t seed)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_start: null handle");
    if (start < SU2G_START_COLD || start > SU2G_START_REF)
        return set_error(h, SU2G_EINVAL, "su2g_start: unknown start mode %d", start);
    cudaSetDevice(h->device);
    h->seed = seed;
    h->hb_sweeps = 0;
    int grid = grid_for(h, 4ll * h->g.V, 8);
    launch_begin(h, SU2G_K_OTHER);
    if (h->prec == SU2G_FP32)
        k_start<float><<<grid, kBlock, 0, h->stream>>>(make_field<float>(h->dirp, h->g.Vh), h->g, start, seed,
                                                      h->replica);
    else
        k_start<double><<<grid, kBlock, 0, h->stream>>>(make_field<double>(h->dirp, h->g.Vh), h->g, start, seed,
                                                        h->replica);
    return launch_end(h, SU2G_K_OTHER, "start kernel");
}

extern "C" int su2g_info(const su2g_lattice* h, int32_t dims[4], int32_t* precision, int64_t* volume,
                         uint32_t* hb_sweeps)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_info: null handle");
    if (dims)
        for (int d = 0; d < 4; ++d) dims[d] = h->g.L[d];
    if (precision) *precision = h->prec;
    if (volume) *volume = h->g.V;
    if (hb_sweeps) *hb_sweeps = h->hb_sweeps;
    return SU2G_OK;
}

extern "C" int su2g_set_beta(su2g_lattice* h, double beta)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_set_beta: null handle");
    if (!(beta >= 0.0) || !std::isfinite(beta)) return set_error(h, SU2G_EINVAL, "su2g_set_beta: bad beta");
    h->beta = beta;
    return SU2G_OK;
}

extern "C" int su2g_set_sweep_counter(su2g_lattice* h, uint32_t hb_sweeps)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_set_sweep_counter: null handle");
    h->hb_sweeps = hb_sweeps;
    return SU2G_OK;
}

extern "C" int su2g_upload_aos_f64(su2g_lattice* h, const double* links)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_upload_aos_f64: null handle");
    if (!links) return set_error(h, SU2G_EINVAL, "su2g_upload_aos_f64: null links");
    cudaSetDevice(h->device);
    int rc = ensure_aos(h);
    if (rc) return rc;
    for (size_t n0 = 0; n0 < (size_t)h->g.V; n0 += h->aos_sites) {
        int cnt = (int)std::min(h->aos_sites, (size_t)h->g.V - n0);
        rc = check_cuda(h, cudaMemcpyAsync(h->d_aos, links + n0 * 16, (size_t)cnt * 16 * sizeof(double),
                                           cudaMemcpyHostToDevice, h->stream),
                        "uploading links");
        if (rc || (rc = aos_to_field(h, h->d_aos, n0, cnt))) return rc;
    }
    return check_cuda(h, cudaStreamSynchronize(h->stream), "uploading links");
}

extern "C" int su2g_download_aos_f64(su2g_lattice* h, double* links)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_download_aos_f64: null handle");
    if (!links) return set_error(h, SU2G_EINVAL, "su2g_download_aos_f64: null links");
    cudaSetDevice(h->device);
    int rc = ensure_aos(h);
    if (rc) return rc;
    for (size_t n0 = 0; n0 < (size_t)h->g.V; n0 += h->aos_sites) {
        int cnt = (int)std::min(h->aos_sites, (size_t)h->g.V - n0);
        if ((rc = field_to_aos(h, h->d_aos, n0, cnt))) return rc;
        rc = check_cuda(h, cudaMemcpyAsync(links + n0 * 16, h->d_aos, (size_t)cnt * 16 * sizeof(double),
                                           cudaMemcpyDeviceToHost, h->stream),
                        "downloading links");
        if (rc) return rc;
    }
    return check_cuda(h, cudaStreamSynchronize(h->stream), "downloading links");
}

extern "C" int su2g_stream(su2g_lattice* h, void** cuda_stream)
{
    if (!h || !cuda_stream) return set_error(h, SU2G_EINVAL, "su2g_stream: null argument");
    *cuda_stream = (void*)h->stream;
    return SU2G_OK;
}

extern "C" int su2g_synchronize(su2g_lattice* h)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_synchronize: null handle");
    return check_cuda(h, cudaStreamSynchronize(h->stream), "synchronising");
}

extern "C" int su2g_timer_begin(su2g_lattice* h)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_timer_begin: null handle");
    return check_cuda(h, cudaEventRecord(h->ev_begin, h->stream), "recording timer event");
}

extern "C" int su2g_timer_end(su2g_lattice* h, double* ms)
{
    if (!h || !ms) return set_error(h, SU2G_EINVAL, "su2g_timer_end: null argument");
    int rc = check_cuda(h, cudaEventRecord(h->ev_end, h->stream), "recording timer event");
    if (!rc) rc = check_cuda(h, cudaEventSynchronize(h->ev_end), "waiting for timer event");
    float f = 0.f;
    if (!rc) rc = check_cuda(h, cudaEventElapsedTime(&f, h->ev_begin, h->ev_end), "reading timer");
    *ms = f;
    return rc;
}

extern "C" int su2g_profile_enable(su2g_lattice* h, int32_t enable)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_profile_enable: null handle");
    drain_profile(h);
    h->profiling = enable != 0;
    for (int k = 0; k < SU2G_K_COUNT; ++k) {
        h->prof_launches[k] = 0;
        h->prof_ms[k] = 0.0;
    }
    return SU2G_OK;
}

extern "C" int su2g_profile_read(su2g_lattice* h, int32_t cls, int64_t* launches, double* ms)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_profile_read: null handle");
    if (cls < 0 || cls >= SU2G_K_COUNT) return set_error(h, SU2G_EINVAL, "su2g_profile_read: bad class %d", cls);
    drain_profile(h);
    if (launches) *launches = h->prof_launches[cls];
    if (ms) *ms = h->prof_ms[cls];
    return SU2G_OK;
}

extern "C" int su2g_host_alloc(size_t bytes, void** ptr)
{
    if (!ptr) return set_error(nullptr, SU2G_EINVAL, "su2g_host_alloc: null argument");
    *ptr = nullptr;
    cudaError_t e = cudaMallocHost(ptr, bytes);
    if (e != cudaSuccess) return check_cuda(nullptr, e, "su2g_host_alloc");
    return SU2G_OK;
}

extern "C" int su2g_host_free(void* ptr)
{
    if (!ptr) return SU2G_OK;
    return check_cuda(nullptr, cudaFreeHost(ptr), "su2g_host_free");
}

extern "C" int su2g_set_kernel_variant(su2g_lattice* h, int32_t kernel_class, int32_t variant)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_set_kernel_variant: null handle");
    if (kernel_class != SU2G_K_APE || variant < 0 || variant > 1)
        return set_error(h, SU2G_EINVAL, "su2g_set_kernel_variant: unknown class/variant (%d, %d)", kernel_class, variant);
    h->ape_variant = variant;
    return SU2G_OK;
}

extern "C" int su2g_kernel_variant(const su2g_lattice* h, int32_t kernel_class, int32_t* active)
{
    if (!h || !active) return set_error(nullptr, SU2G_EINVAL, "su2g_kernel_variant: null argument");
    if (kernel_class != SU2G_K_APE) return set_error(nullptr, SU2G_EINVAL, "su2g_kernel_variant: unknown class");
    const bool tma = h->prec == SU2G_FP32 && h->ape_variant == 1 && ape_tma_rows(h->g, h->max_smem) > 0;
    *active = tma ? 1 : 0;
    return SU2G_OK;
}
