// noalloc.cu -- APE smearing in place on a caller-owned device field, without allocating.
//
// Who this is for: programs that hold their gauge field in device memory they got from somewhere
// else and may not call cudaMalloc themselves -- e.g. a host program whose device memory is handed
// out by another component (a framework's memory pool, or a fixed per-process budget that must
// account for every byte), or a steady-state measurement loop that must not pay the implicit
// device-wide synchronisation of cudaMalloc/cudaFree.  Such a caller cannot create a su2g handle
// (su2g_create allocates the field, the reduction scratch and a pinned result buffer), so this
// entry point works directly on the caller's buffer.
//
// A Jacobi smearing step reads the old field while it writes the new one, so it needs room for a
// second field.  That room is the file-scope array g_noalloc_scratch below: kNoAllocMaxSites
// sites of FP64 links (48 MiB).  Every GPU that loads this library reserves it for the lifetime
// of the process.  All calls share it; calls that overlap on the GPU (different streams, or
// different host threads without ordering) race on it and must not be issued.
#include <mutex>

#include "internal.cuh"

using namespace su2g;

namespace {

// Largest lattice (sites) the static scratch holds: 393216 sites x 4 links x 4 doubles = 48 MiB.
// 24^4 = 331776 sites fits; 26^4 = 456976 does not.
constexpr long long kNoAllocMaxSites = 393216;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxSites * 16];

constexpr int kMaxDevices = 64;
std::mutex g_setup_lock;
void* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on the current device.  In host code the array's name is
// only a host-side stand-in, so the address is looked up once per device (with that device
// current) and cached; a kernel is always given this looked-up address.  The cache lives as long
// as the process: after cudaDeviceReset the module is loaded again and the array may move, so a
// program that resets a device must not call this entry point afterwards (restart the process).
int scratch_address(int dev, void** out)
{
    if (dev < 0 || dev >= kMaxDevices)
        return set_error(nullptr, SU2G_EINVAL, "su2g_ape_inplace_noalloc: device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_setup_lock);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return set_error(nullptr, SU2G_ECUDA, "su2g_ape_inplace_noalloc: cudaGetSymbolAddress failed: %s",
                             cudaGetErrorString(e));
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return SU2G_OK;
}

// A link of the reference's host layout double[V][4][4] (site, direction, c0..c3) on the device.
__device__ __forceinline__ Q<double> aos_ld(const double2* f, int n, int mu)
{
    const double2* a = f + 2 * ((size_t)n * 4 + mu);
    double2 x = a[0], y = a[1];
    return q_make<double>(x.x, x.y, y.x, y.y);
}

__device__ __forceinline__ void aos_st(double2* f, int n, int mu, const Q<double>& q)
{
    double2* a = f + 2 * ((size_t)n * 4 + mu);
    a[0] = make_double2(q.c0, q.c1);
    a[1] = make_double2(q.c2, q.c3);
}

__device__ __forceinline__ bool updates(int mode, int mu)
{
    return mode == SU2G_APE_ALL ? true : (mode == SU2G_APE_SPATIAL ? mu != 0 : mu == 0);
}

// One Jacobi step from `src` into `dst` (both AoS FP64): the links of the smeared directions
// become Proj(U + alpha S) with the staples of smearing.c:42-71; the other directions are copied,
// so that `dst` is complete whatever the scratch held before.
__global__ void __launch_bounds__(kBlock) k_ape_aos(const double2* __restrict__ src, double2* __restrict__ dst,
                                                    Geom g, int mode, double alpha)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.V) return;
    uint32_t t = fdiv((uint32_t)n, g.dS0);
    uint32_t r = (uint32_t)n - t * (uint32_t)g.S[0];
    uint32_t x = fdiv(r, g.dS1);
    r -= x * (uint32_t)g.S[1];
    uint32_t y = fdiv(r, g.dS2);
    uint32_t z = r - y * (uint32_t)g.S[2];
    const int c[4] = {(int)t, (int)x, (int)y, (int)z};
    for (int mu = 0; mu < 4; ++mu) {
        const Q<double> u = aos_ld(src, n, mu);
        if (!updates(mode, mu)) {
            aos_st(dst, n, mu, u);
            continue;
        }
        const int np = n + up_off_rt(g, c, mu);
        Q<double> S = q_zero<double>();
        for (int nu = 0; nu < 4; ++nu) {
            if (nu == mu || (mode != SU2G_APE_ALL && nu == 0)) continue;
            const int nn = n + up_off_rt(g, c, nu);
            const int nm = n + dn_off_rt(g, c, nu);
            // U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag
            S = q_add(S, q_mul_nd(q_mul(aos_ld(src, n, nu), aos_ld(src, nn, mu)), aos_ld(src, np, nu)));
            // U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu)
            S = q_add(S, q_mul(q_mul_dn(aos_ld(src, nm, nu), aos_ld(src, nm, mu)), aos_ld(src, nm + (np - n), nu)));
        }
        aos_st(dst, n, mu, q_project(q_axpy(alpha, S, u)));
    }
}

__global__ void __launch_bounds__(kBlock) k_copy_aos(const double2* __restrict__ src, double2* __restrict__ dst,
                                                     long long n2)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n2) dst[i] = src[i];
}

}  // namespace

extern "C" int su2g_ape_inplace_noalloc(double* links, const int32_t dims[4], int32_t ns, double alpha, int32_t mode,
                                        void* cuda_stream)
{
    if (!links || !dims) return set_error(nullptr, SU2G_EINVAL, "su2g_ape_inplace_noalloc: null argument");
    long long V = 1;
    for (int d = 0; d < 4; ++d) {
        if (dims[d] < 2 || (dims[d] & 1))
            return set_error(nullptr, SU2G_EINVAL,
                             "su2g_ape_inplace_noalloc: extent %d of direction %d must be even and >= 2", dims[d], d);
        V *= dims[d];
    }
    if (V > kNoAllocMaxSites)
        return set_error(nullptr, SU2G_EINVAL,
                         "su2g_ape_inplace_noalloc: lattice of %lld sites exceeds the static scratch of %lld sites "
                         "(48 MiB); use a su2g handle (su2g_create + su2g_ape) for larger lattices",
                         V, kNoAllocMaxSites);
    if (ns < 0 || mode < SU2G_APE_ALL || mode > SU2G_APE_TEMPORAL || !(alpha == alpha))
        return set_error(nullptr, SU2G_EINVAL, "su2g_ape_inplace_noalloc: bad argument (ns=%d, mode=%d)", ns, mode);
    if (ns == 0) return SU2G_OK;

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return set_error(nullptr, SU2G_ECUDA, "su2g_ape_inplace_noalloc: %s", cudaGetErrorString(e));
    // The kernels read and write the field as double2, so it must be 16-byte aligned device (or
    // managed) memory of the current device.  Callers hand in sub-allocations of their own pools,
    // so a bad pointer is refused here instead of faulting on the GPU.  Neither check allocates.
    if (((uintptr_t)links & 15u) != 0)
        return set_error(nullptr, SU2G_EINVAL,
                         "su2g_ape_inplace_noalloc: field pointer %p is not 16-byte aligned", (void*)links);
    cudaPointerAttributes pa;
    e = cudaPointerGetAttributes(&pa, links);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(nullptr, SU2G_EINVAL, "su2g_ape_inplace_noalloc: cannot query pointer %p: %s", (void*)links,
                         cudaGetErrorString(e));
    }
    if ((pa.type != cudaMemoryTypeDevice && pa.type != cudaMemoryTypeManaged) ||
        (pa.type == cudaMemoryTypeDevice && pa.device != dev))
        return set_error(nullptr, SU2G_EINVAL,
                         "su2g_ape_inplace_noalloc: field pointer %p is not device memory of the current device %d",
                         (void*)links, dev);
    void* scratch = nullptr;
    int rc = scratch_address(dev, &scratch);
    if (rc) return rc;

    const Geom g = make_geom(dims);
    cudaStream_t st = (cudaStream_t)cuda_stream;
    const int grid = (int)((V + kBlock - 1) / kBlock);
    double2* field = reinterpret_cast<double2*>(links);
    double2* tmp = reinterpret_cast<double2*>(scratch);
    for (int step = 0; step < ns; ++step) {
        const double2* src = (step & 1) ? tmp : field;
        double2* dst = (step & 1) ? field : tmp;
        k_ape_aos<<<grid, kBlock, 0, st>>>(src, dst, g, mode, alpha);
    }
    if (ns & 1) {   // the last level is in the scratch: copy it back into the caller's field
        const long long n2 = V * 8;
        k_copy_aos<<<(int)((n2 + kBlock - 1) / kBlock), kBlock, 0, st>>>(tmp, field, n2);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return set_error(nullptr, SU2G_ECUDA, "su2g_ape_inplace_noalloc: launch failed: %s", cudaGetErrorString(e));
    return SU2G_OK;
}
