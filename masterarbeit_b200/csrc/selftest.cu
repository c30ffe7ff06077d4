// selftest.cu -- failure detection on the device without a GPU fault.  One CTA arms an mbarrier
// for a bulk copy that is never issued and waits on it with the library's bounded wait; the wait
// runs out, the kernel records the timeout in the handle's status word and returns, and the host
// reports it at the next synchronising call.  No copy is in flight, so nothing can land after the
// kernel has returned.
#include "internal.cuh"
#include "mbarrier.cuh"

using namespace su2g;

namespace {

__global__ void k_bounded_wait(uint32_t limit, unsigned* __restrict__ status)
{
    __shared__ alignas(8) unsigned long long bar;
    const uint32_t b = smem_addr(&bar);
    if (threadIdx.x == 0) {
        mbar_init(b, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) mbar_expect_tx(b, 16u);   // arrival done, 16 bytes expected that never come
    __syncthreads();
    const bool ok = mbar_wait_bounded(b, 0u, limit);
    if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicOr(status, kStatusTmaTimeout);
}

}  // namespace

extern "C" int su2g_selftest_bounded_wait(su2g_lattice* h, uint32_t poll_limit)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_selftest_bounded_wait: null handle");
    if (poll_limit < 1 || poll_limit > (1u << 22))
        return set_error(h, SU2G_EINVAL, "su2g_selftest_bounded_wait: poll limit %u outside [1, 2^22]", poll_limit);
    cudaSetDevice(h->device);
    launch_begin(h, SU2G_K_OTHER);
    k_bounded_wait<<<1, 64, 0, h->stream>>>(poll_limit, h->d_status);
    int rc = launch_end(h, SU2G_K_OTHER, "bounded-wait self-test");
    if (!rc) rc = fetch_results(h, 0, 0);
    return rc;
}
