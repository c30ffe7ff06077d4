// stats.cu -- the reference's analysis of measurement series, on the device.
//
// Reference tools: LGT_Code/Autocorrelation/t_int.c:24-74 (integrated autocorrelation time and
// the corrected error of a series) and Analysis/static potential/static_potential.py:28-146 (block
// jackknife of W(R,T), the effective potential V_eff = log(W(T)/W(T+1)) with its bias correction,
// and weighted plateau fits V(R)).  Both run here in FP64 with every sum in the reference's
// index order and no fused multiply-adds, so results equal the sequential restatement bit for
// bit.  Traces produced on the device (a batch's plaquette trace, measurement results) are
// analysed where they are.
#include <cmath>

#include "internal.cuh"

using namespace su2g;

namespace {

// One CTA per series; lags in chunks of blockDim, each thread computes one Gamma(k) with the
// separate window means of t_int.c:32-41; thread 0 adds them up in lag order until the first
// negative one (t_int.c:44-55).
__global__ void __launch_bounds__(kBlock) k_tau_int(const double* __restrict__ x, long long n, long long si,
                                                    long long ss, double* __restrict__ out, int* __restrict__ resolved)
{
    __shared__ double gam[kBlock];
    __shared__ double t_acc, g0, mean;
    __shared__ int done;
    const double* s = x + (size_t)blockIdx.x * ss;
    if (threadIdx.x == 0) done = 0;
    for (long long k0 = 0; k0 < n; k0 += blockDim.x) {
        const long long k = k0 + threadIdx.x;
        double gk = 0.0;
        if (k < n) {
            const long long m = n - k;
            double a = 0.0, b = 0.0, c = 0.0;
            for (long long i = 0; i < m; ++i) a = __dadd_rn(a, s[i * si]);
            for (long long i = k; i < n; ++i) b = __dadd_rn(b, s[i * si]);
            const double a0 = __ddiv_rn(a, (double)m), ak = __ddiv_rn(b, (double)m);
            for (long long i = 0; i < m; ++i)
                c = __dadd_rn(c, __dmul_rn(__dsub_rn(s[i * si], a0), __dsub_rn(s[(i + k) * si], ak)));
            gk = __ddiv_rn(c, (double)m);
            if (k == 0) mean = a0;   // average(array, 0, N)
        }
        gam[threadIdx.x] = gk;
        __syncthreads();
        if (threadIdx.x == 0) {
            long long j = 0;
            if (k0 == 0) {
                g0 = gam[0];
                t_acc = __dmul_rn(0.5, g0);
                j = 1;
            }
            for (; j < (long long)blockDim.x && k0 + j < n; ++j) {
                if (gam[j] < 0.0) {
                    done = 1;
                    break;
                }
                t_acc = __dadd_rn(t_acc, gam[j]);
            }
        }
        __syncthreads();
        if (done) break;
    }
    if (threadIdx.x == 0) {
        const double tau = __ddiv_rn(t_acc, g0);
        const double naive = sqrt(__ddiv_rn(g0, (double)(n - 1)));
        double* o = out + 4 * (size_t)blockIdx.x;
        o[0] = mean;
        o[1] = tau;
        o[2] = naive;
        o[3] = __dmul_rn(sqrt(__dmul_rn(2.0, tau)), naive);
        if (resolved) resolved[blockIdx.x] = (long long)ceil(__dmul_rn(100.0, tau)) <= n;
    }
}

// static_potential.py:80-146 in one CTA.  ws holds the window means [r][t][1 + B] and the
// jackknife samples of V_eff [r][t][B].
__global__ void __launch_bounds__(kBlock) k_veff(const double* __restrict__ w, int n_conf, int n_r, int n_t, int B,
                                                 const int* __restrict__ t0, const int* __restrict__ t1,
                                                 double* __restrict__ ws, double* __restrict__ veff,
                                                 double* __restrict__ veff_err, double* __restrict__ v,
                                                 double* __restrict__ v_err)
{
    const int L = n_conf / B, nt1 = n_t - 1;
    double* wbar = ws;
    double* vj = ws + (size_t)n_r * n_t * (B + 1);
    // means over all configurations and over all but block k (static_potential.py:80-86)
    for (int p = threadIdx.x; p < n_r * n_t; p += blockDim.x) {
        const int r = p / n_t, t = p % n_t;
        double* wb = wbar + (size_t)p * (B + 1);
        double all = 0.0, blk = 0.0;
        for (int c = 0; c < n_conf; ++c) {
            const double x = w[((size_t)c * n_r + r) * n_t + t];
            all = __dadd_rn(all, x);
            const int k = c / L;
            if (k < B) {
                blk = __dadd_rn(blk, x);
                if (c == (k + 1) * L - 1) {
                    wb[1 + k] = blk;   // block sum for now
                    blk = 0.0;
                }
            }
        }
        wb[0] = __ddiv_rn(all, (double)n_conf);
        for (int k = 0; k < B; ++k) wb[1 + k] = __ddiv_rn(__dsub_rn(all, wb[1 + k]), (double)(n_conf - L));
    }
    __syncthreads();
    // V_eff, its jackknife error and bias correction (static_potential.py:90-113)
    for (int p = threadIdx.x; p < n_r * nt1; p += blockDim.x) {
        const int r = p / nt1, t = p % nt1;
        const double* a = wbar + ((size_t)r * n_t + t) * (B + 1);
        const double* b = a + (B + 1);
        const double full = log(__ddiv_rn(a[0], b[0]));
        double s2 = 0.0, sm = 0.0;
        for (int k = 0; k < B; ++k) {
            const double e = log(__ddiv_rn(a[1 + k], b[1 + k]));
            vj[(size_t)p * B + k] = e;
            const double d = __dsub_rn(e, full);
            s2 = __dadd_rn(s2, __dmul_rn(d, d));
            sm = __dadd_rn(sm, e);
        }
        veff_err[p] = sqrt(__dmul_rn(__ddiv_rn((double)(B - 1), (double)B), s2));
        veff[p] = __dsub_rn(full, __dmul_rn((double)(B - 1), __dsub_rn(__ddiv_rn(sm, (double)B), full)));
    }
    __syncthreads();
    // plateau fits (fitting_constant, static_potential.py:28-42, :117-146)
    for (int r = threadIdx.x; r < n_r; r += blockDim.x) {
        const double* ve = veff + (size_t)r * nt1;
        const double* er = veff_err + (size_t)r * nt1;
        double sig = 0.0;
        for (int t = t0[r]; t < t1[r]; ++t) sig = __dadd_rn(sig, __ddiv_rn(1.0, __dmul_rn(er[t], er[t])));
        double a = 0.0;
        for (int t = t0[r]; t < t1[r]; ++t)
            a = __dadd_rn(a, __ddiv_rn(ve[t], __dmul_rn(__dmul_rn(sig, er[t]), er[t])));
        double s2 = 0.0, sm = 0.0;
        for (int k = 0; k < B; ++k) {
            double f = 0.0;
            for (int t = t0[r]; t < t1[r]; ++t)
                f = __dadd_rn(f, __ddiv_rn(vj[((size_t)r * nt1 + t) * B + k], __dmul_rn(__dmul_rn(sig, er[t]), er[t])));
            const double d = __dsub_rn(f, a);
            s2 = __dadd_rn(s2, __dmul_rn(d, d));
            sm = __dadd_rn(sm, f);
        }
        v_err[r] = sqrt(__dmul_rn(__ddiv_rn((double)(B - 1), (double)B), s2));
        v[r] = __dsub_rn(a, __dmul_rn((double)(B - 1), __dsub_rn(__ddiv_rn(sm, (double)B), a)));
    }
}

bool on_device(const void* p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Device buffers freed on scope exit.
struct Scratch {
    std::vector<void*> p;
    ~Scratch()
    {
        for (void* q : p) cudaFree(q);
    }
    template <typename T>
    int alloc(T** out, size_t n)
    {
        void* q = nullptr;
        int rc = check_cuda(nullptr, cudaMalloc(&q, n * sizeof(T)), "allocating statistics scratch");
        if (!rc) p.push_back(q);
        *out = (T*)q;
        return rc;
    }
};

}  // namespace

int su2g::tau_int_enqueue(const double* d_x, long long n, long long si, long long ss, int n_series, cudaStream_t stream,
                          double* d_out, int* d_resolved)
{
    k_tau_int<<<n_series, kBlock, 0, stream>>>(d_x, n, si, ss, d_out, d_resolved);
    return check_cuda(nullptr, cudaGetLastError(), "tau_int kernel");
}

extern "C" int su2g_stats_tau_int(const double* data, int64_t n, int32_t n_series, int64_t stride_i, int64_t stride_s,
                                  int32_t device, double* out, int32_t* resolved)
{
    if (!data || !out || n < 2 || n_series < 1 || stride_i < 1 || stride_s < 0)
        return set_error(nullptr, SU2G_EINVAL, "su2g_stats_tau_int: bad arguments (n >= 2, series >= 1, strides)");
    int rc = check_cuda(nullptr, cudaSetDevice(device), "su2g_stats_tau_int: selecting the device");
    if (rc) return rc;
    Scratch sc;
    const double* d_x = data;
    if (!on_device(data)) {
        // the series' span in memory: the last element is (n-1) stride_i + (n_series-1) stride_s
        const size_t span = (size_t)(n - 1) * stride_i + (size_t)(n_series - 1) * stride_s + 1;
        double* tmp = nullptr;
        if ((rc = sc.alloc(&tmp, span))) return rc;
        if ((rc = check_cuda(nullptr, cudaMemcpy(tmp, data, span * sizeof(double), cudaMemcpyHostToDevice),
                             "su2g_stats_tau_int: copying the series")))
            return rc;
        d_x = tmp;
    }
    double* d_out = nullptr;
    int* d_res = nullptr;
    if ((rc = sc.alloc(&d_out, 4 * (size_t)n_series)) || (rc = sc.alloc(&d_res, (size_t)n_series))) return rc;
    if ((rc = tau_int_enqueue(d_x, n, stride_i, stride_s, n_series, 0, d_out, d_res))) return rc;
    rc = check_cuda(nullptr, cudaMemcpy(out, d_out, 4 * (size_t)n_series * sizeof(double), cudaMemcpyDeviceToHost),
                    "su2g_stats_tau_int: copying results");
    if (!rc && resolved)
        rc = check_cuda(nullptr, cudaMemcpy(resolved, d_res, (size_t)n_series * sizeof(int), cudaMemcpyDeviceToHost),
                        "su2g_stats_tau_int: copying results");
    return rc;
}

extern "C" int su2g_stats_veff(const double* w, int32_t n_conf, int32_t n_r, int32_t n_t, int32_t n_bins,
                               const int32_t* t_fit_start, const int32_t* t_fit_end, int32_t device, double* veff,
                               double* veff_err, double* v, double* v_err)
{
    if (!w || !t_fit_start || !t_fit_end || !veff || !veff_err || !v || !v_err || n_r < 1 || n_t < 2 || n_bins < 2 ||
        n_conf / (n_bins > 0 ? n_bins : 1) < 1)
        return set_error(nullptr, SU2G_EINVAL, "su2g_stats_veff: bad arguments (n_t >= 2, 2 <= n_bins <= n_conf)");
    for (int r = 0; r < n_r; ++r)
        if (t_fit_start[r] < 0 || t_fit_end[r] > n_t - 1 || t_fit_start[r] >= t_fit_end[r])
            return set_error(nullptr, SU2G_EINVAL, "su2g_stats_veff: fit range %d of R index %d outside [0, %d)",
                             t_fit_start[r], r, n_t - 1);
    int rc = check_cuda(nullptr, cudaSetDevice(device), "su2g_stats_veff: selecting the device");
    if (rc) return rc;
    Scratch sc;
    const size_t nw = (size_t)n_conf * n_r * n_t, nt1 = (size_t)n_t - 1;
    const double* d_w = w;
    if (!on_device(w)) {
        double* tmp = nullptr;
        if ((rc = sc.alloc(&tmp, nw))) return rc;
        if ((rc = check_cuda(nullptr, cudaMemcpy(tmp, w, nw * sizeof(double), cudaMemcpyHostToDevice),
                             "su2g_stats_veff: copying the loops")))
            return rc;
        d_w = tmp;
    }
    int *d_t0 = nullptr, *d_t1 = nullptr;
    double *ws = nullptr, *d_ve = nullptr, *d_er = nullptr, *d_v = nullptr, *d_verr = nullptr;
    if ((rc = sc.alloc(&d_t0, n_r)) || (rc = sc.alloc(&d_t1, n_r)) ||
        (rc = sc.alloc(&ws, (size_t)n_r * n_t * (n_bins + 1) + (size_t)n_r * nt1 * n_bins)) ||
        (rc = sc.alloc(&d_ve, n_r * nt1)) || (rc = sc.alloc(&d_er, n_r * nt1)) || (rc = sc.alloc(&d_v, n_r)) ||
        (rc = sc.alloc(&d_verr, n_r)))
        return rc;
    cudaMemcpy(d_t0, t_fit_start, n_r * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(d_t1, t_fit_end, n_r * sizeof(int), cudaMemcpyHostToDevice);
    k_veff<<<1, kBlock>>>(d_w, n_conf, n_r, n_t, n_bins, d_t0, d_t1, ws, d_ve, d_er, d_v, d_verr);
    if ((rc = check_cuda(nullptr, cudaGetLastError(), "su2g_stats_veff: kernel"))) return rc;
    const struct {
        double* dst;
        const double* src;
        size_t n;
    } copies[] = {{veff, d_ve, n_r * nt1}, {veff_err, d_er, n_r * nt1}, {v, d_v, (size_t)n_r}, {v_err, d_verr, (size_t)n_r}};
    for (const auto& c : copies)
        if ((rc = check_cuda(nullptr, cudaMemcpy(c.dst, c.src, c.n * sizeof(double), cudaMemcpyDeviceToHost),
                             "su2g_stats_veff: copying results")))
            return rc;
    return SU2G_OK;
}
