// config_io.cu -- configuration files in the reference's binary format, streamed between the file
// and the device field.
//
// Reference: writeConfig / readConfig / readConfigForThermalisation
// (LGT_Code/modules/io/config_IO.c:40-117, :537-621, :348-535).  The file is
//   int32 {DIM = 4, SUN = 2}, int32 {L_t, L_x, L_y, L_z}, double plaquette,
//   then for every site n (lexicographic) and direction mu the doubles c0..c3 of U_mu(n).
// The reference byte-swaps on big-endian hosts, so its files are little-endian everywhere.
//
// The body moves in chunks through two pinned host buffers and the two halves of the handle's
// AoS staging: while the GPU copies and converts chunk k, the host reads (or writes) chunk k+1
// (k-1).  After reading, the plaquette is checked against the header as readConfig does
// (config_IO.c:612-614): |P - P_file| <= sqrt(6 V) DBL_EPSILON.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "internal.cuh"

using namespace su2g;

namespace {

bool little_endian()
{
    const uint32_t one = 1;
    unsigned char b;
    std::memcpy(&b, &one, 1);
    return b == 1;
}

struct File {
    FILE* f = nullptr;
    ~File()
    {
        if (f) fclose(f);
    }
};

struct Pinned {
    double* p = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    ~Pinned()
    {
        if (p) cudaFreeHost(p);
        for (auto e : ev)
            if (e) cudaEventDestroy(e);
    }
    int init(su2g_lattice* h, size_t doubles)
    {
        int rc = check_cuda(h, cudaHostAlloc((void**)&p, doubles * sizeof(double), cudaHostAllocDefault),
                            "allocating pinned file buffers");
        for (auto& e : ev)
            if (!rc) rc = check_cuda(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "creating events");
        return rc;
    }
};

int read_header(su2g_lattice* h, FILE* f, const char* path, const int32_t expect[4], double* plaq0)
{
    int32_t info[2], dims[4];
    double plaq = 0.0;
    // the fields are read one by one: the file has no padding between the int32s and the double
    if (fread(info, sizeof(int32_t), 2, f) != 2 || fread(dims, sizeof(int32_t), 4, f) != 4 ||
        fread(&plaq, sizeof(double), 1, f) != 1)
        return set_error(h, SU2G_EFILE, "%s: read error in the header", path);
    if (info[0] != 4 || info[1] != 2)
        return set_error(h, SU2G_EFILE, "%s: incompatible parameters (dimension %d, SU(%d))", path, info[0], info[1]);
    for (int mu = 0; mu < 4; ++mu)
        if (dims[mu] != expect[mu])
            return set_error(h, SU2G_EFILE, "%s: incompatible lattice size (%dx%dx%dx%d, expected %dx%dx%dx%d)", path,
                             dims[0], dims[1], dims[2], dims[3], expect[0], expect[1], expect[2], expect[3]);
    *plaq0 = plaq;
    return SU2G_OK;
}

// Read `nsites` sites of links from f and hand each chunk, once on the device, to consume(d, n0, cnt).
template <typename F>
int stream_in(su2g_lattice* h, FILE* f, const char* path, size_t nsites, F&& consume)
{
    int rc = ensure_aos(h);
    if (rc) return rc;
    const size_t chunk = std::max<size_t>(1, h->aos_sites / 2);
    Pinned buf;
    if ((rc = buf.init(h, 2 * chunk * 16))) return rc;
    size_t k = 0;
    for (size_t n0 = 0; n0 < nsites && !rc; n0 += chunk, ++k) {
        const int b = (int)(k & 1);
        const size_t cnt = std::min(chunk, nsites - n0);
        double* hb = buf.p + b * chunk * 16;
        double* db = h->d_aos + b * chunk * 16;
        // host buffer b is free once the copy out of it (two chunks ago) has run; the device half b
        // is free by stream order (its conversion kernel precedes this copy)
        if (k >= 2 && (rc = check_cuda(h, cudaEventSynchronize(buf.ev[b]), "waiting for a copy"))) break;
        if (fread(hb, 16 * sizeof(double), cnt, f) != cnt) {
            rc = set_error(h, SU2G_EFILE, "%s: read error (file shorter than the lattice)", path);
            break;
        }
        rc = check_cuda(h, cudaMemcpyAsync(db, hb, cnt * 16 * sizeof(double), cudaMemcpyHostToDevice, h->stream),
                        "copying links");
        if (!rc) rc = check_cuda(h, cudaEventRecord(buf.ev[b], h->stream), "recording an event");
        if (!rc) rc = consume(db, n0, (int)cnt);
    }
    const int rs = check_cuda(h, cudaStreamSynchronize(h->stream), "reading a configuration");
    return rc ? rc : rs;
}

int check_plaquette(su2g_lattice* h, const char* path, double plaq0, double* plaq_file, double* plaq)
{
    double p = 0.0;
    int rc = su2g_plaquette(h, &p);
    if (rc) return rc;
    if (plaq_file) *plaq_file = plaq0;
    if (plaq) *plaq = p;
    const double eps = h->prec == SU2G_FP64 ? std::sqrt(6.0 * (double)h->g.V) * DBL_EPSILON : 1e-5;
    if (!(std::fabs(p - plaq0) <= eps))
        return set_error(h, SU2G_EFILE, "%s: plaquette test failed (file %.15e, computed %.15e)", path, plaq0, p);
    return SU2G_OK;
}

// readConfigForThermalisation (config_IO.c:348-535).  Image k (0..15) mirrors direction j when
// bit j of k is set.  In image k the link U_mu(c) of small-lattice site c lands at the site X of
// the full lattice with, per direction j,
//   X_j = L_j - c_j - 1                      if j == mu and j is mirrored (the link is reversed),
//   X_j = (c_j == 0 ? L_j / 2 : L_j - c_j)   if j != mu and j is mirrored,
//   X_j = c_j                                otherwise,
// and holds U_mu(c)^dag when mu is mirrored.  Every full-lattice link is written exactly once.
template <typename R>
__global__ void __launch_bounds__(kBlock) k_reflect_in(const double2* __restrict__ aos, Field<R> U, Geom g, int n0,
                                                       int count)
{
    int hl[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) hl[j] = g.L[j] / 2;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        int rem = n0 + i, c[4];
#pragma unroll
        for (int j = 3; j >= 0; --j) {
            c[j] = rem % hl[j];
            rem /= hl[j];
        }
        const double2* src = aos + (size_t)i * 8;
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) {
            const double2 a = src[2 * mu], b = src[2 * mu + 1];
            const Q<R> u = q_make<R>((R)a.x, (R)a.y, (R)b.x, (R)b.y);
            const Q<R> ud = q_dag(u);
            for (int k = 0; k < 16; ++k) {
                int n = 0, psum = 0;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    int x = c[j];
                    if ((k >> j) & 1) x = j == mu ? g.L[j] - c[j] - 1 : (c[j] == 0 ? hl[j] : g.L[j] - c[j]);
                    n += x * g.S[j];
                    psum += x;
                }
                U.sth(mu, psum & 1, n >> 1, ((k >> mu) & 1) ? ud : u);
            }
        }
    }
}

}  // namespace

extern "C" int su2g_read_config(su2g_lattice* h, const char* path, double* plaq_file, double* plaq)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_read_config: null handle");
    if (!path) return set_error(h, SU2G_EINVAL, "su2g_read_config: null path");
    if (!little_endian()) return set_error(h, SU2G_EFILE, "su2g_read_config: big-endian hosts are not supported");
    cudaSetDevice(h->device);
    File f;
    if (!(f.f = fopen(path, "rb"))) return set_error(h, SU2G_EFILE, "unable to read input file %s", path);
    double plaq0 = 0.0;
    int rc = read_header(h, f.f, path, h->g.L, &plaq0);
    if (rc) return rc;
    rc = stream_in(h, f.f, path, (size_t)h->g.V,
                   [h](const double* d, size_t n0, int cnt) { return aos_to_field(h, d, n0, cnt); });
    if (rc) return rc;
    return check_plaquette(h, path, plaq0, plaq_file, plaq);
}

extern "C" int su2g_read_config_reflect(su2g_lattice* h, const char* path, double* plaq_file, double* plaq)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_read_config_reflect: null handle");
    if (!path) return set_error(h, SU2G_EINVAL, "su2g_read_config_reflect: null path");
    if (!little_endian())
        return set_error(h, SU2G_EFILE, "su2g_read_config_reflect: big-endian hosts are not supported");
    cudaSetDevice(h->device);
    int32_t half[4];
    for (int mu = 0; mu < 4; ++mu) {
        if (h->g.L[mu] % 2) return set_error(h, SU2G_EINVAL, "su2g_read_config_reflect: odd extent %d", h->g.L[mu]);
        half[mu] = h->g.L[mu] / 2;
    }
    File f;
    if (!(f.f = fopen(path, "rb"))) return set_error(h, SU2G_EFILE, "unable to read input file %s", path);
    double plaq0 = 0.0;
    int rc = read_header(h, f.f, path, half, &plaq0);
    if (rc) return rc;
    const size_t vsmall = (size_t)h->g.V / 16;
    rc = stream_in(h, f.f, path, vsmall, [h](const double* d, size_t n0, int cnt) {
        const int grid = grid_for(h, cnt, 8);
        launch_begin(h, SU2G_K_OTHER);
        if (h->prec == SU2G_FP32)
            k_reflect_in<float><<<grid, kBlock, 0, h->stream>>>((const double2*)d, make_field<float>(h->dirp, h->g.Vh),
                                                                h->g, (int)n0, cnt);
        else
            k_reflect_in<double><<<grid, kBlock, 0, h->stream>>>((const double2*)d,
                                                                 make_field<double>(h->dirp, h->g.Vh), h->g, (int)n0,
                                                                 cnt);
        return launch_end(h, SU2G_K_OTHER, "reflection");
    });
    if (rc) return rc;
    return check_plaquette(h, path, plaq0, plaq_file, plaq);
}

extern "C" int su2g_write_config(su2g_lattice* h, const char* path, double* plaq)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_write_config: null handle");
    if (!path) return set_error(h, SU2G_EINVAL, "su2g_write_config: null path");
    if (!little_endian()) return set_error(h, SU2G_EFILE, "su2g_write_config: big-endian hosts are not supported");
    cudaSetDevice(h->device);
    double p = 0.0;
    int rc = su2g_plaquette(h, &p);
    if (rc) return rc;
    if (plaq) *plaq = p;
    if ((rc = ensure_aos(h))) return rc;
    File f;
    if (!(f.f = fopen(path, "wb"))) return set_error(h, SU2G_EFILE, "unable to create output file %s", path);
    const int32_t info[2] = {4, 2};
    if (fwrite(info, sizeof(int32_t), 2, f.f) != 2 || fwrite(h->g.L, sizeof(int32_t), 4, f.f) != 4 ||
        fwrite(&p, sizeof(double), 1, f.f) != 1)
        return set_error(h, SU2G_EFILE, "%s: write error", path);
    const size_t chunk = std::max<size_t>(1, h->aos_sites / 2), V = (size_t)h->g.V;
    Pinned buf;
    if ((rc = buf.init(h, 2 * chunk * 16))) return rc;
    size_t prev_cnt = 0;
    // iteration k enqueues chunk k (conversion into staging half b, copy into host buffer b) and
    // then writes chunk k-1 to the file while chunk k is in flight; one extra iteration flushes
    for (size_t n0 = 0, k = 0; !rc; n0 += chunk, ++k) {
        const int b = (int)(k & 1);
        const size_t cnt = n0 < V ? std::min(chunk, V - n0) : 0;
        if (cnt) {
            double* db = h->d_aos + b * chunk * 16;
            rc = field_to_aos(h, db, n0, (int)cnt);
            if (!rc)
                rc = check_cuda(h, cudaMemcpyAsync(buf.p + b * chunk * 16, db, cnt * 16 * sizeof(double),
                                                   cudaMemcpyDeviceToHost, h->stream),
                                "copying links");
            if (!rc) rc = check_cuda(h, cudaEventRecord(buf.ev[b], h->stream), "recording an event");
        }
        if (!rc && prev_cnt) {
            const int pb = 1 - b;
            rc = check_cuda(h, cudaEventSynchronize(buf.ev[pb]), "waiting for a copy");
            if (!rc && fwrite(buf.p + pb * chunk * 16, 16 * sizeof(double), prev_cnt, f.f) != prev_cnt)
                rc = set_error(h, SU2G_EFILE, "%s: write error", path);
        }
        prev_cnt = cnt;
        if (!cnt) break;
    }
    const int rs = check_cuda(h, cudaStreamSynchronize(h->stream), "writing a configuration");
    if (rc || rs) return rc ? rc : rs;
    if (fflush(f.f) != 0) return set_error(h, SU2G_EFILE, "%s: write error", path);
    return SU2G_OK;
}
