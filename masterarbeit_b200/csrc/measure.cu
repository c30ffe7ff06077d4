// measure.cu -- one configuration's measurement of the meas / qtop drivers as one CUDA graph.
//
// Reference flow (LGT_Code/main_meas/meas.c:93-126; LGT_Code/main_qtop/qtop.c:76-91):
//   charge:  readConfig, smearing_APE_all(ism_tc, smpar_tc), topologicalCharge
//            (qtop.c: Q after every APE_all step from N_APE_start to N_APE_finish);
//   loops:   readConfig again, smearing_APE_temporal(ismt, smpart), smearing_APE_spatial(isms,
//            smpars), measureWilsonLoop.
// Here the field is read once (by the caller) and each branch smears a device copy, so the
// handle's field is left as it was.  The sequence -- copies, smearing steps, charges, loop
// chunks and their reductions -- is captured once per measurement spec and replayed for every
// configuration; the results come back with one copy.
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.cuh"

using namespace su2g;

struct su2g_meas_graph {
    cudaGraphExec_t exec = nullptr;
    std::vector<int32_t> q_ape, R, T;
    double alpha_q = 0, alpha_t = 0, alpha_s = 0;
    int ns_t = 0, ns_s = 0;
    void* dirp[4] = {nullptr, nullptr, nullptr, nullptr};
    const void* partials = nullptr;
    int ape_variant = 0;
    std::vector<int> wslot;   // d_out slot of each loop
    int nres = 0;             // d_out slots to fetch
};

namespace {

int ensure_work(su2g_lattice* h)
{
    if (h->meas_work) return SU2G_OK;
    const size_t bytes = 4ull * h->g.V * h->link_bytes;
    int rc = check_cuda(h, cudaMalloc(&h->meas_work, bytes), "allocating the measurement field");
    if (!rc) rc = check_cuda(h, cudaMalloc(&h->meas_alt, bytes), "allocating the measurement field");
    if (rc) {
        cudaFree(h->meas_work);
        cudaFree(h->meas_alt);
        h->meas_work = h->meas_alt = nullptr;
    }
    return rc;
}

void work_dirs(su2g_lattice* h, void* base, void* dirs[4])
{
    for (int mu = 0; mu < 4; ++mu) dirs[mu] = (char*)base + (size_t)mu * 2 * h->g.Vh * h->link_bytes;
}

int copy_field(su2g_lattice* h, void* const dst[4])
{
    const size_t bytes = 2ull * h->g.Vh * h->link_bytes;
    for (int mu = 0; mu < 4; ++mu) {
        int rc = check_cuda(h, cudaMemcpyAsync(dst[mu], h->dirp[mu], bytes, cudaMemcpyDeviceToDevice, h->stream),
                            "copying the field");
        if (rc) return rc;
    }
    return SU2G_OK;
}

int enqueue_measurement(su2g_lattice* h, su2g_meas_graph& m)
{
    int rc = SU2G_OK;
    void *cur[4], *alt[4];
    const int nq = (int)m.q_ape.size(), nw = (int)m.R.size();
    if (nq) {
        work_dirs(h, h->meas_work, cur);
        work_dirs(h, h->meas_alt, alt);
        if ((rc = copy_field(h, cur))) return rc;
        int done = 0;
        for (int i = 0; i < nq; ++i) {
            if ((rc = ape_run(h, cur, alt, m.q_ape[i] - done, SU2G_APE_ALL, m.alpha_q))) return rc;
            done = m.q_ape[i];
            // Q and sum |q| into d_out[2i], d_out[2i + 1]
            if ((rc = qtop_enqueue(h, cur, 2 * i))) return rc;
        }
    }
    if (nw) {
        work_dirs(h, h->meas_work, cur);
        work_dirs(h, h->meas_alt, alt);
        if ((rc = copy_field(h, cur))) return rc;
        if ((rc = ape_run(h, cur, alt, m.ns_t, SU2G_APE_TEMPORAL, m.alpha_t))) return rc;
        if ((rc = ape_run(h, cur, alt, m.ns_s, SU2G_APE_SPATIAL, m.alpha_s))) return rc;
        m.wslot.assign(nw, 0);
        const int off = 2 * nq;
        if ((rc = wilson_enqueue(h, cur, m.R.data(), m.T.data(), nw, off, kOutSlots - 2 - off, m.wslot.data())))
            return rc;
    }
    m.nres = 2 * nq;
    for (int s : m.wslot) m.nres = std::max(m.nres, s + 1);
    return SU2G_OK;
}

bool same(const su2g_meas_graph& m, const su2g_lattice* h, const su2g_meas_spec* sp)
{
    if (!m.exec || m.ape_variant != h->ape_variant || m.partials != h->partials) return false;
    for (int mu = 0; mu < 4; ++mu)
        if (m.dirp[mu] != h->dirp[mu]) return false;
    if ((int)m.q_ape.size() != sp->n_q || (int)m.R.size() != sp->n_w) return false;
    if (sp->n_q && (m.alpha_q != sp->alpha_q || std::memcmp(m.q_ape.data(), sp->q_ape, sp->n_q * sizeof(int32_t))))
        return false;
    if (sp->n_w && (m.ns_t != sp->ns_t || m.ns_s != sp->ns_s || m.alpha_t != sp->alpha_t || m.alpha_s != sp->alpha_s ||
                    std::memcmp(m.R.data(), sp->R, sp->n_w * sizeof(int32_t)) ||
                    std::memcmp(m.T.data(), sp->T, sp->n_w * sizeof(int32_t))))
        return false;
    return true;
}

int capture(su2g_lattice* h, const su2g_meas_spec* sp)
{
    release_meas_graph(h);
    auto* m = new su2g_meas_graph;
    m->q_ape.assign(sp->q_ape, sp->q_ape + sp->n_q);
    m->R.assign(sp->R, sp->R + sp->n_w);
    m->T.assign(sp->T, sp->T + sp->n_w);
    m->alpha_q = sp->alpha_q;
    m->alpha_t = sp->alpha_t;
    m->alpha_s = sp->alpha_s;
    m->ns_t = sp->ns_t;
    m->ns_s = sp->ns_s;
    m->ape_variant = h->ape_variant;
    for (int mu = 0; mu < 4; ++mu) m->dirp[mu] = h->dirp[mu];
    const bool prof = h->profiling;
    h->profiling = false;   // no per-launch events inside the graph
    int rc = check_cuda(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal),
                        "beginning graph capture");
    cudaGraph_t graph = nullptr;
    if (!rc) {
        rc = enqueue_measurement(h, *m);
        const cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
        if (!rc) rc = check_cuda(h, e, "ending graph capture");
    }
    h->profiling = prof;
    if (!rc) rc = check_cuda(h, cudaGraphInstantiate(&m->exec, graph, 0), "instantiating the measurement graph");
    if (graph) cudaGraphDestroy(graph);
    if (rc) {
        cudaGetLastError();
        delete m;
        return rc;
    }
    m->partials = h->partials;
    h->meas = m;
    return SU2G_OK;
}

}  // namespace

void su2g::release_meas_graph(su2g_lattice* h)
{
    if (!h->meas) return;
    if (h->meas->exec) cudaGraphExecDestroy(h->meas->exec);
    delete h->meas;
    h->meas = nullptr;
}

extern "C" int su2g_measure(su2g_lattice* h, const su2g_meas_spec* sp, double* q, double* w)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_measure: null handle");
    if (!sp || sp->n_q < 0 || sp->n_w < 0 || (sp->n_q && (!sp->q_ape || !q)) || (sp->n_w && (!sp->R || !sp->T || !w)))
        return set_error(h, SU2G_EINVAL, "su2g_measure: bad specification");
    if (sp->n_q == 0 && sp->n_w == 0) return SU2G_OK;
    for (int i = 0; i < sp->n_q; ++i)
        if (sp->q_ape[i] < 0 || (i && sp->q_ape[i] < sp->q_ape[i - 1]))
            return set_error(h, SU2G_EINVAL, "su2g_measure: APE step counts must be >= 0 and ascending");
    if (sp->n_w && (sp->ns_t < 0 || sp->ns_s < 0))
        return set_error(h, SU2G_EINVAL, "su2g_measure: negative smearing steps");
    if (!std::isfinite(sp->alpha_q) || !std::isfinite(sp->alpha_t) || !std::isfinite(sp->alpha_s))
        return set_error(h, SU2G_EINVAL, "su2g_measure: smearing parameter not finite");
    int rc = sp->n_w ? wilson_check(h, sp->R, sp->T, sp->n_w, "su2g_measure") : SU2G_OK;
    if (rc) return rc;
    if (2 * sp->n_q > kOutSlots - 2) return set_error(h, SU2G_EINVAL, "su2g_measure: too many charges");
    cudaSetDevice(h->device);
    if (!h->meas || !same(*h->meas, h, sp)) {
        // everything the graph uses is allocated before the capture starts
        if ((rc = ensure_work(h))) return rc;
        if ((rc = ensure_partials(h, 8 * 32))) return rc;
        if ((rc = ensure_partial_entries(h, 2 * (size_t)((h->g.V + kBlock - 1) / kBlock)))) return rc;
        if (sp->n_q > 0 && (rc = ensure_lines(h))) return rc;
        if ((rc = capture(h, sp))) return rc;
    }
    if ((rc = check_cuda(h, cudaGraphLaunch(h->meas->exec, h->stream), "replaying the measurement graph"))) return rc;
    if ((rc = fetch_results(h, 0, h->meas->nres))) return rc;
    for (int i = 0; i < sp->n_q; ++i) q[i] = h->h_out[2 * i];
    for (int i = 0; i < sp->n_w; ++i) w[i] = h->h_out[h->meas->wslot[i]];
    return SU2G_OK;
}

extern "C" int su2g_measure_release(su2g_lattice* h)
{
    if (!h) return set_error(nullptr, SU2G_EINVAL, "su2g_measure_release: null handle");
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    release_meas_graph(h);
    cudaFree(h->meas_work);
    cudaFree(h->meas_alt);
    h->meas_work = h->meas_alt = nullptr;
    return SU2G_OK;
}
