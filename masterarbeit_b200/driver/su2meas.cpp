// su2meas -- native measurement driver over libsu2g: the flows of the reference's meas and qtop
// programs (LGT_Code/main_meas/meas.c:38-133, LGT_Code/main_qtop/qtop.c:17-99) with every
// configuration read straight into device memory (su2g_read_config) and each configuration's
// smearing + charge + Wilson-loop sequence replayed from one CUDA graph (su2g_measure).
//
//   su2meas -i meas.in -d TxXxYxZ [-p fp64|fp32] [--device N]
//       reads the reference's meas input file (keys of readInputFileForMeas, inp_IO.c:250-360) and
//       writes <odir>/<T>x<X>x<Y>x<Z>_SU2_b<beta %.6f>_id<outFileId>.meas with the reference's lines:
//       "QTOP %.8e", "WIL %d %d\t%.8e" and the progress lines around them.  The configuration is read
//       once per number (the reference reads it once per observable), so its reading lines appear once.
//   su2meas --qtop <dir> -d TxXxYxZ [--beta 2.3] [--alpha 0.1] [--ape 0:20:1] [--conf 1:1:1] [--id 1]
//       the qtop program: "QTOP %d %d %e %+.8e" for every APE_all step count of the range; the
//       defaults are the values qtop.c hard-codes.
//
// Differences from the reference's programs: the lattice extents are a command-line argument (the
// reference compiles them in, headers.h:22-25); Q is normalised with pi (the reference's meas never
// sets its global PI and logs "QTOP inf"); two-point functions (mcorrs) are not on this path and
// are refused.
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "su2g.h"

namespace {

std::string g_log;

void die(const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    fprintf(stderr, "su2meas: ");
    vfprintf(stderr, fmt, ap);
    fprintf(stderr, "\n");
    va_end(ap);
    exit(1);
}

// Append one formatted record to the .meas file (the reference's logging(), IO_utils.c:47-58).
void logging(const char* fmt, ...)
{
    FILE* f = fopen(g_log.c_str(), "a");
    if (!f) die("unable to open %s", g_log.c_str());
    va_list ap;
    va_start(ap, fmt);
    vfprintf(f, fmt, ap);
    va_end(ap);
    fclose(f);
}

double now()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

void check(su2g_lattice* h, int rc, const char* what)
{
    if (rc) die("%s: %s", what, su2g_last_error(h));
}

bool parse_dims(const char* s, int32_t d[4])
{
    return sscanf(s, "%dx%dx%dx%d", &d[0], &d[1], &d[2], &d[3]) == 4;
}

// "a:b:c" -> a, b, c
bool parse_range(const char* s, int& a, int& b, int& c)
{
    return sscanf(s, "%d:%d:%d", &a, &b, &c) == 3 && c > 0 && b >= a;
}

std::string base_name(const int32_t d[4], double beta, int id)
{
    char buf[256];
    snprintf(buf, sizeof buf, "%dx%dx%dx%d_SU2_b%.6f_id%d", d[0], d[1], d[2], d[3], beta, id);
    return buf;
}

su2g_lattice* open_lattice(const int32_t dims[4], int precision, int device)
{
    su2g_params p;
    memset(&p, 0, sizeof p);
    for (int i = 0; i < 4; ++i) p.dims[i] = dims[i];
    p.precision = precision;
    p.start = SU2G_START_COLD;
    p.seed = 1;
    p.device = device;
    su2g_lattice* h = nullptr;
    if (su2g_create(&p, &h)) die("%s", su2g_last_error(nullptr));
    return h;
}

// readConfig's log and stdout lines (config_IO.c:549, :613, :620) around su2g_read_config.
void read_config(su2g_lattice* h, const std::string& file)
{
    const double t1 = now();
    logging("\nReading configuration %s:\n", file.c_str());
    double p0 = 0, p = 0;
    check(h, su2g_read_config(h, file.c_str(), &p0, &p), "reading a configuration");
    printf("read plaq %.6e, calc plaq %.6e\n", p0, p);
    logging("\nConfiguration imported (took %.3e sec)!\n", now() - t1);
}

// meas.in: "key values..." per line, the keys of readInputFileForMeas.
struct MeasInput {
    std::map<std::string, std::vector<std::string>> kv;
    const std::vector<std::string>& get(const char* key, size_t n) const
    {
        auto it = kv.find(key);
        if (it == kv.end() || it->second.size() < n) die("input file: missing or short field '%s'", key);
        return it->second;
    }
    int i(const char* key, size_t k = 0) const { return atoi(get(key, k + 1)[k].c_str()); }
    double d(const char* key, size_t k = 0) const { return atof(get(key, k + 1)[k].c_str()); }
};

MeasInput read_input(const char* path)
{
    FILE* f = fopen(path, "r");
    if (!f) die("unable to open input file %s", path);
    MeasInput in;
    char line[4096];
    while (fgets(line, sizeof line, f)) {
        std::istringstream ss(line);
        std::string key, v;
        if (!(ss >> key)) continue;
        auto& vals = in.kv[key];
        while (ss >> v) vals.push_back(v);
    }
    fclose(f);
    return in;
}

int run_meas(const char* input, const int32_t dims[4], int precision, int device)
{
    const MeasInput in = read_input(input);
    const int id = in.i("outFileId");
    const std::string odir = in.get("odir", 1)[0];
    const double beta = in.d("beta");
    const int sconf = in.i("sconf"), fconf = in.i("fconf"), econf = in.i("econf");
    const int mtop = in.i("mtopcharge");
    const int ism_tc = in.i("smear_tc", 0);
    const double smpar_tc = in.d("smear_tc", 1);
    const int mwil = in.i("mwil", 0), mode = in.i("mwil", 1);
    const int ismt = in.i("tSmear", 0), isms = in.i("rSmear", 0);
    const double smpart = in.d("tSmear", 1), smpars = in.d("rSmear", 1);
    if (in.kv.count("mcorrs") && in.i("mcorrs"))
        die("two-point functions (mcorrs 1) are not on the GPU path; run the reference's meas for them");
    if (econf <= 0) die("econf must be positive");
    // loop pairs: a grid (mwil_mode <= 0, inp_IO.c:316-330) or an explicit list
    std::vector<int32_t> R, T;
    if (mwil) {
        if (mode <= 0) {
            const int ts = in.i("tLoopExtent", 0), tf = in.i("tLoopExtent", 1), dt = in.i("tLoopExtent", 2);
            const int rs = in.i("rLoopExtent", 0), rf = in.i("rLoopExtent", 1), dr = in.i("rLoopExtent", 2);
            if (dt <= 0 || dr <= 0) die("loop extent steps must be positive");
            const int nt = (tf - ts) / dt + 1, nr = (rf - rs) / dr + 1;
            for (int a = 0; a < nr; ++a)
                for (int b = 0; b < nt; ++b) {
                    R.push_back(rs + a * dr);
                    T.push_back(ts + b * dt);
                }
        } else {
            for (int k = 0; k < mode; ++k) {
                T.push_back(in.i("tLoopExtent", k));
                R.push_back(in.i("rLoopExtent", k));
            }
        }
    }
    const std::string base = base_name(dims, beta, id);
    g_log = odir + "/" + base + ".meas";
    FILE* f = fopen(g_log.c_str(), "w");
    if (!f) die("unable to create %s", g_log.c_str());
    fclose(f);

    su2g_lattice* h = open_lattice(dims, precision, device);
    const int32_t q_ape[1] = {ism_tc};
    su2g_meas_spec spec;
    memset(&spec, 0, sizeof spec);
    spec.n_q = mtop ? 1 : 0;
    spec.q_ape = q_ape;
    spec.alpha_q = smpar_tc;
    spec.n_w = (int32_t)R.size();
    spec.R = R.data();
    spec.T = T.data();
    spec.ns_t = ismt;
    spec.alpha_t = smpart;
    spec.ns_s = isms;
    spec.alpha_s = smpars;
    std::vector<double> w(R.size());
    for (int n = sconf; n <= fconf; n += econf) {
        const std::string cfg = odir + "/" + base + "_n" + std::to_string(n);
        logging("\nMeasuring on configuration:\n %s\n", cfg.c_str());
        const double t1 = now();
        read_config(h, cfg);
        double q = 0.0;
        const double tm = now();
        if (spec.n_q || spec.n_w) check(h, su2g_measure(h, &spec, &q, w.data()), "measuring");
        if (spec.n_q) {
            logging("calculating topological charge ..\n");
            logging("measurement done (took %.3e sec)\n", now() - tm);
            logging("QTOP %.8e\n", q);
        }
        for (size_t k = 0; k < w.size(); ++k) logging("WIL %d %d\t%.8e\n", R[k], T[k], w[k]);
        logging("\nMeasurement complete (took %.3e sec)\n\n", now() - t1);
    }
    su2g_destroy(h);
    return 0;
}

int run_qtop(const char* dir, const int32_t dims[4], int precision, int device, double beta, double alpha, int a0,
             int a1, int as, int c0, int c1, int cs, int id)
{
    g_log = std::string(dir) + "/" + base_name(dims, beta, id) + ".meas";
    FILE* f = fopen(g_log.c_str(), "w");
    if (!f) die("unable to create %s", g_log.c_str());
    fclose(f);
    su2g_lattice* h = open_lattice(dims, precision, device);
    std::vector<int32_t> q_ape;
    for (int N = a0; N <= a1; N += as) q_ape.push_back(N);
    su2g_meas_spec spec;
    memset(&spec, 0, sizeof spec);
    spec.n_q = (int32_t)q_ape.size();
    spec.q_ape = q_ape.data();
    spec.alpha_q = alpha;
    std::vector<double> q(q_ape.size());
    for (int n = c0; n <= c1; n += cs) {
        const double t1 = now();
        const std::string cfg = std::string(dir) + "/" + base_name(dims, beta, id) + "_n" + std::to_string(n);
        printf("Configuration : %04d\n%s\n", n, cfg.c_str());
        logging("measuring on Configuration %s", cfg.c_str());
        read_config(h, cfg);
        const double tm = now();
        check(h, su2g_measure(h, &spec, q.data(), nullptr), "measuring");
        const double per = (now() - tm) / (double)q.size();
        for (size_t k = 0; k < q.size(); ++k) {
            logging("calculating topological charge ..\n");
            logging("measurement done (took %.3e sec)\n", per);
            logging("QTOP %d %d %e %+.8e\n", n, q_ape[k], alpha, q[k]);
        }
        logging("measurement took %.3e sec\n\n", now() - t1);
    }
    su2g_destroy(h);
    return 0;
}

void usage()
{
    fprintf(stderr,
            "usage: su2meas -i <meas.in> -d TxXxYxZ [-p fp64|fp32] [--device N]\n"
            "       su2meas --qtop <dir> -d TxXxYxZ [--beta 2.3] [--alpha 0.1] [--ape 0:20:1] [--conf 1:1:1]\n"
            "               [--id 1] [-p fp64|fp32] [--device N]\n");
    exit(2);
}

}  // namespace

int main(int argc, char** argv)
{
    const char *input = nullptr, *qdir = nullptr;
    int32_t dims[4] = {0, 0, 0, 0};
    bool have_dims = false;
    int precision = SU2G_FP64, device = 0, id = 1;
    double beta = 2.3, alpha = 0.1;
    int a0 = 0, a1 = 20, as = 1, c0 = 1, c1 = 1, cs = 1;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto next = [&]() -> const char* {
            if (i + 1 >= argc) usage();
            return argv[++i];
        };
        if (a == "-i") input = next();
        else if (a == "--qtop") qdir = next();
        else if (a == "-d") have_dims = parse_dims(next(), dims);
        else if (a == "-p") {
            const std::string p = next();
            if (p == "fp64") precision = SU2G_FP64;
            else if (p == "fp32") precision = SU2G_FP32;
            else usage();
        } else if (a == "--device") device = atoi(next());
        else if (a == "--beta") beta = atof(next());
        else if (a == "--alpha") alpha = atof(next());
        else if (a == "--id") id = atoi(next());
        else if (a == "--ape") {
            if (!parse_range(next(), a0, a1, as)) usage();
        } else if (a == "--conf") {
            if (!parse_range(next(), c0, c1, cs)) usage();
        } else usage();
    }
    if (!have_dims || (!input == !qdir)) usage();
    if (input) return run_meas(input, dims, precision, device);
    return run_qtop(qdir, dims, precision, device, beta, alpha, a0, a1, as, c0, c1, cs, id);
}
