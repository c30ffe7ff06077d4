// su2qcd -- native thermalisation/production driver over libsu2g: the flow of the reference's qcd
// program (LGT_Code/main/qcd.c:26-79) with the sweeps between two configuration writes replayed
// from one CUDA graph (su2g_graph_run) and configurations written from device memory
// (su2g_write_config).
//
//   su2qcd -i qcd.in -d TxXxYxZ [-c cfg | -t cfg] [-p fp64|fp32] [--or N] [--utype 0|1] [--stype 0|1]
//          [--device N]
//
// qcd.in has the keys of readInputFile (LGT_Code/modules/io/inp_IO.c:54-134): outFileId,
// outputDir, start (0 cold, 1 hot with the reference's su2RandomMatrix formula), beta, epsilon,
// nconf, ntherm, ndecorr (read but, as in qcd.c, unused), writeConfFreq, seed.  Output:
// <outputDir>/<T>x<X>x<Y>x<Z>_SU2_b<beta %.6f>_id<outFileId>.log with the reference's start-up block
// (printStartupInfo, inp_IO.c:190-247) and per sweep its update record (update.c:169-173) and
// "plaq\t%.8f" (qcd.c:60); configurations <base>_n<k> after the same sweeps as qcd.c:64-69; an empty
// .out file.  Like the reference it refuses to overwrite an existing .log or .out.
//
// Differences: the extents are a command-line argument (the reference compiles them in); --or N adds
// N overrelaxation sweeps after every heatbath sweep (the reference has none; default 0); the
// random numbers are Philox keyed by `seed`, not RANLUX, so chains agree with the reference's
// statistically; the update record's time is the mean over a graph block.
#include <chrono>
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
    fprintf(stderr, "su2qcd: ");
    vfprintf(stderr, fmt, ap);
    fprintf(stderr, "\n");
    va_end(ap);
    exit(1);
}

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

bool exists(const std::string& p)
{
    FILE* f = fopen(p.c_str(), "r");
    if (f) fclose(f);
    return f != nullptr;
}

std::map<std::string, std::vector<std::string>> read_input(const char* path)
{
    FILE* f = fopen(path, "r");
    if (!f) die("unable to open input file %s", path);
    std::map<std::string, std::vector<std::string>> kv;
    char line[4096];
    while (fgets(line, sizeof line, f)) {
        std::istringstream ss(line);
        std::string key, v;
        if (!(ss >> key)) continue;
        auto& vals = kv[key];
        while (ss >> v) vals.push_back(v);
    }
    fclose(f);
    for (const char* k : {"outFileId", "outputDir", "start", "beta", "epsilon", "nconf", "ntherm", "ndecorr",
                          "writeConfFreq", "seed"})
        if (!kv.count(k) || kv[k].empty()) die("input file: missing field '%s'", k);
    return kv;
}

void usage()
{
    fprintf(stderr,
            "usage: su2qcd -i <qcd.in> -d TxXxYxZ [-c cfg | -t cfg] [-p fp64|fp32] [--or N] [--utype 0|1]\n"
            "              [--stype 0|1] [--device N]\n");
    exit(2);
}

}  // namespace

int main(int argc, char** argv)
{
    const char *input = nullptr, *cfg = nullptr;
    bool reflect = false, have_dims = false;
    int32_t dims[4] = {0, 0, 0, 0};
    int precision = SU2G_FP64, device = 0, n_or = 0, utype = 1, stype = 0;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto next = [&]() -> const char* {
            if (i + 1 >= argc) usage();
            return argv[++i];
        };
        if (a == "-i") input = next();
        else if (a == "-c" || a == "-t") {
            if (cfg) usage();
            cfg = next();
            reflect = a == "-t";
        } else if (a == "-d") have_dims = sscanf(next(), "%dx%dx%dx%d", &dims[0], &dims[1], &dims[2], &dims[3]) == 4;
        else if (a == "-p") {
            const std::string p = next();
            if (p == "fp64") precision = SU2G_FP64;
            else if (p == "fp32") precision = SU2G_FP32;
            else usage();
        } else if (a == "--or") n_or = atoi(next());
        else if (a == "--utype") utype = atoi(next());
        else if (a == "--stype") stype = atoi(next());
        else if (a == "--device") device = atoi(next());
        else usage();
    }
    if (!input || !have_dims || n_or < 0 || (utype != 0 && utype != 1) || (stype != 0 && stype != 1)) usage();
    auto kv = read_input(input);
    auto I = [&](const char* k) { return atoi(kv[k][0].c_str()); };
    auto D = [&](const char* k) { return atof(kv[k][0].c_str()); };
    const int id = I("outFileId"), start = I("start"), nconf = I("nconf"), ntherm = I("ntherm");
    const int ndecorr = I("ndecorr"), wfreq = I("writeConfFreq"), seed = I("seed");
    const double beta = D("beta"), eps = D("epsilon");
    const std::string dir = kv["outputDir"][0];

    char base[512];
    snprintf(base, sizeof base, "%dx%dx%dx%d_SU2_b%.6f_id%d", dims[0], dims[1], dims[2], dims[3], beta, id);
    const std::string stem = dir + "/" + base;
    g_log = stem + ".log";
    if (exists(g_log)) die("try to overwrite existing .log file %s", g_log.c_str());
    if (exists(stem + ".out")) die("try to overwrite existing .out file %s.out", stem.c_str());
    for (const std::string& f : {g_log, stem + ".out"}) {
        FILE* fp = fopen(f.c_str(), "w");
        if (!fp) die("unable to create %s", f.c_str());
        fclose(fp);
    }
    // printStartupInfo (inp_IO.c:190-247)
    logging("*******************************\nLATTICE QCD CODE\n*******************************\n"
            "Global parameters:\n*******************************\n");
    logging("Using a four -dimensional lattice:\nlatt  :\t%dx%dx%dx%d\n", dims[0], dims[1], dims[2], dims[3]);
    logging("beta :\t%.6f\nepsilon :\t%.6f\nnconf :\t%d\nndecorr :\t%d\nntherm :\t%d\nwriteConfFreq :\t%d\nseed :\t%d\n",
            beta, eps, nconf, ndecorr, ntherm, wfreq, seed);
    logging("*******************************\nInline measurements:\nNone at the moment!\n"
            "*******************************\n");
    logging("Start from \"%s\" configuration:\n*******************************\n", cfg ? cfg : "");

    su2g_params p;
    memset(&p, 0, sizeof p);
    for (int i = 0; i < 4; ++i) p.dims[i] = dims[i];
    p.precision = precision;
    p.start = start ? SU2G_START_REF : SU2G_START_COLD;
    p.beta = beta;
    p.seed = (uint64_t)(uint32_t)seed;
    p.device = device;
    su2g_lattice* h = nullptr;
    if (su2g_create(&p, &h)) die("%s", su2g_last_error(nullptr));
    if (cfg) {
        double p0 = 0, p1 = 0;
        const double t1 = now();
        logging(reflect ? "\nReading configuration for thermalisation %s:\n" : "\nReading configuration %s:\n", cfg);
        check(h, reflect ? su2g_read_config_reflect(h, cfg, &p0, &p1) : su2g_read_config(h, cfg, &p0, &p1),
              "reading the start configuration");
        printf("read plaq %.6e, calc plaq %.6e\n", p0, p1);
        logging(reflect ? "\nConfiguration imported for thermalisation(took %.3e sec)!\n"
                        : "\nConfiguration imported (took %.3e sec)!\n",
                now() - t1);
    }

    // sweeps n whose end writes a configuration (qcd.c:64): n > ntherm, (n - ntherm + 1) % wfreq == 0
    auto writes_after = [&](int n) { return wfreq > 0 && n > ntherm && (n - ntherm + 1) % wfreq == 0; };
    std::vector<double> plaq, acc;
    int nw = 0;
    for (int n0 = 0; n0 < nconf;) {
        int n1 = n0;
        while (n1 < nconf - 1 && !writes_after(n1)) ++n1;   // block n0..n1 ends at a write or the last sweep
        const int nb = n1 - n0 + 1;
        plaq.assign(nb, 0.0);
        acc.assign(nb, 0.0);
        const double t1 = now();
        if (utype == 1 && stype == 0) {
            check(h, su2g_graph_run(h, nb, 1, 1, n_or, plaq.data(), acc.data()), "sweeping");
        } else {
            for (int b = 0; b < nb; ++b) {
                check(h, su2g_gauge_update(h, 1, utype, stype, eps, 1, &acc[b]), "sweeping");
                if (n_or) check(h, su2g_sweep(h, 1, 0, n_or, nullptr), "overrelaxation");
                check(h, su2g_plaquette(h, &plaq[b]), "plaquette");
            }
        }
        const double per = (now() - t1) / nb;
        for (int b = 0; b < nb; ++b) {
            const int n = n0 + b;
            logging("\nUpdate %d done:\n(algorithm %d; sweep %d; acc=%.3f)\nupdate took %.9f seconds\n", n + 1, utype,
                    stype, acc[b], per);
            logging("plaq\t%.8f\n", plaq[b]);
            if (writes_after(n)) {
                ++nw;
                const std::string f = stem + "_n" + std::to_string(nw);
                const double tw = now();
                logging("\nWriting configuration %s:\n", f.c_str());
                check(h, su2g_write_config(h, f.c_str(), nullptr), "writing a configuration");
                logging("\nConfiguration exported (took %.3e sec)!\n", now() - tw);
            }
            printf("\nSweep %d done (took %.3e sec)!\n", n, per);
        }
        n0 = n1 + 1;
    }
    su2g_destroy(h);
    return 0;
}
