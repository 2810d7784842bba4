// Command-line driver over the FastLBP reference's public API, compiled with
// the reference sources into oracle/_ref/ref_bp by oracle/Makefile. It runs
// the reference's own GPU FP64 CausalBP (updates=PARALL, or the schedule in
// the environment variable REF_BP_UPDATES: SEQFIX or TOPO) the way
// examples/fl_wrapper.cu does: read the graph, clamp by label, rebuild the
// graph from its factors, construct, init, run.
//
// TEST / BASELINE INFRASTRUCTURE ONLY (golden vectors and the benchmark's
// reference arm).
//
//   ref_bp <graph.causal_fg> <clamps.txt|-> <out.txt|-> fixed  <sweeps>
//   ref_bp <graph.causal_fg> <clamps.txt|-> <out.txt|-> tol    <tol> <maxiter>
//   ref_bp <graph.causal_fg> <clamps.txt|-> <out.txt|-> lowpass <tol> <min> <max> <hist>
//   (append "repeat <n>" to time n construct+init+run repetitions)
//
// clamps.txt holds "label 0|1" lines. out.txt receives "label belief" lines at
// 17 significant digits (newBelief() for fixed/lowpass, belief() for tol).
// One JSON line with timings goes to stdout.

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include <ext/causal_bp.h>
#include <lbp/properties.h>
#include <utils/utils.h>

using namespace lbp;

int main(int argc, char **argv) {
    if (argc < 6) {
        fprintf(stderr, "usage: ref_bp graph clamps out mode args...\n");
        return 2;
    }
    std::string graph = argv[1], clampf = argv[2], outf = argv[3], mode = argv[4];
    int a = 5;
    double tol = 1e-6;
    size_t n1 = 0, n2 = 0, n3 = 0;
    if (mode == "fixed") {
        n1 = std::stoull(argv[a++]);
    } else if (mode == "tol") {
        tol = std::stod(argv[a++]);
        n1 = std::stoull(argv[a++]);
    } else if (mode == "lowpass") {
        tol = std::stod(argv[a++]);
        n1 = std::stoull(argv[a++]);
        n2 = std::stoull(argv[a++]);
        n3 = std::stoull(argv[a++]);
    } else {
        fprintf(stderr, "bad mode\n");
        return 2;
    }
    int repeat = 1;
    if (a + 1 < argc && std::string(argv[a]) == "repeat") repeat = std::atoi(argv[a + 1]);

    cudaFree(0);
    double t0 = toc();
    CausalFactorGraph fg;
    fg.ReadFromFile(graph.c_str());
    double t_read = toc() - t0;

    std::map<size_t, size_t> clamps;
    if (clampf != "-") {
        std::ifstream in(clampf);
        long lab, val;
        while (in >> lab >> val) clamps[(size_t)lab] = (size_t)val;
    }
    for (auto &c : clamps)
        for (size_t i = 0; i < fg.nrVars(); i++)
            if (fg.var(i).label() == c.first) fg.clamp(i, c.second);
    CausalFactorGraph nfg(fg.factors());

    PropertySet opts;
    opts.set("maxiter", n1 ? n1 : (size_t)10000);
    opts.set("maxtime", Real(57600));
    opts.set("tol", Real(tol));
    opts.set("verbose", (size_t)(getenv("REF_BP_VERBOSE") ? 1 : 0));
    const char *upd = getenv("REF_BP_UPDATES");
    opts.set("updates", std::string(upd ? upd : "PARALL"));
    opts.set("logdomain", false);

    double best_construct = 1e30, best_run = 1e30, best_run_ev = 1e30;
    std::vector<double> all_construct, all_run_ev;
    double ret = 0;
    std::unique_ptr<CausalBP> bp;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int r = 0; r < repeat; r++) {
        bp.reset();
        cudaDeviceSynchronize();
        double c0 = toc();
        bp.reset(new CausalBP(nfg, opts));
        bp->init();
        cudaDeviceSynchronize();
        double c1 = toc();
        cudaEventRecord(e0);
        if (mode == "fixed") ret = bp->run(tol, n1, 1);
        else if (mode == "tol") bp->run();
        else ret = bp->run(tol, n1, n2, n3);
        cudaEventRecord(e1);
        cudaDeviceSynchronize();
        double c2 = toc();
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        best_construct = std::min(best_construct, c1 - c0);
        best_run = std::min(best_run, c2 - c1);
        best_run_ev = std::min(best_run_ev, (double)ms / 1e3);
        all_construct.push_back(c1 - c0);
        all_run_ev.push_back((double)ms / 1e3);
    }
    std::string runs = "[", cons = "[";
    for (size_t r = 0; r < all_run_ev.size(); r++) {
        runs += (r ? ", " : "") + std::to_string(all_run_ev[r]);
        cons += (r ? ", " : "") + std::to_string(all_construct[r]);
    }
    runs += "]";
    cons += "]";
    cudaError_t err = cudaGetLastError();

    if (outf != "-") {
        FILE *f = fopen(outf.c_str(), "w");
        for (size_t i = 0; i < nfg.nrVars(); i++) {
            double b = (mode == "tol") ? bp->belief(VarSet(nfg.var(i)))[1] : bp->newBelief(i);
            fprintf(f, "%zu %.17g\n", nfg.var(i).label(), b);
        }
        fclose(f);
    }
    size_t E = 0;
    for (size_t I = 0; I < nfg.nrFactors(); I++) E += nfg.factor(I).vars().size();
    printf("{\"vars\": %zu, \"factors\": %zu, \"slots\": %zu, \"read_s\": %.6f, \"construct_s\": %.6f, "
           "\"run_s\": %.6f, \"run_event_s\": %.6f, \"ret\": %.17g, \"repeat\": %d, \"cuda\": \"%s\", "
           "\"run_event_all_s\": %s, \"construct_all_s\": %s}\n",
           nfg.nrVars(), nfg.nrFactors(), E, t_read, best_construct, best_run, best_run_ev, ret, repeat,
           cudaGetErrorString(err), runs.c_str(), cons.c_str());
    return err == cudaSuccess ? 0 : 1;
}
