// ctypes-facing wrapper around the FastLBP reference's own graph model
// (CausalFactorGraph / CausalFactor / BipartiteGraph), compiled from the
// reference sources into oracle/_ref/ by oracle/Makefile.
//
// TEST INFRASTRUCTURE ONLY: it pins the oracle's reader, graph construction
// and clamping against the reference itself, on the CPU. The array layouts
// match the orc_* functions of causal_bp_oracle.cpp so tests can compare the
// two element by element.

#include <cstdint>
#include <string>
#include <vector>

#include <ext/causal_fg.h>

using lbp::CausalFactorGraph;

extern "C" {

void *ref_read_file(const char *path) {
    auto *g = new CausalFactorGraph();
    g->ReadFromFile(path);
    return g;
}

void ref_free(void *g) { delete (CausalFactorGraph *)g; }

void ref_clamp(void *g, int64_t i, int64_t x) { ((CausalFactorGraph *)g)->clamp((size_t)i, (size_t)x); }

// fl_wrapper's rebuild step: CausalFactorGraph(causal_fg.factors()).
void *ref_rebuild(void *g) { return new CausalFactorGraph(((CausalFactorGraph *)g)->factors()); }

int64_t ref_nr_vars(void *g) { return (int64_t)((CausalFactorGraph *)g)->nrVars(); }
int64_t ref_nr_factors(void *g) { return (int64_t)((CausalFactorGraph *)g)->nrFactors(); }
int64_t ref_nr_edges(void *g) { return (int64_t)((CausalFactorGraph *)g)->nrEdges(); }

void ref_vars(void *g, int64_t *labels) {
    auto &G = *(CausalFactorGraph *)g;
    for (size_t i = 0; i < G.nrVars(); i++) labels[i] = (int64_t)G.var(i).label();
}

void ref_factor_info(void *g, int32_t *type, int64_t *head, double *p, double *q, int32_t *clamped, double *m0,
                     double *m1, int64_t *nvars) {
    auto &G = *(CausalFactorGraph *)g;
    for (size_t I = 0; I < G.nrFactors(); I++) {
        const auto &f = G.factor(I);
        type[I] = f.type();
        head[I] = (int64_t)f.head().label();
        p[I] = f.prob();
        q[I] = f.prob_default();
        clamped[I] = f.head_clamped ? 1 : 0;
        m0[I] = f.head_mask[0];
        m1[I] = f.head_mask[1];
        nvars[I] = (int64_t)f.vars().size();
    }
}

void ref_factor_vars(void *g, int64_t *off, int64_t *labels) {
    auto &G = *(CausalFactorGraph *)g;
    int64_t k = 0;
    off[0] = 0;
    for (size_t I = 0; I < G.nrFactors(); I++) {
        for (const auto &v : G.factor(I).vars()) labels[k++] = (int64_t)v.label();
        off[I + 1] = k;
    }
}

void ref_neighbors(void *g, int which_factor, int64_t *off, int64_t *node, int64_t *iter, int64_t *dual) {
    auto &G = *(CausalFactorGraph *)g;
    size_t n = which_factor ? G.nrFactors() : G.nrVars();
    int64_t k = 0;
    off[0] = 0;
    for (size_t a = 0; a < n; a++) {
        const auto &nb = which_factor ? G.nbF(a) : G.nbV(a);
        for (const auto &x : nb) {
            node[k] = (int64_t)x.node;
            iter[k] = (int64_t)x.iter;
            dual[k] = (int64_t)x.dual;
            k++;
        }
        off[a + 1] = k;
    }
}

}  // extern "C"
