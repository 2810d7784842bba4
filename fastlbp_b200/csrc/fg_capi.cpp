// Graph-model half of the C ABI (flbp_fg_*): the CausalFactorGraph of the
// C++ API behind an opaque handle, for callers without C++.

#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include <ext/causal_fg.h>

#include "../../include/fastlbp_b200.h"
#include "engine_internal.h"
#include "model_internal.h"

struct flbp_fg {
    lbp::CausalFactorGraph g;
};

namespace {

template <class F>
int guarded(F &&f) {
    try {
        return f();
    } catch (const lbp::detail::BadFactorType &) {
        flbp::set_error("Unreachable: factor type must be 'I', '*' or '+'");
        return FLBP_ERR_INVALID;
    } catch (const std::bad_alloc &) {
        flbp::set_error("host allocation failed");
        return FLBP_ERR_NOMEM;
    } catch (const std::exception &e) {
        flbp::set_error(std::string("malformed input: ") + e.what());
        return FLBP_ERR_INVALID;
    }
}

}  // namespace

extern "C" {

int flbp_fg_read_file(const char *path, flbp_fg **out) {
    if (!path || !out) {
        flbp::set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    *out = nullptr;
    return guarded([&] {
        std::ifstream in(path);
        if (!in.is_open()) {
            flbp::set_error(std::string("Cannot read from file ") + path + ".");
            return FLBP_ERR_INVALID;
        }
        auto *h = new flbp_fg{lbp::detail::read_causal_fg_file(in)};
        *out = h;
        return FLBP_OK;
    });
}

int flbp_fg_read_string(const char *text, flbp_fg **out) {
    if (!text || !out) {
        flbp::set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    *out = nullptr;
    return guarded([&] {
        *out = new flbp_fg{lbp::detail::parse_causal_fg_text(text, std::strlen(text))};
        return FLBP_OK;
    });
}

int flbp_fg_from_factors(int64_t n, const int32_t *type, const int64_t *head, const int64_t *body_off,
                         const int64_t *body, const double *p, const double *q, flbp_fg **out) {
    if (!out || n < 0 || (n > 0 && (!type || !head || !body_off || !p || !q))) {
        flbp::set_error("null or invalid argument");
        return FLBP_ERR_INVALID;
    }
    *out = nullptr;
    return guarded([&] {
        std::vector<lbp::CausalFactor> facs;
        facs.reserve((size_t)n);
        for (int64_t I = 0; I < n; I++) {
            const lbp::Var h((size_t)head[I], 2);
            if (type[I] == FLBP_SINGLETON) {
                facs.emplace_back(h, p[I]);
            } else if (type[I] == FLBP_AND || type[I] == FLBP_OR) {
                std::vector<lbp::Var> bv;
                for (int64_t k = body_off[I]; k < body_off[I + 1]; k++) bv.emplace_back((size_t)body[k], 2);
                facs.emplace_back(h, lbp::VarSet(bv.begin(), bv.end(), bv.size()), type[I] == FLBP_AND, p[I], q[I]);
            } else {
                flbp::set_error("unknown factor type at factor " + std::to_string(I));
                return FLBP_ERR_INVALID;
            }
        }
        *out = new flbp_fg{lbp::CausalFactorGraph(facs)};
        return FLBP_OK;
    });
}

int flbp_fg_destroy(flbp_fg *fg) {
    delete fg;
    return FLBP_OK;
}

int flbp_fg_clamp(flbp_fg *fg, int64_t i, int64_t x) {
    if (!fg || i < 0 || (size_t)i >= fg->g.nrVars() || (x != 0 && x != 1)) {
        flbp::set_error("clamp needs a valid variable index and a value of 0 or 1");
        return FLBP_ERR_INVALID;
    }
    return guarded([&] {
        fg->g.clamp((size_t)i, (size_t)x);
        return FLBP_OK;
    });
}

int flbp_fg_rebuild(const flbp_fg *fg, flbp_fg **out) {
    if (!fg || !out) {
        flbp::set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    return guarded([&] {
        *out = new flbp_fg{lbp::CausalFactorGraph(fg->g.factors())};
        return FLBP_OK;
    });
}

int flbp_fg_sizes(const flbp_fg *fg, int64_t *c) {
    if (!fg || !c) {
        flbp::set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    int64_t slots = 0;
    for (const auto &f : fg->g.factors()) slots += (int64_t)f.vars().size();
    c[0] = (int64_t)fg->g.nrVars();
    c[1] = (int64_t)fg->g.nrFactors();
    c[2] = (int64_t)fg->g.nrEdges();
    c[3] = slots;
    return FLBP_OK;
}

int flbp_fg_var_labels(const flbp_fg *fg, int64_t *labels, int64_t n) {
    if (!fg || !labels || n != (int64_t)fg->g.nrVars()) {
        flbp::set_error("labels buffer must hold one entry per variable");
        return FLBP_ERR_INVALID;
    }
    for (int64_t i = 0; i < n; i++) labels[i] = (int64_t)fg->g.var((size_t)i).label();
    return FLBP_OK;
}

int flbp_fg_factors(const flbp_fg *fg, int32_t *type, int64_t *head, double *p, double *q, int32_t *clamped,
                    double *mask0, double *mask1, int64_t *vars_off, int64_t *vars) {
    if (!fg) {
        flbp::set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    const auto &G = fg->g;
    int64_t k = 0;
    if (vars_off) vars_off[0] = 0;
    for (size_t I = 0; I < G.nrFactors(); I++) {
        const auto &f = G.factor(I);
        if (type) type[I] = f.type();
        if (head) head[I] = (int64_t)f.head().label();
        if (p) p[I] = f.prob();
        if (q) q[I] = f.prob_default();
        if (clamped) clamped[I] = f.head_clamped ? 1 : 0;
        if (mask0) mask0[I] = f.head_mask[0];
        if (mask1) mask1[I] = f.head_mask[1];
        for (const auto &v : f.vars()) {
            if (vars) vars[k] = (int64_t)v.label();
            k++;
        }
        if (vars_off) vars_off[I + 1] = k;
    }
    return FLBP_OK;
}

int flbp_fg_neighbors(const flbp_fg *fg, int32_t which, int64_t *off, int64_t *node, int64_t *iter, int64_t *dual) {
    if (!fg || !off || !node || !iter || !dual) {
        flbp::set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    const auto &G = fg->g;
    const size_t n = which ? G.nrFactors() : G.nrVars();
    int64_t k = 0;
    off[0] = 0;
    for (size_t a = 0; a < n; a++) {
        const auto &nb = which ? G.nbF(a) : G.nbV(a);
        for (const auto &x : nb) {
            node[k] = (int64_t)x.node;
            iter[k] = (int64_t)x.iter;
            dual[k] = (int64_t)x.dual;
            k++;
        }
        off[a + 1] = k;
    }
    return FLBP_OK;
}

int flbp_fg_construct(const flbp_fg *fg, int64_t *factor_offsets, int64_t *slot_var, int64_t *factor_head,
                      int64_t *row_ptr_fv, int64_t *col_ind_fv) {
    if (!fg) {
        flbp::set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    return guarded([&] {
        lbp::detail::GraphArrays a;
        std::string err;
        if (lbp::detail::build_arrays(fg->g, a, err)) {
            flbp::set_error(err);
            return FLBP_ERR_INVALID;
        }
        const size_t F = a.offsets.size() - 1, E = a.slot_var.size(), V = fg->g.nrVars();
        if (factor_offsets) std::copy(a.offsets.begin(), a.offsets.end(), factor_offsets);
        if (slot_var) std::copy(a.slot_var.begin(), a.slot_var.end(), slot_var);
        if (factor_head) std::copy(a.head.begin(), a.head.end(), factor_head);
        // Variable-major CSR: a stable counting sort of the factor-major slots by variable
        // (coo2csr of csrc/ext/causal_bp.cu:556-581 over the nbV order).
        std::vector<int64_t> rp(V + 1, 0);
        for (size_t e = 0; e < E; e++) rp[(size_t)a.slot_var[e] + 1]++;
        for (size_t i = 0; i < V; i++) rp[i + 1] += rp[i];
        if (row_ptr_fv) std::copy(rp.begin(), rp.end(), row_ptr_fv);
        if (col_ind_fv) {
            std::vector<int64_t> cur(rp.begin(), rp.end() - 1);
            for (size_t I = 0; I < F; I++)
                for (int64_t e = a.offsets[I]; e < a.offsets[I + 1]; e++)
                    col_ind_fv[cur[(size_t)a.slot_var[(size_t)e]]++] = (int64_t)I;
        }
        return FLBP_OK;
    });
}

int flbp_engine_create_from_fg(const flbp_fg *fg, const flbp_engine_opts *opts, flbp_engine **out) {
    if (!fg || !out) {
        flbp::set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    return guarded([&] {
        lbp::detail::GraphArrays a;
        std::string err;
        if (lbp::detail::build_arrays(fg->g, a, err)) {
            flbp::set_error(err);
            return FLBP_ERR_INVALID;
        }
        return flbp_engine_create(&a.desc, opts, out);
    });
}

}  // extern "C"
