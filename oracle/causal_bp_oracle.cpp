// FP64 CPU restatement of FastLBP's causal loopy-BP path: the PARALL sweep and
// the sequential SEQFIX / TOPO schedules.
//
// TEST INFRASTRUCTURE ONLY. This file is the correctness oracle: only the
// tests, the smoke check and the CPU-baseline leg of the benchmark may load
// it, and only as the checker. The product path (fastlbp_b200/) never links,
// loads or calls anything in oracle/.
//
// Every routine restates one piece of the reference (paths relative to the
// FastLBP project root) in plain double-precision C++:
//   * .causal_fg reader ........ csrc/ext/causal_fg.cpp:129-279, include/utils/utils.h:109-113
//   * graph construction ....... csrc/ext/causal_fg.cpp:28-68, csrc/lbp/bipgraph.cpp:24-42
//   * clamping ................. csrc/ext/causal_fg.cpp:17-26, csrc/ext/causal_factor.cpp:63-100
//   * CSR + edge records ....... csrc/ext/causal_bp.cu:310-407, 556-581, 724-817
//   * init ..................... csrc/ext/causal_bp.cu:824-856
//   * f->v kernel (types 0-8) .. csrc/kernel/causal_bp_parall.cu:14-18, 94-398
//   * per-variable product ..... csrc/kernel/causal_bp_parall.cu:20-53
//   * v->f kernel .............. csrc/kernel/causal_bp_parall.cu:55-92
//   * beliefs .................. csrc/kernel/causal_bp_seq.cu:102-111, csrc/ext/causal_bp.cu:483-515
//   * run loops ................ csrc/ext/causal_bp.cu:858-910, 912-1004, 1006-1143 (+ HostBeliefHistory :28-78)
//   * SEQFIX / TOPO orders ..... csrc/ext/causal_bp.cu:186-201, 203-304
//   * conflict-free batches .... csrc/ext/causal_bp.cu:583-722
//   * sequential sweep ......... csrc/kernel/causal_bp_seq.cu:13-83, 113-459, csrc/ext/causal_bp.cu:446-476
//
// Damping is not part of the reference. It is defined here once, for the
// oracle and the GPU engine alike: after the f->v sweep each new f->v message
// is mixed geometrically with the previous one, m <- m_new^(1-d) * m_old^d,
// then normalised; a (0,0) result becomes (0.5,0.5) (the reference's rule for
// an all-zero message). With d == 0 the mixing step is skipped entirely, so
// the restatement reduces exactly to the reference.
//
// Built with -ffp-contract=off so results are deterministic; expect agreement
// with the reference GPU binary to ~1e-12, not bit-exactly (nvcc contracts
// multiply-adds into FMAs by default).
//
// Two arithmetic modes. The default restates the reference's arithmetic:
// message pairs in probability space, rescaled by their larger component
// after every product (causal_bp_parall.cu:14-18) and exact zeros counted
// (:36-45, 74-83). Once the smaller component of a pair falls below the
// double range (log-odds beyond about +-745) it becomes an exact zero, which
// the zero-count rules then treat as hard evidence. The log-odds mode
// ("lodds") runs the same PARALL recurrence - the same case split of the nine
// factor/clamp/direction types, the same zero-count and fallback rules,
// damping and run loops - with every message held as an FP64 log-odds value
// and every product taken as a sum of logs, so nothing underflows: exact
// zeros arise only where the reference's arithmetic gives them with exact
// inputs (a p or q of 0 or 1, a clamp). On graphs whose messages stay in
// range both modes agree to rounding. With underflow tracking on, the
// default mode also marks every message and belief that depends on an
// underflow: a message whose probability-space result has an exact zero (or
// a product that reached zero without an exact-zero input) where the
// log-odds evaluation of the same inputs is finite, and everything computed
// from it in later sweeps.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <map>
#include <queue>
#include <random>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <sys/time.h>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------- graph model

struct OFactor {
    int type = 0;                 // 0 Singleton 'I', 1 DefiniteAnd '*', 2 DefiniteOr '+'
    uint64_t head = 0;            // label
    std::vector<uint64_t> body;   // sorted unique labels
    std::vector<uint64_t> vars;   // sorted unique labels of body + head
    double p = 0.0, q = 0.0;
    bool head_clamped = false;
    double mask0 = 1.0, mask1 = 1.0;
};

struct ONb {
    size_t iter, node, dual;
};

struct OGraph {
    std::vector<OFactor> factors;
    std::vector<uint64_t> vars;           // sorted labels
    std::vector<std::vector<ONb>> nbV;    // per variable: factors in factor order
    std::vector<std::vector<ONb>> nbF;    // per factor: variables in label order
};

void insert_sorted(std::vector<uint64_t> &s, uint64_t x) {
    auto it = std::lower_bound(s.begin(), s.end(), x);
    if (it == s.end() || *it != x) s.insert(it, x);
}

void erase_sorted(std::vector<uint64_t> &s, uint64_t x) {
    auto it = std::lower_bound(s.begin(), s.end(), x);
    if (it != s.end() && *it == x) s.erase(it);
}

OFactor make_singleton(uint64_t v, double p) {
    OFactor f;
    f.type = 0;
    f.head = v;
    f.p = p;
    f.q = 0.0;
    f.vars = {v};
    return f;
}

OFactor make_rule(uint64_t head, std::vector<uint64_t> body, bool is_and, double p, double q) {
    OFactor f;
    f.type = is_and ? 1 : 2;
    f.head = head;
    std::sort(body.begin(), body.end());
    body.erase(std::unique(body.begin(), body.end()), body.end());
    f.body = body;
    f.vars = body;
    insert_sorted(f.vars, head);
    f.p = p;
    f.q = q;
    return f;
}

// csrc/ext/causal_fg.cpp:50-68 and :28-48; csrc/lbp/bipgraph.cpp:24-42 (no duplicate check).
OGraph build_graph(const std::vector<OFactor> &facs) {
    OGraph g;
    g.factors = facs;
    std::set<uint64_t> vs;
    for (auto &f : facs) vs.insert(f.vars.begin(), f.vars.end());
    g.vars.assign(vs.begin(), vs.end());
    std::unordered_map<uint64_t, size_t> idx;
    idx.reserve(g.vars.size() * 2 + 1);
    for (size_t i = 0; i < g.vars.size(); i++) idx[g.vars[i]] = i;
    g.nbV.assign(g.vars.size(), {});
    g.nbF.assign(facs.size(), {});
    for (size_t I = 0; I < facs.size(); I++) {
        for (uint64_t lab : facs[I].vars) {
            size_t i = idx[lab];
            ONb n1{g.nbV[i].size(), I, g.nbF[I].size()};
            ONb n2{n1.dual, i, n1.iter};
            g.nbV[i].push_back(n1);
            g.nbF[I].push_back(n2);
        }
    }
    return g;
}

// include/utils/utils.h:109-113: skip following lines that start with '#'.
void skip_annotation(std::istream &is) {
    std::string tmp;
    while (is.peek() == '#') std::getline(is, tmp);
}

// csrc/ext/causal_fg.cpp:129-279.
std::vector<OFactor> parse_causal_fg(std::istream &is) {
    std::vector<OFactor> facs;
    std::string line;
    std::getline(is, line);
    skip_annotation(is);
    size_t nr = (size_t)std::stoi(line);
    std::set<uint64_t> heads, all_vars;
    for (size_t I = 0; I < nr; I++) {
        std::getline(is, line);  // the separating blank line (content ignored)
        std::getline(is, line);
        skip_annotation(is);
        uint64_t head = (uint64_t)(size_t)std::stoi(line);
        heads.insert(head);
        all_vars.insert(head);
        std::getline(is, line);
        skip_annotation(is);
        char ch = line.front();
        if (ch != 'I' && ch != '*' && ch != '+') throw std::runtime_error("Unreachable");
        if (ch == 'I') {
            std::getline(is, line);
            skip_annotation(is);
            double prob = (double)std::stold(line);
            facs.push_back(make_singleton(head, prob));
        } else {
            double prob = 1.0, prob_default = 0.0;
            if (line.length() > 1) {
                size_t sp = line.find(';');
                if (sp > 1) prob = (double)std::stold(line.substr(1, sp - 1));
                if (sp != std::string::npos && sp + 1 != line.length())
                    prob_default = (double)std::stold(line.substr(sp + 1));
            }
            std::getline(is, line);
            skip_annotation(is);
            size_t blen = (size_t)std::stoi(line);
            std::getline(is, line);
            skip_annotation(is);
            std::istringstream ss(line);
            std::vector<uint64_t> body;
            for (size_t b = 0; b < blen; b++) {
                long id = 0;
                ss >> id;
                body.push_back((uint64_t)(size_t)id);
                all_vars.insert((uint64_t)(size_t)id);
            }
            facs.push_back(make_rule(head, body, ch == '*', prob, prob_default));
        }
    }
    for (uint64_t v : all_vars)
        if (!heads.count(v)) facs.push_back(make_singleton(v, 0.5));
    return facs;
}

// csrc/ext/causal_factor.cpp:63-100.
OFactor gen_clamped(const OFactor &f, uint64_t v, size_t x) {
    OFactor nf = f;
    if (f.type == 0) {
        if (v == f.head) nf.p = (double)x;
        return nf;
    }
    if (v == f.head) {
        nf.head_clamped = true;
        double m0 = (x == 0) ? 1.0 : 0.0, m1 = (x == 1) ? 1.0 : 0.0;
        if (x > 1) throw std::out_of_range("clamp value");
        if (f.head_clamped) {
            m0 *= f.mask0;
            m1 *= f.mask1;
        }
        nf.mask0 = m0;
        nf.mask1 = m1;
    } else if (std::binary_search(f.body.begin(), f.body.end(), v)) {
        erase_sorted(nf.body, v);
        erase_sorted(nf.vars, v);
        if ((x == 0 && f.type == 1) || (x > 0 && f.type == 2)) {
            nf.p = f.q;
            nf.body.clear();
            nf.vars = {f.head};
        }
    }
    return nf;
}

// csrc/ext/causal_fg.cpp:17-26 (topology is deliberately left as it was).
void clamp_graph(OGraph &g, size_t i, size_t x) {
    std::map<size_t, OFactor> nf;
    for (auto &n : g.nbV[i]) nf.emplace(n.node, gen_clamped(g.factors[n.node], g.vars[i], x));
    for (auto &kv : nf) g.factors[kv.first] = kv.second;
}

// ------------------------------------------------------------ CSR + records

struct ORec {  // Index6Real4 of include/utils/utils.h:48-51
    size_t type, v, src, start, end, head;
    double q, p, m0, m1;
};

struct OVfRec {  // Index3 of include/utils/utils.h:29-31
    size_t ind, v, src;
};

struct OLayout {
    std::vector<size_t> row_ptr_vf, col_ind_vf, row_ptr_fv, col_ind_fv, head;
    std::vector<ORec> rec;     // variable-major order
    std::vector<OVfRec> vf;    // factor-major order
};

// csrc/ext/causal_bp.cu:556-581.
void coo2csr(const std::vector<size_t> &rows, const std::vector<size_t> &cols, size_t nrows,
             std::vector<size_t> &ptr, std::vector<size_t> &ind) {
    ptr.assign(nrows + 1, 0);
    ind.assign(rows.size(), 0);
    std::vector<size_t> cnt(nrows, 0);
    for (size_t r : rows) cnt[r]++;
    for (size_t i = 0; i < nrows; i++) ptr[i + 1] = ptr[i] + cnt[i];
    std::vector<size_t> cur(nrows, 0);
    for (size_t k = 0; k < rows.size(); k++) {
        size_t r = rows[k];
        ind[ptr[r] + cur[r]++] = cols[k];
    }
}

// csrc/ext/causal_bp.cu:310-407 and :724-817 (PARALL branch).
OLayout construct(const OGraph &g) {
    OLayout L;
    size_t F = g.factors.size(), V = g.vars.size();
    size_t len = 0;
    for (auto &f : g.factors) len += f.vars.size();
    std::vector<size_t> rows(len), cols(len);
    L.head.assign(F, 0);
    size_t idx = 0;
    for (size_t I = 0; I < F; I++) {
        uint64_t hl = g.factors[I].head;
        for (auto &n : g.nbF[I]) {
            rows[idx] = I;
            cols[idx] = n.node;
            if (g.vars[n.node] == hl) L.head[I] = idx;
            idx++;
        }
    }
    coo2csr(rows, cols, F, L.row_ptr_vf, L.col_ind_vf);
    idx = 0;
    for (size_t i = 0; i < V; i++) {
        for (auto &n : g.nbV[i]) {
            rows[idx] = i;
            cols[idx] = n.node;
            idx++;
        }
    }
    coo2csr(rows, cols, V, L.row_ptr_fv, L.col_ind_fv);

    L.rec.reserve(len);
    for (size_t i = 0; i < V; i++) {
        for (auto &n : g.nbV[i]) {
            size_t I = n.node;
            const OFactor &f = g.factors[I];
            ORec r;
            r.v = i;
            r.src = L.row_ptr_vf[I] + n.dual;
            r.start = L.row_ptr_vf[I];
            r.end = L.row_ptr_vf[I + 1];
            r.head = L.head[I];
            r.q = f.q;
            r.p = f.p;
            r.m0 = f.mask0;
            r.m1 = f.mask1;
            bool is_head = (f.head == g.vars[i]);
            if (f.type == 0) r.type = 0;
            else if (f.type == 1) r.type = f.head_clamped ? (is_head ? 3 : 7) : (is_head ? 1 : 5);
            else r.type = f.head_clamped ? (is_head ? 4 : 8) : (is_head ? 2 : 6);
            L.rec.push_back(r);
        }
    }
    L.vf.reserve(len);
    for (size_t I = 0; I < F; I++)
        for (auto &n : g.nbF[I])
            L.vf.push_back({L.row_ptr_vf[I] + n.iter, n.node, L.row_ptr_fv[n.node] + n.dual});
    return L;
}

// ------------------------------------------------------------------ kernels

inline void scale_parall(double &x, double &y) {  // csrc/kernel/causal_bp_parall.cu:14-18
    double m = std::fmax(x, y);
    x /= m;
    y /= m;
}

// csrc/kernel/causal_bp_seq.cu:13-23: the sequential kernels' rescaling; it
// differs from the PARALL one only for two equal values (both become 1, so
// (0, 0) gives (1, 1) instead of NaN).
inline void scale_seq(double &x, double &y) {
    if (x < y) {
        x = x / y;
        y = 1.0;
    } else if (y < x) {
        y = y / x;
        x = 1.0;
    } else {
        x = y = 1.0;
    }
}

// One f->v message, csrc/kernel/causal_bp_parall.cu:102-397 (PARALL) and
// csrc/kernel/causal_bp_seq.cu:162-452 (SEQ): the same formulas, with the
// rescaling of the schedule's kernels.
template <bool SEQ>
void fv_message_t(const ORec &r, const double *vf0, const double *vf1, double &out0, double &out1) {
    auto scale2 = [](double &x, double &y) {
        if (SEQ) scale_seq(x, y);
        else scale_parall(x, y);
    };
    const size_t type = r.type, src = r.src, h = r.head, s = r.start, e = r.end;
    const double p0 = r.q, p1 = r.p, mask0 = r.m0, mask1 = r.m1;
    double marg0 = 0.0, marg1 = 0.0;
    if (type == 0) {
        marg0 = 1 - p1;
        marg1 = p1;
    } else if (type == 1 || type == 3) {
        double prod_1 = 1.0, prod_10 = 1.0;
        if (e - s == 1) {
            marg0 = 1 - p1;
            marg1 = p1;
        } else if (e - s == 2) {
            size_t j = s;
            if (s == src) j++;
            double m_0 = vf0[j], m_1 = vf1[j];
            marg0 = (1 - p1) * m_1 + (1 - p0) * m_0;
            marg1 = p1 * m_1 + p0 * m_0;
        } else {
            double e1 = 0;
            for (size_t j = s; j < e; j++) {
                if (j == src) continue;
                double m_0 = vf0[j], m_1 = vf1[j];
                double a0 = m_0 + m_1, a1 = m_1;
                prod_1 *= a1;
                prod_10 *= a0;
                scale2(prod_1, prod_10);
                double delta = m_0;
                if (a1 != 0 && a0 == a1 && delta != 0) e1 += delta / a1;
            }
            marg0 = (1 - p1) * prod_1 + (1 - p0) * (e1 * prod_10 + (prod_10 - prod_1));
            marg1 = p1 * prod_1 + p0 * (e1 * prod_10 + (prod_10 - prod_1));
        }
        if (type == 3) {
            marg0 *= mask0;
            marg1 *= mask1;
        }
        double marg = marg0 + marg1;
        if (marg != 0) {
            marg0 = marg0 / marg;
            marg1 = marg1 / marg;
        } else if (type == 3 && mask0 == 0) {
            marg0 = 0.0;
            marg1 = 1.0;
        } else if (type == 3 && mask1 == 0) {
            marg0 = 1.0;
            marg1 = 0.0;
        } else {
            marg0 = 0.5;
            marg1 = 0.5;
        }
    } else if (type == 2 || type == 4) {
        double prod_0 = 1.0, prod_10 = 1.0;
        if (e - s == 1) {
            marg0 = p1;
            marg1 = 1 - p1;
        } else if (e - s == 2) {
            size_t j = s;
            if (s == src) j++;
            double m_0 = vf0[j], m_1 = vf1[j];
            marg0 = p1 * m_0 + p0 * m_1;
            marg1 = (1 - p1) * m_0 + (1 - p0) * m_1;
        } else {
            double e1 = 0;
            for (size_t j = s; j < e; j++) {
                if (j == src) continue;
                double m_0 = vf0[j], m_1 = vf1[j];
                double a0 = m_0 + m_1, a1 = m_0;
                prod_0 *= a1;
                prod_10 *= a0;
                scale2(prod_0, prod_10);
                double delta = m_1;
                if (a1 != 0 && a0 == a1 && delta != 0) e1 += delta / a1;
            }
            marg0 = p1 * prod_0 + p0 * (e1 * prod_10 + (prod_10 - prod_0));
            marg1 = (1 - p1) * prod_0 + (1 - p0) * (e1 * prod_10 + (prod_10 - prod_0));
        }
        if (type == 4) {
            marg0 *= mask0;
            marg1 *= mask1;
        }
        double marg = marg0 + marg1;
        if (marg != 0) {
            marg0 = marg0 / marg;
            marg1 = marg1 / marg;
        } else if (type == 4 && mask0 == 0) {
            marg0 = 0.0;
            marg1 = 1.0;
        } else if (type == 4 && mask1 == 0) {
            marg0 = 1.0;
            marg1 = 0.0;
        } else {
            marg0 = 0.5;
            marg1 = 0.5;
        }
    } else if (type == 5 || type == 7) {
        double m0h = vf0[h], m1h = vf1[h];
        double prod_1, prod_10;
        if (type == 5) {
            prod_1 = (p1 - p0) * (m1h - m0h);
            prod_10 = p0 * m1h + (1 - p0) * m0h;
        } else {
            prod_1 = (p1 - p0) * (m1h * mask1 - m0h * mask0);
            prod_10 = p0 * m1h * mask1 + (1 - p0) * m0h * mask0;
        }
        scale2(prod_1, prod_10);
        if (prod_10 != 0) {
            for (size_t j = s; j < e; j++) {
                if (j == src || j == h) continue;
                double m0 = vf0[j], m1 = vf1[j], m = m0 + m1;
                prod_10 *= m;
                prod_1 *= m1;
                scale2(prod_1, prod_10);
            }
        }
        marg0 = prod_10;
        marg1 = prod_10 + prod_1;
        double marg = marg0 + marg1;
        if (marg != 0) {
            marg0 = marg0 / marg;
            marg1 = marg1 / marg;
        } else {
            marg0 = 0.5;
            marg1 = 0.5;
        }
    } else {  // 6 or 8
        double m0h = vf0[h], m1h = vf1[h];
        double prod_0, prod_10;
        if (type == 6) {
            prod_0 = (p1 - p0) * (m0h - m1h);
            prod_10 = p0 * m0h + (1 - p0) * m1h;
        } else {
            prod_0 = (p1 - p0) * (m0h * mask0 - m1h * mask1);
            prod_10 = p0 * m0h * mask0 + (1 - p0) * m1h * mask1;
        }
        scale2(prod_0, prod_10);
        if (prod_10 != 0) {
            for (size_t j = s; j < e; j++) {
                if (j == src || j == h) continue;
                double m0 = vf0[j], m1 = vf1[j], m = m0 + m1;
                prod_10 *= m;
                prod_0 *= m0;
                scale2(prod_0, prod_10);
            }
        }
        marg0 = prod_0 + prod_10;
        marg1 = prod_10;
        double marg = marg0 + marg1;
        if (marg != 0) {
            marg0 = marg0 / marg;
            marg1 = marg1 / marg;
        } else {
            marg0 = 0.5;
            marg1 = 0.5;
        }
    }
    out0 = marg0;
    out1 = marg1;
}

void fv_message(const ORec &r, const double *vf0, const double *vf1, double &out0, double &out1) {
    fv_message_t<false>(r, vf0, vf1, out0, out1);
}

// --------------------------------------------------------- log-odds mode
//
// A message (m0, m1), normalised, is held as lambda = log m1 - log m0:
// +inf is (0, 1), -inf is (1, 0), 0 is (0.5, 0.5), NaN is the reference's
// NaN pair.

constexpr double kInfD = std::numeric_limits<double>::infinity();

// log sigmoid(x) = log of the normalised m1 of lambda x; +inf -> 0, -inf -> -inf.
inline double lsig(double x) {
    if (std::isnan(x)) return x;
    return x >= 0 ? -std::log1p(std::exp(-x)) : x - std::log1p(std::exp(x));
}

// log(e^a + e^b), exact zeros (-inf) allowed.
inline double lae(double a, double b) {
    if (a == -kInfD) return b;
    if (b == -kInfD) return a;
    const double m = std::fmax(a, b);
    return m + std::log1p(std::exp(-std::fabs(a - b)));
}

// log(1 - e^x) for x <= 0.
inline double log1mexp(double x) {
    if (x == -kInfD) return 0.0;
    if (x == 0.0) return -kInfD;
    return x > -M_LN2 ? std::log(-std::expm1(x)) : std::log1p(-std::exp(x));
}

inline double lmask(double m) { return m == 0.0 ? -kInfD : 0.0; }  // masks are 0 or 1

// Pair (log a, log b) of a noisy-AND over a body whose product of sigma is
// e^lP: a = p P + q (1 - P), b = (1 - p) P + (1 - q)(1 - P).
inline void and_pair(double lP, double p, double q, double &la, double &lb) {
    const double l1 = log1mexp(lP);
    la = lae(std::log(p) + lP, std::log(q) + l1);
    lb = lae(std::log1p(-p) + lP, std::log1p(-q) + l1);
}

// One f->v message in log-odds: the nine types of
// csrc/kernel/causal_bp_parall.cu:102-397 with every product taken as a sum
// of logs. OR factors are AND factors with the states swapped.
double fv_message_lodds(const ORec &r, const double *lvf) {
    const size_t type = r.type, src = r.src, h = r.head, s = r.start, e = r.end;
    const double p = r.p, q = r.q;
    if (type == 0) return std::log(p) - std::log1p(-p);  // (1-p, p), :110-112
    if (type <= 4) {  // into the head: AND 1 / 3, OR 2 / 4 (:113-288)
        const bool is_or = (type == 2 || type == 4);
        const double sg = is_or ? -1.0 : 1.0;
        double lP = 0.0;  // log product of the body's sigma (AND orientation)
        for (size_t j = s; j < e; j++)
            if (j != src) lP += lsig(sg * lvf[j]);
        double la, lb;
        and_pair(lP, p, q, la, lb);
        // AND: (marg0, marg1) = (b, a); OR: (a, b)
        double l0 = is_or ? la : lb, l1 = is_or ? lb : la;
        if (type >= 3) {
            l0 += lmask(r.m0);
            l1 += lmask(r.m1);
        }
        if (l0 == -kInfD && l1 == -kInfD) {  // marg == 0: the mask's one-hot fallback, else (0.5, 0.5)
            if (type >= 3 && r.m0 == 0.0) return kInfD;
            if (type >= 3 && r.m1 == 0.0) return -kInfD;
            return 0.0;
        }
        return l1 - l0;
    }
    // into a body slot: AND 5 / 7, OR 6 / 8 (:289-393), in AND orientation
    const bool is_or = (type == 6 || type == 8);
    const double sg = is_or ? -1.0 : 1.0;
    double lh1 = lsig(sg * lvf[h]), lh0 = lsig(-sg * lvf[h]);  // head message, oriented
    if (type >= 7) {
        lh1 += lmask(is_or ? r.m0 : r.m1);
        lh0 += lmask(is_or ? r.m1 : r.m0);
    }
    // prod_10 = q m1h + (1 - q) m0h; the reference skips its loop when it is 0
    const double lden = lae(std::log(q) + lh1, std::log1p(-q) + lh0);
    if (lden == -kInfD) {
        // scale() of (prod_1, 0): (1, 0) if prod_1 = (p - q)(m1h - m0h) > 0, else NaN
        const double dh = (lh1 > lh0) ? 1.0 : (lh1 < lh0) ? -1.0 : 0.0;
        return ((p - q) * dh > 0.0) ? sg * kInfD : std::numeric_limits<double>::quiet_NaN();
    }
    double lPo = 0.0;  // the other body slots
    for (size_t j = s; j < e; j++)
        if (j != src && j != h) lPo += lsig(sg * lvf[j]);
    double la, lb;
    and_pair(lPo, p, q, la, lb);
    const double lnum = lae(lh1 + la, lh0 + lb);  // prod_10 + prod_1 = m1h a + m0h b
    return sg * (lnum - lden);
}

// Damping in log-odds: (1 - d) new + d old, with exact zeros dominating and
// opposite zeros giving (0.5, 0.5) - the probability-space rule of the
// default mode.
inline double damp_lodds(double nw, double old, double d) {
    const bool ni = std::isinf(nw), oi = std::isinf(old);
    if (ni || oi) {
        if (ni && oi) return (nw == old) ? nw : 0.0;
        return ni ? nw : old;
    }
    return (1.0 - d) * nw + d * old;
}

inline double lodds_of(double m0, double m1) { return std::log(m1) - std::log(m0); }

double now_s() {
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return (double)tv.tv_sec + (double)tv.tv_usec / 1e6;
}

// ------------------------------------------------------------- BP engine

struct OBP {
    OGraph g;  // CausalBP copies the graph (include/lbp/daialg.h:21)
    OLayout L;
    size_t V = 0, E = 0;
    double damping = 0.0;
    int nthreads = 1;
    std::vector<double> fv0, fv1, vf0, vf1, prod0, prod1, bel0, bel1;
    std::vector<size_t> nz0, nz1;
    std::vector<double> oldBeliefs, beliefs, lowpass;
    std::vector<double> damp_old0, damp_old1;
    size_t iters = 0;
    double maxdiff_member = 0.0;
    bool logdomain = false;
    // log-odds mode: f->v (variable-major) and v->f (factor-major) log-odds,
    // per-variable finite sums; nz0 / nz1 count the +inf / -inf inputs
    bool lodds = false;
    std::vector<double> lfv, lvf, lS;
    // underflow tracking (default mode): per message / variable, 1 = depends on an underflow
    bool track = false;
    std::vector<uint8_t> t_fv, t_vf, t_var;
    size_t underflow_events = 0;
    // sequential schedule (updates=SEQFIX / TOPO): per batch its v->f records
    // and its f->v records (indices into L.rec); empty for PARALL
    bool seq = false;
    std::vector<std::vector<OVfRec>> seq_vf;
    std::vector<std::vector<size_t>> seq_fv;
    std::vector<size_t> seq_slots;   // the update sequence as factor-major slots
    std::vector<size_t> slot_batch;  // batch of every factor-major slot
};

void bp_init(OBP &b) {  // csrc/ext/causal_bp.cu:824-856
    if (b.lodds) {  // every message (1, 1): log-odds 0
        b.lfv.assign(b.E, 0.0);
        b.lvf.assign(b.E, 0.0);
        b.lS.assign(b.V, 0.0);
    }
    if (b.track) {
        b.t_fv.assign(b.E, 0);
        b.t_vf.assign(b.E, 0);
        b.t_var.assign(b.V, 0);
        b.underflow_events = 0;
    }
    double c = b.logdomain ? 0.0 : 1.0;
    std::fill(b.fv0.begin(), b.fv0.end(), c);
    std::fill(b.fv1.begin(), b.fv1.end(), c);
    std::fill(b.vf0.begin(), b.vf0.end(), c);
    std::fill(b.vf1.begin(), b.vf1.end(), c);
    std::fill(b.prod0.begin(), b.prod0.end(), c);
    std::fill(b.prod1.begin(), b.prod1.end(), c);
    std::fill(b.nz0.begin(), b.nz0.end(), 0);
    std::fill(b.nz1.begin(), b.nz1.end(), 0);
}

inline double powz(double x, double a) {  // x^a with 0^0 = 1 and 0^a = 0 for a > 0
    if (a == 0.0) return 1.0;
    if (x == 0.0) return 0.0;
    return std::pow(x, a);
}

// Underflow tracking, f->v side: the message at variable-major position i
// depends on an underflow if an input v->f message does, or if its
// probability-space result (o0, o1) differs in kind (an exact zero, NaN)
// from the log-odds evaluation of the same inputs, or by more than 1e-9 in
// log-odds (denormal products). Inputs are the v->f messages of the factor's
// other slots.
uint8_t fv_taint(const OBP &b, const ORec &r, double o0, double o1, std::vector<double> &scratch) {
    uint8_t t = 0;
    if (r.type != 0)
        for (size_t j = r.start; j < r.end; j++)
            if (j != r.src) t |= b.t_vf[j];
    if (t) return 1;
    if (r.type == 0) return 0;
    // log-odds of the same inputs (only the factor's own slots are read)
    if (scratch.size() < b.E) scratch.resize(b.E);
    for (size_t j = r.start; j < r.end; j++) scratch[j] = lodds_of(b.vf0[j], b.vf1[j]);
    const double want = fv_message_lodds(r, scratch.data());
    const double got = lodds_of(o0, o1);
    if (std::isnan(want) || std::isnan(got)) return (uint8_t)(std::isnan(want) != std::isnan(got));
    if (std::isinf(want) || std::isinf(got)) return (uint8_t)(want != got);
    return (uint8_t)(std::fabs(want - got) > 1e-9 * std::fmax(1.0, std::fabs(want)));
}

// csrc/ext/causal_bp.cu:409-444 in log-odds (see fv_message_lodds): f->v,
// per-variable sums with +-inf counts, v->f.
void bp_sweep_parall_lodds(OBP &b) {
    const long E = (long)b.E, V = (long)b.V;
    const double d = b.damping;
    const ORec *rec = b.L.rec.data();
#pragma omp parallel for schedule(dynamic, 4096) num_threads(b.nthreads)
    for (long i = 0; i < E; i++) {
        double o = fv_message_lodds(rec[i], b.lvf.data());
        if (d != 0.0) o = damp_lodds(o, b.lfv[i], d);
        b.lfv[i] = o;
    }
    const size_t *rp = b.L.row_ptr_fv.data();
#pragma omp parallel for schedule(dynamic, 4096) num_threads(b.nthreads)
    for (long i = 0; i < V; i++) {  // csrc/kernel/causal_bp_parall.cu:30-52
        double S = 0.0;
        size_t z0 = 0, z1 = 0;
        for (size_t j = rp[i]; j < rp[i + 1]; j++) {
            const double x = b.lfv[j];
            if (x == kInfD) z0++;        // m0 == 0
            else if (x == -kInfD) z1++;  // m1 == 0
            else S += x;                 // NaN stays NaN, as the reference's product
        }
        b.lS[i] = S;
        b.nz0[i] = z0;
        b.nz1[i] = z1;
    }
    const OVfRec *vr = b.L.vf.data();
#pragma omp parallel for schedule(dynamic, 4096) num_threads(b.nthreads)
    for (long k = 0; k < E; k++) {  // csrc/kernel/causal_bp_parall.cu:67-91
        const OVfRec &x = vr[k];
        const double ms = b.lfv[x.src];
        const bool zero0 = b.nz0[x.v] - (size_t)(ms == kInfD) > 0;
        const bool zero1 = b.nz1[x.v] - (size_t)(ms == -kInfD) > 0;
        double o;
        if (zero0 && zero1) o = 0.0;  // (0.5, 0.5)
        else if (zero0) o = kInfD;
        else if (zero1) o = -kInfD;
        else o = b.lS[x.v] - (std::isinf(ms) ? 0.0 : ms);
        b.lvf[x.ind] = o;
    }
}

// csrc/ext/causal_bp.cu:409-444: f->v, per-variable product, v->f.
void bp_sweep_parall(OBP &b) {
    if (b.lodds) {
        bp_sweep_parall_lodds(b);
        return;
    }
    const long E = (long)b.E, V = (long)b.V;
    const double d = b.damping;
    const ORec *rec = b.L.rec.data();
    std::vector<uint8_t> t_fv_new(b.track ? b.E : 0);
    size_t events = 0;
#pragma omp parallel for schedule(dynamic, 4096) num_threads(b.nthreads) reduction(+ : events)
    for (long i = 0; i < E; i++) {
        double o0, o1;
        fv_message(rec[i], b.vf0.data(), b.vf1.data(), o0, o1);
        if (b.track) {
            thread_local std::vector<double> scratch;
            const uint8_t t = fv_taint(b, rec[i], o0, o1, scratch);
            t_fv_new[i] = t | (d != 0.0 ? b.t_fv[i] : 0);
            if (t && rec[i].type != 0) {
                bool in = false;
                for (size_t j = rec[i].start; j < rec[i].end; j++)
                    if (j != rec[i].src) in |= b.t_vf[j] != 0;
                events += in ? 0 : 1;
            }
        }
        if (d != 0.0) {
            double n0 = powz(o0, 1.0 - d) * powz(b.fv0[i], d);
            double n1 = powz(o1, 1.0 - d) * powz(b.fv1[i], d);
            if (n0 == 0 && n1 == 0) {
                n0 = 0.5;
                n1 = 0.5;
            }
            double s = n0 + n1;
            o0 = n0 / s;
            o1 = n1 / s;
        }
        b.fv0[i] = o0;
        b.fv1[i] = o1;
    }
    if (b.track) b.t_fv.swap(t_fv_new);
    const size_t *rp = b.L.row_ptr_fv.data();
#pragma omp parallel for schedule(dynamic, 4096) num_threads(b.nthreads) reduction(+ : events)
    for (long i = 0; i < V; i++) {  // csrc/kernel/causal_bp_parall.cu:30-52
        double pr0 = 1.0, pr1 = 1.0;
        size_t z0 = 0, z1 = 0;
        for (size_t j = rp[i]; j < rp[i + 1]; j++) {
            double m0 = b.fv0[j], m1 = b.fv1[j];
            if (m0 == 0) z0++;
            else pr0 *= m0;
            if (m1 == 0) z1++;
            else pr1 *= m1;
            scale_parall(pr0, pr1);
        }
        b.prod0[i] = pr0;
        b.prod1[i] = pr1;
        b.nz0[i] = z0;
        b.nz1[i] = z1;
        if (b.track) {  // the variable's totals depend on every incoming message; a product that
                        // reached zero without an exact-zero input underflowed here
            uint8_t t = 0;
            for (size_t j = rp[i]; j < rp[i + 1]; j++) t |= b.t_fv[j];
            const bool uf = (pr0 == 0 && z0 == 0) || (pr1 == 0 && z1 == 0);
            events += (uf && !t) ? 1 : 0;
            b.t_var[i] = t | (uint8_t)uf;
        }
    }
    if (b.track) b.underflow_events += events;
    const OVfRec *vr = b.L.vf.data();
#pragma omp parallel for schedule(dynamic, 4096) num_threads(b.nthreads)
    for (long k = 0; k < E; k++) {  // csrc/kernel/causal_bp_parall.cu:67-91
        const OVfRec &x = vr[k];
        size_t c0 = b.nz0[x.v], c1 = b.nz1[x.v];
        double ms0 = b.fv0[x.src], ms1 = b.fv1[x.src];
        double pr0 = b.prod0[x.v], pr1 = b.prod1[x.v];
        if (c0 >= 2 || (c0 == 1 && ms0 != 0)) pr0 = 0.0;
        else if (ms0 != 0) pr0 = pr0 / ms0;
        if (c1 >= 2 || (c1 == 1 && ms1 != 0)) pr1 = 0.0;
        else if (ms1 != 0) pr1 = pr1 / ms1;
        if (pr0 == 0 && pr1 == 0) pr0 = pr1 = 0.5;
        double pr = pr0 + pr1;
        b.vf0[x.ind] = pr0 / pr;
        b.vf1[x.ind] = pr1 / pr;
        if (b.track) b.t_vf[x.ind] = b.t_var[x.v];
    }
}

// ------------------------------------------------------ sequential schedules

using OEdge = std::pair<size_t, size_t>;  // (variable, dual): Edge of include/ext/causal_bp.h

// csrc/ext/causal_bp.cu:186-201: factors in an order shuffled by the
// thread-local std::mt19937 (seeded 42 at start-up, csrc/ext/causal_bp.cu:116),
// every factor's edges in its neighbour order.
std::vector<OEdge> seqfix_order(const OGraph &g, uint32_t seed) {
    std::mt19937 rng(seed);
    std::vector<int> numbers(g.factors.size());
    for (int i = 0; i < (int)numbers.size(); ++i) numbers[i] = i;
    std::shuffle(numbers.begin(), numbers.end(), rng);
    std::vector<OEdge> seq;
    for (size_t I = 0; I < numbers.size(); I++)
        for (const ONb &n : g.nbF[numbers[I]]) seq.push_back({n.node, n.dual});
    return seq;
}

// csrc/ext/causal_bp.cu:203-304: breadth-first order over variables (nodes
// 0..V-1) and factors (V..V+F-1), roots in node order, neighbours in node
// order; edges ranked by (later endpoint, earlier endpoint, factor, variable,
// dual).
std::vector<OEdge> topo_order(const OGraph &g) {
    const size_t V = g.vars.size(), F = g.factors.size(), N = V + F;
    std::vector<std::vector<size_t>> adj(N);
    for (size_t I = 0; I < F; I++)
        for (const ONb &n : g.nbF[I]) {
            adj[V + I].push_back(n.node);
            adj[n.node].push_back(V + I);
        }
    for (auto &a : adj) {
        std::sort(a.begin(), a.end());
        a.erase(std::unique(a.begin(), a.end()), a.end());
    }
    std::vector<size_t> order(N, N);
    size_t next = 0;
    std::queue<size_t> ready;
    for (size_t r = 0; r < N; r++) {
        if (order[r] != N) continue;
        ready.push(r);
        order[r] = next++;
        while (!ready.empty()) {
            const size_t i = ready.front();
            ready.pop();
            for (size_t x : adj[i]) {
                if (order[x] != N) continue;
                order[x] = next++;
                ready.push(x);
            }
        }
    }
    struct Ranked {
        size_t rank, src, factor, var, dual;
    };
    std::vector<Ranked> rs;
    for (size_t I = 0; I < F; I++)
        for (const ONb &n : g.nbF[I]) {
            const size_t a = order[V + I], c = order[n.node];
            rs.push_back({std::max(a, c), std::min(a, c), I, n.node, n.dual});
        }
    std::stable_sort(rs.begin(), rs.end(), [](const Ranked &x, const Ranked &y) {
        if (x.rank != y.rank) return x.rank < y.rank;
        if (x.src != y.src) return x.src < y.src;
        if (x.factor != y.factor) return x.factor < y.factor;
        if (x.var != y.var) return x.var < y.var;
        return x.dual < y.dual;
    });
    std::vector<OEdge> seq;
    for (const Ranked &r : rs) seq.push_back({r.var, r.dual});
    return seq;
}

// csrc/ext/causal_bp.cu:583-722: cut the sequence into batches. An edge
// (i, I) opens a new batch when a v->f message of I it needs is not yet in
// the batch while its variable already receives a batch f->v message from
// another factor (for TOPO only if that edge precedes it in the sequence),
// or when i itself already receives one. Every batch records its new v->f
// messages (factor-major) and its f->v records.
void seq_batches(OBP &b, const std::vector<OEdge> &seq, bool respect_preorder) {
    const OGraph &g = b.g;
    std::map<OEdge, size_t> rank;
    for (size_t k = 0; k < seq.size(); k++) rank[seq[k]] = k;
    b.seq_vf.clear();
    b.seq_fv.clear();
    b.seq_slots.clear();
    b.slot_batch.assign(b.E, 0);
    std::set<OEdge> fv_set, vf_set;
    std::set<size_t> v_set;
    std::vector<OVfRec> cur_vf;
    std::vector<size_t> cur_fv;
    for (const OEdge &e : seq) {
        const size_t i = e.first;
        const size_t I = g.nbV[i][e.second].node;
        bool conflict = false;
        for (const ONb &j : g.nbF[I]) {
            if (j.node == i) continue;
            if (vf_set.find({I, j.iter}) == vf_set.end()) {
                for (const ONb &J : g.nbV[j.node]) {
                    if (J.node == I) continue;
                    const OEdge fv_e(j.node, J.iter);
                    if (fv_set.find(fv_e) != fv_set.end() && (!respect_preorder || rank[fv_e] < rank[e])) {
                        conflict = true;
                        break;
                    }
                }
            }
            if (conflict) break;
        }
        if (!conflict && v_set.find(i) != v_set.end()) conflict = true;
        if (conflict) {
            b.seq_vf.push_back(cur_vf);
            b.seq_fv.push_back(cur_fv);
            v_set.clear();
            fv_set.clear();
            vf_set.clear();
            cur_vf.clear();
            cur_fv.clear();
        }
        v_set.insert(i);
        fv_set.insert(e);
        cur_fv.push_back(b.L.row_ptr_fv[i] + e.second);
        const size_t slot = b.L.row_ptr_vf[I] + g.nbV[i][e.second].dual;
        b.seq_slots.push_back(slot);
        b.slot_batch[slot] = b.seq_fv.size();
        for (const ONb &j : g.nbF[I]) {
            if (j.node == i || vf_set.find({I, j.iter}) != vf_set.end()) continue;
            vf_set.insert({I, j.iter});
            cur_vf.push_back({b.L.row_ptr_vf[I] + j.iter, j.node, b.L.row_ptr_fv[j.node] + j.dual});
        }
    }
    b.seq_vf.push_back(cur_vf);
    b.seq_fv.push_back(cur_fv);
}

// csrc/kernel/causal_bp_seq.cu:34-83: replace one f->v message and update
// its variable's product and zero counts in place.
void update_message(OBP &b, size_t ind, size_t v, double marg0, double marg1) {
    const double old0 = b.fv0[ind], old1 = b.fv1[ind];
    double p0 = b.prod0[v], p1 = b.prod1[v];
    size_t z0 = b.nz0[v], z1 = b.nz1[v];
    if (old0 == 0) z0--;
    else p0 /= old0;
    if (marg0 == 0) z0++;
    else p0 *= marg0;
    if (old1 == 0) z1--;
    else p1 /= old1;
    if (marg1 == 0) z1++;
    else p1 *= marg1;
    scale_seq(p0, p1);
    b.prod0[v] = p0;
    b.prod1[v] = p1;
    b.nz0[v] = z0;
    b.nz1[v] = z1;
    b.fv0[ind] = marg0;
    b.fv1[ind] = marg1;
}

// One sequential sweep (csrc/ext/causal_bp.cu:446-476 for every batch in
// order): the batch's v->f messages from the current products
// (causal_bp_seq.cu:113-147), then its f->v messages, each folded into its
// variable's product at once (:149-459). The f->v records of a batch have
// distinct variables, so their order inside the batch does not matter.
// Damping (not in the reference) mixes each new message with the one it
// replaces, as in the PARALL sweep.
void bp_sweep_seq(OBP &b) {
    const double d = b.damping;
    for (size_t k = 0; k < b.seq_fv.size(); k++) {
        for (const OVfRec &x : b.seq_vf[k]) {
            const size_t c0 = b.nz0[x.v], c1 = b.nz1[x.v];
            const double ms0 = b.fv0[x.src], ms1 = b.fv1[x.src];
            double pr0 = b.prod0[x.v], pr1 = b.prod1[x.v];
            if (c0 >= 2 || (c0 == 1 && ms0 != 0)) pr0 = 0.0;
            else if (ms0 != 0) pr0 = pr0 / ms0;
            if (c1 >= 2 || (c1 == 1 && ms1 != 0)) pr1 = 0.0;
            else if (ms1 != 0) pr1 = pr1 / ms1;
            const double pr = pr0 + pr1;
            b.vf0[x.ind] = pr0 / pr;
            b.vf1[x.ind] = pr1 / pr;
        }
        for (size_t r : b.seq_fv[k]) {
            double o0, o1;
            fv_message_t<true>(b.L.rec[r], b.vf0.data(), b.vf1.data(), o0, o1);
            if (d != 0.0) {
                double n0 = powz(o0, 1.0 - d) * powz(b.fv0[r], d);
                double n1 = powz(o1, 1.0 - d) * powz(b.fv1[r], d);
                if (n0 == 0 && n1 == 0) {
                    n0 = 0.5;
                    n1 = 0.5;
                }
                const double s = n0 + n1;
                o0 = n0 / s;
                o1 = n1 / s;
            }
            update_message(b, r, b.L.rec[r].v, o0, o1);
        }
    }
}

void bp_sweep(OBP &b) {
    if (b.seq && (b.lodds || b.track)) throw std::runtime_error("the log-odds mode and underflow tracking are PARALL only");
    if (b.seq) bp_sweep_seq(b);
    else bp_sweep_parall(b);
}

// csrc/ext/causal_bp.cu:483-515 with getBeliefsV (causal_bp_seq.cu:102-111).
void bp_beliefs(const OBP &b, std::vector<double> &out) {
    out.resize(b.V);
    if (b.lodds) {  // b_s = P_s [zeros_s == 0], belief = b1 / (b0 + b1), from the log-odds sum
        for (size_t i = 0; i < b.V; i++) {
            const bool z0 = b.nz0[i] != 0, z1 = b.nz1[i] != 0;
            const double S = b.lS[i];
            out[i] = (z0 && z1) ? std::numeric_limits<double>::quiet_NaN()
                     : z0       ? 1.0
                     : z1       ? 0.0
                     : (S >= 0 ? 1.0 / (1.0 + std::exp(-S)) : std::exp(S) / (1.0 + std::exp(S)));
        }
        return;
    }
    for (size_t i = 0; i < b.V; i++) {
        double x = b.prod0[i] * (double)(!b.nz0[i]);
        double y = b.prod1[i] * (double)(!b.nz1[i]);
        out[i] = y / (x + y);
    }
}

OBP *bp_create(const OGraph &g, double damping, int nthreads) {
    OBP *b = new OBP();
    b->g = g;
    b->L = construct(b->g);
    b->V = g.vars.size();
    b->E = b->L.rec.size();
    b->damping = damping;
    b->nthreads = nthreads < 1 ? 1 : nthreads;
    b->fv0.assign(b->E, 0);
    b->fv1.assign(b->E, 0);
    b->vf0.assign(b->E, 0);
    b->vf1.assign(b->E, 0);
    b->prod0.assign(b->V, 0);
    b->prod1.assign(b->V, 0);
    b->nz0.assign(b->V, 0);
    b->nz1.assign(b->V, 0);
    b->oldBeliefs.assign(b->V, 0.0);  // value-initialised device vector (causal_bp.cu:371)
    b->beliefs.assign(b->V, 0.0);
    return b;
}

// csrc/ext/causal_bp.cu:858-910.
void bp_run_tol(OBP &b, double tol, size_t maxiter, double maxtime, double *maxdiff_out) {
    double tic = now_s();
    double maxDiff = INFINITY;
    std::vector<double> nb;
    for (; b.iters < maxiter && maxDiff > tol && (now_s() - tic) < maxtime; b.iters++) {
        bp_sweep(b);
        maxDiff = -INFINITY;
        bp_beliefs(b, nb);
        double diff = 0.0;  // thrust::reduce(max) with init 0.0
        for (size_t i = 0; i < b.V; i++) {
            double dd = std::fabs(b.oldBeliefs[i] - nb[i]);
            diff = (diff < dd) ? dd : diff;  // thrust::maximum keeps the left operand on NaN
        }
        maxDiff = std::max(diff, maxDiff);
        b.oldBeliefs = nb;
    }
    b.beliefs = b.oldBeliefs;
    if (maxdiff_out) *maxdiff_out = maxDiff;
}

// csrc/ext/causal_bp.cu:912-1004: exactly maxIters sweeps, beliefs once at the end.
double bp_run_fixed(OBP &b, double /*tol*/, size_t maxIters, size_t /*hist*/) {
    for (size_t n = 0; n < maxIters; n++, b.iters++) bp_sweep(b);
    std::vector<double> nb;
    bp_beliefs(b, nb);
    b.oldBeliefs = nb;
    b.beliefs = b.oldBeliefs;
    b.lowpass = b.beliefs;
    return 1.0;
}

// csrc/ext/causal_bp.cu:1006-1143 with HostBeliefHistory (:28-78).
double bp_run_lowpass(OBP &b, double tol, size_t minIters, size_t maxIters, size_t hist, double maxtime,
                      int *reason_out, size_t *sweeps_out) {
    double tic = now_s();
    size_t numIters = 0;
    double maxDiff = INFINITY, frac = 1.0, nodeFracTol = 0.0;
    const size_t V = b.V;
    std::vector<double> hvals(V * (hist ? hist : 1));
    std::vector<size_t> hnext(V, 0), hcount(V, 0);
    int reason = 2;  // 0 ALL_CONVERGED, 1 BIG_FRAC_CONVERGED, 2 DIVERGED
    std::vector<double> nb;
    for (;; numIters++, b.iters++) {
        if (numIters >= minIters) nodeFracTol = (double)(numIters - minIters) / (double)(maxIters - minIters);
        if (maxDiff <= tol) {
            reason = 0;
            break;
        } else if (numIters > minIters && frac < nodeFracTol) {
            reason = 1;
            break;
        } else if (numIters > maxIters) {
            reason = 2;
            break;
        } else if ((now_s() - tic) > maxtime) {
            reason = 2;
            break;
        }
        bp_sweep(b);
        bp_beliefs(b, nb);
        double diff = 0.0;
        size_t nonconv = 0;
        for (size_t i = 0; i < V; i++) {
            double dd = std::fabs(b.oldBeliefs[i] - nb[i]);
            diff = (diff < dd) ? dd : diff;
            nonconv += (size_t)(dd > tol);
        }
        b.oldBeliefs = nb;
        maxDiff = std::max(diff, -(double)INFINITY);
        for (size_t i = 0; i < V; i++) {
            double v = nb[i];
            int c = std::fpclassify(v);
            if (c != FP_NORMAL && c != FP_SUBNORMAL && c != FP_ZERO) continue;
            size_t slot = hnext[i];
            hvals[slot * V + i] = v;
            if (++slot == hist) slot = 0;
            hnext[i] = slot;
            if (hcount[i] < hist) hcount[i]++;
        }
        frac = V ? (double)nonconv / (double)V : NAN;
    }
    if (maxDiff > b.maxdiff_member) b.maxdiff_member = maxDiff;
    b.beliefs = b.oldBeliefs;
    b.lowpass.assign(V, 0.0);
    for (size_t i = 0; i < V; i++) {
        if (reason == 0) {
            b.lowpass[i] = b.beliefs[i];
        } else {
            size_t cnt = hcount[i];
            size_t slot = (cnt == hist) ? hnext[i] : 0;
            double sum = 0.0;
            for (size_t s = 0; s < cnt; s++) {
                sum += hvals[slot * V + i];
                if (++slot == hist) slot = 0;
            }
            if (cnt > 0) sum /= (double)cnt;
            b.lowpass[i] = sum;
        }
    }
    if (reason_out) *reason_out = reason;
    if (sweeps_out) *sweeps_out = numIters;
    return frac;
}

thread_local std::string g_err;

template <class F>
int guarded(F &&f) {
    try {
        f();
        return 0;
    } catch (const std::exception &e) {
        g_err = e.what();
        return -1;
    }
}

}  // namespace

// ------------------------------------------------------------------ C ABI

extern "C" {

const char *orc_last_error() { return g_err.c_str(); }

void *orc_read_file(const char *path) {
    OGraph *g = nullptr;
    int rc = guarded([&] {
        std::ifstream in(path);
        if (!in.is_open()) throw std::runtime_error(std::string("Cannot read from file ") + path);
        g = new OGraph(build_graph(parse_causal_fg(in)));
    });
    return rc ? nullptr : g;
}

void *orc_read_string(const char *text) {
    OGraph *g = nullptr;
    int rc = guarded([&] {
        std::istringstream in(text);
        g = new OGraph(build_graph(parse_causal_fg(in)));
    });
    return rc ? nullptr : g;
}

// Factors given as parallel arrays; body labels in CSR form (body_off has n+1 entries).
void *orc_from_factors(int64_t n, const int32_t *type, const int64_t *head, const int64_t *body_off,
                       const int64_t *body, const double *p, const double *q) {
    OGraph *g = nullptr;
    int rc = guarded([&] {
        std::vector<OFactor> facs;
        facs.reserve((size_t)n);
        for (int64_t I = 0; I < n; I++) {
            if (type[I] == 0) {
                facs.push_back(make_singleton((uint64_t)head[I], p[I]));
            } else {
                std::vector<uint64_t> b;
                for (int64_t k = body_off[I]; k < body_off[I + 1]; k++) b.push_back((uint64_t)body[k]);
                facs.push_back(make_rule((uint64_t)head[I], b, type[I] == 1, p[I], q[I]));
            }
        }
        g = new OGraph(build_graph(facs));
    });
    return rc ? nullptr : g;
}

void orc_free(void *g) { delete (OGraph *)g; }

int orc_clamp(void *g, int64_t i, int64_t x) {
    return guarded([&] { clamp_graph(*(OGraph *)g, (size_t)i, (size_t)x); });
}

void *orc_rebuild(void *g) { return new OGraph(build_graph(((OGraph *)g)->factors)); }

int64_t orc_nr_vars(void *g) { return (int64_t)((OGraph *)g)->vars.size(); }
int64_t orc_nr_factors(void *g) { return (int64_t)((OGraph *)g)->factors.size(); }
int64_t orc_nr_edges(void *g) {
    int64_t s = 0;
    for (auto &n : ((OGraph *)g)->nbV) s += (int64_t)n.size();
    return s;
}
// Sum of |vars()| over factors (the message length of causal_bp.cu:319-322).
int64_t orc_nr_slots(void *g) {
    int64_t s = 0;
    for (auto &f : ((OGraph *)g)->factors) s += (int64_t)f.vars.size();
    return s;
}

void orc_vars(void *g, int64_t *labels) {
    auto &G = *(OGraph *)g;
    for (size_t i = 0; i < G.vars.size(); i++) labels[i] = (int64_t)G.vars[i];
}

void orc_factor_info(void *g, int32_t *type, int64_t *head, double *p, double *q, int32_t *clamped,
                     double *m0, double *m1, int64_t *nvars) {
    auto &G = *(OGraph *)g;
    for (size_t I = 0; I < G.factors.size(); I++) {
        auto &f = G.factors[I];
        type[I] = f.type;
        head[I] = (int64_t)f.head;
        p[I] = f.p;
        q[I] = f.q;
        clamped[I] = f.head_clamped ? 1 : 0;
        m0[I] = f.mask0;
        m1[I] = f.mask1;
        nvars[I] = (int64_t)f.vars.size();
    }
}

// Per-factor vars() labels in CSR form (off has F+1 entries).
void orc_factor_vars(void *g, int64_t *off, int64_t *labels) {
    auto &G = *(OGraph *)g;
    int64_t k = 0;
    off[0] = 0;
    for (size_t I = 0; I < G.factors.size(); I++) {
        for (uint64_t l : G.factors[I].vars) labels[k++] = (int64_t)l;
        off[I + 1] = k;
    }
}

// nbV / nbF neighbour lists (node, iter, dual) in CSR form.
void orc_neighbors(void *g, int which_factor, int64_t *off, int64_t *node, int64_t *iter, int64_t *dual) {
    auto &G = *(OGraph *)g;
    auto &nb = which_factor ? G.nbF : G.nbV;
    int64_t k = 0;
    off[0] = 0;
    for (size_t a = 0; a < nb.size(); a++) {
        for (auto &n : nb[a]) {
            node[k] = (int64_t)n.node;
            iter[k] = (int64_t)n.iter;
            dual[k] = (int64_t)n.dual;
            k++;
        }
        off[a + 1] = k;
    }
}

// construct() outputs. Sizes: row_ptr_vf F+1, col_ind_vf E, row_ptr_fv V+1, col_ind_fv E, head F,
// rec_* E (variable-major), vf_* E (factor-major).
void orc_construct(void *g, int64_t *row_ptr_vf, int64_t *col_ind_vf, int64_t *row_ptr_fv, int64_t *col_ind_fv,
                   int64_t *head, int64_t *rec_i, double *rec_r, int64_t *vf_i) {
    OLayout L = construct(*(OGraph *)g);
    for (size_t a = 0; a < L.row_ptr_vf.size(); a++) row_ptr_vf[a] = (int64_t)L.row_ptr_vf[a];
    for (size_t a = 0; a < L.col_ind_vf.size(); a++) col_ind_vf[a] = (int64_t)L.col_ind_vf[a];
    for (size_t a = 0; a < L.row_ptr_fv.size(); a++) row_ptr_fv[a] = (int64_t)L.row_ptr_fv[a];
    for (size_t a = 0; a < L.col_ind_fv.size(); a++) col_ind_fv[a] = (int64_t)L.col_ind_fv[a];
    for (size_t a = 0; a < L.head.size(); a++) head[a] = (int64_t)L.head[a];
    for (size_t k = 0; k < L.rec.size(); k++) {
        const ORec &r = L.rec[k];
        int64_t *o = rec_i + 6 * k;
        o[0] = (int64_t)r.type;
        o[1] = (int64_t)r.v;
        o[2] = (int64_t)r.src;
        o[3] = (int64_t)r.start;
        o[4] = (int64_t)r.end;
        o[5] = (int64_t)r.head;
        double *d = rec_r + 4 * k;
        d[0] = r.q;
        d[1] = r.p;
        d[2] = r.m0;
        d[3] = r.m1;
    }
    for (size_t k = 0; k < L.vf.size(); k++) {
        vf_i[3 * k] = (int64_t)L.vf[k].ind;
        vf_i[3 * k + 1] = (int64_t)L.vf[k].v;
        vf_i[3 * k + 2] = (int64_t)L.vf[k].src;
    }
}

void *orc_bp_create(void *g, double damping, int nthreads, int logdomain) {
    OBP *b = bp_create(*(OGraph *)g, damping, nthreads);
    b->logdomain = logdomain != 0;
    return b;
}

// Arithmetic mode (takes effect at the next init): 0 the reference's
// probability-space arithmetic, 1 log-odds (no underflow), 2 the reference's
// arithmetic with underflow tracking.
int orc_bp_set_mode(void *b, int mode) {
    auto &B = *(OBP *)b;
    if (mode < 0 || mode > 2) return -1;
    B.lodds = mode == 1;
    B.track = mode == 2;
    return 0;
}

// Underflow tracking: per variable 1 if its belief depends on an underflow;
// returns the number of underflow events since init (messages or totals that
// underflowed from inputs that did not).
int64_t orc_bp_underflow(void *b, uint8_t *var_taint) {
    auto &B = *(OBP *)b;
    if (!B.track) return -1;
    for (size_t i = 0; i < B.V; i++) var_taint[i] = B.t_var.empty() ? 0 : B.t_var[i];
    return (int64_t)B.underflow_events;
}
void orc_bp_free(void *b) { delete (OBP *)b; }
int64_t orc_bp_nr_vars(void *b) { return (int64_t)((OBP *)b)->V; }
int64_t orc_bp_nr_slots(void *b) { return (int64_t)((OBP *)b)->E; }
int64_t orc_bp_iters(void *b) { return (int64_t)((OBP *)b)->iters; }
void orc_bp_set_threads(void *b, int n) { ((OBP *)b)->nthreads = n < 1 ? 1 : n; }
void orc_bp_init(void *b) { bp_init(*(OBP *)b); }
void orc_bp_sweep(void *b) { bp_sweep(*(OBP *)b); }

double orc_bp_run_tol(void *b, double tol, int64_t maxiter, double maxtime) {
    double md = 0;
    bp_run_tol(*(OBP *)b, tol, (size_t)maxiter, maxtime, &md);
    return md;
}

double orc_bp_run_fixed(void *b, double tol, int64_t maxIters, int64_t hist) {
    return bp_run_fixed(*(OBP *)b, tol, (size_t)maxIters, (size_t)hist);
}

double orc_bp_run_lowpass(void *b, double tol, int64_t minIters, int64_t maxIters, int64_t hist, double maxtime,
                          int32_t *reason, int64_t *sweeps) {
    size_t sw = 0;
    int rs = 0;
    double r = bp_run_lowpass(*(OBP *)b, tol, (size_t)minIters, (size_t)maxIters, (size_t)hist, maxtime, &rs, &sw);
    if (reason) *reason = rs;
    if (sweeps) *sweeps = (int64_t)sw;
    return r;
}

// _beliefsV (host copy after a run), _lowPassBeliefs, and the current b1/(b0+b1).
void orc_bp_beliefs(void *b, double *out) {
    auto &B = *(OBP *)b;
    for (size_t i = 0; i < B.V; i++) out[i] = B.beliefs[i];
}
int orc_bp_lowpass(void *b, double *out) {
    auto &B = *(OBP *)b;
    if (B.lowpass.size() != B.V) return -1;
    for (size_t i = 0; i < B.V; i++) out[i] = B.lowpass[i];
    return 0;
}
void orc_bp_current_beliefs(void *b, double *out) {
    std::vector<double> nb;
    bp_beliefs(*(OBP *)b, nb);
    for (size_t i = 0; i < nb.size(); i++) out[i] = nb[i];
}

// Messages: f->v in variable-major order, v->f in factor-major order.
void orc_bp_messages(void *b, double *fv0, double *fv1, double *vf0, double *vf1) {
    auto &B = *(OBP *)b;
    if (B.lodds) {  // normalised pairs of the log-odds
        auto pair = [](double l, double &m0, double &m1) {
            if (std::isnan(l)) {
                m0 = m1 = l;
                return;
            }
            m1 = std::exp(lsig(l));
            m0 = std::exp(lsig(-l));
        };
        for (size_t k = 0; k < B.E; k++) {
            pair(B.lfv[k], fv0[k], fv1[k]);
            pair(B.lvf[k], vf0[k], vf1[k]);
        }
        return;
    }
    for (size_t k = 0; k < B.E; k++) {
        fv0[k] = B.fv0[k];
        fv1[k] = B.fv1[k];
        vf0[k] = B.vf0[k];
        vf1[k] = B.vf1[k];
    }
}

// Switch to a sequential schedule: kind 1 SEQFIX with the factor order
// shuffled by std::mt19937(seed), kind 2 TOPO. Returns the number of batches.
int64_t orc_bp_set_schedule(void *b, int kind, uint32_t seed) {
    auto &B = *(OBP *)b;
    if (kind == 1) seq_batches(B, seqfix_order(B.g, seed), false);
    else if (kind == 2) seq_batches(B, topo_order(B.g), true);
    else return -1;
    B.seq = true;
    return (int64_t)B.seq_fv.size();
}

// The update sequence as factor-major slots (row_ptr_vf[I] + iter) and the
// batch of every slot.
void orc_bp_schedule(void *b, int64_t *seq_slots, int64_t *slot_batch) {
    auto &B = *(OBP *)b;
    for (size_t k = 0; k < B.seq_slots.size(); k++) seq_slots[k] = (int64_t)B.seq_slots[k];
    for (size_t k = 0; k < B.slot_batch.size(); k++) slot_batch[k] = (int64_t)B.slot_batch[k];
}

// Overwrite v->f messages (factor-major); lets tests drive single f->v evaluations.
void orc_bp_set_vf(void *b, const double *vf0, const double *vf1) {
    auto &B = *(OBP *)b;
    for (size_t k = 0; k < B.E; k++) {
        B.vf0[k] = vf0[k];
        B.vf1[k] = vf1[k];
    }
}

}  // extern "C"
