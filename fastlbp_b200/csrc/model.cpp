// Host implementation of the libDAI-style graph model of the drop-in API:
// multi-index helpers, the generic FactorGraph reader, CausalFactor,
// CausalFactorGraph (.causal_fg reader, construction, clamping) and the
// conversion of a CausalFactorGraph into the engine's reference-order arrays.

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <climits>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <map>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <string_view>
#include <unordered_map>
#include <vector>

#include <ext/causal_bp.h>
#include <ext/causal_factor.h>
#include <ext/causal_fg.h>
#include <lbp/factorgraph.h>
#include <lbp/index.h>
#include <utils/log.h>
#include <utils/utils.h>

#include "model_internal.h"

namespace lbp {

thread_local rnd_gen_type rnd_gen(42U);

// ------------------------------------------------------------------ IndexFor

IndexFor::IndexFor(const VarSet &indexVars, const VarSet &forVars) : _state(forVars.size(), 0) {
    // Mixed-radix counter over forVars (first variable fastest). _sum[k] is the
    // stride of forVars[k] inside indexVars, or 0 when it is not an index variable.
    long stride = 1;
    auto j = forVars.begin();
    for (auto i = indexVars.begin(); i != indexVars.end(); ++i) {
        for (; j != forVars.end() && *j <= *i; ++j) {
            _ranges.push_back(j->states());
            _sum.push_back((*i == *j) ? stride : 0);
        }
        stride *= (long)i->states();
    }
    for (; j != forVars.end(); ++j) {
        _ranges.push_back(j->states());
        _sum.push_back(0);
    }
    _index = 0;
}

IndexFor &IndexFor::reset() {
    std::fill(_state.begin(), _state.end(), 0);
    _index = 0;
    return *this;
}

IndexFor &IndexFor::operator++() {
    if (_index < 0) return *this;
    size_t k = 0;
    for (; k < _state.size(); k++) {
        _index += _sum[k];
        if (++_state[k] < _ranges[k]) break;
        _index -= _sum[k] * (long)_ranges[k];
        _state[k] = 0;
    }
    if (k == _state.size()) _index = -1;
    return *this;
}

Permute::Permute(const std::vector<Var> &vars, bool reverse) {
    // _ranges: state counts in the given order; _sigma[j]: given position of the
    // j-th variable in label order.
    const size_t n = vars.size();
    std::vector<size_t> order(n);
    for (size_t k = 0; k < n; k++) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return vars[a] < vars[b]; });
    for (size_t k = 0; k < n; k++) _ranges.push_back(vars[k].states());
    _sigma = order;
    if (reverse) {
        std::vector<size_t> inv(n);
        for (size_t k = 0; k < n; k++) inv[order[k]] = k;
        _sigma = inv;
    }
}

size_t Permute::convertLinearIndex(size_t li) const {
    // Decode li in the given variable order (first fastest), re-encode in label order.
    const size_t n = _ranges.size();
    std::vector<size_t> st(n);
    for (size_t k = 0; k < n; k++) {
        st[k] = li % _ranges[k];
        li /= _ranges[k];
    }
    size_t out = 0, stride = 1;
    for (size_t j = 0; j < n; j++) {
        out += st[_sigma[j]] * stride;
        stride *= _ranges[_sigma[j]];
    }
    return out;
}

// --------------------------------------------------------------- FactorGraph

void FactorGraph::constructGraph(size_t nrEdges) {
    std::unordered_map<size_t, size_t> idx;
    for (size_t i = 0; i < _vars.size(); i++) idx[_vars[i].label()] = i;
    std::vector<Edge> edges;
    edges.reserve(nrEdges);
    for (size_t I = 0; I < _factors.size(); I++)
        for (const auto &v : _factors[I].vars()) edges.push_back(Edge(idx[v.label()], I));
    _G.construct(_vars.size(), _factors.size(), edges.begin(), edges.end());
}

FactorGraph::FactorGraph(const std::vector<Factor> &P) {
    std::set<Var> vs;
    size_t nrEdges = 0;
    _factors.reserve(P.size());
    for (const auto &f : P) {
        _factors.push_back(f);
        vs.insert(f.vars().begin(), f.vars().end());
        nrEdges += f.vars().size();
    }
    _vars.assign(vs.begin(), vs.end());
    constructGraph(nrEdges);
}

size_t FactorGraph::findVar(const Var &n) const {
    size_t i = std::find(_vars.begin(), _vars.end(), n) - _vars.begin();
    if (i == nrVars()) std::cerr << "var not found \n";
    return i;
}

void FactorGraph::ReadFromFile(const char *filename) {
    std::ifstream in(filename);
    if (!in.is_open()) exit(1);
    in >> *this;
}

// libDAI ".fg" format: factor count, then per factor the member count, member
// labels, member state counts, the number of listed entries and
// (linear index, value) pairs in the listed member order.
std::istream &operator>>(std::istream &is, FactorGraph &fg) {
    std::string line;
    size_t nr;
    read_annotation(is, line);
    is >> nr;
    if (is.fail()) exit(1);
    std::getline(is, line);
    if (is.fail() || line.size() > 0) exit(1);
    std::map<long, size_t> dims_seen;
    std::vector<Factor> facs;
    for (size_t I = 0; I < nr; I++) {
        size_t m;
        read_annotation(is, line);
        is >> m;
        std::vector<long> labels(m);
        for (auto &l : labels) {
            read_annotation(is, line);
            is >> l;
        }
        std::vector<size_t> dims(m);
        for (auto &d : dims) {
            read_annotation(is, line);
            is >> d;
        }
        std::vector<Var> ivars;
        for (size_t k = 0; k < m; k++) {
            auto it = dims_seen.find(labels[k]);
            if (it != dims_seen.end() && it->second != dims[k]) exit(1);
            dims_seen[labels[k]] = dims[k];
            ivars.push_back(Var((size_t)labels[k], dims[k]));
        }
        facs.push_back(Factor(VarSet(ivars.begin(), ivars.end(), ivars.size()), (Real)0.0));
        Permute perm(ivars);
        size_t nnz;
        read_annotation(is, line);
        is >> nnz;
        for (size_t k = 0; k < nnz; k++) {
            size_t li;
            Real val;
            read_annotation(is, line);
            is >> li;
            read_annotation(is, line);
            is >> val;
            facs.back().set(perm.convertLinearIndex(li), val);
        }
    }
    fg = FactorGraph(facs);
    return is;
}

// -------------------------------------------------------------- CausalFactor

CausalFactor::CausalFactor(const Var &v, Real p) : _type(Singleton), _head(v), _body(), _p(p) {
    _vs = VarSet(_head);
    head_clamped = false;
    head_mask = Prob(2, 1);
}

CausalFactor::CausalFactor(const Var &head, const VarSet &body, bool isAnd, Real p, Real q)
    : _type(isAnd ? DefiniteAnd : DefiniteOr), _head(head), _body(body), _p(p), _q(q) {
    _vs = VarSet(_body);
    _vs.insert(_head);
    head_clamped = false;
    head_mask = Prob(2, 1);
}

int CausalFactor::type() const {
    switch (_type) {
        case Singleton: return 0;
        case DefiniteAnd: return 1;
        case DefiniteOr: return 2;
    }
    LOG_FATAL("unreachable");
}

CausalFactor CausalFactor::gen_clamped(Var i, size_t x) const {
    CausalFactor nf(*this);
    if (_type == Singleton) {
        if (i == _head) nf._p = (Real)x;
        else std::cerr << "Clamp unrelated var " << i << " in factor " << *this << std::endl;
        return nf;
    }
    if (i == _head) {
        nf.head_clamped = true;
        nf.head_mask = Prob(2, 0);
        nf.head_mask.set(x, 1);  // throws std::out_of_range for x > 1, as Prob::set does
        if (head_clamped) {
            std::cerr << "Duplicate clamp head of factor " << *this << "with val " << x << std::endl;
            nf.head_mask *= head_mask;
        }
    } else if (_body.contains(i)) {
        nf._body.erase(i);
        nf._vs.erase(i);
        const bool resolves = (x == 0 && _type == DefiniteAnd) || (x > 0 && _type == DefiniteOr);
        if (resolves) {  // the rule's outcome no longer depends on its body
            nf._p = _q;
            nf._body = VarSet();
            nf._vs = VarSet(_head);
        }
    }
    return nf;
}

std::ostream &operator<<(std::ostream &os, const CausalFactor &f) {
    os << f.head() << std::endl << static_cast<char>(f._type);
    if (f._type == CausalFactor::Singleton) {
        os << std::endl << std::setw(os.precision() + 4) << f.prob() << std::endl;
    } else {
        os << std::setw(os.precision() + 4) << f.prob() << ";" << std::setw(os.precision() + 4) << f.prob_default()
           << std::endl;
        os << f.body().size() << std::endl;
        for (const auto &v : f.body()) os << v.label() << " ";
        os << std::endl;
    }
    return os << std::endl;
}

// ---------------------------------------------------------- CausalFactorGraph

void CausalFactorGraph::constructGraph(size_t nrEdges) {
    // label -> variable index: a direct table when the labels are dense
    // (the usual 0..V-1), else a hash map
    const size_t V = _vars.size();
    const size_t max_label = V ? _vars.back().label() : 0;  // _vars is sorted by label
    std::vector<uint32_t> dense;
    std::unordered_map<size_t, size_t> idx;
    const bool use_dense = V && V < UINT32_MAX && max_label < 4 * V + 1024;
    if (use_dense) {
        dense.assign(max_label + 1, UINT32_MAX);
        for (size_t i = 0; i < V; i++) dense[_vars[i].label()] = (uint32_t)i;
    } else {
        idx.reserve(V * 2 + 1);
        for (size_t i = 0; i < V; i++) idx[_vars[i].label()] = i;
    }
    std::vector<Edge> edges;
    edges.reserve(nrEdges);
    for (size_t I = 0; I < _factors.size(); I++)
        for (const auto &v : _factors[I].vars())
            edges.push_back(Edge(use_dense ? (size_t)dense[v.label()] : idx[v.label()], I));
    _G.construct(V, _factors.size(), edges.begin(), edges.end(), false);
}

CausalFactorGraph::CausalFactorGraph(const std::vector<CausalFactor> &P) : CausalFactorGraph(std::vector<CausalFactor>(P)) {}

CausalFactorGraph::CausalFactorGraph(std::vector<CausalFactor> &&P) {
    _factors = std::move(P);
    size_t nrEdges = 0, max_label = 0;
    for (const auto &f : _factors) {
        nrEdges += f.vars().size();
        for (const auto &v : f.vars()) max_label = std::max(max_label, v.label());
    }
    // the variables in ascending label order without repeats, each as first met
    // (what inserting them all into a std::set<Var> keeps)
    std::vector<Var> vs;
    if (nrEdges && max_label < 4 * nrEdges + 1024) {  // dense labels: a table of first occurrences
        std::vector<const Var *> first(max_label + 1, nullptr);
        for (const auto &f : _factors)
            for (const auto &v : f.vars())
                if (!first[v.label()]) first[v.label()] = &v;
        for (const Var *v : first)
            if (v) vs.push_back(*v);
    } else {
        vs.reserve(nrEdges);
        for (const auto &f : _factors) vs.insert(vs.end(), f.vars().begin(), f.vars().end());
        std::stable_sort(vs.begin(), vs.end());
        vs.erase(std::unique(vs.begin(), vs.end(), [](const Var &a, const Var &b) { return !(a < b) && !(b < a); }),
                 vs.end());
    }
    _vars = std::move(vs);
    constructGraph(nrEdges);
}

size_t CausalFactorGraph::findVar(const Var &n) const {
    size_t i = std::lower_bound(_vars.begin(), _vars.end(), n) - _vars.begin();
    if (i < _vars.size() && _vars[i] == n) return i;
    i = std::find(_vars.begin(), _vars.end(), n) - _vars.begin();  // labels are sorted; kept for safety
    if (i == nrVars()) std::cerr << "var not found \n";
    return i;
}

void CausalFactorGraph::clamp(size_t i, size_t x) {
    std::map<size_t, CausalFactor> nf;
    for (const Neighbor &I : nbV(i)) nf.emplace(I.node, factor(I).gen_clamped(var(i), x));
    setFactors(nf);
}

void CausalFactorGraph::ReadFromFile(const char *filename) {
    std::ifstream in(filename);
    if (!in.is_open()) LOG_FATAL("Cannot read from file %s.", filename);
    try {
        *this = detail::read_causal_fg_file(in);
    } catch (const detail::BadFactorType &) {
        LOG_FATAL("Unreachable");
    }
}

std::istream &operator>>(std::istream &is, CausalFactorGraph &fg) {
    try {
        fg = detail::parse_causal_fg(is);
    } catch (const detail::BadFactorType &) {
        LOG_FATAL("Unreachable");
    }
    return is;
}

namespace detail {

// Line sources of the reader, with the semantics of std::getline (false
// when nothing could be read: the stream's failbit) and of peeking at the
// next character.
struct StreamLines {
    std::istream &is;
    std::string buf;
    bool next(std::string_view &line) {
        std::getline(is, buf);
        line = buf;
        return !is.fail();
    }
    bool peek_hash() { return is.peek() == '#'; }
};

struct BufferLines {
    const char *p, *end;
    bool next(std::string_view &line) {
        if (p >= end) {
            line = std::string_view();
            return false;
        }
        const char *nl = static_cast<const char *>(std::memchr(p, '\n', (size_t)(end - p)));
        const char *e = nl ? nl : end;
        line = std::string_view(p, (size_t)(e - p));
        p = nl ? nl + 1 : end;
        return true;
    }
    bool peek_hash() { return p < end && *p == '#'; }
};

// std::stoi / std::stold on a line: the same conversion (strtol / strtold on
// the line alone) and the same exceptions.
int line_stoi(std::string_view s) {
    char buf[64];
    if (s.size() >= sizeof buf) return std::stoi(std::string(s));
    std::memcpy(buf, s.data(), s.size());
    buf[s.size()] = 0;
    char *e = nullptr;
    errno = 0;
    const long v = std::strtol(buf, &e, 10);
    if (e == buf) throw std::invalid_argument("stoi");
    if (errno == ERANGE || v < INT_MIN || v > INT_MAX) throw std::out_of_range("stoi");
    return (int)v;
}

long double line_stold(std::string_view s) {
    char buf[128];
    if (s.size() >= sizeof buf) return std::stold(std::string(s));
    std::memcpy(buf, s.data(), s.size());
    buf[s.size()] = 0;
    char *e = nullptr;
    errno = 0;
    const long double v = std::strtold(buf, &e);
    if (e == buf) throw std::invalid_argument("stold");
    if (errno == ERANGE) throw std::out_of_range("stold");
    return v;
}

// Successive `long` extractions from a line as an istringstream performs
// them: leading white space skipped; after a failed extraction (no number,
// or out of range: LONG_MAX / LONG_MIN) every later one yields 0.
struct LongReader {
    const char *p, *end;
    bool ok = true;
    long next() {
        if (!ok) return 0;
        while (p < end && std::isspace((unsigned char)*p)) p++;
        const char *q = p;
        bool neg = false;
        if (q < end && (*q == '+' || *q == '-')) neg = *q++ == '-';
        if (q >= end || !std::isdigit((unsigned char)*q)) {
            ok = false;
            return 0;
        }
        unsigned long long mag = 0;
        bool over = false;
        for (; q < end && std::isdigit((unsigned char)*q); q++) {
            const unsigned d = (unsigned)(*q - '0');
            if (mag > (ULLONG_MAX - d) / 10) over = true;
            else mag = mag * 10 + d;
        }
        p = q;
        const unsigned long long lim = neg ? (unsigned long long)LONG_MAX + 1ull : (unsigned long long)LONG_MAX;
        if (over || mag > lim) {
            ok = false;
            return neg ? LONG_MIN : LONG_MAX;
        }
        return neg ? (long)(0ull - mag) : (long)mag;
    }
};

// The .causal_fg grammar of csrc/ext/causal_fg.cpp:129-279: a factor count;
// per factor a separating blank line, the head id, a type line ("I", or "*" /
// "+" optionally followed by "p;q", defaults p=1, q=0), then for "I" the
// probability, else the body length and the body ids on one line. Lines
// starting with '#' directly after a consumed line are skipped. Variables
// never used as a head get Singleton(0.5), appended in ascending label order.
template <typename Lines>
CausalFactorGraph parse_lines(Lines &in) {
    std::vector<CausalFactor> facs;
    std::string_view line;
    auto skip_annotation = [&] {
        std::string_view c;
        while (in.peek_hash()) in.next(c);
    };
    in.next(line);
    skip_annotation();
    const size_t nr = (size_t)line_stoi(line);
    std::vector<size_t> heads, all_vars;  // sorted and de-duplicated at the end
    facs.reserve(nr);
    heads.reserve(nr);
    std::vector<Var> body_vars;
    for (size_t I = 0; I < nr; I++) {
        if (!in.next(line) || line.size() > 0) LOG_ERROR("Expecting empty line");
        in.next(line);
        skip_annotation();
        const size_t head_id = (size_t)line_stoi(line);
        const Var head(head_id, 2);
        heads.push_back(head_id);
        all_vars.push_back(head_id);
        in.next(line);
        skip_annotation();
        const char ch = line.empty() ? '\0' : line.front();
        if (ch != CausalFactor::Singleton && ch != CausalFactor::DefiniteAnd && ch != CausalFactor::DefiniteOr)
            throw BadFactorType();
        if (ch == CausalFactor::Singleton) {
            in.next(line);
            skip_annotation();
            const Real prob = static_cast<Real>(line_stold(line));
            facs.emplace_back(head, prob);
            continue;
        }
        Real prob = 1, prob_default = 0;
        if (line.length() > 1) {
            const size_t sp = line.find(';');
            if (sp > 1) prob = static_cast<Real>(line_stold(line.substr(1, sp - 1)));
            if (sp != std::string_view::npos && sp + 1 != line.length())
                prob_default = static_cast<Real>(line_stold(line.substr(sp + 1)));
        }
        in.next(line);
        skip_annotation();
        const size_t blen = (size_t)line_stoi(line);
        in.next(line);
        skip_annotation();
        LongReader ids{line.data(), line.data() + line.size()};
        body_vars.clear();
        body_vars.reserve(blen);
        for (size_t b = 0; b < blen; b++) {
            const long id = ids.next();
            body_vars.emplace_back((size_t)id, 2);
            all_vars.push_back((size_t)id);
        }
        VarSet body(body_vars.begin(), body_vars.end(), body_vars.size());
        facs.emplace_back(head, body, ch == CausalFactor::DefiniteAnd, prob, prob_default);
    }
    std::sort(heads.begin(), heads.end());
    heads.erase(std::unique(heads.begin(), heads.end()), heads.end());
    std::sort(all_vars.begin(), all_vars.end());
    all_vars.erase(std::unique(all_vars.begin(), all_vars.end()), all_vars.end());
    for (size_t v : all_vars)
        if (!std::binary_search(heads.begin(), heads.end(), v)) facs.emplace_back(Var(v, 2), 0.5);
    return CausalFactorGraph(std::move(facs));
}

CausalFactorGraph parse_causal_fg(std::istream &is) {
    StreamLines in{is, {}};
    return parse_lines(in);
}

CausalFactorGraph parse_causal_fg_text(const char *text, size_t n) {
    BufferLines in{text, text + n};
    return parse_lines(in);
}

CausalFactorGraph read_causal_fg_file(std::ifstream &f) {
    std::string buf;
    f.seekg(0, std::ios::end);
    const std::streamoff sz = f.tellg();
    f.seekg(0, std::ios::beg);
    if (sz > 0) {
        buf.resize((size_t)sz);
        f.read(&buf[0], sz);
        buf.resize((size_t)f.gcount());
    }
    return parse_causal_fg_text(buf.data(), buf.size());
}

int build_arrays(const CausalFactorGraph &fg, GraphArrays &a, std::string &err) {
    const size_t V = fg.nrVars(), F = fg.nrFactors();
    // label -> variable index: a direct table when the labels are dense, else a hash map
    size_t max_label = 0;
    for (size_t i = 0; i < V; i++) max_label = std::max(max_label, fg.var(i).label());
    const bool use_dense = V && V < UINT32_MAX && max_label < 4 * V + 1024;
    std::vector<uint32_t> dense;
    std::unordered_map<size_t, size_t> idx;
    if (use_dense) {
        dense.assign(max_label + 1, UINT32_MAX);
        for (size_t i = 0; i < V; i++) dense[fg.var(i).label()] = (uint32_t)i;
    } else {
        idx.reserve(V * 2 + 1);
        for (size_t i = 0; i < V; i++) idx[fg.var(i).label()] = i;
    }
    auto index_of = [&](size_t label, size_t &out) {
        if (use_dense) {
            if (label > max_label || dense[label] == UINT32_MAX) return false;
            out = dense[label];
            return true;
        }
        auto it = idx.find(label);
        if (it == idx.end()) return false;
        out = it->second;
        return true;
    };
    a = GraphArrays();
    a.offsets.assign(F + 1, 0);
    a.head.assign(F, 0);
    a.type.assign(F, 0);
    a.p.assign(F, 0);
    a.q.assign(F, 0);
    a.clamped.assign(F, 0);
    a.m0.assign(F, 1);
    a.m1.assign(F, 1);
    size_t E = 0;
    for (size_t I = 0; I < F; I++) E += fg.factor(I).vars().size();
    a.slot_var.reserve(E);
    for (size_t I = 0; I < F; I++) {
        const CausalFactor &f = fg.factor(I);
        const size_t hl = f.head().label();
        bool found = false;
        for (const auto &v : f.vars()) {
            size_t vi = 0;
            if (!index_of(v.label(), vi)) {
                err = "factor " + std::to_string(I) + " uses variable x" + std::to_string(v.label()) +
                      " that is not in the graph";
                return 1;
            }
            if (v.label() == hl) {
                a.head[I] = (int64_t)a.slot_var.size();
                found = true;
            }
            a.slot_var.push_back((int64_t)vi);
        }
        if (!found) {
            err = "factor " + std::to_string(I) + " does not contain its head";
            return 1;
        }
        a.offsets[I + 1] = (int64_t)a.slot_var.size();
        a.type[I] = f.type();
        a.p[I] = f.prob();
        a.q[I] = f.prob_default();
        a.clamped[I] = f.head_clamped ? 1 : 0;
        a.m0[I] = f.head_mask.size() > 0 ? f.head_mask[0] : 1.0;
        a.m1[I] = f.head_mask.size() > 1 ? f.head_mask[1] : 1.0;
    }
    a.desc.n_vars = (int64_t)V;
    a.desc.n_factors = (int64_t)F;
    a.desc.n_slots = (int64_t)a.slot_var.size();
    a.desc.factor_offsets = a.offsets.data();
    a.desc.slot_var = a.slot_var.data();
    a.desc.factor_head = a.head.data();
    a.desc.factor_type = a.type.data();
    a.desc.factor_p = a.p.data();
    a.desc.factor_q = a.q.data();
    a.desc.factor_head_clamped = a.clamped.data();
    a.desc.factor_mask0 = a.m0.data();
    a.desc.factor_mask1 = a.m1.data();
    return 0;
}

}  // namespace detail

}  // namespace lbp
