// Host-side construction of the engine's device layout from a graph in the
// reference's factor-major order (the arrays of CausalBP::construct(),
// csrc/ext/causal_bp.cu:310-407).
//
// What differs from the reference layout, and why:
// * Factors whose f->v messages never depend on other messages are folded
//   into per-variable priors instead of being recomputed every sweep:
//   singletons (type 0, causal_bp_parall.cu:110-112), AND/OR factors reduced
//   to their head (the `end_ind - start_ind == 1` cases, :115-117, :154-156),
//   and the head output of head-clamped factors (types 3/4, :222-238: with a
//   0/1 mask the normalised result is always the mask's one-hot state).
// * Factors and variables are sorted by degree and stored as sliced ELL of
//   width 32 (see engine_internal.h), so a warp handles 32 items of equal
//   degree with coalesced loads and no divergence; the head of every factor
//   is its slot 0.
// * All offsets and indices are 32-bit.
//
// The build runs on all host threads (OpenMP) and gives the same layout as
// a sequential build: parallel counting sorts keep items in index order
// within each class, and every per-item result is written by one thread.

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <string>
#include <vector>

#include "engine_internal.h"
#include "logodds.h"

namespace flbp {

namespace {

constexpr double kInf = std::numeric_limits<double>::infinity();

inline double logit(double p) { return det_logit(p); }

// Items [0, n) cut into T contiguous chunks (T = 1 for small n), one per
// parallel iteration, so that per-chunk results combine in index order.
constexpr int64_t kParMin = 1 << 15;

struct Chunks {
    int T;
    int64_t n, len;
    int64_t lo(int t) const { return std::min(n, (int64_t)t * len); }
    int64_t hi(int t) const { return std::min(n, (int64_t)(t + 1) * len); }
};

Chunks chunks(int64_t n, size_t nk = 1) {
    int T = n >= kParMin ? omp_get_max_threads() : 1;
    // per-chunk class counters stay below 32 M words
    T = (int)std::max<int64_t>(1, std::min<int64_t>(T, (int64_t)(32u << 20) / (int64_t)std::max<size_t>(1, nk)));
    return {T, n, std::max<int64_t>(1, (n + T - 1) / T)};
}

// Counting sort in two steps. class_counts: per chunk, the number of items
// of each class k < nk (key(i) >= nk: not placed). class_place: put(i, pos)
// for every placed item, pos = start[k] + the number of items of class k
// before i, i.e. classes at the given starts, items of a class in index
// order.
template <typename Key>
std::vector<uint64_t> class_counts(const Chunks &c, size_t nk, Key key) {
    std::vector<uint64_t> cnt((size_t)c.T * nk, 0);
#pragma omp parallel for schedule(static, 1) if (c.T > 1)
    for (int t = 0; t < c.T; t++) {
        uint64_t *h = &cnt[(size_t)t * nk];
        for (int64_t i = c.lo(t); i < c.hi(t); i++) {
            const size_t k = key(i);
            if (k < nk) h[k]++;
        }
    }
    return cnt;
}

template <typename Key, typename Put>
void class_place(const Chunks &c, size_t nk, const std::vector<uint64_t> &cnt, const std::vector<uint64_t> &start,
                 Key key, Put put) {
    std::vector<uint64_t> at((size_t)c.T * nk);
    for (size_t k = 0; k < nk; k++) {
        uint64_t p = start[k];
        for (int t = 0; t < c.T; t++) {
            at[(size_t)t * nk + k] = p;
            p += cnt[(size_t)t * nk + k];
        }
    }
#pragma omp parallel for schedule(static, 1) if (c.T > 1)
    for (int t = 0; t < c.T; t++) {
        uint64_t *a = &at[(size_t)t * nk];
        for (int64_t i = c.lo(t); i < c.hi(t); i++) {
            const size_t k = key(i);
            if (k < nk) put(i, a[k]++);
        }
    }
}

// Sizes of the classes (summed over chunks) and their starts from `base`.
std::vector<uint64_t> class_starts(const Chunks &c, size_t nk, const std::vector<uint64_t> &cnt, uint64_t base,
                                   std::vector<uint64_t> *sizes = nullptr) {
    std::vector<uint64_t> start(nk + 1, base);
    for (size_t k = 0; k < nk; k++) {
        uint64_t sz = 0;
        for (int t = 0; t < c.T; t++) sz += cnt[(size_t)t * nk + k];
        start[k + 1] = start[k] + sz;
    }
    if (sizes) {
        sizes->resize(nk);
        for (size_t k = 0; k < nk; k++) (*sizes)[k] = start[k + 1] - start[k];
    }
    return start;
}

inline void atomic_min_u32(uint32_t *p, uint32_t v) {
    uint32_t cur = __atomic_load_n(p, __ATOMIC_RELAXED);
    while (v < cur && !__atomic_compare_exchange_n(p, &cur, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
    }
}

// v = n copies of x, filled by all threads (first touch spread over them).
template <class T, class X>
void par_assign(hvec<T> &v, size_t n, const X &x) {
    hvec<T>().swap(v);
    v.resize(n);  // default-initialised: nothing written yet
    T *d = v.data();
    const T val = (T)x;
#pragma omp parallel for if ((int64_t)n >= kParMin)
    for (int64_t i = 0; i < (int64_t)n; i++) d[i] = val;
}

template <class T, class X>
hvec<T> par_vec(size_t n, const X &x) {
    hvec<T> v;
    par_assign(v, n, x);
    return v;
}

// v = the range [first, first + n), copied by all threads.
template <class T, class S>
void par_copy(hvec<T> &v, const S *first, size_t n) {
    hvec<T>().swap(v);
    v.resize(n);
    T *d = v.data();
#pragma omp parallel for if ((int64_t)n >= kParMin)
    for (int64_t i = 0; i < (int64_t)n; i++) d[i] = (T)first[i];
}

}  // namespace

bool classify_factor(const flbp_graph_desc &g, int64_t I, uint8_t &active, uint8_t &head_state, double &fconst,
                     std::string *msg) {
    auto fail = [&](const std::string &m) {
        if (msg) *msg = m;
        return false;
    };
    const int64_t *off = g.factor_offsets;
    active = 0;
    head_state = HEAD_FREE;
    fconst = 0.0;
    const int64_t d = off[I + 1] - off[I];
    const int32_t t = g.factor_type[I];
    const double p = g.factor_p[I], q = g.factor_q[I];
    if (t != FLBP_SINGLETON && t != FLBP_AND && t != FLBP_OR)
        return fail("unknown factor type at factor " + std::to_string(I));
    if (!(p >= 0.0 && p <= 1.0) || !(q >= 0.0 && q <= 1.0))
        return fail("factor probabilities must lie in [0,1] (factor " + std::to_string(I) + ")");
    if (d < 1) return fail("factor without variables at factor " + std::to_string(I));
    const int64_t h = g.factor_head[I];
    if (h < off[I] || h >= off[I + 1]) return fail("factor_head outside the factor's slots at factor " + std::to_string(I));
    if (t == FLBP_SINGLETON) {
        if (d != 1) return fail("singleton factor with more than one variable at factor " + std::to_string(I));
        fconst = logit(p);  // (1-p, p), causal_bp_parall.cu:110-112
        return true;
    }
    bool clamped = g.factor_head_clamped && g.factor_head_clamped[I];
    if (clamped) {
        const double m0 = g.factor_mask0 ? g.factor_mask0[I] : 1.0;
        const double m1 = g.factor_mask1 ? g.factor_mask1[I] : 1.0;
        if (!((m0 == 0.0 || m0 == 1.0) && (m1 == 0.0 || m1 == 1.0)))
            return fail("head_mask entries must be 0 or 1 (factor " + std::to_string(I) + ")");
        if (m0 == 1.0 && m1 == 1.0) {
            clamped = false;  // multiplying by (1,1) changes nothing
        } else {
            // causal_bp_parall.cu:222-238 / 271-287: marg*mask normalised, else the mask fallback.
            fconst = (m0 == 0.0) ? kInf : -kInf;
            head_state = (m0 == 0.0 && m1 == 1.0) ? HEAD_ONE : (m0 == 1.0 && m1 == 0.0) ? HEAD_ZERO : HEAD_NONE;
        }
    }
    if (d == 1) {
        if (!clamped) fconst = (t == FLBP_AND) ? logit(p) : -logit(p);  // :115-117, :154-156
        return true;
    }
    active = 1;
    return true;
}


int check_graph_shape(const flbp_graph_desc &g, std::string &err) {
    const int64_t V = g.n_vars, F = g.n_factors, E = g.n_slots;
    if (V < 0 || F < 0 || E < 0) {
        err = "negative graph size";
        return FLBP_ERR_INVALID;
    }
    if ((F > 0 || E > 0) && (!g.factor_offsets || !g.slot_var || !g.factor_head || !g.factor_type ||
                             !g.factor_p || !g.factor_q)) {
        err = "missing graph array";
        return FLBP_ERR_INVALID;
    }
    if (V >= (int64_t)UINT32_MAX || E >= (int64_t)UINT32_MAX) {
        err = "graph exceeds 2^32-1 variables or edge slots";
        return FLBP_ERR_LIMIT;
    }
    const int64_t *off = g.factor_offsets;
    if (F > 0 && (off[0] != 0 || off[F] != E)) {
        err = "factor_offsets must start at 0 and end at n_slots";
        return FLBP_ERR_INVALID;
    }
    if (F == 0 && E != 0) {
        err = "edge slots without factors";
        return FLBP_ERR_INVALID;
    }
    return FLBP_OK;
}

// Tiles of both passes and their headers, and the per-tile constants of the
// large items, from the layout's group bases and large-item runs; big_kind /
// big_pq hold the kind and (p, q) of every large factor (internal order).
// Large items that fit a tile come first (a warp per item, staged like the
// sliced-ELL groups); the sliced-ELL tiles follow. Items too large for a
// tile (the first ones, by decreasing degree) are left to the warp path.
void build_tiles(HostLayout &L, const uint8_t *big_kind, const double *big_pq) {
    L.nf_huge = 0;
    while (L.nf_huge < L.nf_big && L.fb_deg[L.nf_huge] - 1 > kBigFactorBody) L.nf_huge++;
    L.nv_huge = 0;
    while (L.nv_huge < L.nv_big && L.vb_deg[L.nv_huge] > kTileSlotsHost) L.nv_huge++;
    auto push_hdr = [](hvec<uint32_t> &h, uint32_t first, uint32_t nflag, const uint32_t *offs, uint32_t n,
                       uint32_t ordinal) {
        const size_t at = h.size();
        h.push_back(first);
        h.push_back(nflag);
        for (uint32_t j = 0; j + 2 < kHdrWordsHost; j++) h.push_back(offs[std::min(j, n)]);
        if (nflag & kBigTileFlag) h[at + kHdrWordsHost - 1] = ordinal;
    };
    auto big_tiles = [&](const hvec<uint32_t> &boff, const hvec<uint32_t> &bdeg, uint32_t b0, uint32_t nb,
                         hvec<uint32_t> &hdr, std::vector<uint32_t> &firsts) -> uint32_t {
        uint32_t nt = 0, b = b0;
        while (b < nb) {
            const uint32_t start = b;
            do b++;  // every item fits a tile by itself (larger ones are left to the warp path)
            while (b < nb && b - start < kTileGroupsHost && boff[b + 1] - boff[start] <= kTileSlotsHost);
            push_hdr(hdr, start, (b - start) | kBigTileFlag, &boff[start], b - start, nt);
            firsts.push_back(start);
            nt++;
        }
        (void)bdeg;
        return nt;
    };
    auto sell_tiles = [&](const hvec<uint32_t> &base, hvec<uint32_t> &hdr) -> uint32_t {
        const uint32_t ng = base.empty() ? 0 : (uint32_t)base.size() - 1;
        uint32_t g = 0, nt = 0;
        while (g < ng) {
            const uint32_t g0 = g;
            uint32_t slots = 0;
            while (g < ng && g - g0 < kTileGroupsHost && slots + (base[g + 1] - base[g]) <= kTileSlotsHost) {
                slots += base[g + 1] - base[g];
                g++;
            }
            push_hdr(hdr, g0, g - g0, &base[g0], g - g0, 0);
            nt++;
        }
        return nt;
    };
    L.fhdr.clear();
    L.vhdr.clear();
    std::vector<uint32_t> fbt_first, vbt_first;
    L.n_fbtiles = big_tiles(L.fb_off, L.fb_deg, L.nf_huge, L.nf_big, L.fhdr, fbt_first);
    L.n_ftiles = L.n_fbtiles + sell_tiles(L.fg_base, L.fhdr);
    L.n_vbtiles = big_tiles(L.vb_off, L.vb_deg, L.nv_huge, L.nv_big, L.vhdr, vbt_first);
    L.n_vtiles = L.n_vbtiles + sell_tiles(L.vg_base, L.vhdr);
    // per large tile constants: degrees and kinds (factor side), degrees (variable side)
    L.fbt_deg.assign((size_t)kTileGroupsHost * L.n_fbtiles, 0);
    L.fbt_kind.assign((size_t)kTileGroupsHost * L.n_fbtiles, 0);
    L.fbt_pq.assign((size_t)2 * kTileGroupsHost * L.n_fbtiles, 0.0);
    for (uint32_t t = 0; t < L.n_fbtiles; t++) {
        const uint32_t b0 = fbt_first[t], n = L.fhdr[(size_t)kHdrWordsHost * t + 1] & ~kBigTileFlag;
        for (uint32_t j = 0; j < n; j++) {
            const size_t k = (size_t)kTileGroupsHost * t + j, fi = (size_t)L.nf_sell + b0 + j;
            L.fbt_deg[k] = L.fb_deg[b0 + j];
            L.fbt_kind[k] = big_kind[fi - L.nf_sell];
            L.fbt_pq[2 * k] = big_pq[2 * (fi - L.nf_sell)];
            L.fbt_pq[2 * k + 1] = big_pq[2 * (fi - L.nf_sell) + 1];
        }
    }
    L.vbt_deg.assign((size_t)kTileGroupsHost * L.n_vbtiles, 0);
    for (uint32_t t = 0; t < L.n_vbtiles; t++) {
        const uint32_t b0 = vbt_first[t], n = L.vhdr[(size_t)kHdrWordsHost * t + 1] & ~kBigTileFlag;
        for (uint32_t j = 0; j < n; j++) L.vbt_deg[(size_t)kTileGroupsHost * t + j] = L.vb_deg[b0 + j];
    }
}

int build_layout(const flbp_graph_desc &g, HostLayout &L, std::string &err, const GraphIds *graphs) {
    const int64_t V = g.n_vars, F = g.n_factors, E = g.n_slots;
    if (int rc = check_graph_shape(g, err)) return rc;
    const int64_t *off = g.factor_offsets;
    {  // first offending index, as a sequential scan reports it
        int64_t bad_f = F, bad_e = E;
#pragma omp parallel for reduction(min : bad_f) if (F >= kParMin)
        for (int64_t I = 0; I < F; I++)
            if (off[I + 1] < off[I]) bad_f = std::min(bad_f, I);
        if (bad_f < F) {
            err = "factor_offsets not monotone at factor " + std::to_string(bad_f);
            return FLBP_ERR_INVALID;
        }
#pragma omp parallel for reduction(min : bad_e) if (E >= kParMin)
        for (int64_t e = 0; e < E; e++)
            if (g.slot_var[e] < 0 || g.slot_var[e] >= V) bad_e = std::min(bad_e, e);
        if (bad_e < E) {
            err = "slot_var out of range at slot " + std::to_string(bad_e);
            return FLBP_ERR_INVALID;
        }
    }

    L = HostLayout();
    L.V = V;
    L.F = F;
    L.E = E;

    // --- classify factors -------------------------------------------------
    hvec<uint8_t> active = par_vec<uint8_t>(F, 0);
    hvec<uint8_t> head_state = par_vec<uint8_t>(F, HEAD_FREE);
    hvec<double> fconst = par_vec<double>(F, 0.0);  // constant message of non-active factors / clamped heads
    // classify factor I; false (with the message in *msg when given) for a malformed factor
    auto classify = [&](int64_t I, std::string *msg) -> bool {
        uint8_t act = 0, hs = HEAD_FREE;
        double c = 0.0;
        const bool ok = classify_factor(g, I, act, hs, c, msg);
        active[I] = act;
        head_state[I] = hs;
        fconst[I] = c;
        return ok;
    };
    {
        int64_t bad = F;
#pragma omp parallel for reduction(min : bad) if (F >= kParMin)
        for (int64_t I = 0; I < F; I++)
            if (!classify(I, nullptr)) bad = std::min(bad, I);
        if (bad < F) {
            classify(bad, &err);
            return FLBP_ERR_INVALID;
        }
    }

    // --- internal factor order: sliced-ELL factors by (graph, degree), then big ones ---
    // Batched engines (graph ids given) keep each graph's items together so
    // that the tiles of a graph that has stopped can be skipped; a single
    // graph is graph 0 throughout.
    const uint32_t G = graphs ? graphs->n_graphs : 1;
    auto fgraph = [&](int64_t I) -> uint32_t { return graphs ? graphs->factor_graph[I] : 0u; };
    auto vgraph = [&](int64_t i) -> uint32_t { return graphs ? graphs->var_graph[i] : 0u; };
    hvec<int64_t> fact_of_int;
    uint32_t nf_sell = 0, nf_big = 0;
    {
        // classes (graph, degree) of the sliced-ELL factors, then one class of the large ones
        constexpr uint32_t D = kSellFactorDegree + 1;
        const size_t nk = (size_t)G * D + 1;
        auto key = [&](int64_t I) -> size_t {
            if (!active[I]) return nk;
            const uint64_t d = (uint64_t)(off[I + 1] - off[I]);
            return d <= kSellFactorDegree ? (size_t)fgraph(I) * D + d : nk - 1;
        };
        const Chunks c = chunks(F, nk);
        const std::vector<uint64_t> cnt = class_counts(c, nk, key);
        const std::vector<uint64_t> start = class_starts(c, nk, cnt, 0);
        nf_sell = (uint32_t)start[nk - 1];
        nf_big = (uint32_t)(start[nk] - start[nk - 1]);
        fact_of_int.resize((size_t)nf_sell + nf_big);  // every position is placed below
        class_place(c, nk, cnt, start, key, [&](int64_t I, uint64_t at) { fact_of_int[at] = I; });
        // large factors: those too large for a tile first, then by (graph, decreasing
        // degree); warps deal them round-robin, largest first
        auto deg = [&](int64_t I) { return off[I + 1] - off[I]; };
        std::stable_sort(fact_of_int.begin() + nf_sell, fact_of_int.end(), [&](int64_t x, int64_t y) {
            const bool hx = deg(x) - 1 > (int64_t)kBigFactorBody, hy = deg(y) - 1 > (int64_t)kBigFactorBody;
            if (hx != hy) return hx;
            if (!hx && fgraph(x) != fgraph(y)) return fgraph(x) < fgraph(y);
            return deg(x) > deg(y);
        });
    }
    const uint32_t nf = nf_sell + nf_big;
    par_copy(L.factor_of_internal, fact_of_int.data(), fact_of_int.size());
    L.nf_sell = nf_sell;
    L.nf_big = nf_big;
    par_assign(L.f_kind, nf, 0);
    par_assign(L.f_deg, nf_sell, 0);
    par_assign(L.f_pq, 2 * (size_t)nf, 0.0);
#pragma omp parallel for if (nf >= kParMin)
    for (uint32_t f = 0; f < nf; f++) {
        const int64_t I = fact_of_int[f];
        L.f_kind[f] = (uint8_t)((g.factor_type[I] == FLBP_OR ? KIND_OR : 0) | head_state[I]);
        L.f_pq[2 * f] = g.factor_p[I];
        L.f_pq[2 * f + 1] = g.factor_q[I];
        if (f < nf_sell) L.f_deg[f] = (uint8_t)(off[I + 1] - off[I]);
    }

    // --- device slots --------------------------------------------------------------
    hvec<uint32_t> dev_slot = par_vec<uint32_t>(E, UINT32_MAX);  // reference slot -> device slot
    {
        // group widths and bases, then the big runs (sizes first, 64-bit), then the slots
        const uint32_t ng = (nf_sell + 31) / 32;
        std::vector<uint64_t> gbase((size_t)ng + 1, 0);
#pragma omp parallel for if (ng >= kParMin / 32)
        for (uint32_t gi = 0; gi < ng; gi++) {
            uint32_t w = 0;
            for (uint32_t f = gi * 32; f < std::min(nf_sell, gi * 32 + 32); f++) w = std::max<uint32_t>(w, L.f_deg[f]);
            gbase[gi + 1] = 32ull * w;
        }
        for (uint32_t gi = 0; gi < ng; gi++) gbase[gi + 1] += gbase[gi];
        std::vector<uint64_t> boff((size_t)nf_big + 1, gbase[ng]);
        for (uint32_t b = 0; b < nf_big; b++) {
            const int64_t I = fact_of_int[nf_sell + b];
            boff[b + 1] = (boff[b] + (uint64_t)(off[I + 1] - off[I]) + kRunAlign - 1) & ~(uint64_t)(kRunAlign - 1);
        }
        const uint64_t next = boff[nf_big];
        if (next >= UINT32_MAX) {
            err = "graph exceeds 2^32-1 device slots";
            return FLBP_ERR_LIMIT;
        }
        par_copy(L.fg_base, gbase.data(), gbase.size());
        par_copy(L.fb_off, boff.data(), boff.size());
        L.fb_deg.assign(nf_big, 0);
#pragma omp parallel for if (nf_sell >= kParMin)
        for (uint32_t f = 0; f < nf_sell; f++) {
            const int64_t I = fact_of_int[f];
            const uint64_t base = gbase[f / 32] + (f % 32);
            uint64_t k = 0;
            dev_slot[g.factor_head[I]] = (uint32_t)base;
            for (int64_t e = off[I]; e < off[I + 1]; e++)
                if (e != g.factor_head[I]) dev_slot[e] = (uint32_t)(base + 32ull * (++k));
        }
#pragma omp parallel for if (nf_big >= kParMin / 64)
        for (uint32_t b = 0; b < nf_big; b++) {
            const int64_t I = fact_of_int[nf_sell + b];
            uint64_t at = boff[b];
            L.fb_deg[b] = (uint32_t)(off[I + 1] - off[I]);
            dev_slot[g.factor_head[I]] = (uint32_t)at++;
            for (int64_t e = off[I]; e < off[I + 1]; e++)
                if (e != g.factor_head[I]) dev_slot[e] = (uint32_t)at++;
        }
        L.n_slots = next;
    }

    // --- variable entries ----------------------------------------------------------
    // A reference slot reaches its variable through the engine when it is an
    // active body slot or the head slot of an active factor with a free head.
    hvec<uint8_t> entry = par_vec<uint8_t>(E, 0);
    hvec<uint32_t> vdeg = par_vec<uint32_t>(V, 0);
    hvec<uint32_t> var_of_dev = par_vec<uint32_t>(L.n_slots, UINT32_MAX);  // device slot -> variable of its entry
    uint64_t n_act = 0;
#pragma omp parallel for reduction(+ : n_act) if (F >= kParMin)
    for (int64_t I = 0; I < F; I++) {
        if (!active[I]) continue;
        n_act += (uint64_t)(off[I + 1] - off[I]);
        for (int64_t e = off[I]; e < off[I + 1]; e++) {
            if (e == g.factor_head[I] && head_state[I] != HEAD_FREE) continue;
            entry[e] = 1;
            const uint32_t v = (uint32_t)g.slot_var[e];
            __atomic_fetch_add(&vdeg[v], 1u, __ATOMIC_RELAXED);
            var_of_dev[dev_slot[e]] = v;
        }
    }
    L.n_active_slots = n_act;

    // Internal variable order: sliced-ELL variables by (graph, degree) and,
    // within that, by their first device slot (so that variables reached from
    // neighbouring factors sit together), then the large ones: those too large
    // for a tile first, the rest by (graph, decreasing degree). One scan over
    // the device slots in increasing order finds every variable's first slot.
    uint32_t nv_sell = 0;
    hvec<uint32_t> order(V);  // every position is placed below
    {
        // classes (graph, degree) of the sliced-ELL variables, then one class of the large ones
        constexpr uint32_t D = kSellVarDegree + 1;
        const size_t nk = (size_t)G * D + 1;
        auto vkey = [&](int64_t i) -> size_t {
            return vdeg[i] <= kSellVarDegree ? (size_t)vgraph(i) * D + vdeg[i] : nk - 1;
        };
        const Chunks cv = chunks(V, nk);
        const std::vector<uint64_t> start = class_starts(cv, nk, class_counts(cv, nk, vkey), 0);
        nv_sell = (uint32_t)start[nk - 1];
        // variables without entries and the large ones in index order
        auto key0 = [&](int64_t i) -> size_t {
            const size_t k = vkey(i);
            return (vdeg[i] == 0 || k == nk - 1) ? k : nk;
        };
        class_place(cv, nk, class_counts(cv, nk, key0), start, key0,
                    [&](int64_t i, uint64_t at) { order[at] = (uint32_t)i; });
        // the others in the order of their first device slot
        hvec<uint32_t> first = par_vec<uint32_t>(V, UINT32_MAX);
#pragma omp parallel for if (L.n_slots >= (uint64_t)kParMin)
        for (int64_t sl = 0; sl < (int64_t)L.n_slots; sl++) {
            const uint32_t v = var_of_dev[sl];
            if (v != UINT32_MAX) atomic_min_u32(&first[v], (uint32_t)sl);
        }
        auto skey = [&](int64_t sl) -> size_t {
            const uint32_t v = var_of_dev[sl];
            if (v == UINT32_MAX || first[v] != (uint32_t)sl || vdeg[v] > kSellVarDegree) return nk;
            return (size_t)vgraph(v) * D + vdeg[v];
        };
        const Chunks cs = chunks((int64_t)L.n_slots, nk);
        class_place(cs, nk, class_counts(cs, nk, skey), start, skey,
                    [&](int64_t sl, uint64_t at) { order[at] = var_of_dev[sl]; });
        std::stable_sort(order.begin() + nv_sell, order.end(), [&](uint32_t x, uint32_t y) {
            const bool hx = vdeg[x] > kTileSlotsHost, hy = vdeg[y] > kTileSlotsHost;
            if (hx != hy) return hx;
            if (!hx && vgraph(x) != vgraph(y)) return vgraph(x) < vgraph(y);
            return vdeg[x] > vdeg[y];
        });
    }
    L.nv_sell = nv_sell;
    L.nv_big = (uint32_t)V - nv_sell;
    par_copy(L.var_of_internal, order.data(), order.size());
    L.internal_of_var.resize(V);  // a permutation: every position is written below
#pragma omp parallel for if (V >= kParMin)
    for (int64_t iv = 0; iv < V; iv++) L.internal_of_var[order[iv]] = (uint32_t)iv;

    // Entry positions: group base + 32 k + lane for sliced-ELL variables, a
    // contiguous run for large ones; entry k of a variable is its k-th device
    // slot in increasing order.
    {
        const uint32_t ng = (nv_sell + 31) / 32;
        std::vector<uint64_t> gbase((size_t)ng + 1, 0);
#pragma omp parallel for if (ng >= kParMin / 32)
        for (uint32_t gi = 0; gi < ng; gi++) {
            uint32_t w = 0;
            for (uint32_t iv = gi * 32; iv < std::min(nv_sell, gi * 32 + 32); iv++) w = std::max(w, vdeg[order[iv]]);
            gbase[gi + 1] = 32ull * w;
        }
        for (uint32_t gi = 0; gi < ng; gi++) gbase[gi + 1] += gbase[gi];
        const uint64_t nent = gbase[ng];
        L.vg_base.assign(ng + 1, 0);
        uint64_t nbig = 0;
        for (uint32_t iv = nv_sell; iv < (uint32_t)V; iv++) nbig += (vdeg[order[iv]] + kRunAlign - 1) & ~(kRunAlign - 1);
        if (nent + nbig >= UINT32_MAX) {
            err = "graph exceeds 2^32-1 variable entries";
            return FLBP_ERR_LIMIT;
        }
        std::copy(gbase.begin(), gbase.end(), L.vg_base.begin());
        L.vb_off.assign((size_t)L.nv_big + 1, 0);
        L.vb_deg.assign(L.nv_big, 0);
        uint64_t pos = nent;
        for (uint32_t b = 0; b < L.nv_big; b++) {
            L.vb_off[b] = (uint32_t)pos;
            L.vb_deg[b] = vdeg[order[nv_sell + b]];
            pos = (pos + L.vb_deg[b] + kRunAlign - 1) & ~(uint64_t)(kRunAlign - 1);  // 16-byte aligned runs
        }
        L.vb_off[L.nv_big] = (uint32_t)pos;
        // first entry position and stride of every variable
        hvec<uint32_t> epos(V), estride(V);  // written for every variable below
#pragma omp parallel for if (V >= kParMin)
        for (int64_t iv = 0; iv < V; iv++) {
            const uint32_t v = order[iv];
            if (iv < nv_sell) {
                epos[v] = L.vg_base[iv / 32] + (iv % 32);
                estride[v] = 32;
            } else {
                epos[v] = L.vb_off[iv - nv_sell];
                estride[v] = 1;
            }
        }
        par_assign(L.v_ent, pos, kSentinel);
        par_assign(L.f_pos, L.n_slots, kSentinel);  // slot -> entry receiving its f->v message
        // The (variable, device slot) pairs in the reference's factor-major
        // slot order, stably radix-sorted by variable (11-bit digits): each
        // variable's slots end up together, and entry k of a variable is its
        // k-th slot in the reference's order. That order belongs to the graph,
        // not to the layout, so a variable sums its messages in the same order
        // whether its graph is solved alone or in a batch.
        hvec<uint32_t> kv, ks, kv2, ks2;  // variable, slot
        {
            constexpr int kBits = 11;
            constexpr size_t nk = size_t(1) << kBits;
            int passes = 1;
            while (passes * kBits < 32 && ((uint64_t)V - 1) >> (passes * kBits)) passes++;
            uint64_t n_ent = 0;
            for (int64_t i = 0; i < V; i++) n_ent += vdeg[i];
            kv.resize(n_ent);
            ks.resize(n_ent);
            kv2.resize(n_ent);
            ks2.resize(n_ent);
            for (int ps = 0; ps < passes; ps++) {
                const int sh = ps * kBits;
                if (ps == 0) {  // straight from the reference slots that are entries
                    const Chunks c = chunks(E, nk);
                    auto key = [&](int64_t e) -> size_t {
                        return entry[e] ? ((uint32_t)g.slot_var[e] & (nk - 1)) : nk;
                    };
                    const std::vector<uint64_t> cnt = class_counts(c, nk, key);
                    class_place(c, nk, cnt, class_starts(c, nk, cnt, 0), key, [&](int64_t e, uint64_t at) {
                        kv2[at] = (uint32_t)g.slot_var[e];
                        ks2[at] = dev_slot[e];
                    });
                } else {
                    const Chunks c = chunks((int64_t)n_ent, nk);
                    auto key = [&](int64_t i) -> size_t { return (kv[i] >> sh) & (nk - 1); };
                    const std::vector<uint64_t> cnt = class_counts(c, nk, key);
                    class_place(c, nk, cnt, class_starts(c, nk, cnt, 0), key, [&](int64_t i, uint64_t at) {
                        kv2[at] = kv[i];
                        ks2[at] = ks[i];
                    });
                }
                kv.swap(kv2);
                ks.swap(ks2);
            }
            hvec<uint32_t>().swap(kv2);
            hvec<uint32_t>().swap(ks2);
        }
        // run starts: the first pair of every variable
        hvec<uint64_t> vstart((size_t)V);
#pragma omp parallel for if ((int64_t)kv.size() >= kParMin)
        for (int64_t i = 0; i < (int64_t)kv.size(); i++)
            if (i == 0 || kv[i - 1] != kv[i]) vstart[kv[i]] = (uint64_t)i;
#pragma omp parallel for if ((int64_t)kv.size() >= kParMin)
        for (int64_t i = 0; i < (int64_t)kv.size(); i++) {
            const uint32_t v = kv[i], k = (uint32_t)(i - vstart[v]), sl = ks[i];
            const uint32_t ep = epos[v] + k * estride[v];
            L.v_ent[ep] = sl;
            L.f_pos[sl] = ep;
        }
    }

    // --- tiles and their headers, per large tile constants ---------------------------
    std::vector<uint8_t> big_kind(L.f_kind.begin() + nf_sell, L.f_kind.end());
    std::vector<double> big_pq(L.f_pq.begin() + 2 * (size_t)nf_sell, L.f_pq.end());
    build_tiles(L, big_kind.data(), big_pq.data());
    // batched engines: the range of graphs of every tile's items
    if (graphs) {
        auto stamp = [&](hvec<uint32_t> &hdr, uint32_t nt, uint32_t n_sell_items, auto item_graph) {
            for (uint32_t t = 0; t < nt; t++) {
                uint32_t *h = &hdr[(size_t)kHdrWordsHost * t];
                const bool big = h[1] & kBigTileFlag;
                const uint32_t n = h[1] & ~kBigTileFlag;
                uint32_t lo = UINT32_MAX, hi = 0;
                auto see = [&](uint32_t item) {
                    const uint32_t gr = item_graph(item);
                    lo = std::min(lo, gr);
                    hi = std::max(hi, gr);
                };
                if (big) {
                    for (uint32_t j = 0; j < n; j++) see(n_sell_items + h[0] + j);
                } else {
                    for (uint32_t i = 32 * h[0]; i < std::min(n_sell_items, 32 * (h[0] + n)); i++) see(i);
                }
                h[kHdrGraphLo] = lo;
                h[kHdrGraphHi] = hi;
            }
        };
        stamp(L.fhdr, L.n_ftiles, nf_sell, [&](uint32_t f) { return fgraph(fact_of_int[f]); });
        stamp(L.vhdr, L.n_vtiles, nv_sell, [&](uint32_t iv) { return vgraph(order[iv]); });
    }

    // --- priors ------------------------------------------------------------------
    par_assign(L.prior_fin, V, 0.0);
    par_assign(L.prior_cnt, V, 0);
    {
        hvec<double> fin = par_vec<double>(V, 0.0);
        hvec<uint32_t> head_iv(F);  // internal variable of every folded factor's head (all written below)
#pragma omp parallel for if (F >= kParMin)
        for (int64_t I = 0; I < F; I++)
            head_iv[I] = (active[I] && head_state[I] == HEAD_FREE) ? UINT32_MAX
                                                                   : L.internal_of_var[g.slot_var[g.factor_head[I]]];
        for (int64_t I = 0; I < F; I++) {  // in factor order: the sums and lists are order-dependent
            if (head_iv[I] == UINT32_MAX) continue;
            const uint32_t iv = head_iv[I];
            const double c = fconst[I];
            if (c == kInf) {
                if ((L.prior_cnt[iv] & 0xffffu) != 0xffffu) L.prior_cnt[iv] += 1u;
            } else if (c == -kInf) {
                if (((L.prior_cnt[iv] >> 16) & 0x7fffu) != 0x7fffu) L.prior_cnt[iv] += 1u << 16;
            } else {
                fin[iv] += c;
                // finite constant: +-logit(p) of a singleton or of an AND/OR factor reduced to its head
                L.prior_factor.push_back((uint32_t)I);
                L.prior_var.push_back(iv);
                L.prior_sign.push_back(g.factor_type[I] == FLBP_OR ? -1 : 1);
            }
        }
        L.prior_fin.swap(fin);
    }

    // --- reference-order data for message export (maps built on first use) ----------
    par_copy(L.ref_off, off, (size_t)F + 1);
    L.ref_slot_var.resize(E);  // both written for every slot below
    L.ref_ent.resize(E);
#pragma omp parallel for if (E >= kParMin)
    for (int64_t e = 0; e < E; e++) {
        L.ref_slot_var[e] = (uint32_t)g.slot_var[e];
        L.ref_ent[e] = entry[e] ? L.f_pos[dev_slot[e]] : kSentinel;
    }
    L.ref_fconst = std::move(fconst);
    return FLBP_OK;
}

void build_export_maps(HostLayout &L) {
    if (L.export_ready) return;
    const int64_t V = L.V, F = L.F, E = L.E;
    L.row_ptr_fv.assign((size_t)V + 1, 0);
    for (int64_t e = 0; e < E; e++) L.row_ptr_fv[L.ref_slot_var[e] + 1]++;
    for (int64_t i = 0; i < V; i++) L.row_ptr_fv[i + 1] += L.row_ptr_fv[i];
    L.ref_fv_src.assign(E, 0);
    L.ref_const.assign(E, 0.0);
    L.fm_to_vm.assign(E, 0);
    L.vm_var.assign(E, 0);
    hvec<int64_t> cur(L.row_ptr_fv.begin(), L.row_ptr_fv.end() - 1);
    for (int64_t I = 0; I < F; I++) {
        for (int64_t e = L.ref_off[I]; e < L.ref_off[I + 1]; e++) {
            const int64_t pos = cur[L.ref_slot_var[e]]++;
            L.fm_to_vm[e] = pos;
            L.vm_var[pos] = L.ref_slot_var[e];
            if (L.ref_ent[e] != kSentinel) {
                L.ref_fv_src[pos] = L.ref_ent[e];
            } else {
                const double c = L.ref_fconst[I];
                L.ref_fv_src[pos] = (c == kInf) ? -2 : (c == -kInf) ? -3 : -1;
                L.ref_const[pos] = c;
            }
        }
    }
    L.export_ready = true;
}

}  // namespace flbp

// Digest of the host layout of a graph (no GPU needed): an FNV-1a hash over
// every layout array and count, built with `threads` host threads (0: all).
extern "C" int flbp_layout_digest(const flbp_graph_desc *graph, const uint32_t *factor_graph,
                                  const uint32_t *var_graph, uint32_t n_graphs, int32_t threads, uint64_t *digest) {
    using namespace flbp;
    if (!graph || !digest || (n_graphs && (!factor_graph || !var_graph))) {
        set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    const int saved = omp_get_max_threads();
    if (threads > 0) omp_set_num_threads(threads);
    HostLayout L;
    std::string err;
    const GraphIds ids{n_graphs, factor_graph, var_graph};
    const int rc = build_layout(*graph, L, err, n_graphs ? &ids : nullptr);
    omp_set_num_threads(saved);
    if (rc) {
        set_error(err);
        return rc;
    }
    uint64_t h = 1469598103934665603ull;
    auto bytes = [&](const void *p, size_t n) {
        const unsigned char *c = static_cast<const unsigned char *>(p);
        for (size_t i = 0; i < n; i++) h = (h ^ c[i]) * 1099511628211ull;
    };
    auto arr = [&](const auto &v) {
        const uint64_t n = v.size();
        bytes(&n, sizeof n);
        if (n) bytes(v.data(), n * sizeof(v[0]));
    };
    arr(L.fg_base), arr(L.fb_off), arr(L.fb_deg), arr(L.f_kind), arr(L.f_deg), arr(L.f_pq), arr(L.vg_base);
    arr(L.vb_off), arr(L.vb_deg), arr(L.v_ent), arr(L.f_pos), arr(L.prior_fin), arr(L.prior_cnt);
    arr(L.prior_factor), arr(L.prior_var), arr(L.prior_sign), arr(L.var_of_internal), arr(L.factor_of_internal);
    arr(L.internal_of_var), arr(L.ref_off), arr(L.ref_slot_var), arr(L.ref_ent), arr(L.ref_fconst), arr(L.fhdr);
    arr(L.vhdr), arr(L.fbt_deg), arr(L.fbt_kind), arr(L.fbt_pq), arr(L.vbt_deg);
    const uint64_t sc[] = {L.nf_sell, L.nf_big, L.nf_huge, L.nv_sell, L.nv_big, L.nv_huge, L.n_slots,
                           L.n_active_slots, L.n_ftiles, L.n_vtiles, L.n_fbtiles, L.n_vbtiles};
    bytes(sc, sizeof sc);
    *digest = h;
    return FLBP_OK;
}

