// Sequential update schedules of CausalBP (updates=SEQFIX / TOPO) on the
// host: the update sequences (csrc/ext/causal_bp.cu:186-201, 203-304), their
// conflict-free batches (:583-722) and the per-batch device layout.
//
// A sequence lists every edge once as a factor-major slot (the position of
// the edge in row_ptr_vf / col_ind_vf). The reference cuts it into batches
// scanning edges in order: edge (i, I) opens a new batch when one of the
// factor's other variables j still needs its v->f message to I computed in
// the batch while j already receives an f->v message from another factor in
// the batch, or when i already receives one. Its sets become per-variable and
// per-factor stamps here: a variable receives at most one batch f->v message,
// and after the first edge of a factor in a batch every v->f message of the
// factor but the one from that edge's variable is in the batch, so the scan
// is O(slots) plus O(degree) per (factor, batch) pair. TOPO's extra test
// (the conflicting edge must precede the current one in the sequence) always
// holds, since the batch only holds earlier edges of the sequence.

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <utility>
#include <vector>

#include "../../include/fastlbp_b200.h"
#include "engine_internal.h"

namespace flbp {

namespace {

constexpr uint32_t kNone = 0xffffffffu;

// Offsets monotone, variables in range, distinct variables within a factor.
int check_graph(const flbp_graph_desc &g, std::string &err) {
    if (g.n_vars < 0 || g.n_factors < 0 || g.n_slots < 0 || g.n_vars >= (int64_t)kNone ||
        g.n_factors >= (int64_t)kNone || g.n_slots >= (int64_t)kNone) {
        err = "graph sizes out of range";
        return FLBP_ERR_INVALID;
    }
    if ((g.n_factors > 0 && (!g.factor_offsets || !g.factor_head)) || (g.n_slots > 0 && !g.slot_var)) {
        err = "missing graph arrays";
        return FLBP_ERR_INVALID;
    }
    const int64_t *off = g.factor_offsets;
    if (g.n_factors > 0 && (off[0] != 0 || off[g.n_factors] != g.n_slots)) {
        err = "factor_offsets must run from 0 to n_slots";
        return FLBP_ERR_INVALID;
    }
    std::vector<uint32_t> stamp((size_t)g.n_vars, kNone);
    for (int64_t I = 0; I < g.n_factors; I++) {
        if (off[I + 1] < off[I]) {
            err = "factor_offsets not monotone at factor " + std::to_string(I);
            return FLBP_ERR_INVALID;
        }
        if (g.factor_head[I] < off[I] || g.factor_head[I] >= off[I + 1]) {
            err = "factor_head outside the factor's slots at factor " + std::to_string(I);
            return FLBP_ERR_INVALID;
        }
        for (int64_t s = off[I]; s < off[I + 1]; s++) {
            const int64_t v = g.slot_var[s];
            if (v < 0 || v >= g.n_vars) {
                err = "slot_var out of range at slot " + std::to_string(s);
                return FLBP_ERR_INVALID;
            }
            if (stamp[v] == (uint32_t)I) {
                err = "variable listed twice in factor " + std::to_string(I);
                return FLBP_ERR_INVALID;
            }
            stamp[v] = (uint32_t)I;
        }
    }
    return FLBP_OK;
}

}  // namespace

int seq_batches(const flbp_graph_desc &g, const int64_t *seq, int64_t n, std::vector<uint32_t> &slot_batch,
                uint32_t &n_batches, std::string &err) {
    int rc = check_graph(g, err);
    if (rc) return rc;
    const int64_t V = g.n_vars, F = g.n_factors, E = g.n_slots;
    if (n != E || (E > 0 && !seq)) {
        err = "the update sequence must list every slot once";
        return FLBP_ERR_INVALID;
    }
    std::vector<uint32_t> fos((size_t)E);
    for (int64_t I = 0; I < F; I++)
        for (int64_t s = g.factor_offsets[I]; s < g.factor_offsets[I + 1]; s++) fos[s] = (uint32_t)I;
    slot_batch.assign((size_t)E, kNone);
    std::vector<uint32_t> vstamp((size_t)V, kNone), vfac((size_t)V, 0);  // batch f->v message into a variable: from vfac
    std::vector<uint32_t> fstamp((size_t)F, kNone), fmiss((size_t)F, kNone);  // factor's slot still without its v->f
    uint32_t cur = 0;
    for (int64_t k = 0; k < n; k++) {
        const int64_t s = seq[k];
        if (s < 0 || s >= E || slot_batch[s] != kNone) {
            err = "the update sequence must list every slot once (position " + std::to_string(k) + ")";
            return FLBP_ERR_INVALID;
        }
        const uint32_t I = fos[s];
        const int64_t i = g.slot_var[s];
        // does variable j still need its v->f message to I while it already receives
        // a batch f->v message from another factor?
        auto blocks = [&](int64_t r) {
            const int64_t j = g.slot_var[r];
            return j != i && vstamp[j] == cur && vfac[j] != I;
        };
        bool conflict = false;
        if (fstamp[I] != cur) {
            for (int64_t r = g.factor_offsets[I]; r < g.factor_offsets[I + 1] && !conflict; r++) conflict = blocks(r);
        } else if (fmiss[I] != kNone) {
            conflict = blocks(fmiss[I]);
        }
        if (!conflict && vstamp[i] == cur) conflict = true;
        if (conflict) cur++;
        vstamp[i] = cur;
        vfac[i] = I;
        slot_batch[s] = cur;
        if (fstamp[I] != cur) {  // every v->f message of I but i's is now in the batch
            fstamp[I] = cur;
            fmiss[I] = (uint32_t)s;
        } else {
            fmiss[I] = kNone;  // and i's, from the factor's earlier edge in the batch
        }
    }
    n_batches = E > 0 ? cur + 1 : 0;
    return FLBP_OK;
}

int topo_seq(const flbp_graph_desc &g, std::vector<int64_t> &seq, std::string &err) {
    int rc = check_graph(g, err);
    if (rc) return rc;
    const int64_t V = g.n_vars, F = g.n_factors, E = g.n_slots;
    const int64_t N = V + F;
    // variable -> its factors (ascending), factor -> its variables (ascending)
    std::vector<int64_t> voff((size_t)V + 1, 0), vadj((size_t)E);
    for (int64_t s = 0; s < E; s++) voff[g.slot_var[s] + 1]++;
    for (int64_t v = 0; v < V; v++) voff[v + 1] += voff[v];
    {
        std::vector<int64_t> at(voff.begin(), voff.end() - 1);
        for (int64_t I = 0; I < F; I++)
            for (int64_t s = g.factor_offsets[I]; s < g.factor_offsets[I + 1]; s++) vadj[at[g.slot_var[s]]++] = I;
    }
    std::vector<int64_t> fadj(g.slot_var, g.slot_var + E);
    for (int64_t I = 0; I < F; I++) std::sort(fadj.begin() + g.factor_offsets[I], fadj.begin() + g.factor_offsets[I + 1]);
    // breadth-first order, roots in node order (variables 0..V-1, then factors)
    std::vector<int64_t> order((size_t)N, -1), queue;
    queue.reserve((size_t)N);
    int64_t next = 0;
    for (int64_t r = 0; r < N; r++) {
        if (order[r] >= 0) continue;
        order[r] = next++;
        queue.clear();
        queue.push_back(r);
        for (size_t h = 0; h < queue.size(); h++) {
            const int64_t x = queue[h];
            auto visit = [&](int64_t y) {
                if (order[y] < 0) {
                    order[y] = next++;
                    queue.push_back(y);
                }
            };
            if (x < V) {
                for (int64_t k = voff[x]; k < voff[x + 1]; k++) visit(V + vadj[k]);
            } else {
                const int64_t I = x - V;
                for (int64_t k = g.factor_offsets[I]; k < g.factor_offsets[I + 1]; k++) visit(fadj[k]);
            }
        }
    }
    // edges by (later endpoint, earlier endpoint): both orders name the edge
    std::vector<std::pair<uint64_t, uint64_t>> key((size_t)E);
    std::vector<int64_t> idx((size_t)E);
    for (int64_t I = 0; I < F; I++)
        for (int64_t s = g.factor_offsets[I]; s < g.factor_offsets[I + 1]; s++) {
            const int64_t a = order[V + I], b = order[g.slot_var[s]];
            key[s] = {(uint64_t)std::max(a, b), (uint64_t)std::min(a, b)};
        }
    std::iota(idx.begin(), idx.end(), 0);
    std::sort(idx.begin(), idx.end(), [&](int64_t x, int64_t y) { return key[x] < key[y]; });
    seq.assign(idx.begin(), idx.end());
    return FLBP_OK;
}

int build_seq_layout(const flbp_graph_desc &g, const HostLayout &L, const int64_t *seq, int64_t n, SeqLayout &S,
                     std::string &err) {
    std::vector<uint32_t> slot_batch;
    uint32_t nb = 0;
    int rc = seq_batches(g, seq, n, slot_batch, nb, err);
    if (rc) return rc;
    const int64_t F = g.n_factors, E = g.n_slots;
    S = SeqLayout();
    S.n_batches = nb;
    S.foff.resize((size_t)F + 1);
    S.dslot.resize((size_t)E);
    S.var.resize((size_t)E);
    S.kind.assign((size_t)F, 0);
    S.cst.assign((size_t)F, 0.0);
    S.pq.assign(2 * (size_t)F, 0.0);
    std::vector<uint32_t> internal((size_t)F, kNone);
    for (size_t f = 0; f < L.factor_of_internal.size(); f++) internal[L.factor_of_internal[f]] = (uint32_t)f;
    for (int64_t I = 0; I < F; I++) {
        const int64_t o = g.factor_offsets[I], h = g.factor_head[I];
        S.foff[I] = (uint32_t)o;
        for (int64_t r = o; r < g.factor_offsets[I + 1]; r++) {  // head first, then the body in slot order
            const int64_t d = (r == h) ? o : (r < h ? r + 1 : r);
            S.dslot[r] = (uint32_t)d;
            S.var[d] = L.internal_of_var[g.slot_var[r]];
        }
        S.cst[I] = L.ref_fconst[I];
        S.pq[2 * I] = g.factor_p[I];
        S.pq[2 * I + 1] = g.factor_q[I];
        S.kind[I] = (internal[I] == kNone) ? kSeqConst : L.f_kind[internal[I]];
    }
    S.foff[F] = (uint32_t)E;
    // batches are consecutive runs of the sequence: targets in sequence order,
    // items (factors with a target in the batch) in order of first target
    S.toff.assign((size_t)nb + 1, 0);
    S.ioff.assign((size_t)nb + 1, 0);
    S.tgt.resize((size_t)E);
    S.items.clear();
    std::vector<uint32_t> seen((size_t)F, kNone);
    std::vector<uint32_t> fos((size_t)E);
    for (int64_t I = 0; I < F; I++)
        for (int64_t s = g.factor_offsets[I]; s < g.factor_offsets[I + 1]; s++) fos[s] = (uint32_t)I;
    for (int64_t k = 0; k < n; k++) {
        const int64_t s = seq[k];
        const uint32_t b = slot_batch[s], I = fos[s];
        S.tgt[k] = S.dslot[s];
        S.toff[b + 1] = (uint32_t)(k + 1);
        if (seen[I] != b) {
            seen[I] = b;
            S.items.push_back(I);
        }
        S.ioff[b + 1] = (uint32_t)S.items.size();
    }
    S.irec.resize(4 * S.items.size());
    for (size_t it = 0; it < S.items.size(); it++) {
        const uint32_t I = S.items[it];
        S.irec[4 * it] = S.foff[I];
        S.irec[4 * it + 1] = S.foff[I + 1] - S.foff[I];
        S.irec[4 * it + 2] = S.kind[I];
        S.irec[4 * it + 3] = I;
    }
    S.tvar.resize((size_t)E);
    for (int64_t k = 0; k < E; k++) S.tvar[k] = S.var[S.tgt[k]];
    S.bo.resize(2 * ((size_t)nb + 1));
    for (uint32_t b = 0; b <= nb; b++) {
        S.bo[2 * b] = S.ioff[b];
        S.bo[2 * b + 1] = S.toff[b];
    }
    S.max_items = S.max_tgt = 0;
    for (uint32_t b = 0; b < nb; b++) {
        S.max_items = std::max(S.max_items, S.ioff[b + 1] - S.ioff[b]);
        S.max_tgt = std::max(S.max_tgt, S.toff[b + 1] - S.toff[b]);
    }
    return FLBP_OK;
}

}  // namespace flbp

using namespace flbp;

extern "C" {

int flbp_update_seq(const flbp_graph_desc *g, int32_t kind, const int32_t *factor_order, int64_t *seq_out) {
    if (!g || (!seq_out && g->n_slots > 0)) {
        set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    std::string err;
    if (kind == FLBP_UPDATES_TOPO) {
        std::vector<int64_t> seq;
        int rc = topo_seq(*g, seq, err);
        if (rc) {
            set_error(err);
            return rc;
        }
        if (!seq.empty()) std::memcpy(seq_out, seq.data(), seq.size() * sizeof(int64_t));
        return FLBP_OK;
    }
    if (kind != FLBP_UPDATES_SEQFIX) {
        set_error("kind must be FLBP_UPDATES_SEQFIX or FLBP_UPDATES_TOPO");
        return FLBP_ERR_INVALID;
    }
    int rc = check_graph(*g, err);
    if (rc) {
        set_error(err);
        return rc;
    }
    if (!factor_order && g->n_factors > 0) {
        set_error("SEQFIX needs a factor order");
        return FLBP_ERR_INVALID;
    }
    std::vector<uint8_t> used((size_t)g->n_factors, 0);
    int64_t k = 0;
    for (int64_t x = 0; x < g->n_factors; x++) {
        const int64_t I = factor_order[x];
        if (I < 0 || I >= g->n_factors || used[I]) {
            set_error("factor_order must be a permutation of the factors");
            return FLBP_ERR_INVALID;
        }
        used[I] = 1;
        for (int64_t s = g->factor_offsets[I]; s < g->factor_offsets[I + 1]; s++) seq_out[k++] = s;
    }
    return FLBP_OK;
}

int flbp_shuffled_factors(int64_t n, uint32_t seed, int32_t *order) {
    if (n < 0 || n > INT32_MAX || (n > 0 && !order)) {
        set_error("invalid factor count or null output");
        return FLBP_ERR_INVALID;
    }
    std::vector<int> numbers((size_t)n);
    std::iota(numbers.begin(), numbers.end(), 0);
    std::mt19937 rng(seed);
    std::shuffle(numbers.begin(), numbers.end(), rng);
    for (int64_t i = 0; i < n; i++) order[i] = numbers[i];
    return FLBP_OK;
}

int flbp_seq_batches(const flbp_graph_desc *g, const int64_t *seq, int64_t n, int64_t *slot_batch,
                     int64_t *n_batches) {
    if (!g) {
        set_error("null graph");
        return FLBP_ERR_INVALID;
    }
    std::vector<uint32_t> sb;
    uint32_t nb = 0;
    std::string err;
    int rc = seq_batches(*g, seq, n, sb, nb, err);
    if (rc) {
        set_error(err);
        return rc;
    }
    if (slot_batch)
        for (size_t s = 0; s < sb.size(); s++) slot_batch[s] = sb[s];
    if (n_batches) *n_batches = nb;
    return FLBP_OK;
}

}  // extern "C"
