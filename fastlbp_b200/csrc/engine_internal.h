// Internal declarations shared by the host layout builder (layout.cpp) and
// the CUDA engine (engine.cu). Not part of the public interface.
#pragma once

#include <sys/mman.h>

#include <cstdint>
#include <cstdlib>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "../../include/fastlbp_b200.h"

namespace flbp {

// Allocator of the host layout's arrays: blocks of 2 MiB and more are
// 2 MiB-aligned and hinted for transparent huge pages, and elements are
// default-initialised (resize() writes nothing), so that large arrays are
// first touched by the parallel loops that fill them instead of being
// zeroed page by page by one thread.
template <class T>
struct HostAlloc {
    using value_type = T;
    static constexpr size_t kHuge = size_t(2) << 20;
    HostAlloc() = default;
    template <class U>
    HostAlloc(const HostAlloc<U> &) {}
    T *allocate(size_t n) {
        const size_t bytes = n * sizeof(T);
        if (bytes < kHuge) return static_cast<T *>(::operator new(bytes));
        const size_t al = (bytes + kHuge - 1) & ~(kHuge - 1);
        void *p = std::aligned_alloc(kHuge, al);
        if (!p) throw std::bad_alloc();
        madvise(p, al, MADV_HUGEPAGE);
        return static_cast<T *>(p);
    }
    void deallocate(T *p, size_t n) {
        if (n * sizeof(T) < kHuge) ::operator delete(p);
        else std::free(p);
    }
    template <class U>
    void construct(U *p) noexcept {
        ::new (static_cast<void *>(p)) U;
    }
    template <class U, class... A>
    void construct(U *p, A &&...a) {
        ::new (static_cast<void *>(p)) U(std::forward<A>(a)...);
    }
};
template <class T, class U>
bool operator==(const HostAlloc<T> &, const HostAlloc<U> &) {
    return true;
}
template <class T, class U>
bool operator!=(const HostAlloc<T> &, const HostAlloc<U> &) {
    return false;
}
template <class T>
using hvec = std::vector<T, HostAlloc<T>>;

// Kind byte of an active AND/OR factor.
enum : uint8_t {
    KIND_OR = 1,          // bit 0: OR factor (else AND)
    HEAD_FREE = 0 << 1,   // head message comes from the head variable
    HEAD_ONE = 1 << 1,    // head clamped to 1: effective head log-odds +inf
    HEAD_ZERO = 2 << 1,   // head clamped to 0: effective head log-odds -inf
    HEAD_NONE = 3 << 1,   // head mask (0,0): the reference's arithmetic yields NaN
    HEAD_MASK = 3 << 1,
};

// Items up to these degrees go to the sliced-ELL (one item per lane) paths,
// larger ones to the warp-per-item paths.
constexpr uint32_t kSellFactorDegree = 16;
constexpr uint32_t kSellVarDegree = 16;
constexpr uint32_t kSentinel = 0xffffffffu;  // padding entry in the variable layout
constexpr uint32_t kTileGroupsHost = 16;     // groups (large items) per tile = consumer warps of a block
constexpr uint32_t kTileSlotsHost = 2048;    // slot budget of a tile (shared-memory stage size)
constexpr uint32_t kHdrWordsHost = 32;       // words per tile header
constexpr uint32_t kBigTileFlag = 0x80000000u;  // header word 1: a tile of large items
constexpr uint32_t kBigFactorBody = 256;     // body slots of the largest factor evaluated from a tile
constexpr uint32_t kRunAlign = 4;            // large items' slot / entry runs start on 4-element boundaries
constexpr uint32_t kHdrGraphLo = 29, kHdrGraphHi = 30;  // tile header words: graph range (batched engines)

// Host-built device layout.
//
// Active factors are the AND/OR factors with at least one body variable; all
// other factors (singletons, AND/OR factors reduced to their head, and the
// head output of head-clamped factors) send constant messages and are folded
// into per-variable priors.
//
// Factor side, "sliced ELL" of width 32: active factors with degree <=
// kSellFactorDegree are sorted by degree (stable) and cut into groups of 32;
// group g owns slots [fg_base[g], fg_base[g+1]) laid out column-major, slot k
// of the group's lane-th factor at fg_base[g] + 32*k + lane, k = 0 being the
// head. Larger factors follow as contiguous runs (fb_off), head first.
//
// Variable side: variables are sorted by degree (stable) and cut into groups
// of 32 the same way; entry k of the lane-th variable of group g is
// v_ent[vg_base[g] + 32*k + lane], the factor-side slot whose message
// reaches the variable (kSentinel for padding). Variables of larger degree
// follow with contiguous entry runs (vb_off).
//
// Messages: vf (variable -> factor) is indexed by factor-side slot, fv
// (factor -> variable) by variable entry; f_pos maps each slot to the entry
// that receives its f->v message, v_ent each entry back to its slot, so that
// both passes read contiguously and scatter their outputs.
struct HostLayout {
    int64_t V = 0, F = 0, E = 0;  // reference sizes
    // false: built on the device (dlayout.h); only the counts and the small
    // arrays (group bases, large-item runs, tiles) are filled
    bool complete = true;

    uint32_t nf_sell = 0, nf_big = 0;  // active factors per path
    hvec<uint32_t> fg_base;     // n_fgroups + 1
    hvec<uint32_t> fb_off;      // nf_big + 1 (absolute slot ids; runs padded to kRunAlign)
    hvec<uint32_t> fb_deg;      // per big factor: degree (head included)
    uint32_t nf_huge = 0;              // big factors [0, nf_huge) are too large for a tile
    hvec<uint8_t> f_kind;       // per active factor (internal order)
    hvec<uint8_t> f_deg;        // per sell factor
    hvec<double> f_pq;          // 2 per active factor: p, q
    uint64_t n_slots = 0;              // slots incl. padding

    uint32_t nv_sell = 0, nv_big = 0;
    hvec<uint32_t> vg_base;     // n_vgroups + 1 (entry ids)
    hvec<uint32_t> vb_off;      // nv_big + 1 (entry ids; runs padded to kRunAlign)
    hvec<uint32_t> vb_deg;      // per big variable: number of entries
    uint32_t nv_huge = 0;              // big variables [0, nv_huge) are too large for a tile
    hvec<uint32_t> v_ent;       // entries incl. padding
    hvec<uint32_t> f_pos;       // per slot: entry of its f->v message (kSentinel: none)
    hvec<double> prior_fin;     // per internal variable: finite constant log-odds (damping-scaled)
    hvec<uint32_t> prior_cnt;   // per internal variable: (#+inf) | (#-inf << 16)
    // The finite constant messages folded into prior_fin: reference factor,
    // internal variable and sign (the constant is sign * logit(p)).
    hvec<uint32_t> prior_factor, prior_var;
    hvec<int8_t> prior_sign;
    hvec<uint32_t> var_of_internal;  // internal variable -> reference variable
    hvec<uint32_t> factor_of_internal;  // internal (active) factor -> reference factor
    hvec<uint32_t> internal_of_var;  // reference variable -> internal variable
    uint64_t n_active_slots = 0;       // real (non-padding) slots of active factors

    // Reference order, kept for message export: factor offsets, slot ->
    // variable, slot -> fv entry of its message (kSentinel: constant message),
    // factor -> its constant message.
    hvec<int64_t> ref_off;
    hvec<uint32_t> ref_slot_var;
    hvec<uint32_t> ref_ent;
    hvec<double> ref_fconst;
    // Built by build_export_maps() on first use. Reference variable-major
    // slot (row_ptr_fv order) -> source of its f->v message: >= 0 fv entry;
    // -1 constant finite (value in ref_const, damping-scaled); -2 constant
    // +inf; -3 constant -inf.
    bool export_ready = false;
    hvec<int64_t> ref_fv_src;
    hvec<double> ref_const;
    hvec<int64_t> row_ptr_fv;  // reference variable-major CSR (V+1)
    hvec<int64_t> fm_to_vm;    // reference factor-major slot -> variable-major position
    hvec<int64_t> vm_var;      // variable-major position -> reference variable

    // Tiles: kHdrWordsHost-word headers. Word 0: first group (sliced ELL) or
    // first big item; word 1: item count n, | kBigTileFlag for a tile of big
    // items; words 2..2+n: slot (entry) offsets of the items and the end; the
    // remaining words repeat the end offset, except that word 31 of a big
    // tile holds its ordinal among the big tiles. Big tiles come first.
    hvec<uint32_t> fhdr, vhdr;
    uint32_t n_ftiles = 0, n_vtiles = 0, n_fbtiles = 0, n_vbtiles = 0;
    // per big tile, kTileGroupsHost entries each: degree, kind, (p, q) of its factors;
    // number of entries of its variables
    hvec<uint32_t> fbt_deg;
    hvec<uint8_t> fbt_kind;
    hvec<double> fbt_pq;
    hvec<uint32_t> vbt_deg;

    uint32_t n_fgroups() const { return fg_base.empty() ? 0 : (uint32_t)fg_base.size() - 1; }
    uint32_t n_vgroups() const { return vg_base.empty() ? 0 : (uint32_t)vg_base.size() - 1; }
};

// Graph of every reference factor and variable of a batched engine (the
// disjoint union of n_graphs graphs).
struct GraphIds {
    uint32_t n_graphs;
    const uint32_t *factor_graph;
    const uint32_t *var_graph;
};

// Sequential schedule (updates=SEQFIX / TOPO) of one engine. Every edge is a
// message of its own here, constants included, because the reference folds
// a message into its variable's product only when the edge's turn comes.
// Device slots are the reference's factor-major slots with each factor's
// head moved to the front (the order the factor kernels read).
constexpr uint8_t kSeqConst = 0x80;  // kind flag: the factor sends one constant message
struct SeqLayout {
    uint32_t n_batches = 0;
    uint32_t max_items = 0, max_tgt = 0;  // largest batch
    hvec<uint32_t> foff;   // per reference factor: first device slot (F + 1)
    hvec<uint32_t> dslot;  // reference factor-major slot -> device slot
    hvec<uint32_t> var;    // per device slot: internal variable
    hvec<uint8_t> kind;    // per reference factor: active factors' kind, else kSeqConst
    hvec<double> cst;      // per reference factor: its constant message (a clamped head's output)
    hvec<double> pq;       // per reference factor: p, q
    hvec<uint32_t> ioff, items;  // per batch: its factors
    hvec<uint32_t> toff, tgt;    // per batch: its target device slots
    hvec<uint32_t> irec;         // per item: first device slot, degree, kind, factor (4 words)
    hvec<uint32_t> tvar;         // per target: its internal variable
    hvec<uint32_t> bo;           // per batch and the end: first item, first target (2 words)
};

// Conflict-free batches of an update sequence (every factor-major slot once):
// the batch of every slot and the number of batches.
int seq_batches(const flbp_graph_desc &g, const int64_t *seq, int64_t n, std::vector<uint32_t> &slot_batch,
                uint32_t &n_batches, std::string &err);
// The TOPO update sequence.
int topo_seq(const flbp_graph_desc &g, std::vector<int64_t> &seq, std::string &err);
// The device layout of a sequential schedule over an engine's layout L.
int build_seq_layout(const flbp_graph_desc &g, const HostLayout &L, const int64_t *seq, int64_t n, SeqLayout &S,
                     std::string &err);

// Builds the layout; returns FLBP_OK or an error code with `err` filled in.
// With `graphs`, items are ordered graph by graph and every tile header also
// names the range of graphs its items belong to (words kHdrGraphLo/Hi).
int build_layout(const flbp_graph_desc &g, HostLayout &L, std::string &err, const GraphIds *graphs = nullptr);

// The checks of a graph's sizes and offsets that come before any per-factor
// work (both layout builds).
int check_graph_shape(const flbp_graph_desc &g, std::string &err);

// Fills the variable-major export maps of L (idempotent).
void build_export_maps(HostLayout &L);

// One factor of a graph: whether it is evaluated every sweep (active), the
// state of its head (HEAD_*) and the constant message of a folded factor or
// clamped head. False, with the message in *msg when given, for a malformed
// factor.
bool classify_factor(const flbp_graph_desc &g, int64_t I, uint8_t &active, uint8_t &head_state, double &fconst,
                     std::string *msg);

// Tiles and headers of both passes, and the large items' per-tile
// constants, from L's group bases and large-item runs; big_kind / big_pq:
// kind and (p, q) of every large factor in internal order.
void build_tiles(HostLayout &L, const uint8_t *big_kind, const double *big_pq);

void set_error(const std::string &msg);

}  // namespace flbp
