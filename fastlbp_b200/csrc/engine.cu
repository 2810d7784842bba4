// C-ABI engine: device buffers, sweep launches, the three run loops of
// CausalBP and host exports. Kernels live in kernels.cuh.

#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <numeric>
#include <queue>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstddef>
#include <cstring>
#include <limits>
#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <tuple>
#include <string>
#include <unordered_set>
#include <utility>
#include <vector>

#include "engine_internal.h"
#include "kernels.cuh"
#include "adjoint.cuh"
#include "direct_launch.h"
#include "dlayout.h"
#include "logodds.h"
#include "seq.cuh"

namespace flbp {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

#define FLBP_CUDA(call)                                                                             \
    do {                                                                                            \
        cudaError_t err_ = (call);                                                                  \
        if (err_ != cudaSuccess) {                                                                  \
            set_error(std::string("CUDA error: ") + cudaGetErrorString(err_) + " at " #call);      \
            return err_ == cudaErrorMemoryAllocation ? FLBP_ERR_NOMEM : FLBP_ERR_CUDA;              \
        }                                                                                           \
    } while (0)

}  // namespace flbp

using namespace flbp;

struct flbp_engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int prec = 32;
    double damping = 0.0;
    HostLayout L;
    size_t tsize = 4;

    void *d_vf = nullptr;   // per slot
    void *d_fv = nullptr;   // per variable entry
    void *d_fvd = nullptr;  // per variable entry: damped f->v messages (damping only)
    void *d_f_pq = nullptr;
    uint32_t *d_f_pos = nullptr;  // per slot: entry of its f->v message
    size_t n_ent = 0;
    uint32_t *d_fg_base = nullptr, *d_fb_off = nullptr, *d_vg_base = nullptr, *d_vb_off = nullptr, *d_v_ent = nullptr;
    uint32_t *d_ftiles = nullptr, *d_vtiles = nullptr;  // kHdrWords-word headers per tile
    uint32_t *d_fb_deg = nullptr, *d_vb_deg = nullptr;   // big items' degrees
    uint32_t *d_fbt_deg = nullptr, *d_vbt_deg = nullptr;  // per big tile: degrees of its items
    uint8_t *d_fbt_kind = nullptr;                        // per big tile: kinds of its factors
    void *d_fbt_pq = nullptr;                             // per big tile: (p, q) of its factors
    void *d_vbt_prior = nullptr;                          // per big tile: priors of its variables
    uint32_t f_tile_blocks = 0, v_tile_blocks = 0;
    // Batched solves: the engine holds the disjoint union of n_graphs graphs.
    uint32_t n_graphs = 0;
    std::vector<int64_t> graph_var_off;  // n_graphs + 1: variable ranges in the union's order
    uint32_t *d_f_graph = nullptr, *d_v_graph = nullptr;  // internal factor / variable -> graph
    int *d_gstate = nullptr;  // [4][n_graphs]: stopped, moved, sweeps, stop reason
    uint2 *d_ftrange = nullptr, *d_vtrange = nullptr;  // per tile: range of its items' graphs
    uint32_t *d_act_f = nullptr, *d_act_v = nullptr;   // batched runs: the passes' tiles that hold a live graph
    uint8_t *d_act_flag = nullptr;                      // their flags (factor tiles, then variable tiles)
    void *d_cub_tmp = nullptr;                          // and the compaction's temporary storage
    size_t cub_tmp_bytes = 0;
    // Adjoint: checkpoints of vf every adj_k sweeps of the last adjoint forward
    // run (adj_t sweeps), per-sweep states of one segment, and derivatives.
    long long adj_t = 0, adj_k = 0;
    bool adj_last_seg = false;  // the segment buffers hold the last segment's states (from the forward run)
    void *d_ckpt = nullptr, *d_seg_vf = nullptr, *d_seg_fv = nullptr;
    // in the message type: lambdas per entry (two), mu per slot, dL/dp and
    // dL/dq per internal factor, dL/dprior and dL/dS per internal variable
    void *d_lam = nullptr, *d_lam2 = nullptr, *d_mu = nullptr, *d_gp = nullptr, *d_gq = nullptr;
    void *d_gprior = nullptr, *d_gs = nullptr;
    size_t adj_ckpt_n = 0, adj_seg_n = 0;
    // staged factor pass: each block's tiles (FactorArgs::tile_list / tile_off)
    uint32_t *d_ftlist = nullptr, *d_ftoff = nullptr;
    uint32_t *d_int_of_var = nullptr, *d_f_of_int = nullptr;  // caller variable -> internal; internal factor -> caller
    uint32_t *d_pri_fac = nullptr, *d_pri_var = nullptr;      // folded constants: caller factor, internal variable
    double *d_pri_coef = nullptr;                             // their d(constant)/dp
    bool pri_coef_valid = false;
    // flbp_set_factor_probs_device: the maps it uses (big-tile (p, q) and
    // prior copies' sources, the prior entries grouped by variable), the
    // last p and q it took, and whether the host copies lag behind them
    uint32_t *d_fbt_src = nullptr, *d_vbt_src = nullptr, *d_pri_uvar = nullptr, *d_pri_uoff = nullptr,
             *d_pri_ord = nullptr;
    double *d_pri_sign = nullptr, *d_p_keep = nullptr, *d_q_keep = nullptr;
    unsigned long long *d_bad = nullptr;
    uint32_t n_pri_uvar = 0;
    bool probs_maps = false, host_probs_stale = false;
    double *d_adj_in = nullptr, *d_adj_out = nullptr;         // staging of the host-buffer backward call
    uint32_t *d_adj_groups = nullptr;  // sliced-ELL group ids by width class (see adj_group_n)
    double *d_ref_out = nullptr;       // per-variable results in the caller's order (readback staging)
    uint32_t adj_group_n[4] = {0, 0, 0, 0};
    std::vector<double> factor_p_host;  // every reference factor's p (for derivatives of folded constants)
    std::vector<double> factor_q_host;  // every reference factor's q
    std::vector<int64_t> ref_head;      // every reference factor's head slot
    // Sequential schedule (updates=SEQFIX / TOPO): its layout and device state.
    bool seq = false;
    SeqLayout SQ;
    uint32_t *d_sq_foff = nullptr, *d_sq_var = nullptr, *d_sq_items = nullptr, *d_sq_tgt = nullptr;
    uint32_t *d_sq_iota = nullptr, *d_sq_irec = nullptr, *d_sq_tvar = nullptr, *d_sq_bo = nullptr;
    int seq_kernel = 0;        // 0: choose, 1: two launches per batch, 2: one cluster per sweep, 3: as 1 with
                               // programmatic dependent launch
    bool seq_cluster = false;  // the sweep runs as one cluster kernel
    uint8_t *d_sq_kind = nullptr;
    void *d_sq_cst = nullptr, *d_sq_pq = nullptr, *d_sq_fv = nullptr, *d_sq_vf = nullptr, *d_sq_nw = nullptr;
    double *d_sq_S = nullptr;
    int2 *d_sq_cnt = nullptr;
    std::vector<int8_t> clamp_state;    // per reference variable: -1 free, else the value it is clamped to
    // (slot, value) of every slot of a clamped variable: its v->f message is
    // +-inf from init() on, as if the variable had left the factor
    std::vector<uint32_t> clamp_slots;
    uint32_t *d_clamp_slots = nullptr;
    size_t clamp_slots_cap = 0;
    uint32_t *d_clamp_upd = nullptr;  // a clamp call's update lists (grow-only)
    size_t clamp_upd_cap = 0;
    uint8_t *d_f_kind = nullptr, *d_f_deg = nullptr;
    void *d_prior = nullptr;
    double *d_belief = nullptr, *d_lowpass = nullptr, *d_hist = nullptr;
    double *d_scratch = nullptr;  // beliefs evaluated on demand (leave the run state untouched)
    uint32_t *d_hist_next = nullptr, *d_hist_count = nullptr;
    uint32_t hist_cap = 0;
    Ctl *d_ctl = nullptr;
    Ctl *h_ctl = nullptr;  // pinned mirror

    int factor_grid = 1, var_grid = 1;
    // Form of each pass (flbp_tuning): 0 staged, 1/2 direct; grids of the direct forms.
    int f_form = 0, v_form = 0;
    int f_grid_direct = 1, v_grid_direct = 1;
    int sms = 148;
    std::map<std::pair<int, int>, cudaGraphExec_t> graphs;  // (mode, sweeps) -> executable graph
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.f;

    long long iters = 0;   // the reference's _iters (sweeps since construction)
    long long t = 0;       // sweeps since init()
    long long launches = 0;
    bool lowpass_valid = false;
    size_t bytes = 0;
    size_t h2d_bytes = 0;  // host->device bytes copied by create
    // Evidence sets on one graph (flbp_sets_create): n_sets copies of the
    // messages, priors and beliefs at these strides (elements); (set, entry)
    // pairs that no message reaches, (set, slot, value, -) of the clamped
    // variables' slots; the sweep's grid width.
    uint32_t n_sets = 0;
    uint64_t set_vs = 0, set_es = 0, set_nv = 0;
    uint2 *d_set_cut = nullptr;
    uint32_t n_set_cut = 0;
    uint4 *d_set_slots = nullptr;
    uint32_t n_set_slots = 0;
    unsigned set_fgx = 1, set_vgx = 1;
    // Layout built on the device (dlayout.h): the caller's graph arrays stay
    // on the device until the complete host layout is first needed.
    bool dev_layout = false;
    DevGraphIn din;
    void *d_in[9] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    // wall time (us) of the phases of create: host layout, device allocation,
    // host->device copies (with the host-side packing they need), the rest
    int64_t create_us[4] = {0, 0, 0, 0};

    // Per-kernel timing mode: sweeps are launched without graphs, with events
    // around each pass; collect_kernel_times() folds them into kt_ms / kt_n.
    bool ktime = false;
    std::vector<cudaEvent_t> kev;
    size_t kev_used = 0;
    std::vector<cudaGraphExec_t> kgraphs;  // timing-mode graphs of the current call
    double kt_ms[2] = {0.0, 0.0};
    long long kt_n[2] = {0, 0};
};

namespace {

template <typename T>
FactorArgs factor_args(flbp_engine *e) {
    FactorArgs a;
    a.fg_base = e->d_fg_base;
    a.fb_off = e->d_fb_off;
    a.f_pos = e->d_f_pos;
    a.f_kind = e->d_f_kind;
    a.f_deg = e->d_f_deg;
    a.f_pq = e->d_f_pq;
    a.fb_deg = e->d_fb_deg;
    a.bt_deg = e->d_fbt_deg;
    a.bt_kind = e->d_fbt_kind;
    a.bt_pq = e->d_fbt_pq;
    a.nf_sell = e->L.nf_sell;
    a.nf_big = e->L.nf_big;
    a.nf_huge = e->L.nf_huge;
    a.n_fgroups = e->L.n_fgroups();
    a.thdr = reinterpret_cast<const uint4 *>(e->d_ftiles);
    a.tile_list = e->d_ftlist;
    a.tile_off = e->d_ftoff;
    a.n_tiles = e->L.n_ftiles;
    a.n_tile_blocks = e->f_tile_blocks;
    a.f_graph = nullptr;
    a.gdone = nullptr;
    a.trange = nullptr;
    a.n_graphs = 0;
    return a;
}

VarArgs var_args(flbp_engine *e) {
    VarArgs a;
    a.vg_base = e->d_vg_base;
    a.vb_off = e->d_vb_off;
    a.vb_deg = e->d_vb_deg;
    a.bt_deg = e->d_vbt_deg;
    a.bt_prior = e->d_vbt_prior;
    a.v_ent = e->d_v_ent;
    a.prior = e->d_prior;
    a.belief = e->d_belief;
    a.hist = e->d_hist;
    a.hist_next = e->d_hist_next;
    a.hist_count = e->d_hist_count;
    a.nv_sell = e->L.nv_sell;
    a.nv_big = e->L.nv_big;
    a.nv_huge = e->L.nv_huge;
    a.n_vgroups = e->L.n_vgroups();
    a.thdr = reinterpret_cast<const uint4 *>(e->d_vtiles);
    a.n_tiles = e->L.n_vtiles;
    a.n_tile_blocks = e->v_tile_blocks;
    a.hist_len = e->hist_cap;
    a.v_graph = nullptr;
    a.gstate = nullptr;
    a.trange = nullptr;
    a.n_graphs = 0;
    return a;
}

SeqArgs seq_args(flbp_engine *e) {
    SeqArgs a;
    a.irec = reinterpret_cast<const uint4 *>(e->d_sq_irec);
    a.tvar = e->d_sq_tvar;
    a.bo = reinterpret_cast<const uint2 *>(e->d_sq_bo);
    a.foff = e->d_sq_foff;
    a.var = e->d_sq_var;
    a.kind = e->d_sq_kind;
    a.cst = e->d_sq_cst;
    a.pq = e->d_sq_pq;
    a.items = e->d_sq_items;
    a.tgt = e->d_sq_tgt;
    a.iota = e->d_sq_iota;
    a.fv = e->d_sq_fv;
    a.vf = e->d_sq_vf;
    a.nw = e->d_sq_nw;
    a.S = e->d_sq_S;
    a.cnt = e->d_sq_cnt;
    return a;
}

unsigned int seq_belief_grid(const flbp_engine *e) {
    const uint64_t b = ((uint64_t)e->L.V + 255) / 256;
    return (unsigned int)std::max<uint64_t>(1, std::min<uint64_t>(b, 148ull * 8));
}

// Kernels of one sequential sweep: `which` bit 0 the batches (with the
// sweep's opening kernel), bit 1 the beliefs of the tolerance / low-pass loops.
long long seq_sweep_launches(const flbp_engine *e, int mode, int which) {
    const long long batches = e->seq_cluster ? 1 : 1 + 2LL * e->SQ.n_batches;
    return ((which & 1) ? batches : 0) + (((which & 2) && (mode == 1 || mode == 2)) ? 1 : 0);
}

// One cluster per sweep where batches hold a few factors on average (TOPO's
// hold two or three: a batch then takes 3.3 us on the cluster against 3.9 us
// as two launches on a B200), else two launches per batch over the whole GPU
// (SEQFIX's batches of a few hundred factors: 5.4 against 6.2 us).
bool choose_seq_cluster(const flbp_engine *e) {
    if (e->seq_kernel == 1 || e->seq_kernel == 3) return false;
    if (e->seq_kernel == 2) return true;
    const SeqLayout &Q = e->SQ;
    return Q.n_batches > 0 && Q.items.size() <= (size_t)Q.n_batches * 32;
}

// A kernel launch on the engine's stream, with programmatic dependent launch
// when asked for (the kernels wait for their predecessor in pdl_enter).
template <typename... K, typename... A>
void launch_seq(flbp_engine *e, bool pdl, void (*kern)(K...), unsigned grid, unsigned block, A... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.stream = e->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kern, args...);
}

template <typename T>
void launch_seq_sweep(flbp_engine *e, int mode, int which) {
    const SeqArgs a = seq_args(e);
    const SeqLayout &Q = e->SQ;
    const bool pdl = (e->seq_kernel == 3);
    if ((which & 1) && e->seq_cluster) {
        if (e->damping != 0.0)
            seq_sweep_cluster_kernel<T, true><<<kSeqClusterCtas, 32 * kSeqClusterWarps, 0, e->stream>>>(
                a, Q.n_batches, (T)e->damping, e->d_ctl);
        else
            seq_sweep_cluster_kernel<T, false><<<kSeqClusterCtas, 32 * kSeqClusterWarps, 0, e->stream>>>(
                a, Q.n_batches, (T)0, e->d_ctl);
    } else if (which & 1) {
        launch_seq(e, pdl, seq_begin_kernel, 1, 1, e->d_ctl);
        const T d = (T)e->damping;
        for (uint32_t b = 0; b < Q.n_batches; b++) {
            const uint32_t i0 = Q.ioff[b], i1 = Q.ioff[b + 1], t0 = Q.toff[b], t1 = Q.toff[b + 1];
            launch_seq(e, pdl, seq_factor_kernel<T>, (i1 - i0 + kSeqWarps - 1) / kSeqWarps, 32 * kSeqWarps, a, i0, i1,
                       e->d_ctl);
            if (e->damping != 0.0)
                launch_seq(e, pdl, seq_apply_kernel<T, true>, (t1 - t0 + 255) / 256, 256, a, t0, t1, d, e->d_ctl);
            else
                launch_seq(e, pdl, seq_apply_kernel<T, false>, (t1 - t0 + 255) / 256, 256, a, t0, t1, d, e->d_ctl);
        }
    }
    if ((which & 2) && (mode == 1 || mode == 2)) {
        const VarArgs va = var_args(e);
        const uint32_t V = (uint32_t)e->L.V;
        if (mode == 1)
            launch_seq(e, pdl, seq_belief_kernel<1>, seq_belief_grid(e), 256, va, (const double *)e->d_sq_S,
                       (const int2 *)e->d_sq_cnt, V, e->d_ctl);
        else
            launch_seq(e, pdl, seq_belief_kernel<2>, seq_belief_grid(e), 256, va, (const double *)e->d_sq_S,
                       (const int2 *)e->d_sq_cnt, V, e->d_ctl);
    }
}

constexpr int kStages = 3;  // bulk-copy pipeline depth of the variable pass (and of the FP64 factor pass)
// FP32 factor-pass stages are small enough for a fourth with two blocks per
// SM, and without the batched solves' per-factor graph (GID false: one
// graph) for a fifth
template <typename T, bool GID>
constexpr int kFactorStages = sizeof(T) == 4 ? (GID ? 4 : 5) : 3;
constexpr int kBlockThreads = kBlockThreadsDev;  // 16 consumer warps + 1 producer warp

template <typename T, bool GID>
constexpr size_t factor_smem() {
    return (size_t)kFactorStages<T, GID> * FactorStage<T, GID>::bytes;
}

template <typename T, bool DAMP>
constexpr size_t var_smem() {
    return (size_t)kStages * VarStage<T, DAMP>::bytes;
}
static_assert(factor_smem<double, true>() <= 227 * 1024 && factor_smem<double, false>() <= 227 * 1024,
              "factor-pass stages exceed shared memory");
// two blocks per SM (228 KB) with the static shared memory and 1 KB reserved per block
static_assert(2 * (factor_smem<float, false>() + 6 * 1024) <= 228 * 1024, "single-graph FP32 stages: two blocks per SM");
static_assert(var_smem<double, true>() <= 227 * 1024, "variable-pass stages exceed shared memory");
static_assert(kTileGroupsHost == (uint32_t)kTileGroups && kTileSlotsHost == (uint32_t)kTileSlots,
              "host tiling must match the kernels' stage sizes");

// Opt every kernel instantiation of precision T into its dynamic shared
// memory size; returns the resident blocks per SM of the factor and
// variable passes.
template <typename T>
cudaError_t configure_kernels(bool damp, int *fb, int *vb) {
    cudaError_t err = cudaSuccess;
    auto set = [&](const void *fn, size_t bytes) {
        cudaError_t e2 = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e2 != cudaSuccess) err = e2;
    };
    set((const void *)factor_pass_kernel<T, kFactorStages<T, true>, true>, factor_smem<T, true>());
    set((const void *)factor_pass_kernel<T, kFactorStages<T, false>, false>, factor_smem<T, false>());
    if (err == cudaSuccess)  // the single-graph stages fill two blocks' worth of the SM's shared memory
        err = cudaFuncSetAttribute((const void *)factor_pass_kernel<T, kFactorStages<T, false>, false>,
                                   cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    set((const void *)var_pass_kernel<T, 0, true, false, kStages>, var_smem<T, false>());
    set((const void *)var_pass_kernel<T, 1, true, false, kStages>, var_smem<T, false>());
    set((const void *)var_pass_kernel<T, 2, true, false, kStages>, var_smem<T, false>());
    set((const void *)var_pass_kernel<T, 0, true, true, kStages>, var_smem<T, true>());
    set((const void *)var_pass_kernel<T, 1, true, true, kStages>, var_smem<T, true>());
    set((const void *)var_pass_kernel<T, 2, true, true, kStages>, var_smem<T, true>());
    set((const void *)var_pass_kernel<T, 4, true, false, kStages>, var_smem<T, false>());
    set((const void *)var_pass_kernel<T, 4, true, true, kStages>, var_smem<T, true>());
    set((const void *)var_pass_kernel<T, 3, false, false, kStages>, var_smem<T, false>());
    // one grid for both kernels: the fewer resident blocks of the two
    int fb1 = 0, fb2 = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fb1, factor_pass_kernel<T, kFactorStages<T, true>, true>,
                                                  kBlockThreads, factor_smem<T, true>());
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fb2, factor_pass_kernel<T, kFactorStages<T, false>, false>,
                                                  kBlockThreads, factor_smem<T, false>());
    *fb = std::min(fb1, fb2);
    if (damp)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(vb, var_pass_kernel<T, 2, true, true, kStages>, kBlockThreads,
                                                      var_smem<T, true>());
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(vb, var_pass_kernel<T, 2, true, false, kStages>, kBlockThreads,
                                                      var_smem<T, false>());
    return err;
}

template <typename T, int BMODE, bool DAMP>
void launch_var(flbp_engine *e, const VarArgs &va) {
    if (e->v_form) {
        direct_var_launch<T>(e->v_form, BMODE, DAMP, (unsigned)e->v_grid_direct, va, (const T *)e->d_fv, (T *)e->d_vf,
                             (T *)e->d_fvd, (T)e->damping, e->d_ctl, e->stream);
        return;
    }
    var_pass_kernel<T, BMODE, true, DAMP, kStages><<<e->var_grid, kBlockThreads, var_smem<T, DAMP>(), e->stream>>>(
        va, (const T *)e->d_fv, (T *)e->d_vf, (T *)e->d_fvd, (T)e->damping, e->d_ctl);
}

template <typename T>
void launch_factor(flbp_engine *e, const FactorArgs &fa, const void *vf, void *fv) {
    if (e->f_form) {
        direct_factor_launch<T>(e->f_form, (unsigned)e->f_grid_direct, fa, (const T *)vf, (T *)fv, e->d_ctl,
                                e->stream);
        return;
    }
    if (fa.f_graph)
        factor_pass_kernel<T, kFactorStages<T, true>, true>
            <<<e->factor_grid, kBlockThreads, factor_smem<T, true>(), e->stream>>>(fa, (const T *)vf, (T *)fv, e->d_ctl);
    else
        factor_pass_kernel<T, kFactorStages<T, false>, false>
            <<<e->factor_grid, kBlockThreads, factor_smem<T, false>(), e->stream>>>(fa, (const T *)vf, (T *)fv, e->d_ctl);
}

template <typename T, bool DAMP>
void launch_var_mode(flbp_engine *e, const VarArgs &va, int mode) {
    if (mode == 0) launch_var<T, 0, DAMP>(e, va);
    else if (mode == 1) launch_var<T, 1, DAMP>(e, va);
    else if (mode == 2) launch_var<T, 2, DAMP>(e, va);
    else launch_var<T, 4, DAMP>(e, va);
}

// mode 0: bare sweep; 1: tolerance loop sweep; 2: low-pass loop sweep;
// 3: batched tolerance sweep (stopped graphs frozen, per-graph stop rules).
// which: bit 0 launches the factor pass, bit 1 the variable pass.
template <typename T>
void launch_sweep(flbp_engine *e, int mode, int which = 3) {
    if (e->n_sets) {  // evidence sets: the direct form over grid.y = set, per-set stop rules
        if (which & 1) {
            FactorArgs fa = factor_args<T>(e);
            fa.set_done = e->d_gstate;
            fa.set_vf_stride = e->set_vs;
            fa.set_fv_stride = e->set_es;
            sets_factor_launch<T>(e->set_fgx, e->n_sets, fa, (const T *)e->d_vf, (T *)e->d_fv, e->d_ctl, e->d_set_cut,
                                  e->n_set_cut, e->stream);
        }
        if (which & 2) {
            VarArgs va = var_args(e);
            va.gstate = e->d_gstate;
            va.n_graphs = e->n_sets;
            va.set_vf_stride = e->set_vs;
            va.set_fv_stride = e->set_es;
            va.set_prior_stride = e->set_nv * (e->prec == 64 ? 16 : 8);
            va.set_belief_stride = e->set_nv;
            sets_var_launch<T>(e->damping != 0.0, e->set_vgx, e->n_sets, va, (const T *)e->d_fv, (T *)e->d_vf,
                               (T *)e->d_fvd, (T)e->damping, e->d_ctl, e->stream);
        }
        return;
    }
    // batched staged passes walk the live tiles only (the direct forms skip stopped graphs' items themselves)
    const bool live_lists = mode == 3 && e->d_act_f && (e->f_form == 0 || e->v_form == 0);
    if (which & 1) {
        FactorArgs fa = factor_args<T>(e);
        if (mode == 3) {
            fa.f_graph = e->d_f_graph;
            fa.gdone = e->d_gstate;
            fa.trange = e->d_ftrange;
            fa.n_graphs = e->n_graphs;
            if (live_lists) {  // flags, then the live tiles of each pass in tile order
                live_tile_flags_kernel<<<e->sms, 256, 0, e->stream>>>(e->d_ftrange, e->L.n_ftiles, e->d_vtrange,
                                                                      e->L.n_vtiles, e->d_gstate, e->d_act_flag,
                                                                      e->d_act_flag + e->L.n_ftiles, e->d_ctl);
                thrust::counting_iterator<uint32_t> it(0);
                size_t tb = e->cub_tmp_bytes;
                cub::DeviceSelect::Flagged(e->d_cub_tmp, tb, it, e->d_act_flag, e->d_act_f, &e->d_ctl->n_act_f,
                                           (int)e->L.n_ftiles, e->stream);
                tb = e->cub_tmp_bytes;
                cub::DeviceSelect::Flagged(e->d_cub_tmp, tb, it, e->d_act_flag + e->L.n_ftiles, e->d_act_v,
                                           &e->d_ctl->n_act_v, (int)e->L.n_vtiles, e->stream);
                fa.act_list = e->d_act_f;
                fa.n_act = &e->d_ctl->n_act_f;
            }
        }
        launch_factor<T>(e, fa, e->d_vf, e->d_fv);
    }
    if (!(which & 2)) return;
    VarArgs va = var_args(e);
    if (mode == 3) {
        va.v_graph = e->d_v_graph;
        va.gstate = e->d_gstate;
        va.trange = e->d_vtrange;
        va.n_graphs = e->n_graphs;
        if (live_lists) {
            va.act_list = e->d_act_v;
            va.n_act = &e->d_ctl->n_act_v;
        }
    }
    if (e->damping != 0.0) launch_var_mode<T, true>(e, va, mode);
    else launch_var_mode<T, false>(e, va, mode);
}

void launch_sweep_any(flbp_engine *e, int mode, int which = 3) {
    if (e->seq) {
        if (e->prec == 64) launch_seq_sweep<double>(e, mode, which);
        else launch_seq_sweep<float>(e, mode, which);
        return;
    }
    if (e->prec == 64) launch_sweep<double>(e, mode, which);
    else launch_sweep<float>(e, mode, which);
}

// Beliefs of the current messages (the damped ones under damping), without
// touching the run state.
template <typename T>
void launch_beliefs_only_t(flbp_engine *e, double *dst) {
    VarArgs a = var_args(e);
    a.belief = dst;
    const T *src = (const T *)(e->damping != 0.0 ? e->d_fvd : e->d_fv);
    // the tile counter of the variable pass is reset by the factor pass; none ran since the last one
    cudaMemsetAsync(reinterpret_cast<char *>(e->d_ctl) + offsetof(Ctl, vnext), 0, sizeof(unsigned int), e->stream);
    var_pass_kernel<T, 3, false, false, kStages><<<e->var_grid, kBlockThreads, var_smem<T, false>(), e->stream>>>(
        a, src, (T *)e->d_vf, nullptr, (T)0, e->d_ctl);
}

void launch_beliefs_only(flbp_engine *e, double *dst) {
    if (e->seq) {
        VarArgs va = var_args(e);
        va.belief = dst;
        seq_belief_kernel<3><<<seq_belief_grid(e), 256, 0, e->stream>>>(va, e->d_sq_S, e->d_sq_cnt, (uint32_t)e->L.V,
                                                                        e->d_ctl);
    } else if (e->prec == 64) launch_beliefs_only_t<double>(e, dst);
    else launch_beliefs_only_t<float>(e, dst);
    e->launches += 1;
}

// Executable graph of `n` consecutive sweeps of a mode, captured once.
int sweep_graph(flbp_engine *e, int mode, int n, cudaGraphExec_t *out) {
    auto key = std::make_pair(mode, n);
    auto it = e->graphs.find(key);
    if (it != e->graphs.end()) {
        *out = it->second;
        return FLBP_OK;
    }
    cudaGraph_t g = nullptr;
    FLBP_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < n; i++) launch_sweep_any(e, mode);
    FLBP_CUDA(cudaStreamEndCapture(e->stream, &g));
    cudaGraphExec_t x = nullptr;
    cudaError_t err = cudaGraphInstantiateWithFlags(&x, g, 0);
    cudaGraphDestroy(g);
    if (err != cudaSuccess) {
        set_error(std::string("CUDA graph instantiation failed: ") + cudaGetErrorString(err));
        return FLBP_ERR_CUDA;
    }
    e->graphs[key] = x;
    *out = x;
    return FLBP_OK;
}

// Launch n sweeps as power-of-two graph chunks (of at most 64 sweeps, and for
// a sequential schedule of about 2048 kernels).
int launch_sweeps(flbp_engine *e, int mode, long long n) {
    if (e->L.nf_sell + e->L.nf_big == 0 && e->L.V == 0) return FLBP_OK;
    const long long per = e->seq ? seq_sweep_launches(e, mode, 3)
                                 : 2 + (e->n_sets && e->n_set_cut ? 1 : 0) +
                                       (mode == 3 && e->d_act_f && (e->f_form == 0 || e->v_form == 0) ? 3 : 0);
    int kmax = 64;
    if (e->seq)
        while (kmax > 1 && (long long)kmax * per > 2048) kmax /= 2;
    if (e->ktime) {
        // Events around each pass, recorded by event nodes of a captured graph,
        // so that the passes run back to back as in the graph-replayed sweeps.
        while (n > 0) {
            const long long k = std::min<long long>(n, kmax);
            while (e->kev.size() < e->kev_used + 3 * (size_t)k) {
                cudaEvent_t ev;
                FLBP_CUDA(cudaEventCreate(&ev));
                e->kev.push_back(ev);
            }
            cudaGraph_t g = nullptr;
            FLBP_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
            for (long long i = 0; i < k; i++) {
                cudaEvent_t *ev = &e->kev[e->kev_used];
                e->kev_used += 3;
                cudaEventRecordWithFlags(ev[0], e->stream, cudaEventRecordExternal);
                launch_sweep_any(e, mode, 1);
                cudaEventRecordWithFlags(ev[1], e->stream, cudaEventRecordExternal);
                launch_sweep_any(e, mode, 2);
                cudaEventRecordWithFlags(ev[2], e->stream, cudaEventRecordExternal);
            }
            FLBP_CUDA(cudaStreamEndCapture(e->stream, &g));
            cudaGraphExec_t x = nullptr;
            cudaError_t err = cudaGraphInstantiateWithFlags(&x, g, 0);
            cudaGraphDestroy(g);
            if (err != cudaSuccess) {
                set_error(std::string("CUDA graph instantiation failed: ") + cudaGetErrorString(err));
                return FLBP_ERR_CUDA;
            }
            e->kgraphs.push_back(x);
            FLBP_CUDA(cudaGraphLaunch(x, e->stream));
            e->launches += per * k;
            n -= k;
        }
        return FLBP_OK;
    }
    while (n > 0) {
        int k = 1;
        while ((long long)k * 2 <= n && k < kmax) k *= 2;
        cudaGraphExec_t x;
        int rc = sweep_graph(e, mode, k, &x);
        if (rc) return rc;
        FLBP_CUDA(cudaGraphLaunch(x, e->stream));
        e->launches += per * k;
        n -= k;
    }
    return FLBP_OK;
}

int upload_ctl(flbp_engine *e) {
    FLBP_CUDA(cudaMemcpyAsync(e->d_ctl, e->h_ctl, sizeof(Ctl), cudaMemcpyHostToDevice, e->stream));
    return FLBP_OK;
}

int download_ctl(flbp_engine *e) {
    FLBP_CUDA(cudaMemcpyAsync(e->h_ctl, e->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, e->stream));
    FLBP_CUDA(cudaStreamSynchronize(e->stream));
    if (e->h_ctl->status != 0) {
        set_error("a device-side wait for a shared-memory copy timed out; results of this call are invalid");
        return FLBP_ERR_TIMEOUT;
    }
    return FLBP_OK;
}

void reset_ctl_for_run(flbp_engine *e, int mode) {
    Ctl &c = *e->h_ctl;
    std::memset(&c, 0, sizeof(Ctl));
    c.t = e->t;
    c.mode = mode;
    c.iters0 = e->iters;
    c.n_vars = e->L.V;
    c.maxtime_ns = 1e300;
    c.reason = FLBP_DIVERGED;
    c.damping = e->damping;
    c.pscale = (e->damping == 0.0) ? 1.0 : 1.0 - std::pow(e->damping, (double)e->t);
}

// Frees a buffer of dalloc in the order of the engine's stream (work
// already queued there may still read it).
inline void dfree(flbp_engine *e, void *p) {
    if (p) cudaFreeAsync(p, e->stream);
}

template <typename X>
int dalloc(flbp_engine *e, X **p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    FLBP_CUDA(pool_malloc((void **)p, n * sizeof(X), e->stream));
    e->bytes += n * sizeof(X);
    return FLBP_OK;
}

template <typename X, typename A>
int upload(flbp_engine *e, X *dst, const std::vector<X, A> &src) {
    if (src.empty()) return FLBP_OK;
    FLBP_CUDA(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(X), cudaMemcpyHostToDevice, e->stream));
    e->h2d_bytes += src.size() * sizeof(X);
    return FLBP_OK;
}

int begin_call(flbp_engine *e) {
    if (!e) {
        set_error("null engine handle");
        return FLBP_ERR_INVALID;
    }
    FLBP_CUDA(cudaSetDevice(e->device));
    return FLBP_OK;
}

// Entry points of the PARALL layout that a sequential schedule does not support.
int refuse_seq(flbp_engine *e, const char *what) {
    if (!e->seq) return FLBP_OK;
    set_error(std::string(what) + " is not available with a sequential update schedule");
    return FLBP_ERR_STATE;
}

// Entry points of a single graph's run state that an engine of evidence sets does not support.
int refuse_sets(flbp_engine *e, const char *what) {
    if (!e->n_sets) return FLBP_OK;
    set_error(std::string(what) + " is not available on an engine of evidence sets (use flbp_sets_run_tol)");
    return FLBP_ERR_STATE;
}

int record_start(flbp_engine *e) {
    FLBP_CUDA(cudaEventRecord(e->ev0, e->stream));
    return FLBP_OK;
}

int record_stop(flbp_engine *e) {
    FLBP_CUDA(cudaEventRecord(e->ev1, e->stream));
    FLBP_CUDA(cudaEventSynchronize(e->ev1));
    FLBP_CUDA(cudaEventElapsedTime(&e->last_ms, e->ev0, e->ev1));
    FLBP_CUDA(cudaGetLastError());
    // fold per-pass event pairs of the timing mode
    for (size_t k = 0; k + 3 <= e->kev_used; k += 3) {
        float a = 0.f, b = 0.f;
        FLBP_CUDA(cudaEventElapsedTime(&a, e->kev[k], e->kev[k + 1]));
        FLBP_CUDA(cudaEventElapsedTime(&b, e->kev[k + 1], e->kev[k + 2]));
        e->kt_ms[0] += a;
        e->kt_ms[1] += b;
        e->kt_n[0]++;
        e->kt_n[1]++;
    }
    e->kev_used = 0;
    for (auto x : e->kgraphs) cudaGraphExecDestroy(x);
    e->kgraphs.clear();
    return FLBP_OK;
}

void fill_info(flbp_engine *e, flbp_run_info *info, long long sweeps, long long launches0) {
    if (!info) return;
    info->sweeps = sweeps;
    info->total_sweeps = e->iters;
    info->maxdiff = e->h_ctl->mode ? e->h_ctl->maxdiff : std::numeric_limits<double>::quiet_NaN();
    info->frac = e->h_ctl->mode == 2 ? e->h_ctl->frac : 1.0;
    info->reason = e->h_ctl->reason;
    info->status = e->h_ctl->status;
    info->launches = e->launches - launches0;
}

// Stop-rule driven loop: chunks of sweeps until the device sets ctl->done.
int run_loop(flbp_engine *e, int mode, long long cap) {
    long long launched = 0;
    int k = 1;
    while (launched < cap) {
        const long long n = std::min<long long>(k, cap - launched);
        int rc = launch_sweeps(e, mode, n);
        if (rc) return rc;
        launched += n;
        rc = download_ctl(e);
        if (rc) return rc;
        if (e->h_ctl->done) break;
        k = std::min(k * 2, 64);
    }
    return FLBP_OK;
}

double sigmoid_d(double x) { return x >= 0 ? 1.0 / (1.0 + std::exp(-x)) : std::exp(x) / (1.0 + std::exp(x)); }

}  // namespace

extern "C" {

const char *flbp_last_error(void) { return g_last_error.c_str(); }

const char *flbp_version(void) { return "fastlbp_b200 0.1 (sm_100a)"; }

}  // extern "C"

namespace {

// Graph of every reference factor and variable of a batched engine (the
// concatenation order of its graphs); null for a single graph.
struct BatchSpec {
    std::vector<uint32_t> factor_graph, var_graph;
    std::vector<int64_t> var_off;
};

int create_engine(const flbp_graph_desc *graph, const flbp_engine_opts *opts, flbp_engine **out,
                  const BatchSpec *batch, bool host_layout = false);

// Cost of one factor of a tile, in slots, for dealing tiles to blocks.
constexpr double kTileCostFactorItem = 0.3;

}  // namespace

extern "C" int flbp_engine_create(const flbp_graph_desc *graph, const flbp_engine_opts *opts, flbp_engine **out) {
    return create_engine(graph, opts, out, nullptr);
}

namespace {

// Device words of the per-variable priors (finite part, +-inf counts) and of
// the big-tile copies of them.
void packed_priors(const flbp_engine *e, size_t nv_pad, std::vector<uint32_t> &prior, std::vector<uint32_t> &bt_prior) {
    const HostLayout &L = e->L;
    const size_t psz = e->prec == 64 ? 16 : 8;
    prior.assign(std::max<size_t>(1, nv_pad) * (psz / 4), 0u);
    // bit 31 of the count word: the variable has a folded finite constant
    // (its dL/dprior feeds a factor's dL/dp)
    std::vector<uint8_t> folded((size_t)L.V, 0);
    for (uint32_t v : L.prior_var) folded[v] = 1;
#pragma omp parallel for if (L.V >= (1 << 15))
    for (int64_t i = 0; i < L.V; i++) {
        const uint32_t cnt = L.prior_cnt[i] | (folded[i] ? 0x80000000u : 0u);
        if (e->prec == 64) {
            std::memcpy(&prior[4 * i], &L.prior_fin[i], 8);
            prior[4 * i + 2] = cnt;
        } else {
            const float f = (float)L.prior_fin[i];
            std::memcpy(&prior[2 * i], &f, 4);
            prior[2 * i + 1] = cnt;
        }
    }
    // priors of the variables of every big tile, in tile order
    bt_prior.assign(std::max<size_t>(1, L.vbt_deg.size()) * (psz / 4), 0u);
    for (uint32_t t = 0; t < L.n_vbtiles; t++) {
        const uint32_t *h = &L.vhdr[(size_t)kHdrWordsHost * t];
        const uint32_t b0 = h[0], n = h[1] & ~kBigTileFlag;
        for (uint32_t j = 0; j < n; j++) {
            const size_t k = (size_t)kTileGroupsHost * t + j, iv = (size_t)L.nv_sell + b0 + j;
            std::copy(&prior[iv * (psz / 4)], &prior[(iv + 1) * (psz / 4)], &bt_prior[k * (psz / 4)]);
        }
    }
    bt_prior.resize(L.vbt_deg.size() * (psz / 4));
}

// Which builder makes a new engine's layout: 0 the device for graphs of at
// least 2^18 edge slots (below that the host build is as fast), 1 always
// the host, 2 always the device (flbp_set_layout_builder).
std::atomic<int> g_layout_builder{0};

bool use_device_layout(const flbp_graph_desc &g) {
    const int mode = g_layout_builder.load();
    if (mode == 1) return false;
    const bool fits = g.n_slots < (1ll << 30) && g.n_factors < (1ll << 30) && g.n_vars < (1ll << 30);
    return fits && (mode == 2 || g.n_slots >= (1ll << 18));
}

// The host copies of the caller's factor p, q and heads that later calls
// (schedules, gradients, new probabilities) read.
void keep_host_graph(flbp_engine *e, const flbp_graph_desc &g) {
    if (g.n_factors > 0 && g.factor_p) e->factor_p_host.assign(g.factor_p, g.factor_p + g.n_factors);
    if (g.n_factors > 0 && g.factor_q) e->factor_q_host.assign(g.factor_q, g.factor_q + g.n_factors);
    if (g.n_factors > 0) e->ref_head.assign(g.factor_head, g.factor_head + g.n_factors);
}

// Device build of the layout: the caller's arrays are copied to the device
// (and kept there for ensure_host_layout), then dlayout.cu builds the layout.
// Host -> device copies of a graph's inputs go through a pair of pinned
// staging buffers per device (allocated once per process): the host threads
// pack the next chunk while the previous one is copied.
struct PinnedStage {
    std::mutex mu;
    char *buf[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
};
constexpr size_t kStageBytes = 8u << 20;
std::mutex g_stage_mu;
std::map<int, std::unique_ptr<PinnedStage>> g_stages;

// The staging buffers of `dev` (the current device); null if they cannot be had.
PinnedStage *stage_for(int dev) {
    std::lock_guard<std::mutex> lock(g_stage_mu);
    auto &slot = g_stages[dev];
    if (!slot) {
        auto st = std::make_unique<PinnedStage>();
        for (int k = 0; k < 2; k++)
            if (cudaHostAlloc((void **)&st->buf[k], kStageBytes, cudaHostAllocDefault) != cudaSuccess ||
                cudaEventCreateWithFlags(&st->done[k], cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                for (int j = 0; j < 2; j++) {
                    if (st->buf[j]) cudaFreeHost(st->buf[j]);
                    if (st->done[j]) cudaEventDestroy(st->done[j]);
                }
                return nullptr;
            }
        slot = std::move(st);
    }
    return slot.get();
}

// n elements get(i) of type X to dst on the engine's stream, through the
// staging buffers S (held by the caller), or straight from `plain` (n
// elements already of type X) without them.
template <typename X, typename Get>
cudaError_t staged_h2d(flbp_engine *e, PinnedStage *S, X *dst, size_t n, Get get, const X *plain = nullptr) {
    if (!S) {
        if (plain) return cudaMemcpyAsync(dst, plain, n * sizeof(X), cudaMemcpyHostToDevice, e->stream);
        std::vector<X> tmp(n);
#pragma omp parallel for if (n >= (1 << 15))
        for (int64_t i = 0; i < (int64_t)n; i++) tmp[(size_t)i] = get((size_t)i);
        cudaError_t ce = cudaMemcpyAsync(dst, tmp.data(), n * sizeof(X), cudaMemcpyHostToDevice, e->stream);
        return ce == cudaSuccess ? cudaStreamSynchronize(e->stream) : ce;
    }
    const size_t per = kStageBytes / sizeof(X);
    int k = 0;
    for (size_t c = 0; c < n; c += per, k ^= 1) {
        const size_t m = std::min(per, n - c);
        cudaError_t ce = cudaEventSynchronize(S->done[k]);  // the buffer's previous chunk has been copied
        if (ce != cudaSuccess) return ce;
        X *b = reinterpret_cast<X *>(S->buf[k]);
#pragma omp parallel for if (m >= (1 << 15))
        for (int64_t i = 0; i < (int64_t)m; i++) b[i] = get(c + (size_t)i);
        if ((ce = cudaMemcpyAsync(dst + c, b, m * sizeof(X), cudaMemcpyHostToDevice, e->stream)) != cudaSuccess ||
            (ce = cudaEventRecord(S->done[k], e->stream)) != cudaSuccess)
            return ce;
    }
    return cudaSuccess;
}

// Pinned host copies of the engines' control blocks: slots of a few pinned
// slabs shared by all engines of the process (a pinned allocation of its own
// per engine would cost more than the rest of a small engine's creation).
struct CtlSlots {
    std::mutex mu;
    std::vector<Ctl *> free;
};
CtlSlots g_ctl_slots;
constexpr size_t kCtlSlab = 256;

Ctl *ctl_slot_get() {
    std::lock_guard<std::mutex> lock(g_ctl_slots.mu);
    if (g_ctl_slots.free.empty()) {
        Ctl *slab = nullptr;
        if (cudaHostAlloc((void **)&slab, kCtlSlab * sizeof(Ctl), cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        for (size_t i = 0; i < kCtlSlab; i++) g_ctl_slots.free.push_back(slab + (kCtlSlab - 1 - i));
    }
    Ctl *c = g_ctl_slots.free.back();
    g_ctl_slots.free.pop_back();
    std::memset(c, 0, sizeof(Ctl));
    return c;
}

void ctl_slot_put(Ctl *c) {
    std::lock_guard<std::mutex> lock(g_ctl_slots.mu);
    g_ctl_slots.free.push_back(c);
}

// n elements from device memory to the caller's host memory through the
// staging buffers S (held by the caller; without them a plain copy): each
// chunk's device copy is in flight while the host threads copy out the
// previous one. Returns once dst holds everything.
template <typename X>
cudaError_t staged_d2h(flbp_engine *e, PinnedStage *S, X *dst, const X *src, size_t n) {
    cudaError_t ce;
    if (!S) {
        if ((ce = cudaMemcpyAsync(dst, src, n * sizeof(X), cudaMemcpyDeviceToHost, e->stream)) != cudaSuccess)
            return ce;
        return cudaStreamSynchronize(e->stream);
    }
    const size_t per = kStageBytes / sizeof(X), nch = (n + per - 1) / per;
    auto issue = [&](size_t c) -> cudaError_t {
        const size_t o = c * per, m = std::min(per, n - o);
        cudaError_t r = cudaMemcpyAsync(S->buf[c & 1], src + o, m * sizeof(X), cudaMemcpyDeviceToHost, e->stream);
        return r == cudaSuccess ? cudaEventRecord(S->done[c & 1], e->stream) : r;
    };
    for (size_t c = 0; c < nch && c < 2; c++)
        if ((ce = issue(c)) != cudaSuccess) return ce;
    for (size_t c = 0; c < nch; c++) {
        if ((ce = cudaEventSynchronize(S->done[c & 1])) != cudaSuccess) return ce;
        const size_t o = c * per, m = std::min(per, n - o);
        const X *b = reinterpret_cast<const X *>(S->buf[c & 1]);
#pragma omp parallel for if (m >= (1 << 15))
        for (int64_t i = 0; i < (int64_t)m; i++) dst[o + (size_t)i] = b[i];
        if (c + 2 < nch && (ce = issue(c + 2)) != cudaSuccess) return ce;
    }
    return cudaSuccess;
}

// device_layout's answer when the compact device input cannot hold the
// graph (a value beyond int32, a factor type or head mask the build
// rejects): the host build takes it, and reports what is wrong.
constexpr int kUseHostBuild = -1;

int device_layout(flbp_engine *e, const flbp_graph_desc &g, DevLayout &D) {
    std::string err;
    int rc = check_graph_shape(g, err);
    if (rc) {
        set_error(err);
        return rc;
    }
    const size_t F = (size_t)g.n_factors, E = (size_t)g.n_slots;
    // the compact device input (DevGraphIn): int32 offsets, slot variables
    // and heads, int8 types, the head masks as one code, p and q as given
    std::atomic<int> bad{0};
    auto i32 = [&](int64_t x) -> int32_t {
        if (x < INT32_MIN || x > INT32_MAX) {
            bad.store(1, std::memory_order_relaxed);
            return 0;
        }
        return (int32_t)x;
    };
    const bool any_clamped = g.factor_head_clamped != nullptr && F > 0;
    const size_t sz[7] = {F ? (F + 1) * 4 : 0, E * 4, F * 4, F, F * 8, F * 8, any_clamped ? F : 0};
    for (int k = 0; k < 7; k++) {
        if (!sz[k]) continue;
        FLBP_CUDA(pool_malloc(&e->d_in[k], sz[k], e->stream));
        e->h2d_bytes += sz[k];
    }
    PinnedStage *S = stage_for(e->device);
    std::unique_lock<std::mutex> lock;
    if (S) lock = std::unique_lock<std::mutex>(S->mu);
    cudaError_t ce = cudaSuccess;
    auto go = [&](cudaError_t c) {
        if (ce == cudaSuccess) ce = c;
    };
    const int64_t *off = g.factor_offsets, *sv = g.slot_var, *hd = g.factor_head;
    const int32_t *ty = g.factor_type, *cl = g.factor_head_clamped;
    const double *m0 = g.factor_mask0, *m1 = g.factor_mask1;
    if (F) go(staged_h2d<int32_t>(e, S, (int32_t *)e->d_in[0], F + 1, [&](size_t i) { return i32(off[i]); }));
    if (E) go(staged_h2d<int32_t>(e, S, (int32_t *)e->d_in[1], E, [&](size_t i) { return i32(sv[i]); }));
    if (F) {
        go(staged_h2d<int32_t>(e, S, (int32_t *)e->d_in[2], F, [&](size_t i) { return i32(hd[i]); }));
        go(staged_h2d<int8_t>(e, S, (int8_t *)e->d_in[3], F, [&](size_t i) -> int8_t {
            const int32_t t = ty[i];
            if (t != FLBP_SINGLETON && t != FLBP_AND && t != FLBP_OR) {
                bad.store(1, std::memory_order_relaxed);
                return 0;
            }
            return (int8_t)t;
        }));
        go(staged_h2d<double>(e, S, (double *)e->d_in[4], F, [&](size_t i) { return g.factor_p[i]; }, g.factor_p));
        go(staged_h2d<double>(e, S, (double *)e->d_in[5], F, [&](size_t i) { return g.factor_q[i]; }, g.factor_q));
    }
    if (any_clamped)
        go(staged_h2d<uint8_t>(e, S, (uint8_t *)e->d_in[6], F, [&](size_t i) -> uint8_t {
            if (!cl[i] || ty[i] == FLBP_SINGLETON) return kMaskFree;
            const double a = m0 ? m0[i] : 1.0, b = m1 ? m1[i] : 1.0;
            if (!((a == 0.0 || a == 1.0) && (b == 0.0 || b == 1.0))) {
                bad.store(1, std::memory_order_relaxed);
                return kMaskFree;
            }
            return a == 1.0 ? (b == 1.0 ? kMaskFree : kMaskZero) : (b == 1.0 ? kMaskOne : kMaskNone);
        }));
    if (S) {  // the buffers are free again once their last copies have landed
        if (ce == cudaSuccess) ce = cudaEventSynchronize(S->done[0]);
        if (ce == cudaSuccess) ce = cudaEventSynchronize(S->done[1]);
        lock.unlock();
    }
    if (ce != cudaSuccess) {
        set_error(std::string("graph upload failed: ") + cudaGetErrorString(ce));
        return FLBP_ERR_CUDA;
    }
    if (bad.load()) {
        for (void *&b : e->d_in)
            if (b) {
                cudaFree(b);
                b = nullptr;
            }
        e->h2d_bytes = 0;
        return kUseHostBuild;
    }
    DevGraphIn &in = e->din;
    in.off = (const int32_t *)e->d_in[0];
    in.slot_var = (const int32_t *)e->d_in[1];
    in.head = (const int32_t *)e->d_in[2];
    in.type = (const int8_t *)e->d_in[3];
    in.p = (const double *)e->d_in[4];
    in.q = (const double *)e->d_in[5];
    in.mcode = (const uint8_t *)e->d_in[6];
    rc = build_layout_device(g, in, e->prec, e->L, D, err, e->stream);
    if (rc) {
        free_dev_layout(D, e->stream);
        set_error(err);
        return rc;
    }
    e->dev_layout = true;
    return FLBP_OK;
}

void adopt_dev_layout(flbp_engine *e, DevLayout &D) {
    e->d_f_pos = D.f_pos;
    e->d_fg_base = D.fg_base;
    e->d_fb_off = D.fb_off;
    e->d_fb_deg = D.fb_deg;
    e->d_vg_base = D.vg_base;
    e->d_vb_off = D.vb_off;
    e->d_vb_deg = D.vb_deg;
    e->d_v_ent = D.v_ent;
    e->d_ftiles = D.ftiles;
    e->d_vtiles = D.vtiles;
    e->d_fbt_deg = D.fbt_deg;
    e->d_vbt_deg = D.vbt_deg;
    e->d_int_of_var = D.int_of_var;
    e->d_f_kind = D.f_kind;
    e->d_f_deg = D.f_deg;
    e->d_fbt_kind = D.fbt_kind;
    e->d_f_pq = D.f_pq;
    e->d_fbt_pq = D.fbt_pq;
    e->d_prior = D.prior;
    e->d_vbt_prior = D.vbt_prior;
    e->bytes += D.bytes;
    D = DevLayout();
}

// Deals the tiles of a pass to its `nb` blocks so that every block's total
// cost is about the same (largest first, each to the least loaded block;
// the huge items a block takes first count towards its load). A tile costs
// its slots plus `per_item` per item (a factor's head and denominators cost
// more than one slot). Each block's tiles are kept in tile order.
void deal_tiles(const hvec<uint32_t> &hdr, uint32_t n_tiles, uint32_t nb, double per_item,
                const std::vector<double> &huge_load, std::vector<uint32_t> &list, std::vector<uint32_t> &off) {
    std::vector<std::pair<double, uint32_t>> cost(n_tiles);
    for (uint32_t t = 0; t < n_tiles; t++) {
        const uint32_t *h = &hdr[(size_t)kHdrWordsHost * t];
        const uint32_t n = h[1] & ~kBigTileFlag;
        const double items = (h[1] & kBigTileFlag) ? n : 32.0 * n;
        cost[t] = {(double)(h[2 + n] - h[2]) + per_item * items, t};
    }
    std::stable_sort(cost.begin(), cost.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
    typedef std::pair<double, uint32_t> Load;  // (load, block)
    std::priority_queue<Load, std::vector<Load>, std::greater<Load>> q;
    for (uint32_t b = 0; b < nb; b++) q.push({b < huge_load.size() ? huge_load[b] : 0.0, b});
    std::vector<std::vector<uint32_t>> per(nb);
    for (const auto &c : cost) {
        Load l = q.top();
        q.pop();
        per[l.second].push_back(c.second);
        l.first += c.first;
        q.push(l);
    }
    list.clear();
    off.assign(1, 0u);
    for (auto &p : per) {
        std::sort(p.begin(), p.end());
        list.insert(list.end(), p.begin(), p.end());
        off.push_back((uint32_t)list.size());
    }
    if (list.empty()) list.push_back(0u);
}

int create_engine(const flbp_graph_desc *graph, const flbp_engine_opts *opts, flbp_engine **out,
                  const BatchSpec *batch, bool host_layout) {
    auto clk = [] { return std::chrono::steady_clock::now(); };
    auto us = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
        return (int64_t)std::chrono::duration_cast<std::chrono::microseconds>(b - a).count();
    };
    const auto t_begin = clk();
    if (!graph || !out) {
        set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    *out = nullptr;
    flbp_engine_opts o{32, -1, 0.0, nullptr};
    if (opts) o = *opts;
    if (o.precision != 32 && o.precision != 64) {
        set_error("precision must be 32 or 64");
        return FLBP_ERR_INVALID;
    }
    if (!(o.damping >= 0.0 && o.damping < 1.0)) {
        set_error("damping must lie in [0,1)");
        return FLBP_ERR_INVALID;
    }
    flbp_engine *e = new (std::nothrow) flbp_engine();
    if (!e) {
        set_error("host allocation failed");
        return FLBP_ERR_NOMEM;
    }
    std::string err;
    int rc = FLBP_OK;
    // The host build runs first (a malformed graph is reported without a
    // GPU); the device build needs the engine's device and stream.
    bool on_device = !batch && !host_layout && use_device_layout(*graph);
    if (!on_device) {
        GraphIds ids{0, nullptr, nullptr};
        if (batch)
            ids = GraphIds{(uint32_t)(batch->var_off.size() - 1), batch->factor_graph.data(), batch->var_graph.data()};
        auto tc0 = clk();
        rc = build_layout(*graph, e->L, err, batch ? &ids : nullptr);
        e->create_us[0] = us(tc0, clk());
        if (rc) {
            set_error(err);
            delete e;
            return rc;
        }
        keep_host_graph(e, *graph);
    }
    e->prec = o.precision;
    e->tsize = o.precision == 64 ? 8 : 4;
    e->damping = o.damping;
    auto fail = [&](int code) {
        std::string msg = g_last_error;
        flbp_engine_destroy(e);
        set_error(msg);
        return code;
    };
    if (o.device >= 0) {
        cudaError_t ce = cudaSetDevice(o.device);
        if (ce != cudaSuccess) {
            set_error(std::string("cudaSetDevice failed: ") + cudaGetErrorString(ce));
            delete e;
            return FLBP_ERR_CUDA;
        }
    }
    if (cudaGetDevice(&e->device) != cudaSuccess) {
        set_error("no CUDA device");
        delete e;
        return FLBP_ERR_CUDA;
    }
    if (o.stream) {
        e->stream = (cudaStream_t)o.stream;
    } else {
        if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
            set_error("stream creation failed");
            delete e;
            return FLBP_ERR_CUDA;
        }
        e->own_stream = true;
    }
    if (cudaEventCreate(&e->ev0) != cudaSuccess || cudaEventCreate(&e->ev1) != cudaSuccess) {
        set_error("event creation failed");
        return fail(FLBP_ERR_CUDA);
    }
    DevLayout DL;
    if (on_device) {
        auto tc0 = clk();
        rc = device_layout(e, *graph, DL);
        if (rc == kUseHostBuild) {  // the host build takes the graph (and reports what is wrong with it)
            if ((rc = build_layout(*graph, e->L, err, nullptr))) {
                set_error(err);
                return fail(rc);
            }
            keep_host_graph(e, *graph);
        } else if (rc) {
            return fail(rc);
        }
        e->create_us[0] = us(tc0, clk());
    }
    const HostLayout &L = e->L;
    const uint32_t nf = L.nf_sell + L.nf_big;
    const size_t ns = std::max<uint64_t>(1, L.n_slots);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
    e->sms = sms;
    // One full wave of resident blocks; the kernels stride over tiles and large items.
    int fb = 1, vb = 1;
    const bool damp = e->damping != 0.0;
    cudaError_t cfg =
        (e->prec == 64) ? configure_kernels<double>(damp, &fb, &vb) : configure_kernels<float>(damp, &fb, &vb);
    if (cfg != cudaSuccess) {
        set_error(std::string("kernel configuration failed: ") + cudaGetErrorString(cfg));
        return fail(FLBP_ERR_CUDA);
    }
    fb = std::max(fb, 1);
    vb = std::max(vb, 1);
    // One wave of resident blocks; every block's consumer warps first take the
    // items too large for a tile (one per warp), then the block's tiles.
    auto grid = [&](uint32_t n_tiles, uint32_t n_huge, int per_sm, uint32_t &tile_blocks) -> int {
        const uint64_t total = (uint64_t)sms * (uint64_t)per_sm;
        const uint64_t g = std::max<uint64_t>(
            1, std::min<uint64_t>(total, std::max<uint64_t>(n_tiles, (n_huge + kConsumerWarps - 1) / kConsumerWarps)));
        tile_blocks = (uint32_t)g;
        return (int)g;
    };
    e->factor_grid = grid(L.n_ftiles, L.nf_huge, fb, e->f_tile_blocks);
    e->var_grid = grid(L.n_vtiles, L.nv_huge, vb, e->v_tile_blocks);

    // Per-item arrays are padded to whole groups of 32 so that the tile copies
    // of the last group stay in bounds.
    const size_t nf_pad = std::max<size_t>(nf, 32ull * L.n_fgroups());
    const size_t nv_pad = std::max<size_t>((size_t)L.V, 32ull * L.n_vgroups());
    const size_t psz = e->prec == 64 ? 16 : 8;
    e->n_ent = std::max<size_t>(1, e->dev_layout ? DL.n_ent : L.v_ent.size());
    const size_t ne = e->n_ent;
    auto tc1 = clk();
    auto tc2 = tc1;
    if (e->dev_layout) {  // the layout's buffers are built; the run state's follow
        adopt_dev_layout(e, DL);
        if ((rc = dalloc(e, (char **)&e->d_vf, ns * e->tsize)) || (rc = dalloc(e, (char **)&e->d_fv, ne * e->tsize)) ||
            (damp && (rc = dalloc(e, (char **)&e->d_fvd, ne * e->tsize))) || (rc = dalloc(e, &e->d_belief, nv_pad)) ||
            (rc = dalloc(e, &e->d_lowpass, (size_t)L.V)) || (rc = dalloc(e, &e->d_ctl, 1)) ||
            (rc = dalloc(e, &e->d_ref_out, (size_t)L.V)))
            return fail(rc);
        if (!(e->h_ctl = ctl_slot_get())) {
            set_error("pinned allocation failed");
            return fail(FLBP_ERR_NOMEM);
        }
        std::memset(e->h_ctl, 0, sizeof(Ctl));
        tc2 = clk();
        e->create_us[1] = us(tc1, tc2);
    } else {
        if ((rc = dalloc(e, (char **)&e->d_vf, ns * e->tsize)) || (rc = dalloc(e, (char **)&e->d_fv, ne * e->tsize)) ||
            (damp && (rc = dalloc(e, (char **)&e->d_fvd, ne * e->tsize))) || (rc = dalloc(e, &e->d_f_pos, ns)) ||
            (rc = dalloc(e, (char **)&e->d_f_pq, 2 * nf_pad * e->tsize)) ||
            (rc = dalloc(e, &e->d_fg_base, L.fg_base.size())) || (rc = dalloc(e, &e->d_fb_off, L.fb_off.size())) ||
            (rc = dalloc(e, &e->d_f_kind, nf_pad)) || (rc = dalloc(e, &e->d_f_deg, nf_pad)) ||
            (rc = dalloc(e, &e->d_vg_base, L.vg_base.size())) || (rc = dalloc(e, &e->d_vb_off, L.vb_off.size())) ||
            (rc = dalloc(e, &e->d_v_ent, L.v_ent.size())) || (rc = dalloc(e, &e->d_ftiles, L.fhdr.size())) ||
            (rc = dalloc(e, &e->d_vtiles, L.vhdr.size())) || (rc = dalloc(e, &e->d_fb_deg, L.fb_deg.size())) ||
            (rc = dalloc(e, &e->d_vb_deg, L.vb_deg.size())) || (rc = dalloc(e, &e->d_fbt_deg, L.fbt_deg.size())) ||
            (rc = dalloc(e, &e->d_vbt_deg, L.vbt_deg.size())) || (rc = dalloc(e, &e->d_fbt_kind, L.fbt_kind.size())) ||
            (rc = dalloc(e, (char **)&e->d_fbt_pq, L.fbt_pq.size() * e->tsize)) ||
            (rc = dalloc(e, (char **)&e->d_vbt_prior, L.vbt_deg.size() * psz)) ||
            (rc = dalloc(e, (char **)&e->d_prior, std::max<size_t>(1, nv_pad) * psz)) ||
            (rc = dalloc(e, &e->d_belief, nv_pad)) || (rc = dalloc(e, &e->d_lowpass, (size_t)L.V)) ||
            (rc = dalloc(e, &e->d_ctl, 1)))
            return fail(rc);
        if (!(e->h_ctl = ctl_slot_get())) {
            set_error("pinned allocation failed");
            return fail(FLBP_ERR_NOMEM);
        }
        std::memset(e->h_ctl, 0, sizeof(Ctl));
        tc2 = clk();
        e->create_us[1] = us(tc1, tc2);
        std::vector<uint32_t> prior, bt_prior;
        packed_priors(e, nv_pad, prior, bt_prior);
        std::vector<uint8_t> kind_pad(nf_pad, 0), deg_pad(nf_pad, 0);
        std::copy(L.f_kind.begin(), L.f_kind.end(), kind_pad.begin());
        std::copy(L.f_deg.begin(), L.f_deg.end(), deg_pad.begin());
        // (p, q) of every factor in the message type, padded with zeros
        auto padded_pq = [&](auto zero) {
            using X = decltype(zero);
            hvec<X> v(2 * nf_pad);
            const int64_t n = (int64_t)v.size(), nr = (int64_t)L.f_pq.size();
    #pragma omp parallel for if (n >= (1 << 15))
            for (int64_t i = 0; i < n; i++) v[i] = i < nr ? (X)L.f_pq[i] : X(0);
            return v;
        };
        if (e->prec == 64) {
            if ((rc = upload(e, (double *)e->d_f_pq, padded_pq(0.0))) ||
                (rc = upload(e, (double *)e->d_fbt_pq, L.fbt_pq)))
                return fail(rc);
        } else {
            std::vector<float> bpq32(L.fbt_pq.begin(), L.fbt_pq.end());
            if ((rc = upload(e, (float *)e->d_f_pq, padded_pq(0.0f))) || (rc = upload(e, (float *)e->d_fbt_pq, bpq32)))
                return fail(rc);
        }
        if ((rc = upload(e, e->d_fg_base, L.fg_base)) || (rc = upload(e, e->d_fb_off, L.fb_off)) ||
            (rc = upload(e, e->d_f_pos, L.f_pos)) ||
            (rc = upload(e, e->d_f_kind, kind_pad)) || (rc = upload(e, e->d_f_deg, deg_pad)) ||
            (rc = upload(e, e->d_vg_base, L.vg_base)) || (rc = upload(e, e->d_vb_off, L.vb_off)) ||
            (rc = upload(e, e->d_v_ent, L.v_ent)) || (rc = upload(e, (uint32_t *)e->d_prior, prior)) ||
            (rc = upload(e, e->d_ftiles, L.fhdr)) || (rc = upload(e, e->d_vtiles, L.vhdr)) ||
            (rc = upload(e, e->d_fb_deg, L.fb_deg)) || (rc = upload(e, e->d_vb_deg, L.vb_deg)) ||
            (rc = upload(e, e->d_fbt_deg, L.fbt_deg)) || (rc = upload(e, e->d_vbt_deg, L.vbt_deg)) ||
            (rc = upload(e, e->d_fbt_kind, L.fbt_kind)) || (rc = upload(e, (uint32_t *)e->d_vbt_prior, bt_prior)) ||
            (rc = dalloc(e, &e->d_int_of_var, L.internal_of_var.size())) ||
            (rc = upload(e, e->d_int_of_var, L.internal_of_var)) || (rc = dalloc(e, &e->d_ref_out, (size_t)L.V)))
            return fail(rc);
    }
    cudaError_t ce = cudaSuccess;
    if ((ce = cudaStreamSynchronize(e->stream)) != cudaSuccess) {
        set_error(std::string("device initialisation failed: ") + cudaGetErrorString(ce));
        return fail(FLBP_ERR_CUDA);
    }
    e->create_us[2] = us(tc2, clk());
    if ((ce = cudaMemsetAsync(e->d_belief, 0, std::max<size_t>(1, nv_pad) * sizeof(double), e->stream)) != cudaSuccess ||
        (ce = cudaMemsetAsync(e->d_vf, 0, ns * e->tsize, e->stream)) != cudaSuccess ||
        (ce = cudaMemsetAsync(e->d_fv, 0, ne * e->tsize, e->stream)) != cudaSuccess ||
        (damp && (ce = cudaMemsetAsync(e->d_fvd, 0, ne * e->tsize, e->stream)) != cudaSuccess) ||
        (ce = cudaStreamSynchronize(e->stream)) != cudaSuccess) {
        set_error(std::string("device initialisation failed: ") + cudaGetErrorString(ce));
        return fail(FLBP_ERR_CUDA);
    }
    if (batch) {  // graph ids in the kernels' orders, padded like the per-item arrays
        e->n_graphs = (uint32_t)(batch->var_off.size() - 1);
        e->graph_var_off = batch->var_off;
        std::vector<uint32_t> fg(nf_pad, 0), vg(std::max<size_t>(1, nv_pad), 0);
        for (uint32_t f = 0; f < nf; f++) fg[f] = batch->factor_graph[L.factor_of_internal[f]];
        for (uint32_t iv = 0; iv < (uint32_t)L.V; iv++) vg[iv] = batch->var_graph[L.var_of_internal[iv]];
        auto ranges = [](const hvec<uint32_t> &hdr, uint32_t nt) {
            std::vector<uint2> r(std::max<uint32_t>(1, nt));
            for (uint32_t t = 0; t < nt; t++)
                r[t] = make_uint2(hdr[(size_t)kHdrWordsHost * t + kHdrGraphLo], hdr[(size_t)kHdrWordsHost * t + kHdrGraphHi]);
            return r;
        };
        const std::vector<uint2> fr = ranges(L.fhdr, L.n_ftiles), vr = ranges(L.vhdr, L.n_vtiles);
        if ((rc = dalloc(e, &e->d_f_graph, fg.size())) || (rc = dalloc(e, &e->d_v_graph, vg.size())) ||
            (rc = dalloc(e, &e->d_gstate, 4 * (size_t)e->n_graphs)) || (rc = upload(e, e->d_f_graph, fg)) ||
            (rc = upload(e, e->d_v_graph, vg)) || (rc = dalloc(e, &e->d_ftrange, fr.size())) ||
            (rc = dalloc(e, &e->d_vtrange, vr.size())) || (rc = upload(e, e->d_ftrange, fr)) ||
            (rc = upload(e, e->d_vtrange, vr)) || (rc = dalloc(e, &e->d_act_f, fr.size())) ||
            (rc = dalloc(e, &e->d_act_v, vr.size())) || (rc = dalloc(e, &e->d_act_flag, fr.size() + vr.size())))
            return fail(rc);
        {
            thrust::counting_iterator<uint32_t> it(0);
            size_t a = 0, b = 0;
            cub::DeviceSelect::Flagged(nullptr, a, it, e->d_act_flag, e->d_act_f, (unsigned int *)nullptr,
                                       (int)fr.size(), e->stream);
            cub::DeviceSelect::Flagged(nullptr, b, it, e->d_act_flag, e->d_act_v, (unsigned int *)nullptr,
                                       (int)vr.size(), e->stream);
            e->cub_tmp_bytes = std::max<size_t>({a, b, 16});
            if ((rc = dalloc(e, (char **)&e->d_cub_tmp, e->cub_tmp_bytes))) return fail(rc);
        }
        FLBP_CUDA(cudaMemsetAsync(e->d_gstate, 0, 4 * sizeof(int) * std::max<size_t>(1, e->n_graphs), e->stream));
        FLBP_CUDA(cudaStreamSynchronize(e->stream));
    }
    {  // each staged factor block's tiles (the variable pass keeps tiles b, b + grid, ...: measured faster)
        std::vector<double> fh((size_t)e->factor_grid, 0.0);
        for (uint32_t b = 0; b < L.nf_huge; b++) fh[b % e->factor_grid] += (double)L.fb_deg[b];
        std::vector<uint32_t> fl, fo;
        deal_tiles(L.fhdr, L.n_ftiles, (uint32_t)e->factor_grid, kTileCostFactorItem, fh, fl, fo);
        if ((rc = dalloc(e, &e->d_ftlist, fl.size())) || (rc = upload(e, e->d_ftlist, fl)) ||
            (rc = dalloc(e, &e->d_ftoff, fo.size())) || (rc = upload(e, e->d_ftoff, fo)))
            return fail(rc);
        FLBP_CUDA(cudaStreamSynchronize(e->stream));
    }
    e->create_us[3] = us(t_begin, clk()) - e->create_us[0] - e->create_us[1] - e->create_us[2];
    *out = e;
    return FLBP_OK;
}

// Installs the forms of the two passes (0 staged, 1/2 direct) with one wave
// of resident blocks for a direct form; captured sweep graphs are dropped.
int apply_forms(flbp_engine *e, int ff, int vf) {
    const bool damp = e->damping != 0.0;
    const HostLayout &L = e->L;
    auto grid = [&](int form, bool var, uint64_t items, uint64_t huge) -> int {
        const int bps = e->prec == 64 ? direct_blocks_per_sm<double>(form, var, damp)
                                      : direct_blocks_per_sm<float>(form, var, damp);
        const uint64_t need = std::max<uint64_t>((items + kConsumerWarps - 1) / kConsumerWarps, huge);
        return (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)e->sms * (uint64_t)bps, need));
    };
    if (ff) e->f_grid_direct = grid(ff, false, (uint64_t)(L.nf_big - L.nf_huge) + L.n_fgroups(), L.nf_huge);
    if (vf) e->v_grid_direct = grid(vf, true, (uint64_t)(L.nv_big - L.nv_huge) + L.n_vgroups(), L.nv_huge);
    FLBP_CUDA(cudaGetLastError());
    e->f_form = ff;
    e->v_form = vf;
    for (auto &kv : e->graphs) cudaGraphExecDestroy(kv.second);
    e->graphs.clear();
    return FLBP_OK;
}

// The complete host layout of an engine whose layout was built on the device
// (message export, gradients, clamps, schedules and new probabilities read
// it): the caller's graph arrays come back from the device and the host
// build runs on them; its result equals the device build's (tested).
int ensure_host_layout(flbp_engine *e) {
    if (e->L.complete) return FLBP_OK;
    // the compact device input (device_layout) back to the caller's arrays
    const size_t F = (size_t)e->L.F, E = (size_t)e->L.E;
    std::vector<int32_t> off32(F ? F + 1 : 0), sv32(E), head32(F);
    std::vector<int8_t> type8(F);
    std::vector<uint8_t> mcode(e->d_in[6] ? F : 0);
    std::vector<double> p(F), q(F);
    void *dst[7] = {off32.data(), sv32.data(), head32.data(), type8.data(), p.data(), q.data(), mcode.data()};
    const size_t bytes[7] = {off32.size() * 4, E * 4, F * 4, F, F * 8, F * 8, mcode.size()};
    for (int k = 0; k < 7; k++)
        if (e->d_in[k] && bytes[k])
            FLBP_CUDA(cudaMemcpyAsync(dst[k], e->d_in[k], bytes[k], cudaMemcpyDeviceToHost, e->stream));
    FLBP_CUDA(cudaStreamSynchronize(e->stream));
    std::vector<int64_t> off(off32.begin(), off32.end()), sv(sv32.begin(), sv32.end()), head(head32.begin(), head32.end());
    std::vector<int32_t> type(type8.begin(), type8.end()), clamped(mcode.size());
    std::vector<double> m0(mcode.size()), m1(mcode.size());
    for (size_t I = 0; I < mcode.size(); I++) {
        clamped[I] = mcode[I] != kMaskFree;
        m0[I] = (mcode[I] == kMaskOne || mcode[I] == kMaskNone) ? 0.0 : 1.0;
        m1[I] = (mcode[I] == kMaskZero || mcode[I] == kMaskNone) ? 0.0 : 1.0;
    }
    flbp_graph_desc g{};
    g.n_vars = e->L.V;
    g.n_factors = (int64_t)F;
    g.n_slots = (int64_t)E;
    g.factor_offsets = off.empty() ? nullptr : off.data();
    g.slot_var = sv.data();
    g.factor_head = head.data();
    g.factor_type = type.data();
    g.factor_p = p.data();
    g.factor_q = q.data();
    g.factor_head_clamped = clamped.empty() ? nullptr : clamped.data();
    g.factor_mask0 = m0.empty() ? nullptr : m0.data();
    g.factor_mask1 = m1.empty() ? nullptr : m1.data();
    HostLayout L;
    std::string err;
    int rc = build_layout(g, L, err, nullptr);
    if (rc) {
        set_error("host layout of a device-built engine: " + err);
        return rc;
    }
    keep_host_graph(e, g);
    e->L = std::move(L);
    for (void *&b : e->d_in)
        if (b) {
            cudaFree(b);
            b = nullptr;
        }
    return FLBP_OK;
}

// The v->f messages of clamped variables: +inf (clamped to 1) or -inf (0).
template <typename T>
__global__ void clamp_slots_kernel(const uint32_t *__restrict__ pairs, uint32_t n, T *vf) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) vf[pairs[2 * i]] = pairs[2 * i + 1] ? Num<T>::inf() : -Num<T>::inf();
}

int launch_clamp_slots(flbp_engine *e, uint32_t n) {
    if (!n) return FLBP_OK;
    if (e->prec == 64)
        clamp_slots_kernel<double><<<(n + 255) / 256, 256, 0, e->stream>>>(e->d_clamp_slots, n, (double *)e->d_vf);
    else
        clamp_slots_kernel<float><<<(n + 255) / 256, 256, 0, e->stream>>>(e->d_clamp_slots, n, (float *)e->d_vf);
    e->launches += 1;
    FLBP_CUDA(cudaGetLastError());
    return FLBP_OK;
}

int apply_clamp_slots(flbp_engine *e) { return launch_clamp_slots(e, (uint32_t)(e->clamp_slots.size() / 2)); }

}  // namespace

extern "C" {

int flbp_engine_destroy(flbp_engine *e) {
    if (!e) return FLBP_OK;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    for (auto &kv : e->graphs) cudaGraphExecDestroy(kv.second);
    for (auto ev : e->kev) cudaEventDestroy(ev);
    for (auto x : e->kgraphs) cudaGraphExecDestroy(x);
    void *bufs[] = {e->d_vf,     e->d_fv,       e->d_fvd,    e->d_f_pos,     e->d_f_pq,   e->d_fg_base,   e->d_fb_off,     e->d_f_kind,
                    e->d_f_deg,  e->d_vg_base,  e->d_vb_off, e->d_v_ent,     e->d_prior,      e->d_belief,
                    e->d_lowpass, e->d_hist,    e->d_hist_next, e->d_hist_count, e->d_ctl,    e->d_scratch,
                    e->d_ftiles, e->d_vtiles,  e->d_fb_deg, e->d_vb_deg, e->d_fbt_deg, e->d_vbt_deg,
                    e->d_fbt_kind, e->d_fbt_pq, e->d_vbt_prior, e->d_f_graph, e->d_v_graph, e->d_gstate, e->d_ftrange, e->d_vtrange,
                    e->d_ckpt, e->d_seg_vf, e->d_seg_fv, e->d_lam, e->d_lam2, e->d_mu, e->d_gp, e->d_gq,
                    e->d_gprior, e->d_gs, e->d_int_of_var, e->d_f_of_int, e->d_pri_fac, e->d_pri_var, e->d_pri_coef,
                    e->d_adj_in, e->d_adj_out, e->d_adj_groups, e->d_ref_out, e->d_clamp_slots, e->d_clamp_upd,
                    e->d_sq_foff, e->d_sq_var, e->d_sq_items, e->d_sq_tgt, e->d_sq_iota, e->d_sq_kind,
                    e->d_sq_cst, e->d_sq_pq, e->d_sq_fv, e->d_sq_vf, e->d_sq_nw, e->d_sq_S, e->d_sq_cnt};
    for (void *b : bufs)
        if (b) cudaFree(b);
    for (void *b : e->d_in)
        if (b) cudaFree(b);
    if (e->d_set_cut) cudaFree(e->d_set_cut);
    for (void *b : {(void *)e->d_ftlist, (void *)e->d_ftoff, (void *)e->d_act_f, (void *)e->d_act_v,
                    (void *)e->d_act_flag, e->d_cub_tmp})
        if (b) cudaFree(b);
    for (void *b : {(void *)e->d_fbt_src, (void *)e->d_vbt_src, (void *)e->d_pri_uvar, (void *)e->d_pri_uoff,
                    (void *)e->d_pri_ord, (void *)e->d_pri_sign, (void *)e->d_p_keep, (void *)e->d_q_keep,
                    (void *)e->d_bad})
        if (b) cudaFree(b);
    if (e->d_set_slots) cudaFree(e->d_set_slots);
    if (e->h_ctl) ctl_slot_put(e->h_ctl);
    if (e->ev0) cudaEventDestroy(e->ev0);
    if (e->ev1) cudaEventDestroy(e->ev1);
    if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return FLBP_OK;
}

int flbp_init(flbp_engine *e) {
    int rc = begin_call(e);
    if (rc) return rc;
    if (e->n_sets) {  // every set's messages uniform, its clamped variables' v->f messages +-inf, its
                      // beliefs 0 (those of a new engine, for the tolerance rule's first sweep)
        FLBP_CUDA(cudaMemsetAsync(e->d_vf, 0, e->n_sets * e->set_vs * e->tsize, e->stream));
        FLBP_CUDA(cudaMemsetAsync(e->d_belief, 0, e->n_sets * e->set_nv * sizeof(double), e->stream));
        FLBP_CUDA(cudaMemsetAsync(e->d_fv, 0, e->n_sets * e->set_es * e->tsize, e->stream));
        if (e->d_fvd) FLBP_CUDA(cudaMemsetAsync(e->d_fvd, 0, e->n_sets * e->set_es * e->tsize, e->stream));
        FLBP_CUDA(e->prec == 64 ? sets_init_slots<double>(e->d_set_slots, e->n_set_slots, (double *)e->d_vf, e->set_vs,
                                                          e->stream)
                                : sets_init_slots<float>(e->d_set_slots, e->n_set_slots, (float *)e->d_vf, e->set_vs,
                                                         e->stream));
        e->launches += e->n_set_slots ? 1 : 0;
        e->t = 0;
        e->lowpass_valid = false;
        return FLBP_OK;
    }
    const size_t ns = std::max<size_t>(1, e->L.n_slots);
    FLBP_CUDA(cudaMemsetAsync(e->d_vf, 0, ns * e->tsize, e->stream));
    FLBP_CUDA(cudaMemsetAsync(e->d_fv, 0, e->n_ent * e->tsize, e->stream));
    if (e->d_fvd) FLBP_CUDA(cudaMemsetAsync(e->d_fvd, 0, e->n_ent * e->tsize, e->stream));
    if (e->seq) {  // every message (1, 1): log-odds 0; totals and counts 0 (causal_bp.cu:824-856)
        FLBP_CUDA(cudaMemsetAsync(e->d_sq_fv, 0, std::max<size_t>(1, (size_t)e->L.E) * e->tsize, e->stream));
        FLBP_CUDA(cudaMemsetAsync(e->d_sq_S, 0, std::max<size_t>(1, (size_t)e->L.V) * sizeof(double), e->stream));
        FLBP_CUDA(cudaMemsetAsync(e->d_sq_cnt, 0, std::max<size_t>(1, (size_t)e->L.V) * sizeof(int2), e->stream));
    }
    if ((rc = apply_clamp_slots(e))) return rc;
    e->t = 0;
    e->lowpass_valid = false;
    return FLBP_OK;
}

int flbp_sweep(flbp_engine *e, int64_t n) {
    int rc = begin_call(e);
    if (rc || (rc = refuse_sets(e, "flbp_sweep"))) return rc;
    if (n < 0) {
        set_error("negative sweep count");
        return FLBP_ERR_INVALID;
    }
    reset_ctl_for_run(e, 0);
    if ((rc = upload_ctl(e)) || (rc = launch_sweeps(e, 0, n)) || (rc = download_ctl(e))) return rc;
    e->t += n;
    e->iters += n;
    return FLBP_OK;
}

int flbp_run_fixed(flbp_engine *e, int64_t sweeps, flbp_run_info *info) {
    int rc = begin_call(e);
    if (rc || (rc = refuse_sets(e, "flbp_run_fixed"))) return rc;
    if (sweeps < 0) {
        set_error("negative sweep count");
        return FLBP_ERR_INVALID;
    }
    const long long l0 = e->launches;
    reset_ctl_for_run(e, 0);
    if ((rc = record_start(e)) || (rc = upload_ctl(e)) || (rc = launch_sweeps(e, 0, sweeps))) return rc;
    launch_beliefs_only(e, e->d_belief);
    FLBP_CUDA(cudaMemcpyAsync(e->d_lowpass, e->d_belief, std::max<size_t>(1, e->L.V) * sizeof(double),
                              cudaMemcpyDeviceToDevice, e->stream));
    if ((rc = record_stop(e)) || (rc = download_ctl(e))) return rc;
    e->t += sweeps;
    e->iters += sweeps;
    e->lowpass_valid = true;
    fill_info(e, info, sweeps, l0);
    if (info) info->frac = 1.0;
    return FLBP_OK;
}

int flbp_reset_counts(flbp_engine *e) {
    int rc = begin_call(e);
    if (rc) return rc;
    const size_t nv = e->n_sets ? e->n_sets * e->set_nv
                                : std::max<size_t>({(size_t)1, (size_t)e->L.V, 32ull * e->L.n_vgroups()});
    FLBP_CUDA(cudaMemsetAsync(e->d_belief, 0, nv * sizeof(double), e->stream));
    FLBP_CUDA(cudaStreamSynchronize(e->stream));
    e->iters = 0;
    e->lowpass_valid = false;
    return FLBP_OK;
}

int flbp_run_tol(flbp_engine *e, double tol, int64_t maxiter, double maxtime, flbp_run_info *info) {
    int rc = begin_call(e);
    if (rc || (rc = refuse_sets(e, "flbp_run_tol"))) return rc;
    const long long l0 = e->launches;
    reset_ctl_for_run(e, 1);
    Ctl &c = *e->h_ctl;
    c.tol = tol;
    c.maxiter = maxiter;
    c.maxtime_ns = maxtime * 1e9;
    c.maxdiff = INFINITY;
    if ((rc = record_start(e))) return rc;
    long long done_sweeps = 0;
    if (e->iters < maxiter && maxtime > 0.0 && INFINITY > tol) {
        if ((rc = upload_ctl(e)) || (rc = run_loop(e, 1, maxiter - e->iters))) return rc;
        if ((rc = download_ctl(e))) return rc;
        done_sweeps = e->h_ctl->run_sweeps;
    }
    if ((rc = record_stop(e))) return rc;
    e->t += done_sweeps;
    e->iters += done_sweeps;
    fill_info(e, info, done_sweeps, l0);
    return FLBP_OK;
}

int flbp_run_lowpass(flbp_engine *e, double tol, int64_t min_iters, int64_t max_iters, int64_t hist_length,
                     double maxtime, flbp_run_info *info) {
    int rc = begin_call(e);
    if (rc || (rc = refuse_sets(e, "flbp_run_lowpass"))) return rc;
    if (hist_length <= 0) {
        set_error("belief history length must be positive");
        return FLBP_ERR_INVALID;
    }
    if (max_iters <= min_iters || min_iters < 0) {
        set_error("low-pass run needs 0 <= minIters < maxIters");
        return FLBP_ERR_INVALID;
    }
    const size_t V = (size_t)e->L.V;
    if ((uint64_t)hist_length > e->hist_cap) {
        dfree(e, e->d_hist);
        dfree(e, e->d_hist_next);
        dfree(e, e->d_hist_count);
        e->d_hist = nullptr;
        e->d_hist_next = e->d_hist_count = nullptr;
        e->hist_cap = 0;
        if ((rc = dalloc(e, &e->d_hist, std::max<size_t>(1, V) * (size_t)hist_length)) ||
            (rc = dalloc(e, &e->d_hist_next, V)) || (rc = dalloc(e, &e->d_hist_count, V)))
            return rc;
    }
    e->hist_cap = (uint32_t)hist_length;
    FLBP_CUDA(cudaMemsetAsync(e->d_hist_next, 0, std::max<size_t>(1, V) * sizeof(uint32_t), e->stream));
    FLBP_CUDA(cudaMemsetAsync(e->d_hist_count, 0, std::max<size_t>(1, V) * sizeof(uint32_t), e->stream));
    // Graphs captured with a different history length are stale.
    for (auto it = e->graphs.begin(); it != e->graphs.end();) {
        if (it->first.first == 2) {
            cudaGraphExecDestroy(it->second);
            it = e->graphs.erase(it);
        } else {
            ++it;
        }
    }
    const long long l0 = e->launches;
    reset_ctl_for_run(e, 2);
    Ctl &c = *e->h_ctl;
    c.tol = tol;
    c.min_iters = min_iters;
    c.max_iters = max_iters;
    c.maxtime_ns = maxtime * 1e9;
    c.frac = 1.0;
    c.maxdiff = INFINITY;
    if ((rc = record_start(e))) return rc;
    long long done_sweeps = 0;
    if (maxtime >= 0.0) {
        if ((rc = upload_ctl(e)) || (rc = run_loop(e, 2, max_iters + 1))) return rc;
        if ((rc = download_ctl(e))) return rc;
        done_sweeps = e->h_ctl->run_sweeps;
    }
    if (e->h_ctl->reason == FLBP_ALL_CONVERGED && done_sweeps > 0) {
        FLBP_CUDA(cudaMemcpyAsync(e->d_lowpass, e->d_belief, std::max<size_t>(1, V) * sizeof(double),
                                  cudaMemcpyDeviceToDevice, e->stream));
    } else if (V > 0) {
        lowpass_kernel<<<(unsigned)((V + 255) / 256), 256, 0, e->stream>>>(
            e->d_hist, e->d_hist_next, e->d_hist_count, e->hist_cap, (uint32_t)V, e->d_lowpass);
        e->launches += 1;
    }
    if ((rc = record_stop(e))) return rc;
    e->t += done_sweeps;
    e->iters += done_sweeps;
    e->lowpass_valid = true;
    fill_info(e, info, done_sweeps, l0);
    if (info && done_sweeps == 0) info->frac = 1.0;
    return FLBP_OK;
}

// A per-variable device array in the caller's variable order, gathered on
// the device and copied straight into `out`.
static int fetch_internal(flbp_engine *e, const double *dsrc, double *out, int64_t n) {
    if (n != e->L.V) {
        set_error("output length must equal the number of variables");
        return FLBP_ERR_INVALID;
    }
    if (!n) return FLBP_OK;
    int rc;
    if (!e->d_int_of_var) {
        std::vector<uint32_t> iov(e->L.internal_of_var.begin(), e->L.internal_of_var.end());
        if ((rc = dalloc(e, &e->d_int_of_var, iov.size())) || (rc = upload(e, e->d_int_of_var, iov))) return rc;
    }
    if (!e->d_ref_out && (rc = dalloc(e, &e->d_ref_out, (size_t)n))) return rc;
    gather_vars_kernel<<<(unsigned)((n + 255) / 256), 256, 0, e->stream>>>(dsrc, e->d_int_of_var, n, e->d_ref_out);
    e->launches += 1;
    FLBP_CUDA(cudaGetLastError());
    PinnedStage *S = n >= (1 << 16) ? stage_for(e->device) : nullptr;  // large outputs through the staging buffers
    std::unique_lock<std::mutex> lock;
    if (S) lock = std::unique_lock<std::mutex>(S->mu);
    FLBP_CUDA(staged_d2h<double>(e, S, out, e->d_ref_out, (size_t)n));
    return FLBP_OK;
}

int flbp_get_beliefs(flbp_engine *e, double *out, int64_t n) {
    int rc = begin_call(e);
    if (rc) return rc;
    if (e->n_sets) {  // set k's beliefs at [k V, (k + 1) V)
        const int64_t V = e->L.V;
        if (n != V * (int64_t)e->n_sets) {
            set_error("output length must equal the number of sets times the number of variables");
            return FLBP_ERR_INVALID;
        }
        for (uint32_t k = 0; k < e->n_sets; k++)
            if ((rc = fetch_internal(e, e->d_belief + (size_t)k * e->set_nv, out + (size_t)k * V, V))) return rc;
        return FLBP_OK;
    }
    return fetch_internal(e, e->d_belief, out, n);
}

int flbp_get_lowpass(flbp_engine *e, double *out, int64_t n) {
    int rc = begin_call(e);
    if (rc || (rc = refuse_sets(e, "flbp_get_lowpass"))) return rc;
    if (!e->lowpass_valid) return fetch_internal(e, e->d_belief, out, n);
    return fetch_internal(e, e->d_lowpass, out, n);
}

int flbp_compute_beliefs(flbp_engine *e, double *out, int64_t n) {
    int rc = begin_call(e);
    if (rc || (rc = refuse_sets(e, "flbp_compute_beliefs"))) return rc;
    reset_ctl_for_run(e, 0);
    if (!e->d_scratch && (rc = dalloc(e, &e->d_scratch, (size_t)e->L.V))) return rc;
    if ((rc = upload_ctl(e))) return rc;
    launch_beliefs_only(e, e->d_scratch);
    FLBP_CUDA(cudaGetLastError());
    return fetch_internal(e, e->d_scratch, out, n);
}

// f->v messages in the reference's variable-major slot order: from the
// entry array in use (the damped one under damping) for computed messages,
// the folded constants otherwise.
static int fv_lambda(flbp_engine *e, std::vector<double> &lam) {
    build_export_maps(e->L);
    const HostLayout &L = e->L;
    if (e->seq) {  // one message per edge, in device-slot order
        const size_t ne = std::max<size_t>(1, (size_t)L.E);
        std::vector<double> m(ne);
        if (e->prec == 64) {
            FLBP_CUDA(cudaMemcpyAsync(m.data(), e->d_sq_fv, ne * 8, cudaMemcpyDeviceToHost, e->stream));
        } else {
            std::vector<float> f(ne);
            FLBP_CUDA(cudaMemcpyAsync(f.data(), e->d_sq_fv, ne * 4, cudaMemcpyDeviceToHost, e->stream));
            FLBP_CUDA(cudaStreamSynchronize(e->stream));
            for (size_t i = 0; i < ne; i++) m[i] = f[i];
        }
        FLBP_CUDA(cudaStreamSynchronize(e->stream));
        lam.assign((size_t)L.E, 0.0);
        for (int64_t r = 0; r < L.E; r++) lam[L.fm_to_vm[r]] = m[e->SQ.dslot[r]];
        return FLBP_OK;
    }
    const size_t ne = L.v_ent.size();
    const void *src = e->d_fvd ? e->d_fvd : e->d_fv;
    std::vector<double> ent(ne);
    if (ne) {
        if (e->prec == 64) {
            FLBP_CUDA(cudaMemcpyAsync(ent.data(), src, ne * 8, cudaMemcpyDeviceToHost, e->stream));
        } else {
            std::vector<float> f(ne);
            FLBP_CUDA(cudaMemcpyAsync(f.data(), src, ne * 4, cudaMemcpyDeviceToHost, e->stream));
            FLBP_CUDA(cudaStreamSynchronize(e->stream));
            for (size_t i = 0; i < ne; i++) ent[i] = f[i];
        }
        FLBP_CUDA(cudaStreamSynchronize(e->stream));
    }
    const double scale = (e->damping == 0.0) ? 1.0 : 1.0 - std::pow(e->damping, (double)e->t);
    lam.assign((size_t)L.E, 0.0);
    for (int64_t k = 0; k < L.E; k++) {
        const int64_t s = L.ref_fv_src[k];
        if (s >= 0) lam[k] = ent[s];
        else if (s == -2) lam[k] = INFINITY;
        else if (s == -3) lam[k] = -INFINITY;
        else lam[k] = L.ref_const[k] * scale;
    }
    return FLBP_OK;
}

static void pair_of(double lam, double &m0, double &m1) {
    if (lam == INFINITY) {
        m0 = 0.0;
        m1 = 1.0;
    } else if (lam == -INFINITY) {
        m0 = 1.0;
        m1 = 0.0;
    } else {
        m1 = sigmoid_d(lam);
        m0 = sigmoid_d(-lam);
    }
}

int flbp_get_fv_messages(flbp_engine *e, double *m0, double *m1, int64_t n) {
    int rc = begin_call(e);
    if (rc || (rc = refuse_sets(e, "message export")) || (rc = ensure_host_layout(e))) return rc;
    if (n != e->L.E) {
        set_error("output length must equal the number of edge slots");
        return FLBP_ERR_INVALID;
    }
    if (e->t == 0) {  // init() fills both states with 1 (causal_bp.cu:825-841)
        for (int64_t k = 0; k < n; k++) m0[k] = m1[k] = 1.0;
        return FLBP_OK;
    }
    std::vector<double> lam;
    if ((rc = fv_lambda(e, lam))) return rc;
    for (int64_t k = 0; k < n; k++) pair_of(lam[k], m0[k], m1[k]);
    return FLBP_OK;
}

int flbp_get_vf_messages(flbp_engine *e, double *m0, double *m1, int64_t n) {
    int rc = begin_call(e);
    if (rc || (rc = refuse_sets(e, "message export")) || (rc = ensure_host_layout(e))) return rc;
    const HostLayout &L = e->L;
    if (n != L.E) {
        set_error("output length must equal the number of edge slots");
        return FLBP_ERR_INVALID;
    }
    if (e->t == 0) {
        for (int64_t k = 0; k < n; k++) m0[k] = m1[k] = 1.0;
        return FLBP_OK;
    }
    std::vector<double> lam;
    if ((rc = fv_lambda(e, lam))) return rc;
    std::vector<double> S((size_t)L.V, 0.0);
    std::vector<int> np((size_t)L.V, 0), nn((size_t)L.V, 0);
    for (int64_t k = 0; k < L.E; k++) {
        const int64_t v = L.vm_var[k];
        if (lam[k] == INFINITY) np[v]++;
        else if (lam[k] == -INFINITY) nn[v]++;
        else S[v] += lam[k];
    }
    for (int64_t e_ = 0; e_ < L.E; e_++) {
        const int64_t k = L.fm_to_vm[e_], v = L.vm_var[k];
        double s = S[v];
        int a = np[v], b = nn[v];
        if (lam[k] == INFINITY) a--;
        else if (lam[k] == -INFINITY) b--;
        else s -= lam[k];
        const double x = (a > 0 && b > 0) ? 0.0 : a > 0 ? INFINITY : b > 0 ? -INFINITY : s;
        pair_of(x, m0[e_], m1[e_]);
    }
    return FLBP_OK;
}

int flbp_engine_stats(flbp_engine *e, int64_t *c, int64_t n) {
    if (!e || !c) {
        set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    const int64_t v[20] = {e->L.V, e->L.F, e->L.E, (int64_t)(e->L.nf_sell + e->L.nf_big),
                           (int64_t)e->L.n_active_slots, (int64_t)e->L.nf_big, (int64_t)e->L.nv_big,
                           (int64_t)e->bytes, (int64_t)e->h2d_bytes, (int64_t)e->launches,
                           (int64_t)e->L.nf_huge, (int64_t)e->L.nv_huge, (int64_t)e->L.n_fbtiles,
                           (int64_t)e->L.n_vbtiles, e->create_us[0], e->create_us[1], e->create_us[2],
                           e->create_us[3], (int64_t)e->L.n_ftiles, (int64_t)e->L.n_vtiles};
    for (int64_t i = 0; i < n && i < 20; i++) c[i] = v[i];
    return FLBP_OK;
}

int flbp_set_kernel_timing(flbp_engine *e, int32_t enable) {
    if (!e) {
        set_error("null engine handle");
        return FLBP_ERR_INVALID;
    }
    e->ktime = enable != 0;
    e->kt_ms[0] = e->kt_ms[1] = 0.0;
    e->kt_n[0] = e->kt_n[1] = 0;
    return FLBP_OK;
}

int flbp_kernel_times(flbp_engine *e, double *ms, int64_t *counts) {
    if (!e || !ms || !counts) {
        set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    for (int i = 0; i < 2; i++) {
        ms[i] = e->kt_ms[i];
        counts[i] = e->kt_n[i];
    }
    return FLBP_OK;
}

int flbp_set_tuning(flbp_engine *e, const flbp_tuning *t) {
    int rc = begin_call(e);
    if (rc || (rc = refuse_sets(e, "flbp_set_tuning"))) return rc;
    if (!t || t->factor_form < 0 || t->factor_form > 2 || t->var_form < 0 || t->var_form > 2) {
        set_error("flbp_set_tuning: forms must be 0 (staged), 1 or 2 (direct)");
        return FLBP_ERR_INVALID;
    }
    return apply_forms(e, t->factor_form, t->var_form);
}

int flbp_get_tuning(flbp_engine *e, flbp_tuning *t) {
    if (!e || !t) {
        set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    t->factor_form = e->f_form;
    t->var_form = e->v_form;
    t->factor_blocks = e->f_form ? e->f_grid_direct : e->factor_grid;
    t->var_blocks = e->v_form ? e->v_grid_direct : e->var_grid;
    return FLBP_OK;
}

// ---- autotuner: the form of each pass, timed on the engine's own graph ----

namespace {

struct TuneKey {
    int prec, damped, batched, kind, lv, le, big;
    bool operator<(const TuneKey &o) const {
        return std::tie(prec, damped, batched, kind, lv, le, big) <
               std::tie(o.prec, o.damped, o.batched, o.kind, o.lv, o.le, o.big);
    }
};
std::mutex g_tune_mu;
std::map<TuneKey, std::pair<int, int>> g_tune_cache;

int ilog2(uint64_t x) {
    int r = 0;
    while (x > 1) {
        x >>= 1;
        r++;
    }
    return r;
}

// Size class of the graph: log2 of variables and slots, and the share of
// slots held by items too wide for a lane (the fan-in histogram's tail) in
// eighths.
TuneKey tune_key(const flbp_engine *e, int kind) {
    const HostLayout &L = e->L;
    uint64_t wide = 0;
    for (uint32_t b = 0; b < L.nf_big; b++) wide += L.fb_deg[b];
    for (uint32_t b = 0; b < L.nv_big; b++) wide += L.vb_deg[b];
    const uint64_t tot = std::max<uint64_t>(1, 2 * L.n_active_slots);
    return TuneKey{e->prec, e->damping != 0.0 ? 1 : 0, e->n_graphs ? 1 : 0, kind, ilog2((uint64_t)L.V + 1),
                   ilog2((uint64_t)L.E + 1), (int)std::min<uint64_t>(8, (8 * wide + tot - 1) / tot)};
}

}  // namespace

int flbp_autotune(flbp_engine *e, int32_t kind, int64_t sweeps, double tol, int32_t reps, flbp_tuning *chosen) {
    int rc = begin_call(e);
    if (rc || (rc = refuse_sets(e, "flbp_autotune"))) return rc;
    if ((rc = refuse_seq(e, "flbp_autotune"))) return rc;
    if (kind < 0 || kind > 1 || sweeps < 1 || reps < 1) {
        set_error("flbp_autotune: kind must be 0 (fixed sweeps) or 1 (tolerance run), sweeps and reps positive");
        return FLBP_ERR_INVALID;
    }
    const TuneKey key = tune_key(e, kind);
    std::pair<int, int> best{-1, -1};
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) best = it->second;
    }
    if (best.first < 0) {
        // Keep what a run changes: the sweep counts and the previous beliefs
        // of the tolerance rule (device), restored after the timing runs.
        const long long iters0 = e->iters, t0 = e->t;
        const bool lp0 = e->lowpass_valid;
        const size_t nb = std::max<size_t>((size_t)e->L.V, 32ull * e->L.n_vgroups());
        double *saved = nullptr;
        FLBP_CUDA(cudaMalloc((void **)&saved, std::max<size_t>(1, nb) * sizeof(double)));
        FLBP_CUDA(cudaMemcpyAsync(saved, e->d_belief, std::max<size_t>(1, nb) * sizeof(double), cudaMemcpyDeviceToDevice,
                                  e->stream));
        auto time_one = [&](int ff, int vf, double *ms) -> int {
            int r = apply_forms(e, ff, vf);
            if (r) return r;
            std::vector<double> ts;
            for (int i = 0; i <= reps; i++) {  // the first run captures the sweep graphs
                if ((r = flbp_init(e))) return r;
                e->iters = 0;
                if (kind == 0) r = flbp_run_fixed(e, sweeps, nullptr);
                else if (e->n_graphs) r = flbp_batch_run_tol(e, tol, sweeps, 1e9, nullptr, nullptr, nullptr);
                else r = flbp_run_tol(e, tol, sweeps, 1e9, nullptr);
                if (r) return r;
                if (i > 0) ts.push_back(e->last_ms);
            }
            std::sort(ts.begin(), ts.end());
            *ms = ts[ts.size() / 2];
            return FLBP_OK;
        };
        // coordinate descent: the factor pass's form with the variable pass
        // staged, then the variable pass's form with that factor form
        double bms = 0.0, ms = 0.0;
        int bf = 0, bv = 0;
        rc = time_one(0, 0, &bms);
        for (int ff = 1; ff <= 2 && !rc; ff++) {
            rc = time_one(ff, 0, &ms);
            if (!rc && ms < bms) bms = ms, bf = ff;
        }
        for (int vf = 1; vf <= 2 && !rc; vf++) {
            rc = time_one(bf, vf, &ms);
            if (!rc && ms < bms) bms = ms, bv = vf;
        }
        e->iters = iters0;
        e->t = t0;
        e->lowpass_valid = lp0;
        cudaMemcpyAsync(e->d_belief, saved, std::max<size_t>(1, nb) * sizeof(double), cudaMemcpyDeviceToDevice,
                        e->stream);
        cudaStreamSynchronize(e->stream);
        cudaFree(saved);
        if (rc) return rc;
        best = {bf, bv};
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune_cache[key] = best;
    }
    if ((rc = apply_forms(e, best.first, best.second))) return rc;
    if ((rc = flbp_init(e))) return rc;
    if (chosen) {
        chosen->factor_form = e->f_form;
        chosen->var_form = e->v_form;
        chosen->factor_blocks = e->f_form ? e->f_grid_direct : e->factor_grid;
        chosen->var_blocks = e->v_form ? e->v_grid_direct : e->var_grid;
    }
    return FLBP_OK;
}

int flbp_set_layout_builder(int32_t mode) {
    if (mode < 0 || mode > 2) {
        set_error("flbp_set_layout_builder: mode must be 0 (choose by size), 1 (host) or 2 (device)");
        return FLBP_ERR_INVALID;
    }
    g_layout_builder.store(mode);
    return FLBP_OK;
}

int flbp_engine_layout_digest(flbp_engine *e, uint64_t *digest, int32_t *built_on_device) {
    int rc = begin_call(e);
    if (rc) return rc;
    if (!digest) {
        set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    const HostLayout &L = e->L;
    const size_t psz = e->prec == 64 ? 16 : 8, nf = L.nf_sell + L.nf_big;
    const size_t nf_pad = std::max<size_t>(nf, 32ull * L.n_fgroups());
    const size_t nv_pad = std::max<size_t>((size_t)L.V, 32ull * L.n_vgroups());
    uint64_t h = 1469598103934665603ull;
    auto bytes = [&](const void *p, size_t n) {
        const unsigned char *c = static_cast<const unsigned char *>(p);
        for (size_t i = 0; i < n; i++) h = (h ^ c[i]) * 1099511628211ull;
    };
    std::vector<unsigned char> buf;
    auto dev = [&](const void *p, size_t n) -> int {
        const uint64_t len = n;
        bytes(&len, sizeof len);
        if (!n) return FLBP_OK;
        buf.resize(n);
        FLBP_CUDA(cudaMemcpyAsync(buf.data(), p, n, cudaMemcpyDeviceToHost, e->stream));
        FLBP_CUDA(cudaStreamSynchronize(e->stream));
        bytes(buf.data(), n);
        return FLBP_OK;
    };
    if ((rc = dev(e->d_fg_base, L.fg_base.size() * 4)) || (rc = dev(e->d_fb_off, L.fb_off.size() * 4)) ||
        (rc = dev(e->d_fb_deg, L.fb_deg.size() * 4)) || (rc = dev(e->d_f_kind, nf_pad)) ||
        (rc = dev(e->d_f_deg, nf_pad)) || (rc = dev(e->d_f_pq, 2 * nf_pad * e->tsize)) ||
        (rc = dev(e->d_vg_base, L.vg_base.size() * 4)) || (rc = dev(e->d_vb_off, L.vb_off.size() * 4)) ||
        (rc = dev(e->d_vb_deg, L.vb_deg.size() * 4)) || (rc = dev(e->d_v_ent, e->n_ent * 4)) ||
        (rc = dev(e->d_f_pos, std::max<uint64_t>(1, L.n_slots) * 4)) || (rc = dev(e->d_prior, nv_pad * psz)) ||
        (rc = dev(e->d_ftiles, L.fhdr.size() * 4)) || (rc = dev(e->d_vtiles, L.vhdr.size() * 4)) ||
        (rc = dev(e->d_fbt_deg, L.fbt_deg.size() * 4)) || (rc = dev(e->d_vbt_deg, L.vbt_deg.size() * 4)) ||
        (rc = dev(e->d_fbt_kind, L.fbt_kind.size())) || (rc = dev(e->d_fbt_pq, L.fbt_pq.size() * e->tsize)) ||
        (rc = dev(e->d_vbt_prior, L.vbt_deg.size() * psz)) || (rc = dev(e->d_int_of_var, (size_t)L.V * 4)))
        return rc;
    const uint64_t sc[] = {L.nf_sell, L.nf_big, L.nf_huge, L.nv_sell, L.nv_big, L.nv_huge, L.n_slots,
                           L.n_active_slots, L.n_ftiles, L.n_vtiles, L.n_fbtiles, L.n_vbtiles, (uint64_t)e->n_ent};
    bytes(sc, sizeof sc);
    *digest = h;
    if (built_on_device) *built_on_device = e->dev_layout ? 1 : 0;
    return FLBP_OK;
}

int flbp_last_run_ms(flbp_engine *e, double *ms) {
    if (!e || !ms) {
        set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    *ms = e->last_ms;
    return FLBP_OK;
}

// ------------------------------------------------------------------ batched solves

// Tolerance run of G independently stopping groups (graphs of a batched
// engine, or evidence sets): group g stops after the first sweep in which
// none of its beliefs moved by more than tol, or after maxiter sweeps.
static int run_groups_tol(flbp_engine *e, uint32_t G, double tol, int64_t maxiter, double maxtime, int64_t *sweeps,
                          int32_t *reasons, flbp_run_info *info) {
    int rc;
    const long long l0 = e->launches;
    FLBP_CUDA(cudaMemsetAsync(e->d_gstate, 0, 4 * sizeof(int) * G, e->stream));
    reset_ctl_for_run(e, 3);
    Ctl &c = *e->h_ctl;
    c.iters0 = 0;  // every group's sweep count starts at this call
    c.tol = tol;
    c.maxiter = maxiter;
    c.maxtime_ns = maxtime * 1e9;
    c.maxdiff = INFINITY;
    if ((rc = record_start(e))) return rc;
    long long done_sweeps = 0;
    if (maxiter > 0 && maxtime > 0.0) {
        if ((rc = upload_ctl(e)) || (rc = run_loop(e, 3, maxiter))) return rc;
        if ((rc = download_ctl(e))) return rc;
        done_sweeps = e->h_ctl->run_sweeps;
    }
    if ((rc = record_stop(e))) return rc;
    std::vector<int> st(4 * (size_t)G);
    FLBP_CUDA(cudaMemcpyAsync(st.data(), e->d_gstate, st.size() * sizeof(int), cudaMemcpyDeviceToHost, e->stream));
    FLBP_CUDA(cudaStreamSynchronize(e->stream));
    for (uint32_t g = 0; g < G; g++) {
        if (sweeps) sweeps[g] = st[2 * (size_t)G + g];
        if (reasons) reasons[g] = st[g] ? st[3 * (size_t)G + g] : FLBP_DIVERGED;
    }
    e->t += done_sweeps;
    e->iters += done_sweeps;
    fill_info(e, info, done_sweeps, l0);
    return FLBP_OK;
}

int flbp_batch_create(const flbp_graph_desc *graphs, int64_t n_graphs, const flbp_engine_opts *opts,
                      flbp_engine **out) {
    if (!graphs || !out || n_graphs <= 0) {
        set_error("batch needs at least one graph");
        return FLBP_ERR_INVALID;
    }
    *out = nullptr;
    int64_t V = 0, F = 0, E = 0;
    for (int64_t g = 0; g < n_graphs; g++) {
        const flbp_graph_desc &d = graphs[g];
        if (d.n_vars < 0 || d.n_factors < 0 || d.n_slots < 0 || (d.n_factors > 0 && !d.factor_offsets)) {
            set_error("graph " + std::to_string(g) + " of the batch is malformed");
            return FLBP_ERR_INVALID;
        }
        if (d.n_factors > 0 && (d.factor_offsets[0] != 0 || d.factor_offsets[d.n_factors] != d.n_slots)) {
            set_error("graph " + std::to_string(g) + ": factor_offsets must start at 0 and end at n_slots");
            return FLBP_ERR_INVALID;
        }
        if ((d.n_factors > 0 || d.n_slots > 0) &&
            (!d.slot_var || !d.factor_head || !d.factor_type || !d.factor_p || !d.factor_q)) {
            set_error("graph " + std::to_string(g) + " of the batch lacks an array");
            return FLBP_ERR_INVALID;
        }
        V += d.n_vars;
        F += d.n_factors;
        E += d.n_slots;
    }
    if (V >= (int64_t)UINT32_MAX || E >= (int64_t)UINT32_MAX || n_graphs >= (int64_t)INT32_MAX) {
        set_error("batch exceeds 2^32-1 variables or edge slots");
        return FLBP_ERR_LIMIT;
    }
    // the disjoint union, graphs in order
    std::vector<int64_t> off(F + 1, 0), sv(E), head(F);
    std::vector<int32_t> type(F), clamped(F, 0);
    std::vector<double> p(F), q(F), m0(F, 1.0), m1(F, 1.0);
    BatchSpec spec;
    spec.factor_graph.resize(F);
    spec.var_graph.resize(V);
    spec.var_off.assign(n_graphs + 1, 0);
    int64_t vo = 0, fo = 0, so = 0;
    for (int64_t g = 0; g < n_graphs; g++) {
        const flbp_graph_desc &d = graphs[g];
        for (int64_t I = 0; I < d.n_factors; I++) {
            off[fo + I + 1] = so + d.factor_offsets[I + 1];
            head[fo + I] = so + d.factor_head[I];
            type[fo + I] = d.factor_type[I];
            p[fo + I] = d.factor_p[I];
            q[fo + I] = d.factor_q[I];
            if (d.factor_head_clamped) clamped[fo + I] = d.factor_head_clamped[I];
            if (d.factor_mask0) m0[fo + I] = d.factor_mask0[I];
            if (d.factor_mask1) m1[fo + I] = d.factor_mask1[I];
            spec.factor_graph[fo + I] = (uint32_t)g;
        }
        for (int64_t e = 0; e < d.n_slots; e++) {
            if (d.slot_var[e] < 0 || d.slot_var[e] >= d.n_vars) {
                set_error("graph " + std::to_string(g) + ": slot_var out of range at slot " + std::to_string(e));
                return FLBP_ERR_INVALID;
            }
            sv[so + e] = vo + d.slot_var[e];
        }
        for (int64_t i = 0; i < d.n_vars; i++) spec.var_graph[vo + i] = (uint32_t)g;
        vo += d.n_vars;
        fo += d.n_factors;
        so += d.n_slots;
        spec.var_off[g + 1] = vo;
    }
    flbp_graph_desc u{V, F, E, off.data(), sv.data(), head.data(), type.data(), p.data(), q.data(),
                      clamped.data(), m0.data(), m1.data()};
    return create_engine(&u, opts, out, &spec);
}

int flbp_batch_info(flbp_engine *e, int64_t *n_graphs, int64_t *var_off) {
    int rc = begin_call(e);
    if (rc) return rc;
    if (n_graphs) *n_graphs = e->n_graphs;
    if (var_off)
        for (size_t g = 0; g < e->graph_var_off.size(); g++) var_off[g] = e->graph_var_off[g];
    return FLBP_OK;
}

int flbp_batch_run_tol(flbp_engine *e, double tol, int64_t maxiter, double maxtime, int64_t *sweeps, int32_t *reasons,
                       flbp_run_info *info) {
    int rc = begin_call(e);
    if (rc) return rc;
    if (e->n_graphs == 0) {
        set_error("not a batched engine (create it with flbp_batch_create)");
        return FLBP_ERR_INVALID;
    }
    return run_groups_tol(e, e->n_graphs, tol, maxiter, maxtime, sweeps, reasons, info);
}

}  // extern "C"

// ------------------------------------------------------------------ adjoint

namespace {

AdjArgs adj_args(flbp_engine *e) {
    AdjArgs a;
    a.fg_base = e->d_fg_base;
    a.fb_off = e->d_fb_off;
    a.fb_deg = e->d_fb_deg;
    a.f_pos = e->d_f_pos;
    a.f_kind = e->d_f_kind;
    a.f_deg = e->d_f_deg;
    a.f_pq = e->d_f_pq;
    a.nf_sell = e->L.nf_sell;
    a.nf_big = e->L.nf_big;
    a.vg_base = e->d_vg_base;
    a.vb_off = e->d_vb_off;
    a.vb_deg = e->d_vb_deg;
    a.v_ent = e->d_v_ent;
    a.prior = e->d_prior;
    a.nv_sell = e->L.nv_sell;
    a.nv_big = e->L.nv_big;
    return a;
}

unsigned int blocks_for(uint64_t threads, unsigned int per_block) {
    return (unsigned int)std::max<uint64_t>(1, (threads + per_block - 1) / per_block);
}

// One backward step: lam_next = dL/dvf_{t+1} -> lam = dL/dvf_t, with the
// parameter gradients of sweep t accumulated (dL/dq only with want_q).
template <typename T>
void launch_adjoint_step(flbp_engine *e, const void *vf, const void *fv, const void *lam_next, const void *gs,
                         void *lam, bool want_q) {
    const AdjArgs a = adj_args(e);
    T *mu = (T *)e->d_mu, *gp = (T *)e->d_gp, *gq = want_q ? (T *)e->d_gq : nullptr, *gprior = (T *)e->d_gprior;
    const uint32_t *gl = e->d_adj_groups;
    const uint32_t *c = e->adj_group_n;  // narrow var, wide var, narrow factor, wide factor groups
    const uint32_t o1 = c[0], o2 = o1 + c[1], o3 = o2 + c[2];
    int n = 0;
    auto go = [&](uint32_t cnt) { n += cnt ? 1 : 0; return cnt != 0; };
    if (go(c[0]))
        var_adjoint_kernel<T, false><<<blocks_for(32ull * c[0], 128), 128, 0, e->stream>>>(
            a, gl, c[0], (const T *)fv, (const T *)lam_next, (const T *)gs, mu, gprior);
    if (go(c[1]))
        var_adjoint_wide_kernel<T><<<(unsigned)((c[1] + 1) / 2), 128, 0, e->stream>>>(
            a, gl + o1, c[1], (const T *)fv, (const T *)lam_next, (const T *)gs, mu, gprior);
    if (go(a.nv_big))
        var_adjoint_big_kernel<T><<<blocks_for((uint64_t)kBigVarLanes * a.nv_big, 128), 128, 0, e->stream>>>(
            a, (const T *)fv, (const T *)lam_next, (const T *)gs, mu, gprior);
    if (go(c[2]))
        factor_adjoint_sell_kernel<T, false><<<blocks_for(32ull * c[2], 128), 128, 0, e->stream>>>(
            a, gl + o2, c[2], (const T *)vf, mu, (T *)lam, gp, gq);
    if (go(c[3]))
        factor_adjoint_sell_kernel<T, true><<<blocks_for(32ull * c[3], 128), 128, 0, e->stream>>>(
            a, gl + o3, c[3], (const T *)vf, mu, (T *)lam, gp, gq);
    if (go(a.nf_big))
        factor_adjoint_big_kernel<T><<<blocks_for(32ull * a.nf_big, 128), 128, 0, e->stream>>>(a, (const T *)vf, mu,
                                                                                                (T *)lam, gp, gq);
    e->launches += n;
}

// Undamped sweep halves on explicit message arrays (the recomputation of a
// segment writes each sweep's states straight into the segment buffers).
template <typename T>
void launch_factor_pass_on(flbp_engine *e, const void *vf, void *fv) {
    const FactorArgs fa = factor_args<T>(e);
    launch_factor<T>(e, fa, vf, fv);
    e->launches += 1;
}

template <typename T>
void launch_var_pass_on(flbp_engine *e, const void *fv, void *vf) {
    const VarArgs va = var_args(e);
    if (e->v_form)
        direct_var_launch<T>(e->v_form, 0, false, (unsigned)e->v_grid_direct, va, (const T *)fv, (T *)vf, nullptr,
                             (T)0, e->d_ctl, e->stream);
    else
        var_pass_kernel<T, 0, true, false, kStages><<<e->var_grid, kBlockThreads, var_smem<T, false>(), e->stream>>>(
            va, (const T *)fv, (T *)vf, nullptr, (T)0, e->d_ctl);
    e->launches += 1;
}

// State buffers of the checkpointed runs: checkpoint c (vf at sweep c K),
// and sweep i of the segment being differentiated (vf_i: the checkpoint for
// i = 0, else segment slot i; fv_i: segment slot i).
char *adj_ckpt(flbp_engine *e, long long c) {
    return (char *)e->d_ckpt + (size_t)c * std::max<uint64_t>(1, e->L.n_slots) * e->tsize;
}
char *adj_seg_vf(flbp_engine *e, long long c, long long i) {
    return i == 0 ? adj_ckpt(e, c) : (char *)e->d_seg_vf + (size_t)i * std::max<uint64_t>(1, e->L.n_slots) * e->tsize;
}
char *adj_seg_fv(flbp_engine *e, long long i) {
    return (char *)e->d_seg_fv + (size_t)i * std::max<size_t>(1, e->n_ent) * e->tsize;
}

// The checkpointed forward run on explicit buffers: each segment's sweeps
// start from its checkpoint, the last sweep of a segment writes the next
// checkpoint, and the last segment keeps every state in the segment buffers
// (its final variable pass writes the engine's vf, and fv_{T-1} is copied
// to the engine's fv, so the engine state is that of T plain sweeps).
template <typename T>
int adjoint_forward_t(flbp_engine *e, long long T_, long long K) {
    const size_t ns = std::max<uint64_t>(1, e->L.n_slots);
    const long long nck = (T_ + K - 1) / K;
    FLBP_CUDA(cudaMemcpyAsync(adj_ckpt(e, 0), e->d_vf, ns * e->tsize, cudaMemcpyDeviceToDevice,
                              e->stream));  // the state after init()
    for (long long c = 0; c < nck; c++) {
        const long long n1 = std::min<long long>(K, T_ - c * K);
        const bool last = c == nck - 1;
        for (long long i = 0; i < n1; i++) {
            const void *vin = i == 0 ? adj_ckpt(e, c) : (last ? adj_seg_vf(e, c, i) : e->d_vf);
            void *fout = last ? adj_seg_fv(e, i) : e->d_fv;
            void *vout = i + 1 < n1 ? (last ? adj_seg_vf(e, c, i + 1) : e->d_vf) : (last ? e->d_vf : adj_ckpt(e, c + 1));
            launch_factor_pass_on<T>(e, vin, fout);
            launch_var_pass_on<T>(e, fout, vout);
        }
        if (last && e->n_ent)
            FLBP_CUDA(cudaMemcpyAsync(e->d_fv, adj_seg_fv(e, n1 - 1), e->n_ent * e->tsize, cudaMemcpyDeviceToDevice,
                                      e->stream));
    }
    return FLBP_OK;
}

template <typename T>
void launch_adjoint_seed(flbp_engine *e, const double *grad_b) {
    const int64_t V = e->L.V;
    if (V)
        adjoint_seed_kernel<T><<<blocks_for(V, 256), 256, 0, e->stream>>>(grad_b, e->d_int_of_var, e->d_belief, V,
                                                                          (T *)e->d_gs);
    e->launches += V ? 1 : 0;
}

template <typename T>
void launch_adjoint_out(flbp_engine *e, double *gp_out, double *gq_out) {
    const uint32_t nf = e->L.nf_sell + e->L.nf_big, np = (uint32_t)e->L.prior_factor.size();
    if (nf)
        adjoint_factor_out_kernel<T><<<blocks_for(nf, 256), 256, 0, e->stream>>>(
            (const T *)e->d_gp, (const T *)e->d_gq, e->d_f_of_int, nf, gp_out, gq_out);
    if (np && gp_out)
        adjoint_prior_out_kernel<T><<<blocks_for(np, 256), 256, 0, e->stream>>>(
            (const T *)e->d_gprior, e->d_pri_fac, e->d_pri_var, e->d_pri_coef, np, gp_out);
    e->launches += (nf ? 1 : 0) + ((np && gp_out) ? 1 : 0);
}

// Device maps between the caller's order and the internal one, and the
// coefficients of the folded constants, for the adjoint (built on first use;
// the coefficients again after flbp_set_factor_probs).
int ensure_adjoint_maps(flbp_engine *e) {
    if (int rc0 = ensure_host_layout(e)) return rc0;
    int rc;
    const HostLayout &L = e->L;
    if (!e->d_adj_groups) {
        // sliced-ELL groups by width class: narrow var, wide var, narrow factor, wide factor
        std::vector<uint32_t> lists[4];
        for (uint32_t g = 0; g < L.n_vgroups(); g++)
            lists[(L.vg_base[g + 1] - L.vg_base[g]) / 32 > kNarrowWidth ? 1 : 0].push_back(g);
        for (uint32_t g = 0; g < L.n_fgroups(); g++)
            lists[(L.fg_base[g + 1] - L.fg_base[g]) / 32 > kNarrowWidth ? 3 : 2].push_back(g);
        std::vector<uint32_t> all;
        for (int k = 0; k < 4; k++) {
            e->adj_group_n[k] = (uint32_t)lists[k].size();
            all.insert(all.end(), lists[k].begin(), lists[k].end());
        }
        if ((rc = dalloc(e, &e->d_adj_groups, all.size())) || (rc = upload(e, e->d_adj_groups, all))) return rc;
        const uint32_t nf = L.nf_sell + L.nf_big;
        std::vector<uint32_t> foi(L.factor_of_internal.begin(), L.factor_of_internal.begin() + nf);
        if ((rc = dalloc(e, &e->d_f_of_int, foi.size())) || (rc = upload(e, e->d_f_of_int, foi)) ||
            (rc = dalloc(e, &e->d_pri_fac, L.prior_factor.size())) || (rc = upload(e, e->d_pri_fac, L.prior_factor)) ||
            (rc = dalloc(e, &e->d_pri_var, L.prior_var.size())) || (rc = upload(e, e->d_pri_var, L.prior_var)) ||
            (rc = dalloc(e, &e->d_pri_coef, L.prior_factor.size())))
            return rc;
        e->pri_coef_valid = false;
    }
    if (!e->pri_coef_valid) {
        std::vector<double> coef(L.prior_factor.size(), 0.0);
        for (size_t k = 0; k < coef.size(); k++) {
            const double p = e->factor_p_host[L.prior_factor[k]];
            if (p > 0.0 && p < 1.0) coef[k] = L.prior_sign[k] / (p * (1.0 - p));
        }
        if ((rc = upload(e, e->d_pri_coef, coef))) return rc;
        e->pri_coef_valid = true;
    }
    return FLBP_OK;
}

// The backward pass on device buffers in the caller's orders: dL/dbeliefs
// in, dL/dp and dL/dq out (either may be null). Leaves the work queued on
// the engine's stream.
template <typename T>
int adjoint_backward_t(flbp_engine *e, const double *grad_b, double *gp_out, double *gq_out) {
    int rc;
    const HostLayout &L = e->L;
    const size_t ts = sizeof(T);
    const size_t ns = std::max<uint64_t>(1, L.n_slots), ne = std::max<size_t>(1, e->n_ent);
    const size_t nv = std::max<int64_t>(1, L.V), nf = std::max<size_t>(1, (size_t)L.nf_sell + L.nf_big);
    if ((rc = ensure_adjoint_maps(e))) return rc;
    if (!e->d_lam && ((rc = dalloc(e, (char **)&e->d_lam, ne * ts)) || (rc = dalloc(e, (char **)&e->d_lam2, ne * ts)) ||
                      (rc = dalloc(e, (char **)&e->d_mu, ns * ts)) || (rc = dalloc(e, (char **)&e->d_gp, nf * ts)) ||
                      (rc = dalloc(e, (char **)&e->d_gq, nf * ts)) ||
                      (rc = dalloc(e, (char **)&e->d_gprior, nv * ts)) || (rc = dalloc(e, (char **)&e->d_gs, nv * ts))))
        return rc;
    FLBP_CUDA(cudaMemsetAsync(e->d_gp, 0, nf * ts, e->stream));
    if (gq_out) FLBP_CUDA(cudaMemsetAsync(e->d_gq, 0, nf * ts, e->stream));
    FLBP_CUDA(cudaMemsetAsync(e->d_gprior, 0, nv * ts, e->stream));
    FLBP_CUDA(cudaMemsetAsync(e->d_lam, 0, ne * ts, e->stream));
    FLBP_CUDA(cudaMemsetAsync(e->d_lam2, 0, ne * ts, e->stream));
    FLBP_CUDA(cudaMemsetAsync(e->d_mu, 0, ns * ts, e->stream));
    launch_adjoint_seed<T>(e, grad_b);
    reset_ctl_for_run(e, 0);
    if ((rc = upload_ctl(e))) return rc;
    const long long T_ = e->adj_t, K = e->adj_k;
    const long long nck = (T_ + K - 1) / K;
    void *lam_next = e->d_lam, *lam_cur = e->d_lam2;
    for (long long c = nck - 1; c >= 0; c--) {
        const long long t0 = c * K, n1 = std::min<long long>(K, T_ - t0);
        // the segment's states: vf_i = adj_seg_vf(c, i), fv_i in seg_fv(i), recomputed
        // from the checkpoint unless the forward run left them (last segment)
        if (!(c == nck - 1 && e->adj_last_seg)) {
            for (long long i = 0; i < n1; i++) {
                launch_factor_pass_on<T>(e, adj_seg_vf(e, c, i), adj_seg_fv(e, i));
                if (i + 1 < n1) launch_var_pass_on<T>(e, adj_seg_fv(e, i), adj_seg_vf(e, c, i + 1));
            }
        }
        e->adj_last_seg = false;  // the segment buffers are reused from here on
        for (long long i = n1 - 1; i >= 0; i--) {
            const void *gsp = (t0 + i == T_ - 1) ? e->d_gs : nullptr;
            launch_adjoint_step<T>(e, adj_seg_vf(e, c, i), adj_seg_fv(e, i), lam_next, gsp, lam_cur,
                                   gq_out != nullptr);
            std::swap(lam_next, lam_cur);
        }
    }
    launch_adjoint_out<T>(e, gp_out, gq_out);
    FLBP_CUDA(cudaGetLastError());
    return download_ctl(e);  // synchronises; reports a timed-out pass
}

int adjoint_backward_dev(flbp_engine *e, const double *grad_b, double *gp_out, double *gq_out) {
    if (e->adj_t == 0) {
        set_error("no adjoint forward run to differentiate (call flbp_adjoint_forward first)");
        return FLBP_ERR_INVALID;
    }
    if (e->L.F) {
        if (gp_out) FLBP_CUDA(cudaMemsetAsync(gp_out, 0, (size_t)e->L.F * sizeof(double), e->stream));
        if (gq_out) FLBP_CUDA(cudaMemsetAsync(gq_out, 0, (size_t)e->L.F * sizeof(double), e->stream));
    }
    if (e->prec == 64) return adjoint_backward_t<double>(e, grad_b, gp_out, gq_out);
    return adjoint_backward_t<float>(e, grad_b, gp_out, gq_out);
}

}  // namespace

namespace {

// The host copies of new factor probabilities (reference factor order): the
// factors' (p, q) in the internal order and in the big-tile copies, and the
// finite prior constants of the folded singletons, summed in prior-entry
// order.
void apply_probs_host(flbp_engine *e, const double *p, const double *q) {
    HostLayout &L = e->L;
    e->factor_p_host.assign(p, p + L.F);
    e->factor_q_host.assign(q, q + L.F);
    const uint32_t nf = L.nf_sell + L.nf_big;
    for (uint32_t f = 0; f < nf; f++) {
        L.f_pq[2 * f] = p[L.factor_of_internal[f]];
        L.f_pq[2 * f + 1] = q[L.factor_of_internal[f]];
    }
    for (uint32_t t = 0; t < L.n_fbtiles; t++) {
        const uint32_t *h = &L.fhdr[(size_t)kHdrWordsHost * t];
        for (uint32_t j = 0; j < (h[1] & ~kBigTileFlag); j++) {
            const size_t k = (size_t)kTileGroupsHost * t + j, fi = (size_t)L.nf_sell + h[0] + j;
            L.fbt_pq[2 * k] = L.f_pq[2 * fi];
            L.fbt_pq[2 * k + 1] = L.f_pq[2 * fi + 1];
        }
    }
    std::fill(L.prior_fin.begin(), L.prior_fin.end(), 0.0);
    for (size_t k = 0; k < L.prior_factor.size(); k++) {
        const double pk = p[L.prior_factor[k]];
        L.prior_fin[L.prior_var[k]] += L.prior_sign[k] * det_logit(pk);
    }
    e->host_probs_stale = false;
}

// Brings the host copies up to the probabilities last given on the device.
int sync_host_probs(flbp_engine *e) {
    if (!e->host_probs_stale) return FLBP_OK;
    const size_t F = (size_t)e->L.F;
    std::vector<double> p(F), q(F);
    FLBP_CUDA(cudaMemcpyAsync(p.data(), e->d_p_keep, F * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    FLBP_CUDA(cudaMemcpyAsync(q.data(), e->d_q_keep, F * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    FLBP_CUDA(cudaStreamSynchronize(e->stream));
    apply_probs_host(e, p.data(), q.data());
    return FLBP_OK;
}

// The maps of flbp_set_factor_probs_device, built once per engine.
int ensure_prob_maps(flbp_engine *e) {
    if (e->probs_maps) return FLBP_OK;
    int rc;
    if ((rc = ensure_adjoint_maps(e))) return rc;  // internal factor -> caller factor, prior entries
    const HostLayout &L = e->L;
    std::vector<uint32_t> fbt_src(std::max<size_t>(1, L.fbt_pq.size() / 2), UINT32_MAX);
    for (uint32_t t = 0; t < L.n_fbtiles; t++) {
        const uint32_t *h = &L.fhdr[(size_t)kHdrWordsHost * t];
        for (uint32_t j = 0; j < (h[1] & ~kBigTileFlag); j++) fbt_src[(size_t)kTileGroupsHost * t + j] = L.nf_sell + h[0] + j;
    }
    std::vector<uint32_t> vbt_src(std::max<size_t>(1, L.vbt_deg.size()), UINT32_MAX);
    for (uint32_t t = 0; t < L.n_vbtiles; t++) {
        const uint32_t *h = &L.vhdr[(size_t)kHdrWordsHost * t];
        for (uint32_t j = 0; j < (h[1] & ~kBigTileFlag); j++) vbt_src[(size_t)kTileGroupsHost * t + j] = L.nv_sell + h[0] + j;
    }
    // prior entries grouped by variable, in entry order within a variable
    const size_t np = L.prior_var.size();
    std::vector<uint32_t> ord(std::max<size_t>(1, np), 0), uvar, uoff;
    std::iota(ord.begin(), ord.begin() + np, 0u);
    std::stable_sort(ord.begin(), ord.begin() + np, [&](uint32_t a, uint32_t b) { return L.prior_var[a] < L.prior_var[b]; });
    for (size_t i = 0; i < np; i++)
        if (i == 0 || L.prior_var[ord[i]] != L.prior_var[ord[i - 1]]) {
            uvar.push_back(L.prior_var[ord[i]]);
            uoff.push_back((uint32_t)i);
        }
    uoff.push_back((uint32_t)np);
    if (uvar.empty()) uvar.push_back(0);
    std::vector<double> sign(std::max<size_t>(1, np), 0.0);
    for (size_t k = 0; k < np; k++) sign[k] = L.prior_sign[k];
    if ((rc = dalloc(e, &e->d_fbt_src, fbt_src.size())) || (rc = upload(e, e->d_fbt_src, fbt_src)) ||
        (rc = dalloc(e, &e->d_vbt_src, vbt_src.size())) || (rc = upload(e, e->d_vbt_src, vbt_src)) ||
        (rc = dalloc(e, &e->d_pri_ord, ord.size())) || (rc = upload(e, e->d_pri_ord, ord)) ||
        (rc = dalloc(e, &e->d_pri_uvar, uvar.size())) || (rc = upload(e, e->d_pri_uvar, uvar)) ||
        (rc = dalloc(e, &e->d_pri_uoff, uoff.size())) || (rc = upload(e, e->d_pri_uoff, uoff)) ||
        (rc = dalloc(e, &e->d_pri_sign, sign.size())) || (rc = upload(e, e->d_pri_sign, sign)) ||
        (rc = dalloc(e, &e->d_p_keep, (size_t)L.F)) || (rc = dalloc(e, &e->d_q_keep, (size_t)L.F)) ||
        (rc = dalloc(e, &e->d_bad, 1)))
        return rc;
    e->n_pri_uvar = np ? (uint32_t)(uoff.size() - 1) : 0u;
    e->probs_maps = true;
    return FLBP_OK;
}

// The first factor (reference order) whose p or q lies outside [0, 1] (NaN included).
__global__ void probs_check_kernel(const double *__restrict__ p, const double *__restrict__ q, int64_t F,
                                   unsigned long long *bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < F; i += (int64_t)gridDim.x * blockDim.x) {
        const double a = p[i], b = q[i];
        if (!(a >= 0.0 && a <= 1.0) || !(b >= 0.0 && b <= 1.0)) atomicMin(bad, (unsigned long long)i);
    }
}

// (p, q) of every internal factor and of every big-tile copy, in the message type.
template <typename T>
__global__ void probs_pq_kernel(const double *__restrict__ p, const double *__restrict__ q,
                                const uint32_t *__restrict__ f_of_int, uint32_t nf, T *f_pq,
                                const uint32_t *__restrict__ fbt_src, uint32_t n_fbt, T *fbt_pq) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < max(nf, n_fbt); i += gridDim.x * blockDim.x) {
        if (i < nf) {
            const uint32_t I = f_of_int[i];
            f_pq[2 * i] = (T)p[I];
            f_pq[2 * i + 1] = (T)q[I];
        }
        if (i < n_fbt && fbt_src[i] != UINT32_MAX) {
            const uint32_t I = f_of_int[fbt_src[i]];
            fbt_pq[2 * i] = (T)p[I];
            fbt_pq[2 * i + 1] = (T)q[I];
        }
    }
}

// Finite prior constants of the folded singletons (the sum over a variable's
// prior entries of sign det_logit(p), in entry order) into the
// engine's prior words, and each entry's d(constant)/dp for the adjoint.
template <typename T>
__global__ void probs_prior_kernel(const double *__restrict__ p, const uint32_t *__restrict__ uvar,
                                   const uint32_t *__restrict__ uoff, uint32_t n_uvar, const uint32_t *__restrict__ ord,
                                   const uint32_t *__restrict__ pri_fac, const double *__restrict__ sign, uint32_t np,
                                   double *coef, uint32_t *prior_words) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < max(n_uvar, np); i += gridDim.x * blockDim.x) {
        if (i < n_uvar) {
            double s = 0.0;
            for (uint32_t j = uoff[i]; j < uoff[i + 1]; j++) {
                const uint32_t k = ord[j];
                const double pk = p[pri_fac[k]];
                s += sign[k] * det_logit(pk);
            }
            const uint32_t v = uvar[i];
            if (sizeof(T) == 8) {
                *reinterpret_cast<double *>(prior_words + 4 * (size_t)v) = s;
            } else {
                *reinterpret_cast<float *>(prior_words + 2 * (size_t)v) = (float)s;
            }
        }
        if (i < np) {
            const double pk = p[pri_fac[i]];
            coef[i] = (pk > 0.0 && pk < 1.0) ? sign[i] / (pk * (1.0 - pk)) : 0.0;
        }
    }
}

// The big-tile copies of the priors (pw words each).
__global__ void probs_bt_prior_kernel(const uint32_t *__restrict__ src, uint32_t n, uint32_t pw,
                                      const uint32_t *__restrict__ prior_words, uint32_t *bt_prior_words) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t v = src[i];
        if (v == UINT32_MAX) continue;
        for (uint32_t w = 0; w < pw; w++) bt_prior_words[(size_t)pw * i + w] = prior_words[(size_t)pw * v + w];
    }
}

}  // namespace

extern "C" {

int flbp_adjoint_forward(flbp_engine *e, int64_t sweeps, int64_t every, double *beliefs, int64_t n) {
    int rc = begin_call(e);
    if (rc || (rc = refuse_sets(e, "the adjoint")) || (rc = refuse_seq(e, "the adjoint")) || (rc = ensure_host_layout(e))) return rc;
    if (e->damping != 0.0) {
        set_error("the adjoint needs an engine without damping");
        return FLBP_ERR_INVALID;
    }
    if (sweeps < 1 || every < 1) {
        set_error("sweeps and checkpoint interval must be positive");
        return FLBP_ERR_INVALID;
    }
    if (beliefs && n != e->L.V) {
        set_error("output length must equal the number of variables");
        return FLBP_ERR_INVALID;
    }
    const size_t ns = std::max<uint64_t>(1, e->L.n_slots), ne = std::max<size_t>(1, e->n_ent);
    const size_t nck = (size_t)((sweeps + every - 1) / every);
    const size_t nseg = (size_t)std::min<int64_t>(every, sweeps);
    if (nck > e->adj_ckpt_n) {
        dfree(e, e->d_ckpt);
        e->d_ckpt = nullptr;
        e->adj_ckpt_n = 0;
        if ((rc = dalloc(e, (char **)&e->d_ckpt, nck * ns * e->tsize))) return rc;
        e->adj_ckpt_n = nck;
    }
    if (nseg > e->adj_seg_n) {
        dfree(e, e->d_seg_vf);
        dfree(e, e->d_seg_fv);
        e->d_seg_vf = e->d_seg_fv = nullptr;
        e->adj_seg_n = 0;
        if ((rc = dalloc(e, (char **)&e->d_seg_vf, nseg * ns * e->tsize)) ||
            (rc = dalloc(e, (char **)&e->d_seg_fv, nseg * ne * e->tsize)))
            return rc;
        // positions that no pass writes (padding) keep the value init() gives the
        // engine's own arrays, zero; the segment recomputation writes the rest
        FLBP_CUDA(cudaMemsetAsync(e->d_seg_vf, 0, nseg * ns * e->tsize, e->stream));
        FLBP_CUDA(cudaMemsetAsync(e->d_seg_fv, 0, nseg * ne * e->tsize, e->stream));
        e->adj_seg_n = nseg;
    }
    if ((rc = flbp_init(e))) return rc;
    e->adj_t = 0;
    e->adj_last_seg = false;
    reset_ctl_for_run(e, 0);
    if ((rc = upload_ctl(e))) return rc;
    if ((rc = e->prec == 64 ? adjoint_forward_t<double>(e, sweeps, every) : adjoint_forward_t<float>(e, sweeps, every)))
        return rc;
    launch_beliefs_only(e, e->d_belief);
    if ((rc = download_ctl(e))) return rc;
    e->t += sweeps;
    e->iters += sweeps;
    e->adj_t = sweeps;
    e->adj_k = every;
    e->adj_last_seg = true;
    if (beliefs) return fetch_internal(e, e->d_belief, beliefs, n);
    return FLBP_OK;
}

int flbp_adjoint_backward(flbp_engine *e, const double *grad_beliefs, double *grad_p, double *grad_q) {
    int rc = begin_call(e);
    if (rc || (rc = refuse_sets(e, "the adjoint")) || (rc = refuse_seq(e, "the adjoint")) || (rc = ensure_host_layout(e))) return rc;
    const HostLayout &L = e->L;
    const size_t nv = std::max<int64_t>(1, L.V), nF = std::max<int64_t>(1, L.F);
    if (!e->d_adj_in && ((rc = dalloc(e, &e->d_adj_in, nv)) || (rc = dalloc(e, &e->d_adj_out, 2 * nF)))) return rc;
    if (L.V) {
        if (grad_beliefs)
            FLBP_CUDA(cudaMemcpyAsync(e->d_adj_in, grad_beliefs, (size_t)L.V * sizeof(double), cudaMemcpyHostToDevice,
                                      e->stream));
        else
            FLBP_CUDA(cudaMemsetAsync(e->d_adj_in, 0, (size_t)L.V * sizeof(double), e->stream));
    }
    if ((rc = adjoint_backward_dev(e, e->d_adj_in, e->d_adj_out, e->d_adj_out + nF))) return rc;
    if (L.F) {
        if (grad_p)
            FLBP_CUDA(cudaMemcpyAsync(grad_p, e->d_adj_out, (size_t)L.F * sizeof(double), cudaMemcpyDeviceToHost,
                                      e->stream));
        if (grad_q)
            FLBP_CUDA(cudaMemcpyAsync(grad_q, e->d_adj_out + nF, (size_t)L.F * sizeof(double), cudaMemcpyDeviceToHost,
                                      e->stream));
    }
    FLBP_CUDA(cudaStreamSynchronize(e->stream));
    return FLBP_OK;
}

int flbp_adjoint_backward_device(flbp_engine *e, const double *grad_beliefs, double *grad_p, double *grad_q) {
    int rc = begin_call(e);
    if (rc || (rc = refuse_sets(e, "the adjoint")) || (rc = refuse_seq(e, "the adjoint")) || (rc = ensure_host_layout(e))) return rc;
    if (!grad_beliefs && e->L.V) {
        set_error("grad_beliefs is required");
        return FLBP_ERR_INVALID;
    }
    return adjoint_backward_dev(e, grad_beliefs, grad_p, grad_q);
}

int flbp_get_beliefs_device(flbp_engine *e, double *out, int64_t n) {
    int rc = begin_call(e);
    if (rc || (rc = refuse_sets(e, "flbp_get_beliefs_device"))) return rc;
    if (n != e->L.V) {
        set_error("output length must equal the number of variables");
        return FLBP_ERR_INVALID;
    }
    if (!e->d_int_of_var && (rc = ensure_adjoint_maps(e))) return rc;
    if (n) {
        gather_vars_kernel<<<blocks_for(n, 256), 256, 0, e->stream>>>(e->d_belief, e->d_int_of_var, n, out);
        e->launches += 1;
    }
    FLBP_CUDA(cudaGetLastError());
    FLBP_CUDA(cudaStreamSynchronize(e->stream));
    return FLBP_OK;
}

int flbp_set_factor_probs(flbp_engine *e, const double *p, const double *q) {
    int rc = begin_call(e);
    if (rc || (rc = refuse_sets(e, "flbp_set_factor_probs")) || (rc = refuse_seq(e, "flbp_set_factor_probs")) ||
        (rc = ensure_host_layout(e)))
        return rc;
    HostLayout &L = e->L;
    if (L.F > 0 && (!p || !q)) {
        set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    for (int64_t I = 0; I < L.F; I++) {
        if (!(p[I] >= 0.0 && p[I] <= 1.0) || !(q[I] >= 0.0 && q[I] <= 1.0)) {
            set_error("factor probabilities must lie in [0,1] (factor " + std::to_string(I) + ")");
            return FLBP_ERR_INVALID;
        }
    }
    apply_probs_host(e, p, q);
    e->pri_coef_valid = false;
    const uint32_t nf = L.nf_sell + L.nf_big;
    const size_t nf_pad = std::max<size_t>(nf, 32ull * L.n_fgroups());
    const size_t nv_pad = std::max<size_t>((size_t)L.V, 32ull * L.n_vgroups());
    std::vector<double> pq64(2 * nf_pad, 0.0);
    std::copy(L.f_pq.begin(), L.f_pq.end(), pq64.begin());
    if (e->prec == 64) {
        if ((rc = upload(e, (double *)e->d_f_pq, pq64)) || (rc = upload(e, (double *)e->d_fbt_pq, L.fbt_pq))) return rc;
    } else {
        std::vector<float> a(pq64.begin(), pq64.end()), b(L.fbt_pq.begin(), L.fbt_pq.end());
        if ((rc = upload(e, (float *)e->d_f_pq, a)) || (rc = upload(e, (float *)e->d_fbt_pq, b))) return rc;
    }
    std::vector<uint32_t> prior, bt_prior;
    packed_priors(e, nv_pad, prior, bt_prior);
    if ((rc = upload(e, (uint32_t *)e->d_prior, prior)) || (rc = upload(e, (uint32_t *)e->d_vbt_prior, bt_prior)))
        return rc;
    FLBP_CUDA(cudaStreamSynchronize(e->stream));
    return FLBP_OK;
}

int flbp_set_factor_probs_device(flbp_engine *e, const double *p, const double *q) {
    int rc = begin_call(e);
    if (rc || (rc = refuse_sets(e, "flbp_set_factor_probs_device")) ||
        (rc = refuse_seq(e, "flbp_set_factor_probs_device")) || (rc = ensure_host_layout(e)))
        return rc;
    const HostLayout &L = e->L;
    if (L.F == 0) return FLBP_OK;
    if (!p || !q) {
        set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    if ((rc = ensure_prob_maps(e))) return rc;
    // the range check first: a bad value leaves the engine as it was
    const unsigned gF = (unsigned)std::min<int64_t>((L.F + 255) / 256, 8192);
    FLBP_CUDA(cudaMemsetAsync(e->d_bad, 0xff, sizeof(unsigned long long), e->stream));
    probs_check_kernel<<<gF, 256, 0, e->stream>>>(p, q, L.F, e->d_bad);
    FLBP_CUDA(cudaGetLastError());
    unsigned long long bad = 0;
    FLBP_CUDA(cudaMemcpyAsync(&bad, e->d_bad, sizeof bad, cudaMemcpyDeviceToHost, e->stream));
    FLBP_CUDA(cudaStreamSynchronize(e->stream));
    if (bad != ~0ull) {
        set_error("factor probabilities must lie in [0,1] (factor " + std::to_string(bad) + ")");
        return FLBP_ERR_INVALID;
    }
    FLBP_CUDA(cudaMemcpyAsync(e->d_p_keep, p, (size_t)L.F * sizeof(double), cudaMemcpyDeviceToDevice, e->stream));
    FLBP_CUDA(cudaMemcpyAsync(e->d_q_keep, q, (size_t)L.F * sizeof(double), cudaMemcpyDeviceToDevice, e->stream));
    const uint32_t nf = L.nf_sell + L.nf_big, n_fbt = (uint32_t)(L.fbt_pq.size() / 2);
    const uint32_t n_vbt = (uint32_t)L.vbt_deg.size();
    auto blocks = [](uint64_t n) { return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 8192)); };
    const uint32_t pw = e->prec == 64 ? 4 : 2;
    if (e->prec == 64) {
        probs_pq_kernel<double><<<blocks(std::max(nf, n_fbt)), 256, 0, e->stream>>>(
            e->d_p_keep, e->d_q_keep, e->d_f_of_int, nf, (double *)e->d_f_pq, e->d_fbt_src, n_fbt, (double *)e->d_fbt_pq);
        probs_prior_kernel<double><<<blocks(std::max<uint64_t>(e->n_pri_uvar, L.prior_var.size())), 256, 0, e->stream>>>(
            e->d_p_keep, e->d_pri_uvar, e->d_pri_uoff, e->n_pri_uvar, e->d_pri_ord, e->d_pri_fac, e->d_pri_sign,
            (uint32_t)L.prior_var.size(), e->d_pri_coef, (uint32_t *)e->d_prior);
    } else {
        probs_pq_kernel<float><<<blocks(std::max(nf, n_fbt)), 256, 0, e->stream>>>(
            e->d_p_keep, e->d_q_keep, e->d_f_of_int, nf, (float *)e->d_f_pq, e->d_fbt_src, n_fbt, (float *)e->d_fbt_pq);
        probs_prior_kernel<float><<<blocks(std::max<uint64_t>(e->n_pri_uvar, L.prior_var.size())), 256, 0, e->stream>>>(
            e->d_p_keep, e->d_pri_uvar, e->d_pri_uoff, e->n_pri_uvar, e->d_pri_ord, e->d_pri_fac, e->d_pri_sign,
            (uint32_t)L.prior_var.size(), e->d_pri_coef, (uint32_t *)e->d_prior);
    }
    if (n_vbt)
        probs_bt_prior_kernel<<<blocks(n_vbt), 256, 0, e->stream>>>(e->d_vbt_src, n_vbt, pw, (const uint32_t *)e->d_prior,
                                                                     (uint32_t *)e->d_vbt_prior);
    e->launches += 3 + (n_vbt ? 1 : 0);
    FLBP_CUDA(cudaGetLastError());
    e->pri_coef_valid = true;
    e->host_probs_stale = true;
    return FLBP_OK;
}

}  // extern "C"

// ------------------------------------------------------ incremental clamping

namespace {

// Applies a clamp batch: zero the listed f->v entries (and their damped
// copies), mark the listed slots as sending to no entry, and write the
// listed prior count words (engine priors and big-tile copies).
template <typename T>
__global__ void clamp_apply_kernel(const uint32_t *__restrict__ ents, uint32_t n_e, const uint32_t *__restrict__ pw,
                                   uint32_t n_p, const uint32_t *__restrict__ bw, uint32_t n_b, T *fv, T *fvd,
                                   uint32_t *f_pos, uint32_t *prior_words, uint32_t *bt_prior_words) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_e) {
        fv[ents[2 * i]] = T(0);
        if (fvd) fvd[ents[2 * i]] = T(0);
        f_pos[ents[2 * i + 1]] = kSentinel;
    }
    if (i < n_p) prior_words[pw[2 * i]] = pw[2 * i + 1];
    if (i < n_b) bt_prior_words[bw[2 * i]] = bw[2 * i + 1];
}

// The changes a set of clamps makes to an engine (flbp_clamp_vars), from
// the layout L as it is and the variables' current clamp states: the
// entries no message reaches any more ((entry, slot) pairs), the new prior
// count words ((word, value) pairs, engine priors and big-tile copies), the
// (slot, value) pairs of the clamped variables' v->f messages (appended to
// `slots`), and the host-side updates.
struct ClampPlan {
    std::vector<uint32_t> ents, pw, bw, cut_slots, slots;
    std::vector<std::pair<int64_t, int8_t>> new_state;
    std::vector<std::pair<uint32_t, uint32_t>> new_cnt;  // (internal variable, count word)
};

// Checks a clamp list against the current states; "" when valid.
std::string check_clamps(const HostLayout &L, const std::vector<int8_t> &state, int64_t n, const int64_t *vars,
                         const int32_t *values) {
    if (n < 0 || (n > 0 && (!vars || !values))) return "clamp list is malformed";
    for (int64_t k = 0; k < n; k++) {
        if (vars[k] < 0 || vars[k] >= L.V) return "clamped variable out of range: " + std::to_string(vars[k]);
        if (values[k] != 0 && values[k] != 1)
            return "clamp value must be 0 or 1 (variable " + std::to_string(vars[k]) + ")";
        const int8_t st = state[vars[k]];
        if (st >= 0 && st != values[k])
            return "variable " + std::to_string(vars[k]) + " is already clamped to the other value";
        for (int64_t j = 0; j < k; j++)
            if (vars[j] == vars[k] && values[j] != values[k])
                return "variable " + std::to_string(vars[k]) + " is clamped to both values";
    }
    return "";
}

void clamp_plan(const HostLayout &L, int prec, const std::vector<int8_t> &state, int64_t n, const int64_t *vars,
                const int32_t *values, ClampPlan &P) {
    std::vector<uint8_t> folded((size_t)L.V, 0);
    for (uint32_t v : L.prior_var) folded[v] = 1;
    const size_t pwords = prec == 64 ? 4 : 2, cword = prec == 64 ? 2 : 1;
    std::vector<uint32_t> &ents = P.ents, &pw = P.pw, &bw = P.bw, &cut_slots = P.cut_slots, &slots = P.slots;
    std::unordered_set<int64_t> in_call;
    std::unordered_set<uint32_t> cut_now;
    for (int64_t k = 0; k < n; k++) {
        // clamping again to the same value changes nothing
        if (state[vars[k]] >= 0 || !in_call.insert(vars[k]).second) continue;
        P.new_state.push_back({vars[k], (int8_t)values[k]});
        const uint32_t iv = L.internal_of_var[vars[k]];
        // the clamp: one exact-zero count in the variable's prior
        uint32_t cnt = L.prior_cnt[iv];
        if (values[k]) {
            if ((cnt & 0xffffu) != 0xffffu) cnt += 1u;
        } else if (((cnt >> 16) & 0x7fffu) != 0x7fffu) {
            cnt += 1u << 16;
        }
        P.new_cnt.push_back({iv, cnt});
        const uint32_t word = cnt | (folded[iv] ? 0x80000000u : 0u);
        pw.push_back((uint32_t)(pwords * iv + cword));
        pw.push_back(word);
        // its entries: no factor's message reaches it any more; its v->f
        // messages are +-inf from init() on (it leaves every body it is in);
        // a factor it kills (0 in an AND body, 1 in an OR body) leaves its
        // other body variables too
        auto cut = [&](uint32_t sl) {  // no message from slot sl any more
            const uint32_t en = L.f_pos[sl];
            if (en == kSentinel || !cut_now.insert(sl).second) return;
            ents.push_back(en);
            ents.push_back(sl);
            cut_slots.push_back(sl);
        };
        auto entry = [&](uint32_t en) {
            const uint32_t sl = L.v_ent[en];
            if (sl == kSentinel) return;
            cut(sl);
            slots.push_back(sl);
            slots.push_back((uint32_t)values[k]);
            // the factor of slot sl, and sl's position in it (0 = head)
            uint32_t f, pos, base, stride, deg;
            if (sl < L.fg_base.back()) {
                const uint32_t g = (uint32_t)(std::upper_bound(L.fg_base.begin(), L.fg_base.end(), sl) - L.fg_base.begin()) - 1;
                const uint32_t off = sl - L.fg_base[g];
                f = 32u * g + off % 32u;
                pos = off / 32u;
                base = L.fg_base[g] + off % 32u;
                stride = 32;
                deg = L.f_deg[f];
            } else {
                const uint32_t b = (uint32_t)(std::upper_bound(L.fb_off.begin(), L.fb_off.end(), sl) - L.fb_off.begin()) - 1;
                f = L.nf_sell + b;
                pos = sl - L.fb_off[b];
                base = L.fb_off[b];
                stride = 1;
                deg = L.fb_deg[b];
            }
            const bool is_or = L.f_kind[f] & KIND_OR;
            if (pos > 0 && ((values[k] == 0 && !is_or) || (values[k] == 1 && is_or)))
                for (uint32_t j = 1; j < deg; j++)
                    if (j != pos) cut(base + stride * j);
        };
        if (iv < L.nv_sell) {
            const uint32_t g = iv / 32, lane = iv % 32, w = (L.vg_base[g + 1] - L.vg_base[g]) / 32;
            for (uint32_t j = 0; j < w; j++) entry(L.vg_base[g] + 32u * j + lane);
        } else {
            const uint32_t b = iv - L.nv_sell;
            for (uint32_t j = 0; j < L.vb_deg[b]; j++) entry(L.vb_off[b] + j);
            for (uint32_t t = 0; t < L.n_vbtiles; t++) {  // the big-tile copy of its prior
                const uint32_t *h = &L.vhdr[(size_t)kHdrWordsHost * t];
                const uint32_t b0 = h[0], nb = h[1] & ~kBigTileFlag;
                if (b >= b0 && b < b0 + nb) {
                    bw.push_back((uint32_t)(pwords * ((size_t)kTileGroupsHost * t + (b - b0)) + cword));
                    bw.push_back(word);
                    break;
                }
            }
        }
    }
}

}  // namespace

extern "C" {

int flbp_clamp_vars(flbp_engine *e, int64_t n, const int64_t *vars, const int32_t *values) {
    int rc = begin_call(e);
    if (rc || (rc = refuse_seq(e, "flbp_clamp_vars")) || (rc = refuse_sets(e, "flbp_clamp_vars")) ||
        (rc = ensure_host_layout(e)))
        return rc;
    HostLayout &L = e->L;
    if (n < 0 || (n > 0 && (!vars || !values))) {
        set_error("clamp list is malformed");
        return FLBP_ERR_INVALID;
    }
    if (e->clamp_state.empty()) e->clamp_state.assign((size_t)L.V, -1);
    const std::string bad = check_clamps(L, e->clamp_state, n, vars, values);
    if (!bad.empty()) {
        set_error(bad);
        return FLBP_ERR_INVALID;
    }
    // Every change is staged and the engine's host state is updated only once
    // the device has taken them.
    ClampPlan P;
    P.slots = e->clamp_slots;
    clamp_plan(L, e->prec, e->clamp_state, n, vars, values, P);
    std::vector<uint32_t> &ents = P.ents, &pw = P.pw, &bw = P.bw, &cut_slots = P.cut_slots, &slots = P.slots;
    auto &new_state = P.new_state;
    auto &new_cnt = P.new_cnt;
    const uint32_t n_e = (uint32_t)(ents.size() / 2), n_p = (uint32_t)(pw.size() / 2), n_b = (uint32_t)(bw.size() / 2);
    const uint32_t m = std::max(n_e, std::max(n_p, n_b));
    if (m == 0) return FLBP_OK;
    // the device side: the clamped slots' list, the run state a new engine
    // starts with (previous beliefs 0, for the tolerance rule), the updates
    if (slots.size() > e->clamp_slots_cap) {
        dfree(e, e->d_clamp_slots);
        e->d_clamp_slots = nullptr;
        e->clamp_slots_cap = 0;
        if ((rc = dalloc(e, &e->d_clamp_slots, 2 * slots.size()))) return rc;
        e->clamp_slots_cap = 2 * slots.size();
    }
    if ((rc = upload(e, e->d_clamp_slots, slots)) || (rc = launch_clamp_slots(e, (uint32_t)(slots.size() / 2))))
        return rc;
    FLBP_CUDA(cudaMemsetAsync(e->d_belief, 0, (size_t)std::max<int64_t>(1, L.V) * sizeof(double), e->stream));
    const size_t n_upd = ents.size() + pw.size() + bw.size();
    if (n_upd > e->clamp_upd_cap) {  // kept between calls: no allocation per label in a labelling loop
        dfree(e, e->d_clamp_upd);
        e->d_clamp_upd = nullptr;
        e->clamp_upd_cap = 0;
        if ((rc = dalloc(e, &e->d_clamp_upd, 2 * n_upd))) return rc;
        e->clamp_upd_cap = 2 * n_upd;
    }
    uint32_t *d = e->d_clamp_upd;
    cudaError_t ce = cudaSuccess;
    auto put = [&](const std::vector<uint32_t> &v, size_t at) {
        if (!v.empty() && ce == cudaSuccess)
            ce = cudaMemcpyAsync(d + at, v.data(), v.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, e->stream);
    };
    put(ents, 0);
    put(pw, ents.size());
    put(bw, ents.size() + pw.size());
    if (ce == cudaSuccess) {
        const unsigned blocks = (m + 255) / 256;
        uint32_t *pwords_d = reinterpret_cast<uint32_t *>(e->d_prior), *bw_d = reinterpret_cast<uint32_t *>(e->d_vbt_prior);
        if (e->prec == 64)
            clamp_apply_kernel<double><<<blocks, 256, 0, e->stream>>>(
                d, n_e, d + ents.size(), n_p, d + ents.size() + pw.size(), n_b, (double *)e->d_fv, (double *)e->d_fvd,
                e->d_f_pos, pwords_d, bw_d);
        else
            clamp_apply_kernel<float><<<blocks, 256, 0, e->stream>>>(
                d, n_e, d + ents.size(), n_p, d + ents.size() + pw.size(), n_b, (float *)e->d_fv, (float *)e->d_fvd,
                e->d_f_pos, pwords_d, bw_d);
        e->launches += 1;
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) {
        set_error(std::string("clamp update failed: ") + cudaGetErrorString(ce));
        return FLBP_ERR_CUDA;
    }
    // the host side, now that the device holds the update; like a new engine,
    // no sweeps since construction (the reference's maxiter counts them)
    for (const auto &st : new_state) e->clamp_state[st.first] = st.second;
    for (const auto &c : new_cnt) L.prior_cnt[c.first] = c.second;
    for (uint32_t sl : cut_slots) L.f_pos[sl] = kSentinel;
    e->clamp_slots.swap(slots);
    e->iters = 0;
    e->lowpass_valid = false;
    return FLBP_OK;
}

int flbp_sets_create(const flbp_graph_desc *graph, int64_t n_sets, const int64_t *set_off, const int64_t *set_vars,
                     const int32_t *set_vals, const flbp_engine_opts *opts, flbp_engine **out) {
    if (!out) {
        set_error("null argument");
        return FLBP_ERR_INVALID;
    }
    *out = nullptr;
    if (n_sets <= 0 || n_sets > 65535 || !set_off || set_off[0] != 0) {
        set_error("evidence sets: between 1 and 65535 sets, offsets starting at 0");
        return FLBP_ERR_INVALID;
    }
    for (int64_t k = 0; k < n_sets; k++)
        if (set_off[k + 1] < set_off[k]) {
            set_error("evidence set offsets must not decrease (set " + std::to_string(k) + ")");
            return FLBP_ERR_INVALID;
        }
    if (set_off[n_sets] > 0 && (!set_vars || !set_vals)) {
        set_error("evidence sets lack their clamp arrays");
        return FLBP_ERR_INVALID;
    }
    flbp_engine *e = nullptr;
    int rc = create_engine(graph, opts, &e, nullptr, true);
    if (rc) return rc;
    auto fail = [&](int code) {
        std::string msg = g_last_error;
        flbp_engine_destroy(e);
        set_error(msg);
        return code;
    };
    const HostLayout &L = e->L;
    const uint32_t S = (uint32_t)n_sets;
    const size_t nv_pad = std::max<size_t>({(size_t)1, (size_t)L.V, 32ull * L.n_vgroups()});
    const size_t ns = std::max<size_t>(1, L.n_slots), ne = e->n_ent;
    // every set's clamps: validity, then its cut entries, prior words and slots
    std::vector<uint32_t> base_prior, bt_prior;
    packed_priors(e, nv_pad, base_prior, bt_prior);
    std::vector<uint32_t> prior(base_prior.size() * S);
    std::vector<uint2> cut;
    std::vector<uint4> slots;
    const std::vector<int8_t> state((size_t)L.V, -1);
    for (uint32_t k = 0; k < S; k++) {
        const int64_t n = set_off[k + 1] - set_off[k];
        const int64_t *vars = n ? set_vars + set_off[k] : nullptr;
        const int32_t *vals = n ? set_vals + set_off[k] : nullptr;
        const std::string bad = check_clamps(L, state, n, vars, vals);
        if (!bad.empty()) {
            set_error("evidence set " + std::to_string(k) + ": " + bad);
            return fail(FLBP_ERR_INVALID);
        }
        ClampPlan P;
        clamp_plan(L, e->prec, state, n, vars, vals, P);
        uint32_t *pk = prior.data() + (size_t)k * base_prior.size();
        std::copy(base_prior.begin(), base_prior.end(), pk);
        for (size_t i = 0; i + 1 < P.pw.size(); i += 2) pk[P.pw[i]] = P.pw[i + 1];
        for (size_t i = 0; i + 1 < P.ents.size(); i += 2) cut.push_back(make_uint2(k, P.ents[i]));
        for (size_t i = 0; i + 1 < P.slots.size(); i += 2) slots.push_back(make_uint4(k, P.slots[i], P.slots[i + 1], 0));
    }
    if (cut.size() >= UINT32_MAX || slots.size() >= UINT32_MAX) {
        set_error("evidence sets: too many clamped entries");
        return fail(FLBP_ERR_LIMIT);
    }
    // S copies of the run state; the layout stays single
    for (void **b : {(void **)&e->d_vf, (void **)&e->d_fv, (void **)&e->d_fvd, (void **)&e->d_belief,
                     (void **)&e->d_prior, (void **)&e->d_gstate})
        if (*b) {
            dfree(e, *b);
            *b = nullptr;
        }
    const bool damp = e->damping != 0.0;
    if ((rc = dalloc(e, (char **)&e->d_vf, S * ns * e->tsize)) || (rc = dalloc(e, (char **)&e->d_fv, S * ne * e->tsize)) ||
        (damp && (rc = dalloc(e, (char **)&e->d_fvd, S * ne * e->tsize))) ||
        (rc = dalloc(e, &e->d_belief, S * nv_pad)) || (rc = dalloc(e, &e->d_gstate, 4 * (size_t)S)) ||
        (rc = dalloc(e, (uint32_t **)&e->d_prior, prior.size())) || (rc = upload(e, (uint32_t *)e->d_prior, prior)) ||
        (!cut.empty() && ((rc = dalloc(e, &e->d_set_cut, cut.size())) || (rc = upload(e, e->d_set_cut, cut)))) ||
        (!slots.empty() && ((rc = dalloc(e, &e->d_set_slots, slots.size())) || (rc = upload(e, e->d_set_slots, slots)))))
        return fail(rc);
    FLBP_CUDA(cudaMemsetAsync(e->d_belief, 0, S * nv_pad * sizeof(double), e->stream));
    FLBP_CUDA(cudaMemsetAsync(e->d_gstate, 0, 4 * sizeof(int) * S, e->stream));
    FLBP_CUDA(cudaStreamSynchronize(e->stream));
    e->n_sets = S;
    e->set_vs = ns;
    e->set_es = ne;
    e->set_nv = nv_pad;
    e->n_set_cut = (uint32_t)cut.size();
    e->n_set_slots = (uint32_t)slots.size();
    // Grid width per set: one wave of the direct form's resident blocks over
    // all sets, at least one block and at most one per 16 items of a set.
    auto width = [&](bool var, uint64_t items, uint64_t huge) -> unsigned {
        const int bps = e->prec == 64 ? direct_blocks_per_sm<double>(1, var, damp) : direct_blocks_per_sm<float>(1, var, damp);
        const uint64_t wave = (uint64_t)e->sms * (uint64_t)std::max(bps, 1);
        const uint64_t need = std::max<uint64_t>(1, std::max<uint64_t>((items + kConsumerWarps - 1) / kConsumerWarps, huge));
        return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(need, wave / S));
    };
    e->set_fgx = width(false, (uint64_t)(L.nf_big - L.nf_huge) + L.n_fgroups(), L.nf_huge);
    e->set_vgx = width(true, (uint64_t)(L.nv_big - L.nv_huge) + L.n_vgroups(), L.nv_huge);
    *out = e;
    return FLBP_OK;
}

int flbp_sets_run_tol(flbp_engine *e, double tol, int64_t maxiter, double maxtime, int64_t *sweeps, int32_t *reasons,
                      flbp_run_info *info) {
    int rc = begin_call(e);
    if (rc) return rc;
    if (!e->n_sets) {
        set_error("not an engine of evidence sets (create it with flbp_sets_create)");
        return FLBP_ERR_INVALID;
    }
    return run_groups_tol(e, e->n_sets, tol, maxiter, maxtime, sweeps, reasons, info);
}

int flbp_sets_info(flbp_engine *e, int64_t *n_sets, int64_t *n_vars) {
    int rc = begin_call(e);
    if (rc) return rc;
    if (n_sets) *n_sets = e->n_sets;
    if (n_vars) *n_vars = e->L.V;
    return FLBP_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ sequential schedules

namespace {

void free_seq(flbp_engine *e) {
    void *bufs[] = {e->d_sq_foff, e->d_sq_var, e->d_sq_items, e->d_sq_tgt, e->d_sq_iota, e->d_sq_kind, e->d_sq_cst,
                    e->d_sq_pq,   e->d_sq_fv,  e->d_sq_vf,    e->d_sq_nw,  e->d_sq_S,    e->d_sq_cnt, e->d_sq_irec,
                    e->d_sq_tvar, e->d_sq_bo};
    for (void *b : bufs)
        dfree(e, b);
    e->d_sq_foff = e->d_sq_var = e->d_sq_items = e->d_sq_tgt = e->d_sq_iota = nullptr;
    e->d_sq_irec = e->d_sq_tvar = e->d_sq_bo = nullptr;
    e->seq_cluster = false;
    e->d_sq_kind = nullptr;
    e->d_sq_cst = e->d_sq_pq = e->d_sq_fv = e->d_sq_vf = e->d_sq_nw = nullptr;
    e->d_sq_S = nullptr;
    e->d_sq_cnt = nullptr;
    e->SQ = SeqLayout();
    e->seq = false;
}

template <typename T>
int upload_seq_consts(flbp_engine *e) {
    const SeqLayout &Q = e->SQ;
    std::vector<T> cst(Q.cst.begin(), Q.cst.end()), pq(Q.pq.begin(), Q.pq.end());
    int rc;
    if ((rc = dalloc(e, (T **)&e->d_sq_cst, cst.size())) || (rc = dalloc(e, (T **)&e->d_sq_pq, pq.size())) ||
        (rc = upload(e, (T *)e->d_sq_cst, cst)) || (rc = upload(e, (T *)e->d_sq_pq, pq)))
        return rc;
    const size_t ne = std::max<size_t>(1, (size_t)e->L.E);
    if ((rc = dalloc(e, (T **)&e->d_sq_fv, ne)) || (rc = dalloc(e, (T **)&e->d_sq_vf, ne)) ||
        (rc = dalloc(e, (T **)&e->d_sq_nw, ne)))
        return rc;
    FLBP_CUDA(cudaStreamSynchronize(e->stream));  // the host vectors above go out of scope
    return FLBP_OK;
}

}  // namespace

extern "C" {

int flbp_set_update_seq(flbp_engine *e, const int64_t *seq, int64_t n) {
    int rc = begin_call(e);
    if (rc || (rc = refuse_sets(e, "sequential schedules")) || (rc = ensure_host_layout(e))) return rc;
    if (e->n_graphs > 0) {
        set_error("sequential update schedules are not available on batched engines");
        return FLBP_ERR_STATE;
    }
    for (int8_t st : e->clamp_state)
        if (st >= 0) {
            set_error("sequential update schedules are not available after flbp_clamp_vars");
            return FLBP_ERR_STATE;
        }
    if ((rc = sync_host_probs(e))) return rc;
    const HostLayout &L = e->L;
    SeqLayout Q;
    if (seq) {  // build before touching the engine, so that a bad sequence leaves it as it was
        std::vector<int64_t> slot_var(L.ref_slot_var.begin(), L.ref_slot_var.end());
        flbp_graph_desc g{};
        g.n_vars = L.V;
        g.n_factors = L.F;
        g.n_slots = L.E;
        g.factor_offsets = L.ref_off.data();
        g.slot_var = slot_var.data();
        g.factor_head = e->ref_head.data();
        g.factor_p = e->factor_p_host.data();
        g.factor_q = e->factor_q_host.data();
        std::string err;
        if ((rc = build_seq_layout(g, L, seq, n, Q, err))) {
            set_error(err);
            return rc;
        }
    }
    FLBP_CUDA(cudaStreamSynchronize(e->stream));
    for (auto &kv : e->graphs) cudaGraphExecDestroy(kv.second);  // captured for the previous schedule
    e->graphs.clear();
    free_seq(e);
    if (seq) {
        e->SQ = std::move(Q);
        const SeqLayout &S = e->SQ;
        const size_t nv = std::max<size_t>(1, (size_t)L.V), ne = std::max<size_t>(1, (size_t)L.E);
        std::vector<uint32_t> iota(ne);
        for (size_t k = 0; k < ne; k++) iota[k] = (uint32_t)k;
        if ((rc = dalloc(e, &e->d_sq_foff, S.foff.size())) || (rc = upload(e, e->d_sq_foff, S.foff)) ||
            (rc = dalloc(e, &e->d_sq_var, S.var.size())) || (rc = upload(e, e->d_sq_var, S.var)) ||
            (rc = dalloc(e, &e->d_sq_kind, S.kind.size())) || (rc = upload(e, e->d_sq_kind, S.kind)) ||
            (rc = dalloc(e, &e->d_sq_items, S.items.size())) || (rc = upload(e, e->d_sq_items, S.items)) ||
            (rc = dalloc(e, &e->d_sq_tgt, S.tgt.size())) || (rc = upload(e, e->d_sq_tgt, S.tgt)) ||
            (rc = dalloc(e, &e->d_sq_iota, ne)) || (rc = upload(e, e->d_sq_iota, iota)) ||
            (rc = dalloc(e, &e->d_sq_irec, S.irec.size())) || (rc = upload(e, e->d_sq_irec, S.irec)) ||
            (rc = dalloc(e, &e->d_sq_tvar, S.tvar.size())) || (rc = upload(e, e->d_sq_tvar, S.tvar)) ||
            (rc = dalloc(e, &e->d_sq_bo, S.bo.size())) || (rc = upload(e, e->d_sq_bo, S.bo)) ||
            (rc = dalloc(e, &e->d_sq_S, nv)) || (rc = dalloc(e, &e->d_sq_cnt, nv)) ||
            (rc = (e->prec == 64 ? upload_seq_consts<double>(e) : upload_seq_consts<float>(e)))) {
            free_seq(e);
            return rc;
        }
        e->seq = true;
        e->seq_cluster = choose_seq_cluster(e);
    }
    if ((rc = flbp_init(e))) return rc;
    FLBP_CUDA(cudaStreamSynchronize(e->stream));
    return FLBP_OK;
}

int flbp_set_seq_kernel(flbp_engine *e, int32_t kind) {
    int rc = begin_call(e);
    if (rc) return rc;
    if (kind < 0 || kind > 3) {
        set_error("kind must be 0 (choose), 1 (two launches per batch), 2 (one cluster per sweep) or 3 (two "
                  "launches per batch with programmatic dependent launch)");
        return FLBP_ERR_INVALID;
    }
    FLBP_CUDA(cudaStreamSynchronize(e->stream));
    for (auto &kv : e->graphs) cudaGraphExecDestroy(kv.second);
    e->graphs.clear();
    e->seq_kernel = kind;
    e->seq_cluster = e->seq && choose_seq_cluster(e);
    return FLBP_OK;
}

int flbp_update_info(flbp_engine *e, int32_t *sequential, int64_t *n_batches) {
    if (!e) {
        set_error("null engine handle");
        return FLBP_ERR_INVALID;
    }
    if (sequential) *sequential = e->seq ? 1 : 0;
    if (n_batches) *n_batches = e->seq ? (int64_t)e->SQ.n_batches : 1;
    return FLBP_OK;
}

}  // extern "C"
