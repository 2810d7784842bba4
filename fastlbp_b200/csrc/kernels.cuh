// sm_100a kernels of one synchronous (PARALL) causal-BP sweep.
//
// Messages are log-odds lambda = log(m1/m0) in two arrays: vf (variable ->
// factor) in factor-slot order and fv (factor -> variable) in variable-entry
// order, so that each pass reads its inputs as contiguous streams and
// scatters its outputs into the other pass's order (stores only; no pass
// waits on a gather). A sweep is
//   factor pass:   fv <- f(vf) for every active factor, all its outputs;
//   variable pass: per variable the sum of its incoming fv plus its constant
//                  prior, then vf <- total - own message, beliefs, residual.
// This is the reference's FV -> Prod -> VF sequence
// (csrc/ext/causal_bp.cu:409-444) restated in log-odds. With damping the
// variable pass mixes each new f->v message with the previous damped one
// (array fvd, variable-entry order) before using it.
//
// Exact zeros of the reference's probability arithmetic become +-inf
// log-odds. On the factor side zeros flow through sums of log-sigmoids as
// -inf (prefix/suffix sums never subtract); on the variable side +inf / -inf
// counts play the role of the reference's num_zeros counters
// (causal_bp_parall.cu:36-45, 74-83).
//
// OR factors are evaluated as AND factors on negated log-odds (the states 0
// and 1 swap roles, causal_bp_parall.cu:152-190 vs :113-151) and their
// outputs negated back.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "engine_internal.h"

namespace flbp {

// Control block of one engine (device memory). Written by block 0 of the
// factor pass (sweep counters, residual reset) and by the last block of the
// variable pass (stop decision); read by every block at kernel entry.
struct Ctl {
    unsigned long long maxdiff_bits;  // max |belief change| of this sweep, double bits
    unsigned long long nonconv;       // variables with |belief change| > tol
    unsigned int arrive;              // variable-pass blocks finished this sweep
    int done;                         // set: every kernel returns at entry
    long long t;                      // sweeps since init (damping exponent)
    long long run_sweeps;             // sweeps of the current run call
    long long iters0;                 // reference _iters at the start of the run call
    unsigned long long t_start_ns;    // %globaltimer at the first sweep of the run call
    int mode;                         // 0 none, 1 tolerance loop, 2 low-pass loop
    int reason;
    int status;
    int pad;
    double tol;
    long long maxiter;                // mode 1
    long long min_iters, max_iters;   // mode 2
    double maxtime_ns;
    double maxdiff;                   // last sweep's residual (decoded)
    double frac;                      // last sweep's non-converged fraction
    double node_frac_tol;
    long long n_vars;
    double damping;
    double pscale;                    // 1 - damping^t: weight of the finite constant priors
    unsigned int fnext, vnext;        // next chunk of tiles of the factor / variable pass (reset by the other pass)
    // batched solves: number of tiles of the factor / variable pass that hold a live graph
    unsigned int n_act_f, n_act_v;
};

template <typename T>
struct Num;

template <>
struct Num<float> {
    static __device__ __forceinline__ float inf() { return __int_as_float(0x7f800000); }
    static __device__ __forceinline__ float nan() { return __int_as_float(0x7fffffff); }
    static __device__ __forceinline__ float exp(float x) { return __expf(x); }
    static __device__ __forceinline__ float log(float x) { return __logf(x); }
    static __device__ __forceinline__ float log1p(float x) { return ::log1pf(x); }
    static __device__ __forceinline__ float expm1(float x) { return ::expm1f(x); }
    static __device__ __forceinline__ float rcp(float x) { return __fdividef(1.0f, x); }  // x in [1, 2] here
    static __device__ __forceinline__ float tiny() { return 1.17549435e-38f; }           // smallest normal
};

template <>
struct Num<double> {
    static __device__ __forceinline__ double inf() { return __longlong_as_double(0x7ff0000000000000ll); }
    static __device__ __forceinline__ double nan() { return __longlong_as_double(0x7fffffffffffffffll); }
    static __device__ __forceinline__ double exp(double x) { return ::exp(x); }
    static __device__ __forceinline__ double log(double x) { return ::log(x); }
    static __device__ __forceinline__ double log1p(double x) { return ::log1p(x); }
    static __device__ __forceinline__ double expm1(double x) { return ::expm1(x); }
    static __device__ __forceinline__ double rcp(double x) { return 1.0 / x; }
    static __device__ __forceinline__ double tiny() { return 2.2250738585072014e-308; }  // smallest normal
};

template <typename T>
__device__ __forceinline__ bool is_nan(T x) {
    return x != x;
}

// Streaming loads (read once per sweep): evict-first in L2 so that the
// message arrays, reused every pass, stay resident.
__device__ __forceinline__ uint32_t ld_stream(const uint32_t *p) { return __ldcs(p); }
__device__ __forceinline__ uint2 ld_stream(const uint2 *p) { return __ldcs(p); }
__device__ __forceinline__ uint8_t ld_stream(const uint8_t *p) {
    return (uint8_t)__ldcs(reinterpret_cast<const unsigned char *>(p));
}
__device__ __forceinline__ float ld_stream(const float *p) { return __ldcs(p); }
__device__ __forceinline__ double ld_stream(const double *p) { return __ldcs(p); }

// log(sigmoid(x)) = min(x,0) - log1p(exp(-|x|)); +inf -> 0, -inf -> -inf, NaN -> NaN.
template <typename T>
__device__ __forceinline__ T log_sigmoid(T x) {
    return fmin(x, T(0)) - Num<T>::log1p(Num<T>::exp(-fabs(x)));
}

// AND -> head (causal_bp_parall.cu:113-151 in log-odds). With P = product of
// sigma over the body = exp(lo) and R = 1 - P:
//   m1 ~ p P + q R,   m0 ~ (1-p) P + (1-q) R   (m0 + m1 = 1).
// lp = log p, used for q == 0 so that tiny P does not underflow.
template <typename T>
__device__ __forceinline__ T head_out(T lo, T p, T q, T lp) {
    const T P = Num<T>::exp(lo), R = -Num<T>::expm1(lo);
    const T B = fma(T(1) - p, P, (T(1) - q) * R);
    const T la = (q == T(0)) ? lp + lo : Num<T>::log(fma(p, P, q * R));
    return la - Num<T>::log(B);
}

// AND -> body (types 5/7, causal_bp_parall.cu:289-314, 341-366). With
// Po = product of sigma over the other body slots = exp(lo), Ro = 1 - Po,
// a = p Po + q Ro, b = 1 - a and head log-odds lh:
//   m1 ~ sigma(lh) a + sigma(-lh) b,   m0 ~ sigma(lh) q + sigma(-lh) (1-q).
// Both are divided by max(sigma(lh), sigma(-lh)); r = exp(-|lh|). Terms that
// are exactly zero are taken in log space so that large |lh| cannot
// underflow them. When m0 == 0 exactly (the reference's prod_10 == 0, which
// skips its loop) the result is +inf if (p-q)(m1h-m0h) > 0 and NaN
// otherwise, as the reference's scale() of (x, 0) and (0, 0) gives.
// The m0 side depends only on the factor (head message, q), so it is
// evaluated once per factor: lden = log of the scaled m0 and the value
// returned when m0 == 0 exactly.
// With u = a, w = b for lh >= 0 and u = b, w = a otherwise, the scaled
// numerator is u + r w, taken as log(w) - |lh| when u == 0 (so that r cannot
// underflow it), and the denominator likewise with (q, 1-q). Both forms are
// selected without branches.
template <typename T>
struct BodyDen {
    T lden, zero_out, r, alh;  // alh = |lh|
    T pu, qu, pw, qw;          // u = pu Po + qu Ro, w = pw Po + qw Ro of a body slot
    bool dead;                 // lden == -inf: every body output is zero_out
};

template <typename T>
__device__ __forceinline__ BodyDen<T> body_den(T lh, T p, T q) {
    BodyDen<T> D;
    const bool pos = lh >= T(0);
    D.alh = fabs(lh);
    D.r = Num<T>::exp(-D.alh);
    const T u = pos ? q : T(1) - q, w = pos ? T(1) - q : q;
    D.lden = Num<T>::log(u == T(0) ? w : fma(D.r, w, u)) - (u == T(0) ? D.alh : T(0));
    const T s = pos ? (p - q) : (q - p);
    D.zero_out = is_nan(lh) ? lh : ((s > T(0)) ? Num<T>::inf() : Num<T>::nan());
    if (is_nan(lh)) D.lden = -Num<T>::inf();
    D.dead = D.lden == -Num<T>::inf();
    // a = p Po + q Ro, b = (1-p) Po + (1-q) Ro; u = a, w = b for lh >= 0, swapped otherwise
    D.pu = pos ? p : T(1) - p;
    D.qu = pos ? q : T(1) - q;
    D.pw = pos ? T(1) - p : p;
    D.qw = pos ? T(1) - q : q;
    return D;
}

// Body output from the pair (Po, Ro = 1 - Po) of the other body slots.
template <typename T>
__device__ __forceinline__ T body_out_pr(T Po, T Ro, T p, T q, const BodyDen<T> &D) {
    // explicit fused forms: the result must not depend on how a caller's code is contracted
    const T u = fma(D.pu, Po, D.qu * Ro), w = fma(D.pw, Po, D.qw * Ro);
    const T lnum = Num<T>::log(u == T(0) ? w : fma(D.r, w, u)) - (u == T(0) ? D.alh : T(0));
    return D.dead ? D.zero_out : lnum - D.lden;
}

// Body output from lo = log Po.
template <typename T>
__device__ __forceinline__ T body_out(T lo, T p, T q, const BodyDen<T> &D) {
    return body_out_pr<T>(Num<T>::exp(lo), -Num<T>::expm1(lo), p, q, D);
}

// Damping of an f->v message in log-odds: (1-d) new + d old, with exact
// zeros dominating (0^(1-d) = 0^d = 0) and opposite zeros giving (0.5, 0.5).
template <typename T>
__device__ __forceinline__ T damp_mix(T nw, T old, T d) {
    const T inf = Num<T>::inf();
    const bool ni = fabs(nw) == inf, oi = fabs(old) == inf;
    if (ni || oi) {
        if (ni && oi) return (nw == old) ? nw : T(0);
        return ni ? nw : old;
    }
    return fma(T(1) - d, nw, d * old);
}

struct FactorArgs {
    const uint32_t *fg_base;  // sliced-ELL groups (n_fgroups + 1)
    const uint32_t *fb_off;   // big factors (nf_big + 1)
    const uint32_t *f_pos;    // per device slot: fv position of its output (kSentinel: none)
    const uint8_t *f_kind;
    const uint8_t *f_deg;
    const void *f_pq;         // T[2 * nf]
    const uint32_t *fb_deg;   // per big factor: degree
    const uint32_t *bt_deg;   // per big tile: kTileGroups degrees
    const uint8_t *bt_kind;   // per big tile: kTileGroups kinds
    const void *bt_pq;        // per big tile: kTileGroups (p, q), T
    const uint4 *thdr;        // kHdrWords-word header per tile (see TileHdr)
    const uint32_t *f_graph;  // batched solves: graph of every internal factor, else null
    const int *gdone;         // batched solves: per graph, nonzero once it has stopped
    const uint2 *trange;      // batched solves: per tile, the range of its items' graphs
    uint32_t n_graphs;        // batched solves: number of graphs
    uint32_t nf_sell, nf_big, nf_huge, n_fgroups, n_tiles, n_tile_blocks;
    // Staged form on one graph: block b's tiles tile_list[tile_off[b] ..
    // tile_off[b + 1]) (null: tiles b, b + gridDim.x, ...).
    const uint32_t *tile_list = nullptr, *tile_off = nullptr;
    // Staged form of a batched solve: the tiles that hold a live graph,
    // act_list[0 .. *n_act) (null: every tile).
    const uint32_t *act_list = nullptr;
    const unsigned int *n_act = nullptr;
    // Evidence sets on one graph (direct form, set = blockIdx.y): per-set
    // message strides and stopped flags; null / 0 otherwise.
    const int *set_done = nullptr;
    uint64_t set_vf_stride = 0, set_fv_stride = 0;
};

struct VarArgs {
    const uint32_t *vg_base;  // sliced-ELL groups (n_vgroups + 1)
    const uint32_t *vb_off;   // big variables (nv_big + 1)
    const uint32_t *vb_deg;   // per big variable: number of entries
    const uint32_t *bt_deg;   // per big tile: kTileGroups entry counts
    const void *bt_prior;     // per big tile: kTileGroups priors (layout of `prior`)
    const uint32_t *v_ent;    // per entry: device slot of the factor side (kSentinel: padding)
    const void *prior;        // per variable: FP32 engines uint2 (float bits of the finite prior,
                              // +inf | -inf << 16 counts); FP64 engines uint4 (double bits, counts, 0)
    double *belief;           // per internal variable, previous / current belief
    double *hist;             // low-pass history [hist_len][n_vars], or null
    uint32_t *hist_next;      // per variable ring cursor
    uint32_t *hist_count;     // per variable number of stored samples
    const uint4 *thdr;        // kHdrWords-word header per tile (see TileHdr)
    uint32_t nv_sell, nv_big, nv_huge, n_vgroups, n_tiles, n_tile_blocks;
    uint32_t hist_len;
    // Batched solves (BMODE 4): graph of every internal variable and the
    // per-graph state gstate[4][n_graphs] = stopped flag, "some belief moved
    // by more than tol this sweep" flag, sweeps, stop reason.
    const uint32_t *v_graph;
    int *gstate;
    const uint2 *trange;      // per tile, the range of its items' graphs
    uint32_t n_graphs;
    // Staged form of a batched solve: the live tiles (see FactorArgs).
    const uint32_t *act_list = nullptr;
    const unsigned int *n_act = nullptr;
    // Evidence sets on one graph (direct form, set = blockIdx.y): per-set
    // strides of messages, priors (bytes) and beliefs; gstate / n_graphs
    // then hold the sets' stop state.
    uint64_t set_vf_stride = 0, set_fv_stride = 0, set_prior_stride = 0, set_belief_stride = 0;
};

// ------------------------------------------------------------ accumulators
//
// Sums of log-odds (a variable's incoming messages and prior) and of
// log-sigmoids (a large factor's body). FP64 engines sum in double. FP32
// engines keep the sweep in FP32: a plain float sum where at most 16 terms
// meet (the sliced-ELL variables), and a compensated two-float sum
// (Neumaier's variant of Kahan summation) for wider items, whose error does
// not grow with the number of terms. FP64 then appears in an FP32 sweep only
// in the residual and in the belief normalisation (belief_of).
struct F2 {
    float hi, lo;  // value = hi + lo
};

template <typename A>
struct AccOps;

template <>
struct AccOps<double> {
    static __device__ __forceinline__ double zero() { return 0.0; }
    static __device__ __forceinline__ double of(double x) { return x; }
    static __device__ __forceinline__ void add(double &s, double x) { s += x; }
    static __device__ __forceinline__ void combine(double &s, double o) { s += o; }
    static __device__ __forceinline__ double value(double s) { return s; }
    // s - x rounded once to the message type
    template <typename T>
    static __device__ __forceinline__ T excl(double s, T x) {
        return (T)(s - (double)x);
    }
    static __device__ __forceinline__ double shfl_xor(double s, int o) { return __shfl_xor_sync(0xffffffffu, s, o); }
};

template <>
struct AccOps<float> {
    static __device__ __forceinline__ float zero() { return 0.f; }
    static __device__ __forceinline__ float of(float x) { return x; }
    static __device__ __forceinline__ void add(float &s, float x) { s += x; }
    static __device__ __forceinline__ void combine(float &s, float o) { s += o; }
    static __device__ __forceinline__ double value(float s) { return (double)s; }
    template <typename T>
    static __device__ __forceinline__ T excl(float s, T x) {
        return (T)(s - (float)x);
    }
    static __device__ __forceinline__ float shfl_xor(float s, int o) { return __shfl_xor_sync(0xffffffffu, s, o); }
};

template <>
struct AccOps<F2> {
    static __device__ __forceinline__ F2 zero() { return F2{0.f, 0.f}; }
    static __device__ __forceinline__ F2 of(float x) { return F2{x, 0.f}; }
    static __device__ __forceinline__ void add(F2 &s, float x) {  // Neumaier: the error of hi + x into lo
        const float t = s.hi + x;
        s.lo += (fabsf(s.hi) >= fabsf(x)) ? (s.hi - t) + x : (x - t) + s.hi;
        s.hi = t;
    }
    static __device__ __forceinline__ void combine(F2 &s, F2 o) {
        add(s, o.hi);
        s.lo += o.lo;
    }
    static __device__ __forceinline__ double value(F2 s) { return (double)s.hi + (double)s.lo; }
    template <typename T>
    static __device__ __forceinline__ T excl(F2 s, T x) {
        return (T)((s.hi - (float)x) + s.lo);
    }
    static __device__ __forceinline__ F2 shfl_xor(F2 s, int o) {
        return F2{__shfl_xor_sync(0xffffffffu, s.hi, o), __shfl_xor_sync(0xffffffffu, s.lo, o)};
    }
};

// Accumulator of the sliced-ELL variables (<= 16 terms) and of wider items.
template <typename T>
struct NarrowAcc {
    typedef T type;
};
template <typename T>
struct WideAcc;
template <>
struct WideAcc<float> {
    typedef F2 type;
};
template <>
struct WideAcc<double> {
    typedef double type;
};

template <typename T>
__device__ __forceinline__ T head_effective(uint8_t kind, T vf_head) {
    const uint8_t hs = kind & HEAD_MASK;
    const T inf = Num<T>::inf();
    if (hs == HEAD_FREE) return vf_head;
    if (hs == HEAD_ONE) return inf;
    if (hs == HEAD_ZERO) return -inf;
    return Num<T>::nan();
}

// ------------------------------------------------------------------ TMA staging
//
// Both passes run persistent blocks of kConsumerWarps consumer warps plus one
// producer warp over "tiles" of up to kTileGroups sliced-ELL groups and
// kTileSlots slots (entries). The producer brings each tile's contiguous
// streams (messages, scatter indices, per-item constants) into a
// STAGES-deep shared-memory ring with 1-D bulk copies (cp.async.bulk,
// completion tracked by one mbarrier per stage, no multicast). Each consumer
// warp takes one group of the staged tile (lane = item), scatters its
// outputs to global memory and releases the stage; warps never wait for one
// another. All waits are bounded: on a timeout the block records
// FLBP_ERR_TIMEOUT in ctl->status, lets its own copies land and returns.

constexpr int kConsumerWarps = 16;
constexpr int kConsumers = 32 * kConsumerWarps;    // consumer threads per block
constexpr int kBlockThreadsDev = kConsumers + 32;  // + one producer warp
constexpr int kTileGroups = 16;                    // groups per tile = consumer warps
constexpr int kTileItems = 32 * kTileGroups;       // factors / variables per tile
constexpr int kTileSlots = 2048;                   // slot (entry) budget of a tile
constexpr int kHdrWords = 32;                      // tile header: 128 bytes
static_assert(kTileGroups == kConsumerWarps, "one consumer warp per group of a tile");
static_assert(kHdrWords == (int)kHdrWordsHost && kTileGroups == (int)kTileGroupsHost, "tile format");
constexpr long long kWaitCycles = 4000000000ll;    // ~2 s at 2 GHz

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for a stage; false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;  // the common case: no clock read
    const long long t0 = clock64();
    for (uint32_t i = 1;; i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 15u) == 0 && clock64() - t0 > kWaitCycles) return false;
    }
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void record_timeout(Ctl *ctl) { atomicExch(&ctl->status, FLBP_ERR_TIMEOUT); }

// Barrier among the consumer threads only (the producer warp never joins).
__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kConsumers) : "memory"); }


// Waits for a stage on every lane of a warp; true on all lanes, or false on
// all lanes when any of them gave up.
__device__ __forceinline__ bool warp_wait_stage(uint64_t *bar, uint32_t parity) {
    return __all_sync(0xffffffffu, mbar_wait_bounded(bar, parity));
}

// Per-tile header (kHdrWords words, host-built): [0] first group (first big
// item), [1] number of groups (big items) n in 1..kTileGroups, with
// kBigTileFlag set for a tile of big items, [2 + j] slot (entry) offset of
// item j for j = 0..n, the remaining words repeating the end offset, except
// that word kHdrWords - 1 of a big tile holds its ordinal among the big
// tiles (the index of its per-tile constants). The producer loads
// the next tile's header into registers while the current tile's copies are
// in flight, so that header latency stays off the pipeline's critical path.
struct TileHdr {
    uint4 w[kHdrWords / 4];
    __device__ __forceinline__ void load(const uint4 *src) {
#pragma unroll
        for (int i = 0; i < kHdrWords / 4; i++) w[i] = __ldcg(src + i);
    }
    __device__ __forceinline__ void store(uint32_t *dst) const {
        uint4 *d = reinterpret_cast<uint4 *>(dst);
#pragma unroll
        for (int i = 0; i < kHdrWords / 4; i++) d[i] = w[i];
    }
};

constexpr uint32_t kEndTile = 0x40000000u;  // header word 1 of the stage that ends a block's tiles
constexpr int kDoneWords = 128;              // graphs whose stopped flag is cached in shared memory, / 32

// Batched solves: stopped flags of graphs [0, 32 kDoneWords) as bits in
// shared memory, taken at kernel entry (they change only between launches).
__device__ __forceinline__ void load_done_bits(uint32_t *s_done, const int *gdone, uint32_t n_graphs, int lane,
                                               int wid, int nwarps) {
    const uint32_t words = min((n_graphs + 31) / 32, (uint32_t)kDoneWords);
    for (uint32_t w = wid; w < words; w += nwarps) {
        const uint32_t g = 32 * w + lane;
        const uint32_t bits = __ballot_sync(0xffffffffu, g < n_graphs && gdone[g] != 0);
        if (lane == 0) s_done[w] = bits;
    }
}

__device__ __forceinline__ bool graph_done(const uint32_t *s_done, const int *gdone, uint32_t g) {
    return g < 32u * kDoneWords ? ((s_done[g >> 5] >> (g & 31)) & 1u) != 0 : gdone[g] != 0;
}

// Producer warp of a pass. A single graph's pass walks the block's own
// tiles in order: the list the engine dealt it (tile_list / tile_off, tiles
// of about equal total cost per block, so that all SMs finish together), or
// without a list tiles blockIdx.x + i gridDim.x. A batched solve instead takes chunks of kChunkTiles consecutive
// tiles from the pass's counter, so that blocks whose tiles belong to stopped
// graphs take more, and leaves out tiles whose graphs have all stopped. One
// stage per remaining tile is filled with fill(stage, header in shared
// memory, full barrier); a stage whose header word 1 is kEndTile closes the
// stream. All lanes call it; lane 0 issues the copies. After a timeout it
// records FLBP_ERR_TIMEOUT, lets its own copies land and returns false.
constexpr uint32_t kChunkTiles = 4;

template <int STAGES, typename Fill>
__device__ bool produce_tiles(const uint4 *thdr, const uint2 *trange, const uint32_t *tile_list,
                              const uint32_t *tile_off, const uint32_t *act_list, const unsigned int *n_act,
                              const uint32_t *s_done, const int *gdone, uint32_t n_tiles, unsigned int *counter,
                              unsigned char *smem, size_t stage_bytes, uint64_t *full, uint64_t *empty, int lane,
                              Ctl *ctl, Fill fill) {
    uint32_t issued = 0;
    bool ok = true;
    const bool dynamic = trange != nullptr;
    // round r covers tiles tile_at(r, 0..width-1)
    const uint32_t width = dynamic ? kChunkTiles : 32u;
    const uint32_t nb = gridDim.x;
    uint32_t round = dynamic ? __shfl_sync(0xffffffffu, lane == 0 ? atomicAdd(counter, 1u) : 0u, 0) : 0u;
    const bool listed = !dynamic && tile_list != nullptr;
    const uint32_t l0 = listed ? tile_off[blockIdx.x] : 0u, ln = listed ? tile_off[blockIdx.x + 1] - l0 : 0u;
    const bool live_list = dynamic && act_list != nullptr;
    const uint32_t n_live = live_list ? *(volatile const unsigned int *)n_act : 0u;
    auto tile_at = [&](uint32_t r, uint32_t k) -> uint32_t {  // n_tiles when out of range
        if (listed) {
            const uint64_t i = (uint64_t)r * width + k;
            return i < ln ? tile_list[l0 + i] : n_tiles;
        }
        if (live_list) {
            const uint64_t i = (uint64_t)r * width + k;
            return i < n_live ? act_list[i] : n_tiles;
        }
        const uint64_t t = dynamic ? (uint64_t)r * width + k : (uint64_t)blockIdx.x + ((uint64_t)r * width + k) * nb;
        return t < n_tiles ? (uint32_t)t : n_tiles;
    };
    // The round's tile headers, one per lane, loaded by the whole warp at
    // once, so that lane 0 issues every stage's copies without waiting for a
    // header load.
    __shared__ uint4 s_hdr[32][kHdrWords / 4];
    while (ok && tile_at(round, 0) < n_tiles) {
        const uint32_t next = dynamic ? __shfl_sync(0xffffffffu, lane == 0 ? atomicAdd(counter, 1u) : 0u, 0)
                                      : round + 1;
        const uint32_t t = (uint32_t)lane < width ? tile_at(round, lane) : n_tiles;
        bool act = t < n_tiles;
        if (act && dynamic) {  // active unless every graph of the tile has stopped
            const uint2 r = trange[t];
            bool stopped = r.y >= r.x && r.y - r.x <= 32;
            for (uint32_t g = r.x; stopped && g <= r.y; g++) stopped = graph_done(s_done, gdone, g);
            act = !stopped;
        }
        uint32_t bits = __ballot_sync(0xffffffffu, act);
        if (act) {  // global -> shared without registers (16 B asynchronous copies)
            const uint4 *src = thdr + (size_t)(kHdrWords / 4) * t;
            const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&s_hdr[lane][0]);
#pragma unroll
            for (int i = 0; i < kHdrWords / 4; i++)
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst + 16u * i), "l"(src + i) : "memory");
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncwarp();
        if (lane == 0) {
            int j = bits ? __ffs(bits) - 1 : -1;
            while (j >= 0) {
                bits &= bits - 1;
                const int s = (int)(issued % STAGES);
                if (issued >= (uint32_t)STAGES && !mbar_wait_bounded(&empty[s], ((issued / STAGES) - 1) & 1u)) {
                    ok = false;
                    break;
                }
                unsigned char *st = smem + (size_t)s * stage_bytes;
                uint32_t *gb = reinterpret_cast<uint32_t *>(st);
#pragma unroll
                for (int i = 0; i < kHdrWords / 4; i++) reinterpret_cast<uint4 *>(gb)[i] = s_hdr[j][i];
                fill(st, gb, &full[s]);
                issued++;
                j = bits ? __ffs(bits) - 1 : -1;
            }
        }
        __syncwarp();  // s_hdr is rewritten next round
        ok = __shfl_sync(0xffffffffu, ok, 0);
        round = next;
    }
    if (lane == 0) {
        if (ok) {  // end marker
            const int s = (int)(issued % STAGES);
            if (issued >= (uint32_t)STAGES && !mbar_wait_bounded(&empty[s], ((issued / STAGES) - 1) & 1u)) {
                ok = false;
            } else {
                reinterpret_cast<uint32_t *>(smem + (size_t)s * stage_bytes)[1] = kEndTile;
                mbar_arrive_expect_tx(&full[s], 0);
                issued++;
            }
        }
        if (!ok) {
            record_timeout(ctl);
            // let this block's own loads in flight land before the block moves on
            for (uint32_t k = issued > (uint32_t)STAGES ? issued - STAGES : 0; k < issued; k++)
                mbar_wait_bounded(&full[k % STAGES], (k / STAGES) & 1u);
        }
    }
    return __shfl_sync(0xffffffffu, ok, 0);
}

// Shared-memory layout of one factor-pass stage. Batched solves (GID) also
// stage the graph of every factor; a single graph's pass has no use for it,
// and the room it leaves takes a fifth FP32 stage at two blocks per SM.
template <typename T, bool GID = true>
struct FactorStage {
    static constexpr size_t hdr = 0;                                   // uint32[kHdrWords]
    static constexpr size_t vbuf = 128;                                // T[kTileSlots]: incoming vf
    static constexpr size_t pos = vbuf + sizeof(T) * kTileSlots;       // uint32[kTileSlots]: fv position per slot
    static constexpr size_t deg = pos + 4 * kTileSlots;                // uint8[kTileItems]
    static constexpr size_t kind = deg + kTileItems;                   // uint8[kTileItems]
    static constexpr size_t pq = kind + kTileItems;                    // T[2 * kTileItems]
    static constexpr size_t gid = pq + 2 * sizeof(T) * kTileItems;     // uint32[kTileItems]: graph (batched solves)
    static constexpr size_t bytes = (gid + (GID ? 4 * kTileItems : 0) + 127) & ~(size_t)127;
};

// Shared-memory layout of one variable-pass stage.
template <typename T, bool DAMP>
struct VarStage {
    static constexpr size_t hdr = 0;                                             // uint32[kHdrWords]
    static constexpr size_t ent = 128;                                           // uint32[kTileSlots]
    static constexpr size_t x = ent + 4 * kTileSlots;                            // T[kTileSlots]: incoming fv
    static constexpr size_t xo = x + sizeof(T) * kTileSlots;                     // T[kTileSlots]: previous damped fv
    static constexpr size_t prior = xo + (DAMP ? sizeof(T) * kTileSlots : 0);   // uint2 / uint4 [kTileItems]
    static constexpr size_t bold = prior + (sizeof(T) == 4 ? 8 : 16) * kTileItems;  // double[kTileItems]
    static constexpr size_t gid = bold + 8 * kTileItems;                        // uint32[kTileItems]: graph (batched)
    static constexpr size_t bytes = gid + 4 * kTileItems;
};

// sigma(x) and 1 - sigma(x) without cancellation, from e = exp(-|x|):
// +inf -> (1, 0), -inf -> (0, 1), NaN -> (NaN, NaN).
template <typename T>
__device__ __forceinline__ void sig_pair(T x, T &sg, T &tau) {
    const T e = Num<T>::exp(-fabs(x));
    const T inv = Num<T>::rcp(T(1) + e);
    const bool pos = x >= T(0);
    sg = pos ? inv : e * inv;
    tau = pos ? e * inv : inv;
}

template <typename T>
__device__ __forceinline__ void put_fv(T *__restrict__ fv, uint32_t e, T o) {
    if (e != kSentinel) fv[e] = o;
}

// Head output of an AND factor from the pair (P, R = 1 - P) of its whole
// body: m1 ~ p P + q R, m0 ~ (1-p) P + (1-q) R (causal_bp_parall.cu:113-151
// in log-odds). With q == 0 and P not a normal number, p P is taken in log
// space from lP(), the sum of the body's log-sigmoids.
template <typename T, typename LogP>
__device__ __forceinline__ T head_from_pair(T P, T R, T p, T q, LogP lP) {
    const T la = (q == T(0) && P < Num<T>::tiny()) ? Num<T>::log(p) + lP() : Num<T>::log(fma(p, P, q * R));
    return la - Num<T>::log(fma(T(1) - p, P, (T(1) - q) * R));
}

// One factor of a sliced-ELL group of width W, one lane, all in registers:
// vb(k) is the message of slot k of the factor (head at k = 0) and ps(k) the
// fv position of its output, read from a staged tile in shared memory or
// from registers that the direct form loaded. With sigma_k, tau_k = 1 - sigma_k of the
// body messages (AND orientation), pairs combine as
//   (P1, R1) o (P2, R2) = (P1 P2, R1 + P1 R2),
// a product and its complement: every term is non-negative, so P and 1 - P
// both keep full relative precision and exact zeros stay exact. Prefix and
// suffix pairs give each body slot the pair of all other body slots without
// a division; its output is body_out_pr (causal_bp_parall.cu:289-314,
// 341-366 in log-odds; OR = AND on negated log-odds). Widths up to 8 keep
// sigma, tau and the suffix pairs of every slot (4 W registers); wider
// groups keep only the prefix pairs and evaluate sigma again on the way back.
template <typename T, int W, typename VB, typename PS>
__device__ __forceinline__ void factor_reg(VB vb, PS ps, int deg, uint8_t kind, T p, T q, T *__restrict__ fv) {
    const T sgn = (kind & KIND_OR) ? T(-1) : T(1);
    auto logP = [&]() {
        T l = T(0);
#pragma unroll
        for (int k = 1; k < W; k++)
            if (k < deg) l += log_sigmoid<T>(sgn * vb(k));
        return l;
    };
    const T lh = sgn * head_effective<T>(kind, vb(0));
    if constexpr (W <= 8) {
        T sg[W], ta[W];
#pragma unroll
        for (int k = 1; k < W; k++) {
            if (k < deg) {
                sig_pair<T>(sgn * vb(k), sg[k], ta[k]);
            } else {  // padding slot: the identity pair
                sg[k] = T(1);
                ta[k] = T(0);
            }
        }
        T sP[W], sR[W];
        T P = T(1), R = T(0);
#pragma unroll
        for (int k = W - 1; k >= 1; k--) {
            sP[k] = P;
            sR[k] = R;
            R = fma(sg[k], R, ta[k]);
            P = sg[k] * P;
        }
        (void)P;
        (void)R;
        const BodyDen<T> D = body_den<T>(lh, p, q);
        T Pp = T(1), Rp = T(0);
#pragma unroll
        for (int k = 1; k < W; k++) {
            if (k < deg)
                put_fv<T>(fv, ps(k), sgn * body_out_pr<T>(Pp * sP[k], fma(Pp, sR[k], Rp), p, q, D));
            Rp = fma(Pp, ta[k], Rp);
            Pp = Pp * sg[k];
        }
        // the head from the forward product, as in the wider form below, so that a
        // factor's outputs do not depend on the width of the group it lands in
        if ((kind & HEAD_MASK) == HEAD_FREE) put_fv<T>(fv, ps(0), sgn * head_from_pair<T>(Pp, Rp, p, q, logP));
    } else {
        T pP[W], pR[W];
        T P = T(1), R = T(0);
#pragma unroll
        for (int k = 1; k < W; k++) {
            pP[k] = P;
            pR[k] = R;
            if (k < deg) {
                T sk, tk;
                sig_pair<T>(sgn * vb(k), sk, tk);
                R = fma(P, tk, R);
                P = P * sk;
            }
        }
        if ((kind & HEAD_MASK) == HEAD_FREE) put_fv<T>(fv, ps(0), sgn * head_from_pair<T>(P, R, p, q, logP));
        const BodyDen<T> D = body_den<T>(lh, p, q);
        T Ps = T(1), Rs = T(0);
#pragma unroll
        for (int k = W - 1; k >= 1; k--) {
            if (k < deg) {
                T sk, tk;
                sig_pair<T>(sgn * vb(k), sk, tk);
                put_fv<T>(fv, ps(k), sgn * body_out_pr<T>(pP[k] * Ps, fma(pP[k], Rs, pR[k]), p, q, D));
                Rs = fma(sk, Rs, tk);
                Ps = sk * Ps;
            }
        }
    }
}

template <typename T>
__device__ __forceinline__ void factor_group(int w, const T *vb, const uint32_t *ps, int deg, uint8_t kind, T p, T q,
                                             int lane, T *__restrict__ fv) {
    switch (w) {
#define FLBP_W(N) \
    case N:                                                                                           \
        factor_reg<T, N>([&](int k) { return vb[32 * k + lane]; }, [&](int k) { return ps[32 * k + lane]; }, deg, \
                         kind, p, q, fv);                                                                     \
        break;
        FLBP_W(2) FLBP_W(3) FLBP_W(4) FLBP_W(5) FLBP_W(6) FLBP_W(7) FLBP_W(8) FLBP_W(9) FLBP_W(10) FLBP_W(11)
        FLBP_W(12) FLBP_W(13) FLBP_W(14) FLBP_W(15) FLBP_W(16)
#undef FLBP_W
        default: break;
    }
}
static_assert(kSellFactorDegree == 16, "factor_group instantiates widths 2..16");

// Pair of a warp's lanes 0..lane (forward) combined with a shuffle scan.
template <typename T>
__device__ __forceinline__ void warp_scan_pairs(T &P, T &R, int lane) {
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const T oP = __shfl_up_sync(0xffffffffu, P, off), oR = __shfl_up_sync(0xffffffffu, R, off);
        if (lane >= off) {
            R = fma(oP, R, oR);
            P = oP * P;
        }
    }
}

// Pair of a warp's lanes lane..31 (backward).
template <typename T>
__device__ __forceinline__ void warp_rscan_pairs(T &P, T &R, int lane) {
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const T oP = __shfl_down_sync(0xffffffffu, P, off), oR = __shfl_down_sync(0xffffffffu, R, off);
        if (lane + off < 32) {
            R = fma(P, oR, R);
            P = P * oP;
        }
    }
}

// One large factor of a staged big tile, one warp, with at most 32 NV body
// slots: vb[0] / ps[0] are the head's message and fv position, vb[1 + k] /
// ps[1 + k] those of body slot k. Lane l holds body slots [l NV, l NV + NV)
// as (sigma, tau) pairs. Each slot's leave-one-out pair is
//   (lanes before) o (own earlier slots) o (own later slots) o (lanes after),
// from two shuffle scans over the lanes' pairs; no division, exact zeros
// stay exact.
template <typename T, int NV>
__device__ __forceinline__ void factor_tile_big(const T *vb, const uint32_t *ps, uint32_t nbody, uint8_t kind, T p, T q,
                                                int lane, T *__restrict__ fv) {
    const T sgn = (kind & KIND_OR) ? T(-1) : T(1);
    const uint32_t k0 = (uint32_t)lane * NV;  // first body slot of this lane (body index)
    T sg[NV], ta[NV];
#pragma unroll
    for (int u = 0; u < NV; u++) {
        const bool in = k0 + u < nbody;
        const T x = in ? vb[1 + k0 + u] : T(0);
        if (in) {
            sig_pair<T>(sgn * x, sg[u], ta[u]);
        } else {
            sg[u] = T(1);
            ta[u] = T(0);
        }
    }
    const T vh = vb[0];
    T lP = T(1), lR = T(0);  // this lane's slots
#pragma unroll
    for (int u = 0; u < NV; u++) {
        lR = fma(lP, ta[u], lR);
        lP = lP * sg[u];
    }
    T fP = lP, fR = lR, bP = lP, bR = lR;
    warp_scan_pairs<T>(fP, fR, lane);
    warp_rscan_pairs<T>(bP, bR, lane);
    const T P = __shfl_sync(0xffffffffu, fP, 31), R = __shfl_sync(0xffffffffu, fR, 31);
    T eP = __shfl_up_sync(0xffffffffu, fP, 1), eR = __shfl_up_sync(0xffffffffu, fR, 1);  // lanes before
    T xP = __shfl_down_sync(0xffffffffu, bP, 1), xR = __shfl_down_sync(0xffffffffu, bR, 1);  // lanes after
    if (lane == 0) eP = T(1), eR = T(0);
    if (lane == 31) xP = T(1), xR = T(0);
    if ((kind & HEAD_MASK) == HEAD_FREE) {
        auto logP = [&]() {  // rare: whole-body log-sigmoid sum, by the whole warp, -inf terms counted apart
            typedef AccOps<typename WideAcc<T>::type> O;
            typename WideAcc<T>::type l = O::zero();
            int nz = 0;
            for (uint32_t k = lane; k < nbody; k += 32) {
                const T ls = log_sigmoid<T>(sgn * vb[1 + k]);
                if (ls == -Num<T>::inf()) nz++;
                else O::add(l, ls);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                O::combine(l, O::shfl_xor(l, o));
                nz += __shfl_xor_sync(0xffffffffu, nz, o);
            }
            return nz ? -Num<T>::inf() : (T)O::value(l);
        };
        const T o = sgn * head_from_pair<T>(P, R, p, q, logP);
        if (lane == 0) put_fv<T>(fv, ps[0], o);
    }
    const BodyDen<T> D = body_den<T>(sgn * head_effective<T>(kind, vh), p, q);
    // own later slots, then the lanes after: suffix pairs, backwards
    T sP[NV], sR[NV];
    T cP = xP, cR = xR;
#pragma unroll
    for (int u = NV - 1; u >= 0; u--) {
        sP[u] = cP;
        sR[u] = cR;
        cR = fma(sg[u], cR, ta[u]);
        cP = sg[u] * cP;
    }
    T Pp = eP, Rp = eR;
#pragma unroll
    for (int u = 0; u < NV; u++) {
        if (k0 + u < nbody)
            put_fv<T>(fv, ps[1 + k0 + u], sgn * body_out_pr<T>(Pp * sP[u], fma(Pp, sR[u], Rp), p, q, D));
        Rp = fma(Pp, ta[u], Rp);
        Pp = Pp * sg[u];
    }
}

// A factor too large for a tile (big factor b, internal index nf_sell + b),
// spread over all consumer threads of a block (called by all of them): a
// log-sigmoid sum of the body (WideAcc) with a count of -inf terms, reduced
// over the block in a fixed order, then every slot removes its own term.
template <typename T>
__device__ void factor_block_huge(const FactorArgs &a, uint32_t b, int tid, const T *__restrict__ vf,
                                  T *__restrict__ fv, typename WideAcc<T>::type *s_l, int *s_nz) {
    typedef typename WideAcc<T>::type A;
    typedef AccOps<A> O;
    const uint32_t fi = a.nf_sell + b;
    if (a.f_graph && a.gdone[a.f_graph[fi]]) return;  // batched solve: its graph has stopped (same for all)
    const uint32_t s0 = a.fb_off[b], s1 = s0 + a.fb_deg[b];
    const uint8_t kind = a.f_kind[fi];
    const T *pq = reinterpret_cast<const T *>(a.f_pq);
    const T p = pq[2 * fi], q = pq[2 * fi + 1];
    const T s = (kind & KIND_OR) ? T(-1) : T(1);
    const T inf = Num<T>::inf();
    const int lane = tid & 31, wid = tid >> 5;
    A L = O::zero();
    int nz = 0;
    for (uint32_t k = s0 + 1 + tid; k < s1; k += kConsumers) {
        const T ls = log_sigmoid<T>(s * vf[k]);
        if (ls == -inf) nz++;
        else O::add(L, ls);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        O::combine(L, O::shfl_xor(L, o));
        nz += __shfl_xor_sync(0xffffffffu, nz, o);
    }
    if (lane == 0) {
        s_l[wid] = L;
        s_nz[wid] = nz;
    }
    consumer_sync();
    L = O::zero();
    nz = 0;
    for (int w = 0; w < kConsumerWarps; w++) {
        O::combine(L, s_l[w]);
        nz += s_nz[w];
    }
    consumer_sync();  // the partials are reused by the next factor
    if ((kind & HEAD_MASK) == HEAD_FREE && tid == 0)
        put_fv<T>(fv, a.f_pos[s0], s * head_out<T>(nz ? -inf : (T)O::value(L), p, q, Num<T>::log(p)));
    const BodyDen<T> D = body_den<T>(s * head_effective<T>(kind, vf[s0]), p, q);
    for (uint32_t k = s0 + 1 + tid; k < s1; k += kConsumers) {
        const T ls = log_sigmoid<T>(s * vf[k]);
        const bool z = (ls == -inf);
        const T lo = (nz - (int)z) ? -inf : (z ? (T)O::value(L) : O::template excl<T>(L, ls));
        put_fv<T>(fv, a.f_pos[k], s * body_out<T>(lo, p, q, D));
    }
}

// Item `wid` of a staged big tile: dispatch on its body size.
template <typename T>
__device__ __forceinline__ void factor_tile_item(const T *vb, const uint32_t *ps, uint32_t deg, uint8_t kind, T p, T q,
                                                 int lane, T *__restrict__ fv) {
    const uint32_t nbody = deg - 1;
    if (nbody <= 32) factor_tile_big<T, 1>(vb, ps, nbody, kind, p, q, lane, fv);
    else if (nbody <= 64) factor_tile_big<T, 2>(vb, ps, nbody, kind, p, q, lane, fv);
    else if (nbody <= 128) factor_tile_big<T, 4>(vb, ps, nbody, kind, p, q, lane, fv);
    else factor_tile_big<T, 8>(vb, ps, nbody, kind, p, q, lane, fv);
}
static_assert(kBigFactorBody == 256, "factor_tile_item covers bodies of up to 256 slots");

// Opens a sweep (thread 0 of block 0 of the factor pass, either form): sweep
// counters, damping weight of the constant priors, residual reset.
__device__ __forceinline__ void sweep_open(Ctl *ctl) {
    unsigned long long now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    if (ctl->run_sweeps == 0) ctl->t_start_ns = now;
    ctl->t += 1;
    ctl->run_sweeps += 1;
    ctl->pscale = (ctl->damping == 0.0) ? 1.0 : 1.0 - pow(ctl->damping, (double)ctl->t);
    ctl->maxdiff_bits = 0ull;
    ctl->nonconv = 0ull;
    ctl->arrive = 0u;
    ctl->vnext = 0u;  // the variable pass of this sweep starts after this kernel
}

// Factor pass. Every block runs a STAGES-deep pipeline over its tiles (tile
// blockIdx.x + i gridDim.x): warp kConsumerWarps (one lane) is the producer -
// it waits until the consumer warps have released a stage and bulk-loads the
// next tile (messages, fv positions, per-factor constants) into it; consumer
// warp j evaluates item j of the staged tile - the 32 factors of sliced-ELL
// group j, one per lane, or big factor j with the whole warp - and scatters
// the outputs to fv. Factors too large for a tile are taken first, one per
// warp, while the producer's first loads are in flight.
// GID: the kernel of batched solves (a.f_graph set), which stages every
// factor's graph; without it a.f_graph must be null.
template <typename T, int STAGES, bool GID>
__global__ void __launch_bounds__(kBlockThreadsDev) factor_pass_kernel(FactorArgs a, const T *__restrict__ vf,
                                                                       T *__restrict__ fv, Ctl *ctl) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES];
    typedef FactorStage<T, GID> FS;
    if (*(volatile int *)&ctl->done) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) sweep_open(ctl);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t n_tiles = a.n_tiles;
    __shared__ uint32_t s_done[kDoneWords];  // batched solves: stopped graphs
    if (a.f_graph) load_done_bits(s_done, a.gdone, a.n_graphs, lane, wid, blockDim.x >> 5);
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kConsumerWarps);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (wid == kConsumerWarps) {  // producer warp
        const T *pq_g = reinterpret_cast<const T *>(a.f_pq);
        auto fill = [&](unsigned char *st, uint32_t *gb, uint64_t *bar) {
            const uint32_t g0 = gb[0], n = gb[1] & ~kBigTileFlag;
            const uint32_t ns = gb[2 + n] - gb[2];
            if (gb[1] & kBigTileFlag) {  // big factors: degrees, kinds and (p, q) from the tile's constants
                const size_t bt = gb[kHdrWords - 1];
                constexpr uint32_t cbytes = 4u * kTileGroups + kTileGroups + 2u * kTileGroups * (uint32_t)sizeof(T);
                mbar_arrive_expect_tx(bar, ns * (uint32_t)(sizeof(T) + 4) + cbytes);
                bulk_g2s(st + FS::deg, a.bt_deg + kTileGroups * bt, 4u * kTileGroups, bar);
                bulk_g2s(st + FS::kind, a.bt_kind + kTileGroups * bt, kTileGroups, bar);
                bulk_g2s(st + FS::pq, reinterpret_cast<const T *>(a.bt_pq) + 2 * kTileGroups * bt,
                         2u * kTileGroups * (uint32_t)sizeof(T), bar);
            } else {
                const uint32_t items = 32u * n;
                const bool gid = GID && a.f_graph;
                mbar_arrive_expect_tx(bar, ns * (uint32_t)(sizeof(T) + 4) + 2u * items +
                                               2u * items * (uint32_t)sizeof(T) + (gid ? 4u * items : 0u));
                bulk_g2s(st + FS::deg, a.f_deg + 32ull * g0, items, bar);
                bulk_g2s(st + FS::kind, a.f_kind + 32ull * g0, items, bar);
                bulk_g2s(st + FS::pq, pq_g + 64ull * g0, 2u * items * (uint32_t)sizeof(T), bar);
                if (gid) bulk_g2s(st + FS::gid, a.f_graph + 32ull * g0, 4u * items, bar);
            }
            if (ns) {
                bulk_g2s(st + FS::vbuf, vf + gb[2], ns * (uint32_t)sizeof(T), bar);
                bulk_g2s(st + FS::pos, a.f_pos + gb[2], ns * 4u, bar);
            }
        };
        produce_tiles<STAGES>(a.thdr, a.f_graph ? a.trange : nullptr, a.tile_list, a.tile_off, a.act_list, a.n_act,
                              s_done, a.gdone, n_tiles, &ctl->fnext, smem, FS::bytes, full, empty, lane, ctl, fill);
        return;
    }

    {  // factors too large for a tile first, one per block, while the producer's first loads are in flight
        __shared__ typename WideAcc<T>::type s_l[kConsumerWarps];
        __shared__ int s_nz[kConsumerWarps];
        for (uint32_t b = blockIdx.x; b < a.nf_huge; b += gridDim.x)
            factor_block_huge<T>(a, b, threadIdx.x, vf, fv, s_l, s_nz);
    }
    for (uint32_t it = 0;; it++) {
        const int s = (int)(it % STAGES);
        if (!warp_wait_stage(&full[s], (it / STAGES) & 1u)) {
            if (lane == 0) record_timeout(ctl);
            return;
        }
        const unsigned char *st = smem + (size_t)s * FS::bytes;
        const uint32_t *gb = reinterpret_cast<const uint32_t *>(st + FS::hdr);
        if (gb[1] == kEndTile) break;
        if (gb[1] & kBigTileFlag) {  // one big factor per warp
            if ((uint32_t)wid < (gb[1] & ~kBigTileFlag) &&
                !(a.f_graph && graph_done(s_done, a.gdone, a.f_graph[a.nf_sell + gb[0] + wid]))) {
                const uint32_t base = gb[2 + wid] - gb[2];
                const T *pq = reinterpret_cast<const T *>(st + FS::pq);
                factor_tile_item<T>(reinterpret_cast<const T *>(st + FS::vbuf) + base,
                                    reinterpret_cast<const uint32_t *>(st + FS::pos) + base,
                                    reinterpret_cast<const uint32_t *>(st + FS::deg)[wid], st[FS::kind + wid],
                                    pq[2 * wid], pq[2 * wid + 1], lane, fv);
            }
        } else if ((uint32_t)wid < gb[1]) {
            const uint32_t base = gb[2 + wid] - gb[2], f = 32u * wid + lane;
            const int w = (int)((gb[3 + wid] - gb[2 + wid]) >> 5);
            int deg = st[FS::deg + f];
            if (GID && a.f_graph && graph_done(s_done, a.gdone, reinterpret_cast<const uint32_t *>(st + FS::gid)[f]))
                deg = 0;  // stopped graph
            const T *pq = reinterpret_cast<const T *>(st + FS::pq);
            if (deg > 0)
                factor_group<T>(w, reinterpret_cast<const T *>(st + FS::vbuf) + base,
                                reinterpret_cast<const uint32_t *>(st + FS::pos) + base, deg, st[FS::kind + f],
                                pq[2 * f], pq[2 * f + 1], lane, fv);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
}

// Leave-one-out message of a variable to the factor of one entry: remove
// `x` from (S, npos, nneg); both kinds of zero left -> (0.5,0.5); otherwise
// the remaining zero wins (causal_bp_parall.cu:74-90).
template <typename T, typename A>
__device__ __forceinline__ T excl_msg(const A &S, int npos, int nneg, T x) {
    const T inf = Num<T>::inf();
    const bool fin = !(x == inf || x == -inf);
    if (x == inf) npos--;
    else if (x == -inf) nneg--;
    if (npos > 0 && nneg > 0) return T(0);
    if (npos > 0) return inf;
    if (nneg > 0) return -inf;
    return fin ? AccOps<A>::template excl<T>(S, x) : (T)AccOps<A>::value(S);
}

// Belief P(x=1): b_s = prod_s * [zeros_s == 0], belief = b1 / (b0 + b1)
// (causal_bp_seq.cu:102-111, causal_bp.cu:510-514).
__device__ __forceinline__ double belief_of(double S, int npos, int nneg) {
    if (npos > 0 && nneg > 0) return __longlong_as_double(0x7ff8000000000000ll);
    if (npos > 0) return 1.0;
    if (nneg > 0) return 0.0;
    return 1.0 / (1.0 + ::exp(-S));
}

// BMODE: 0 no beliefs; 1 beliefs + residual; 2 beliefs + residual + count +
// history; 3 beliefs only (no residual, no history); 4 beliefs + residual of
// a batched solve (per-graph stop rules).
template <int BMODE>
__device__ __forceinline__ double var_finish(const VarArgs &a, uint32_t v, double S, int npos, int nneg, double tol,
                                             double bold, unsigned long long &cnt) {
    double diff = 0.0;
    if (BMODE != 0) {
        const double b = belief_of(S, npos, nneg);
        if (BMODE == 1 || BMODE == 2 || BMODE == 4) {
            const double dd = fabs(bold - b);
            diff = dd;
            if (BMODE == 2) {
                if (dd > tol) cnt++;
                if (isfinite(b)) {
                    uint32_t slot = a.hist_next[v];
                    a.hist[(size_t)slot * (a.nv_sell + a.nv_big) + v] = b;
                    if (++slot == a.hist_len) slot = 0;
                    a.hist_next[v] = slot;
                    if (a.hist_count[v] < a.hist_len) a.hist_count[v]++;
                }
            }
        }
        a.belief[v] = b;
    }
    return diff;
}

// Prior of internal variable i: its finite constant log-odds times the
// damping weight pscale (FP32 engines: in float; an accumulator A of a
// wider type receives it exactly), and its +-inf counts.
template <typename T, typename A>
__device__ __forceinline__ void decode_prior(const void *pr, uint32_t i, double pscale, A &S, int &npos, int &nneg) {
    uint32_t cnt;
    if (sizeof(T) == 4) {
        const uint2 x = reinterpret_cast<const uint2 *>(pr)[i];
        S = AccOps<A>::of(__uint_as_float(x.x) * (float)pscale);
        cnt = x.y;
    } else {
        const uint4 x = reinterpret_cast<const uint4 *>(pr)[i];
        S = AccOps<A>::of(__hiloint2double((int)x.y, (int)x.x) * pscale);
        cnt = x.z;
    }
    npos = (int)(cnt & 0xffffu);
    nneg = (int)((cnt >> 16) & 0x7fffu);  // bit 31: the variable has a folded finite constant (adjoint)
}


// Incoming f->v message of one entry: the new one, or with damping the mix
// of the new one with the previous damped one, which is then stored back.
template <typename T, bool DAMP>
__device__ __forceinline__ T take_fv(T x, T old, T d) {
    return DAMP ? damp_mix(x, old, d) : x;
}

// One big variable of a staged big tile, one warp: its entries are en[k],
// x[k] (and xo[k], the previous damped messages), k < deg, in the stage;
// fvd_run is its run of damped messages in global memory.
template <typename T, int BMODE, bool WRITE_VF, bool DAMP>
__device__ __forceinline__ double var_tile_big(const VarArgs &a, uint32_t v, uint32_t deg, const uint32_t *en, T *x,
                                               const T *xo, T *__restrict__ fvd_run, const void *prior, uint32_t pidx,
                                               int lane, T *__restrict__ vf, T d, double pscale, double tol,
                                               unsigned long long &cnt) {
    typedef typename WideAcc<T>::type A;
    typedef AccOps<A> O;
    const T inf = Num<T>::inf();
    A S = O::zero();
    int npos = 0, nneg = 0;
    for (uint32_t k = lane; k < deg; k += 32) {
        T xv = x[k];
        if (DAMP) {
            xv = take_fv<T, DAMP>(xv, xo[k], d);
            x[k] = xv;
            fvd_run[k] = xv;
        }
        if (xv == inf) npos++;
        else if (xv == -inf) nneg++;
        else O::add(S, xv);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        O::combine(S, O::shfl_xor(S, o));
        npos += __shfl_xor_sync(0xffffffffu, npos, o);
        nneg += __shfl_xor_sync(0xffffffffu, nneg, o);
    }
    A S0;
    int p0, n0;
    decode_prior<T>(prior, pidx, pscale, S0, p0, n0);
    O::combine(S, S0);
    npos += p0;
    nneg += n0;
    if (WRITE_VF) {
        for (uint32_t k = lane; k < deg; k += 32) {
            const uint32_t e = en[k];
            if (e != kSentinel) vf[e] = excl_msg<T>(S, npos, nneg, x[k]);
        }
    }
    constexpr bool RESID = (BMODE == 1 || BMODE == 2 || BMODE == 4);
    return (lane == 0) ? var_finish<BMODE>(a, v, O::value(S), npos, nneg, tol, RESID ? a.belief[v] : 0.0, cnt) : 0.0;
}

// A variable too large for a tile (big variable b, internal index
// nv_sell + b), spread over all consumer threads of a block (called by all
// of them): a WideAcc sum with +-inf counts reduced over the block in a fixed
// order, then every entry's leave-one-out message. Returns the belief change
// on thread 0 (0 elsewhere).
template <typename T, int BMODE, bool WRITE_VF, bool DAMP>
__device__ double var_block_huge(const VarArgs &a, uint32_t b, int tid, const T *__restrict__ fv,
                                 T *__restrict__ vf, T *__restrict__ fvd, T d, double pscale, double tol,
                                 unsigned long long &cnt, typename WideAcc<T>::type *s_s, int *s_np, int *s_nn) {
    typedef typename WideAcc<T>::type A;
    typedef AccOps<A> O;
    constexpr bool RESID = (BMODE == 1 || BMODE == 2 || BMODE == 4);
    const uint32_t v = a.nv_sell + b, k0 = a.vb_off[b], k1 = k0 + a.vb_deg[b];
    const T inf = Num<T>::inf();
    const T *src = DAMP ? fvd : fv;  // after the first loop, fvd holds the messages in use
    const int lane = tid & 31, wid = tid >> 5;
    A S = O::zero();
    int npos = 0, nneg = 0;
    for (uint32_t k = k0 + tid; k < k1; k += kConsumers) {
        T x = fv[k];
        if (DAMP) {
            x = take_fv<T, DAMP>(x, fvd[k], d);
            fvd[k] = x;
        }
        if (x == inf) npos++;
        else if (x == -inf) nneg++;
        else O::add(S, x);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        O::combine(S, O::shfl_xor(S, o));
        npos += __shfl_xor_sync(0xffffffffu, npos, o);
        nneg += __shfl_xor_sync(0xffffffffu, nneg, o);
    }
    if (lane == 0) {
        s_s[wid] = S;
        s_np[wid] = npos;
        s_nn[wid] = nneg;
    }
    consumer_sync();
    S = O::zero();
    npos = nneg = 0;
    for (int w = 0; w < kConsumerWarps; w++) {
        O::combine(S, s_s[w]);
        npos += s_np[w];
        nneg += s_nn[w];
    }
    consumer_sync();  // the partials are reused by the next variable
    A S0;
    int p0, n0;
    decode_prior<T>(a.prior, v, pscale, S0, p0, n0);
    O::combine(S, S0);
    npos += p0;
    nneg += n0;
    if (WRITE_VF) {
        for (uint32_t k = k0 + tid; k < k1; k += kConsumers) {
            const uint32_t e = a.v_ent[k];
            if (e != kSentinel) vf[e] = excl_msg<T>(S, npos, nneg, src[k]);
        }
    }
    return (tid == 0) ? var_finish<BMODE>(a, v, O::value(S), npos, nneg, tol, RESID ? a.belief[v] : 0.0, cnt) : 0.0;
}

__device__ __forceinline__ double warp_max(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// Stop rules evaluated after a sweep by the last block of the variable pass,
// so that the next launches see ctl->done.
static __device__ void stop_rules(Ctl *ctl) {
    const double maxdiff = __longlong_as_double((long long)ctl->maxdiff_bits);
    ctl->maxdiff = maxdiff;
    unsigned long long now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    const double elapsed = (double)(now - ctl->t_start_ns);
    const long long n = ctl->run_sweeps;
    if (ctl->status != 0) {  // a device wait gave up: stop the run
        ctl->done = 1;
        ctl->reason = FLBP_DIVERGED;
        return;
    }
    if (ctl->mode == 1) {  // causal_bp.cu:866
        const long long iters = ctl->iters0 + n;
        const bool cont = iters < ctl->maxiter && maxdiff > ctl->tol && elapsed < ctl->maxtime_ns;
        if (!cont) {
            ctl->done = 1;
            ctl->reason = (maxdiff > ctl->tol) ? FLBP_DIVERGED : FLBP_ALL_CONVERGED;
        }
    } else if (ctl->mode == 2) {  // causal_bp.cu:1037-1054, evaluated for the next numIters
        const double frac = (double)ctl->nonconv / (double)ctl->n_vars;
        ctl->frac = frac;
        if (n >= ctl->min_iters)
            ctl->node_frac_tol = (double)(n - ctl->min_iters) / (double)(ctl->max_iters - ctl->min_iters);
        if (maxdiff <= ctl->tol) {
            ctl->done = 1;
            ctl->reason = FLBP_ALL_CONVERGED;
        } else if (n > ctl->min_iters && frac < ctl->node_frac_tol) {
            ctl->done = 1;
            ctl->reason = FLBP_BIG_FRAC_CONVERGED;
        } else if (n > ctl->max_iters) {
            ctl->done = 1;
            ctl->reason = FLBP_DIVERGED;
        } else if (elapsed > ctl->maxtime_ns) {
            ctl->done = 1;
            ctl->reason = FLBP_DIVERGED;
        }
    }
}

// Per-graph stop rules of a batched tolerance solve (the rule of stop_rules
// mode 1 applied to each graph: it stops after the sweep in which no belief
// moved by more than tol, or after maxiter sweeps; it is then frozen), run by
// every thread of the last block of the variable pass. The run ends when all
// graphs have stopped, or at maxtime.
static __device__ void batch_stop_rules(Ctl *ctl, const VarArgs &a) {
    __shared__ int s_open;
    if (threadIdx.x == 0) s_open = 0;
    __syncthreads();
    const uint32_t G = a.n_graphs;
    int *done = a.gstate, *moved = a.gstate + G, *iters = a.gstate + 2 * G, *reason = a.gstate + 3 * G;
    int open = 0;
    for (uint32_t g = threadIdx.x; g < G; g += blockDim.x) {
        if (done[g]) continue;
        iters[g] += 1;
        if (!moved[g]) {
            done[g] = 1;
            reason[g] = FLBP_ALL_CONVERGED;
        } else if (ctl->iters0 + iters[g] >= ctl->maxiter) {
            done[g] = 1;
            reason[g] = FLBP_DIVERGED;
        } else {
            open++;
        }
        moved[g] = 0;
    }
    if (open) atomicAdd(&s_open, open);
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->maxdiff = __longlong_as_double((long long)ctl->maxdiff_bits);
        unsigned long long now;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
        if (ctl->status != 0 || s_open == 0 || (double)(now - ctl->t_start_ns) >= ctl->maxtime_ns) {
            ctl->done = 1;
            ctl->reason = (s_open == 0 && ctl->status == 0) ? FLBP_ALL_CONVERGED : FLBP_DIVERGED;
        }
        __threadfence();
    }
}

// Batched solves, before a sweep's factor pass: per tile of each pass,
// whether its graph range holds a live graph (ranges of more than 32
// graphs count as live). The engine compacts the flags into the passes'
// tile lists, in tile order.
static __global__ void live_tile_flags_kernel(const uint2 *ftr, uint32_t nft, const uint2 *vtr, uint32_t nvt,
                                              const int *done, uint8_t *fflag, uint8_t *vflag, const Ctl *ctl) {
    if (*(volatile const int *)&ctl->done) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nft + nvt; i += gridDim.x * blockDim.x) {
        const uint2 r = i < nft ? ftr[i] : vtr[i - nft];
        bool stopped = r.y >= r.x && r.y - r.x <= 32;
        for (uint32_t g = r.x; stopped && g <= r.y; g++) stopped = done[g] != 0;
        if (i < nft) fflag[i] = stopped ? 0 : 1;
        else vflag[i - nft] = stopped ? 0 : 1;
    }
}

// Batched solves: graph g had a belief move by more than tol this sweep.
// Graphs below kMovedWords * 32 are collected in a shared-memory bit set and
// written out once per block at the end of the pass (a store per graph and
// block instead of one per variable, which would all hit a few addresses).
constexpr int kMovedWords = 128;
__device__ __forceinline__ void mark_moved(uint32_t *s_moved, const VarArgs &a, uint32_t g) {
    if (g < 32u * kMovedWords) {
        const uint32_t bit = 1u << (g & 31);
        if (!(s_moved[g >> 5] & bit)) atomicOr(&s_moved[g >> 5], bit);
    } else {
        a.gstate[a.n_graphs + g] = 1;
    }
}

// End of a variable pass with a residual (BMODE 1, 2, 4), called by every
// thread of the block: the block's maximum belief change (and count of
// changes above tol) into the control block, the batched per-graph flags,
// and in the last block to finish, the run's stop rules.
template <int BMODE>
__device__ __forceinline__ void var_close(const VarArgs &a, Ctl *ctl, double dmax, unsigned long long cnt,
                                          const uint32_t *s_moved, int lane, int wid) {
    __shared__ double s_max[kConsumerWarps + 1];
    __shared__ unsigned long long s_cnt[kConsumerWarps + 1];
    __shared__ bool s_last;
    dmax = warp_max(dmax);
    cnt = warp_sum(cnt);
    if (lane == 0) {
        s_max[wid] = dmax;
        s_cnt[wid] = cnt;
    }
    __syncthreads();
    if (BMODE == 4) {  // the block's per-graph flags, one store per graph
        const uint32_t words = min((a.n_graphs + 31) / 32, (uint32_t)kMovedWords);
        for (uint32_t w = threadIdx.x; w < words; w += blockDim.x) {
            uint32_t bits = s_moved[w];
            while (bits) {
                const int b = __ffs(bits) - 1;
                bits &= bits - 1;
                a.gstate[a.n_graphs + 32 * w + b] = 1;
            }
        }
        __threadfence();
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double m = 0.0;
        unsigned long long c = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) {
            m = fmax(m, s_max[i]);
            c += s_cnt[i];
        }
        atomicMax(&ctl->maxdiff_bits, (unsigned long long)__double_as_longlong(m));
        if (BMODE == 2) atomicAdd(&ctl->nonconv, c);
        __threadfence();
        const unsigned int prev = atomicAdd(&ctl->arrive, 1u);
        s_last = (prev == gridDim.x * gridDim.y - 1);
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        if (BMODE == 4) batch_stop_rules(ctl, a);  // the whole block
        else if (threadIdx.x == 0) stop_rules(ctl);
    }
}

// Variable pass, warp-specialised like the factor pass: the producer warp
// bulk-loads each tile's entries (factor-side slots), incoming messages, the
// previous damped messages (with damping), priors and (with a residual)
// previous beliefs; consumer warp j takes group j, one variable per lane:
// the FP64 sum of its incoming messages with +-inf counts and its prior,
// belief and residual, then the leave-one-out messages scattered to vf; a
// big variable of a big tile takes the whole warp. Variables too large for a
// tile are taken first, one per warp. With BMODE 1/2 the
// block maxima of |belief change| are combined with an atomic max and the
// last block to finish applies the stop rules. DAMP mixes each new message
// with the previous damped one (fvd) and stores the result back to fvd.
template <typename T, int BMODE, bool WRITE_VF, bool DAMP, int STAGES>
__global__ void __launch_bounds__(kBlockThreadsDev) var_pass_kernel(VarArgs a, const T *__restrict__ fv,
                                                                    T *__restrict__ vf, T *__restrict__ fvd, T d,
                                                                    Ctl *ctl) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES];
    typedef VarStage<T, DAMP> VS;
    constexpr bool RESID = (BMODE == 1 || BMODE == 2 || BMODE == 4);
    constexpr uint32_t psz = sizeof(T) == 4 ? 8u : 16u;
    if (*(volatile int *)&ctl->done) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl->fnext = 0u;  // the next factor pass starts after this kernel
    const double pscale = ctl->pscale;
    const double tol = ctl->tol;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t n_tiles = a.n_tiles;
    const T inf = Num<T>::inf();
    double dmax = 0.0;
    unsigned long long cnt = 0;
    __shared__ uint32_t s_moved[BMODE == 4 ? kMovedWords : 1];  // batched: graphs with a belief moved > tol
    __shared__ uint32_t s_done[kDoneWords];                      // batched: stopped graphs
    if (BMODE == 4)
        for (int w = threadIdx.x; w < kMovedWords; w += blockDim.x) s_moved[w] = 0u;
    if (a.v_graph) load_done_bits(s_done, a.gstate, a.n_graphs, lane, wid, blockDim.x >> 5);
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kConsumerWarps);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (wid == kConsumerWarps) {  // producer warp
        auto fill = [&](unsigned char *st, uint32_t *gb, uint64_t *bar) {
            const uint32_t g0 = gb[0], n = gb[1] & ~kBigTileFlag;
            const uint32_t ns = gb[2 + n] - gb[2];
            const uint32_t mbytes = ns * (4u + (DAMP ? 2u : 1u) * (uint32_t)sizeof(T));
            if (gb[1] & kBigTileFlag) {  // big variables: entry counts and priors from the tile's constants
                const size_t bt = gb[kHdrWords - 1];
                mbar_arrive_expect_tx(bar, mbytes + psz * kTileGroups + 4u * kTileGroups);
                bulk_g2s(st + VS::prior, reinterpret_cast<const unsigned char *>(a.bt_prior) + psz * kTileGroups * bt,
                         psz * kTileGroups, bar);
                bulk_g2s(st + VS::bold, a.bt_deg + kTileGroups * bt, 4u * kTileGroups, bar);
            } else {
                const uint32_t items = 32u * n;
                mbar_arrive_expect_tx(bar, mbytes + psz * items + (RESID ? 8u * items : 0u) + (a.v_graph ? 4u * items : 0u));
                bulk_g2s(st + VS::prior, reinterpret_cast<const unsigned char *>(a.prior) + 32ull * g0 * psz,
                         psz * items, bar);
                if (RESID) bulk_g2s(st + VS::bold, a.belief + 32ull * g0, 8u * items, bar);
                if (a.v_graph) bulk_g2s(st + VS::gid, a.v_graph + 32ull * g0, 4u * items, bar);
            }
            if (ns) {
                bulk_g2s(st + VS::ent, a.v_ent + gb[2], ns * 4u, bar);
                bulk_g2s(st + VS::x, fv + gb[2], ns * (uint32_t)sizeof(T), bar);
                if (DAMP) bulk_g2s(st + VS::xo, fvd + gb[2], ns * (uint32_t)sizeof(T), bar);
            }
        };
        produce_tiles<STAGES>(a.thdr, a.v_graph ? a.trange : nullptr, nullptr, nullptr, a.act_list, a.n_act, s_done,
                              a.gstate, n_tiles, &ctl->vnext, smem, VS::bytes, full, empty, lane, ctl, fill);
    } else {  // consumer warps: variables too large for a tile first
        {  // one per block
            __shared__ typename WideAcc<T>::type s_s[kConsumerWarps];
            __shared__ int s_np[kConsumerWarps], s_nn[kConsumerWarps];
            for (uint32_t b = blockIdx.x; b < a.nv_huge; b += gridDim.x) {
                const uint32_t g = a.v_graph ? a.v_graph[a.nv_sell + b] : 0;
                if (a.v_graph && graph_done(s_done, a.gstate, g)) continue;  // stopped graph (batched solve)
                const double dd = var_block_huge<T, BMODE, WRITE_VF, DAMP>(a, b, threadIdx.x, fv, vf, fvd, d, pscale,
                                                                           tol, cnt, s_s, s_np, s_nn);
                dmax = fmax(dmax, dd);
                if (BMODE == 4 && dd > tol) mark_moved(s_moved, a, g);
            }
        }
        for (uint32_t it = 0;; it++) {
            const int s = (int)(it % STAGES);
            if (!warp_wait_stage(&full[s], (it / STAGES) & 1u)) {
                if (lane == 0) record_timeout(ctl);
                break;
            }
            unsigned char *st = smem + (size_t)s * VS::bytes;
            const uint32_t *gb = reinterpret_cast<const uint32_t *>(st + VS::hdr);
            if (gb[1] == kEndTile) break;
            if (gb[1] & kBigTileFlag) {  // one big variable per warp
                const uint32_t v = a.nv_sell + gb[0] + wid;
                const uint32_t g = a.v_graph && (uint32_t)wid < (gb[1] & ~kBigTileFlag) ? a.v_graph[v] : 0;
                if ((uint32_t)wid < (gb[1] & ~kBigTileFlag) && !(a.v_graph && graph_done(s_done, a.gstate, g))) {
                    const uint32_t base = gb[2 + wid] - gb[2];
                    const double dd = var_tile_big<T, BMODE, WRITE_VF, DAMP>(
                        a, v, reinterpret_cast<const uint32_t *>(st + VS::bold)[wid],
                        reinterpret_cast<const uint32_t *>(st + VS::ent) + base, reinterpret_cast<T *>(st + VS::x) + base,
                        reinterpret_cast<const T *>(st + VS::xo) + base, fvd + gb[2] + base, st + VS::prior, wid, lane,
                        vf, d, pscale, tol, cnt);
                    dmax = fmax(dmax, dd);
                    if (BMODE == 4 && dd > tol) mark_moved(s_moved, a, g);
                }
            } else if ((uint32_t)wid < gb[1]) {
                const uint32_t base = gb[2 + wid] - gb[2];
                const int w = (int)((gb[3 + wid] - gb[2 + wid]) >> 5);
                const uint32_t t = 32u * wid + lane, v = 32u * gb[0] + t;
                const uint32_t *en = reinterpret_cast<const uint32_t *>(st + VS::ent) + base;
                T *x = reinterpret_cast<T *>(st + VS::x) + base;
                const T *xo = reinterpret_cast<const T *>(st + VS::xo) + base;
                const uint32_t g = a.v_graph ? reinterpret_cast<const uint32_t *>(st + VS::gid)[t] : 0;
                const bool live = !(a.v_graph && graph_done(s_done, a.gstate, g));  // stopped graph: no work
                const int wl = live ? w : 0;
                typedef typename NarrowAcc<T>::type A;
                A S = AccOps<A>::zero();
                int npos = 0, nneg = 0;
                if (v < a.nv_sell) decode_prior<T>(st + VS::prior, t, pscale, S, npos, nneg);
                for (int k = 0; k < wl; k++) {  // padding entries hold 0
                    const int i = 32 * k + lane;
                    T xv = x[i];
                    if (DAMP) {
                        xv = take_fv<T, DAMP>(xv, xo[i], d);
                        x[i] = xv;
                        fvd[gb[2] + base + i] = xv;
                    }
                    if (xv == inf) npos++;
                    else if (xv == -inf) nneg++;
                    else AccOps<A>::add(S, xv);
                }
                if (v < a.nv_sell && live) {
                    const double dd = var_finish<BMODE>(
                        a, v, AccOps<A>::value(S), npos, nneg, tol, RESID ? reinterpret_cast<const double *>(st + VS::bold)[t] : 0.0, cnt);
                    dmax = fmax(dmax, dd);
                    if (BMODE == 4 && dd > tol) mark_moved(s_moved, a, g);
                }
                if (WRITE_VF) {
                    for (int k = 0; k < wl; k++) {
                        const int i = 32 * k + lane;
                        const uint32_t e = en[i];
                        if (e != kSentinel) vf[e] = excl_msg<T>(S, npos, nneg, x[i]);
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
        }
    }
    if (RESID) var_close<BMODE>(a, ctl, dmax, cnt, s_moved, lane, wid);
}

// Low-pass belief mean, oldest to newest, then one division
// (HostBeliefHistory::mean, causal_bp.cu:65-77).
static __global__ void lowpass_kernel(const double *hist, const uint32_t *hist_next, const uint32_t *hist_count,
                               uint32_t hist_len, uint32_t n, double *out) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const uint32_t cnt = hist_count[v];
    uint32_t slot = (cnt == hist_len) ? hist_next[v] : 0;
    double sum = 0.0;
    for (uint32_t s = 0; s < cnt; s++) {
        sum += hist[(size_t)slot * n + v];
        if (++slot == hist_len) slot = 0;
    }
    if (cnt > 0) sum /= (double)cnt;
    out[v] = sum;
}

}  // namespace flbp
