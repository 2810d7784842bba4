// Direct-load form of the two sweep passes (no shared-memory staging).
//
// The staged form (factor_pass_kernel / var_pass_kernel) feeds consumer
// warps from a producer warp's bulk copies. This form has no producer: every
// warp of a persistent grid takes work items in turn (one sliced-ELL group
// of 32 items, one per lane, or one large item per warp) and issues all
// loads of an item - messages, scatter positions, per-item constants - before
// it uses any of them, so that an item costs one memory round trip and the
// SM's resident warps keep many items in flight. The item of the next turn
// has its header (group offsets, per-item constants) loaded before the
// current item is evaluated. Streams read once per sweep (positions,
// constants, priors) are loaded with the evict-first hint so that the
// message arrays, reused by the next pass, stay in L2.
//
// Both forms share the arithmetic (factor_reg, factor_tile_item,
// factor_block_huge, excl_msg, var_finish, var_close), so a sweep gives the
// same bits in either form; the engine's tuner picks the faster one per
// graph.
#pragma once

#include "kernels.cuh"

namespace flbp {

constexpr int kDirectThreads = kConsumers;  // 16 warps: the huge-item paths synchronise all consumer threads

template <typename T>
struct Pair2;
template <>
struct Pair2<float> {
    typedef float2 type;
};
template <>
struct Pair2<double> {
    typedef double2 type;
};

// (p, q) of internal factor f, streamed.
template <typename T>
__device__ __forceinline__ void load_pq(const void *f_pq, uint32_t f, T &p, T &q) {
    const typename Pair2<T>::type v = __ldcs(reinterpret_cast<const typename Pair2<T>::type *>(f_pq) + f);
    p = v.x;
    q = v.y;
}

// One sliced-ELL factor group of width W, direct: lane = factor, slots of
// the group at base + 32 k + lane. All 2 W loads are issued first.
template <typename T, int W>
__device__ __forceinline__ void factor_group_direct(const T *__restrict__ vf, const uint32_t *__restrict__ f_pos,
                                                    uint32_t base, int deg, uint8_t kind, T p, T q, int lane,
                                                    T *__restrict__ fv) {
    T x[W];
    uint32_t ps[W];
#pragma unroll
    for (int k = 0; k < W; k++) x[k] = vf[base + 32u * k + lane];
#pragma unroll
    for (int k = 0; k < W; k++) ps[k] = ld_stream(f_pos + base + 32u * k + lane);
    if (deg > 0) factor_reg<T, W>([&](int k) { return x[k]; }, [&](int k) { return ps[k]; }, deg, kind, p, q, fv);
}

template <typename T>
__device__ __forceinline__ void factor_group_direct_w(int w, const T *__restrict__ vf,
                                                      const uint32_t *__restrict__ f_pos, uint32_t base, int deg,
                                                      uint8_t kind, T p, T q, int lane, T *__restrict__ fv) {
    switch (w) {
#define FLBP_W(N) \
    case N: factor_group_direct<T, N>(vf, f_pos, base, deg, kind, p, q, lane, fv); break;
        FLBP_W(2) FLBP_W(3) FLBP_W(4) FLBP_W(5) FLBP_W(6) FLBP_W(7) FLBP_W(8) FLBP_W(9) FLBP_W(10) FLBP_W(11)
        FLBP_W(12) FLBP_W(13) FLBP_W(14) FLBP_W(15) FLBP_W(16)
#undef FLBP_W
        default: break;
    }
}

// Header of a factor-pass item: a sliced-ELL group (its slot range and this
// lane's factor constants) or a large factor (one per warp).
template <typename T>
struct FItem {
    uint32_t base, end;  // group: slot range; large factor: slot run start, degree in `end`
    uint32_t fi;         // internal factor of this lane (group) or of the warp (large)
    int deg;
    uint8_t kind;
    T p, q;
    bool big, live;
};

// Items: [0, nbig) the large factors that fit a warp (largest first), then
// the sliced-ELL groups.
template <typename T>
__device__ __forceinline__ FItem<T> factor_item(const FactorArgs &a, uint32_t it, uint32_t nbig, int lane) {
    FItem<T> h;
    if (it < nbig) {
        const uint32_t b = a.nf_huge + it;
        h.big = true;
        h.fi = a.nf_sell + b;
        h.base = __ldcs(a.fb_off + b);
        h.end = __ldcs(a.fb_deg + b);
        h.deg = 0;
        h.kind = ld_stream(a.f_kind + h.fi);
        load_pq<T>(a.f_pq, h.fi, h.p, h.q);
        h.live = !(a.f_graph && a.gdone[a.f_graph[h.fi]]);
    } else {
        const uint32_t g = it - nbig;
        h.big = false;
        h.fi = 32u * g + lane;
        h.base = __ldcs(a.fg_base + g);
        h.end = __ldcs(a.fg_base + g + 1);
        h.deg = ld_stream(a.f_deg + h.fi);
        h.kind = ld_stream(a.f_kind + h.fi);
        load_pq<T>(a.f_pq, h.fi, h.p, h.q);
        h.live = !(a.f_graph && a.gdone[a.f_graph[h.fi]]);  // batched solve: stopped graph
    }
    return h;
}

// Factor pass, direct form. Blocks of 16 warps, one wave of resident blocks;
// factors too large for a warp first (one per block), then every warp takes
// items it = warp, warp + all warps, ... (neighbouring warps work on
// neighbouring items, which keeps the scattered stores of a pass close
// together). SETS: evidence set blockIdx.y of an engine of sets (its
// messages at the set's strides; a stopped set does no work).
template <typename T, int MINB, bool SETS = false>
__global__ void __launch_bounds__(kDirectThreads, MINB) factor_direct_kernel(FactorArgs a, const T *__restrict__ vf,
                                                                             T *__restrict__ fv, Ctl *ctl) {
    if (*(volatile int *)&ctl->done) return;
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) sweep_open(ctl);
    if (SETS) {
        if (a.set_done[blockIdx.y]) return;
        vf += blockIdx.y * a.set_vf_stride;
        fv += blockIdx.y * a.set_fv_stride;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    {
        __shared__ typename WideAcc<T>::type s_l[kConsumerWarps];
        __shared__ int s_nz[kConsumerWarps];
        for (uint32_t b = blockIdx.x; b < a.nf_huge; b += gridDim.x)
            factor_block_huge<T>(a, b, threadIdx.x, vf, fv, s_l, s_nz);
    }
    const uint32_t nbig = a.nf_big - a.nf_huge;
    const uint32_t n_items = nbig + a.n_fgroups;
    const uint32_t stride = gridDim.x * (uint32_t)kConsumerWarps;
    uint32_t it = blockIdx.x * (uint32_t)kConsumerWarps + wid;
    if (it >= n_items) return;
    FItem<T> h = factor_item<T>(a, it, nbig, lane);
    for (;;) {
        const uint32_t nx = it + stride;
        FItem<T> hn;
        if (nx < n_items) hn = factor_item<T>(a, nx, nbig, lane);  // next header in flight during this item
        if (h.big) {
            if (h.live)
                factor_tile_item<T>(vf + h.base, a.f_pos + h.base, h.end, h.kind, h.p, h.q, lane, fv);
        } else {
            factor_group_direct_w<T>((int)((h.end - h.base) >> 5), vf, a.f_pos, h.base, h.live ? h.deg : 0, h.kind,
                                     h.p, h.q, lane, fv);
        }
        if (nx >= n_items) break;
        it = nx;
        h = hn;
    }
}

// One sliced-ELL variable group of width W, direct: lane = variable, entries
// at base + 32 k + lane (padding entries hold 0 and kSentinel). W = 0: a
// group of variables without entries (their beliefs come from the priors).
template <typename T, int W, int BMODE, bool WRITE_VF, bool DAMP>
__device__ __forceinline__ double var_group_direct(const VarArgs &a, const T *__restrict__ fv, T *__restrict__ vf,
                                                   T *__restrict__ fvd, T d, uint32_t base, uint32_t v, bool live,
                                                   double pscale, double tol, int lane, unsigned long long &cnt) {
    constexpr bool RESID = (BMODE == 1 || BMODE == 2 || BMODE == 4);
    const T inf = Num<T>::inf();
    T x[W > 0 ? W : 1];
    T xo[DAMP && W > 0 ? W : 1];
    uint32_t en[W > 0 ? W : 1];
#pragma unroll
    for (int k = 0; k < W; k++) x[k] = fv[base + 32u * k + lane];
    if (DAMP) {
#pragma unroll
        for (int k = 0; k < W; k++) xo[k] = fvd[base + 32u * k + lane];
    }
    if (WRITE_VF) {
#pragma unroll
        for (int k = 0; k < W; k++) en[k] = ld_stream(a.v_ent + base + 32u * k + lane);
    }
    const bool real = v < a.nv_sell;
    typedef typename NarrowAcc<T>::type A;
    A S = AccOps<A>::zero();
    int npos = 0, nneg = 0;
    if (real) decode_prior<T>(a.prior, v, pscale, S, npos, nneg);
    const double bold = (RESID && real) ? a.belief[v] : 0.0;
    if (!live) return 0.0;
#pragma unroll
    for (int k = 0; k < W; k++) {
        T xv = x[k];
        if (DAMP) {
            xv = take_fv<T, DAMP>(xv, xo[k], d);
            x[k] = xv;
            fvd[base + 32u * k + lane] = xv;
        }
        if (xv == inf) npos++;
        else if (xv == -inf) nneg++;
        else AccOps<A>::add(S, xv);
    }
    double dd = 0.0;
    if (real) dd = var_finish<BMODE>(a, v, AccOps<A>::value(S), npos, nneg, tol, bold, cnt);
    if (WRITE_VF) {
#pragma unroll
        for (int k = 0; k < W; k++)
            if (en[k] != kSentinel) vf[en[k]] = excl_msg<T>(S, npos, nneg, x[k]);
    }
    return dd;
}

template <typename T, int BMODE, bool WRITE_VF, bool DAMP>
__device__ __forceinline__ double var_group_direct_w(int w, const VarArgs &a, const T *__restrict__ fv,
                                                     T *__restrict__ vf, T *__restrict__ fvd, T d, uint32_t base,
                                                     uint32_t v, bool live, double pscale, double tol, int lane,
                                                     unsigned long long &cnt) {
    switch (w) {
#define FLBP_W(N) \
    case N: return var_group_direct<T, N, BMODE, WRITE_VF, DAMP>(a, fv, vf, fvd, d, base, v, live, pscale, tol, lane, cnt);
        FLBP_W(0) FLBP_W(1) FLBP_W(2) FLBP_W(3) FLBP_W(4) FLBP_W(5) FLBP_W(6) FLBP_W(7) FLBP_W(8) FLBP_W(9)
        FLBP_W(10) FLBP_W(11) FLBP_W(12) FLBP_W(13) FLBP_W(14) FLBP_W(15) FLBP_W(16)
#undef FLBP_W
        default: return 0.0;
    }
}
static_assert(kSellVarDegree == 16, "var_group_direct_w instantiates widths 0..16");

// One large variable that fits a warp (big variable b, internal index
// nv_sell + b), direct: the warp's lanes stride over its entries. Returns the
// belief change on lane 0 (0 elsewhere).
template <typename T, int BMODE, bool WRITE_VF, bool DAMP>
__device__ __forceinline__ double var_warp_direct(const VarArgs &a, uint32_t b, const T *__restrict__ fv,
                                                  T *__restrict__ vf, T *__restrict__ fvd, T d, double pscale,
                                                  double tol, int lane, unsigned long long &cnt) {
    constexpr bool RESID = (BMODE == 1 || BMODE == 2 || BMODE == 4);
    const uint32_t v = a.nv_sell + b, k0 = __ldcs(a.vb_off + b), k1 = k0 + __ldcs(a.vb_deg + b);
    const T inf = Num<T>::inf();
    const T *src = DAMP ? fvd : fv;  // after the first loop, fvd holds the messages in use
    typedef typename WideAcc<T>::type A;
    typedef AccOps<A> O;
    A S = O::zero();
    int npos = 0, nneg = 0;
    for (uint32_t k = k0 + lane; k < k1; k += 32) {
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
    A S0;
    int p0, n0;
    decode_prior<T>(a.prior, v, pscale, S0, p0, n0);
    O::combine(S, S0);
    npos += p0;
    nneg += n0;
    if (WRITE_VF) {
        for (uint32_t k = k0 + lane; k < k1; k += 32) {
            const uint32_t e = ld_stream(a.v_ent + k);
            if (e != kSentinel) vf[e] = excl_msg<T>(S, npos, nneg, src[k]);
        }
    }
    return (lane == 0) ? var_finish<BMODE>(a, v, O::value(S), npos, nneg, tol, RESID ? a.belief[v] : 0.0, cnt) : 0.0;
}

// Variable pass, direct form: variables too large for a warp first (one per
// block), then items it = warp, warp + all warps, ...: [0, nbig) the large
// variables that fit a warp, then the sliced-ELL groups (lane = variable).
// Residual, counts and stop rules as in the staged form (var_close). SETS:
// evidence set blockIdx.y of an engine of sets (BMODE 4 with the set as the
// graph); the blocks of a stopped set do no work but still take part in
// the end-of-pass count.
template <typename T, int BMODE, bool WRITE_VF, bool DAMP, int MINB, bool SETS = false>
__global__ void __launch_bounds__(kDirectThreads, MINB) var_direct_kernel(VarArgs a, const T *__restrict__ fv,
                                                                          T *__restrict__ vf, T *__restrict__ fvd, T d,
                                                                          Ctl *ctl) {
    constexpr bool RESID = (BMODE == 1 || BMODE == 2 || BMODE == 4);
    if (*(volatile int *)&ctl->done) return;
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0)
        ctl->fnext = 0u;  // the next staged factor pass starts after this kernel
    const double pscale = ctl->pscale;
    const double tol = ctl->tol;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double dmax = 0.0;
    unsigned long long cnt = 0;
    __shared__ uint32_t s_moved[BMODE == 4 ? kMovedWords : 1];  // batched: graphs with a belief moved > tol
    __shared__ uint32_t s_done[kDoneWords];                      // batched: stopped graphs
    if (BMODE == 4)
        for (int w = threadIdx.x; w < kMovedWords; w += blockDim.x) s_moved[w] = 0u;
    if (a.v_graph) load_done_bits(s_done, a.gstate, a.n_graphs, lane, wid, blockDim.x >> 5);
    const uint32_t set = SETS ? blockIdx.y : 0u;
    bool set_live = true;
    if (SETS) {
        set_live = a.gstate[set] == 0;
        fv += set * a.set_fv_stride;
        vf += set * a.set_vf_stride;
        if (DAMP) fvd += set * a.set_fv_stride;
        a.prior = reinterpret_cast<const unsigned char *>(a.prior) + set * a.set_prior_stride;
        a.belief += set * a.set_belief_stride;
    }
    __syncthreads();
    if (set_live) {
        {
            __shared__ typename WideAcc<T>::type s_s[kConsumerWarps];
            __shared__ int s_np[kConsumerWarps], s_nn[kConsumerWarps];
            for (uint32_t b = blockIdx.x; b < a.nv_huge; b += gridDim.x) {
                const uint32_t g = SETS ? set : a.v_graph ? a.v_graph[a.nv_sell + b] : 0;
                if (a.v_graph && graph_done(s_done, a.gstate, g)) continue;  // stopped graph (batched solve)
                const double dd = var_block_huge<T, BMODE, WRITE_VF, DAMP>(a, b, threadIdx.x, fv, vf, fvd, d, pscale,
                                                                           tol, cnt, s_s, s_np, s_nn);
                dmax = fmax(dmax, dd);
                if (BMODE == 4 && dd > tol) mark_moved(s_moved, a, g);
            }
        }
        const uint32_t nbig = a.nv_big - a.nv_huge;
        const uint32_t n_items = nbig + a.n_vgroups;
        const uint32_t stride = gridDim.x * (uint32_t)kConsumerWarps;
        for (uint32_t it = blockIdx.x * (uint32_t)kConsumerWarps + wid; it < n_items; it += stride) {
            if (it < nbig) {
                const uint32_t b = a.nv_huge + it;
                const uint32_t g = SETS ? set : a.v_graph ? a.v_graph[a.nv_sell + b] : 0;
                if (a.v_graph && graph_done(s_done, a.gstate, g)) continue;
                const double dd =
                    var_warp_direct<T, BMODE, WRITE_VF, DAMP>(a, b, fv, vf, fvd, d, pscale, tol, lane, cnt);
                dmax = fmax(dmax, dd);
                if (BMODE == 4 && dd > tol) mark_moved(s_moved, a, g);
            } else {
                const uint32_t grp = it - nbig;
                const uint32_t base = __ldcs(a.vg_base + grp), end = __ldcs(a.vg_base + grp + 1);
                const uint32_t v = 32u * grp + lane;
                const uint32_t g = SETS ? set : a.v_graph ? a.v_graph[v] : 0;
                const bool live = !(a.v_graph && graph_done(s_done, a.gstate, g));
                const double dd = var_group_direct_w<T, BMODE, WRITE_VF, DAMP>(
                    (int)((end - base) >> 5), a, fv, vf, fvd, d, base, v, live, pscale, tol, lane, cnt);
                dmax = fmax(dmax, dd);
                if (BMODE == 4 && dd > tol) mark_moved(s_moved, a, g);
            }
        }
    }
    if (RESID) var_close<BMODE>(a, ctl, dmax, cnt, s_moved, lane, wid);
}

}  // namespace flbp
