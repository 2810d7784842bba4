// Kernels of the sequential schedules (updates=SEQFIX / TOPO).
//
// A sweep runs the schedule's batches in order, each in two phases:
//   seq_factor_kernel  one warp per factor of the batch: the v->f message of
//                      every slot from the current variable totals (the
//                      reference's calcMessageVFKernel, causal_bp_seq.cu:
//                      113-147), then every output of the factor into the
//                      staging array (the f->v math of the PARALL pass);
//   seq_apply_kernel   one thread per target edge of the batch: its new f->v
//                      message replaces the old one in its variable's total
//                      and +-inf counts (update_message, :34-83).
// The factor kernel reads only state as it was before the batch, which is
// what the reference's two kernels per batch see, and the targets of a batch
// have distinct variables, so the apply kernel has no conflicts. A factor's
// outputs to slots that are not targets of the batch are staged but not
// applied. seq_begin_kernel opens a sweep; seq_belief_kernel closes it with
// the beliefs, residuals and stop rules of the run loops.
//
// seq_sweep_cluster_kernel runs all batches of a sweep in one launch on one
// cluster of kSeqClusterCtas blocks: the two phases of a batch are
// separated by cluster barriers (release / acquire) instead of kernel
// boundaries. Every thread passes exactly two barriers per batch and none
// leaves early, so the barriers cannot wait for a thread that is gone. State
// that other blocks write (totals, counts, messages, staged messages) is
// read with ld.global.cg, from L2, never from a stale L1 line.
#pragma once

#include "kernels.cuh"

namespace flbp {

struct SeqArgs {
    const uint4 *irec;      // per item: first device slot, degree, kind, factor
    const uint32_t *tvar;   // per target: its variable
    const uint2 *bo;        // per batch: (first item, first target), n_batches + 1
    const uint32_t *foff;   // per factor: first device slot (F + 1)
    const uint32_t *var;    // per device slot: internal variable
    const uint8_t *kind;    // per factor
    const void *cst;        // per factor: constant message, T
    const void *pq;         // per factor: p, q, T
    const uint32_t *items;  // factors of the batches
    const uint32_t *tgt;    // target device slots of the batches
    const uint32_t *iota;   // iota[s] = s: output positions of a factor's slots
    void *fv;               // per device slot: current f->v message, T
    void *vf;               // per device slot: v->f message of the current batch, T
    void *nw;               // per device slot: staged f->v message, T
    double *S;              // per internal variable: sum of its finite f->v messages
    int2 *cnt;              // per internal variable: (+inf count, -inf count)
};

// Programmatic dependent launch: a kernel lets the next one in the stream
// launch at once and waits (in hardware) for the previous one to finish and
// its memory to be visible before it reads any state. Both are no-ops for a
// kernel launched without the attribute.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

constexpr int kSeqWarps = 8;           // warps per block of the factor kernel
constexpr int kSeqClusterCtas = 8;     // blocks of the one-cluster sweep kernel (portable cluster size)
constexpr int kSeqClusterWarps = 16;   // warps per block of that kernel (FP64 item code: ~92 registers)

static __global__ void seq_begin_kernel(Ctl *ctl) {
    pdl_enter();
    if (*(volatile int *)&ctl->done) return;
    unsigned long long now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    if (ctl->run_sweeps == 0) ctl->t_start_ns = now;
    ctl->t += 1;
    ctl->run_sweeps += 1;
    ctl->maxdiff_bits = 0ull;
    ctl->nonconv = 0ull;
    ctl->arrive = 0u;
}

// A factor with more than kBigFactorBody body slots, one warp: a log-sigmoid
// sum of the body in FP64 with a count of -inf terms, then every slot removes
// its own term (the warp form of factor_block_huge). vb[0] is the head's
// v->f message, vb[1 + k] body slot k's; outputs go to out[0] (head) and
// out[1 + k].
template <typename T>
__device__ void seq_factor_huge(const T *vb, uint32_t nbody, uint8_t kind, T p, T q, int lane, T *out) {
    const T s = (kind & KIND_OR) ? T(-1) : T(1);
    const T inf = Num<T>::inf();
    double L = 0.0;
    int nz = 0;
    for (uint32_t k = 1 + lane; k <= nbody; k += 32) {
        const T ls = log_sigmoid<T>(s * vb[k]);
        if (ls == -inf) nz++;
        else L += (double)ls;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        L += __shfl_xor_sync(0xffffffffu, L, o);
        nz += __shfl_xor_sync(0xffffffffu, nz, o);
    }
    if ((kind & HEAD_MASK) == HEAD_FREE && lane == 0) out[0] = s * head_out<T>(nz ? -inf : (T)L, p, q, Num<T>::log(p));
    const BodyDen<T> D = body_den<T>(s * head_effective<T>(kind, vb[0]), p, q);
    for (uint32_t k = 1 + lane; k <= nbody; k += 32) {
        const T ls = log_sigmoid<T>(s * vb[k]);
        const bool z = (ls == -inf);
        const T lo = (nz - (int)z) ? -inf : (T)(z ? L : L - (double)ls);
        out[k] = s * body_out<T>(lo, p, q, D);
    }
}

// Item `it` of the batches' item list, one whole warp: every v->f message of
// the factor from the current totals, then all its outputs into the staging
// array.
template <typename T>
__device__ __forceinline__ void seq_factor_item(const SeqArgs &a, uint32_t it, int lane) {
    const uint4 r = a.irec[it];  // first slot, degree, kind, factor
    const uint32_t s0 = r.x, deg = r.y, f = r.w;
    const uint8_t kind = (uint8_t)r.z;
    T *nw = reinterpret_cast<T *>(a.nw);
    const T c = reinterpret_cast<const T *>(a.cst)[f];
    if (kind & kSeqConst) {  // singleton, or an AND/OR factor reduced to its head
        if (lane == 0) nw[s0] = c;
        return;
    }
    const T *fv = reinterpret_cast<const T *>(a.fv);
    T *vf = reinterpret_cast<T *>(a.vf);
    for (uint32_t k = lane; k < deg; k += 32) {
        const uint32_t s = s0 + k, v = a.var[s];
        const T x = __ldcg(fv + s);
        const int2 n = __ldcg(a.cnt + v);
        vf[s] = excl_msg<T>(__ldcg(a.S + v), n.x, n.y, x);
    }
    __syncwarp();  // orders the v->f stores before the other lanes' loads
    const T *pq = reinterpret_cast<const T *>(a.pq);
    const T p = pq[2 * f], q = pq[2 * f + 1];
    if (deg - 1 <= kBigFactorBody) factor_tile_item<T>(vf + s0, a.iota + s0, deg, kind, p, q, lane, nw);
    else seq_factor_huge<T>(vf + s0, deg - 1, kind, p, q, lane, nw + s0);
    if ((kind & HEAD_MASK) != HEAD_FREE && lane == 0) nw[s0] = c;  // a clamped head's constant
}

// Target k of the batches' target list: its staged message replaces the old
// one in its variable's total and counts.
template <typename T, bool DAMP>
__device__ __forceinline__ void seq_apply_one(const SeqArgs &a, uint32_t k, T d) {
    const uint32_t s = a.tgt[k], v = a.tvar[k];
    T *fv = reinterpret_cast<T *>(a.fv);
    const T old = __ldcg(fv + s);
    T x = __ldcg(reinterpret_cast<const T *>(a.nw) + s);
    double S = __ldcg(a.S + v);
    int2 n = __ldcg(a.cnt + v);
    if (DAMP) x = damp_mix<T>(x, old, d);
    const T inf = Num<T>::inf();
    if (old == inf) n.x--;
    else if (old == -inf) n.y--;
    else S -= (double)old;
    if (x == inf) n.x++;
    else if (x == -inf) n.y++;
    else S += (double)x;
    a.S[v] = S;
    a.cnt[v] = n;
    fv[s] = x;
}

// Items [i0, i1) of the batches' item list: one warp per factor.
template <typename T>
__global__ void __launch_bounds__(32 * kSeqWarps) seq_factor_kernel(SeqArgs a, uint32_t i0, uint32_t i1, Ctl *ctl) {
    pdl_enter();
    if (*(volatile int *)&ctl->done) return;
    const uint32_t it = i0 + blockIdx.x * kSeqWarps + (threadIdx.x >> 5);
    if (it >= i1) return;  // whole warps leave together
    seq_factor_item<T>(a, it, threadIdx.x & 31);
}

// Targets [t0, t1) of the batches' target list.
template <typename T, bool DAMP>
__global__ void seq_apply_kernel(SeqArgs a, uint32_t t0, uint32_t t1, T d, Ctl *ctl) {
    pdl_enter();
    if (*(volatile int *)&ctl->done) return;
    const uint32_t k = t0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= t1) return;
    seq_apply_one<T, DAMP>(a, k, d);
}

__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}

// One whole sweep (its opening included) on one cluster; grid = one cluster.
template <typename T, bool DAMP>
__global__ void __cluster_dims__(kSeqClusterCtas, 1, 1) __launch_bounds__(32 * kSeqClusterWarps, 1)
    seq_sweep_cluster_kernel(SeqArgs a, uint32_t n_batches, T d, Ctl *ctl) {
    if (*(volatile int *)&ctl->done) return;  // the same for every thread: only earlier launches write it
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        unsigned long long now;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
        if (ctl->run_sweeps == 0) ctl->t_start_ns = now;
        ctl->t += 1;
        ctl->run_sweeps += 1;
        ctl->maxdiff_bits = 0ull;
        ctl->nonconv = 0ull;
        ctl->arrive = 0u;
    }
    const int lane = threadIdx.x & 31;
    const uint32_t gw = blockIdx.x * kSeqClusterWarps + (threadIdx.x >> 5), nwarps = gridDim.x * kSeqClusterWarps;
    const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
    uint2 lo = a.bo[0];
    for (uint32_t b = 0; b < n_batches; b++) {
        const uint2 hi = a.bo[b + 1];
        for (uint32_t it = lo.x + gw; it < hi.x; it += nwarps) seq_factor_item<T>(a, it, lane);
        cluster_barrier();
        for (uint32_t k = lo.y + gt; k < hi.y; k += nthreads) seq_apply_one<T, DAMP>(a, k, d);
        cluster_barrier();
        lo = hi;
    }
}

// Beliefs of every internal variable from its total and counts, with the
// residual, history and stop rules of the run loop's mode (BMODE of
// var_finish: 1 tolerance loop, 2 low-pass loop, 3 beliefs only).
template <int BMODE>
__global__ void __launch_bounds__(256) seq_belief_kernel(VarArgs va, const double *S, const int2 *cnt, uint32_t V,
                                                         Ctl *ctl) {
    constexpr bool RESID = (BMODE == 1 || BMODE == 2);
    pdl_enter();
    if (BMODE != 3 && *(volatile int *)&ctl->done) return;
    const double tol = ctl->tol;
    double dmax = 0.0;
    unsigned long long c = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const int2 n = cnt[v];
        const double dd = var_finish<BMODE>(va, v, S[v], n.x, n.y, tol, RESID ? va.belief[v] : 0.0, c);
        dmax = fmax(dmax, dd);
    }
    if (!RESID) return;
    __shared__ double s_max[8];
    __shared__ unsigned long long s_cnt[8];
    __shared__ bool s_last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    dmax = warp_max(dmax);
    c = warp_sum(c);
    if (lane == 0) {
        s_max[wid] = dmax;
        s_cnt[wid] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        unsigned long long t = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) {
            m = fmax(m, s_max[i]);
            t += s_cnt[i];
        }
        atomicMax(&ctl->maxdiff_bits, (unsigned long long)__double_as_longlong(m));
        if (BMODE == 2) atomicAdd(&ctl->nonconv, t);
        __threadfence();
        s_last = (atomicAdd(&ctl->arrive, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (s_last && threadIdx.x == 0) {
        __threadfence();
        stop_rules(ctl);
    }
}

}  // namespace flbp
