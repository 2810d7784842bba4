// Adjoint (reverse-mode derivative) of one synchronous sweep, for gradients
// of a loss on the beliefs after T sweeps with respect to every factor's p
// and q. FastLBP has no counterpart: it only runs the forward sweep.
//
// Forward sweep t (damping 0), in log-odds, as the kernels of kernels.cuh
// compute it:
//   fv_t = F(vf_t; p, q)                         factor pass
//   S_v  = prior_v + sum over entries e of v of fv_t[e]
//   vf_{t+1}[s] = S_v - fv_t[e(s)]               variable pass
//   belief_v = sigmoid(S_v) after the last sweep
// Backward, given lambda_{t+1} = dL/dvf_{t+1}:
//   variable adjoint: mu_t[e] = dL/dfv_t[e] = Lambda_v - lambda_{t+1}[s(e)]
//     with Lambda_v = sum over the slots of v of lambda_{t+1}, and
//     dL/dprior_v += Lambda_v (plus dL/dS_v at the last sweep);
//   factor adjoint: lambda_t = dL/dvf_t and dL/dp, dL/dq from mu_t through
//     the closed forms of the factor outputs (AND orientation, OR = AND on
//     negated log-odds), with sigma_j = sigmoid(y_j), tau_j = 1 - sigma_j,
//     P = prod sigma over the body, Po_k / Ro_k the same without slot k,
//     head: f_h = log(pP + qR) - log((1-p)P + (1-q)R),
//     body: f_k = log(s_h a_k + t_h (1 - a_k)) - log(s_h q + t_h (1 - q)),
//           a_k = p Po_k + q Ro_k, (s_h, t_h) = sigmoid of +-(head log-odds).
// Messages that are exact zeros (+-inf) carry no derivative, and an output
// that is an exact zero passes none back. The derivative arithmetic and the
// adjoint arrays use the engine's message type T (FP32 engines differentiate
// in FP32, FP64 engines in FP64).
//
// Layout, as in the forward passes: lambda is stored in variable-entry order
// (lambda of slot s at entry f_pos[s]) and mu in slot order (mu of entry e at
// slot v_ent[e]), so that each kernel reads its inputs coalesced and
// scatters its outputs through the map the forward pass of the same side
// uses. Every kernel writes the same set of positions at every step (the
// entries of each body slot of a factor with a head, and of the head slot of
// a factor whose head is free; the slot of every entry), so positions
// outside that set keep the zero they were given once.
#pragma once

#include "kernels.cuh"

namespace flbp {

struct AdjArgs {
    const uint32_t *fg_base, *fb_off, *fb_deg, *f_pos;
    const uint8_t *f_kind, *f_deg;
    const void *f_pq;  // T[2 * nf]
    uint32_t nf_sell, nf_big;
    const uint32_t *vg_base, *vb_off, *vb_deg, *v_ent;
    const void *prior;  // as in VarArgs
    uint32_t nv_sell, nv_big;
};

// Counts of exact-zero priors (clamps) of internal variable iv, and whether
// it has a folded finite constant (bit 31 of the count word), the only
// variables whose dL/dprior is accumulated.
template <typename T>
__device__ __forceinline__ bool prior_info(const void *prior, uint32_t iv, int &npos, int &nneg) {
    double S;
    decode_prior<T>(prior, iv, 1.0, S, npos, nneg);
    const uint32_t cnt = sizeof(T) == 4 ? reinterpret_cast<const uint2 *>(prior)[iv].y
                                        : reinterpret_cast<const uint4 *>(prior)[iv].z;
    return (cnt >> 31) != 0u;
}

// Head-output terms of the factor adjoint, given the body pair (P, R) and
// whether P is an exact zero: H = mu_h (p - q) P (1/A + 1/B) (the coefficient
// of tau_j in every body slot's derivative), and the contributions to dL/dp
// and dL/dq. With q == 0, (p - q) P / A = 1 and P / A = 1 / p exactly, also
// where P underflows (the forward pass takes log A = log p + log P there).
template <typename T>
__device__ __forceinline__ void head_terms(T mh, T p, T q, T P, T R, bool pzero, T &H, T &dgp, T &dgq) {
    H = T(0);
    if (mh == T(0) || pzero) return;
    const T A = p * P + q * R, B = (T(1) - p) * P + (T(1) - q) * R;
    if (!(B > T(0))) return;
    T r1, pa;
    if (q == T(0)) {
        if (!(p > T(0))) return;
        r1 = T(1);
        pa = T(1) / p;
    } else {
        if (!(A > T(0))) return;
        r1 = (p - q) * P / A;
        pa = P / A;
    }
    H = mh * (r1 + (p - q) * P / B);
    dgp += mh * (pa + P / B);
    dgq += mh * ((A > T(0) ? R / A : T(0)) + R / B);
}

// Lambda_v from the per-entry sums: with no exact-zero input every outgoing
// message is finite and Lambda is the sum over all slots; with exactly one
// exact zero only the slot of that entry receives a finite message.
template <typename T>
__device__ __forceinline__ T lambda_of(int npos, int nneg, T Lf, T Lp, T Ln) {
    if (npos == 0 && nneg == 0) return Lf;
    if (npos == 1 && nneg == 0) return Lp;
    if (npos == 0 && nneg == 1) return Ln;
    return T(0);
}

// Variable adjoint of one sliced-ELL variable (group width W, one lane):
// entries at base_lane + 32 k (lam in entry order), mu scattered to the
// entries' slots; messages and lambdas held in registers between the two
// passes.
template <typename T, int W>
__device__ __forceinline__ void var_adjoint_reg(const AdjArgs &a, uint32_t iv, uint32_t base_lane,
                                                const T *__restrict__ fv, const T *__restrict__ lam, const T *gS,
                                                T *__restrict__ mu, T *__restrict__ gprior) {
    int npos, nneg;
    const bool folded = prior_info<T>(a.prior, iv, npos, nneg);
    T x[W], l[W];
    uint32_t sl[W];
    // every load of the row first (padding entries are in bounds), so that they overlap
#pragma unroll
    for (int k = 0; k < W; k++) {
        sl[k] = a.v_ent[base_lane + 32u * k];
        x[k] = fv[base_lane + 32u * k];
        l[k] = lam[base_lane + 32u * k];
    }
    T Lf = T(0), Lp = T(0), Ln = T(0);
#pragma unroll
    for (int k = 0; k < W; k++) {
        if (sl[k] != kSentinel) {
            if (x[k] == Num<T>::inf()) {
                npos++;
                Lp += l[k];
            } else if (x[k] == -Num<T>::inf()) {
                nneg++;
                Ln += l[k];
            } else {
                Lf += l[k];
            }
        }
    }
    const bool fin = npos == 0 && nneg == 0;
    const T Lam = lambda_of<T>(npos, nneg, Lf, Lp, Ln);
    const T gs = (gS && fin) ? gS[iv] : T(0);
#pragma unroll
    for (int k = 0; k < W; k++)
        if (sl[k] != kSentinel) mu[sl[k]] = isfinite(x[k]) ? Lam - (fin ? l[k] : T(0)) + gs : T(0);
    if (folded) gprior[iv] += Lam + gs;
}

// Sliced-ELL groups of one width class, a warp per group: groups[0..n) are
// group ids whose widths are at most 8 (WIDE false) or 9..16 (WIDE true), so
// that the narrow groups, the common case, do not pay the registers of the
// wide ones.
constexpr uint32_t kNarrowWidth = 8;

template <typename T, bool WIDE>
__global__ void var_adjoint_kernel(AdjArgs a, const uint32_t *__restrict__ groups, uint32_t n, const T *__restrict__ fv,
                                   const T *__restrict__ lam, const T *gS, T *__restrict__ mu,
                                   T *__restrict__ gprior) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if ((t >> 5) >= n) return;
    const uint32_t g = groups[t >> 5], iv = 32u * g + (t & 31);
    if (iv >= a.nv_sell) return;
    const uint32_t base = a.vg_base[g];
    const uint32_t w = (a.vg_base[g + 1] - base) >> 5, bl = base + (t & 31);
#define FLBP_VW(N) \
    case N: var_adjoint_reg<T, N>(a, iv, bl, fv, lam, gS, mu, gprior); break;
    if (WIDE) {
        switch (w) {  // warp-uniform
            FLBP_VW(9) FLBP_VW(10) FLBP_VW(11) FLBP_VW(12) FLBP_VW(13) FLBP_VW(14) FLBP_VW(15) FLBP_VW(16)
            default: break;
        }
    } else {
        switch (w) {
            FLBP_VW(1) FLBP_VW(2) FLBP_VW(3) FLBP_VW(4) FLBP_VW(5) FLBP_VW(6) FLBP_VW(7) FLBP_VW(8)
            default: break;
        }
    }
#undef FLBP_VW
}
static_assert(kSellVarDegree == 16, "var_adjoint_kernel instantiates widths 1..16");

// Wide sliced-ELL groups (9-16 entries), two warps per group: warp h of the
// pair takes entries h, h + 2, ... of the group's 32 variables (one per
// lane), the pair combines its partial sums in shared memory, and each warp
// writes the mu of its own entries. Blocks of 128 threads hold two groups.
template <typename T>
__global__ void __launch_bounds__(128) var_adjoint_wide_kernel(AdjArgs a, const uint32_t *__restrict__ groups,
                                                                uint32_t n, const T *__restrict__ fv,
                                                                const T *__restrict__ lam, const T *gS,
                                                                T *__restrict__ mu, T *__restrict__ gprior) {
    __shared__ int s_cnt[4][32][2];
    __shared__ T s_sum[4][32][3];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31, h = warp & 1;
    const uint32_t gi = 2 * blockIdx.x + (warp >> 1);
    const bool live_g = gi < n;
    const uint32_t g = live_g ? groups[gi] : 0u, iv = 32u * g + lane;
    const bool live = live_g && iv < a.nv_sell;
    const uint32_t base = live ? a.vg_base[g] : 0u;
    const uint32_t w = live ? (a.vg_base[g + 1] - base) >> 5 : 0u, bl = base + lane;
    constexpr int R = (kSellVarDegree + 1) / 2;  // entries per warp at most
    T x[R], l[R];
    uint32_t sl[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
        const uint32_t k = h + 2u * r;
        sl[r] = kSentinel;
        if (k < w) {
            sl[r] = a.v_ent[bl + 32u * k];
            x[r] = fv[bl + 32u * k];
            l[r] = lam[bl + 32u * k];
        }
    }
    int npos = 0, nneg = 0;
    T Lf = T(0), Lp = T(0), Ln = T(0);
#pragma unroll
    for (int r = 0; r < R; r++) {
        if (sl[r] == kSentinel) continue;
        if (x[r] == Num<T>::inf()) {
            npos++;
            Lp += l[r];
        } else if (x[r] == -Num<T>::inf()) {
            nneg++;
            Ln += l[r];
        } else {
            Lf += l[r];
        }
    }
    s_cnt[warp][lane][0] = npos;
    s_cnt[warp][lane][1] = nneg;
    s_sum[warp][lane][0] = Lf;
    s_sum[warp][lane][1] = Lp;
    s_sum[warp][lane][2] = Ln;
    __syncthreads();
    const uint32_t o = warp ^ 1u;  // the pair's other warp; entries added in the order (even, odd)
    const int np = h ? s_cnt[o][lane][0] + npos : npos + s_cnt[o][lane][0];
    const int nn = h ? s_cnt[o][lane][1] + nneg : nneg + s_cnt[o][lane][1];
    const T lf = h ? s_sum[o][lane][0] + Lf : Lf + s_sum[o][lane][0];
    const T lp = h ? s_sum[o][lane][1] + Lp : Lp + s_sum[o][lane][1];
    const T ln = h ? s_sum[o][lane][2] + Ln : Ln + s_sum[o][lane][2];
    if (!live) return;
    int p0, n0;
    const bool folded = prior_info<T>(a.prior, iv, p0, n0);
    const int tp = np + p0, tn = nn + n0;
    const bool fin = tp == 0 && tn == 0;
    const T Lam = lambda_of<T>(tp, tn, lf, lp, ln);
    const T gs = (gS && fin) ? gS[iv] : T(0);
#pragma unroll
    for (int r = 0; r < R; r++)
        if (sl[r] != kSentinel) mu[sl[r]] = isfinite(x[r]) ? Lam - (fin ? l[r] : T(0)) + gs : T(0);
    if (h == 0 && folded) gprior[iv] += Lam + gs;
}

// Variables too large for a sliced-ELL group, kBigVarLanes lanes each: lane
// j of a variable takes entries e0 + j, e0 + j + kBigVarLanes, ..., the first
// kBigVarRegs of them held in registers between the two passes.
constexpr int kBigVarLanes = 8, kBigVarRegs = 8;

template <typename T>
__global__ void var_adjoint_big_kernel(AdjArgs a, const T *__restrict__ fv, const T *__restrict__ lam, const T *gS,
                                       T *__restrict__ mu, T *__restrict__ gprior) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t b = t / kBigVarLanes, j = t % kBigVarLanes;
    // whole warps stay in the shuffles below; lanes past the last variable carry no entries
    const bool live = b < a.nv_big;
    const uint32_t iv = a.nv_sell + b;
    const uint32_t e0 = live ? a.vb_off[b] : 0u, e1 = live ? e0 + a.vb_deg[b] : 0u;
    int npos = 0, nneg = 0;
    T Lf = T(0), Lp = T(0), Ln = T(0);
    T xr[kBigVarRegs], lr[kBigVarRegs];
    uint32_t sr[kBigVarRegs];
#pragma unroll
    for (int r = 0; r < kBigVarRegs; r++) {
        const uint32_t e = e0 + j + (uint32_t)(r * kBigVarLanes);
        sr[r] = kSentinel;
        if (e < e1) {
            sr[r] = a.v_ent[e];
            xr[r] = fv[e];
            lr[r] = lam[e];
        }
    }
    auto add = [&](uint32_t s, T x, T l) {
        if (s == kSentinel) return;
        if (x == Num<T>::inf()) {
            npos++;
            Lp += l;
        } else if (x == -Num<T>::inf()) {
            nneg++;
            Ln += l;
        } else {
            Lf += l;
        }
    };
#pragma unroll
    for (int r = 0; r < kBigVarRegs; r++) add(sr[r], xr[r], lr[r]);
    for (uint32_t e = e0 + j + kBigVarRegs * kBigVarLanes; e < e1; e += kBigVarLanes) add(a.v_ent[e], fv[e], lam[e]);
    for (int o = kBigVarLanes / 2; o > 0; o >>= 1) {
        npos += __shfl_xor_sync(0xffffffffu, npos, o);
        nneg += __shfl_xor_sync(0xffffffffu, nneg, o);
        Lf += __shfl_xor_sync(0xffffffffu, Lf, o);
        Lp += __shfl_xor_sync(0xffffffffu, Lp, o);
        Ln += __shfl_xor_sync(0xffffffffu, Ln, o);
    }
    if (!live) return;
    int p0, n0;
    const bool folded = prior_info<T>(a.prior, iv, p0, n0);
    npos += p0;
    nneg += n0;
    const bool fin = npos == 0 && nneg == 0;
    const T Lam = lambda_of<T>(npos, nneg, Lf, Lp, Ln);
    const T gs = (gS && fin) ? gS[iv] : T(0);
    auto put = [&](uint32_t s, T x, T l) {
        if (s != kSentinel) mu[s] = isfinite(x) ? Lam - (fin ? l : T(0)) + gs : T(0);
    };
#pragma unroll
    for (int r = 0; r < kBigVarRegs; r++) put(sr[r], xr[r], lr[r]);
    for (uint32_t e = e0 + j + kBigVarRegs * kBigVarLanes; e < e1; e += kBigVarLanes) put(a.v_ent[e], fv[e], lam[e]);
    if (j == 0 && folded) gprior[iv] += Lam + gs;
}

// Factor adjoint of one sliced-ELL factor (group width W, one lane): slot k
// of the factor at base + 32 k (head at k = 0), mu in slot order, lam
// scattered to the slots' entries. Sigmoids, prefix pairs and per-slot terms
// stay in registers; leave-one-out pairs are prefix x suffix.
template <typename T, int W>
__device__ __forceinline__ void factor_adjoint_reg(const AdjArgs &a, uint32_t base, int deg, uint8_t kind, T p, T q,
                                                   const T *__restrict__ vf, const T *__restrict__ mu,
                                                   T *__restrict__ lam, T *__restrict__ gp, T *__restrict__ gq) {
    const uint8_t hs = kind & HEAD_MASK;
    if (hs == HEAD_NONE) return;
    // every load of the row first (padding slots are in bounds), so that they overlap
    T y[W], m[W];
    uint32_t ep[W];
#pragma unroll
    for (int k = 0; k < W; k++) {
        y[k] = vf[base + 32u * k];
        m[k] = mu[base + 32u * k];
        ep[k] = a.f_pos[base + 32u * k];
    }
    const T gp0 = *gp, gq0 = gq ? *gq : T(0);
    const T sgn = (kind & KIND_OR) ? T(-1) : T(1);
    // the head's log-odds in the factor's orientation, as the forward pass takes it
    const T lh = sgn * (hs == HEAD_FREE ? y[0] : (hs == HEAD_ONE ? Num<T>::inf() : -Num<T>::inf()));
    T sh, th;
    sig_pair<T>(lh, sh, th);
    auto mu_of = [&](int k) { return sgn * m[k]; };
    auto put_lam = [&](int k, T v) {
        if (ep[k] != kSentinel) lam[ep[k]] = v;
    };
    T sg[W], ta[W], pP[W], pR[W];
    uint32_t fin = 0;
    T P = T(1), R = T(0);
    bool pzero = false;
#pragma unroll
    for (int k = 1; k < W; k++) {
        sg[k] = T(1);
        ta[k] = T(0);
        if (k < deg) {
            const T yk = sgn * y[k];
            if (isfinite(yk)) fin |= 1u << k;
            sig_pair<T>(yk, sg[k], ta[k]);
        }
        pP[k] = P;
        pR[k] = R;
        pzero |= sg[k] == T(0);
        R = fma(P, ta[k], R);
        P = P * sg[k];
    }
    const T m0 = sh * q + th * (T(1) - q);
    const T r0 = m0 > T(0) ? T(1) / m0 : T(0), d0 = (T(2) * q - T(1)) * r0, shth = sh * th, smt = sh - th;
    T H = T(0), dgp = T(0), dgq = T(0), gh = T(0);
    if (hs == HEAD_FREE) head_terms<T>(mu_of(0), p, q, P, R, pzero, H, dgp, dgq);
    T c[W];
    T C = T(0), Ps = T(1), Rs = T(0);
#pragma unroll
    for (int k = W - 1; k >= 1; k--) {
        c[k] = T(0);
        if (k < deg) {
            const T Po = pP[k] * Ps, Ro = fma(pP[k], Rs, pR[k]);
            const T ak = p * Po + q * Ro, bk = (T(1) - p) * Po + (T(1) - q) * Ro;
            const T m1 = sh * ak + th * bk;
            const T mk = mu_of(k);
            if (m1 > T(0) && m0 > T(0) && mk != T(0)) {
                const T r1 = T(1) / m1, wk = mk * smt * r1;
                c[k] = wk * (p - q) * Po;
                dgp += wk * Po;
                dgq += wk * Ro - mk * smt * r0;
                gh += mk * shth * ((ak - bk) * r1 - d0);
            }
            C += c[k];
            Rs = fma(sg[k], Rs, ta[k]);
            Ps = sg[k] * Ps;
        }
    }
#pragma unroll
    for (int k = 1; k < W; k++)
        if (k < deg) put_lam(k, (fin & (1u << k)) ? sgn * ta[k] * (H + C - c[k]) : T(0));
    if (hs == HEAD_FREE) put_lam(0, isfinite(lh) ? sgn * gh : T(0));
    *gp = gp0 + dgp;
    if (gq) *gq = gq0 + dgq;
}

template <typename T, bool WIDE>
__global__ void __launch_bounds__(128, (!WIDE && sizeof(T) == 4) ? 8 : 1) factor_adjoint_sell_kernel(AdjArgs a, const uint32_t *__restrict__ groups, uint32_t n,
                                           const T *__restrict__ vf, const T *__restrict__ mu, T *__restrict__ lam,
                                           T *__restrict__ gp, T *__restrict__ gq) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if ((t >> 5) >= n) return;
    const uint32_t g = groups[t >> 5], f = 32u * g + (t & 31);
    if (f >= a.nf_sell) return;
    const uint32_t gb = a.fg_base[g];
    const uint32_t w = (a.fg_base[g + 1] - gb) >> 5, base = gb + (t & 31);
    const T *pq = reinterpret_cast<const T *>(a.f_pq);
    const int deg = a.f_deg[f];
    const uint8_t kind = a.f_kind[f];
    const T p = pq[2 * f], q = pq[2 * f + 1];
#define FLBP_FW(N) \
    case N: factor_adjoint_reg<T, N>(a, base, deg, kind, p, q, vf, mu, lam, gp + f, gq ? gq + f : nullptr); break;
    if (WIDE) {
        switch (w) {  // warp-uniform
            FLBP_FW(9) FLBP_FW(10) FLBP_FW(11) FLBP_FW(12) FLBP_FW(13) FLBP_FW(14) FLBP_FW(15) FLBP_FW(16)
            default: break;
        }
    } else {
        switch (w) {
            FLBP_FW(2) FLBP_FW(3) FLBP_FW(4) FLBP_FW(5) FLBP_FW(6) FLBP_FW(7) FLBP_FW(8)
            default: break;  // width 1: a head without a body has a constant output
        }
    }
#undef FLBP_FW
}
static_assert(kSellFactorDegree == 16, "factor_adjoint_sell_kernel instantiates widths 2..16");

// Big factors, one warp each: leave-one-out products from a sum of
// log-sigmoids with a count of exact zeros (inputs at -inf after the
// orientation sign).
template <typename T>
__global__ void factor_adjoint_big_kernel(AdjArgs a, const T *__restrict__ vf, const T *__restrict__ mu,
                                          T *__restrict__ lam, T *__restrict__ gp, T *__restrict__ gq) {
    const uint32_t b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (b >= a.nf_big) return;
    const uint32_t f = a.nf_sell + b, s0 = a.fb_off[b], s1 = s0 + a.fb_deg[b];
    const uint8_t kind = a.f_kind[f];
    const uint8_t hs = kind & HEAD_MASK;
    if (hs == HEAD_NONE) return;
    const T *pqa = reinterpret_cast<const T *>(a.f_pq);
    const T p = pqa[2 * f], q = pqa[2 * f + 1];
    const T sgn = (kind & KIND_OR) ? T(-1) : T(1);
    const T lh = sgn * (hs == HEAD_FREE ? vf[s0] : (hs == HEAD_ONE ? Num<T>::inf() : -Num<T>::inf()));
    T sh, th;
    sig_pair<T>(lh, sh, th);
    auto mu_of = [&](uint32_t s) { return sgn * mu[s]; };
    auto put_lam = [&](uint32_t s, T v) {
        const uint32_t e = a.f_pos[s];
        if (e != kSentinel) lam[e] = v;
    };
    T L = T(0);
    int nz = 0;
    for (uint32_t k = s0 + 1 + lane; k < s1; k += 32) {
        const T y = sgn * vf[k];
        if (y == -Num<T>::inf()) nz++;
        else L += log_sigmoid<T>(y);
    }
    for (int o = 16; o > 0; o >>= 1) {
        L += __shfl_xor_sync(0xffffffffu, L, o);
        nz += __shfl_xor_sync(0xffffffffu, nz, o);
    }
    const T P = nz ? T(0) : Num<T>::exp(L), R = nz ? T(1) : -Num<T>::expm1(L);
    const T m0 = sh * q + th * (T(1) - q);
    // (Po_k, Ro_k) of body slot k from its log-sigmoid
    auto loo = [&](T y, T &Po, T &Ro) {
        const bool z = y == -Num<T>::inf();
        if (nz - (int)z) {
            Po = T(0);
            Ro = T(1);
        } else {
            const T lo = z ? L : L - log_sigmoid<T>(y);
            Po = Num<T>::exp(lo);
            Ro = -Num<T>::expm1(lo);
        }
    };
    T C = T(0), dgp = T(0), dgq = T(0), gh = T(0);
    for (uint32_t k = s0 + 1 + lane; k < s1; k += 32) {
        T Po, Ro;
        loo(sgn * vf[k], Po, Ro);
        const T ak = p * Po + q * Ro, bk = (T(1) - p) * Po + (T(1) - q) * Ro;
        const T m1 = sh * ak + th * bk, mk = mu_of(k);
        if (m1 > T(0) && m0 > T(0) && mk != T(0)) {
            const T wk = mk * (sh - th) / m1;
            C += wk * (p - q) * Po;
            dgp += wk * Po;
            dgq += wk * Ro - mk * (sh - th) / m0;
            gh += mk * sh * th * ((ak - bk) / m1 - (T(2) * q - T(1)) / m0);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        C += __shfl_xor_sync(0xffffffffu, C, o);
        dgp += __shfl_xor_sync(0xffffffffu, dgp, o);
        dgq += __shfl_xor_sync(0xffffffffu, dgq, o);
        gh += __shfl_xor_sync(0xffffffffu, gh, o);
    }
    T H = T(0);
    if (hs == HEAD_FREE) head_terms<T>(mu_of(s0), p, q, P, R, nz > 0, H, dgp, dgq);
    for (uint32_t k = s0 + 1 + lane; k < s1; k += 32) {
        const T y = sgn * vf[k];
        T Po, Ro, ck = T(0), sk, tk;
        loo(y, Po, Ro);
        sig_pair<T>(y, sk, tk);
        const T ak = p * Po + q * Ro, bk = (T(1) - p) * Po + (T(1) - q) * Ro;
        const T m1 = sh * ak + th * bk, mk = mu_of(k);
        if (m1 > T(0) && m0 > T(0) && mk != T(0)) ck = mk * (sh - th) / m1 * (p - q) * Po;
        put_lam(k, isfinite(y) ? sgn * tk * (H + C - ck) : T(0));
    }
    if (lane == 0) {
        if (hs == HEAD_FREE) put_lam(s0, isfinite(lh) ? sgn * gh : T(0));
        gp[f] += dgp;
        if (gq) gq[f] += dgq;
    }
}

// dL/dS_v = dL/db_v * b_v (1 - b_v) at the final beliefs, from the loss
// gradient in the caller's variable order (internal_of_var maps it).
template <typename T>
__global__ void adjoint_seed_kernel(const double *__restrict__ grad_b, const uint32_t *__restrict__ internal_of_var,
                                    const double *__restrict__ belief, int64_t n, T *__restrict__ gs) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t iv = internal_of_var[i];
    const double b = belief[iv];
    gs[iv] = isfinite(b) ? (T)(grad_b[i] * b * (1.0 - b)) : T(0);
}

// Parameter gradients in the caller's factor order: internal factor f's
// accumulators to factor factor_of_internal[f] (one internal factor per
// caller factor at most; the outputs start at zero).
template <typename T>
__global__ void adjoint_factor_out_kernel(const T *__restrict__ gp, const T *__restrict__ gq,
                                          const uint32_t *__restrict__ factor_of_internal, uint32_t nf,
                                          double *__restrict__ out_p, double *__restrict__ out_q) {
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const uint32_t I = factor_of_internal[f];
    if (out_p) out_p[I] += (double)gp[f];
    if (out_q) out_q[I] += (double)gq[f];
}

// Folded constants sign * logit(p) of singleton and reduced factors: their
// dL/dp = dL/dprior_v * coef, coef = sign / (p (1 - p)) (0 at p = 0 or 1).
// Several folded factors may share a caller factor's variable, never a
// caller factor: plain adds.
template <typename T>
__global__ void adjoint_prior_out_kernel(const T *__restrict__ gprior, const uint32_t *__restrict__ prior_factor,
                                         const uint32_t *__restrict__ prior_var, const double *__restrict__ coef,
                                         uint32_t n, double *__restrict__ out_p) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    out_p[prior_factor[k]] += (double)gprior[prior_var[k]] * coef[k];
}

// Reference-order copy of an internal per-variable array.
__global__ void gather_vars_kernel(const double *__restrict__ src, const uint32_t *__restrict__ internal_of_var,
                                   int64_t n, double *__restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = src[internal_of_var[i]];
}

}  // namespace flbp
