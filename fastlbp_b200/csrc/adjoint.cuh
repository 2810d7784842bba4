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
// Backward, given lambda_{t+1} = dL/dvf_{t+1} (slot order):
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
// that is an exact zero passes none back. All derivative arithmetic is FP64.
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

__device__ __forceinline__ double sigm(double y) { return y >= 0.0 ? 1.0 / (1.0 + exp(-y)) : exp(y) / (1.0 + exp(y)); }

__device__ __forceinline__ bool zero_msg(double x) { return !isfinite(x); }

template <typename T>
__device__ __forceinline__ void prior_counts(const void *prior, uint32_t iv, int &npos, int &nneg) {
    double S;
    decode_prior<T>(prior, iv, 1.0, S, npos, nneg);
}

// Head-output terms of the factor adjoint, given the body pair (P, R) and
// whether P is an exact zero: H = mu_h (p - q) P (1/A + 1/B) (the coefficient
// of tau_j in every body slot's derivative), and the contributions to dL/dp
// and dL/dq. With q == 0, (p - q) P / A = 1 and P / A = 1 / p exactly, also
// where P underflows (the forward pass takes log A = log p + log P there).
__device__ __forceinline__ void head_terms(double mh, double p, double q, double P, double R, bool pzero, double &H,
                                           double &dgp, double &dgq) {
    H = 0.0;
    if (mh == 0.0 || pzero) return;
    const double A = p * P + q * R, B = (1.0 - p) * P + (1.0 - q) * R;
    if (!(B > 0.0)) return;
    double r1, pa;
    if (q == 0.0) {
        if (!(p > 0.0)) return;
        r1 = 1.0;
        pa = 1.0 / p;
    } else {
        if (!(A > 0.0)) return;
        r1 = (p - q) * P / A;
        pa = P / A;
    }
    H = mh * (r1 + (p - q) * P / B);
    dgp += mh * (pa + P / B);
    dgq += mh * ((A > 0.0 ? R / A : 0.0) + R / B);
}

// Variable adjoint for the entries en[k * stride] (k < n) of internal
// variable iv. gS: dL/dS_v at the last sweep (or null).
template <typename T>
__device__ void var_adjoint_one(const AdjArgs &a, uint32_t iv, const uint32_t *en, uint32_t stride, uint32_t n,
                                const T *__restrict__ fv, const double *__restrict__ lam, const double *gS,
                                double *__restrict__ mu, double *__restrict__ gprior, uint32_t e0) {
    int npos, nneg;
    prior_counts<T>(a.prior, iv, npos, nneg);
    for (uint32_t k = 0; k < n; k++) {
        const uint32_t e = e0 + k * stride;
        if (en[k * stride] == kSentinel) continue;
        const double x = (double)fv[e];
        if (x == INFINITY) npos++;
        else if (x == -INFINITY) nneg++;
    }
    // the message to the slot of entry e is finite iff no zero is left without x
    auto out_finite = [&](double x) {
        return (npos - (x == INFINITY)) == 0 && (nneg - (x == -INFINITY)) == 0;
    };
    double Lam = 0.0;
    for (uint32_t k = 0; k < n; k++) {
        const uint32_t s = en[k * stride];
        if (s == kSentinel) continue;
        if (out_finite((double)fv[e0 + k * stride])) Lam += lam[s];
    }
    const double gs = (gS && npos == 0 && nneg == 0) ? gS[iv] : 0.0;
    for (uint32_t k = 0; k < n; k++) {
        const uint32_t e = e0 + k * stride, s = en[k * stride];
        if (s == kSentinel) continue;
        const double x = (double)fv[e];
        mu[e] = zero_msg(x) ? 0.0 : Lam - (out_finite(x) ? lam[s] : 0.0) + gs;
    }
    gprior[iv] += Lam + gs;
}

template <typename T>
__global__ void var_adjoint_kernel(AdjArgs a, const T *__restrict__ fv, const double *__restrict__ lam,
                                   const double *gS, double *__restrict__ mu, double *__restrict__ gprior) {
    const uint32_t iv = blockIdx.x * blockDim.x + threadIdx.x;
    if (iv < a.nv_sell) {
        const uint32_t g = iv >> 5, lane = iv & 31, base = a.vg_base[g];
        const uint32_t w = (a.vg_base[g + 1] - base) >> 5;
        var_adjoint_one<T>(a, iv, a.v_ent + base + lane, 32, w, fv, lam, gS, mu, gprior, base + lane);
    } else if (iv < a.nv_sell + a.nv_big) {
        const uint32_t b = iv - a.nv_sell;
        var_adjoint_one<T>(a, iv, a.v_ent + a.vb_off[b], 1, a.vb_deg[b], fv, lam, gS, mu, gprior, a.vb_off[b]);
    }
}

// Factor adjoint of one factor whose slot k (head at k = 0) is slot(k).
// Leave-one-out pairs come from prefix and suffix products (in FP64).
template <typename T, typename Slot>
__device__ void factor_adjoint_one(int deg, uint8_t kind, double p, double q, Slot slot, const AdjArgs &a,
                                   const T *__restrict__ vf, const double *__restrict__ mu, double *__restrict__ lam,
                                   double *gp, double *gq) {
    const double sgn = (kind & KIND_OR) ? -1.0 : 1.0;
    const uint8_t hs = kind & HEAD_MASK;
    if (hs == HEAD_NONE) return;
    const double lh = hs == HEAD_FREE ? sgn * (double)vf[slot(0)] : (hs == HEAD_ONE ? INFINITY : -INFINITY);
    const double sh = sigm(lh), th = sigm(-lh);
    auto mu_of = [&](int k) {
        const uint32_t e = a.f_pos[slot(k)];
        return e == kSentinel ? 0.0 : sgn * mu[e];
    };
    // prefix pairs forward, then suffix pairs backward with the outputs
    double Pp[kSellFactorDegree + 1], Rp[kSellFactorDegree + 1];
    double P = 1.0, R = 0.0;
    bool pzero = false;
    for (int k = 1; k < deg; k++) {
        Pp[k] = P;
        Rp[k] = R;
        const double y = sgn * (double)vf[slot(k)];
        const double sk = sigm(y), tk = sigm(-y);
        pzero |= sk == 0.0;
        R = fma(P, tk, R);
        P = P * sk;
    }
    const double m0 = sh * q + th * (1.0 - q);
    double H = 0.0, dgp = 0.0, dgq = 0.0, gh = 0.0;
    if (hs == HEAD_FREE) head_terms(mu_of(0), p, q, P, R, pzero, H, dgp, dgq);
    double c[kSellFactorDegree + 1];
    double C = 0.0, Ps = 1.0, Rs = 0.0;
    for (int k = deg - 1; k >= 1; k--) {
        const double Po = Pp[k] * Ps, Ro = fma(Pp[k], Rs, Rp[k]);
        const double ak = p * Po + q * Ro, bk = (1.0 - p) * Po + (1.0 - q) * Ro;
        const double m1 = sh * ak + th * bk;
        const double mk = mu_of(k);
        c[k] = 0.0;
        if (m1 > 0.0 && m0 > 0.0 && mk != 0.0) {
            const double wk = mk * (sh - th) / m1;
            c[k] = wk * (p - q) * Po;
            dgp += wk * Po;
            dgq += wk * Ro - mk * (sh - th) / m0;
            gh += mk * sh * th * ((ak - bk) / m1 - (2.0 * q - 1.0) / m0);
        }
        C += c[k];
        const double y = sgn * (double)vf[slot(k)];
        const double sk = sigm(y), tk = sigm(-y);
        Rs = fma(sk, Rs, tk);
        Ps = sk * Ps;
    }
    for (int k = 1; k < deg; k++) {
        const double y = sgn * (double)vf[slot(k)];
        lam[slot(k)] = isfinite(y) ? sgn * sigm(-y) * (H + C - c[k]) : 0.0;
    }
    if (hs == HEAD_FREE) lam[slot(0)] = isfinite(lh) ? sgn * gh : 0.0;
    *gp += dgp;
    *gq += dgq;
}

template <typename T>
__global__ void factor_adjoint_sell_kernel(AdjArgs a, const T *__restrict__ vf, const double *__restrict__ mu,
                                           double *__restrict__ lam, double *__restrict__ gp,
                                           double *__restrict__ gq) {
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= a.nf_sell) return;
    const uint32_t base = a.fg_base[f >> 5] + (f & 31);
    const T *pq = reinterpret_cast<const T *>(a.f_pq);
    factor_adjoint_one<T>(a.f_deg[f], a.f_kind[f], (double)pq[2 * f], (double)pq[2 * f + 1],
                          [&](int k) { return base + 32u * k; }, a, vf, mu, lam, gp + f, gq + f);
}

// Big factors, one warp each: leave-one-out products from an FP64 sum of
// log-sigmoids with a count of exact zeros.
template <typename T>
__global__ void factor_adjoint_big_kernel(AdjArgs a, const T *__restrict__ vf, const double *__restrict__ mu,
                                          double *__restrict__ lam, double *__restrict__ gp, double *__restrict__ gq) {
    const uint32_t b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (b >= a.nf_big) return;
    const uint32_t f = a.nf_sell + b, s0 = a.fb_off[b], s1 = s0 + a.fb_deg[b];
    const uint8_t kind = a.f_kind[f];
    const T *pqa = reinterpret_cast<const T *>(a.f_pq);
    const double p = (double)pqa[2 * f], q = (double)pqa[2 * f + 1];
    const double sgn = (kind & KIND_OR) ? -1.0 : 1.0;
    const uint8_t hs = kind & HEAD_MASK;
    if (hs == HEAD_NONE) return;
    const double lh = hs == HEAD_FREE ? sgn * (double)vf[s0] : (hs == HEAD_ONE ? INFINITY : -INFINITY);
    const double sh = sigm(lh), th = sigm(-lh);
    auto mu_of = [&](uint32_t s) {
        const uint32_t e = a.f_pos[s];
        return e == kSentinel ? 0.0 : sgn * mu[e];
    };
    double L = 0.0;
    int nz = 0;
    for (uint32_t k = s0 + 1 + lane; k < s1; k += 32) {
        const double sk = sigm(sgn * (double)vf[k]);
        if (sk == 0.0) nz++;
        else L += log(sk);
    }
    for (int o = 16; o > 0; o >>= 1) {
        L += __shfl_xor_sync(0xffffffffu, L, o);
        nz += __shfl_xor_sync(0xffffffffu, nz, o);
    }
    const double P = nz ? 0.0 : exp(L), R = 1.0 - P;
    const double m0 = sh * q + th * (1.0 - q);
    auto loo = [&](double sk) {  // Po_k
        const bool z = sk == 0.0;
        return (nz - (int)z) ? 0.0 : exp(z ? L : L - log(sk));
    };
    double C = 0.0, dgp = 0.0, dgq = 0.0, gh = 0.0;
    for (uint32_t k = s0 + 1 + lane; k < s1; k += 32) {
        const double sk = sigm(sgn * (double)vf[k]);
        const double Po = loo(sk), Ro = 1.0 - Po;
        const double ak = p * Po + q * Ro, bk = (1.0 - p) * Po + (1.0 - q) * Ro;
        const double m1 = sh * ak + th * bk, mk = mu_of(k);
        if (m1 > 0.0 && m0 > 0.0 && mk != 0.0) {
            const double wk = mk * (sh - th) / m1;
            C += wk * (p - q) * Po;
            dgp += wk * Po;
            dgq += wk * Ro - mk * (sh - th) / m0;
            gh += mk * sh * th * ((ak - bk) / m1 - (2.0 * q - 1.0) / m0);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        C += __shfl_xor_sync(0xffffffffu, C, o);
        dgp += __shfl_xor_sync(0xffffffffu, dgp, o);
        dgq += __shfl_xor_sync(0xffffffffu, dgq, o);
        gh += __shfl_xor_sync(0xffffffffu, gh, o);
    }
    double H = 0.0;
    if (hs == HEAD_FREE) head_terms(mu_of(s0), p, q, P, R, nz > 0, H, dgp, dgq);
    for (uint32_t k = s0 + 1 + lane; k < s1; k += 32) {
        const double y = sgn * (double)vf[k];
        double ck = 0.0;
        const double sk = sigm(y), Po = loo(sk), Ro = 1.0 - Po;
        const double ak = p * Po + q * Ro, bk = (1.0 - p) * Po + (1.0 - q) * Ro;
        const double m1 = sh * ak + th * bk, mk = mu_of(k);
        if (m1 > 0.0 && m0 > 0.0 && mk != 0.0) ck = mk * (sh - th) / m1 * (p - q) * Po;
        lam[k] = isfinite(y) ? sgn * sigm(-y) * (H + C - ck) : 0.0;
    }
    if (lane == 0) {
        if (hs == HEAD_FREE) lam[s0] = isfinite(lh) ? sgn * gh : 0.0;
        gp[f] += dgp;
        gq[f] += dgq;
    }
}

}  // namespace flbp
