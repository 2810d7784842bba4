// Device construction of the engine's layout (dlayout.h): the steps of the
// host build (layout.cpp, build_layout) as kernels and device-wide sorts and
// scans, with the same results bit for bit. Counting sorts of the host build
// become stable radix sorts of (class, tie-break) keys whose input is in
// index order, so items of equal key keep index order as on the host. The
// folded constants' log-odds (det_logit, the same bits on host and device)
// are summed per variable in factor order, as the host build sums them.

#include <cub/cub.cuh>
#include <cuda_runtime.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include <algorithm>
#include <cstring>
#include <limits>
#include <mutex>
#include <map>
#include <vector>

#include "dlayout.h"
#include "logodds.h"

namespace flbp {

namespace {

constexpr unsigned kTPB = 256;

unsigned grid_for(uint64_t n) {
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + kTPB - 1) / kTPB, 148ull * 16));
}

// Sum over a warp (every lane active). Counters that every item adds to
// take one atomic per warp: thousands of them instead of millions on one
// address, which the memory system would serialise.
__device__ __forceinline__ unsigned long long warp_sum(unsigned long long x) {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

__device__ __forceinline__ void warp_add(unsigned long long *dst, unsigned long long x) {
    x = warp_sum(x);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(dst, x);
}

#define GS_LOOP(i, n)                                                                                  \
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < (uint64_t)(n); \
         i += (uint64_t)gridDim.x * blockDim.x)

__device__ __forceinline__ bool classify_ok(const DevGraphIn &in, int64_t I) {
    const int64_t s0 = in.off[I], s1 = in.off[I + 1], d = s1 - s0;
    const int32_t t = in.type[I];
    const double p = in.p[I], q = in.q[I];
    if (t != FLBP_SINGLETON && t != FLBP_AND && t != FLBP_OR) return false;
    if (!(p >= 0.0 && p <= 1.0) || !(q >= 0.0 && q <= 1.0)) return false;
    if (d < 1) return false;
    const int64_t h = in.head[I];
    if (h < s0 || h >= s1) return false;
    if (t == FLBP_SINGLETON) return d == 1;
    return true;  // head masks other than 0 / 1 never reach the device build
}

// bad[0]: first factor whose offsets decrease; bad[1]: first slot whose
// variable is out of range; bad[2]: first malformed factor.
__global__ void k_validate(DevGraphIn in, int64_t V, int64_t F, int64_t E, unsigned long long *bad) {
    GS_LOOP(i, (F > E ? F : E)) {
        if ((int64_t)i < F) {
            if (in.off[i + 1] < in.off[i]) atomicMin(&bad[0], (unsigned long long)i);
            else if (!classify_ok(in, (int64_t)i)) atomicMin(&bad[2], (unsigned long long)i);
        }
        if ((int64_t)i < E) {
            const int64_t v = in.slot_var[i];
            if (v < 0 || v >= V) atomicMin(&bad[1], (unsigned long long)i);
        }
    }
}

// Sort key of an active factor: sliced-ELL ones by degree, then the large
// ones, too large for a tile first, by decreasing degree; inactive factors
// last. 38 bits.
constexpr int kFactorKeyBits = 38;
constexpr uint64_t kInactiveKey = (1ull << kFactorKeyBits) - 1;

// Active / head state / constant message of every factor (the host's
// classify_factor: +-det_logit(p) of singletons and of unclamped factors of
// one slot, +-inf of clamped heads), the factor sort keys and counts:
// cnt[0] sliced-ELL factors, cnt[1] large ones, cnt[2] slots of active
// factors.
__global__ void k_classify(DevGraphIn in, int64_t F, uint8_t *active, uint8_t *hstate, double *fconst,
                           uint64_t *fkey, uint32_t *fidx, unsigned long long *cnt) {
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    unsigned long long n_sell = 0, n_big = 0, n_slots = 0;
    GS_LOOP(i, F) {
        const int64_t I = (int64_t)i;
        const int64_t d = in.off[I + 1] - in.off[I];
        const int32_t t = in.type[I];
        uint8_t act = 0, hs = HEAD_FREE;
        double c = 0.0;
        if (t == FLBP_SINGLETON) {
            c = det_logit(in.p[I]);
        } else {
            const uint8_t m = in.mcode ? in.mcode[I] : kMaskFree;
            if (m != kMaskFree) {  // m0 == 0: +inf; (0, 1) head 1, (1, 0) head 0, (0, 0) neither
                c = (m == kMaskZero) ? -inf : inf;
                hs = (m == kMaskOne) ? HEAD_ONE : (m == kMaskZero) ? HEAD_ZERO : HEAD_NONE;
            } else if (d == 1) {
                const double l = det_logit(in.p[I]);
                c = (t == FLBP_AND) ? l : -l;
            }
            act = d > 1 ? 1 : 0;
        }
        active[I] = act;
        hstate[I] = hs;
        fconst[I] = c;
        fidx[I] = (uint32_t)I;
        uint64_t key = kInactiveKey;
        if (act) {
            if (d <= (int64_t)kSellFactorDegree) {
                key = (uint64_t)d << 33;
                n_sell++;
            } else {
                const uint64_t huge = (uint64_t)(d - 1 > (int64_t)kBigFactorBody ? 0 : 1);
                key = (17ull << 33) | (huge << 32) | (uint64_t)(0xffffffffu - (uint32_t)d);
                n_big++;
            }
            n_slots += (unsigned long long)d;
        }
        fkey[I] = key;
    }
    warp_add(&cnt[0], n_sell);
    warp_add(&cnt[1], n_big);
    warp_add(&cnt[2], n_slots);
}

// Per active factor in internal order: kind, (p, q), degree; large ones'
// degrees, 4-aligned run sizes and (p, q) in double.
template <typename T>
__global__ void k_fill_factor(DevGraphIn in, const uint32_t *foi, uint32_t nf, uint32_t nf_sell,
                              const uint8_t *hstate, uint8_t *f_kind, uint8_t *f_deg, T *f_pq, double *pq64,
                              uint32_t *fb_deg, uint64_t *bsz) {
    GS_LOOP(f, nf) {
        const uint32_t I = foi[f];
        const uint32_t d = (uint32_t)(in.off[I + 1] - in.off[I]);
        f_kind[f] = (uint8_t)((in.type[I] == FLBP_OR ? KIND_OR : 0) | hstate[I]);
        f_pq[2 * f] = (T)in.p[I];
        f_pq[2 * f + 1] = (T)in.q[I];
        if (f < nf_sell) {
            f_deg[f] = (uint8_t)d;
        } else {
            const uint32_t b = (uint32_t)f - nf_sell;
            fb_deg[b] = d;
            bsz[b] = (d + kRunAlign - 1) & ~(uint64_t)(kRunAlign - 1);
            pq64[2 * b] = in.p[I];
            pq64[2 * b + 1] = in.q[I];
        }
    }
}

// Group sizes 32 * width of n items sorted by ascending degree within the
// sliced-ELL range: the width of a group is the degree of its last item.
__global__ void k_group_sizes(const uint8_t *deg8, const uint32_t *deg32, const uint32_t *order, uint32_t n,
                              uint32_t ng, uint64_t *gsz) {
    GS_LOOP(gi, ng) {
        const uint64_t l64 = 32ull * gi + 31, nm1 = (uint64_t)n - 1;
        const uint32_t last = (uint32_t)(l64 < nm1 ? l64 : nm1);
        const uint32_t w = deg8 ? deg8[last] : deg32[order[last]];
        gsz[gi] = 32ull * w;
    }
}

// Device slot of every slot of an active factor: sliced-ELL factor f at
// base + 32 k (k = 0 the head, the others in reference order), a large
// factor's run contiguously, head first.
__global__ void k_dev_slot(DevGraphIn in, const uint32_t *foi, uint32_t nf, uint32_t nf_sell, const uint64_t *gbase,
                           const uint64_t *boff, uint32_t *dev_slot) {
    GS_LOOP(f, nf) {
        const uint32_t I = foi[f];
        uint64_t base, stride;
        if (f < nf_sell) {
            base = gbase[f / 32] + (f % 32);
            stride = 32;
        } else {
            base = boff[f - nf_sell];
            stride = 1;
        }
        const int64_t h = in.head[I];
        dev_slot[h] = (uint32_t)base;
        uint64_t k = 0;
        for (int64_t e = in.off[I]; e < in.off[I + 1]; e++)
            if (e != h) dev_slot[e] = (uint32_t)(base + stride * (++k));
    }
}

// Entries: every slot of an active factor reaches its variable, except a
// clamped head. Entry flags of the reference slots, variable degrees, the
// variable of each device slot, and every variable's first device slot.
__global__ void k_entries(DevGraphIn in, const uint32_t *foi, uint32_t nf, const uint8_t *hstate,
                          const uint32_t *dev_slot, uint8_t *is_entry, uint32_t *vdeg, uint32_t *var_of_dev,
                          uint32_t *first) {
    GS_LOOP(f, nf) {
        const uint32_t I = foi[f];
        const int64_t h = in.head[I];
        for (int64_t e = in.off[I]; e < in.off[I + 1]; e++) {
            if (e == h && hstate[I] != HEAD_FREE) continue;
            const uint32_t v = (uint32_t)in.slot_var[e];
            is_entry[e] = 1;
            atomicAdd(&vdeg[v], 1u);
            var_of_dev[dev_slot[e]] = v;
            atomicMin(&first[v], dev_slot[e]);
        }
    }
}

// Sort key of a variable: sliced-ELL classes by degree (degree 0 in index
// order, the others by first device slot), then the large ones, too large
// for a tile first, by decreasing degree. 39 bits. cnt: sliced-ELL count.
constexpr int kVarKeyBits = 39;
__global__ void k_var_keys(const uint32_t *vdeg, const uint32_t *first, uint64_t V, uint64_t *vkey, uint32_t *vidx,
                           unsigned long long *cnt) {
    unsigned long long n_sell = 0;
    GS_LOOP(v, V) {
        const uint32_t d = vdeg[v];
        uint64_t key;
        if (d <= kSellVarDegree) {
            key = ((uint64_t)d << 34) | (d == 0 ? 0ull : (uint64_t)first[v]);
            n_sell++;
        } else {
            const uint64_t huge = d > kTileSlotsHost ? 0 : 1;
            key = (17ull << 34) | (huge << 32) | (uint64_t)(0xffffffffu - d);
        }
        vkey[v] = key;
        vidx[v] = (uint32_t)v;
    }
    warp_add(cnt, n_sell);
}

__global__ void k_inverse(const uint32_t *order, uint64_t n, uint32_t *inv) {
    GS_LOOP(i, n) inv[order[i]] = (uint32_t)i;
}

__global__ void k_big_var(const uint32_t *order, const uint32_t *vdeg, uint32_t nv_sell, uint32_t nv_big,
                          uint32_t *vb_deg, uint64_t *vsz) {
    GS_LOOP(b, nv_big) {
        const uint32_t d = vdeg[order[nv_sell + b]];
        vb_deg[b] = d;
        vsz[b] = (d + kRunAlign - 1) & ~(uint64_t)(kRunAlign - 1);
    }
}

// First entry position and stride of every variable.
__global__ void k_epos(const uint32_t *inv, uint64_t V, uint32_t nv_sell, const uint64_t *vgb, const uint64_t *vbo,
                       uint32_t *epos, uint32_t *estride) {
    GS_LOOP(v, V) {
        const uint32_t iv = inv[v];
        if (iv < nv_sell) {
            epos[v] = (uint32_t)(vgb[iv / 32] + (iv % 32));
            estride[v] = 32;
        } else {
            epos[v] = (uint32_t)vbo[iv - nv_sell];
            estride[v] = 1;
        }
    }
}

__global__ void k_fill_u32(uint32_t *a, uint64_t n, uint32_t x) {
    GS_LOOP(i, n) a[i] = x;
}

__global__ void k_u64_to_u32(const uint64_t *a, uint64_t n, uint32_t *b) {
    GS_LOOP(i, n) b[i] = (uint32_t)a[i];
}

// (variable, device slot) of every entry, reference slots in increasing order.
__global__ void k_pair_vars(const uint32_t *ref_slots, const int32_t *slot_var, const uint32_t *dev_slot, uint64_t n,
                            uint32_t *vars, uint32_t *dslots) {
    GS_LOOP(i, n) {
        const uint32_t e = ref_slots[i];
        vars[i] = (uint32_t)slot_var[e];
        dslots[i] = dev_slot[e];
    }
}

struct ToU64 {
    __host__ __device__ __forceinline__ uint64_t operator()(uint32_t x) const { return x; }
};

// Entry k of a variable is its k-th slot in the reference's factor-major
// order: the pairs sorted by variable (stably, reference slots ascending);
// vstart = start of each variable's run.
__global__ void k_place(const uint32_t *kv, const uint32_t *ks, uint64_t n, const uint64_t *vstart,
                        const uint32_t *epos, const uint32_t *estride, uint32_t *v_ent, uint32_t *f_pos) {
    GS_LOOP(i, n) {
        const uint32_t v = kv[i], sl = ks[i];
        const uint32_t k = (uint32_t)(i - vstart[v]);
        const uint32_t ep = epos[v] + k * estride[v];
        v_ent[ep] = sl;
        f_pos[sl] = ep;
    }
}

// Folded constants: +-inf counts per internal variable; finite ones flagged
// for the ordered sums.
__global__ void k_prior_counts(DevGraphIn in, int64_t F, const uint8_t *active, const uint8_t *hstate,
                               const double *fconst, const uint32_t *inv, uint32_t *cpos, uint32_t *cneg,
                               uint8_t *finite, uint32_t *fin_var) {
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    GS_LOOP(i, F) {
        uint8_t fl = 0;
        if (!(active[i] && hstate[i] == HEAD_FREE)) {
            const uint32_t iv = inv[in.slot_var[in.head[i]]];
            const double c = fconst[i];
            if (c == inf) atomicAdd(&cpos[iv], 1u);
            else if (c == -inf) atomicAdd(&cneg[iv], 1u);
            else fl = 1;
            fin_var[i] = iv;
        }
        finite[i] = fl;
    }
}

// Sum of each variable's finite constants in factor order (runs of equal
// variable in the stably sorted list), from 0.0 as the host build adds them.
__global__ void k_prior_sums(const uint32_t *kv, const uint32_t *kf, uint64_t n, const double *fconst, double *fin,
                             uint8_t *folded) {
    GS_LOOP(i, n) {
        if (i > 0 && kv[i - 1] == kv[i]) continue;
        double s = 0.0;
        for (uint64_t j = i; j < n && kv[j] == kv[i]; j++) s += fconst[kf[j]];
        fin[kv[i]] = s;
        folded[kv[i]] = 1;
    }
}

// Packed priors in internal variable order: FP32 uint2 (float bits of the
// sum, counts); FP64 uint4 (double bits, counts, 0). Counts saturate at
// 0xffff (+inf) and 0x7fff (-inf); bit 31: a folded finite constant.
__global__ void k_pack_prior(const double *fin, const uint32_t *cpos, const uint32_t *cneg, const uint8_t *folded,
                             uint64_t V, int prec, uint32_t *out) {
    GS_LOOP(iv, V) {
        const uint32_t cnt =
            min(cpos[iv], 0xffffu) | (min(cneg[iv], 0x7fffu) << 16) | (folded[iv] ? 0x80000000u : 0u);
        if (prec == 32) {
            const float f = (float)fin[iv];
            out[2 * iv] = __float_as_uint(f);
            out[2 * iv + 1] = cnt;
        } else {
            const unsigned long long b = (unsigned long long)__double_as_longlong(fin[iv]);
            out[4 * iv] = (uint32_t)b;
            out[4 * iv + 1] = (uint32_t)(b >> 32);
            out[4 * iv + 2] = cnt;
            out[4 * iv + 3] = 0;
        }
    }
}

// Device memory of engines and of their layout builds comes from a memory
// pool per device that keeps up to kPoolKeep bytes reserved when it is
// freed: the next engine's buffers and build temporaries are then taken
// from memory already mapped instead of new cudaMalloc calls (which cost
// more than the rest of a small engine's creation, and milliseconds for a
// large one). Allocations are ordered on the creating stream; buffers are
// freed with cudaFreeAsync on the stream that uses them, or with cudaFree
// once that stream has finished (cudaFree does not wait for work that still
// reads pool memory). If the pool cannot be made, the device's default
// pool serves.
constexpr uint64_t kPoolKeep = 4ull << 30;
std::mutex g_pool_mu;
std::map<int, cudaMemPool_t> g_pools;

cudaMemPool_t device_pool() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    auto it = g_pools.find(dev);
    if (it != g_pools.end()) return it->second;
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
        cudaGetLastError();
        pool = nullptr;
    } else {
        uint64_t keep = kPoolKeep;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    g_pools[dev] = pool;
    return pool;
}

struct Pool {
    cudaStream_t st;
    cudaMemPool_t pool = device_pool();
    std::vector<void *> tmp;
    cudaError_t err = cudaSuccess;
    template <typename X>
    X *get(size_t n) {
        void *p = nullptr;
        const size_t bytes = std::max<size_t>(1, n) * sizeof(X);
        if (err == cudaSuccess)
            err = pool ? cudaMallocFromPoolAsync(&p, bytes, pool, st) : cudaMallocAsync(&p, bytes, st);
        if (p) tmp.push_back(p);
        return static_cast<X *>(p);
    }
    ~Pool() {
        for (void *p : tmp) cudaFreeAsync(p, st);
    }
};

template <typename X>
cudaError_t dalloc_out(X **p, size_t n, DevLayout &D, cudaStream_t st) {
    *p = nullptr;
    const size_t bytes = std::max<size_t>(1, n) * sizeof(X);
    cudaError_t e = pool_malloc((void **)p, bytes, st);
    if (e == cudaSuccess) D.bytes += bytes;
    return e;
}

}  // namespace

cudaError_t pool_malloc(void **p, size_t bytes, cudaStream_t st) {
    *p = nullptr;
    cudaMemPool_t pool = device_pool();
    return pool ? cudaMallocFromPoolAsync(p, bytes, pool, st) : cudaMallocAsync(p, bytes, st);
}

void free_dev_layout(DevLayout &D, cudaStream_t st) {
    void *bufs[] = {D.f_pos,      D.fg_base, D.fb_off, D.fb_deg,   D.vg_base, D.vb_off, D.vb_deg,
                    D.v_ent,      D.ftiles,  D.vtiles, D.fbt_deg,  D.vbt_deg, D.int_of_var, D.f_kind,
                    D.f_deg,      D.fbt_kind, D.f_pq,  D.fbt_pq,   D.prior,   D.vbt_prior};
    for (void *b : bufs)
        if (b) cudaFreeAsync(b, st);
    D = DevLayout();
}

#define DL_CHECK(call)                                                     \
    do {                                                                   \
        cudaError_t e_ = (call);                                           \
        if (e_ != cudaSuccess) {                                           \
            err = std::string("device layout: ") + cudaGetErrorString(e_); \
            return FLBP_ERR_CUDA;                                          \
        }                                                                  \
    } while (0)

int build_layout_device(const flbp_graph_desc &g, const DevGraphIn &in, int prec, HostLayout &L, DevLayout &D,
                        std::string &err, cudaStream_t st) {
    const int64_t V = g.n_vars, F = g.n_factors, E = g.n_slots;
    L = HostLayout();
    L.complete = false;
    L.V = V;
    L.F = F;
    L.E = E;
    Pool P{st};
    const size_t tsz = prec == 64 ? 8 : 4, psz = prec == 64 ? 16 : 8;

    // device-wide primitives with their temporary storage from the pool
    auto sort_pairs = [&](const uint64_t *ki, uint64_t *ko, const uint32_t *vi, uint32_t *vo, size_t n, int bits) {
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, ki, ko, vi, vo, n, 0, bits, st);
        void *t = P.get<char>(tb);
        if (P.err != cudaSuccess) return P.err;
        return cub::DeviceRadixSort::SortPairs(t, tb, ki, ko, vi, vo, n, 0, bits, st);
    };
    auto sort_pairs32 = [&](const uint32_t *ki, uint32_t *ko, const uint32_t *vi, uint32_t *vo, size_t n, int bits) {
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, ki, ko, vi, vo, n, 0, bits, st);
        void *t = P.get<char>(tb);
        if (P.err != cudaSuccess) return P.err;
        return cub::DeviceRadixSort::SortPairs(t, tb, ki, ko, vi, vo, n, 0, bits, st);
    };
    // b[0] = init, b[i] = init + a[0] + ... + a[i-1], i <= n
    auto excl_scan = [&](const uint64_t *a, uint64_t *b, size_t n, uint64_t init) {
        size_t tb = 0;
        cub::DeviceScan::ExclusiveScan(nullptr, tb, a, b, cub::Sum(), init, n + 1, st);
        void *t = P.get<char>(tb);
        if (P.err != cudaSuccess) return P.err;
        return cub::DeviceScan::ExclusiveScan(t, tb, a, b, cub::Sum(), init, n + 1, st);
    };
    auto bits_for = [](uint64_t n) {
        int b = 1;
        while (b < 32 && ((n - 1) >> b)) b++;
        return b;
    };
    auto read = [&](void *dst, const void *src, size_t bytes) -> cudaError_t {
        cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st);
        return e == cudaSuccess ? cudaStreamSynchronize(st) : e;
    };

    // --- validation: the host build's checks, the first offender of each ----------------
    {
        unsigned long long *bad = P.get<unsigned long long>(3);
        DL_CHECK(P.err);
        DL_CHECK(cudaMemsetAsync(bad, 0xff, 3 * sizeof(unsigned long long), st));
        if (F > 0 || E > 0) k_validate<<<grid_for((uint64_t)std::max(F, E)), kTPB, 0, st>>>(in, V, F, E, bad);
        unsigned long long hb[3];
        DL_CHECK(cudaGetLastError());
        DL_CHECK(read(hb, bad, sizeof(hb)));
        if (hb[0] != ~0ull) {
            err = "factor_offsets not monotone at factor " + std::to_string(hb[0]);
            return FLBP_ERR_INVALID;
        }
        if (hb[1] != ~0ull) {
            err = "slot_var out of range at slot " + std::to_string(hb[1]);
            return FLBP_ERR_INVALID;
        }
        if (hb[2] != ~0ull) {
            uint8_t a, h;
            double c;
            classify_factor(g, (int64_t)hb[2], a, h, c, &err);
            return FLBP_ERR_INVALID;
        }
    }

    // --- classify, folded log-odds, internal factor order --------------------
    uint8_t *active = P.get<uint8_t>(F), *hstate = P.get<uint8_t>(F);
    double *fconst = P.get<double>(F);
    uint64_t *fkey = P.get<uint64_t>(F), *fkey2 = P.get<uint64_t>(F);
    uint32_t *fidx = P.get<uint32_t>(F), *foi = P.get<uint32_t>(F);
    unsigned long long *cnt = P.get<unsigned long long>(4);
    DL_CHECK(P.err);
    DL_CHECK(cudaMemsetAsync(cnt, 0, 4 * sizeof(unsigned long long), st));
    if (F > 0) k_classify<<<grid_for(F), kTPB, 0, st>>>(in, F, active, hstate, fconst, fkey, fidx, cnt);
    if (F > 0) DL_CHECK(sort_pairs(fkey, fkey2, fidx, foi, (size_t)F, kFactorKeyBits));
    unsigned long long hc[4];
    DL_CHECK(cudaGetLastError());
    DL_CHECK(read(hc, cnt, sizeof(hc)));
    const uint32_t nf_sell = (uint32_t)hc[0], nf_big = (uint32_t)hc[1], nf = nf_sell + nf_big;
    L.nf_sell = nf_sell;
    L.nf_big = nf_big;
    L.n_active_slots = hc[2];
    const uint32_t ngf = (nf_sell + 31) / 32;
    D.nf_pad = std::max<size_t>(nf, 32ull * ngf);

    // --- per-factor arrays, device slots -----------------------------------------------------
    DL_CHECK(dalloc_out(&D.f_kind, D.nf_pad, D, st));
    DL_CHECK(dalloc_out(&D.f_deg, D.nf_pad, D, st));
    DL_CHECK(dalloc_out((char **)&D.f_pq, 2 * D.nf_pad * tsz, D, st));
    DL_CHECK(dalloc_out(&D.fb_deg, nf_big, D, st));
    DL_CHECK(cudaMemsetAsync(D.f_kind, 0, D.nf_pad, st));
    DL_CHECK(cudaMemsetAsync(D.f_deg, 0, D.nf_pad, st));
    DL_CHECK(cudaMemsetAsync(D.f_pq, 0, 2 * D.nf_pad * tsz, st));
    double *bpq = P.get<double>(2 * (size_t)nf_big);
    uint64_t *bsz = P.get<uint64_t>((size_t)nf_big + 1), *gsz = P.get<uint64_t>((size_t)ngf + 1);
    uint64_t *gbase = P.get<uint64_t>((size_t)ngf + 1), *boff = P.get<uint64_t>((size_t)nf_big + 1);
    DL_CHECK(P.err);
    if (nf > 0) {
        if (prec == 64)
            k_fill_factor<double><<<grid_for(nf), kTPB, 0, st>>>(in, foi, nf, nf_sell, hstate, D.f_kind, D.f_deg,
                                                                 (double *)D.f_pq, bpq, D.fb_deg, bsz);
        else
            k_fill_factor<float><<<grid_for(nf), kTPB, 0, st>>>(in, foi, nf, nf_sell, hstate, D.f_kind, D.f_deg,
                                                                (float *)D.f_pq, bpq, D.fb_deg, bsz);
    }
    if (ngf > 0) k_group_sizes<<<grid_for(ngf), kTPB, 0, st>>>(D.f_deg, nullptr, nullptr, nf_sell, ngf, gsz);
    DL_CHECK(excl_scan(gsz, gbase, ngf, 0));
    uint64_t h_gend = 0;
    DL_CHECK(cudaGetLastError());
    DL_CHECK(read(&h_gend, gbase + ngf, 8));
    DL_CHECK(excl_scan(bsz, boff, nf_big, h_gend));
    uint64_t n_slots = 0;
    DL_CHECK(read(&n_slots, boff + nf_big, 8));
    if (n_slots >= UINT32_MAX) {
        err = "graph exceeds 2^32-1 device slots";
        return FLBP_ERR_LIMIT;
    }
    L.n_slots = n_slots;
    uint32_t *dev_slot = P.get<uint32_t>(E);
    DL_CHECK(P.err);
    DL_CHECK(cudaMemsetAsync(dev_slot, 0xff, std::max<int64_t>(1, E) * 4, st));
    if (nf > 0) k_dev_slot<<<grid_for(nf), kTPB, 0, st>>>(in, foi, nf, nf_sell, gbase, boff, dev_slot);
    // group bases and run offsets as 32-bit arrays, and their host copies
    DL_CHECK(dalloc_out(&D.fg_base, (size_t)ngf + 1, D, st));
    DL_CHECK(dalloc_out(&D.fb_off, (size_t)nf_big + 1, D, st));
    k_u64_to_u32<<<grid_for((uint64_t)ngf + 1), kTPB, 0, st>>>(gbase, (uint64_t)ngf + 1, D.fg_base);
    k_u64_to_u32<<<grid_for((uint64_t)nf_big + 1), kTPB, 0, st>>>(boff, (uint64_t)nf_big + 1, D.fb_off);
    L.fg_base.resize((size_t)ngf + 1);
    L.fb_off.resize((size_t)nf_big + 1);
    L.fb_deg.resize(nf_big);
    std::vector<uint8_t> big_kind(nf_big);
    std::vector<double> big_pq(2 * (size_t)nf_big);
    DL_CHECK(cudaGetLastError());
    DL_CHECK(cudaMemcpyAsync(L.fg_base.data(), D.fg_base, L.fg_base.size() * 4, cudaMemcpyDeviceToHost, st));
    DL_CHECK(cudaMemcpyAsync(L.fb_off.data(), D.fb_off, L.fb_off.size() * 4, cudaMemcpyDeviceToHost, st));
    if (nf_big) {
        DL_CHECK(cudaMemcpyAsync(L.fb_deg.data(), D.fb_deg, (size_t)nf_big * 4, cudaMemcpyDeviceToHost, st));
        DL_CHECK(cudaMemcpyAsync(big_kind.data(), D.f_kind + nf_sell, nf_big, cudaMemcpyDeviceToHost, st));
        DL_CHECK(cudaMemcpyAsync(big_pq.data(), bpq, big_pq.size() * 8, cudaMemcpyDeviceToHost, st));
    }

    // --- variable entries and the internal variable order -------------------------------------
    uint32_t *vdeg = P.get<uint32_t>(V), *first = P.get<uint32_t>(V), *var_of_dev = P.get<uint32_t>(n_slots);
    uint8_t *is_entry = P.get<uint8_t>(E);
    uint64_t *vkey = P.get<uint64_t>(V), *vkey2 = P.get<uint64_t>(V);
    uint32_t *vidx = P.get<uint32_t>(V), *order = P.get<uint32_t>(V);
    DL_CHECK(P.err);
    DL_CHECK(dalloc_out(&D.int_of_var, (size_t)V, D, st));
    DL_CHECK(cudaMemsetAsync(vdeg, 0, std::max<int64_t>(1, V) * 4, st));
    DL_CHECK(cudaMemsetAsync(first, 0xff, std::max<int64_t>(1, V) * 4, st));
    DL_CHECK(cudaMemsetAsync(var_of_dev, 0xff, std::max<uint64_t>(1, n_slots) * 4, st));
    DL_CHECK(cudaMemsetAsync(is_entry, 0, std::max<int64_t>(1, E), st));
    if (nf > 0)
        k_entries<<<grid_for(nf), kTPB, 0, st>>>(in, foi, nf, hstate, dev_slot, is_entry, vdeg, var_of_dev, first);
    DL_CHECK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), st));
    if (V > 0) {
        k_var_keys<<<grid_for(V), kTPB, 0, st>>>(vdeg, first, V, vkey, vidx, cnt);
        DL_CHECK(sort_pairs(vkey, vkey2, vidx, order, (size_t)V, kVarKeyBits));
        k_inverse<<<grid_for(V), kTPB, 0, st>>>(order, V, D.int_of_var);
    }
    DL_CHECK(cudaGetLastError());
    DL_CHECK(read(hc, cnt, 8));
    const uint32_t nv_sell = (uint32_t)hc[0], nv_big = (uint32_t)(V - nv_sell);
    L.nv_sell = nv_sell;
    L.nv_big = nv_big;
    const uint32_t ngv = (nv_sell + 31) / 32;
    D.nv_pad = std::max<size_t>((size_t)V, 32ull * ngv);

    // --- entry positions ---------------------------------------------------------------------
    uint64_t *vgsz = P.get<uint64_t>((size_t)ngv + 1), *vgb = P.get<uint64_t>((size_t)ngv + 1);
    uint64_t *vsz = P.get<uint64_t>((size_t)nv_big + 1), *vbo = P.get<uint64_t>((size_t)nv_big + 1);
    DL_CHECK(P.err);
    DL_CHECK(dalloc_out(&D.vb_deg, nv_big, D, st));
    if (ngv > 0) k_group_sizes<<<grid_for(ngv), kTPB, 0, st>>>(nullptr, vdeg, order, nv_sell, ngv, vgsz);
    DL_CHECK(excl_scan(vgsz, vgb, ngv, 0));
    if (nv_big > 0) k_big_var<<<grid_for(nv_big), kTPB, 0, st>>>(order, vdeg, nv_sell, nv_big, D.vb_deg, vsz);
    uint64_t nent = 0;
    DL_CHECK(cudaGetLastError());
    DL_CHECK(read(&nent, vgb + ngv, 8));
    DL_CHECK(excl_scan(vsz, vbo, nv_big, nent));
    uint64_t n_ent = 0;
    DL_CHECK(read(&n_ent, vbo + nv_big, 8));
    if (n_ent >= UINT32_MAX) {
        err = "graph exceeds 2^32-1 variable entries";
        return FLBP_ERR_LIMIT;
    }
    D.n_ent = n_ent;
    DL_CHECK(dalloc_out(&D.vg_base, (size_t)ngv + 1, D, st));
    DL_CHECK(dalloc_out(&D.vb_off, (size_t)nv_big + 1, D, st));
    k_u64_to_u32<<<grid_for((uint64_t)ngv + 1), kTPB, 0, st>>>(vgb, (uint64_t)ngv + 1, D.vg_base);
    k_u64_to_u32<<<grid_for((uint64_t)nv_big + 1), kTPB, 0, st>>>(vbo, (uint64_t)nv_big + 1, D.vb_off);
    uint32_t *epos = P.get<uint32_t>(V), *estride = P.get<uint32_t>(V);
    DL_CHECK(P.err);
    if (V > 0) k_epos<<<grid_for(V), kTPB, 0, st>>>(D.int_of_var, V, nv_sell, vgb, vbo, epos, estride);
    DL_CHECK(dalloc_out(&D.v_ent, n_ent, D, st));
    DL_CHECK(dalloc_out(&D.f_pos, n_slots, D, st));
    k_fill_u32<<<grid_for(n_ent), kTPB, 0, st>>>(D.v_ent, n_ent, kSentinel);
    k_fill_u32<<<grid_for(n_slots), kTPB, 0, st>>>(D.f_pos, n_slots, kSentinel);
    {
        // the (variable, device slot) pairs in reference slot order, stably sorted by variable
        uint32_t *refs = P.get<uint32_t>(E), *vars = P.get<uint32_t>(E), *dsl = P.get<uint32_t>(E);
        uint32_t *kv = P.get<uint32_t>(E), *ks = P.get<uint32_t>(E);
        int *nsel = P.get<int>(1);
        uint64_t *vstart = P.get<uint64_t>((size_t)V + 1);
        DL_CHECK(P.err);
        thrust::counting_iterator<uint32_t> it(0);
        size_t tb = 0;
        cub::DeviceSelect::Flagged(nullptr, tb, it, is_entry, refs, nsel, (int)E, st);
        void *t = P.get<char>(tb);
        DL_CHECK(P.err);
        DL_CHECK(cub::DeviceSelect::Flagged(t, tb, it, is_entry, refs, nsel, (int)E, st));
        int h_nsel = 0;
        DL_CHECK(read(&h_nsel, nsel, sizeof(int)));
        const uint64_t npairs = (uint64_t)h_nsel;
        if (npairs > 0) {
            k_pair_vars<<<grid_for(npairs), kTPB, 0, st>>>(refs, in.slot_var, dev_slot, npairs, vars, dsl);
            DL_CHECK(sort_pairs32(vars, kv, dsl, ks, npairs, bits_for((uint64_t)std::max<int64_t>(V, 2))));
            // run starts: exclusive scan of the degrees in variable order
            auto d64 = thrust::make_transform_iterator(vdeg, ToU64());
            size_t tb2 = 0;
            cub::DeviceScan::ExclusiveSum(nullptr, tb2, d64, vstart, (int)V, st);
            void *t2 = P.get<char>(tb2);
            DL_CHECK(P.err);
            DL_CHECK(cub::DeviceScan::ExclusiveSum(t2, tb2, d64, vstart, (int)V, st));
            k_place<<<grid_for(npairs), kTPB, 0, st>>>(kv, ks, npairs, vstart, epos, estride, D.v_ent, D.f_pos);
        }
    }
    L.vg_base.resize((size_t)ngv + 1);
    L.vb_off.resize((size_t)nv_big + 1);
    L.vb_deg.resize(nv_big);
    DL_CHECK(cudaGetLastError());
    DL_CHECK(cudaMemcpyAsync(L.vg_base.data(), D.vg_base, L.vg_base.size() * 4, cudaMemcpyDeviceToHost, st));
    DL_CHECK(cudaMemcpyAsync(L.vb_off.data(), D.vb_off, L.vb_off.size() * 4, cudaMemcpyDeviceToHost, st));
    if (nv_big) DL_CHECK(cudaMemcpyAsync(L.vb_deg.data(), D.vb_deg, (size_t)nv_big * 4, cudaMemcpyDeviceToHost, st));

    // --- priors -----------------------------------------------------------------------------
    {
        uint32_t *cpos = P.get<uint32_t>(D.nv_pad), *cneg = P.get<uint32_t>(D.nv_pad);
        uint8_t *finite = P.get<uint8_t>(F), *folded = P.get<uint8_t>(D.nv_pad);
        uint32_t *fin_var = P.get<uint32_t>(F), *sel_f = P.get<uint32_t>(F), *sel_v = P.get<uint32_t>(F);
        uint32_t *kv = P.get<uint32_t>(F), *kf = P.get<uint32_t>(F);
        double *fin = P.get<double>(D.nv_pad);
        int *nsel = P.get<int>(1);
        DL_CHECK(P.err);
        DL_CHECK(cudaMemsetAsync(cpos, 0, D.nv_pad * 4, st));
        DL_CHECK(cudaMemsetAsync(cneg, 0, D.nv_pad * 4, st));
        DL_CHECK(cudaMemsetAsync(folded, 0, D.nv_pad, st));
        DL_CHECK(cudaMemsetAsync(fin, 0, D.nv_pad * 8, st));
        DL_CHECK(dalloc_out((char **)&D.prior, D.nv_pad * psz, D, st));
        DL_CHECK(cudaMemsetAsync(D.prior, 0, D.nv_pad * psz, st));
        if (F > 0) {
            k_prior_counts<<<grid_for(F), kTPB, 0, st>>>(in, F, active, hstate, fconst, D.int_of_var, cpos, cneg,
                                                        finite, fin_var);
            thrust::counting_iterator<uint32_t> it(0);
            size_t tb = 0;
            cub::DeviceSelect::Flagged(nullptr, tb, it, finite, sel_f, nsel, (int)F, st);
            void *t = P.get<char>(tb);
            DL_CHECK(P.err);
            DL_CHECK(cub::DeviceSelect::Flagged(t, tb, it, finite, sel_f, nsel, (int)F, st));
            size_t tb2 = 0;
            cub::DeviceSelect::Flagged(nullptr, tb2, fin_var, finite, sel_v, nsel, (int)F, st);
            void *t2 = P.get<char>(tb2);
            DL_CHECK(P.err);
            DL_CHECK(cub::DeviceSelect::Flagged(t2, tb2, fin_var, finite, sel_v, nsel, (int)F, st));
            int h_n = 0;
            DL_CHECK(read(&h_n, nsel, sizeof(int)));
            if (h_n > 0) {
                DL_CHECK(sort_pairs32(sel_v, kv, sel_f, kf, (size_t)h_n,
                                      bits_for((uint64_t)std::max<size_t>(D.nv_pad, 2))));
                k_prior_sums<<<grid_for(h_n), kTPB, 0, st>>>(kv, kf, (uint64_t)h_n, fconst, fin, folded);
            }
        }
        k_pack_prior<<<grid_for(D.nv_pad), kTPB, 0, st>>>(fin, cpos, cneg, folded, D.nv_pad, prec,
                                                          (uint32_t *)D.prior);
        DL_CHECK(cudaGetLastError());
    }

    // --- tiles, headers and the large items' per-tile constants (host, small) -------------------
    DL_CHECK(cudaStreamSynchronize(st));
    build_tiles(L, big_kind.data(), big_pq.data());
    std::vector<uint32_t> big_prior((size_t)nv_big * (psz / 4));
    if (nv_big)
        DL_CHECK(read(big_prior.data(), (const char *)D.prior + (size_t)nv_sell * psz, (size_t)nv_big * psz));
    std::vector<uint32_t> bt_prior(std::max<size_t>(1, L.vbt_deg.size()) * (psz / 4), 0u);
    for (uint32_t t = 0; t < L.n_vbtiles; t++) {
        const uint32_t *h = &L.vhdr[(size_t)kHdrWordsHost * t];
        const uint32_t b0 = h[0], n = h[1] & ~kBigTileFlag;
        for (uint32_t j = 0; j < n; j++) {
            const size_t k = (size_t)kTileGroupsHost * t + j, b = (size_t)b0 + j;
            std::copy(&big_prior[b * (psz / 4)], &big_prior[(b + 1) * (psz / 4)], &bt_prior[k * (psz / 4)]);
        }
    }
    bt_prior.resize(L.vbt_deg.size() * (psz / 4));
    auto up = [&](auto **dst, const auto &src, size_t n_elems) -> cudaError_t {
        cudaError_t e = dalloc_out(dst, n_elems, D, st);
        if (e == cudaSuccess && !src.empty())
            e = cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(src[0]), cudaMemcpyHostToDevice, st);
        return e;
    };
    DL_CHECK(up(&D.ftiles, L.fhdr, L.fhdr.size()));
    DL_CHECK(up(&D.vtiles, L.vhdr, L.vhdr.size()));
    DL_CHECK(up(&D.fbt_deg, L.fbt_deg, L.fbt_deg.size()));
    DL_CHECK(up(&D.vbt_deg, L.vbt_deg, L.vbt_deg.size()));
    DL_CHECK(up(&D.fbt_kind, L.fbt_kind, L.fbt_kind.size()));
    std::vector<float> f32;
    if (prec == 64) {
        DL_CHECK(up((double **)&D.fbt_pq, L.fbt_pq, L.fbt_pq.size()));
    } else {
        f32.assign(L.fbt_pq.begin(), L.fbt_pq.end());
        DL_CHECK(up((float **)&D.fbt_pq, f32, f32.size()));
    }
    DL_CHECK(up((uint32_t **)&D.vbt_prior, bt_prior, L.vbt_deg.size() * (psz / 4)));
    DL_CHECK(cudaStreamSynchronize(st));  // the host sources above are released at return
    return FLBP_OK;
}

}  // namespace flbp
