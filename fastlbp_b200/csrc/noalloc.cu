// Allocation-free fixed-sweep solve (flbp_run_fixed_device_noalloc).
//
// Some callers cannot allocate device memory at the moment they need a solve:
// latency-critical serving loops whose policy forbids allocation after
// start-up (cudaMalloc synchronises the device and can stall other work), and
// hosts whose GPU memory is owned by another allocator (a framework's caching
// allocator, a plugin host that hands out fixed pools) that does not allow
// out-of-band cudaMalloc. This entry point lets them run the synchronous
// sweep with buffers they already own: the graph and the belief output are
// the caller's device arrays, and the two message arrays live in one
// file-scope __device__ array of fixed size, held by every GPU that loads the
// library until the process exits.
//
// The kernels restate the engine's sweep in its simplest form (one thread per
// factor, one per variable, FP32 log-odds), computing constant messages
// inline instead of folding them, with the same closed forms as kernels.cuh.

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "engine_internal.h"
#include "kernels.cuh"

namespace flbp {

namespace {

// Message scratch: vf in the first half, fv in the second (FLBP_NOALLOC_MAX_SLOTS each).
__device__ __align__(256) float g_noalloc_scratch[2 * FLBP_NOALLOC_MAX_SLOTS];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
float *g_noalloc_ptr[kMaxDevices] = {nullptr};

__global__ void noalloc_zero(float *m, int32_t n) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m[i] = 0.f;
}

// One factor per thread: every outgoing f->v message of the factor.
__global__ void noalloc_factor(flbp_device_graph g, const float *__restrict__ vf, float *__restrict__ fv, float d) {
    const float inf = Num<float>::inf();
    for (int32_t I = blockIdx.x * blockDim.x + threadIdx.x; I < g.n_factors; I += gridDim.x * blockDim.x) {
        const int32_t s0 = g.factor_offsets[I], s1 = g.factor_offsets[I + 1], h = g.factor_head[I];
        const int32_t type = g.factor_type[I];
        const float p = g.factor_p[I], q = g.factor_q[I];
        const uint8_t hs = g.factor_head_state ? g.factor_head_state[I] : 0;
        auto put = [&](int32_t s, float o) { fv[s] = (d != 0.f) ? damp_mix(o, fv[s], d) : o; };
        if (type == FLBP_SINGLETON) {  // (1-p, p)
            put(s0, logf(p) - log1pf(-p));
            continue;
        }
        const float sg = (type == FLBP_OR) ? -1.f : 1.f;
        if (hs) {  // head-clamped: the mask's one-hot fallback; a (0,0) mask gives (0, 1) like a 1-clamp
                   // (causal_bp_parall.cu:222-238, 271-287), as the engine folds it
            put(h, (hs == 2) ? -inf : inf);
        } else if (s1 - s0 == 1) {  // reduced to its head: (1-p, p) for AND, (p, 1-p) for OR
            put(h, sg * (logf(p) - log1pf(-p)));
            continue;
        }
        if (s1 - s0 == 1) continue;
        float L = 0.f;
        int nz = 0;
        for (int32_t s = s0; s < s1; s++) {
            if (s == h) continue;
            const float ls = log_sigmoid<float>(sg * vf[s]);
            if (ls == -inf) nz++;
            else L += ls;
        }
        if (!hs) put(h, sg * head_out<float>(nz ? -inf : L, p, q, logf(p)));
        const float lh = sg * (hs == 0 ? vf[h] : hs == 1 ? inf : hs == 2 ? -inf : Num<float>::nan());
        const BodyDen<float> D = body_den<float>(lh, p, q);
        for (int32_t s = s0; s < s1; s++) {
            if (s == h) continue;
            const float ls = log_sigmoid<float>(sg * vf[s]);
            const bool z = (ls == -inf);
            const float lo = (nz - (int)z) ? -inf : (z ? L : L - ls);
            put(s, sg * body_out<float>(lo, p, q, D));
        }
    }
}

// One variable per thread: totals, then the leave-one-out v->f messages.
__global__ void noalloc_var(flbp_device_graph g, const float *__restrict__ fv, float *__restrict__ vf,
                            double *beliefs) {
    const float inf = Num<float>::inf();
    for (int32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < g.n_vars; v += gridDim.x * blockDim.x) {
        const int32_t k0 = g.var_offsets[v], k1 = g.var_offsets[v + 1];
        double S = 0.0;
        int npos = 0, nneg = 0;
        for (int32_t k = k0; k < k1; k++) {
            const float x = fv[g.var_slots[k]];
            if (x == inf) npos++;
            else if (x == -inf) nneg++;
            else S += (double)x;
        }
        if (beliefs) {
            beliefs[v] = belief_of(S, npos, nneg);
        } else {
            for (int32_t k = k0; k < k1; k++) {
                const int32_t e = g.var_slots[k];
                vf[e] = excl_msg<float>(S, npos, nneg, fv[e]);
            }
        }
    }
}

int scratch_for_current_device(float **out) {
    int dev = -1;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        set_error(std::string("no usable current CUDA device: ") + cudaGetErrorString(err));
        return FLBP_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (err != cudaSuccess || !p) {
            set_error(std::string("cudaGetSymbolAddress of the message scratch failed: ") + cudaGetErrorString(err));
            return FLBP_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = static_cast<float *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return FLBP_OK;
}

}  // namespace

}  // namespace flbp

using namespace flbp;

extern "C" int flbp_run_fixed_device_noalloc(const flbp_device_graph *g, int64_t sweeps, double damping,
                                             double *beliefs_out, void *stream) {
    if (!g || !beliefs_out || sweeps < 0 || !(damping >= 0.0 && damping < 1.0)) {
        set_error("flbp_run_fixed_device_noalloc: null graph or output, negative sweep count or damping outside [0,1)");
        return FLBP_ERR_INVALID;
    }
    if (g->n_vars < 0 || g->n_factors < 0 || g->n_slots < 0) {
        set_error("flbp_run_fixed_device_noalloc: negative graph size");
        return FLBP_ERR_INVALID;
    }
    if (g->n_slots > FLBP_NOALLOC_MAX_SLOTS) {
        set_error("flbp_run_fixed_device_noalloc: the graph has " + std::to_string(g->n_slots) +
                  " edge slots; the allocation-free path holds at most " + std::to_string(FLBP_NOALLOC_MAX_SLOTS) +
                  " (use flbp_engine_create for larger graphs)");
        return FLBP_ERR_LIMIT;
    }
    // slot_var is not read here (var_offsets / var_slots give the variable side) and may be NULL
    if ((g->n_factors > 0 && (!g->factor_offsets || !g->factor_head || !g->factor_type || !g->factor_p ||
                              !g->factor_q)) ||
        (g->n_vars > 0 && (!g->var_offsets || (g->n_slots > 0 && !g->var_slots)))) {
        set_error("flbp_run_fixed_device_noalloc: missing device array");
        return FLBP_ERR_INVALID;
    }
    float *scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    float *vf = scratch, *fv = scratch + FLBP_NOALLOC_MAX_SLOTS;
    const int threads = 256;
    const int fblocks = (int)std::max<int64_t>(1, std::min<int64_t>((g->n_factors + threads - 1) / threads, 4096));
    const int vblocks = (int)std::max<int64_t>(1, std::min<int64_t>((g->n_vars + threads - 1) / threads, 4096));
    const int zblocks = (int)std::max<int64_t>(1, std::min<int64_t>((g->n_slots + threads - 1) / threads, 4096));
    // The scratch keeps the previous call's messages: start from uniform (log-odds 0).
    if (g->n_slots > 0) {
        noalloc_zero<<<zblocks, threads, 0, st>>>(vf, (int32_t)g->n_slots);
        noalloc_zero<<<zblocks, threads, 0, st>>>(fv, (int32_t)g->n_slots);
    }
    for (int64_t t = 0; t < sweeps; t++) {
        noalloc_factor<<<fblocks, threads, 0, st>>>(*g, vf, fv, (float)damping);
        noalloc_var<<<vblocks, threads, 0, st>>>(*g, fv, vf, nullptr);
    }
    noalloc_var<<<vblocks, threads, 0, st>>>(*g, fv, vf, beliefs_out);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        set_error(std::string("flbp_run_fixed_device_noalloc: launch failed: ") + cudaGetErrorString(err));
        return FLBP_ERR_CUDA;
    }
    return FLBP_OK;
}
