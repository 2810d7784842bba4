// Construction of the engine's device layout on the GPU (dlayout.cu).
//
// The result equals the host build (build_layout, layout.cpp) bit for bit:
// the same item orders, slots, entries, priors and tile headers. The device
// arrays the sweep reads are built and left on the device; the host receives
// only the layout's counts and its small arrays (group bases, large-item
// runs, tile headers and per-tile constants), which is what the launch code
// needs. The per-slot and per-item arrays that other host-side features read
// (message export, gradients, clamps, schedules) are not filled here: the
// engine builds the complete host layout from the graph when one of them is
// first used.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "engine_internal.h"

namespace flbp {

// The caller's graph arrays on the device (reference order), in a compact
// form: offsets, slot variables and heads as int32 (the device build serves
// graphs below 2^30 slots), factor types as int8, and per factor the masks
// of a clamped head as one code (kMaskFree: not clamped or masks (1, 1);
// kMaskOne (0, 1); kMaskZero (1, 0); kMaskNone (0, 0)), null when no head
// is clamped. Values that do not fit (and masks other than 0 / 1) send the
// graph to the host build, which reports them.
constexpr uint8_t kMaskFree = 0, kMaskOne = 1, kMaskZero = 2, kMaskNone = 3;
struct DevGraphIn {
    const int32_t *off = nullptr, *slot_var = nullptr, *head = nullptr;
    const int8_t *type = nullptr;
    const uint8_t *mcode = nullptr;
    const double *p = nullptr, *q = nullptr;
};

// Device buffers of a layout (owned by the caller once built). Per-item
// arrays are padded to whole groups of 32 like the host build's uploads.
struct DevLayout {
    uint32_t *f_pos = nullptr, *fg_base = nullptr, *fb_off = nullptr, *fb_deg = nullptr;
    uint32_t *vg_base = nullptr, *vb_off = nullptr, *vb_deg = nullptr, *v_ent = nullptr;
    uint32_t *ftiles = nullptr, *vtiles = nullptr, *fbt_deg = nullptr, *vbt_deg = nullptr, *int_of_var = nullptr;
    uint8_t *f_kind = nullptr, *f_deg = nullptr, *fbt_kind = nullptr;
    void *f_pq = nullptr, *fbt_pq = nullptr, *prior = nullptr, *vbt_prior = nullptr;
    size_t bytes = 0;      // device memory held by these buffers
    size_t nf_pad = 0, nv_pad = 0, n_ent = 0;
};

// Builds the layout of graph `g` (sizes and, on the host, the arrays that
// the validation messages and the folded constants need) from its device
// copy `in`, for messages of `prec` bits (32 / 64). Fills the counts and
// small arrays of L (L.complete false) and the buffers of D. On a malformed
// graph returns the host build's error code and message.
int build_layout_device(const flbp_graph_desc &g, const DevGraphIn &in, int prec, HostLayout &L, DevLayout &D,
                        std::string &err, cudaStream_t st);

// Frees the buffers of D in the order of stream st.
void free_dev_layout(DevLayout &D, cudaStream_t st);

// Device memory from the per-device pool that engines and layout builds
// share, ordered on st; freed with cudaFreeAsync, or with cudaFree once no
// queued work reads it.
cudaError_t pool_malloc(void **p, size_t bytes, cudaStream_t st);

}  // namespace flbp
