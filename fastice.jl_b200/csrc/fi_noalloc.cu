// fi_noalloc.cu -- residual norms for callers that cannot allocate device memory.
//
// fi_residual_norms_noalloc runs the same fused residual + norm reduction as
// fi_model_residual_norms, on field pointers the caller owns, but keeps the
// per-block partial results in a file-scope static device array instead of a
// buffer allocated by a model.  Callers that cannot call cudaMalloc: a host
// program whose device memory is owned by another runtime's allocator or pool
// (a Julia or Python runtime that hands out device pointers and counts every
// byte), and long-running services that fix their device memory at start-up and
// forbid allocation afterwards (an allocation there could fail or stall a loop).
// The first call on a device looks up the array's device address
// (cudaGetSymbolAddress) and caches it; make that first call before any stream
// capture.  The cache is per process: after cudaDeviceReset (or anything else
// that unloads the library's module on a device) the cached address is stale,
// so a program that resets a device must not call this entry point afterwards.
//
// Limits and sharing.  The reduction runs a grid-stride loop over
// norm_blocks(grid) blocks (at most 148 * 8, whatever the grid size), the same
// block count as the model's own entry point, so the two give identical bits.
// The array holds kNoAllocSlots per-block partials (kNoAllocSlots * 12 doubles,
// 192 KiB), and every loaded device keeps its own copy until the process exits;
// a launch needing more blocks than slots would be rejected with FI_ERR_ARG (no
// grid does with these constants).  All calls on a device share the one array:
// calls whose work overlaps on the GPU (on different streams, or from several
// host threads) race on it and must be serialised by the caller.  Every slot a
// call reads is written by the same call first, so nothing needs clearing
// between calls.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "fi_internal.h"

namespace fi {
namespace {

constexpr int kNoAllocSlots = 2048;
constexpr int kMaxDevices = 64;

// per-block partials (FI_NORMS_LEN-slot layout), one copy per device
static __device__ __align__(256) double g_noalloc_partials[kNoAllocSlots * kNormSlots];
// device address of g_noalloc_partials on each device, filled once per device
// under g_partials_lock (host threads may make their first calls concurrently)
static double *g_partials_addr[kMaxDevices] = {};
static std::mutex g_partials_lock;

fi_status scratch_for_current_device(double **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return set_error("device ordinal beyond the no-alloc table"), FI_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> guard(g_partials_lock);
    if (!g_partials_addr[dev]) {
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_partials);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
        g_partials_addr[dev] = (double *)ptr;
    }
    *out = g_partials_addr[dev];
    return FI_OK;
}

}  // namespace
}  // namespace fi

using namespace fi;

extern "C" fi_status fi_residual_norms_noalloc(const fi_model_desc *desc, const fi_state_view *state, double *out_dev,
                                               void *stream) {
    if (!desc || !state || !out_dev) return set_error("null argument"), FI_ERR_ARG;
    const fi_grid &gr = desc->grid;
    if (gr.nd != 2 && gr.nd != 3) return set_error("grid.nd must be 2 or 3"), FI_ERR_ARG;
    for (int k = 0; k < gr.nd; k++)
        if (gr.n[k] < 3 || !(gr.extent[k] > 0.0)) return set_error("invalid grid"), FI_ERR_ARG;
    if (desc->dtype != FI_F64 && desc->dtype != FI_F32) return set_error("dtype must be FI_F64 or FI_F32"), FI_ERR_ARG;
    if (desc->immersed && gr.nd != 3) return set_error("the immersed-boundary model is 3D only"), FI_ERR_UNSUPPORTED;
    if (state->pitch < (size_t)gr.n[0] + 3) return set_error("state pitch smaller than n0 + 3"), FI_ERR_ARG;
    const bool three = gr.nd == 3;
    if (!state->P || !state->txx || !state->tyy || !state->txy || !state->Vx || !state->Vy ||
        (three && (!state->tzz || !state->txz || !state->tyz || !state->Vz)))
        return set_error("missing state field pointer"), FI_ERR_ARG;
    for (int c = 0; c < gr.nd; c++)
        if (desc->gravity.kind[c] == FI_G_FIELD && !state->g[c]) return set_error("missing gravity field"), FI_ERR_ARG;
    if (desc->immersed)
        for (int c = 0; c < 8; c++)
            if (!state->na[c] || !state->ns[c]) return set_error("missing immersed-boundary mask"), FI_ERR_ARG;

    Geom g{};
    g.nd = gr.nd;
    for (int k = 0; k < 3; k++) g.n[k] = k < gr.nd ? gr.n[k] : 0;
    g.pitch = (long long)state->pitch;
    g.rows = gr.n[1] + 3;
    g.sxy = g.pitch * g.rows;
    g.planes = three ? gr.n[2] + 3 : 1;
    KParams kp{};
    for (int k = 0; k < 3; k++) kp.inv_dx[k] = k < gr.nd ? 1.0 / (gr.extent[k] / gr.n[k]) : 0.0;
    for (int k = 0; k < 3; k++) {
        kp.g_kind[k] = desc->gravity.kind[k];
        kp.g_val[k] = desc->gravity.value[k];
        for (int s = 0; s < 2; s++) kp.bc_kind[k][s] = k < gr.nd ? desc->bc[k][s].kind : FI_BC_TRACTION;
    }
    kp.small = desc->dtype == FI_F64 ? 1e-6 : (double)small_threshold_f32();
    // the model's own block count: a grid-stride reduction whose partials fit the array
    const int blocks = norm_blocks(g);
    if (blocks > kNoAllocSlots)
        return set_error("the reduction needs " + std::to_string(blocks) + " partial slots, the no-alloc scratch has " +
                         std::to_string(kNoAllocSlots)),
               FI_ERR_ARG;

    double *scratch = nullptr;
    fi_status st = scratch_for_current_device(&scratch);
    if (st != FI_OK) return st;

    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    if (desc->dtype == FI_F64) {
        Ptrs<double> f{};
        f.P = (double *)state->P; f.txx = (double *)state->txx; f.tyy = (double *)state->tyy; f.tzz = (double *)state->tzz;
        f.txy = (double *)state->txy; f.txz = (double *)state->txz; f.tyz = (double *)state->tyz;
        f.Vx = (double *)state->Vx; f.Vy = (double *)state->Vy; f.Vz = (double *)state->Vz;
        f.gx = (const double *)state->g[0]; f.gy = (const double *)state->g[1]; f.gz = (const double *)state->g[2];
        for (int c = 0; c < 8; c++) {
            f.wna[c] = (const double *)state->na[c];
            f.wns[c] = (const double *)state->ns[c];
        }
        e = launch_residual_norms<double>(g, kp, f, desc->immersed != 0, scratch, blocks, out_dev, s);
    } else {
        Ptrs<float> f{};
        f.P = (float *)state->P; f.txx = (float *)state->txx; f.tyy = (float *)state->tyy; f.tzz = (float *)state->tzz;
        f.txy = (float *)state->txy; f.txz = (float *)state->txz; f.tyz = (float *)state->tyz;
        f.Vx = (float *)state->Vx; f.Vy = (float *)state->Vy; f.Vz = (float *)state->Vz;
        f.gx = (const float *)state->g[0]; f.gy = (const float *)state->g[1]; f.gz = (const float *)state->g[2];
        for (int c = 0; c < 8; c++) {
            f.wna[c] = (const float *)state->na[c];
            f.wns[c] = (const float *)state->ns[c];
        }
        e = launch_residual_norms<float>(g, kp, f, desc->immersed != 0, scratch, blocks, out_dev, s);
    }
    if (e != cudaSuccess) return cuda_fail(e, "no-alloc residual norms");
    return FI_OK;
}
