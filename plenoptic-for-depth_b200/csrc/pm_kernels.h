// pm_kernels.h -- launchers of the PatchMatch kernels (pm_kernels.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "pm_device.cuh"

// Device-side error flags, OR-ed into the context's error word.
#define PFD_DEVERR_TMA_TIMEOUT 0x1
#define PFD_DEVERR_SWEEP_CHECK 0x10      // a sweep launch's shared-memory plan, scratch or neighbour ids did not fit

namespace pfd {

cudaError_t launch_slice(const uint8_t* raw, int raw_pitch, const int2* origin, int V, int W, int H,
                         int tile_stride, uint8_t* tiles, cudaStream_t st);
// refit: keep each pixel's plane and recompute only its cost, selected views
// and disp (the ACMM matcher's post-refine pass).
cudaError_t launch_init(const FrameDev& F, const PmParams& P, const StateDev& out, int* err, cudaStream_t st,
                        bool refit = false);
cudaError_t launch_ncc(const FrameDev& F, const PmParams& P, int nseg, int npb, const int* seg_vid,
                       const int* seg_start, const int* seg_len, const int* hyp_pxy, const float4* hyp_plane,
                       const int* hyp_out, float* costs, int* err, cudaStream_t st);
// The warp-per-pixel sweep (pm_sweep.cu): grid, shared memory, and the global
// scratch it needs (P.cost_scratch: per warp, the cost vectors of one pixel).
// shape selects one of kSweepShapes launch shapes (warps per CTA and CTAs per
// SM the registers are sized for); every shape computes the same result bit
// for bit.  Shape 0 is the default; tap counting always runs shape 0.
constexpr int kSweepShapes = 4;
int sweep_shape_warps(int shape);
// The sweep fetches neighbour samples from F.tex when the frame has textures
// (tap counting excepted), else from shared-memory quads; tex selects the plan.
cudaError_t sweep_warp_grid(const FrameDev& F, const PmParams& P, int* n_ctas, int shape = 0);
int sweep_warp_smem_bytes(const PmParams& P, bool blur, int shape, bool tex);
size_t sweep_warp_scratch_bytes(const PmParams& P, int n_ctas, int shape = 0);
// Floats of global scratch one warp uses for K neighbours (PmParams::scratch_stride).
int sweep_warp_stride(int K);
cudaError_t launch_sweep_warp(const FrameDev& F, const PmParams& P, const StateDev& prev, const StateDev& next,
                              int iter, int phase, int n_ctas, int* err, cudaStream_t st, int shape = 0);
// One frame's half-sweep in a launch over several frames (pm_sweep_batch_kernel).
struct SweepItem {
    FrameDev F;
    PmParams P;             // P.view_queue: this frame's counter, zeroed before the launch
    StateDev prev, next;
    int iter, phase;
};
// Grid of the batch kernel for `smem` bytes of dynamic shared memory per CTA.
cudaError_t sweep_batch_grid(int smem, bool blur, bool shift, bool tex, int* n_ctas, int shape = 0);
// items: device array of n frames, all with or all without a blur channel, all
// with textures (tex) or none.
cudaError_t launch_sweep_batch(const SweepItem* items, int n, bool blur, bool shift, bool tex, int smem, int n_ctas,
                               int* err, cudaStream_t st, int shape = 0);

// Fills the layered float textures of a frame's tiles: texel (x, y) of layer
// v % layers of surface v / layers is tiles[v * tile_stride + y * W + x].
cudaError_t launch_tex_fill(const uint8_t* tiles, int V, int W, int H, int tile_stride,
                            const cudaSurfaceObject_t* surfs, int layers, cudaStream_t st);

}  // namespace pfd
