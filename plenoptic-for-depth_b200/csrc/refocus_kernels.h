// refocus_kernels.h -- focal-stack render (refocus_kernels.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pfd {

// Lens centres bucketed on a square grid (cell of a centre c:
// floorf((c.x - grid_x0) * (1.0f / cell)), clamped to the grid), view ids
// ascending inside each cell.
struct RefocusFrame {
    int V, m, mh, tile_stride;
    const uint8_t* gray;          // [V][tile_stride] micro-images, m x mh dense
    const float2* centers;        // [V]
    const int* cell_start;        // [grid_w * grid_h + 1]
    const int* cell_ids;          // [V]
    int grid_w, grid_h;
    float grid_x0, grid_y0, cell;
};

constexpr int kMaxRefocusCand = 2048;             // lenses that may reach one 64 x 16 output tile
#define PFD_DEVERR_REFOCUS_LENSES 0x2             // a tile saw more than kMaxRefocusCand lenses

int refocus_smem_bytes(const RefocusFrame& F);
cudaError_t launch_refocus(const RefocusFrame& F, const float* slice_vd, int n_slices, int raw_w, int raw_h, int out_w,
                           int out_h, float* out, int* err, cudaStream_t st);

}  // namespace pfd
