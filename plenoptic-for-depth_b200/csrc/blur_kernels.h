// blur_kernels.h -- the frame's blur channel from its raw image (blur_kernels.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pfd {

// For every view v (window origin[v], mi_w x mi_h) and pixel (x, y) of its
// window: tiles[v * tile_stride + y * mi_w + x] = the 4-neighbour Laplacian of
// the raw frame (W x H, rows raw_pitch bytes apart) at (origin + (x, y)),
// borders reflected without repeating the edge, saturated to [0, 255]; the
// tile's padding bytes are zero.  counts (may be NULL): [V] pixels of the
// window whose Laplacian exceeds 10.
cudaError_t launch_blur(const uint8_t* raw, int raw_pitch, int W, int H, const int2* origin, int V, int mi_w,
                        int mi_h, int tile_stride, uint8_t* tiles, uint32_t* counts, cudaStream_t st);

}  // namespace pfd
