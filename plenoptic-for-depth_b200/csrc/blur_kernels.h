// blur_kernels.h -- the frame's blur and richness channels from its raw image
// (blur_kernels.cu).
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

// The richness channel (GLCM contrast of every 8x8 window of the raw frame,
// normalised to [0, 255] over the frame).  contrast: W * H 16-bit scratch that
// receives the frame's contrast map; cmax: one word, the map's maximum.  For
// every view v and pixel e of its window: score[v * mi_w * mi_h + e] = the
// normalised value, binary[...] = 255 where it exceeds 10 else 0, counts[v] =
// the number of 255s; score, binary and counts may each be NULL.
cudaError_t launch_richness(const uint8_t* raw, int raw_pitch, int W, int H, const int2* origin, int V, int mi_w,
                            int mi_h, uint16_t* contrast, unsigned* cmax, float* score, uint8_t* binary,
                            uint32_t* counts, cudaStream_t st);

}  // namespace pfd
