// select_kernels.h -- micro-image similarity for the neighbour selection (select_kernels.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pfd {

// out[p] = MeasureSimilarity(micro-image pairs[p].x, micro-image pairs[p].y):
// gray [V][tile_stride] (W x H dense), centres [V].
cudaError_t launch_similarity(const uint8_t* gray, int tile_stride, int W, int H, const float2* centers,
                              const int2* pairs, int n, int* out, cudaStream_t st);

}  // namespace pfd
