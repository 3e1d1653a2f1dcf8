// fuse_kernels.h -- virtual-depth fusion and all-in-focus splat (fuse_kernels.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pfd {

constexpr int kFuseMaxList = 128;                 // neighbour-list entries a reference pixel visits

struct FuseFrame {
    int V, m, ppv, tile_stride;
    const uint8_t* gray;          // [V][tile_stride]
    const uint8_t* bgr;           // [V][ppv][3] or nullptr (gray in all channels)
    const float2* centers;        // [V]
    const float4* plane;          // [V * ppv] normal and disparity
    const int* lists;             // [V][max_list] view ids, -1 = no result
    const int* list_counts;       // [V]
    int max_list;
    float mla_base, min_ref_disp, max_reproj_px, max_rel_vd;
    int min_consistent;
    int raw_w, raw_h;
    uint8_t* mask;                // [V * ppv], zero at the start
    unsigned int* winner;         // [raw_h * raw_w]: 1 + sequence number of the last point there, 0 = none
    float* rec;                   // [V * ppv][10]: point, normal, colour, consistent count
    unsigned int* has_rec;        // [V * ppv]: 1 where a point inside the raw frame was recorded
};

// One wavefront step: the reference micro-images views[0..n), one warp each.
cudaError_t launch_fuse_step(const FuseFrame& F, const int* views, int n, cudaStream_t st);
// The maps from the winning points (outputs zeroed where no point landed).
cudaError_t launch_fuse_maps(const FuseFrame& F, float* vd_map, uint8_t* conf, uint8_t* aif, cudaStream_t st);
// Points in sequence order: counts per block of 1024 sequence numbers, then the
// scatter given each block's exclusive offset.
constexpr int kFuseScanBlock = 1024;
cudaError_t launch_fuse_count(const FuseFrame& F, unsigned int* block_counts, cudaStream_t st);
cudaError_t launch_fuse_compact(const FuseFrame& F, const unsigned int* block_offsets, float* points, cudaStream_t st);

}  // namespace pfd
