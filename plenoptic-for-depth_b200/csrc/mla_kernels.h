// mla_kernels.h -- micro-lens centre detection from a white image (mla_kernels.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define PFD_DEVERR_MLA_UNION 0x4                  // a union-find merge did not settle (bounded retries)
#define PFD_DEVERR_MLA_TRACE 0x8                  // a border did not close within its step bound

namespace pfd {

// hist [256] must start at zero.
cudaError_t launch_mla_hist(const uint8_t* bgr, int W, int H, int step, unsigned int* hist, cudaStream_t st);
// fg [W*H], L [W*H]; roots receives up to max_roots component roots (unordered),
// n_roots (starting at zero) their count.
cudaError_t launch_mla_components(const uint8_t* bgr, int W, int H, int step, int threshold, uint8_t* fg, int* L,
                                  int* roots, unsigned int* n_roots, int max_roots, int* err, cudaStream_t st);
// The layout of pfd_mla_lens (include/pfd_abi.h).
struct pfd_mla_lens_dev {
    int col, row;
    float cx, cy, area;
    int abandon;
};
// partial [nblocks][14]: per block, the upper triangle of A^T A (10) and A^T z (4)
// of the hexagonal lattice fit over the lenses.
cudaError_t launch_mla_lattice(const pfd_mla_lens_dev* lens, int n, double* partial, int nblocks, cudaStream_t st);
// sums [n][3]: the contour sums a00, a10, a01 of each start pixel's outer border.
cudaError_t launch_mla_trace(const uint8_t* fg, int W, int H, const int* starts, int n, double* sums, int* err,
                             cudaStream_t st);

}  // namespace pfd
