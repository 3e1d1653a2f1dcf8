/*
 * pfd_host.h -- host-side (CPU) helpers of libpfd.so that prepare the inputs
 * of the device path.  Same conventions as pfd_abi.h.
 */
#ifndef PFD_HOST_H
#define PFD_HOST_H

#include "pfd_abi.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Ordered neighbour lists for matching, the order
 * SelectNeighbors::CollectMIANeighImagesForMatch (MINeighbor/SelectNeighbors.cpp:113-193)
 * produces when no candidate is rejected by its similarity/RANSAC test:
 * hexagonal rings grown breadth-first with the |dist - pitch| < 0.15 pitch test
 * (:195-420), score 1 - normalised baseline (:770-832), std::sort descending
 * over key-ordered candidates (MVStereo/LFDepthInfo.cpp:214-241).
 * centers [n][2], tilekeys [n][2] (column, row); rings >= 1 (the reference
 * collects up to 5); out: nb_ids [n][max_nb] (-1 padded), nb_counts [n]. */
pfd_status pfd_neighbors_by_baseline(const float* centers, const int* tilekeys, int n_views, float pitch,
                                     int rings, int max_nb, int* nb_ids, int* nb_counts);

#ifdef __cplusplus
}
#endif
#endif
