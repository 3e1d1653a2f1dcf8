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

/* Ordered neighbour lists for matching from the lens geometry alone: the
 * lists pfd_select_neighbors produces when no candidate is rejected by its
 * similarity test (every similarity 0), i.e. the reference's ring walk
 * (MINeighbor/SelectNeighbors.cpp:195-417,925-978) over `rings` rings (1..5; the
 * reference searches up to 5) and its normalised-baseline score and sort
 * (:770-832, MVStereo/LFDepthInfo.cpp:214-241,404-429).  The key grid spans the
 * largest column and row present.  centers [n][2], tilekeys [n][2] (column,
 * row); out: nb_ids [n][max_nb] (-1 padded), nb_counts [n] (<= max_nb <= 128). */
pfd_status pfd_neighbors_by_baseline(const float* centers, const int* tilekeys, int n_views, float pitch,
                                     int rings, int max_nb, int* nb_ids, int* nb_counts);

#ifdef __cplusplus
}
#endif
#endif
