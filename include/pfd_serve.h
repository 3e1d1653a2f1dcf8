/*
 * pfd_serve.h -- request loop of libpfd.so: raw frames of any size and lens
 * pitch are submitted as they arrive and matched concurrently on one GPU.
 * Same conventions as pfd_abi.h.
 *
 * A server owns `slots` engine contexts (each with its own stream) and one
 * dispatcher thread.  A submitted request is copied, queued, and admitted in
 * arrival order as soon as a slot is free and its device memory fits the HBM
 * budget beside the requests already running; its frame is uploaded,
 * initialised and swept (the plane/cost state stays on the device across its
 * PatchMatch iterations), optionally filtered, and its state copied back.
 * Requests running in different slots overlap on the device: their kernels
 * come from different streams, and a frame that does not fill the GPU
 * leaves room for the others'.  Every request computes exactly what
 * pfd_frame_upload + pfd_patchmatch (+ pfd_filter) + pfd_download compute for
 * it alone, bit for bit.
 *
 * The reference has no request loop; this is the serving form layered on the
 * drop-in path (the reference processes one frame at a time and resets the
 * device between frames, DepthSolver.cpp:327-433).
 */
#ifndef PFD_SERVE_H
#define PFD_SERVE_H

#include "pfd_abi.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pfd_server pfd_server;

/* One frame to match.  Every pointer is read during pfd_server_submit only. */
typedef struct {
    const uint8_t* raw;            /* W x H 8-bit gray, rows raw_pitch bytes apart */
    int W, H, raw_pitch;
    const float* centers;          /* [n_views][2] */
    const int* tilekeys;           /* [n_views][2] */
    int n_views, mi_w, mi_h;
    const int* nb_ids;             /* [n_views][max_nb] */
    const int* nb_counts;          /* [n_views] */
    int max_nb;
    pfd_pm_params params;          /* params.max_iterations: this request's PatchMatch iterations */
    uint64_t seed;
    int run_filter;                /* 1: pfd_filter after the sweeps */
    pfd_filter_cfg filter_cfg;
    float baseline_unit;           /* for the filter */
} pfd_request;

/* A server on CUDA device `device` (-1: the current one) with `slots`
 * concurrent requests (1..16) inside hbm_budget_bytes of frame memory (0 = no
 * cap). */
pfd_status pfd_server_create(pfd_server** out, int device, size_t hbm_budget_bytes, int slots);
/* Waits for the running requests, drops the queued ones, frees everything. */
void pfd_server_destroy(pfd_server* srv);
/* Queues a copy of the request; never waits for the device.  PFD_EINVAL for a
 * malformed request, PFD_ENOMEM when it alone exceeds the budget. */
pfd_status pfd_server_submit(pfd_server* srv, const pfd_request* req, uint64_t* ticket);
/* Waits up to timeout_ms (< 0: without limit) for the request to finish and
 * copies its state (layout of pfd_download; any pointer may be NULL), then
 * forgets the ticket.  PFD_ETIMEDOUT if it has not finished (the ticket stays
 * valid); the request's own error otherwise.  latency_ms (may be NULL):
 * submission to completion on the device. */
pfd_status pfd_server_wait(pfd_server* srv, uint64_t ticket, int timeout_ms, float* plane, float* cost,
                           float* disp, uint32_t* sel, double* latency_ms);
/* Requests queued, running, and device bytes admitted now. */
pfd_status pfd_server_load(pfd_server* srv, int* queued, int* running, size_t* bytes_admitted);
/* Text of the server's last failure ("" if none). */
const char* pfd_server_last_error(pfd_server* srv);

/* Device bytes a frame of this shape holds (what the budget admission counts). */
size_t pfd_frame_bytes(int W, int H, int n_views, int mi_w, int mi_h, int max_nb, int has_blur);

#ifdef __cplusplus
}
#endif
#endif
