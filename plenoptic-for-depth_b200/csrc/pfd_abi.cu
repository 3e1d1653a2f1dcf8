// pfd_abi.cu -- implementation of include/pfd_abi.h: contexts, frames and the
// PatchMatch entry points.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/pfd_abi.h"
#include "pm_kernels.h"
#include "check_kernels.h"
#include "refocus_kernels.h"
#include "vdrd_kernels.h"
#include "fuse_kernels.h"
#include "mla_kernels.h"
#include "neighbors.h"
#include "select_kernels.h"
#include "blur_kernels.h"

namespace {

// SelectNeighbors' candidate rings of every view, which depend on the lens
// geometry only (ComputeNearestCircleKeys, SelectNeighbors.cpp:195-365), and
// the (view, candidate) pairs whose similarities the device computes.
struct RingPlan {
    int u = 0, v = 0;
    float pitch = 0.0f;
    pfd::LensGrid G;
    std::vector<std::vector<std::vector<int>>> R;
    std::vector<int2> pairs;
    std::vector<size_t> first;       // [view * 5 + ring] offset into pairs
    bool build(const float* centers, const int* keys, int n, int u_size, int v_size, float p)
    {
        if (!G.build(centers, keys, n, u_size, v_size)) return false;
        u = u_size;
        v = v_size;
        pitch = p;
        pfd::collect_rings(G, pitch, 5, R);
        pairs.clear();
        first.assign((size_t)n * 5 + 1, 0);
        for (int i = 0; i < n; ++i)
            for (int k = 0; k < 5; ++k) {
                first[(size_t)i * 5 + k] = pairs.size();
                for (int m : R[i][k]) pairs.push_back(make_int2(i, m));
            }
        first[(size_t)n * 5] = pairs.size();
        return true;
    }
};

// A launch sequence of one frame replayed from a CUDA graph: the key of the
// call it was captured from, and the frame's host-side bookkeeping as the
// sequence leaves it (restored after each replay).
struct FrameGraph {
    std::vector<unsigned char> key;   // the call's arguments and the context modes; empty = none
    bool warm = false;                // one call with this key ran uncaptured (allocations, tuning done)
    cudaGraphExec_t exec = nullptr;
    unsigned long long launches = 0;  // kernels in the graph
    unsigned scratch_gen = 0;         // the context's scratch generation at capture
    int cur = 0;
    unsigned cvec_valid = 0;
    pfd_pm_params cvec_key = {};
    int cvec_mode = 0;
    void reset()
    {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        key.clear();
        warm = false;
    }
};

// One channel of a frame's micro-image tiles (gray or blur) as layered float
// textures for the sweep's fetches: view v is layer v % layers of array
// v / layers.  The surfaces write the same arrays.
struct TexTiles {
    std::vector<cudaArray_t> arr;
    std::vector<cudaTextureObject_t> tex;
    std::vector<cudaSurfaceObject_t> surf;
    cudaTextureObject_t* d_tex = nullptr;     // the texture handles on the device (frame allocation)
    cudaSurfaceObject_t* d_surf = nullptr;    // the surface handles on the device (frame allocation)
    bool stale = true;                        // the tiles changed since the last fill
    bool ready() const { return d_tex != nullptr; }
    void release()
    {
        for (auto t : tex) cudaDestroyTextureObject(t);
        for (auto t : surf) cudaDestroySurfaceObject(t);
        for (auto a : arr) cudaFreeArray(a);
        tex.clear(); surf.clear(); arr.clear();
        d_tex = nullptr; d_surf = nullptr;
        stale = true;
    }
};

struct Frame {
    int W = 0, H = 0;                 // raw frame
    int V = 0, mi_w = 0, mi_h = 0, K = 0, tile_stride = 0;
    bool has_raw = false, has_blur = false;
    bool has_mi = false;              // micro-image tiles filled (from a raw frame or uploaded)
    uint8_t* d_raw = nullptr;
    uint8_t* d_gray = nullptr;
    uint8_t* d_blur = nullptr;
    float2* d_centers = nullptr;
    int2* d_tilekeys = nullptr;
    int2* d_origin = nullptr;
    int* d_nb_ids = nullptr;
    int* d_nb_counts = nullptr;
    pfd::StateDev s[2] = {};
    int cur = 0;                      // s[cur] is the latest state
    // Cost vector of every pixel's current plane ([V*ppv][K]), written by the
    // initialisation and by each sweep for the pixels it updates; bit c of
    // cvec_valid says the vectors of colour c match the latest state under the
    // parameters cvec_key (patch, tap stride, sigmas, base).
    float* d_cvec = nullptr;
    unsigned cvec_valid = 0;
    pfd_pm_params cvec_key = {};
    int cvec_mode = 0;                        // cost_mode() of the context that computed cvec
    bool has_state = false;
    size_t bytes = 0;
    bool registered = false;          // bytes already counted in the context's total
    std::vector<void*> allocs;
    // host copies for scheduling the consistency pass
    std::vector<int> h_keys, h_nb_ids, h_nb_counts;
    uint8_t* d_reason = nullptr;      // filter reject reasons, allocated on first use
    float* d_err = nullptr;           // reprojection-error map, allocated on first use
    int* d_steps = nullptr;           // views grouped by wavefront step
    std::vector<int> step_start;      // [n_steps + 1] offsets into d_steps
    pfd::CycleTileRec* d_cyc_recs = nullptr;   // cycle check: per-view sums, allocated on first use
    unsigned int* d_cyc_hist = nullptr;        // cycle check: masked geometric-error histogram
    float* d_cyc_maps = nullptr;               // cycle check: geo and photo error maps
    uint8_t* d_cyc_tm = nullptr;               // cycle check: texture mask
    bool cyc_done = false;                     // d_cyc_recs / d_cyc_hist hold a cycle check
    std::vector<float> h_centers;              // lens centres, for the refocus bucket grid
    int* d_cells = nullptr;                    // refocus: cell_start [cells + 1] then cell_ids [V]
    int grid_w = 0, grid_h = 0;
    float grid_x0 = 0.f, grid_y0 = 0.f, grid_cell = 0.f;
    float* d_slice_vd = nullptr;               // refocus: slice virtual depths [kMaxSlices]
    float* d_stack = nullptr;                  // refocus: focal stack
    size_t stack_bytes = 0;
    unsigned long long* d_fstats = nullptr;    // filter counters, allocated on first use
    // neighbour selection: the rings of the frame's lens grid, kept for the next call
    std::shared_ptr<RingPlan> rings;
    int2* d_pairs = nullptr;                   // rings->pairs on the device
    int* d_sims = nullptr;                     // their similarities
    size_t n_pairs_alloc = 0;                  // entries d_pairs and d_sims hold
    // CUDA graphs of the enqueue-only PatchMatch and filter (pfd_set_graphs)
    FrameGraph pm_graph, filter_graph;
    // the tiles as textures: [0] gray, [1] blur; tex_layers views per array
    TexTiles tx[2];
    int tex_layers = 0;
};

}  // namespace

struct pfd_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    size_t budget = 0, used = 0;
    int next_id = 1;
    std::map<int, Frame> frames;
    int* d_err = nullptr;
    unsigned long long* d_taps = nullptr;   // tap counter of calibration runs
    int* d_vq = nullptr;                    // sweep: next micro-image to take (reset before each launch)
    bool counting = false;
    int ncc_moments = PFD_NCC_REFERENCE;    // accumulation of the NCC moments (pfd_set_ncc_moments)
    int matcher = PFD_MATCHER_FRAME;        // PatchMatch rules (pfd_set_matcher)
    unsigned long long launches = 0;        // kernels this context has launched
    float* d_scratch = nullptr;             // sweep candidate costs, per resident CTA
    size_t scratch_bytes = 0;
    int sweep_shape = 0;                    // launch shape of the half-sweeps, or PFD_SHAPE_AUTOTUNE
    int sweep_fetch = PFD_FETCH_SHARED;     // where the half-sweeps read neighbour samples
    bool graphs = false;                    // replay pfd_patchmatch / pfd_filter from CUDA graphs
    unsigned scratch_gen = 0;               // bumped whenever d_scratch moves (graphs hold its address)
    std::string last_error;
};

namespace {

pfd_status fail(pfd_ctx* c, pfd_status code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->last_error = buf;
    return code;
}

#define CU(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return fail(ctx, PFD_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        int now = -1;
        cudaGetDevice(&now);
        if (prev >= 0 && now != prev) cudaSetDevice(prev);
    }
};

pfd_status frame_alloc(pfd_ctx* ctx, Frame& f, void** p, size_t bytes)
{
    const size_t pending = f.registered ? 0 : f.bytes;
    if (ctx->budget && ctx->used + pending + bytes > ctx->budget)
        return fail(ctx, PFD_ENOMEM, "HBM budget exceeded: %zu in use + %zu requested > %zu",
                    ctx->used + pending, bytes, ctx->budget);
    // stream-ordered: no device-wide synchronisation, so frames of other contexts
    // (other streams) keep running while this one allocates or frees
    cudaError_t e = cudaMallocAsync(p, bytes, ctx->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, PFD_ENOMEM, "cudaMallocAsync(%zu): %s", bytes, cudaGetErrorString(e));
    }
    f.allocs.push_back(*p);
    f.bytes += bytes;
    if (f.registered) ctx->used += bytes;
    return PFD_OK;
}

// Frees one buffer obtained from frame_alloc.
void frame_free_one(pfd_ctx* ctx, Frame& f, void* p, size_t bytes)
{
    if (!p) return;
    cudaFreeAsync(p, ctx->stream);
    for (size_t i = 0; i < f.allocs.size(); ++i)
        if (f.allocs[i] == p) { f.allocs.erase(f.allocs.begin() + (long)i); break; }
    f.bytes -= bytes;
    if (f.registered) ctx->used -= bytes;
}

// Creates channel c's textures (c = 0 gray, 1 blur) of frame f: float arrays of
// mi_w x mi_h texels, up to the device's layer limit each, with a linear-filter,
// clamped, unnormalised-coordinate texture and a surface on each.
pfd_status tex_create(pfd_ctx* ctx, Frame& f, int c)
{
    TexTiles& T = f.tx[c];
    if (T.ready()) return PFD_OK;
    int max_layers = 0, max_w = 0, max_h = 0;
    cudaDeviceGetAttribute(&max_layers, cudaDevAttrMaxTexture2DLayeredLayers, ctx->device);
    cudaDeviceGetAttribute(&max_w, cudaDevAttrMaxTexture2DLayeredWidth, ctx->device);
    cudaDeviceGetAttribute(&max_h, cudaDevAttrMaxTexture2DLayeredHeight, ctx->device);
    if (max_layers < 1 || f.mi_w > max_w || f.mi_h > max_h)
        return fail(ctx, PFD_EINVAL, "micro-image %dx%d does not fit a layered texture", f.mi_w, f.mi_h);
    const int layers = std::min(max_layers, f.V);
    const int n = (f.V + layers - 1) / layers;
    const size_t bytes = (size_t)f.V * f.mi_w * f.mi_h * sizeof(float);
    const size_t pending = f.registered ? 0 : f.bytes;
    if (ctx->budget && ctx->used + pending + bytes > ctx->budget)
        return fail(ctx, PFD_ENOMEM, "HBM budget exceeded: %zu in use + %zu requested > %zu", ctx->used + pending,
                    bytes, ctx->budget);
    pfd_status st = frame_alloc(ctx, f, (void**)&T.d_tex, sizeof(cudaTextureObject_t) * n);
    if (st == PFD_OK) st = frame_alloc(ctx, f, (void**)&T.d_surf, sizeof(cudaSurfaceObject_t) * n);
    if (st != PFD_OK) { T.d_tex = nullptr; T.d_surf = nullptr; return st; }
    const cudaChannelFormatDesc cd = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < n && e == cudaSuccess; ++i) {
        const int nl = std::min(layers, f.V - i * layers);
        cudaArray_t a = nullptr;
        e = cudaMalloc3DArray(&a, &cd, make_cudaExtent(f.mi_w, f.mi_h, nl), cudaArrayLayered | cudaArraySurfaceLoadStore);
        if (e != cudaSuccess) break;
        T.arr.push_back(a);
        cudaResourceDesc rd = {};
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = a;
        cudaTextureDesc td = {};
        td.addressMode[0] = cudaAddressModeClamp;
        td.addressMode[1] = cudaAddressModeClamp;
        td.addressMode[2] = cudaAddressModeClamp;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 0;
        cudaTextureObject_t t = 0;
        e = cudaCreateTextureObject(&t, &rd, &td, nullptr);
        if (e != cudaSuccess) break;
        T.tex.push_back(t);
        cudaSurfaceObject_t sf = 0;
        e = cudaCreateSurfaceObject(&sf, &rd);
        if (e != cudaSuccess) break;
        T.surf.push_back(sf);
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(T.d_tex, T.tex.data(), sizeof(cudaTextureObject_t) * n, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(T.d_surf, T.surf.data(), sizeof(cudaSurfaceObject_t) * n, cudaMemcpyHostToDevice,
                            ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);      // the handle vectors stay; no staging dies
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaStreamSynchronize(ctx->stream);
        void* dt = T.d_tex; void* ds = T.d_surf;
        T.release();
        frame_free_one(ctx, f, dt, sizeof(cudaTextureObject_t) * n);
        frame_free_one(ctx, f, ds, sizeof(cudaSurfaceObject_t) * n);
        return fail(ctx, PFD_ECUDA, "micro-image textures: %s", cudaGetErrorString(e));
    }
    f.tex_layers = layers;
    f.bytes += bytes;
    if (f.registered) ctx->used += bytes;
    T.stale = true;
    return PFD_OK;
}

// Refills the textures of every channel whose tiles changed since the last
// fill (stream-ordered before the sweeps that read them).  With create, first
// creates the textures the frame lacks when the context fetches from textures
// (an allocation, and a synchronisation of the context's stream).
pfd_status tex_refresh(pfd_ctx* ctx, Frame& f, bool create = true)
{
    if (create && ctx->sweep_fetch == PFD_FETCH_TEXTURE) {
        for (int c = 0; c < (f.has_blur ? 2 : 1); ++c) {
            const pfd_status st = tex_create(ctx, f, c);
            if (st != PFD_OK) return st;
        }
    }
    for (int c = 0; c < 2; ++c) {
        TexTiles& T = f.tx[c];
        const uint8_t* tiles = c == 0 ? f.d_gray : (f.has_blur ? f.d_blur : nullptr);
        if (!T.ready() || !T.stale || !tiles) continue;
        const cudaError_t e = pfd::launch_tex_fill(tiles, f.V, f.mi_w, f.mi_h, f.tile_stride, T.d_surf, f.tex_layers,
                                                   ctx->stream);
        if (e != cudaSuccess) return fail(ctx, PFD_ECUDA, "texture fill: %s", cudaGetErrorString(e));
        ctx->launches += 1;
        T.stale = false;
    }
    return PFD_OK;
}

void frame_release(Frame& f, cudaStream_t s)
{
    f.pm_graph.reset();
    f.filter_graph.reset();
    if (f.tx[0].ready() || f.tx[1].ready() || !f.tx[0].arr.empty() || !f.tx[1].arr.empty()) {
        cudaStreamSynchronize(s);                // no launch in flight reads the arrays
        f.tx[0].release();
        f.tx[1].release();
    }
    for (void* p : f.allocs) cudaFreeAsync(p, s);
    f.allocs.clear();
    f.bytes = 0;
}

Frame* find_frame(pfd_ctx* ctx, int id)
{
    auto it = ctx->frames.find(id);
    return it == ctx->frames.end() ? nullptr : &it->second;
}

pfd_status check_params(pfd_ctx* ctx, const Frame& f, const pfd_pm_params* p)
{
    if (!p) return fail(ctx, PFD_EINVAL, "params is NULL");
    if (p->patch_size < 1 || (p->patch_size & 1) == 0 || p->patch_size > 31)
        return fail(ctx, PFD_EINVAL, "patch_size must be odd in [1, 31], got %d", p->patch_size);
    if (p->radius_increment < 1) return fail(ctx, PFD_EINVAL, "radius_increment must be >= 1");
    if (!(p->sigma_spatial > 0.0f) || !(p->sigma_color > 0.0f))
        return fail(ctx, PFD_EINVAL, "sigma_spatial and sigma_color must be > 0");
    if (!(p->base > 0.0f)) return fail(ctx, PFD_EINVAL, "base (lens pitch) must be > 0");
    if (p->top_k < 1) return fail(ctx, PFD_EINVAL, "top_k must be >= 1");
    if (p->max_iterations < 0) return fail(ctx, PFD_EINVAL, "max_iterations must be >= 0");
    if (!f.has_mi) return fail(ctx, PFD_ESTATE, "frame has no micro-images yet");
    return PFD_OK;
}

pfd::PmParams make_params(const pfd_ctx* ctx, const Frame& f, const pfd_pm_params* p, uint64_t seed)
{
    pfd::PmParams P;
    P.shifted = ctx->ncc_moments == PFD_NCC_SHIFTED ? 1 : 0;
    // the ACMM matcher's blur penalty gain and write-back (AdaptMIPMFrameACMM.cu:99,880-900)
    P.acmm = ctx->matcher == PFD_MATCHER_ACMM ? 1 : 0;
    P.blur_gain = P.acmm ? 0.8f : 2.0f;
    P.W = f.mi_w; P.H = f.mi_h; P.ppv = f.mi_w * f.mi_h;
    P.K = f.K;
    P.radius = p->patch_size / 2;
    P.inc = p->radius_increment;
    P.ntap = (2 * P.radius) / P.inc + 1;
    P.top_k = p->top_k;
    P.ss2 = (2.0f * p->sigma_spatial) * p->sigma_spatial;
    P.cc2 = (2.0f * p->sigma_color) * p->sigma_color;
    P.depth_min = p->depth_min;
    P.depth_max = p->depth_max;
    P.base = p->base;
    P.inv_base = 1.0f / std::max(p->base, 1e-6f);
    P.pert_pi = (float)((double)0.02f * 3.14159265358979323846);
    const float fw = (float)f.mi_w, fh = (float)f.mi_h;
    std::memcpy(&P.W_bits, &fw, 4);
    std::memcpy(&P.H_bits, &fh, 4);
    P.tile_stride = f.tile_stride;
    P.seed = seed;
    P.tap_counter = nullptr;
    P.cost_scratch = nullptr;
    P.scratch_floats = 0;
    P.scratch_stride = pfd::sweep_warp_stride(f.K);
    P.cvec = f.d_cvec;
    P.view_queue = ctx->d_vq;
    P.cvec_ok = 0;
    return P;
}

// The stored cost vectors depend on the parameters that shape an NCC.
bool same_cost_params(const pfd_pm_params& a, const pfd_pm_params& b)
{
    return a.patch_size == b.patch_size && a.radius_increment == b.radius_increment &&
           std::memcmp(&a.sigma_spatial, &b.sigma_spatial, 4) == 0 &&
           std::memcmp(&a.sigma_color, &b.sigma_color, 4) == 0 && std::memcmp(&a.base, &b.base, 4) == 0;
}

// Before a sweep of `phase`: may it use the stored vectors?  After it: the
// updated colour's vectors are valid under `p`.
// Everything of the context that shapes a cost vector besides the parameters:
// the moment mode and the matcher (its blur penalty gain).
int cost_mode(const pfd_ctx* ctx) { return ctx->ncc_moments | (ctx->matcher << 1); }

bool cvec_usable(const Frame& f, const pfd_pm_params& p, int phase, int mode)
{
    return ((f.cvec_valid >> phase) & 1u) && same_cost_params(f.cvec_key, p) && f.cvec_mode == mode;
}
void cvec_swept(Frame& f, const pfd_pm_params& p, int phase, int mode)
{
    if (!same_cost_params(f.cvec_key, p) || f.cvec_mode != mode) f.cvec_valid = 0;
    f.cvec_key = p;
    f.cvec_mode = mode;
    f.cvec_valid |= 1u << phase;
}

pfd::FrameDev frame_dev(const Frame& f)
{
    pfd::FrameDev F;
    F.gray = f.d_gray;
    F.blur = f.has_blur ? f.d_blur : nullptr;
    F.centers = f.d_centers;
    F.nb_ids = f.d_nb_ids;
    F.nb_counts = f.d_nb_counts;
    F.V = f.V;
    F.tex = nullptr;
    F.tex_blur = nullptr;
    F.tex_layers = f.tex_layers;
    return F;
}

// The frame as the sweep sees it: with its textures when the context fetches
// from them and every channel the frame has is held as textures.
pfd::FrameDev sweep_dev(const pfd_ctx* ctx, const Frame& f)
{
    pfd::FrameDev F = frame_dev(f);
    if (ctx->sweep_fetch == PFD_FETCH_TEXTURE && f.tx[0].ready() && (!f.has_blur || f.tx[1].ready())) {
        F.tex = f.tx[0].d_tex;
        F.tex_blur = f.has_blur ? f.tx[1].d_tex : nullptr;
    }
    return F;
}

pfd_status check_device_error(pfd_ctx* ctx)
{
    int h = 0;
    CU(cudaMemcpyAsync(&h, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    if (h) {
        CU(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
        if (h == PFD_DEVERR_REFOCUS_LENSES)
            return fail(ctx, PFD_EINVAL, "refocus: more than %d lenses reach one output tile (slice virtual depth "
                        "too large for this lens density)", pfd::kMaxRefocusCand);
        if (h & PFD_DEVERR_SWEEP_CHECK)
            return fail(ctx, PFD_ECUDA, "sweep launch refused its work: shared-memory plan, scratch or neighbour "
                        "ids out of range (flags 0x%x)", h);
        return fail(ctx, PFD_ETIMEDOUT, "device wait timed out (flags 0x%x)", h);
    }
    return PFD_OK;
}

}  // namespace

extern "C" {

pfd_status pfd_create(pfd_ctx** out, int device, size_t hbm_budget_bytes)
{
    pfd_ctx* ctx = nullptr;
    if (!out) return PFD_EINVAL;
    *out = nullptr;
    int n = 0;
    if (device == -1 && cudaGetDevice(&device) != cudaSuccess) device = -2;   // the caller's current device
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return PFD_ENODEV;
    }
    ctx = new (std::nothrow) pfd_ctx;
    if (!ctx) return PFD_ENOMEM;
    ctx->device = device;
    {
        // frames come and go with every request: keep their memory in this process's
        // pool instead of handing it back to the driver at each synchronisation
        DeviceGuard g0(device);
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaGetLastError();
    }
    ctx->budget = hbm_budget_bytes;
    DeviceGuard g(device);
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&ctx->d_err, sizeof(int)) != cudaSuccess ||
        cudaMemset(ctx->d_err, 0, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&ctx->d_taps, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMemset(ctx->d_taps, 0, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&ctx->d_vq, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        if (ctx->d_err) cudaFree(ctx->d_err);
        if (ctx->d_taps) cudaFree(ctx->d_taps);
        if (ctx->d_vq) cudaFree(ctx->d_vq);
        delete ctx;
        return PFD_ECUDA;
    }
    *out = ctx;
    return PFD_OK;
}

void pfd_destroy(pfd_ctx* ctx)
{
    if (!ctx) return;
    DeviceGuard g(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto& kv : ctx->frames) frame_release(kv.second, ctx->stream);
    ctx->frames.clear();
    cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->d_err);
    cudaFree(ctx->d_taps);
    cudaFree(ctx->d_vq);
    if (ctx->d_scratch) cudaFreeAsync(ctx->d_scratch, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}

pfd_status pfd_set_tap_counting(pfd_ctx* ctx, int enable)
{
    if (!ctx) return PFD_EINVAL;
    ctx->counting = enable != 0;
    return PFD_OK;
}

pfd_status pfd_set_ncc_moments(pfd_ctx* ctx, int mode)
{
    if (!ctx) return PFD_EINVAL;
    if (mode != PFD_NCC_REFERENCE && mode != PFD_NCC_SHIFTED)
        return fail(ctx, PFD_EINVAL, "NCC moment mode %d is neither PFD_NCC_REFERENCE nor PFD_NCC_SHIFTED", mode);
    ctx->ncc_moments = mode;
    return PFD_OK;
}

pfd_status pfd_set_matcher(pfd_ctx* ctx, int matcher)
{
    if (!ctx) return PFD_EINVAL;
    if (matcher != PFD_MATCHER_FRAME && matcher != PFD_MATCHER_ACMM)
        return fail(ctx, PFD_EINVAL, "matcher %d is neither PFD_MATCHER_FRAME nor PFD_MATCHER_ACMM", matcher);
    ctx->matcher = matcher;
    return PFD_OK;
}

pfd_status pfd_read_tap_count(pfd_ctx* ctx, unsigned long long* taps)
{
    if (!ctx || !taps) return PFD_EINVAL;
    DeviceGuard g(ctx->device);
    CU(cudaMemcpyAsync(taps, ctx->d_taps, sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaMemsetAsync(ctx->d_taps, 0, sizeof(unsigned long long), ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return PFD_OK;
}

const char* pfd_last_error(pfd_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

void* pfd_stream(pfd_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

size_t pfd_bytes_in_use(pfd_ctx* ctx) { return ctx ? ctx->used : 0; }

pfd_status pfd_sync(pfd_ctx* ctx)
{
    if (!ctx) return PFD_EINVAL;
    DeviceGuard g(ctx->device);
    return check_device_error(ctx);
}

pfd_status pfd_frame_create(pfd_ctx* ctx, int* frame_id, int W, int H, const float* centers, const int* tilekeys,
                            int n_views, int mi_w, int mi_h, const int* nb_ids, const int* nb_counts, int max_nb,
                            const uint8_t* blur)
{
    if (!ctx || !frame_id) return PFD_EINVAL;
    *frame_id = 0;
    if (W <= 0 || H <= 0 || n_views <= 0 || !centers || !tilekeys || !nb_ids || !nb_counts)
        return fail(ctx, PFD_EINVAL, "frame_create: bad sizes or NULL arrays");
    if (mi_w < 2 || mi_h < 2 || mi_w > 32 || mi_h > 32)
        return fail(ctx, PFD_EINVAL, "micro-image window %dx%d outside [2, 32]", mi_w, mi_h);
    if (max_nb < 1 || max_nb > pfd::kMaxNb)
        return fail(ctx, PFD_EINVAL, "max_nb %d outside [1, 32] (selected-view masks are 32 bits)", max_nb);
    Frame f;
    f.W = W; f.H = H; f.V = n_views; f.mi_w = mi_w; f.mi_h = mi_h; f.K = max_nb;
    f.tile_stride = (mi_w * mi_h + 15) & ~15;
    f.has_blur = blur != nullptr;
    std::vector<int2> origin(n_views);
    for (int v = 0; v < n_views; ++v) {
        const float cx = centers[2 * v], cy = centers[2 * v + 1];
        if (!std::isfinite(cx) || !std::isfinite(cy)) return fail(ctx, PFD_EINVAL, "view %d: centre not finite", v);
        // DepthSolver.cpp:1894-1895 (float minus double, stored as float), then the
        // int conversion of cv::Rect (:1977-1978)
        const float ox = (float)((double)cx - (mi_w - 1) * 0.5);
        const float oy = (float)((double)cy - (mi_h - 1) * 0.5);
        if (!(ox >= 0.0f) || !(oy >= 0.0f))
            return fail(ctx, PFD_EINVAL, "view %d: window origin (%g, %g) outside the frame", v, ox, oy);
        const int ix = (int)ox, iy = (int)oy;
        if (ix + mi_w > W || iy + mi_h > H)
            return fail(ctx, PFD_EINVAL, "view %d: window [%d,%d]+%dx%d outside the %dx%d frame", v, ix, iy, mi_w, mi_h, W, H);
        origin[v] = make_int2(ix, iy);
        if (nb_counts[v] < 0 || nb_counts[v] > max_nb)
            return fail(ctx, PFD_EINVAL, "view %d: neighbour count %d outside [0, %d]", v, nb_counts[v], max_nb);
        for (int k = 0; k < nb_counts[v]; ++k) {
            const int id = nb_ids[v * max_nb + k];
            if (id >= n_views || id < -1 || id == v)
                return fail(ctx, PFD_EINVAL, "view %d: neighbour %d has id %d", v, k, id);
        }
    }
    DeviceGuard g(ctx->device);
    const size_t ppv_tiles = (size_t)n_views * f.tile_stride;
    const size_t px = (size_t)n_views * mi_w * mi_h;
    pfd_status st = PFD_OK;
    auto A = [&](void** p, size_t b) { if (st == PFD_OK) st = frame_alloc(ctx, f, p, b); };
    A((void**)&f.d_raw, (size_t)W * H);
    A((void**)&f.d_gray, ppv_tiles);
    if (blur) A((void**)&f.d_blur, ppv_tiles);
    A((void**)&f.d_centers, sizeof(float2) * n_views);
    A((void**)&f.d_tilekeys, sizeof(int2) * n_views);
    A((void**)&f.d_origin, sizeof(int2) * n_views);
    A((void**)&f.d_nb_ids, sizeof(int) * (size_t)n_views * max_nb);
    A((void**)&f.d_nb_counts, sizeof(int) * n_views);
    A((void**)&f.d_cvec, sizeof(float) * px * max_nb);
    for (int b = 0; b < 2; ++b) {
        A((void**)&f.s[b].plane, sizeof(float4) * px);
        A((void**)&f.s[b].cost, sizeof(float) * px);
        A((void**)&f.s[b].disp, sizeof(float4) * px);
        A((void**)&f.s[b].sel, sizeof(uint32_t) * px);
    }
    if (st != PFD_OK) { frame_release(f, ctx->stream); return st; }
    cudaStream_t s = ctx->stream;
    auto H2D = [&](void* d, const void* h, size_t b) {
        if (st == PFD_OK && cudaMemcpyAsync(d, h, b, cudaMemcpyHostToDevice, s) != cudaSuccess) st = PFD_ECUDA;
    };
    H2D(f.d_centers, centers, sizeof(float2) * n_views);
    H2D(f.d_tilekeys, tilekeys, sizeof(int2) * n_views);
    H2D(f.d_origin, origin.data(), sizeof(int2) * n_views);
    H2D(f.d_nb_ids, nb_ids, sizeof(int) * (size_t)n_views * max_nb);
    H2D(f.d_nb_counts, nb_counts, sizeof(int) * n_views);
    if (blur) {
        // repack [V][mi_h*mi_w] into padded tiles
        std::vector<uint8_t> tiles(ppv_tiles, 0);
        for (int v = 0; v < n_views; ++v)
            std::memcpy(&tiles[(size_t)v * f.tile_stride], blur + (size_t)v * mi_w * mi_h, (size_t)mi_w * mi_h);
        H2D(f.d_blur, tiles.data(), ppv_tiles);
        if (st == PFD_OK && cudaStreamSynchronize(s) != cudaSuccess) st = PFD_ECUDA;
    } else if (st == PFD_OK && cudaStreamSynchronize(s) != cudaSuccess) {
        st = PFD_ECUDA;
    }
    if (st != PFD_OK) {
        cudaGetLastError();
        frame_release(f, ctx->stream);
        return fail(ctx, st, "frame_create: upload failed");
    }
    f.h_keys.assign(tilekeys, tilekeys + 2 * (size_t)n_views);
    f.h_centers.assign(centers, centers + 2 * (size_t)n_views);
    f.h_nb_ids.assign(nb_ids, nb_ids + (size_t)n_views * max_nb);
    f.h_nb_counts.assign(nb_counts, nb_counts + n_views);
    const int id = ctx->next_id++;
    ctx->used += f.bytes;
    f.registered = true;
    ctx->frames.emplace(id, std::move(f));
    *frame_id = id;
    return PFD_OK;
}

static pfd_status set_raw(pfd_ctx* ctx, int frame_id, const uint8_t* raw, int raw_pitch, bool device_src)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    if (!raw || raw_pitch < f->W) return fail(ctx, PFD_EINVAL, "raw is NULL or pitch %d < width %d", raw_pitch, f->W);
    DeviceGuard g(ctx->device);
    CU(cudaMemcpy2DAsync(f->d_raw, f->W, raw, raw_pitch, f->W, f->H,
                         device_src ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
    CU(pfd::launch_slice(f->d_raw, f->W, f->d_origin, f->V, f->mi_w, f->mi_h, f->tile_stride, f->d_gray, ctx->stream));
    ctx->launches += 1;
    f->tx[0].stale = true;
    f->has_raw = true;
    f->has_mi = true;
    f->has_state = false;
    f->cvec_valid = 0;
    return PFD_OK;
}

pfd_status pfd_frame_set_raw(pfd_ctx* ctx, int frame_id, const uint8_t* raw, int raw_pitch)
{
    return set_raw(ctx, frame_id, raw, raw_pitch, false);
}

pfd_status pfd_frame_set_raw_device(pfd_ctx* ctx, int frame_id, const uint8_t* raw_dev, int raw_pitch)
{
    return set_raw(ctx, frame_id, raw_dev, raw_pitch, true);
}

pfd_status pfd_frame_set_micro_images(pfd_ctx* ctx, int frame_id, const uint8_t* images)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    if (!images) return fail(ctx, PFD_EINVAL, "micro-images are NULL");
    DeviceGuard g(ctx->device);
    const size_t ppv = (size_t)f->mi_w * f->mi_h;
    std::vector<uint8_t> tiles((size_t)f->V * f->tile_stride, 0);
    for (int v = 0; v < f->V; ++v) std::memcpy(&tiles[(size_t)v * f->tile_stride], images + (size_t)v * ppv, ppv);
    CU(cudaMemcpyAsync(f->d_gray, tiles.data(), tiles.size(), cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));       // the staging vector dies on return
    f->tx[0].stale = true;
    f->has_mi = true;
    f->has_state = false;
    f->cvec_valid = 0;
    return PFD_OK;
}

pfd_status pfd_frame_compute_blur(pfd_ctx* ctx, int frame_id, uint8_t* blur_out, uint32_t* blureness)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    if (!f->has_raw) return fail(ctx, PFD_EINVAL, "compute_blur: frame %d has no raw image", frame_id);
    DeviceGuard g(ctx->device);
    const size_t ppv_tiles = (size_t)f->V * f->tile_stride;
    if (!f->d_blur) {
        const pfd_status st = frame_alloc(ctx, *f, (void**)&f->d_blur, ppv_tiles);
        if (st != PFD_OK) return st;
    }
    if (f->tx[0].ready() && !f->tx[1].ready()) {      // the frame's sweeps read textures
        const pfd_status st = tex_create(ctx, *f, 1);
        if (st != PFD_OK) return st;
    }
    uint32_t* d_counts = nullptr;
    if (blureness) CU(cudaMallocAsync((void**)&d_counts, sizeof(uint32_t) * f->V, ctx->stream));
    const cudaError_t e = pfd::launch_blur(f->d_raw, f->W, f->W, f->H, f->d_origin, f->V, f->mi_w, f->mi_h,
                                           f->tile_stride, f->d_blur, d_counts, ctx->stream);
    if (e != cudaSuccess) {
        if (d_counts) cudaFreeAsync(d_counts, ctx->stream);
        return fail(ctx, PFD_ECUDA, "launch_blur: %s", cudaGetErrorString(e));
    }
    ctx->launches += 1;
    f->tx[1].stale = true;
    f->has_blur = true;
    f->has_state = false;
    f->cvec_valid = 0;
    pfd_status st = PFD_OK;
    if (blur_out) {
        const size_t ppv = (size_t)f->mi_w * f->mi_h;
        if (cudaMemcpy2DAsync(blur_out, ppv, f->d_blur, f->tile_stride, ppv, f->V, cudaMemcpyDeviceToHost,
                              ctx->stream) != cudaSuccess)
            st = PFD_ECUDA;
    }
    if (d_counts) {
        if (st == PFD_OK && cudaMemcpyAsync(blureness, d_counts, sizeof(uint32_t) * f->V, cudaMemcpyDeviceToHost,
                                            ctx->stream) != cudaSuccess)
            st = PFD_ECUDA;
        cudaFreeAsync(d_counts, ctx->stream);
    }
    if (blur_out || blureness) {
        if (st == PFD_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) st = PFD_ECUDA;
    }
    if (st != PFD_OK) {
        cudaGetLastError();
        return fail(ctx, st, "compute_blur: copy-back failed");
    }
    return PFD_OK;
}

pfd_status pfd_frame_compute_richness(pfd_ctx* ctx, int frame_id, float* score_out, uint8_t* binary_out,
                                      uint32_t* richness)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    if (!f->has_raw) return fail(ctx, PFD_EINVAL, "compute_richness: frame %d has no raw image", frame_id);
    if ((f->H + 15) / 16 > 65535) return fail(ctx, PFD_EINVAL, "compute_richness: frame height %d above 1048560", f->H);
    DeviceGuard g(ctx->device);
    const size_t px = (size_t)f->V * f->mi_w * f->mi_h;
    // one allocation: the 16-bit contrast map, the maximum, then the outputs asked for
    const size_t map_bytes = ((size_t)f->W * f->H * sizeof(uint16_t) + 255) & ~(size_t)255;
    const size_t score_bytes = score_out ? ((px * sizeof(float) + 255) & ~(size_t)255) : 0;
    const size_t binary_bytes = binary_out ? ((px + 255) & ~(size_t)255) : 0;
    const size_t count_bytes = richness ? sizeof(uint32_t) * f->V : 0;
    uint8_t* buf = nullptr;
    CU(cudaMallocAsync((void**)&buf, map_bytes + 256 + score_bytes + binary_bytes + count_bytes, ctx->stream));
    uint16_t* d_map = (uint16_t*)buf;
    unsigned* d_max = (unsigned*)(buf + map_bytes);
    float* d_score = score_out ? (float*)(buf + map_bytes + 256) : nullptr;
    uint8_t* d_binary = binary_out ? buf + map_bytes + 256 + score_bytes : nullptr;
    uint32_t* d_counts = richness ? (uint32_t*)(buf + map_bytes + 256 + score_bytes + binary_bytes) : nullptr;
    pfd_status st = PFD_OK;
    const cudaError_t e = pfd::launch_richness(f->d_raw, f->W, f->W, f->H, f->d_origin, f->V, f->mi_w, f->mi_h, d_map,
                                               d_max, d_score, d_binary, d_counts, ctx->stream);
    if (e != cudaSuccess) {
        cudaFreeAsync(buf, ctx->stream);
        cudaGetLastError();
        return fail(ctx, PFD_ECUDA, "launch_richness: %s", cudaGetErrorString(e));
    }
    ctx->launches += f->V > 0 ? 2 : 1;
    if (score_out && cudaMemcpyAsync(score_out, d_score, px * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream) !=
                         cudaSuccess)
        st = PFD_ECUDA;
    if (st == PFD_OK && binary_out &&
        cudaMemcpyAsync(binary_out, d_binary, px, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess)
        st = PFD_ECUDA;
    if (st == PFD_OK && richness &&
        cudaMemcpyAsync(richness, d_counts, count_bytes, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess)
        st = PFD_ECUDA;
    cudaFreeAsync(buf, ctx->stream);
    if (st == PFD_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) st = PFD_ECUDA;
    if (st != PFD_OK) {
        cudaGetLastError();
        return fail(ctx, st, "compute_richness: copy-back failed");
    }
    return PFD_OK;
}

pfd_status pfd_state_upload(pfd_ctx* ctx, int frame_id, const float* plane, const float* cost, const float* disp,
                            const uint32_t* sel)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    if (!plane || !cost || !disp || !sel) return fail(ctx, PFD_EINVAL, "state_upload: NULL array");
    DeviceGuard g(ctx->device);
    const size_t px = (size_t)f->V * f->mi_w * f->mi_h;
    const pfd::StateDev& s = f->s[f->cur];
    CU(cudaMemcpyAsync(s.plane, plane, sizeof(float4) * px, cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(s.cost, cost, sizeof(float) * px, cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(s.disp, disp, sizeof(float4) * px, cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(s.sel, sel, sizeof(uint32_t) * px, cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));       // host buffers may be reused on return
    f->has_state = true;
    f->cvec_valid = 0;
    return PFD_OK;
}

pfd_status pfd_frame_upload(pfd_ctx* ctx, int* frame_id, const uint8_t* raw, int W, int H, int raw_pitch,
                            const float* centers, const int* tilekeys, int n_views, int mi_w, int mi_h,
                            const int* nb_ids, const int* nb_counts, int max_nb, const uint8_t* blur)
{
    pfd_status st = pfd_frame_create(ctx, frame_id, W, H, centers, tilekeys, n_views, mi_w, mi_h, nb_ids, nb_counts,
                                     max_nb, blur);
    if (st != PFD_OK) return st;
    st = pfd_frame_set_raw(ctx, *frame_id, raw, raw_pitch);
    if (st != PFD_OK) {
        const std::string msg = ctx->last_error;
        pfd_frame_free(ctx, *frame_id);
        *frame_id = 0;
        ctx->last_error = msg;
    }
    return st;
}

pfd_status pfd_frame_free(pfd_ctx* ctx, int frame_id)
{
    if (!ctx) return PFD_EINVAL;
    auto it = ctx->frames.find(frame_id);
    if (it == ctx->frames.end()) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    DeviceGuard g(ctx->device);
    ctx->used -= it->second.bytes;
    frame_release(it->second, ctx->stream);           // ordered after the frame's queued work
    ctx->frames.erase(it);
    return PFD_OK;
}

pfd_status pfd_pm_init(pfd_ctx* ctx, int frame_id, const pfd_pm_params* params, uint64_t seed)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    pfd_status st = check_params(ctx, *f, params);
    if (st != PFD_OK) return st;
    DeviceGuard g(ctx->device);
    pfd::PmParams P = make_params(ctx, *f, params, seed);
    if (ctx->counting) P.tap_counter = ctx->d_taps;
    f->cur = 0;
    f->cvec_valid = 0;
    CU(pfd::launch_init(frame_dev(*f), P, f->s[0], ctx->d_err, ctx->stream));
    ctx->launches += 1;
    f->has_state = true;
    f->cvec_valid = 3u;
    f->cvec_key = *params;
    f->cvec_mode = cost_mode(ctx);
    return PFD_OK;
}

// The context's sweep scratch, grown to `need` bytes when smaller.
static pfd_status ensure_scratch(pfd_ctx* ctx, size_t need)
{
    if (need <= ctx->scratch_bytes) return PFD_OK;
    if (ctx->budget && ctx->used - ctx->scratch_bytes + need > ctx->budget)
        return fail(ctx, PFD_ENOMEM, "HBM budget exceeded by %zu bytes of sweep scratch", need);
    // stream-ordered, like the frames: other contexts' work keeps running
    if (ctx->d_scratch) cudaFreeAsync(ctx->d_scratch, ctx->stream);
    ctx->used -= ctx->scratch_bytes;
    ctx->d_scratch = nullptr;
    ctx->scratch_bytes = 0;
    ++ctx->scratch_gen;
    if (cudaMallocAsync((void**)&ctx->d_scratch, need, ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, PFD_ENOMEM, "cudaMallocAsync(%zu) for sweep scratch failed", need);
    }
    ctx->scratch_bytes = need;
    ctx->used += need;
    return PFD_OK;
}

// ---- launch shapes of the half-sweep and their autotuner -------------------------
//
// Every shape (warps per CTA, CTAs per SM the registers are sized for) computes
// the same state bit for bit; which is fastest depends on the frame's window,
// neighbour count, patch and channels, through the shared-memory plan (CTAs
// that fit an SM), the registers (spills) and the pixels per micro-image
// (warps per staged view).  The autotuner times each shape once per such key
// and device on the frame's own half-sweep and keeps the fastest for the
// process.

namespace {

struct ShapeKey {
    int dev, W, H, K, ntap, inc, blur, shift, acmm, tex;
    bool operator<(const ShapeKey& o) const
    {
        return std::tie(dev, W, H, K, ntap, inc, blur, shift, acmm, tex) <
               std::tie(o.dev, o.W, o.H, o.K, o.ntap, o.inc, o.blur, o.shift, o.acmm, o.tex);
    }
};

std::mutex g_shape_mu;
std::map<ShapeKey, int> g_shape_cache;

ShapeKey shape_key(const pfd_ctx* ctx, const Frame& f, const pfd::PmParams& P)
{
    return ShapeKey{ ctx->device, P.W, P.H, P.K, P.ntap, P.inc, f.has_blur ? 1 : 0, P.shifted, P.acmm,
                     sweep_dev(ctx, f).tex != nullptr ? 1 : 0 };
}

int cached_shape(const ShapeKey& k)
{
    std::lock_guard<std::mutex> lock(g_shape_mu);
    auto it = g_shape_cache.find(k);
    return it == g_shape_cache.end() ? -1 : it->second;
}

}  // namespace

// Runs the frame's half-sweep (iter, phase) once in every shape, from its
// current state into the other buffer, with the stored cost vectors neither
// read nor written (so every trial computes the same state), timing each on
// the context's stream; records the fastest for the frame's key.
static pfd_status tune_shape(pfd_ctx* ctx, Frame& f, pfd::PmParams P, int iter, int phase, int* out)
{
    P.cvec_ok = 0;
    P.cvec = nullptr;
    P.tap_counter = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    CU(cudaEventCreate(&a));
    if (cudaEventCreate(&b) != cudaSuccess) { cudaEventDestroy(a); return fail(ctx, PFD_ECUDA, "event"); }
    int best = 0;
    float best_ms = 0.0f;
    pfd_status st = PFD_OK;
    const pfd::FrameDev F = sweep_dev(ctx, f);
    for (int shape = 0; shape < pfd::kSweepShapes && st == PFD_OK; ++shape) {
        if (pfd::sweep_warp_smem_bytes(P, f.has_blur, shape, F.tex != nullptr) > 227 * 1024) continue;
        int n_ctas = 0;
        if (pfd::sweep_warp_grid(F, P, &n_ctas, shape) != cudaSuccess) {
            cudaGetLastError();                      // this shape does not fit the plan: not a candidate
            continue;
        }
        st = ensure_scratch(ctx, pfd::sweep_warp_scratch_bytes(P, n_ctas, shape));
        if (st != PFD_OK) break;
        pfd::PmParams Q = P;
        Q.cost_scratch = ctx->d_scratch;
        Q.scratch_floats = ctx->scratch_bytes / sizeof(float);
        cudaError_t e = cudaEventRecord(a, ctx->stream);
        if (e == cudaSuccess)
            e = pfd::launch_sweep_warp(F, Q, f.s[f.cur], f.s[f.cur ^ 1], iter, phase, n_ctas, ctx->d_err,
                                       ctx->stream, shape);
        if (e == cudaSuccess) e = cudaEventRecord(b, ctx->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(b);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
        if (e != cudaSuccess) {
            cudaGetLastError();
            st = fail(ctx, PFD_ECUDA, "sweep autotune, shape %d: %s", shape, cudaGetErrorString(e));
            break;
        }
        ctx->launches += 1;
        if (shape == 0 || ms < best_ms) { best = shape; best_ms = ms; }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (st != PFD_OK) return st;
    st = check_device_error(ctx);
    if (st != PFD_OK) return st;
    {
        std::lock_guard<std::mutex> lock(g_shape_mu);
        g_shape_cache[shape_key(ctx, f, P)] = best;
    }
    *out = best;
    return PFD_OK;
}

// The shape the context's next half-sweep of frame f runs: the fixed one, or
// under PFD_SHAPE_AUTOTUNE the tuned one (tuning on this half-sweep when the
// key is new).  Tap counting runs shape 0.
static pfd_status sweep_shape_for(pfd_ctx* ctx, Frame& f, const pfd::PmParams& P, int iter, int phase, int* shape)
{
    *shape = 0;
    if (ctx->counting) return PFD_OK;
    if (ctx->sweep_shape != PFD_SHAPE_AUTOTUNE) {
        *shape = ctx->sweep_shape;
        return PFD_OK;
    }
    const int c = cached_shape(shape_key(ctx, f, P));
    if (c >= 0) {
        *shape = c;
        return PFD_OK;
    }
    return tune_shape(ctx, f, P, iter, phase, shape);
}

pfd_status pfd_set_sweep_shape(pfd_ctx* ctx, int shape)
{
    if (!ctx) return PFD_EINVAL;
    if (shape != PFD_SHAPE_AUTOTUNE && (shape < 0 || shape >= PFD_SWEEP_SHAPES))
        return fail(ctx, PFD_EINVAL, "sweep shape %d: give 0-%d or PFD_SHAPE_AUTOTUNE", shape, PFD_SWEEP_SHAPES - 1);
    ctx->sweep_shape = shape;
    return PFD_OK;
}

pfd_status pfd_sweep_shape_info(int shape, int* warps_per_cta, int* ctas_per_sm)
{
    static const int kMin[PFD_SWEEP_SHAPES] = { 4, 3, 6, 2 };
    static_assert(PFD_SWEEP_SHAPES == pfd::kSweepShapes, "shape tables");
    if (shape < 0 || shape >= PFD_SWEEP_SHAPES) return PFD_EINVAL;
    if (warps_per_cta) *warps_per_cta = pfd::sweep_shape_warps(shape);
    if (ctas_per_sm) *ctas_per_sm = kMin[shape];
    return PFD_OK;
}

pfd_status pfd_tuned_sweep_shape(pfd_ctx* ctx, int frame_id, const pfd_pm_params* params, int* shape)
{
    if (!ctx || !shape) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    const pfd_status st = check_params(ctx, *f, params);
    if (st != PFD_OK) return st;
    *shape = cached_shape(shape_key(ctx, *f, make_params(ctx, *f, params, 0)));
    return PFD_OK;
}

pfd_status pfd_pm_sweep(pfd_ctx* ctx, int frame_id, const pfd_pm_params* params, uint64_t seed, int iter, int phase)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    pfd_status st = check_params(ctx, *f, params);
    if (st != PFD_OK) return st;
    if (!f->has_state) return fail(ctx, PFD_ESTATE, "sweep before pfd_pm_init");
    if (phase != 0 && phase != 1) return fail(ctx, PFD_EINVAL, "phase must be 0 or 1");
    if (iter < 0) return fail(ctx, PFD_EINVAL, "iter must be >= 0");
    DeviceGuard g(ctx->device);
    pfd::PmParams P = make_params(ctx, *f, params, seed);
    if (ctx->counting) P.tap_counter = ctx->d_taps;
    st = tex_refresh(ctx, *f);
    if (st != PFD_OK) return st;
    const pfd::FrameDev F = sweep_dev(ctx, *f);
    if (pfd::sweep_warp_smem_bytes(P, f->has_blur, 0, F.tex != nullptr) > 227 * 1024)
        return fail(ctx, PFD_EINVAL, "window %dx%d with %d neighbours does not fit shared memory", f->mi_w, f->mi_h, f->K);
    int shape = 0;
    st = sweep_shape_for(ctx, *f, P, iter, phase, &shape);
    if (st != PFD_OK) return st;
    int n_ctas = 0;
    CU(pfd::sweep_warp_grid(F, P, &n_ctas, shape));
    st = ensure_scratch(ctx, pfd::sweep_warp_scratch_bytes(P, n_ctas, shape));
    if (st != PFD_OK) return st;
    P.cost_scratch = ctx->d_scratch;
    P.scratch_floats = ctx->scratch_bytes / sizeof(float);
    P.cvec_ok = !ctx->counting && cvec_usable(*f, *params, phase, cost_mode(ctx));
    CU(pfd::launch_sweep_warp(F, P, f->s[f->cur], f->s[f->cur ^ 1], iter, phase, n_ctas, ctx->d_err,
                              ctx->stream, shape));
    ctx->launches += 1;
    f->cur ^= 1;
    if (ctx->counting) f->cvec_valid = 0;        // tap counting evaluates everything and stores nothing
    else cvec_swept(*f, *params, phase, cost_mode(ctx));
    return PFD_OK;
}

static pfd_status patchmatch_enqueue(pfd_ctx* ctx, int frame_id, const pfd_pm_params* params, uint64_t seed)
{
    pfd_status st = pfd_pm_init(ctx, frame_id, params, seed);
    for (int it = 0; st == PFD_OK && it < params->max_iterations; ++it)
        for (int ph = 0; ph < 2 && st == PFD_OK; ++ph) st = pfd_pm_sweep(ctx, frame_id, params, seed, it, ph);
    if (st == PFD_OK && ctx->matcher == PFD_MATCHER_ACMM) st = pfd_acmm_post_refine(ctx, frame_id, params);
    return st;
}

pfd_status pfd_patchmatch(pfd_ctx* ctx, int frame_id, const pfd_pm_params* params, uint64_t seed)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    if (!ctx->graphs || ctx->counting) return patchmatch_enqueue(ctx, frame_id, params, seed);
    pfd_status st = check_params(ctx, *f, params);
    if (st != PFD_OK) return st;
    // the key: the call's arguments and every context mode the launches depend on
    std::vector<unsigned char> key(sizeof(pfd_pm_params) + sizeof(uint64_t) + 4 * sizeof(int));
    const int modes[4] = { ctx->matcher, ctx->ncc_moments, ctx->sweep_shape, ctx->sweep_fetch };
    std::memcpy(key.data(), params, sizeof(pfd_pm_params));
    std::memcpy(key.data() + sizeof(pfd_pm_params), &seed, sizeof(uint64_t));
    std::memcpy(key.data() + sizeof(pfd_pm_params) + sizeof(uint64_t), modes, sizeof(modes));
    FrameGraph& G = f->pm_graph;
    DeviceGuard g(ctx->device);
    st = tex_refresh(ctx, *f);                   // changed tiles are refilled before, not inside, the graph
    if (st != PFD_OK) return st;
    if (G.exec && G.scratch_gen != ctx->scratch_gen) G.reset();   // the scratch moved since the capture
    if (G.exec && G.key == key) {
        CU(cudaGraphLaunch(G.exec, ctx->stream));
        ctx->launches += G.launches;
    } else if (G.warm && G.key == key) {
        // the first call ran uncaptured (scratch sized, launch shape tuned): capture
        // this one's enqueue sequence, then replay it
        const unsigned long long launches0 = ctx->launches;
        CU(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        st = patchmatch_enqueue(ctx, frame_id, params, seed);
        cudaGraph_t graph = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
        if (st == PFD_OK && (ce != cudaSuccess || cudaGraphInstantiate(&G.exec, graph, 0) != cudaSuccess)) {
            cudaGetLastError();
            st = fail(ctx, PFD_ECUDA, "patchmatch: graph capture failed");
        }
        if (graph) cudaGraphDestroy(graph);
        if (st != PFD_OK) { G.reset(); return st; }
        G.launches = ctx->launches - launches0;
        ctx->launches = launches0;
        G.scratch_gen = ctx->scratch_gen;
        G.cur = f->cur;
        G.cvec_valid = f->cvec_valid;
        G.cvec_key = f->cvec_key;
        G.cvec_mode = f->cvec_mode;
        CU(cudaGraphLaunch(G.exec, ctx->stream));
        ctx->launches += G.launches;
    } else {
        G.reset();
        st = patchmatch_enqueue(ctx, frame_id, params, seed);
        if (st != PFD_OK) return st;
        G.key = key;
        G.warm = true;
        return PFD_OK;
    }
    f->has_state = true;
    f->cur = G.cur;
    f->cvec_valid = G.cvec_valid;
    f->cvec_key = G.cvec_key;
    f->cvec_mode = G.cvec_mode;
    return PFD_OK;
}

pfd_status pfd_set_sweep_fetch(pfd_ctx* ctx, int mode)
{
    if (!ctx) return PFD_EINVAL;
    if (mode != PFD_FETCH_TEXTURE && mode != PFD_FETCH_SHARED)
        return fail(ctx, PFD_EINVAL, "sweep fetch %d: give PFD_FETCH_TEXTURE or PFD_FETCH_SHARED", mode);
    ctx->sweep_fetch = mode;
    return PFD_OK;
}

pfd_status pfd_set_graphs(pfd_ctx* ctx, int on)
{
    if (!ctx) return PFD_EINVAL;
    ctx->graphs = on != 0;
    return PFD_OK;
}

pfd_status pfd_patchmatch_batch(pfd_ctx* ctx, const int* frame_ids, int n, const pfd_pm_params* params,
                                const uint64_t* seeds)
{
    if (!ctx) return PFD_EINVAL;
    if (n < 1 || n > 4096 || !frame_ids || !params || !seeds)
        return fail(ctx, PFD_EINVAL, "patchmatch_batch: n must be in [1, 4096] and the arrays non-NULL");
    std::vector<Frame*> fr(n);
    for (int b = 0; b < n; ++b) {
        fr[b] = find_frame(ctx, frame_ids[b]);
        if (!fr[b]) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_ids[b]);
        for (int c = 0; c < b; ++c)
            if (frame_ids[c] == frame_ids[b]) return fail(ctx, PFD_EINVAL, "frame %d listed twice", frame_ids[b]);
        const pfd_status st = check_params(ctx, *fr[b], &params[b]);
        if (st != PFD_OK) return st;
    }
    if (ctx->counting) {                          // tap counting runs frame by frame
        for (int b = 0; b < n; ++b) {
            const pfd_status st = pfd_patchmatch(ctx, frame_ids[b], &params[b], seeds[b]);
            if (st != PFD_OK) return st;
        }
        return PFD_OK;
    }
    DeviceGuard g(ctx->device);
    {
        // A frame whose micro-images fill the sweep's grid four times over or more gains
        // nothing from sharing a launch (its last wave is a small part of its work) and
        // measured 4-5% slower inside one (2048x1536 and 4080x3068 frames of the mixed
        // set); such frames run as their own launches, the others share launches.
        std::vector<int> solo, rest;
        for (int b = 0; b < n; ++b) {
            int n_ctas = 0;
            const pfd::PmParams P = make_params(ctx, *fr[b], &params[b], seeds[b]);
            if (pfd::sweep_warp_grid(sweep_dev(ctx, *fr[b]), P, &n_ctas, 0) != cudaSuccess) {
                cudaGetLastError();
                n_ctas = 0;
            }
            (n_ctas > 0 && fr[b]->V >= 4 * n_ctas ? solo : rest).push_back(b);
        }
        if (!solo.empty()) {
            for (int b : solo) {
                const pfd_status st = pfd_patchmatch(ctx, frame_ids[b], &params[b], seeds[b]);
                if (st != PFD_OK) return st;
            }
            if (rest.empty()) return PFD_OK;
            std::vector<int> ids;
            std::vector<pfd_pm_params> ps;
            std::vector<uint64_t> sd;
            for (int b : rest) {
                ids.push_back(frame_ids[b]);
                ps.push_back(params[b]);
                sd.push_back(seeds[b]);
            }
            return pfd_patchmatch_batch(ctx, ids.data(), (int)ids.size(), ps.data(), sd.data());
        }
    }
    for (int b = 0; b < n; ++b) {
        pfd_status st = pfd_pm_init(ctx, frame_ids[b], &params[b], seeds[b]);
        if (st == PFD_OK) st = tex_refresh(ctx, *fr[b]);
        if (st != PFD_OK) return st;
    }
    // launch shape per blur group: the fixed one, or the one tuned for the group's
    // largest frame (tuned on that frame's first half-sweep when its key is new)
    const bool shift = ctx->ncc_moments == PFD_NCC_SHIFTED;
    int half_sweeps = 0;
    for (int b = 0; b < n; ++b) {
        const pfd::PmParams P = make_params(ctx, *fr[b], &params[b], seeds[b]);
        if (pfd::sweep_warp_smem_bytes(P, fr[b]->has_blur, 0, sweep_dev(ctx, *fr[b]).tex != nullptr) > 227 * 1024)
            return fail(ctx, PFD_EINVAL, "frame %d: window %dx%d with %d neighbours does not fit shared memory",
                        frame_ids[b], fr[b]->mi_w, fr[b]->mi_h, fr[b]->K);
        half_sweeps = std::max(half_sweeps, 2 * params[b].max_iterations);
    }
    int shape_of_blur[2] = { 0, 0 };
    for (int grp = 0; grp < 2; ++grp) {
        int big = -1;
        for (int b = 0; b < n; ++b)
            if ((fr[b]->has_blur ? 1 : 0) == grp && params[b].max_iterations > 0 &&
                (big < 0 || (size_t)fr[b]->V * fr[b]->mi_w * fr[b]->mi_h > (size_t)fr[big]->V * fr[big]->mi_w * fr[big]->mi_h))
                big = b;
        if (big < 0) continue;
        const pfd::PmParams Pb = make_params(ctx, *fr[big], &params[big], seeds[big]);
        const pfd_status st = sweep_shape_for(ctx, *fr[big], Pb, 0, 0, &shape_of_blur[grp]);
        if (st != PFD_OK) return st;
        for (int b = 0; b < n; ++b)          // a shape every frame of the group fits, or the default
            if ((fr[b]->has_blur ? 1 : 0) == grp &&
                pfd::sweep_warp_smem_bytes(make_params(ctx, *fr[b], &params[b], seeds[b]), grp == 1,
                                           shape_of_blur[grp], sweep_dev(ctx, *fr[b]).tex != nullptr) > 227 * 1024)
                shape_of_blur[grp] = 0;
    }
    // launch groups: frames with the same blur channel and fetch whose own
    // shared-memory plans allow the same CTAs per SM share a launch, so no frame
    // runs at the occupancy of a larger frame's plan; a group's plan is its
    // largest member's (same occupancy)
    struct Group { int blur, tex, ctas, smem, shape; std::vector<int> members; };
    std::vector<Group> groups;
    for (int b = 0; b < n; ++b) {
        const int blur = fr[b]->has_blur ? 1 : 0, shape = shape_of_blur[blur];
        const int tex = sweep_dev(ctx, *fr[b]).tex != nullptr ? 1 : 0;
        const int sm = pfd::sweep_warp_smem_bytes(make_params(ctx, *fr[b], &params[b], seeds[b]), blur == 1, shape,
                                                  tex == 1);
        int ctas = 0;
        CU(pfd::sweep_batch_grid(sm, blur == 1, shift, tex == 1, &ctas, shape));
        int g = -1;
        for (size_t k = 0; k < groups.size(); ++k)
            if (groups[k].blur == blur && groups[k].tex == tex && groups[k].ctas == ctas) g = (int)k;
        if (g < 0) {
            groups.push_back(Group{ blur, tex, ctas, 0, shape, {} });
            g = (int)groups.size() - 1;
        }
        groups[g].smem = std::max(groups[g].smem, sm);
        groups[g].members.push_back(b);
    }
    // one warp-scratch stride for every frame (the largest neighbour count's): CTAs of a
    // launch work on different frames at once, and their regions must not overlap
    int k_max = 0;
    for (int b = 0; b < n; ++b) k_max = std::max(k_max, fr[b]->K);
    const int stride = pfd::sweep_warp_stride(k_max);
    size_t scratch = 0;
    for (const Group& g : groups) {
        pfd::PmParams Pk = {};
        Pk.K = k_max;                                  // the scratch of the group's CTAs at that stride
        scratch = std::max(scratch, pfd::sweep_warp_scratch_bytes(Pk, g.ctas, g.shape));
    }
    pfd_status st = ensure_scratch(ctx, scratch);
    if (st != PFD_OK) return st;
    if (half_sweeps == 0) return PFD_OK;
    // one item and one queue counter per (half-sweep, frame), uploaded as the work is enqueued
    pfd::SweepItem* d_items = nullptr;
    int* d_queues = nullptr;
    const size_t n_items = (size_t)half_sweeps * n;
    if (cudaMallocAsync((void**)&d_items, sizeof(pfd::SweepItem) * n_items, ctx->stream) != cudaSuccess ||
        cudaMallocAsync((void**)&d_queues, sizeof(int) * n_items, ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        if (d_items) cudaFreeAsync(d_items, ctx->stream);
        return fail(ctx, PFD_ENOMEM, "patchmatch_batch: %zu launch items", n_items);
    }
    CU(cudaMemsetAsync(d_queues, 0, sizeof(int) * n_items, ctx->stream));
    std::vector<pfd::SweepItem> items;
    const int mode = cost_mode(ctx);
    std::vector<int> count(groups.size());
    for (int s = 0; s < half_sweeps && st == PFD_OK; ++s) {
        const int iter = s / 2, phase = s % 2;
        std::fill(count.begin(), count.end(), 0);
        items.clear();
        for (size_t grp = 0; grp < groups.size(); ++grp)
            for (int b : groups[grp].members) {
                Frame& f = *fr[b];
                if (s >= 2 * params[b].max_iterations) continue;
                pfd::SweepItem it;
                it.F = sweep_dev(ctx, f);
                it.P = make_params(ctx, f, &params[b], seeds[b]);
                it.P.cost_scratch = ctx->d_scratch;
                it.P.scratch_floats = ctx->scratch_bytes / sizeof(float);
                it.P.scratch_stride = stride;
                it.P.cvec_ok = cvec_usable(f, params[b], phase, mode);
                it.P.view_queue = d_queues + (size_t)s * n + items.size();
                it.prev = f.s[f.cur];
                it.next = f.s[f.cur ^ 1];
                it.iter = iter;
                it.phase = phase;
                items.push_back(it);
                ++count[grp];
                f.cur ^= 1;
                cvec_swept(f, params[b], phase, mode);
            }
        pfd::SweepItem* row = d_items + (size_t)s * n;
        if (cudaMemcpyAsync(row, items.data(), sizeof(pfd::SweepItem) * items.size(), cudaMemcpyHostToDevice,
                            ctx->stream) != cudaSuccess) {
            st = fail(ctx, PFD_ECUDA, "patchmatch_batch: item upload");
            break;
        }
        int off = 0;
        for (size_t grp = 0; grp < groups.size(); off += count[grp], ++grp) {
            if (!count[grp]) continue;
            const Group& G = groups[grp];
            const cudaError_t e = pfd::launch_sweep_batch(row + off, count[grp], G.blur == 1, shift, G.tex == 1, G.smem,
                                                          G.ctas, ctx->d_err, ctx->stream, G.shape);
            if (e != cudaSuccess) {
                st = fail(ctx, PFD_ECUDA, "launch_sweep_batch: %s", cudaGetErrorString(e));
                break;
            }
            ctx->launches += 1;
        }
    }
    cudaFreeAsync(d_items, ctx->stream);
    cudaFreeAsync(d_queues, ctx->stream);
    if (st != PFD_OK) return st;
    if (ctx->matcher == PFD_MATCHER_ACMM)
        for (int b = 0; b < n && st == PFD_OK; ++b) st = pfd_acmm_post_refine(ctx, frame_ids[b], &params[b]);
    return st;
}

pfd_status pfd_acmm_post_refine(pfd_ctx* ctx, int frame_id, const pfd_pm_params* params)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    pfd_status st = check_params(ctx, *f, params);
    if (st != PFD_OK) return st;
    if (!f->has_state) return fail(ctx, PFD_ESTATE, "post-refine before pfd_pm_init");
    DeviceGuard g(ctx->device);
    pfd::PmParams P = make_params(ctx, *f, params, 0);
    if (ctx->counting) P.tap_counter = ctx->d_taps;
    CU(pfd::launch_init(frame_dev(*f), P, f->s[f->cur], ctx->d_err, ctx->stream, true));
    ctx->launches += 1;
    // the pass stores every pixel's vector of its current plane
    f->cvec_valid = 3u;
    f->cvec_key = *params;
    f->cvec_mode = cost_mode(ctx);
    return PFD_OK;
}

pfd_status pfd_ncc_costs(pfd_ctx* ctx, int frame_id, const pfd_pm_params* params, const int* vids, const int* pxy,
                         const float* planes, int n, float* costs)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    pfd_status st = check_params(ctx, *f, params);
    if (st != PFD_OK) return st;
    if (n < 0 || (n > 0 && (!vids || !pxy || !planes || !costs))) return fail(ctx, PFD_EINVAL, "ncc_costs: bad arrays");
    if (n == 0) return PFD_OK;
    for (int i = 0; i < n; ++i) {
        if (vids[i] < 0 || vids[i] >= f->V) return fail(ctx, PFD_EINVAL, "hypothesis %d: view %d", i, vids[i]);
        if (pxy[2 * i] < 0 || pxy[2 * i] >= f->mi_w || pxy[2 * i + 1] < 0 || pxy[2 * i + 1] >= f->mi_h)
            return fail(ctx, PFD_EINVAL, "hypothesis %d: pixel outside the window", i);
    }
    // group by view (stable), segments of <= npb hypotheses
    const int npb = 128;
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return vids[a] < vids[b]; });
    std::vector<int> seg_vid, seg_start, seg_len, h_pxy(2 * (size_t)n), h_out(n);
    std::vector<float> h_plane(4 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        const int o = order[i];
        h_pxy[2 * i] = pxy[2 * o]; h_pxy[2 * i + 1] = pxy[2 * o + 1];
        std::memcpy(&h_plane[4 * (size_t)i], planes + 4 * (size_t)o, 16);
        h_out[i] = o;
        if (i == 0 || vids[o] != vids[order[i - 1]] || seg_len.back() == npb) {
            seg_vid.push_back(vids[o]); seg_start.push_back(i); seg_len.push_back(0);
        }
        seg_len.back()++;
    }
    const int nseg = (int)seg_vid.size();
    DeviceGuard g(ctx->device);
    const size_t bytes = sizeof(int) * (3 * (size_t)nseg + 3 * (size_t)n) + sizeof(float) * 4 * (size_t)n +
                         sizeof(float) * (size_t)n * f->K + 64;
    char* d = nullptr;
    CU(cudaMallocAsync((void**)&d, bytes, ctx->stream));
    int* d_segv = (int*)d;
    int* d_segs = d_segv + nseg;
    int* d_segl = d_segs + nseg;
    int* d_pxy = d_segl + nseg;
    int* d_out = d_pxy + 2 * (size_t)n;
    float4* d_plane = (float4*)(((uintptr_t)(d_out + n) + 15) & ~(uintptr_t)15);
    float* d_cost = (float*)(d_plane + n);
    cudaStream_t s = ctx->stream;
    pfd_status rc = PFD_OK;
    auto H2D = [&](void* dd, const void* h, size_t b) {
        if (rc == PFD_OK && cudaMemcpyAsync(dd, h, b, cudaMemcpyHostToDevice, s) != cudaSuccess) rc = PFD_ECUDA;
    };
    H2D(d_segv, seg_vid.data(), sizeof(int) * nseg);
    H2D(d_segs, seg_start.data(), sizeof(int) * nseg);
    H2D(d_segl, seg_len.data(), sizeof(int) * nseg);
    H2D(d_pxy, h_pxy.data(), sizeof(int) * 2 * (size_t)n);
    H2D(d_out, h_out.data(), sizeof(int) * (size_t)n);
    H2D(d_plane, h_plane.data(), sizeof(float) * 4 * (size_t)n);
    const pfd::PmParams P = make_params(ctx, *f, params, 0);
    if (rc == PFD_OK &&
        pfd::launch_ncc(frame_dev(*f), P, nseg, npb, d_segv, d_segs, d_segl, d_pxy, d_plane, d_out, d_cost,
                        ctx->d_err, s) != cudaSuccess)
        rc = PFD_ECUDA;
    else if (rc == PFD_OK)
        ctx->launches += 1;
    if (rc == PFD_OK &&
        cudaMemcpyAsync(costs, d_cost, sizeof(float) * (size_t)n * f->K, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        rc = PFD_ECUDA;
    cudaFreeAsync(d, s);
    if (rc != PFD_OK) {
        const cudaError_t e = cudaGetLastError();
        return fail(ctx, rc, "ncc_costs: %s", cudaGetErrorString(e));
    }
    return check_device_error(ctx);
}

static pfd::CheckFrame check_frame(const Frame& f, float baseline_unit)
{
    pfd::CheckFrame F;
    F.V = f.V; F.W = f.mi_w; F.H = f.mi_h; F.K = f.K; F.tile_stride = f.tile_stride;
    F.gray = f.d_gray; F.centers = f.d_centers; F.nb_ids = f.d_nb_ids; F.nb_counts = f.d_nb_counts;
    F.baseline_unit = baseline_unit;
    return F;
}

static pfd_status check_filter_cfg(pfd_ctx* ctx, const pfd_filter_cfg* cfg, float baseline_unit)
{
    if (!cfg) return fail(ctx, PFD_EINVAL, "filter config is NULL");
    if (cfg->max_triplet < 0 || cfg->max_triplet > 32) return fail(ctx, PFD_EINVAL, "max_triplet outside [0, 32]");
    if (!(baseline_unit > 0.0f)) return fail(ctx, PFD_EINVAL, "baseline_unit must be > 0");
    return PFD_OK;
}

// Groups the views into wavefront steps col + c * row such that every
// neighbour that precedes a view in key order (row, col) lands in an earlier
// step and every one that follows it in a later step.
static pfd_status build_steps(pfd_ctx* ctx, Frame& f)
{
    if (!f.step_start.empty()) return PFD_OK;
    const int V = f.V;
    long long c = 1;
    for (int v = 0; v < V; ++v) {
        const int cv = f.h_keys[2 * v], rv = f.h_keys[2 * v + 1];
        for (int k = 0; k < f.h_nb_counts[v]; ++k) {
            const int u = f.h_nb_ids[(size_t)v * f.K + k];
            if (u < 0) continue;
            const int cu = f.h_keys[2 * u], ru = f.h_keys[2 * u + 1];
            if (ru == rv) continue;
            // earlier row: c (rv - ru) > cu - cv; later row: c (ru - rv) > cv - cu
            const long long num = (ru < rv) ? (long long)cu - cv : (long long)cv - cu;
            const long long den = (ru < rv) ? (long long)rv - ru : (long long)ru - rv;
            long long need = (num >= 0) ? num / den + 1 : 1;
            if (need > c) c = need;
        }
    }
    std::vector<long long> step(V);
    long long smin = LLONG_MAX, smax = LLONG_MIN;
    for (int v = 0; v < V; ++v) {
        step[v] = (long long)f.h_keys[2 * v] + c * (long long)f.h_keys[2 * v + 1];
        smin = std::min(smin, step[v]);
        smax = std::max(smax, step[v]);
    }
    const long long ns = smax - smin + 1;
    if (ns > 100000000LL) return fail(ctx, PFD_EINVAL, "tile keys too sparse for the filter schedule");
    std::vector<int> counts((size_t)ns + 1, 0), order(V);
    for (int v = 0; v < V; ++v) counts[(size_t)(step[v] - smin) + 1]++;
    for (size_t i = 1; i < counts.size(); ++i) counts[i] += counts[i - 1];
    std::vector<int> fill(counts.begin(), counts.end() - 1);
    for (int v = 0; v < V; ++v) order[fill[(size_t)(step[v] - smin)]++] = v;
    // compact away empty steps
    f.step_start.clear();
    for (size_t s = 0; s + 1 < counts.size(); ++s)
        if (counts[s + 1] > counts[s]) f.step_start.push_back(counts[s]);
    f.step_start.push_back(V);
    if (!f.d_steps) {                 // kept when new neighbour lists rebuild the schedule
        void* p = nullptr;
        pfd_status st = frame_alloc(ctx, f, &p, sizeof(int) * (size_t)V);
        if (st != PFD_OK) { f.step_start.clear(); return st; }
        f.d_steps = (int*)p;
    }
    CU(cudaMemcpyAsync(f.d_steps, order.data(), sizeof(int) * (size_t)V, cudaMemcpyHostToDevice, ctx->stream));
    return PFD_OK;
}

pfd_status pfd_filter(pfd_ctx* ctx, int frame_id, const pfd_filter_cfg* cfg, float baseline_unit, uint8_t* reason,
                      long long* stats)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    pfd_status st = check_filter_cfg(ctx, cfg, baseline_unit);
    if (st != PFD_OK) return st;
    if (!f->has_state) return fail(ctx, PFD_ESTATE, "filter before PatchMatch");
    DeviceGuard g(ctx->device);
    if ((st = build_steps(ctx, *f)) != PFD_OK) return st;
    const size_t px = (size_t)f->V * f->mi_w * f->mi_h;
    if (!f->d_reason) {
        void* p = nullptr;
        if ((st = frame_alloc(ctx, *f, &p, px)) != PFD_OK) return st;
        f->d_reason = (uint8_t*)p;
    }
    pfd::FilterCfg fc;
    static_assert(sizeof(fc) == sizeof(pfd_filter_cfg), "filter config layouts differ");
    std::memcpy(&fc, cfg, sizeof(fc));
    const pfd::CheckFrame F = check_frame(*f, baseline_unit);
    if (pfd::filter_smem_bytes(F) > 227 * 1024) return fail(ctx, PFD_EINVAL, "filter tile does not fit shared memory");
    if (!f->d_fstats) {
        void* p = nullptr;
        if ((st = frame_alloc(ctx, *f, &p, 8 * sizeof(unsigned long long))) != PFD_OK) return st;
        f->d_fstats = (unsigned long long*)p;
    }
    unsigned long long* d_stats = f->d_fstats;
    // enqueue-only calls under pfd_set_graphs: the first call with a key runs as
    // usual, the second is captured, later ones replay the graph (it reads the
    // state buffer the frame's current state was in at capture)
    FrameGraph& G = f->filter_graph;
    const bool graph_mode = !stats && !reason && ctx->graphs;
    bool capture = false;
    if (graph_mode) {
        std::vector<unsigned char> key(sizeof(pfd_filter_cfg) + sizeof(float));
        std::memcpy(key.data(), cfg, sizeof(pfd_filter_cfg));
        std::memcpy(key.data() + sizeof(pfd_filter_cfg), &baseline_unit, sizeof(float));
        if (G.exec && G.key == key && G.cur == f->cur) {
            CU(cudaGraphLaunch(G.exec, ctx->stream));
            ctx->launches += G.launches;
            f->cvec_valid = 0;
            return PFD_OK;
        }
        capture = G.warm && !G.exec && G.key == key && G.cur == f->cur;
        if (!capture) {
            G.reset();
            G.key = key;
            G.warm = true;
            G.cur = f->cur;
        }
    }
    if (capture) CU(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const unsigned long long launches0 = ctx->launches;
    pfd_status fst = PFD_OK;
    if (cudaMemsetAsync(d_stats, 0, 8 * sizeof(unsigned long long), ctx->stream) != cudaSuccess)
        fst = fail(ctx, PFD_ECUDA, "filter: counter reset");
    const pfd::StateDev& S = f->s[f->cur];
    f->cvec_valid = 0;                             // rejected pixels get new planes
    for (size_t s = 0; fst == PFD_OK && s + 1 < f->step_start.size(); ++s) {
        const int a = f->step_start[s], b = f->step_start[s + 1];
        cudaError_t e = pfd::launch_filter_step(F, fc, S, f->d_steps + a, b - a, f->d_reason, d_stats, ctx->stream);
        if (e != cudaSuccess) fst = fail(ctx, PFD_ECUDA, "filter step: %s", cudaGetErrorString(e));
        else ctx->launches += 1;
    }
    if (capture) {
        cudaGraph_t graph = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
        if (fst == PFD_OK && (ce != cudaSuccess || cudaGraphInstantiate(&G.exec, graph, 0) != cudaSuccess)) {
            cudaGetLastError();
            fst = fail(ctx, PFD_ECUDA, "filter: graph capture failed");
        }
        if (graph) cudaGraphDestroy(graph);
        if (fst != PFD_OK) { G.reset(); return fst; }
        G.launches = ctx->launches - launches0;
        CU(cudaGraphLaunch(G.exec, ctx->stream));
        return PFD_OK;
    }
    if (fst != PFD_OK) return fst;
    unsigned long long h[8] = {};
    if (stats) CU(cudaMemcpyAsync(h, d_stats, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    if (reason) CU(cudaMemcpyAsync(reason, f->d_reason, px, cudaMemcpyDeviceToHost, ctx->stream));
    if (stats || reason) {
        CU(cudaStreamSynchronize(ctx->stream));
        if (stats) for (int i = 0; i < 8; ++i) stats[i] = (long long)h[i];
    }
    return PFD_OK;
}

pfd_status pfd_reprojection_error(pfd_ctx* ctx, int frame_id, const pfd_filter_cfg* cfg, float baseline_unit, float* err)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    pfd_status st = check_filter_cfg(ctx, cfg, baseline_unit);
    if (st != PFD_OK) return st;
    if (!f->has_state) return fail(ctx, PFD_ESTATE, "reprojection error before PatchMatch");
    DeviceGuard g(ctx->device);
    const size_t px = (size_t)f->V * f->mi_w * f->mi_h;
    if (!f->d_err) {
        void* p = nullptr;
        if ((st = frame_alloc(ctx, *f, &p, px * sizeof(float))) != PFD_OK) return st;
        f->d_err = (float*)p;
    }
    pfd::FilterCfg fc;
    std::memcpy(&fc, cfg, sizeof(fc));
    CU(pfd::launch_reproj(check_frame(*f, baseline_unit), fc, f->s[f->cur], f->d_err, ctx->stream));
    ctx->launches += 1;
    if (err) {
        CU(cudaMemcpyAsync(err, f->d_err, px * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
    }
    return PFD_OK;
}

// CheckGlobal's fold of the per-tile records (MICycleCheck.cpp:541-600, 742-832).
static void fold_cycle_stats(const std::vector<pfd::CycleTileRec>& rec, const unsigned int* hist, pfd_cycle_stats* stats)
{
    pfd_cycle_stats o;
    std::memset(&o, 0, sizeof(o));
    double io_mean_geo = 0.0, io_mean_photo = 0.0, io_sq_geo = 0.0, io_sq_photo = 0.0;
    long long io_num = 0;
    double m_sq_geo = 0.0, m_sq_photo = 0.0, m_sum_geo = 0.0, m_sum_photo = 0.0;
    long long m_count = 0, all_count = 0, c_total = 0, c_good = 0, c_geo = 0, c_photo = 0;
    double geo_min = INFINITY, geo_max = 0.0;
    for (size_t v = 0; v < rec.size(); ++v) {
        const pfd::CycleTileRec& r = rec[v];
        if (r.n > 0) {
            const double mg = r.sum_geo / (double)r.n, mp = r.sum_photo / (double)r.n;
            const long long N0 = io_num + r.n;
            const double den = (double)(N0 > 1 ? N0 : 1);
            io_mean_geo = (io_mean_geo * (double)io_num + mg * (double)r.n) / den;
            io_mean_photo = (io_mean_photo * (double)io_num + mp * (double)r.n) / den;
            io_num = N0;
            io_sq_geo += r.sq_geo;
            io_sq_photo += r.sq_photo;
        }
        m_sq_geo += r.sq_geo_m;
        m_sq_photo += r.sq_photo_m;
        m_sum_geo += r.sum_geo_m;
        m_sum_photo += r.sum_photo_m;
        c_total += r.comp_total;
        c_good += r.comp_good;
        c_geo += r.comp_good_geo;
        c_photo += r.comp_good_photo;
        if ((double)r.min_geo_m < geo_min) geo_min = r.min_geo_m;
        if ((double)r.max_geo_m > geo_max) geo_max = r.max_geo_m;
        m_count += r.n_masked;
        all_count += r.n;
    }
    o.num_samples = io_num;
    o.mean_geo_err_px = io_mean_geo;
    o.mean_photo_err = io_mean_photo;
    o.completeness = c_total > 0 ? (double)c_good / (double)c_total : 0.0;
    o.completeness_geo = c_total > 0 ? (double)c_geo / (double)c_total : 0.0;
    o.completeness_photo = c_total > 0 ? (double)c_photo / (double)c_total : 0.0;
    o.completeness_masked_pixels = c_total;
    o.completeness_good_pixels = c_good;
    o.completeness_good_pixels_geo = c_geo;
    o.completeness_good_pixels_photo = c_photo;
    if (io_num > 0) {
        o.rmse_geo_err_px = std::sqrt(io_sq_geo / (double)io_num);
        o.rmse_photo_err = std::sqrt(io_sq_photo / (double)io_num);
    }
    o.median_geo_err_px = o.mean_geo_err_px;          // as CheckGlobal reports them
    o.p90_geo_err_px = o.mean_geo_err_px;
    o.masked_count = m_count;
    o.all_count = all_count;
    o.masked_geo_mean = m_count > 0 ? m_sum_geo / (double)m_count : 0.0;
    o.masked_photo_mean = m_count > 0 ? m_sum_photo / (double)m_count : 0.0;
    o.masked_geo_rmse = m_count > 0 ? std::sqrt(m_sq_geo / (double)m_count) : 0.0;
    o.masked_photo_rmse = m_count > 0 ? std::sqrt(m_sq_photo / (double)m_count) : 0.0;
    o.coverage = all_count > 0 ? (double)m_count / (double)all_count : 0.0;
    if (m_count > 0) {
        long long cum = 0;
        bool med = false, p90 = false;
        for (int i = 0; i < pfd::kCycleHistBins && !(med && p90); ++i) {
            cum += hist[i];
            if (!med && cum >= (long long)std::ceil(0.5 * (double)m_count)) { o.masked_geo_median_approx = (i + 0.5) * 0.5; med = true; }
            if (!p90 && cum >= (long long)std::ceil(0.9 * (double)m_count)) { o.masked_geo_p90_approx = (i + 0.5) * 0.5; p90 = true; }
        }
    }
    o.masked_geo_min = std::isfinite(geo_min) ? geo_min : 0.0;
    o.masked_geo_max = geo_max;
    *stats = o;
}

pfd_status pfd_cycle_check(pfd_ctx* ctx, int frame_id, const pfd_cycle_cfg* cfg, float baseline_unit,
                           pfd_cycle_stats* stats, float* geo_err, float* pho_err, uint8_t* texmask)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    if (!cfg) return fail(ctx, PFD_EINVAL, "cycle config is NULL");
    if (cfg->max_triplet < 0 || cfg->max_triplet > 32) return fail(ctx, PFD_EINVAL, "max_triplet outside [0, 32]");
    if (!(baseline_unit > 0.0f)) return fail(ctx, PFD_EINVAL, "baseline_unit must be > 0");
    if (!f->has_state) return fail(ctx, PFD_ESTATE, "cycle check before PatchMatch");
    DeviceGuard g(ctx->device);
    const size_t px = (size_t)f->V * f->mi_w * f->mi_h;
    pfd_status st;
    void* p = nullptr;
    if (!f->d_cyc_recs) {
        const size_t rec_bytes = sizeof(pfd::CycleTileRec) * (size_t)f->V;
        if ((st = frame_alloc(ctx, *f, &p, rec_bytes + sizeof(unsigned int) * pfd::kCycleHistBins)) != PFD_OK)
            return st;
        f->d_cyc_recs = (pfd::CycleTileRec*)p;
        f->d_cyc_hist = (unsigned int*)((char*)p + rec_bytes);
    }
    const bool maps = geo_err || pho_err || texmask;
    if (maps && !f->d_cyc_maps) {
        if ((st = frame_alloc(ctx, *f, &p, 2 * sizeof(float) * px + px)) != PFD_OK) return st;
        f->d_cyc_maps = (float*)p;
        f->d_cyc_tm = (uint8_t*)(f->d_cyc_maps + 2 * px);
    }
    pfd::CycleCfg cc;
    static_assert(sizeof(cc) == sizeof(pfd_cycle_cfg), "cycle config layouts differ");
    std::memcpy(&cc, cfg, sizeof(cc));
    const pfd::CheckFrame F = check_frame(*f, baseline_unit);
    if (pfd::cycle_smem_bytes(F) > 227 * 1024) return fail(ctx, PFD_EINVAL, "cycle-check tile does not fit shared memory");
    CU(cudaMemsetAsync(f->d_cyc_hist, 0, sizeof(unsigned int) * pfd::kCycleHistBins, ctx->stream));
    CU(pfd::launch_cycle(F, cc, f->s[f->cur], maps ? f->d_cyc_maps : nullptr, maps ? f->d_cyc_maps + px : nullptr,
                         maps ? f->d_cyc_tm : nullptr, f->d_cyc_recs, f->d_cyc_hist, ctx->stream));
    ctx->launches += 1;
    f->cyc_done = true;
    if (!stats && !geo_err && !pho_err && !texmask) return PFD_OK;   // stays enqueued; pfd_cycle_check_stats folds it later
    std::vector<pfd::CycleTileRec> rec(f->V);
    unsigned int hist[pfd::kCycleHistBins];
    CU(cudaMemcpyAsync(rec.data(), f->d_cyc_recs, sizeof(pfd::CycleTileRec) * rec.size(), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CU(cudaMemcpyAsync(hist, f->d_cyc_hist, sizeof(hist), cudaMemcpyDeviceToHost, ctx->stream));
    if (geo_err) CU(cudaMemcpyAsync(geo_err, f->d_cyc_maps, sizeof(float) * px, cudaMemcpyDeviceToHost, ctx->stream));
    if (pho_err)
        CU(cudaMemcpyAsync(pho_err, f->d_cyc_maps + px, sizeof(float) * px, cudaMemcpyDeviceToHost, ctx->stream));
    if (texmask) CU(cudaMemcpyAsync(texmask, f->d_cyc_tm, px, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    if ((st = check_device_error(ctx)) != PFD_OK) return st;
    if (stats) fold_cycle_stats(rec, hist, stats);
    return PFD_OK;
}

pfd_status pfd_cycle_check_stats(pfd_ctx* ctx, int frame_id, pfd_cycle_stats* stats)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    if (!stats) return fail(ctx, PFD_EINVAL, "cycle_check_stats: NULL output");
    if (!f->cyc_done) return fail(ctx, PFD_ESTATE, "cycle_check_stats before pfd_cycle_check");
    DeviceGuard g(ctx->device);
    std::vector<pfd::CycleTileRec> rec(f->V);
    unsigned int hist[pfd::kCycleHistBins];
    CU(cudaMemcpyAsync(rec.data(), f->d_cyc_recs, sizeof(pfd::CycleTileRec) * rec.size(), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CU(cudaMemcpyAsync(hist, f->d_cyc_hist, sizeof(hist), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    pfd_status st = check_device_error(ctx);
    if (st != PFD_OK) return st;
    fold_cycle_stats(rec, hist, stats);
    return PFD_OK;
}


static const int kMaxSlices = 1024;

// Bucket grid of lens centres for the render (built once per frame): cells of
// 32 px, ids ascending within a cell.
static pfd_status build_lens_grid(pfd_ctx* ctx, Frame& f)
{
    if (f.d_cells) return PFD_OK;
    float x0 = INFINITY, y0 = INFINITY, x1 = -INFINITY, y1 = -INFINITY;
    for (int v = 0; v < f.V; ++v) {
        x0 = std::min(x0, f.h_centers[2 * v]); x1 = std::max(x1, f.h_centers[2 * v]);
        y0 = std::min(y0, f.h_centers[2 * v + 1]); y1 = std::max(y1, f.h_centers[2 * v + 1]);
    }
    const float cell = 32.0f, inv = 1.0f / cell;
    const int gw = std::max(1, (int)std::floor((x1 - x0) * inv) + 1), gh = std::max(1, (int)std::floor((y1 - y0) * inv) + 1);
    std::vector<int> start((size_t)gw * gh + 1, 0), ids(f.V);
    std::vector<int> cell_of(f.V);
    for (int v = 0; v < f.V; ++v) {
        const int cx = std::min(gw - 1, std::max(0, (int)std::floor((f.h_centers[2 * v] - x0) * inv)));
        const int cy = std::min(gh - 1, std::max(0, (int)std::floor((f.h_centers[2 * v + 1] - y0) * inv)));
        cell_of[v] = cy * gw + cx;
        start[cell_of[v] + 1]++;
    }
    for (size_t i = 1; i < start.size(); ++i) start[i] += start[i - 1];
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (int v = 0; v < f.V; ++v) ids[fill[cell_of[v]]++] = v;
    void* p = nullptr;
    pfd_status st = frame_alloc(ctx, f, &p, sizeof(int) * (start.size() + ids.size()) + sizeof(float) * kMaxSlices);
    if (st != PFD_OK) return st;
    f.d_cells = (int*)p;
    f.d_slice_vd = (float*)(f.d_cells + start.size() + ids.size());
    CU(cudaMemcpyAsync(f.d_cells, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(f.d_cells + start.size(), ids.data(), sizeof(int) * ids.size(), cudaMemcpyHostToDevice,
                       ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));      // host vectors go out of scope
    f.grid_w = gw; f.grid_h = gh; f.grid_x0 = x0; f.grid_y0 = y0; f.grid_cell = cell;
    return PFD_OK;
}

// Stream-ordered scratch for the host-array entry points below.
struct AsyncBuf {
    cudaStream_t st;
    void* p = nullptr;
    AsyncBuf(cudaStream_t s, size_t bytes, cudaError_t& e) : st(s) { e = cudaMallocAsync(&p, bytes, s); }
    ~AsyncBuf() { if (p) cudaFreeAsync(p, st); }
};

static pfd_status vd_args(pfd_ctx* ctx, const void* vd, size_t n, const void* out)
{
    if (!ctx) return PFD_EINVAL;
    if (n > 0 && (!vd || !out)) return fail(ctx, PFD_EINVAL, "vd / output array is NULL");
    if (n > ((size_t)1 << 33)) return fail(ctx, PFD_EINVAL, "too many values (%zu)", n);
    return PFD_OK;
}

pfd_status pfd_vd_to_rd_map_device(pfd_ctx* ctx, const float* vd_dev, size_t n, const double c[3], double* rd_dev)
{
    pfd_status st = vd_args(ctx, vd_dev, n, rd_dev);
    if (st != PFD_OK) return st;
    if (!c) return fail(ctx, PFD_EINVAL, "model coefficients are NULL");
    if (n == 0) return PFD_OK;
    DeviceGuard g(ctx->device);
    CU(pfd::launch_vd_to_rd(vd_dev, n, c[0], c[1], c[2], 0, rd_dev, ctx->stream));
    ctx->launches += 1;
    return PFD_OK;
}

static pfd_status vd_host(pfd_ctx* ctx, const float* vd, size_t n, const double c[3], int mode, void* out)
{
    pfd_status st = vd_args(ctx, vd, n, out);
    if (st != PFD_OK) return st;
    if (!c) return fail(ctx, PFD_EINVAL, "model coefficients are NULL");
    if (n == 0) return PFD_OK;
    DeviceGuard g(ctx->device);
    const size_t osz = mode == 0 ? 8 : 4;
    cudaError_t e;
    AsyncBuf buf(ctx->stream, n * 4 + n * osz + 16, e);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(ctx, PFD_ENOMEM, "vd_to_rd: device buffer of %zu bytes", n * (4 + osz)); }
    float* d_vd = (float*)buf.p;
    void* d_out = (void*)(((uintptr_t)(d_vd + n) + 15) & ~(uintptr_t)15);
    CU(cudaMemcpyAsync(d_vd, vd, n * 4, cudaMemcpyHostToDevice, ctx->stream));
    CU(pfd::launch_vd_to_rd(d_vd, n, c[0], c[1], c[2], mode, d_out, ctx->stream));
    ctx->launches += 1;
    CU(cudaMemcpyAsync(out, d_out, n * osz, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return PFD_OK;
}

pfd_status pfd_vd_to_rd_map(pfd_ctx* ctx, const float* vd, size_t n, const double c[3], double* rd)
{
    return vd_host(ctx, vd, n, c, 0, rd);
}

pfd_status pfd_vd_to_rd_points(pfd_ctx* ctx, const float* vd, size_t n, const double c[3], float* rd)
{
    return vd_host(ctx, vd, n, c, 1, rd);
}

pfd_status pfd_vd_to_rd_segments(pfd_ctx* ctx, const float* vd, size_t n, const pfd_vd_segment* segs, int nseg,
                                 float* rd)
{
    pfd_status st = vd_args(ctx, vd, n, rd);
    if (st != PFD_OK) return st;
    if (nseg < 0 || nseg > pfd::kMaxVdSegments || (nseg > 0 && !segs))
        return fail(ctx, PFD_EINVAL, "need 0..%d segments", pfd::kMaxVdSegments);
    if (n == 0) return PFD_OK;
    DeviceGuard g(ctx->device);
    cudaError_t e;
    AsyncBuf buf(ctx->stream, n * 8 + (size_t)nseg * 40 + 32, e);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(ctx, PFD_ENOMEM, "vd_to_rd_segments: device buffer"); }
    double* d_seg = (double*)buf.p;
    float* d_vd = (float*)(d_seg + 5 * (size_t)nseg);
    float* d_out = d_vd + n;
    static_assert(sizeof(pfd_vd_segment) == 5 * sizeof(double), "segment layout");
    if (nseg) CU(cudaMemcpyAsync(d_seg, segs, (size_t)nseg * 40, cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(d_vd, vd, n * 4, cudaMemcpyHostToDevice, ctx->stream));
    CU(pfd::launch_vd_to_rd_segments(d_vd, n, d_seg, nseg, d_out, ctx->stream));
    ctx->launches += 1;
    CU(cudaMemcpyAsync(rd, d_out, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return PFD_OK;
}

pfd_status pfd_fit_behavioral_model(pfd_ctx* ctx, const float* real_depth, const float* vd, size_t n, double c[3])
{
    pfd_status st = vd_args(ctx, vd, n, c);
    if (st != PFD_OK) return st;
    if (!real_depth) return fail(ctx, PFD_EINVAL, "real_depth is NULL");
    if (n < 3) return fail(ctx, PFD_EINVAL, "the behavioural model needs at least 3 pairs, got %zu", n);
    DeviceGuard g(ctx->device);
    const int nb = pfd::fit_blocks(n);
    cudaError_t e;
    AsyncBuf buf(ctx->stream, n * 8 + (size_t)nb * 72 + 72 + 32, e);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(ctx, PFD_ENOMEM, "behavioural fit: device buffer"); }
    double* d_partial = (double*)buf.p;
    double* d_sums = d_partial + (size_t)nb * 9;
    float* d_real = (float*)(d_sums + 9);
    float* d_vd = d_real + n;
    CU(cudaMemcpyAsync(d_real, real_depth, n * 4, cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(d_vd, vd, n * 4, cudaMemcpyHostToDevice, ctx->stream));
    CU(pfd::launch_fit_sums(d_real, d_vd, n, d_partial, d_sums, ctx->stream));
    ctx->launches += 2;
    double h[9];
    CU(cudaMemcpyAsync(h, d_sums, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    // normal equations, Gaussian elimination with partial pivoting
    double M[3][4] = { { h[0], h[1], h[2], h[6] }, { h[1], h[3], h[4], h[7] }, { h[2], h[4], h[5], h[8] } };
    for (int col = 0; col < 3; ++col) {
        int piv = col;
        for (int r = col + 1; r < 3; ++r) if (std::fabs(M[r][col]) > std::fabs(M[piv][col])) piv = r;
        if (!(std::fabs(M[piv][col]) > 1e-300)) return fail(ctx, PFD_EINVAL, "behavioural fit: singular system");
        if (piv != col) for (int q = 0; q < 4; ++q) std::swap(M[col][q], M[piv][q]);
        for (int r = 0; r < 3; ++r) {
            if (r == col) continue;
            const double f = M[r][col] / M[col][col];
            for (int q = col; q < 4; ++q) M[r][q] -= f * M[col][q];
        }
    }
    for (int r = 0; r < 3; ++r) c[r] = M[r][3] / M[r][r];
    return PFD_OK;
}

pfd_status pfd_launch_count(pfd_ctx* ctx, unsigned long long* n)
{
    if (!ctx || !n) return PFD_EINVAL;
    *n = ctx->launches;
    return PFD_OK;
}

pfd_status pfd_refocus(pfd_ctx* ctx, int frame_id, const float* slice_vd, int n_slices, int out_w, int out_h,
                       float* out)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    if (!slice_vd || n_slices < 1 || n_slices > kMaxSlices)
        return fail(ctx, PFD_EINVAL, "refocus: need 1..%d slice virtual depths", kMaxSlices);
    if (out_w < 1 || out_h < 1 || out_w > 65536 || out_h > 65536) return fail(ctx, PFD_EINVAL, "refocus: bad output size");
    for (int i = 0; i < n_slices; ++i)
        if (!(slice_vd[i] > 0.0f) || !std::isfinite(slice_vd[i]))
            return fail(ctx, PFD_EINVAL, "refocus: slice %d virtual depth must be finite and > 0", i);
    if (!f->has_raw) return fail(ctx, PFD_ESTATE, "frame has no raw image yet");
    DeviceGuard g(ctx->device);
    pfd_status st = build_lens_grid(ctx, *f);
    if (st != PFD_OK) return st;
    const size_t need = sizeof(float) * (size_t)n_slices * out_w * out_h;
    if (need > f->stack_bytes) {
        frame_free_one(ctx, *f, f->d_stack, f->stack_bytes);
        f->d_stack = nullptr;
        f->stack_bytes = 0;
        void* p = nullptr;
        if ((st = frame_alloc(ctx, *f, &p, need)) != PFD_OK) return st;
        f->d_stack = (float*)p;
        f->stack_bytes = need;
    }
    pfd::RefocusFrame R;
    R.V = f->V; R.m = f->mi_w; R.mh = f->mi_h; R.tile_stride = f->tile_stride;
    R.gray = f->d_gray; R.centers = f->d_centers;
    R.cell_start = f->d_cells;
    R.cell_ids = f->d_cells + (size_t)f->grid_w * f->grid_h + 1;
    R.grid_w = f->grid_w; R.grid_h = f->grid_h;
    R.grid_x0 = f->grid_x0; R.grid_y0 = f->grid_y0; R.cell = f->grid_cell;
    if (pfd::refocus_smem_bytes(R) > 227 * 1024) return fail(ctx, PFD_EINVAL, "refocus: micro-image too large");
    CU(cudaMemcpyAsync(f->d_slice_vd, slice_vd, sizeof(float) * n_slices, cudaMemcpyHostToDevice, ctx->stream));
    CU(pfd::launch_refocus(R, f->d_slice_vd, n_slices, f->W, f->H, out_w, out_h, f->d_stack, ctx->d_err, ctx->stream));
    ctx->launches += 1;
    if (out) CU(cudaMemcpyAsync(out, f->d_stack, need, cudaMemcpyDeviceToHost, ctx->stream));
    return out ? check_device_error(ctx) : PFD_OK;
}

// Wavefront steps of the fusion: a reference micro-image runs one step after
// the last step that touched any micro-image it touches (itself and its list
// entries), so two micro-images that share one keep the reference's order and
// micro-images of one step touch disjoint sets.
static void fuse_schedule(int V, const int* lists, const int* counts, int max_list, const uint8_t* is_ref,
                          std::vector<int>& order, std::vector<int>& step_start)
{
    std::vector<int> last(V, 0), step(V, 0);
    int nsteps = 0;
    for (int v = 0; v < V; ++v) {
        if (!is_ref[v]) continue;
        const int nl = std::min(counts[v], max_list);
        int s = last[v];
        for (int j = 0; j < nl; ++j) {
            const int u = lists[(size_t)v * max_list + j];
            if (u >= 0) s = std::max(s, last[u]);
        }
        step[v] = ++s;
        last[v] = s;
        for (int j = 0; j < nl; ++j) {
            const int u = lists[(size_t)v * max_list + j];
            if (u >= 0) last[u] = s;
        }
        nsteps = std::max(nsteps, s);
    }
    std::vector<int> cnt((size_t)nsteps + 2, 0);
    for (int v = 0; v < V; ++v)
        if (is_ref[v]) cnt[(size_t)step[v]]++;
    step_start.assign((size_t)nsteps + 1, 0);
    for (int s = 1; s <= nsteps; ++s) step_start[s] = step_start[s - 1] + cnt[(size_t)s];
    order.assign((size_t)step_start[nsteps], 0);
    std::vector<int> fill(step_start.begin(), step_start.end());
    for (int v = 0; v < V; ++v)                       // ascending view order inside a step
        if (is_ref[v]) order[(size_t)fill[(size_t)step[v] - 1]++] = v;
}

pfd_status pfd_fuse_virtual_depth(pfd_ctx* ctx, int frame_id, const pfd_fuse_params* p, const int* lists,
                                  const int* list_counts, int max_list, const uint8_t* is_ref, const uint8_t* bgr,
                                  float* vd_map, uint8_t* conf, uint8_t* aif, float* points, long long* n_points)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    if (!p || !lists || !list_counts || !is_ref) return fail(ctx, PFD_EINVAL, "fuse: NULL argument");
    if (max_list < 1 || max_list > pfd::kFuseMaxList)
        return fail(ctx, PFD_EINVAL, "fuse: max_list %d outside [1, %d]", max_list, pfd::kFuseMaxList);
    if (!std::isfinite(p->mla_base) || !std::isfinite(p->min_ref_disp) || !std::isfinite(p->max_reproj_px) ||
        !std::isfinite(p->max_rel_vd))
        return fail(ctx, PFD_EINVAL, "fuse: parameters must be finite");
    if (f->mi_w != f->mi_h) return fail(ctx, PFD_EINVAL, "fuse: square micro-images only (%dx%d)", f->mi_w, f->mi_h);
    if (!f->has_state) return fail(ctx, PFD_ESTATE, "fuse before PatchMatch");
    if (!bgr && !f->has_mi) return fail(ctx, PFD_ESTATE, "frame has no micro-images yet");
    const int V = f->V;
    for (int v = 0; v < V; ++v) {
        if (list_counts[v] < 0 || list_counts[v] > max_list)
            return fail(ctx, PFD_EINVAL, "fuse: view %d list count %d outside [0, %d]", v, list_counts[v], max_list);
        for (int j = 0; j < list_counts[v]; ++j) {
            const int u = lists[(size_t)v * max_list + j];
            if (u < -1 || u >= V) return fail(ctx, PFD_EINVAL, "fuse: view %d list entry %d is %d", v, j, u);
        }
    }
    DeviceGuard g(ctx->device);
    std::vector<int> order, step_start;
    fuse_schedule(V, lists, list_counts, max_list, is_ref, order, step_start);
    const size_t ppv = (size_t)f->mi_w * f->mi_h, px = (size_t)V * ppv, npix = (size_t)f->W * f->H;
    const size_t nb = (px + pfd::kFuseScanBlock - 1) / pfd::kFuseScanBlock;
    cudaStream_t s = ctx->stream;
    // scratch of this call, from the stream-ordered pool
    struct Scratch {
        cudaStream_t s;
        std::vector<void*> ptrs;
        ~Scratch() { for (void* q : ptrs) cudaFreeAsync(q, s); }
        cudaError_t get(void** q, size_t bytes) {
            cudaError_t e = cudaMallocAsync(q, bytes > 0 ? bytes : 1, s);
            if (e == cudaSuccess) ptrs.push_back(*q);
            return e;
        }
    } S{ s, {} };
    int *d_lists = nullptr, *d_counts = nullptr, *d_order = nullptr;
    uint8_t *d_bgr = nullptr, *d_mask = nullptr, *d_conf = nullptr, *d_aif = nullptr;
    unsigned int *d_winner = nullptr, *d_has = nullptr, *d_bcount = nullptr;
    float *d_rec = nullptr, *d_vd = nullptr, *d_points = nullptr;
    CU(S.get((void**)&d_lists, sizeof(int) * (size_t)V * max_list));
    CU(S.get((void**)&d_counts, sizeof(int) * (size_t)V));
    CU(S.get((void**)&d_order, sizeof(int) * std::max<size_t>(order.size(), 1)));
    if (bgr) CU(S.get((void**)&d_bgr, px * 3));
    CU(S.get((void**)&d_mask, px));
    CU(S.get((void**)&d_winner, sizeof(unsigned int) * npix));
    CU(S.get((void**)&d_has, sizeof(unsigned int) * px));
    CU(S.get((void**)&d_rec, sizeof(float) * 10 * px));
    CU(S.get((void**)&d_vd, sizeof(float) * npix));
    CU(S.get((void**)&d_conf, npix));
    CU(S.get((void**)&d_aif, npix * 3));
    CU(cudaMemcpyAsync(d_lists, lists, sizeof(int) * (size_t)V * max_list, cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(d_counts, list_counts, sizeof(int) * (size_t)V, cudaMemcpyHostToDevice, s));
    if (!order.empty())
        CU(cudaMemcpyAsync(d_order, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice, s));
    if (bgr) CU(cudaMemcpyAsync(d_bgr, bgr, px * 3, cudaMemcpyHostToDevice, s));
    CU(cudaMemsetAsync(d_mask, 0, px, s));
    CU(cudaMemsetAsync(d_winner, 0, sizeof(unsigned int) * npix, s));
    CU(cudaMemsetAsync(d_has, 0, sizeof(unsigned int) * px, s));
    pfd::FuseFrame F;
    F.V = V; F.m = f->mi_w; F.ppv = (int)ppv; F.tile_stride = f->tile_stride;
    F.gray = f->d_gray; F.bgr = d_bgr; F.centers = f->d_centers; F.plane = f->s[f->cur].plane;
    F.lists = d_lists; F.list_counts = d_counts; F.max_list = max_list;
    F.mla_base = p->mla_base; F.min_ref_disp = p->min_ref_disp; F.max_reproj_px = p->max_reproj_px;
    F.max_rel_vd = p->max_rel_vd; F.min_consistent = p->min_consistent;
    F.raw_w = f->W; F.raw_h = f->H;
    F.mask = d_mask; F.winner = d_winner; F.rec = d_rec; F.has_rec = d_has;
    for (size_t k = 0; k + 1 < step_start.size(); ++k) {
        const int a = step_start[k], b = step_start[k + 1];
        CU(pfd::launch_fuse_step(F, d_order + a, b - a, s));
        ctx->launches += 1;
    }
    CU(pfd::launch_fuse_maps(F, d_vd, d_conf, d_aif, s));
    ctx->launches += 1;
    if (vd_map) CU(cudaMemcpyAsync(vd_map, d_vd, sizeof(float) * npix, cudaMemcpyDeviceToHost, s));
    if (conf) CU(cudaMemcpyAsync(conf, d_conf, npix, cudaMemcpyDeviceToHost, s));
    if (aif) CU(cudaMemcpyAsync(aif, d_aif, npix * 3, cudaMemcpyDeviceToHost, s));
    if (points || n_points) {
        CU(S.get((void**)&d_bcount, sizeof(unsigned int) * nb));
        CU(pfd::launch_fuse_count(F, d_bcount, s));
        ctx->launches += 1;
        std::vector<unsigned int> bc(nb);
        CU(cudaMemcpyAsync(bc.data(), d_bcount, sizeof(unsigned int) * nb, cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        unsigned long long total = 0;
        for (size_t i = 0; i < nb; ++i) { const unsigned int c = bc[i]; bc[i] = (unsigned int)total; total += c; }
        if (n_points) *n_points = (long long)total;
        if (points && total) {
            CU(cudaMemcpyAsync(d_bcount, bc.data(), sizeof(unsigned int) * nb, cudaMemcpyHostToDevice, s));
            CU(S.get((void**)&d_points, sizeof(float) * 9 * total));
            CU(pfd::launch_fuse_compact(F, d_bcount, d_points, s));
            ctx->launches += 1;
            CU(cudaMemcpyAsync(points, d_points, sizeof(float) * 9 * total, cudaMemcpyDeviceToHost, s));
        }
    }
    if (vd_map || conf || aif || points || n_points) return check_device_error(ctx);
    return PFD_OK;
}

// ---- matching-neighbour selection ---------------------------------------------

// The selection given the micro-images on the device (tiles tile_stride bytes
// apart) and the centres on the host and the device: every ring candidate's
// similarity on the device, then the per-view ring walk, RANSAC, stop rule and
// sort on the host threads.  out_ids [n][max_nb], out_counts [n].
// The selection given the rings and the micro-images on the device (tiles
// tile_stride bytes apart): every ring candidate's similarity on the device,
// then the per-view RANSAC, stop rule and sort on the host threads.  d_pairs /
// d_out: the plan's pairs already on the device and room for their
// similarities, or NULL to use temporary buffers.  out_ids [n][max_nb],
// out_counts [n].
static pfd_status select_lists(pfd_ctx* ctx, const RingPlan& rp, const int2* d_pairs, int* d_out,
                               const uint8_t* d_img, int tile_stride, int mi_w, int mi_h, const float2* d_c,
                               int max_nb, int* out_ids, int* out_counts)
{
    const int n_views = rp.G.V;
    cudaStream_t s = ctx->stream;
    const size_t np = rp.pairs.size();
    std::vector<int> sims(np);
    int2* tp = nullptr;
    int* to = nullptr;
    cudaError_t e = cudaSuccess;
    if (!d_pairs) {
        e = cudaMallocAsync((void**)&tp, sizeof(int2) * std::max<size_t>(np, 1), s);
        if (e == cudaSuccess) e = cudaMallocAsync((void**)&to, sizeof(int) * std::max<size_t>(np, 1), s);
        if (e == cudaSuccess && np)
            e = cudaMemcpyAsync(tp, rp.pairs.data(), sizeof(int2) * np, cudaMemcpyHostToDevice, s);
        d_pairs = tp;
        d_out = to;
    }
    if (e == cudaSuccess) e = pfd::launch_similarity(d_img, tile_stride, mi_w, mi_h, d_c, d_pairs, (int)np, d_out, s);
    if (e == cudaSuccess && np) e = cudaMemcpyAsync(sims.data(), d_out, sizeof(int) * np, cudaMemcpyDeviceToHost, s);
    for (void* q : { (void*)tp, (void*)to })
        if (q) cudaFreeAsync(q, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, PFD_ECUDA, "select_neighbors: %s", cudaGetErrorString(e));
    }
    ctx->launches += 1;
    pfd::parallel_views(n_views, [&](int a, int b) {
        std::vector<int> list;
        for (int v = a; v < b; ++v) {
            auto sim = [&](int ring, int i) { return (float)(double)sims[rp.first[(size_t)v * 5 + ring] + i]; };
            pfd::select_for_view(rp.G, rp.pitch, v, rp.R[v], sim, list);
            const int n = std::min((int)list.size(), max_nb);
            for (int k = 0; k < max_nb; ++k) out_ids[(size_t)v * max_nb + k] = k < n ? list[k] : -1;
            out_counts[v] = n;
        }
    });
    return PFD_OK;
}

pfd_status pfd_select_neighbors(pfd_ctx* ctx, const float* centers, const int* tilekeys, int n_views, int mla_u_size,
                                int mla_v_size, float pitch, const uint8_t* images, int mi_w, int mi_h, int max_nb,
                                int* nb_ids, int* nb_counts)
{
    if (!ctx) return PFD_EINVAL;
    if (!centers || !tilekeys || !images || !nb_ids || !nb_counts || n_views < 1)
        return fail(ctx, PFD_EINVAL, "select_neighbors: NULL argument or no views");
    if (!(pitch > 0.0f) || mi_w < 2 || mi_h < 2 || mi_w > 64 || mi_h > 64 || max_nb < 1 || max_nb > 128)
        return fail(ctx, PFD_EINVAL, "select_neighbors: bad pitch, window or max_nb");
    if (mla_u_size < 1 || mla_v_size < 1 || (long long)mla_u_size * mla_v_size > (1LL << 28))
        return fail(ctx, PFD_EINVAL, "select_neighbors: bad lens grid %d x %d", mla_u_size, mla_v_size);
    RingPlan rp;
    if (!rp.build(centers, tilekeys, n_views, mla_u_size, mla_v_size, pitch))
        return fail(ctx, PFD_EINVAL, "select_neighbors: a tile key lies outside the grid or is repeated");
    DeviceGuard g(ctx->device);
    cudaStream_t s = ctx->stream;
    const size_t ppv = (size_t)mi_w * mi_h;
    uint8_t* d_img = nullptr;
    float2* d_c = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&d_img, ppv * n_views, s);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&d_c, sizeof(float2) * n_views, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_img, images, ppv * n_views, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_c, centers, sizeof(float2) * n_views, cudaMemcpyHostToDevice, s);
    pfd_status st = PFD_OK;
    if (e != cudaSuccess) {
        cudaGetLastError();
        st = fail(ctx, PFD_ECUDA, "select_neighbors: %s", cudaGetErrorString(e));
    } else {
        st = select_lists(ctx, rp, nullptr, nullptr, d_img, (int)ppv, mi_w, mi_h, d_c, max_nb, nb_ids, nb_counts);
    }
    for (void* q : { (void*)d_img, (void*)d_c })
        if (q) cudaFreeAsync(q, s);
    return st;
}

pfd_status pfd_frame_select_neighbors(pfd_ctx* ctx, int frame_id, int mla_u_size, int mla_v_size, float pitch,
                                      int max_list, int* nb_ids, int* nb_counts)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    if (!f->has_mi) return fail(ctx, PFD_ESTATE, "frame_select_neighbors: frame %d has no micro-images", frame_id);
    if (!(pitch > 0.0f)) return fail(ctx, PFD_EINVAL, "frame_select_neighbors: pitch must be > 0");
    if ((nb_ids != nullptr) != (nb_counts != nullptr) || (nb_ids && (max_list < 1 || max_list > 128)))
        return fail(ctx, PFD_EINVAL, "frame_select_neighbors: give both lists (max_list 1-128) or neither");
    if (mla_u_size < 1 || mla_v_size < 1 || (long long)mla_u_size * mla_v_size > (1LL << 28))
        return fail(ctx, PFD_EINVAL, "frame_select_neighbors: bad lens grid %d x %d", mla_u_size, mla_v_size);
    DeviceGuard g(ctx->device);
    // the rings depend on the lens grid and the pitch only: made once per frame
    if (!f->rings || f->rings->u != mla_u_size || f->rings->v != mla_v_size || f->rings->pitch != pitch) {
        auto rp = std::make_shared<RingPlan>();
        if (!rp->build(f->h_centers.data(), f->h_keys.data(), f->V, mla_u_size, mla_v_size, pitch))
            return fail(ctx, PFD_EINVAL, "frame_select_neighbors: a tile key lies outside the grid or is repeated");
        if (f->d_pairs) { frame_free_one(ctx, *f, f->d_pairs, sizeof(int2) * f->n_pairs_alloc); f->d_pairs = nullptr; }
        if (f->d_sims) { frame_free_one(ctx, *f, f->d_sims, sizeof(int) * f->n_pairs_alloc); f->d_sims = nullptr; }
        const size_t np = std::max<size_t>(rp->pairs.size(), 1);
        f->n_pairs_alloc = np;
        void* p = nullptr;
        pfd_status st = frame_alloc(ctx, *f, &p, sizeof(int2) * np);
        if (st != PFD_OK) return st;
        f->d_pairs = (int2*)p;
        if ((st = frame_alloc(ctx, *f, &p, sizeof(int) * np)) != PFD_OK) return st;
        f->d_sims = (int*)p;
        if (!rp->pairs.empty())
            CU(cudaMemcpyAsync(f->d_pairs, rp->pairs.data(), sizeof(int2) * rp->pairs.size(), cudaMemcpyHostToDevice,
                               ctx->stream));
        f->rings = rp;
    }
    const int L = std::max(f->K, nb_ids ? max_list : 0);
    std::vector<int> ids((size_t)f->V * L), cnt(f->V);
    pfd_status st = select_lists(ctx, *f->rings, f->d_pairs, f->d_sims, f->d_gray, f->tile_stride, f->mi_w, f->mi_h,
                                 f->d_centers, L, ids.data(), cnt.data());
    if (st != PFD_OK) return st;
    // the matcher's lists: the first K of each (AdaptMIPMFrame::BuildViewIndexMap keeps the first 16 views)
    const std::vector<int> old_ids = f->h_nb_ids, old_counts = f->h_nb_counts;
    for (int v = 0; v < f->V; ++v) {
        const int n = std::min(cnt[v], f->K);
        for (int k = 0; k < f->K; ++k) f->h_nb_ids[(size_t)v * f->K + k] = k < n ? ids[(size_t)v * L + k] : -1;
        f->h_nb_counts[v] = n;
        if (nb_ids) {
            const int m = std::min(cnt[v], max_list);
            for (int k = 0; k < max_list; ++k) nb_ids[(size_t)v * max_list + k] = k < m ? ids[(size_t)v * L + k] : -1;
            nb_counts[v] = m;
        }
    }
    CU(cudaMemcpyAsync(f->d_nb_ids, f->h_nb_ids.data(), sizeof(int) * f->h_nb_ids.size(), cudaMemcpyHostToDevice,
                       ctx->stream));
    CU(cudaMemcpyAsync(f->d_nb_counts, f->h_nb_counts.data(), sizeof(int) * f->V, cudaMemcpyHostToDevice, ctx->stream));
    // the host copies are the frame's own (they outlive the copies); the
    // state, the stored cost vectors and the filter's schedule belong to the
    // old lists
    f->has_state = false;
    f->cvec_valid = 0;
    if (f->h_nb_ids != old_ids || f->h_nb_counts != old_counts) {
        f->step_start.clear();        // the filter's schedule and its graph follow the old lists
        f->filter_graph.reset();
    }
    return PFD_OK;
}

// ---- micro-lens centres ------------------------------------------------------

// DepthSolver::Otsu (DepthSolver.cpp:486-546) on the histogram, float arithmetic as written.
static int otsu_threshold(const unsigned int* count, long long pixel_sum)
{
    float pro[256];
    for (int i = 0; i < 256; ++i) pro[i] = (float)count[i] / (float)pixel_sum;
    float deltaMax = 0;
    int threshold = 0;
    for (int i = 0; i < 256; ++i) {
        float w0 = 0, w1 = 0, u0tmp = 0, u1tmp = 0;
        for (int j = 0; j < 256; ++j) {
            if (j <= i) { w0 += pro[j]; u0tmp += j * pro[j]; }
            else { w1 += pro[j]; u1tmp += j * pro[j]; }
        }
        const float u0 = u0tmp / w0, u1 = u1tmp / w1, u = u0tmp + u1tmp;
        const float deltaTmp = w0 * (u0 - u) * (u0 - u) + w1 * (u1 - u) * (u1 - u);
        if (deltaTmp > deltaMax) { deltaMax = deltaTmp; threshold = i; }
    }
    return threshold;
}

pfd_status pfd_mla_centers(pfd_ctx* ctx, const uint8_t* white_bgr, int W, int H, int step, float baseline,
                           int mla_u_size, int mla_v_size, pfd_mla_lens* out, int max_out, int* n_out, int* threshold)
{
    if (!ctx) return PFD_EINVAL;
    if (!white_bgr || !n_out || (!out && max_out > 0)) return fail(ctx, PFD_EINVAL, "mla_centers: NULL argument");
    if (W < 1 || H < 1 || step < 3 * W || (long long)W * H > (1LL << 30))
        return fail(ctx, PFD_EINVAL, "mla_centers: bad image size %dx%d, step %d", W, H, step);
    if (!(baseline > 0.0f) || mla_u_size < 1 || mla_v_size < 1)
        return fail(ctx, PFD_EINVAL, "mla_centers: baseline and lens counts must be positive");
    DeviceGuard g(ctx->device);
    cudaStream_t s = ctx->stream;
    const size_t n = (size_t)W * H;
    const int max_roots = (int)std::min<size_t>(n / 2 + 1, (size_t)1 << 24);
    uint8_t *d_bgr = nullptr, *d_fg = nullptr;
    int *d_L = nullptr, *d_roots = nullptr;
    unsigned int* d_hist = nullptr;
    double* d_sums = nullptr;
    struct Pool {
        cudaStream_t s;
        std::vector<void*> p;
        ~Pool() { for (void* q : p) cudaFreeAsync(q, s); }
        cudaError_t get(void** q, size_t b) { cudaError_t e = cudaMallocAsync(q, b, s); if (!e) p.push_back(*q); return e; }
    } P{ s, {} };
    CU(P.get((void**)&d_bgr, (size_t)step * H));
    CU(P.get((void**)&d_fg, n));
    CU(P.get((void**)&d_L, sizeof(int) * n));
    CU(P.get((void**)&d_roots, sizeof(int) * (size_t)max_roots));
    CU(P.get((void**)&d_hist, sizeof(unsigned int) * (256 + 1)));
    CU(cudaMemcpyAsync(d_bgr, white_bgr, (size_t)step * H, cudaMemcpyHostToDevice, s));
    CU(cudaMemsetAsync(d_hist, 0, sizeof(unsigned int) * (256 + 1), s));
    CU(pfd::launch_mla_hist(d_bgr, W, H, step, d_hist, s));
    unsigned int hist[256];
    CU(cudaMemcpyAsync(hist, d_hist, sizeof(hist), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    const int t = otsu_threshold(hist, (long long)W * H);
    if (threshold) *threshold = t;
    unsigned int* d_nroots = d_hist + 256;
    CU(pfd::launch_mla_components(d_bgr, W, H, step, t, d_fg, d_L, d_roots, d_nroots, max_roots, ctx->d_err, s));
    unsigned int nr = 0;
    CU(cudaMemcpyAsync(&nr, d_nroots, sizeof(nr), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if ((int)nr > max_roots) return fail(ctx, PFD_EINVAL, "mla_centers: %u components exceed %d", nr, max_roots);
    // findContours lists the external contours in reverse order of discovery
    std::vector<int> roots(nr);
    if (nr) CU(cudaMemcpyAsync(roots.data(), d_roots, sizeof(int) * nr, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    std::sort(roots.begin(), roots.end(), [](int a, int b) { return a > b; });
    std::vector<double> sums(3 * (size_t)nr);
    if (nr) {
        CU(P.get((void**)&d_sums, sizeof(double) * 3 * nr));
        CU(cudaMemcpyAsync(d_roots, roots.data(), sizeof(int) * nr, cudaMemcpyHostToDevice, s));
        CU(pfd::launch_mla_trace(d_fg, W, H, d_roots, (int)nr, d_sums, ctx->d_err, s));
        CU(cudaMemcpyAsync(sums.data(), d_sums, sizeof(double) * 3 * nr, cudaMemcpyDeviceToHost, s));
    }
    ctx->launches += 4 + (nr ? 1 : 0);
    pfd_status st = check_device_error(ctx);
    if (st != PFD_OK) return fail(ctx, PFD_EINVAL, "mla_centers: component labelling or border tracing did not finish");

    // ComputeMLACentersFromWhiteImage (:752-868): moments, position filter,
    // rows by running mean y, columns by x, small-area flag.
    struct Info { float x, y, area; int col, row; bool abandon; };
    std::vector<Info> infos;
    double average_area = 0.0;
    for (unsigned k = 0; k < nr; ++k) {
        const double a00 = sums[3 * k], a10 = sums[3 * k + 1], a01 = sums[3 * k + 2];
        double m00 = 0, m10 = 0, m01 = 0;
        if (std::fabs(a00) > 1.1920928955078125e-07) {       // moments() (FLT_EPSILON)
            const double h = a00 > 0 ? 0.5 : -0.5, s6 = a00 > 0 ? 1.0 / 6.0 : -1.0 / 6.0;
            m00 = a00 * h; m10 = a10 * s6; m01 = a01 * s6;
        }
        float x = -1, y = -1;
        if (m00 != 0) { x = (float)(m10 / m00); y = (float)(m01 / m00); }
        if (y >= baseline * 0.5 && y <= baseline * mla_v_size && x >= baseline * 0.5 && x <= baseline * mla_u_size) {
            const double area = std::fabs(a00 * 0.5);                 // contourArea()
            average_area += area;
            infos.push_back({ x, y, (float)area, 0, 0, false });      // MLA_Info::SetArea(float)
        }
    }
    average_area /= (double)nr;
    std::map<int, std::vector<int>> rows;
    float y_ideal_next = 0.0f;
    int y_ideal_next_count = 0;
    for (int row = 0; row < mla_v_size; ++row) {
        std::vector<int> members;
        float y_ideal = 0.0f;
        if (row == 0) {
            y_ideal = baseline * 0.5;
        } else {
            y_ideal = y_ideal_next / y_ideal_next_count;
            y_ideal += baseline;
            y_ideal_next = 0.0f;
            y_ideal_next_count = 0;
        }
        for (int i = 0; i < (int)infos.size(); ++i)
            if (std::fabs(infos[i].y - y_ideal) < baseline * 0.5) {
                members.push_back(i);
                y_ideal_next += infos[i].y;
                y_ideal_next_count++;
            }
        std::map<float, int> by_x;                                   // equal x: the later lens wins
        for (int i = 0; i < (int)members.size(); ++i) by_x[infos[members[i]].x] = i;
        std::vector<int> sorted;
        for (auto& kv : by_x) sorted.push_back(members[kv.second]);
        rows[row] = sorted;
    }
    std::map<std::pair<int, int>, int> keyed;                        // (row, col), the map's key order
    for (auto& kv : rows)
        for (int col = 0; col < (int)kv.second.size(); ++col) {
            Info& I = infos[kv.second[col]];
            I.col = col;
            I.row = kv.first;
            I.abandon = I.area < average_area * 0.8;
            keyed[{ kv.first, col }] = kv.second[col];
        }
    *n_out = (int)keyed.size();
    if ((int)keyed.size() > max_out) return out ? fail(ctx, PFD_EINVAL, "mla_centers: %d lenses, room for %d", *n_out, max_out)
                                                : PFD_OK;
    int i = 0;
    for (auto& kv : keyed) {
        const Info& I = infos[kv.second];
        out[i].col = kv.first.second;
        out[i].row = kv.first.first;
        out[i].cx = I.x;
        out[i].cy = I.y;
        out[i].area = I.area;
        out[i].abandon = I.abandon ? 1 : 0;
        ++i;
    }
    return PFD_OK;
}

pfd_status pfd_mla_lattice_fit(pfd_ctx* ctx, const pfd_mla_lens* lenses, int n, int skip_abandoned, double fit[6])
{
    if (!ctx) return PFD_EINVAL;
    if (!lenses || !fit || n < 1) return fail(ctx, PFD_EINVAL, "mla_lattice_fit: need lenses and an output");
    static_assert(sizeof(pfd_mla_lens) == sizeof(pfd::pfd_mla_lens_dev), "lens layouts differ");
    std::vector<pfd_mla_lens> use;
    for (int i = 0; i < n; ++i)
        if (!(skip_abandoned && lenses[i].abandon) && std::isfinite(lenses[i].cx) && std::isfinite(lenses[i].cy))
            use.push_back(lenses[i]);
    if (use.size() < 3) return fail(ctx, PFD_EINVAL, "mla_lattice_fit: fewer than 3 usable lenses");
    DeviceGuard g(ctx->device);
    cudaStream_t s = ctx->stream;
    const int nb = (int)std::max<size_t>(1, std::min<size_t>((use.size() + 1023) / 1024, 256));
    void *d_l = nullptr, *d_p = nullptr;
    CU(cudaMallocAsync(&d_l, sizeof(pfd_mla_lens) * use.size(), s));
    if (cudaMallocAsync(&d_p, sizeof(double) * 14 * nb, s) != cudaSuccess) {
        cudaFreeAsync(d_l, s);
        return fail(ctx, PFD_ENOMEM, "mla_lattice_fit: scratch");
    }
    std::vector<double> part(14 * (size_t)nb);
    cudaError_t e = cudaMemcpyAsync(d_l, use.data(), sizeof(pfd_mla_lens) * use.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = pfd::launch_mla_lattice((const pfd::pfd_mla_lens_dev*)d_l, (int)use.size(), (double*)d_p, nb, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(part.data(), d_p, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(d_l, s);
    cudaFreeAsync(d_p, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(ctx, PFD_ECUDA, "mla_lattice_fit: %s", cudaGetErrorString(e));
    ctx->launches += 1;
    double S[14] = { 0 };
    for (int b = 0; b < nb; ++b)
        for (int q = 0; q < 14; ++q) S[q] += part[(size_t)b * 14 + q];
    double M[4][5];
    int q = 0;
    for (int i0 = 0; i0 < 4; ++i0)
        for (int i1 = i0; i1 < 4; ++i1, ++q) M[i0][i1] = M[i1][i0] = S[q];
    for (int i0 = 0; i0 < 4; ++i0) M[i0][4] = S[10 + i0];
    // Gaussian elimination with partial pivoting (4 x 4, FP64)
    for (int c = 0; c < 4; ++c) {
        int pr = c;
        for (int r = c + 1; r < 4; ++r)
            if (std::fabs(M[r][c]) > std::fabs(M[pr][c])) pr = r;
        if (!(std::fabs(M[pr][c]) > 1e-300)) return fail(ctx, PFD_EINVAL, "mla_lattice_fit: degenerate lens layout");
        for (int k = 0; k < 5; ++k) std::swap(M[c][k], M[pr][k]);
        for (int r = 0; r < 4; ++r) {
            if (r == c) continue;
            const double f = M[r][c] / M[c][c];
            for (int k = c; k < 5; ++k) M[r][k] -= f * M[c][k];
        }
    }
    const double ox = M[0][4] / M[0][0], oy = M[1][4] / M[1][1], a = M[2][4] / M[2][2], b = M[3][4] / M[3][3];
    double ss = 0.0;
    const double h3 = 0.86602540378443864676;
    for (const pfd_mla_lens& L : use) {
        const double u = L.col + ((L.row & 1) ? 0.5 : 0.0), w = L.row * h3;
        const double ex = ox + u * a - w * b - L.cx, ey = oy + u * b + w * a - L.cy;
        ss += ex * ex + ey * ey;
    }
    fit[0] = ox;
    fit[1] = oy;
    fit[2] = std::sqrt(a * a + b * b);
    fit[3] = std::atan2(b, a);
    fit[4] = std::sqrt(ss / (double)use.size());
    fit[5] = (double)use.size();
    return PFD_OK;
}

pfd_status pfd_download_async(pfd_ctx* ctx, int frame_id, float* plane, float* cost, float* disp, uint32_t* sel)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    if (!f->has_state) return fail(ctx, PFD_ESTATE, "download before PatchMatch");
    DeviceGuard g(ctx->device);
    const size_t px = (size_t)f->V * f->mi_w * f->mi_h;
    const pfd::StateDev& s = f->s[f->cur];
    if (plane) CU(cudaMemcpyAsync(plane, s.plane, sizeof(float4) * px, cudaMemcpyDeviceToHost, ctx->stream));
    if (cost) CU(cudaMemcpyAsync(cost, s.cost, sizeof(float) * px, cudaMemcpyDeviceToHost, ctx->stream));
    if (disp) CU(cudaMemcpyAsync(disp, s.disp, sizeof(float4) * px, cudaMemcpyDeviceToHost, ctx->stream));
    if (sel) CU(cudaMemcpyAsync(sel, s.sel, sizeof(uint32_t) * px, cudaMemcpyDeviceToHost, ctx->stream));
    return PFD_OK;
}

size_t pfd_frame_bytes(int W, int H, int n_views, int mi_w, int mi_h, int max_nb, int has_blur)
{
    if (W < 1 || H < 1 || n_views < 1 || mi_w < 1 || mi_h < 1 || max_nb < 1) return 0;
    const size_t V = (size_t)n_views, px = V * mi_w * mi_h, tiles = V * (((size_t)mi_w * mi_h + 15) & ~(size_t)15);
    size_t b = (size_t)W * H + tiles * (has_blur ? 2 : 1) + 3 * sizeof(int2) * V + sizeof(int) * V * (max_nb + 1);
    b += sizeof(float) * px * max_nb;                              // stored cost vectors
    b += 2 * (sizeof(float4) + sizeof(float) + sizeof(float4) + sizeof(uint32_t)) * px;   // ping-pong state
    b += px + sizeof(int) * V;                                     // filter reasons and schedule
    return b;
}

pfd_status pfd_download(pfd_ctx* ctx, int frame_id, float* plane, float* cost, float* disp, uint32_t* sel)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    if (!f->has_state) return fail(ctx, PFD_ESTATE, "download before PatchMatch");
    DeviceGuard g(ctx->device);
    const size_t px = (size_t)f->V * f->mi_w * f->mi_h;
    const pfd::StateDev& s = f->s[f->cur];
    if (plane) CU(cudaMemcpyAsync(plane, s.plane, sizeof(float4) * px, cudaMemcpyDeviceToHost, ctx->stream));
    if (cost) CU(cudaMemcpyAsync(cost, s.cost, sizeof(float) * px, cudaMemcpyDeviceToHost, ctx->stream));
    if (disp) CU(cudaMemcpyAsync(disp, s.disp, sizeof(float4) * px, cudaMemcpyDeviceToHost, ctx->stream));
    if (sel) CU(cudaMemcpyAsync(sel, s.sel, sizeof(uint32_t) * px, cudaMemcpyDeviceToHost, ctx->stream));
    return check_device_error(ctx);
}

}  // extern "C"

// ---- PatchMatch sweep without allocation --------------------------------------
//
// pfd_pm_sweep takes its candidate-cost scratch from cudaMalloc, grown on the
// first sweep of a larger grid.  Some callers cannot allocate device memory
// once frames are streaming: an application whose memory pool claimed all free
// HBM at start-up (a cudaMalloc then fails, or takes memory the pool counts
// on), or a real-time camera loop that forbids cudaMalloc/cudaFree because they
// can synchronise the whole device and stall its other streams.
// pfd_pm_sweep_noalloc runs the same kernel on a fixed array that is part of
// the library's device image instead.

// 8 MiB, held by every GPU that loads the library until the process exits.
// Each warp of the sweep keeps the cost vectors of its current pixel here,
// (1.5 h max_nb + 3 h) words rounded up to 32 with h = max_nb + 6, seven warps
// per CTA; the array must hold at least one CTA per SM, which it does for every
// max_nb up to 32 on a 148-SM B200 (54.7 KB per CTA at 32 neighbours).  Nothing
// in it needs to start at zero: a sweep writes every entry it reads, earlier
// for the same pixel.
static __device__ __align__(256) float g_noalloc_scratch[(size_t(8) << 20) / sizeof(float)];

namespace {

constexpr size_t kNoAllocScratchBytes = sizeof(g_noalloc_scratch);

// Device address of g_noalloc_scratch on the current device.  In host code the
// array's name stands for a host-side shadow, so the kernel gets the address
// from cudaGetSymbolAddress.  It is looked up on every call (a host-side table
// lookup once the module is loaded): a cached address would outlive a
// cudaDeviceReset, after which the module is loaded again, possibly elsewhere.
pfd_status noalloc_scratch(pfd_ctx* ctx, float** out)
{
    float* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return fail(ctx, PFD_ECUDA, "pfd_pm_sweep_noalloc: cudaGetSymbolAddress of the scratch array: %s",
                    cudaGetErrorString(e));
    }
    *out = p;
    return PFD_OK;
}

}  // namespace

extern "C" pfd_status pfd_pm_sweep_noalloc(pfd_ctx* ctx, int frame_id, const pfd_pm_params* params, uint64_t seed,
                                           int iter, int phase)
{
    if (!ctx) return PFD_EINVAL;
    Frame* f = find_frame(ctx, frame_id);
    if (!f) return fail(ctx, PFD_ENOFRAME, "no frame %d", frame_id);
    pfd_status st = check_params(ctx, *f, params);
    if (st != PFD_OK) return st;
    if (!f->has_state) return fail(ctx, PFD_ESTATE, "sweep before pfd_pm_init");
    if (phase != 0 && phase != 1) return fail(ctx, PFD_EINVAL, "phase must be 0 or 1");
    if (iter < 0) return fail(ctx, PFD_EINVAL, "iter must be >= 0");
    DeviceGuard g(ctx->device);
    pfd::PmParams P = make_params(ctx, *f, params, seed);
    if (ctx->counting) P.tap_counter = ctx->d_taps;
    st = tex_refresh(ctx, *f, false);            // a launch, no allocation (textures only if the frame has them)
    if (st != PFD_OK) return st;
    const pfd::FrameDev F = sweep_dev(ctx, *f);
    if (pfd::sweep_warp_smem_bytes(P, f->has_blur, 0, F.tex != nullptr) > 227 * 1024)
        return fail(ctx, PFD_EINVAL, "window %dx%d with %d neighbours does not fit shared memory", f->mi_w, f->mi_h, f->K);
    int sms = 0;
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    const size_t per_cta = pfd::sweep_warp_scratch_bytes(P, 1);
    const size_t fit = kNoAllocScratchBytes / per_cta;
    if (fit < (size_t)sms) {
        int kmax = 0;                            // largest max_nb whose CTAs still cover every SM
        for (int k = 1; k <= pfd::kMaxNb; ++k) {
            pfd::PmParams Q = P;
            Q.K = k;
            if (kNoAllocScratchBytes / pfd::sweep_warp_scratch_bytes(Q, 1) >= (size_t)sms) kmax = k;
        }
        return fail(ctx, PFD_EINVAL,
                    "pfd_pm_sweep_noalloc: %d neighbours need %zu bytes of scratch per CTA; the fixed %zu-byte "
                    "scratch holds %zu CTAs, fewer than the %d SMs (at most %d neighbours on this device)",
                    f->K, per_cta, kNoAllocScratchBytes, fit, sms, kmax);
    }
    int n_ctas = 0;
    CU(pfd::sweep_warp_grid(F, P, &n_ctas));
    n_ctas = (int)std::min<size_t>((size_t)n_ctas, fit);
    float* scratch = nullptr;
    st = noalloc_scratch(ctx, &scratch);
    if (st != PFD_OK) return st;
    P.cost_scratch = scratch;
    P.scratch_floats = kNoAllocScratchBytes / sizeof(float);
    P.cvec_ok = !ctx->counting && cvec_usable(*f, *params, phase, cost_mode(ctx));
    CU(pfd::launch_sweep_warp(F, P, f->s[f->cur], f->s[f->cur ^ 1], iter, phase, n_ctas, ctx->d_err,
                              ctx->stream));
    ctx->launches += 1;
    f->cur ^= 1;
    if (ctx->counting) f->cvec_valid = 0;        // tap counting evaluates everything and stores nothing
    else cvec_swept(*f, *params, phase, cost_mode(ctx));
    return PFD_OK;
}
