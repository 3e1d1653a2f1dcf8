/*
 * ref_frame_harness.cu -- TEST ORACLE, not product code.
 *
 * Compiles the reference's own frame PatchMatch kernels from their source
 * with the reference's flags (-O3 --use_fast_math --maxrregcount=128,
 * CMakeLists.txt:52) for sm_100a and drives them through a small C API.  The
 * translation units are the reference's: MIStereo/CudaUtil.cu, which includes
 * MIStereo/AdaptMIPMFrame.cu at its end (CudaUtil.cu:1047), is included below
 * from the reference tree, so the frame kernels' static helpers are callable
 * here; MIStereo/AdaptMIPMUtil.cu is a separate object linked with
 * separable compilation, as CUDA_SEPARABLE_COMPILATION does in the
 * reference's build (CMakeLists.txt:27, :112-115).
 *   - pfdref_ncc_costs: ComputeMultiViewCostVector_Frame (AdaptMIPMFrame.cu:
 *     181-225) on given (view, pixel, plane) hypotheses, one thread each;
 *   - pfdref_patchmatch: the reference's RunPatchMatchCUDAForFrame_Impl
 *     (AdaptMIPMFrame.cu:949-995) unchanged (16x16 blocks, grid.z = views, a
 *     device synchronisation after every launch), timed with CUDA events;
 *   - pfdref_init / pfdref_sweep: the same two kernels launched one at a time
 *     with that structure, so a half-sweep can start from a given state.
 * The micro-images are bound to float textures exactly as
 * AdaptMIPMFrame::CreateGrayImageObject / CreateBlurImageObject do
 * (AdaptMIPMFrame.cpp:224-276: one cudaArray per view, linear filtering,
 * wrap addressing, unnormalised coordinates).  Without a blur channel every
 * view's blur texture is one shared all-zero array, which gives the blur
 * penalty 0 (the reference's active pipeline never computes the channel,
 * DepthSolver.cpp:2763-2774).
 *
 * Only tests/ and bench.py's baseline legs load the library this builds
 * (oracle/_ref/libref_frame*.so); the engine never does.
 */
#include "MIStereo/CudaUtil.cu"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

__device__ unsigned long long pfdref_seed;
#ifdef PFD_REF_RNG_PHILOX
__device__ unsigned int pfdref_sweep_id;
__device__ pfdref_rng_state* pfdref_states;
#endif

namespace {
cudaError_t g_first_error = cudaSuccess;
std::string g_error_text;

void note(const std::string& what)
{
    if (g_error_text.empty()) g_error_text = what;
}
}  // namespace

namespace LFMVS {

void pfdref_note_cuda_error(cudaError_t e, const char* file, int line)
{
    if (e != cudaSuccess && g_first_error == cudaSuccess) {
        g_first_error = e;
        char buf[512];
        snprintf(buf, sizeof buf, "%s:%d: %s", file, line, cudaGetErrorString(e));
        note(buf);
    }
}

/* One thread per hypothesis: the reference's cost vector of that hypothesis. */
__global__ void pfdref_ncc_kernel(const cudaTextureObjects* tex, const float2* centers, const int2* tilekeys,
                                  const int* nb_ids, const int* nb_counts, int max_nb, PatchMatchParamsLF params,
                                  const int* vids, const int2* pxy, const float4* planes, int n, float* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float cost[32];
    float2 blur[32];
    float4 disp[32];
    ComputeMultiViewCostVector_Frame(tex, centers, tilekeys, nb_ids, nb_counts, max_nb, params, vids[i], pxy[i],
                                     planes[i], cost, blur, disp);
    for (int k = 0; k < max_nb; ++k) out[(size_t)i * max_nb + k] = cost[k];
}

#ifndef PFD_REF_RNG_PHILOX
/* The reference seeds its states only inside RandomInitializationForFrame;
 * a half-sweep from an uploaded state needs them seeded the same way
 * (AdaptMIPMFrame.cu:498-501). */
__global__ void pfdref_seed_states(curandState* st, int num_views, int ppv)
{
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)num_views * ppv) return;
    const unsigned long long vid = idx / ppv;
    curand_init(clock64(), vid * (unsigned long long)ppv + idx, 0, &st[idx]);
}
#else
__global__ void pfdref_seed_states(curandState* st, int num_views, int ppv)
{
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)num_views * ppv) return;
    curand_init(0, 0, 0, &st[idx]);
}
#endif

}  // namespace LFMVS

using namespace LFMVS;

struct pfdref_params {
    int max_iterations, patch_size, radius_increment, top_k;
    float sigma_spatial, sigma_color, depth_min, depth_max, base;
};

struct pfdref_frame {
    int V = 0, mi = 0, max_nb = 0;
    std::vector<cudaArray_t> arrays;
    cudaTextureObjects* tex_host = nullptr;
    cudaTextureObjects* tex_dev = nullptr;
    float2* centers = nullptr;
    int2* tilekeys = nullptr;
    int* nb_ids = nullptr;
    int* nb_counts = nullptr;
    float4* plane[2] = {nullptr, nullptr};
    float* cost[2] = {nullptr, nullptr};
    float4* disp[2] = {nullptr, nullptr};
    unsigned int* sel[2] = {nullptr, nullptr};
    curandState* states = nullptr;
    int cur = 0;   /* buffer holding the current state */
    bool seeded = false;
};

namespace {

bool ok(cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return true;
    if (g_first_error == cudaSuccess) g_first_error = e;
    note(std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

/* AdaptMIPMFrame::InitGPUParamsFromCPUParams (AdaptMIPMFrame.cpp:126-143)
 * with the caller's matching parameters in place of its defaults. */
PatchMatchParamsLF to_lf(const pfdref_params* p, int mi, int max_nb)
{
    PatchMatchParamsLF q;
    q.max_iterations = p->max_iterations;
    q.patch_size = p->patch_size;
    q.patch_Bound_size = 5;
    q.propagation_Graph_size = 5;
    q.num_images = max_nb + 1;
    q.radius_increment = p->radius_increment;
    q.sigma_spatial = p->sigma_spatial;
    q.sigma_color = p->sigma_color;
    q.top_k = p->top_k;
    q.depth_min = p->depth_min;
    q.depth_max = p->depth_max;
    q.disparity_min = p->depth_min;
    q.disparity_max = p->depth_max;
    q.Base = p->base;
    q.MLA_Mask_Width_Cuda = mi;
    q.MLA_Mask_Height_Cuda = mi;
    q.base_height_ratio = 0.2f;
    q.base_height_sigma = 0.05f;
    return q;
}

cudaTextureObject_t make_texture(cudaArray_t arr)
{
    cudaResourceDesc res;
    memset(&res, 0, sizeof res);
    res.resType = cudaResourceTypeArray;
    res.res.array.array = arr;
    cudaTextureDesc td;
    memset(&td, 0, sizeof td);
    td.addressMode[0] = cudaAddressModeWrap;
    td.addressMode[1] = cudaAddressModeWrap;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    cudaTextureObject_t t = 0;
    ok(cudaCreateTextureObject(&t, &res, &td, nullptr), "cudaCreateTextureObject");
    return t;
}

cudaArray_t make_array(const float* host, int mi)
{
    cudaChannelFormatDesc cd = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
    cudaArray_t a = nullptr;
    if (!ok(cudaMallocArray(&a, &cd, mi, mi), "cudaMallocArray")) return nullptr;
    ok(cudaMemcpy2DToArray(a, 0, 0, host, mi * sizeof(float), mi * sizeof(float), mi, cudaMemcpyHostToDevice),
       "cudaMemcpy2DToArray");
    return a;
}

dim3 grid_of(const pfdref_frame* f)
{
    return dim3((f->mi + 15) / 16, (f->mi + 15) / 16, f->V);
}

bool set_seed(uint64_t seed)
{
    unsigned long long s = seed;
    return ok(cudaMemcpyToSymbol(pfdref_seed, &s, sizeof s), "seed");
}

#ifdef PFD_REF_RNG_PHILOX
bool set_sweep(unsigned int sweep)
{
    return ok(cudaMemcpyToSymbol(pfdref_sweep_id, &sweep, sizeof sweep), "sweep id");
}
#endif

}  // namespace

extern "C" {

const char* pfdref_last_error(void) { return g_error_text.c_str(); }

int pfdref_rng_is_philox(void)
{
#ifdef PFD_REF_RNG_PHILOX
    return 1;
#else
    return 0;
#endif
}

void pfdref_frame_destroy(pfdref_frame* f)
{
    if (!f) return;
    cudaDeviceSynchronize();
    if (f->tex_host) {
        for (int v = 0; v < f->V; ++v) {
            if (f->tex_host->images[v]) cudaDestroyTextureObject(f->tex_host->images[v]);
            if (f->tex_host->blur_images[v]) cudaDestroyTextureObject(f->tex_host->blur_images[v]);
        }
    }
    for (cudaArray_t a : f->arrays) cudaFreeArray(a);
    cudaFree(f->tex_dev);
    cudaFree(f->centers);
    cudaFree(f->tilekeys);
    cudaFree(f->nb_ids);
    cudaFree(f->nb_counts);
    for (int b = 0; b < 2; ++b) {
        cudaFree(f->plane[b]);
        cudaFree(f->cost[b]);
        cudaFree(f->disp[b]);
        cudaFree(f->sel[b]);
    }
    cudaFree(f->states);
    delete f->tex_host;
    delete f;
}

/* gray, blur: [V][mi][mi] 8-bit (blur may be NULL); centers [V][2];
 * tilekeys [V][2]; nb_ids [V][max_nb] (-1 padded); nb_counts [V]. */
int pfdref_frame_create(pfdref_frame** out, int V, int mi, const uint8_t* gray, const uint8_t* blur,
                        const float* centers, const int* tilekeys, const int* nb_ids, const int* nb_counts,
                        int max_nb)
{
    *out = nullptr;
    g_error_text.clear();
    g_first_error = cudaSuccess;
    if (V <= 0 || V > MAX_IMAGES || mi <= 0 || mi > 64 || max_nb <= 0 || max_nb > 32 || !gray) {
        note("pfdref_frame_create: bad sizes");
        return -1;
    }
    pfdref_frame* f = new pfdref_frame;
    f->V = V;
    f->mi = mi;
    f->max_nb = max_nb;
    f->tex_host = new cudaTextureObjects;
    memset(f->tex_host, 0, sizeof(cudaTextureObjects));
    const int ppv = mi * mi;
    std::vector<float> tile(ppv, 0.0f);
    cudaArray_t zero = nullptr;
    if (!blur) {
        zero = make_array(tile.data(), mi);
        f->arrays.push_back(zero);
    }
    for (int v = 0; v < V && g_first_error == cudaSuccess; ++v) {
        for (int i = 0; i < ppv; ++i) tile[i] = (float)gray[(size_t)v * ppv + i];
        cudaArray_t a = make_array(tile.data(), mi);
        f->arrays.push_back(a);
        f->tex_host->images[v] = make_texture(a);
        if (blur) {
            for (int i = 0; i < ppv; ++i) tile[i] = (float)blur[(size_t)v * ppv + i];
            cudaArray_t b = make_array(tile.data(), mi);
            f->arrays.push_back(b);
            f->tex_host->blur_images[v] = make_texture(b);
        } else {
            f->tex_host->blur_images[v] = make_texture(zero);
        }
    }
    const size_t px = (size_t)V * ppv;
    bool good = g_first_error == cudaSuccess;
    good = good && ok(cudaMalloc(&f->tex_dev, sizeof(cudaTextureObjects)), "cudaMalloc");
    good = good && ok(cudaMemcpy(f->tex_dev, f->tex_host, sizeof(cudaTextureObjects), cudaMemcpyHostToDevice), "copy");
    good = good && ok(cudaMalloc(&f->centers, sizeof(float2) * V), "cudaMalloc");
    good = good && ok(cudaMemcpy(f->centers, centers, sizeof(float2) * V, cudaMemcpyHostToDevice), "copy");
    good = good && ok(cudaMalloc(&f->tilekeys, sizeof(int2) * V), "cudaMalloc");
    good = good && ok(cudaMemcpy(f->tilekeys, tilekeys, sizeof(int2) * V, cudaMemcpyHostToDevice), "copy");
    good = good && ok(cudaMalloc(&f->nb_ids, sizeof(int) * V * max_nb), "cudaMalloc");
    good = good && ok(cudaMemcpy(f->nb_ids, nb_ids, sizeof(int) * V * max_nb, cudaMemcpyHostToDevice), "copy");
    good = good && ok(cudaMalloc(&f->nb_counts, sizeof(int) * V), "cudaMalloc");
    good = good && ok(cudaMemcpy(f->nb_counts, nb_counts, sizeof(int) * V, cudaMemcpyHostToDevice), "copy");
    for (int b = 0; b < 2 && good; ++b) {
        good = good && ok(cudaMalloc(&f->plane[b], sizeof(float4) * px), "cudaMalloc");
        good = good && ok(cudaMalloc(&f->cost[b], sizeof(float) * px), "cudaMalloc");
        good = good && ok(cudaMalloc(&f->disp[b], sizeof(float4) * px), "cudaMalloc");
        good = good && ok(cudaMalloc(&f->sel[b], sizeof(unsigned int) * px), "cudaMalloc");
    }
    good = good && ok(cudaMalloc(&f->states, sizeof(curandState) * px), "cudaMalloc");
#ifdef PFD_REF_RNG_PHILOX
    good = good && ok(cudaMemcpyToSymbol(pfdref_states, &f->states, sizeof(f->states)), "states");
#endif
    if (!good) {
        pfdref_frame_destroy(f);
        return -3;
    }
    *out = f;
    return 0;
}

/* vids [n], pxy [n][2], planes [n][4] -> costs [n][max_nb]. */
int pfdref_ncc_costs(pfdref_frame* f, const pfdref_params* p, const int* vids, const int* pxy, const float* planes,
                     int n, float* costs)
{
    if (!f || n < 0) return -1;
    if (n == 0) return 0;
    int* dv = nullptr;
    int2* dp = nullptr;
    float4* dpl = nullptr;
    float* dout = nullptr;
    bool good = ok(cudaMalloc(&dv, sizeof(int) * n), "cudaMalloc") && ok(cudaMalloc(&dp, sizeof(int2) * n), "cudaMalloc") &&
                ok(cudaMalloc(&dpl, sizeof(float4) * n), "cudaMalloc") &&
                ok(cudaMalloc(&dout, sizeof(float) * (size_t)n * f->max_nb), "cudaMalloc");
    good = good && ok(cudaMemcpy(dv, vids, sizeof(int) * n, cudaMemcpyHostToDevice), "copy") &&
           ok(cudaMemcpy(dp, pxy, sizeof(int2) * n, cudaMemcpyHostToDevice), "copy") &&
           ok(cudaMemcpy(dpl, planes, sizeof(float4) * n, cudaMemcpyHostToDevice), "copy");
    if (good) {
        pfdref_ncc_kernel<<<(n + 127) / 128, 128>>>(f->tex_dev, f->centers, f->tilekeys, f->nb_ids, f->nb_counts,
                                                    f->max_nb, to_lf(p, f->mi, f->max_nb), dv, dp, dpl, n, dout);
        good = ok(cudaGetLastError(), "pfdref_ncc_kernel launch") && ok(cudaDeviceSynchronize(), "pfdref_ncc_kernel");
        good = good && ok(cudaMemcpy(costs, dout, sizeof(float) * (size_t)n * f->max_nb, cudaMemcpyDeviceToHost), "copy");
    }
    cudaFree(dv);
    cudaFree(dp);
    cudaFree(dpl);
    cudaFree(dout);
    return good ? 0 : -3;
}

/* The reference's whole run: RunPatchMatchCUDAForFrame_Impl unchanged (the
 * Philox build launches the same kernels with the same structure one by one,
 * setting each launch's sweep id).  ms[0] receives the device time of the
 * initialisation, ms[1] of the half-sweeps (CUDA events on the default
 * stream; the reference synchronises after every launch).  May be NULL. */
int pfdref_patchmatch(pfdref_frame* f, const pfdref_params* p, uint64_t seed, float* ms)
{
    if (!f) return -1;
    g_first_error = cudaSuccess;
    g_error_text.clear();
    PatchMatchParamsLF q = to_lf(p, f->mi, f->max_nb);
    if (!set_seed(seed)) return -3;
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    const dim3 block(16, 16, 1), grid = grid_of(f);
    cudaEventRecord(e0, 0);
#ifdef PFD_REF_RNG_PHILOX
    set_sweep(0);
    RandomInitializationForFrame<<<grid, block>>>(f->tex_dev, f->centers, f->tilekeys, f->nb_ids, f->nb_counts,
                                                  f->max_nb, f->plane[0], f->cost[0], f->disp[0], f->sel[0],
                                                  f->states, q, f->mi, f->mi, f->V);
    CUDA_SAFE_CALL(cudaDeviceSynchronize());
    cudaEventRecord(e1, 0);
    int cur = 0;
    for (int it = 0; it < q.max_iterations; ++it) {
        for (int ph = 0; ph < 2; ++ph) {
            set_sweep(1u + 2u * it + ph);
            CheckerboardUpdateFrame<<<grid, block>>>(f->tex_dev, f->centers, f->tilekeys, f->nb_ids, f->nb_counts,
                                                     f->max_nb, f->plane[cur], f->cost[cur], f->disp[cur], f->sel[cur],
                                                     f->plane[cur ^ 1], f->cost[cur ^ 1], f->disp[cur ^ 1],
                                                     f->sel[cur ^ 1], f->states, q, f->mi, f->mi, f->V, it, ph);
            CUDA_SAFE_CALL(cudaDeviceSynchronize());
            cur ^= 1;
        }
    }
    f->cur = cur;
#else
    /* The initialisation alone first, for its time, then the whole method. */
    RandomInitializationForFrame<<<grid, block>>>(f->tex_dev, f->centers, f->tilekeys, f->nb_ids, f->nb_counts,
                                                  f->max_nb, f->plane[0], f->cost[0], f->disp[0], f->sel[0],
                                                  f->states, q, f->mi, f->mi, f->V);
    CUDA_SAFE_CALL(cudaDeviceSynchronize());
    cudaEventRecord(e1, 0);
    {
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, 0);
        RunPatchMatchCUDAForFrame_Impl(f->tex_dev, f->centers, f->tilekeys, f->nb_ids, f->nb_counts, f->plane[0],
                                       f->plane[1], f->cost[0], f->cost[1], f->disp[0], f->disp[1], f->sel[0],
                                       f->sel[1], f->states, q, f->V, f->max_nb);
        cudaEventRecord(b, 0);
        cudaEventSynchronize(b);
        float whole = 0.0f, init = 0.0f;
        cudaEventElapsedTime(&whole, a, b);
        cudaEventElapsedTime(&init, e0, e1);
        if (ms) {
            ms[0] = init;
            ms[1] = whole - init;
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    f->cur = 0;   /* an even number of swaps leaves the result in buffer 0 */
#endif
    cudaEventRecord(e2, 0);
    cudaEventSynchronize(e2);
#ifdef PFD_REF_RNG_PHILOX
    if (ms) {
        cudaEventElapsedTime(&ms[0], e0, e1);
        cudaEventElapsedTime(&ms[1], e1, e2);
    }
#endif
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    f->seeded = true;
    ok(cudaGetLastError(), "launch");
    return g_first_error == cudaSuccess ? 0 : -3;
}

/* A bounded sample of the reference's whole run: RunPatchMatchCUDAForFrame_Impl
 * launched with num_views = n, so its kernels update views [0, n) only (the
 * caller puts the sampled block of views first).  Every view is initialised
 * first, untimed, and both state buffers get that state, so the views past n
 * that the sample's proposals read hold a valid (initial) plane throughout.
 * ms[0] receives the device time of the sample's initialisation, ms[1] of its
 * half-sweeps (CUDA events on the default stream). */
int pfdref_patchmatch_sample(pfdref_frame* f, const pfdref_params* p, uint64_t seed, int n, float* ms)
{
    if (!f || n < 1 || n > f->V) return -1;
    g_first_error = cudaSuccess;
    g_error_text.clear();
    PatchMatchParamsLF q = to_lf(p, f->mi, f->max_nb);
    if (!set_seed(seed)) return -3;
#ifdef PFD_REF_RNG_PHILOX
    set_sweep(0);
#endif
    const dim3 block(16, 16, 1), grid = grid_of(f);
    RandomInitializationForFrame<<<grid, block>>>(f->tex_dev, f->centers, f->tilekeys, f->nb_ids, f->nb_counts,
                                                  f->max_nb, f->plane[0], f->cost[0], f->disp[0], f->sel[0],
                                                  f->states, q, f->mi, f->mi, f->V);
    CUDA_SAFE_CALL(cudaDeviceSynchronize());
    const size_t px = (size_t)f->V * f->mi * f->mi;
    ok(cudaMemcpy(f->plane[1], f->plane[0], sizeof(float4) * px, cudaMemcpyDeviceToDevice), "copy");
    ok(cudaMemcpy(f->cost[1], f->cost[0], sizeof(float) * px, cudaMemcpyDeviceToDevice), "copy");
    ok(cudaMemcpy(f->disp[1], f->disp[0], sizeof(float4) * px, cudaMemcpyDeviceToDevice), "copy");
    ok(cudaMemcpy(f->sel[1], f->sel[0], sizeof(unsigned int) * px, cudaMemcpyDeviceToDevice), "copy");
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    const dim3 sgrid((f->mi + 15) / 16, (f->mi + 15) / 16, n);
    cudaEventRecord(e0, 0);
    RandomInitializationForFrame<<<sgrid, block>>>(f->tex_dev, f->centers, f->tilekeys, f->nb_ids, f->nb_counts,
                                                   f->max_nb, f->plane[0], f->cost[0], f->disp[0], f->sel[0],
                                                   f->states, q, f->mi, f->mi, n);
    CUDA_SAFE_CALL(cudaDeviceSynchronize());
    cudaEventRecord(e1, 0);
    RunPatchMatchCUDAForFrame_Impl(f->tex_dev, f->centers, f->tilekeys, f->nb_ids, f->nb_counts, f->plane[0],
                                   f->plane[1], f->cost[0], f->cost[1], f->disp[0], f->disp[1], f->sel[0], f->sel[1],
                                   f->states, q, n, f->max_nb);
    cudaEventRecord(e2, 0);
    cudaEventSynchronize(e2);
    float init = 0.0f, whole = 0.0f;
    cudaEventElapsedTime(&init, e0, e1);
    cudaEventElapsedTime(&whole, e1, e2);
    if (ms) {
        ms[0] = init;
        ms[1] = whole - init;   /* the Impl initialises the sample again before its sweeps */
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    f->cur = 0;
    f->seeded = true;
    ok(cudaGetLastError(), "launch");
    return g_first_error == cudaSuccess ? 0 : -3;
}

/* RandomInitializationForFrame alone (AdaptMIPMFrame.cu:474-518). */
int pfdref_init(pfdref_frame* f, const pfdref_params* p, uint64_t seed)
{
    if (!f) return -1;
    g_first_error = cudaSuccess;
    g_error_text.clear();
    if (!set_seed(seed)) return -3;
#ifdef PFD_REF_RNG_PHILOX
    set_sweep(0);
#endif
    RandomInitializationForFrame<<<grid_of(f), dim3(16, 16, 1)>>>(f->tex_dev, f->centers, f->tilekeys, f->nb_ids,
                                                                 f->nb_counts, f->max_nb, f->plane[0], f->cost[0],
                                                                 f->disp[0], f->sel[0], f->states,
                                                                 to_lf(p, f->mi, f->max_nb), f->mi, f->mi, f->V);
    CUDA_SAFE_CALL(cudaDeviceSynchronize());
    ok(cudaGetLastError(), "launch");
    f->cur = 0;
    f->seeded = true;
    return g_first_error == cudaSuccess ? 0 : -3;
}

/* One CheckerboardUpdateFrame launch (AdaptMIPMFrame.cu:520-947) from the
 * current state.  A state set by pfdref_state_upload gets its random states
 * seeded first, as RandomInitializationForFrame seeds them. */
int pfdref_sweep(pfdref_frame* f, const pfdref_params* p, uint64_t seed, int iter, int phase)
{
    if (!f || (phase != 0 && phase != 1) || iter < 0) return -1;
    g_first_error = cudaSuccess;
    g_error_text.clear();
    if (!set_seed(seed)) return -3;
    const size_t px = (size_t)f->V * f->mi * f->mi;
    if (!f->seeded) {
        pfdref_seed_states<<<(unsigned)((px + 255) / 256), 256>>>(f->states, f->V, f->mi * f->mi);
        CUDA_SAFE_CALL(cudaDeviceSynchronize());
        f->seeded = true;
    }
#ifdef PFD_REF_RNG_PHILOX
    set_sweep(1u + 2u * iter + phase);
#endif
    const int c = f->cur;
    CheckerboardUpdateFrame<<<grid_of(f), dim3(16, 16, 1)>>>(
        f->tex_dev, f->centers, f->tilekeys, f->nb_ids, f->nb_counts, f->max_nb, f->plane[c], f->cost[c], f->disp[c],
        f->sel[c], f->plane[c ^ 1], f->cost[c ^ 1], f->disp[c ^ 1], f->sel[c ^ 1], f->states,
        to_lf(p, f->mi, f->max_nb), f->mi, f->mi, f->V, iter, phase);
    CUDA_SAFE_CALL(cudaDeviceSynchronize());
    ok(cudaGetLastError(), "launch");
    f->cur = c ^ 1;
    return g_first_error == cudaSuccess ? 0 : -3;
}

/* Host arrays [V*mi*mi] (plane, disp: [.][4]); any may be NULL on download. */
int pfdref_download(pfdref_frame* f, float* plane, float* cost, float* disp, uint32_t* sel)
{
    if (!f) return -1;
    const size_t px = (size_t)f->V * f->mi * f->mi;
    const int c = f->cur;
    bool good = true;
    if (plane) good = good && ok(cudaMemcpy(plane, f->plane[c], sizeof(float4) * px, cudaMemcpyDeviceToHost), "copy");
    if (cost) good = good && ok(cudaMemcpy(cost, f->cost[c], sizeof(float) * px, cudaMemcpyDeviceToHost), "copy");
    if (disp) good = good && ok(cudaMemcpy(disp, f->disp[c], sizeof(float4) * px, cudaMemcpyDeviceToHost), "copy");
    if (sel) good = good && ok(cudaMemcpy(sel, f->sel[c], sizeof(unsigned int) * px, cudaMemcpyDeviceToHost), "copy");
    return good ? 0 : -3;
}

/* Makes host arrays the current state (all four required).  The random
 * states are seeded afresh before the next half-sweep. */
int pfdref_state_upload(pfdref_frame* f, const float* plane, const float* cost, const float* disp,
                        const uint32_t* sel)
{
    if (!f || !plane || !cost || !disp || !sel) return -1;
    const size_t px = (size_t)f->V * f->mi * f->mi;
    const int c = f->cur;
    bool good = ok(cudaMemcpy(f->plane[c], plane, sizeof(float4) * px, cudaMemcpyHostToDevice), "copy") &&
                ok(cudaMemcpy(f->cost[c], cost, sizeof(float) * px, cudaMemcpyHostToDevice), "copy") &&
                ok(cudaMemcpy(f->disp[c], disp, sizeof(float4) * px, cudaMemcpyHostToDevice), "copy") &&
                ok(cudaMemcpy(f->sel[c], sel, sizeof(unsigned int) * px, cudaMemcpyHostToDevice), "copy");
    f->seeded = false;
    return good ? 0 : -3;
}

}  // extern "C"
