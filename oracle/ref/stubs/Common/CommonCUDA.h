/*
 * Stand-in for the reference's Common/CommonCUDA.h (see Common.h of this
 * directory): the CUDA headers, cudaTextureObjects (CommonCUDA.h:62-66, same
 * members) and CUDA_SAFE_CALL, which here records the first failure for the
 * harness to report instead of exiting the process (the reference's
 * CudaSafeCall exits, Common/CommonCUDA.cpp:77-86).
 *
 * Random numbers.  The reference seeds cuRAND XORWOW from clock64()
 * (AdaptMIPMFrame.cu:501), so no two of its runs agree.  Two builds fix that:
 *  - default: cuRAND XORWOW as the reference uses it, with clock64() replaced
 *    by the harness's seed (every thread gets the same seed and its own
 *    subsequence, the standard cuRAND use).  This is the timed plain method.
 *  - PFD_REF_RNG_PHILOX: curandState, curand_init and curand_uniform are
 *    replaced by the engine's Philox4x32-10 draw streams (Salmon et al.,
 *    SC'11): draw n of pixel idx in sweep s is word n & 3 of the block with
 *    counter (n >> 2, s, idx, 0) under key (seed_lo, seed_hi), as uniform
 *    ((u >> 8) + 1) 2^-24.  The reference's kernels then draw exactly the
 *    numbers the engine and the CPU oracle draw, in the reference's own
 *    order, so the three can be compared on one trajectory.  The harness sets
 *    the sweep id (0 initialisation, 1 + 2 iter + phase a half-sweep) before
 *    each launch; a state whose stored sweep differs restarts its stream.
 */
#ifndef PFD_REF_STUB_COMMONCUDA_H
#define PFD_REF_STUB_COMMONCUDA_H

#include <cuda_runtime.h>
#include <cuda_texture_types.h>
#include <vector_types.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "Common/Common.h"

/* Seed of both builds; set by the harness with cudaMemcpyToSymbol. */
extern __device__ unsigned long long pfdref_seed;

#ifdef PFD_REF_RNG_PHILOX
extern __device__ unsigned int pfdref_sweep_id;
struct pfdref_rng_state;
extern __device__ pfdref_rng_state* pfdref_states;

struct pfdref_rng_state {
    unsigned int sweep, pixel, n, block;
    uint4 buf;
};
typedef pfdref_rng_state curandState;

static __device__ __forceinline__ uint4 pfdref_philox4x32_10(uint4 c, uint2 k)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const unsigned int lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const unsigned int lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

/* The reference's arguments (seed, subsequence, offset) are not used: the
 * stream is keyed by the harness's seed and the state's own pixel index. */
static __device__ __forceinline__ void curand_init(unsigned long long, unsigned long long, unsigned long long,
                                                   curandState* st)
{
    st->pixel = (unsigned int)(st - pfdref_states);
    st->sweep = pfdref_sweep_id;
    st->n = 0;
    st->block = 0xffffffffu;
}

static __device__ __forceinline__ float curand_uniform(curandState* st)
{
    if (st->sweep != pfdref_sweep_id) {
        st->sweep = pfdref_sweep_id;
        st->n = 0;
        st->block = 0xffffffffu;
    }
    const unsigned int b = st->n >> 2;
    if (b != st->block) {
        const unsigned long long s = pfdref_seed;
        st->buf = pfdref_philox4x32_10(make_uint4(b, st->sweep, st->pixel, 0u),
                                       make_uint2((unsigned int)s, (unsigned int)(s >> 32)));
        st->block = b;
    }
    const unsigned int w = st->n & 3u;
    st->n++;
    const unsigned int u = w == 0 ? st->buf.x : (w == 1 ? st->buf.y : (w == 2 ? st->buf.z : st->buf.w));
    return __fmul_rn((float)((u >> 8) + 1u), 0x1p-24f);
}
#else
#include <curand_kernel.h>
#endif

/* clock64() seeds the reference's cuRAND states; both builds read the
 * harness's seed instead.  Defined after the CUDA headers, which declare the
 * real clock64. */
#define clock64() ((long long int)pfdref_seed)

namespace LFMVS {

void pfdref_note_cuda_error(cudaError_t e, const char* file, int line);
#define CUDA_SAFE_CALL(error) LFMVS::pfdref_note_cuda_error((error), __FILE__, __LINE__)
#define CUDA_CHECK_ERROR() LFMVS::pfdref_note_cuda_error(cudaGetLastError(), __FILE__, __LINE__)

struct cudaTextureObjects {
    cudaTextureObject_t images[MAX_IMAGES];
    cudaTextureObject_t blur_images[MAX_IMAGES];
};

}  // namespace LFMVS

#endif
