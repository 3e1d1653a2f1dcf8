/*
 * oracle/canon.h -- canonical scalar arithmetic of the plenoptic PatchMatch path,
 * CPU side.  TEST INFRASTRUCTURE ONLY: this file belongs to the oracle and is
 * never linked into the product library.
 *
 * The reference kernels (MIStereo/AdaptMIPMFrame.cu, MIStereo/CudaUtil.cu,
 * MIStereo/AdaptMIPMUtil.cu) are compiled with --use_fast_math and nvcc's
 * default FMA contraction, and seed cuRAND from clock64(), so their exact bits
 * are not reproducible even run to run.  The oracle therefore fixes ONE
 * arithmetic for every step of the algorithm and the CUDA kernels implement
 * the same arithmetic, so that oracle and GPU agree bit for bit:
 *
 *  - every product that feeds a sum is fused (fmaf), evaluated left to right:
 *    a*b + c*d + e  ==  fmaf(c, d, a*b) + e   (the first product is rounded);
 *    a - b*c        ==  fmaf(-b, c, a).
 *  - divisions and square roots are IEEE (correctly rounded).
 *  - exp is canon_expf below (Cody-Waite reduction + degree-7 Taylor
 *    polynomial, all fmaf), not libm's and not CUDA's.
 *  - random numbers come from Philox4x32-10 (Salmon, Moraes, Dror, Shaw,
 *    "Parallel random numbers: as easy as 1, 2, 3", SC'11), a counter-based
 *    generator, instead of cuRAND XORWOW seeded from clock64().
 *
 * Compile with -ffp-contract=off so that the compiler fuses nothing by itself.
 */
#ifndef PFD_ORACLE_CANON_H
#define PFD_ORACLE_CANON_H

#include <math.h>
#include <stdint.h>
#include <string.h>

static inline float canon_bits_to_float(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline uint32_t canon_float_to_bits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

/* 1.5 * 2^23: adding it to |x| < 2^22 rounds x to the nearest integer (ties to even). */
#define CANON_RNE_MAGIC 12582912.0f

/* exp(x) in float.  Cody-Waite: x = k*ln2 + r with ln2 split in a high part whose
 * low 12 bits are zero (so k*ln2_hi is exact for |k| <= 2^12) and a low part;
 * e^r by the Taylor series to r^7 (|r| <= ln2/2 gives a truncation error below
 * 2^-26 relative); 2^k applied in two exact power-of-two multiplications so that
 * results in the subnormal range round once.  Error <= 2 ulp over [-104, 88.7].
 * Reference call sites: CudaUtil.cu:149 (bilateral weight), AdaptMIPMFrame.cu:219
 * (blur penalty), :818, :829, :837 (view sampling). */
static inline float canon_expf(float x)
{
    if (x != x) return x;
    if (x < -104.0f) return 0.0f;
    if (x > 88.72283935546875f) return INFINITY;
    const float t  = fmaf(x, 0x1.715476p+0f /* log2(e) */, CANON_RNE_MAGIC);
    const float kf = t - CANON_RNE_MAGIC;
    float r = fmaf(kf, -0x1.62e4p-1f /* -ln2_hi, 0x3F317200 */, x);
    r = fmaf(kf, -0x1.7f7d1cp-20f /* -ln2_lo, 0x35BFBE8E */, r);
    float p = fmaf(r, 0x1.a01a02p-13f /* 1/5040 */, 0x1.6c16c2p-10f /* 1/720 */);
    p = fmaf(p, r, 0x1.111112p-7f /* 1/120 */);
    p = fmaf(p, r, 0x1.555556p-5f /* 1/24 */);
    p = fmaf(p, r, 0x1.555556p-3f /* 1/6 */);
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    const int k  = (int)kf;
    const int k1 = k / 2;            /* truncates toward zero */
    const int k2 = k - k1;
    const float s1 = canon_bits_to_float((uint32_t)(k1 + 127) << 23);
    const float s2 = canon_bits_to_float((uint32_t)(k2 + 127) << 23);
    return (p * s1) * s2;
}

/* 1/sqrt(x) as two correctly rounded operations (reference: rsqrtf in
 * CudaUtil.cu:52, AdaptMIPMFrame.cu:46). */
static inline float canon_rsqrtf(float x) { return 1.0f / sqrtf(x); }

/* sin and cos for |a| <= 0.04 (the perturbation angles of CudaUtil.cu:110-119 are
 * at most 0.01*pi): Taylor to a^7 / a^6, error far below 1 ulp there. */
static inline float canon_sin_small(float a)
{
    const float a2 = a * a;
    float p = fmaf(a2, -0x1.a01a02p-13f /* -1/5040 */, 0x1.111112p-7f /* 1/120 */);
    p = fmaf(p, a2, -0x1.555556p-3f /* -1/6 */);
    return fmaf(p, a2 * a, a);
}
static inline float canon_cos_small(float a)
{
    const float a2 = a * a;
    float p = fmaf(a2, -0x1.6c16c2p-10f /* -1/720 */, 0x1.555556p-5f /* 1/24 */);
    p = fmaf(p, a2, -0.5f);
    return fmaf(p, a2, 1.0f);
}

/* ---------------------------------------------------------------------------
 * Philox4x32-10 (SC'11): 10 rounds of two 32x32->64 multiplications with the
 * published multipliers, Weyl-sequence key schedule.
 * ------------------------------------------------------------------------- */
static inline void canon_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4])
{
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * (uint64_t)c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * (uint64_t)c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* One pixel's draw stream for one sweep.  Draw n is word (n & 3) of the Philox
 * block with counter (n >> 2, sweep, pixel, 0) under key (seed_lo, seed_hi).
 * Sweep 0 is the random initialisation; half-sweep (iter, phase) is
 * 1 + 2*iter + phase.  The pixel id is vid*ppv + y*W + x, the reference's idx
 * (AdaptMIPMFrame.cu:498). */
typedef struct {
    uint32_t key[2];
    uint32_t sweep, pixel;
    uint32_t n;
    uint32_t block;      /* index of the cached block, or 0xffffffff */
    uint32_t buf[4];
} canon_rng;

static inline void canon_rng_init(canon_rng* g, uint64_t seed, uint32_t sweep, uint32_t pixel)
{
    g->key[0] = (uint32_t)seed;
    g->key[1] = (uint32_t)(seed >> 32);
    g->sweep = sweep;
    g->pixel = pixel;
    g->n = 0;
    g->block = 0xffffffffu;
}

static inline uint32_t canon_rng_next_u32(canon_rng* g)
{
    const uint32_t b = g->n >> 2;
    if (b != g->block) {
        const uint32_t ctr[4] = { b, g->sweep, g->pixel, 0u };
        canon_philox4x32_10(ctr, g->key, g->buf);
        g->block = b;
    }
    return g->buf[g->n++ & 3u];
}

/* Uniform in (0, 1] like curand_uniform: ((u >> 8) + 1) * 2^-24. */
static inline float canon_uniform(canon_rng* g)
{
    const uint32_t u = canon_rng_next_u32(g);
    return (float)((u >> 8) + 1u) * 0x1p-24f;
}

/* ---------------------------------------------------------------------------
 * Texture emulation.  The reference samples float micro-images with
 * tex2D<float>(tex, x + 0.5f, y + 0.5f), linear filtering, unnormalised
 * coordinates, cudaAddressModeWrap (AdaptMIPMFrame.cpp:240-246,
 * AdaptMIPMFrame.cu:139-143).  Measured on a B200 (driver 580) with the probe
 * in tests/csrc/tex_probe.cu, for integer texels 0..255 (200,000 random fetches
 * plus 1-D sweeps at 2^-16 steps, all bit-exact):
 *   - wrap is not applied to unnormalised coordinates: texel indices clamp;
 *   - the texel-space coordinate is quantised to 1/256 rounding half up:
 *       q = floor(256 * fl(x + 0.5) - 127.5),  i = q >> 8,  a = q & 255
 *     (likewise b for y);
 *   - the four weights are 8-bit fixed point summing to 256, built from the
 *     rounded product  w11 = (a*b + 128) >> 8:
 *       w10 = a - w11,  w01 = b - w11,  w00 = 256 - a - b + w11;
 *   - the result is (w00 T00 + w10 T10 + w01 T01 + w11 T11) / 256, exact in float.
 * ------------------------------------------------------------------------- */
static inline float canon_tex_fetch(const float* img, int W, int H, float sx, float sy)
{
    const float ux = sx + 0.5f, uy = sy + 0.5f;
    /* 256 u - 127.5 is exact in float for u < 32.5 (windows up to 32 pixels) */
    const int qx = (int)floorf(fmaf(ux, 256.0f, -127.5f));
    const int qy = (int)floorf(fmaf(uy, 256.0f, -127.5f));
    int ix = qx >> 8, iy = qy >> 8;
    const int a = qx & 255, b = qy & 255;
    int ix1 = ix + 1, iy1 = iy + 1;
    if (ix < 0) ix = 0; if (ix > W - 1) ix = W - 1;
    if (iy < 0) iy = 0; if (iy > H - 1) iy = H - 1;
    if (ix1 < 0) ix1 = 0; if (ix1 > W - 1) ix1 = W - 1;
    if (iy1 < 0) iy1 = 0; if (iy1 > H - 1) iy1 = H - 1;
    const int t00 = (int)img[iy * W + ix],  t10 = (int)img[iy * W + ix1];
    const int t01 = (int)img[iy1 * W + ix], t11 = (int)img[iy1 * W + ix1];
    const int w11 = (a * b + 128) >> 8;
    const int w10 = a - w11, w01 = b - w11, w00 = 256 - a - b + w11;
    return (float)(w00 * t00 + w10 * t10 + w01 * t01 + w11 * t11) * 0x1p-8f;
}

#endif /* PFD_ORACLE_CANON_H */
