// canon.cuh -- scalar arithmetic shared by every PatchMatch kernel.
//
// The reference kernels (MIStereo/AdaptMIPMFrame.cu, CudaUtil.cu,
// AdaptMIPMUtil.cu) build with --use_fast_math and seed cuRAND from clock64(),
// so their bits are neither specified nor reproducible.  This engine fixes one
// arithmetic and the CPU oracle states the same one:
//   * products feeding sums are fused explicitly with __fmaf_rn, left to right
//     (a*b + c*d + e == fma(c, d, a*b) + e;  a - b*c == fma(-b, c, a)); the
//     library is compiled with -fmad=false so nvcc fuses nothing else;
//   * division and square root are IEEE round-to-nearest;
//   * exp is pfd_expf (Cody-Waite reduction, degree-7 Taylor polynomial);
//   * random numbers are Philox4x32-10 (Salmon et al., SC'11) streams keyed by
//     (seed) and counted by (draw block, sweep, pixel).
#pragma once
#include <cstdint>

namespace pfd {

constexpr float kRneMagic = 12582912.0f;   // 1.5 * 2^23

// exp(x): x = k ln2 + r, ln2 = ln2_hi (0x3F317200, low 12 bits zero) + ln2_lo;
// e^r by Taylor to r^7; 2^k applied as two exact power-of-two products.
__device__ __forceinline__ float pfd_expf(float x)
{
    if (x != x) return x;
    if (x < -104.0f) return 0.0f;
    if (x > 88.72283935546875f) return __int_as_float(0x7f800000);
    const float t  = __fmaf_rn(x, 0x1.715476p+0f, kRneMagic);
    const float kf = __fsub_rn(t, kRneMagic);
    float r = __fmaf_rn(kf, -0x1.62e4p-1f, x);
    r = __fmaf_rn(kf, -0x1.7f7d1cp-20f, r);
    float p = __fmaf_rn(r, 0x1.a01a02p-13f, 0x1.6c16c2p-10f);
    p = __fmaf_rn(p, r, 0x1.111112p-7f);
    p = __fmaf_rn(p, r, 0x1.555556p-5f);
    p = __fmaf_rn(p, r, 0x1.555556p-3f);
    p = __fmaf_rn(p, r, 0.5f);
    p = __fmaf_rn(p, r, 1.0f);
    p = __fmaf_rn(p, r, 1.0f);
    const int k  = __float2int_rz(kf);
    const int k1 = k / 2;
    const int k2 = k - k1;
    const float s1 = __int_as_float((k1 + 127) << 23);
    const float s2 = __int_as_float((k2 + 127) << 23);
    return __fmul_rn(__fmul_rn(p, s1), s2);
}

// exp(x) for x in (-104, 0]: the bilateral weights, whose argument is never
// positive and never NaN.  Same arithmetic as pfd_expf on that range.
__device__ __forceinline__ float pfd_expf_nonpos(float x)
{
    const float t  = __fmaf_rn(x, 0x1.715476p+0f, kRneMagic);
    const float kf = __fsub_rn(t, kRneMagic);
    float r = __fmaf_rn(kf, -0x1.62e4p-1f, x);
    r = __fmaf_rn(kf, -0x1.7f7d1cp-20f, r);
    float p = __fmaf_rn(r, 0x1.a01a02p-13f, 0x1.6c16c2p-10f);
    p = __fmaf_rn(p, r, 0x1.111112p-7f);
    p = __fmaf_rn(p, r, 0x1.555556p-5f);
    p = __fmaf_rn(p, r, 0x1.555556p-3f);
    p = __fmaf_rn(p, r, 0.5f);
    p = __fmaf_rn(p, r, 1.0f);
    p = __fmaf_rn(p, r, 1.0f);
    const int k  = __float_as_int(t) - 0x4B400000;     // the rounded integer
    const int k1 = k / 2;
    const int k2 = k - k1;
    const float v = __fmul_rn(__fmul_rn(p, __int_as_float((k1 + 127) << 23)), __int_as_float((k2 + 127) << 23));
    return (x < -104.0f) ? 0.0f : v;
}

__device__ __forceinline__ float pfd_rsqrtf(float x) { return __fdiv_rn(1.0f, __fsqrt_rn(x)); }

// sin / cos for |a| <= 0.04 (perturbation angles, CudaUtil.cu:110-119).
__device__ __forceinline__ float pfd_sin_small(float a)
{
    const float a2 = __fmul_rn(a, a);
    float p = __fmaf_rn(a2, -0x1.a01a02p-13f, 0x1.111112p-7f);
    p = __fmaf_rn(p, a2, -0x1.555556p-3f);
    return __fmaf_rn(p, __fmul_rn(a2, a), a);
}
__device__ __forceinline__ float pfd_cos_small(float a)
{
    const float a2 = __fmul_rn(a, a);
    float p = __fmaf_rn(a2, -0x1.6c16c2p-10f, 0x1.555556p-5f);
    p = __fmaf_rn(p, a2, -0.5f);
    return __fmaf_rn(p, a2, 1.0f);
}

// Philox4x32-10.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

// One pixel's draw stream in one sweep: draw n = word (n & 3) of block
// (n >> 2, sweep, pixel, 0).
struct DrawStream {
    uint2 key;
    uint32_t sweep, pixel, n, block;
    uint4 buf;

    __device__ __forceinline__ void init(uint64_t seed, uint32_t sw, uint32_t px)
    {
        key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
        sweep = sw; pixel = px; n = 0; block = 0xffffffffu;
    }
    __device__ __forceinline__ uint32_t next_u32()
    {
        const uint32_t b = n >> 2;
        if (b != block) { buf = philox4x32_10(make_uint4(b, sweep, pixel, 0u), key); block = b; }
        const uint32_t w = n & 3u;
        ++n;
        return w == 0 ? buf.x : (w == 1 ? buf.y : (w == 2 ? buf.z : buf.w));
    }
    // (0, 1], like curand_uniform
    __device__ __forceinline__ float uniform() { return __fmul_rn((float)((next_u32() >> 8) + 1u), 0x1p-24f); }
};

}  // namespace pfd
