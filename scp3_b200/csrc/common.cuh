// Device helpers shared by the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace scp3 {

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T>
__device__ __forceinline__ T dist2(const T* a, const T* b)
{
    const T dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    return dx * dx + dy * dy + dz * dz;
}

__device__ __forceinline__ double inv_sqrt(double x) { return 1.0 / sqrt(x); }
// IEEE-rounded in FP32 too: rsqrtf's approximation error is not centred and its
// bias, summed over the ~10^4 kcal/mol of Coulomb terms of a cluster, shows in
// the levels at the 0.1 cm^-1 scale.
__device__ __forceinline__ float inv_sqrt(float x) { return __frsqrt_rn(x); }

// Beasley-Springer-Moro inverse normal CDF, the same formula and branch points
// as the reference (beasley_springer_moro.cpp:14-46); log() is CUDA's.
__device__ __forceinline__ double bsm(double u)
{
    const double y = u - 0.5;
    if (fabs(y) < 0.42) {
        const double r = y * y;
        return y * (((-25.44106049637 * r + 41.39119773534) * r + -18.61500062529) * r + 2.50662823884) /
               ((((3.13082909833 * r + -21.06224101826) * r + 23.08336743743) * r + -8.47351093090) * r + 1);
    }
    const double r = (y > 0) ? log(-log(1 - u)) : log(-log(u));
    const double t = 0.3374754822726147 +
                     r * (0.9761690190917186 +
                          r * (0.1607979714918209 +
                               r * (0.0276438810333863 +
                                    r * (0.0038405729373609 +
                                         r * (0.0003951896511919 +
                                              r * (0.0000321767881768 + r * (0.0000002888167364 +
                                                                              r * 0.0000003960315187)))))));
    return (y < 0) ? -t : t;
}

// The same inverse CDF in FP32 for the FP32 form, split at its branch so that
// a warp can run the central branch over all its items and the rarer tail
// branch (|u - 0.5| >= 0.42, 16 % of the points) over a compacted list of them.
// From the 62-bit Sobol state x (u = x 2^-62):
// * bsm_centred_f32: y = u - 0.5 from the top 32 bits of x as a centred signed
//   integer (truncation below 2^-32, then one rounding to FP32);
// * bsm_central_f32: the rational function of the central branch, divided with
//   __fdividef (the denominator lies in [0.11, 1]; within 2 ulp);
// * bsm_tail_f32: the tail branch, from min(u, 1 - u) formed exactly from the
//   integer state (the upper tail as (2^62 - x) 2^-62); the two logarithms are
//   the __logf intrinsic (3 ulp here: both arguments lie outside [0.5, 2]).
__device__ __forceinline__ float bsm_centred_f32(uint64_t x)
{
    return (float)(int32_t)((uint32_t)(x >> 30) ^ 0x80000000u) * 0x1p-32f;
}

__device__ __forceinline__ float bsm_central_f32(float y)
{
    const float r = y * y;
    return __fdividef(
        y * (((-25.44106049637f * r + 41.39119773534f) * r + -18.61500062529f) * r + 2.50662823884f),
        (((3.13082909833f * r + -21.06224101826f) * r + 23.08336743743f) * r + -8.47351093090f) * r + 1.0f);
}

__device__ __forceinline__ float bsm_tail_f32(uint64_t x)
{
    const bool upper = x >= (1ull << 61);
    const float p = (float)(int64_t)(upper ? (1ull << 62) - x : x) * 0x1p-62f;
    const float r = __logf(-__logf(p));
    const float t = 0.3374754822726147f +
                    r * (0.9761690190917186f +
                         r * (0.1607979714918209f +
                              r * (0.0276438810333863f +
                                   r * (0.0038405729373609f +
                                        r * (0.0003951896511919f +
                                             r * (0.0000321767881768f + r * (0.0000002888167364f +
                                                                             r * 0.0000003960315187f)))))));
    return upper ? t : -t;
}

// The 62-bit Sobol state of point `index` of dimension d: XOR of the direction
// numbers picked by the Gray code of the index (the state i8_sobol reaches by
// walking, sobol.cpp:27796-27856).  vdir is [bit][dims].
__device__ __forceinline__ uint64_t sobol_state(const int64_t* __restrict__ vdir, int dims, int d, uint64_t index)
{
    uint64_t g = index ^ (index >> 1);
    uint64_t x = 0;
    while (g) {
        const int b = __ffsll((long long)g) - 1;
        x ^= (uint64_t)__ldg(vdir + (size_t)b * dims + d);
        g &= g - 1;
    }
    return x;
}

__device__ __forceinline__ double sobol_uniform(uint64_t x) { return (double)(int64_t)x * 0x1p-62; }

}  // namespace scp3
