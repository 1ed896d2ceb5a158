// qTIP4P/f energy, warp-cooperative: one warp per geometry, the geometry and
// M sites staged in the warp's shared memory, lanes strided over the pair
// tasks and the monomers.  Same terms and constants as the reference
// (qtip4pf.cpp:57-145 monomer, 190-286 pair terms); kcal/mol, Angstrom.
#pragma once
#include "common.cuh"

namespace scp3 {
namespace qt {

constexpr double kChargeCon = 18.22234397655801030455;  // qtip4pf.cpp:61
constexpr double kQM = -1.1128 * kChargeCon;
constexpr double kQH = -kQM / 2;
constexpr double kROHeq = 0.9419;
constexpr double kAHOHeqRad = 107.4 * 3.14159265358979323846 / 180.0;  // aHOHeq*M_PI/180.0
constexpr double kEpsilon = 0.1852;
constexpr double kSigma = 3.1589;
constexpr double kAlphaR = 2.287;
constexpr double kDR = 116.09;
constexpr double kKTheta = 87.85;
constexpr double kGammaM = 0.73612;
constexpr double kGamma1 = (1.0 - kGammaM) / 2;

template <typename T>
__device__ __forceinline__ T monomer(const T* w)
{
    T d1[3], d2[3], r1 = 0, r2 = 0, c = 0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        d1[k] = w[3 + k] - w[k];
        d2[k] = w[6 + k] - w[k];
        r1 += d1[k] * d1[k];
        r2 += d2[k] * d2[k];
        c += d1[k] * d2[k];
    }
    r1 = sqrt(r1);
    r2 = sqrt(r2);
    const T x1 = T(kAlphaR) * (r1 - T(kROHeq)), x2 = T(kAlphaR) * (r2 - T(kROHeq));
    const T v1 = x1 * x1 * (T(1) - x1 * (T(1) - T(7.0 / 12.0) * x1)) * T(kDR);
    const T v2 = x2 * x2 * (T(1) - x2 * (T(1) - T(7.0 / 12.0) * x2)) * T(kDR);
    const T th = acos(c * (T(1) / r1 / r2));
    const T dth = th - T(kAHOHeqRad);
    return v1 + v2 + T(0.5) * T(kKTheta) * dth * dth;
}

template <typename T>
__device__ __forceinline__ T pair(uint32_t task, const T* crd, const T* ms)
{
    const uint32_t type = task & 3u, a = (task >> 2) & 0x7fffu, b = task >> 17;
    switch (type) {
        case 0: return T(kQH * kQM) * inv_sqrt(dist2(ms + 3 * a, crd + 3 * b));
        case 1: return T(kQH * kQH) * inv_sqrt(dist2(crd + 3 * a, crd + 3 * b));
        case 2: {
            const T s2 = T(kSigma * kSigma) / dist2(crd + 3 * a, crd + 3 * b);
            const T s6 = s2 * s2 * s2;
            return T(4 * kEpsilon) * s6 * (s6 - T(1));
        }
        default: return T(kQM * kQM) * inv_sqrt(dist2(ms + 3 * a, ms + 3 * b));
    }
}

// Energy of the geometry crd[9nw] (shared memory, T), all lanes return the sum.
// ms is a 3nw shared scratch for the M sites.
template <typename T>
__device__ double energy_warp(const T* crd, T* ms, int nw, const uint32_t* __restrict__ tasks, int ntasks,
                              int lane)
{
    double part = 0;     // terms in T, their sums in FP64
    for (int i = lane; i < nw; i += 32) {
        const T* w = crd + 9 * i;
#pragma unroll
        for (int k = 0; k < 3; k++) ms[3 * i + k] = T(kGammaM) * w[k] + T(kGamma1) * (w[3 + k] + w[6 + k]);
        part += (double)monomer(w);
    }
    __syncwarp();
    for (int t = lane; t < ntasks; t += 32) part += (double)pair(__ldg(tasks + t), crd, ms);
    return warp_sum(part);
}

}  // namespace qt
}  // namespace scp3
