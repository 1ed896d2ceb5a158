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

// Water pair p of the row-major upper triangle of nw waters: a < b.
__host__ __device__ __forceinline__ void water_pair_of(int p, int nw, int& a, int& b)
{
    a = 0;
    while (p >= nw - 1 - a) {
        p -= nw - 1 - a;
        a++;
    }
    b = a + 1 + p;
}

// The ten site pairs of waters a < b that the reference's pair loops visit
// (qtip4pf.cpp:213-283): the M site of each water against the two H of the
// other, the four H/H pairs, O/O (Lennard-Jones) and M/M.  The eight sites are
// read once; each term is formed in T exactly as pair() forms it and summed in
// FP64.
template <typename T>
__device__ __forceinline__ double water_pair(int a, int b, const T* crd, const T* ms)
{
    T s[2][4][3];   // [water][O, H1, H2, M][x, y, z]
#pragma unroll
    for (int k = 0; k < 3; k++) {
#pragma unroll
        for (int l = 0; l < 3; l++) s[0][l][k] = crd[9 * a + 3 * l + k], s[1][l][k] = crd[9 * b + 3 * l + k];
        s[0][3][k] = ms[3 * a + k];
        s[1][3][k] = ms[3 * b + k];
    }
    double e = 0.0;
#pragma unroll
    for (int w = 0; w < 2; w++)
#pragma unroll
        for (int l = 1; l < 3; l++) e += (double)(T(kQH * kQM) * inv_sqrt(dist2(s[w][3], s[1 - w][l])));
#pragma unroll
    for (int l = 1; l < 3; l++)
#pragma unroll
        for (int m = 1; m < 3; m++) e += (double)(T(kQH * kQH) * inv_sqrt(dist2(s[0][l], s[1][m])));
    const T s2 = T(kSigma * kSigma) / dist2(s[0][0], s[1][0]);
    const T s6 = s2 * s2 * s2;
    e += (double)(T(4 * kEpsilon) * s6 * (s6 - T(1)));
    e += (double)(T(kQM * kQM) * inv_sqrt(dist2(s[0][3], s[1][3])));
    return e;
}

// Energies of ng <= 4 geometries crd + j * stride (shared memory, T) at once,
// ms a [4][3nw] shared scratch: lane l works for geometry l % 4 only (M sites and
// monomers as items (water, geometry), pair terms as items (water pair,
// geometry)), so a warp keeps its lanes busy on the per-water and per-pair
// terms; lane l returns the sum of geometry l % 4.
template <typename T>
__device__ double energy_warp4(const T* crd, int stride, T* ms, int nw, int ng, int lane)
{
    const int j = lane & 3;
    const bool on = j < ng;
    const T* cj = crd + j * stride;
    T* mj = ms + j * 3 * nw;
    if (on)
        for (int i = lane >> 2; i < nw; i += 8) {
            const T* w = cj + 9 * i;
#pragma unroll
            for (int k = 0; k < 3; k++) mj[3 * i + k] = T(kGammaM) * w[k] + T(kGamma1) * (w[3 + k] + w[6 + k]);
        }
    __syncwarp();
    double part = 0;    // terms in T, their sums in FP64
    if (on) {
        for (int i = lane >> 2; i < nw; i += 8) part += (double)monomer(cj + 9 * i);
        const int np = nw * (nw - 1) / 2;
        for (int p = lane >> 2; p < np; p += 8) {
            int a, b;
            water_pair_of(p, nw, a, b);
            part += water_pair<T>(a, b, cj, mj);
        }
    }
    part += __shfl_xor_sync(0xffffffffu, part, 4);
    part += __shfl_xor_sync(0xffffffffu, part, 8);
    part += __shfl_xor_sync(0xffffffffu, part, 16);
    return part;
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


// ---------------------------------------------------------------- energy + gradient
// qtip4pf.cpp:252-397 (the E+g operator of the gradient path): the same terms,
// their derivatives in kcal/mol/A.  The M site is gammaM O + gamma1 (H1 + H2), so
// the force on it is spread over the three atoms with those weights.  In the
// precision T (FP64 for the parity form; FP32 for the split form's products),
// each term's energy returned in FP64 and summed in FP64.

template <typename T>
__device__ __forceinline__ double monomer_grad(const T* w, T* g)
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
    const T v1 = x1 * x1 * (T(1.0) - x1 * (T(1.0) - T(7.0 / 12.0) * x1)) * T(kDR);
    const T v2 = x2 * x2 * (T(1.0) - x2 * (T(1.0) - T(7.0 / 12.0) * x2)) * T(kDR);
    const T dv1 = T(kDR) * T(kAlphaR) * x1 * (T(2.0) - x1 * (T(3.0) - T(7.0 / 3.0) * x1));   // dv/dr
    const T dv2 = T(kDR) * T(kAlphaR) * x2 * (T(2.0) - x2 * (T(3.0) - T(7.0 / 3.0) * x2));
    const T cs = c / (r1 * r2);
    const T dth = acos(cs) - T(kAHOHeqRad);
    const T de_dc = -T(kKTheta) * dth / sqrt(T(1.0) - cs * cs);                           // dE/dcos(theta)
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const T u1 = d1[k] / r1, u2 = d2[k] / r2;
        const T gh1 = dv1 * u1 + de_dc * (u2 - cs * u1) / r1;
        const T gh2 = dv2 * u2 + de_dc * (u1 - cs * u2) / r2;
        atomicAdd(g + 3 + k, gh1);
        atomicAdd(g + 6 + k, gh2);
        atomicAdd(g + k, -(gh1 + gh2));
    }
    return (double)(v1 + v2 + T(0.5) * T(kKTheta) * dth * dth);
}

// q q' / |a - b|: energy; gradient into ga (at a) and gb (at b)
template <typename T>
__device__ __forceinline__ double coulomb_grad(double qq, const T* a, const T* b, T* ga, T* gb)
{
    const T d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
    const T ir = T(1.0) / sqrt(d0 * d0 + d1 * d1 + d2 * d2), e = T(qq) * ir, f = -e * ir * ir;
    atomicAdd(ga + 0, f * d0), atomicAdd(ga + 1, f * d1), atomicAdd(ga + 2, f * d2);
    atomicAdd(gb + 0, -f * d0), atomicAdd(gb + 1, -f * d1), atomicAdd(gb + 2, -f * d2);
    return (double)e;
}

template <typename T>
__device__ __forceinline__ double pair_grad(uint32_t task, const T* crd, const T* ms, T* g, T* gm)
{
    const uint32_t type = task & 3u, a = (task >> 2) & 0x7fffu, b = task >> 17;
    switch (type) {
        case 0: return coulomb_grad<T>(kQH * kQM, ms + 3 * a, crd + 3 * b, gm + 3 * a, g + 3 * b);
        case 1: return coulomb_grad<T>(kQH * kQH, crd + 3 * a, crd + 3 * b, g + 3 * a, g + 3 * b);
        case 2: {
            const T d0 = crd[3 * a] - crd[3 * b], d1 = crd[3 * a + 1] - crd[3 * b + 1];
            const T d2 = crd[3 * a + 2] - crd[3 * b + 2];
            const T r2 = d0 * d0 + d1 * d1 + d2 * d2;
            const T s2 = T(kSigma * kSigma) / r2, s6 = s2 * s2 * s2;
            const T f = T(2.0 * 4 * kEpsilon) * (T(3.0) * s6 - T(6.0) * s6 * s6) / r2;   // 2 dE/d(r^2)
            atomicAdd(g + 3 * a, f * d0), atomicAdd(g + 3 * a + 1, f * d1), atomicAdd(g + 3 * a + 2, f * d2);
            atomicAdd(g + 3 * b, -f * d0), atomicAdd(g + 3 * b + 1, -f * d1), atomicAdd(g + 3 * b + 2, -f * d2);
            return (double)(T(4 * kEpsilon) * s6 * (s6 - T(1.0)));
        }
        default: return coulomb_grad<T>(kQM * kQM, ms + 3 * a, ms + 3 * b, gm + 3 * a, gm + 3 * b);
    }
}

// Energy (all lanes) and gradient g[9nw] (shared, complete after the call) of
// the geometry crd; ms[3nw] and gm[3nw] are shared scratch (M sites, their forces).
template <typename T>
__device__ inline double energy_grad_warp(const T* crd, T* ms, T* g, T* gm, int nw,
                                          const uint32_t* __restrict__ tasks, int ntasks, int lane)
{
    for (int c = lane; c < 9 * nw; c += 32) g[c] = T(0);
    for (int c = lane; c < 3 * nw; c += 32) gm[c] = T(0);
    for (int i = lane; i < nw; i += 32) {
        const T* w = crd + 9 * i;
#pragma unroll
        for (int k = 0; k < 3; k++) ms[3 * i + k] = T(kGammaM) * w[k] + T(kGamma1) * (w[3 + k] + w[6 + k]);
    }
    __syncwarp();
    double part = 0;
    for (int i = lane; i < nw; i += 32) part += monomer_grad<T>(crd + 9 * i, g + 9 * i);
    for (int t = lane; t < ntasks; t += 32) part += pair_grad<T>(__ldg(tasks + t), crd, ms, g, gm);
    __syncwarp();
    for (int i = lane; i < nw; i += 32)
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const T f = gm[3 * i + k];
            g[9 * i + k] += T(kGammaM) * f;
            g[9 * i + 3 + k] += T(kGamma1) * f;
            g[9 * i + 6 + k] += T(kGamma1) * f;
        }
    __syncwarp();
    return warp_sum(part);
}

// The ten site pairs of waters a < b with their gradients, as water_pair:
// each term formed in T as pair_grad() forms it, the forces on the eight sites
// gathered in registers and added to g (O, H1, H2) and gm (M) once per site.
template <typename T>
__device__ __forceinline__ double water_pair_grad(int a, int b, const T* crd, const T* ms, T* g, T* gm)
{
    T s[2][4][3], f[2][4][3];   // [water][O, H1, H2, M][x, y, z]: positions, forces
#pragma unroll
    for (int k = 0; k < 3; k++) {
#pragma unroll
        for (int l = 0; l < 3; l++) s[0][l][k] = crd[9 * a + 3 * l + k], s[1][l][k] = crd[9 * b + 3 * l + k];
        s[0][3][k] = ms[3 * a + k];
        s[1][3][k] = ms[3 * b + k];
#pragma unroll
        for (int l = 0; l < 4; l++) f[0][l][k] = f[1][l][k] = T(0);
    }
    double e = 0.0;
    // q q' / |u - v| with its forces, u = site x of water w, v = site y of water 1 - w
    auto coulomb = [&](T qq, int w, int x, int y) {
        const T d0 = s[w][x][0] - s[1 - w][y][0], d1 = s[w][x][1] - s[1 - w][y][1], d2 = s[w][x][2] - s[1 - w][y][2];
        const T ir = T(1.0) / sqrt(d0 * d0 + d1 * d1 + d2 * d2), eu = qq * ir, fu = -eu * ir * ir;
        f[w][x][0] += fu * d0, f[w][x][1] += fu * d1, f[w][x][2] += fu * d2;
        f[1 - w][y][0] -= fu * d0, f[1 - w][y][1] -= fu * d1, f[1 - w][y][2] -= fu * d2;
        e += (double)eu;
    };
#pragma unroll
    for (int w = 0; w < 2; w++)
#pragma unroll
        for (int l = 1; l < 3; l++) coulomb(T(kQH * kQM), w, 3, l);
#pragma unroll
    for (int l = 1; l < 3; l++)
#pragma unroll
        for (int m = 1; m < 3; m++) coulomb(T(kQH * kQH), 0, l, m);
    {
        const T d0 = s[0][0][0] - s[1][0][0], d1 = s[0][0][1] - s[1][0][1], d2 = s[0][0][2] - s[1][0][2];
        const T r2 = d0 * d0 + d1 * d1 + d2 * d2;
        const T s2 = T(kSigma * kSigma) / r2, s6 = s2 * s2 * s2;
        const T fo = T(2.0 * 4 * kEpsilon) * (T(3.0) * s6 - T(6.0) * s6 * s6) / r2;   // 2 dE/d(r^2)
        f[0][0][0] += fo * d0, f[0][0][1] += fo * d1, f[0][0][2] += fo * d2;
        f[1][0][0] -= fo * d0, f[1][0][1] -= fo * d1, f[1][0][2] -= fo * d2;
        e += (double)(T(4 * kEpsilon) * s6 * (s6 - T(1.0)));
    }
    coulomb(T(kQM * kQM), 0, 3, 3);
#pragma unroll
    for (int k = 0; k < 3; k++) {
#pragma unroll
        for (int l = 0; l < 3; l++) atomicAdd(g + 9 * a + 3 * l + k, f[0][l][k]), atomicAdd(g + 9 * b + 3 * l + k, f[1][l][k]);
        atomicAdd(gm + 3 * a + k, f[0][3][k]);
        atomicAdd(gm + 3 * b + k, f[1][3][k]);
    }
    return e;
}

// Energies and gradients of ng <= 4 geometries crd + j * stride at once (the
// FP32 gradient path): lane l works for geometry l % 4 only, as energy_warp4;
// ms [4][3nw], g [4][9nw] and gm [4][3nw] are shared scratch, g complete after
// the call; lane l returns the energy of geometry l % 4.
template <typename T>
__device__ double energy_grad_warp4(const T* crd, int stride, T* ms, T* g, T* gm, int nw, int ng, int lane)
{
    const int j = lane & 3;
    const bool on = j < ng;
    const T* cj = crd + j * stride;
    T* mj = ms + j * 3 * nw;
    T* gj = g + j * 9 * nw;
    T* gmj = gm + j * 3 * nw;
    for (int c = lane; c < 4 * 9 * nw; c += 32) g[c] = T(0);
    for (int c = lane; c < 4 * 3 * nw; c += 32) gm[c] = T(0);
    if (on)
        for (int i = lane >> 2; i < nw; i += 8) {
            const T* w = cj + 9 * i;
#pragma unroll
            for (int k = 0; k < 3; k++) mj[3 * i + k] = T(kGammaM) * w[k] + T(kGamma1) * (w[3 + k] + w[6 + k]);
        }
    __syncwarp();
    double part = 0;
    if (on) {
        for (int i = lane >> 2; i < nw; i += 8) part += monomer_grad<T>(cj + 9 * i, gj + 9 * i);
        const int np = nw * (nw - 1) / 2;
        for (int p = lane >> 2; p < np; p += 8) {
            int a, b;
            water_pair_of(p, nw, a, b);
            part += water_pair_grad<T>(a, b, cj, mj, gj, gmj);
        }
    }
    __syncwarp();
    if (on)
        for (int i = lane >> 2; i < nw; i += 8)
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const T f = gmj[3 * i + k];
                gj[9 * i + k] += T(kGammaM) * f;
                gj[9 * i + 3 + k] += T(kGamma1) * f;
                gj[9 * i + 6 + k] += T(kGamma1) * f;
            }
    __syncwarp();
    part += __shfl_xor_sync(0xffffffffu, part, 4);
    part += __shfl_xor_sync(0xffffffffu, part, 8);
    part += __shfl_xor_sync(0xffffffffu, part, 16);
    return part;
}

}  // namespace qt
}  // namespace scp3
