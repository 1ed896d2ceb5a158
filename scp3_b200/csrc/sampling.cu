// Per-sample kernels: Sobol point (optionally scrambled) -> BSM -> q = y/sqrt(2)
// -> Cartesian back-transform -> water potential -> anharmonic residual.
// One warp per sample; the sample's q and geometry live in the warp's slice of
// shared memory, lanes split the dimensions, the coordinates and the potential's
// pair terms.  The FP64 form follows SCP3.cpp:196-223 operation for operation
// where that is cheap (division by sqrt(2), x0 + MUa q then times bohr).
#include "common.cuh"
#include "internal.h"
#include "pes_qtip4pf.cuh"
#include "pes_ttm3f.cuh"
#include "ps_coeffs.h"

#include <algorithm>
#include <cmath>
#include <mutex>

namespace scp3 {

namespace {

constexpr int kWarpsPerBlock = 8;
constexpr int kRun = 16;          // samples per warp of a batch launch (Gray-code walk)
constexpr int kMinRun = 8;        // fewest samples per warp of a single launch

// Samples a warp carries through the back-transform together, so that every
// shared-memory read of MUa serves this many samples (the back-transform is
// bound by shared-memory bandwidth, MUa being re-read for every sample).
constexpr int kGroup = 4;

template <typename T>
struct WarpSlot {
    T* q;           // [group][qs] normal coordinates (the form's precision)
    T* crd;         // [group][9nw] geometries
    T* ms;          // [group][3nw] M sites
    T* ttm;         // TTM3-F scratch
    double* g;      // 9nw gradient (gradient path)
    double* gm;     // 3nw forces on the M sites
    uint64_t* xs;   // FP32 form: [group][nm0] Sobol states of the group
    uint16_t* tl;   // FP32 form: [group * nm0] items that take the inverse CDF's tail branch
    int qs;         // q stride: nm0 rounded up to even (16-byte aligned rows)
};

// Gradient storage of a warp slot: [9nw] + [3nw] in FP64, or in the FP32 form
// the four geometries' [4][9nw] + [4][3nw].
template <typename T>
__host__ __device__ inline size_t grad_bytes(int nw, int group)
{
    return sizeof(T) == 4 ? sizeof(float) * (size_t)(12 * nw * group) : sizeof(double) * (size_t)(12 * nw);
}

template <typename T>
__host__ __device__ inline size_t slot_bytes(int pes, int nm0, int nw, bool grad = false, int group = 1)
{
    size_t b = sizeof(T) * ((size_t)group * ((nm0 + 1) & ~1) + (size_t)(12 * nw * group));
    if (pes == SCP3GPU_PES_TTM3F) b += sizeof(T) * ttm::scratch_elems(nw, grad);
    b = (b + 7) & ~(size_t)7;
    if (grad) b += grad_bytes<T>(nw, group);
    if (sizeof(T) == 4) b += (size_t)group * nm0 * (sizeof(uint64_t) + sizeof(uint16_t));
    return (b + 15) & ~(size_t)15;
}

template <typename T>
__device__ inline WarpSlot<T> warp_slot(char* base, int pes, int nm0, int nw, bool grad = false, int group = 1)
{
    WarpSlot<T> s;
    s.qs = (nm0 + 1) & ~1;
    s.q = reinterpret_cast<T*>(base);
    s.crd = s.q + (size_t)group * s.qs;
    s.ms = s.crd + 9 * nw * group;
    s.ttm = s.ms + 3 * nw * group;
    size_t off = sizeof(T) * ((size_t)group * s.qs + (size_t)(12 * nw * group));
    if (pes == SCP3GPU_PES_TTM3F) off += sizeof(T) * ttm::scratch_elems(nw, grad);
    off = (off + 7) & ~(size_t)7;
    s.g = grad ? reinterpret_cast<double*>(base + off) : nullptr;
    s.gm = grad ? s.g + 9 * nw : nullptr;
    if (grad) off += grad_bytes<T>(nw, group);
    s.xs = sizeof(T) == 4 ? reinterpret_cast<uint64_t*>(base + off) : nullptr;
    s.tl = sizeof(T) == 4 ? reinterpret_cast<uint16_t*>(base + off + sizeof(uint64_t) * (size_t)group * nm0) : nullptr;
    return s;
}

template <int PES, typename T>
__device__ inline double potential(const T* crd, const WarpSlot<T>& w, int nw, const uint32_t* tasks, int ntasks,
                                   int lane, int* iters)
{
    if (PES == SCP3GPU_PES_QTIP4PF) {
        *iters = 0;
        return qt::energy_warp<T>(crd, w.ms, nw, tasks, ntasks, lane);
    }
    return ttm::energy_warp<T>(crd, w.ms, w.ttm, nw, tasks, ntasks, lane, iters);
}

// MUa is staged in shared memory, in the form's precision, when it fits this
// many bytes, as coordinate pairs: for mode k and coordinate group g (64
// coordinates), lane l reads {MUa[k][64g + l], MUa[k][64g + 32 + l]} as one
// word (zero past the last coordinate).
constexpr size_t kMuaSmemMax = 64 * 1024;

__host__ __device__ inline int mua_groups(int nw) { return (9 * nw + 63) / 64; }

// On the gradient path MUa of the selected modes is also staged transposed,
// [coordinate][selected mode] in FP64, when it fits this many bytes: the lane of
// mode m then reads row c at m (consecutive lanes, consecutive words) where a
// read of MUa[k][c] from global memory touched one cache line per lane.
constexpr size_t kMuaTSmemMax = 48 * 1024;
__host__ __device__ inline size_t muat_smem_bytes(int nw, int nm)
{
    return (sizeof(double) * 9 * (size_t)nw * nm + 15) / 16 * 16;   // the warp slots follow, 16-byte aligned
}
template <typename T>
__host__ __device__ inline size_t mua_smem_bytes(int nw, int nm0)
{
    return sizeof(T) * 64 * (size_t)mua_groups(nw) * nm0;
}

template <typename T>
struct Pair;
template <>
struct Pair<double> {
    using type = double2;
};
template <>
struct Pair<float> {
    using type = float2;
};

// G: the gradient path (dV/dq) is compiled in; the energy-only instances keep
// their registers for the energy path.
template <int PES, typename T, bool G = false>
__device__ __forceinline__ void samples_body(const SampleArgs& a, char* smem);

template <int PES, typename T, bool G>
// Blocks per SM the registers must allow: 4 for the FP32 energy path (64
// registers), 3 for the FP32 gradient path (85: a few spills, 1.3x faster than
// at 2), 2 for FP64.
__global__ void __launch_bounds__(kWarpsPerBlock * 32, sizeof(T) == 4 ? (G ? 3 : 4) : 2)
    samples_kernel(SampleArgs a)
{
    extern __shared__ __align__(16) char smem[];
    samples_body<PES, T, G>(a, smem);
}

// Several clusters of a batch: cluster blockIdx.y takes args[blockIdx.y].
template <int PES, typename T>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) samples_batch_kernel(const SampleArgs* __restrict__ args)
{
    extern __shared__ __align__(16) char smem[];
    // the cluster's arguments in shared memory, read where used (a register copy
    // of the whole block costs occupancy)
    __shared__ SampleArgs a;
    if (threadIdx.x == 0) a = args[blockIdx.y];
    __syncthreads();
    samples_body<PES, T>(a, smem);
}

template <int PES, typename T, bool G>
__device__ __forceinline__ void samples_body(const SampleArgs& a, char* smem)
{
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int nw = a.nw, nm0 = a.nm0, N3 = 9 * nw;
    using T2 = typename Pair<T>::type;
    const size_t mua_b = mua_smem_bytes<T>(nw, nm0);
    const bool mua_in_smem = mua_b <= kMuaSmemMax;
    const int ng = mua_groups(nw);
    const double* MUa = a.MUa;
    T2* mua2 = reinterpret_cast<T2*>(smem);      // [nm0][ng][32] coordinate pairs
    if (mua_in_smem) {
        for (int e = threadIdx.x; e < nm0 * ng * 32; e += blockDim.x) {
            const int l = e & 31, g = (e >> 5) % ng, k = (e >> 5) / ng, c = 64 * g + l;
            T2 m;
            m.x = (T)(c < N3 ? a.MUa[(size_t)k * N3 + c] : 0.0);
            m.y = (T)(c + 32 < N3 ? a.MUa[(size_t)k * N3 + c + 32] : 0.0);
            mua2[e] = m;
        }
        __syncthreads();
    }
    const bool grad = G && a.vq != nullptr;
    const bool muat_in_smem = grad && muat_smem_bytes(nw, a.nm) <= kMuaTSmemMax;
    double* muat = reinterpret_cast<double*>(smem + (mua_in_smem ? mua_b : 0));   // [N3][nm]
    if (muat_in_smem) {
        for (int e = threadIdx.x; e < N3 * a.nm; e += blockDim.x) {
            const int c = e / a.nm, m = e - c * a.nm;
            muat[e] = a.MUa[(size_t)__ldg(a.modes + m) * N3 + c];
        }
        __syncthreads();
    }
    char* slots = smem + (mua_in_smem ? mua_b : 0) + (muat_in_smem ? muat_smem_bytes(nw, a.nm) : 0);
    WarpSlot<T> w = warp_slot<T>(slots + wib * slot_bytes<T>(PES, nm0, nw, grad, kGroup), PES, nm0, nw, grad, kGroup);
    // Each warp takes one contiguous range of samples, the ranges balanced to
    // within one sample (the grid is sized to the SMs, so there is no tail wave):
    // the Sobol state of the first is formed from the Gray code of its index, the
    // next ones by one XOR per dimension (index k differs from k-1 in direction
    // number ctz(k)).  The range goes in groups of kGroup samples: normals for
    // the group, one back-transform pass for the group, then the potential per
    // sample.
    const int64_t nwarps = (int64_t)gridDim.x * kWarpsPerBlock;
    const int64_t gw = (int64_t)blockIdx.x * kWarpsPerBlock + wib;
    constexpr int kDimsPerLane = 4;           // dimensions up to 128 keep their state in registers
    uint64_t st[kDimsPerLane];
    const int64_t s_first = a.n * gw / nwarps, s_end = a.n * (gw + 1) / nwarps;
    const bool sobol = a.normals == nullptr && a.normals32 == nullptr;
    for (int64_t s0 = s_first; s0 < s_end; s0 += kGroup) {
        const int gn = (int)(s_end - s0 < kGroup ? s_end - s0 : kGroup);
        // 1. standard normals -> q   (SCP3.cpp:196-201)
        bool done = false;
        if constexpr (sizeof(T) == 4) {
            if (sobol) {
                // FP32 form: (a) the group's Sobol states, lane-owned by dimension,
                // staged as [sample][dimension] (padding samples get u = 0.5, so
                // q = 0); (b) the central branch over all gn * nm0 items, the warp's
                // lanes strided over them, the tail items listed; (c) the tail
                // branch over the list.
                for (int j = 0; j < gn; j++) {
                    const int64_t s = s0 + j;
                    const uint64_t idx = (uint64_t)(a.index0 + s);
                    uint64_t* xj = w.xs + j * nm0;
                    if (s >= a.nvalid) {
                        for (int d = lane; d < nm0; d += 32) xj[d] = 1ull << 61;
                        continue;
                    }
#pragma unroll
                    for (int jd = 0; jd < kDimsPerLane; jd++) {
                        const int d = lane + 32 * jd;
                        if (d >= nm0) break;
                        if (s == s_first) st[jd] = sobol_state(a.vdir, nm0, d, idx);
                        else st[jd] ^= (uint64_t)__ldg(a.vdir + (size_t)(__ffsll((long long)idx) - 1) * nm0 + d);
                        xj[d] = a.shift ? st[jd] ^ __ldg(a.shift + d) : st[jd];
                    }
                    for (int d = lane + 32 * kDimsPerLane; d < nm0; d += 32)
                        xj[d] = (a.shift ? __ldg(a.shift + d) : 0ull) ^ sobol_state(a.vdir, nm0, d, idx);
                }
                __syncwarp();
                const int items = gn * nm0;
                const float inv_nm0 = 1.0f / (float)nm0;   // item i is (i / nm0, i % nm0); exact for i < 2^16
                // two items per lane and round (i, i + 32): two independent chains;
                // every item runs the central formula, the tail items' values are
                // dropped (their denominator may vanish; nothing reads the quotient)
                int ntail = 0;
                const unsigned below = (1u << lane) - 1u;
                for (int i0 = 0; i0 < items; i0 += 64) {
                    const int ia = i0 + lane, ib = ia + 32;
                    const float ya = ia < items ? bsm_centred_f32(w.xs[ia]) : 0.0f;
                    const float yb = ib < items ? bsm_centred_f32(w.xs[ib]) : 0.0f;
                    const float va = bsm_central_f32(ya), vb = bsm_central_f32(yb);
                    const bool ta = ia < items && !(fabsf(ya) < 0.42f);
                    const bool tb = ib < items && !(fabsf(yb) < 0.42f);
                    if (ia < items && !ta) {
                        const int j = (int)(((float)ia + 0.5f) * inv_nm0);
                        w.q[j * w.qs + (ia - j * nm0)] = (T)(va * 0.70710678f);
                    }
                    if (ib < items && !tb) {
                        const int j = (int)(((float)ib + 0.5f) * inv_nm0);
                        w.q[j * w.qs + (ib - j * nm0)] = (T)(vb * 0.70710678f);
                    }
                    const unsigned ma = __ballot_sync(0xffffffffu, ta);
                    if (ta) w.tl[ntail + __popc(ma & below)] = (uint16_t)ia;
                    ntail += __popc(ma);
                    const unsigned mb = __ballot_sync(0xffffffffu, tb);
                    if (tb) w.tl[ntail + __popc(mb & below)] = (uint16_t)ib;
                    ntail += __popc(mb);
                }
                __syncwarp();
                for (int t = lane; t < ntail; t += 32) {
                    const int i = w.tl[t];
                    const int j = (int)(((float)i + 0.5f) * inv_nm0);
                    w.q[j * w.qs + (i - j * nm0)] = (T)(bsm_tail_f32(w.xs[i]) * 0.70710678f);
                }
                done = true;
            }
        }
        for (int j = 0; j < gn && !done; j++) {
            const int64_t s = s0 + j;
            T* q = w.q + j * w.qs;
            if (s >= a.nvalid) {        // padding sample (the range's tail): contributes nothing
                for (int d = lane; d < nm0; d += 32) q[d] = T(0);
                continue;
            }
            const uint64_t idx = (uint64_t)(a.index0 + s);
#pragma unroll
            for (int jd = 0; jd < kDimsPerLane; jd++) {
                const int d = lane + 32 * jd;
                if (d >= nm0) break;
                double y;
                if (!sobol) {
                    y = a.normals ? a.normals[s * nm0 + d] : (double)a.normals32[s * nm0 + d];
                } else {
                    if (s == s_first) st[jd] = sobol_state(a.vdir, nm0, d, idx);
                    else st[jd] ^= (uint64_t)__ldg(a.vdir + (size_t)(__ffsll((long long)idx) - 1) * nm0 + d);
                    const uint64_t x = a.shift ? st[jd] ^ __ldg(a.shift + d) : st[jd];
                    y = bsm(sobol_uniform(x));
                }
                q[d] = (T)(y / 1.4142135623730951);   // by /= sqrt(2.0)
            }
            for (int d = lane + 32 * kDimsPerLane; d < nm0; d += 32) {   // beyond 128 dimensions
                double y = sobol ? bsm(sobol_uniform((a.shift ? __ldg(a.shift + d) : 0ull) ^
                                                     sobol_state(a.vdir, nm0, d, idx)))
                                 : a.normals ? a.normals[s * nm0 + d] : (double)a.normals32[s * nm0 + d];
                q[d] = (T)(y / 1.4142135623730951);
            }
        }
        __syncwarp();
        // 2. r = bohr * (x0 + MUa q)   (SCP3.cpp:208), in the form's precision (FP64
        // for the plain form); a lane's two coordinates (c, c + 32) of every sample
        // of the group in one pass, each summed over k in order (samples past gn
        // compute stale values that are not used)
        if (mua_in_smem) {
            for (int g = 0; g < ng; g++) {
                const int c = 64 * g + lane;
                const T2* mg = mua2 + g * 32 + lane;
                const int kstride = ng * 32;
                T acc0[kGroup], acc1[kGroup];
#pragma unroll
                for (int j = 0; j < kGroup; j++) acc0[j] = acc1[j] = T(0);
                int k = 0;
                for (; k + 1 < nm0; k += 2) {
                    const T2 m0 = mg[k * kstride], m1 = mg[(k + 1) * kstride];
#pragma unroll
                    for (int j = 0; j < kGroup; j++) {
                        const T2 qq = reinterpret_cast<const T2*>(w.q + j * w.qs)[k >> 1];
                        acc0[j] += m0.x * qq.x;
                        acc1[j] += m0.y * qq.x;
                        acc0[j] += m1.x * qq.y;
                        acc1[j] += m1.y * qq.y;
                    }
                }
                if (k < nm0) {
                    const T2 m0 = mg[k * kstride];
#pragma unroll
                    for (int j = 0; j < kGroup; j++) {
                        const T qk = w.q[j * w.qs + k];
                        acc0[j] += m0.x * qk;
                        acc1[j] += m0.y * qk;
                    }
                }
                const T x0a = (T)(c < N3 ? __ldg(a.x0 + c) : 0.0), x0b = (T)(c + 32 < N3 ? __ldg(a.x0 + c + 32) : 0.0);
#pragma unroll
                for (int j = 0; j < kGroup; j++) {
                    if (j >= gn) break;
                    T* crd = w.crd + j * N3;
                    if (c < N3) crd[c] = (T)kBohr * (x0a + acc0[j]);
                    if (c + 32 < N3) crd[c + 32] = (T)kBohr * (x0b + acc1[j]);
                }
            }
        } else {
            for (int j = 0; j < gn; j++) {
                const T* q = w.q + j * w.qs;
                T* crd = w.crd + j * N3;
                for (int c = lane; c < N3; c += 64) {
                    const bool two = c + 32 < N3;
                    double acc0 = 0.0, acc1 = 0.0;
#pragma unroll 4
                    for (int k = 0; k < nm0; k++) {
                        const double qk = (double)q[k];
                        acc0 += MUa[(size_t)k * N3 + c] * qk;
                        if (two) acc1 += MUa[(size_t)k * N3 + c + 32] * qk;
                    }
                    crd[c] = (T)(kBohr * (__ldg(a.x0 + c) + acc0));
                    if (two) crd[c + 32] = (T)(kBohr * (__ldg(a.x0 + c + 32) + acc1));
                }
            }
        }
        __syncwarp();
        // qTIP4P/f energies of the whole group in one warp pass
        double e4 = 0.0;
        if constexpr (PES == SCP3GPU_PES_QTIP4PF) {
            if (!a.skip_pes && !grad) e4 = qt::energy_warp4<T>(w.crd, N3, w.ms, nw, gn, lane);
        }
        if constexpr (PES == SCP3GPU_PES_QTIP4PF && sizeof(T) == 4) {
            if (grad) {
                // FP32 gradient path (the split form's products): energies and
                // gradients of the group in one warp pass, then dV_anh/dq of the
                // group's (sample, mode) items over the lanes, summed in FP64
                T* g4 = reinterpret_cast<T*>(w.g);
                T* gm4 = g4 + 4 * 9 * nw;
                e4 = qt::energy_grad_warp4<T>(w.crd, N3, w.ms, g4, gm4, nw, gn, lane);
                for (int it = lane; it < gn * a.nm; it += 32) {
                    const int j = it / a.nm, m = it - j * a.nm;
                    const int k = __ldg(a.modes + m);
                    const T* gj = g4 + j * 9 * nw;
                    double acc = 0.0;
                    if (muat_in_smem)
                        for (int c = 0; c < N3; c++) acc += muat[(size_t)c * a.nm + m] * (double)gj[c];
                    else
                        for (int c = 0; c < N3; c++) acc += MUa[(size_t)k * N3 + c] * (double)gj[c];
                    a.vq[(s0 + j) * a.nm + m] =
                        acc * (kBohr / kAuToKcalPerMol) - __ldg(a.omega + k) * (double)w.q[j * w.qs + k];
                }
                __syncwarp();
            }
        }
        for (int j = 0; j < gn; j++) {
            const int64_t s = s0 + j;
            const T* q = w.q + j * w.qs;
            const T* crd = w.crd + j * N3;
            const double e4j = __shfl_sync(0xffffffffu, e4, j);
            if (s >= a.nvalid) {
                if (lane == 0) a.v[s] = 0.0;
                for (int m = lane; m < a.nm; m += 32) {
                    if (a.q64) a.q64[s * a.nm + m] = 0.0;
                    if (a.q32) a.q32[s * a.nm + m] = 0.0f;
                    if (a.vq) a.vq[s * a.nm + m] = 0.0;
                }
                continue;
            }
            // 3. V in hartree, anharmonic residual   (SCP3.cpp:219-223)
            int iters = 0;
            double V = 0.0;
            if constexpr (sizeof(T) == 8) {
                if (grad) {
                    // gradient path (SCP3.cpp:209-216): V and dV/dr, then
                    // dV_anh/dq = MUa^T (bohr dV/dr / autokcal) - omega % q, selected modes
                    double e;
                    if constexpr (PES == SCP3GPU_PES_QTIP4PF)
                        e = qt::energy_grad_warp(reinterpret_cast<const double*>(crd),
                                                 reinterpret_cast<double*>(w.ms), w.g, w.gm, nw, a.tasks, a.ntasks,
                                                 lane);
                    else
                        e = ttm::energy_grad_warp(reinterpret_cast<const double*>(crd),
                                                  reinterpret_cast<double*>(w.ms), reinterpret_cast<double*>(w.ttm),
                                                  w.g, nw, a.tasks, a.ntasks, lane, &iters);
                    double h = 0.0;
                    for (int d = lane; d < nm0; d += 32) h += (double)q[d] * (__ldg(a.omega + d) * (double)q[d]);
                    h = warp_sum(h);
                    V = e / kAuToKcalPerMol - 0.5 * h;
                    for (int m = lane; m < a.nm; m += 32) {
                        const int k = __ldg(a.modes + m);
                        double acc = 0.0;
                        if (muat_in_smem)
                            for (int c = 0; c < N3; c++) acc += muat[(size_t)c * a.nm + m] * w.g[c];
                        else
                            for (int c = 0; c < N3; c++) acc += MUa[(size_t)k * N3 + c] * w.g[c];
                        a.vq[s * a.nm + m] = acc * (kBohr / kAuToKcalPerMol) - __ldg(a.omega + k) * (double)q[k];
                    }
                }
            } else if constexpr (PES == SCP3GPU_PES_QTIP4PF) {
                if (grad) {
                    // the FP32 form: the group's energies and dV/dq came from the
                    // group pass above
                    double h = 0.0;
                    for (int d = lane; d < nm0; d += 32) h += (double)q[d] * (__ldg(a.omega + d) * (double)q[d]);
                    h = warp_sum(h);
                    V = e4j / kAuToKcalPerMol - 0.5 * h;
                }
            }
            if (!a.skip_pes && !grad) {
                const double e = PES == SCP3GPU_PES_QTIP4PF ? e4j
                                                             : potential<PES, T>(crd, w, nw, a.tasks, a.ntasks, lane, &iters);
                double h = 0.0;
                for (int d = lane; d < nm0; d += 32) h += (double)q[d] * (__ldg(a.omega + d) * (double)q[d]);
                h = warp_sum(h);
                V = e / kAuToKcalPerMol - 0.5 * h;
            }
            if (lane == 0) {
                a.v[s] = V;
                if (!isfinite(V)) atomicAdd(a.counters + 0, 1ull);
                if (iters > kTtmMaxIter) atomicAdd(a.counters + 1, 1ull);
            }
            // 4. selected modes, coalesced per sample
            for (int m = lane; m < a.nm; m += 32) {
                const T qm = q[__ldg(a.modes + m)];
                if (a.q64) a.q64[s * a.nm + m] = (double)qm;
                if (a.q32) a.q32[s * a.nm + m] = (float)qm;
            }
            __syncwarp();
        }
    }
}

template <int PES>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
    pes_energy_kernel(int nw, int64_t n, const double* __restrict__ crd, double* __restrict__ E,
                      int* __restrict__ iters_out, const uint32_t* __restrict__ tasks, int ntasks)
{
    extern __shared__ __align__(16) char smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    WarpSlot<double> w = warp_slot<double>(smem + wib * slot_bytes<double>(PES, 0, nw), PES, 0, nw);
    const int64_t nwarps = (int64_t)gridDim.x * kWarpsPerBlock;
    for (int64_t g = (int64_t)blockIdx.x * kWarpsPerBlock + wib; g < n; g += nwarps) {
        for (int c = lane; c < 9 * nw; c += 32) w.crd[c] = crd[g * 9 * nw + c];
        __syncwarp();
        int iters = 0;
        const double e = potential<PES, double>(w.crd, w, nw, tasks, ntasks, lane, &iters);
        if (lane == 0) {
            E[g] = e;
            if (iters_out) iters_out[g] = iters;
        }
        __syncwarp();
    }
}

// qTIP4P/f energy and gradient of n geometries, one warp each (the E+g operator,
// qtip4pf.cpp:252-397).
template <int PES>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
    pes_energy_grad_kernel(int nw, int64_t n, const double* __restrict__ crd, double* __restrict__ E,
                           double* __restrict__ G, int* __restrict__ iters_out, const uint32_t* __restrict__ tasks,
                           int ntasks)
{
    extern __shared__ __align__(16) double gsm[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const size_t per = 24 * (size_t)nw + (PES == SCP3GPU_PES_TTM3F ? ttm::scratch_elems(nw, true) : 0);
    double* x = gsm + (size_t)wib * per;
    double *ms = x + 9 * nw, *g = ms + 3 * nw, *gm = g + 9 * nw, *sc = gm + 3 * nw;
    const int64_t nwarps = (int64_t)gridDim.x * kWarpsPerBlock;
    for (int64_t k = (int64_t)blockIdx.x * kWarpsPerBlock + wib; k < n; k += nwarps) {
        for (int c = lane; c < 9 * nw; c += 32) x[c] = crd[k * 9 * nw + c];
        __syncwarp();
        int iters = 0;
        double e;
        if constexpr (PES == SCP3GPU_PES_QTIP4PF) e = qt::energy_grad_warp(x, ms, g, gm, nw, tasks, ntasks, lane);
        else e = ttm::energy_grad_warp(x, ms, sc, g, nw, tasks, ntasks, lane, &iters);
        if (lane == 0) {
            E[k] = e;
            if (iters_out) iters_out[k] = iters;
        }
        for (int c = lane; c < 9 * nw; c += 32) G[k * 9 * nw + c] = g[c];
        __syncwarp();
    }
}

// SCP1 per-sample stage (SCP1.cpp:52-63): one warp per sample, contiguous
// balanced ranges per warp with the Gray-code Sobol walk, isqrtM_U staged in
// shared memory, the potential's energy and gradient (the gradient estimator's
// warp code).
constexpr int kS1Warps = 8;

__host__ __device__ inline size_t scp1_slot(int pes, int nw, int dim)
{
    return 2 * (size_t)dim + 24 * (size_t)nw + (pes == SCP3GPU_PES_TTM3F ? ttm::scratch_elems(nw, true) : 0);
}

template <int PES>
__global__ void __launch_bounds__(kS1Warps * 32) scp1_samples_kernel(Scp1Args a)
{
    extern __shared__ __align__(16) double s1[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int nw = a.nw, dim = a.dim;
    double* U = s1;
    for (int e = threadIdx.x; e < dim * dim; e += blockDim.x) U[e] = a.U[e];
    double* y = s1 + (size_t)dim * dim + (size_t)wib * scp1_slot(PES, nw, dim);
    double* dq = y + dim;
    double* x = dq + dim;
    double* ms = x + 9 * nw;
    double* g = ms + 3 * nw;
    double* gm = g + 9 * nw;
    double* sc = gm + 3 * nw;
    __syncthreads();
    const int64_t nwarps = (int64_t)gridDim.x * kS1Warps;
    const int64_t gw = (int64_t)blockIdx.x * kS1Warps + wib;
    const int64_t s_first = a.n * gw / nwarps, s_end = a.n * (gw + 1) / nwarps;
    constexpr int kDimsPerLane = 4;
    uint64_t st[kDimsPerLane];
    for (int64_t s = s_first; s < s_end; s++) {
        const uint64_t idx = (uint64_t)(a.index0 + s);
        // y = std_normal % sqrt(d)   (SCP1.cpp:54-58)
#pragma unroll
        for (int jd = 0; jd < kDimsPerLane; jd++) {
            const int d = lane + 32 * jd;
            if (d >= dim) break;
            if (s == s_first) st[jd] = sobol_state(a.vdir, dim, d, idx);
            else st[jd] ^= (uint64_t)__ldg(a.vdir + (size_t)(__ffsll((long long)idx) - 1) * dim + d);
            y[d] = bsm(sobol_uniform(st[jd])) * __ldg(a.sqd + d);
        }
        for (int d = lane + 32 * kDimsPerLane; d < dim; d += 32)
            y[d] = bsm(sobol_uniform(sobol_state(a.vdir, dim, d, idx))) * __ldg(a.sqd + d);
        __syncwarp();
        // dq = isqrtM_U y, r = bohr (q + dq)   (SCP1.cpp:60-61), k in order
        for (int c = lane; c < dim; c += 32) {
            double acc = 0.0;
            for (int k = 0; k < dim; k++) acc += U[(size_t)k * dim + c] * y[k];
            dq[c] = acc;
            x[c] = kBohr * (__ldg(a.q + c) + acc);
        }
        __syncwarp();
        int it = 0;
        double e;
        if constexpr (PES == SCP3GPU_PES_QTIP4PF)
            e = qt::energy_grad_warp(x, ms, g, gm, nw, a.tasks, a.ntasks, lane);
        else
            e = ttm::energy_grad_warp(x, ms, sc, g, nw, a.tasks, a.ntasks, lane, &it);
        if (lane == 0) {
            a.V[s] = e / kAuToKcalPerMol;
            if (a.iters) a.iters[s] = it;
        }
        for (int c = lane; c < dim; c += 32) {
            a.G[s * dim + c] = g[c] * (kBohr / kAuToKcalPerMol);    // UX_ *= bohr/autokcalpmol
            a.D[s * dim + c] = dq[c];
        }
        __syncwarp();
    }
}

__global__ void std_normal_kernel(int dims, int64_t index0, int64_t n, const int64_t* __restrict__ vdir,
                                  const uint64_t* __restrict__ shift, double* __restrict__ out)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * dims) return;
    const int64_t s = t / dims;
    const int d = (int)(t - s * dims);
    uint64_t x = sobol_state(vdir, dims, d, (uint64_t)(index0 + s));
    if (shift) x ^= shift[d];
    out[t] = bsm(sobol_uniform(x));
}

// Blocks of the per-sample kernel: one warp per kMinRun samples at least, and
// no more blocks than the SMs hold at once.
template <typename K>
int sample_grid(K kern, size_t smem, int64_t n)
{
    int dev = 0, sms = 148, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kWarpsPerBlock * 32, smem) != cudaSuccess || per < 1)
        per = 1;
    const int64_t want = (n + (int64_t)kMinRun * kWarpsPerBlock - 1) / ((int64_t)kMinRun * kWarpsPerBlock);
    const int64_t cap = (int64_t)per * sms;
    return (int)std::max<int64_t>(1, std::min(want, cap));
}

int grid_for(int64_t nwarps_needed)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int64_t blocks = (nwarps_needed + kWarpsPerBlock - 1) / kWarpsPerBlock;
    const int64_t cap = (int64_t)sms * 8;
    return (int)(blocks < cap ? (blocks > 0 ? blocks : 1) : cap);
}

template <int PES, typename T>
int launch_samples_t(const SampleArgs& a, cudaStream_t s)
{
    const size_t mua_b = mua_smem_bytes<T>(a.nw, a.nm0);
    const size_t muat_b = muat_smem_bytes(a.nw, a.nm);
    const size_t sm = kWarpsPerBlock * slot_bytes<T>(PES, a.nm0, a.nw, a.vq != nullptr, kGroup) +
                      (mua_b <= kMuaSmemMax ? mua_b : 0) + (a.vq && muat_b <= kMuaTSmemMax ? muat_b : 0);
    auto kern = a.vq ? samples_kernel<PES, T, true> : samples_kernel<PES, T, false>;
    if (sm > 48 * 1024) SCP3_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    kern<<<sample_grid(kern, sm, a.n), kWarpsPerBlock * 32, sm, s>>>(a);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

template <int PES, typename T>
int launch_samples_batch_t(const SampleArgs* args_host, const SampleArgs* args_dev, int ncl, int64_t n, cudaStream_t s)
{
    // Shared memory for the largest cluster: warp slots of the largest (nm0, nw)
    // plus the largest MUa that a cluster stages (each cluster decides as the
    // single-cluster kernel does, so its layout fits).
    int nm0 = 0, nw = 0;
    size_t mua = 0;
    for (int c = 0; c < ncl; c++) {
        nm0 = std::max(nm0, args_host[c].nm0);
        nw = std::max(nw, args_host[c].nw);
        const size_t b = mua_smem_bytes<T>(args_host[c].nw, args_host[c].nm0);
        if (b <= kMuaSmemMax) mua = std::max(mua, b);
    }
    const size_t sm = kWarpsPerBlock * slot_bytes<T>(PES, nm0, nw, false, kGroup) + mua;
    if (sm > 48 * 1024) SCP3_CUDA(cudaFuncSetAttribute(samples_batch_kernel<PES, T>,
                                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    const int per = grid_for((n + kRun - 1) / kRun);   // per cluster; the clusters share the SMs
    samples_batch_kernel<PES, T><<<dim3((unsigned)per, (unsigned)ncl), kWarpsPerBlock * 32, sm, s>>>(args_dev);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

}  // namespace

int launch_samples_batch(int pes, bool fp32, const SampleArgs* args_host, const SampleArgs* args_dev, int ncl,
                         int64_t n, cudaStream_t s)
{
    if (n <= 0 || ncl <= 0) return SCP3GPU_OK;
    if (pes == SCP3GPU_PES_QTIP4PF)
        return fp32 ? launch_samples_batch_t<SCP3GPU_PES_QTIP4PF, float>(args_host, args_dev, ncl, n, s)
                    : launch_samples_batch_t<SCP3GPU_PES_QTIP4PF, double>(args_host, args_dev, ncl, n, s);
    if (pes == SCP3GPU_PES_TTM3F)
        return fp32 ? launch_samples_batch_t<SCP3GPU_PES_TTM3F, float>(args_host, args_dev, ncl, n, s)
                    : launch_samples_batch_t<SCP3GPU_PES_TTM3F, double>(args_host, args_dev, ncl, n, s);
    return fail(SCP3GPU_ERR_ARG, "unknown potential id");
}

int ttm_init_device()
{
    static std::mutex mu;
    static bool done[128] = {false};
    int dev = 0;
    SCP3_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 0 || dev >= 128) return fail(SCP3GPU_ERR_ARG, "device ordinal out of range");
    if (done[dev]) return SCP3GPU_OK;
    ttm::Consts c;
    c.AA_HH = std::pow(0.496 * 0.496, 1.0 / 6.0);
    c.AA_HM = std::pow(0.496 * 0.837, 1.0 / 6.0);
    c.AA_MM = std::pow(0.837 * 0.837, 1.0 / 6.0);
    c.aXX13 = std::pow(0.175, 1.0 / 3.0);
    for (int i = 0; i < 245; i++)   // ps.cpp:508-511: f5z, fbasis, fcore, frest
        c.c5z[i] = 0.999677885 * scp3_ps_c5zA[i] + 0.15860145369897 * scp3_ps_cbasis[i] +
                   -1.6351695982132 * scp3_ps_ccore[i] + 1.0 * scp3_ps_crest[i];
    c.phh1 = 0.999677885 * 16.94879431193463 * std::exp(12.66426998162947);
    for (int i = 0; i < 84; i++) c.coefD[i] = scp3_ps_coefD[i];
    for (int i = 0; i < 245; i++) {
        c.idx1[i] = scp3_ps_idx1[i];
        c.idx2[i] = scp3_ps_idx2[i];
        c.idx3[i] = scp3_ps_idx3[i];
    }
    for (int i = 0; i < 84; i++) {
        c.idxD0[i] = scp3_ps_idxD0[i];
        c.idxD1[i] = scp3_ps_idxD1[i];
        c.idxD2[i] = scp3_ps_idxD2[i];
    }
    SCP3_CUDA(cudaMemcpyToSymbol(ttm::kC, &c, sizeof(c)));
    done[dev] = true;
    return SCP3GPU_OK;
}

int launch_samples(int pes, bool fp32, const SampleArgs& a, cudaStream_t s)
{
    if (a.n <= 0) return SCP3GPU_OK;
    if (a.vq && fp32 && pes != SCP3GPU_PES_QTIP4PF)
        return fail(SCP3GPU_ERR_UNSUPPORTED, "gradient path: FP32 potential for qTIP4P/f only");
    if (pes == SCP3GPU_PES_QTIP4PF)
        return fp32 ? launch_samples_t<SCP3GPU_PES_QTIP4PF, float>(a, s)
                    : launch_samples_t<SCP3GPU_PES_QTIP4PF, double>(a, s);
    if (pes == SCP3GPU_PES_TTM3F)
        return fp32 ? launch_samples_t<SCP3GPU_PES_TTM3F, float>(a, s)
                    : launch_samples_t<SCP3GPU_PES_TTM3F, double>(a, s);
    return fail(SCP3GPU_ERR_ARG, "unknown potential id");
}

int launch_pes_energy_grad(int pes, int nw, int64_t n, const double* crd, double* E, double* G, int* iters,
                           const uint32_t* tasks, int ntasks, cudaStream_t s)
{
    if (n <= 0) return SCP3GPU_OK;
    const bool ttm = pes == SCP3GPU_PES_TTM3F;
    const size_t per = 24 * (size_t)nw + (ttm ? ttm::scratch_elems(nw, true) : 0);
    const size_t sm = sizeof(double) * kWarpsPerBlock * per;
    auto kern = ttm ? pes_energy_grad_kernel<SCP3GPU_PES_TTM3F> : pes_energy_grad_kernel<SCP3GPU_PES_QTIP4PF>;
    if (sm > 48 * 1024) SCP3_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    kern<<<grid_for(n), kWarpsPerBlock * 32, sm, s>>>(nw, n, crd, E, G, iters, tasks, ntasks);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

int launch_scp1_samples(int pes, const Scp1Args& a, cudaStream_t s)
{
    if (a.n <= 0) return SCP3GPU_OK;
    if (pes != SCP3GPU_PES_QTIP4PF && pes != SCP3GPU_PES_TTM3F) return fail(SCP3GPU_ERR_ARG, "unknown potential id");
    const size_t sm = sizeof(double) * ((size_t)a.dim * a.dim + kS1Warps * scp1_slot(pes, a.nw, a.dim));
    auto kern = pes == SCP3GPU_PES_QTIP4PF ? scp1_samples_kernel<SCP3GPU_PES_QTIP4PF>
                                            : scp1_samples_kernel<SCP3GPU_PES_TTM3F>;
    SCP3_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int dev = 0, sms = 148, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kS1Warps * 32, sm) != cudaSuccess || per < 1) per = 1;
    const int64_t want = (a.n + 4 * kS1Warps - 1) / (4 * kS1Warps);     // >= 4 samples per warp
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)per * sms));
    kern<<<grid, kS1Warps * 32, sm, s>>>(a);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

int launch_pes_energy(int pes, int nw, int64_t n, const double* crd, double* E, int* iters, const uint32_t* tasks,
                      int ntasks, cudaStream_t s)
{
    if (n <= 0) return SCP3GPU_OK;
    const size_t sm = kWarpsPerBlock * slot_bytes<double>(pes, 0, nw);
    if (pes == SCP3GPU_PES_QTIP4PF) {
        pes_energy_kernel<SCP3GPU_PES_QTIP4PF><<<grid_for(n), kWarpsPerBlock * 32, sm, s>>>(nw, n, crd, E, iters,
                                                                                          tasks, ntasks);
    } else if (pes == SCP3GPU_PES_TTM3F) {
        if (sm > 48 * 1024)
            SCP3_CUDA(cudaFuncSetAttribute(pes_energy_kernel<SCP3GPU_PES_TTM3F>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        pes_energy_kernel<SCP3GPU_PES_TTM3F><<<grid_for(n), kWarpsPerBlock * 32, sm, s>>>(nw, n, crd, E, iters,
                                                                                        tasks, ntasks);
    } else {
        return fail(SCP3GPU_ERR_ARG, "unknown potential id");
    }
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

int launch_std_normal(int dims, int64_t index0, int64_t n, const int64_t* vdir, const uint64_t* shift, double* out,
                      cudaStream_t s)
{
    const int64_t total = n * dims;
    if (total <= 0) return SCP3GPU_OK;
    std_normal_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(dims, index0, n, vdir, shift, out);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

}  // namespace scp3

// Host-only view of the water-pair items of the four-sample qTIP4P/f kernels, for
// tests: ab[2 p], ab[2 p + 1] = the waters a < b of pair p, p < nw (nw - 1) / 2.
extern "C" int scp3gpu_internal_water_pairs(int nw, int* ab)
{
    if (nw < 1 || nw > 64 || !ab) return SCP3GPU_ERR_ARG;
    const int np = nw * (nw - 1) / 2;
    for (int p = 0; p < np; p++) scp3::qt::water_pair_of(p, nw, ab[2 * p], ab[2 * p + 1]);
    return SCP3GPU_OK;
}
