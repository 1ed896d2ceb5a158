// The gradient (default) estimator of SCP3: addEpot(q, V, Vq, M)
// (ScaledMatrixElements.cpp:102-725 with the formulas of TripleExcitations.h),
// FP64, as dense products on the FP64 pipe.
//
// Every formula of the reference follows one rule.  For the pair (i, j) let S be
// the modes either function excites and p_m(q_m) = h_a(q_m) h_b(q_m) the
// product of their oscillator factors in mode m (levels a, b).  Writing
// p_m = p_m(0) + q_m r_m(q_m), the Stein identity E[q g(q)] = E[g'(q)] / 2
// (q ~ N(0, 1/2)) moves one power of q_m onto V:
//     T_m = prod_{m' != m} p_m' * [ (p_m(0) + r_m'/2) V + (r_m / 2) dV/dq_m ],
// and the estimate of <i|V|j> is the mean of T_m over m in S (<0|V|0>: V).
// With d_a = (h_a - h_a(0)) / q, r_ab = d_a h_b + h_a(0) d_b, so every factor is
// a short polynomial in q_m.  One formula of the reference departs from the
// rule and is reproduced as written: <3_m|V|3_m> (TripleExcitations.h:763-773)
// carries (q^2 - 3) V where the identity gives (10 q^2 - 3) V.
//
// As products.  prod_{m' != m} p_m' = R_i^m R_j^m, where R_i^m is function i
// without its mode-m factor, and the bracket is K^m_ab = u_ab(q_m) V + w_ab(q_m)
// dV/dq_m, which depends on the pair only through the levels (a, b) of i and j
// in mode m.  When j does not excite m (b = 0), R_j^m = Phi_j, so
//     T^m_ij = sum_s [R_i^m K^m_a0](s) Phi_j(s)
// is one row of a product W Phi^T, with one "virtual row" W_(m,i) = R_i^m K^m_a0
// per (mode, function exciting it): 2352 rows against 1225 columns for the
// hexamer doubles basis, an FP64 GEMM (contract_fp64.cu, rectangular form).
// When both excite m, T^m_ij = sum_s R_i^m R_j^m K^m_ab is a pair sum over the
// functions exciting m, kept per mode (stein_pairs_kernel; 48 x 49^2 pairs for
// the hexamer doubles basis against 48 x 49 x 1225 products in the GEMM).  The
// read-out forms each element from its |S| <= 6 terms and divides by |S|;
// <0|V|0> comes from one more virtual row, W = V, against Phi_0 = 1.
//
// Every sum runs over samples in a fixed order per (split, tile) and the splits
// are added in order at read-out, so results are deterministic.
#include <cuda_bf16.h>

#include <algorithm>
#include <array>
#include <map>

#include "internal.h"
#include "tc.h"

namespace scp3 {

namespace {

// (mode, level) list of a basis descriptor (kind | m << 3 | n << 11 | p << 19)
__host__ __device__ __forceinline__ int decode(uint32_t d, int* m, int* l)
{
    const int kind = (int)(d & 7u), a = (int)((d >> 3) & 255u), b = (int)((d >> 11) & 255u), c = (int)(d >> 19);
    switch (kind) {
        case kGround: return 0;
        case kHo1: m[0] = a, l[0] = 1; return 1;
        case kHo2: m[0] = a, l[0] = 2; return 1;
        case kHo1Ho1: m[0] = a, l[0] = 1, m[1] = b, l[1] = 1; return 2;
        case kHo3: m[0] = a, l[0] = 3; return 1;
        case kHo2Ho1: m[0] = a, l[0] = 2, m[1] = b, l[1] = 1; return 2;
        case kHo1Ho2: m[0] = a, l[0] = 1, m[1] = b, l[1] = 2; return 2;
        default: m[0] = a, l[0] = 1, m[1] = b, l[1] = 1, m[2] = c, l[2] = 1; return 3;
    }
}

// h_l(q) (HarmonicOscillatorBasis.cpp: 1, sqrt2 q, (2q^2 - 1)/sqrt2, (2q^3 - 3q)/sqrt3)
__device__ __forceinline__ double ho(int l, double q)
{
    switch (l) {
        case 0: return 1.0;
        case 1: return 1.4142135623730951 * q;
        case 2: return (2.0 * q * q - 1.0) * 0.70710678118654752;
        default: return (2.0 * q * q - 3.0) * q * 0.57735026918962576;
    }
}

// h_a(q), h_a(0), h_a'(q), d_a(q), d_a'(q) for the oscillator functions h_0..h_3
__device__ __forceinline__ void ho_parts(int a, double q, double& h, double& h0, double& dh, double& d, double& dd)
{
    constexpr double s2 = 1.4142135623730951, is2 = 0.70710678118654752, is3 = 0.57735026918962576;
    switch (a) {
        case 0: h = 1, h0 = 1, dh = 0, d = 0, dd = 0; break;
        case 1: h = s2 * q, h0 = 0, dh = s2, d = s2, dd = 0; break;
        case 2: h = (2 * q * q - 1) * is2, h0 = -is2, dh = 2 * s2 * q, d = s2 * q, dd = s2; break;
        default: h = (2 * q * q - 3) * q * is3, h0 = 0, dh = (6 * q * q - 3) * is3, d = (2 * q * q - 3) * is3,
                 dd = 4 * q * is3; break;
    }
}

// K_ab = u V + w dV/dq_m for mode m at q_m = x, levels (a, b)
__device__ __forceinline__ double stein_weight(int a, int b, double x, double V, double Vm)
{
    double ha, ha0, dha, da, dda, hb, hb0, dhb, db, ddb;
    ho_parts(a, x, ha, ha0, dha, da, dda);
    ho_parts(b, x, hb, hb0, dhb, db, ddb);
    const double r = da * hb + ha0 * db;
    const double dr = dda * hb + da * dhb + ha0 * ddb;
    double u = ha0 * hb0 + 0.5 * dr;
    const double w = 0.5 * r;
    if (a == 3 && b == 3) u = (2 * x * x - 3) * (x * x - 3) * (1.0 / 6.0);   // TripleExcitations.h:763-773
    return u * V + w * Vm;
}

// Virtual row descriptor: m | a << 8 | m1 << 10 | l1 << 18 | m2 << 20 | l2 << 28,
// (m1, l1), (m2, l2) the function's other factors (level 0: none); bit 30: the
// ground row (W = V).
constexpr uint32_t kGroundRow = 1u << 30;

__device__ __forceinline__ double reduced(uint32_t vd, const double* qs, int stride, int j)
{
    const int m1 = (vd >> 10) & 255, l1 = (vd >> 18) & 3, m2 = (vd >> 20) & 255, l2 = (vd >> 28) & 3;
    double r = 1.0;
    if (l1) r *= ho(l1, qs[m1 * stride + j]);
    if (l2) r *= ho(l2, qs[m2 * stride + j]);
    return r;
}

constexpr int kExpS = 64, kExpR = 128;
constexpr int kExpLd = kExpS + 1;   // odd row stride of the staged q: a warp's rows read different modes conflict-free

// Phi [s][j] (ld nb_pad) and W [s][r] (ld nv_pad) for 64 samples; one thread per
// row of the stacked [Phi rows | W rows], coalesced 1 KB stores per sample.
__global__ void __launch_bounds__(kExpR) stein_expand_kernel(const uint32_t* __restrict__ desc, int nb, int nb_pad,
                                                             const uint32_t* __restrict__ vrdesc, int nv,
                                                             int nv_pad, int nm, const double* __restrict__ q,
                                                             const double* __restrict__ v,
                                                             const double* __restrict__ vq, int64_t n,
                                                             double* __restrict__ Phi, double* __restrict__ W)
{
    extern __shared__ double st[];          // q [nm][65], vq [nm][65], V [64]
    double* qs = st;
    double* vqs = st + (size_t)nm * kExpLd;
    double* vs = vqs + (size_t)nm * kExpLd;
    const int t = threadIdx.x;
    const int64_t s0 = (int64_t)blockIdx.x * kExpS;
    for (int e = t; e < nm * kExpS; e += kExpR) {
        const int ss = e / nm, m = e - ss * nm;          // coalesced reads of row s0 + ss
        const bool ok = s0 + ss < n;
        qs[m * kExpLd + ss] = ok ? q[(s0 + ss) * nm + m] : 0.0;
        vqs[m * kExpLd + ss] = ok ? vq[(s0 + ss) * nm + m] : 0.0;
    }
    for (int ss = t; ss < kExpS; ss += kExpR) vs[ss] = s0 + ss < n ? v[s0 + ss] : 0.0;
    __syncthreads();
    const int ns = (int)min((int64_t)kExpS, n - s0);
    const int row = blockIdx.y * kExpR + t;
    if (row < nb_pad) {
        int mm[3], ll[3], k = 0;
        if (row < nb) k = decode(__ldg(desc + row), mm, ll);
        for (int j = 0; j < ns; j++) {
            double x = row < nb ? 1.0 : 0.0;
            for (int u = 0; u < k; u++) x *= ho(ll[u], qs[mm[u] * kExpLd + j]);
            Phi[(size_t)(s0 + j) * nb_pad + row] = x;
        }
    } else {
        const int r = row - nb_pad;
        const uint32_t vd = r < nv ? __ldg(vrdesc + r) : 0u;
        const int m = vd & 255, a = (vd >> 8) & 3;
        for (int j = 0; j < ns; j++) {
            double x = 0.0;
            if (r < nv) {
                if (vd & kGroundRow) x = vs[j];
                else x = reduced(vd, qs, kExpLd, j) *
                         stein_weight(a, 0, qs[m * kExpLd + j], vs[j], vqs[m * kExpLd + j]);
            }
            W[(size_t)(s0 + j) * nv_pad + r] = x;
        }
    }
}

// Split form: x = hi + lo in BF16 for two values, each half packed in one
// 32-bit word (the first value in the low 16 bits), round-to-nearest.
__device__ __forceinline__ void split_bf16x2(float x0, float x1, uint32_t& hi, uint32_t& lo)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
    const float2 hf = __bfloat1622float2(h);
    const __nv_bfloat162 l = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = *reinterpret_cast<const uint32_t*>(&l);
}

constexpr int kSxSlots = 32, kSxThreads = 256, kSxLd = 33;
constexpr int kSxBlocksPerFlush = tc::kSlotsPerFlush / kSxSlots;   // 130: the last two hold only padding slots
constexpr uint32_t kSxZeroRow = 0xffffffffu;                        // padding row: never written
constexpr int kSxMaxTable = 1024;                                   // table rows (10-bit indices)

// Kinds of table rows (TableSpec: kind | a << 4 | b << 6 | mode << 8)
enum : uint32_t { kTOne = 0, kTHo = 1, kTKa0 = 2, kTV = 3, kTKab = 4 };

// h_a(q), h_a(0), h_a'(q), d_a(q), d_a'(q) in FP32 (as ho_parts)
__device__ __forceinline__ void ho_parts_f(int a, float q, float& h, float& h0, float& dh, float& d, float& dd)
{
    constexpr float s2 = 1.41421356f, is2 = 0.70710678f, is3 = 0.57735027f;
    switch (a) {
        case 0: h = 1, h0 = 1, dh = 0, d = 0, dd = 0; break;
        case 1: h = s2 * q, h0 = 0, dh = s2, d = s2, dd = 0; break;
        case 2: h = (2 * q * q - 1) * is2, h0 = -is2, dh = 2 * s2 * q, d = s2 * q, dd = s2; break;
        default: h = (2 * q * q - 3) * q * is3, h0 = 0, dh = (6 * q * q - 3) * is3, d = (2 * q * q - 3) * is3,
                 dd = 4 * q * is3; break;
    }
}

// K_ab in FP32 (as stein_weight, including the reference's <3|V|3> form)
__device__ __forceinline__ float stein_weight_f(int a, int b, float x, float V, float Vm)
{
    float ha, ha0, dha, da, dda, hb, hb0, dhb, db, ddb;
    ho_parts_f(a, x, ha, ha0, dha, da, dda);
    ho_parts_f(b, x, hb, hb0, dhb, db, ddb);
    const float r = da * hb + ha0 * db;
    const float dr = dda * hb + da * dhb + ha0 * ddb;
    float u = ha0 * hb0 + 0.5f * dr;
    const float w = 0.5f * r;
    if (a == 3 && b == 3) u = (2 * x * x - 3) * (x * x - 3) * (1.0f / 6.0f);   // TripleExcitations.h:763-773
    return u * V + w * Vm;
}

// level pair (a <= b, levels 1..3) -> 0..5: 11, 12, 13, 22, 23, 33
__host__ __device__ __forceinline__ int level_pair(int a, int b)
{
    const int lo = a < b ? a : b, hi = a < b ? b : a;
    return lo == 1 ? hi - 1 : lo == 2 ? hi + 1 : 5;
}

// Table entry of row r for slot l (0..31): slots 8g..8g+3 at 4g..4g+3 and
// 8g+4..8g+7 at 16+4g..16+4g+3, the two halves swapped on odd rows, so that the
// 4 threads of an operand row read 64 contiguous bytes per load and rows of
// different parity fall in different banks.
__device__ __forceinline__ int sx_col(int r, int l)
{
    return ((((l >> 2) & 1) << 4) ^ ((r & 1) << 4)) | ((l >> 3) << 2) | (l & 3);
}

// The split operand of a pass: the W rows (reduced function x Stein weight K^m_a0,
// and the ground row V) from row 0, the W_b rows (R_i^m K^m_ab) after them and the
// Phi rows last, as BF16 hi + lo in the 32-slot, 64-byte-swizzled boxes the
// tensor-core contraction reads ([row block][k-block][hi, lo][128 x 32], 16-byte
// chunk c of row r at c ^ ((r >> 1) & 3)).  K slot l of 4096-sample block f holds
// sample 4096 f + l (l < 4096); the block's last 64 slots and the padding rows
// are never written (zero since creation).
//
// Per 32-slot block the CTA tabulates in FP32 the entries the operand's rows use
// (tspec: 1, h_l(q_m), K^m_a0, V, K^m_ab; with b = 0 the Stein weights of
// stein_weight reduce to K_10 = Vm / sqrt2, K_20 = q Vm / sqrt2, K_30 = (2 q /
// sqrt3) V + (2 q^2 - 3) / (2 sqrt3) Vm); a warp fills one table row at a time, so
// its kind is uniform.  Every operand row is the product of three table entries
// (xdesc: three 10-bit indices, 0 = the constant 1).  The values are rounded to
// FP32 before the BF16 split in any case.  CTA: one 32-slot block x `per` rows;
// thread (g, r) writes slots 8g..8g+7 of rows 4r..4r+3, 4r+256..4r+259, ...: one
// 16-byte chunk of the hi box and one of the lo box each.
__global__ void __launch_bounds__(kSxThreads) stein_expand_split_kernel(
    const uint32_t* __restrict__ tspec, int trows, const uint32_t* __restrict__ xdesc, int rows, int nsum, int per,
    int nm, const double* __restrict__ q, const double* __restrict__ v, const double* __restrict__ vq, int64_t n,
    int64_t nkb_alloc, uint16_t* __restrict__ xop, float* __restrict__ spart)
{
    extern __shared__ __align__(16) float tx[];   // table [trows][32]; q, Vm [nm][33]; V [32]
    const int kb = blockIdx.x;
    const int f = kb / kSxBlocksPerFlush, lb = kb - f * kSxBlocksPerFlush;
    if (lb * kSxSlots >= tc::kFlush) return;
    const int t = threadIdx.x;
    const int64_t s0 = (int64_t)f * tc::kFlush + (int64_t)lb * kSxSlots;
    float* qs = tx + (size_t)trows * kSxSlots;
    float* vms = qs + (size_t)nm * kSxLd;
    float* vs = vms + (size_t)nm * kSxLd;
    for (int e = t; e < nm * kSxSlots; e += kSxThreads) {
        const int l = e / nm, m = e - l * nm;      // coalesced reads of sample s0 + l
        const bool ok = s0 + l < n;
        qs[m * kSxLd + l] = ok ? (float)q[(s0 + l) * nm + m] : 0.0f;
        vms[m * kSxLd + l] = ok ? (float)vq[(s0 + l) * nm + m] : 0.0f;
    }
    for (int l = t; l < kSxSlots; l += kSxThreads) vs[l] = s0 + l < n ? (float)v[s0 + l] : 0.0f;
    __syncthreads();
    for (int e = t; e < trows * kSxSlots; e += kSxThreads) {
        const int r = e / kSxSlots, l = e - r * kSxSlots;
        const uint32_t sp = __ldg(tspec + r);
        const int kind = sp & 15, a = (sp >> 4) & 3, b = (sp >> 6) & 3, m = sp >> 8;
        float val = 1.0f;
        if (kind == kTV) {
            val = vs[l];
        } else if (kind != kTOne) {
            const float x = qs[m * kSxLd + l];
            if (kind == kTHo) {
                const float x2 = 2.0f * x * x;
                val = a == 1 ? 1.41421356f * x : a == 2 ? (x2 - 1.0f) * 0.70710678f : (x2 - 3.0f) * x * 0.57735027f;
            } else if (kind == kTKa0) {
                const float vm = vms[m * kSxLd + l];
                val = a == 1 ? 0.70710678f * vm
                             : a == 2 ? 0.70710678f * x * vm
                                      : 1.15470054f * x * vs[l] + (2.0f * x * x - 3.0f) * 0.28867513f * vm;
            } else {
                val = stein_weight_f(a, b, x, vs[l], vms[m * kSxLd + l]);
            }
        }
        tx[r * kSxSlots + sx_col(r, l)] = val;
    }
    __syncthreads();
    const int g = t & 3, rl = t >> 2;
    const float4* tab4 = reinterpret_cast<const float4*>(tx);
    const int64_t box_k = kb;                                  // the block's 32-slot box
    auto rd = [&](uint32_t i, float4& lo4, float4& hi4) {
        const uint32_t sw = (i & 1u) << 2;                      // swapped halves (in float4 units)
        lo4 = tab4[i * (kSxSlots / 4) + (sw ^ 0u) + g];
        hi4 = tab4[i * (kSxSlots / 4) + (sw ^ 4u) + g];
    };
    const int r0 = blockIdx.y * per, r1 = min(rows + nsum, r0 + per);
    // four consecutive rows per thread: consecutive rows mostly share their first
    // factor (the weight K^m of one mode and level, or the first Hermite factor of
    // a pair), read once
    for (int rb = r0 + 4 * rl; rb < r1; rb += kSxThreads) {
        uint32_t pia = 0xffffffffu;
        float4 f0 = make_float4(0.f, 0.f, 0.f, 0.f), f1 = f0;
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int row = rb + u;
            if (row >= r1) break;
            const uint32_t d = __ldg(xdesc + row);
            const bool has = d != kSxZeroRow;
            float4 a0 = f0, a1 = f1;
            if (has) {
                const uint32_t ia = d & 1023u, ib = (d >> 10) & 1023u, ic = d >> 20;
                if (ia != pia) {
                    rd(ia, f0, f1);
                    pia = ia;
                }
                a0 = f0, a1 = f1;
                if (ib) {
                    float4 b0, b1;
                    rd(ib, b0, b1);
                    a0.x *= b0.x, a0.y *= b0.y, a0.z *= b0.z, a0.w *= b0.w;
                    a1.x *= b1.x, a1.y *= b1.y, a1.z *= b1.z, a1.w *= b1.w;
                }
                if (ic) {
                    float4 c0, c1;
                    rd(ic, c0, c1);
                    a0.x *= c0.x, a0.y *= c0.y, a0.z *= c0.z, a0.w *= c0.w;
                    a1.x *= c1.x, a1.y *= c1.y, a1.z *= c1.z, a1.w *= c1.w;
                }
            }
            if (row >= rows) {
                // a summed row: its 32 values added, in FP32, into this block's partial
                float x = has ? ((a0.x + a0.y) + (a0.z + a0.w)) + ((a1.x + a1.y) + (a1.z + a1.w)) : 0.0f;
                const unsigned grp = 0xfu << (threadIdx.x & 28);     // the 4 lanes of this row
                x += __shfl_xor_sync(grp, x, 1);
                x += __shfl_xor_sync(grp, x, 2);
                if (g == 0) spart[(size_t)kb * nsum + (row - rows)] = x;
                continue;
            }
            if (!has) continue;
            uint4 hi, lo;
            split_bf16x2(a0.x, a0.y, hi.x, lo.x);
            split_bf16x2(a0.z, a0.w, hi.y, lo.y);
            split_bf16x2(a1.x, a1.y, hi.z, lo.z);
            split_bf16x2(a1.z, a1.w, hi.w, lo.w);
            const int rin = row & (tc::kTile - 1);
            uint16_t* box = xop + ((size_t)(row / tc::kTile) * nkb_alloc + box_k) * (2 * tc::kTile * tc::kKBlock2);
            const int off = rin * tc::kKBlock2 + ((g ^ ((rin >> 1) & 3)) << 3);
            *reinterpret_cast<uint4*>(box + off) = hi;
            *reinterpret_cast<uint4*>(box + tc::kTile * tc::kKBlock2 + off) = lo;
        }
    }
}

// Same-mode pair sums D^m[ri][rj] += sum_s R_i^m R_j^m K^m_{a_i b_j} over the
// functions exciting m (ranks ri <= rj), one 64 x 64 tile of ranks per CTA,
// 4 x 4 elements per thread; samples in chunks of kPS staged in shared memory.
constexpr int kPS = 16, kPT = 64;

__global__ void __launch_bounds__(256) stein_pairs_kernel(const int4* __restrict__ tasks,
                                                          const uint32_t* __restrict__ vrdesc,
                                                          const int* __restrict__ voff,
                                                          const int64_t* __restrict__ doff, int nm,
                                                          const double* __restrict__ q,
                                                          const double* __restrict__ v,
                                                          const double* __restrict__ vq, int64_t kps,
                                                          int64_t dsize, double* __restrict__ D)
{
    extern __shared__ double ps[];   // q [kPS][nm], V [kPS], Vm [kPS], Rr [kPS][64], Rc [kPS][64], K [kPS][16]
    double* qs = ps;
    double* vs = qs + (size_t)kPS * nm;
    double* vms = vs + kPS;
    double* Rr = vms + kPS;
    double* Rc = Rr + kPS * kPT;
    double* K = Rc + kPS * kPT;
    const int4 task = tasks[blockIdx.x];
    const int m = task.x, ti = task.y, tj = task.z;
    const int v0 = voff[m], e = voff[m + 1] - v0;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    // levels of the thread's rows and columns; past e (R = 0) they take the first
    // one's, so that a thread whose functions share one level pair reads one
    // weight per sample (the functions are ordered by level: most threads do)
    int arow[4], bcol[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int rr = ti * kPT + ty + 16 * r, rc = tj * kPT + tx + 16 * r;
        arow[r] = rr < e ? (int)((vrdesc[v0 + rr] >> 8) & 3u) : -1;
        bcol[r] = rc < e ? (int)((vrdesc[v0 + rc] >> 8) & 3u) : -1;
    }
    bool uni = true;
#pragma unroll
    for (int r = 0; r < 4; r++) {
        if (arow[r] < 0) arow[r] = max(arow[0], 0);
        if (bcol[r] < 0) bcol[r] = max(bcol[0], 0);
        uni = uni && arow[r] == arow[0] && bcol[r] == bcol[0];
    }
    double acc[4][4];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[r][c] = 0.0;
    const int64_t s0 = (int64_t)blockIdx.y * kps;
    for (int64_t c0 = 0; c0 < kps; c0 += kPS) {
        const int nc = (int)min((int64_t)kPS, kps - c0);
        __syncthreads();
        for (int x = tid; x < nc * nm; x += 256) qs[x] = q[(s0 + c0) * nm + x];
        for (int j = tid; j < nc; j += 256) {
            vs[j] = v[s0 + c0 + j];
            vms[j] = vq[(s0 + c0 + j) * nm + m];
        }
        __syncthreads();
        for (int x = tid; x < nc * (2 * kPT + 16); x += 256) {
            const int j = x / (2 * kPT + 16), y = x - j * (2 * kPT + 16);
            if (y < 2 * kPT) {
                const int rk = (y < kPT ? ti : tj) * kPT + (y & (kPT - 1));
                double val = 0.0;
                if (rk < e) val = reduced(vrdesc[v0 + rk], qs + (size_t)j * nm, 1, 0);
                (y < kPT ? Rr : Rc)[j * kPT + (y & (kPT - 1))] = val;
            } else {
                const int ab = y - 2 * kPT, a = ab >> 2, b = ab & 3;
                K[j * 16 + ab] = (a && b) ? stein_weight(a, b, qs[(size_t)j * nm + m], vs[j], vms[j]) : 0.0;
            }
        }
        __syncthreads();
        if (uni) {
            const int k0 = arow[0] * 4 + bcol[0];
            for (int j = 0; j < nc; j++) {
                double rr[4], rc[4];
                const double kk = K[j * 16 + k0];
#pragma unroll
                for (int r = 0; r < 4; r++) rr[r] = Rr[j * kPT + ty + 16 * r], rc[r] = Rc[j * kPT + tx + 16 * r] * kk;
#pragma unroll
                for (int r = 0; r < 4; r++)
#pragma unroll
                    for (int c = 0; c < 4; c++) acc[r][c] = fma(rr[r], rc[c], acc[r][c]);
            }
            continue;
        }
        for (int j = 0; j < nc; j++) {
            double rr[4], rc[4];
#pragma unroll
            for (int r = 0; r < 4; r++) rr[r] = Rr[j * kPT + ty + 16 * r], rc[r] = Rc[j * kPT + tx + 16 * r];
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[r][c] = fma(rr[r], rc[c] * K[j * 16 + arow[r] * 4 + bcol[c]], acc[r][c]);
        }
    }
    double* Dp = D + (size_t)blockIdx.y * dsize + doff[m];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int rr = ti * kPT + ty + 16 * r, rc = tj * kPT + tx + 16 * c;
            if (rr < e && rc < e && rr <= rc) Dp[(size_t)rr * e + rc] += acc[r][c];
        }
}

// The same sums for modes with few exciting functions (e <= kTriMax; 49 for
// every mode of the hexamer doubles basis), where most of a 64 x 64 tile would
// be idle: one CTA per mode (and sample range), thread t owning the t-th 4 x 4
// block (bi <= bj) of the mode's upper e x e triangle, so a sample costs a
// thread four 16-byte loads of R and 16 weight loads for 16 products.  R values
// (zero past e) and the level-pair weights of a sample chunk are staged in
// shared memory.
constexpr int kTriMax = 64, kTriThreads = 160, kFS = 32;

__global__ void __launch_bounds__(kTriThreads) stein_pairs_tri_kernel(const int* __restrict__ modes,
                                                                      const uint32_t* __restrict__ vrdesc,
                                                                      const int* __restrict__ voff,
                                                                      const int64_t* __restrict__ doff, int nm,
                                                                      const double* __restrict__ q,
                                                                      const double* __restrict__ v,
                                                                      const double* __restrict__ vq, int64_t kps,
                                                                      int64_t dsize, double* __restrict__ D)
{
    extern __shared__ __align__(16) double fs[];   // q [kFS][nm], V [kFS], Vm [kFS], R [kFS][64], K [kFS][16]
    double* qs = fs;
    double* vs = qs + (size_t)kFS * nm;
    double* vms = vs + kFS;
    double* R = vms + kFS;          // 16-byte aligned: kFS * (nm + 2) doubles is even
    double* K = R + kFS * kTriMax;
    const int m = modes[blockIdx.x];
    const int v0 = voff[m], e = voff[m + 1] - v0;
    const int nbk = (e + 3) / 4, tid = threadIdx.x;
    // this thread's block (bi, bj), row-major over bi <= bj
    int bi = -1, bj = 0;
    if (tid < nbk * (nbk + 1) / 2) {
        int p = tid, r = 0;
        while (p >= nbk - r) p -= nbk - r, r++;
        bi = r, bj = r + p;
    }
    // level pairs of the block; rows and columns past e (R = 0) take the block's
    // first level, so that a block whose functions share one level pair reads one
    // weight per sample (the functions are ordered by level: most blocks do)
    int ab[4][4];
    bool uni = true;
    {
        int la[4], lb[4];
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int ri = 4 * bi + r, rc = 4 * bj + r;
            la[r] = (bi >= 0 && ri < e) ? (int)((vrdesc[v0 + ri] >> 8) & 3u) : -1;
            lb[r] = (bi >= 0 && rc < e) ? (int)((vrdesc[v0 + rc] >> 8) & 3u) : -1;
        }
#pragma unroll
        for (int r = 1; r < 4; r++) {
            if (la[r] < 0) la[r] = la[0];
            if (lb[r] < 0) lb[r] = lb[0];
        }
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int c = 0; c < 4; c++) {
                ab[r][c] = max(la[r], 0) * 4 + max(lb[c], 0);
                uni = uni && ab[r][c] == ab[0][0];
            }
    }
    double acc[4][4];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[r][c] = 0.0;
    const int64_t s0 = (int64_t)blockIdx.y * kps;
    for (int64_t c0 = 0; c0 < kps; c0 += kFS) {
        const int nc = (int)min((int64_t)kFS, kps - c0);
        __syncthreads();
        for (int x = tid; x < nc * nm; x += kTriThreads) qs[x] = q[(s0 + c0) * nm + x];
        for (int j = tid; j < nc; j += kTriThreads) {
            vs[j] = v[s0 + c0 + j];
            vms[j] = vq[(s0 + c0 + j) * nm + m];
        }
        __syncthreads();
        for (int x = tid; x < nc * (kTriMax + 16); x += kTriThreads) {
            const int j = x / (kTriMax + 16), y = x - j * (kTriMax + 16);
            if (y < kTriMax) {
                R[j * kTriMax + y] = y < e ? reduced(vrdesc[v0 + y], qs + (size_t)j * nm, 1, 0) : 0.0;
            } else {
                const int k = y - kTriMax, a = k >> 2, b = k & 3;
                K[j * 16 + k] = (a && b) ? stein_weight(a, b, qs[(size_t)j * nm + m], vs[j], vms[j]) : 0.0;
            }
        }
        __syncthreads();
        if (bi < 0) continue;
        if (uni) {
            const int k0 = ab[0][0];
            for (int j = 0; j < nc; j++) {
                const double2* Rj = reinterpret_cast<const double2*>(R + j * kTriMax);
                const double2 r01 = Rj[2 * bi], r23 = Rj[2 * bi + 1], c01 = Rj[2 * bj], c23 = Rj[2 * bj + 1];
                const double kk = K[j * 16 + k0];
                const double rr[4] = {r01.x, r01.y, r23.x, r23.y};
                const double rc[4] = {c01.x * kk, c01.y * kk, c23.x * kk, c23.y * kk};
#pragma unroll
                for (int r = 0; r < 4; r++)
#pragma unroll
                    for (int c = 0; c < 4; c++) acc[r][c] = fma(rr[r], rc[c], acc[r][c]);
            }
            continue;
        }
        for (int j = 0; j < nc; j++) {
            const double2* Rj = reinterpret_cast<const double2*>(R + j * kTriMax);
            const double2 r01 = Rj[2 * bi], r23 = Rj[2 * bi + 1], c01 = Rj[2 * bj], c23 = Rj[2 * bj + 1];
            const double rr[4] = {r01.x, r01.y, r23.x, r23.y}, rc[4] = {c01.x, c01.y, c23.x, c23.y};
            const double* Kj = K + j * 16;
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[r][c] = fma(rr[r], rc[c] * Kj[ab[r][c]], acc[r][c]);
        }
    }
    if (bi < 0) return;
    double* Dp = D + (size_t)blockIdx.y * dsize + doff[m];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int ri = 4 * bi + r, rc = 4 * bj + c;
            if (ri < e && rc < e && ri <= rc) Dp[(size_t)ri * e + rc] += acc[r][c];
        }
}

// sums[i] += the summed rows' partials of a pass (the last two blocks of every
// 4096-sample block hold only padding slots and are skipped).  CTA: 32 rows;
// warp w adds the blocks b = w mod 8 (a coalesced 128-byte read per block), the
// eight warp sums are then added in warp order, so the result does not depend
// on scheduling.
__global__ void __launch_bounds__(256) stein_rowsum_kernel(const float* __restrict__ spart, int nsum, int nblocks,
                                                           double* __restrict__ sums)
{
    __shared__ double ws[8][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int i = blockIdx.x * 32 + lane;
    constexpr int kValid = tc::kFlush / kSxSlots;     // 128 sample blocks per 130
    const int nvalid = nblocks / kSxBlocksPerFlush * kValid;
    double acc = 0.0;
    if (i < nsum) {
#pragma unroll 8
        for (int vb = w; vb < nvalid; vb += 8) {
            const int b = vb / kValid * kSxBlocksPerFlush + vb % kValid;
            acc += (double)__ldg(spart + (size_t)b * nsum + i);
        }
    }
    ws[w][lane] = acc;
    __syncthreads();
    if (w == 0 && i < nsum) {
        double t = 0.0;
        for (int k = 0; k < 8; k++) t += ws[k][lane];
        sums[i] += t;
    }
}

// Element (i, j) of the dense matrix from its terms: for each mode m that r =
// min(i, j) or c = max(i, j) excites, C at virtual row (m, r) column c, or at
// (m, c) column r, or the pair sum D^m when both excite m; the mean over those
// modes; <0|V|0> from the ground row.  C: FP64 tiles of 128 x 128, row-major,
// `ct` per tile row (N256 = false); or the split form's 128 x 256 unit partials
// (N256 = true), tile (row panel r, column panel pair q) at tile_of[r * ct + q]
// with `ct` = column panel pairs, tile-local column-major.  With wb_off (the
// split form's pair sums as products) the term of a pair exciting m in both
// functions is C at W_b row (m, rank of r, level of c in m), column
// red3(c without its mode-m factor).
template <bool N256>
__global__ void stein_unpack_kernel(const uint32_t* __restrict__ desc, const int* __restrict__ rank3,
                                    const int* __restrict__ voff, const int64_t* __restrict__ doff, int nb, int nv,
                                    int ct, int nsplit, int dsplit, const double* __restrict__ C,
                                    const double* __restrict__ D,
                                    int64_t csize, int64_t dsize, double divisor, const double* __restrict__ diag,
                                    double zpe, double* __restrict__ M, int64_t ld,
                                    const int* __restrict__ tile_of, const int* __restrict__ red3,
                                    const int* __restrict__ wb_off, const int* __restrict__ sum_off,
                                    const double* __restrict__ sums)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)nb * nb) return;
    const int j = (int)(e / nb), i = (int)(e - (int64_t)j * nb);
    const int r = min(i, j), c = max(i, j);
    // a term whose tile the plan did not make reads NaN into the element (never,
    // by construction; a visible result rather than an out-of-range read)
    auto cidx = [&](int vr, int col) -> int64_t {
        if (N256) {
            const int t = tile_of[(vr >> 7) * ct + (col >> 8)];
            if (t < 0) return -1;
            return (int64_t)t * (128 * 256) + (int64_t)(((col >> 7) & 1) * 128 + (col & 127)) * 128 + (vr & 127);
        }
        return ((int64_t)(vr >> 7) * ct + (col >> 7)) * (128 * 128) + (int64_t)(vr & 127) * 128 + (col & 127);
    };
    auto csum = [&](int64_t x) {
        if (x < 0) return __longlong_as_double(0x7ff8000000000000ll);
        double t = 0.0;
        for (int s = 0; s < nsplit; s++) t += C[s * csize + x];
        return t;
    };
    int mr[3], lr[3], mc[3], lc[3];
    const int nr = decode(desc[r], mr, lr), ncn = decode(desc[c], mc, lc);
    double val = 0.0;
    if (nr + ncn == 0) {   // <0|V|0>
        const int64_t x = cidx(nv - 1, 0);
        val += csum(x);
    } else {
        int ns = 0;
        for (int a = 0; a < nr; a++) {
            int b = -1;
            for (int k = 0; k < ncn; k++)
                if (mc[k] == mr[a]) b = k;
            const int m = mr[a];
            double t = 0.0;
            if (b < 0) {
                const int64_t x = cidx(voff[m] + rank3[3 * r + a], c);
                t += csum(x);
            } else if (sum_off && sum_off[m * 4 + lc[b]] >= 0) {
                // summed row (m, rank of r, level of c in m): c without m is the constant
                t = sums[sum_off[m * 4 + lc[b]] + rank3[3 * r + a]];
            } else if (wb_off) {
                // W_b row (m, rank of r, level of c in m) against Phi of c without m
                const int64_t x = cidx(wb_off[m * 4 + lc[b]] + rank3[3 * r + a], red3[3 * c + b]);
                t += csum(x);
            } else {
                // D holds the upper triangle of ranks (functions ordered by level in m)
                const int en = voff[m + 1] - voff[m];
                const int ra = rank3[3 * r + a], rb = rank3[3 * c + b];
                const int64_t x = doff[m] + (int64_t)min(ra, rb) * en + max(ra, rb);
                for (int s = 0; s < dsplit; s++) t += D[s * dsize + x];
            }
            val += t;
            ns++;
        }
        for (int b = 0; b < ncn; b++) {
            bool shared = false;
            for (int a = 0; a < nr; a++) shared |= mr[a] == mc[b];
            if (shared) continue;
            const int64_t x = cidx(voff[mc[b]] + rank3[3 * c + b], r);
            double t = 0.0;
            t += csum(x);
            val += t;
            ns++;
        }
        val /= (double)ns;
    }
    val = val / divisor;
    if (diag && i == j) val = (val + diag[i]) + zpe;
    M[(size_t)j * ld + i] = val;
}

int64_t round_up(int64_t a, int64_t b) { return (a + b - 1) / b * b; }

}  // namespace

// red3[3 j + a]: the basis index of function j without its a-th factor (decode
// order), -1 where that function is not in the basis; *closed: none is missing.
std::vector<int> reduced_functions(const std::vector<uint32_t>& desc, bool* closed)
{
    const int nb = (int)desc.size();
    std::map<std::array<int, 6>, int> index_of;     // sorted (mode, level) factors -> basis index
    auto key_of = [](const int* mm, const int* ll, int k, int skip) {
        std::array<int, 6> key{-1, -1, -1, -1, -1, -1};
        std::vector<std::pair<int, int>> f;
        for (int a = 0; a < k; a++)
            if (a != skip) f.push_back({mm[a], ll[a]});
        std::sort(f.begin(), f.end());
        for (size_t u = 0; u < f.size(); u++) key[2 * u] = f[u].first, key[2 * u + 1] = f[u].second;
        return key;
    };
    for (int j = 0; j < nb; j++) {
        int mm[3], ll[3];
        const int k = decode(desc[j], mm, ll);
        index_of[key_of(mm, ll, k, -1)] = j;
    }
    std::vector<int> red3((size_t)nb * 3, -1);
    *closed = true;
    for (int j = 0; j < nb; j++) {
        int mm[3], ll[3];
        const int k = decode(desc[j], mm, ll);
        for (int a = 0; a < k; a++) {
            const auto it = index_of.find(key_of(mm, ll, k, a));
            if (it == index_of.end()) *closed = false;
            else red3[(size_t)3 * j + a] = it->second;
        }
    }
    return red3;
}

int stein_create(SteinPlan& p, const std::vector<uint32_t>& desc, int nm, int64_t chunk_cfg, int sms, bool split)
{
    p = SteinPlan{};
    p.nb = (int)desc.size();
    p.nm = nm;
    p.nb_pad = (int)round_up(p.nb, 128);
    if (sizeof(double) * (2 * (size_t)nm * kExpLd + kExpS) > 227 * 1024)
        return fail(SCP3GPU_ERR_ARG, "stein: too many modes for the expansion's shared memory (at most 220)");
    if (split && 6 * nm + 2 > kSxMaxTable)
        return fail(SCP3GPU_ERR_ARG, "stein: too many modes for the split expansion's table (at most 170)");
    // functions exciting each mode, in basis order; rank of each in its mode's list
    std::vector<std::vector<int>> E(nm);
    std::vector<std::vector<int>> lev(nm);
    std::vector<int> rank3((size_t)p.nb * 3, 0);
    std::vector<uint32_t> vr_of_rank;
    std::vector<std::vector<int>> slot(nm);   // factor index, within its function, of mode m
    for (int i = 0; i < p.nb; i++) {
        int mm[3], ll[3];
        const int k = decode(desc[i], mm, ll);
        for (int a = 0; a < k; a++) {
            if (mm[a] >= nm) return fail(SCP3GPU_ERR_ARG, "stein: basis mode out of range");
            E[mm[a]].push_back(i);
            lev[mm[a]].push_back(ll[a]);
            slot[mm[a]].push_back(a);
        }
    }
    // each mode's functions ordered by their level in that mode (stable), so that
    // the pair sums' 4 x 4 blocks mostly share one level pair (one weight)
    for (int m = 0; m < nm; m++) {
        std::vector<int> ord(E[m].size());
        for (size_t r = 0; r < ord.size(); r++) ord[r] = (int)r;
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return lev[m][x] < lev[m][y]; });
        std::vector<int> e2, l2;
        for (size_t r = 0; r < ord.size(); r++) {
            const int i = E[m][ord[r]];
            e2.push_back(i);
            l2.push_back(lev[m][ord[r]]);
            rank3[(size_t)3 * i + slot[m][ord[r]]] = (int)r;
        }
        E[m].swap(e2);
        lev[m].swap(l2);
    }
    std::vector<int> voff(nm + 1, 0);
    std::vector<int64_t> doff(nm, 0);
    std::vector<uint32_t> vrdesc;
    std::vector<int4> tasks;      // 64 x 64 rank tiles of modes with many exciting functions
    std::vector<int> ftasks;      // modes with few (one CTA each)
    int64_t dsz = 0;
    for (int m = 0; m < nm; m++) {
        voff[m] = (int)vrdesc.size();
        doff[m] = dsz;
        const int en = (int)E[m].size();
        dsz += (int64_t)en * en;
        for (int r = 0; r < en; r++) {
            int mm[3], ll[3];
            const int k = decode(desc[E[m][r]], mm, ll);
            uint32_t d = (uint32_t)m | ((uint32_t)lev[m][r] << 8);
            int o = 0;
            for (int a = 0; a < k; a++) {
                if (mm[a] == m) continue;
                d |= o == 0 ? ((uint32_t)mm[a] << 10) | ((uint32_t)ll[a] << 18)
                            : ((uint32_t)mm[a] << 20) | ((uint32_t)ll[a] << 28);
                o++;
            }
            vrdesc.push_back(d);
        }
        if (en <= kTriMax) {
            if (en > 0) ftasks.push_back(m);
        } else {
            const int nt = (en + kPT - 1) / kPT;
            for (int a = 0; a < nt; a++)
                for (int b = a; b < nt; b++) tasks.push_back(make_int4(m, a, b, 0));
        }
    }
    voff[nm] = (int)vrdesc.size();
    vrdesc.push_back(kGroundRow);
    p.nv = (int)vrdesc.size();
    p.nv_pad = (int)round_up(p.nv, 128);
    p.rt = p.nv_pad / 128;
    p.ct = p.nb_pad / 128;
    p.dsize = std::max<int64_t>(dsz, 1);
    p.ndtasks = (int)tasks.size();
    p.nftasks = (int)ftasks.size();
    int rc;
    if (!split) {
        // passes of 2^14 samples (fewer while W and Phi of a pass would pass ~4 GB);
        // sample ranges per tile as the plain form chooses them, the C partials of
        // all ranges held under ~8 GB (one range if a single one is larger)
        int64_t chunk = chunk_cfg > 0 ? chunk_cfg : 16384;
        while (chunk > 4096 && (int64_t)(p.nv_pad + p.nb_pad) * chunk * 8 > (4ll << 30)) chunk /= 2;
        p.chunk = chunk;
        const int64_t csize = (int64_t)p.rt * p.ct * 128 * 128;
        double best = 1e300;
        p.nsplit = 1;
        for (int ns = 1; chunk / ns >= 2048 && chunk % (16ll * ns) == 0; ns *= 2) {
            if (ns > 1 && (csize + p.dsize) * 8 * ns > (8ll << 30)) break;
            const int64_t units = (int64_t)p.rt * p.ct * ns;
            const double cost = (double)((units + sms - 1) / sms) / ns;
            if (cost < best - 1e-9) best = cost, p.nsplit = ns;
        }
        // sample ranges of the same-mode pair sums: a multiple of the products' (so a
        // pass of 16 * nsplit samples divides), up to 4x finer while their sums stay
        // small -- those kernels have one CTA per mode and range, too few for the GPU
        // at the products' split (48 x 8 for the hexamer doubles basis)
        p.dsplit = p.nsplit;
        while (p.dsplit < 4 * p.nsplit && p.dsplit * 2 * p.dsize * 8 <= (256ll << 20)) p.dsplit *= 2;
        if ((rc = dalloc(&p.W, (size_t)p.chunk * p.nv_pad)) || (rc = dalloc(&p.Phi, (size_t)p.chunk * p.nb_pad)) ||
            (rc = dalloc(&p.C, (size_t)csize * p.nsplit))) {
            stein_destroy(p);
            return rc;
        }
    } else {
        // The products W Phi^T on the tensor cores: tiles of one W panel against a
        // pair of Phi panels (one panel when ct is odd), K slots in blocks of 4160
        // per 4096 samples (the contraction's sign groups, here all positive).
        // Passes of 2^16 samples (fewer while the operand would pass ~4 GB); sample
        // ranges per tile minimising waves per range, at most 16, partials under ~4 GB.
        p.split = true;
        p.bpairs = (p.ct + 1) / 2;
        // The same-mode pair sums as products too, when every function j exciting m
        // is, without its mode-m factor, again a basis function (red3) and the
        // expansion's table holds the weights of the level pairs present:
        // T^m_ij = sum_s [R_i^m K^m_{a_i b_j}] Phi_{red(j, m)}.
        bool closed = true;
        const std::vector<int> red3 = reduced_functions(desc, &closed);
        std::vector<int> levmask(nm, 0);
        for (int m = 0; m < nm; m++)
            for (int l : lev[m]) levmask[m] |= 1 << l;
        // the expansion's table holds at most 1 + 3 nm Hermite values, 3 nm weights
        // K_a0, V and 6 nm weights K_ab: 10-bit indices
        p.tcpairs = closed && 12 * nm + 2 <= kSxMaxTable;
        // W_b blocks (m, b), one per level b present in mode m, e_m rows each: in the
        // operand, or summed when every function of level b in m reduces to the
        // constant (its only Phi column would be the ground function's)
        std::vector<int> wb_off((size_t)nm * 4, -1), sum_off((size_t)nm * 4, -1);
        auto reduces_to_ground = [&](int m, int b) {
            for (size_t r = 0; r < E[m].size(); r++) {
                if (lev[m][r] != b) continue;
                int mm[3], ll[3];
                const int k = decode(desc[E[m][r]], mm, ll);
                for (int a = 0; a < k; a++)
                    if (mm[a] == m && red3[(size_t)3 * E[m][r] + a] != 0) return false;
            }
            return true;
        };
        // The products of the W_b blocks pay whole tiles for the few columns each
        // needs: worth it while they add no more tiles than the direct terms have
        // (hexamer doubles basis: 19 against 95); otherwise (triples bases, where
        // each block reaches Phi pairs all over the basis) the pair sums stay FP64.
        if (p.tcpairs) {
            int64_t est = 0;
            for (int m = 0; m < nm; m++)
                for (int b = 1; b <= 3; b++) {
                    if (!((levmask[m] >> b) & 1) || reduces_to_ground(m, b)) continue;
                    std::vector<char> pairs((size_t)p.bpairs, 0);
                    for (size_t r = 0; r < E[m].size(); r++) {
                        if (lev[m][r] != b) continue;
                        int mm[3], ll[3];
                        const int k = decode(desc[E[m][r]], mm, ll);
                        for (int a = 0; a < k; a++)
                            if (mm[a] == m) pairs[red3[(size_t)3 * E[m][r] + a] / 256] = 1;
                    }
                    int np = 0;
                    for (char c : pairs) np += c;
                    est += (int64_t)np * (int64_t)E[m].size();     // tile rows: 128 per tile
                }
            if (est > (int64_t)128 * p.rt * p.bpairs) p.tcpairs = false;
        }
        int nwb = 0;
        p.nsum = 0;
        if (p.tcpairs)
            for (int m = 0; m < nm; m++)
                for (int b = 1; b <= 3; b++) {
                    if (!((levmask[m] >> b) & 1)) continue;
                    if (reduces_to_ground(m, b)) {
                        sum_off[(size_t)m * 4 + b] = p.nsum;
                        p.nsum += (int)E[m].size();
                    } else {
                        wb_off[(size_t)m * 4 + b] = p.nv_pad + nwb;
                        nwb += (int)E[m].size();
                    }
                }
        p.nwb_pad = (int)round_up(nwb, 128);
        const int wpanels = (p.nv_pad + p.nwb_pad) / 128;
        const int phi0 = p.nv_pad + p.nwb_pad;     // first Phi row
        const int64_t rows = (int64_t)phi0 + p.nb_pad;
        auto slots_of = [](int64_t k) { return k / tc::kFlush * tc::kSlotsPerFlush; };
        int64_t chunk = chunk_cfg > 0 ? chunk_cfg : 65536;
        while (chunk > tc::kFlush && rows * slots_of(chunk) * 4 > (4ll << 30)) chunk /= 2;
        chunk = std::max<int64_t>(chunk / tc::kFlush * tc::kFlush, tc::kFlush);
        p.chunk = chunk;
        p.slots = slots_of(chunk);
        // tiles: every W panel of the direct terms against every Phi pair (pair-major,
        // so a wave's tiles share their pairs), then every W_b panel against the pairs
        // that hold its rows' reduced functions
        std::vector<int4> tl;
        std::vector<int> tile_of((size_t)wpanels * p.bpairs, -1);
        auto add_tile = [&](int r, int q) {
            const int b0 = phi0 + 2 * q * 128, b1 = 2 * q + 1 < p.ct ? b0 + 128 : b0;
            tile_of[(size_t)r * p.bpairs + q] = (int)tl.size();
            tl.push_back(make_int4(r * 128, b0, 0, b1));
        };
        for (int q = 0; q < p.bpairs; q++)
            for (int r = 0; r < p.rt; r++) add_tile(r, q);
        if (p.tcpairs) {
            std::vector<std::vector<char>> need((size_t)wpanels, std::vector<char>((size_t)p.bpairs, 0));
            for (int m = 0; m < nm; m++)
                for (int b = 1; b <= 3; b++) {
                    const int o = wb_off[(size_t)m * 4 + b], en = (int)E[m].size();
                    if (o < 0) continue;
                    for (int r = 0; r < en; r++) {
                        if (lev[m][r] != b) continue;
                        int mm[3], ll[3];
                        const int k = decode(desc[E[m][r]], mm, ll);
                        for (int a = 0; a < k; a++)
                            if (mm[a] == m)
                                for (int pr = o / 128; pr <= (o + en - 1) / 128; pr++)
                                    need[pr][red3[(size_t)3 * E[m][r] + a] / 256] = 1;
                    }
                }
            for (int r = p.rt; r < wpanels; r++)
                for (int q = 0; q < p.bpairs; q++)
                    if (need[r][q]) add_tile(r, q);
        }
        p.ntiles2 = (int)tl.size();
        double best = 1e300;
        p.nsplit = 1;
        for (int m = 1; m <= 16; m++) {
            const int64_t units = (int64_t)p.ntiles2 * m;
            if (m > 1 && units * 128 * 256 * 8 > (4ll << 30)) break;
            const double cost = (double)((units + sms - 1) / sms) / m;
            if (cost < best - 1e-12) best = cost, p.nsplit = m;
        }
        p.dsplit = 1;
        while (!p.tcpairs && p.dsplit < 64 && p.dsplit * 2 * p.dsize * 8 <= (256ll << 20)) p.dsplit *= 2;
        const std::vector<int> nosign((size_t)(chunk / tc::kFlush), tc::kSlotsPerFlush / 16);
        const size_t xop_elems = (size_t)2 * rows * p.slots;
        // per operand row, three indices into the expansion's table (0 = the constant 1);
        // the table holds the entries the rows use, numbered as they are first needed
        std::map<uint32_t, uint32_t> tslot;
        std::vector<uint32_t> tspec{kTOne};
        auto tab = [&](uint32_t kind, int a, int b, int m) -> uint32_t {
            const uint32_t key = kind | (uint32_t)a << 4 | (uint32_t)b << 6 | (uint32_t)m << 8;
            const auto it = tslot.find(key);
            if (it != tslot.end()) return it->second;
            const uint32_t i = (uint32_t)tspec.size();
            tspec.push_back(key);
            tslot[key] = i;
            return i;
        };
        auto hidx = [&](int m, int l) { return l ? tab(kTHo, l, 0, m) : 0u; };
        std::vector<uint32_t> xd((size_t)rows + p.nsum, kSxZeroRow);   // operand rows, then summed rows
        for (int r = 0; r < p.nv; r++) {
            const uint32_t vd = vrdesc[r];
            if (vd & kGroundRow) {
                xd[r] = tab(kTV, 0, 0, 0);
                continue;
            }
            const int m = vd & 255, a = (vd >> 8) & 3;
            xd[r] = tab(kTKa0, a, 0, m) | hidx((vd >> 10) & 255, (vd >> 18) & 3) << 10 |
                    hidx((vd >> 20) & 255, (vd >> 28) & 3) << 20;
        }
        for (int m = 0; m < nm; m++)        // W_b(m, r) = R^m_{E_m[r]} K^m_{a_r b}
            for (int b = 1; b <= 3; b++) {
                const int o = wb_off[(size_t)m * 4 + b] >= 0 ? wb_off[(size_t)m * 4 + b]
                              : sum_off[(size_t)m * 4 + b] >= 0 ? (int)rows + sum_off[(size_t)m * 4 + b]
                                                                 : -1;
                if (o < 0) continue;
                for (size_t r = 0; r < E[m].size(); r++) {
                    const uint32_t vd = vrdesc[voff[m] + r];
                    const int a = lev[m][r];
                    xd[(size_t)o + r] = tab(kTKab, std::min(a, b), std::max(a, b), m) |
                                        hidx((vd >> 10) & 255, (vd >> 18) & 3) << 10 |
                                        hidx((vd >> 20) & 255, (vd >> 28) & 3) << 20;
                }
            }
        for (int j = 0; j < p.nb; j++) {
            int mm[3] = {0, 0, 0}, ll[3] = {0, 0, 0};
            decode(desc[j], mm, ll);
            xd[(size_t)phi0 + j] = hidx(mm[0], ll[0]) | hidx(mm[1], ll[1]) << 10 | hidx(mm[2], ll[2]) << 20;
        }
        p.trows = (int)tspec.size();
        if (p.trows > kSxMaxTable) {
            stein_destroy(p);
            return fail(SCP3GPU_ERR_ARG, "stein: the split expansion's table exceeds 1024 rows");
        }
        if ((rc = upload(&p.xdesc, xd.data(), xd.size())) || (rc = upload(&p.tspec, tspec.data(), tspec.size())) ||
            (rc = upload(&p.tiles2, tl.data(), tl.size())) ||
            (rc = upload(&p.tile_of, tile_of.data(), tile_of.size())) ||
            (p.tcpairs && ((rc = upload(&p.red3, red3.data(), red3.size())) ||
                           (rc = upload(&p.wb_off, wb_off.data(), wb_off.size())) ||
                           (rc = upload(&p.sum_off, sum_off.data(), sum_off.size())))) ||
            (p.nsum && ((rc = dalloc(&p.spart, (size_t)(chunk / tc::kFlush) * kSxBlocksPerFlush * p.nsum)) ||
                        (rc = dalloc(&p.sums, (size_t)p.nsum)))) ||
            (rc = upload(&p.nosign, nosign.data(), nosign.size())) ||
            (rc = dalloc(&p.xop, xop_elems)) || (rc = dalloc(&p.P, (size_t)p.nsplit * p.ntiles2 * 128 * 256)) ||
            (rc = dalloc(&p.err, (size_t)1))) {
            stein_destroy(p);
            return rc;
        }
        // padding rows and the slots closing each 4096-sample block are never written
        SCP3_CUDA(cudaMemset(p.xop, 0, sizeof(uint16_t) * xop_elems));
        if (p.spart)   // the blocks of padding slots are never written
            SCP3_CUDA(cudaMemset(p.spart, 0,
                                 sizeof(float) * (size_t)(chunk / tc::kFlush) * kSxBlocksPerFlush * p.nsum));
        SCP3_CUDA(cudaMemset(p.err, 0, sizeof(int)));
        const size_t es = sizeof(float) * ((size_t)p.trows * kSxSlots + 2 * (size_t)nm * kSxLd + kSxSlots);
        if (es > 48 * 1024)
            SCP3_CUDA(cudaFuncSetAttribute(stein_expand_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)es));
    }
    if ((rc = upload(&p.vrdesc, vrdesc.data(), vrdesc.size())) || (rc = upload(&p.rank3, rank3.data(), rank3.size())) ||
        (rc = upload(&p.voff, voff.data(), voff.size())) || (rc = upload(&p.doff, doff.data(), doff.size())) ||
        (p.ndtasks && (rc = upload(&p.dtasks, tasks.data(), tasks.size()))) ||
        (p.nftasks && (rc = upload(&p.ftasks, ftasks.data(), ftasks.size()))) ||
        (!p.tcpairs && (rc = dalloc(&p.D, (size_t)p.dsize * p.dsplit)))) {
        stein_destroy(p);
        return rc;
    }
    return SCP3GPU_OK;
}

int64_t stein_pass_samples(const SteinPlan& p, int64_t nvalid)
{
    return p.split ? round_up(nvalid, tc::kFlush) : round_up(nvalid, 16ll * p.nsplit);
}

void stein_destroy(SteinPlan& p)
{
    cudaFree(p.vrdesc), cudaFree(p.rank3), cudaFree(p.voff), cudaFree(p.doff), cudaFree(p.dtasks), cudaFree(p.ftasks);
    cudaFree(p.W), cudaFree(p.Phi), cudaFree(p.C), cudaFree(p.D);
    cudaFree(p.xop), cudaFree(p.xdesc), cudaFree(p.tiles2), cudaFree(p.nosign), cudaFree(p.P), cudaFree(p.err);
    cudaFree(p.tile_of), cudaFree(p.red3), cudaFree(p.wb_off), cudaFree(p.tspec);
    cudaFree(p.sum_off), cudaFree(p.spart), cudaFree(p.sums);
    p = SteinPlan{};
}

int stein_zero(const SteinPlan& p, cudaStream_t s)
{
    if (p.split) {
        SCP3_CUDA(cudaMemsetAsync(p.P, 0, sizeof(double) * (size_t)p.nsplit * p.ntiles2 * 128 * 256, s));
        SCP3_CUDA(cudaMemsetAsync(p.err, 0, sizeof(int), s));
    } else {
        SCP3_CUDA(cudaMemsetAsync(p.C, 0, sizeof(double) * (size_t)p.rt * p.ct * 128 * 128 * p.nsplit, s));
    }
    if (p.D) SCP3_CUDA(cudaMemsetAsync(p.D, 0, sizeof(double) * (size_t)p.dsize * p.dsplit, s));
    if (p.sums) SCP3_CUDA(cudaMemsetAsync(p.sums, 0, sizeof(double) * (size_t)p.nsum, s));
    return SCP3GPU_OK;
}

int stein_pass(const SteinPlan& p, const uint32_t* desc, const double* q, const double* v, const double* vq,
               int64_t k, cudaStream_t s)
{
    if (k == 0) return SCP3GPU_OK;
    if (k > p.chunk || k != stein_pass_samples(p, k)) return fail(SCP3GPU_ERR_ARG, "stein: pass not tiled");
    int rc;
    if (p.split) {
        const int nflush = (int)(k / tc::kFlush);
        const int rows = p.nv_pad + p.nwb_pad + p.nb_pad;
        const size_t es = sizeof(float) * ((size_t)p.trows * kSxSlots + 2 * (size_t)p.nm * kSxLd + kSxSlots);
        // rows in chunks of at most 16384 per CTA: each chunk builds the block's table
        // again, and the table build is a third of a 2816-row chunk's time (measured:
        // 8496 rows in one chunk instead of three took the split pass from 31.2 to
        // 32.8 M samples/s)
        const int vrows = rows + p.nsum;   // operand rows, then summed rows
        const int ny = (vrows + 16383) / 16384, per = (int)round_up((vrows + ny - 1) / ny, 64);
        dim3 eg((unsigned)(nflush * kSxBlocksPerFlush), (unsigned)ny);
        stein_expand_split_kernel<<<eg, kSxThreads, es, s>>>(p.tspec, p.trows, p.xdesc, rows, p.nsum, per, p.nm, q,
                                                             v, vq, k, p.slots / tc::kKBlock2, p.xop, p.spart);
        SCP3_CUDA(cudaGetLastError());
        if (p.nsum)
            stein_rowsum_kernel<<<(p.nsum + 31) / 32, 256, 0, s>>>(p.spart, p.nsum, nflush * kSxBlocksPerFlush,
                                                                   p.sums);
        SCP3_CUDA(cudaGetLastError());
        const int units = p.ntiles2 * p.nsplit;
        int sms = 148, dev = 0;
        SCP3_CUDA(cudaGetDevice(&dev));
        SCP3_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        rc = tc::launch_contract(p.xop, p.slots / tc::kKBlock2, p.tiles2, p.ntiles2, p.nsplit,
                                 nflush * (tc::kSlotsPerFlush / tc::kKBlock2), p.nosign, false, p.P, p.err,
                                 std::min(units, sms), s);
    } else {
        const size_t es = sizeof(double) * (2 * (size_t)p.nm * kExpLd + kExpS);
        if (es > 48 * 1024)
            SCP3_CUDA(cudaFuncSetAttribute(stein_expand_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)es));
        dim3 eg((unsigned)((k + kExpS - 1) / kExpS), (unsigned)((p.nb_pad + p.nv_pad) / kExpR));
        stein_expand_kernel<<<eg, kExpR, es, s>>>(desc, p.nb, p.nb_pad, p.vrdesc, p.nv, p.nv_pad, p.nm, q, v, vq, k,
                                                  p.Phi, p.W);
        SCP3_CUDA(cudaGetLastError());
        rc = launch_gemm_fp64_rect(p.W, p.nv_pad, p.Phi, p.nb_pad, k, p.rt, p.ct, p.nsplit, p.C, s);
    }
    if (rc) return rc;
    if (p.tcpairs) return SCP3GPU_OK;      // the pair sums were part of the products
    if (p.ndtasks) {
        const size_t ps = sizeof(double) * ((size_t)kPS * p.nm + 2 * kPS + 2 * kPS * kPT + 16 * kPS);
        if (ps > 48 * 1024)
            SCP3_CUDA(cudaFuncSetAttribute(stein_pairs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ps));
        dim3 pg((unsigned)p.ndtasks, (unsigned)p.dsplit);
        stein_pairs_kernel<<<pg, 256, ps, s>>>(p.dtasks, p.vrdesc, p.voff, p.doff, p.nm, q, v, vq, k / p.dsplit,
                                               p.dsize, p.D);
        SCP3_CUDA(cudaGetLastError());
    }
    if (p.nftasks) {
        const size_t fsm = sizeof(double) * ((size_t)kFS * p.nm + 2 * kFS + (size_t)kFS * kTriMax + 16 * kFS);
        if (fsm > 48 * 1024)
            SCP3_CUDA(cudaFuncSetAttribute(stein_pairs_tri_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)fsm));
        dim3 fg((unsigned)p.nftasks, (unsigned)p.dsplit);
        stein_pairs_tri_kernel<<<fg, kTriThreads, fsm, s>>>(p.ftasks, p.vrdesc, p.voff, p.doff, p.nm, q, v, vq,
                                                            k / p.dsplit, p.dsize, p.D);
        SCP3_CUDA(cudaGetLastError());
    }
    return SCP3GPU_OK;
}

int stein_unpack(const SteinPlan& p, const uint32_t* desc, double divisor, const double* diag, double zpe,
                 double* M, int64_t ld, cudaStream_t s)
{
    const int64_t total = (int64_t)p.nb * p.nb;
    const unsigned grid = (unsigned)((total + 255) / 256);
    if (p.split) {
        int err = 0;
        SCP3_CUDA(cudaMemcpyAsync(&err, p.err, sizeof(int), cudaMemcpyDeviceToHost, s));
        SCP3_CUDA(cudaStreamSynchronize(s));
        if (err) return fail(SCP3GPU_ERR_TIMEOUT, "tensor-core contraction: a bounded pipeline wait expired");
        stein_unpack_kernel<true><<<grid, 256, 0, s>>>(desc, p.rank3, p.voff, p.doff, p.nb, p.nv, p.bpairs, p.nsplit,
                                                       p.dsplit, p.P, p.D, (int64_t)p.ntiles2 * 128 * 256, p.dsize,
                                                       divisor, diag, zpe, M, ld, p.tile_of, p.red3,
                                                       p.tcpairs ? p.wb_off : nullptr,
                                                       p.nsum ? p.sum_off : nullptr, p.sums);
    } else {
        stein_unpack_kernel<false><<<grid, 256, 0, s>>>(desc, p.rank3, p.voff, p.doff, p.nb, p.nv, p.ct, p.nsplit,
                                                        p.dsplit, p.C, p.D, (int64_t)p.rt * p.ct * 128 * 128, p.dsize,
                                                        divisor, diag, zpe, M, ld, nullptr, nullptr, nullptr,
                                                        nullptr, nullptr);
    }
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

}  // namespace scp3

// Host-only view of the split gradient estimator's reduced functions, for tests:
// red3 (nb * 3 ints, may be null) as reduced_functions gives it for the basis of
// (nmodes, n2, n3); returns 1 when the basis is closed under removing a factor,
// 0 when it is not, negative on bad arguments.
extern "C" int scp3gpu_internal_reduced(int nmodes, int n2, int n3, int* red3)
{
    if (scp3gpu_basis_size(nmodes, n2, n3) < 0) return -1;
    bool closed = true;
    const std::vector<int> r = scp3::reduced_functions(scp3::basis_descriptors(nmodes, n2, n3), &closed);
    if (red3) std::copy(r.begin(), r.end(), red3);
    return closed ? 1 : 0;
}
