// The gradient (default) estimator of SCP3: addEpot(q, V, Vq, M)
// (ScaledMatrixElements.cpp:102-725 with the formulas of TripleExcitations.h),
// FP64, on the upper-triangle 64x64 tiles of the plain form.
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
// Layout: a CTA owns one upper 64x64 tile and one range of samples (split);
// 256 threads hold a 4x4 fragment each.  Every factor above depends on one
// mode, its two levels and the sample, so the samples are taken in small
// chunks and, per sample and mode, a table of the 16 level pairs (a, b) holds
// p_ab and t_ab = (p_ab(0) + r_ab'/2) V + (r_ab/2) dV/dq_m.  An element is
// then up to six table slots (its mode set; spare slots point at an entry with
// p = 1, t = 0, and <0|V|0> at one with t = V), and its estimate is
// (1/|S|) sum_u t_u prod_{u' != u} p_u' from prefix and suffix products.  The
// slot indices of the thread's 16 elements are formed once and kept in
// registers.  Partials: [split][tile][64 x 64] row-major within the tile, as
// the plain -G form, so the same read-out applies.
#include <algorithm>

#include "internal.h"

namespace scp3 {

namespace {

constexpr int kT = 64;
constexpr int kMaxS = 6;

// (mode, level) list of a basis descriptor (kind | m << 3 | n << 11 | p << 19)
__device__ __forceinline__ int decode(uint32_t d, int* m, int* l)
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

// h_a(q), h_a(0), h_a'(q), d_a(q), d_a'(q) for the oscillator functions h_0..h_3
// (HarmonicOscillatorBasis.cpp: sqrt2 q, (2q^2 - 1)/sqrt2, (2q^3 - 3q)/sqrt3)
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

// Table entry of mode m, levels (a, b) at q = x: p and the two Stein coefficients.
__device__ __forceinline__ void stein_entry(int a, int b, double x, double& p, double& u, double& w)
{
    double ha, ha0, dha, da, dda, hb, hb0, dhb, db, ddb;
    ho_parts(a, x, ha, ha0, dha, da, dda);
    ho_parts(b, x, hb, hb0, dhb, db, ddb);
    const double r = da * hb + ha0 * db;
    const double dr = dda * hb + da * dhb + ha0 * ddb;
    p = ha * hb;
    u = ha0 * hb0 + 0.5 * dr;
    w = 0.5 * r;
    if (a == 3 && b == 3) u = (2 * x * x - 3) * (x * x - 3) * (1.0 / 6.0);   // TripleExcitations.h:763-773
}

constexpr int kSlots = 6;
__constant__ double kInvNs[kSlots + 1] = {0.0, 1.0, 1.0 / 2, 1.0 / 3, 1.0 / 4, 1.0 / 5, 1.0 / 6};

__global__ void __launch_bounds__(256, 2) stein_fp64_kernel(const uint32_t* __restrict__ desc, int nb, int nm,
                                                             const double* __restrict__ q,
                                                             const double* __restrict__ v,
                                                             const double* __restrict__ vq, int64_t kps, int chunk,
                                                             int nt, int ntiles, double* __restrict__ partial)
{
    extern __shared__ __align__(16) double2 tab[];   // [chunk][nm * 16 + 2] (p, t), then the slot words
    const int per = nm * 16 + 2;                     // + the p = 1, t = 0 entry and the t = V entry
    uint32_t* slw = reinterpret_cast<uint32_t*>(tab + (size_t)chunk * per);   // [16 x 3 words][thread]
    const int kOne = nm * 16, kV = nm * 16 + 1;
    int t = blockIdx.x, ti = 0;
    while (t >= nt - ti) {
        t -= nt - ti;
        ti++;
    }
    const int tj = ti + t;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;

    // slot indices of the thread's 16 elements, two 16-bit indices per word; the
    // element's |S| rides in bits 12-15 of word 0 (|S| <= 6; 0 = skip).  Kept in
    // shared memory, [word][thread], so the registers stay with the arithmetic.
    auto SL = [&](int e, int wd) -> uint32_t& { return slw[(size_t)(3 * e + wd) * 256 + tid]; };
#pragma unroll 1
    for (int e = 0; e < 16; e++) {
        const int gi = ti * kT + ty + 16 * (e >> 2), gj = tj * kT + tx + 16 * (e & 3);
        int idx[kSlots];
#pragma unroll
        for (int u = 0; u < kSlots; u++) idx[u] = kOne;
        int ns = 0;
        if (gi <= gj && gj < nb) {
            int mi[3], li[3], mj[3], lj[3];
            const int ni = decode(__ldg(desc + gi), mi, li), nj = decode(__ldg(desc + gj), mj, lj);
            int S[kSlots], A[kSlots], B[kSlots];
            for (int k = 0; k < ni; k++) S[ns] = mi[k], A[ns] = li[k], B[ns] = 0, ns++;
            for (int k = 0; k < nj; k++) {
                int f = -1;
                for (int u = 0; u < ns; u++)
                    if (S[u] == mj[k]) f = u;
                if (f >= 0) B[f] = lj[k];
                else S[ns] = mj[k], A[ns] = 0, B[ns] = lj[k], ns++;
            }
#pragma unroll
            for (int u = 0; u < kSlots; u++)
                if (u < ns) idx[u] = S[u] * 16 + A[u] * 4 + B[u];
            if (ns == 0) {                 // <0|V|0> = V
                idx[0] = kV;
                ns = 1;
            }
        }
        SL(e, 0) = (uint32_t)idx[0] | ((uint32_t)ns << 12) | ((uint32_t)idx[1] << 16);
        SL(e, 1) = (uint32_t)idx[2] | ((uint32_t)idx[3] << 16);
        SL(e, 2) = (uint32_t)idx[4] | ((uint32_t)idx[5] << 16);
    }
    double acc[16];
#pragma unroll
    for (int e = 0; e < 16; e++) acc[e] = 0.0;

    const int64_t s0 = (int64_t)blockIdx.y * kps;
    for (int64_t c0 = 0; c0 < kps; c0 += chunk) {
        const int nc = (int)(kps - c0 < chunk ? kps - c0 : chunk);
        __syncthreads();
        for (int k = tid; k < nc * per; k += blockDim.x) {
            const int j = k / per, id = k - j * per;
            const int64_t smp = s0 + c0 + j;
            double2 ent;
            if (id >= kOne) {
                ent = make_double2(1.0, id == kV ? v[smp] : 0.0);
            } else {
                const int m = id >> 4, a = (id >> 2) & 3, b = id & 3;
                double p, u, w;
                stein_entry(a, b, q[smp * nm + m], p, u, w);
                ent = make_double2(p, u * v[smp] + w * vq[smp * nm + m]);
            }
            tab[k] = ent;
        }
        __syncthreads();
        for (int j = 0; j < nc; j++) {
            const double2* T = tab + (size_t)j * per;
#pragma unroll
            for (int e = 0; e < 16; e++) {
                const uint32_t w0 = SL(e, 0);
                const int ns = (int)((w0 >> 12) & 15u);
                if (ns == 0) continue;
                const uint32_t w1 = SL(e, 1), w2 = SL(e, 2);
                double2 x[kSlots];
                x[0] = T[w0 & 0xfffu];
                x[1] = T[w0 >> 16];
                x[2] = T[w1 & 0xffffu];
                x[3] = T[w1 >> 16];
                x[4] = T[w2 & 0xffffu];
                x[5] = T[w2 >> 16];
                // sum_u t_u prod_{u' != u} p_u' over the six slots (spare ones p = 1, t = 0)
                double pre = 1.0, tot = 0.0;
                double suf[kSlots];
                suf[kSlots - 1] = 1.0;
#pragma unroll
                for (int u = kSlots - 1; u > 0; u--) suf[u - 1] = suf[u] * x[u].x;
#pragma unroll
                for (int u = 0; u < kSlots; u++) {
                    tot += x[u].y * (pre * suf[u]);
                    pre *= x[u].x;
                }
                acc[e] += tot * kInvNs[ns];
            }
        }
    }
    double* P = partial + ((size_t)blockIdx.y * ntiles + blockIdx.x) * (kT * kT);
#pragma unroll
    for (int e = 0; e < 16; e++) {
        const int lr = ty + 16 * (e >> 2), lc = tx + 16 * (e & 3);
        P[lr * kT + lc] += acc[e];
    }
}

}  // namespace

int launch_stein_fp64(const uint32_t* desc, int nb, int nm, const double* q, const double* v, const double* vq,
                      int64_t k, const TileMap& tm, int nsplit, double* partial, cudaStream_t s)
{
    if (tm.tile != kT || k % nsplit != 0) return fail(SCP3GPU_ERR_ARG, "stein: shapes not tiled");
    if (nm * 16 + 2 > 0xfff) return fail(SCP3GPU_ERR_ARG, "stein: too many modes for the slot encoding");
    if (k == 0) return SCP3GPU_OK;
    const size_t per = (size_t)(nm * 16 + 2) * sizeof(double2);
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>(4, (48 * 1024) / per));
    const size_t sm = per * chunk + sizeof(uint32_t) * 48 * 256;   // table chunk + slot words
    if (sm > 48 * 1024) SCP3_CUDA(cudaFuncSetAttribute(stein_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       (int)sm));
    dim3 grid(tm.ntiles, nsplit);
    stein_fp64_kernel<<<grid, 256, sm, s>>>(desc, nb, nm, q, v, vq, k / nsplit, chunk, tm.nt, tm.ntiles, partial);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

}  // namespace scp3
