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
// 256 threads hold a 4x4 fragment each.  The samples' q, V and dV/dq (FP64,
// sample-major) are staged in shared memory in chunks; every thread forms the
// mode set of each of its elements from the row and column descriptors and
// sums the estimate over the chunk.  Partials: [split][tile][64 x 64] row-major
// within the tile, as the plain -G form, so the same read-out applies.
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

__global__ void __launch_bounds__(256) stein_fp64_kernel(const uint32_t* __restrict__ desc, int nb, int nm,
                                                          const double* __restrict__ q, const double* __restrict__ v,
                                                          const double* __restrict__ vq, int64_t kps, int chunk,
                                                          int nt, int ntiles, double* __restrict__ partial)
{
    extern __shared__ __align__(16) double sm[];
    double* sq = sm;                              // [chunk][nm]
    double* svq = sq + (size_t)chunk * nm;        // [chunk][nm]
    double* sv = svq + (size_t)chunk * nm;        // [chunk]
    __shared__ uint32_t rdesc[kT], cdesc[kT];
    int t = blockIdx.x, ti = 0;
    while (t >= nt - ti) {
        t -= nt - ti;
        ti++;
    }
    const int tj = ti + t;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    if (tid < kT) {
        const int r = ti * kT + tid, c = tj * kT + tid;
        rdesc[tid] = r < nb ? desc[r] : 0xffffffffu;
        cdesc[tid] = c < nb ? desc[c] : 0xffffffffu;
    }
    const int64_t s0 = (int64_t)blockIdx.y * kps;
    double acc[16];
#pragma unroll
    for (int e = 0; e < 16; e++) acc[e] = 0.0;
    for (int64_t c0 = 0; c0 < kps; c0 += chunk) {
        const int nc = (int)(kps - c0 < chunk ? kps - c0 : chunk);
        __syncthreads();
        for (int e = tid; e < nc * nm; e += blockDim.x) {
            sq[e] = q[(s0 + c0) * nm + e];
            svq[e] = vq[(s0 + c0) * nm + e];
        }
        for (int e = tid; e < nc; e += blockDim.x) sv[e] = v[s0 + c0 + e];
        __syncthreads();
#pragma unroll 1
        for (int e = 0; e < 16; e++) {
            const int lr = ty + 16 * (e >> 2), lc = tx + 16 * (e & 3);
            const int gi = ti * kT + lr, gj = tj * kT + lc;
            if (gi > gj || rdesc[lr] == 0xffffffffu || cdesc[lc] == 0xffffffffu) continue;
            // the mode set S of the pair and the two levels in each mode
            int mi[3], li[3], mj[3], lj[3];
            const int ni = decode(rdesc[lr], mi, li), nj = decode(cdesc[lc], mj, lj);
            int S[kMaxS], A[kMaxS], B[kMaxS], ns = 0;
            for (int k = 0; k < ni; k++) S[ns] = mi[k], A[ns] = li[k], B[ns] = 0, ns++;
            for (int k = 0; k < nj; k++) {
                int f = -1;
                for (int u = 0; u < ns; u++)
                    if (S[u] == mj[k]) f = u;
                if (f >= 0) B[f] = lj[k];
                else S[ns] = mj[k], A[ns] = 0, B[ns] = lj[k], ns++;
            }
            double sum = 0.0;
            if (ns == 0) {
                for (int s = 0; s < nc; s++) sum += sv[s];
            } else {
                const double inv_ns = 1.0 / ns;
                for (int s = 0; s < nc; s++) {
                    const double* qs = sq + (size_t)s * nm;
                    const double* gs = svq + (size_t)s * nm;
                    double p[kMaxS], term[kMaxS];
#pragma unroll
                    for (int u = 0; u < kMaxS; u++) {
                        if (u >= ns) break;
                        const double x = qs[S[u]];
                        double ha, ha0, dha, da, dda, hb, hb0, dhb, db, ddb;
                        ho_parts(A[u], x, ha, ha0, dha, da, dda);
                        ho_parts(B[u], x, hb, hb0, dhb, db, ddb);
                        const double r = da * hb + ha0 * db;
                        const double dr = dda * hb + da * dhb + ha0 * ddb;
                        double uu = ha0 * hb0 + 0.5 * dr;
                        if (A[u] == 3 && B[u] == 3) uu = (2 * x * x - 3) * (x * x - 3) * (1.0 / 6.0);
                        p[u] = ha * hb;
                        term[u] = uu * sv[s] + 0.5 * r * gs[S[u]];
                    }
                    // sum_u term_u prod_{u' != u} p_u'  (prefix and suffix products)
                    double pre = 1.0, tot = 0.0, suf[kMaxS];
                    suf[ns - 1] = 1.0;
                    for (int u = ns - 1; u > 0; u--) suf[u - 1] = suf[u] * p[u];
                    for (int u = 0; u < ns; u++) {
                        tot += term[u] * pre * suf[u];
                        pre *= p[u];
                    }
                    sum += tot * inv_ns;
                }
            }
            acc[e] += sum;
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
    if (k == 0) return SCP3GPU_OK;
    const int chunk = (int)std::max<int64_t>(1, std::min<int64_t>(32, (40 * 1024) / (int64_t)(16 * nm + 8)));
    const size_t sm = sizeof(double) * ((size_t)chunk * (2 * nm + 1));
    if (sm > 48 * 1024) SCP3_CUDA(cudaFuncSetAttribute(stein_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       (int)sm));
    dim3 grid(tm.ntiles, nsplit);
    stein_fp64_kernel<<<grid, 256, sm, s>>>(desc, nb, nm, q, v, vq, k / nsplit, chunk, tm.nt, tm.ntiles, partial);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

}  // namespace scp3
