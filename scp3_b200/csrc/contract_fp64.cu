// Plain-form (FP64) contraction M_ij += sum_s Phi_i(s) V_s Phi_j(s) over the
// upper-triangle tiles only -- what dsyr2k('U','N',0.5,bra,ket,1,M) computes in
// the reference (ScaledMatrixElements.cpp:942-949, 970) -- plus the unpack of
// the tile partial sums into a dense column-major matrix.
//
// FP64 has no tcgen05 path; this is a register-tiled DFMA kernel: 64x64 tile per
// CTA, 256 threads each owning a 4x4 fragment, 16-deep K slices double-buffered
// in shared memory.  Samples are split across `nsplit` CTAs per tile; each
// (split, tile) owns a private FP64 partial that it read-modify-writes, so the
// sums are deterministic and need no atomics.
#include "internal.h"

namespace scp3 {

namespace {

constexpr int kT = 64, kBK = 16, kPad = 1;

__global__ void __launch_bounds__(256) contract_fp64_kernel(const double* __restrict__ phi,
                                                             const double* __restrict__ w, int64_t ldk, int64_t kps,
                                                             int nt, int ntiles, double* __restrict__ partial)
{
    __shared__ double As[2][kBK][kT + kPad];
    __shared__ double Bs[2][kBK][kT + kPad];
    // tile index -> (ti, tj), ti <= tj, row-major over the upper triangle
    int t = blockIdx.x, ti = 0;
    while (t >= nt - ti) {
        t -= nt - ti;
        ti++;
    }
    const int tj = ti + t;
    const int split = blockIdx.y;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int lrow = tid >> 2, lk = (tid & 3) * 4;
    const int64_t kbeg = (int64_t)split * kps;
    const double* pa = phi + (size_t)(ti * kT + lrow) * ldk + kbeg + lk;
    const double* pb = w + (size_t)(tj * kT + lrow) * ldk + kbeg + lk;
    const int nkb = (int)(kps / kBK);

    double acc[4][4];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[r][c] = 0.0;

    double2 a0 = *reinterpret_cast<const double2*>(pa), a1 = *reinterpret_cast<const double2*>(pa + 2);
    double2 b0 = *reinterpret_cast<const double2*>(pb), b1 = *reinterpret_cast<const double2*>(pb + 2);
    auto stash = [&](int buf) {
        As[buf][lk + 0][lrow] = a0.x;
        As[buf][lk + 1][lrow] = a0.y;
        As[buf][lk + 2][lrow] = a1.x;
        As[buf][lk + 3][lrow] = a1.y;
        Bs[buf][lk + 0][lrow] = b0.x;
        Bs[buf][lk + 1][lrow] = b0.y;
        Bs[buf][lk + 2][lrow] = b1.x;
        Bs[buf][lk + 3][lrow] = b1.y;
    };
    stash(0);
    __syncthreads();
    for (int kb = 0; kb < nkb; kb++) {
        const int cur = kb & 1;
        const bool more = kb + 1 < nkb;
        if (more) {
            const double* na = pa + (size_t)(kb + 1) * kBK;
            const double* nb = pb + (size_t)(kb + 1) * kBK;
            a0 = *reinterpret_cast<const double2*>(na);
            a1 = *reinterpret_cast<const double2*>(na + 2);
            b0 = *reinterpret_cast<const double2*>(nb);
            b1 = *reinterpret_cast<const double2*>(nb + 2);
        }
#pragma unroll
        for (int k = 0; k < kBK; k++) {
            double av[4], bv[4];
#pragma unroll
            for (int r = 0; r < 4; r++) av[r] = As[cur][k][ty + 16 * r];
#pragma unroll
            for (int c = 0; c < 4; c++) bv[c] = Bs[cur][k][tx + 16 * c];
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[r][c] = fma(av[r], bv[c], acc[r][c]);
        }
        if (more) stash(cur ^ 1);
        __syncthreads();
    }
    double* P = partial + ((size_t)split * ntiles + blockIdx.x) * (kT * kT);
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int idx = (ty + 16 * r) * kT + tx + 16 * c;
            P[idx] += acc[r][c];
        }
}

// One thread per element (i, j) of the dense nb x nb matrix; rows fastest.
__global__ void unpack_kernel(const double* __restrict__ partial, int T, int nt, int ntiles, int nsplit, int nb,
                              double divisor, const double* __restrict__ diag, double zpe, double* __restrict__ M,
                              int64_t ld)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)nb * nb) return;
    const int j = (int)(e / nb), i = (int)(e - (int64_t)j * nb);
    const int r = min(i, j), c = max(i, j);
    const int ti = r / T, tj = c / T;
    const int t = ti * nt - ti * (ti - 1) / 2 + (tj - ti);
    const size_t off = (size_t)t * T * T + (size_t)(r - ti * T) * T + (c - tj * T);
    double v = 0.0;
    for (int s = 0; s < nsplit; s++) v += partial[(size_t)s * ntiles * T * T + off];
    v = v / divisor;
    if (diag && i == j) v = (v + diag[i]) + zpe;
    M[(size_t)j * ld + i] = v;
}

}  // namespace

int launch_contract_fp64(const double* phi, const double* w, int64_t ldk, int64_t k, int nb_pad, const TileMap& tm,
                         int nsplit, double* partial, cudaStream_t s)
{
    if (tm.tile != kT || nb_pad != tm.nt * kT || k % ((int64_t)nsplit * kBK) != 0 || ldk % 2 != 0)
        return fail(SCP3GPU_ERR_ARG, "contract_fp64: shapes not tiled");
    if (k == 0) return SCP3GPU_OK;
    dim3 grid(tm.ntiles, nsplit);
    contract_fp64_kernel<<<grid, 256, 0, s>>>(phi, w, ldk, k / nsplit, tm.nt, tm.ntiles, partial);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

int launch_unpack(const double* partial, const TileMap& tm, int nsplit, int nb, double divisor, const double* diag,
                  double zpe, double* M, int64_t ld, cudaStream_t s)
{
    const int64_t total = (int64_t)nb * nb;
    unpack_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(partial, tm.tile, tm.nt, tm.ntiles, nsplit, nb,
                                                                   divisor, diag, zpe, M, ld);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

}  // namespace scp3
