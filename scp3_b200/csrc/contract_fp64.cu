// Plain-form (FP64) contraction M_ij += sum_s Phi_i(s) V_s Phi_j(s) over the
// upper-triangle tiles only -- what dsyr2k('U','N',0.5,bra,ket,1,M) computes in
// the reference (ScaledMatrixElements.cpp:942-949, 970) -- plus the unpack of
// the tile partial sums into a dense column-major matrix.
//
// FP64 has no tcgen05 path; both kernels here are register-tiled DFMA.  The first
// (the addEpot entry without device allocation uses it) takes a 64x64 tile per
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

// ---------------------------------------------------------------------------
// The build's FP64 contraction: 128 x 128 tiles over sample-major operands.
//
// phi and w are [sample][row] (rows contiguous, leading dimension ld = nb_pad, a
// multiple of 128), so a K slice of a tile's 128 rows is kBK2 contiguous 1 KB
// runs that 16-byte cp.async copies put straight into shared memory as
// [k][row], in three stages.  256 threads each own an 8 x 8 block of the tile:
// rows 32g + 2*ty + {0,1} and columns 32g + 2*tx + {0,1} for g = 0..3, so per K
// step a thread reads its 8 A and 8 B values with four 16-byte loads each
// (a warp's A loads touch two addresses, its B loads 256 contiguous bytes) and
// issues 64 DFMAs: one shared-memory load per 8 DFMAs, where the 64 x 64 kernel
// above needs one per 2.  The partial is the same [split][tile][T*T] row-major
// layout with T = 128, so launch_unpack reads it unchanged.
constexpr int kT2 = 128, kBK2 = 16, kStages2 = 3;
constexpr size_t kSmem2 = sizeof(double) * kStages2 * 2 * kBK2 * kT2;   // 96 KB

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// kRect = false: the upper-triangle tiles of A A'-shaped work (A = phi, B = w,
// one leading dimension), tile index row-major over ti <= tj.  kRect = true:
// every tile of an (rt x nt)-tile rectangle, A and B with their own leading
// dimensions (tile t = ti * nt + tj).
template <bool kRect>
__global__ void __launch_bounds__(256, 1) contract_fp64_t128_kernel(const double* __restrict__ phi,
                                                                     const double* __restrict__ w, int64_t lda,
                                                                     int64_t ldb, int64_t kps, int nt, int ntiles,
                                                                     double* __restrict__ partial)
{
    extern __shared__ __align__(16) double sm2[];   // [stage][A, B][kBK2][kT2]
    int ti = 0, tj = 0;
    if (kRect) {
        ti = blockIdx.x / nt;
        tj = blockIdx.x - ti * nt;
    } else {
        int t = blockIdx.x;
        while (t >= nt - ti) {
            t -= nt - ti;
            ti++;
        }
        tj = ti + t;
    }
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int64_t k0 = (int64_t)blockIdx.y * kps;
    const double* ga = phi + k0 * lda + (size_t)ti * kT2;
    const double* gb = w + k0 * ldb + (size_t)tj * kT2;
    const int nkb = (int)(kps / kBK2);

    // stage load: 2 x kBK2 x 128 doubles = 2 x 1024 chunks of 16 B, 4 + 4 per thread
    auto load = [&](int stage, int kb) {
        double* sa = sm2 + (size_t)stage * 2 * kBK2 * kT2;
        double* sb = sa + kBK2 * kT2;
        const size_t ka = (size_t)kb * kBK2 * lda, kb_ = (size_t)kb * kBK2 * ldb;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int c = tid + 256 * i, k = c >> 6, col = (c & 63) * 2;
            cp_async16(sa + k * kT2 + col, ga + ka + (size_t)k * lda + col);
            cp_async16(sb + k * kT2 + col, gb + kb_ + (size_t)k * ldb + col);
        }
    };

    double acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = 0.0;

#pragma unroll
    for (int st = 0; st < kStages2 - 1; st++) {
        if (st < nkb) load(st, st);
        cp_async_commit();
    }
    for (int kb = 0; kb < nkb; kb++) {
        cp_async_wait<kStages2 - 2>();   // stage kb has landed (this thread's copies)
        __syncthreads();                 // ... and every thread's; stage kb-1 is free again
        if (kb + kStages2 - 1 < nkb) load((kb + kStages2 - 1) % kStages2, kb + kStages2 - 1);
        cp_async_commit();
        const double* sa = sm2 + (size_t)(kb % kStages2) * 2 * kBK2 * kT2;
        const double* sb = sa + kBK2 * kT2;
#pragma unroll
        for (int k = 0; k < kBK2; k++) {
            double a[8], b[8];
#pragma unroll
            for (int g = 0; g < 4; g++) {
                const double2 va = *reinterpret_cast<const double2*>(sa + k * kT2 + 32 * g + 2 * ty);
                const double2 vb = *reinterpret_cast<const double2*>(sb + k * kT2 + 32 * g + 2 * tx);
                a[2 * g] = va.x, a[2 * g + 1] = va.y;
                b[2 * g] = vb.x, b[2 * g + 1] = vb.y;
            }
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 8; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
    }
    cp_async_wait<0>();
    double* P = partial + ((size_t)blockIdx.y * ntiles + blockIdx.x) * (kT2 * kT2);
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int r = 32 * (i >> 1) + 2 * ty + (i & 1);
#pragma unroll
        for (int g = 0; g < 4; g++) {
            double2* p = reinterpret_cast<double2*>(P + r * kT2 + 32 * g + 2 * tx);
            double2 o = *p;
            o.x += acc[i][2 * g];
            o.y += acc[i][2 * g + 1];
            *p = o;
        }
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

int launch_contract_fp64_t128(const double* phi, const double* w, int64_t ld, int64_t k, const TileMap& tm,
                              int nsplit, double* partial, cudaStream_t s)
{
    if (tm.tile != kT2 || ld != (int64_t)tm.nt * kT2 || k % ((int64_t)nsplit * kBK2) != 0)
        return fail(SCP3GPU_ERR_ARG, "contract_fp64_t128: shapes not tiled");
    if (k == 0) return SCP3GPU_OK;
    SCP3_CUDA(cudaFuncSetAttribute(contract_fp64_t128_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)kSmem2));
    dim3 grid(tm.ntiles, nsplit);
    contract_fp64_t128_kernel<false><<<grid, 256, kSmem2, s>>>(phi, w, ld, ld, k / nsplit, tm.nt, tm.ntiles, partial);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

int launch_gemm_fp64_rect(const double* A, int64_t lda, const double* B, int64_t ldb, int64_t k, int rt, int ct,
                          int nsplit, double* partial, cudaStream_t s)
{
    if (lda < (int64_t)rt * kT2 || ldb < (int64_t)ct * kT2 || lda % 2 || ldb % 2 || k % ((int64_t)nsplit * kBK2))
        return fail(SCP3GPU_ERR_ARG, "gemm_fp64_rect: shapes not tiled");
    if (k == 0) return SCP3GPU_OK;
    SCP3_CUDA(cudaFuncSetAttribute(contract_fp64_t128_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)kSmem2));
    dim3 grid(rt * ct, nsplit);
    contract_fp64_t128_kernel<true><<<grid, 256, kSmem2, s>>>(A, B, lda, ldb, k / nsplit, ct, rt * ct, partial);
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
