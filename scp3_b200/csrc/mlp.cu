// The learned surrogate V_nn(q) of the control-variate estimator: a
// 48 -> 256 -> 256 -> 256 -> 1 multilayer perceptron with GELU activations,
// BF16 weights and FP32 accumulation, trained and evaluated on the GPU by the
// kernels below (the reference has no surrogate; SCP3 evaluates the exact
// potential at every point, SCP3.cpp:205-225).
//
//   forward    gemm_bias_gelu_tc: Y = GELU(X W^T + b) on the tcgen05 tensor
//              cores, persistent (one CTA per SM, the layer's weights resident
//              in shared memory), 128-sample tiles against all outputs (M = 128,
//              N = hidden, K = 16 MMAs into one of two FP32 TMEM accumulators,
//              the next tile loaded and multiplied while the last is drained),
//              activations stored BF16 for the next layer and FP32
//              pre-activations kept for training;
//              head_kernel: y = h3 . w4 + b4, one warp per sample
//   backward   FP32 register-tiled GEMMs for dX = dZ W and dW = dZ^T X,
//              gelu_backward for dZ = dH * GELU'(Z), a per-column reduction for
//              the bias gradients
//   update     adam_kernel on FP32 master weights, refreshing the BF16 copies
//
// Layout: weights W_l row-major [out][in] (in padded to a multiple of 32);
// activations row-major [sample][feature].
#include <cuda_bf16.h>

#include <cmath>
#include <utility>
#include <vector>
#include <algorithm>

#include "internal.h"
#include "mlp.h"

namespace scp3 {
namespace mlp {

namespace {

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float z)
{
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

constexpr unsigned long long kWaitNs = 4000000000ull;
#include "tc_ptx.cuh"

// 16-byte cp.async into shared memory, zero-filled (nothing read) when !valid
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(valid ? 16 : 0)
                 : "memory");
}

// Y[M][N] = act(X[M][K] W[N][K]^T + b) on the tensor cores.  X, W BF16
// row-major (K contiguous); N a multiple of 32 up to 256, K a multiple of 32 up
// to 256, any M.  Persistent: a CTA stages all of W once, then takes 128-row
// tiles of X in turn (tile blockIdx.x, + gridDim.x, ...), in the K-major
// 64-byte-swizzled layout the MMA descriptors read (per 32-column K box, row r's
// 16-byte chunk c at c ^ ((r >> 1) & 3)).  Warps 0-3 load a tile with cp.async
// once the previous tile's MMAs have read their buffer, and thread 0 issues its
// K / 16 MMAs of M = 128, N, K = 16 into one of two FP32 TMEM accumulators; warps
// 4-15 drain the other accumulator meanwhile -- warp w reads rows 32 ((w - 4) % 4)
// .. +31 (its TMEM lane quadrant) and every third 32-column chunk from
// 32 ((w - 4) / 4) -- add the bias and write Z (FP32, may be null) and
// H = GELU(Z) (BF16).  Every wait is bounded; after an expiry the CTA stops
// issuing and the tiles it could not finish are written as NaN, which the
// build's non-finite counters report.
constexpr int kTM = 128, kTcThreads = 512, kLoadThreads = 128, kEpiWarpsL = 12;

__host__ __device__ inline size_t tc_smem_bytes(int N, int K)
{
    return (size_t)(K / 32) * (kTM + N) * 64 + 128 + (size_t)N * 4 + 1024;   // operands, barriers, bias, alignment
}

__global__ void __launch_bounds__(kTcThreads, 1) gemm_bias_gelu_tc(const __nv_bfloat16* __restrict__ X,
                                                                const __nv_bfloat16* __restrict__ W,
                                                                const float* __restrict__ b, int M, int N, int K,
                                                                float* __restrict__ Z,
                                                                __nv_bfloat16* __restrict__ H, int apply_gelu)
{
    extern __shared__ uint8_t sm_raw[];
    uint8_t* sm = (uint8_t*)(((uintptr_t)sm_raw + 1023) & ~(uintptr_t)1023);
    const int nkb = K / 32;
    uint8_t* As = sm;                                  // [nkb][128 rows][64 B]
    uint8_t* Bs = sm + (size_t)nkb * kTM * 64;         // [nkb][N rows][64 B]
    uint64_t* done = reinterpret_cast<uint64_t*>(Bs + (size_t)nkb * N * 64);   // [2] MMAs of a tile complete
    uint64_t* freed = done + 2;                        // [2] accumulator drained
    uint32_t* tslot = reinterpret_cast<uint32_t*>(freed + 2);
    volatile int* abort = reinterpret_cast<volatile int*>(tslot + 1);
    volatile int* stop = abort + 1;                    // the loaders' own exit flag, written by thread 0
    float* bias = reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(done) + 128);   // [N]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ntiles = (M + kTM - 1) / kTM;
    const uint32_t ncol = N <= 32 ? 32u : N <= 64 ? 64u : N <= 128 ? 128u : 256u;   // per accumulator
    if (tid == 0) {
        for (int a = 0; a < 2; a++) {
            mbar_init(done + a, 1);
            mbar_init(freed + a, kEpiWarpsL);
        }
        *abort = 0;
        *stop = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(2 * ncol));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    const int kc = K / 8;                              // 16-byte chunks per row
    for (int j = tid; j < N; j += kTcThreads) bias[j] = b[j];
    for (int e = tid; e < N * kc; e += kTcThreads) {
        const int r = e / kc, c = e - r * kc, cc = c & 3;
        cp_async16(Bs + (size_t)(c >> 2) * N * 64 + r * 64 + ((cc ^ ((r >> 1) & 3)) << 4), W + (size_t)r * K + c * 8,
                   true);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // the tensor core reads what was copied
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (warp < kLoadThreads / 32) {
        // loaders and, on thread 0, the MMA issue
        const uint32_t idesc =
            (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kTM >> 4) << 24);
        // Thread 0 alone waits and decides; the other loaders learn the outcome
        // from *stop after a named barrier, so all 128 take the same path
        int i = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, i++) {
            const int a = i & 1;
            // the buffer is free once the previous tile's MMAs have read it
            if (tid == 0 && i > 0 && !mbar_wait(done + ((i - 1) & 1), ((i - 1) >> 1) & 1, abort)) *stop = 1;
            asm volatile("bar.sync 1, %0;" ::"n"(kLoadThreads) : "memory");
            if (*stop) break;
            const int m0 = t * kTM;
            for (int e = tid; e < kTM * kc; e += kLoadThreads) {
                const int r = e / kc, c = e - r * kc, cc = c & 3;
                const bool ok = m0 + r < M;
                cp_async16(As + (size_t)(c >> 2) * kTM * 64 + r * 64 + ((cc ^ ((r >> 1) & 3)) << 4),
                           X + (size_t)(ok ? m0 + r : 0) * K + c * 8, ok);
            }
            asm volatile("cp.async.wait_all;" ::: "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("bar.sync 1, %0;" ::"n"(kLoadThreads) : "memory");
            if (tid == 0) {
                if (!mbar_wait(freed + a, ((i >> 1) & 1) ^ 1, abort)) {   // the epilogue is done with it
                    *stop = 1;
                    *abort = 1;
                } else {
                    tc_fence_after();
                    const uint32_t d = tmem + (uint32_t)a * ncol;
                    for (int kb = 0; kb < nkb; kb++) {
                        const uint64_t ad = smem_desc64(As + (size_t)kb * kTM * 64);
                        const uint64_t bd = smem_desc64(Bs + (size_t)kb * N * 64);
#pragma unroll
                        for (int kk = 0; kk < 2; kk++) mma_bf16(d, ad + 2 * kk, bd + 2 * kk, idesc, (kb | kk) != 0);
                    }
                    mma_commit(done + a);
                }
            }
        }
        // the epilogue waits for the last tile's MMAs before the CTA frees TMEM
    } else {
        const int ew = warp - kLoadThreads / 32, quad = ew & 3, grp = ew >> 2;
        int i = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, i++) {
            const int a = i & 1;
            // warp-uniform outcome: the TMEM loads below are warp-collective
            const bool ok = __all_sync(0xffffffffu, mbar_wait(done + a, (i >> 1) & 1, abort));
            tc_fence_after();
            const int row = t * kTM + quad * 32 + lane;
            for (int c0 = grp * 32; c0 < N; c0 += 32 * (kEpiWarpsL / 4)) {
                float v[32];
                __syncwarp();
                if (ok) tmem_ld32(tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(a * ncol + c0), v);
                if (row < M) {
                    // 8 columns at a time: one 16-byte store of H, two of Z
#pragma unroll
                    for (int j = 0; j < 32; j += 8) {
                        const float4 b0 = *reinterpret_cast<const float4*>(bias + c0 + j);
                        const float4 b1 = *reinterpret_cast<const float4*>(bias + c0 + j + 4);
                        const float bj[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
                        float z[8];
#pragma unroll
                        for (int e = 0; e < 8; e++) z[e] = ok ? v[j + e] + bj[e] : __int_as_float(0x7fc00000);
                        if (Z) {
                            float4* zp = reinterpret_cast<float4*>(Z + (size_t)row * N + c0 + j);
                            zp[0] = make_float4(z[0], z[1], z[2], z[3]);
                            zp[1] = make_float4(z[4], z[5], z[6], z[7]);
                        }
                        uint32_t hv[4];
#pragma unroll
                        for (int e = 0; e < 4; e++) {
                            const float h0 = apply_gelu ? gelu(z[2 * e]) : z[2 * e];
                            const float h1 = apply_gelu ? gelu(z[2 * e + 1]) : z[2 * e + 1];
                            const __nv_bfloat162 hb = __floats2bfloat162_rn(h0, h1);
                            hv[e] = *reinterpret_cast<const uint32_t*>(&hb);
                        }
                        *reinterpret_cast<uint4*>(H + (size_t)row * N + c0 + j) = make_uint4(hv[0], hv[1], hv[2], hv[3]);
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(freed + a);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * ncol));
    }
}

int launch_layer(const __nv_bfloat16* X, const __nv_bfloat16* W, const float* b, int M, int N, int K, float* Z,
                 __nv_bfloat16* H, cudaStream_t s)
{
    if (N % 32 || N > 256 || K % 32 || K > 256) return fail(SCP3GPU_ERR_ARG, "mlp layer: shape out of range");
    const size_t sm = tc_smem_bytes(N, K);
    SCP3_CUDA(cudaFuncSetAttribute(gemm_bias_gelu_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int dev = 0, sms = 148;
    SCP3_CUDA(cudaGetDevice(&dev));
    SCP3_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int tiles = (M + kTM - 1) / kTM;
    gemm_bias_gelu_tc<<<(unsigned)std::max(1, std::min(tiles, sms)), kTcThreads, sm, s>>>(X, W, b, M, N, K, Z, H, 1);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

// y[m] = H[m][:] . w + b, one warp per sample.
__global__ void head_kernel(const __nv_bfloat16* __restrict__ H, const float* __restrict__ w, float b, int M, int K,
                            float scale, float shift, float* __restrict__ y)
{
    const int m = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (m >= M) return;
    float s = 0.0f;
    for (int k = lane; k < K; k += 32) s += __bfloat162float(H[(size_t)m * K + k]) * w[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[m] = (s + b) * scale + shift;
}

// Input features: q (M x nin, FP32) -> BF16 rows of width kin (zero padded).
__global__ void input_kernel(const float* __restrict__ q, int M, int nin, int kin, __nv_bfloat16* __restrict__ X)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)M * kin) return;
    const int m = (int)(e / kin), k = (int)(e - (int64_t)m * kin);
    X[e] = __float2bfloat16_rn(k < nin ? q[(size_t)m * nin + k] : 0.0f);
}

// Generic FP32 GEMM C[M][N] = sum_k A(m,k) B(k,n) with strided operands (A(m,k)
// at A[m*sam + k*sak], B(k,n) at B[k*sbk + n*sbn]), 64x64 tiles, 4x4 per thread.
template <typename TA, typename TB>
__global__ void __launch_bounds__(256) gemm_f32(const TA* __restrict__ A, int64_t sam, int64_t sak,
                                                 const TB* __restrict__ B, int64_t sbk, int64_t sbn, int M, int N, int K,
                                                 float* __restrict__ C, int64_t ldc, float beta)
{
    __shared__ float As[16][65], Bs[16][65];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int m0 = blockIdx.x * 64, n0 = blockIdx.y * 64;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += 16) {
        for (int e = tid; e < 64 * 16; e += 256) {
            const int r = e >> 4, k = e & 15;
            const int m = m0 + r, n = n0 + r, kk = k0 + k;
            As[k][r] = (m < M && kk < K) ? (float)A[m * sam + kk * sak] : 0.0f;
            Bs[k][r] = (n < N && kk < K) ? (float)B[kk * sbk + n * sbn] : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; k++) {
            float av[4], bv[4];
#pragma unroll
            for (int i = 0; i < 4; i++) av[i] = As[k][ty + 16 * i], bv[i] = Bs[k][tx + 16 * i];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] += av[i] * bv[j];
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int m = m0 + ty + 16 * i, n = n0 + tx + 16 * j;
            if (m < M && n < N) C[(size_t)m * ldc + n] = acc[i][j] + (beta != 0.0f ? beta * C[(size_t)m * ldc + n] : 0.0f);
        }
}

__global__ void gelu_backward(const float* __restrict__ Z, float* __restrict__ dH, int64_t n)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) dH[e] *= gelu_grad(Z[e]);
}

// Column sums (bias gradient): out[n] = sum_m D[m][n].
__global__ void colsum(const float* __restrict__ D, int M, int N, float* __restrict__ out)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.0f;
    for (int m = 0; m < M; m++) s += D[(size_t)m * N + n];
    out[n] = s;
}

// MSE loss on normalised targets: d = (y - t)/M ... dy = 2 (y - t) / M, loss accumulated.
__global__ void mse_grad(const float* __restrict__ y, const float* __restrict__ t, int M, float* __restrict__ dy,
                         float* __restrict__ loss)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (m < M) {
        const float d = y[m] - t[m];
        dy[m] = 2.0f * d / M;
        l = d * d / M;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                            float* __restrict__ m2, int64_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2, __nv_bfloat16* __restrict__ pb, int rows, int cols, int cols_pad)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const float gr = g[e];
    const float a = m1[e] = b1 * m1[e] + (1 - b1) * gr;
    const float s = m2[e] = b2 * m2[e] + (1 - b2) * gr * gr;
    const float v = p[e] -= lr * (a / c1) / (sqrtf(s / c2) + eps);
    if (pb) {
        const int r = (int)(e / cols), c = (int)(e - (int64_t)r * cols);
        pb[(size_t)r * cols_pad + c] = __float2bfloat16_rn(v);
    }
}

int blocks(int64_t n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

__global__ void normalise_kernel(const float* y, const float* t, int M, float scale, float shift, float* yr, float* tr)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    yr[m] = (y[m] - shift) / scale;
    tr[m] = (t[m] - shift) / scale;
}

// ------------------------------------------------------------------ host side

int Net::alloc(int n_in_, int hidden_, int max_batch_)
{
    n_in = n_in_;
    hid = hidden_;
    kin = (n_in + 31) / 32 * 32;
    max_batch = (max_batch_ + 63) / 64 * 64;
    const int ins[4] = {n_in, hid, hid, hid}, outs[4] = {hid, hid, hid, 1};
    for (int l = 0; l < 4; l++) {
        in[l] = ins[l];
        out[l] = outs[l];
        inpad[l] = l == 0 ? kin : hid;
        const size_t nw = (size_t)out[l] * in[l];
        SCP3_CUDA(cudaMalloc(&w[l], sizeof(float) * nw));
        SCP3_CUDA(cudaMalloc(&b[l], sizeof(float) * out[l]));
        SCP3_CUDA(cudaMalloc(&gw[l], sizeof(float) * nw));
        SCP3_CUDA(cudaMalloc(&gb[l], sizeof(float) * out[l]));
        SCP3_CUDA(cudaMalloc(&mw[l], sizeof(float) * nw * 2));
        SCP3_CUDA(cudaMalloc(&mb[l], sizeof(float) * out[l] * 2));
        SCP3_CUDA(cudaMemset(mw[l], 0, sizeof(float) * nw * 2));
        SCP3_CUDA(cudaMemset(mb[l], 0, sizeof(float) * out[l] * 2));
        SCP3_CUDA(cudaMalloc(&wb[l], sizeof(__nv_bfloat16) * (size_t)out[l] * inpad[l]));
        SCP3_CUDA(cudaMemset(wb[l], 0, sizeof(__nv_bfloat16) * (size_t)out[l] * inpad[l]));
    }
    SCP3_CUDA(cudaMalloc(&X, sizeof(__nv_bfloat16) * (size_t)max_batch * kin));
    for (int l = 0; l < 3; l++) {
        SCP3_CUDA(cudaMalloc(&Z[l], sizeof(float) * (size_t)max_batch * hid));
        SCP3_CUDA(cudaMalloc(&H[l], sizeof(__nv_bfloat16) * (size_t)max_batch * hid));
    }
    SCP3_CUDA(cudaMalloc(&dA, sizeof(float) * (size_t)max_batch * hid));
    SCP3_CUDA(cudaMalloc(&dB, sizeof(float) * (size_t)max_batch * hid));
    SCP3_CUDA(cudaMalloc(&ybuf, sizeof(float) * max_batch));
    SCP3_CUDA(cudaMalloc(&dy, sizeof(float) * max_batch));
    SCP3_CUDA(cudaMalloc(&loss, sizeof(float)));
    return SCP3GPU_OK;
}

void Net::free_all()
{
    for (int l = 0; l < 4; l++) {
        void* ps[] = {w[l], b[l], gw[l], gb[l], mw[l], mb[l], wb[l]};
        for (void* p : ps)
            if (p) cudaFree(p);
    }
    void* ps[] = {X, Z[0], Z[1], Z[2], H[0], H[1], H[2], dA, dB, ybuf, dy, loss};
    for (void* p : ps)
        if (p) cudaFree(p);
}

// Refresh the BF16 copy of layer l's weights from the FP32 masters.
__global__ void to_bf16_padded(const float* __restrict__ w, int rows, int cols, int cols_pad,
                               __nv_bfloat16* __restrict__ wb)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)rows * cols) return;
    const int r = (int)(e / cols), c = (int)(e - (int64_t)r * cols);
    wb[(size_t)r * cols_pad + c] = __float2bfloat16_rn(w[e]);
}

int Net::sync_bf16(cudaStream_t s)
{
    for (int l = 0; l < 4; l++) {
        const int64_t n = (int64_t)out[l] * in[l];
        to_bf16_padded<<<blocks(n, 256), 256, 0, s>>>(w[l], out[l], in[l], inpad[l], wb[l]);
    }
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

// Forward for M samples (M <= max_batch, any M): y (device, M floats) in
// target units (y_raw * scale + shift).
int Net::forward(const float* q, int M, float* y, cudaStream_t s)
{
    if (M <= 0) return SCP3GPU_OK;
    if (M > max_batch) return fail(SCP3GPU_ERR_ARG, "mlp forward: batch larger than the allocation");
    const int Mp = (M + 63) / 64 * 64;
    input_kernel<<<blocks((int64_t)Mp * kin, 256), 256, 0, s>>>(q, M, n_in, kin, X);
    if (Mp > M) SCP3_CUDA(cudaMemsetAsync(X + (size_t)M * kin, 0, sizeof(__nv_bfloat16) * (size_t)(Mp - M) * kin, s));
    const __nv_bfloat16* in_act = X;
    for (int l = 0; l < 3; l++) {
        if (int rc = launch_layer(in_act, wb[l], b[l], Mp, hid, inpad[l], Z[l], H[l], s)) return rc;
        in_act = H[l];
    }
    head_kernel<<<blocks(M, 8), 256, 0, s>>>(H[2], w[3], 0.0f, M, hid, 1.0f, 0.0f, y);
    SCP3_CUDA(cudaGetLastError());
    // head bias and output scaling are applied by a small kernel
    return apply_output(y, M, s);
}

__global__ void affine_kernel(float* y, int M, const float* b, float scale, float shift);

size_t Net::infer_workspace(int M) const
{
    const size_t Mp = (size_t)(M + 63) / 64 * 64;
    return Mp * kin + 2 * Mp * hid;
}

int Net::infer(const float* q, int M, float* y, cudaStream_t s, __nv_bfloat16* Xw, __nv_bfloat16* Ha,
               __nv_bfloat16* Hb) const
{
    if (M <= 0) return SCP3GPU_OK;
    const int Mp = (M + 63) / 64 * 64;
    input_kernel<<<blocks((int64_t)Mp * kin, 256), 256, 0, s>>>(q, M, n_in, kin, Xw);
    if (Mp > M) SCP3_CUDA(cudaMemsetAsync(Xw + (size_t)M * kin, 0, sizeof(__nv_bfloat16) * (size_t)(Mp - M) * kin, s));
    const __nv_bfloat16* in_act = Xw;
    __nv_bfloat16* outs[3] = {Ha, Hb, Ha};
    for (int l = 0; l < 3; l++) {
        if (int rc = launch_layer(in_act, wb[l], b[l], Mp, hid, inpad[l], nullptr, outs[l], s)) return rc;
        in_act = outs[l];
    }
    head_kernel<<<blocks(M, 8), 256, 0, s>>>(in_act, w[3], 0.0f, M, hid, 1.0f, 0.0f, y);
    affine_kernel<<<blocks(M, 256), 256, 0, s>>>(y, M, b[3], out_scale, out_shift);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

__global__ void affine_kernel(float* y, int M, const float* b, float scale, float shift)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < M) y[m] = (y[m] + b[0]) * scale + shift;
}

int Net::apply_output(float* y, int M, cudaStream_t s)
{
    affine_kernel<<<blocks(M, 256), 256, 0, s>>>(y, M, b[3], out_scale, out_shift);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

// Loss and gradients of the mean squared error against targets t (device, in
// target units) for M samples (multiple of 64); gradients land in gw/gb.
int Net::backward(const float* q, const float* t, int M, cudaStream_t s, float* loss_out)
{
    if (M % 64 != 0 || M > max_batch) return fail(SCP3GPU_ERR_ARG, "mlp backward: batch must be a multiple of 64");
    int rc = forward(q, M, ybuf, s);
    if (rc) return rc;
    // normalised residual: dL/dy_raw with y_raw = (y - shift)/scale
    SCP3_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), s));
    {
        // targets into raw units in dB (scratch), outputs into raw units in dA
        normalise_kernel<<<blocks(M, 256), 256, 0, s>>>(ybuf, t, M, out_scale, out_shift, dA, dB);
        mse_grad<<<blocks(M, 256), 256, 0, s>>>(dA, dB, M, dy, loss);
    }
    // head: gw3[k] = sum_m dy[m] H2[m][k]; gb3 = sum dy; dH2 = dy w3^T
    gemm_f32<float, __nv_bfloat16><<<dim3(1, blocks(hid, 64)), 256, 0, s>>>(dy, 0, 1, H[2], hid, 1, 1, hid, M,
                                                                              gw[3], hid, 0.0f);
    colsum<<<1, 32, 0, s>>>(dy, M, 1, gb[3]);
    gemm_f32<float, float><<<dim3(blocks(M, 64), blocks(hid, 64)), 256, 0, s>>>(dy, 1, 0, w[3], 0, 1, M, hid, 1,
                                                                              dA, hid, 0.0f);
    for (int l = 2; l >= 0; l--) {
        gelu_backward<<<blocks((int64_t)M * hid, 256), 256, 0, s>>>(Z[l], dA, (int64_t)M * hid);   // dZ_l
        // gw_l[o][i] = sum_m dZ[m][o] Xin[m][i]
        const __nv_bfloat16* Xin = l == 0 ? X : H[l - 1];
        const int ld_in = inpad[l];
        gemm_f32<float, __nv_bfloat16><<<dim3(blocks(hid, 64), blocks(in[l], 64)), 256, 0, s>>>(
            dA, 1, hid, Xin, ld_in, 1, hid, in[l], M, gw[l], in[l], 0.0f);
        colsum<<<blocks(hid, 128), 128, 0, s>>>(dA, M, hid, gb[l]);
        if (l > 0) {   // dH_{l-1}[m][i] = sum_o dZ[m][o] W_l[o][i]
            gemm_f32<float, float><<<dim3(blocks(M, 64), blocks(hid, 64)), 256, 0, s>>>(dA, hid, 1, w[l], in[l], 1, M,
                                                                                      hid, hid, dB, hid, 0.0f);
            std::swap(dA, dB);
        }
    }
    SCP3_CUDA(cudaGetLastError());
    if (loss_out) {
        SCP3_CUDA(cudaMemcpyAsync(loss_out, loss, sizeof(float), cudaMemcpyDeviceToHost, s));
        SCP3_CUDA(cudaStreamSynchronize(s));
    }
    return SCP3GPU_OK;
}

int Net::adam(float lr, cudaStream_t s)
{
    step++;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    for (int l = 0; l < 4; l++) {
        const int64_t nw = (int64_t)out[l] * in[l];
        adam_kernel<<<blocks(nw, 256), 256, 0, s>>>(w[l], gw[l], mw[l], mw[l] + nw, nw, lr, b1, b2, eps, c1, c2,
                                                    l < 3 ? wb[l] : nullptr, out[l], in[l], inpad[l]);
        adam_kernel<<<blocks(out[l], 256), 256, 0, s>>>(b[l], gb[l], mb[l], mb[l] + out[l], out[l], lr, b1, b2, eps,
                                                        c1, c2, nullptr, 1, 1, 1);
    }
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

}  // namespace mlp
}  // namespace scp3

// ------------------------------------------------------------------ C ABI
using namespace scp3;

struct scp3gpu_mlp {
    mlp::Net net;
    int dev = 0;
    cudaStream_t s = nullptr;
    float* qbuf = nullptr;   // staging for host calls: max_batch x n_in
    float* tbuf = nullptr;
};

namespace {

uint64_t sm64(uint64_t& x)
{
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct Dev {
    int prev = -1;
    explicit Dev(int d)
    {
        cudaGetDevice(&prev);
        if (prev != d) cudaSetDevice(d);
    }
    ~Dev()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

__global__ void gather_rows(const float* __restrict__ src, const int* __restrict__ idx, int n, int w,
                            float* __restrict__ dst)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * w) return;
    const int r = (int)(e / w), c = (int)(e - (int64_t)r * w);
    dst[e] = src[(size_t)idx[r] * w + c];
}

}  // namespace

extern "C" {

int64_t scp3gpu_mlp_num_params(const scp3gpu_mlp* m)
{
    if (!m) return -1;
    int64_t n = 0;
    for (int l = 0; l < 4; l++) n += (int64_t)m->net.out[l] * m->net.in[l] + m->net.out[l];
    return n;
}

int scp3gpu_mlp_destroy(scp3gpu_mlp* m)
{
    if (!m) return SCP3GPU_OK;
    Dev g(m->dev);
    if (m->s) cudaStreamSynchronize(m->s);
    m->net.free_all();
    if (m->qbuf) cudaFree(m->qbuf);
    if (m->tbuf) cudaFree(m->tbuf);
    if (m->s) cudaStreamDestroy(m->s);
    delete m;
    return SCP3GPU_OK;
}

int scp3gpu_mlp_create(int n_in, int hidden, int max_batch, uint64_t seed, int device, scp3gpu_mlp** out)
{
    (void)cudaGetLastError();
    if (!out || n_in < 1 || n_in > 256 || hidden < 64 || hidden > 256 || hidden % 64 != 0 || max_batch < 64)
        return fail(SCP3GPU_ERR_ARG, "mlp_create: n_in 1..256, hidden 64, 128, 192 or 256, max_batch >= 64");
    *out = nullptr;
    int nd = 0;
    if (cudaGetDeviceCount(&nd) != cudaSuccess || device < 0 || device >= nd)
        return fail(SCP3GPU_ERR_UNSUPPORTED, "no such CUDA device");
    Dev g(device);
    scp3gpu_mlp* m = new scp3gpu_mlp();
    m->dev = device;
    int rc = m->net.alloc(n_in, hidden, max_batch);
    if (!rc && cudaStreamCreateWithFlags(&m->s, cudaStreamNonBlocking) != cudaSuccess)
        rc = fail(SCP3GPU_ERR_CUDA, "stream creation failed");
    if (!rc && (cudaMalloc(&m->qbuf, sizeof(float) * (size_t)m->net.max_batch * n_in) != cudaSuccess ||
                cudaMalloc(&m->tbuf, sizeof(float) * (size_t)m->net.max_batch) != cudaSuccess))
        rc = fail(SCP3GPU_ERR_NOMEM, "mlp staging allocation failed");
    if (rc) {
        scp3gpu_mlp_destroy(m);
        return rc;
    }
    // Glorot-uniform weights, zero biases, from one splitmix64 stream
    uint64_t st = seed;
    for (int l = 0; l < 4; l++) {
        const int fi = m->net.in[l], fo = m->net.out[l];
        const double a = std::sqrt(6.0 / (fi + fo));
        std::vector<float> w((size_t)fi * fo), b(fo, 0.0f);
        for (float& x : w) x = (float)(a * (2.0 * ((sm64(st) >> 11) * 0x1p-53) - 1.0));
        if (cudaMemcpy(m->net.w[l], w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(m->net.b[l], b.data(), sizeof(float) * b.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
            scp3gpu_mlp_destroy(m);
            return fail(SCP3GPU_ERR_CUDA, "mlp init copy failed");
        }
    }
    if ((rc = m->net.sync_bf16(m->s)) || cudaStreamSynchronize(m->s) != cudaSuccess) {
        scp3gpu_mlp_destroy(m);
        return rc ? rc : fail(SCP3GPU_ERR_CUDA, "mlp init failed");
    }
    *out = m;
    return SCP3GPU_OK;
}

int scp3gpu_mlp_set_output(scp3gpu_mlp* m, float scale, float shift)
{
    if (!m || !(scale > 0.0f)) return fail(SCP3GPU_ERR_ARG, "mlp_set_output: scale must be positive");
    m->net.out_scale = scale;
    m->net.out_shift = shift;
    return SCP3GPU_OK;
}

int scp3gpu_mlp_get_params(scp3gpu_mlp* m, float* p, int64_t n)
{
    if (!m || !p || n != scp3gpu_mlp_num_params(m)) return fail(SCP3GPU_ERR_ARG, "mlp_get_params: bad size");
    Dev g(m->dev);
    SCP3_CUDA(cudaStreamSynchronize(m->s));
    for (int l = 0; l < 4; l++) {
        const size_t nw = (size_t)m->net.out[l] * m->net.in[l];
        SCP3_CUDA(cudaMemcpy(p, m->net.w[l], sizeof(float) * nw, cudaMemcpyDeviceToHost));
        p += nw;
        SCP3_CUDA(cudaMemcpy(p, m->net.b[l], sizeof(float) * m->net.out[l], cudaMemcpyDeviceToHost));
        p += m->net.out[l];
    }
    return SCP3GPU_OK;
}

int scp3gpu_mlp_set_params(scp3gpu_mlp* m, const float* p, int64_t n)
{
    (void)cudaGetLastError();
    if (!m || !p || n != scp3gpu_mlp_num_params(m)) return fail(SCP3GPU_ERR_ARG, "mlp_set_params: bad size");
    Dev g(m->dev);
    SCP3_CUDA(cudaStreamSynchronize(m->s));
    for (int l = 0; l < 4; l++) {
        const size_t nw = (size_t)m->net.out[l] * m->net.in[l];
        SCP3_CUDA(cudaMemcpy(m->net.w[l], p, sizeof(float) * nw, cudaMemcpyHostToDevice));
        p += nw;
        SCP3_CUDA(cudaMemcpy(m->net.b[l], p, sizeof(float) * m->net.out[l], cudaMemcpyHostToDevice));
        p += m->net.out[l];
    }
    int rc = m->net.sync_bf16(m->s);
    if (rc) return rc;
    SCP3_CUDA(cudaStreamSynchronize(m->s));
    return SCP3GPU_OK;
}

int scp3gpu_mlp_forward(scp3gpu_mlp* m, const float* q, int64_t n, float* y)
{
    (void)cudaGetLastError();
    if (!m || n < 0 || (n > 0 && (!q || !y))) return fail(SCP3GPU_ERR_ARG, "mlp_forward: bad arguments");
    Dev g(m->dev);
    const int nin = m->net.n_in, B = m->net.max_batch;
    for (int64_t off = 0; off < n; off += B) {
        const int c = (int)std::min<int64_t>(B, n - off);
        SCP3_CUDA(cudaMemcpyAsync(m->qbuf, q + off * nin, sizeof(float) * c * nin, cudaMemcpyHostToDevice, m->s));
        int rc = m->net.forward(m->qbuf, c, m->tbuf, m->s);
        if (rc) return rc;
        SCP3_CUDA(cudaMemcpyAsync(y + off, m->tbuf, sizeof(float) * c, cudaMemcpyDeviceToHost, m->s));
    }
    SCP3_CUDA(cudaStreamSynchronize(m->s));
    return SCP3GPU_OK;
}

int scp3gpu_mlp_grad(scp3gpu_mlp* m, const float* q, const float* t, int n, float* loss, float* grad)
{
    (void)cudaGetLastError();
    if (!m || !q || !t || n < 64 || n % 64 != 0 || n > m->net.max_batch)
        return fail(SCP3GPU_ERR_ARG, "mlp_grad: n must be a multiple of 64 within the batch size");
    Dev g(m->dev);
    float* td = nullptr;
    SCP3_CUDA(cudaMalloc(&td, sizeof(float) * n));
    SCP3_CUDA(cudaMemcpyAsync(m->qbuf, q, sizeof(float) * (size_t)n * m->net.n_in, cudaMemcpyHostToDevice, m->s));
    SCP3_CUDA(cudaMemcpyAsync(td, t, sizeof(float) * n, cudaMemcpyHostToDevice, m->s));
    int rc = m->net.backward(m->qbuf, td, n, m->s, loss);
    cudaFree(td);
    if (rc) return rc;
    if (grad)
        for (int l = 0; l < 4; l++) {
            const size_t nw = (size_t)m->net.out[l] * m->net.in[l];
            SCP3_CUDA(cudaMemcpy(grad, m->net.gw[l], sizeof(float) * nw, cudaMemcpyDeviceToHost));
            grad += nw;
            SCP3_CUDA(cudaMemcpy(grad, m->net.gb[l], sizeof(float) * m->net.out[l], cudaMemcpyDeviceToHost));
            grad += m->net.out[l];
        }
    return SCP3GPU_OK;
}

// Adam on the mean squared error of normalised targets, cosine-decayed
// learning rate, a seeded shuffle per epoch; the data stay on the device.
int scp3gpu_mlp_train(scp3gpu_mlp* m, const float* q, const float* t, int64_t n, int epochs, int batch, float lr,
                      uint64_t seed, float* final_loss)
{
    (void)cudaGetLastError();
    if (!m || !q || !t || n < batch || batch < 64 || batch % 64 != 0 || batch > m->net.max_batch || epochs < 1)
        return fail(SCP3GPU_ERR_ARG, "mlp_train: bad sizes");
    Dev g(m->dev);
    const int nin = m->net.n_in;
    float *qd = nullptr, *td = nullptr;
    int* idx = nullptr;
    int rc = SCP3GPU_OK;
    if (cudaMalloc(&qd, sizeof(float) * (size_t)n * nin) != cudaSuccess || cudaMalloc(&td, sizeof(float) * n) != cudaSuccess ||
        cudaMalloc(&idx, sizeof(int) * n) != cudaSuccess) {
        cudaFree(qd), cudaFree(td), cudaFree(idx);
        return fail(SCP3GPU_ERR_NOMEM, "mlp_train: data allocation failed");
    }
    if (cudaMemcpyAsync(qd, q, sizeof(float) * (size_t)n * nin, cudaMemcpyHostToDevice, m->s) != cudaSuccess ||
        cudaMemcpyAsync(td, t, sizeof(float) * n, cudaMemcpyHostToDevice, m->s) != cudaSuccess) {
        cudaFree(qd), cudaFree(td), cudaFree(idx);
        return fail(SCP3GPU_ERR_CUDA, "mlp_train: data copy failed");
    }
    std::vector<int> perm(n);
    for (int64_t i = 0; i < n; i++) perm[i] = (int)i;
    uint64_t st = seed;
    const int64_t nbatch = n / batch, total = nbatch * epochs;
    int64_t k = 0;
    float loss = 0.0f;
    for (int e = 0; e < epochs && !rc; e++) {
        for (int64_t i = n - 1; i > 0; i--) std::swap(perm[i], perm[sm64(st) % (uint64_t)(i + 1)]);
        if (cudaMemcpyAsync(idx, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, m->s) != cudaSuccess)
            rc = fail(SCP3GPU_ERR_CUDA, "mlp_train: permutation copy failed");
        for (int64_t bi = 0; bi < nbatch && !rc; bi++, k++) {
            gather_rows<<<(unsigned)((batch * nin + 255) / 256), 256, 0, m->s>>>(qd, idx + bi * batch, batch, nin, m->qbuf);
            gather_rows<<<(unsigned)((batch + 255) / 256), 256, 0, m->s>>>(td, idx + bi * batch, batch, 1, m->tbuf);
            const bool last = k == total - 1;
            rc = m->net.backward(m->qbuf, m->tbuf, batch, m->s, last ? &loss : nullptr);
            const float lr_k = lr * (0.05f + 0.95f * 0.5f * (1.0f + cosf(3.14159265f * (float)k / (float)total)));
            if (!rc) rc = m->net.adam(lr_k, m->s);
        }
        cudaStreamSynchronize(m->s);   // the host permutation is reused next epoch
    }
    cudaError_t ce = cudaStreamSynchronize(m->s);
    cudaFree(qd), cudaFree(td), cudaFree(idx);
    if (rc) return rc;
    if (ce != cudaSuccess) return cuda_fail(ce, "mlp_train");
    if (final_loss) *final_loss = loss;
    return SCP3GPU_OK;
}

}  // extern "C"

namespace scp3 {
mlp::Net* mlp_net(scp3gpu_mlp* m) { return m ? &m->net : nullptr; }
int mlp_device(const scp3gpu_mlp* m) { return m ? m->dev : -1; }
}  // namespace scp3
