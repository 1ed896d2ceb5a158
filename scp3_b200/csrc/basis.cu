// Basis expansion: for every sample s and basis function i (getBasisSize order,
// ScaledMatrixElements.cpp:870-930), Phi_i(q_s) from the Hermite functions of
// HarmonicOscillatorBasis.cpp:23-41 -- the columns of `bra`, written K-major
// (samples contiguous) so the contraction reads them as its A/B operands.
#include "common.cuh"
#include "internal.h"

namespace scp3 {

namespace {

constexpr int kExpSamples = 64;   // samples per block (threads)
constexpr int kExpRows = 128;     // basis rows per block

__device__ __forceinline__ double ho1(double y) { return 1.4142135623730951 * y; }              // sqrt(2.0)*y
__device__ __forceinline__ double ho2(double y) { return (2.0 * y * y - 1.0) / 1.4142135623730951; }
__device__ __forceinline__ double ho3(double y) { return (2.0 * y * y - 3.0) * y / 1.7320508075688772; }

// qs: [mode][ld] staged q values, sample t of the block
template <int ld = kExpSamples>
__device__ __forceinline__ double basis_value(uint32_t d, const double* qs, int t)
{
    const int m = (d >> 3) & 255, n = (d >> 11) & 255, p = (d >> 19) & 255;
    const double qm = qs[m * ld + t];
    switch (d & 7u) {
        case kGround: return 1.0;
        case kHo1: return ho1(qm);
        case kHo2: return ho2(qm);
        case kHo1Ho1: return ho1(qm) * ho1(qs[n * ld + t]);
        case kHo3: return ho3(qm);
        case kHo2Ho1: return ho2(qm) * ho1(qs[n * ld + t]);
        case kHo1Ho2: return ho1(qm) * ho2(qs[n * ld + t]);
        default: return ho1(qm) * ho1(qs[n * ld + t]) * ho1(qs[p * ld + t]);
    }
}

// grid: x = sample blocks of 64, y = row blocks of 128.  phi/w: [nb_pad][ldk].
__global__ void __launch_bounds__(kExpSamples) expand_fp64_kernel(const uint32_t* __restrict__ desc, int nb,
                                                                   int nb_pad, int nm, const double* __restrict__ q,
                                                                   const double* __restrict__ v, int64_t n,
                                                                   int64_t ldk, double* __restrict__ phi,
                                                                   double* __restrict__ w)
{
    extern __shared__ double qs[];   // [nm][64]
    const int t = threadIdx.x;
    const int64_t s0 = (int64_t)blockIdx.x * kExpSamples;
    for (int e = t; e < nm * kExpSamples; e += kExpSamples) {
        const int ss = e / nm, m = e - ss * nm;          // coalesced read of q[s0+ss][m]
        qs[m * kExpSamples + ss] = (s0 + ss < n) ? q[(s0 + ss) * nm + m] : 0.0;
    }
    __syncthreads();
    const int64_t s = s0 + t;
    if (s >= n) return;
    const double vs = v[s];
    const int r0 = blockIdx.y * kExpRows, r1 = min(r0 + kExpRows, nb_pad);
    for (int i = r0; i < r1; i++) {
        const double val = (i < nb) ? basis_value(__ldg(desc + i), qs, t) : 0.0;
        phi[(size_t)i * ldk + s] = val;
        w[(size_t)i * ldk + s] = val * vs;     // ket = bra * V (ScaledMatrixElements.cpp:964-967)
    }
}

// Sample-major form for the 128 x 128 FP64 contraction: phi/w [n][ld], rows
// contiguous.  grid: x = sample blocks of 64, y = row blocks of 128; 512 threads,
// thread t owning row t % 128 for every fourth sample from t / 128, so each
// sample's 128 rows are one coalesced 1 KB store and four warps per row group
// keep stores in flight.
constexpr int kExpSmThreads = 4 * kExpRows;
constexpr int kExpSmLd = kExpSamples + 1;   // odd stride: a warp's rows read different modes conflict-free

__global__ void __launch_bounds__(kExpSmThreads) expand_fp64_sm_kernel(const uint32_t* __restrict__ desc, int nb,
                                                                       int nm, const double* __restrict__ q,
                                                                       const double* __restrict__ v, int64_t n,
                                                                       int64_t ld, double* __restrict__ phi,
                                                                       double* __restrict__ w)
{
    extern __shared__ double qs[];   // [nm][65]
    const int t = threadIdx.x;
    const int64_t s0 = (int64_t)blockIdx.x * kExpSamples;
    for (int e = t; e < nm * kExpSamples; e += kExpSmThreads) {
        const int ss = e / nm, m = e - ss * nm;          // coalesced read of q[s0+ss][m]
        qs[m * kExpSmLd + ss] = (s0 + ss < n) ? q[(s0 + ss) * nm + m] : 0.0;
    }
    __syncthreads();
    const int i = blockIdx.y * kExpRows + (t % kExpRows);   // < ld: ld is a whole number of row blocks
    const uint32_t d = i < nb ? __ldg(desc + i) : 0u;
    const int ns = (int)min((int64_t)kExpSamples, n - s0);
    for (int ss = t / kExpRows; ss < ns; ss += kExpSmThreads / kExpRows) {
        const double val = (i < nb) ? basis_value<kExpSmLd>(d, qs, ss) : 0.0;
        phi[(size_t)(s0 + ss) * ld + i] = val;
        w[(size_t)(s0 + ss) * ld + i] = val * v[s0 + ss];   // ket = bra * V (ScaledMatrixElements.cpp:964-967)
    }
}

}  // namespace

int launch_expand_fp64_sm(const uint32_t* desc, int nb, int nm, const double* q, const double* v, int64_t n,
                          int64_t ld, double* phi, double* w, cudaStream_t s)
{
    if (n <= 0) return SCP3GPU_OK;
    if (ld % kExpRows != 0) return fail(SCP3GPU_ERR_ARG, "expand_fp64_sm: ld is not a whole number of row blocks");
    const size_t sm = sizeof(double) * nm * kExpSmLd;
    if (sm > 48 * 1024)
        SCP3_CUDA(cudaFuncSetAttribute(expand_fp64_sm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    dim3 grid((unsigned)((n + kExpSamples - 1) / kExpSamples), (unsigned)(ld / kExpRows));
    expand_fp64_sm_kernel<<<grid, kExpSmThreads, sm, s>>>(desc, nb, nm, q, v, n, ld, phi, w);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

int launch_expand_fp64(const uint32_t* desc, int nb, int nb_pad, int nm, const double* q, const double* v, int64_t n,
                       int64_t ldk, double* phi, double* w, cudaStream_t s)
{
    if (n <= 0) return SCP3GPU_OK;
    const size_t sm = sizeof(double) * nm * kExpSamples;
    if (sm > 48 * 1024)
        SCP3_CUDA(cudaFuncSetAttribute(expand_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    dim3 grid((unsigned)((n + kExpSamples - 1) / kExpSamples), (unsigned)((nb_pad + kExpRows - 1) / kExpRows));
    expand_fp64_kernel<<<grid, kExpSamples, sm, s>>>(desc, nb, nb_pad, nm, q, v, n, ldk, phi, w);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

}  // namespace scp3
