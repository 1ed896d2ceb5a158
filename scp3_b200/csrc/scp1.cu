// SCP1 thermal averages (SCP1.cpp:34-90, SCP1::average) on the GPU.
//
// For Sobol points i of the unscrambled sequence at offset `skip` (dimension
// dim = 9 nw, every Cartesian coordinate), each sample is
//
//   y  = std_normal(dim) % sqrt(d)                       (SCP1.cpp:54-58)
//   dq = isqrtM_U y,   r = bohr (q + dq)                  (SCP1.cpp:60-61)
//   V  = pes(r) / autokcal,  g = dV/dr * bohr / autokcal  (SCP1.cpp:62-63)
//
// and the call returns the sums over its points of V, g and g dq^T (the
// reference's per-rank partials before its MPI_Allreduce, SCP1.cpp:65-80).
//
// Two kernels per chunk of samples:
//   scp1_samples_kernel   (sampling.cu, beside the potentials' constant tables)
//                         one warp per sample (contiguous, balanced ranges per
//                         warp, Gray-code Sobol walk), isqrtM_U staged in
//                         shared memory, the potential's energy and gradient
//                         (the same warp code as the gradient estimator); writes
//                         V, g and dq per sample.
//   scp1_reduce_kernel    R = sum_s [g_s, V_s] [dq_s, 1]^T, a (dim+1)^2 grid of
//                         FP64 sums: every block owns a fixed sample range and
//                         adds into its own partial, so the result does not
//                         depend on scheduling; a last kernel adds the block
//                         partials in block order.
#include "common.cuh"
#include "internal.h"

#include <algorithm>
#include <cmath>
#include <vector>

struct scp3gpu_scp1 {
    int pes = 0, nw = 0, dim = 0, device = 0;
    int64_t chunk = 0;
    int blocks = 0;                 // reduction blocks (fixed per handle)
    cudaStream_t stream = nullptr;
    int64_t* vdir = nullptr;        // [62][dim] direction numbers
    uint32_t* tasks = nullptr;
    int ntasks = 0;
    double* q = nullptr;            // [dim]
    double* sqd = nullptr;          // [dim] sqrt(d)
    double* U = nullptr;            // [dim*dim] isqrtM_U, column-major
    double* V = nullptr;            // [chunk]
    double* G = nullptr;            // [chunk][dim]
    double* D = nullptr;            // [chunk][dim]
    double* P = nullptr;            // [blocks][(dim+1)^2] block partials
    double* R = nullptr;            // [(dim+1)^2]
    int* iters = nullptr;           // [chunk] TTM3-F dipole iterations
    long long not_converged = 0;
};

namespace scp3 {
namespace {

constexpr int kRedThreads = 256, kRedPer = 16, kRedRows = 32;

// P[block] += sum over the block's samples of [g, V] [dq, 1]^T, column-major
// (dim+1) x (dim+1); element page blockIdx.y of kRedThreads * kRedPer elements.
__global__ void __launch_bounds__(kRedThreads) scp1_reduce_kernel(int dim, int64_t n, const double* __restrict__ V,
                                                                  const double* __restrict__ G,
                                                                  const double* __restrict__ D, double* __restrict__ P)
{
    __shared__ double sg[kRedRows][80], sd[kRedRows][80];    // dim + 1 <= 80
    const int E1 = dim + 1, E = E1 * E1;
    const int t = threadIdx.x;
    const int e0 = blockIdx.y * kRedThreads * kRedPer;
    int ia[kRedPer], ib[kRedPer];
    double acc[kRedPer];
#pragma unroll
    for (int k = 0; k < kRedPer; k++) {
        const int e = e0 + t + kRedThreads * k;
        ia[k] = e < E ? e % E1 : 0;
        ib[k] = e < E ? e / E1 : 0;
        acc[k] = 0.0;
    }
    const int64_t s0 = n * blockIdx.x / gridDim.x, s1 = n * (blockIdx.x + 1) / gridDim.x;
    for (int64_t c0 = s0; c0 < s1; c0 += kRedRows) {
        const int rows = (int)(s1 - c0 < kRedRows ? s1 - c0 : kRedRows);
        __syncthreads();
        for (int e = t; e < rows * E1; e += kRedThreads) {
            const int r = e / E1, c = e - r * E1;
            const int64_t s = c0 + r;
            sg[r][c] = c < dim ? G[s * dim + c] : V[s];
            sd[r][c] = c < dim ? D[s * dim + c] : 1.0;
        }
        __syncthreads();
        for (int r = 0; r < rows; r++) {
#pragma unroll
            for (int k = 0; k < kRedPer; k++) acc[k] += sg[r][ia[k]] * sd[r][ib[k]];
        }
    }
    double* Pb = P + (size_t)blockIdx.x * E;
#pragma unroll
    for (int k = 0; k < kRedPer; k++) {
        const int e = e0 + t + kRedThreads * k;
        if (e < E) Pb[e] += acc[k];
    }
}

__global__ void scp1_sum_kernel(int E, int blocks, const double* __restrict__ P, double* __restrict__ R)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    double s = 0.0;
    for (int b = 0; b < blocks; b++) s += P[(size_t)b * E + e];
    R[e] = s;
}

void free_all(scp3gpu_scp1* h)
{
    void* p[] = {h->vdir, h->tasks, h->q, h->sqd, h->U, h->V, h->G, h->D, h->P, h->R, h->iters};
    for (void* x : p)
        if (x) cudaFree(x);
    if (h->stream) cudaStreamDestroy(h->stream);
}

}  // namespace
}  // namespace scp3

using namespace scp3;

extern "C" {

int scp3gpu_scp1_create(int pes, int nw, int64_t chunk, int device, scp3gpu_scp1** out)
{
    (void)cudaGetLastError();
    if (!out) return fail(SCP3GPU_ERR_ARG, "scp1_create: null handle pointer");
    *out = nullptr;
    if (pes != SCP3GPU_PES_QTIP4PF && pes != SCP3GPU_PES_TTM3F) return fail(SCP3GPU_ERR_ARG, "unknown potential");
    if (nw < 1 || nw > 8) return fail(SCP3GPU_ERR_ARG, "scp1: 1 <= nw <= 8");
    if (chunk < 0) return fail(SCP3GPU_ERR_ARG, "scp1: negative chunk");
    int rc = check_device(device);
    if (rc) return rc;
    DeviceGuard guard(device);
    if (pes == SCP3GPU_PES_TTM3F && (rc = ttm_init_device())) return rc;
    scp3gpu_scp1* h = new scp3gpu_scp1;
    h->pes = pes;
    h->nw = nw;
    h->dim = 9 * nw;
    h->device = device;
    h->chunk = chunk > 0 ? (chunk + 31) / 32 * 32 : (1 << 16);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    h->blocks = 2 * sms;
    const int dim = h->dim, E = (dim + 1) * (dim + 1);
    std::vector<int64_t> v;
    std::vector<uint64_t> sh;
    const std::vector<uint32_t> t = pair_tasks(nw);
    h->ntasks = (int)t.size();
    if ((rc = sobol_tables(dim, 0, 0, v, sh)) || (rc = upload(&h->vdir, v.data(), v.size())) ||
        (rc = upload(&h->tasks, t.data(), t.size())) || (rc = dalloc(&h->q, dim)) || (rc = dalloc(&h->sqd, dim)) ||
        (rc = dalloc(&h->U, (size_t)dim * dim)) || (rc = dalloc(&h->V, h->chunk)) ||
        (rc = dalloc(&h->G, (size_t)h->chunk * dim)) || (rc = dalloc(&h->D, (size_t)h->chunk * dim)) ||
        (rc = dalloc(&h->P, (size_t)h->blocks * E)) || (rc = dalloc(&h->R, E)) || (rc = dalloc(&h->iters, h->chunk))) {
        free_all(h);
        delete h;
        return rc;
    }
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        free_all(h);
        delete h;
        return fail(SCP3GPU_ERR_CUDA, "scp1: stream creation failed");
    }
    *out = h;
    return SCP3GPU_OK;
}

int scp3gpu_scp1_average(scp3gpu_scp1* h, const double* q, const double* d, const double* isqrtM_U, int64_t skip,
                         int64_t i0, int64_t i1, double* Upot, double* UX, double* UX_q)
{
    (void)cudaGetLastError();
    if (!h || !q || !d || !isqrtM_U || !Upot || !UX || !UX_q)
        return fail(SCP3GPU_ERR_ARG, "scp1_average: null handle or pointer");
    if (skip < 0 || i0 < 0 || i1 < i0 || skip + i1 >= (1ll << kLogMax))
        return fail(SCP3GPU_ERR_ARG, "scp1_average: bad Sobol range");
    DeviceGuard guard(h->device);
    const int dim = h->dim, E1 = dim + 1, E = E1 * E1;
    std::vector<double> sqd(dim);
    for (int k = 0; k < dim; k++) {
        if (!(d[k] >= 0.0)) return fail(SCP3GPU_ERR_ARG, "scp1_average: d must be >= 0");
        sqd[k] = std::sqrt(d[k]);
    }
    cudaStream_t s = h->stream;
    SCP3_CUDA(cudaMemcpyAsync(h->q, q, sizeof(double) * dim, cudaMemcpyHostToDevice, s));
    SCP3_CUDA(cudaMemcpyAsync(h->sqd, sqd.data(), sizeof(double) * dim, cudaMemcpyHostToDevice, s));
    SCP3_CUDA(cudaMemcpyAsync(h->U, isqrtM_U, sizeof(double) * dim * dim, cudaMemcpyHostToDevice, s));
    SCP3_CUDA(cudaMemsetAsync(h->P, 0, sizeof(double) * (size_t)h->blocks * E, s));
    std::vector<int> it;
    int rc = SCP3GPU_OK;
    for (int64_t c0 = i0; c0 < i1; c0 += h->chunk) {
        const int64_t n = std::min<int64_t>(h->chunk, i1 - c0);
        Scp1Args a{h->nw, dim, h->q, h->sqd, h->U, h->vdir, skip + c0, n, h->tasks, h->ntasks, h->V, h->G, h->D,
                   h->iters};
        if ((rc = launch_scp1_samples(h->pes, a, s))) return rc;
        const int pages = (E + kRedThreads * kRedPer - 1) / (kRedThreads * kRedPer);
        scp1_reduce_kernel<<<dim3(h->blocks, pages), kRedThreads, 0, s>>>(dim, n, h->V, h->G, h->D, h->P);
        SCP3_CUDA(cudaGetLastError());
        if (h->pes == SCP3GPU_PES_TTM3F) {
            it.resize(n);
            SCP3_CUDA(cudaMemcpyAsync(it.data(), h->iters, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
            SCP3_CUDA(cudaStreamSynchronize(s));
            for (int64_t k = 0; k < n; k++) h->not_converged += it[k] > kTtmMaxIter;
        }
    }
    scp1_sum_kernel<<<(E + 255) / 256, 256, 0, s>>>(E, h->blocks, h->P, h->R);
    SCP3_CUDA(cudaGetLastError());
    std::vector<double> R(E);
    SCP3_CUDA(cudaMemcpyAsync(R.data(), h->R, sizeof(double) * E, cudaMemcpyDeviceToHost, s));
    SCP3_CUDA(cudaStreamSynchronize(s));
    for (int j = 0; j < dim; j++)
        for (int i = 0; i < dim; i++) UX_q[(size_t)j * dim + i] = R[(size_t)j * E1 + i];
    for (int i = 0; i < dim; i++) UX[i] = R[(size_t)dim * E1 + i];
    *Upot = R[(size_t)dim * E1 + dim];
    return SCP3GPU_OK;
}

int scp3gpu_scp1_status(const scp3gpu_scp1* h, int64_t* not_converged)
{
    if (!h || !not_converged) return fail(SCP3GPU_ERR_ARG, "scp1_status: null handle or pointer");
    *not_converged = h->not_converged;
    return SCP3GPU_OK;
}

void scp3gpu_scp1_destroy(scp3gpu_scp1* h)
{
    if (!h) return;
    DeviceGuard guard(h->device);
    free_all(h);
    delete h;
}

}  // extern "C"
