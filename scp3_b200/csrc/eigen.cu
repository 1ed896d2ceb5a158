// The lowest eigenpairs of a symmetric matrix on the device: dsyevr(A, IU, &C)
// of eigensolver.cpp:20-84 (LAPACK dsyevr with RANGE = 'I', IL = 1), here
// cuSOLVER's syevdx in FP64.  The triangle read follows the reference: the upper
// one unless A(0, n-1) == 0 (eigensolver.cpp:27-30), which is how a matrix
// holding only its lower triangle is recognised.
#include <cusolverDn.h>

#include <algorithm>

#include "internal.h"

using namespace scp3;

extern "C" int scp3gpu_syevr_lowest(const double* A, int64_t n, int64_t lda, int k, double* W, double* Z, int64_t ldz,
                                    int device)
{
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    if (!A || !W || n < 1 || n > (1ll << 31) - 1 || lda < n || k < 1 || k > n || (Z && ldz < n))
        return fail(SCP3GPU_ERR_ARG, "syevr_lowest: bad arguments");
    int rc = check_device(device);
    if (rc) return rc;
    DeviceGuard g(device);
    const int N = (int)n;
    const cublasFillMode_t uplo = A[(size_t)(n - 1) * lda] == 0.0 ? CUBLAS_FILL_MODE_LOWER : CUBLAS_FILL_MODE_UPPER;
    const cusolverEigMode_t jobz = Z ? CUSOLVER_EIG_MODE_VECTOR : CUSOLVER_EIG_MODE_NOVECTOR;
    double *dA = nullptr, *dW = nullptr, *work = nullptr;
    int* info = nullptr;
    cudaStream_t s = nullptr;
    cusolverDnHandle_t sol = nullptr;
    int lwork = 0, meig = 0, hinfo = 0;
    auto done = [&](int code) {
        if (sol) cusolverDnDestroy(sol);
        if (s) cudaStreamSynchronize(s), cudaStreamDestroy(s);
        cudaFree(dA), cudaFree(dW), cudaFree(work), cudaFree(info);
        return code;
    };
    if ((rc = dalloc(&dA, (size_t)N * N)) || (rc = dalloc(&dW, (size_t)N)) || (rc = dalloc(&info, 1))) return done(rc);
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
        return done(fail(SCP3GPU_ERR_CUDA, "stream creation failed"));
    if (cudaMemcpy2DAsync(dA, sizeof(double) * N, A, sizeof(double) * lda, sizeof(double) * N, N,
                          cudaMemcpyHostToDevice, s) != cudaSuccess)
        return done(fail(SCP3GPU_ERR_CUDA, "syevr_lowest: copy in failed"));
    if (cusolverDnCreate(&sol) != CUSOLVER_STATUS_SUCCESS) return done(fail(SCP3GPU_ERR_CUDA, "cusolverDnCreate failed"));
    cusolverDnSetStream(sol, s);
    if (cusolverDnDsyevdx_bufferSize(sol, jobz, CUSOLVER_EIG_RANGE_I, uplo, N, dA, N, 0.0, 0.0, 1, k, &meig, dW,
                                     &lwork) != CUSOLVER_STATUS_SUCCESS)
        return done(fail(SCP3GPU_ERR_CUDA, "syevdx buffer query failed"));
    if ((rc = dalloc(&work, (size_t)std::max(lwork, 1)))) return done(rc);
    if (cusolverDnDsyevdx(sol, jobz, CUSOLVER_EIG_RANGE_I, uplo, N, dA, N, 0.0, 0.0, 1, k, &meig, dW, work, lwork,
                          info) != CUSOLVER_STATUS_SUCCESS)
        return done(fail(SCP3GPU_ERR_CUDA, "syevdx failed"));
    cudaMemcpyAsync(W, dW, sizeof(double) * k, cudaMemcpyDeviceToHost, s);
    // eigenvectors overwrite the first k columns of the device copy
    if (Z) cudaMemcpy2DAsync(Z, sizeof(double) * ldz, dA, sizeof(double) * N, sizeof(double) * N, k,
                             cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return done(cuda_fail(e, "syevr_lowest"));
    if (hinfo != 0) return done(fail(SCP3GPU_ERR_CUDA, "syevdx did not converge"));
    if (meig != k) return done(fail(SCP3GPU_ERR_CUDA, "#EW returned is different from requested"));
    return done(SCP3GPU_OK);
}
