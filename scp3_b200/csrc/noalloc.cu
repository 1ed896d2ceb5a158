// scp3gpu_add_epot_static: the FP64 accumulation of the -G path on caller device
// buffers, for callers that cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is unavailable or not allowed --
// inside a memory pool or arena owned by someone else (a framework that hands
// out only pre-planned buffers), in a process whose allocator is locked down by
// a host application, or in a latency-critical loop that must never touch the
// allocator.  Such callers own q, V and M but cannot give the contraction its
// working space.  This entry point takes that working space from one
// file-scope __device__ array of kStaticScratchBytes (64 MiB), which every GPU
// that loads the library keeps until the process exits.
//
// It computes what scp3gpu_hbuild_add_epot computes, sum_s Phi(q_s) V_s
// Phi(q_s)^T added into M, in FP64 with the same basis expansion; its
// contraction is the 64 x 64 tile kernel, whose partial sums take a quarter of
// the space of the build's 128 x 128 tiles.
//
// Rules of use:
//  * The first call on a device looks up the array's device address
//    (cudaGetSymbolAddress, once per device, with that device current); make
//    that first call before any stream capture on that device.
//  * All calls share the one array and it keeps the last call's contents; each
//    call clears what must start at zero.  Calls whose work overlaps on the GPU
//    (different streams, or different host threads, without ordering between
//    them) race on the array: order them on one stream or synchronise.
//  * Bases that do not fit the array (see the size check) are rejected with
//    SCP3GPU_ERR_ARG; nothing here calls cudaMalloc, cudaFree or any allocating
//    library routine.
#include <mutex>

#include "internal.h"

namespace scp3 {

namespace {

constexpr size_t kStaticScratchBytes = 64ull << 20;
__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_static_mu;
void* g_static_addr[128] = {nullptr};

int static_scratch(void** out)
{
    int dev = 0;
    SCP3_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 128) return fail(SCP3GPU_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(static scratch)");
        g_static_addr[dev] = p;
    }
    *out = g_static_addr[dev];
    return SCP3GPU_OK;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Adds the tile partials (split-summed) into M, both triangles.
__global__ void add_partials_kernel(const double* __restrict__ partial, int nt, int ntiles, int nsplit, int nb,
                                    double* __restrict__ M, int64_t ld)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)nb * nb) return;
    const int j = (int)(e / nb), i = (int)(e - (int64_t)j * nb);
    const int r = min(i, j), c = max(i, j);
    const int ti = r / 64, tj = c / 64;
    const int t = ti * nt - ti * (ti - 1) / 2 + (tj - ti);
    const size_t off = (size_t)t * 64 * 64 + (size_t)(r - ti * 64) * 64 + (c - tj * 64);
    double v = 0.0;
    for (int s = 0; s < nsplit; s++) v += partial[(size_t)s * ntiles * 64 * 64 + off];
    M[(size_t)j * ld + i] += v;
}

}  // namespace
}  // namespace scp3

using namespace scp3;

extern "C" int scp3gpu_add_epot_static(int nmodes, int n2, int n3, const double* q_dev, const double* V_dev, int64_t n,
                                       double* M_dev, int64_t ld, void* stream)
{
    (void)cudaGetLastError();
    const int64_t nb64 = scp3gpu_basis_size(nmodes, n2, n3);
    if (nb64 < 0 || nmodes < 1 || nmodes > kMaxModes) return fail(SCP3GPU_ERR_ARG, "add_epot_static: bad mode counts");
    if (n < 0 || (n > 0 && (!q_dev || !V_dev)) || !M_dev || ld < nb64)
        return fail(SCP3GPU_ERR_ARG, "add_epot_static: bad sample count, pointer or leading dimension");
    if (n == 0) return SCP3GPU_OK;
    const int nb = (int)nb64;
    TileMap tm;
    tm.tile = 64;
    tm.nt = (nb + 63) / 64;
    tm.ntiles = tm.nt * (tm.nt + 1) / 2;
    const int nb_pad = tm.nt * 64;
    // fit: descriptors + Phi and W of one chunk + the tile partials
    const size_t desc_b = align256(sizeof(uint32_t) * nb);
    const size_t part_tile_b = sizeof(double) * 64 * 64 * tm.ntiles;
    int64_t chunk = 4096;
    int nsplit = 4;
    auto need = [&](int64_t k, int s) { return desc_b + align256(sizeof(double) * nb_pad * k) * 2 + part_tile_b * s; };
    while (nsplit > 1 && need(16 * nsplit, nsplit) > kStaticScratchBytes) nsplit /= 2;
    while (chunk > 16 * nsplit && need(chunk, nsplit) > kStaticScratchBytes) chunk /= 2;
    if (need(chunk, nsplit) > kStaticScratchBytes)
        return fail(SCP3GPU_ERR_ARG, "add_epot_static: a basis of " + std::to_string(nb) +
                                         " functions does not fit the 64 MiB static scratch (at most 4032)");
    void* base = nullptr;
    int rc = static_scratch(&base);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char* p = static_cast<unsigned char*>(base);
    uint32_t* desc = reinterpret_cast<uint32_t*>(p);
    double* phi = reinterpret_cast<double*>(p + desc_b);
    double* w = reinterpret_cast<double*>(p + desc_b + align256(sizeof(double) * nb_pad * chunk));
    double* partial = reinterpret_cast<double*>(p + desc_b + 2 * align256(sizeof(double) * nb_pad * chunk));

    const std::vector<uint32_t> d = basis_descriptors(nmodes, n2, n3);
    SCP3_CUDA(cudaMemcpyAsync(desc, d.data(), sizeof(uint32_t) * d.size(), cudaMemcpyHostToDevice, s));
    SCP3_CUDA(cudaMemsetAsync(partial, 0, part_tile_b * nsplit, s));
    for (int64_t off = 0; off < n; off += chunk) {
        const int64_t c = std::min(chunk, n - off);
        const int64_t kpad = (c + 16 * nsplit - 1) / (16 * nsplit) * (16 * nsplit);
        if (kpad != c) {   // columns past the last sample must hold zeros, not the previous call's values
            SCP3_CUDA(cudaMemsetAsync(phi, 0, sizeof(double) * nb_pad * chunk, s));
            SCP3_CUDA(cudaMemsetAsync(w, 0, sizeof(double) * nb_pad * chunk, s));
        }
        if ((rc = launch_expand_fp64(desc, nb, nb_pad, nmodes, q_dev + off * nmodes, V_dev + off, c, chunk, phi, w,
                                     s)))
            return rc;
        if ((rc = launch_contract_fp64(phi, w, chunk, kpad, nb_pad, tm, nsplit, partial, s))) return rc;
    }
    const int64_t total = (int64_t)nb * nb;
    add_partials_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(partial, tm.nt, tm.ntiles, nsplit, nb, M_dev,
                                                                        ld);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}
