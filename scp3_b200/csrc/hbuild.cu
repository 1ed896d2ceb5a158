// The C ABI of libscp3gpu.so (include/scp3gpu.h): handle lifecycle, the chunked
// sample loop of SCP3_a (SCP3.cpp:154-272) on the device, the -r normals path,
// read-out, eigenvalues and status.
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "internal.h"
#include "tc.h"
#include "mlp.h"

namespace scp3 {
mlp::Net* mlp_net(scp3gpu_mlp* m);
int mlp_device(const scp3gpu_mlp* m);
}

namespace scp3 {

static thread_local std::string g_err;
void set_error(const std::string& m) { g_err = m; }
int fail(int code, const std::string& m)
{
    g_err = m;
    return code;
}
int cuda_fail(cudaError_t e, const char* what)
{
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? SCP3GPU_ERR_NOMEM : SCP3GPU_ERR_CUDA;
}

}  // namespace scp3

using namespace scp3;

struct scp3gpu_hbuild {
    scp3gpu_config cfg{};
    std::vector<double> omega_sel;
    double zpe_inactive = 0.0;
    int dev = 0, sms = 148;
    cudaStream_t stream = nullptr, copy_stream = nullptr, prep_stream = nullptr;
    cudaEvent_t copied[2] = {nullptr, nullptr}, consumed[2] = {nullptr, nullptr};
    cudaEvent_t prepared[2] = {nullptr, nullptr}, contracted[2] = {nullptr, nullptr};
    cudaEvent_t head_done[2] = {nullptr, nullptr};   // a pass's whole waves of contraction units done
    int64_t pass = 0;                 // split form: passes launched (buffer = pass & 1)
    int nb = 0, nb_pad = 0, ntasks = 0, nsplit = 1;
    int64_t chunk = 0;
    TileMap tm{};
    bool split_form = false;
    bool pes_fp32 = false;
    // tables
    int64_t* vdir = nullptr;
    uint64_t* shift = nullptr;
    double *x0 = nullptr, *MUa = nullptr, *omega = nullptr;
    int* modes = nullptr;
    uint32_t *tasks = nullptr, *desc = nullptr;
    // per chunk
    double* q64 = nullptr;
    float* q32 = nullptr;             // split form: q32 / vv[buffer]
    double* v = nullptr;
    float* q32b[2] = {nullptr, nullptr};
    double* vb[2] = {nullptr, nullptr};
    double* normals[2] = {nullptr, nullptr};
    double *phi = nullptr, *w = nullptr;
    double* vq = nullptr;             // gradient path: dV_anh/dq of the selected modes, [chunk][nmodes]
    bool gradient = false;
    SteinPlan sp{};                   // gradient path: tables, operands and sums
    double* partial = nullptr;
    tc::Plan tcp{};
    // read-out
    double* dense = nullptr;
    double* hodiag = nullptr;
    unsigned long long* counters = nullptr;
    int64_t count = 0;
    // learned surrogate
    scp3gpu_mlp* sur = nullptr;
    int sur_mode = SCP3GPU_SURROGATE_NONE;
    float* ybuf = nullptr;
    __nv_bfloat16* sur_ws = nullptr;  // the network's activations for this build's passes
    // kernel timing
    bool prof = false;
    std::vector<cudaEvent_t> pev;
    std::vector<int> pkind;
};

namespace {

int64_t round_up(int64_t a, int64_t b) { return (a + b - 1) / b * b; }

// Records an event on the handle's stream before (open) and after (close) a
// launch when timing is on.
struct Timed {
    scp3gpu_hbuild* h;
    int kind;
    cudaStream_t st;
    Timed(scp3gpu_hbuild* h_, int kind_, cudaStream_t s = nullptr) : h(h_), kind(kind_), st(s ? s : h_->stream)
    {
        mark();
    }
    ~Timed() { mark(); }
    void mark()
    {
        if (!h->prof) return;
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        cudaEventRecord(e, st);
        h->pev.push_back(e);
        h->pkind.push_back(kind);
    }
};

// Samples per device pass and the split of each pass over CTAs of a tile, plain
// FP64 form with the direct estimator: 128 x 128 tiles with one CTA per SM
// (contract_fp64_t128_kernel), in passes of 2^16 samples by default (fewer where
// Phi and W of a pass would pass ~4 GB), so a unit's partial write-back is spread
// over at least 8192 samples at the usual split.  Sample ranges per tile (nsplit, a
// power of two, each range at least 2048 samples) minimise the waves of units
// per unit of work: the units of a pass run in ceil(units / sms) waves.  (The
// gradient estimator plans its own passes: stein_create.)
void plan_fp64(scp3gpu_hbuild* h, int sms)
{
    const int T = 128;
    h->tm.tile = T;
    h->tm.nt = (h->nb + T - 1) / T;
    h->tm.ntiles = h->tm.nt * (h->tm.nt + 1) / 2;
    h->nb_pad = h->tm.nt * T;
    int64_t chunk = h->cfg.chunk > 0 ? h->cfg.chunk : 65536;
    // keep Phi and W of one pass under ~4 GB
    while (chunk > 4096 && (int64_t)h->nb_pad * chunk * 16 > (4ll << 30)) chunk /= 2;
    h->chunk = chunk;
    int nsplit = 1;
    double best = 1e300;
    for (int ns = 1; chunk / ns >= 2048 && chunk % (16ll * ns) == 0; ns *= 2) {
        const int64_t units = (int64_t)h->tm.ntiles * ns;
        const double cost = (double)((units + sms - 1) / sms) / ns;   // waves per unit of work
        if (cost < best - 1e-9) best = cost, nsplit = ns;
    }
    h->nsplit = nsplit;
}

}  // namespace
namespace scp3 {
namespace hb {
int launch_combine(int mode, double* v, const float* y, int64_t nvalid, cudaStream_t s);
}
}  // namespace scp3
namespace {

// One pass.  Plain form: everything on the handle's stream.  Split form: the
// per-sample kernel, sign partition and expansion run on the prepare stream into
// pass buffer (pass & 1), alongside the previous pass's contraction on the main
// stream when that contraction leaves SMs free (otherwise after it); events
// order buffer reuse.  `copied` (may be null): event the normals copy of
// this pass completes; the pass records `consumed` once it has read them.
int launch_chunk(scp3gpu_hbuild* h, int64_t index0, int64_t nvalid, const double* normals_dev,
                 const float* normals32_dev = nullptr, cudaEvent_t copied = nullptr, cudaEvent_t consumed = nullptr)
{
    const bool fp32 = h->pes_fp32;
    const int b = (int)(h->pass & 1);
    SampleArgs a{};
    a.nw = h->cfg.nw;
    a.nm0 = h->cfg.nmodes0;
    a.nm = h->cfg.nmodes;
    a.x0 = h->x0;
    a.MUa = h->MUa;
    a.omega = h->omega;
    a.modes = h->modes;
    a.vdir = h->vdir;
    a.shift = h->shift;
    a.tasks = h->tasks;
    a.ntasks = h->ntasks;
    a.normals = normals_dev;
    a.normals32 = normals32_dev;
    a.index0 = index0;
    a.n = h->split_form ? tc::pass_samples(h->tcp, nvalid)
                        : h->gradient ? stein_pass_samples(h->sp, nvalid) : round_up(nvalid, 16ll * h->nsplit);
    a.nvalid = nvalid;
    a.q64 = h->split_form ? nullptr : h->q64;
    a.q32 = h->split_form ? h->q32b[b] : nullptr;
    a.v = h->split_form ? h->vb[b] : h->v;
    a.counters = h->counters;
    a.skip_pes = h->sur_mode == SCP3GPU_SURROGATE_REPLACE;
    a.vq = h->gradient ? h->vq : nullptr;
    int rc;
    if (h->split_form) {
        cudaStream_t ps = h->prep_stream;
        SCP3_CUDA(cudaStreamWaitEvent(ps, h->contracted[b], 0));   // buffer b free again
        // A contraction with a CTA on (nearly) every SM leaves no room for the
        // preparation kernels (released with it, they would take SMs its CTAs
        // wait for): prepare once its whole waves are done, on the SMs its last,
        // partial wave leaves idle.  Smaller contractions share the GPU with the
        // next pass's preparation.
        if (h->tcp.grid * 8 >= h->sms * 7) SCP3_CUDA(cudaStreamWaitEvent(ps, h->head_done[b ^ 1], 0));
        if (copied) SCP3_CUDA(cudaStreamWaitEvent(ps, copied, 0));
        {
            Timed t(h, 0, ps);
            rc = launch_samples(h->cfg.pes, fp32, a, ps);
        }
        if (rc) return rc;
        if (consumed) SCP3_CUDA(cudaEventRecord(consumed, ps));
        if (h->sur) {
            Timed t(h, 1, ps);
            const mlp::Net* net = mlp_net(h->sur);
            const size_t mp = (size_t)(a.n + 63) / 64 * 64;
            __nv_bfloat16* X = h->sur_ws;
            __nv_bfloat16* Ha = X + mp * net->kin;
            rc = net->infer(a.q32, (int)a.n, h->ybuf, ps, X, Ha, Ha + mp * net->hid);
            if (!rc) rc = hb::launch_combine(h->sur_mode, a.v, h->ybuf, nvalid, ps);
            if (rc) return rc;
        }
        rc = tc::prepare(h->tcp, b, h->nb, h->cfg.nmodes, a.q32, a.v, a.n, ps, h->prof ? &h->pev : nullptr,
                         h->prof ? &h->pkind : nullptr);
        if (rc) return rc;
        SCP3_CUDA(cudaEventRecord(h->prepared[b], ps));
        SCP3_CUDA(cudaStreamWaitEvent(h->stream, h->prepared[b], 0));
        rc = tc::contract(h->tcp, b, a.n, h->stream, h->prof ? &h->pev : nullptr, h->prof ? &h->pkind : nullptr,
                          h->head_done[b]);
        if (rc) return rc;
        SCP3_CUDA(cudaEventRecord(h->contracted[b], h->stream));
        h->pass++;
        return SCP3GPU_OK;
    }
    if (copied) SCP3_CUDA(cudaStreamWaitEvent(h->stream, copied, 0));
    {
        Timed t(h, 0);
        rc = launch_samples(h->cfg.pes, fp32, a, h->stream);
    }
    if (rc) return rc;
    if (consumed) SCP3_CUDA(cudaEventRecord(consumed, h->stream));
    if (h->gradient) {
        Timed t(h, 2);
        return stein_pass(h->sp, h->desc, h->q64, h->v, h->vq, a.n, h->stream);
    }
    {
        Timed t(h, 1);
        rc = launch_expand_fp64_sm(h->desc, h->nb, h->cfg.nmodes, h->q64, h->v, a.n, h->nb_pad, h->phi, h->w,
                                   h->stream);
    }
    if (rc) return rc;
    Timed t(h, 2);
    return launch_contract_fp64_t128(h->phi, h->w, h->nb_pad, a.n, h->tm, h->nsplit, h->partial, h->stream);
}

}  // namespace

namespace scp3 {
namespace hb {
__global__ void combine_kernel(int mode, double* __restrict__ v, const float* __restrict__ y, int64_t n)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    v[s] = mode == SCP3GPU_SURROGATE_REPLACE ? (double)y[s] : v[s] - (double)y[s];
}

int launch_combine(int mode, double* v, const float* y, int64_t nvalid, cudaStream_t s)
{
    if (nvalid <= 0) return SCP3GPU_OK;
    combine_kernel<<<(unsigned)((nvalid + 255) / 256), 256, 0, s>>>(mode, v, y, nvalid);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}
}  // namespace hb
}  // namespace scp3

namespace {

// Work on the prepare stream (split form) finished before the host goes on.
int drain_prep(scp3gpu_hbuild* h)
{
    if (h->prep_stream) SCP3_CUDA(cudaStreamSynchronize(h->prep_stream));
    return SCP3GPU_OK;
}

int zero_sums(scp3gpu_hbuild* h)
{
    if (h->split_form) return tc::zero(h->tcp, h->stream);
    if (h->gradient) return stein_zero(h->sp, h->stream);
    SCP3_CUDA(cudaMemsetAsync(h->partial, 0, sizeof(double) * (size_t)h->nsplit * h->tm.ntiles * h->tm.tile *
                                                 h->tm.tile, h->stream));
    return SCP3GPU_OK;
}


// The -r path for normals of type T (double, or float for the FP32 entry): the
// host buffer goes in piece by piece into two device buffers (FP64-sized, so
// either type fits), each copy on the copy stream overlapped with the previous
// piece's pass.  The first copy overlaps nothing, so the pieces ramp up: 2^15,
// 2^15, 2^16, 2^17, 2^17, then 2^18 samples (at ~50 GB/s a piece's FP32
// normals copy in about 0.7 of its pass; the second 2^17 piece lets the copies
// get ahead before they double again, and the longer pieces after it make
// fewer passes).
template <typename T>
int accumulate_host_normals(scp3gpu_hbuild* h, const T* normals, int64_t n, const char* who)
{
    if (!h || n < 0 || (n > 0 && !normals)) return fail(SCP3GPU_ERR_ARG, who);
    DeviceGuard g(h->dev);
    (void)cudaGetLastError();
    const int nm0 = h->cfg.nmodes0;
    int rc = SCP3GPU_OK;
    for (int b = 0; b < 2 && !h->normals[b]; b++)
        if ((rc = dalloc(&h->normals[b], (size_t)h->chunk * nm0))) return rc;
    // A failed step ends the loop but not the function: copies already queued
    // from the caller's buffer are waited for before returning, so the caller
    // may free or reuse that buffer as soon as the call returns, error or not.
    // h->count then holds the samples whose passes were queued.
    auto step = [&](int64_t off, int64_t c, int b) -> int {
        T* dst = reinterpret_cast<T*>(h->normals[b]);
        // the copy into buffer b may start once the pass that last read it is done
        SCP3_CUDA(cudaStreamWaitEvent(h->copy_stream, h->consumed[b], 0));
        SCP3_CUDA(cudaMemcpyAsync(dst, normals + off * nm0, sizeof(T) * c * nm0, cudaMemcpyHostToDevice,
                                  h->copy_stream));
        SCP3_CUDA(cudaEventRecord(h->copied[b], h->copy_stream));
        const double* d64 = sizeof(T) == 8 ? reinterpret_cast<const double*>(dst) : nullptr;
        const float* d32 = sizeof(T) == 4 ? reinterpret_cast<const float*>(dst) : nullptr;
        return launch_chunk(h, 0, c, d64, d32, h->copied[b], h->consumed[b]);
    };
    int k = 0;
    for (int64_t off = 0, c = 0; off < n && rc == SCP3GPU_OK; off += c, k++) {
        static const int kRamp[] = {15, 15, 16, 17, 17};
        const int64_t part = (int64_t)1 << (k < 5 ? kRamp[k] : 18);
        c = std::min(std::min(h->chunk, part), n - off);
        if ((rc = step(off, c, k & 1)) == SCP3GPU_OK) h->count += c;
    }
    const cudaError_t e = cudaStreamSynchronize(h->copy_stream);
    if (rc != SCP3GPU_OK) return rc;
    if (e != cudaSuccess) return scp3::cuda_fail(e, "accumulate_host_normals: copy stream");
    return SCP3GPU_OK;
}
}  // namespace

extern "C" {

const char* scp3gpu_last_error(void) { return g_err.c_str(); }
int scp3gpu_version(void) { return 100; }

int64_t scp3gpu_basis_size(int nm, int n2, int n3)
{
    if (nm < 0 || n2 < 0 || n3 < 0 || n2 > nm || n3 > nm) return -1;
    return 1 + (int64_t)nm + (int64_t)n2 * (n2 + 1) / 2 + (int64_t)n3 * (1 + n3) * (2 + n3) / 6;
}

int64_t scp3gpu_sub_basis_size(int nm, int n2, int n3, int level)
{
    if (scp3gpu_basis_size(nm, n2, n3) < 0) return -1;
    int64_t s = 0;
    if (level >= 3) s += (int64_t)n3 * (1 + n3) * (2 + n3) / 6;
    if (level >= 2) s += (int64_t)n2 * (n2 + 1) / 2;
    if (level >= 1) s += nm;
    if (level >= 0) s += 1;
    return s;
}

int scp3gpu_pes_energy_dev(int pes, int nw, int64_t n, const double* crd_dev, double* E_dev, int device)
{
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    if (pes != SCP3GPU_PES_QTIP4PF && pes != SCP3GPU_PES_TTM3F) return fail(SCP3GPU_ERR_ARG, "unknown potential");
    if (nw < 1 || nw > kMaxWaters || n < 0 || (n > 0 && (!crd_dev || !E_dev)))
        return fail(SCP3GPU_ERR_ARG, "pes_energy: bad nw, n or pointer");
    int rc = check_device(device);
    if (rc) return rc;
    DeviceGuard g(device);
    if (pes == SCP3GPU_PES_TTM3F && (rc = ttm_init_device())) return rc;
    std::vector<uint32_t> t = pair_tasks(nw);
    uint32_t* td = nullptr;
    if ((rc = upload(&td, t.data(), t.size()))) return rc;
    rc = launch_pes_energy(pes, nw, n, crd_dev, E_dev, nullptr, td, (int)t.size(), 0);
    cudaError_t e = cudaStreamSynchronize(0);
    cudaFree(td);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "pes_energy");
    return SCP3GPU_OK;
}

int scp3gpu_pes_energy(int pes, int nw, int64_t n, const double* crd, double* E, int* iters)
{
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    if (pes != SCP3GPU_PES_QTIP4PF && pes != SCP3GPU_PES_TTM3F) return fail(SCP3GPU_ERR_ARG, "unknown potential");
    if (nw < 1 || nw > kMaxWaters || n < 0 || (n > 0 && (!crd || !E)))
        return fail(SCP3GPU_ERR_ARG, "pes_energy: bad nw, n or pointer");
    if (n == 0) return SCP3GPU_OK;
    int dev = 0;
    cudaGetDevice(&dev);
    int rc = check_device(dev);
    if (rc) return rc;
    if (pes == SCP3GPU_PES_TTM3F && (rc = ttm_init_device())) return rc;
    std::vector<uint32_t> t = pair_tasks(nw);
    uint32_t* td = nullptr;
    double *cd = nullptr, *ed = nullptr;
    int* id = nullptr;
    if ((rc = upload(&td, t.data(), t.size())) || (rc = upload(&cd, crd, (size_t)n * 9 * nw)) ||
        (rc = dalloc(&ed, (size_t)n)) || (rc = dalloc(&id, (size_t)n))) {
        cudaFree(td), cudaFree(cd), cudaFree(ed), cudaFree(id);
        return rc;
    }
    rc = launch_pes_energy(pes, nw, n, cd, ed, id, td, (int)t.size(), 0);
    std::vector<int> it(n);
    if (!rc) {
        cudaError_t e = cudaMemcpy(E, ed, sizeof(double) * n, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(it.data(), id, sizeof(int) * n, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = cuda_fail(e, "pes_energy copy-out");
    }
    cudaFree(td), cudaFree(cd), cudaFree(ed), cudaFree(id);
    if (rc) return rc;
    bool capped = false;
    for (int64_t k = 0; k < n; k++) {
        if (iters) iters[k] = it[k];
        capped |= it[k] > kTtmMaxIter;
    }
    return capped ? fail(SCP3GPU_ERR_NOT_CONVERGED, "TTM3-F dipoles hit the iteration cap") : SCP3GPU_OK;
}

int scp3gpu_pes_energy_grad(int pes, int nw, int64_t n, const double* crd, double* E, double* grad)
{
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    if (pes != SCP3GPU_PES_QTIP4PF && pes != SCP3GPU_PES_TTM3F) return fail(SCP3GPU_ERR_ARG, "unknown potential");
    if (nw < 1 || nw > kMaxWaters || n < 0 || (n > 0 && (!crd || !E || !grad)))
        return fail(SCP3GPU_ERR_ARG, "pes_energy_grad: bad nw, n or pointer");
    if (pes == SCP3GPU_PES_TTM3F && nw > 8) return fail(SCP3GPU_ERR_ARG, "TTM3-F kernel supports nw <= 8");
    if (n == 0) return SCP3GPU_OK;
    int dev = 0;
    cudaGetDevice(&dev);
    int rc = check_device(dev);
    if (rc) return rc;
    if (pes == SCP3GPU_PES_TTM3F && (rc = ttm_init_device())) return rc;
    std::vector<uint32_t> t = pair_tasks(nw);
    uint32_t* td = nullptr;
    double *cd = nullptr, *ed = nullptr, *gd = nullptr;
    int* id = nullptr;
    if ((rc = upload(&td, t.data(), t.size())) || (rc = upload(&cd, crd, (size_t)n * 9 * nw)) ||
        (rc = dalloc(&ed, (size_t)n)) || (rc = dalloc(&gd, (size_t)n * 9 * nw)) || (rc = dalloc(&id, (size_t)n))) {
        cudaFree(td), cudaFree(cd), cudaFree(ed), cudaFree(gd), cudaFree(id);
        return rc;
    }
    rc = launch_pes_energy_grad(pes, nw, n, cd, ed, gd, id, td, (int)t.size(), 0);
    std::vector<int> it(n);
    if (!rc) {
        cudaError_t e = cudaMemcpy(E, ed, sizeof(double) * n, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(grad, gd, sizeof(double) * n * 9 * nw, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(it.data(), id, sizeof(int) * n, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = cuda_fail(e, "pes_energy_grad copy-out");
    }
    cudaFree(td), cudaFree(cd), cudaFree(ed), cudaFree(gd), cudaFree(id);
    if (rc) return rc;
    for (int64_t k = 0; k < n; k++)
        if (it[k] > kTtmMaxIter) return fail(SCP3GPU_ERR_NOT_CONVERGED, "TTM3-F dipoles hit the iteration cap");
    return SCP3GPU_OK;
}

int scp3gpu_sobol_std_normal(int dims, int64_t index0, int64_t n, int scramble, uint64_t seed, double* out)
{
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    if (dims < 1 || dims > 1111 || index0 < 0 || n < 0 || (n > 0 && !out))
        return fail(SCP3GPU_ERR_ARG, "sobol_std_normal: bad dims, index or pointer");
    if (n == 0) return SCP3GPU_OK;
    int dev = 0;
    cudaGetDevice(&dev);
    int rc = check_device(dev);
    if (rc) return rc;
    std::vector<int64_t> v;
    std::vector<uint64_t> sh;
    if ((rc = sobol_tables(dims, scramble, seed, v, sh))) return rc;
    int64_t* vd = nullptr;
    uint64_t* sd = nullptr;
    double* od = nullptr;
    if ((rc = upload(&vd, v.data(), v.size())) || (rc = upload(&sd, sh.data(), sh.size())) ||
        (rc = dalloc(&od, (size_t)n * dims))) {
        cudaFree(vd), cudaFree(sd), cudaFree(od);
        return rc;
    }
    rc = launch_std_normal(dims, index0, n, vd, scramble ? sd : nullptr, od, 0);
    if (!rc) {
        cudaError_t e = cudaMemcpy(out, od, sizeof(double) * n * dims, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = cuda_fail(e, "sobol copy-out");
    }
    cudaFree(vd), cudaFree(sd), cudaFree(od);
    return rc;
}

int scp3gpu_hbuild_destroy(scp3gpu_hbuild* h)
{
    if (!h) return SCP3GPU_OK;
    DeviceGuard g(h->dev);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
    if (h->prep_stream) cudaStreamSynchronize(h->prep_stream);
    void* ptrs[] = {h->sur_ws, h->vq, h->ybuf, h->vdir, h->shift, h->x0, h->MUa, h->omega, h->modes, h->tasks, h->desc, h->q64, h->q32b[0],
                    h->q32b[1], h->vb[0], h->vb[1],
                    h->v, h->normals[0], h->normals[1], h->phi, h->w, h->partial, h->dense, h->hodiag,
                    h->counters};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    tc::destroy(h->tcp);
    stein_destroy(h->sp);
    for (int b = 0; b < 2; b++) {
        if (h->copied[b]) cudaEventDestroy(h->copied[b]);
        if (h->consumed[b]) cudaEventDestroy(h->consumed[b]);
        if (h->prepared[b]) cudaEventDestroy(h->prepared[b]);
        if (h->contracted[b]) cudaEventDestroy(h->contracted[b]);
        if (h->head_done[b]) cudaEventDestroy(h->head_done[b]);
    }
    if (h->prep_stream) cudaStreamDestroy(h->prep_stream);
    if (h->stream) cudaStreamDestroy(h->stream);
    if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
    delete h;
    return SCP3GPU_OK;
}

int scp3gpu_hbuild_create(const scp3gpu_config* c, scp3gpu_hbuild** out)
{
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    if (!c || !out) return fail(SCP3GPU_ERR_ARG, "null config or output");
    *out = nullptr;
    if (c->nw < 1 || c->nw > kMaxWaters) return fail(SCP3GPU_ERR_ARG, "nw must be 1..16");
    if (c->nmodes0 != 9 * c->nw - 6) return fail(SCP3GPU_ERR_ARG, "nmodes0 must be 9*nw-6");
    if (c->nmodes < 1 || c->nmodes > c->nmodes0 || c->nmodes > kMaxModes)
        return fail(SCP3GPU_ERR_ARG, "nmodes out of range");
    // SCP3.cpp:156-160
    if (c->n2 < 0 || c->n3 < 0 || c->n2 > c->nmodes || c->n3 > c->nmodes)
        return fail(SCP3GPU_ERR_ARG, "Number of double or triple excitations exceed number of modes.");
    if (!c->x0 || !c->MUa || !c->omega || !c->modes) return fail(SCP3GPU_ERR_ARG, "null geometry or mode arrays");
    if (c->pes != SCP3GPU_PES_QTIP4PF && c->pes != SCP3GPU_PES_TTM3F) return fail(SCP3GPU_ERR_ARG, "unknown potential");
    if (c->precision != SCP3GPU_PREC_FP64 && c->precision != SCP3GPU_PREC_BF16X3 &&
        c->precision != SCP3GPU_PREC_BF16X3_PES64 && c->precision != SCP3GPU_PREC_F16X3 &&
        c->precision != SCP3GPU_PREC_F16X3_PES64)
        return fail(SCP3GPU_ERR_ARG, "unknown precision");
    if (c->pes == SCP3GPU_PES_TTM3F && c->nw > 8) return fail(SCP3GPU_ERR_ARG, "TTM3-F kernel supports nw <= 8");
    if (c->chunk < 0 || c->chunk % 4096 != 0) return fail(SCP3GPU_ERR_ARG, "chunk must be a multiple of 4096");
    if (c->estimator != SCP3GPU_ESTIMATOR_DIRECT && c->estimator != SCP3GPU_ESTIMATOR_GRADIENT)
        return fail(SCP3GPU_ERR_ARG, "unknown estimator");
    if (c->estimator == SCP3GPU_ESTIMATOR_GRADIENT && c->precision != SCP3GPU_PREC_FP64 &&
        c->precision != SCP3GPU_PREC_BF16X3 && c->precision != SCP3GPU_PREC_BF16X3_PES64)
        return fail(SCP3GPU_ERR_UNSUPPORTED, "gradient estimator: plain FP64 or BF16x3 products only");
    for (int m = 0; m < c->nmodes; m++)
        if (c->modes[m] < 0 || c->modes[m] >= c->nmodes0) return fail(SCP3GPU_ERR_ARG, "mode index out of range");
    int rc = check_device(c->device);
    if (rc) return rc;
    DeviceGuard g(c->device);
    if (c->pes == SCP3GPU_PES_TTM3F && (rc = ttm_init_device())) return rc;

    scp3gpu_hbuild* h = new scp3gpu_hbuild();
    h->cfg = *c;
    h->cfg.x0 = h->cfg.MUa = h->cfg.omega = nullptr;
    h->cfg.modes = nullptr;
    h->dev = c->device;
    // The gradient estimator keeps its own pass structure in every form (stein.cu):
    // its products in FP64 or BF16x3; the potential and its gradient in FP64, or in
    // FP32 for qTIP4P/f with SCP3GPU_PREC_BF16X3.
    const bool gradient = c->estimator == SCP3GPU_ESTIMATOR_GRADIENT;
    h->split_form = c->precision != SCP3GPU_PREC_FP64 && !gradient;
    h->pes_fp32 = (c->precision == SCP3GPU_PREC_BF16X3 || c->precision == SCP3GPU_PREC_F16X3) &&
                  (!gradient || c->pes == SCP3GPU_PES_QTIP4PF);
    const int nm0 = c->nmodes0, N3 = 9 * c->nw;
    h->nb = (int)scp3gpu_basis_size(c->nmodes, c->n2, c->n3);
    // HO diagonal of the selected modes and the inactive-mode zero point (SCP3.cpp:239)
    double sum_all = 0, sum_sel = 0;
    for (int k = 0; k < nm0; k++) sum_all += c->omega[k];
    for (int m = 0; m < c->nmodes; m++) {
        h->omega_sel.push_back(c->omega[c->modes[m]]);
        sum_sel += c->omega[c->modes[m]];
    }
    h->zpe_inactive = 0.5 * (sum_all - sum_sel);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    h->sms = sms;

    auto bail = [&](int code) {
        scp3gpu_hbuild_destroy(h);
        return code;
    };
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->prep_stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(SCP3GPU_ERR_CUDA, "stream creation failed"));
    for (int b = 0; b < 2; b++)
        if (cudaEventCreateWithFlags(&h->copied[b], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->consumed[b], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->prepared[b], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->contracted[b], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->head_done[b], cudaEventDisableTiming) != cudaSuccess)
            return bail(fail(SCP3GPU_ERR_CUDA, "event creation failed"));

    std::vector<int64_t> vd;
    std::vector<uint64_t> sh;
    if ((rc = sobol_tables(nm0, c->scramble, c->scramble_seed, vd, sh))) return bail(rc);
    std::vector<uint32_t> tasks = pair_tasks(c->nw), desc = basis_descriptors(c->nmodes, c->n2, c->n3);
    h->ntasks = (int)tasks.size();
    if ((rc = upload(&h->vdir, vd.data(), vd.size())) ||
        (c->scramble && (rc = upload(&h->shift, sh.data(), sh.size()))) ||
        (rc = upload(&h->x0, c->x0, (size_t)N3)) || (rc = upload(&h->MUa, c->MUa, (size_t)N3 * nm0)) ||
        (rc = upload(&h->omega, c->omega, (size_t)nm0)) || (rc = upload(&h->modes, c->modes, (size_t)c->nmodes)) ||
        (rc = upload(&h->tasks, tasks.data(), tasks.size())) || (rc = upload(&h->desc, desc.data(), desc.size())) ||
        (rc = dalloc(&h->counters, 2)))
        return bail(rc);
    SCP3_CUDA(cudaMemset(h->counters, 0, 2 * sizeof(unsigned long long)));

    if (h->split_form) {
        const bool f16 = c->precision == SCP3GPU_PREC_F16X3 || c->precision == SCP3GPU_PREC_F16X3_PES64;
        if ((rc = tc::create(h->tcp, h->nb, c->nmodes, c->n2, c->n3, c->chunk, sms, f16)))
            return bail(rc);
        h->chunk = h->tcp.chunk;
        h->nb_pad = h->tcp.nb_pad;
        for (int b = 0; b < 2; b++)
            if ((rc = dalloc(&h->q32b[b], (size_t)h->chunk * c->nmodes)) || (rc = dalloc(&h->vb[b], (size_t)h->chunk)))
                return bail(rc);
        h->q32 = h->q32b[0];
        h->v = h->vb[0];
    } else {
        h->gradient = c->estimator == SCP3GPU_ESTIMATOR_GRADIENT;
        if (h->gradient) {
            if ((rc = stein_create(h->sp, desc, c->nmodes, c->chunk, sms, c->precision != SCP3GPU_PREC_FP64)))
                return bail(rc);
            h->chunk = h->sp.chunk;
            h->nsplit = h->sp.nsplit;
            h->nb_pad = h->sp.nb_pad;
            if ((rc = dalloc(&h->q64, (size_t)h->chunk * c->nmodes)) || (rc = dalloc(&h->v, (size_t)h->chunk)) ||
                (rc = dalloc(&h->vq, (size_t)h->chunk * c->nmodes)))
                return bail(rc);
        } else {
            plan_fp64(h, sms);
            if ((rc = dalloc(&h->q64, (size_t)h->chunk * c->nmodes)) || (rc = dalloc(&h->v, (size_t)h->chunk)) ||
                (rc = dalloc(&h->partial, (size_t)h->nsplit * h->tm.ntiles * h->tm.tile * h->tm.tile)) ||
                (rc = dalloc(&h->phi, (size_t)h->nb_pad * h->chunk)) || (rc = dalloc(&h->w, (size_t)h->nb_pad * h->chunk)))
                return bail(rc);
        }
    }
    if ((rc = zero_sums(h))) return bail(rc);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return bail(fail(SCP3GPU_ERR_CUDA, "create sync failed"));
    *out = h;
    return SCP3GPU_OK;
}

int scp3gpu_hbuild_reset(scp3gpu_hbuild* h)
{
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    if (!h) return fail(SCP3GPU_ERR_ARG, "null handle");
    DeviceGuard g(h->dev);
    int rc = drain_prep(h);
    if (!rc) rc = zero_sums(h);
    if (rc) return rc;
    SCP3_CUDA(cudaMemsetAsync(h->counters, 0, 2 * sizeof(unsigned long long), h->stream));
    h->count = 0;
    return SCP3GPU_OK;
}

int64_t scp3gpu_hbuild_basis_size(const scp3gpu_hbuild* h) { return h ? h->nb : -1; }
void* scp3gpu_hbuild_stream(const scp3gpu_hbuild* h) { return h ? (void*)h->stream : nullptr; }
int64_t scp3gpu_hbuild_sample_count(const scp3gpu_hbuild* h) { return h ? h->count : -1; }

int scp3gpu_hbuild_accumulate(scp3gpu_hbuild* h, int64_t index0, int64_t n)
{
    if (!h || index0 < 0 || n < 0) return fail(SCP3GPU_ERR_ARG, "accumulate: bad handle or range");
    if (index0 + n > (1ll << 62)) return fail(SCP3GPU_ERR_ARG, "accumulate: Sobol index beyond 2^62");
    DeviceGuard g(h->dev);
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    for (int64_t off = 0; off < n; off += h->chunk) {
        const int64_t c = std::min(h->chunk, n - off);
        int rc = launch_chunk(h, index0 + off, c, nullptr);
        if (rc) return rc;
        h->count += c;
    }
    return SCP3GPU_OK;
}

int scp3gpu_hbuild_accumulate_normals(scp3gpu_hbuild* h, const double* normals, int64_t n)
{
    return accumulate_host_normals(h, normals, n, "accumulate_normals: bad arguments");
}

int scp3gpu_hbuild_accumulate_normals_f32(scp3gpu_hbuild* h, const float* normals, int64_t n)
{
    return accumulate_host_normals(h, normals, n, "accumulate_normals_f32: bad arguments");
}

int scp3gpu_hbuild_add_epot(scp3gpu_hbuild* h, const double* q, const double* V, int64_t n)
{
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    if (!h || n < 0 || (n > 0 && (!q || !V))) return fail(SCP3GPU_ERR_ARG, "add_epot: bad arguments");
    if (h->gradient) return fail(SCP3GPU_ERR_ARG, "add_epot: a gradient-estimator build takes add_epot_grad");
    DeviceGuard g(h->dev);
    const int nm = h->cfg.nmodes;
    if (int rc0 = drain_prep(h)) return rc0;
    SCP3_CUDA(cudaStreamSynchronize(h->stream));
    for (int64_t off = 0; off < n; off += h->chunk) {
        const int64_t c = std::min(h->chunk, n - off);
        const int64_t kn = h->split_form ? tc::pass_samples(h->tcp, c) : round_up(c, 16ll * h->nsplit);
        SCP3_CUDA(cudaMemsetAsync(h->v, 0, sizeof(double) * kn, h->stream));
        SCP3_CUDA(cudaMemcpyAsync(h->v, V + off, sizeof(double) * c, cudaMemcpyHostToDevice, h->stream));
        int rc;
        if (h->split_form) {
            std::vector<float> qf((size_t)kn * nm, 0.0f);
            for (int64_t i = 0; i < c * nm; i++) qf[i] = (float)q[off * nm + i];
            SCP3_CUDA(cudaMemcpyAsync(h->q32, qf.data(), sizeof(float) * qf.size(), cudaMemcpyHostToDevice, h->stream));
            rc = tc::accumulate_pass(h->tcp, h->desc, h->nb, nm, h->q32, h->v, kn, h->stream, nullptr, nullptr);
            SCP3_CUDA(cudaStreamSynchronize(h->stream));
        } else {
            SCP3_CUDA(cudaMemsetAsync(h->q64, 0, sizeof(double) * kn * nm, h->stream));
            SCP3_CUDA(cudaMemcpyAsync(h->q64, q + off * nm, sizeof(double) * c * nm, cudaMemcpyHostToDevice, h->stream));
            rc = launch_expand_fp64_sm(h->desc, h->nb, nm, h->q64, h->v, kn, h->nb_pad, h->phi, h->w, h->stream);
            if (!rc) rc = launch_contract_fp64_t128(h->phi, h->w, h->nb_pad, kn, h->tm, h->nsplit, h->partial,
                                                    h->stream);
            SCP3_CUDA(cudaStreamSynchronize(h->stream));
        }
        if (rc) return rc;
        h->count += c;
    }
    return SCP3GPU_OK;
}

int scp3gpu_hbuild_add_epot_grad(scp3gpu_hbuild* h, const double* q, const double* V, const double* Vq, int64_t n)
{
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    if (!h || n < 0 || (n > 0 && (!q || !V || !Vq))) return fail(SCP3GPU_ERR_ARG, "add_epot_grad: bad arguments");
    if (!h->gradient) return fail(SCP3GPU_ERR_ARG, "add_epot_grad: the build was created with the direct estimator");
    DeviceGuard g(h->dev);
    const int nm = h->cfg.nmodes;
    SCP3_CUDA(cudaStreamSynchronize(h->stream));
    for (int64_t off = 0; off < n; off += h->chunk) {
        const int64_t c = std::min(h->chunk, n - off);
        const int64_t kn = stein_pass_samples(h->sp, c);
        // padding samples carry V = 0 and dV/dq = 0 and so contribute nothing
        SCP3_CUDA(cudaMemsetAsync(h->v, 0, sizeof(double) * kn, h->stream));
        SCP3_CUDA(cudaMemsetAsync(h->q64, 0, sizeof(double) * kn * nm, h->stream));
        SCP3_CUDA(cudaMemsetAsync(h->vq, 0, sizeof(double) * kn * nm, h->stream));
        SCP3_CUDA(cudaMemcpyAsync(h->v, V + off, sizeof(double) * c, cudaMemcpyHostToDevice, h->stream));
        SCP3_CUDA(cudaMemcpyAsync(h->q64, q + off * nm, sizeof(double) * c * nm, cudaMemcpyHostToDevice, h->stream));
        SCP3_CUDA(cudaMemcpyAsync(h->vq, Vq + off * nm, sizeof(double) * c * nm, cudaMemcpyHostToDevice, h->stream));
        int rc = stein_pass(h->sp, h->desc, h->q64, h->v, h->vq, kn, h->stream);
        SCP3_CUDA(cudaStreamSynchronize(h->stream));
        if (rc) return rc;
        h->count += c;
    }
    return SCP3GPU_OK;
}

static int build_dense(scp3gpu_hbuild* h, int mode)
{
    int rc;
    if (!h->dense && (rc = dalloc(&h->dense, (size_t)h->nb * h->nb))) return rc;
    const double* diag = nullptr;
    double divisor = 1.0, zpe = 0.0;
    if (mode == 1) {
        if (h->count <= 0) return fail(SCP3GPU_ERR_ARG, "read: no samples accumulated");
        if (!h->hodiag) {
            const std::vector<double> d = ho_diagonal(h->omega_sel, h->cfg.n2, h->cfg.n3);
            if ((rc = upload(&h->hodiag, d.data(), d.size()))) return rc;
        }
        diag = h->hodiag;
        divisor = (double)h->count;
        zpe = h->zpe_inactive;
    }
    Timed t(h, 3);
    if (h->split_form) return tc::unpack(h->tcp, h->nb, divisor, diag, zpe, h->dense, h->nb, h->stream);
    if (h->gradient) return stein_unpack(h->sp, h->desc, divisor, diag, zpe, h->dense, h->nb, h->stream);
    return launch_unpack(h->partial, h->tm, h->nsplit, h->nb, divisor, diag, zpe, h->dense, h->nb, h->stream);
}

int scp3gpu_hbuild_read(scp3gpu_hbuild* h, double* M, int64_t ld, int mode)
{
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    if (!h || !M || ld < h->nb || (mode != 0 && mode != 1)) return fail(SCP3GPU_ERR_ARG, "read: bad arguments");
    DeviceGuard g(h->dev);
    int rc = build_dense(h, mode);
    if (rc) return rc;
    SCP3_CUDA(cudaMemcpy2DAsync(M, sizeof(double) * ld, h->dense, sizeof(double) * h->nb, sizeof(double) * h->nb,
                                h->nb, cudaMemcpyDeviceToHost, h->stream));
    SCP3_CUDA(cudaStreamSynchronize(h->stream));
    return SCP3GPU_OK;
}

int scp3gpu_hbuild_read_dev(scp3gpu_hbuild* h, double* M_dev, int64_t ld, int mode)
{
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    if (!h || !M_dev || ld < h->nb || (mode != 0 && mode != 1)) return fail(SCP3GPU_ERR_ARG, "read_dev: bad arguments");
    DeviceGuard g(h->dev);
    int rc = build_dense(h, mode);
    if (rc) return rc;
    SCP3_CUDA(cudaMemcpy2DAsync(M_dev, sizeof(double) * ld, h->dense, sizeof(double) * h->nb, sizeof(double) * h->nb,
                                h->nb, cudaMemcpyDeviceToDevice, h->stream));
    return SCP3GPU_OK;
}

int scp3gpu_hbuild_eigvals(scp3gpu_hbuild* h, int64_t nsub, int k, double* evals)
{
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    if (!h || nsub < 1 || nsub > h->nb || k < 1 || k > nsub || !evals)
        return fail(SCP3GPU_ERR_ARG, "eigvals: bad arguments");
    DeviceGuard g(h->dev);
    int rc = build_dense(h, 1);
    if (rc) return rc;
    const int n = (int)nsub;
    double *A = nullptr, *W = nullptr, *work = nullptr;
    int* info = nullptr;
    if ((rc = dalloc(&A, (size_t)n * n)) || (rc = dalloc(&W, (size_t)n)) || (rc = dalloc(&info, 1))) {
        cudaFree(A), cudaFree(W), cudaFree(info);
        return rc;
    }
    cudaMemcpy2DAsync(A, sizeof(double) * n, h->dense, sizeof(double) * h->nb, sizeof(double) * n, n,
                      cudaMemcpyDeviceToDevice, h->stream);
    cusolverDnHandle_t sol = nullptr;
    int lwork = 0, meig = 0, hinfo = 0;
    rc = SCP3GPU_OK;
    if (cusolverDnCreate(&sol) != CUSOLVER_STATUS_SUCCESS) rc = fail(SCP3GPU_ERR_CUDA, "cusolverDnCreate failed");
    if (!rc) cusolverDnSetStream(sol, h->stream);
    if (!rc && cusolverDnDsyevdx_bufferSize(sol, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_RANGE_I,
                                            CUBLAS_FILL_MODE_UPPER, n, A, n, 0.0, 0.0, 1, k, &meig, W,
                                            &lwork) != CUSOLVER_STATUS_SUCCESS)
        rc = fail(SCP3GPU_ERR_CUDA, "syevdx buffer query failed");
    if (!rc && (rc = dalloc(&work, (size_t)std::max(lwork, 1)))) {}
    if (!rc && cusolverDnDsyevdx(sol, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_RANGE_I, CUBLAS_FILL_MODE_UPPER, n, A,
                                 n, 0.0, 0.0, 1, k, &meig, W, work, lwork, info) != CUSOLVER_STATUS_SUCCESS)
        rc = fail(SCP3GPU_ERR_CUDA, "syevdx failed");
    if (!rc) {
        cudaMemcpyAsync(evals, W, sizeof(double) * k, cudaMemcpyDeviceToHost, h->stream);
        cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
        cudaError_t e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) rc = cuda_fail(e, "eigvals");
        else if (hinfo != 0) rc = fail(SCP3GPU_ERR_CUDA, "syevdx did not converge");
    }
    if (sol) cusolverDnDestroy(sol);
    cudaFree(A), cudaFree(W), cudaFree(work), cudaFree(info);
    return rc;
}

int scp3gpu_hbuild_set_surrogate(scp3gpu_hbuild* h, scp3gpu_mlp* m, int mode)
{
    if (!h) return fail(SCP3GPU_ERR_ARG, "null handle");
    if (mode == SCP3GPU_SURROGATE_NONE) {
        h->sur = nullptr;
        h->sur_mode = mode;
        return SCP3GPU_OK;
    }
    if (mode != SCP3GPU_SURROGATE_REPLACE && mode != SCP3GPU_SURROGATE_RESIDUAL)
        return fail(SCP3GPU_ERR_ARG, "unknown surrogate mode");
    if (!m || !h->split_form) return fail(SCP3GPU_ERR_ARG, "a surrogate needs a split-form build and a network");
    mlp::Net* net = mlp_net(m);
    if (net->n_in != h->cfg.nmodes || net->max_batch < h->chunk || mlp_device(m) != h->dev)
        return fail(SCP3GPU_ERR_ARG, "surrogate: input width must equal nmodes, max_batch >= pass size, same device");
    DeviceGuard g(h->dev);
    if (int rc = drain_prep(h)) return rc;
    if (!h->ybuf && cudaMalloc(&h->ybuf, sizeof(float) * (size_t)h->chunk) != cudaSuccess)
        return fail(SCP3GPU_ERR_NOMEM, "surrogate output buffer");
    // a workspace per build, so builds sharing one network can run at once
    if (h->sur_ws) cudaFree(h->sur_ws);
    h->sur_ws = nullptr;
    if (cudaMalloc(&h->sur_ws, sizeof(__nv_bfloat16) * net->infer_workspace((int)h->chunk)) != cudaSuccess)
        return fail(SCP3GPU_ERR_NOMEM, "surrogate workspace");
    h->sur = m;
    h->sur_mode = mode;
    return SCP3GPU_OK;
}

int scp3gpu_hbuild_sample(scp3gpu_hbuild* h, int64_t index0, int64_t n, float* q, double* v)
{
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    if (!h || index0 < 0 || n < 0 || (n > 0 && (!q || !v))) return fail(SCP3GPU_ERR_ARG, "sample: bad arguments");
    DeviceGuard g(h->dev);
    if (int rc = drain_prep(h)) return rc;
    SCP3_CUDA(cudaStreamSynchronize(h->stream));
    const int nm = h->cfg.nmodes;
    std::vector<double> qd;
    for (int64_t off = 0; off < n; off += h->chunk) {
        const int64_t c = std::min(h->chunk, n - off);
        SampleArgs a{};
        a.nw = h->cfg.nw, a.nm0 = h->cfg.nmodes0, a.nm = nm;
        a.x0 = h->x0, a.MUa = h->MUa, a.omega = h->omega, a.modes = h->modes, a.vdir = h->vdir, a.shift = h->shift;
        a.tasks = h->tasks, a.ntasks = h->ntasks, a.index0 = index0 + off, a.n = c, a.nvalid = c;
        a.q64 = h->split_form ? nullptr : h->q64;
        a.q32 = h->split_form ? h->q32b[0] : nullptr;
        a.v = h->split_form ? h->vb[0] : h->v;
        a.counters = h->counters;
        int rc = launch_samples(h->cfg.pes, h->pes_fp32, a, h->stream);
        if (rc) return rc;
        if (h->split_form) {
            SCP3_CUDA(cudaMemcpyAsync(q + off * nm, a.q32, sizeof(float) * c * nm, cudaMemcpyDeviceToHost, h->stream));
        } else {
            qd.resize((size_t)c * nm);
            SCP3_CUDA(cudaMemcpyAsync(qd.data(), a.q64, sizeof(double) * c * nm, cudaMemcpyDeviceToHost, h->stream));
        }
        SCP3_CUDA(cudaMemcpyAsync(v + off, a.v, sizeof(double) * c, cudaMemcpyDeviceToHost, h->stream));
        SCP3_CUDA(cudaStreamSynchronize(h->stream));
        if (!h->split_form)
            for (size_t i = 0; i < qd.size(); i++) q[off * nm + i] = (float)qd[i];
    }
    return SCP3GPU_OK;
}

int scp3gpu_hbuild_profile(scp3gpu_hbuild* h, int enable, double* ms, int64_t* launches)
{
    if (!h) return fail(SCP3GPU_ERR_ARG, "null handle");
    DeviceGuard g(h->dev);
    double tot[4] = {0, 0, 0, 0};
    int64_t cnt[4] = {0, 0, 0, 0};
    int rc = SCP3GPU_OK;
    if (!enable) {
        if (h->prep_stream) cudaStreamSynchronize(h->prep_stream);
        cudaError_t e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) rc = cuda_fail(e, "profile sync");
        for (size_t k = 0; !rc && k + 1 < h->pev.size(); k += 2) {
            float t = 0;
            cudaEventElapsedTime(&t, h->pev[k], h->pev[k + 1]);
            const int kind = h->pkind[k] & 3;
            tot[kind] += t;
            cnt[kind]++;
        }
    }
    for (cudaEvent_t e : h->pev) cudaEventDestroy(e);
    h->pev.clear();
    h->pkind.clear();
    h->prof = enable != 0;
    if (ms) std::copy(tot, tot + 4, ms);
    if (launches) std::copy(cnt, cnt + 4, launches);
    return rc;
}

int scp3gpu_hbuild_status(scp3gpu_hbuild* h, int64_t* nonfinite, int64_t* not_converged)
{
    if (!h) return fail(SCP3GPU_ERR_ARG, "null handle");
    DeviceGuard g(h->dev);
    unsigned long long c[2] = {0, 0};
    int rc0 = drain_prep(h);
    if (rc0) return rc0;
    SCP3_CUDA(cudaMemcpyAsync(c, h->counters, sizeof(c), cudaMemcpyDeviceToHost, h->stream));
    SCP3_CUDA(cudaStreamSynchronize(h->stream));
    if (nonfinite) *nonfinite = (int64_t)c[0];
    if (not_converged) *not_converged = (int64_t)c[1];
    if (c[0]) return fail(SCP3GPU_ERR_NONFINITE, "samples with non-finite V were accumulated");
    if (c[1]) return fail(SCP3GPU_ERR_NOT_CONVERGED, "TTM3-F samples hit the iteration cap");
    return SCP3GPU_OK;
}

}  // extern "C"
