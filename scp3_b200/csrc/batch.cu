// Batched build: several clusters of uneven size and basis accumulated together.
//
// Every stage of a pass runs as ONE launch over all clusters: the per-sample
// kernel (grid.y = cluster, each cluster with its own geometry, modes and Sobol
// tables), the sign partition (grid.y = cluster), the split-operand expansion
// (grid.z = cluster) into one operand whose rows hold the clusters' bases one
// after another (each padded to 256 rows), and one tensor-core contraction
// over the concatenated list of every cluster's 128 x 256 tiles.  The
// passes of an accumulate call are captured once into a CUDA graph (the
// prepare stream fills pass buffer p&1 while the main stream contracts the
// other) and replayed; per-pass arguments (Sobol offsets) live in device
// memory and are refreshed by one copy before each replay.
//
// The work shape of the contraction: the number of tiles and of sample ranges
// per tile come from the tiling (the fewest waves per unit of work); whether one
// CTA runs per work unit or a persistent grid of one CTA per SM loops over them
// is chosen at creation by timing both on a pass of the batch's own operand.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "internal.h"
#include "tc.h"

using namespace scp3;

namespace {

struct Cluster {
    scp3gpu_config cfg{};              // host copy, pointers cleared
    int nb = 0, nb_pad = 0, nt = 0, row0 = 0;
    int64_t qoff = 0;                  // offset of the cluster's q in a pass buffer (floats)
    int tindex_off = 0;                // offset of its block-owner table
    std::vector<double> omega_sel;
    double zpe_inactive = 0.0;
    // device tables
    int64_t* vdir = nullptr;
    uint64_t* shift = nullptr;
    double *x0 = nullptr, *MUa = nullptr, *omega = nullptr, *hodiag = nullptr;
    int* modes = nullptr;
    uint32_t *tasks = nullptr, *factors = nullptr;
    int ntasks = 0;
};

constexpr int kBuffers = 2;

}  // namespace

struct scp3gpu_batch {
    int dev = 0, ncl = 0, pes = 0, precision = 0, sms = 148;
    bool pes_fp32 = false, f16 = false, use_graph = true;
    std::vector<Cluster> cl;
    int rows = 0, max_nb = 0, max_nm = 0;
    int64_t chunk = 0, slots = 0;     // samples and K slots per pass
    int nflush = 0;
    // contraction work
    int ntiles = 0, nsplit = 1;        // 128 x 256 tiles of all clusters; sample ranges per pass
    int ctas = 0;                      // chosen grid (one per unit, or one per SM looping over units)
    double tuned_ms = 0.0;
    int4* tiles = nullptr;
    int* tile_index = nullptr;         // per cluster, owner of block (ti <= tj): 4 * tile + 2 * transposed + half
    double* partial = nullptr;
    int* err_flag = nullptr;
    // pass buffers
    float* q32[kBuffers] = {};
    double* v[kBuffers] = {};
    int* slot_of[kBuffers] = {};
    int* neg[kBuffers] = {};
    uint16_t* x[kBuffers] = {};        // the operand (32-slot box layout of contract_tc.cu), rows x slots x 2 halves
    tc::ExpandDesc* desc_dev[kBuffers] = {};
    // per-pass sample arguments [pass][cluster]
    SampleArgs* args_dev = nullptr;
    SampleArgs* args_pinned = nullptr;
    std::vector<SampleArgs> args_host;
    int64_t args_cap = 0;              // passes args_dev holds
    cudaEvent_t args_copied = nullptr;
    // streams, events, graph
    cudaStream_t stream = nullptr, prep = nullptr;
    cudaEvent_t prepared[kBuffers] = {}, contracted[kBuffers] = {}, fork = nullptr, join = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t graph_passes = -1, graph_last = -1;
    // read-out and status
    double* dense = nullptr;
    unsigned long long* counters = nullptr;   // [ncl][2]
    int64_t count = 0;
};

namespace {

int64_t round_up(int64_t a, int64_t b) { return (a + b - 1) / b * b; }

void free_graph(scp3gpu_batch* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    b->graph_passes = b->graph_last = -1;
}

int ensure_args(scp3gpu_batch* b, int64_t passes)
{
    if (passes <= b->args_cap) return SCP3GPU_OK;
    free_graph(b);   // the graph points into the old argument array
    if (b->args_dev) cudaFree(b->args_dev);
    if (b->args_pinned) cudaFreeHost(b->args_pinned);
    b->args_dev = nullptr;
    b->args_pinned = nullptr;
    b->args_cap = 0;
    const int64_t cap = std::max<int64_t>(passes, 16);
    SCP3_CUDA(cudaMalloc(&b->args_dev, sizeof(SampleArgs) * (size_t)cap * b->ncl));
    SCP3_CUDA(cudaMallocHost(&b->args_pinned, sizeof(SampleArgs) * (size_t)cap * b->ncl));
    b->args_cap = cap;
    return SCP3GPU_OK;
}

// Sample arguments of pass p, cluster c (host side).
SampleArgs make_args(scp3gpu_batch* b, int c, int buf, int64_t index0, int64_t npad, int64_t nvalid)
{
    const Cluster& k = b->cl[c];
    SampleArgs a{};
    a.nw = k.cfg.nw;
    a.nm0 = k.cfg.nmodes0;
    a.nm = k.cfg.nmodes;
    a.x0 = k.x0;
    a.MUa = k.MUa;
    a.omega = k.omega;
    a.modes = k.modes;
    a.vdir = k.vdir;
    a.shift = k.shift;
    a.tasks = k.tasks;
    a.ntasks = k.ntasks;
    a.normals = nullptr;
    a.index0 = index0;
    a.n = npad;
    a.nvalid = nvalid;
    a.q64 = nullptr;
    a.q32 = b->q32[buf] + k.qoff;
    a.v = b->v[buf] + (size_t)c * b->chunk;
    a.counters = b->counters + 2 * c;
    a.skip_pes = 0;
    return a;
}

// Enqueues passes [0, passes) (the last one `last` samples, padded) on the two
// streams: pass p prepares into buffer p&1 on the prepare stream and contracts
// on the main stream.  Usable both directly and under stream capture: every
// event waited on is recorded earlier in the same sequence.
int enqueue(scp3gpu_batch* b, int64_t passes, int64_t last)
{
    SCP3_CUDA(cudaEventRecord(b->fork, b->stream));
    SCP3_CUDA(cudaStreamWaitEvent(b->prep, b->fork, 0));
    for (int64_t p = 0; p < passes; p++) {
        const int buf = (int)(p & 1);
        const int64_t npad = p + 1 < passes ? b->chunk : round_up(last, tc::kFlush);
        const int nflush = (int)(npad / tc::kFlush);
        const int64_t slots = (int64_t)nflush * tc::kSlotsPerFlush;
        if (p >= kBuffers) SCP3_CUDA(cudaStreamWaitEvent(b->prep, b->contracted[buf], 0));
        int rc = launch_samples_batch(b->pes, b->pes_fp32, &b->args_host[(size_t)p * b->ncl],
                                      b->args_dev + (size_t)p * b->ncl, b->ncl, npad, b->prep);
        if (!rc) rc = tc::launch_partition(b->v[buf], b->chunk, b->slot_of[buf], b->slots, b->neg[buf], b->nflush,
                                           nflush, b->ncl, b->prep);
        if (!rc) rc = tc::launch_expand(b->desc_dev[buf], b->ncl, round_up(b->max_nb, 2 * tc::kTile), b->max_nm, slots,
                                        b->slots / tc::kKBlock2, b->x[buf], b->f16, b->prep);
        if (rc) return rc;
        SCP3_CUDA(cudaEventRecord(b->prepared[buf], b->prep));
        SCP3_CUDA(cudaStreamWaitEvent(b->stream, b->prepared[buf], 0));
        rc = tc::launch_contract(b->x[buf], b->slots / tc::kKBlock2, b->tiles, b->ntiles, b->nsplit,
                                  (int)(slots / tc::kKBlock2), b->neg[buf], b->f16,
                                  b->partial, b->err_flag, b->ctas, b->stream);
        if (rc) return rc;
        SCP3_CUDA(cudaEventRecord(b->contracted[buf], b->stream));
    }
    SCP3_CUDA(cudaEventRecord(b->join, b->prep));
    SCP3_CUDA(cudaStreamWaitEvent(b->stream, b->join, 0));
    return SCP3GPU_OK;
}

// Writes the per-pass arguments of an accumulate call and copies them to the device.
int stage_args(scp3gpu_batch* b, int64_t index0, int64_t n, int64_t passes)
{
    int rc = ensure_args(b, passes);
    if (rc) return rc;
    SCP3_CUDA(cudaEventSynchronize(b->args_copied));   // the previous copy has read the pinned buffer
    b->args_host.resize((size_t)passes * b->ncl);
    for (int64_t p = 0; p < passes; p++) {
        const int64_t nvalid = std::min(b->chunk, n - p * b->chunk);
        const int64_t npad = p + 1 < passes ? b->chunk : round_up(nvalid, tc::kFlush);
        for (int c = 0; c < b->ncl; c++)
            b->args_host[(size_t)p * b->ncl + c] = make_args(b, c, (int)(p & 1), index0 + p * b->chunk, npad, nvalid);
    }
    std::memcpy(b->args_pinned, b->args_host.data(), sizeof(SampleArgs) * b->args_host.size());
    SCP3_CUDA(cudaMemcpyAsync(b->args_dev, b->args_pinned, sizeof(SampleArgs) * b->args_host.size(),
                              cudaMemcpyHostToDevice, b->stream));
    SCP3_CUDA(cudaEventRecord(b->args_copied, b->stream));
    return SCP3GPU_OK;
}

int run_passes(scp3gpu_batch* b, int64_t passes, int64_t last)
{
    if (!b->use_graph) return enqueue(b, passes, last);
    const int64_t last_pad = round_up(last, tc::kFlush);
    if (!b->exec || b->graph_passes != passes || b->graph_last != last_pad) {
        free_graph(b);
        SCP3_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed));
        int rc = enqueue(b, passes, last);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return cuda_fail(e, "batch: graph capture");
        const cudaError_t ei = cudaGraphInstantiate(&b->exec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            b->exec = nullptr;
            return cuda_fail(ei, "batch: graph instantiate");
        }
        b->graph_passes = passes;
        b->graph_last = last_pad;
    }
    SCP3_CUDA(cudaGraphLaunch(b->exec, b->stream));
    return SCP3GPU_OK;
}

int zero_sums(scp3gpu_batch* b)
{
    SCP3_CUDA(cudaMemsetAsync(b->partial, 0, sizeof(double) * (size_t)b->nsplit * b->ntiles * tc::kTile * 2 * tc::kTile,
                              b->stream));
    SCP3_CUDA(cudaMemsetAsync(b->err_flag, 0, sizeof(int), b->stream));
    SCP3_CUDA(cudaMemsetAsync(b->counters, 0, sizeof(unsigned long long) * 2 * b->ncl, b->stream));
    return SCP3GPU_OK;
}

// Times both grid forms of the contraction (one CTA per work unit; one CTA per
// SM looping over the units) on one prepared pass (buffer 0) and keeps the
// faster.  The trial sums are discarded afterwards.
int autotune(scp3gpu_batch* b)
{
    int rc = stage_args(b, 1ll << 30, b->chunk, 1);   // trial points from the reference's default skip
    if (rc) return rc;
    const int units = b->ntiles * b->nsplit;
    // one direct pass prepares buffer 0 (and sets the kernels' attributes before any capture)
    b->ctas = std::min(units, b->sms);
    if ((rc = enqueue(b, 1, b->chunk))) return rc;
    cudaEvent_t e0, e1;
    SCP3_CUDA(cudaEventCreate(&e0));
    SCP3_CUDA(cudaEventCreate(&e1));
    double best = 1e30;
    int best_ctas = b->ctas;
    const int cand[2] = {std::min(units, b->sms), units};
    for (int ci = 0; ci < 2 && rc == 0; ci++) {
        float ms_best = 1e30f;
        for (int rep = 0; rep < 3 && rc == 0; rep++) {
            cudaEventRecord(e0, b->stream);
            rc = tc::launch_contract(b->x[0], b->slots / tc::kKBlock2, b->tiles, b->ntiles, b->nsplit,
                                      (int)(b->slots / tc::kKBlock2), b->neg[0], b->f16,
                                      b->partial, b->err_flag, cand[ci], b->stream);
            cudaEventRecord(e1, b->stream);
            if (cudaEventSynchronize(e1) != cudaSuccess) rc = fail(SCP3GPU_ERR_CUDA, "batch: autotune sync");
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) ms_best = std::min(ms_best, ms);   // first run warms the caches
        }
        if (rc == 0 && ms_best < best) {
            best = ms_best;
            best_ctas = cand[ci];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    b->ctas = best_ctas;
    b->tuned_ms = best;
    int err = 0;
    SCP3_CUDA(cudaMemcpy(&err, b->err_flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return fail(SCP3GPU_ERR_TIMEOUT, "batch autotune: a bounded pipeline wait expired");
    return zero_sums(b);
}

int check_config(const scp3gpu_config* c)
{
    if (c->nw < 1 || c->nw > kMaxWaters) return fail(SCP3GPU_ERR_ARG, "nw must be 1..16");
    if (c->nmodes0 != 9 * c->nw - 6) return fail(SCP3GPU_ERR_ARG, "nmodes0 must be 9*nw-6");
    if (c->nmodes < 1 || c->nmodes > c->nmodes0 || c->nmodes > kMaxModes)
        return fail(SCP3GPU_ERR_ARG, "nmodes out of range");
    if (c->n2 < 0 || c->n3 < 0 || c->n2 > c->nmodes || c->n3 > c->nmodes)
        return fail(SCP3GPU_ERR_ARG, "Number of double or triple excitations exceed number of modes.");
    if (!c->x0 || !c->MUa || !c->omega || !c->modes) return fail(SCP3GPU_ERR_ARG, "null geometry or mode arrays");
    if (c->pes == SCP3GPU_PES_TTM3F && c->nw > 8) return fail(SCP3GPU_ERR_ARG, "TTM3-F kernel supports nw <= 8");
    for (int m = 0; m < c->nmodes; m++)
        if (c->modes[m] < 0 || c->modes[m] >= c->nmodes0) return fail(SCP3GPU_ERR_ARG, "mode index out of range");
    return SCP3GPU_OK;
}

int upload_cluster(Cluster& k, const scp3gpu_config* c)
{
    std::vector<int64_t> vd;
    std::vector<uint64_t> sh;
    int rc = sobol_tables(c->nmodes0, c->scramble, c->scramble_seed, vd, sh);
    if (rc) return rc;
    const std::vector<uint32_t> tasks = pair_tasks(c->nw);
    const std::vector<uint32_t> fac = basis_factor_table(c->nmodes, c->n2, c->n3);
    const std::vector<double> hod = ho_diagonal(k.omega_sel, c->n2, c->n3);
    k.ntasks = (int)tasks.size();
    const int N3 = 9 * c->nw;
    if ((rc = upload(&k.vdir, vd.data(), vd.size())) || (c->scramble && (rc = upload(&k.shift, sh.data(), sh.size()))) ||
        (rc = upload(&k.x0, c->x0, (size_t)N3)) || (rc = upload(&k.MUa, c->MUa, (size_t)N3 * c->nmodes0)) ||
        (rc = upload(&k.omega, c->omega, (size_t)c->nmodes0)) || (rc = upload(&k.modes, c->modes, (size_t)c->nmodes)) ||
        (rc = upload(&k.tasks, tasks.data(), tasks.size())) || (rc = upload(&k.factors, fac.data(), fac.size())) ||
        (rc = upload(&k.hodiag, hod.data(), hod.size())))
        return rc;
    return SCP3GPU_OK;
}

}  // namespace

extern "C" {

int scp3gpu_batch_destroy(scp3gpu_batch* b)
{
    if (!b) return SCP3GPU_OK;
    DeviceGuard g(b->dev);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->prep) cudaStreamSynchronize(b->prep);
    free_graph(b);
    for (Cluster& k : b->cl) {
        void* ptrs[] = {k.vdir, k.shift, k.x0, k.MUa, k.omega, k.hodiag, k.modes, k.tasks, k.factors};
        for (void* p : ptrs)
            if (p) cudaFree(p);
    }
    for (int i = 0; i < kBuffers; i++) {
        void* ptrs[] = {b->q32[i], b->v[i], b->slot_of[i], b->neg[i], b->x[i], b->desc_dev[i]};
        for (void* p : ptrs)
            if (p) cudaFree(p);
        if (b->prepared[i]) cudaEventDestroy(b->prepared[i]);
        if (b->contracted[i]) cudaEventDestroy(b->contracted[i]);
    }
    void* ptrs[] = {b->tiles, b->tile_index, b->partial, b->err_flag, b->args_dev, b->dense, b->counters};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (b->args_pinned) cudaFreeHost(b->args_pinned);
    cudaEvent_t evs[] = {b->args_copied, b->fork, b->join};
    for (cudaEvent_t e : evs)
        if (e) cudaEventDestroy(e);
    if (b->prep) cudaStreamDestroy(b->prep);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return SCP3GPU_OK;
}

int scp3gpu_batch_create(const scp3gpu_config* cfgs, int ncl, int64_t chunk, int flags, scp3gpu_batch** out)
{
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    if (!cfgs || !out || ncl < 1 || ncl > 65535) return fail(SCP3GPU_ERR_ARG, "batch: null configs/output or bad count");
    *out = nullptr;
    if (chunk < 0 || chunk % tc::kFlush != 0) return fail(SCP3GPU_ERR_ARG, "batch: chunk must be a multiple of 4096");
    const scp3gpu_config& c0 = cfgs[0];
    if (c0.precision == SCP3GPU_PREC_FP64)
        return fail(SCP3GPU_ERR_UNSUPPORTED, "batch: the batched build runs the split (tensor-core) precisions");
    if (c0.precision != SCP3GPU_PREC_BF16X3 && c0.precision != SCP3GPU_PREC_BF16X3_PES64 &&
        c0.precision != SCP3GPU_PREC_F16X3 && c0.precision != SCP3GPU_PREC_F16X3_PES64)
        return fail(SCP3GPU_ERR_ARG, "unknown precision");
    if (c0.pes != SCP3GPU_PES_QTIP4PF && c0.pes != SCP3GPU_PES_TTM3F) return fail(SCP3GPU_ERR_ARG, "unknown potential");
    int rc;
    for (int c = 0; c < ncl; c++) {
        if ((rc = check_config(&cfgs[c]))) return rc;
        if (cfgs[c].pes != c0.pes || cfgs[c].precision != c0.precision || cfgs[c].device != c0.device)
            return fail(SCP3GPU_ERR_ARG, "batch: all clusters share one potential, precision and device");
    }
    if ((rc = check_device(c0.device))) return rc;
    DeviceGuard g(c0.device);
    if (c0.pes == SCP3GPU_PES_TTM3F && (rc = ttm_init_device())) return rc;

    scp3gpu_batch* b = new scp3gpu_batch();
    auto bail = [&](int code) {
        scp3gpu_batch_destroy(b);
        return code;
    };
    b->dev = c0.device;
    b->ncl = ncl;
    b->pes = c0.pes;
    b->precision = c0.precision;
    b->pes_fp32 = c0.precision == SCP3GPU_PREC_BF16X3 || c0.precision == SCP3GPU_PREC_F16X3;
    b->f16 = c0.precision == SCP3GPU_PREC_F16X3 || c0.precision == SCP3GPU_PREC_F16X3_PES64;
    b->use_graph = !(flags & SCP3GPU_BATCH_NO_GRAPH);
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->dev);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->prep, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(SCP3GPU_ERR_CUDA, "stream creation failed"));
    cudaEvent_t* evs[] = {&b->prepared[0], &b->prepared[1], &b->contracted[0], &b->contracted[1],
                          &b->fork, &b->join, &b->args_copied};
    for (cudaEvent_t* e : evs)
        if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess)
            return bail(fail(SCP3GPU_ERR_CUDA, "event creation failed"));

    // clusters: basis sizes, operand rows, tables
    int64_t sum_nm = 0;
    b->cl.resize(ncl);
    for (int c = 0; c < ncl; c++) {
        Cluster& k = b->cl[c];
        const scp3gpu_config& cf = cfgs[c];
        k.cfg = cf;
        k.cfg.x0 = k.cfg.MUa = k.cfg.omega = nullptr;
        k.cfg.modes = nullptr;
        k.nb = (int)scp3gpu_basis_size(cf.nmodes, cf.n2, cf.n3);
        k.nb_pad = (int)round_up(k.nb, 2 * tc::kTile);    // whole 256-row panel pairs
        k.nt = k.nb_pad / tc::kTile;
        k.row0 = b->rows;
        b->rows += k.nb_pad;
        b->max_nb = std::max(b->max_nb, k.nb);
        b->max_nm = std::max(b->max_nm, cf.nmodes);
        k.qoff = 0;   // set below, once the chunk is known
        sum_nm += cf.nmodes;
        double sum_all = 0, sum_sel = 0;   // SCP3.cpp:239
        for (int m = 0; m < cf.nmodes0; m++) sum_all += cf.omega[m];
        for (int m = 0; m < cf.nmodes; m++) {
            k.omega_sel.push_back(cf.omega[cf.modes[m]]);
            sum_sel += cf.omega[cf.modes[m]];
        }
        k.zpe_inactive = 0.5 * (sum_all - sum_sel);
        if ((rc = upload_cluster(k, &cf))) return bail(rc);
    }
    // samples per pass: up to 2^17 (long work units amortise each unit's pipeline
    // fill and FP64 write-back), with each pass buffer's split operand under ~8 GB
    int64_t ch = chunk > 0 ? chunk : (int64_t)tc::kFlush * 32;
    while (ch > tc::kFlush && (int64_t)b->rows * (ch / tc::kFlush) * tc::kSlotsPerFlush * 4 > (8ll << 30)) ch /= 2;
    b->chunk = ch / tc::kFlush * tc::kFlush;
    b->nflush = (int)(b->chunk / tc::kFlush);
    b->slots = (int64_t)b->nflush * tc::kSlotsPerFlush;
    {
        int64_t off = 0;
        for (Cluster& k : b->cl) {
            k.qoff = off;
            off += b->chunk * k.cfg.nmodes;
        }
    }
    // 128 x 256 tiles of every cluster, cluster by cluster
    std::vector<tc::BaseTile> base;
    std::vector<int> cnt;
    for (int c = 0; c < ncl; c++) {
        const Cluster& k = b->cl[c];
        tc::add_cluster_tiles(base, c, k.nt, (k.nb + tc::kTile - 1) / tc::kTile, k.row0, c * b->nflush);
        cnt.push_back(k.nt);
    }
    std::vector<int4> tiles;
    std::vector<std::vector<int>> owners;
    tc::finish_tiling(base, cnt, b->sms, tiles, owners, b->nsplit);
    b->ntiles = (int)tiles.size();
    std::vector<int> tindex;
    for (int c = 0; c < ncl; c++) {
        b->cl[c].tindex_off = (int)tindex.size();
        tindex.insert(tindex.end(), owners[c].begin(), owners[c].end());
    }
    b->ctas = std::min(b->ntiles * b->nsplit, b->sms);
    if ((rc = upload(&b->tiles, tiles.data(), tiles.size())) || (rc = upload(&b->tile_index, tindex.data(), tindex.size())) ||
        (rc = dalloc(&b->partial, (size_t)b->nsplit * b->ntiles * tc::kTile * 2 * tc::kTile)) ||
        (rc = dalloc(&b->err_flag, 1)) || (rc = dalloc(&b->counters, (size_t)2 * ncl)))
        return bail(rc);
    for (int i = 0; i < kBuffers; i++) {
        if ((rc = dalloc(&b->q32[i], (size_t)b->chunk * sum_nm)) || (rc = dalloc(&b->v[i], (size_t)b->chunk * ncl)) ||
            (rc = dalloc(&b->slot_of[i], (size_t)b->slots * ncl)) || (rc = dalloc(&b->neg[i], (size_t)b->nflush * ncl)) ||
            (rc = dalloc(&b->x[i], (size_t)2 * b->rows * b->slots)))
            return bail(rc);
        // each cluster's padding rows are never written by the expansion: zero once
        if (cudaMemset(b->x[i], 0, sizeof(uint16_t) * 2 * (size_t)b->rows * b->slots) != cudaSuccess)
            return bail(fail(SCP3GPU_ERR_CUDA, "batch: operand zeroing failed"));
        std::vector<tc::ExpandDesc> d(ncl);
        for (int c = 0; c < ncl; c++) {
            const Cluster& k = b->cl[c];
            d[c] = tc::ExpandDesc{k.factors, k.nb, k.nb_pad, k.cfg.nmodes, k.row0, b->q32[i] + k.qoff,
                                  b->v[i] + (size_t)c * b->chunk, b->slot_of[i] + (size_t)c * b->slots};
        }
        if ((rc = upload(&b->desc_dev[i], d.data(), d.size()))) return bail(rc);
    }
    SCP3_CUDA(cudaEventRecord(b->args_copied, b->stream));
    if ((rc = zero_sums(b))) return bail(rc);
    if (!(flags & SCP3GPU_BATCH_NO_AUTOTUNE)) {
        if ((rc = autotune(b))) return bail(rc);
    } else {
        // set the kernels' attributes outside any capture with one direct pass, then clear its sums
        if ((rc = stage_args(b, 1ll << 30, b->chunk, 1)) || (rc = enqueue(b, 1, b->chunk)) || (rc = zero_sums(b)))
            return bail(rc);
    }
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return bail(fail(SCP3GPU_ERR_CUDA, "batch create sync failed"));
    *out = b;
    return SCP3GPU_OK;
}

int scp3gpu_batch_reset(scp3gpu_batch* b)
{
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    if (!b) return fail(SCP3GPU_ERR_ARG, "null handle");
    DeviceGuard g(b->dev);
    int rc = zero_sums(b);
    if (rc) return rc;
    b->count = 0;
    return SCP3GPU_OK;
}

int scp3gpu_batch_size(const scp3gpu_batch* b) { return b ? b->ncl : -1; }
int64_t scp3gpu_batch_basis_size(const scp3gpu_batch* b, int c)
{
    return (b && c >= 0 && c < b->ncl) ? b->cl[c].nb : -1;
}
int64_t scp3gpu_batch_sample_count(const scp3gpu_batch* b) { return b ? b->count : -1; }
void* scp3gpu_batch_stream(const scp3gpu_batch* b) { return b ? (void*)b->stream : nullptr; }

int scp3gpu_batch_shape(const scp3gpu_batch* b, int* nsplit, int* ctas, int64_t* chunk, double* ms)
{
    if (!b) return fail(SCP3GPU_ERR_ARG, "null handle");
    if (nsplit) *nsplit = b->nsplit;
    if (ctas) *ctas = b->ctas;
    if (chunk) *chunk = b->chunk;
    if (ms) *ms = b->tuned_ms;
    return SCP3GPU_OK;
}

int scp3gpu_batch_accumulate(scp3gpu_batch* b, int64_t index0, int64_t n)
{
    if (!b || index0 < 0 || n < 0) return fail(SCP3GPU_ERR_ARG, "batch accumulate: bad handle or range");
    if (index0 + n > (1ll << 62)) return fail(SCP3GPU_ERR_ARG, "batch accumulate: Sobol index beyond 2^62");
    if (n == 0) return SCP3GPU_OK;
    DeviceGuard g(b->dev);
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    const int64_t passes = (n + b->chunk - 1) / b->chunk;
    const int64_t last = n - (passes - 1) * b->chunk;
    int rc = stage_args(b, index0, n, passes);
    if (!rc) rc = run_passes(b, passes, last);
    if (rc) return rc;
    b->count += n;
    return SCP3GPU_OK;
}

int scp3gpu_batch_read(scp3gpu_batch* b, int c, double* M, int64_t ld, int mode)
{
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    if (!b || c < 0 || c >= b->ncl || !M || (mode != 0 && mode != 1) || ld < b->cl[c].nb)
        return fail(SCP3GPU_ERR_ARG, "batch read: bad arguments");
    const Cluster& k = b->cl[c];
    if (mode == 1 && b->count <= 0) return fail(SCP3GPU_ERR_ARG, "read: no samples accumulated");
    DeviceGuard g(b->dev);
    int rc;
    if (!b->dense && (rc = dalloc(&b->dense, (size_t)b->max_nb * b->max_nb))) return rc;
    int err = 0;
    SCP3_CUDA(cudaMemcpyAsync(&err, b->err_flag, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    SCP3_CUDA(cudaStreamSynchronize(b->stream));
    if (err) return fail(SCP3GPU_ERR_TIMEOUT, "tensor-core contraction: a bounded pipeline wait expired");
    rc = tc::launch_unpack(b->partial, b->tile_index + k.tindex_off, k.nt, b->ntiles, b->nsplit, k.nb,
                            mode == 1 ? (double)b->count : 1.0, mode == 1 ? k.hodiag : nullptr,
                            mode == 1 ? k.zpe_inactive : 0.0, b->dense, k.nb, b->stream);
    if (rc) return rc;
    SCP3_CUDA(cudaMemcpy2DAsync(M, sizeof(double) * ld, b->dense, sizeof(double) * k.nb, sizeof(double) * k.nb, k.nb,
                                cudaMemcpyDeviceToHost, b->stream));
    SCP3_CUDA(cudaStreamSynchronize(b->stream));
    return SCP3GPU_OK;
}

int scp3gpu_batch_status(scp3gpu_batch* b, int c, int64_t* nonfinite, int64_t* not_converged)
{
    (void)cudaGetLastError();   // a pending error of an earlier, unrelated call is not this call's
    if (!b || c < 0 || c >= b->ncl) return fail(SCP3GPU_ERR_ARG, "batch status: bad arguments");
    DeviceGuard g(b->dev);
    unsigned long long h[2] = {0, 0};
    SCP3_CUDA(cudaMemcpyAsync(h, b->counters + 2 * c, sizeof(h), cudaMemcpyDeviceToHost, b->stream));
    SCP3_CUDA(cudaStreamSynchronize(b->stream));
    if (nonfinite) *nonfinite = (int64_t)h[0];
    if (not_converged) *not_converged = (int64_t)h[1];
    if (h[0]) return fail(SCP3GPU_ERR_NONFINITE, "non-finite potential values were sampled");
    if (h[1]) return fail(SCP3GPU_ERR_NOT_CONVERGED, "TTM3-F dipole iterations hit the cap");
    return SCP3GPU_OK;
}

}  // extern "C"
