"""Benchmark of the B200 Hamiltonian build (one JSON line on rank 0).

Workload (one step): the hexamer-prism doubles build -- six waters relaxed on
qTIP4P/f, 48 modes, N2 = 48 (1225 basis functions), 2^20 scrambled Sobol points
per step and per GPU (weak scaling), each point through BSM, the back-transform,
the potential and the accumulation of <i|V|j>.  Inputs are synthetic: the
geometry is built and relaxed by scp3_b200.inputs, the Sobol points are
generated on the device.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision bf16x3|fp64]
  python bench.py --impl reference ...   # the reference's CPU build, timed on this host

value   samples/s over all ranks, device-timed (CUDA events on the build's stream,
        max over ranks), L2 flushed between steps (256 MB write)
e2e     samples/s through the C ABI with host buffers: the -r path (SCP3.cpp:188-194)
        with 2^20 x 48 FP64 normals copied in from pinned memory and Mout read back
"""
import argparse
import json
import os
import subprocess
import sys
import time

# Thread pools of the reference's CPU build (cpu_baseline and --impl reference):
# OpenBLAS and OpenMP threads sleep when idle instead of spinning against each
# other's phase of the block loop.  Set before numpy and torch load their BLAS
# and OpenMP runtimes, which read these once; the reference's build shares the
# OpenMP runtime torch loads.
REF_THREAD_ENV = {"OPENBLAS_THREAD_TIMEOUT": "4", "OMP_WAIT_POLICY": "PASSIVE"}
for _k, _v in REF_THREAD_ENV.items():
    os.environ.setdefault(_k, _v)

import numpy as np  # noqa: E402

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SAMPLES = 1 << 20
TRIPLES_SAMPLES = 1 << 18       # the default line's triples sub-record: two 2^17 chunks, a dump after each
INPUT = "prism_qtip4pf"
SCRAMBLE_SEED = 0x5C3
WORKLOAD = "hexamer prism qTIP4P/f, 48 modes, doubles basis Nb=1225, 2^20 scrambled Sobol points per GPU per step"
METRIC = "Sobol samples/s (hexamer H-build) at <=0.1 cm^-1 on 10 lowest levels vs FP64"
FP64_NOMINAL_TFLOPS = 37.0   # B200 FP64 (vector and tensor) nominal; no measured FP64 peak on this pool
# DRAM bytes (read + write) of the BF16x3 contraction on the hexamer doubles basis, from an ncu
# capture of one 2^18-sample pass (one launch of 140 CTAs: dram__bytes_read.sum +
# dram__bytes_write.sum = 1522.6 + 11.8 MB); per launch it grows with the samples the launch covers
CONTRACT_DRAM_BYTES_PER_SAMPLE = (1522.616320e6 + 11.786240e6) / 262144


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "of measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "of fallback"


class Clocks:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""

    def __init__(self, gpu):
        # the raw samples stay beside the summary (BENCH_CLOCKS_DIR, default bench_out/)
        out = os.environ.get("BENCH_CLOCKS_DIR", os.path.join(ROOT, "bench_out"))
        self.path = os.path.join(out, "clocks_%d.csv" % os.getpid())
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons)}


def launch_ranks(n, argv, limit_s=1800):
    """`--gpus N` started without a launcher: run N local ranks of this script
    under torch.distributed.run (one per GPU, rendezvous on 127.0.0.1) and
    return their exit code.  `timeout -k 60` bounds the whole job well above the
    process group's own timeout, so ranks that wait for one another end."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = ["timeout", "-k", "60", str(limit_s), sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node", str(n), "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.abspath(__file__)] + list(argv)
    return subprocess.call(cmd)


def dist_setup(n_gpus, backend="nccl"):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != n_gpus:
        raise SystemExit("bench.py: --gpus %d but the launcher started %d ranks" % (n_gpus, world))
    if world > 1:
        import datetime
        import torch.distributed as dist
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def exchange(hb, Mdev, stream):
    """The ranks' one exchange (sample-range sharding): the rank's matrix is
    written into Mdev on the build's stream, the current stream waits for that
    write, then Mdev is summed over the ranks in place.  `stream` is None for
    the host stand-in, whose read is synchronous."""
    from scp3_b200 import shard
    hb.read_dev(Mdev.data_ptr(), Mdev.shape[0], 0)
    if stream is not None:
        import torch
        ev = torch.cuda.Event()
        ev.record(stream)
        torch.cuda.current_stream().wait_event(ev)
    shard.reduce_matrix(Mdev)


class HostStandIn:
    """`--standin`: a small numpy build on the host that takes the calls the
    benchmark step makes of a build (accumulate, read_dev, reset, status,
    close), so the CPU tests can run the rank launcher, the sample-range split
    and the exchange without a GPU.  Sample s contributes phi(s) v(s) phi(s)^T
    with phi and v fixed functions of the Sobol index, so any split of the
    indices over ranks sums to the same matrix.  Not a Hamiltonian build."""

    def __init__(self, nb=6):
        self.nb = nb
        self.M = np.zeros((nb, nb))
        self.n = 0

    @staticmethod
    def terms(index0, n, nb):
        s = (index0 + np.arange(n, dtype=np.float64))[None, :]
        k = np.arange(1, nb + 1, dtype=np.float64)[:, None]
        return np.cos(1e-3 * k * s + 0.1 * k), np.sin(7e-4 * s[0]) - 0.25

    def accumulate(self, index0, n):
        phi, v = self.terms(index0, n, self.nb)
        self.M += (phi * v) @ phi.T
        self.n += n

    def read_dev(self, ptr, ld, mode=0):
        import ctypes
        out = np.ctypeslib.as_array((ctypes.c_double * (ld * self.nb)).from_address(ptr)).reshape(self.nb, ld)
        out[:, :self.nb] = self.M      # symmetric: row- and column-major agree

    def reset(self):
        self.M[:] = 0.0
        self.n = 0

    def status(self):
        return 0, 0, 0

    def close(self):
        pass


def cpu_reference(nw, x0, MUa, omega, modes, n2, n3, normals, target_s=12.0, max_samples=None):
    """The reference's own build (oracle/_ref, release flags) on this host: samples/s."""
    import oracle
    fast = oracle.ref_available(fast=True)
    if not (fast or oracle.ref_available()):
        return None
    block = 1024
    n = block * 4
    M, t, _ = oracle.ref_hbuild(0, nw, x0, MUa, omega, modes, n2, n3, n, block, normals=normals[:n], fast=fast)
    per = max(t.sum(), 1e-6) / n
    n = int(min(max(block * 4, target_s / per), normals.shape[0] if max_samples is None else max_samples))
    n -= n % block
    M.fill(0.0)          # the timed run's matrix holds its own n samples only
    t0 = time.perf_counter()
    M, t, _ = oracle.ref_hbuild(0, nw, x0, MUa, omega, modes, n2, n3, n, block, normals=normals[:n], fast=fast, M=M)
    wall = time.perf_counter() - t0
    return {"value": n / wall, "unit": "samples/s", "cores": os.cpu_count(), "kind": "reference" if fast else "port",
            "sample": "%d of the %d samples (blocks of %d, -r normals path: PES + get_bra + dsyr2k, OpenMP/OpenBLAS on "
                      "all host threads); Sobol skip walk excluded" % (n, SAMPLES, block),
            "split_s": {"pes": float(t[0]), "bra": float(t[1]), "dsyr2k": float(t[2])},
            "threads": oracle.ref_thread_env(), "_M": M, "_n": n}


def levels_vs_reference(ref, nw, x0, MUa, omega, normals, precision, device):
    """The 10 lowest levels of Mout = M/n + HO diagonal from the reference's own
    build (cpu_reference's matrix, dsyr2k 'U') against the GPU build of the same
    normals through the -r path, in the benchmark's precision: the level gate
    of the metric pinned to the reference itself."""
    import oracle
    import scp3_b200
    M, n = ref.pop("_M"), ref.pop("_n")
    Mref = np.asfortranarray(np.triu(M) + np.triu(M, 1).T) / n
    oracle.add_ho_diagonal(Mref, omega, 48, 0, 0.0)
    e_ref = np.linalg.eigvalsh(Mref)[:10]
    hb = scp3_b200.HBuild(nw, x0, MUa, omega, n2=48, n3=0, pes="qtip4pf", precision=precision,
                          scramble_seed=SCRAMBLE_SEED, device=device)
    hb.accumulate_normals(np.ascontiguousarray(normals[:n]))
    e_gpu = np.linalg.eigvalsh(hb.read(1))[:10]
    hb.close()
    autocm = scp3_b200.constants.autocm
    return {"samples": int(n), "precision": precision,
            "max_abs_err_cm1": float(np.abs(e_gpu - e_ref).max() * autocm),
            "lowest10_cm1_reference": [float(x * autocm) for x in e_ref],
            "note": "the reference's build (oracle/_ref) and the GPU build on the same normals; levels of a "
                    "2^17-point build are dominated by Monte Carlo noise, so this compares arithmetic, not physics"}


def run_standin(args, world, rank):
    """The benchmark's rank logic with HostStandIn as the build (CPU tests):
    the same sample ranges, warm-up, reset, barrier, exchange and max-over-ranks
    timing as the GPU step, host-clocked.  --dump-matrix writes rank 0's
    reduced matrix after the timed steps."""
    import torch
    import torch.distributed as dist
    from scp3_b200 import shard
    hb = HostStandIn()
    Mdev = torch.zeros((hb.nb, hb.nb), dtype=torch.float64)
    base, _ = shard.sample_range(rank, world, 0, SAMPLES, "weak")

    def step(k):
        hb.accumulate(base + k * SAMPLES, SAMPLES)
        if world > 1:
            exchange(hb, Mdev, None)

    for k in range(args.warmup):
        step(k)
    hb.reset()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        step(args.warmup + k)
    total_ms = 1e3 * (time.perf_counter() - t0)
    if world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    else:
        exchange(hb, Mdev, None)
    if rank == 0:
        if args.dump_matrix:
            np.save(args.dump_matrix, Mdev.numpy())
        print(json.dumps({"metric": "stand-in build rank exchange (host)", "value": world * SAMPLES * args.steps /
                          (total_ms / 1e3), "unit": "samples/s", "n_gpus": world, "steps": args.steps,
                          "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "data": "stand-in",
                          "config": {"workload": "HostStandIn nb=%d, %d samples per rank per step" % (hb.nb, SAMPLES),
                                     "parallelism": "dp%d (sample ranges)" % world, "base": base}}))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def bench_config(precision, nb, world):
    """The `config` of the benchmark line, the same in both arms."""
    return {"workload": WORKLOAD, "precision": precision, "nb": nb, "samples_per_step": SAMPLES,
            "l2": "flushed between steps (256 MB write)", "parallelism": "dp%d (sample ranges)" % world}


def run_reference(args, rank):
    if rank != 0:
        return
    from scp3_b200 import inputs, std_normals
    nw, x0, MUa, omega = inputs.load(INPUT)
    modes = np.arange(omega.size, dtype=np.int32)
    import oracle
    if not (oracle.ref_available(fast=True) or oracle.ref_available()):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference built from its sources) "
                                                              "is not present on this host"}))
        return
    per_step = 1 << 14
    normals = oracle.std_normals(omega.size, 0, per_step, scramble_seed=SCRAMBLE_SEED)
    fast = oracle.ref_available(fast=True)
    times = []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.ref_hbuild(0, nw, x0, MUa, omega, modes, 48, 0, per_step, 1024, normals=normals, fast=fast)
        if k >= args.warmup:
            times.append(time.perf_counter() - t0)
    v = per_step * len(times) / sum(times)
    nb = oracle.basis_size(omega.size, 48, 0)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "samples/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(args.precision, nb, args.gpus),
            "reference_step": "a bounded 2^14-sample slice of the workload per step (samples/s is a rate)",
            "cpu_baseline": {"value": v, "unit": "samples/s", "cores": os.cpu_count(),
                             "kind": "reference" if fast else "port",
                             "sample": "2^14 samples per step of the same workload, -r normals path",
                             "threads": oracle.ref_thread_env()},
            "e2e": {"value": v, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def timed_accumulate(hb, index0, n):
    """Device time (ms) of one accumulate call: CUDA events on the build's stream,
    which every pass of the call joins before it returns."""
    import torch
    st = torch.cuda.ExternalStream(hb.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    hb.accumulate(index0, n)
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1)


def triples_record(total, precision, dump=True, deflate=6):
    """The triples configuration: TTM3-F hexamer prism, N2 = N3 = 48 (20825 basis
    functions), `total` scrambled points in 2^17-sample chunks, after each chunk
    Mout read back and written as sM_<n>.h5 in the reference's layout (chunked,
    deflate 6; SCP3.cpp:252-255, DiskIO.cpp:201-227) for the split form; the 10
    lowest levels (FP64 eigensolve) of the split form against the FP64 form on
    the same points.  samples_per_s is device-timed over the accumulate calls;
    the dumps and the eigensolve are timed apart."""
    import tempfile

    import torch
    import scp3_b200
    from scp3_b200 import h5, inputs
    nw, x0, MUa, omega = inputs.load("prism_ttm3f")
    chunk = 1 << 17
    res = {}
    outdir = tempfile.mkdtemp(prefix="scp3_triples_")
    autocm = scp3_b200.constants.autocm
    for prec in (precision, "fp64"):
        hb = scp3_b200.HBuild(nw, x0, MUa, omega, n2=48, n3=48, pes="ttm3f", precision=prec,
                              scramble_seed=SCRAMBLE_SEED)
        nb = hb.nb
        hb.accumulate(1 << 45, 4096)           # warm-up, then start clean
        hb.reset()
        torch.cuda.synchronize()
        ms, t_dump, dumps = 0.0, 0.0, []
        Mh = np.zeros((nb, nb), order="F") if prec != "fp64" and dump else None
        kms = np.zeros(4)
        for c0 in range(0, total, chunk):
            hb.profile(True)
            ms += timed_accumulate(hb, c0, min(chunk, total - c0))
            kms += hb.profile(False)[0]
            if Mh is not None:
                t1 = time.perf_counter()
                hb.read(1, out=Mh)
                path = os.path.join(outdir, "sM_%07d.h5" % (c0 + chunk))
                h5.save(path, Mh, deflate=deflate)
                t_dump += time.perf_counter() - t1
                dumps.append({"file": os.path.basename(path), "bytes": os.path.getsize(path)})
                os.remove(path)           # 1.7 GB of float32 before compression
        t0 = time.perf_counter()
        ev = hb.eigvals(10)
        t_eig = time.perf_counter() - t0
        rc, nonfinite, notconv = hb.status()
        res[prec] = dict(samples_per_s=total / (ms * 1e-3), compute_ms=ms,
                         kernel_ms={"per_sample": kms[0], "expand": kms[1], "contract": kms[2]},
                         dump_s=t_dump, dumps=dumps,
                         eig_s=t_eig, levels_cm1=[float(x * autocm) for x in ev], rc=rc, nonfinite=nonfinite,
                         not_converged=notconv)
        hb.close()
    os.rmdir(outdir)
    sp, dp = res[precision], res["fp64"]
    err = float(np.abs(np.array(sp["levels_cm1"]) - np.array(dp["levels_cm1"])).max())
    return {"config": {"workload": "hexamer prism TTM3-F, 48 modes, triples basis Nb=20825, %d scrambled Sobol "
                                   "points in 2^17 chunks, an sM_*.h5 (chunked, deflate %d) after each chunk of the "
                                   "split form" % (total, deflate), "precision": precision, "nb": 20825},
            "split": sp, "fp64": dp, "speedup_vs_fp64": sp["samples_per_s"] / dp["samples_per_s"],
            "max_abs_err_cm1_vs_fp64": err,
            "note": "levels of a %d-point build are dominated by Monte Carlo noise (the plain estimator collapses "
                    "at these sizes); the error compares two arithmetic forms on the same points" % total}


def run_triples(args):
    """--config triples: triples_record at 2^21 points (one JSON line)."""
    import torch
    torch.cuda.set_device(0)
    print(json.dumps(triples_record(args.samples, args.precision, dump=not args.no_dump)))


def guarded(fn, *a):
    """A sub-record of the default line: its dict, or {"error": ...} if it failed,
    so the benchmark line itself is always printed."""
    try:
        return fn(*a)
    except Exception as e:            # noqa: BLE001
        import traceback
        traceback.print_exc()
        return {"error": "%s: %s" % (type(e).__name__, e)}


def fp64_record(nw, x0, MUa, omega, steps, device):
    """The plain FP64 form on the benchmark's workload (the hexamer doubles
    build, 2^20 points per step): device-timed samples/s and the contraction's
    algorithmic FP64 rate against the B200's nominal FP64 peak."""
    import scp3_b200
    hb = scp3_b200.HBuild(nw, x0, MUa, omega, n2=48, n3=0, pes="qtip4pf", precision="fp64",
                          scramble_seed=SCRAMBLE_SEED, device=device)
    nb = hb.nb
    timed_accumulate(hb, 1 << 44, SAMPLES)        # warm-up
    hb.reset()
    hb.profile(True)
    ms = [timed_accumulate(hb, k * SAMPLES, SAMPLES) for k in range(steps)]
    kms, launches = hb.profile(False)
    hb.close()
    achieved = nb * (nb + 1) * SAMPLES * steps / (kms[2] * 1e-3) / 1e12
    return {"value": SAMPLES * steps / (sum(ms) * 1e-3), "unit": "samples/s", "steps": steps,
            "ms_per_step": sum(ms) / steps,
            "kernel_ms": {"per_sample": kms[0], "expand": kms[1], "contract": kms[2]},
            "contraction": {"achieved": achieved, "unit": "TFLOP/s", "peak": FP64_NOMINAL_TFLOPS,
                            "frac": achieved / FP64_NOMINAL_TFLOPS,
                            "peak_source": "nominal B200 FP64 (no measured FP64 peak)",
                            "work": "Nb(Nb+1) FLOP per sample, upper triangle"}}


def cv_record(precision, epochs):
    """The learned control variate on the TTM3-F hexamer prism, doubles basis
    (1225 functions): the surrogate trained on 2^18 exact samples, then
    V_nn over 2^24 points + (V - V_nn) over 2^20 exact points, against the
    plain exact estimator with 2^21 points and with as many points as the
    control variate's GPU time buys; level errors against a 2^26-point exact
    build.  One JSON line; not the benchmark's default."""
    import torch
    import scp3_b200
    from scp3_b200 import inputs, surrogate
    nw, x0, MUa, omega = inputs.load("prism_ttm3f")
    autocm = scp3_b200.constants.autocm
    prec = precision

    def make():
        return scp3_b200.HBuild(nw, x0, MUa, omega, n2=48, n3=0, pes="ttm3f", precision=prec,
                                scramble_seed=SCRAMBLE_SEED)

    sme = scp3_b200.ScaledMatrixElements(omega, 48, 0)

    def levels(Mavg):
        M = np.asfortranarray(Mavg.copy())
        sme.addHODiagonal(M)
        return np.linalg.eigvalsh(M)[:10] * autocm

    def plain(n, i0=0):
        hb = make()
        hb.accumulate(1 << 45, 1 << 17)    # warm-up, as the control variate's builds
        hb.reset()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        hb.accumulate(i0, n)
        M = hb.read(0) / n
        t = time.perf_counter() - t0
        hb.close()
        return M, t

    M_ref, t_ref = plain(1 << 26, 1 << 42)
    e_ref = levels(M_ref)
    hb = make()
    t0 = time.perf_counter()
    q, v = surrogate.sample(hb, 1 << 44, 1 << 18)
    t_sample = time.perf_counter() - t0
    hb.close()
    net = surrogate.MLP(48, hidden=256, max_batch=1 << 18, seed=11)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    loss = net.fit(q, v.astype(np.float32), epochs=epochs, batch=4096, lr=2e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    y = net(q[:1 << 16])
    r2 = 1.0 - float(np.var(v[:1 << 16] - y) / np.var(v[:1 << 16]))
    # the two builds of the control variate, created and warmed up outside the timed region
    # (as plain() creates its build before timing)
    hb_nn, hb_res = make(), make()
    surrogate.attach(hb_nn, net, surrogate.SURROGATE_REPLACE)
    surrogate.attach(hb_res, net, surrogate.SURROGATE_RESIDUAL)
    for hb in (hb_nn, hb_res):
        hb.accumulate(1 << 45, 1 << 17)
        hb.reset()
    err = lambda M: float(np.abs(levels(M) - e_ref).max())
    # three trials with independent Sobol ranges for the exact points of each estimator
    offsets = [0, 1 << 36, 1 << 37]
    cv_trials, t_cv = [], 0.0
    for k, off in enumerate(offsets):
        hb_nn.reset()
        hb_res.reset()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        hb_nn.accumulate((1 << 40) + k * (1 << 24), 1 << 24)
        hb_res.accumulate(off, 1 << 20)
        M_cv = hb_nn.read(0) / (1 << 24) + hb_res.read(0) / (1 << 20)
        torch.cuda.synchronize()
        t_cv = max(t_cv, time.perf_counter() - t0)
        cv_trials.append(err(M_cv))
    hb_nn.close()
    hb_res.close()
    M_p21, t_p21 = plain(1 << 21)
    n_eq = int(min(1 << 24, (1 << 21) * t_cv / t_p21)) // 4096 * 4096
    eq_trials, t_eq = [], 0.0
    for off in offsets:
        M_eq, t = plain(n_eq, off)
        t_eq = max(t_eq, t)
        eq_trials.append(err(M_eq))
    return {"config": {"workload": "hexamer prism TTM3-F, doubles basis Nb=1225; surrogate 48-256-256-256-1 "
                                             "GELU trained on 2^18 exact samples; V_nn over 2^24 + residual over 2^20",
                                 "precision": prec, "trials": "3 independent Sobol ranges for the exact points"},
                      "train": {"samples": 1 << 18, "epochs": epochs, "sample_s": t_sample,
                                "train_s": t_train, "final_batch_loss": loss, "r2_heldin": r2},
                      "control_variate": {"gpu_s": t_cv, "max_level_err_cm1": cv_trials,
                                          "mean": float(np.mean(cv_trials))},
                      "plain_2^21": {"gpu_s": t_p21, "max_level_err_cm1": err(M_p21)},
                      "plain_equal_time": {"samples": n_eq, "gpu_s": t_eq, "max_level_err_cm1": eq_trials,
                                           "mean": float(np.mean(eq_trials))},
                      "reference": {"samples": 1 << 26, "gpu_s": t_ref, "lowest10_cm1": [float(x) for x in e_ref]}}


def run_cv(args):
    """--config cv: cv_record (one JSON line)."""
    import torch
    torch.cuda.set_device(0)
    print(json.dumps(cv_record(args.precision, args.cv_epochs)))


def batch_record(precision, n, steps, warmup):
    """The batched build: 32 qTIP4P/f clusters of 2..8 waters (doubles bases of
    91..946 functions, scp3_b200.inputs.batch_clusters), n scrambled points per
    cluster, built in one batch (one CUDA graph replay per step, autotuned
    contraction work shape) against 32 sequential single builds of the same
    precision and 32 sequential plain FP64 builds.  Levels of every cluster
    against its FP64 build."""
    import torch
    import scp3_b200
    from scp3_b200 import inputs
    cl = inputs.batch_clusters()
    for c in cl:
        c["scramble_seed"] = SCRAMBLE_SEED
    spec = [{k: v for k, v in c.items() if k != "name"} for c in cl]
    autocm = scp3_b200.constants.autocm
    t0 = time.perf_counter()
    b = scp3_b200.Batch(spec, precision=precision)
    t_create = time.perf_counter() - t0
    nsplit, ctas, chunk, tuned_ms = b.shape()

    def timed_batch(bb, steps, warmup):
        st = torch.cuda.ExternalStream(bb.stream)
        for k in range(warmup):
            bb.reset()
            bb.accumulate(k * n, n)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms = []
        for k in range(steps):
            bb.reset()
            e0.record(st)
            bb.accumulate(0, n)
            e1.record(st)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return float(np.median(ms))

    ms_graph = timed_batch(b, steps, warmup)
    bd = scp3_b200.Batch(spec, precision=precision, graph=False)
    ms_direct = timed_batch(bd, steps, 1)
    bd.close()

    def sequential(prec):
        hbs = [scp3_b200.HBuild(c["nw"], c["x0"], c["MUa"], c["omega"], modes=c["modes"], n2=c["n2"], n3=0,
                                precision=prec, scramble_seed=SCRAMBLE_SEED) for c in spec]
        for hb in hbs:             # warm-up
            hb.accumulate(0, 4096)
        torch.cuda.synchronize()
        for hb in hbs:
            hb.reset()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for hb in hbs:
            hb.accumulate(0, n)
        torch.cuda.synchronize()
        return hbs, 1e3 * (time.perf_counter() - t0)

    seq, ms_seq = sequential(precision)
    seq64, ms_seq64 = sequential("fp64")
    # accuracy: the batch against the same-precision single builds (same kernels) and FP64 levels
    b.reset()
    b.accumulate(0, n)
    worst_same, worst_lvl, per = 0.0, 0.0, []
    for i, c in enumerate(cl):
        M = b.read(i, 0)
        R = seq[i].read(0)
        worst_same = max(worst_same, float(np.abs(M - R).max() / np.abs(R).max()))
        e_b = np.linalg.eigvalsh(b.read(i, 1))[:10] * autocm
        e_64 = np.linalg.eigvalsh(seq64[i].read(1))[:10] * autocm
        err = float(np.abs(e_b - e_64).max())
        worst_lvl = max(worst_lvl, err)
        per.append({"name": c["name"], "nw": c["nw"], "nmodes": int(c["modes"].size), "nb": b.nb[i],
                    "max_level_err_cm1": err})
    for hb in seq + seq64:
        hb.close()
    basis_sizes = list(b.nb)
    b.close()
    total = len(cl) * n
    return {
        "config": {"workload": "32 qTIP4P/f clusters, 2..8 waters, 12..42 modes, doubles bases 91..946, "
                               "%d scrambled Sobol points per cluster" % n, "precision": precision,
                   "clusters": len(cl), "samples_per_cluster": n, "basis_sizes": basis_sizes},
        "metric": "cluster-samples/s", "unit": "samples/s",
        "batch_graph": {"ms": ms_graph, "value": total / (ms_graph * 1e-3)},
        "batch_direct": {"ms": ms_direct, "value": total / (ms_direct * 1e-3)},
        "sequential_same_precision": {"ms": ms_seq, "value": total / (ms_seq * 1e-3)},
        "sequential_fp64": {"ms": ms_seq64, "value": total / (ms_seq64 * 1e-3)},
        "speedup_vs_sequential": ms_seq / ms_graph, "speedup_vs_sequential_fp64": ms_seq64 / ms_graph,
        "work_shape": {"nsplit": nsplit, "ctas": ctas, "samples_per_pass": chunk, "tuned_contract_ms": tuned_ms,
                       "create_s": t_create},
        "max_rel_diff_vs_single_builds": worst_same, "max_level_err_cm1_vs_fp64": worst_lvl, "clusters": per}


def run_batch(args):
    """--config batch: batch_record at 2^18 points per cluster (one JSON line)."""
    import torch
    torch.cuda.set_device(0)
    n = args.samples if args.samples != 1 << 20 else 1 << 18
    print(json.dumps(batch_record(args.precision, n, args.steps, args.warmup)))


def gradient_form(prec, nw, x0, MUa, omega, n, steps, warmup):
    """One form of the gradient-estimator build on the hexamer doubles basis:
    device-timed samples/s over `steps` accumulate calls of n points, the kernel
    split, and the 10 lowest levels (cm^-1) of Mout over those points."""
    import scp3_b200
    hb = scp3_b200.HBuild(nw, x0, MUa, omega, n2=48, n3=0, pes="qtip4pf", precision=prec,
                          scramble_seed=SCRAMBLE_SEED, estimator="gradient")
    for k in range(max(warmup, 1)):
        timed_accumulate(hb, (1 << 44) + k * n, n)
    hb.reset()
    hb.profile(True)
    ms = [timed_accumulate(hb, k * n, n) for k in range(steps)]
    kms, launches = hb.profile(False)
    rc, nonfinite, notconv = hb.status()
    levels = np.sort(np.linalg.eigvalsh(hb.read(1)))[:10] * scp3_b200.constants.autocm
    nb = hb.nb
    hb.close()
    t = sum(ms) / len(ms)
    return {"value": n / (t * 1e-3), "ms_per_step": t, "nb": nb,
            "kernel_ms": {"per_sample": kms[0] / steps, "stein": kms[2] / steps},
            "status": {"rc": rc, "nonfinite": nonfinite, "not_converged": notconv}, "levels": levels}


def gradient_record(nw, x0, MUa, omega, n, steps):
    """The gradient (Stein) estimator on the hexamer doubles basis: the BF16x3 form
    against the FP64 form on the same points (samples/s, ratio, level error)."""
    split = gradient_form("bf16x3", nw, x0, MUa, omega, n, steps, 1)
    ref = gradient_form("fp64", nw, x0, MUa, omega, n, steps, 1)
    return {"workload": "hexamer prism qTIP4P/f, doubles basis Nb=%d, %d scrambled Sobol points per step, Stein "
                        "estimator (SCP3's default path)" % (split["nb"], n),
            "bf16x3": {"value": split["value"], "unit": "samples/s", "kernel_ms": split["kernel_ms"]},
            "fp64": {"value": ref["value"], "unit": "samples/s", "kernel_ms": ref["kernel_ms"]},
            "speedup_vs_fp64": split["value"] / ref["value"],
            "max_abs_err_cm1_vs_fp64": float(np.abs(split["levels"] - ref["levels"]).max()),
            "status": split["status"]}


def run_gradient(args):
    """The reference's default estimator (no -G): the Stein estimator of every
    upper element from V and dV/dq (ScaledMatrixElements.cpp:102-725,
    TripleExcitations.h) on the hexamer prism doubles basis (Nb = 1225, 48 modes,
    qTIP4P/f energy and gradient per sample).  --precision bf16x3 (default): the
    products W Phi^T on the tensor cores (BF16x3), the potential, its gradient
    and the same-mode pair sums in FP64, against the FP64 form on the same
    points (rate ratio and level error); --precision fp64: the FP64 form alone.
    value: samples/s, device-timed.  One JSON line; not the benchmark's default."""
    import torch
    from scp3_b200 import inputs
    torch.cuda.set_device(0)
    nw, x0, MUa, omega = inputs.load(INPUT)
    n = args.samples
    prec = "fp64" if args.precision == "fp64" else "bf16x3"
    clocks = Clocks(0)
    main = gradient_form(prec, nw, x0, MUa, omega, n, args.steps, args.warmup)
    clk = clocks.stop()
    line = {
        "metric": "gradient-estimator build: Sobol samples/s (hexamer doubles)", "value": main["value"],
        "unit": "samples/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": main["ms_per_step"], "higher_is_better": True,
        "dtype": "bf16x3/f64" if prec != "fp64" else "f64", "data": "synthetic",
        "config": {"workload": "hexamer prism qTIP4P/f, 48 modes, doubles basis Nb=%d, %d scrambled Sobol points per "
                               "step, the Stein estimator of SCP3's default path" % (main["nb"], n),
                   "precision": prec},
        "kernel_ms": main["kernel_ms"], "clocks": clk, "status": main["status"]}
    if prec != "fp64":
        ref = gradient_form("fp64", nw, x0, MUa, omega, n, args.steps, 1)
        line["fp64"] = {"value": ref["value"], "ms_per_step": ref["ms_per_step"], "kernel_ms": ref["kernel_ms"]}
        line["speedup_vs_fp64"] = main["value"] / ref["value"]
        line["levels"] = {"max_abs_err_cm1_vs_fp64": float(np.abs(main["levels"] - ref["levels"]).max()),
                          "lowest10_cm1_fp64": [float(x) for x in ref["levels"]],
                          "samples": n * args.steps}
    print(json.dumps(line))


def _ref_scp1_rate(job):
    """One process of the CPU reference arm of --config scp1: the reference's own
    std_normal and qTIP4P/f operator in SCP1.cpp's sample loop (single-threaded,
    as one MPI rank)."""
    pes, nw, q, d, iU, skip, i0, i1 = job
    from oracle import scp1_oracle
    t0 = time.perf_counter()
    scp1_oracle.ref_average_sums(pes, nw, q, d, iU, skip, i0, i1, fast=True)
    return (i1 - i0) / (time.perf_counter() - t0)


def run_scp1(args):
    """SCP1 averages: SCP1::average (SCP1.cpp:34-90) on the hexamer prism input --
    per point the qTIP4P/f energy and gradient at bohr (q + isqrtM_U (y % sqrt(d))),
    summed into <V>, <UX> and <UX dq^T> -- over 2^20 unscrambled Sobol points
    (SCP1_main's default NSobol), harmonic density of the input Hessian at T = 0.
    value: points/s of one scp3gpu_scp1_average call (host clock around the
    synchronous C-ABI call, inputs and sums copied inside).  cpu_baseline: the
    reference's own functions in the same loop, one process per host core as
    MPI ranks would run it.  One JSON line; not the benchmark's default."""
    import multiprocessing as mproc

    import torch
    import scp3_b200
    from scp3_b200 import constants as C, modes, scp1
    torch.cuda.set_device(0)
    n = args.samples
    species, mass, x0, H = modes.read_input(os.path.join(ROOT, "scp3_b200", "data", INPUT + ".dat"))
    _, mass, x0, H = modes.ohhohh(mass, x0, H)
    nw = x0.size // 9
    w2, U = scp1.eig_sym(H)
    omega = np.sqrt(np.abs(w2))
    d = np.zeros_like(omega)
    keep = omega >= 50.0 / C.autocm
    d[keep] = 0.5 / omega[keep]
    iU = U / np.sqrt(mass)[:, None]
    skip = 1 << (int(np.floor(np.log2(float(n)))) + 1)
    g = scp3_b200.SCP1Average("qtip4pf", nw)
    for k in range(max(args.warmup, 1)):
        g.sums(x0, d, iU, skip, 0, 1 << 14)
    clocks = Clocks(0)
    times = []
    for k in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        up, UX, UXq = g.sums(x0, d, iU, skip, 0, n)
        times.append(time.perf_counter() - t0)
    clk = clocks.stop()
    g.close()
    t = float(np.median(times))
    cpu = None
    if not args.no_cpu_baseline:
        try:
            import oracle
            if oracle.ref_available(fast=True):
                procs = min(16, os.cpu_count() or 1)
                per = 1 << 15
                jobs = [("qtip4pf", nw, x0, d, iU, skip, r * per, (r + 1) * per) for r in range(procs)]
                with mproc.get_context("spawn").Pool(procs) as pool:
                    rates = pool.map(_ref_scp1_rate, jobs)
                cpu = {"value": float(np.sum(rates)), "unit": "samples/s", "cores": procs, "kind": "reference",
                       "sample": "%d processes x %d points each (the reference's std_normal + qTIP4P/f "
                                 "operator in SCP1.cpp's loop, oracle/_ref release flags)" % (procs, per)}
        except Exception as e:          # noqa: BLE001
            cpu = {"unavailable": str(e)}
    chunks = (n + 65535) // 65536
    print(json.dumps({
        "metric": "SCP1 average: Sobol points/s (hexamer, qTIP4P/f energy + gradient per point)",
        "value": n / t, "unit": "samples/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "hexamer prism qTIP4P/f, 54 Cartesian dims, %d unscrambled Sobol points, T = 0 "
                               "harmonic density of the input Hessian" % n},
        "timing": "host clock around the synchronous scp3gpu_scp1_average call (inputs and sums copied inside)",
        "gpu_launches": 2 * chunks + 1, "clocks": clk, "cpu_baseline": cpu,
        "check": {"mean_V_hartree": up / n, "max_abs_mean_UX": float(np.abs(UX).max() / n)}}))


def main():
    global SAMPLES
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="bf16x3", choices=["fp64", "bf16x3", "f16x3"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--config", default="doubles", choices=["doubles", "triples", "cv", "batch", "scp1", "gradient"],
                    help="doubles: the benchmark (hexamer, Nb=1225); triples: the TTM3-F triples build; "
                         "cv: the learned control variate; batch: 32 clusters in one batched build; "
                         "scp1: the SCP1 effective-Hessian averages; gradient: the default (Stein) estimator")
    ap.add_argument("--cv-epochs", type=int, default=100)
    ap.add_argument("--no-levels", action="store_true", help="skip the FP64 level check (profiler captures)")
    ap.add_argument("--no-dump", action="store_true", help="triples: skip the sM_*.h5 dumps")
    ap.add_argument("--samples", type=int, default=SAMPLES,
                    help="samples per step (the benchmark is 2^20; smaller only for profiler captures)")
    ap.add_argument("--no-subrecords", action="store_true",
                    help="skip the fp64 and triples sub-records of the default line")
    ap.add_argument("--standin", action="store_true",
                    help="CPU tests: ranks over gloo with a host stand-in build (no GPU, not a benchmark)")
    ap.add_argument("--dump-matrix", default=None, help="--standin: save rank 0's reduced matrix (.npy)")
    args = ap.parse_args()
    SAMPLES = args.samples
    if args.config == "cv":
        run_cv(args)
        return
    if args.config == "batch":
        run_batch(args)
        return
    if args.config == "scp1":
        run_scp1(args)
        return
    if args.config == "gradient":
        run_gradient(args)
        return
    if args.config == "triples":
        if args.samples == 1 << 20:
            args.samples = 1 << 21
        run_triples(args)
        return
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(launch_ranks(args.gpus, sys.argv[1:]))
    if args.impl == "reference":
        # rank 0 alone times the CPU build; the other ranks exit without work
        run_reference(args, int(os.environ.get("RANK", "0")))
        return
    world, rank, local = dist_setup(args.gpus, "gloo" if args.standin else "nccl")
    if args.standin:
        run_standin(args, world, rank)
        return

    import torch
    torch.cuda.set_device(local)
    import scp3_b200
    from scp3_b200 import inputs
    nw, x0, MUa, omega = inputs.load(INPUT)
    nm0 = omega.size
    hb = scp3_b200.HBuild(nw, x0, MUa, omega, n2=48, n3=0, pes="qtip4pf", precision=args.precision,
                          scramble_seed=SCRAMBLE_SEED, device=local)
    nb = hb.nb
    stream = torch.cuda.ExternalStream(hb.stream, device=local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=local)
    Mdev = torch.zeros((nb, nb), dtype=torch.float64, device=local)
    from scp3_b200 import shard
    base, _ = shard.sample_range(rank, world, 0, SAMPLES, "weak")   # disjoint Sobol ranges per rank

    def step(k):
        hb.accumulate(base + k * SAMPLES, SAMPLES)
        if world > 1:
            exchange(hb, Mdev, stream)

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()
    hb.reset()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    hb.profile(True)
    total_ms = 0.0
    for k in range(args.steps):
        flush.fill_(k & 0xff)          # L2 flush between steps, outside the timed events
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step(args.warmup + k)
        e1.record(torch.cuda.current_stream() if world > 1 else stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    ms, launches = hb.profile(False)
    torch.cuda.synchronize()
    clk = clocks.stop()
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([total_ms], dtype=torch.float64, device=local)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    value = world * SAMPLES * args.steps / (total_ms / 1e3)
    rc, nonfinite, notconv = hb.status()

    # dominant kernel: the contraction; algorithmic work Nb(Nb+1) flops per sample
    peaks, peak_src = load_peaks()
    flops_per_sample = nb * (nb + 1)
    cont_launches = int(launches[2])
    avg_ms = ms[2] / max(cont_launches, 1)
    samples_per_launch = SAMPLES * args.steps / max(cont_launches, 1)
    achieved = flops_per_sample * samples_per_launch / (avg_ms / 1e3) / 1e12
    if args.precision == "fp64":
        roof = {"bound": "fp64", "achieved": achieved, "peak": FP64_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                "frac": achieved / FP64_NOMINAL_TFLOPS, "traffic": None,
                "note": "FP64 DFMA contraction; peak is B200 nominal FP64 (no measured FP64 peak)"}
    else:
        pk = peaks["bf16_tflops"]
        traffic = CONTRACT_DRAM_BYTES_PER_SAMPLE * samples_per_launch if nb == 1225 else None
        roof = {"bound": "tensor", "achieved": achieved, "peak": pk, "unit": "TFLOP/s", "frac": achieved / pk,
                "traffic": traffic, "note": "algorithmic Nb(Nb+1) flops/sample; BF16x3 issues 3 tensor products each "
                                            "(ceiling 1/3); peak " + peak_src + "; traffic: ncu DRAM bytes per "
                                            "launch (read + write; operand 5200 B/sample)",
                "traffic_source": "not measured in this run: a constant per sample from one ncu capture of the "
                                  "contraction (profiles/), scaled to the samples of an average launch"}

    line = {"metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "bf16x3/f32/f64",
            "data": "synthetic",
            "config": bench_config(args.precision, nb, world),
            "roofline": roof,
            # the handle's timing counts a split-form preparation (sign partition + expansion) as one
            # launch of kind 1; it is two kernels
            "gpu_launches": int(launches[0] + launches[2] + launches[3] +
                                launches[1] * (1 if args.precision == "fp64" else 2)),
            "kernel_ms": {"per_sample": ms[0], "expand": ms[1], "contract": ms[2], "readout": ms[3]},
            "clocks": clk, "status": {"rc": rc, "nonfinite": nonfinite, "not_converged": notconv}}

    if rank == 0 and args.precision != "fp64" and not args.no_levels:
        # quality gate of the metric: the same 2^20 points through the FP64 plain form
        hb.reset()
        hb.accumulate(base, SAMPLES)
        e_split = hb.eigvals(10)
        hb64 = scp3_b200.HBuild(nw, x0, MUa, omega, n2=48, n3=0, pes="qtip4pf", precision="fp64",
                                scramble_seed=SCRAMBLE_SEED, device=local)
        hb64.accumulate(base, SAMPLES)
        e64 = hb64.eigvals(10)
        hb64.close()
        autocm = scp3_b200.constants.autocm
        line["levels"] = {"max_abs_err_cm1_vs_fp64": float(np.abs(e_split - e64).max() * autocm),
                          "lowest10_cm1_fp64": [float(x * autocm) for x in e64],
                          "samples": SAMPLES}
    if not args.no_e2e:
        # the -r path with host buffers on every rank: normals in from pinned memory, Mout
        # back to host; the slowest rank's time is the job's
        normals = torch.from_numpy(scp3_b200.std_normals(nm0, (1 << 41) + rank * SAMPLES, SAMPLES,
                                                          scramble_seed=SCRAMBLE_SEED))
        if args.precision != "fp64":
            # the split forms compute q in FP32: their normals go in as FP32, half the bytes
            normals = normals.float()
        normals = normals.pin_memory().numpy()
        Mh = np.asfortranarray(torch.empty((nb, nb), dtype=torch.float64).pin_memory().numpy().T)
        hb.reset()
        hb.accumulate_normals(normals)
        hb.read(1, out=Mh)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        t0 = time.perf_counter()
        ne = args.steps
        for k in range(ne):
            hb.accumulate_normals(normals)
            hb.read(1, out=Mh)
        e2e_s = (time.perf_counter() - t0) / ne
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([e2e_s], dtype=torch.float64, device=local)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        line["e2e"] = {"value": world * SAMPLES / e2e_s, "unit": "samples/s",
                       "h2d_bytes_per_step": int(normals.nbytes), "d2h_bytes_per_step": int(nb * nb * 8),
                       "path": ("scp3gpu_hbuild_accumulate_normals" + ("" if args.precision == "fp64" else "_f32") +
                                " + scp3gpu_hbuild_read(mode 1), host buffers, every rank; bytes per rank")}
    if rank == 0 and world == 1 and args.precision != "fp64" and not args.no_subrecords:
        # the plain form on the same workload, and the triples configuration with its
        # split-vs-FP64 ratio: the two other numbers the metric's target is read from
        hb.close()
        line["fp64"] = guarded(fp64_record, nw, x0, MUa, omega, 3, local)
        line["triples"] = guarded(triples_record, TRIPLES_SAMPLES, args.precision)
        t, f = line["triples"], line["fp64"]
        if "error" not in t and "error" not in f:
            line["target"] = {"triples_speedup_vs_fp64": t["speedup_vs_fp64"], "wanted": ">= 10",
                              "triples_max_level_err_cm1": t["max_abs_err_cm1_vs_fp64"], "wanted_cm1": "<= 0.1",
                              "doubles_speedup_vs_fp64": value / f["value"]}
        # configs C4 and C5 in compact form (their full lines: --config batch, --config cv)
        bt = guarded(batch_record, args.precision, 1 << 18, 3, 1)
        line["batch"] = bt if "error" in bt else {k: v for k, v in bt.items() if k != "clusters"}
        line["cv"] = guarded(cv_record, args.precision, 100)
        # the reference's default estimator (no -G) in compact form (full line: --config gradient)
        line["gradient"] = guarded(gradient_record, nw, x0, MUa, omega, 1 << 18, 3)
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        normals = scp3_b200.std_normals(nm0, 0, 1 << 17, scramble_seed=SCRAMBLE_SEED)
        cb = cpu_reference(nw, x0, MUa, omega, np.arange(nm0, dtype=np.int32), 48, 0, normals)
        if cb is not None:
            line["levels_vs_reference"] = guarded(levels_vs_reference, cb, nw, x0, MUa, omega, normals,
                                                  args.precision, local)
            cb.pop("_M", None)
            cb.pop("_n", None)
        line["cpu_baseline"] = cb
    if rank == 0:
        print(json.dumps(line))
    hb.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
