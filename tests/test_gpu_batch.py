"""GPU tests of the batched build (scp3gpu_batch_*).

Clusters of uneven size and basis built in one batch give, cluster by
cluster, the matrix that a single split-form build of the same config gives:
both run the same per-sample, partition and expansion code on the same BF16 (or
FP16) operand values; both contract 128 x 256 tiles, but the batch splits
its passes by the tiling of all clusters and a single build by its own, so the
FP32 runs end at different samples and they agree to the FP32 accumulation
error (1e-5 of max|M|).  Graph replay equals direct launches bit for bit, several
accumulate calls equal one call over the same points, and the batch stays
within the split form's tolerance of the reference's golden matrices."""
import numpy as np
import pytest

from conftest import load_hbuild_case, upper_to_full

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scp3():
    import torch
    assert torch.cuda.is_available()
    import scp3_b200
    return scp3_b200


def _cluster(c, **over):
    sseed = int(c["scramble_seed"])
    d = dict(nw=int(c["nw"]), x0=c["x0"], MUa=c["MUa"], omega=c["omega"], modes=c["modes"], n2=int(c["n2"]),
             n3=int(c["n3"]), scramble_seed=None if sseed < 0 else sseed)
    d.update(over)
    return d


def _single(scp3, d, pes, precision):
    return scp3.HBuild(d["nw"], d["x0"], d["MUa"], d["omega"], modes=d["modes"], n2=d["n2"], n3=d["n3"], pes=pes,
                       precision=precision, scramble_seed=d["scramble_seed"])


QT_CASES = ["dimer_qtip4pf", "dimer_qtip4pf_unscrambled", "hexamer_qtip4pf", "hexamer_qtip4pf_modesel"]


def _qt_clusters():
    cl = [_cluster(load_hbuild_case(n)) for n in QT_CASES]
    # a doubles-only hexamer (1225 functions) and a dimer with the triples of all modes
    hx = load_hbuild_case("hexamer_qtip4pf")
    cl.append(_cluster(hx, modes=np.arange(48), n2=48, n3=0))
    dm = load_hbuild_case("dimer_qtip4pf")
    cl.append(_cluster(dm, n3=12))
    return cl


@pytest.mark.parametrize("prec", ["bf16x3", "f16x3_pes64"])
def test_batch_matches_single_builds(scp3, prec):
    cl = _qt_clusters()
    n = 3 * 4096 + 1000          # ragged: the last pass is padded
    b = scp3.Batch(cl, pes="qtip4pf", precision=prec, chunk=8192)
    assert len(set(b.nb)) == len(cl)      # every basis size differs
    b.accumulate(7, n)
    for i, d in enumerate(cl):
        hb = _single(scp3, d, "qtip4pf", prec)
        hb.accumulate(7, n)
        ref = hb.read(0)
        M = b.read(i, 0)
        assert M.shape == ref.shape
        scale = np.abs(ref).max()
        assert np.abs(M - ref).max() <= 1e-5 * scale, (i, np.abs(M - ref).max() / scale)
        M1, R1 = b.read(i, 1), hb.read(1)
        assert np.abs(M1 - R1).max() <= 1e-5 * np.abs(R1).max()
        assert b.status(i)[0] == 0
        hb.close()
    assert b.sample_count() == n


def test_batch_graph_equals_direct_and_calls_compose(scp3):
    cl = _qt_clusters()[:4]
    g = scp3.Batch(cl, precision="bf16x3", chunk=4096, graph=True, autotune=False)
    d = scp3.Batch(cl, precision="bf16x3", chunk=4096, graph=False, autotune=False)
    assert g.shape()[:3] == d.shape()[:3]
    i0 = 1 << 30                         # the reference's skip: point 0 of the unscrambled sequence is u = 0
    g.accumulate(i0, 3 * 4096)           # one graph of three passes
    g.accumulate(i0 + 3 * 4096, 2 * 4096)    # a second graph (two passes) ...
    g.accumulate(i0 + 5 * 4096, 2 * 4096)    # ... replayed with new Sobol offsets
    d.accumulate(i0, 7 * 4096)
    for i in range(len(cl)):
        A, B = g.read(i, 0), d.read(i, 0)
        assert np.array_equal(A, B), i


def test_batch_autotuned_shape_is_valid(scp3):
    cl = _qt_clusters()
    b = scp3.Batch(cl, precision="bf16x3", chunk=16384)
    nsplit, ctas, chunk, ms = b.shape()
    assert chunk == 16384 and 1 <= nsplit <= 16 and ms > 0
    assert ctas >= 1
    # tuning trials leave no trace in the sums
    b.accumulate(7, 4096)
    ref = scp3.Batch(cl, precision="bf16x3", chunk=16384, autotune=False)
    ref.accumulate(7, 4096)
    for i in range(len(cl)):
        A, B = b.read(i, 0), ref.read(i, 0)
        assert np.abs(A - B).max() <= 1e-11 * np.abs(B).max()


def test_batch_against_golden(scp3, oracle_mod):
    """Each cluster of a batch against the reference's golden matrix, same bound
    as the single split-form build: 5e-4 of sum_s |Phi_i||V||Phi_j|."""
    cases = ["dimer_qtip4pf", "hexamer_qtip4pf", "hexamer_qtip4pf_modesel"]
    cs = [load_hbuild_case(n) for n in cases]
    # one Sobol range for all: the golden cases all start at index 0
    ns = min(int(c["nsamples"]) for c in cs)
    b = scp3.Batch([_cluster(c) for c in cs], precision="f16x3")
    b.accumulate(0, ns)
    for i, c in enumerate(cs):
        sseed = int(c["scramble_seed"])
        normals = oracle_mod.std_normals(c["omega"].size, 0, ns, scramble_seed=None if sseed < 0 else sseed)
        q, v = oracle_mod.samples(int(c["pes"]), int(c["nw"]), c["x0"], c["MUa"], c["omega"], normals)
        ref = oracle_mod.accumulate(q[:, c["modes"]], v, int(c["n2"]), int(c["n3"]))
        ref = ref + np.triu(ref, 1).T
        A = oracle_mod.accumulate(q[:, c["modes"]], v, int(c["n2"]), int(c["n3"]), absolute=True)
        A = A + np.triu(A, 1).T
        M = b.read(i, 0)
        rel = np.abs(M - ref) / np.maximum(A, 1e-300)
        assert rel.max() <= 5e-4, (cases[i], rel.max())


def test_batch_ttm3f(scp3):
    cs = [load_hbuild_case(n) for n in ["dimer_ttm3f", "hexamer_ttm3f"]]
    cl = [_cluster(c) for c in cs]
    b = scp3.Batch(cl, pes="ttm3f", precision="bf16x3", chunk=4096)
    b.accumulate(7, 4096)
    for i, d in enumerate(cl):
        hb = _single(scp3, d, "ttm3f", "bf16x3")
        hb.accumulate(7, 4096)
        ref = hb.read(0)
        assert np.abs(b.read(i, 0) - ref).max() <= 1e-5 * np.abs(ref).max()
        assert b.status(i)[0] == 0
        hb.close()


def test_batch_rejects(scp3):
    c = _cluster(load_hbuild_case("dimer_qtip4pf"))
    with pytest.raises(scp3.SCP3GPUError):
        scp3.Batch([c], precision="fp64")
    with pytest.raises(scp3.SCP3GPUError):
        scp3.Batch([c], precision="bf16x3", chunk=1000)
