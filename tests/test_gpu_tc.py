"""GPU parity of the split-precision forms (BF16x3 or FP16x3 tcgen05
contraction, FP32 accumulation in TMEM drained to FP64 every 256 K slots, FP32
or FP64 potential) against the reference's golden matrices and the FP64 form.

Tolerance per element: 5e-4 of sum_s |Phi_i||V||Phi_j| (a bound on one FP32
accumulation run plus ~1e-5 from the split products and the FP32 potential);
median 2e-5.  Levels of Mout: within 0.1 cm^-1 of the FP64 form -- for the
contraction alone on the small golden cases, for the whole split form on the
2^16-sample hexamer doubles build."""
import numpy as np
import pytest

from conftest import load_hbuild_case, upper_to_full

pytestmark = pytest.mark.gpu
AUTOCM = 2.194746313e5


@pytest.fixture(scope="module")
def scp3():
    import torch
    assert torch.cuda.is_available()
    import scp3_b200
    return scp3_b200


def _build(scp3, c, precision):
    sseed = int(c["scramble_seed"])
    return scp3.HBuild(int(c["nw"]), c["x0"], c["MUa"], c["omega"], modes=c["modes"], n2=int(c["n2"]),
                       n3=int(c["n3"]), pes=int(c["pes"]), precision=precision,
                       scramble_seed=None if sseed < 0 else sseed)


@pytest.mark.parametrize("prec", ["bf16x3", "f16x3", "bf16x3_pes64", "f16x3_pes64"])
@pytest.mark.parametrize("name", ["dimer_qtip4pf", "hexamer_qtip4pf", "dimer_ttm3f", "hexamer_qtip4pf_modesel"])
def test_split_matches_reference(scp3, oracle_mod, name, prec):
    c = load_hbuild_case(name)
    ns = int(c["nsamples"])
    hb = _build(scp3, c, prec)
    hb.accumulate(int(c["index0"]), ns)
    M = hb.read(0)
    assert hb.status()[0] == 0
    nb = M.shape[0]
    ref = upper_to_full(c["M_upper"], nb)
    sseed = int(c["scramble_seed"])
    normals = oracle_mod.std_normals(c["omega"].size, int(c["index0"]), ns, scramble_seed=None if sseed < 0 else sseed)
    q, v = oracle_mod.samples(int(c["pes"]), int(c["nw"]), c["x0"], c["MUa"], c["omega"], normals)
    A = oracle_mod.accumulate(q[:, c["modes"]], v, int(c["n2"]), int(c["n3"]), absolute=True)
    A = A + np.triu(A, 1).T
    rel = np.abs(M - ref) / np.maximum(A, 1e-300)
    assert rel.max() <= 5e-4, rel.max()
    assert np.median(rel) <= 2e-5, np.median(rel)
    if prec.endswith("pes64"):
        # the contraction's own error in the levels, potential in FP64 (the FP32
        # potential adds per-sample noise that only a long run averages).  FP16
        # halves stay within 0.1 cm^-1 even on a few hundred samples; BF16 halves
        # (8-bit significands) reach 0.13 cm^-1 on the 512-sample triples case
        # and are held to 0.2 there -- at the benchmark's 2^20 samples both are
        # under 0.05 (test_split_hexamer_doubles_levels, bench.py levels)
        hb64 = _build(scp3, c, "fp64")
        hb64.accumulate(int(c["index0"]), ns)
        e32 = hb.eigvals(min(10, nb))
        e64 = hb64.eigvals(min(10, nb))
        tol = 0.1 if prec.startswith("f16") else 0.2
        assert np.abs(e32 - e64).max() * AUTOCM <= tol, (e32 - e64) * AUTOCM


@pytest.mark.parametrize("prec", ["bf16x3", "f16x3"])
def test_split_hexamer_doubles_levels(scp3, prec):
    from scp3_b200 import inputs
    nw, x0, MUa, omega = inputs.load("prism_qtip4pf", build_if_missing=False)
    ns = 1 << 16
    out = {}
    for p in (prec, "fp64"):
        hb = scp3.HBuild(nw, x0, MUa, omega, n2=48, n3=0, precision=p, scramble_seed=0x5C3)
        hb.accumulate(0, ns)
        assert hb.sample_count() == ns and hb.status()[0] == 0
        out[p] = (hb.read(1), hb.eigvals(10))
    (M32, e32), (M64, e64) = out[prec], out["fp64"]
    assert np.abs(e32 - e64).max() * AUTOCM <= 0.1, (e32 - e64) * AUTOCM
    assert np.linalg.norm(M32 - M64) <= 1e-4 * np.linalg.norm(M64)


def test_split_uneven_passes_and_host_normals(scp3):
    """The same 2^17 hexamer points through the BF16x3 form three ways: one call
    (one pass, shorter than the 2^18-sample plan), uneven calls (passes of 3, 9
    and 20 flush blocks of 4096), and the FP32 host-normals entry (its pieces
    ramp 2^15, 2^15, 2^16).  Every pass cuts its work units' k-block ranges from
    its own length; a missing or repeated k-block range would move the sums by
    ~1/14 of a pass, far beyond the FP32 regrouping and the normals' FP32
    rounding that the three builds differ by."""
    from scp3_b200 import inputs
    nw, x0, MUa, omega = inputs.load("prism_qtip4pf", build_if_missing=False)
    ns = 1 << 17

    def make():
        return scp3.HBuild(nw, x0, MUa, omega, n2=48, n3=0, precision="bf16x3", scramble_seed=0x5C3)

    hb = make()
    hb.accumulate(0, ns)
    M1 = hb.read(0)
    hb2 = make()
    for a, b in ((0, 3 * 4096), (3 * 4096, 12 * 4096), (12 * 4096, ns)):
        hb2.accumulate(a, b - a)
    M2 = hb2.read(0)
    hb3 = make()
    hb3.accumulate_normals(scp3.std_normals(omega.size, 0, ns, scramble_seed=0x5C3).astype(np.float32))
    M3 = hb3.read(0)
    for h in (hb, hb2, hb3):
        assert h.sample_count() == ns and h.status() == (0, 0, 0)
        h.close()
    n1 = np.linalg.norm(M1)
    assert np.linalg.norm(M2 - M1) <= 1e-5 * n1, np.linalg.norm(M2 - M1) / n1
    assert np.linalg.norm(M3 - M1) <= 1e-4 * n1, np.linalg.norm(M3 - M1) / n1
