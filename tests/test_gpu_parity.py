"""GPU parity: the CUDA path through the C ABI against the reference's golden
vectors (tests/golden) and the oracle (oracle/scp3_oracle.c), FP64 plain form.

Tolerances: Sobol integer states and uniforms bit-exact; normals <= 1e-14
relative (device log vs glibc log); potentials <= 1e-12 relative; matrix
elements <= 1e-12 of sum_s |Phi_i||V||Phi_j| (the scale a near-cancelling
element is measured against)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, hbuild_case_names, load_hbuild_case, upper_to_full

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scp3():
    import torch
    assert torch.cuda.is_available()
    import scp3_b200
    scp3_b200._lib.lib()
    return scp3_b200


def test_std_normal_reference_stream(scp3, oracle_mod):
    z = np.load(os.path.join(GOLDEN, "sobol_ref.npz"))
    g = scp3.std_normals(48, 1 << 30, 16)
    assert np.allclose(g, z["std_normal48_from2_30"], rtol=1e-14, atol=0)
    g0 = scp3.std_normals(66, 1, 63)            # index 0 is u = 0 -> -inf in the reference too
    o0 = oracle_mod.std_normals(66, 1, 63)
    assert np.allclose(g0, o0, rtol=1e-14, atol=0)
    seed = [1 << 30]
    first = scp3.std_normal(48, seed)
    assert seed[0] == (1 << 30) + 1
    assert first[0] == pytest.approx(-5.943267008474047, abs=1e-14)


def test_std_normal_scrambled_matches_oracle(scp3, oracle_mod):
    g = scp3.std_normals(48, 12345, 4096, scramble_seed=0x5C3)
    o = oracle_mod.std_normals(48, 12345, 4096, scramble_seed=0x5C3)
    assert np.allclose(g, o, rtol=1e-14, atol=1e-15)


@pytest.mark.parametrize("pes", ["qtip4pf", "ttm3f"])
def test_pes_energies_match_reference(scp3, pes):
    z = np.load(os.path.join(GOLDEN, "pes_ref.npz"), allow_pickle=True)
    p = scp3.PES(pes)
    for nw in sorted(set(int(x) for x in z["nw"])):
        idx = [k for k, n in enumerate(z["nw"]) if n == nw]
        X = np.stack([z["geoms"][k] for k in idx])
        E, it = p.energies(X, return_iters=True)
        ref = z["e_" + pes][idx]
        assert np.allclose(E, ref, rtol=1e-12, atol=1e-11), (nw, np.abs(E - ref).max())
        if pes == "ttm3f":
            assert np.all((it >= 1) & (it <= 500))
    # PES::operator()(nw, crd), the reference's call shape
    assert p(6, z["geoms"][0]) == pytest.approx(float(z["e_" + pes][0]), rel=1e-12)


def _build(scp3, c, precision="fp64", chunk=0):
    sseed = int(c["scramble_seed"])
    return scp3.HBuild(int(c["nw"]), c["x0"], c["MUa"], c["omega"], modes=c["modes"], n2=int(c["n2"]),
                       n3=int(c["n3"]), pes=int(c["pes"]), precision=precision,
                       scramble_seed=None if sseed < 0 else sseed, chunk=chunk)


def _scale(oracle_mod, c):
    sseed = int(c["scramble_seed"])
    normals = oracle_mod.std_normals(c["omega"].size, int(c["index0"]), int(c["nsamples"]),
                                     scramble_seed=None if sseed < 0 else sseed)
    q, v = oracle_mod.samples(int(c["pes"]), int(c["nw"]), c["x0"], c["MUa"], c["omega"], normals)
    A = oracle_mod.accumulate(q[:, c["modes"]], v, int(c["n2"]), int(c["n3"]), absolute=True)
    return normals, q, v, A + np.triu(A, 1).T


@pytest.mark.parametrize("name", hbuild_case_names())
def test_hbuild_fp64_matches_reference(scp3, oracle_mod, name):
    c = load_hbuild_case(name)
    hb = _build(scp3, c)
    hb.accumulate(int(c["index0"]), int(c["nsamples"]))
    M = hb.read(0)
    nb = M.shape[0]
    ref = upper_to_full(c["M_upper"], nb)
    normals, q, v, A = _scale(oracle_mod, c)
    err = np.abs(M - ref)
    assert np.all(err <= 1e-12 * A + 1e-300), (err / np.maximum(A, 1e-300)).max()
    assert np.array_equal(M, M.T)
    rc, nonfinite, notconv = hb.status()
    assert (rc, nonfinite, notconv) == (0, 0, 0)
    assert hb.sample_count() == int(c["nsamples"])


@pytest.mark.parametrize("name", ["dimer_qtip4pf", "hexamer_ttm3f"])
def test_hbuild_normals_path_and_chunking(scp3, oracle_mod, name):
    c = load_hbuild_case(name)
    normals, q, v, A = _scale(oracle_mod, c)
    ns = int(c["nsamples"])
    # the -r path (host normals), fed in two uneven calls
    hb = _build(scp3, c)
    hb.accumulate_normals(normals[: ns // 3])
    hb.accumulate_normals(normals[ns // 3:])
    M = hb.read(0)
    ref = upper_to_full(c["M_upper"], M.shape[0])
    assert np.all(np.abs(M - ref) <= 1e-12 * A + 1e-300)
    # device Sobol in pieces that do not align with the pass size
    hb2 = _build(scp3, c)
    i0 = int(c["index0"])
    for a, b in ((0, 5), (5, 1000), (1000, ns)):
        if a < min(b, ns):
            hb2.accumulate(i0 + a, min(b, ns) - a)
    M2 = hb2.read(0)
    assert np.all(np.abs(M2 - ref) <= 1e-12 * A + 1e-300)



@pytest.mark.parametrize("precision", ["fp64", "bf16x3"])
def test_hbuild_normals_f32_entry(scp3, oracle_mod, precision):
    """scp3gpu_hbuild_accumulate_normals_f32 equals the FP64 entry on the same
    values widened to double, bit for bit, over several chunks."""
    c = load_hbuild_case("hexamer_qtip4pf")
    normals, q, v, A = _scale(oracle_mod, c)
    n32 = np.ascontiguousarray(normals, dtype=np.float32)
    hb = _build(scp3, c, precision=precision, chunk=1 << 12)
    hb.accumulate_normals(n32)
    M32 = hb.read(0)
    hb2 = _build(scp3, c, precision=precision, chunk=1 << 12)
    hb2.accumulate_normals(n32.astype(np.float64))
    M64 = hb2.read(0)
    assert np.array_equal(M32, M64)
    assert hb.sample_count() == normals.shape[0]
    assert hb.status() == (0, 0, 0)
    hb.close(), hb2.close()


def test_add_epot_matches_oracle(scp3, oracle_mod):
    rng = np.random.default_rng(3)
    nm, n2, n3 = 9, 7, 5
    q = rng.normal(scale=np.sqrt(0.5), size=(nm, 777))
    V = rng.normal(scale=1e-3, size=777)
    sme = scp3.ScaledMatrixElements(np.linspace(0.001, 0.02, nm), n2, n3)
    nb = sme.getBasisSize()
    assert nb == oracle_mod.basis_size(nm, n2, n3)
    M = np.zeros((nb, nb), order="F")
    sme.addEpot(q, V, M)
    sme.addEpot(q, V, M)       # adds, as the reference's addEpot does
    ref = oracle_mod.accumulate(np.ascontiguousarray(q.T), V, n2, n3)
    ref = 2 * (ref + np.triu(ref, 1).T)
    A = oracle_mod.accumulate(np.ascontiguousarray(q.T), V, n2, n3, absolute=True)
    A = 2 * (A + np.triu(A, 1).T)
    assert np.all(np.abs(M - ref) <= 1e-12 * A + 1e-300)
    D = np.zeros((nb, nb), order="F")
    sme.addHODiagonal(D)
    R = np.zeros((nb, nb), order="F")
    oracle_mod.add_ho_diagonal(R, sme.omega, n2, n3)
    assert np.array_equal(D, R)


def test_mout_and_eigenvalues(scp3, oracle_mod):
    c = load_hbuild_case("hexamer_qtip4pf_modesel")
    hb = _build(scp3, c)
    ns = int(c["nsamples"])
    hb.accumulate(int(c["index0"]), ns)
    Mout = hb.read(1)
    ref = upper_to_full(c["M_upper"], Mout.shape[0]) / ns
    ref = np.asfortranarray(ref)
    sel = c["modes"]
    zpe = 0.5 * (c["omega"].sum() - c["omega"][sel].sum())
    oracle_mod.add_ho_diagonal(ref, c["omega"][sel], int(c["n2"]), int(c["n3"]), zpe)
    assert np.allclose(Mout, ref, rtol=1e-11, atol=1e-13)
    ev = hb.eigvals(10)
    evr = np.linalg.eigvalsh(ref)[:10]
    assert np.allclose(ev, evr, rtol=1e-12, atol=1e-12)
    n1 = hb.getSubBasisSize(1)
    ev1 = hb.eigvals(1, nsub=n1)
    assert ev1[0] == pytest.approx(np.linalg.eigvalsh(ref[:n1, :n1])[0], rel=1e-12)


def test_bad_arguments_return_status(scp3):
    with pytest.raises(scp3.SCP3GPUError) as e:
        scp3.HBuild(2, np.zeros(18), np.zeros((18, 12)), np.ones(12), n2=13)
    assert e.value.code == 1
    with pytest.raises(ValueError):
        scp3.PES("whbb")
