"""GPU parity of the gradient (default) path: the qTIP4P/f and TTM3-F gradients
in the per-sample kernel, dV/dq = MUa^T dV/dr - omega q (SCP3.cpp:209-216),
and the Stein estimator of every upper element (ScaledMatrixElements.cpp:102-725,
TripleExcitations.h) in FP64.

Against the reference: the dimer matrices of tests/golden/stein_ref.npz (N2 =
12, N3 = 4, 256 scrambled points, both potentials), summed from the
reference's own formulas with the reference's potential gradients, to 1e-11 of
the largest element; the gradients themselves on the pes_ref geometries.
Against the oracle: addEpot(q, V, Vq) on hexamer bases with N3 = 6.

The split form (BF16x3 products W Phi^T on the tensor cores, the same-mode pair
sums and the potential in FP64): against the oracle on that basis, every upper
element within 2e-5 of the largest; on the hexamer doubles basis (N2 = 48,
Nb = 1225) from device Sobol points, against the FP64 form on the same points,
elements within 2e-5 of the largest and the 10 lowest levels within 0.1 cm^-1."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scp3():
    import torch
    assert torch.cuda.is_available()
    import scp3_b200
    return scp3_b200


@pytest.fixture(scope="module")
def z():
    return np.load(os.path.join(GOLDEN, "stein_ref.npz"), allow_pickle=True)


@pytest.mark.parametrize("tag,pes", [("dimer", "qtip4pf"), ("dimer_ttm3f", "ttm3f")])
def test_dimer_gradient_build_matches_reference(scp3, z, tag, pes):
    n2, n3, ns = int(z[tag + "_n2"]), int(z[tag + "_n3"]), int(z[tag + "_nsamples"])
    hb = scp3.HBuild(2, z[tag + "_x0"], z[tag + "_MUa"], z[tag + "_omega"], n2=n2, n3=n3, pes=pes,
                     scramble_seed=int(z[tag + "_scramble_seed"]), estimator="gradient")
    hb.accumulate(0, ns)
    M = hb.read(0)
    assert hb.status()[0] == 0
    got = M.T[np.tril_indices(M.shape[0])]        # upper triangle column by column
    ref = z[tag + "_M_upper"]
    assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max(), np.abs(got - ref).max() / np.abs(ref).max()
    # Mout adds the same HO diagonal as the direct path
    d = scp3.HBuild(2, z[tag + "_x0"], z[tag + "_MUa"], z[tag + "_omega"], n2=n2, n3=n3, pes=pes,
                    scramble_seed=int(z[tag + "_scramble_seed"]))
    d.accumulate(0, ns)
    diag_g = np.diag(hb.read(1)) - np.diag(M) / ns
    diag_d = np.diag(d.read(1)) - np.diag(d.read(0)) / ns
    assert np.allclose(diag_g, diag_d, rtol=0, atol=1e-12)


@pytest.mark.parametrize("tag,pes", [("dimer", "qtip4pf"), ("dimer_ttm3f", "ttm3f")])
def test_dimer_split_gradient_build_matches_reference(scp3, z, tag, pes):
    """The BF16x3 form of the gradient build (device Sobol, the potential's FP64
    gradient, products and pair sums on the tensor cores) against the same
    reference matrices: every upper element within 2e-5 of the largest."""
    n2, n3, ns = int(z[tag + "_n2"]), int(z[tag + "_n3"]), int(z[tag + "_nsamples"])
    hb = scp3.HBuild(2, z[tag + "_x0"], z[tag + "_MUa"], z[tag + "_omega"], n2=n2, n3=n3, pes=pes,
                     scramble_seed=int(z[tag + "_scramble_seed"]), estimator="gradient", precision="bf16x3")
    hb.accumulate(0, ns)
    M = hb.read(0)
    assert hb.status()[0] == 0
    got = M.T[np.tril_indices(M.shape[0])]
    ref = z[tag + "_M_upper"]
    err = np.abs(got - ref) / np.abs(ref).max()
    print("\nsplit gradient, %s: max %.2e median %.2e of max|M|" % (tag, err.max(), np.median(err)))
    assert err.max() <= 2e-5, err.max()


def test_add_epot_grad_matches_oracle(scp3, oracle_mod):
    c = np.load(os.path.join(GOLDEN, "hbuild_ref.npz"))
    omega = c["hexamer_qtip4pf__omega"]
    rng = np.random.default_rng(8)
    n, nm, n2, n3 = 300, 48, 10, 6
    q = rng.normal(scale=np.sqrt(0.5), size=(n, nm))
    V = rng.normal(scale=1e-3, size=n)
    Vq = rng.normal(scale=1e-3, size=(n, nm))
    hb = scp3.HBuild(6, c["hexamer_qtip4pf__x0"], c["hexamer_qtip4pf__MUa"], omega, n2=n2, n3=n3,
                     estimator="gradient")
    hb.add_epot_grad(q, V, Vq)
    M = hb.read(0)
    ref = oracle_mod.accumulate_stein(q, V, Vq, n2, n3)
    iu = np.triu_indices(M.shape[0])
    assert np.abs(M[iu] - ref[iu]).max() <= 1e-12 * np.abs(ref).max()
    assert hb.sample_count() == n


def test_gradient_estimator_limits(scp3, z):
    with pytest.raises(scp3.SCP3GPUError):
        scp3.HBuild(2, z["dimer_x0"], z["dimer_MUa"], z["dimer_omega"], estimator="gradient", precision="f16x3")
    d = scp3.HBuild(2, z["dimer_x0"], z["dimer_MUa"], z["dimer_omega"])
    with pytest.raises(scp3.SCP3GPUError):
        d.add_epot_grad(np.zeros((4, 12)), np.zeros(4), np.zeros((4, 12)))


@pytest.mark.parametrize("pes,ekey,gkey", [("qtip4pf", "e_qtip4pf", "pes_geoms_grad"),
                                           ("ttm3f", "e_ttm3f", "pes_geoms_grad_ttm3f")])
def test_pes_energy_grad_matches_reference(scp3, z, pes, ekey, gkey):
    """h2o::PES::operator()(nw, crd, grad) on the GPU against the reference's
    gradients (qtip4pf.cpp:252-397, ttm3f.cpp:325-720) on the pes_ref geometries."""
    p = np.load(os.path.join(GOLDEN, "pes_ref.npz"), allow_pickle=True)
    P = scp3.PES(pes)
    for x, e_ref, g_ref in zip(p["geoms"], p[ekey], z[gkey]):
        x = np.asarray(x, dtype=np.float64)
        E, G = P.energies_grad(x[None, :])
        assert abs(E[0] - e_ref) <= 1e-11 * max(1.0, abs(e_ref)), (E[0], e_ref)
        assert np.abs(G[0] - g_ref).max() <= 1e-10 * max(1.0, np.abs(g_ref).max()), np.abs(G[0] - g_ref).max()


def test_split_gradient_add_epot_grad_matches_oracle(scp3, oracle_mod):
    """BF16x3 products on tcgen05 against the oracle's addEpot(q, V, Vq) on a
    315-function basis (N2 = 20, N3 = 6: three Phi panels, so a two-panel and a
    one-panel tile per W panel): a ragged pass (5000 samples: one whole
    4096-sample block and a partial one), then a short second call after
    reset() on the same handle."""
    c = np.load(os.path.join(GOLDEN, "hbuild_ref.npz"))
    omega = c["hexamer_qtip4pf__omega"]
    rng = np.random.default_rng(21)
    nm, n2, n3 = 48, 20, 6
    hb = scp3.HBuild(6, c["hexamer_qtip4pf__x0"], c["hexamer_qtip4pf__MUa"], omega, n2=n2, n3=n3,
                     estimator="gradient", precision="bf16x3")
    for call, n in enumerate((5000, 300)):
        q = rng.normal(scale=np.sqrt(0.5), size=(n, nm))
        V = -0.077 + rng.normal(scale=2e-3, size=n)          # V_anh carries the binding energy
        Vq = rng.normal(scale=2e-3, size=(n, nm))
        hb.reset()
        hb.add_epot_grad(q, V, Vq)
        M = hb.read(0)
        assert hb.status()[0] == 0
        ref = oracle_mod.accumulate_stein(q, V, Vq, n2, n3)
        iu = np.triu_indices(M.shape[0])
        err = np.abs(M[iu] - ref[iu]) / np.abs(ref).max()
        print("\nsplit gradient, call %d, %d samples: max %.2e median %.2e of max|M|" % (call, n, err.max(),
                                                                                      np.median(err)))
        assert err.max() <= 2e-5 and np.median(err) <= 1e-6, (call, err.max(), np.median(err))
        assert hb.sample_count() == n


def test_split_gradient_build_hexamer_doubles(scp3):
    """The hexamer prism's doubles basis (N2 = 48, Nb = 1225: 2353 virtual rows
    against 1225 functions, 19 x 5 tiles of 128 x 256), 2^15 scrambled device
    Sobol points, qTIP4P/f: the BF16x3 build against the FP64 build on the same
    points."""
    from scp3_b200 import inputs
    nw, x0, MUa, omega = inputs.load("prism_qtip4pf", build_if_missing=False)
    n = 1 << 15
    builds = {}
    for prec in ("fp64", "bf16x3"):
        hb = scp3.HBuild(nw, x0, MUa, omega, n2=48, n3=0, pes="qtip4pf", precision=prec, scramble_seed=0x5C3,
                         estimator="gradient")
        hb.accumulate(0, n)
        builds[prec] = (hb.read(0), np.sort(np.linalg.eigvalsh(hb.read(1)))[:10] * 2.194746313e5)
        assert hb.status()[0] == 0
        hb.close()
    (M64, l64), (Ms, ls) = builds["fp64"], builds["bf16x3"]
    iu = np.triu_indices(M64.shape[0])
    err = np.abs(Ms[iu] - M64[iu]) / np.abs(M64).max()
    dl = np.abs(ls - l64).max()
    print("\nsplit gradient, hexamer doubles, 2^15 points: elements max %.2e median %.2e of max|M|; "
          "levels max %.4f cm^-1 (lowest %.1f)" % (err.max(), np.median(err), dl, l64[0]))
    assert err.max() <= 2e-5 and np.median(err) <= 1e-6, (err.max(), np.median(err))
    assert dl <= 0.1, dl
