"""GPU tests of the SCP1 averages (scp3gpu_scp1_average) and the SCP1 driver
on the GPU, against the oracle (oracle/scp1_oracle.py): the sums of V, UX and
UX dq^T over the same Sobol points, chunked or not, for both potentials; the
central-difference Hessian from the GPU gradients; and two driver iterations."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scp3():
    import torch
    assert torch.cuda.is_available()
    import scp3_b200
    return scp3_b200


def _start(name):
    from conftest import load_hbuild_case
    from oracle import scp1_oracle
    from scp3_b200 import constants as C
    c = load_hbuild_case(name)
    x0 = np.array(c["x0"], dtype=np.float64)
    nw = x0.size // 9
    mass = np.tile(np.repeat([C.Omass, C.Hmass, C.Hmass], 3), nw)
    pes = "ttm3f" if name.endswith("ttm3f") else "qtip4pf"
    if pes == "qtip4pf":
        H = scp1_oracle.fd_hessian(pes, x0, 1e-3)
    else:
        from scp3_b200 import scp1
        H = scp1.get_hessian(__import__("scp3_b200").PES(pes).energies_grad, x0, 1e-3)
    H = H / np.sqrt(np.outer(mass, mass))
    H = scp1_oracle.project(scp1_oracle.transrot(list(x0), list(mass)), H)
    w2, U = np.linalg.eigh(H, UPLO="U")
    omega = np.sqrt(np.abs(w2))
    d = scp1_oracle.corr(omega, 0.0, 50.0 / 2.194746313e5)
    return pes, nw, mass, x0, H, d, U / np.sqrt(mass)[:, None]


def _close(a, b, tv, tm):
    assert abs(a[0] - b[0]) <= tv * abs(b[0]), (a[0], b[0])
    assert np.abs(a[1] - b[1]).max() <= tm * np.abs(b[1]).max()
    assert np.abs(a[2] - b[2]).max() <= tm * np.abs(b[2]).max()


@pytest.mark.parametrize("name", ["dimer_qtip4pf", "hexamer_qtip4pf"])
def test_average_matches_oracle(scp3, name):
    from oracle import scp1_oracle
    pes, nw, mass, x0, H, d, iU = _start(name)
    n = 2000 if nw == 2 else 400
    g = scp3.SCP1Average(pes, nw)
    a = g.sums(x0, d, iU, 1 << 11, 5, 5 + n)
    b = scp1_oracle.average_sums(pes, nw, x0, d, iU, 1 << 11, 5, 5 + n)
    _close(a, b, 1e-12, 1e-10)
    # several device passes (chunk 96) give the same sums
    g2 = scp3.SCP1Average(pes, nw, chunk=96)
    c = g2.sums(x0, d, iU, 1 << 11, 5, 5 + n)
    _close(c, a, 1e-13, 1e-12)
    g.close(), g2.close()


def test_average_ttm3f_matches_reference_functions(scp3, oracle_mod):
    from oracle import scp1_oracle
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref not built (the reference's sources were absent)")
    pes, nw, mass, x0, H, d, iU = _start("dimer_ttm3f")
    g = scp3.SCP1Average(pes, nw)
    a = g.sums(x0, d, iU, 1 << 9, 0, 256)
    b = scp1_oracle.ref_average_sums(pes, nw, x0, d, iU, 1 << 9, 0, 256)
    _close(a, b, 1e-10, 1e-8)
    assert g.not_converged() == 0
    g.close()


def test_hessian_from_gpu_gradients(scp3):
    from oracle import scp1_oracle
    from scp3_b200 import scp1
    _, nw, mass, x0, H, d, iU = _start("dimer_qtip4pf")
    H1 = scp1.get_hessian(scp3.PES("qtip4pf").energies_grad, x0, 1e-3)
    H2 = scp1_oracle.fd_hessian("qtip4pf", x0, 1e-3)
    # gradients agree to ~1e-12 relative; the difference quotient divides by 2e-3
    assert np.abs(H1 - H2).max() <= 1e-8 * np.abs(H2).max()


def test_driver_on_gpu_matches_oracle_averages(scp3, tmp_path):
    from scp3_b200 import scp1
    from oracle import scp1_oracle
    pes, nw, mass, x0, H, d, iU = _start("dimer_qtip4pf")
    runs = []
    for av in (None, lambda q, dd, U, skip, i0, i1: scp1_oracle.average_sums(pes, nw, q, dd, U, skip, i0, i1)):
        s = scp1.SCP1(mass, pes, 1 << 10, averager=av, outdir=str(tmp_path / str(len(runs))), verbose=False)
        q = x0.copy()
        F = s(q, 0.0, H.copy(), max_iterations=2)
        runs.append((F, q, s.Ks))
        s.close()
    (F1, q1, K1), (F2, q2, K2) = runs
    assert abs(F1 - F2) <= 1e-9 * abs(F2)
    assert np.abs(q1 - q2).max() <= 1e-9 * np.abs(q2).max()
    assert np.abs(K1 - K2).max() <= 1e-8 * np.abs(K2).max()


def test_average_rejects(scp3):
    with pytest.raises(scp3.SCP3GPUError):
        scp3.SCP1Average("qtip4pf", 9)
    g = scp3.SCP1Average("qtip4pf", 2)
    with pytest.raises(scp3.SCP3GPUError):
        g.sums(np.zeros(18), -np.ones(18), np.eye(18), 0, 0, 4)
    with pytest.raises(scp3.SCP3GPUError):
        g.sums(np.zeros(18), np.ones(18), np.eye(18), 0, 5, 4)
    g.close()
