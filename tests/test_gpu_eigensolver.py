"""The eigensolver tool (eigensolver.cpp) over the library: sM_*.h5 in the
reference's chunked + deflate layout -> lowest eigenpairs on the GPU
(scp3gpu_syevr_lowest, cuSOLVER syevdx) -> eigenpairs*.dat, checked against
LAPACK dsyevr (RANGE = 'I', scipy's OpenBLAS) on the same float32-stored
matrix: eigenvalues to 1e-11 of the spectral radius, eigenvectors to 1e-8 up
to sign."""
import os
import subprocess

import numpy as np
import pytest
import scipy.linalg

from conftest import ROOT, load_hbuild_case

pytestmark = pytest.mark.gpu
EIG = os.path.join(ROOT, "scp3_b200", "eigensolver")


@pytest.fixture(scope="module")
def scp3():
    import torch
    assert torch.cuda.is_available()
    import scp3_b200
    return scp3_b200


def _ref(A, k, lower=False):
    return scipy.linalg.eigh(A, lower=lower, subset_by_index=[0, k - 1], driver="evr")


def _check(W, C, A, k, lower=False):
    w, v = _ref(A, k, lower)
    scale = np.abs(scipy.linalg.eigvalsh(A, lower=lower)).max()
    assert np.abs(W - w).max() <= 1e-11 * scale
    ov = np.abs(np.sum(C * v, axis=0))
    assert np.abs(ov - 1).max() <= 1e-8, ov


def test_cli_matches_dsyevr(scp3, tmp_path):
    from scp3_b200 import h5
    rng = np.random.default_rng(3)
    n, k = 400, 20
    X = rng.normal(size=(n, n))
    A = (X + X.T) / 2 + np.diag(np.arange(n) * 0.05)
    h5.save(str(tmp_path / "sM_0131072.h5"), A, deflate=6)
    r = subprocess.run([EIG, "sM_0131072.h5", str(k)], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lines = (tmp_path / "eigenpairs_0131072.dat").read_text().splitlines()
    assert lines[0] == "# Lowest %d eigenvalues" % k
    W = np.array([float(x) for x in lines[1:1 + k]])
    assert lines[1 + k] == "# Corresponding eigenvectors, one per line."
    C = np.array([[float(x) for x in ln.split()] for ln in lines[2 + k:2 + 2 * k]]).T
    A32 = A.astype(np.float32).astype(np.float64)
    _check(W, C, A32, k)


@pytest.mark.parametrize("tri", ["upper", "lower"])
def test_triangle_rule(scp3, tri):
    """SCP3's M holds the upper triangle only (dsyr2k 'U'); a matrix with
    A[0, n-1] == 0 is read from its lower triangle (eigensolver.cpp:27-30)."""
    rng = np.random.default_rng(4)
    n, k = 128, 10
    X = rng.normal(size=(n, n))
    S = X + X.T
    A = np.triu(S) if tri == "upper" else np.tril(S)
    W, C = scp3.dsyevr(A, k)
    _check(W, C, A, k, lower=(tri == "lower"))


def test_mout_levels_via_h5(scp3, tmp_path):
    """A build's Mout written chunked, read back, solved: the same levels as the
    build's own eigensolve, within the float32 storage of the file."""
    from scp3_b200 import h5
    c = load_hbuild_case("dimer_qtip4pf")
    hb = scp3.HBuild(int(c["nw"]), c["x0"], c["MUa"], c["omega"], modes=c["modes"], n2=int(c["n2"]),
                     n3=int(c["n3"]), scramble_seed=int(c["scramble_seed"]))
    hb.accumulate(0, 8192)
    M = hb.read(1)
    p = str(tmp_path / "sM_0008192.h5")
    h5.save(p, np.triu(M), deflate=6)
    W = scp3.dsyevr(h5.load(p), 10, vectors=False)
    ref = hb.eigvals(10)
    assert np.abs(W - ref).max() <= 1e-6 * np.abs(ref).max()
