"""The scp3 command-line host (scp3_b200/csrc/scp3_main.cpp, SCP3.cpp's options
over the C ABI): its input reader, O H H reorder and normal-mode setup run on
the host, so omega0.dat (SCP3.cpp:300-302) is checked here without a GPU."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

CLI = os.path.join(ROOT, "scp3_b200", "scp3")


@pytest.fixture(scope="module")
def cli():
    if not os.path.exists(CLI):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "scp3_b200", "csrc")], check=True)
    return CLI


def test_omega0_matches_numpy_modes(cli, tmp_path):
    import torch
    from scp3_b200 import constants as C, modes
    inp = os.path.join(ROOT, "scp3_b200", "data", "prism_qtip4pf.dat")
    r = subprocess.run([cli, "-G", "-N", "14", inp], cwd=tmp_path, capture_output=True, text=True)
    if not torch.cuda.is_available():
        assert r.returncode == 1 and "no CUDA device" in r.stderr
    w = np.loadtxt(tmp_path / "omega0.dat")
    sp, mass, x0, H = modes.read_input(inp)
    _, mass, x0, H = modes.ohhohh(mass, x0, H)
    ref = np.sqrt(np.abs(np.linalg.eigvalsh(H))) * C.autocm
    assert w.shape == ref.shape
    assert np.allclose(w[6:], ref[6:], rtol=1e-5)


def test_cli_gradient_path_limits_and_bad_options(cli, tmp_path):
    """Without -G the gradient estimator runs (products in FP64 or BF16x3); the
    FP16 form is told to use -G."""
    inp = os.path.join(ROOT, "scp3_b200", "data", "prism_qtip4pf.dat")
    r = subprocess.run([cli, "--precision", "f16x3", inp], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1 and "-G" in r.stderr
    r = subprocess.run([cli, "-G", "-N", "50", inp], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1 and "too large" in r.stderr
    r = subprocess.run([cli, "-G"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1 and "No input file" in r.stderr


def test_eigensolver_cli_arguments(cli, tmp_path):
    """eigensolver (eigensolver.cpp over the library): usage and file errors are
    reported before any GPU work."""
    eig = os.path.join(ROOT, "scp3_b200", "eigensolver")
    r = subprocess.run([eig], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1 and "usage" in r.stderr
    r = subprocess.run([eig, "sM_missing.h5", "5"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1 and "cannot open" in r.stderr
    from scp3_b200 import h5
    h5.save(str(tmp_path / "sM_0000001.h5"), np.eye(4), deflate=6)
    r = subprocess.run([eig, "sM_0000001.h5", "9"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1 and "n_eigenpairs" in r.stderr
