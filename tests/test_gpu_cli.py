"""The scp3 command line on the GPU: SCP3_a's periodic readout (SCP3.cpp:234-263)
against the reference's own build on the same points.

`scp3 -G -N 17 -m 0-7 -2 6 -3 3` on the hexamer prism input samples 2^17
unscrambled Sobol points from the default skip 2^30 in blocks of 1024.  Every
2^14 samples it writes a row of E0_sd.dat (n, lowest level of the singles and
of the doubles sub-block of Mout = M/n + HO diagonal + inactive-mode ZPE, their
difference, cm^-1); at 2^17 it writes sM_0131072.h5 (Mout as float32, upper
triangle, chunked + deflate).  The reference side is oracle/_ref's ref_hbuild
(the reference's potential and Hermite functions, dsyr2k 'U') over the same
normals, with the modes the run wrote (--write-modes), read out the same way."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
CLI = os.path.join(ROOT, "scp3_b200", "scp3")
AUTOCM = 2.194746313e5


def test_cli_readout_loop_matches_reference(tmp_path):
    import torch
    import oracle
    from scp3_b200 import h5
    assert torch.cuda.is_available()
    if not oracle.ref_available():
        pytest.fail("oracle/_ref (the reference built from its sources) is missing")
    inp = os.path.join(ROOT, "scp3_b200", "data", "prism_qtip4pf.dat")
    r = subprocess.run([CLI, "-G", "-N", "17", "-m", "0-7", "-2", "6", "-3", "3", "--write-modes", "modes.txt", inp],
                       cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    rows = np.loadtxt(tmp_path / "E0_sd.dat")
    assert rows.shape == (8, 4)
    assert np.array_equal(rows[:, 0], (np.arange(8) + 1) * (1 << 14))
    assert sorted(os.listdir(tmp_path)) == ["E0_sd.dat", "modes.txt", "omega0.dat", "sM_0131072.h5"]

    with open(tmp_path / "modes.txt") as f:
        x0 = np.array(f.readline().split(), dtype=np.float64)
        tab = np.array([line.split() for line in f], dtype=np.float64)
    omega, MUa = tab[:, 0], np.asfortranarray(tab[:, 1:].T)
    nw, nm0 = x0.size // 9, omega.size
    modes = np.arange(8, dtype=np.int32)
    n2, n3 = 6, 3
    nb = oracle.basis_size(8, n2, n3)
    n1, n2s = 1 + 8, 1 + 8 + n2 * (n2 + 1) // 2
    zpe = 0.5 * (omega.sum() - omega[modes].sum())

    normals = oracle.std_normals(nm0, 1 << 30, 1 << 17)          # the reference's stream from 2^30
    M = None
    for k in range(8):
        M, _, _ = oracle.ref_hbuild(0, nw, x0, MUa, omega, modes, n2, n3, 1 << 14, 1024,
                                    normals=normals[k << 14:(k + 1) << 14], M=M)
        n = (k + 1) << 14
        Mout = np.asfortranarray(np.triu(M) / n)
        oracle.add_ho_diagonal(Mout, omega[modes], n2, n3, zpe)
        e1 = np.linalg.eigvalsh(Mout[:n1, :n1], UPLO="U")[0] * AUTOCM
        e2 = np.linalg.eigvalsh(Mout[:n2s, :n2s], UPLO="U")[0] * AUTOCM
        # E0_sd.dat prints 10 decimals of cm^-1; FP64 parity is ~1e-12 relative
        assert abs(rows[k, 1] - e1) <= 1e-6, (k, rows[k, 1], e1)
        assert abs(rows[k, 2] - e2) <= 1e-6, (k, rows[k, 2], e2)
        assert abs(rows[k, 3] - (rows[k, 2] - rows[k, 1])) <= 1e-9

    D = h5.load(tmp_path / "sM_0131072.h5")
    assert D.shape == (nb, nb)
    ref32 = Mout.astype(np.float32).astype(np.float64)
    assert np.all(np.tril(D, -1) == 0.0)                           # upper triangle, as the reference's file
    ulp = np.abs(np.spacing(Mout.astype(np.float32))).astype(np.float64)
    assert np.all(np.abs(D - ref32) <= ulp), np.abs(D - ref32).max()


def test_cli_default_estimator_split_form_matches_fp64(tmp_path):
    """scp3 without -G runs the reference's default (gradient) estimator; with
    --precision bf16x3 its products run on the tensor cores.  Its periodic
    readout (E0_sd.dat, SCP3.cpp:234-250) matches the FP64 form's on the same
    points within 0.1 cm^-1."""
    import torch
    assert torch.cuda.is_available()
    inp = os.path.join(ROOT, "scp3_b200", "data", "prism_qtip4pf.dat")
    rows = {}
    for prec in ("fp64", "bf16x3"):
        d = tmp_path / prec
        d.mkdir()
        r = subprocess.run([CLI, "-N", "15", "-m", "0-7", "-2", "6", "-3", "3", "--precision", prec, inp],
                           cwd=d, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        rows[prec] = np.loadtxt(d / "E0_sd.dat")
    assert rows["fp64"].shape == (2, 4)
    assert np.array_equal(rows["fp64"][:, 0], rows["bf16x3"][:, 0])
    err = np.abs(rows["fp64"][:, 1:3] - rows["bf16x3"][:, 1:3]).max()
    print("\nCLI gradient estimator, bf16x3 vs fp64 E0_sd levels: max %.4f cm^-1" % err)
    assert err <= 0.1, err
