"""SCP1 effective-Hessian iteration (scp3_b200.scp1) on CPU: the oracle's sample
loop against the reference's own functions, the driver's host arithmetic
against the oracle's restatement of SCP1.cpp:123-170, the finite-difference
Hessian, the output files and options, and two gloo ranks splitting the points
and all-reducing the sums as SCP1.cpp:71-78 does.  The oracle's sums stand in
for the GPU here (tests/test_gpu_scp1.py checks the GPU against them)."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp



def _dimer():
    """The relaxed qTIP4P/f dimer of the golden fixtures, with the mass-scaled,
    translation/rotation-projected central-difference Hessian of the oracle's
    gradient (the SCP1 start when the input has no Hessian)."""
    from conftest import load_hbuild_case
    from oracle import scp1_oracle
    from scp3_b200 import constants as C
    x0 = np.array(load_hbuild_case("dimer_qtip4pf")["x0"], dtype=np.float64)
    mass = np.tile(np.repeat([C.Omass, C.Hmass, C.Hmass], 3), 2)
    H = scp1_oracle.fd_hessian("qtip4pf", x0, 1e-3)
    H = H / np.sqrt(np.outer(mass, mass))
    H = scp1_oracle.project(scp1_oracle.transrot(list(x0), list(mass)), H)
    return mass, x0, H


def _oracle_averager(pes="qtip4pf", nw=2):
    from oracle import scp1_oracle
    return lambda q, d, U, skip, i0, i1: scp1_oracle.average_sums(pes, nw, q, d, U, skip, i0, i1)


def test_oracle_loop_matches_reference_functions(oracle_mod):
    from oracle import scp1_oracle
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref not built (the reference's sources were absent)")
    mass, x0, H = _dimer()
    w2, U = np.linalg.eigh(H, UPLO="U")
    omega = np.sqrt(np.abs(w2))
    d = np.where(omega < 50 / 2.194746313e5, 0.0, 0.5 / np.maximum(omega, 1e-30))
    iU = U / np.sqrt(mass)[:, None]
    a = scp1_oracle.average_sums("qtip4pf", 2, x0, d, iU, 1 << 7, 3, 67)
    b = scp1_oracle.ref_average_sums("qtip4pf", 2, x0, d, iU, 1 << 7, 3, 67)
    assert abs(a[0] - b[0]) <= 1e-12 * abs(b[0])
    assert np.abs(a[1] - b[1]).max() <= 1e-11 * np.abs(b[1]).max()
    assert np.abs(a[2] - b[2]).max() <= 1e-11 * np.abs(b[2]).max()


def test_driver_iterations_match_oracle_restatement(tmp_path):
    from oracle import scp1_oracle
    from scp3_b200 import scp1
    mass, x0, H = _dimer()
    nsobol = 32
    s = scp1.SCP1(mass, "qtip4pf", nsobol, averager=_oracle_averager(), outdir=str(tmp_path), verbose=False)
    assert s.sobol_skip == 64                       # 1 << (floor(log2 32) + 1), SCP1.h:57
    q = x0.copy()
    F = s(q, 0.0, H.copy(), max_iterations=3)
    s.close()
    # the oracle's own loop from the same start
    qo = x0.copy()
    w2, U = np.linalg.eigh(H, UPLO="U")
    omega = np.sqrt(np.abs(w2))
    d = scp1_oracle.corr(omega, 0.0, 50.0 / 2.194746313e5)
    for it in range(3):
        iU = U / np.sqrt(mass)[:, None]
        up, UX, UXq = scp1_oracle.average_sums("qtip4pf", 2, qo, d, iU, 64, 0, nsobol)
        qo, Ks, U, omega, d, Fo = scp1_oracle.iteration(qo, U, d, mass, up / nsobol, UX / nsobol, UXq / nsobol)
    # the two restatements round differently (matrix products, eigensolver
    # calls); three iterations amplify that to ~1e-10
    assert np.abs(q - qo).max() <= 1e-9 * np.abs(qo).max()
    assert abs(F - Fo) <= 1e-9 * abs(Fo)
    assert np.abs(s.Ks - Ks).max() <= 1e-9 * np.abs(Ks).max()
    # files: one line per iteration, and coord.xyz in the input format
    assert len(open(tmp_path / "omega_scp1.dat").read().splitlines()) == 3
    fe = [float(x) for x in open(tmp_path / "free_energy.dat").read().split()]
    assert len(fe) == 3 and abs(fe[-1] - F) <= 1e-15 * abs(F)
    from scp3_b200 import modes
    species, m2, xq, Hq = modes.read_input(str(tmp_path / "coord.xyz"))
    assert species == ["O", "H", "H"] * 2
    assert np.abs(xq - q).max() <= 1e-14 * np.abs(q).max()
    assert np.abs(Hq - np.triu(s.Ks) - np.triu(s.Ks, 1).T).max() <= 1e-14 * np.abs(s.Ks).max()


def test_initial_hessian_from_gradients():
    """No Hessian in the input: the driver's central differences (one batch of
    2N gradients) equal the reference's column loop (Hessian.cpp:12-43)."""
    import oracle
    from oracle import scp1_oracle
    from scp3_b200 import scp1
    mass, x0, _ = _dimer()

    def batched(crd):
        out = [oracle.qtip4pf_grad(c) for c in np.atleast_2d(crd)]
        return np.array([e for e, _ in out]), np.array([g for _, g in out])

    H1 = scp1.get_hessian(batched, x0, 1e-3)
    H2 = scp1_oracle.fd_hessian("qtip4pf", x0, 1e-3)
    assert np.array_equal(H1, H2)


def test_transrot_projection():
    from oracle import scp1_oracle
    from scp3_b200 import scp1
    mass, x0, H = _dimer()
    U1 = scp1.transrot_basis(x0, mass)
    U2 = scp1_oracle.transrot(list(x0), list(mass))
    assert np.abs(U1 - U2).max() <= 1e-14
    assert np.abs(U1.T @ U1 - np.eye(6)).max() <= 1e-12
    K = H.copy()
    scp1.regtransrot(U1, K)
    assert np.abs(K @ U1).max() <= 1e-10 * np.abs(H).max()


def test_options_and_errors():
    from scp3_b200 import scp1
    a = scp1.parse_args(["-N", "12", "-L", "5", "-c", "30", "-p", "ttm3f", "x.dat"])
    assert (a.NSobol, a.max_iterations, a.cutoff, a.PES, a.input) == (12, 5, 30.0, "ttm3f", "x.dat")
    with pytest.raises(SystemExit):
        scp1.parse_args(["-N", "33", "x.dat"])
    with pytest.raises(SystemExit):
        scp1.parse_args([])


def _rank_worker(rank, world, port, out, tmp):
    import torch.distributed as dist
    from scp3_b200 import scp1
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mass, x0, H = _dimer()
    s = scp1.SCP1(mass, "qtip4pf", 40, averager=_oracle_averager(), outdir=tmp, verbose=False)
    q = x0.copy()
    F = s(q, 0.0, H.copy(), max_iterations=2)
    s.close()
    if rank == 0:
        np.save(out, np.concatenate([[F], q]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_split_points_and_allreduce(tmp_path):
    """Two gloo ranks, each averaging its half of the points (SCP1.cpp:49-50),
    all-reduced: the same iterate as one process over all points."""
    from scp3_b200 import scp1
    out = str(tmp_path / "r.npy")
    port = 29400 + (os.getpid() % 900)
    mp.start_processes(_rank_worker, args=(2, port, out, str(tmp_path / "ranks")), nprocs=2, start_method="spawn",
                       join=True)
    r = np.load(out)
    mass, x0, H = _dimer()
    s = scp1.SCP1(mass, "qtip4pf", 40, averager=_oracle_averager(), outdir=str(tmp_path / "one"), verbose=False)
    q = x0.copy()
    F = s(q, 0.0, H.copy(), max_iterations=2)
    s.close()
    # two partial sums added differ from one sum in the last bits; two
    # iterations amplify that to ~1e-10
    assert abs(r[0] - F) <= 1e-9 * abs(F)
    assert np.abs(r[1:] - q).max() <= 1e-9 * np.abs(q).max()
