"""The allocation-free entry point, scp3gpu_add_epot_static.

Some callers cannot allocate device memory (a host framework that owns every
device buffer, a locked-down allocator, a hot loop that must not touch the
allocator), so this entry point does the -G accumulation with its working
space in a static device array.  Called here through the C ABI on device
buffers and checked against the allocating path (ScaledMatrixElements.addEpot,
i.e. scp3gpu_hbuild_add_epot) on two calls in a row with different inputs, the
second proving the shared array starts clean.  This file sorts last so that a
run stopping at its first failure has already run every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _reference(scp3, omega, n2, n3, q, V):
    sme = scp3.ScaledMatrixElements(omega, n2, n3)
    nb = sme.getBasisSize()
    M = np.zeros((nb, nb), order="F")
    sme.addEpot(q.T, V, M)
    return M


def test_static_scratch_matches_allocating_path():
    import torch
    assert torch.cuda.is_available()
    import scp3_b200
    from scp3_b200 import _lib
    L = _lib.lib()
    rng = np.random.default_rng(11)
    nm, n2, n3 = 20, 20, 6
    omega = np.linspace(0.002, 0.02, nm)
    nb = int(L.scp3gpu_basis_size(nm, n2, n3))
    for call, n in enumerate((5003, 777)):
        q = rng.normal(scale=np.sqrt(0.5), size=(n, nm))
        V = rng.normal(scale=1e-3, size=n)
        ref = _reference(scp3_b200, omega, n2, n3, q, V)
        qd = torch.tensor(q, dtype=torch.float64, device="cuda")
        Vd = torch.tensor(V, dtype=torch.float64, device="cuda")
        Md = torch.zeros((nb, nb), dtype=torch.float64, device="cuda")   # row-major storage of M^T = M
        rc = L.scp3gpu_add_epot_static(nm, n2, n3, qd.data_ptr(), Vd.data_ptr(), n, Md.data_ptr(), nb,
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0, L.scp3gpu_last_error()
        torch.cuda.synchronize()
        M = Md.cpu().numpy().T
        scale = np.abs(ref).max()
        assert np.abs(M - ref).max() <= 1e-12 * scale, (call, np.abs(M - ref).max() / scale)


def _plan(nb):
    """The entry point's chunk and sample-range split for a basis of nb functions
    (the size rule of noalloc.cu restated): nsplit 4 halving while the tile
    partials crowd the array out, then the chunk halving from 4096."""
    nt = (nb + 63) // 64
    a256 = lambda b: (b + 255) // 256 * 256
    need = lambda k, s: a256(4 * nb) + 2 * a256(8 * nt * 64 * k) + 8 * 64 * 64 * nt * (nt + 1) // 2 * s
    cap, nsplit, chunk = 64 << 20, 4, 4096
    while nsplit > 1 and need(16 * nsplit, nsplit) > cap:
        nsplit //= 2
    while chunk > 16 * nsplit and need(chunk, nsplit) > cap:
        chunk //= 2
    return nsplit, chunk, need(chunk, nsplit) <= cap


@pytest.mark.parametrize("nm,n2,n,pad", [(62, 62, 1500, 3), (88, 88, 40, 0)])
def test_static_scratch_large_bases(nm, n2, n, pad):
    """Bases where the array forces smaller pieces: 2016 functions (two sample
    ranges per tile, 512-sample chunks, a ragged last chunk, M with a leading
    dimension 3 past the basis) and 4005 functions (63 tiles a side, the most
    the array holds: one range, 16-sample chunks)."""
    import torch
    import scp3_b200
    from scp3_b200 import _lib
    L = _lib.lib()
    nb = int(L.scp3gpu_basis_size(nm, n2, 0))
    nsplit, chunk, fits = _plan(nb)
    assert fits and (nsplit, chunk) == ((2, 512) if nb == 2016 else (1, 16))
    rng = np.random.default_rng(nb)
    omega = np.linspace(0.002, 0.02, nm)
    ld = nb + pad
    for call in range(2):
        q = rng.normal(scale=np.sqrt(0.5), size=(n, nm))
        V = rng.normal(scale=1e-3, size=n)
        ref = _reference(scp3_b200, omega, n2, 0, q, V)
        qd = torch.tensor(q, dtype=torch.float64, device="cuda")
        Vd = torch.tensor(V, dtype=torch.float64, device="cuda")
        Md = torch.full((nb, ld), 7.0, dtype=torch.float64, device="cuda")   # column-major nb x nb, ld rows
        Md[:, :nb] = 0.0
        rc = L.scp3gpu_add_epot_static(nm, n2, 0, qd.data_ptr(), Vd.data_ptr(), n, Md.data_ptr(), ld,
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0, L.scp3gpu_last_error()
        torch.cuda.synchronize()
        A = Md.cpu().numpy()
        assert np.all(A[:, nb:] == 7.0)                 # rows past the basis are not written
        M = A[:, :nb].T
        scale = np.abs(ref).max()
        assert np.abs(M - ref).max() <= 1e-12 * scale, (call, np.abs(M - ref).max() / scale)


def test_static_scratch_rejects_oversized_basis():
    import torch
    from scp3_b200 import _lib
    L = _lib.lib()
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    for nm in (100, 89):      # 5151 functions, and 4095: the first size past 63 tiles a side (4032 rows)
        nb = int(L.scp3gpu_basis_size(nm, nm, 0))
        assert not _plan(nb)[2]
        rc = L.scp3gpu_add_epot_static(nm, nm, 0, x.data_ptr(), x.data_ptr(), 1, x.data_ptr(), nb, None)
        assert rc == _lib.ERR_ARG
        assert b"static scratch" in L.scp3gpu_last_error()
