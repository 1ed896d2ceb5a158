"""CPU-side checks of the product: the C-ABI library loads and exports every
symbol include/scp3gpu.h declares, its host-only entry points, and the host
setup code (input reader, O H H reorder, normal modes)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "scp3gpu.h")).read()
    return sorted(set(re.findall(r"\b(scp3gpu_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    from scp3_b200 import _lib
    L = _lib.lib()
    decl = declared_symbols()
    assert decl, "no declarations found"
    for name in decl:
        assert hasattr(L, name), name
    assert sorted(_lib.EXPORTS) == decl


def test_basis_sizes_through_abi():
    from scp3_b200 import _lib, modes
    L = _lib.lib()
    for nm, n2, n3, nb in ((12, 12, 0, 91), (48, 48, 0, 1225), (48, 48, 48, 20825)):
        assert L.scp3gpu_basis_size(nm, n2, n3) == nb == modes.basis_size(nm, n2, n3)
        for level in range(4):
            assert L.scp3gpu_sub_basis_size(nm, n2, n3, level) == modes.sub_basis_size(nm, n2, n3, level)
    assert L.scp3gpu_basis_size(4, 5, 0) == -1


def test_no_device_is_an_error_status_not_a_crash():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from scp3_b200 import _lib
    out = np.zeros(12)
    rc = _lib.lib().scp3gpu_sobol_std_normal(12, 0, 1, 0, 0, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == _lib.ERR_UNSUPPORTED


def test_input_roundtrip_and_modes(tmp_path):
    from scp3_b200 import clusters, constants as C, modes
    import oracle
    def en(X):
        return np.array([oracle.qtip4pf(x) for x in np.atleast_2d(X)])
    x, e, g, it = clusters.relax(en, clusters.dimer(), maxiter=300)
    mass = np.tile(np.repeat([C.Omass, C.Hmass, C.Hmass], 3), 2)
    H, x0 = clusters.hessian(en, x, mass)
    # write H-first order to exercise the O H H reorder
    orig = ["O", "H", "H", "O", "H", "H"]
    perm = [1, 0, 2, 4, 3, 5]             # file order: H O H H O H
    p3 = np.concatenate([[3 * a, 3 * a + 1, 3 * a + 2] for a in perm])
    path = str(tmp_path / "d.dat")
    modes.write_input(path, [orig[a] for a in perm], x0[p3], H[np.ix_(p3, p3)])
    sp, m2, x2, H2 = modes.read_input(path)
    _, m3, x3, H3 = modes.ohhohh(m2, x2, H2)
    assert np.allclose(x3, x0, atol=1e-14) and np.allclose(H3, H, atol=1e-14)
    omega, MUa, w2 = modes.normal_modes(H3, m3)
    assert omega.size == 12 and np.all(omega > 0)
    assert np.all(np.abs(w2[:6]) < 1e-10)
    # mass-weighted orthonormality: MUa^T M MUa = diag(1/omega)
    G = MUa.T @ (m3[:, None] * MUa)
    assert np.allclose(G, np.diag(1 / omega), rtol=1e-10)
    assert list(modes.parse_modes("0-3,7,9-10")) == [0, 1, 2, 3, 7, 9, 10]


def test_argument_errors_before_any_device_work():
    """Entry points reject bad shapes and options with SCP3GPU_ERR_ARG (or
    UNSUPPORTED for a form that is not built) before they touch a device, so the
    checks run here without a GPU."""
    from scp3_b200 import _lib, api
    L = _lib.lib()
    dp = ctypes.POINTER(ctypes.c_double)
    # batch: FP64 is not a batched form; chunk must be whole 4096-sample blocks
    class K:
        pass
    k = K()
    x0 = np.zeros(18)
    api._fill_config(k, 2, x0, np.zeros((18, 12)), np.ones(12), None, 12, 0, "qtip4pf", "fp64", None, 0, 0)
    arr = (_lib.Config * 1)(k._cfg)
    h = ctypes.c_void_p()
    assert L.scp3gpu_batch_create(arr, 1, 0, 0, ctypes.byref(h)) == _lib.ERR_UNSUPPORTED
    k._cfg.precision = _lib.PREC_BF16X3
    arr = (_lib.Config * 1)(k._cfg)
    assert L.scp3gpu_batch_create(arr, 1, 1000, 0, ctypes.byref(h)) == _lib.ERR_ARG
    assert L.scp3gpu_batch_create(arr, 0, 0, 0, ctypes.byref(h)) == _lib.ERR_ARG
    # a build: unknown estimator; gradient estimator in a split precision
    k._cfg.estimator = 7
    assert L.scp3gpu_hbuild_create(ctypes.byref(k._cfg), ctypes.byref(h)) == _lib.ERR_ARG
    k._cfg.estimator = _lib.ESTIMATOR_GRADIENT
    assert L.scp3gpu_hbuild_create(ctypes.byref(k._cfg), ctypes.byref(h)) == _lib.ERR_UNSUPPORTED
    # eigenpairs: k out of range, null matrix
    A = np.eye(4)
    W = np.zeros(4)
    assert L.scp3gpu_syevr_lowest(A.ctypes.data_as(dp), 4, 4, 5, W.ctypes.data_as(dp), None, 4, 0) == _lib.ERR_ARG
    assert L.scp3gpu_syevr_lowest(None, 4, 4, 2, W.ctypes.data_as(dp), None, 4, 0) == _lib.ERR_ARG
    # energies and gradients: unknown potential, too many waters for TTM3-F
    E = np.zeros(1)
    G = np.zeros(9 * 9)
    crd = np.zeros(9 * 9)
    assert L.scp3gpu_pes_energy_grad(5, 9, 1, crd.ctypes.data_as(dp), E.ctypes.data_as(dp),
                                     G.ctypes.data_as(dp)) == _lib.ERR_ARG
    assert L.scp3gpu_pes_energy_grad(1, 9, 1, crd.ctypes.data_as(dp), E.ctypes.data_as(dp),
                                     G.ctypes.data_as(dp)) == _lib.ERR_ARG
    assert "TTM3-F" in L.scp3gpu_last_error().decode()
    # the -r path's two entries: no handle, negative count, no buffer
    fp = ctypes.POINTER(ctypes.c_float)
    n32 = np.zeros(48, dtype=np.float32)
    assert L.scp3gpu_hbuild_accumulate_normals(None, x0.ctypes.data_as(dp), 1) == _lib.ERR_ARG
    assert L.scp3gpu_hbuild_accumulate_normals_f32(None, n32.ctypes.data_as(fp), 1) == _lib.ERR_ARG
    assert L.scp3gpu_hbuild_accumulate_normals_f32(None, None, -1) == _lib.ERR_ARG
    assert "accumulate_normals_f32" in L.scp3gpu_last_error().decode()


def test_mlp_shape_limits_without_device():
    """The surrogate's forward layers run on the tensor cores with N = hidden and
    K = padded inputs, both at most 256: larger shapes are refused at creation."""
    from scp3_b200 import _lib
    L = _lib.lib()
    h = ctypes.c_void_p()
    for n_in, hidden in ((300, 256), (48, 320), (48, 96), (0, 256)):
        assert L.scp3gpu_mlp_create(n_in, hidden, 4096, 1, 0, ctypes.byref(h)) == _lib.ERR_ARG
    assert b"hidden 64, 128, 192 or 256" in L.scp3gpu_last_error()


def test_scp1_argument_errors_without_device():
    from scp3_b200 import _lib
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.scp3gpu_scp1_create(5, 2, 0, 0, ctypes.byref(h)) == _lib.ERR_ARG
    assert L.scp3gpu_scp1_create(0, 9, 0, 0, ctypes.byref(h)) == _lib.ERR_ARG
    assert L.scp3gpu_scp1_create(0, 2, -1, 0, ctypes.byref(h)) == _lib.ERR_ARG
    assert L.scp3gpu_scp1_create(0, 2, 0, 0, None) == _lib.ERR_ARG
    # a valid request on a host without a GPU: an error status, not a crash
    assert L.scp3gpu_scp1_create(0, 2, 0, 0, ctypes.byref(h)) == _lib.ERR_UNSUPPORTED
    assert not h.value
    assert L.scp3gpu_scp1_average(None, None, None, None, 0, 0, 0, None, None, None) == _lib.ERR_ARG
    L.scp3gpu_scp1_destroy(None)


def test_inverse_cdf_item_split_is_exact():
    """The FP32 per-sample kernel (sampling.cu) splits item i of a sample group
    into (sample, dimension) as j = (int)((i + 0.5f) * (1.0f / nm0)) instead of an
    integer division; restated here in IEEE float32, it equals i // nm0 for every
    mode count the library admits (nm0 <= 144: at most 16 waters) and every
    i < 2^16, a bound far above the 4 * nm0 items of a group."""
    for nm0 in range(1, 145):
        inv = np.float32(1.0) / np.float32(nm0)
        i = np.arange(1 << 16, dtype=np.int64)
        j = ((i.astype(np.float32) + np.float32(0.5)) * inv).astype(np.int32)
        assert np.array_equal(j, i // nm0), nm0
