"""TEST INFRASTRUCTURE ONLY -- the oracle.

ctypes access to two CPU libraries that check the product and are never part of it:

* ``liboracle.so`` (built from ``scp3_oracle.c``): our plain-C, FP64 restatement of
  the reference's Hamiltonian-build path (Sobol, BSM, qTIP4P/f, TTM3-F, get_bra,
  the -G accumulation, the HO diagonal).  Always available once built.
* ``_ref/libscp3ref*.so`` (built by ``oracle/Makefile`` from the reference's own
  sources where they lie): the reference itself.  Used to pin the restatement
  and as the timed CPU baseline.  Absent wherever the reference tree was absent
  at build time and no prebuilt copy travelled.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_c_dp = ctypes.POINTER(ctypes.c_double)
_c_i64p = ctypes.POINTER(ctypes.c_int64)
_c_u64p = ctypes.POINTER(ctypes.c_uint64)


def _dp(a):
    return a.ctypes.data_as(_c_dp)


def build(reference=None):
    """Compile the restatement, and oracle/_ref when a reference tree is given
    (the argument, else $SCP3_REFERENCE) and exists."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    ref = reference or os.environ.get("SCP3_REFERENCE")
    if ref and os.path.isdir(ref):
        subprocess.run(["make", "-s", "-C", HERE, "ref", "REF=" + ref], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.or_sobol_dirnums.argtypes = [ctypes.c_int, _c_i64p]
        L.or_scramble_params.argtypes = [ctypes.c_int, ctypes.c_uint64, _c_u64p, _c_u64p]
        L.or_sobol_uniforms.argtypes = [ctypes.c_int, _c_i64p, _c_u64p, _c_u64p, ctypes.c_int64,
                                        ctypes.c_int64, _c_dp]
        L.or_bsm.argtypes = [ctypes.c_int64, _c_dp, _c_dp]
        L.or_qtip4pf.restype = ctypes.c_double
        L.or_qtip4pf.argtypes = [ctypes.c_int, _c_dp]
        L.or_ttm3f.restype = ctypes.c_double
        L.or_ttm3f.argtypes = [ctypes.c_int, _c_dp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.or_ps_pot.restype = ctypes.c_double
        L.or_ps_pot.argtypes = [_c_dp]
        L.or_ps_dms.argtypes = [_c_dp, _c_dp]
        L.or_basis_size.restype = ctypes.c_size_t
        L.or_basis_size.argtypes = [ctypes.c_int] * 3
        L.or_get_bra.argtypes = [ctypes.c_int] * 3 + [_c_dp, _c_dp]
        L.or_add_ho_diagonal.argtypes = [ctypes.c_int, _c_dp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                         _c_dp, ctypes.c_int64]
        L.or_samples.argtypes = [ctypes.c_int, ctypes.c_int, _c_dp, _c_dp, _c_dp, ctypes.c_int, _c_dp,
                                 ctypes.c_int64, _c_dp, _c_dp]
        L.or_accumulate.argtypes = [ctypes.c_int] * 3 + [_c_dp, _c_dp, ctypes.c_int64, _c_dp]
        L.or_accumulate_abs.argtypes = [ctypes.c_int] * 3 + [_c_dp, _c_dp, ctypes.c_int64, _c_dp]
        L.or_basis_modes.restype = ctypes.c_int
        L.or_basis_modes.argtypes = [ctypes.c_int] * 3 + [ctypes.c_int64, ctypes.POINTER(ctypes.c_int),
                                                          ctypes.POINTER(ctypes.c_int)]
        L.or_qtip4pf_grad.restype = ctypes.c_double
        L.or_qtip4pf_grad.argtypes = [ctypes.c_int, _c_dp, _c_dp]
        L.or_samples_grad.argtypes = [ctypes.c_int, _c_dp, _c_dp, _c_dp, ctypes.c_int, _c_dp, ctypes.c_int64,
                                      _c_dp, _c_dp, _c_dp]
        ip = ctypes.POINTER(ctypes.c_int)
        L.or_stein_term.restype = ctypes.c_double
        L.or_stein_term.argtypes = [_c_dp, ctypes.c_double, _c_dp, ctypes.c_int, ip, ip, ctypes.c_int, ip, ip]
        L.or_accumulate_stein.argtypes = [ctypes.c_int] * 3 + [_c_dp, _c_dp, _c_dp, ctypes.c_int64, _c_dp]
        _lib = L
    return _lib


# ---------------------------------------------------------------- restatement
def sobol_dirnums(dims):
    v = np.zeros((dims, 62), dtype=np.int64)
    if lib().or_sobol_dirnums(dims, v.ctypes.data_as(_c_i64p)) != 0:
        raise ValueError("dims out of range")
    return v


def scramble_params(dims, seed):
    masks = np.zeros((dims, 62), dtype=np.uint64)
    shift = np.zeros(dims, dtype=np.uint64)
    lib().or_scramble_params(dims, seed, masks.ctypes.data_as(_c_u64p), shift.ctypes.data_as(_c_u64p))
    return masks, shift


def sobol_uniforms(dims, index0, n, scramble_seed=None):
    v = sobol_dirnums(dims)
    out = np.zeros((n, dims))
    if scramble_seed is None:
        lib().or_sobol_uniforms(dims, v.ctypes.data_as(_c_i64p), None, None, index0, n, _dp(out))
    else:
        masks, shift = scramble_params(dims, scramble_seed)
        lib().or_sobol_uniforms(dims, v.ctypes.data_as(_c_i64p), masks.ctypes.data_as(_c_u64p),
                                shift.ctypes.data_as(_c_u64p), index0, n, _dp(out))
    return out


def bsm(u):
    u = np.ascontiguousarray(u, dtype=np.float64)
    x = np.zeros_like(u)
    lib().or_bsm(u.size, _dp(u), _dp(x))
    return x


def std_normals(dims, index0, n, scramble_seed=None):
    """n x dims standard normals: Sobol (optionally scrambled) through BSM."""
    return bsm(sobol_uniforms(dims, index0, n, scramble_seed))


def qtip4pf(crd):
    crd = np.ascontiguousarray(crd, dtype=np.float64)
    return lib().or_qtip4pf(crd.size // 9, _dp(crd))


def ttm3f(crd, maxiter=500, with_iters=False):
    crd = np.ascontiguousarray(crd, dtype=np.float64)
    it = ctypes.c_int(0)
    e = lib().or_ttm3f(crd.size // 9, _dp(crd), maxiter, ctypes.byref(it))
    return (e, it.value) if with_iters else e


def basis_size(nm, n2, n3):
    return lib().or_basis_size(nm, n2, n3)


def get_bra(q, n2, n3):
    q = np.ascontiguousarray(q, dtype=np.float64)
    out = np.zeros(basis_size(q.size, n2, n3))
    lib().or_get_bra(q.size, n2, n3, _dp(q), _dp(out))
    return out


def samples(pes_id, nw, x0, MUa, omega, normals):
    """Per-sample stage: (q n x nm0, V_anh n) from standard normals n x nm0."""
    x0 = np.ascontiguousarray(x0, dtype=np.float64)
    MUa_f = np.asfortranarray(MUa, dtype=np.float64)
    omega = np.ascontiguousarray(omega, dtype=np.float64)
    normals = np.ascontiguousarray(normals, dtype=np.float64)
    n, nm0 = normals.shape
    q = np.zeros((n, nm0))
    v = np.zeros(n)
    lib().or_samples(pes_id, nw, _dp(x0), MUa_f.ctypes.data_as(_c_dp), _dp(omega), nm0, _dp(normals), n,
                     _dp(q), _dp(v))
    return q, v


def accumulate(q_sel, v, n2, n3, M=None, absolute=False):
    """Upper triangle of sum_s bra(q_s) V_s bra(q_s)^T, returned column-major (Fortran) nb x nb."""
    q_sel = np.ascontiguousarray(q_sel, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    n, nm = q_sel.shape
    nb = basis_size(nm, n2, n3)
    if M is None:
        M = np.zeros((nb, nb), order="F")
    fn = lib().or_accumulate_abs if absolute else lib().or_accumulate
    fn(nm, n2, n3, _dp(q_sel), _dp(v), n, M.ctypes.data_as(_c_dp))
    return M


def add_ho_diagonal(M, omega_sel, n2, n3, zpe_inactive=0.0):
    omega_sel = np.ascontiguousarray(omega_sel, dtype=np.float64)
    assert M.flags.f_contiguous
    lib().or_add_ho_diagonal(omega_sel.size, _dp(omega_sel), n2, n3, zpe_inactive, M.ctypes.data_as(_c_dp),
                             M.shape[0])
    return M


# ---------------------------------------------------------------- the reference itself
_ref = {}


def basis_modes(nm, n2, n3, R):
    """(mode, level) pairs of basis function R (the order of get_bra)."""
    m = (ctypes.c_int * 3)()
    lv = (ctypes.c_int * 3)()
    k = lib().or_basis_modes(nm, n2, n3, R, m, lv)
    return [(m[t], lv[t]) for t in range(k)]


def qtip4pf_grad(crd):
    crd = np.ascontiguousarray(crd, dtype=np.float64)
    g = np.zeros(crd.size)
    e = lib().or_qtip4pf_grad(crd.size // 9, _dp(crd), _dp(g))
    return e, g


def samples_grad(nw, x0, MUa, omega, normals):
    """(q, V_anh, dV_anh/dq) of the gradient path, all nm0 modes (qTIP4P/f)."""
    normals = np.ascontiguousarray(normals, dtype=np.float64)
    n, nm0 = normals.shape
    MUa = np.asfortranarray(MUa, dtype=np.float64)
    q = np.zeros((n, nm0))
    v = np.zeros(n)
    vq = np.zeros((n, nm0))
    lib().or_samples_grad(nw, _dp(np.ascontiguousarray(x0, dtype=np.float64)), _dp(MUa),
                          _dp(np.ascontiguousarray(omega, dtype=np.float64)), nm0, _dp(normals), n, _dp(q), _dp(v),
                          _dp(vq))
    return q, v, vq


def stein_term(q, V, vq, bra, ket):
    """One sample's gradient-estimator value for <bra|V|ket>, each a list of (mode, level)."""
    q = np.ascontiguousarray(q, dtype=np.float64)
    vq = np.ascontiguousarray(vq, dtype=np.float64)
    mi = (ctypes.c_int * 3)(*[b[0] for b in bra])
    li = (ctypes.c_int * 3)(*[b[1] for b in bra])
    mj = (ctypes.c_int * 3)(*[b[0] for b in ket])
    lj = (ctypes.c_int * 3)(*[b[1] for b in ket])
    return lib().or_stein_term(_dp(q), float(V), _dp(vq), len(bra), mi, li, len(ket), mj, lj)


def accumulate_stein(q_sel, v, vq_sel, n2, n3, M=None):
    """Upper triangle of sum_s estimate_ij(s) (addEpot(q, V, Vq, M)), column-major nb x nb."""
    q_sel = np.ascontiguousarray(q_sel, dtype=np.float64)
    vq_sel = np.ascontiguousarray(vq_sel, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    n, nm = q_sel.shape
    nb = basis_size(nm, n2, n3)
    out = np.zeros((nb, nb), order="F") if M is None else M
    lib().or_accumulate_stein(nm, n2, n3, _dp(q_sel), _dp(v), _dp(vq_sel), n, out.ctypes.data_as(_c_dp))
    return out


def ref_available(fast=False):
    return os.path.exists(os.path.join(HERE, "_ref", "libscp3ref_fast.so" if fast else "libscp3ref.so"))


# Threading of the reference's CPU build.  Its block loop alternates an OpenMP
# region (get_bra and the ket, ScaledMatrixElements.cpp:956-968) with a threaded
# BLAS dsyr2k (:970).  With the libraries' defaults both thread pools busy-wait
# after their work (OpenBLAS for 2^28 cycles, libgomp for its spin count), so
# each phase ran against the other's spinning threads on the same cores: the
# get_bra phase took 3x as long as dsyr2k for a tenth of its work.  The
# reference's production build shares one OpenMP pool between its loop and
# MKL; here the two pools are told to sleep when idle instead.  Both variables
# are read when the libraries load, so they are set before the first load;
# values the caller exported win.
REF_THREAD_ENV = {"OPENBLAS_THREAD_TIMEOUT": "4", "OMP_WAIT_POLICY": "PASSIVE"}


def ref_thread_env():
    """The thread settings in force for the reference's CPU build."""
    return {k: os.environ.get(k) for k in REF_THREAD_ENV}


def ref_lib(fast=False):
    """The reference's own sources compiled by oracle/Makefile (parity or release flags)."""
    key = "fast" if fast else "parity"
    if key not in _ref:
        for k, v in REF_THREAD_ENV.items():
            os.environ.setdefault(k, v)
        L = ctypes.CDLL(os.path.join(HERE, "_ref", "libscp3ref_fast.so" if fast else "libscp3ref.so"))
        for fn in ("ref_qtip4pf_energy", "ref_ttm3f_energy"):
            getattr(L, fn).restype = ctypes.c_double
            getattr(L, fn).argtypes = [ctypes.c_int, _c_dp]
        L.ref_i8_sobol.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_longlong), _c_dp]
        L.ref_std_normal.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_longlong), _c_dp]
        L.ref_ho.restype = ctypes.c_double
        L.ref_ho.argtypes = [ctypes.c_int, ctypes.c_double]
        L.ref_get_bra.argtypes = [ctypes.c_int] * 3 + [_c_dp, _c_dp]
        L.ref_basis_size.restype = ctypes.c_size_t
        L.ref_basis_size.argtypes = [ctypes.c_int] * 3
        L.ref_hbuild.restype = ctypes.c_int
        L.ref_hbuild.argtypes = [ctypes.c_int, ctypes.c_int, _c_dp, _c_dp, _c_dp, ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_longlong), _c_dp, ctypes.c_longlong, ctypes.c_int,
                                 _c_dp, _c_dp]
        # The reference's TTM3-F reads its induced-field buffer before writing it
        # (ttm3f.cpp:108-109 zeroes from Efq on); one call on a sane geometry
        # leaves that buffer finite so later calls converge.
        w = np.array([0.0, 0.0, 0.0, 0.7572, 0.5865, 0.0, -0.7572, 0.5865, 0.0])
        for _ in range(2):
            L.ref_ttm3f_energy(1, _dp(w))
        _ref[key] = L
    return _ref[key]


def ref_hbuild(pes_id, nw, x0, MUa, omega, modes, n2, n3, nsamples, block, normals=None, seed=1 << 30,
               fast=False, M=None):
    """The reference's -G sample loop (see ref_hbuild.cpp).  Returns (M, timings, next_seed)."""
    L = ref_lib(fast)
    x0 = np.ascontiguousarray(x0, dtype=np.float64)
    MUa_f = np.asfortranarray(MUa, dtype=np.float64)
    omega = np.ascontiguousarray(omega, dtype=np.float64)
    modes = np.ascontiguousarray(modes, dtype=np.int32)
    nm0 = omega.size
    nb = L.ref_basis_size(modes.size, n2, n3)
    if M is None:
        M = np.zeros((nb, nb), order="F")
    t = np.zeros(3)
    s = ctypes.c_longlong(seed)
    nrm = None
    if normals is not None:
        nrm = np.ascontiguousarray(normals, dtype=np.float64)
    rc = L.ref_hbuild(pes_id, nw, _dp(x0), MUa_f.ctypes.data_as(_c_dp), _dp(omega), nm0,
                      modes.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), modes.size, n2, n3, ctypes.byref(s),
                      None if nrm is None else _dp(nrm), nsamples, block, M.ctypes.data_as(_c_dp), _dp(t))
    if rc != 0:
        raise ValueError("ref_hbuild rejected its arguments")
    return M, t, s.value
