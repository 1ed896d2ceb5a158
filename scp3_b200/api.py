"""Host-side mirror of the reference's interfaces for the Hamiltonian build,
running on the B200 through libscp3gpu.so.

  PES / qtip4pf / ttm3f     h2o::PES::operator()(nw, crd)   (PES.h:14-22)
  std_normal                sobol::std_normal(dims, &seed, u) (sobol.hpp:31)
  ScaledMatrixElements      ScaledMatrixElements(omega, N2, N3), getBasisSize,
                            getSubBasisSize, addEpot(q, V, M) (-G), addHODiagonal
                            (ScaledMatrixElements.h:75-96)
  HBuild                    the sample loop of SCP3_a (SCP3.cpp:154-272) fused on
                            the device, with the periodic readout's Mout and
                            eigenvalues

Arrays follow the reference's conventions: geometries in Angstrom, O H H per
water; energies from PES in kcal/mol; q, V, omega, M in atomic units; M is a
column-major (Fortran-ordered) Nb x Nb float64 array.
"""
import ctypes

import numpy as np

from . import _lib
from . import constants as C
from . import modes as _modes

_dp = ctypes.POINTER(ctypes.c_double)


def _p(a):
    return a.ctypes.data_as(_dp)


class PES:
    """A water potential evaluated on the GPU, one warp per geometry."""

    def __init__(self, name):
        if name not in C.PES_IDS:
            raise ValueError("Unknown H2O potential: %s" % name)   # h2o.h:38-41
        self.pes_id = C.PES_IDS[name]
        self._name = name

    def name(self):
        return {"qtip4pf": "q-TIP4P/F", "ttm3f": "TTM3-F"}[self._name]

    def energies(self, crd, return_iters=False):
        """Energies (kcal/mol) of a batch of geometries: crd is (n, 9*nw) Angstrom."""
        crd = np.ascontiguousarray(np.atleast_2d(crd), dtype=np.float64)
        n, w = crd.shape
        if w % 9:
            raise ValueError("a geometry has 9*nw coordinates")
        E = np.zeros(n)
        it = np.zeros(n, dtype=np.int32)
        rc = _lib.lib().scp3gpu_pes_energy(self.pes_id, w // 9, n, _p(crd), _p(E),
                                           it.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        if rc != _lib.ERR_NOT_CONVERGED:
            _lib.check(rc)
        return (E, it) if return_iters else E

    def energies_grad(self, crd):
        """Energies (kcal/mol) and gradients (kcal/mol/A, n x 9nw) of a batch of
        geometries (qTIP4P/f)."""
        crd = np.ascontiguousarray(np.atleast_2d(crd), dtype=np.float64)
        n, w = crd.shape
        if w % 9:
            raise ValueError("a geometry has 9*nw coordinates")
        E = np.zeros(n)
        G = np.zeros((n, w))
        _lib.check(_lib.lib().scp3gpu_pes_energy_grad(self.pes_id, w // 9, n, _p(crd), _p(E), _p(G)))
        return E, G

    def __call__(self, nw, crd, grad=None):
        """h2o::PES::operator()(nw, crd[, grad]) (PES.h:14-22): the energy; with a
        9nw array `grad`, the gradient is written into it."""
        crd = np.asarray(crd, dtype=np.float64).reshape(1, -1)
        if crd.shape[1] != 9 * nw:
            raise ValueError("crd must hold 9*nw coordinates")
        if grad is not None:
            E, G = self.energies_grad(crd)
            grad[:] = G[0]
            return float(E[0])
        return float(self.energies(crd)[0])


def qtip4pf():
    return PES("qtip4pf")


def ttm3f():
    return PES("ttm3f")


def PESFromString(name):
    """h2o::PESFromString (h2o.h:20-47), with TTM3-F selectable."""
    return PES(name)


def std_normals(dims, index0, n, scramble_seed=None):
    """n x dims standard normals of Sobol points index0.. (scrambled if a seed is given)."""
    out = np.zeros((n, dims))
    scr = _lib.SOBOL_SCRAMBLED if scramble_seed is not None else _lib.SOBOL_REFERENCE
    _lib.check(_lib.lib().scp3gpu_sobol_std_normal(dims, index0, n, scr, scramble_seed or 0, _p(out)))
    return out


def std_normal(dims, seed):
    """sobol::std_normal: seed is a one-element list [index]; returns the point and advances it."""
    u = std_normals(dims, seed[0], 1)[0]
    seed[0] += 1
    return u


PRECISIONS = {"fp64": _lib.PREC_FP64, "bf16x3": _lib.PREC_BF16X3, "bf16x3_pes64": _lib.PREC_BF16X3_PES64,
              "f16x3": _lib.PREC_F16X3, "f16x3_pes64": _lib.PREC_F16X3_PES64}


def _fill_config(obj, nw, x0, MUa, omega, modes, n2, n3, pes, precision, scramble_seed, chunk, device,
                 estimator="direct"):
    """Fill obj._cfg (a Config) and keep the arrays it points to alive on obj."""
    obj.x0 = np.ascontiguousarray(x0, dtype=np.float64)
    obj.MUa = np.asfortranarray(MUa, dtype=np.float64)
    obj.omega = np.ascontiguousarray(omega, dtype=np.float64)
    nm0 = obj.omega.size
    obj.modes = np.arange(nm0, dtype=np.int32) if modes is None else np.ascontiguousarray(modes, dtype=np.int32)
    n2 = obj.modes.size if n2 is None else n2      # SCP3.cpp:305
    obj.n2, obj.n3 = n2, n3
    cfg = _lib.Config()
    cfg.nw, cfg.nmodes0 = nw, nm0
    cfg.x0, cfg.MUa, cfg.omega = _p(obj.x0), obj.MUa.ctypes.data_as(_dp), _p(obj.omega)
    cfg.nmodes = obj.modes.size
    cfg.modes = obj.modes.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    cfg.n2, cfg.n3 = n2, n3
    cfg.pes = C.PES_IDS[pes] if isinstance(pes, str) else int(pes)
    cfg.precision = PRECISIONS[precision]
    cfg.scramble = _lib.SOBOL_SCRAMBLED if scramble_seed is not None else _lib.SOBOL_REFERENCE
    cfg.scramble_seed = scramble_seed or 0
    cfg.chunk, cfg.device = chunk, device
    cfg.estimator = {"direct": _lib.ESTIMATOR_DIRECT, "gradient": _lib.ESTIMATOR_GRADIENT}[estimator]
    obj._cfg = cfg


class HBuild:
    """One device-side Hamiltonian build: ScaledMatrixElements + the SCP3_a loop."""

    def __init__(self, nw, x0, MUa, omega, modes=None, n2=None, n3=0, pes="qtip4pf", precision="fp64",
                 scramble_seed=None, chunk=0, device=0, estimator="direct"):
        """estimator: "direct" (-G, sum Phi V Phi^T) or "gradient" (the reference's
        default Stein estimator from V and dV/dq; FP64, qTIP4P/f)."""
        _fill_config(self, nw, x0, MUa, omega, modes, n2, n3, pes, precision, scramble_seed, chunk, device,
                     estimator)
        self.estimator = estimator
        cfg = self._cfg
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().scp3gpu_hbuild_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self.nb = int(_lib.lib().scp3gpu_hbuild_basis_size(h))
        self.precision = precision

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().scp3gpu_hbuild_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        return _lib.lib().scp3gpu_hbuild_stream(self._h)

    def getBasisSize(self):
        return self.nb

    def getSubBasisSize(self, level):
        return _modes.sub_basis_size(self.modes.size, self.n2, self.n3, level)

    def reset(self):
        _lib.check(_lib.lib().scp3gpu_hbuild_reset(self._h))

    def accumulate(self, index0, n):
        _lib.check(_lib.lib().scp3gpu_hbuild_accumulate(self._h, index0, n))

    def accumulate_normals(self, normals):
        """The -r path: n x nmodes0 standard normals, sample-major.  A float32 array
        goes in as FP32 (scp3gpu_hbuild_accumulate_normals_f32, half the copy);
        anything else as FP64."""
        if isinstance(normals, np.ndarray) and normals.dtype == np.float32:
            normals = np.ascontiguousarray(normals)
            _lib.check(_lib.lib().scp3gpu_hbuild_accumulate_normals_f32(
                self._h, normals.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), normals.shape[0]))
            return
        normals = np.ascontiguousarray(normals, dtype=np.float64)
        _lib.check(_lib.lib().scp3gpu_hbuild_accumulate_normals(self._h, _p(normals), normals.shape[0]))

    def add_epot(self, q, V):
        q = np.ascontiguousarray(q, dtype=np.float64)
        V = np.ascontiguousarray(V, dtype=np.float64)
        _lib.check(_lib.lib().scp3gpu_hbuild_add_epot(self._h, _p(q), _p(V), V.size))

    def add_epot_grad(self, q, V, Vq):
        """addEpot(q, V, Vq, M) of the gradient path: q, Vq n x nmodes, V n."""
        q = np.ascontiguousarray(q, dtype=np.float64)
        V = np.ascontiguousarray(V, dtype=np.float64)
        Vq = np.ascontiguousarray(Vq, dtype=np.float64)
        _lib.check(_lib.lib().scp3gpu_hbuild_add_epot_grad(self._h, _p(q), _p(V), _p(Vq), V.size))

    def sample_count(self):
        return int(_lib.lib().scp3gpu_hbuild_sample_count(self._h))

    def read(self, mode=0, out=None):
        """mode 0: the raw sum M; mode 1: Mout = M/n + HO diagonal + inactive ZPE."""
        M = out if out is not None else np.zeros((self.nb, self.nb), order="F")
        _lib.check(_lib.lib().scp3gpu_hbuild_read(self._h, M.ctypes.data_as(_dp), M.shape[0], mode))
        return M

    def read_dev(self, ptr, ld, mode=0):
        """Write the matrix into device memory at `ptr` (leading dimension ld), stream-ordered."""
        _lib.check(_lib.lib().scp3gpu_hbuild_read_dev(self._h, ctypes.c_void_p(ptr), ld, mode))

    def eigvals(self, k=10, nsub=None):
        ev = np.zeros(k)
        _lib.check(_lib.lib().scp3gpu_hbuild_eigvals(self._h, nsub or self.nb, k, _p(ev)))
        return ev

    def profile(self, enable):
        """Start (True) or stop (False) kernel timing; stop returns (ms[4], launches[4]) per kind:
        per-sample, expansion/partition, contraction, read-out."""
        ms = np.zeros(4)
        n = np.zeros(4, dtype=np.int64)
        _lib.check(_lib.lib().scp3gpu_hbuild_profile(self._h, 1 if enable else 0, _p(ms),
                                                     n.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        return ms, n

    def status(self):
        a, b = ctypes.c_int64(), ctypes.c_int64()
        rc = _lib.lib().scp3gpu_hbuild_status(self._h, ctypes.byref(a), ctypes.byref(b))
        return rc, a.value, b.value


class ScaledMatrixElements:
    """ScaledMatrixElements(omega, N2, N3) of the -G path: addEpot accumulates
    sum_s bra(q_s) V_s bra(q_s)^T into the caller's M (upper triangle and its
    mirror), exactly as the reference's addEpot(q, V, M) adds into M."""

    def __init__(self, omega, Nmodes2=0, Nmodes3=0, precision="fp64", device=0):
        self.omega = np.ascontiguousarray(omega, dtype=np.float64)
        self.Nmodes, self.Nmodes2, self.Nmodes3 = self.omega.size, Nmodes2, Nmodes3
        nm = self.Nmodes
        # a one-water placeholder geometry: addEpot takes q and V from the caller
        nw = max(1, -(-(nm + 6) // 9))
        nm0 = 9 * nw - 6
        om = np.concatenate([self.omega, np.ones(nm0 - nm)])
        self._hb = HBuild(nw, np.zeros(9 * nw), np.zeros((9 * nw, nm0)), om, modes=np.arange(nm), n2=Nmodes2,
                          n3=Nmodes3, precision=precision, device=device)

    def getBasisSize(self):
        return self._hb.nb

    def getSubBasisSize(self, n):
        return _modes.sub_basis_size(self.Nmodes, self.Nmodes2, self.Nmodes3, n)

    def addEpot(self, q, V, M):
        """q: Nmodes x B (column per sample, as in the reference), V: B, M: Nb x Nb (updated)."""
        q = np.asarray(q, dtype=np.float64)
        self._hb.reset()
        self._hb.add_epot(np.ascontiguousarray(q.T), V)
        M += self._hb.read(0)
        return M

    def addHODiagonal(self, M):
        """diag += E0 + sum n_k omega_k (ScaledMatrixElements.cpp:735-784)."""
        w = self.omega
        e0 = 0.5 * w.sum()
        d = [e0] + [e0 + w[k] for k in range(self.Nmodes)] + [e0 + 2 * w[k] for k in range(self.Nmodes2)]
        d += [e0 + w[k] + w[l] for k in range(self.Nmodes2) for l in range(k + 1, self.Nmodes2)]
        d += [e0 + 3.0 * w[k] for k in range(self.Nmodes3)]
        for k in range(self.Nmodes3):
            for l in range(k + 1, self.Nmodes3):
                d += [e0 + 2.0 * w[k] + w[l], e0 + w[k] + 2.0 * w[l]]
        d += [e0 + w[k] + w[l] + w[j] for k in range(self.Nmodes3) for l in range(k + 1, self.Nmodes3)
              for j in range(l + 1, self.Nmodes3)]
        M[np.diag_indices(len(d))] += np.array(d)
        return M


def dsyevr(A, IU=0, vectors=True, device=0):
    """The lowest IU eigenpairs of the symmetric matrix A on the GPU (FP64), as
    dsyevr(A, IU, &C) of the eigensolver tool (eigensolver.cpp:20-84): the upper
    triangle is read unless A[0, n-1] == 0.  IU = 0: all of them.  Returns W, or
    (W, C) with the eigenvectors as columns of C."""
    A = np.asfortranarray(A, dtype=np.float64)
    n = A.shape[0]
    k = n if IU <= 0 else IU
    W = np.zeros(k)
    C = np.zeros((n, k), order="F") if vectors else None
    _lib.check(_lib.lib().scp3gpu_syevr_lowest(A.ctypes.data_as(_dp), n, n, k, _p(W),
                                               C.ctypes.data_as(_dp) if vectors else None, n, device))
    return (W, C) if vectors else W


class _ClusterCfg:
    pass


class Batch:
    """Several clusters built together (scp3gpu_batch_*): one launch per stage
    for all clusters, each accumulate one CUDA graph replay.

    clusters: sequence of dicts with keys nw, x0, MUa, omega and optionally
    modes, n2, n3, scramble_seed (default: the batch's)."""

    def __init__(self, clusters, pes="qtip4pf", precision="bf16x3", scramble_seed=None, chunk=0, graph=True,
                 autotune=True, device=0):
        self._keep = []
        arr = (_lib.Config * len(clusters))()
        for i, c in enumerate(clusters):
            k = _ClusterCfg()
            _fill_config(k, c["nw"], c["x0"], c["MUa"], c["omega"], c.get("modes"), c.get("n2"), c.get("n3", 0),
                         pes, precision, c.get("scramble_seed", scramble_seed), 0, device)
            self._keep.append(k)
            arr[i] = k._cfg
        flags = (0 if graph else _lib.BATCH_NO_GRAPH) | (0 if autotune else _lib.BATCH_NO_AUTOTUNE)
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().scp3gpu_batch_create(arr, len(clusters), chunk, flags, ctypes.byref(h)))
        self._h = h
        self.ncl = len(clusters)
        self.nb = [int(_lib.lib().scp3gpu_batch_basis_size(h, i)) for i in range(self.ncl)]
        self.precision = precision

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().scp3gpu_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        return _lib.lib().scp3gpu_batch_stream(self._h)

    def shape(self):
        """(nsplit, ctas, samples per pass, timed contraction ms) of the chosen work shape."""
        ns, ct, ch, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_int64(), ctypes.c_double()
        _lib.check(_lib.lib().scp3gpu_batch_shape(self._h, ctypes.byref(ns), ctypes.byref(ct), ctypes.byref(ch),
                                                  ctypes.byref(ms)))
        return ns.value, ct.value, ch.value, ms.value

    def reset(self):
        _lib.check(_lib.lib().scp3gpu_batch_reset(self._h))

    def accumulate(self, index0, n):
        _lib.check(_lib.lib().scp3gpu_batch_accumulate(self._h, index0, n))

    def sample_count(self):
        return int(_lib.lib().scp3gpu_batch_sample_count(self._h))

    def read(self, cluster, mode=0):
        nb = self.nb[cluster]
        M = np.zeros((nb, nb), order="F")
        _lib.check(_lib.lib().scp3gpu_batch_read(self._h, cluster, M.ctypes.data_as(_dp), nb, mode))
        return M

    def status(self, cluster):
        a, b = ctypes.c_int64(), ctypes.c_int64()
        rc = _lib.lib().scp3gpu_batch_status(self._h, cluster, ctypes.byref(a), ctypes.byref(b))
        return rc, a.value, b.value


class SCP1Average:
    """The sample loop of SCP1::average (SCP1.cpp:34-90) on one GPU: for Sobol
    points i0 <= i < i1 (offset `skip`, dimension 9*nw), the sums of V, dV/dr
    and dV/dr dq^T.  The caller all-reduces the sums over ranks and divides by
    NSobol, as SCP1.cpp:71-88 does."""

    def __init__(self, pes, nw, chunk=0, device=0):
        if pes not in C.PES_IDS:
            raise ValueError("Unknown H2O potential: %s" % pes)
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().scp3gpu_scp1_create(C.PES_IDS[pes], nw, chunk, device, ctypes.byref(h)))
        self._h = h
        self.nw = nw
        self.dim = 9 * nw

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().scp3gpu_scp1_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sums(self, q, d, isqrtM_U, skip, i0, i1):
        """(sum V, sum UX[dim], sum UX dq^T [dim x dim]) over points i0..i1-1."""
        q = np.ascontiguousarray(q, dtype=np.float64)
        d = np.ascontiguousarray(d, dtype=np.float64)
        U = np.asfortranarray(isqrtM_U, dtype=np.float64)
        if q.size != self.dim or d.size != self.dim or U.shape != (self.dim, self.dim):
            raise ValueError("q, d and isqrtM_U must have 9*nw rows")
        up = ctypes.c_double()
        UX = np.zeros(self.dim)
        UXq = np.zeros((self.dim, self.dim), order="F")
        _lib.check(_lib.lib().scp3gpu_scp1_average(self._h, _p(q), _p(d), U.ctypes.data_as(_dp), int(skip), int(i0),
                                                  int(i1), ctypes.byref(up), _p(UX), UXq.ctypes.data_as(_dp)))
        return up.value, UX, UXq

    def not_converged(self):
        n = ctypes.c_int64()
        _lib.check(_lib.lib().scp3gpu_scp1_status(self._h, ctypes.byref(n)))
        return n.value
