"""TEST INFRASTRUCTURE ONLY -- the oracle of the SCP1 effective-Hessian iteration.

* average_sums: NumPy restatement of SCP1::average's sample loop
  (SCP1.cpp:49-69) over the oracle's Sobol/BSM (pinned bit for bit against the
  reference's i8_sobol) and potential gradients: scp3_oracle.c's qTIP4P/f
  gradient (pinned against qtip4pf.cpp), or the reference's own TTM3-F
  gradient from oracle/_ref.
* ref_average_sums: the same loop written in C over the reference's own
  std_normal and potentials (oracle/ref_shim.cpp, ref_scp1_average).
* iteration: one pass of SCP1::operator()'s loop body (SCP1.cpp:123-170),
  restated with explicit index loops.

SCP1.cpp itself needs Armadillo and MPI and is not built here, so the update
formulas are pinned only through this restatement; the sample loop is pinned
by the two independent sums above agreeing.

Only tests/ and the CPU-baseline leg of bench.py use this module.
"""
import ctypes
import math

import numpy as np

from . import _dp, lib, qtip4pf_grad, ref_available, ref_lib, std_normals

BOHR = 0.52917721092
AUTOKCAL = 627.509474277194


def _grad_fn(pes):
    if pes == "qtip4pf":
        return qtip4pf_grad
    if not ref_available():
        raise RuntimeError("TTM3-F gradients need oracle/_ref (the reference's sources)")
    L = ref_lib()
    L.ref_ttm3f_energy_grad.restype = ctypes.c_double
    L.ref_ttm3f_energy_grad.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_double)]

    def f(crd):
        crd = np.ascontiguousarray(crd, dtype=np.float64)
        g = np.zeros(crd.size)
        e = L.ref_ttm3f_energy_grad(crd.size // 9, _dp(crd), _dp(g))
        return e, g
    return f


def average_sums(pes, nw, q, d, isqrtM_U, skip, i0, i1):
    """(sum V, sum UX, sum UX dq^T) over Sobol points skip+i0 .. skip+i1-1."""
    dim = 9 * nw
    grad = _grad_fn(pes)
    n = i1 - i0
    y = std_normals(dim, skip + i0, n) * np.sqrt(np.asarray(d, dtype=np.float64))[None, :]
    U = np.asarray(isqrtM_U, dtype=np.float64)
    up = 0.0
    UX = np.zeros(dim)
    UXq = np.zeros((dim, dim))
    for s in range(n):
        dq = np.zeros(dim)
        for k in range(dim):          # k in order, as the kernels sum
            dq += U[:, k] * y[s, k]
        e, g = grad(BOHR * (q + dq))
        up += e / AUTOKCAL
        g = g * (BOHR / AUTOKCAL)
        UX += g
        UXq += np.outer(g, dq)
    return up, UX, UXq


def ref_average_sums(pes, nw, q, d, isqrtM_U, skip, i0, i1, fast=False):
    """The same sums from the reference's own functions (ref_scp1_average)."""
    L = ref_lib(fast)
    f = L.ref_scp1_average
    f.restype = None
    dp = ctypes.POINTER(ctypes.c_double)
    f.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong,
                  dp, dp, dp]
    dim = 9 * nw
    q = np.ascontiguousarray(q, dtype=np.float64)
    d = np.ascontiguousarray(d, dtype=np.float64)
    U = np.asfortranarray(isqrtM_U, dtype=np.float64)
    up = ctypes.c_double()
    UX = np.zeros(dim)
    UXq = np.zeros((dim, dim), order="F")
    f(0 if pes == "qtip4pf" else 1, nw, _dp(q), _dp(d), U.ctypes.data_as(dp), skip, i0, i1, ctypes.byref(up),
      _dp(UX), UXq.ctypes.data_as(dp))
    return up.value, UX, UXq


def transrot(q, mass):
    """Hessian.cpp:98-131, with explicit loops."""
    n = len(q)
    U = [[0.0] * 6 for _ in range(n)]
    tm = sum(mass) / 3.0
    for i in range(0, n, 3):
        qs = [q[i + k] * math.sqrt(mass[i + k]) for k in range(3)]
        for k in range(3):
            U[i + k][k] = math.sqrt(mass[i + k] / tm)
        U[i + 1][3], U[i + 2][3] = -qs[2], qs[1]
        U[i][4], U[i + 2][4] = qs[2], -qs[0]
        U[i][5], U[i + 1][5] = -qs[1], qs[0]
    U = np.array(U)
    for i in range(3, 6):
        for j in range(i):
            U[:, i] = U[:, i] - U[:, j] * float(U[:, i] @ U[:, j])
        U[:, i] = U[:, i] / math.sqrt(float(U[:, i] @ U[:, i]))
    return U


def project(U, H):
    HP = H - (H @ U) @ U.T
    return HP - U @ (U.T @ HP)


def corr(omega, kT, cutoff):
    out = np.zeros_like(omega)
    for i, w in enumerate(omega):
        if w < cutoff:
            continue
        out[i] = 0.5 / w if kT == 0.0 else 0.5 / (w * math.tanh(0.5 / kT * w))
    return out


def iteration(q, U, d, mass, Upot, UX, UX_q, kT=0.0, cutoff=50.0 / 2.194746313e5, qeps=2.0):
    """One pass of SCP1.cpp:123-170 from the averages (<V>, <UX>, <UX dq^T>) at
    (q, U, d): returns (q_new, Ks, U_new, omega, d_new, F)."""
    n = len(q)
    A = np.array(UX_q, dtype=np.float64)
    for i in range(n):
        for j in range(n):
            A[j, i] *= math.sqrt(mass[i] / mass[j])
    KD = A @ U
    for i in range(n):
        KD[:, i] = KD[:, i] / d[i] if d[i] != 0.0 else 0.0
    Ks = KD @ U.T
    Ks = 0.5 * (Ks + Ks.T)
    Ks = project(transrot(q, mass), Ks)
    w2, U2 = np.linalg.eigh(Ks, UPLO="U")
    omega = np.sqrt(np.abs(w2))
    d2 = corr(omega, kT, cutoff)
    iU = U2 / np.sqrt(mass)[:, None]
    qn = q - qeps * (iU @ (d2 * (iU.T @ UX)))
    we = omega[6:]
    if kT > 0.0:
        F = Upot + kT * float(np.sum(np.log(2.0 * np.sinh(0.5 / kT * we)))) - 0.25 * float(
            np.sum(we / np.tanh(0.5 / kT * we)))
    else:
        F = Upot + 0.25 * float(np.sum(we))
    return qn, Ks, U2, omega, d2, F


def fd_hessian(pes, r_au, s=1e-3):
    """Hessian.cpp:12-43 over the oracle's gradient."""
    grad = _grad_fn(pes)
    n = r_au.size
    r = r_au * BOHR
    H = np.zeros((n, n))
    for i in range(n):
        rp = r.copy()
        rp[i] += s * BOHR
        rm = r.copy()
        rm[i] -= s * BOHR
        H[:, i] = (grad(rp)[1] - grad(rm)[1]) / (2.0 * s * AUTOKCAL)
    for i in range(1, n):
        H[:i, i] = 0.5 * (H[:i, i] + H[i, :i])
    return H


__all__ = ["average_sums", "ref_average_sums", "iteration", "fd_hessian", "transrot", "project", "corr", "lib"]
