"""SCP1: the self-consistent phonon iteration that produces the effective
Hessians of SCP3's input files (SCP1.h:25-103, SCP1.cpp:95-190, Hessian.cpp,
SCP1_main.cpp:34-133).

Each iteration averages the potential, its gradient and gradient x displacement
over NSobol Sobol points drawn from the current harmonic density (SCP1.cpp:34-90;
on the GPU through scp3gpu_scp1_average, one rank's share of the points per
process), all-reduces the three sums over ranks (torch.distributed: NCCL
between GPUs, gloo on the host), and updates the mass-scaled effective Hessian
Ks, the frequencies, the displacement variances d and the centroid q
(SCP1.cpp:123-170).  Rank 0 writes omega_scp1.dat, free_energy.dat and
coord.xyz (the input-file format, DiskIO.cpp:118-140) every iteration.

    python -m scp3_b200.scp1 [-N log2 NSobol] [-L iterations] [-c cutoff_cm1] [-p PES] input.dat

Under torchrun every rank takes points [rank N / P, (rank + 1) N / P) on its
own GPU.  As in the reference, -S and -r are accepted and have no effect
(SCP1_main.cpp sets a global skip the SCP1 object never reads and opens a file
it never reads).
"""
import argparse
import math
import os
import sys

import numpy as np

from . import constants as C, modes


def transrot_basis(q, mass):
    """Orthonormal mass-weighted translations and rotations at q (Hessian.cpp:98-131)."""
    n = q.size
    U = np.zeros((n, 6))
    qs = q * np.sqrt(mass)
    total = mass.sum() / 3.0
    for i in range(0, n, 3):
        U[i, 0] = math.sqrt(mass[i] / total)
        U[i + 1, 1] = math.sqrt(mass[i + 1] / total)
        U[i + 2, 2] = math.sqrt(mass[i + 2] / total)
        U[i + 1, 3], U[i + 2, 3] = -qs[i + 2], qs[i + 1]
        U[i, 4], U[i + 2, 4] = qs[i + 2], -qs[i]
        U[i, 5], U[i + 1, 5] = -qs[i + 1], qs[i]
    for i in range(3, 6):
        for j in range(i):
            U[:, i] -= U[:, j] * np.dot(U[:, i], U[:, j])
        U[:, i] /= np.linalg.norm(U[:, i])
    return U


def regtransrot(U, H):
    """H projected off the span of U from both sides (Hessian.cpp:134-141), in place."""
    HP = H - (H @ U) @ U.T
    H[:] = HP - U @ (U.T @ HP)
    return H


def mass_scale_hessian(mass, H):
    """H_ij / sqrt(m_i m_j), in place (Hessian.cpp:46-56)."""
    isq = 1.0 / np.sqrt(mass)
    H *= isq[:, None] * isq[None, :]
    return H


def get_hessian(grad_fn, r_au, s=1e-3):
    """Central differences of the gradient, step s bohr (Hessian.cpp:12-43).
    grad_fn maps an (m, 9nw) batch of Angstrom geometries to (E, G) in kcal/mol
    and kcal/mol/A; all 2N displaced geometries go in one batch.  Only the upper
    triangle is symmetrised, as in the reference."""
    n = r_au.size
    r = r_au * C.bohr
    crd = np.repeat(r[None, :], 2 * n, axis=0)
    for i in range(n):
        crd[2 * i, i] = r[i] + s * C.bohr
        crd[2 * i + 1, i] = r[i] - s * C.bohr
    _, G = grad_fn(crd)
    H = np.zeros((n, n))
    for i in range(n):
        H[:, i] = (G[2 * i] - G[2 * i + 1]) / (2.0 * s * C.autokcalpmol)
    for i in range(1, n):
        H[:i, i] = 0.5 * (H[:i, i] + H[i, :i])
    return H


def eig_sym(K):
    """Eigenpairs from the upper triangle (the triangle LAPACK ?syev reads for Armadillo's eig_sym)."""
    return np.linalg.eigh(K, UPLO="U")


class SCP1:
    """SCP1(mass, PES name, NSobol[, append]) (SCP1.h:48-67).

    averager(q, d, isqrtM_U, skip, i0, i1) -> (sum V, sum UX, sum UX dq^T) over
    points i0..i1-1; default: the GPU (scp3gpu_scp1_average).  grad_fn is the
    batched energy-and-gradient call the initial Hessian uses (default: the GPU
    potential).  The three sums are all-reduced over torch.distributed's
    default group when it is initialised with more than one rank."""

    def __init__(self, mass, pes="qtip4pf", nsobol=1 << 20, append=False, averager=None, grad_fn=None, device=0,
                 outdir=".", verbose=True):
        self.mass = np.asarray(mass, dtype=np.float64)
        self.pes = pes
        self.nsobol = int(nsobol)
        self.omega_cutoff = 50.0 / C.autocm
        self.epsrel = 1e-4
        self.qeps = 2.0
        self.sobol_skip = 1 << (int(math.floor(math.log2(float(np.float32(self.nsobol))))) + 1)
        self.rank, self.nprocs = 0, 1
        try:
            import torch.distributed as dist
            if dist.is_available() and dist.is_initialized():
                self.rank, self.nprocs = dist.get_rank(), dist.get_world_size()
        except ImportError:
            pass
        self.device = device
        self._averager = averager
        self._grad_fn = grad_fn
        self._gpu = None
        self.verbose = verbose
        self.outdir = outdir
        self.iterations = 0
        self.converged = False
        if self.rank == 0:
            mode = "a" if append else "w"
            os.makedirs(outdir, exist_ok=True)
            self._omega_out = open(os.path.join(outdir, "omega_scp1.dat"), mode)
            self._free_out = open(os.path.join(outdir, "free_energy.dat"), mode)

    # setters of SCP1.h:68-97
    def set_sobol_skip(self, s):
        self.sobol_skip = int(s)
        return self

    def set_epsrel(self, e):
        self.epsrel = float(e)
        return self

    def set_qeps(self, e):
        self.qeps = float(e)
        return self

    def set_cutoff(self, w):
        self.omega_cutoff = float(w)
        return self

    def close(self):
        for f in ("_omega_out", "_free_out"):
            if getattr(self, f, None):
                getattr(self, f).close()
                setattr(self, f, None)
        if self._gpu is not None:
            self._gpu.close()
            self._gpu = None

    def disp_disp_corr_diag(self, omega, kT):
        """Harmonic <dq^2> per mode, zero below the cutoff (SCP1.cpp:18-32)."""
        with np.errstate(divide="ignore", invalid="ignore"):
            if kT == 0.0:
                d = 0.5 / omega
            else:
                d = 0.5 / (omega * np.tanh(0.5 / kT * omega))
        d[omega < self.omega_cutoff] = 0.0
        return d

    def _allreduce(self, x):
        if self.nprocs == 1:
            return x
        import torch
        import torch.distributed as dist
        on_gpu = dist.get_backend() == "nccl"
        t = torch.from_numpy(np.ascontiguousarray(x))
        if on_gpu:
            t = t.to("cuda:%d" % torch.cuda.current_device())
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return t.cpu().numpy()

    def average(self, q, d, isqrtM_U):
        """(<V>, <UX>, <UX dq^T>) over NSobol points (SCP1.cpp:34-90)."""
        dim = q.size
        i0 = (self.rank * self.nsobol) // self.nprocs
        i1 = ((self.rank + 1) * self.nsobol) // self.nprocs
        if self._averager is not None:
            up, UX, UXq = self._averager(q, d, isqrtM_U, self.sobol_skip, i0, i1)
        else:
            if self._gpu is None:
                from .api import SCP1Average
                self._gpu = SCP1Average(self.pes, dim // 9, device=self.device)
            up, UX, UXq = self._gpu.sums(q, d, isqrtM_U, self.sobol_skip, i0, i1)
        packed = np.concatenate([[up], np.asarray(UX).ravel(), np.asarray(UXq).ravel(order="F")])
        packed = self._allreduce(packed)
        up = packed[0]
        UX = packed[1:1 + dim].copy()
        UXq = packed[1 + dim:].reshape((dim, dim), order="F").copy()
        return up / self.nsobol, UX / self.nsobol, UXq / self.nsobol

    def _isqrtM_U(self, U):
        return U / np.sqrt(self.mass)[:, None]

    def __call__(self, q, kT, Ks=None, max_iterations=200):
        """SCP1::operator() (SCP1.cpp:95-190): iterates max_iterations times (the
        reference computes a convergence flag and does not stop on it; it is kept
        in self.converged).  q (bohr) is updated in place; returns F (hartree);
        self.Ks, self.omega, self.Upot and self.UX hold the last iterate."""
        mass = self.mass
        if Ks is None or np.size(Ks) == 0:
            grad_fn = self._grad_fn
            if grad_fn is None:
                from .api import PES
                grad_fn = PES(self.pes).energies_grad
            Ks = get_hessian(grad_fn, q, 1e-3)
            mass_scale_hessian(mass, Ks)
            regtransrot(transrot_basis(q, mass), Ks)
        Ks = np.array(Ks, dtype=np.float64)
        omegasq, U = eig_sym(Ks)
        omega = np.sqrt(np.abs(omegasq))
        d = self.disp_disp_corr_diag(omega, kT)
        isqrtM_U = self._isqrtM_U(U)
        F = 0.0
        Upot, UX = 0.0, np.zeros(q.size)
        for niter in range(max_iterations):
            d_old = d.copy()
            q_old = q.copy()
            Upot, UX, UX_q = self.average(q, d, isqrtM_U)
            UX_q = UX_q * np.sqrt(mass[None, :] / mass[:, None])      # (j, i) *= sqrt(m_i / m_j)
            KD = UX_q @ U
            nz = d != 0.0
            KD[:, nz] /= d[nz]
            KD[:, ~nz] = 0.0
            Ks = KD @ U.T
            KD = Ks + Ks.T
            Ks = 0.5 * KD
            regtransrot(transrot_basis(q, mass), Ks)
            omegasq, U = eig_sym(Ks)
            isqrtM_U = self._isqrtM_U(U)
            omega = np.sqrt(np.abs(omegasq))
            d = self.disp_disp_corr_diag(omega, kT)
            q -= self.qeps * (isqrtM_U @ (d * (isqrtM_U.T @ UX)))
            self.converged = bool(np.all(np.abs(q - q_old) <= np.abs(q_old) * self.epsrel) and
                                  np.all(np.abs(d - d_old) <= np.abs(d_old) * self.epsrel))
            F = Upot
            we = omega[6:]
            if kT > 0.0:
                F += kT * np.sum(np.log(2.0 * np.sinh(0.5 / kT * we))) - 0.25 * np.sum(we / np.tanh(0.5 / kT * we))
            else:
                F += 0.25 * np.sum(we)
            self.iterations = niter + 1
            if self.rank == 0:
                self._omega_out.write(" ".join("%.10e" % w for w in omega) + "\n")
                self._omega_out.flush()
                self._free_out.write("%.17g\n" % F)
                self._free_out.flush()
                species = ["O", "H", "H"] * (q.size // 9)
                modes.write_input(os.path.join(self.outdir, "coord.xyz"), species, q, Ks,
                                  comment="Free energy = %.17g" % F)
                if self.verbose:
                    print("iter: %d" % niter)
        if self.rank == 0 and self.verbose:
            print("omega = " + " ".join("%.4f" % w for w in omega * C.autocm))
            print("<U> = %.17g" % Upot)
            print("<UX> = " + " ".join("%.6e" % x for x in UX))
            print("F = %.17g kcal/mol" % (F * C.autokcalpmol))
        self.Ks, self.omega, self.Upot, self.UX = Ks, omega, Upot, UX
        return F


def parse_args(argv):
    """SCP1_main.cpp:34-107 options (long names as the reference spells them)."""
    ap = argparse.ArgumentParser(prog="scp1", description=__doc__.split("\n\n")[0])
    ap.add_argument("-N", "--NSobol", type=int, default=20, help="NSobol = 2^N (N <= 32)")
    ap.add_argument("-S", "--skip", type=int, default=22, help="accepted; no effect, as in the reference")
    ap.add_argument("-r", "--rng-file", default=None, help="accepted; not read, as in the reference")
    ap.add_argument("-p", "--PES", default="qtip4pf")
    ap.add_argument("-L", "--max-itertions", dest="max_iterations", type=int, default=200)
    ap.add_argument("-c", "--cutoff", type=float, default=-1.0, help="frequency cutoff in cm^-1")
    ap.add_argument("input")
    a = ap.parse_args(argv)
    if a.NSobol > 32:
        ap.error("-N <N>: <N>is too large, NSobol = 2^<N>")
    if a.skip > 32:
        ap.error("-S <N>: <N>is too large, sobol_skip = 2^<N>")
    return a


def main(argv=None):
    a = parse_args(sys.argv[1:] if argv is None else argv)
    device = 0
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import datetime

        import torch
        import torch.distributed as dist
        device = int(os.environ.get("LOCAL_RANK", "0"))
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(device)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    species, mass, x0, H = modes.read_input(a.input)
    _, mass, x0, H = modes.ohhohh(mass, x0, H)
    scp1 = SCP1(mass, a.PES, 1 << a.NSobol, append=H is not None, device=device)
    if a.cutoff > 0:
        scp1.set_cutoff(a.cutoff / C.autocm)
    F0 = scp1(x0, 0.0, H, a.max_iterations)
    if scp1.rank == 0:
        print("F0 = %.17g" % F0)
    scp1.close()
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
