"""The synthetic inputs of the benchmark configurations, in the reference's
input-file format (DiskIO.cpp:72-116), built with this package's GPU
potentials and cached under scp3_b200/data/.

  dimer_qtip4pf   two waters, r(OH) 0.96 A, HOH 104.5 deg, O-O 2.9 A, linear
                  donor-acceptor, relaxed on qTIP4P/f: 12 modes
  prism_qtip4pf   six waters on a triangular prism with 2.8 A edges, relaxed on
                  qTIP4P/f: 48 modes
  prism_ttm3f     the same start relaxed on TTM3-F
  cluster_<n>_<seed>  seeded random n-water cluster relaxed on qTIP4P/f

batch_clusters() assembles the batched-build workload from cluster_<n>_<seed>
inputs.
"""
import os

import numpy as np

from . import clusters, constants as C, modes

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


def _start(name):
    if name.startswith("dimer"):
        return clusters.dimer()
    if name.startswith("prism"):
        return clusters.prism()
    if name.startswith("cluster_"):
        _, n, seed = name.split("_")[:3]
        return clusters.random_cluster(int(n), int(seed))
    raise ValueError("unknown input %r" % name)


def _pes_of(name):
    return "ttm3f" if name.endswith("ttm3f") else "qtip4pf"


def build_input(name, path=None, energy=None):
    """Relax the starting geometry of `name` and write its input file."""
    from .api import PES
    x = _start(name)
    nw = x.size // 9
    mass = np.tile(np.repeat([C.Omass, C.Hmass, C.Hmass], 3), nw)
    if energy is None and _pes_of(name) == "qtip4pf" and name.startswith("cluster_"):
        # analytic gradients of the GPU potential: L-BFGS and a gradient-difference Hessian
        eg = PES("qtip4pf").energies_grad
        xr, e, g, it = clusters.relax_grad(eg, x)
        H, x0 = clusters.hessian_grad(eg, xr, mass)
    else:
        en = energy or PES(_pes_of(name)).energies
        xr, e, g, it = clusters.relax(en, x)
        H, x0 = clusters.hessian(en, xr, mass)
    species = ["O", "H", "H"] * nw
    path = path or os.path.join(DATA, name + ".dat")
    os.makedirs(os.path.dirname(path), exist_ok=True)
    modes.write_input(path, species, x0, H, comment="E = %.12f kcal/mol, |g|max = %.2e, %s" % (e, g, _pes_of(name)))
    return path


def load(name, build_if_missing=True):
    """(nw, x0 bohr, MUa, omega) of input `name`: read, reorder O H H, normal modes."""
    path = os.path.join(DATA, name + ".dat")
    if not os.path.exists(path):
        if not build_if_missing:
            raise FileNotFoundError(path)
        build_input(name, path)
    species, mass, x0, H = modes.read_input(path)
    _, mass, x0, H = modes.ohhohh(mass, x0, H)
    omega, MUa, _ = modes.normal_modes(H, mass)
    return x0.size // 9, x0, MUa, omega


def batch_clusters(count=32, seed=7, max_modes=42, min_omega_cm1=20.0, build_if_missing=True):
    """The batched-build workload: `count` clusters, n drawn uniformly from 2..8
    waters (numpy generator seeded with `seed`), each a seeded random placement
    relaxed on qTIP4P/f (input cluster_<n>_<s>, s = 100 * i + t); a placement
    whose relaxed Hessian has a frequency below min_omega_cm1 or an imaginary one
    (a saddle point or an unconverged relaxation) is replaced by the next t.
    Active modes: the max_modes highest-frequency modes (every mode up to five
    waters), N2 = all active modes, no triples -- 12..42 modes and doubles bases
    of 91..946 functions.  Returns a list of dicts for scp3_b200.Batch (plus
    'name')."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(2, 9, size=count)
    out = []
    for i, n in enumerate(ns):
        for t in range(100):
            name = "cluster_%d_%d" % (n, 100 * i + t)
            nw, x0, MUa, omega = load(name, build_if_missing)
            if np.all(np.isfinite(omega)) and omega.min() * C.autocm >= min_omega_cm1:
                break
        else:
            raise RuntimeError("no valid placement for cluster %d" % i)
        nm0 = omega.size
        nm = min(nm0, max_modes)
        modes = np.arange(nm0 - nm, nm0, dtype=np.int32)    # normal modes come in ascending frequency
        out.append(dict(name=name, nw=nw, x0=x0, MUa=MUa, omega=omega, modes=modes, n2=nm, n3=0))
    return out
