"""Water-cluster inputs for the Hamiltonian build: starting geometries, a
minimiser and a finite-difference Hessian.

The reference reads pre-relaxed geometries and Hessians from files
(DiskIO.cpp:72-116; isomers/README:1-2 says they were optimised elsewhere), so
it has no minimiser.  This module makes the synthetic inputs the benchmarks
need: it takes any batched energy function ``energy(X) -> E`` (X: n x 9nw in
Angstrom, O H H order; E in kcal/mol) -- the product passes the GPU potential
-- and returns geometries and mass-weighted Hessians in atomic units.

Units: the Hessian is built from energies in hartree and displacements in bohr,
then mass-weighted (Hessian.cpp:45-55), so ``eig`` gives omega^2 in hartree^2.
(The reference's own ``getHessian``, Hessian.cpp:33, divides kcal/mol/Angstrom
gradient differences by 2 s autokcalpmol without the Angstrom->bohr factor; SCP3
never calls it, and this module uses consistent atomic units instead.)
"""
import numpy as np

from . import constants as C


def water(r=0.96, theta_deg=104.5):
    """One H2O in its own frame: O at the origin, bisector along +y, in the xy plane."""
    t = np.deg2rad(theta_deg) / 2
    return np.array([[0, 0, 0], [r * np.sin(t), r * np.cos(t), 0], [-r * np.sin(t), r * np.cos(t), 0]])


def _rot(axis, ang):
    axis = np.asarray(axis, float) / np.linalg.norm(axis)
    K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * K @ K


def _place(w, O, donate_dir=None, rng=None):
    """Rotate water `w` so that H1 points along donate_dir (or randomly), O at O."""
    w = w - w[0]
    if donate_dir is None:
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        a, b, c, d = q
        R = np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                      [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                      [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])
        return O + w @ R.T
    h1 = w[1] / np.linalg.norm(w[1])
    t = np.asarray(donate_dir, float) / np.linalg.norm(donate_dir)
    v = np.cross(h1, t)
    s = np.linalg.norm(v)
    R = np.eye(3) if s < 1e-12 else _rot(v, np.arctan2(s, h1 @ t))
    w = w @ R.T
    # spin about the O-H1 bond by a seeded angle so H2 is not degenerate
    if rng is not None:
        w = w @ _rot(t, rng.uniform(0, 2 * np.pi)).T
    return O + w


def dimer(roo=2.9, r=0.96, theta_deg=104.5):
    """Linear donor-acceptor water dimer: donor O-H along +x to the acceptor O at
    distance roo; the acceptor's bisector points away from the donor along +x,
    its plane perpendicular to the donor's."""
    w = water(r, theta_deg)
    t = np.deg2rad(theta_deg) / 2
    # donor: H1 on +x
    donor = np.array([[0, 0, 0], [r, 0, 0], [r * np.cos(2 * t), r * np.sin(2 * t), 0]])
    acc = np.array([[roo, 0, 0],
                    [roo + r * np.cos(t), 0, r * np.sin(t)],
                    [roo + r * np.cos(t), 0, -r * np.sin(t)]])
    del w
    return np.concatenate([donor, acc]).ravel()


def prism(edge=2.8, r=0.96, theta_deg=104.5, seed=0):
    """Six waters with their oxygens on the vertices of a triangular prism of
    edge `edge` (two equilateral triangles a distance `edge` apart).  Each water
    donates its first H along a prism edge (a cyclic pattern on each triangle and
    up/down along the vertical edges alternately); the rest is seeded."""
    rng = np.random.default_rng(seed)
    rc = edge / np.sqrt(3)
    O = []
    for z in (-edge / 2, edge / 2):
        for k in range(3):
            a = 2 * np.pi * k / 3
            O.append([rc * np.cos(a), rc * np.sin(a), z])
    O = np.array(O)
    target = [1, 2, 0, 0, 3, 4]          # bottom ring cyclic; top: one down, two around the ring
    w = water(r, theta_deg)
    out = [_place(w, O[i], O[target[i]] - O[i], rng) for i in range(6)]
    return np.concatenate(out).ravel()


def random_cluster(nw, seed, r=0.96, theta_deg=104.5, roo=2.8):
    """Seeded random placement of nw waters: oxygens grown one at a time at
    distance ~roo from a random earlier oxygen, rejecting clashes (< 2.5 A)."""
    rng = np.random.default_rng(seed)
    O = [np.zeros(3)]
    while len(O) < nw:
        base = O[rng.integers(len(O))]
        d = rng.normal(size=3)
        cand = base + roo * d / np.linalg.norm(d)
        if min(np.linalg.norm(cand - o) for o in O) >= 2.5:
            O.append(cand)
    w = water(r, theta_deg)
    out = []
    for i in range(nw):
        others = [j for j in range(nw) if j != i]
        j = min(others, key=lambda j: np.linalg.norm(O[j] - O[i])) if others else None
        out.append(_place(w, O[i], None if j is None else O[j] - O[i], rng))
    return np.concatenate(out).ravel()


def _fd_grad(energy, x, h):
    n = x.size
    X = np.repeat(x[None, :], 2 * n, axis=0)
    idx = np.arange(n)
    X[2 * idx, idx] += h
    X[2 * idx + 1, idx] -= h
    E = energy(X)
    return (E[0::2] - E[1::2]) / (2 * h)


def relax(energy, x, gtol=1e-7, maxiter=2000, h=1e-5):
    """Quasi-Newton (BFGS, backtracking line search) minimisation with central
    finite-difference gradients.  x in Angstrom; returns (x, E, |g|max, iters)."""
    x = np.array(x, dtype=np.float64)
    n = x.size
    Hinv = np.eye(n) * 1e-3
    e = float(energy(x[None, :])[0])
    g = _fd_grad(energy, x, h)
    it = 0
    for it in range(maxiter):
        if np.abs(g).max() < gtol:
            break
        p = -Hinv @ g
        if p @ g >= 0:
            Hinv = np.eye(n) * 1e-3
            p = -Hinv @ g
        step = 1.0
        while True:
            xn = x + step * p
            en = float(energy(xn[None, :])[0])
            if en <= e + 1e-4 * step * (p @ g) or step < 1e-10:
                break
            step *= 0.5
        gn = _fd_grad(energy, xn, h)
        s, y = xn - x, gn - g
        sy = s @ y
        if sy > 1e-14:
            rho = 1.0 / sy
            I = np.eye(n)
            Hinv = (I - rho * np.outer(s, y)) @ Hinv @ (I - rho * np.outer(y, s)) + rho * np.outer(s, s)
        x, e, g = xn, en, gn
    return x, e, float(np.abs(g).max()), it


def _transrot_basis(x_bohr, mass):
    """Orthonormal mass-weighted translation/rotation vectors (cf. Hessian.cpp:57-130)."""
    n = x_bohr.size // 3
    r = x_bohr.reshape(n, 3)
    m = mass.reshape(n, 3)[:, 0]
    com = (m[:, None] * r).sum(0) / m.sum()
    r = r - com
    sm = np.sqrt(m)
    B = []
    for k in range(3):
        v = np.zeros((n, 3))
        v[:, k] = sm
        B.append(v.ravel())
    for k in range(3):
        e = np.zeros(3)
        e[k] = 1
        v = np.cross(e[None, :], r) * sm[:, None]
        B.append(v.ravel())
    B = np.array(B).T
    Q, R = np.linalg.qr(B)
    keep = np.abs(np.diag(R)) > 1e-8
    return Q[:, keep]


def hessian(energy, x_angstrom, mass, h=1e-3):
    """Mass-weighted Hessian in atomic units at x (Angstrom), from central
    second differences of the energy with step h (bohr), with translations and
    rotations projected out.  Returns (H, x0_bohr)."""
    xb = np.asarray(x_angstrom, dtype=np.float64) / C.bohr
    n = xb.size
    idx = [(i, j) for i in range(n) for j in range(i, n)]
    X = np.zeros((4 * len(idx), n))
    for k, (i, j) in enumerate(idx):
        for t, (si, sj) in enumerate(((1, 1), (1, -1), (-1, 1), (-1, -1))):
            v = xb.copy()
            v[i] += si * h
            v[j] += sj * h
            X[4 * k + t] = v
    E = energy(X * C.bohr) / C.autokcalpmol
    K = np.zeros((n, n))
    for k, (i, j) in enumerate(idx):
        e = E[4 * k:4 * k + 4]
        K[i, j] = K[j, i] = (e[0] - e[1] - e[2] + e[3]) / (4 * h * h)
    ism = 1.0 / np.sqrt(mass)
    H = K * ism[:, None] * ism[None, :]
    T = _transrot_basis(xb, mass)
    P = np.eye(n) - T @ T.T
    H = P @ H @ P
    return 0.5 * (H + H.T), xb


def relax_grad(energy_grad, x, gtol=1e-7, maxiter=5000):
    """Minimisation with analytic gradients: ``energy_grad(X) -> (E, G)`` for a
    batch X (n x 9nw, Angstrom; kcal/mol, kcal/mol/A).  L-BFGS (scipy), then the
    same |g|max test as relax().  Returns (x, E, |g|max, iterations)."""
    from scipy.optimize import minimize
    x = np.array(x, dtype=np.float64)

    def fg(v):
        E, G = energy_grad(v[None, :])
        return float(E[0]), G[0]

    res = minimize(fg, x, jac=True, method="L-BFGS-B",
                   options=dict(maxiter=maxiter, gtol=gtol, ftol=1e-15, maxcor=50))
    e, g = fg(res.x)
    return res.x, e, float(np.abs(g).max()), int(res.nit)


def hessian_grad(energy_grad, x_angstrom, mass, h=1e-4):
    """As hessian(), from central differences of analytic gradients (step h bohr):
    one batch of 2n gradient evaluations."""
    xb = np.asarray(x_angstrom, dtype=np.float64) / C.bohr
    n = xb.size
    X = np.repeat(xb[None, :], 2 * n, axis=0)
    idx = np.arange(n)
    X[2 * idx, idx] += h
    X[2 * idx + 1, idx] -= h
    _, G = energy_grad(X * C.bohr)
    G = G * C.bohr / C.autokcalpmol                  # hartree / bohr
    K = (G[0::2] - G[1::2]) / (2 * h)
    K = 0.5 * (K + K.T)
    ism = 1.0 / np.sqrt(mass)
    H = K * ism[:, None] * ism[None, :]
    T = _transrot_basis(xb, mass)
    P = np.eye(n) - T @ T.T
    H = P @ H @ P
    return 0.5 * (H + H.T), xb
