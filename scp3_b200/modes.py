"""Host-side normal-mode setup of the Hamiltonian build (numpy, FP64).

Mirrors the reference's input handling and mode construction:

* ``read_input``   -- ``load_from_vladimir`` (DiskIO.cpp:72-116): atom count, a
  comment line, ``El x y z`` in Angstrom (stored in bohr), then the upper
  triangle of the mass-weighted Hessian, column by column.  A missing Hessian
  leaves ``H`` as ``None`` (the reference resets it, DiskIO.cpp:104-108).
* ``write_input``  -- ``save_for_vladimir`` (DiskIO.cpp:118-140).
* ``ohhohh``       -- the O H H O H H reordering (DiskIO.cpp:142-195).
* ``normal_modes`` -- ``eig_sym`` of H, drop the six lowest, ``omega = sqrt``,
  ``MUa = U[:,6:] / (sqrt(mass) * sqrt(omega))`` (SCP3.cpp:296-314).
* ``parse_modes``  -- the ``-m "0-5,7"`` mode-list syntax (SCP3.cpp:63-89).
"""
import numpy as np

from . import constants as C


class InputError(ValueError):
    pass


def read_input(path):
    with open(path) as f:
        text = f.read().split("\n")
    try:
        n = int(text[0].split()[0])
    except (IndexError, ValueError):
        raise InputError("%s: first line must hold the atom count" % path)
    species, x0 = [], []
    for i in range(n):
        parts = text[2 + i].split()
        if len(parts) < 4:
            raise InputError("%s: atom line %d is truncated" % (path, i + 1))
        if parts[0] not in C.NUCLEAR_MASS:
            raise InputError("%s: unknown species %r" % (path, parts[0]))
        species.append(parts[0])
        x0.extend(float(v) for v in parts[1:4])
    mass = np.repeat([C.NUCLEAR_MASS[s] for s in species], 3).astype(np.float64)
    x0 = np.array(x0) / C.bohr
    vals = " ".join(text[2 + n:]).split()
    need = 3 * n * (3 * n + 1) // 2
    H = None
    if len(vals) >= need:
        H = np.zeros((3 * n, 3 * n))
        k = 0
        for i in range(3 * n):
            for j in range(i + 1):
                H[j, i] = H[i, j] = float(vals[k])
                k += 1
    return species, mass, x0, H


def write_input(path, species, x0_bohr, H, comment="Free energy = 0"):
    n = len(species)
    with open(path, "w") as f:
        f.write("%d\n%s\n" % (n, comment))
        for i, s in enumerate(species):
            r = x0_bohr[3 * i:3 * i + 3] * C.bohr
            f.write("%s %.17g %.17g %.17g\n" % (s, r[0], r[1], r[2]))
        for i in range(3 * n):
            for j in range(i + 1):
                f.write("%.17g\n" % H[j, i])


def ohhohh(mass, x0, H=None):
    """Permutation putting each O before its two H (DiskIO.cpp:142-195); returns
    (perm, mass, x0, H) with the permutation applied."""
    n3 = mass.size
    p = np.zeros(n3, dtype=np.int64)
    iO, iH, i = 0, 3, 0
    while i < n3:
        if mass[i] == C.Omass:
            p[iO:iO + 3] = np.arange(i, i + 3)
            iO += 9
        elif mass[i] in (C.Hmass, C.Dmass):
            p[iH:iH + 3] = np.arange(i, i + 3)
            iH += 3
            iH += 3 * (iH % 9 == 0)
        else:
            raise InputError("unknown mass at %d" % i)
        i += 3
    H2 = None if H is None else H[np.ix_(p, p)]
    return p, mass[p], x0[p], H2


def normal_modes(H, mass):
    """(omega[3N-6], MUa[3N x 3N-6], omegasq0[3N]) from the mass-weighted Hessian."""
    w2, U = np.linalg.eigh(H)
    n3 = mass.size
    omega = np.sqrt(w2[6:n3])
    MUa = U[:, 6:n3] / (np.sqrt(mass)[:, None] * np.sqrt(omega)[None, :])
    return omega, MUa, w2


def parse_modes(desc, nmodes=None):
    modes = []
    for part in desc.split(","):
        part = part.strip()
        if not part:
            continue
        if "-" in part[1:]:
            a, b = part.split("-", 1)
            modes.extend(range(int(a), int(b) + 1))
        else:
            modes.append(int(part))
    if nmodes is not None and any(m < 0 or m >= nmodes for m in modes):
        raise InputError("mode index out of range 0..%d" % (nmodes - 1))
    return np.array(modes, dtype=np.int32)


def basis_size(nm, n2, n3):
    """getBasisSize (ScaledMatrixElements.cpp:73-78)."""
    return 1 + nm + n2 * (n2 + 1) // 2 + n3 * (1 + n3) * (2 + n3) // 6


def sub_basis_size(nm, n2, n3, level):
    """getSubBasisSize (ScaledMatrixElements.cpp:81-99): ground through `level`-fold excitations."""
    s = 0
    if level >= 3:
        s += n3 * (1 + n3) * (2 + n3) // 6
    if level >= 2:
        s += n2 * (n2 + 1) // 2
    if level >= 1:
        s += nm
    if level >= 0:
        s += 1
    return s
