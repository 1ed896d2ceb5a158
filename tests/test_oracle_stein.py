"""The oracle of the gradient (default) path, pinned against the reference:
every formula of TripleExcitations.h, the qTIP4P/f gradient
(qtip4pf.cpp:252-397), the per-sample V and dV/dq of SCP3.cpp:205-223, and a
dimer matrix summed from the reference's formulas (tests/golden/stein_ref.npz,
made by make_golden.py from the reference's sources)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN


@pytest.fixture(scope="module")
def z():
    return np.load(os.path.join(GOLDEN, "stein_ref.npz"), allow_pickle=True)


def _parse(name, params):
    bra, ket = ("", name[2:]) if name.startswith("f_") else name.split("_f_")
    side = lambda t: [(params.index(tok[0]), int(tok[1])) for tok in t.split("_") if tok]
    return side(bra), side(ket)


def test_every_reference_formula(oracle_mod, z):
    q, V, Vq = z["q"], z["V"], z["Vq"]
    names, params = list(z["names"]), [p.split(",") for p in z["params"]]
    assert len(names) == 74
    for i, name in enumerate(names):
        pb, pk = _parse(name, params[i])
        a = z["args"][i]
        bra = [(int(a[p]), lv) for p, lv in pb]
        ket = [(int(a[p]), lv) for p, lv in pk]
        terms = np.array([oracle_mod.stein_term(q[s], V[s], Vq[s], bra, ket) for s in range(V.size)])
        ref = z["values"][i]
        assert abs(terms.sum() - ref) <= 1e-12 * max(1.0, np.abs(terms).sum()), (name, terms.sum(), ref)


def test_qtip4pf_gradient(oracle_mod, z):
    geoms = np.load(os.path.join(GOLDEN, "pes_ref.npz"), allow_pickle=True)["geoms"]
    for x, g_ref in zip(geoms, z["pes_geoms_grad"]):
        e, g = oracle_mod.qtip4pf_grad(np.asarray(x, dtype=np.float64))
        assert np.abs(g - g_ref).max() <= 1e-12 * max(1.0, np.abs(g_ref).max())


def test_dimer_gradient_path(oracle_mod, z):
    nm0 = z["dimer_omega"].size
    n2, n3 = int(z["dimer_n2"]), int(z["dimer_n3"])
    normals = oracle_mod.std_normals(nm0, 0, int(z["dimer_nsamples"]), scramble_seed=int(z["dimer_scramble_seed"]))
    q, v, vq = oracle_mod.samples_grad(2, z["dimer_x0"], z["dimer_MUa"], z["dimer_omega"], normals)
    assert np.array_equal(q, z["dimer_q"])
    assert np.abs(v - z["dimer_V"]).max() <= 1e-13
    assert np.abs(vq - z["dimer_Vq"]).max() <= 1e-12 * np.abs(z["dimer_Vq"]).max()
    M = oracle_mod.accumulate_stein(z["dimer_q"], z["dimer_V"], z["dimer_Vq"], n2, n3)
    nb = M.shape[0]
    got = M.T[np.tril_indices(nb)]        # upper triangle column by column, as the fixture stores it
    ref = z["dimer_M_upper"]
    assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max(), np.abs(got - ref).max()


def test_dimer_ttm3f_gradient_path_matrix(oracle_mod, z):
    """The same rule on V and dV/dq from the reference's TTM3-F E+g operator
    (ttm3f.cpp:325-720)."""
    n2, n3 = int(z["dimer_ttm3f_n2"]), int(z["dimer_ttm3f_n3"])
    M = oracle_mod.accumulate_stein(z["dimer_ttm3f_q"], z["dimer_ttm3f_V"], z["dimer_ttm3f_Vq"], n2, n3)
    got = M.T[np.tril_indices(M.shape[0])]
    ref = z["dimer_ttm3f_M_upper"]
    assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max()
