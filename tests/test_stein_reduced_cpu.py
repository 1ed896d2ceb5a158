"""The split gradient estimator's reduced functions, host side only.

The same-mode pair sums of the Stein estimator (ScaledMatrixElements.cpp:102-725)
become products when every function j exciting a mode m is, without its mode-m
factor, again a basis function red(j, m).  The library's table is checked here
against an independent restatement of the basis order of get_bra
(ScaledMatrixElements.cpp:870-930; ground, singles, h2, h1 h1 pairs, h3,
(h2 h1, h1 h2) pairs, h1 h1 h1 triples), and the basis is closed under removing a
factor whenever N3 <= N2."""
import ctypes
import itertools

import numpy as np
import pytest


def basis_factors(nm, n2, n3):
    """Each basis function as its (mode, level) factors, in the reference's order;
    the factor order is that of the library's descriptors."""
    f = [()]
    f += [((m, 1),) for m in range(nm)]
    f += [((m, 2),) for m in range(n2)]
    f += [((m, 1), (n, 1)) for m, n in itertools.combinations(range(n2), 2)]
    f += [((m, 3),) for m in range(n3)]
    for m, n in itertools.combinations(range(n3), 2):
        f += [((m, 2), (n, 1)), ((m, 1), (n, 2))]
    f += [((m, 1), (n, 1), (p, 1)) for m, n, p in itertools.combinations(range(n3), 3)]
    return f


@pytest.fixture(scope="module")
def reduced():
    from scp3_b200 import _lib
    L = _lib.lib()
    fn = L.scp3gpu_internal_reduced
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]

    def run(nm, n2, n3):
        nb = int(L.scp3gpu_basis_size(nm, n2, n3))
        red = np.full(3 * nb, -7, dtype=np.int32)
        closed = fn(nm, n2, n3, red.ctypes.data)
        return closed, red.reshape(nb, 3)

    return run


@pytest.mark.parametrize("nm,n2,n3", [(12, 12, 0), (12, 12, 4), (48, 48, 0), (48, 20, 6), (20, 20, 20),
                                      (48, 10, 6)])
def test_reduced_functions_match_the_basis_order(reduced, nm, n2, n3):
    closed, red = reduced(nm, n2, n3)
    funcs = basis_factors(nm, n2, n3)
    assert red.shape[0] == len(funcs)
    index = {tuple(sorted(f)): i for i, f in enumerate(funcs)}
    for j, f in enumerate(funcs):
        for a in range(3):
            if a < len(f):
                want = index.get(tuple(sorted(f[:a] + f[a + 1:])), -1)
                assert red[j, a] == want, (j, f, a)
            else:
                assert red[j, a] == -1
    assert closed == 1
    # the doubles basis: a pair reduces to a single, h1 and h2 to the ground function
    if n2 == nm and n3 == 0:
        assert np.all(red[1:1 + nm + n2, 0] == 0)


def test_basis_not_closed_when_triples_pass_doubles(reduced):
    """With N3 > N2 the (h2 h1) pairs of modes past N2 lose their h1 to an h2 the
    basis does not hold: the estimator then keeps its pair sums in FP64."""
    closed, red = reduced(12, 4, 6)
    assert closed == 0
    assert (red == -1).any()
