"""The split contraction's 128 x 256 tiling, host side only: every needed
128 x 128 block of the upper triangle is owned by exactly one tile half, as
itself or transposed, and the tiles are as few as the triangle allows,
ceil(n (n + 1) / 4) for n panels before the wave-filling splits."""
import ctypes

import numpy as np
import pytest


@pytest.fixture(scope="module")
def tiling():
    from scp3_b200 import _lib
    L = _lib.lib()
    f = L.scp3gpu_internal_tiling
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                  ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]

    def run(n, sms):
        nt_, ns_ = ctypes.c_int(), ctypes.c_int()
        assert f(n, sms, ctypes.byref(nt_), ctypes.byref(ns_), None, 0, None) == 0
        nt = (n + 1) // 2 * 2
        tiles = np.zeros((nt_.value, 3), dtype=np.int32)
        owner = np.zeros(nt * nt, dtype=np.int32)
        assert f(n, sms, ctypes.byref(nt_), ctypes.byref(ns_), tiles.ctypes.data, tiles.shape[0],
                 owner.ctypes.data) == 0
        return tiles, owner.reshape(nt, nt), ns_.value

    return run


@pytest.mark.parametrize("sms", [148, 132, 7])
def test_every_block_owned_once_by_a_matching_half(tiling, sms):
    for n in list(range(1, 41)) + [163]:
        tiles, owner, nsplit = tiling(n, sms)
        assert 1 <= nsplit <= 16
        fewest = (n * (n + 1) + 3) // 4
        assert fewest <= tiles.shape[0] <= 2 * fewest, (n, tiles.shape[0])
        used = set()
        for i in range(owner.shape[0]):
            for j in range(owner.shape[1]):
                o = owner[i, j]
                if i > j or j >= n:
                    assert o == -1, (n, i, j, o)
                    continue
                assert o >= 0, (n, i, j)
                t, tr, h = o >> 2, (o >> 1) & 1, o & 1
                a, b = tiles[t, 0], tiles[t, 1 + h]
                assert (a, b) == ((j, i) if tr else (i, j)), (n, i, j, tiles[t], tr, h)
                assert tr == 0 or i != j
                assert (t, h) not in used
                used.add((t, h))
        assert np.all(tiles >= 0) and np.all(tiles < n)


def test_hexamer_doubles_basis_takes_28_tiles(tiling):
    # Nb = 1225: ten panels, 55 needed blocks; aligned column pairs took 30 tiles
    tiles, owner, nsplit = tiling(10, 1 << 20)
    assert tiles.shape[0] == 28
