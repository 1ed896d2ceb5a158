"""The four-sample qTIP4P/f kernels take one item per (water pair, sample): the
decode of pair index p into waters a < b, host side only.  Every unordered pair
of waters must appear once, in the row-major order of the reference's pair loops
(qtip4pf.cpp:213-283, `for i < nw: for j > i`); the ten site pairs formed for each
water pair are checked through the energies of the GPU parity tests."""
import ctypes
import itertools

import numpy as np
import pytest


@pytest.fixture(scope="module")
def water_pairs():
    from scp3_b200 import _lib
    L = _lib.lib()
    f = L.scp3gpu_internal_water_pairs
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_void_p]

    def run(nw):
        np_ = nw * (nw - 1) // 2
        ab = np.full((max(np_, 1), 2), -1, dtype=np.int32)
        assert f(nw, ab.ctypes.data) == 0
        return [tuple(int(x) for x in r) for r in ab[:np_]]

    return run


@pytest.mark.parametrize("nw", list(range(1, 17)) + [33, 64])
def test_every_water_pair_once_in_loop_order(water_pairs, nw):
    assert water_pairs(nw) == list(itertools.combinations(range(nw), 2))


def test_rejects_bad_arguments():
    from scp3_b200 import _lib
    f = _lib.lib().scp3gpu_internal_water_pairs
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_void_p]
    buf = np.zeros(8, dtype=np.int32)
    assert f(0, buf.ctypes.data) != 0
    assert f(3, None) != 0
