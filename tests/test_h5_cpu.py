"""The sM_*.h5 writer (scp3gpu_save_h5, host code) and its reader: layout of
save_hdf5 (DiskIO.cpp:201-227) -- dataset "M", dims {n_cols, n_rows} from
column-major memory, float32."""
import struct

import numpy as np


def test_h5_roundtrip_and_layout(tmp_path):
    from scp3_b200 import h5
    rng = np.random.default_rng(5)
    M = np.asfortranarray(rng.normal(size=(37, 23)))
    p = str(tmp_path / "sM_0131072.h5")
    h5.save(p, M)
    R = h5.load(p)
    assert R.shape == M.shape
    assert np.array_equal(R, M.astype(np.float32).astype(np.float64))
    buf = open(p, "rb").read()
    assert buf[:8] == b"\x89HDF\r\n\x1a\n"
    assert struct.unpack_from("<Q", buf, 40)[0] == len(buf)          # end-of-file address
    # the float32 payload is the column-major matrix, verbatim
    assert np.array_equal(np.frombuffer(buf[-M.size * 4:], "<f4"), M.T.ravel().astype(np.float32))


def test_h5_symmetric_mout(tmp_path):
    from scp3_b200 import h5
    A = np.random.default_rng(1).normal(size=(50, 50))
    M = np.asfortranarray(A + A.T)
    p = str(tmp_path / "m.h5")
    h5.save(p, M)
    assert np.allclose(h5.load(p), M, rtol=1e-7)
