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


def _py_read_chunked(buf):
    """An independent pure-Python walk of the chunked dataset: object header
    messages, the raw-data chunk B-tree, zlib inflation of every chunk."""
    import zlib
    root_oh = struct.unpack_from("<Q", buf, 64)[0]

    def msgs(oh):
        n = struct.unpack_from("<H", buf, oh + 2)[0]
        p, out = oh + 16, {}
        for _ in range(n):
            t, sz = struct.unpack_from("<HH", buf, p)
            out[t] = buf[p + 8:p + 8 + sz]
            p += 8 + sz
        return out

    st = msgs(root_oh)[0x0011]
    btree, heap = struct.unpack_from("<QQ", st)
    snod = struct.unpack_from("<Q", buf, btree + 32)[0]
    oh = struct.unpack_from("<Q", buf, snod + 16)[0]
    m = msgs(oh)
    dims = struct.unpack_from("<2Q", m[0x0001], 8)
    lay = m[0x0008]
    assert lay[0] == 3 and lay[1] == 2 and lay[2] == 3
    root = struct.unpack_from("<Q", lay, 3)[0]
    c0, c1, es = struct.unpack_from("<3I", lay, 11)
    filt = m[0x000B]
    fid, _, _, ncv, level = struct.unpack_from("<HHHHI", filt, 8)
    chunks = []

    def walk(node):
        assert buf[node:node + 4] == b"TREE" and buf[node + 4] == 1
        lvl, used = buf[node + 5], struct.unpack_from("<H", buf, node + 6)[0]
        for e in range(used):
            k = node + 24 + e * 40
            size, mask, col = struct.unpack_from("<IIQ", buf, k)
            child = struct.unpack_from("<Q", buf, k + 32)[0]
            if lvl:
                walk(child)
            else:
                chunks.append((col, zlib.decompress(buf[child:child + size])))
        return lvl

    depth = walk(root)
    n_cols, n_rows = dims
    out = np.zeros(n_cols * n_rows, dtype=np.float32)
    for col, raw in chunks:
        a = np.frombuffer(raw, "<f4")
        assert a.size == c0 * c1
        ncols = min(c0, n_cols - col)
        out[col * n_rows:(col + ncols) * n_rows] = a[:ncols * n_rows]
    return out.reshape(n_cols, n_rows).T, dict(c0=c0, c1=c1, es=es, fid=fid, ncv=ncv, level=level, depth=depth,
                                                nchunks=len(chunks))


def test_h5_chunked_deflate_layout(tmp_path):
    """The reference's storage (DiskIO.cpp:211-216): chunks of whole columns,
    min(n_cols, ceil(131072 / n_rows)) wide, deflate level 6; 69 chunks, so the
    chunk B-tree has two levels and the last chunk is partial."""
    from scp3_b200 import h5
    rng = np.random.default_rng(9)
    n_rows, n_cols = 8192, 1100
    M = np.asfortranarray(rng.normal(size=(n_rows, n_cols)))
    p = str(tmp_path / "sM_0262144.h5")
    h5.save(p, M, deflate=6)
    want = M.astype(np.float32).astype(np.float64)
    assert np.array_equal(h5.load(p), want)
    R, info = _py_read_chunked(open(p, "rb").read())
    assert np.array_equal(R.astype(np.float64), want)
    assert info == dict(c0=16, c1=n_rows, es=4, fid=1, ncv=1, level=6, depth=1, nchunks=69)


def test_h5_small_chunked_and_reader_errors(tmp_path):
    from scp3_b200 import h5, SCP3GPUError
    import pytest
    M = np.asfortranarray(np.arange(12.0).reshape(3, 4))
    p = str(tmp_path / "a.h5")
    h5.save(p, M, deflate=1)      # one chunk holding the whole matrix
    assert np.array_equal(h5.load(p), M)
    bad = tmp_path / "bad.h5"
    bad.write_bytes(b"not hdf5" * 20)
    with pytest.raises(SCP3GPUError):
        h5.load(str(bad))
    with pytest.raises(SCP3GPUError):
        h5.load(str(tmp_path / "missing.h5"))
