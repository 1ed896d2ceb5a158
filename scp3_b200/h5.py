"""sM_*.h5 files: writing through the library (scp3gpu_save_h5, the layout of
save_hdf5, DiskIO.cpp:201-227) and reading them back (load_hdf5,
DiskIO.cpp:267-289) for the files this library writes: superblock v0, root
symbol table, dataset "M" with a contiguous float32 layout."""
import ctypes
import struct

import numpy as np

from . import _lib


def save(path, M):
    """Write the column-major matrix M (n_rows x n_cols) as dataset "M" (float32)."""
    M = np.asfortranarray(M, dtype=np.float64)
    _lib.check(_lib.lib().scp3gpu_save_h5(path.encode(), M.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                          M.shape[0], M.shape[1]))


def _messages(buf, oh):
    ver, _, nmsg, _, size = struct.unpack_from("<BBHII", buf, oh)
    if ver != 1:
        raise ValueError("object header version %d" % ver)
    p, out = oh + 16, {}
    for _ in range(nmsg):
        mtype, msize, _flags = struct.unpack_from("<HHB", buf, p)
        out[mtype] = buf[p + 8:p + 8 + msize]
        p += 8 + msize
    return out


def load(path):
    """Read dataset "M" back as an n_rows x n_cols float64 array (Fortran order)."""
    buf = open(path, "rb").read()
    if buf[:8] != b"\x89HDF\r\n\x1a\n" or buf[8] != 0:
        raise ValueError("not a version-0 HDF5 superblock")
    root_oh = struct.unpack_from("<Q", buf, 64)[0]
    st = _messages(buf, root_oh)[0x0011]
    btree, heap = struct.unpack_from("<QQ", st, 0)
    assert buf[heap:heap + 4] == b"HEAP" and buf[btree:btree + 4] == b"TREE"
    heap_data = struct.unpack_from("<Q", buf, heap + 24)[0]
    snod = struct.unpack_from("<Q", buf, btree + 24 + 8)[0]
    assert buf[snod:snod + 4] == b"SNOD"
    nsym = struct.unpack_from("<H", buf, snod + 6)[0]
    for k in range(nsym):
        name_off, oh = struct.unpack_from("<QQ", buf, snod + 8 + 40 * k)
        name = buf[heap_data + name_off:buf.index(b"\0", heap_data + name_off)].decode()
        if name == "M":
            break
    else:
        raise KeyError("dataset M not found")
    msgs = _messages(buf, oh)
    space, dtype, layout = msgs[0x0001], msgs[0x0003], msgs[0x0008]
    rank = space[1]
    dims = struct.unpack_from("<%dQ" % rank, space, 8)
    assert dtype[0] & 0x0F == 1 and struct.unpack_from("<I", dtype, 4)[0] == 4, "float32 expected"
    assert layout[0] == 3 and layout[1] == 1, "contiguous layout expected"
    addr, size = struct.unpack_from("<QQ", layout, 2)
    data = np.frombuffer(buf, dtype="<f4", count=size // 4, offset=addr).astype(np.float64)
    n_cols, n_rows = dims
    return data.reshape(n_cols, n_rows).T
