"""sM_*.h5 files through the library: save_hdf5 (DiskIO.cpp:201-227) as
scp3gpu_save_h5_layout -- the reference's chunked + deflate layout, or
contiguous -- and load_hdf5 (DiskIO.cpp:267-289) as scp3gpu_load_h5."""
import ctypes

import numpy as np

from . import _lib

_dp = ctypes.POINTER(ctypes.c_double)


def save(path, M, deflate=-1):
    """Write the column-major matrix M (n_rows x n_cols) as dataset "M" (float32):
    deflate=-1 contiguous, 0..9 chunked and deflated (the reference uses 6)."""
    M = np.asfortranarray(M, dtype=np.float64)
    _lib.check(_lib.lib().scp3gpu_save_h5_layout(str(path).encode(), M.ctypes.data_as(_dp), M.shape[0], M.shape[1],
                                                 int(deflate)))


def load(path):
    """Dataset "M" as an n_rows x n_cols float64 array (Fortran order)."""
    r, c = ctypes.c_int64(), ctypes.c_int64()
    L = _lib.lib()
    _lib.check(L.scp3gpu_load_h5(str(path).encode(), None, ctypes.byref(r), ctypes.byref(c)))
    M = np.zeros((r.value, c.value), order="F")
    _lib.check(L.scp3gpu_load_h5(str(path).encode(), M.ctypes.data_as(_dp), ctypes.byref(r), ctypes.byref(c)))
    return M
