"""The learned control variate (no counterpart in the reference).

MLP wraps the library's network (scp3gpu_mlp_*): 48 -> 256 -> 256 -> 256 -> 1,
GELU, BF16 weights, FP32 accumulation, trained on the GPU by the library's own
forward/backward/Adam kernels.  control_variate() forms

    M_cv = (1/N_a) sum_{a} V_nn(q_a) Phi Phi^T  +  (1/N_b) sum_{b} (V - V_nn)(q_b) Phi Phi^T

with the surrogate over N_a Sobol points and the exact residual over N_b
points from a disjoint index range, both through the split contraction."""
import ctypes

import numpy as np

from . import _lib
from .api import HBuild

_fp = ctypes.POINTER(ctypes.c_float)


def _f(a):
    return a.ctypes.data_as(_fp)


def _bind():
    L = _lib.lib()
    if getattr(L, "_mlp_bound", False):
        return L
    vp, i64 = ctypes.c_void_p, ctypes.c_int64
    L.scp3gpu_mlp_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_int,
                                     ctypes.POINTER(vp)]
    L.scp3gpu_mlp_destroy.argtypes = [vp]
    L.scp3gpu_mlp_num_params.restype = i64
    L.scp3gpu_mlp_num_params.argtypes = [vp]
    L.scp3gpu_mlp_get_params.argtypes = [vp, _fp, i64]
    L.scp3gpu_mlp_set_params.argtypes = [vp, _fp, i64]
    L.scp3gpu_mlp_set_output.argtypes = [vp, ctypes.c_float, ctypes.c_float]
    L.scp3gpu_mlp_forward.argtypes = [vp, _fp, i64, _fp]
    L.scp3gpu_mlp_grad.argtypes = [vp, _fp, _fp, ctypes.c_int, _fp, _fp]
    L.scp3gpu_mlp_train.argtypes = [vp, _fp, _fp, i64, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_uint64,
                                    _fp]
    L.scp3gpu_hbuild_set_surrogate.argtypes = [vp, vp, ctypes.c_int]
    L.scp3gpu_hbuild_sample.argtypes = [vp, i64, i64, _fp, ctypes.POINTER(ctypes.c_double)]
    L._mlp_bound = True
    return L


SURROGATE_NONE, SURROGATE_REPLACE, SURROGATE_RESIDUAL = 0, 1, 2


class MLP:
    def __init__(self, n_in, hidden=256, max_batch=1 << 18, seed=1, device=0):
        L = _bind()
        h = ctypes.c_void_p()
        _lib.check(L.scp3gpu_mlp_create(n_in, hidden, max_batch, seed, device, ctypes.byref(h)))
        self._h, self.n_in, self.hidden = h, n_in, hidden

    def close(self):
        if getattr(self, "_h", None):
            _bind().scp3gpu_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def num_params(self):
        return int(_bind().scp3gpu_mlp_num_params(self._h))

    def get_params(self):
        p = np.zeros(self.num_params(), dtype=np.float32)
        _lib.check(_bind().scp3gpu_mlp_get_params(self._h, _f(p), p.size))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _lib.check(_bind().scp3gpu_mlp_set_params(self._h, _f(p), p.size))

    def set_output(self, scale, shift):
        _lib.check(_bind().scp3gpu_mlp_set_output(self._h, scale, shift))

    def __call__(self, q):
        q = np.ascontiguousarray(q, dtype=np.float32)
        y = np.zeros(q.shape[0], dtype=np.float32)
        _lib.check(_bind().scp3gpu_mlp_forward(self._h, _f(q), q.shape[0], _f(y)))
        return y

    def loss_and_grad(self, q, t):
        q = np.ascontiguousarray(q, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        g = np.zeros(self.num_params(), dtype=np.float32)
        _lib.check(_bind().scp3gpu_mlp_grad(self._h, _f(q), _f(t), q.shape[0], _f(loss), _f(g)))
        return float(loss[0]), g

    def fit(self, q, t, epochs=30, batch=4096, lr=2e-3, seed=7):
        """Normalise the targets (mean/std), then Adam on the MSE; returns the last batch loss."""
        q = np.ascontiguousarray(q, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        self.set_output(float(t.std()) or 1.0, float(t.mean()))
        loss = np.zeros(1, dtype=np.float32)
        _lib.check(_bind().scp3gpu_mlp_train(self._h, _f(q), _f(t), q.shape[0], epochs, batch, lr, seed, _f(loss)))
        return float(loss[0])


def sample(hb, index0, n):
    """(q n x nmodes float32, V_anh n float64) of points index0.. through the build's per-sample stage."""
    L = _bind()
    q = np.zeros((n, hb.modes.size), dtype=np.float32)
    v = np.zeros(n)
    _lib.check(L.scp3gpu_hbuild_sample(hb._h, index0, n, _f(q), v.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return q, v


def attach(hb, net, mode):
    """Attach the network to a split-form build: SURROGATE_REPLACE (V_nn for V)
    or SURROGATE_RESIDUAL (V - V_nn); SURROGATE_NONE detaches."""
    _lib.check(_bind().scp3gpu_hbuild_set_surrogate(hb._h, net.handle if net is not None else None, mode))


def control_variate(make_build, net, n_replace, n_residual, index_replace, index_residual):
    """Raw control-variate matrix M_cv (the estimate of sum V Phi Phi^T / N) from two
    builds made by make_build(): the surrogate alone over n_replace points and the
    exact residual over n_residual points."""
    L = _bind()
    out = []
    for mode, i0, n in ((SURROGATE_REPLACE, index_replace, n_replace), (SURROGATE_RESIDUAL, index_residual, n_residual)):
        hb = make_build()
        _lib.check(L.scp3gpu_hbuild_set_surrogate(hb._h, net.handle, mode))
        hb.accumulate(i0, n)
        out.append(hb.read(0) / n)
        hb.close()
    return out[0] + out[1]
