"""ctypes binding of libscp3gpu.so (the C ABI of include/scp3gpu.h).

The library is built in-tree (``scp3_b200/libscp3gpu.so``) by ``build()``; there
is no fallback: if it is missing or fails to load, every call raises.
"""
import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libscp3gpu.so")

OK, ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_NOT_CONVERGED, ERR_NONFINITE, ERR_TIMEOUT, ERR_UNSUPPORTED = range(8)
PREC_FP64, PREC_BF16X3, PREC_BF16X3_PES64, PREC_F16X3, PREC_F16X3_PES64 = 0, 1, 2, 3, 4
SOBOL_REFERENCE, SOBOL_SCRAMBLED = 0, 1
BATCH_NO_GRAPH, BATCH_NO_AUTOTUNE = 1, 2
ESTIMATOR_DIRECT, ESTIMATOR_GRADIENT = 0, 1

# every symbol include/scp3gpu.h declares (checked by the CPU tests)
EXPORTS = [
    "scp3gpu_last_error", "scp3gpu_version", "scp3gpu_pes_energy", "scp3gpu_pes_energy_dev", "scp3gpu_pes_energy_grad",
    "scp3gpu_sobol_std_normal", "scp3gpu_basis_size", "scp3gpu_sub_basis_size", "scp3gpu_hbuild_create",
    "scp3gpu_hbuild_destroy", "scp3gpu_hbuild_reset", "scp3gpu_hbuild_basis_size", "scp3gpu_hbuild_stream",
    "scp3gpu_hbuild_accumulate", "scp3gpu_hbuild_accumulate_normals", "scp3gpu_hbuild_accumulate_normals_f32",
    "scp3gpu_hbuild_add_epot", "scp3gpu_hbuild_sample_count", "scp3gpu_hbuild_read", "scp3gpu_hbuild_read_dev", "scp3gpu_hbuild_eigvals", "scp3gpu_hbuild_status",
    "scp3gpu_hbuild_profile", "scp3gpu_add_epot_static", "scp3gpu_save_h5", "scp3gpu_save_h5_layout",
    "scp3gpu_load_h5", "scp3gpu_syevr_lowest",
    "scp3gpu_mlp_create", "scp3gpu_mlp_destroy", "scp3gpu_mlp_num_params", "scp3gpu_mlp_get_params",
    "scp3gpu_mlp_set_params", "scp3gpu_mlp_set_output", "scp3gpu_mlp_forward", "scp3gpu_mlp_grad", "scp3gpu_mlp_train",
    "scp3gpu_hbuild_set_surrogate", "scp3gpu_hbuild_sample", "scp3gpu_hbuild_add_epot_grad",
    "scp3gpu_batch_create", "scp3gpu_batch_destroy", "scp3gpu_batch_reset", "scp3gpu_batch_size",
    "scp3gpu_batch_basis_size", "scp3gpu_batch_sample_count", "scp3gpu_batch_stream", "scp3gpu_batch_shape",
    "scp3gpu_batch_accumulate", "scp3gpu_batch_read", "scp3gpu_batch_status",
    "scp3gpu_scp1_create", "scp3gpu_scp1_average", "scp3gpu_scp1_status", "scp3gpu_scp1_destroy",
]


class SCP3GPUError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("scp3gpu error %d: %s" % (code, msg))
        self.code = code


class Config(ctypes.Structure):
    _fields_ = [
        ("nw", ctypes.c_int), ("nmodes0", ctypes.c_int),
        ("x0", ctypes.POINTER(ctypes.c_double)), ("MUa", ctypes.POINTER(ctypes.c_double)),
        ("omega", ctypes.POINTER(ctypes.c_double)),
        ("nmodes", ctypes.c_int), ("modes", ctypes.POINTER(ctypes.c_int)),
        ("n2", ctypes.c_int), ("n3", ctypes.c_int), ("pes", ctypes.c_int), ("precision", ctypes.c_int),
        ("scramble", ctypes.c_int), ("scramble_seed", ctypes.c_uint64), ("chunk", ctypes.c_int),
        ("device", ctypes.c_int), ("estimator", ctypes.c_int),
    ]


def build(force=False):
    """Compile libscp3gpu.so for sm_100a with nvcc (make in csrc/)."""
    args = ["make", "-s", "-C", os.path.join(HERE, "csrc"), "-j8"]
    if force:
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "csrc"), "clean"], check=True)
    subprocess.run(args, check=True)


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise SCP3GPUError(ERR_UNSUPPORTED, "libscp3gpu.so is not built (run scp3_b200._lib.build())")
    L = ctypes.CDLL(LIB_PATH)
    dp, ip, vp = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), ctypes.c_void_p
    i64 = ctypes.c_int64
    L.scp3gpu_last_error.restype = ctypes.c_char_p
    L.scp3gpu_pes_energy.argtypes = [ctypes.c_int, ctypes.c_int, i64, dp, dp, ip]
    L.scp3gpu_pes_energy_grad.argtypes = [ctypes.c_int, ctypes.c_int, i64, dp, dp, dp]
    L.scp3gpu_pes_energy_dev.argtypes = [ctypes.c_int, ctypes.c_int, i64, vp, vp, ctypes.c_int]
    L.scp3gpu_sobol_std_normal.argtypes = [ctypes.c_int, i64, i64, ctypes.c_int, ctypes.c_uint64, dp]
    L.scp3gpu_basis_size.restype = i64
    L.scp3gpu_basis_size.argtypes = [ctypes.c_int] * 3
    L.scp3gpu_sub_basis_size.restype = i64
    L.scp3gpu_sub_basis_size.argtypes = [ctypes.c_int] * 4
    L.scp3gpu_hbuild_create.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(vp)]
    L.scp3gpu_hbuild_destroy.argtypes = [vp]
    L.scp3gpu_hbuild_reset.argtypes = [vp]
    L.scp3gpu_hbuild_basis_size.restype = i64
    L.scp3gpu_hbuild_basis_size.argtypes = [vp]
    L.scp3gpu_hbuild_stream.restype = vp
    L.scp3gpu_hbuild_stream.argtypes = [vp]
    L.scp3gpu_hbuild_accumulate.argtypes = [vp, i64, i64]
    L.scp3gpu_hbuild_accumulate_normals.argtypes = [vp, dp, i64]
    L.scp3gpu_hbuild_accumulate_normals_f32.argtypes = [vp, ctypes.POINTER(ctypes.c_float), i64]
    L.scp3gpu_hbuild_add_epot.argtypes = [vp, dp, dp, i64]
    L.scp3gpu_hbuild_add_epot_grad.argtypes = [vp, dp, dp, dp, i64]
    L.scp3gpu_hbuild_sample_count.restype = i64
    L.scp3gpu_hbuild_sample_count.argtypes = [vp]
    L.scp3gpu_hbuild_read.argtypes = [vp, dp, i64, ctypes.c_int]
    L.scp3gpu_hbuild_read_dev.argtypes = [vp, vp, i64, ctypes.c_int]
    L.scp3gpu_hbuild_eigvals.argtypes = [vp, i64, ctypes.c_int, dp]
    L.scp3gpu_hbuild_profile.argtypes = [vp, ctypes.c_int, dp, ctypes.POINTER(i64)]
    L.scp3gpu_add_epot_static.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, i64, vp, i64, vp]
    L.scp3gpu_save_h5.argtypes = [ctypes.c_char_p, dp, i64, i64]
    L.scp3gpu_save_h5_layout.argtypes = [ctypes.c_char_p, dp, i64, i64, ctypes.c_int]
    L.scp3gpu_syevr_lowest.argtypes = [dp, i64, i64, ctypes.c_int, dp, dp, i64, ctypes.c_int]
    L.scp3gpu_load_h5.argtypes = [ctypes.c_char_p, dp, ctypes.POINTER(i64), ctypes.POINTER(i64)]
    L.scp3gpu_hbuild_status.argtypes = [vp, ctypes.POINTER(i64), ctypes.POINTER(i64)]
    L.scp3gpu_scp1_create.argtypes = [ctypes.c_int, ctypes.c_int, i64, ctypes.c_int, ctypes.POINTER(vp)]
    L.scp3gpu_scp1_average.argtypes = [vp, dp, dp, dp, i64, i64, i64, dp, dp, dp]
    L.scp3gpu_scp1_status.argtypes = [vp, ctypes.POINTER(i64)]
    L.scp3gpu_scp1_destroy.argtypes = [vp]
    L.scp3gpu_scp1_destroy.restype = None
    L.scp3gpu_batch_create.argtypes = [ctypes.POINTER(Config), ctypes.c_int, i64, ctypes.c_int, ctypes.POINTER(vp)]
    L.scp3gpu_batch_destroy.argtypes = [vp]
    L.scp3gpu_batch_reset.argtypes = [vp]
    L.scp3gpu_batch_size.argtypes = [vp]
    L.scp3gpu_batch_basis_size.restype = i64
    L.scp3gpu_batch_basis_size.argtypes = [vp, ctypes.c_int]
    L.scp3gpu_batch_sample_count.restype = i64
    L.scp3gpu_batch_sample_count.argtypes = [vp]
    L.scp3gpu_batch_stream.restype = vp
    L.scp3gpu_batch_stream.argtypes = [vp]
    L.scp3gpu_batch_shape.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(i64), dp]
    L.scp3gpu_batch_accumulate.argtypes = [vp, i64, i64]
    L.scp3gpu_batch_read.argtypes = [vp, ctypes.c_int, dp, i64, ctypes.c_int]
    L.scp3gpu_batch_status.argtypes = [vp, ctypes.c_int, ctypes.POINTER(i64), ctypes.POINTER(i64)]
    _lib = L
    return L


def check(rc):
    if rc != OK:
        raise SCP3GPUError(rc, lib().scp3gpu_last_error().decode())
    return rc
