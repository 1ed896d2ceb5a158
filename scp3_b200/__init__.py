"""B200-native Hamiltonian build of SCP3: Sobol -> BSM -> water potential ->
<i|V|j> over Hermite product functions, as hand-written sm_100a kernels behind
a C ABI (include/scp3gpu.h, libscp3gpu.so)."""
from . import constants, modes, clusters  # noqa: F401
from ._lib import SCP3GPUError, build  # noqa: F401
from .api import (PES, Batch, HBuild, PESFromString, SCP1Average, dsyevr, ScaledMatrixElements, qtip4pf,  # noqa: F401
                  std_normal, std_normals, ttm3f)
