"""zhijian_b200: B200-native (sm_100a) Flux-Reconstruction residual and SSP-RK3
stepper behind a C-ABI (include/zj_fr.h).  The compute path is
libzj_fr.so; this package holds the build script, the ctypes binding, the
reference-named solver facade and the synthetic mesh generators."""
from . import _lib
from .meshgen import QuadMesh, structured_quads, vortex_mesh, tgv_mesh
from .solver import FRSolver, make_params

__all__ = ["FRSolver", "make_params", "QuadMesh", "structured_quads", "vortex_mesh",
           "tgv_mesh", "_lib"]
