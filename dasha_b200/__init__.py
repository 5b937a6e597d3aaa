"""dasha_b200: a B200 (sm_100a) CUDA implementation of the RK4 Hall-MHD time step of the
reference Fortran program t3dsdsc.f (Alan66666/dasha), behind a C-ABI (include/dasha_capi.h)."""
from . import harris  # noqa: F401
