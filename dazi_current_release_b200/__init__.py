"""B200-native depth-kernel stage of DAzi (surface-wave azimuthal anisotropy
tomography): Rayleigh phase velocities and the dc/dVs and Gc/Gs sensitivity
kernels (and Love waves and group velocities with their kernels, in both
forms), computed by hand-written sm_100a CUDA kernels behind a C-ABI
(include/dazi_dk.h).  The Python side mirrors the reference's Fortran
interfaces `depthkernel` and `depthkernelTI`.
"""
from .depthkernel import (depthkernel, depthkernel_vpvsrho, depthkernelTI,  # noqa: F401
                          depthkernel_fused, DepthKernelError)
from ._lib import (DaziError, FORM_PLAIN, FORM_ADJOINT, FORM_SCAN_FP32,  # noqa: F401
                   FORM_LOVE, FORM_GROUP, FORM_FAST_ROOT, FORM_FULL_STACK)

__all__ = ["depthkernel", "depthkernel_vpvsrho", "depthkernelTI", "depthkernel_fused",
           "DepthKernelError", "DaziError",
           "FORM_PLAIN", "FORM_ADJOINT", "FORM_SCAN_FP32", "FORM_LOVE", "FORM_GROUP",
           "FORM_FAST_ROOT", "FORM_FULL_STACK"]
