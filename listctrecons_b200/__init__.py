"""B200-native helical cone-beam FDK hot path of LISTCTRecons.

The compute path is liblct.so (hand-written sm_100a CUDA kernels behind the C ABI in
include/lct.h).  This package is its host side: the ctypes binding (capi), the .prm format
(prm), scan generation (scan), and the planner / reconstruction / mirror of the reference's
stage interfaces (recon).  liblct.so is loaded on first use; every entry point raises if it
is missing (there is no other implementation).
"""
from . import capi

from .prm import FileParams, ParameterError  # noqa: E402
from .recon import (  # noqa: E402
    FDKReconstructor,
    Plan,
    ReconData,
    Reconstruction,
    ReconstrctorAbstractFactory,
    recon_opts,
)

__all__ = [
    "capi", "FileParams", "ParameterError", "FDKReconstructor", "Plan", "ReconData",
    "Reconstruction", "ReconstrctorAbstractFactory", "recon_opts",
]
