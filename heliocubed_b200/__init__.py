"""B200-native (sm_100a, FP64) per-box MHD update of HelioCubed.

The second-order cubed-sphere operator (PLM minmod/MC, Rusanov and Roe
8-wave fluxes, Powell and gravity sources, CFL reduction) and the classical
RK4 stage update that consumes it, as hand-written CUDA behind the C ABI of
include/hc_abi.h.  `Shell` (heliocubed_b200.level) is the host-side mirror of
the reference's level/operator interface.
"""
from ._native import HcBox, HcCone, HcConeSpec, HcError, HcInit, HcParams, lib  # noqa: F401
from .level import C_MP, C_SR, ConeSpec, InitSpec, Params, Shell, make_box, prepare_cone  # noqa: F401

__all__ = ["Shell", "Params", "InitSpec", "ConeSpec", "prepare_cone", "make_box", "HcBox", "HcParams", "HcInit",
           "HcCone", "HcConeSpec", "HcError", "lib", "C_SR", "C_MP"]
