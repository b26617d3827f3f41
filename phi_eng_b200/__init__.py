"""phi_eng_b200: B200-native (sm_100a) re-implementation of PhiEng's 2D SPH fluid step.

The product is libphieng_sph.so (C ABI in include/phieng_sph.h); this
package builds it (``phi_eng_b200.build``), binds it (``_abi``) and mirrors
the reference's World2 / FluidState2 API in Python (``world``).
"""
from ._abi import FluidConfig2Ffi, default_config  # noqa: F401

__all__ = ["FluidConfig2Ffi", "default_config"]
