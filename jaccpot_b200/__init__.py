"""jaccpot_b200: jaccpot's real-basis FMM evaluation pass on Blackwell (sm_100a).

Public entry point: :class:`FastMultipoleMethod` (same signature as
``jaccpot.FastMultipoleMethod`` for the real basis).  The kernels live in the
in-tree shared library ``_lib/libjaccpot_b200.so`` (C ABI in
include/jaccpot_b200.h); there is no CPU fallback.
"""

from .solver import FastMultipoleMethod, FMMPreparedState

__all__ = ["FastMultipoleMethod", "FMMPreparedState"]
