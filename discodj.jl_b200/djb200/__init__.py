"""djb200 — host-side mirror of DiscoDJNative's PM interface over libdjb200.so.

The B200 kernels live in the shared library (C ABI, include/djb200.h); this
package gives them the reference's Julia names and argument meanings
(native/DiscoDJNative/src/nbody/pm.jl, run_nbody.jl, analysis/power_spectrum.jl)
so that tests read like the reference's own. Importing fails if the library is
missing: there is no CPU fallback.
"""
from ._lib import DJBError, DJBInvalidOption, LIB_PATH, lib  # noqa: F401
from .cosmology import Cosmology, stepper_coefficients  # noqa: F401
from .nbody import bullfrog_ics, nbody_ics_lpt, run_nbody  # noqa: F401
from .pm import (PMConfig, PMSolver, logical_view, native_host, native_view,  # noqa: F401
                 pm_acceleration, pm_acceleration_)
from .power import evaluate_power_spectrum  # noqa: F401

__all__ = ["Cosmology", "stepper_coefficients", "run_nbody", "bullfrog_ics", "nbody_ics_lpt", "PMConfig",
           "PMSolver", "pm_acceleration", "pm_acceleration_", "evaluate_power_spectrum", "native_view",
           "logical_view", "native_host", "DJBError", "DJBInvalidOption"]
