"""Cosmology and stepper coefficients, computed by libdjb200's float64 host code.

Mirrors `Cosmology`, `compute_timetables`, the timetable lookups
(native/DiscoDJNative/src/cosmology/Cosmology.jl, src/nbody/timetables.jl) and
`stepper_coefficients` (src/nbody/run_nbody.jl:48-101).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, dptr, lib

_TABLES = {"a": 0, "Dplus": 1, "Dplusda": 2, "D2plus": 3, "D2plusda": 4, "superconft": 5,
           "f1": 6, "f2": 7, "D3a": 8, "D3b": 9, "D3c": 10}


class Cosmology:
    """`Cosmology(name)` or `Cosmology(Omega_c=..., ...)` with its timetables."""

    PARAMS = ("Omega_c", "Omega_b", "h", "sigma8", "n_s", "Omega_k", "w0", "wa")
    DEFAULTS = (0.259622, 0.0488911, 0.67742, 0.8105, 0.96822, 0.0, -1.0, 0.0)

    def __init__(self, name: str | None = None, *, n_pts: int = 2500, a_ini: float = 1e-10, **params):
        h = C.c_void_p()
        if name is not None:
            if params:
                raise ValueError("give either a predefined name or parameters")
            check(lib.djb_cosmology_create_named(name.encode(), C.byref(h)))
        else:
            unknown = set(params) - set(self.PARAMS)
            if unknown:
                raise TypeError(f"unknown cosmology parameters {sorted(unknown)}")
            p = np.array([float(params.get(k, d)) for k, d in zip(self.PARAMS, self.DEFAULTS)])
            check(lib.djb_cosmology_create(dptr(p), int(n_pts), float(a_ini), C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib.djb_cosmology_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def table(self, which: str) -> np.ndarray:
        n = C.c_int32()
        check(lib.djb_cosmology_table_size(self._h, C.byref(n)))
        out = np.empty(n.value)
        check(lib.djb_cosmology_table(self._h, _TABLES[which], dptr(out), n.value))
        return out

    @property
    def params(self) -> dict:
        out = np.empty(8)
        check(lib.djb_cosmology_params(self._h, dptr(out)))
        return dict(zip(self.PARAMS, out.tolist()))

    @property
    def D1_unnormed_at_1(self) -> float:
        v = C.c_double()
        check(lib.djb_cosmology_d1_unnormed(self._h, C.byref(v)))
        return v.value

    def _eval(self, what: int, x: float) -> float:
        v = C.c_double()
        check(lib.djb_cosmology_eval(self._h, what, float(x), C.byref(v)))
        return v.value

    def Dplus(self, a):
        return self._eval(0, a)

    def growth_Dplusda(self, a):
        return self._eval(1, a)

    def D2plus(self, a):
        return self._eval(2, a)

    def growth_D2plusda(self, a):
        return self._eval(3, a)

    def superconft(self, a):
        return self._eval(4, a)

    def a_of_superconft(self, s):
        return self._eval(5, s)

    def a_of_Dplus(self, D):
        return self._eval(6, D)

    def Fplus(self, a):
        return self._eval(7, a)

    def hubble_E(self, a):
        return self._eval(8, a)

    @property
    def Omega_m(self):
        return self._eval(9, 0.0)


def stepper_coefficients(cosmo: Cosmology, stepper: str, a_ini: float, a_end: float, n_steps: int,
                         time_var="D") -> dict:
    """run_nbody.jl:48-101 -> dict(alpha, beta, ddrift1, ddrift2, all_a) (float64)."""
    if stepper not in _lib.STEPPERS:
        raise _lib.DJBInvalidOption(_lib.DJB_ERR_INVALID, "stepper must be :bullfrog, :fastpm or :symplectic")
    ns = int(n_steps)
    out = {k: np.empty(ns) for k in ("alpha", "beta", "ddrift1", "ddrift2")}
    out["all_a"] = np.empty(ns + 1)
    if isinstance(time_var, str):
        if time_var not in _lib.TIME_VARS:
            raise _lib.DJBInvalidOption(
                _lib.DJB_ERR_INVALID,
                "time_var must be :a, :log_a, :D, :superconft or a vector of scale factors")
        tv, arr = _lib.TIME_VARS[time_var], None
    else:
        arr = np.ascontiguousarray(time_var, dtype=np.float64)
        if arr.shape != (ns + 1,):
            raise _lib.DJBInvalidOption(_lib.DJB_ERR_INVALID, "time_var vector must have n_steps + 1 entries")
        tv = _lib.TIME_ARRAY
    check(lib.djb_stepper_coefficients(
        cosmo.handle, _lib.STEPPERS[stepper], tv, dptr(arr) if arr is not None else None,
        float(a_ini), float(a_end), ns, dptr(out["alpha"]), dptr(out["beta"]), dptr(out["ddrift1"]),
        dptr(out["ddrift2"]), dptr(out["all_a"])))
    return out
