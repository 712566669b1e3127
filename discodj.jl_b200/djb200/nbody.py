"""`run_nbody` on the B200 (native/DiscoDJNative/src/nbody/run_nbody.jl:107-225).

The particle state (Ψ, Mom) stays resident in HBM for the whole run; host code
only computes the float64 stepper coefficients (in libdjb200) and issues one
`djb_run` (or one `djb_step` per step when callbacks or histories are asked for).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .cosmology import Cosmology, stepper_coefficients
from .pm import PMConfig, PMSolver


def _canon_scales(c: Cosmology, stepper: str, a: float):
    """(p_div, p_mul) of `canon(M, a) = T.(_v_to_pi(M, a) .* Fplus(a))` (run_nbody.jl:149)."""
    F = c.Fplus(a)
    return (F if stepper == "symplectic" else 1.0), F


def run_nbody(c: Cosmology, psi_ini, pi_ini, *, boxsize, a_ini, a_end, n_steps, res_pm, time_var="D",
              stepper="bullfrog", antialias=0, grad_kernel_order=4, laplace_kernel_order=0, worder=2,
              deconvolve=False, n_resample=1, resampling_method="fourier", collect_all=False,
              return_all_a=False, return_displacement=False, step_callback=None, callback_when=None,
              lean=False, device=0, solver: PMSolver | None = None):
    """run_nbody.jl:124-172 -> (X or Ψ, P, a_end | all_a). Arrays are (n,n,n,3) float32."""
    n = int(np.shape(psi_ini)[0])
    L = float(boxsize)
    if n_steps is None:
        if isinstance(time_var, str):
            raise _lib.DJBInvalidOption(_lib.DJB_ERR_INVALID,
                                        "n_steps = nothing requires an explicit time_var vector")
        n_steps = len(time_var) - 1
    co = stepper_coefficients(c, stepper, a_ini, a_end, n_steps, time_var=time_var)
    cfg = PMConfig(res_pm=res_pm, n_part=n, boxsize=L, worder=worder, deconvolve=deconvolve,
                   antialias=antialias, grad_order=grad_kernel_order, lap_order=laplace_kernel_order,
                   n_resample=n_resample, resampling=resampling_method)
    own = solver is None
    S = PMSolver(cfg, lean=lean, device=device) if own else solver
    try:
        S.set_state(psi_ini, pi_ini, mom_scale=c.Fplus(a_ini) if stepper == "symplectic" else 1.0)
        all_a = co["all_a"]
        want = (lambda k: step_callback is not None
                and (callback_when is None or callback_when(k, all_a[k])))

        def snapshot(k, wrap):
            pd, pm = _canon_scales(c, stepper, all_a[k])
            return S.output(wrap=wrap, p_div=pd, p_mul=pm)

        hist = []
        if want(0):
            X, P = snapshot(0, 2)
            step_callback(0, all_a[0], X, P)
        if collect_all:
            hist.append(snapshot(0, 0 if return_displacement else 1))
        if step_callback is None and not collect_all:
            S.run(co["ddrift1"], co["alpha"], co["beta"], co["ddrift2"])
        else:
            for k in range(n_steps):
                S.step(co["ddrift1"][k], co["alpha"][k], co["beta"][k], co["ddrift2"][k])
                if want(k + 1):
                    X, P = snapshot(k + 1, 2)
                    step_callback(k + 1, all_a[k + 1], X, P)
                if collect_all:
                    hist.append(snapshot(k + 1, 0 if return_displacement else 1))
            S.synchronize()
        if collect_all:
            return [h[0] for h in hist], [h[1] for h in hist], all_a
        pd, pm = _canon_scales(c, stepper, a_end)
        X, P = S.output(wrap=0 if return_displacement else 1, p_div=pd, p_mul=pm)
        return X, P, (all_a if return_all_a else a_end)
    finally:
        if own:
            S.close()


def nbody_ics_lpt(c: Cosmology, shapes: dict, a: float, n_order: int, exact_growth: bool = False):
    """run_nbody.jl:180-208 for EdS shapes: Ψ = Σ Dⁿψₙ, Π = Σ n Dⁿ⁻¹ψₙ (array dtype kept)."""
    if exact_growth:
        raise NotImplementedError("exact-growth shapes: combine compute_core_exact fields with the growth tables")
    D = c.Dplus(a)
    psi1 = shapes["psi_1"]
    single = str(psi1.dtype).endswith("float32")
    coef = lambda x: float(np.float32(x)) if single else float(x)  # T(x) of the reference
    Psi = psi1 * 0
    Pi = psi1 * 0
    for m in range(1, n_order + 1):
        pn = shapes[f"psi_{m}"]
        Psi = Psi + coef(D ** m) * pn
        Pi = Pi + coef(m * D ** (m - 1)) * pn
    return Psi, Pi


def bullfrog_ics(c: Cosmology, psi1, a_ini: float, *, boxsize, res_pm, device=0, **settings):
    """run_nbody.jl:217-225: one BullFrog step 0 -> a_ini with the discreteness-suppressing
    defaults (antialias=1, ik gradient, −1/k², PCS, deconvolution, 2³ Fourier resampling)."""
    s = dict(time_var="D", stepper="bullfrog", antialias=1, grad_kernel_order=0, laplace_kernel_order=0,
             worder=4, deconvolve=True, n_resample=2, resampling_method="fourier")
    s.update(settings)
    psi1 = np.asarray(psi1, dtype=np.float32)
    D0 = np.float32(c.Dplus(0.0))
    Psi, P, _ = run_nbody(c, D0 * psi1, psi1.copy(), boxsize=boxsize, a_ini=0.0, a_end=a_ini, n_steps=1,
                          res_pm=res_pm, return_displacement=True, device=device, **s)
    return Psi, P / np.float32(c.Fplus(a_ini))
