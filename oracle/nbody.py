"""N-body time integration (float64): stepper coefficients and the DKD loop.

Restates `native/DiscoDJNative/src/nbody/run_nbody.jl:22-225`.
Test infrastructure only (see `oracle/__init__.py`).

Particle arrays are (n,n,n,3) indexed [i,j,k,c] (c = 0 is x), the reference's
logical layout (`src/nbody/pm.jl:15-17`).
"""
from __future__ import annotations

import math

import numpy as np

from . import cosmology as cz
from . import pm as pmo

# run_nbody.jl:24-25 (5-point Gauss-Legendre nodes and weights)
_GL5_X = (-0.906179845938664, -0.5384693101056831, 0.0, 0.5384693101056831, 0.906179845938664)
_GL5_W = (0.23692688505618928, 0.4786286704993663, 0.5688888888888887, 0.4786286704993663,
          0.23692688505618928)


def nplinspace(s: float, e: float, num: int) -> np.ndarray:
    """run_nbody.jl:22 (numpy.linspace: y = s + i·step, y[end] = e)."""
    st = (e - s) / (num - 1)
    y = np.array([s + i * st for i in range(num)], dtype=np.float64)
    y[-1] = e
    return y


def _a_to_internal(c, tv, a):
    """run_nbody.jl:27-33"""
    if tv == "a":
        return a
    if tv == "log_a":
        return math.log(a)
    if tv == "D":
        return cz.Dplus(c, a)
    if tv == "superconft":
        return cz.superconft(c, a)
    raise ValueError("time_var must be :a, :log_a, :D, :superconft or a vector of scale factors")


def _internal_to_a(c, tv, x):
    """run_nbody.jl:34-40"""
    if tv == "a":
        return x
    if tv == "log_a":
        return math.exp(x)
    if tv == "D":
        return cz.a_of_Dplus(c, x)
    if tv == "superconft":
        return cz.a_of_superconft(c, x)
    raise ValueError(f"unknown time_var {tv}")


def stepper_coefficients(c, stepper, a_ini, a_end, n_steps, time_var="D"):
    """run_nbody.jl:48-101 -> dict(alpha, beta, ddrift1, ddrift2, all_a)."""
    if not isinstance(time_var, str):
        tvv = np.asarray(time_var, dtype=np.float64)
        if len(tvv) != n_steps + 1:
            raise ValueError("time_var vector must have n_steps + 1 entries")
        tgrid = nplinspace(0.0, float(n_steps), n_steps + 1)
        itoa = lambda x: cz.jinterp(x, tgrid, tvv)
        all_int = nplinspace(0.0, float(n_steps), n_steps + 1)
    else:
        s = _a_to_internal(c, time_var, float(a_ini))
        e = _a_to_internal(c, time_var, float(a_end))
        itoa = lambda x: _internal_to_a(c, time_var, x)
        all_int = nplinspace(s, e, n_steps + 1)
    all_a = np.array([itoa(x) for x in all_int])
    int_mid = (all_int[:-1] + all_int[1:]) / 2
    a_mid = np.array([itoa(x) for x in int_mid])
    ab, ae = all_a[:-1], all_a[1:]
    if stepper == "bullfrog":
        D1 = c.D1_unnormed_at_1
        Du = lambda a: cz.Dplus(c, a) * D1
        Ddau = lambda a: cz.growth_Dplusda(c, a) * D1
        D2u = lambda a: cz.D2plus(c, a) * D1 ** 2
        D2dau = lambda a: cz.growth_D2plusda(c, a) * D1 ** 2
        all_D = np.array([Du(a) for a in all_a])
        all_Dda = np.array([Ddau(a) for a in all_a])
        all_D2 = np.array([D2u(a) for a in all_a])
        all_D2da = np.array([D2dau(a) for a in all_a])
        D_b, D_e = all_D[:-1], all_D[1:]
        dD = D_e - D_b
        xi = D_b / dD
        Dda_b, Dda_e = all_Dda[:-1], all_Dda[1:]
        D2_b = all_D2[:-1]
        D2da_b, D2da_e = all_D2da[:-1], all_D2da[1:]
        bracket = (D2_b + D2da_b / Dda_b * dD / 2) / ((xi + 0.5) * dD) - (xi + 0.5) * dD
        alpha = (D2da_e / Dda_e - bracket) / (D2da_b / Dda_b - bracket)
        D_mid = np.array([cz.Dplus(c, a) for a in a_mid])
        beta = (1 - alpha) / D_mid
        dd1 = D_mid - D_b / D1
        dd2 = D_e / D1 - D_mid
    elif stepper == "fastpm":
        alpha = np.array([cz.Fplus(c, a) for a in ab]) / np.array([cz.Fplus(c, a) for a in ae])
        D_mid = np.array([cz.Dplus(c, a) for a in a_mid])
        beta = (1 - alpha) / D_mid
        all_D = np.array([cz.Dplus(c, a) for a in all_a])
        dd1 = D_mid - all_D[:-1]
        dd2 = all_D[1:] - D_mid
    elif stepper == "symplectic":
        alpha = np.ones(len(a_mid))
        f = lambda a: 1 / (a ** 2 * float(cz.hubble_E(c, a)))

        def integ(b, e):
            return 0.5 * (e - b) * sum(_GL5_W[i] * f(0.5 * (e - b) * _GL5_X[i] + 0.5 * (b + e))
                                       for i in range(5))

        beta = 1.5 * cz.Omega_m(c) * np.array([integ(b, e) for b, e in zip(ab, ae)])
        sc = np.array([cz.superconft(c, a) for a in all_a])
        scm = np.array([cz.superconft(c, a) for a in a_mid])
        dd1 = scm - sc[:-1]
        dd2 = sc[1:] - scm
    else:
        raise ValueError("stepper must be :bullfrog, :fastpm or :symplectic")
    return dict(alpha=np.asarray(alpha, dtype=np.float64), beta=np.asarray(beta),
                ddrift1=np.asarray(dd1), ddrift2=np.asarray(dd2), all_a=all_a)


def _pi_to_v(c, stepper, P, a):
    """run_nbody.jl:104"""
    return P * cz.Fplus(c, a) if stepper == "symplectic" else P


def _v_to_pi(c, stepper, v, a):
    """run_nbody.jl:105"""
    return v / cz.Fplus(c, a) if stepper == "symplectic" else v


def lagrangian_q(n: int, L: float) -> np.ndarray:
    """pm.jl:186 `_lagr1d`: q_i = i·L/n (0-based)."""
    return np.array([i * (L / n) for i in range(n)], dtype=np.float64)


def add_q(psi: np.ndarray, L: float) -> np.ndarray:
    """X = q + Ψ for (n,n,n,3) arrays (run_nbody.jl:148)."""
    n = psi.shape[0]
    q = lagrangian_q(n, L)
    X = np.empty_like(psi)
    X[..., 0] = psi[..., 0] + q[:, None, None]
    X[..., 1] = psi[..., 1] + q[None, :, None]
    X[..., 2] = psi[..., 2] + q[None, None, :]
    return X


def run_nbody(c, psi_ini, pi_ini, *, boxsize, a_ini, a_end, n_steps, res_pm, time_var="D",
              stepper="bullfrog", antialias=0, grad_kernel_order=4, laplace_kernel_order=0,
              worder=2, deconvolve=False, n_resample=1, resampling_method="fourier",
              return_displacement=False, step_callback=None, callback_when=None, force=None):
    """run_nbody.jl:124-172 (forward DKD loop, FP64). Returns (X or Ψ, P, a_end).

    `force(cfg, psi)` overrides the PM acceleration (default: `pm.pm_acceleration`)."""
    n = psi_ini.shape[0]
    L = float(boxsize)
    if n_steps is None:
        if isinstance(time_var, str):
            raise ValueError("n_steps = nothing requires an explicit time_var vector")
        n_steps = len(time_var) - 1
    co = stepper_coefficients(c, stepper, a_ini, a_end, n_steps, time_var=time_var)
    cfg = pmo.PMConfig(res_pm=res_pm, n_part=n, boxsize=L, worder=worder, deconvolve=deconvolve,
                       antialias=antialias, grad_order=grad_kernel_order,
                       lap_order=laplace_kernel_order, n_resample=n_resample,
                       resampling=resampling_method)
    acc = force if force is not None else pmo.pm_acceleration
    Psi = np.array(psi_ini, dtype=np.float64, copy=True)
    Mom = np.asarray(_pi_to_v(c, stepper, np.asarray(pi_ini, dtype=np.float64), a_ini))
    canon = lambda M, a: _v_to_pi(c, stepper, M, a) * cz.Fplus(c, a)
    want = lambda k: step_callback is not None and (callback_when is None
                                                    or callback_when(k, co["all_a"][k]))
    if want(0):
        step_callback(0, co["all_a"][0], add_q(Psi, L), canon(Mom, co["all_a"][0]))
    for k in range(n_steps):
        Psi = Psi + co["ddrift1"][k] * Mom
        Mom = co["alpha"][k] * Mom + co["beta"][k] * acc(cfg, Psi)
        Psi = Psi + co["ddrift2"][k] * Mom
        if want(k + 1):
            step_callback(k + 1, co["all_a"][k + 1], add_q(Psi, L), canon(Mom, co["all_a"][k + 1]))
    P = canon(Mom, a_end)
    if return_displacement:
        return Psi, P, a_end
    X = add_q(Psi, L)
    return np.mod(X + L, L), P, a_end


def nbody_ics_lpt(c, shapes, a, n_order, exact_growth=False):
    """run_nbody.jl:180-208 for the EdS shapes (Ψ = Σ Dⁿψₙ, Π = Σ n Dⁿ⁻¹ψₙ)."""
    if exact_growth:
        raise NotImplementedError("exact-growth shapes are not restated in the oracle")
    D = cz.Dplus(c, a)
    psi1 = shapes["psi_1"]
    Psi = np.zeros_like(psi1)
    Pi = np.zeros_like(psi1)
    for m in range(1, n_order + 1):
        psin = shapes[f"psi_{m}"]
        Psi = Psi + D ** m * psin
        Pi = Pi + (m * D ** (m - 1)) * psin
    return Psi, Pi


def bullfrog_ics(c, psi1, a_ini, *, boxsize, res_pm, **settings):
    """run_nbody.jl:217-225: one BullFrog step 0 -> a_ini with the suppression defaults."""
    s = dict(time_var="D", stepper="bullfrog", antialias=1, grad_kernel_order=0,
             laplace_kernel_order=0, worder=4, deconvolve=True, n_resample=2,
             resampling_method="fourier")
    s.update(settings)
    D0 = cz.Dplus(c, 0.0)
    Psi, P, _ = run_nbody(c, D0 * psi1, psi1.copy(), boxsize=boxsize, a_ini=0.0, a_end=a_ini,
                          n_steps=1, res_pm=res_pm, return_displacement=True, **s)
    return Psi, P / cz.Fplus(c, a_ini)
