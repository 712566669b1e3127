"""Background cosmology, growth tables and timetable lookups (float64).

Restates `native/DiscoDJNative/src/cosmology/Cosmology.jl:22-115,145-165`,
`src/cosmology/growth.jl:23-96` and `src/nbody/timetables.jl:10-45`.
Test infrastructure only (see `oracle/__init__.py`).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# Cosmology.jl:145-150
PREDEFINED_COSMOLOGIES = {
    "Planck18EEBAOSN": dict(Omega_c=0.259622, Omega_b=0.0488911, h=0.67742, sigma8=0.8105,
                            n_s=0.96822, Omega_k=0.0, w0=-1.0, wa=0.0),
    "Planck15": dict(Omega_c=0.2589, Omega_b=0.0486, h=0.6774, sigma8=0.8159, n_s=0.9667,
                     Omega_k=0.0, w0=-1.0, wa=0.0),
    "Quijote": dict(Omega_c=0.3175, Omega_b=0.049, h=0.6711, sigma8=0.834, n_s=0.9624,
                    Omega_k=0.0, w0=-1.0, wa=0.0),
    "CamelsCV": dict(Omega_c=0.2514, Omega_b=0.049, h=0.6711, sigma8=0.818, n_s=0.9624,
                     Omega_k=0.0, w0=-1.0, wa=0.0),
}


@dataclass
class Cosmology:
    """Cosmology.jl:22-45 (parameters + timetables)."""
    Omega_c: float = 0.259622
    Omega_b: float = 0.0488911
    h: float = 0.67742
    sigma8: float = 0.8105
    n_s: float = 0.96822
    Omega_k: float = 0.0
    w0: float = -1.0
    wa: float = 0.0
    a_table: np.ndarray = field(default=None, repr=False)
    D1_table: np.ndarray = field(default=None, repr=False)
    D2_table: np.ndarray = field(default=None, repr=False)
    D3a_table: np.ndarray = field(default=None, repr=False)
    D3b_table: np.ndarray = field(default=None, repr=False)
    D3c_table: np.ndarray = field(default=None, repr=False)
    f1_table: np.ndarray = field(default=None, repr=False)
    f2_table: np.ndarray = field(default=None, repr=False)
    f3a_table: np.ndarray = field(default=None, repr=False)
    f3b_table: np.ndarray = field(default=None, repr=False)
    superconft_table: np.ndarray = field(default=None, repr=False)
    D1_unnormed_at_1: float = float("nan")

    @classmethod
    def named(cls, name: str) -> "Cosmology":
        """Cosmology.jl:158-165: predefined cosmology with timetables."""
        if name not in PREDEFINED_COSMOLOGIES:
            raise ValueError(f"Unknown cosmology: {name}")
        return compute_timetables(cls(**PREDEFINED_COSMOLOGIES[name]))

    @property
    def Omega_m(self) -> float:
        return self.Omega_c + self.Omega_b


def Omega_m(c: Cosmology) -> float:
    return c.Omega_c + c.Omega_b


def Omega_de(c: Cosmology, a):
    """Cosmology.jl:48"""
    return (1 - Omega_m(c) - c.Omega_k) * a ** (-3 * (1 + c.w0 + c.wa)) * np.exp(-3 * c.wa * (1 - a))


def hubble_E(c: Cosmology, a):
    """Cosmology.jl:55-58: E(a) = sqrt(Ωm a⁻³ + Ωk a⁻² + Ωde(a))."""
    return np.sqrt(Omega_m(c) * a ** (-3) + c.Omega_k * a ** (-2) + Omega_de(c, a))


def _growth_derivs(c: Cosmology, lna, y):
    """growth.jl:23-45 (state y = [ln D1, f1, ln|D2|, f2, ln D3a, f3a, ln|D3b|, f3b, ln D3c])."""
    a = math.exp(lna)
    Esq = float(hubble_E(c, a)) ** 2
    Om_a = (Omega_m(c) * a ** (-3)) / Esq
    Ox_a = float(Omega_de(c, a)) / Esq
    w_a = c.w0 + c.wa * (1 - a)
    drag = 1 - 0.5 * (Om_a + (1 + 3 * w_a) * Ox_a)
    y1, f1, y2, f2, y3a, f3a, y3b, f3b, y3c = y
    D1 = math.exp(y1)
    D1sq = D1 * D1
    D1cu = D1sq * D1
    D2 = -math.exp(y2)
    D3a = math.exp(y3a)
    D3b = -math.exp(y3b)
    D3c = math.exp(y3c)
    df1 = 1.5 * Om_a - f1 ** 2 - f1 * drag
    df2 = 1.5 * Om_a * (1 - D1sq / D2) - f2 ** 2 - f2 * drag
    df3a = 1.5 * Om_a * (1 + 2 * D1cu / D3a) - f3a ** 2 - f3a * drag
    df3b = 1.5 * Om_a * (1 + (2 * D1 * D2 - 2 * D1cu) / D3b) - f3b ** 2 - f3b * drag
    dy3c = D1 * D2 / D3c * (f1 - f2)
    return (f1, df1, f2, df2, f3a, df3a, f3b, df3b, dy3c)


def _rk4_growth(c, lna, y, dl):
    """growth.jl:49-55"""
    k1 = _growth_derivs(c, lna, y)
    k2 = _growth_derivs(c, lna + dl / 2, tuple(y[i] + dl / 2 * k1[i] for i in range(9)))
    k3 = _growth_derivs(c, lna + dl / 2, tuple(y[i] + dl / 2 * k2[i] for i in range(9)))
    k4 = _growth_derivs(c, lna + dl, tuple(y[i] + dl * k3[i] for i in range(9)))
    return tuple(y[i] + dl / 6 * (k1[i] + 2 * k2[i] + 2 * k3[i] + k4[i]) for i in range(9))


def _julia_linrange(a: float, b: float, n: int) -> np.ndarray:
    """Julia `LinRange(a, b, n)` element values: (1-t)·a + t·b with t = j/(n-1)."""
    j = np.arange(n, dtype=np.float64)
    d = float(n - 1)
    t = j / d
    out = (1 - t) * a + t * b
    out[0], out[-1] = a, b
    return out


def compute_timetables(c: Cosmology, n_pts: int = 2500, a_ini: float = 1e-10) -> Cosmology:
    """Cosmology.jl:86-115 with growth.jl:57-96 (growth tables + superconformal time)."""
    a_table = 10.0 ** _julia_linrange(math.log10(a_ini), 0.0, n_pts)
    n = n_pts
    amin = a_table[0]
    y = (math.log(amin), 1.0, math.log(3 / 7 * amin ** 2), 2.0, math.log(1 / 3 * amin ** 3), 3.0,
         math.log(10 / 21 * amin ** 3), 3.0, math.log(1 / 7 * amin ** 3))
    lna = np.log(a_table)
    rows = np.empty((n, 9))
    rows[0] = y
    for i in range(1, n):
        y = _rk4_growth(c, float(lna[i - 1]), y, float(lna[i] - lna[i - 1]))
        rows[i] = y
    D1 = np.exp(rows[:, 0])
    F1 = rows[:, 1].copy()
    D2 = -np.exp(rows[:, 2])
    F2 = rows[:, 3].copy()
    D3a = np.exp(rows[:, 4])
    F3a = rows[:, 5].copy()
    D3b = -np.exp(rows[:, 6])
    F3b = rows[:, 7].copy()
    D3c = np.exp(rows[:, 8])
    D1_at1 = float(np.interp(1.0, a_table, D1))
    c.a_table = a_table
    c.D1_table = D1 / D1_at1
    c.D2_table = D2 / D1_at1 ** 2
    c.D3a_table = D3a / D1_at1 ** 3
    c.D3b_table = D3b / D1_at1 ** 3
    c.D3c_table = D3c / D1_at1 ** 3
    c.f1_table, c.f2_table, c.f3a_table, c.f3b_table = F1, F2, F3a, F3b
    # growth.jl:88-96 superconformal time: reverse cumulative trapezoid of 1/(E a³)
    f = 1.0 / (hubble_E(c, a_table) * a_table ** 3)
    s = np.zeros(n)
    for i in range(n - 2, -1, -1):
        s[i] = s[i + 1] - (a_table[i + 1] - a_table[i]) * (f[i] + f[i + 1]) / 2
    c.superconft_table = s - s[-1]
    c.D1_unnormed_at_1 = D1_at1
    return c


# ── timetables.jl ─────────────────────────────────────────────────────────────
def jinterp(x: float, xp: np.ndarray, fp: np.ndarray) -> float:
    """timetables.jl:10-18: `jnp.interp` semantics (clamp outside the table)."""
    x = float(x)
    if x <= xp[0]:
        return float(fp[0])
    if x >= xp[-1]:
        return float(fp[-1])
    i = int(np.searchsorted(xp, x, side="right")) - 1  # xp[i] <= x < xp[i+1]
    if i >= len(xp) - 1:
        return float(fp[-1])
    t = (x - xp[i]) / (xp[i + 1] - xp[i])
    return float(fp[i] + t * (fp[i + 1] - fp[i]))


def Dplusda_tab(c):
    """timetables.jl:23"""
    return c.f1_table * c.D1_table / c.a_table


def D2plusda_tab(c):
    """timetables.jl:24"""
    return c.f2_table * c.D2_table / c.a_table


def growth_Dplusda(c, a):
    return jinterp(a, c.a_table, Dplusda_tab(c))


def growth_D2plusda(c, a):
    return jinterp(a, c.a_table, D2plusda_tab(c))


def superconft(c, a):
    return jinterp(a, c.a_table, c.superconft_table)


def a_of_superconft(c, s):
    return jinterp(s, c.superconft_table, c.a_table)


def a_of_Dplus(c, D):
    return jinterp(D, c.D1_table, c.a_table)


def Fplus(c, a):
    """timetables.jl:40: F₊ = a³ E(a) dD₊/da."""
    return a ** 3 * float(hubble_E(c, a)) * growth_Dplusda(c, a)


def Dplus(c, a):
    """timetables.jl:44"""
    return jinterp(a, c.a_table, c.D1_table)


def D2plus(c, a):
    """timetables.jl:45"""
    return jinterp(a, c.a_table, c.D2_table)
