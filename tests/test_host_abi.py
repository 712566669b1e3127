"""CPU-side checks of libdjb200: the shared library loads and exports every symbol
include/djb200.h declares; its float64 host code (cosmology tables, stepper
coefficients) matches the golden vectors; option validation raises like the
reference; the IC generator reproduces the fixture's 2LPT initial conditions.
None of these launch a kernel."""
from __future__ import annotations

import json
import os
import re

import numpy as np
import pytest

from conftest import PARITY_CONFIGS, ROOT, rel, run_kwargs

djb200 = pytest.importorskip("djb200")

HEADER = os.path.join(ROOT, "include", "djb200.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"DJB_API\s+(?:const\s+char\s*\*|int)\s+(djb_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(djb200.lib, s), s
    # the ctypes signature table covers the header exactly
    from djb200 import _lib
    assert sorted(_lib.SIGNATURES) == syms


def test_julia_binding_calls_only_declared_symbols():
    """Every `ccall` of the Julia host binding names an entry point of the header (the
    binding is not executed here: Julia is not installed)."""
    jl = open(os.path.join(ROOT, "discodj.jl_b200", "julia", "DiscoDJB200.jl")).read()
    called = set(re.findall(r"ccall\(\(:(djb_\w+)", jl))
    assert len(called) >= 15
    assert called <= set(declared_symbols()), sorted(called - set(declared_symbols()))


def test_lpt_work_area_sizes_and_rejections():
    """djb_lpt_ics_work_bytes (no device needed): the third order needs more than the
    second, the area grows with n, and invalid sizes and orders are rejected."""
    import ctypes as C

    from djb200 import _lib
    out = C.c_int64(0)

    def wb(n, order, npk=64):
        rc = _lib.lib.djb_lpt_ics_work_bytes(n, order, npk, C.byref(out))
        return rc, out.value

    rc2, b2 = wb(32, 2)
    rc3, b3 = wb(32, 3)
    assert rc2 == rc3 == 0 and 0 < b2 < b3
    ext = 48
    assert b3 >= 4 * ext ** 3 * 14       # P, Q, mu2 and two ext spectra
    assert wb(64, 3)[1] > 7 * b3
    for n, order in ((30, 2), (32, 4), (32, 1)):
        assert wb(n, order)[0] == _lib.DJB_ERR_INVALID
    assert wb(32, 2, npk=1)[0] == _lib.DJB_ERR_INVALID


def test_version_and_error_text():
    assert b"sm_100a" in djb200.lib.djb_version()
    assert djb200.lib.djb_last_error() is not None


@pytest.fixture(scope="module")
def cosmo():
    return djb200.Cosmology("Planck18EEBAOSN")


def test_cosmology_tables(golden, cosmo):
    assert rel(cosmo.table("Dplus"), golden["cosmo/Dplus"]) < 1e-13
    assert rel(cosmo.table("Dplusda"), golden["cosmo/Dplusda"]) < 1e-13
    assert rel(cosmo.table("D2plus"), golden["cosmo/D2plus"]) < 1e-13
    assert rel(cosmo.table("D2plusda"), golden["cosmo/D2plusda"]) < 1e-13
    assert rel(cosmo.table("superconft"), golden["cosmo/superconft"]) < 1e-13
    ref = json.loads(str(golden["cosmo/attrs"]))["Dplus_unnormed_at_1"]
    assert abs(cosmo.D1_unnormed_at_1 / ref - 1) < 1e-13
    assert abs(cosmo.Omega_m - json.loads(str(golden["cosmo/attrs"]))["Omega_m"]) < 1e-15


def test_cosmology_matches_oracle():
    from oracle import cosmology as cz
    p = dict(Omega_c=0.261, Omega_b=0.049, h=0.677, sigma8=0.81, n_s=0.965)
    a = djb200.Cosmology(**p)
    b = cz.compute_timetables(cz.Cosmology(**p))
    assert rel(a.table("Dplus"), b.D1_table) < 1e-14
    assert rel(a.table("D3a"), b.D3a_table) < 1e-13
    for x in (1e-3, 0.02, 0.5, 1.0):
        assert abs(a.Fplus(x) / cz.Fplus(b, x) - 1) < 1e-13
        assert abs(a.Dplus(x) / cz.Dplus(b, x) - 1) < 1e-14


@pytest.mark.parametrize("name", PARITY_CONFIGS)
def test_stepper_coefficients(golden, cosmo, name):
    kw = run_kwargs(golden, name)
    co = djb200.stepper_coefficients(cosmo, kw["stepper"], kw["a_ini"], kw["a_end"], kw["n_steps"],
                                     time_var=kw["time_var"])
    for k in ("alpha", "beta", "ddrift1", "ddrift2", "all_a"):
        assert rel(co[k], golden[f"{name}/{k}"]) < 1e-12, k


def test_unknown_cosmology_and_stepper_raise(cosmo):
    with pytest.raises(djb200.DJBInvalidOption, match="Unknown cosmology"):
        djb200.Cosmology("NotACosmology")
    with pytest.raises(djb200.DJBInvalidOption, match="stepper must be"):
        djb200.stepper_coefficients(cosmo, "leapfrog", 0.05, 1.0, 4)
    with pytest.raises(djb200.DJBInvalidOption, match="time_var"):
        djb200.stepper_coefficients(cosmo, "fastpm", 0.05, 1.0, 4, time_var="t")
    with pytest.raises(djb200.DJBInvalidOption, match="n_steps \\+ 1"):
        djb200.stepper_coefficients(cosmo, "fastpm", 0.05, 1.0, 4, time_var=np.array([0.1, 0.5, 1.0]))


@pytest.mark.parametrize("field,value,msg", [
    ("worder", 5, "worder must be 2, 3 or 4"),
    ("grad_order", 3, "grad_order must be 0, 2, 4 or 6"),
    ("lap_order", 1, "lap_order must be 0, 2, 4 or 6"),
    ("antialias", 4, "antialias must be -1, 0, 1, 2 or 3"),
    ("resampling", "cubic", "resampling must be :fourier or :linear"),
])
def test_invalid_pm_options_raise_before_touching_the_device(field, value, msg):
    cfg = djb200.PMConfig(res_pm=32, n_part=16, boxsize=100.0)
    setattr(cfg, field, value)
    with pytest.raises(djb200.DJBInvalidOption, match=msg):
        djb200.PMSolver(cfg)


def test_lean_restrictions_raise():
    """PMSolverLean supports antialias = 0, n_resample = 1, FD gradients (pm.jl:570-571)."""
    for kw in (dict(antialias=1), dict(n_resample=2), dict(grad_order=0)):
        cfg = djb200.PMConfig(res_pm=32, n_part=16, boxsize=100.0, **kw)
        with pytest.raises(djb200.DJBInvalidOption, match="PMSolverLean supports"):
            djb200.PMSolver(cfg, lean=True)


def test_lpt_ics_match_fixture(golden, cosmo):
    """fphi -> compute_core(n_order=2) -> nbody_ics_lpt reproduces the fixture's
    Ψ, Π at a = 0.05 (nbody_parity_tests.jl:28-34, tolerance 1e-12)."""
    import torch

    from djb200 import ics
    fphi = torch.from_numpy(golden["ics/fphi_re"] + 1j * golden["ics/fphi_im"])
    shapes = {k: v.numpy() for k, v in ics.compute_core(fphi, 100.0, n_order=2).items()}
    psi, pi = djb200.nbody_ics_lpt(cosmo, shapes, 0.05, 2)
    assert rel(psi, golden["ics/psi_ini"]) < 1e-12
    assert rel(pi, golden["ics/pi_ini"]) < 1e-12
    # 1LPT shape at a = 1 (the fixture's psi1 is dΨ/dD of 1LPT)
    assert rel(shapes["psi_1"], golden["ics/psi1"]) < 1e-12


def test_3lpt_shapes_are_transverse_free_at_second_order_and_scale_cubically(golden):
    """3LPT ψ₃ scales as φ³ and ψ₂ as φ² (EdS shapes are homogeneous in φ)."""
    import torch

    from djb200 import ics
    fphi = torch.from_numpy(golden["ics/fphi_re"] + 1j * golden["ics/fphi_im"])
    a = ics.compute_core(fphi, 100.0, n_order=3)
    b = ics.compute_core(2.0 * fphi, 100.0, n_order=3)
    assert rel(b["psi_2"].numpy(), 4.0 * a["psi_2"].numpy()) < 1e-12
    assert rel(b["psi_3"].numpy(), 8.0 * a["psi_3"].numpy()) < 1e-12
    assert float(a["psi_3"].abs().max()) > 0


def _eds_growth_known_answers(D1, Dda, D2, D3):
    """The reference's growth known answers (test/runtests.jl:40-54): EdS-like growth at
    high redshift, D(0.04)/D(0.02) = 2 within 0.05 and f(0.02) = 1 within 0.05; the
    higher-order growth factors at their EdS limits at a = 0.01 within 2%
    (D2 = -3/7 D1², D3a = 1/3 D1³, D3b = -10/21 D1³, D3c = 1/7 D1³); D2(1) < 0."""
    assert abs(D1(0.04) / D1(0.02) - 2.0) < 0.05
    assert abs(0.02 * Dda(0.02) / D1(0.02) - 1.0) < 0.05
    a = 0.01
    d1 = D1(a)
    assert abs(D2(a) / (-3 / 7 * d1 ** 2) - 1) < 2e-2
    for name, coef in (("D3a", 1 / 3), ("D3b", -10 / 21), ("D3c", 1 / 7)):
        assert abs(D3(name, a) / (coef * d1 ** 3) - 1) < 2e-2, name
    assert D2(1.0) < 0


def test_growth_known_answers_library_and_oracle():
    from oracle import cosmology as cz
    c = djb200.Cosmology("Planck18EEBAOSN")
    at = c.table("a")
    _eds_growth_known_answers(c.Dplus, c.growth_Dplusda, c.D2plus,
                              lambda name, x: float(np.interp(x, at, c.table(name))))
    o = cz.compute_timetables(cz.Cosmology.named("Planck18EEBAOSN"))
    _eds_growth_known_answers(lambda x: cz.Dplus(o, x), lambda x: cz.growth_Dplusda(o, x),
                              lambda x: cz.D2plus(o, x),
                              lambda name, x: float(np.interp(x, o.a_table, getattr(o, name + "_table"))))


def test_transfer_and_sigma8_known_answers():
    """The reference's transfer and linear-P(k) known answers (test/runtests.jl:56-86):
    the Eisenstein-Hu T(k) lies in (0, 1] and tends to 1 at k = 1e-3 h/Mpc (within 0.05);
    σ8 integrated back from the P(k) table with the 8 Mpc/h top hat (trapezoid in k)
    is the cosmology's σ8 within 1%. For the package's generator and the oracle's."""
    import math

    from djb200 import ics
    from oracle import ics as oi
    p = djb200.Cosmology("Planck18EEBAOSN").params
    p = p() if callable(p) else p
    k = 10.0 ** np.linspace(-3, 1, 100)
    tables = []
    for T, (kk, pk) in ((ics.eisenstein_hu(p, k), ics.linear_power_spectrum(p)),
                        (oi.eisenstein_hu(p["Omega_c"], p["Omega_b"], p["h"], k),
                         oi.linear_power_spectrum(p["Omega_c"], p["Omega_b"], p["h"], p["n_s"], p["sigma8"]))):
        assert np.all((T > 0) & (T <= 1.0))
        assert abs(T[0] - 1.0) < 0.05
        assert np.all(pk > 0)
        x = kk * 8.0
        W = 3 * (np.sin(x) - x * np.cos(x)) / x ** 3
        W[x < 1e-3] = 1.0
        integ = kk ** 2 * pk * W ** 2 / (2 * math.pi ** 2)
        s8 = math.sqrt(np.sum(0.5 * (integ[:-1] + integ[1:]) * np.diff(kk)))
        assert abs(s8 - p["sigma8"]) / p["sigma8"] < 0.01
        tables.append(pk)
    assert rel(tables[0], tables[1]) < 1e-12


@pytest.mark.parametrize("generator", ["package", "oracle"])
def test_lpt_known_answers(generator):
    """The reference's IC known answers (test/runtests.jl:121-171) at 16³, L = 100, for
    the package's CPU generator (white noise -> φ -> compute_core) and the oracle's
    invariant-form shapes: 1LPT has no bulk motion (|mean Ψ_x| < 0.1); rms Ψ grows as
    D ∝ a in matter domination (rms(a=0.04)/rms(a=0.02) = 2 within 0.05); 2LPT differs
    from 1LPT at a = 0.02, by less than 5% of the rms; positions mod(q + Ψ, L) at a = 0.1
    lie in [0, L)."""
    import torch

    from djb200 import ics
    from oracle import ics as oi
    n, L = 16, 100.0
    c = djb200.Cosmology("Planck18EEBAOSN")
    p = c.params() if callable(c.params) else c.params
    fphi = ics.white_noise_to_fphi(ics.white_noise(42, n), L, ics.linear_power_spectrum(p))
    if generator == "package":
        shp = {k: v.numpy() for k, v in ics.compute_core(fphi, L, n_order=2).items()}
        s1, s2 = shp["psi_1"], shp["psi_2"]
    else:
        s1, s2 = oi.lpt_shapes(fphi.numpy(), L, order=2)

    def psi(a, order):
        D = c.Dplus(a)
        return D * s1 + (D * D * s2 if order == 2 else 0.0)

    rms = lambda x: float(np.sqrt(np.mean(x ** 2)))
    assert abs(float(np.mean(psi(0.02, 1)[..., 0]))) < 0.1
    assert abs(rms(psi(0.04, 1)) / rms(psi(0.02, 1)) - 2.0) < 0.05
    frac = rms(psi(0.02, 1) - psi(0.02, 2)) / rms(psi(0.02, 1))
    assert 0 < frac < 0.05
    q = (np.stack(np.meshgrid(*(np.arange(n),) * 3, indexing="ij"), axis=-1)) * (L / n)
    pos = np.mod(q + psi(0.1, 1), L)
    assert np.all((pos >= 0) & (pos < L))


def test_power_spectrum_white_noise_known_answer():
    """The reference's P(k) known answer (test/runtests.jl:175-187) for the oracle's
    `evaluate_power_spectrum` (the checker of the library's P(k)): white noise on 32³,
    L = 100, 10 bins: 10 values, P ≥ 0, bin centres increasing, and the mean of the
    non-empty bins within a factor 2 of the shot noise V/N (not V²/N)."""
    from oracle import power as opw
    rng = np.random.default_rng(0)
    res, L = 32, 100.0
    k, pk, nm = opw.evaluate_power_spectrum(rng.standard_normal((res, res, res)), L, bins=10)
    assert len(k) == 10 and np.all(pk >= 0) and np.all(np.diff(k) > 0)
    Vn = L ** 3 / res ** 3
    nz = pk[pk > 0]
    assert 0.5 * Vn < nz.mean() < 2.0 * Vn
