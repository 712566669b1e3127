"""The CPU oracle against the reference's JAX golden vectors, at the reference's own
tolerances (native/DiscoDJNative/test/nbody_parity_tests.jl:17-61)."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, PARITY_CONFIGS, REFERENCE_H5, config_attrs, rel, run_kwargs
from oracle import cosmology as cz
from oracle import nbody as onb
from oracle import pm as opm


@pytest.fixture(scope="module")
def cosmo():
    return cz.Cosmology.named("Planck18EEBAOSN")


def test_golden_archive_matches_reference_fixture():
    """The committed npz is a faithful conversion of the reference's HDF5 file."""
    if not REFERENCE_H5 or not os.path.exists(REFERENCE_H5):
        pytest.skip("reference checkout not present (set DISCODJ_REFERENCE to its root)")
    from golden.make_golden import extract

    src = extract(REFERENCE_H5)
    d = np.load(GOLDEN)
    assert set(src) == set(d.files)
    for k, v in src.items():
        if v.dtype.kind in "fc":
            assert np.array_equal(v, d[k]), k
        else:
            assert str(v) == str(d[k]), k


def test_timetables(golden, cosmo):
    assert rel(cosmo.D1_table, golden["cosmo/Dplus"]) < 1e-13
    assert rel(cz.Dplusda_tab(cosmo), golden["cosmo/Dplusda"]) < 1e-13
    assert rel(cosmo.D2_table, golden["cosmo/D2plus"]) < 1e-13
    assert rel(cz.D2plusda_tab(cosmo), golden["cosmo/D2plusda"]) < 1e-13
    assert rel(cosmo.superconft_table, golden["cosmo/superconft"]) < 1e-13
    ref = json.loads(str(golden["cosmo/attrs"]))["Dplus_unnormed_at_1"]
    assert abs(cosmo.D1_unnormed_at_1 / ref - 1) < 1e-13


@pytest.mark.parametrize("name", PARITY_CONFIGS)
def test_stepper_coefficients(golden, cosmo, name):
    kw = run_kwargs(golden, name)
    co = onb.stepper_coefficients(cosmo, kw["stepper"], kw["a_ini"], kw["a_end"], kw["n_steps"],
                                  time_var=kw["time_var"])
    for k in ("alpha", "beta", "ddrift1", "ddrift2", "all_a"):
        assert rel(co[k], golden[f"{name}/{k}"]) < 1e-12, k


def _cfg(golden, name):
    kw = run_kwargs(golden, name)
    return opm.PMConfig(res_pm=kw["res_pm"], n_part=16, boxsize=100.0, worder=kw["worder"],
                        deconvolve=kw["deconvolve"], antialias=kw["antialias"], grad_order=kw["grad_kernel_order"],
                        lap_order=kw["laplace_kernel_order"], n_resample=kw["n_resample"],
                        resampling=kw["resampling_method"])


@pytest.mark.parametrize("name", PARITY_CONFIGS)
def test_pm_acceleration(golden, name):
    acc = opm.pm_acceleration(_cfg(golden, name), golden["ics/psi_ini"])
    assert rel(acc, golden[f"{name}/acc_ini"]) < 1e-12


@pytest.mark.parametrize("name", PARITY_CONFIGS)
def test_run_nbody(golden, cosmo, name):
    kw = run_kwargs(golden, name)
    a = config_attrs(golden, name)
    if a["ic_method"] == "bullfrog":
        p0, m0 = onb.bullfrog_ics(cosmo, golden["ics/psi1"], kw["a_ini"], boxsize=100.0, res_pm=kw["res_pm"])
    else:
        p0, m0 = golden["ics/psi_ini"], golden["ics/pi_ini"]
    psi, p, _ = onb.run_nbody(cosmo, p0, m0, return_displacement=True, **kw)
    assert rel(psi, golden[f"{name}/psi_out"]) < 1e-11
    assert rel(p, golden[f"{name}/p_out"]) < 1e-11


def test_linear_bug_group_is_not_the_fixed_one(golden):
    """The upstream linear-resampling bug group differs from the fixed one; the
    oracle follows the fixed coordinate (pm.jl:23-26)."""
    a = golden["bullfrog_resample_linear/acc_ini"]
    b = golden["bullfrog_resample_linear_fixed/acc_ini"]
    assert rel(a, b) > 1e-6


def test_fd_gradient_equals_fourier_kernel(golden):
    """Circulant identity behind the real-space FD stencil (pm.jl:309-311): the
    order-2/4/6 stencil on φ equals the Fourier gradient kernel."""
    cfg = opm.PMConfig(res_pm=32, n_part=16, boxsize=100.0, grad_order=6)
    X = onb.add_q(golden["ics/psi_ini"], 100.0)
    phi = opm.potential(cfg, X)
    c1, c2, c3 = opm.fd_coeffs(6, 100.0 / 32)
    fx = -(c1 * (np.roll(phi, -1, 0) - np.roll(phi, 1, 0)) + c2 * (np.roll(phi, -2, 0) - np.roll(phi, 2, 0))
           + c3 * (np.roll(phi, -3, 0) - np.roll(phi, 3, 0)))
    K = opm.PMKernels(cfg)
    fk = opm.irfftn(-(K.gx * opm.rfftn(phi)), 32)
    assert rel(fx, fk) < 1e-12


def test_invalid_options_raise():
    cfg = opm.PMConfig(res_pm=32, n_part=16, boxsize=100.0, grad_order=3)
    with pytest.raises(ValueError, match="grad_order must be 0, 2, 4 or 6"):
        opm.pm_acceleration(cfg, np.zeros((16, 16, 16, 3)))
    with pytest.raises(ValueError, match="antialias"):
        opm.aa_shifts(5, 0.1)


def test_oracle_zeldovich_shape_matches_fixture(golden):
    """The oracle's 1LPT shape −∇φ (used for the CPU-side ICs) reproduces the fixture's
    psi1 from its fphi (nbody_parity_tests.jl:28-34 tolerance 1e-12)."""
    from oracle import ics as oi
    fphi = golden["ics/fphi_re"] + 1j * golden["ics/fphi_im"]
    assert rel(oi.zeldovich_shape(fphi, 100.0), golden["ics/psi1"]) < 1e-12


def test_oracle_2lpt_matches_fixture(golden, cosmo):
    """The oracle's invariant-form nLPT (oracle/ics.py `lpt_shapes`) at second order gives
    the fixture's 2LPT Ψ, Π at a = 0.05 from its fphi (tolerance 1e-12)."""
    from oracle import ics as oi
    fphi = golden["ics/fphi_re"] + 1j * golden["ics/fphi_im"]
    psi1, psi2 = oi.lpt_shapes(fphi, 100.0, order=2)
    tabs = cz.compute_timetables(cosmo)
    D = cz.Dplus(tabs, 0.05)
    assert rel(D * psi1 + D * D * psi2, golden["ics/psi_ini"]) < 1e-12
    assert rel(psi1 + 2 * D * psi2, golden["ics/pi_ini"]) < 1e-12


@pytest.mark.parametrize("n", [16, 32])
def test_oracle_3lpt_pins_the_index_table_restatement(golden, n):
    """The third order has no golden vector; the oracle's invariant form (μ₂(A,B) =
    tr A tr B − Σ A_ba B_ab, μ₃ = det A, the transverse part from A·B − (A·B)ᵀ) and the
    package's restatement with the reference's index tables (`djb200.ics.compute_core`,
    whose third-order shape the GPU generator is tested against) agree at round-off."""
    import torch

    from djb200 import ics
    from oracle import ics as oi
    rng = np.random.default_rng(n)
    white = rng.standard_normal((n, n, n))
    pk = oi.linear_power_spectrum(0.261, 0.049, 0.677, 0.965, 0.81)
    fphi = oi.fphi_from_white(white, 0.5 * n * 2.0, pk)
    ref = oi.lpt_shapes(fphi, 0.5 * n * 2.0, order=3)
    got = ics.compute_core(torch.from_numpy(fphi), 0.5 * n * 2.0, n_order=3)
    for m in (1, 2, 3):
        assert rel(got[f"psi_{m}"].numpy(), ref[m - 1]) < 1e-12


def test_oracle_plane_wave_linear_growth(cosmo):
    """nbody_parity_tests.jl:68-90 on the float64 oracle, at the reference's own bars: a
    1e-3 fundamental plane wave stays one-dimensional (transverse < 1e-12) and grows as
    D(a) to within 1e-2 at 32³ for BullFrog (1 and 16 steps), FastPM (16) and the
    symplectic stepper (64), the error falling more than 3x from 16³ to 32³."""
    from oracle import nbody as onb
    c = cz.compute_timetables(cosmo)
    L, a0 = 100.0, 0.05
    D0, D1 = cz.Dplus(c, a0), cz.Dplus(c, 1.0)
    for st, ns in (("bullfrog", 1), ("bullfrog", 16), ("fastpm", 16), ("symplectic", 64)):
        err = {}
        for n in (16, 32):
            q = np.arange(n) * (L / n)
            psi1 = np.zeros((n, n, n, 3))
            psi1[..., 0] = (1e-3 * np.sin(2 * np.pi * q / L))[:, None, None]
            Psi, _, _ = onb.run_nbody(c, D0 * psi1, psi1.copy(), boxsize=L, a_ini=a0, a_end=1.0, n_steps=ns,
                                      res_pm=2 * n, stepper=st, return_displacement=True)
            assert np.max(np.abs(Psi[..., 1:])) < 1e-12
            err[n] = abs(np.sum(Psi[..., 0] * psi1[..., 0]) / np.sum(psi1[..., 0] ** 2) / D1 - 1)
        assert err[32] < 1e-2, (st, ns)
        assert err[16] / err[32] > 3, (st, ns)
