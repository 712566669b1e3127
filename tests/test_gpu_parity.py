"""GPU parity: the CUDA path through the C ABI against the float64 oracle and the
reference's golden vectors, every PM option of the fixture (16³ particles, 32³ mesh).

Tolerances (float32 kernels vs float64 references, metric max|x−y|/max|y|):
  acceleration 2e-5, displacement and momentum after the run 2e-5, P(k) 1e-4 per bin.
  Runs with deconvolution get 6e-5: the sinc^(-2W) window amplifies float32 round-off
  at high k; a float32 CPU restatement of the same run already sits at 1.1e-5 (Ψ) and
  3.4e-5 (P) from the float64 golden vectors for `symplectic_a_pcs_deconv`.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import PARITY_CONFIGS, config_attrs, rel, run_kwargs

pytestmark = pytest.mark.gpu

ACC_TOL = 2e-5
RUN_TOL = 2e-5
RUN_TOL_DECONV = 6e-5
PK_TOL = 1e-4


@pytest.fixture(scope="module")
def djb(cuda_device):
    import djb200
    return djb200


@pytest.fixture(scope="module")
def cosmo(djb):
    return djb.Cosmology("Planck18EEBAOSN")


def _cfg(djb, golden, name):
    kw = run_kwargs(golden, name)
    return djb.PMConfig(res_pm=kw["res_pm"], n_part=16, boxsize=100.0, worder=kw["worder"],
                        deconvolve=kw["deconvolve"], antialias=kw["antialias"], grad_order=kw["grad_kernel_order"],
                        lap_order=kw["laplace_kernel_order"], n_resample=kw["n_resample"],
                        resampling=kw["resampling_method"])


@pytest.mark.parametrize("name", PARITY_CONFIGS)
def test_pm_acceleration_vs_golden(djb, golden, name):
    acc = djb.pm_acceleration(golden["ics/psi_ini"], _cfg(djb, golden, name))
    assert acc.shape == (16, 16, 16, 3) and acc.dtype == np.float32
    assert rel(acc, golden[f"{name}/acc_ini"]) < ACC_TOL


@pytest.mark.parametrize("name", PARITY_CONFIGS)
def test_run_nbody_vs_golden(djb, golden, cosmo, name):
    kw = run_kwargs(golden, name)
    a = config_attrs(golden, name)
    if a["ic_method"] == "bullfrog":
        p0, m0 = djb.bullfrog_ics(cosmo, golden["ics/psi1"], kw["a_ini"], boxsize=100.0, res_pm=kw["res_pm"])
    else:
        p0, m0 = golden["ics/psi_ini"], golden["ics/pi_ini"]
    psi, p, a_end = djb.run_nbody(cosmo, p0, m0, return_displacement=True, **kw)
    assert a_end == kw["a_end"]
    # bullfrog ICs come from a PCS + deconvolution step (run_nbody.jl:219-220)
    tol = RUN_TOL_DECONV if (kw["deconvolve"] or a["ic_method"] == "bullfrog") else RUN_TOL
    assert rel(psi, golden[f"{name}/psi_out"]) < tol
    assert rel(p, golden[f"{name}/p_out"]) < tol


def test_wrapped_positions_and_all_a(djb, golden, cosmo):
    kw = run_kwargs(golden, "bullfrog_D_cic")
    X, P, all_a = djb.run_nbody(cosmo, golden["ics/psi_ini"], golden["ics/pi_ini"], return_all_a=True, **kw)
    assert np.all(X >= 0) and np.all(X < 100.0)
    from oracle import nbody as onb
    Xr = np.mod(onb.add_q(golden["bullfrog_D_cic/psi_out"], 100.0) + 100.0, 100.0)
    d = np.abs(X - Xr)
    d = np.minimum(d, 100.0 - d)  # periodic distance
    assert d.max() < 1e-3
    assert rel(all_a, golden["bullfrog_D_cic/all_a"]) < 1e-12


def test_callbacks_and_history(djb, golden, cosmo):
    """step_callback/callback_when select steps (pm_lean_tests.jl:121-124); collect_all
    returns every step; the per-step path equals the fused run."""
    kw = run_kwargs(golden, "fastpm_D_tsc")
    seen = []
    djb.run_nbody(cosmo, golden["ics/psi_ini"], golden["ics/pi_ini"], return_displacement=True,
                  step_callback=lambda k, a, X, P: seen.append(k), callback_when=lambda k, a: k in (0, 4, 6), **kw)
    assert seen == [0, 4, 6]
    hx, hp, all_a = djb.run_nbody(cosmo, golden["ics/psi_ini"], golden["ics/pi_ini"], return_displacement=True,
                                  collect_all=True, **kw)
    assert len(hx) == kw["n_steps"] + 1 and len(all_a) == kw["n_steps"] + 1
    assert rel(hx[0], golden["ics/psi_ini"]) < 1e-6
    assert rel(hx[-1], golden["fastpm_D_tsc/psi_out"]) < RUN_TOL
    assert rel(hp[-1], golden["fastpm_D_tsc/p_out"]) < RUN_TOL


def test_lean_equals_full(djb):
    """PMSolverLean ≡ PMSolver (pm_lean_tests.jl:96-107): n=24, res=48, L=120."""
    rng = np.random.default_rng(5)
    psi = (3 * rng.standard_normal((24, 24, 24, 3))).astype(np.float32)
    for W, g in ((2, 4), (3, 2), (4, 6)):
        cfg = djb.PMConfig(res_pm=48, n_part=24, boxsize=120.0, worder=W, grad_order=g)
        with djb.PMSolver(cfg) as a, djb.PMSolver(cfg, lean=True) as b:
            x, y = a.acceleration(psi), b.acceleration(psi)
        assert rel(x, y) < 2e-5


@pytest.mark.parametrize("W,g,aa,lap,dec", [(2, 4, 0, 0, False), (3, 2, 0, 4, False), (4, 6, 1, 0, True),
                                            (2, 6, 2, 6, False), (4, 0, 1, 0, True), (3, 4, -1, 2, True)])
def test_random_particles_vs_oracle(djb, W, g, aa, lap, dec):
    """Strongly clustered random displacements (n=24, res=48) against the float64 oracle."""
    from oracle import pm as opm
    rng = np.random.default_rng(7 + W)
    psi = (3 * rng.standard_normal((24, 24, 24, 3)))
    cfg_o = opm.PMConfig(res_pm=48, n_part=24, boxsize=120.0, worder=W, grad_order=g, antialias=aa,
                         lap_order=lap, deconvolve=dec)
    cfg_d = djb.PMConfig(res_pm=48, n_part=24, boxsize=120.0, worder=W, grad_order=g, antialias=aa,
                         lap_order=lap, deconvolve=dec)
    ref = opm.pm_acceleration(cfg_o, psi.astype(np.float32).astype(np.float64))
    got = djb.pm_acceleration(psi.astype(np.float32), cfg_d)
    assert rel(got, ref) < ACC_TOL


def test_device_arrays_roundtrip(djb, golden):
    """CuArray-style call: device pointers in, device pointers out."""
    import torch
    cfg = _cfg(djb, golden, "bullfrog_D_cic")
    psi_d = djb.native_view(torch.from_numpy(golden["ics/psi_ini"].astype(np.float32)).cuda())
    with djb.PMSolver(cfg) as S:
        acc_d = S.acceleration(psi_d)
        acc_h = S.acceleration(golden["ics/psi_ini"])
    got = djb.logical_view(acc_d).cpu().numpy()
    # float atomics in the mass assignment sum in a run-dependent order
    assert rel(got, acc_h) < 1e-6


def test_power_spectrum_vs_oracle(djb):
    from oracle import power as opw
    rng = np.random.default_rng(3)
    field = rng.standard_normal((32, 32, 32))
    field[3:9, 4:7, 10:20] += 4.0
    k, pk, nm = djb.evaluate_power_spectrum(field.astype(np.float32), 250.0, bins=32, logarithmic=True)
    kr, pkr, nmr = opw.evaluate_power_spectrum(field.astype(np.float32).astype(np.float64), 250.0, bins=32)
    assert np.array_equal(nm, nmr)
    assert rel(k, kr) < 1e-13
    nz = nmr > 0
    assert np.max(np.abs(pk[nz] / pkr[nz] - 1)) < PK_TOL
    assert np.all(pk[~nz] == 0)
    kl, pl, nl = djb.evaluate_power_spectrum(field.astype(np.float32), 250.0, bins=12, logarithmic=False)
    klr, plr, nlr = opw.evaluate_power_spectrum(field.astype(np.float32).astype(np.float64), 250.0, bins=12,
                                                logarithmic=False)
    assert np.array_equal(nl, nlr) and np.max(np.abs(pl / plr - 1)) < PK_TOL


def test_state_power_spectrum_vs_oracle(djb, golden):
    """CIC deposit of the resident state -> δ -> P(k) (measure.jl:430-447)."""
    from oracle import nbody as onb
    from oracle import pm as opm
    from oracle import power as opw
    cfg = _cfg(djb, golden, "bullfrog_D_cic")
    with djb.PMSolver(cfg) as S:
        S.set_state(golden["ics/psi_ini"], golden["ics/pi_ini"])
        k, pk, nm = S.state_power_spectrum(bins=16)
    X = onb.add_q(golden["ics/psi_ini"].astype(np.float32).astype(np.float64), 100.0).reshape(-1, 3)
    mesh = opm.pm_scatter(np.zeros((32, 32, 32)), X, 32, 100.0, 2)
    kr, pkr, nmr = opw.evaluate_power_spectrum(opw.density_contrast(mesh, 16), 100.0, bins=16)
    assert np.array_equal(nm, nmr)
    nz = nmr > 0
    assert np.max(np.abs(pk[nz] / pkr[nz] - 1)) < PK_TOL


def test_nonfinite_position_is_reported_not_faulted(djb, golden):
    """A NaN displacement sets the kernels' device error word; the call fails with
    DJB_ERR_DEVICE and the solver stays usable."""
    cfg = _cfg(djb, golden, "bullfrog_D_cic")
    psi = golden["ics/psi_ini"].astype(np.float32).copy()
    psi[3, 4, 5, 1] = np.nan
    with djb.PMSolver(cfg) as S:
        with pytest.raises(djb.DJBError, match="non-finite"):
            S.acceleration(psi)
        acc = S.acceleration(golden["ics/psi_ini"])
    assert rel(acc, golden["bullfrog_D_cic/acc_ini"]) < ACC_TOL


def test_state_calls_need_state(djb, golden):
    cfg = _cfg(djb, golden, "bullfrog_D_cic")
    with djb.PMSolver(cfg) as S:
        with pytest.raises(djb.DJBError, match="no particle state"):
            S.step(0.1, 1.0, 0.0, 0.1)


@pytest.mark.parametrize("W,n,res,clump,aa", [(4, 24, 48, 3000, 0), (4, 24, 48, 3000, 1), (3, 24, 48, 6000, 0),
                                               (2, 24, 48, 5000, 0), (4, 32, 64, 20000, 0)])
def test_dense_clump_vs_oracle(djb, W, n, res, clump, aa):
    """Thousands of particles on one node (a collapsed halo core): the brick deposit's
    32-bit fixed point must not wrap. `clump` particles sit on one mesh node and the
    rest stay near their lattice sites. The bricks holding the clump take reduced
    fixed-point units: 2^21 (PCS, 3000), 2^20 (TSC, 6000), 2^19 (CIC, 5000; PCS, 20000)."""
    from oracle import nbody as onb
    from oracle import pm as opm
    L = 120.0
    rng = np.random.default_rng(31 + W + n)
    psi = 0.3 * rng.standard_normal((n, n, n, 3))
    X = onb.add_q(psi, L)
    node = np.array([17.0, 9.0, 30.0]) * (L / res)           # one mesh node
    idx = rng.choice(n ** 3, size=clump, replace=False)
    flat = X.reshape(-1, 3)
    flat[idx] = node
    q = onb.add_q(np.zeros_like(psi), L)
    psi = (X - q).astype(np.float32)
    cfg_o = opm.PMConfig(res_pm=res, n_part=n, boxsize=L, worder=W, grad_order=4, antialias=aa)
    cfg_d = djb.PMConfig(res_pm=res, n_part=n, boxsize=L, worder=W, grad_order=4, antialias=aa)
    ref = opm.pm_acceleration(cfg_o, psi.astype(np.float64))
    got = djb.pm_acceleration(psi, cfg_d)
    # a wrapped node sum would corrupt the force everywhere; the clump's own particles are
    # left out: their force is the float32 residue of the clump's symmetric self-force,
    # thousands of times larger in each term than in the sum
    keep = np.ones(n ** 3, dtype=bool)
    keep[idx] = False
    g = got.reshape(-1, 3)[keep]
    r = ref.reshape(-1, 3)[keep]
    assert rel(g, r) < ACC_TOL


def test_state_density_modes_vs_oracle(djb):
    """measure.jl:80-91 `density_modes`: CIC δ of the particle state, Fourier modes / res³,
    CIC window divided out; against the float64 oracle's deposit and numpy's FFT."""
    from oracle import nbody as onb
    from oracle import pm as opm
    n, res, L = 32, 32, 100.0
    rng = np.random.default_rng(17)
    psi = (1.5 * rng.standard_normal((n, n, n, 3))).astype(np.float32)
    modes = rng.integers(-res // 2 + 1, res // 2 + 1, size=(40, 3))
    modes[0] = (0, 0, 0)
    modes[1] = (1, 0, 0)
    modes[2] = (-3, 2, -1)
    with djb.PMSolver(djb.PMConfig(res_pm=res, n_part=n, boxsize=L)) as S:
        S.set_state(psi, psi)
        got = S.state_density_modes(modes)
    X = onb.add_q(psi.astype(np.float64), L).reshape(-1, 3)
    mesh = opm.pm_scatter(np.zeros((res, res, res)), X, res, L, 2)       # [ix,iy,iz]
    delta = mesh * (res ** 3 / n ** 3) - 1.0
    dk = np.fft.fftn(delta) / res ** 3
    ref = np.array([dk[m[0] % res, m[1] % res, m[2] % res] for m in modes])
    W = np.prod(np.sinc(modes / res) ** 2, axis=1)
    ref = ref / W
    ref[0] = 0.0
    assert np.max(np.abs(got - ref)) < 1e-5 * np.max(np.abs(ref))


def test_bounded_wait_runs_out_and_reports(djb):
    """The bulk-copy kernels' mbarrier wait is bounded: made to run out (a barrier that
    nothing completes), it sets error bit 8 and returns; the device stays usable."""
    import ctypes as C

    from djb200 import _lib
    err = C.c_int32(-1)
    _lib.check(_lib.lib.djb_selftest_bounded_wait(0, 1, 1 << 20, C.byref(err)))
    assert err.value == 0                      # the barrier completed
    _lib.check(_lib.lib.djb_selftest_bounded_wait(0, 0, 1 << 20, C.byref(err)))
    assert err.value & 8                       # the wait ran out and said so
    # the context is intact: an ordinary force call still works
    rng = np.random.default_rng(2)
    psi = rng.standard_normal((16, 16, 16, 3)).astype(np.float32)
    acc = djb.pm_acceleration(psi, djb.PMConfig(res_pm=32, n_part=16, boxsize=100.0, worder=4, grad_order=4))
    assert np.all(np.isfinite(acc))


def test_lpt_ics_on_the_gpu_match_the_pinned_cpu_path(djb):
    """The initial conditions run the same torch restatement on the GPU in float32 as on
    the CPU in float64, where 2LPT is pinned to the fixture at 1e-12: white noise → φ →
    2LPT / 3LPT shapes → (Ψ, Π) at a = 0.02, 32³ particles, L = 62.5."""
    import torch

    from djb200 import ics
    c = djb.Cosmology("Planck18EEBAOSN")
    w = ics.white_noise(5, 32, device="cpu", dtype=torch.float64)
    for order in (2, 3):
        p64, m64 = ics.lpt_ics(c, 32, 62.5, 0.02, n_order=order, white=w)
        p32, m32 = ics.lpt_ics(c, 32, 62.5, 0.02, n_order=order, device="cuda", dtype=torch.float32,
                               white=w.float().cuda())
        assert rel(p32.cpu().numpy(), p64.numpy()) < 1e-5
        assert rel(m32.cpu().numpy(), m64.numpy()) < 1e-5


@pytest.mark.parametrize("n,L", [(32, 62.5), (64, 250.0)])
def test_native_2lpt_ics_match_the_pinned_cpu_path(djb, n, L):
    """The CUDA 2LPT generator (djb_lpt2_ics) against the torch restatement in float64 on
    the CPU, whose 2LPT reproduces the fixture's ICs at 1e-12: same white noise, a = 0.02."""
    import torch

    from djb200 import ics
    c = djb.Cosmology("Planck18EEBAOSN")
    w = ics.white_noise(9, n, device="cpu", dtype=torch.float64)
    p64, m64 = ics.lpt_ics(c, n, L, 0.02, n_order=2, white=w)
    psi, pi = ics.lpt2_ics_native(c, n, L, 0.02, white=w.float())
    got_p = djb.logical_view(psi).cpu().numpy()
    got_m = djb.logical_view(pi).cpu().numpy()
    assert rel(got_p, p64.numpy()) < 1e-5
    assert rel(got_m, m64.numpy()) < 1e-5
    # the second-order part itself: Π − Ψ/D = D ψ₂
    D = c.Dplus(0.02)
    s2 = got_m - got_p / D
    r2 = (m64 - p64 / D).numpy()
    assert rel(s2, r2) < 1e-3


@pytest.mark.parametrize("n,L", [(32, 62.5), (64, 250.0)])
def test_native_3lpt_ics_match_the_cpu_path(djb, n, L):
    """The CUDA 3LPT generator (djb_lpt_ics, n_order = 3) against the torch restatement of
    compute_core in float64 on the CPU (whose 2LPT part the fixture pins): same white
    noise, at a = 0.02 (the configuration's start) and at a = 1, where the third-order
    shape is a sizeable part of Ψ and is compared on its own (3LPT minus 2LPT)."""
    import torch

    from djb200 import ics
    c = djb.Cosmology("Planck18EEBAOSN")
    w = ics.white_noise(5, n, device="cpu", dtype=torch.float64)
    for a in (0.02, 1.0):
        p64, m64 = ics.lpt_ics(c, n, L, a, n_order=3, white=w)
        psi, pi = ics.lpt_ics_native(c, n, L, a, n_order=3, white=w.float())
        got_p = djb.logical_view(psi).cpu().numpy()
        got_m = djb.logical_view(pi).cpu().numpy()
        assert rel(got_p, p64.numpy()) < 1e-5
        assert rel(got_m, m64.numpy()) < 1e-5
    # a = 1: the third-order displacement alone
    q64, _ = ics.lpt_ics(c, n, L, 1.0, n_order=2, white=w)
    q32, _ = ics.lpt_ics_native(c, n, L, 1.0, n_order=2, white=w.float())
    d_ref = (p64 - q64).numpy()
    d_got = got_p - djb.logical_view(q32).cpu().numpy()
    assert np.abs(d_ref).max() > 1e-3 * np.abs(p64.numpy()).max()   # a real third-order term
    assert rel(d_got, d_ref) < 1e-3


@pytest.mark.parametrize("W,g,aa", [(4, 6, 1), (3, 4, 2), (2, 2, 3), (4, 4, -1)])
def test_sorted_partial_sums_change_no_bit(djb, monkeypatch, W, g, aa):
    """The brick interpolation keeps its sums across the interlacing shifts (and the
    call's Ψ) in sorted order instead of going through the acceleration array in
    particle order (DJB_GATHER_PART=0): the same additions in the same order, so the
    force and three steps give identical bits, for one launch of two shifts (aa = 1),
    several launches (aa = 2, 3) and a single shift (aa = -1)."""
    rng = np.random.default_rng(11 + W + aa)
    n, res, L = 32, 64, 100.0
    psi = np.asfortranarray((2.0 * rng.standard_normal((n, n, n, 3))).astype(np.float32))
    mom = np.asfortranarray(rng.standard_normal((n, n, n, 3)).astype(np.float32))
    out = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("DJB_GATHER_PART", mode)
        cfg = djb.PMConfig(res_pm=res, n_part=n, boxsize=L, worder=W, grad_order=g, antialias=aa)
        with djb.PMSolver(cfg) as S:
            acc = S.acceleration(psi)
            S.set_state(psi, mom)
            for _ in range(3):
                S.step(0.05, 0.9, 0.4, 0.05)
            out[mode] = (acc, *S.output(wrap=False))
    for a, b in zip(out["0"], out["1"]):
        assert np.array_equal(a, b)
