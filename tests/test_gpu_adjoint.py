"""GPU adjoints (no reference counterpart): the force VJP, the step VJP and the P(k)
VJP through the C ABI against the float64 restatements of oracle/adjoint.py (which
test_adjoint_oracle.py pins with finite differences), and the gradient of a P(k) loss
through a checkpointed run against central finite differences of the float64 oracle."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

COSMO = dict(Omega_c=0.31 - 0.049, Omega_b=0.049, h=0.677, n_s=0.965, sigma8=0.81)
VJP_TOL = 2e-4  # float32 kernels against float64 sums of the same terms


@pytest.fixture(scope="module")
def djb(cuda_device):
    import djb200
    return djb200


def _clustered(n, L, seed, amp=3.0):
    return (amp * np.random.default_rng(seed).standard_normal((n, n, n, 3))).astype(np.float32)


@pytest.mark.parametrize("W,g,aa,lap,dec", [(2, 2, 0, 0, False), (3, 4, 1, 4, False), (4, 6, 1, 0, True),
                                            (4, 4, -1, 2, False), (3, 6, 2, 0, True)])
def test_force_vjp_vs_oracle(djb, W, g, aa, lap, dec):
    from oracle import adjoint as oad
    from oracle import pm as opm
    n, res, L = 16, 32, 100.0
    psi = _clustered(n, L, 3 + W)
    abar = np.random.default_rng(9 + g).standard_normal((n, n, n, 3)).astype(np.float32)
    cfg = djb.PMConfig(res_pm=res, n_part=n, boxsize=L, worder=W, grad_order=g, antialias=aa, lap_order=lap,
                       deconvolve=dec)
    with djb.PMSolver(cfg) as S:
        gb = S.acceleration_vjp(psi, abar)
    ocfg = opm.PMConfig(res_pm=res, n_part=n, boxsize=L, worder=W, grad_order=g, antialias=aa, lap_order=lap,
                        deconvolve=dec)
    ref = oad.pm_acceleration_vjp(ocfg, psi.astype(np.float64), abar.astype(np.float64))
    assert rel(gb, ref) < VJP_TOL


def test_force_vjp_device_arrays_and_ik_rejected(djb):
    import torch
    n, res, L = 16, 32, 100.0
    psi = _clustered(n, L, 4)
    abar = np.random.default_rng(2).standard_normal((n, n, n, 3)).astype(np.float32)
    cfg = djb.PMConfig(res_pm=res, n_part=n, boxsize=L, worder=4, grad_order=4, antialias=1)
    with djb.PMSolver(cfg) as S:
        host = S.acceleration_vjp(psi, abar)
        dev = S.acceleration_vjp(djb.native_view(torch.from_numpy(psi).cuda()),
                                 djb.native_view(torch.from_numpy(abar).cuda()))
    assert rel(djb.logical_view(dev).cpu().numpy(), host) < 1e-5  # float atomics reorder only
    with djb.PMSolver(djb.PMConfig(res_pm=res, n_part=n, boxsize=L, grad_order=0)) as S:
        with pytest.raises(djb.DJBInvalidOption):
            S.acceleration_vjp(psi, abar)


def test_stencils_16_byte_staging_at_1024_mesh(djb, monkeypatch):
    """On the dense 1024³ meshes the FD stencil kernels (network inputs, VJP) stage
    their planes with 16-byte copies; the 4-byte path (DJB_FD_SCALAR=1, the one the
    padded meshes of the oracle comparisons take) must give the same fields."""
    n, res, L = 32, 1024, 1000.0
    psi = _clustered(n, L, 5, amp=8.0)
    abar = np.random.default_rng(4).standard_normal((n, n, n, 3)).astype(np.float32)
    cfg = djb.PMConfig(res_pm=res, n_part=n, boxsize=L, worder=4, grad_order=6, antialias=1)
    out = {}
    for scalar in ("0", "1"):
        monkeypatch.setenv("DJB_FD_SCALAR", scalar)
        with djb.PMSolver(cfg) as S:
            f = S.mesh_fields(psi)
            out[scalar] = (f[1:].copy(), S.acceleration_vjp(psi, abar))
        del f
    (f16, g16), (f4, g4) = out["0"], out["1"]
    assert np.isfinite(f16).all() and np.abs(f16).max() > 0
    assert rel(f16, f4) < 1e-5        # float atomics of the deposit reorder only
    assert rel(g16, g4) < 1e-5


def test_vjp_bulk_tensor_boxes_at_1024_mesh(djb, monkeypatch):
    """On the dense 1024³ meshes the adjoint's brick kernels stage and flush their boxes
    with bulk tensor copies; with those off (DJB_TMA=0: asynchronous copies and vector
    reductions, the form the oracle comparisons at small sizes take) the step VJP must
    agree."""
    n, res, L = 32, 1024, 1000.0
    psi = _clustered(n, L, 6, amp=8.0)
    mom = np.random.default_rng(5).standard_normal((n, n, n, 3)).astype(np.float32)
    pb = np.random.default_rng(6).standard_normal((n, n, n, 3)).astype(np.float32)
    mb = np.random.default_rng(7).standard_normal((n, n, n, 3)).astype(np.float32)
    cfg = djb.PMConfig(res_pm=res, n_part=n, boxsize=L, worder=4, grad_order=6, antialias=1)
    out = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("DJB_TMA", flag)
        with djb.PMSolver(cfg) as S:
            out[flag] = S.step_vjp(0.01, 0.9, 0.05, 0.01, psi, mom, pb, mb)
    for a, b in zip(out["1"], out["0"]):
        assert np.isfinite(a).all()
        assert rel(a, b) < 1e-5   # float atomics and reductions reorder only


def test_step_vjp_vs_oracle(djb):
    from oracle import adjoint as oad
    from oracle import pm as opm
    n, res, L = 16, 32, 100.0
    rng = np.random.default_rng(21)
    psi0 = _clustered(n, L, 6)
    mom0 = rng.standard_normal((n, n, n, 3)).astype(np.float32)
    pbar = rng.standard_normal((n, n, n, 3)).astype(np.float32)
    mbar = rng.standard_normal((n, n, n, 3)).astype(np.float32)
    dd1, alpha, beta, dd2 = 0.3, 0.9, 0.7, 0.25
    cfg = djb.PMConfig(res_pm=res, n_part=n, boxsize=L, worder=4, grad_order=6, antialias=1)
    with djb.PMSolver(cfg) as S:
        gp, gm = S.step_vjp(dd1, alpha, beta, dd2, psi0, mom0, pbar, mbar)
    ocfg = opm.PMConfig(res_pm=res, n_part=n, boxsize=L, worder=4, grad_order=6, antialias=1)
    p1 = psi0.astype(np.float64) + np.float32(dd1) * mom0.astype(np.float64)
    mb = mbar.astype(np.float64) + dd2 * pbar.astype(np.float64)
    pb = pbar.astype(np.float64) + oad.pm_acceleration_vjp(ocfg, p1, beta * mb)
    mb0 = alpha * mb + dd1 * pb
    assert rel(gp, pb) < VJP_TOL
    assert rel(gm, mb0) < VJP_TOL


def test_power_spectrum_vjp_vs_oracle(djb):
    from oracle import adjoint as oad
    n, res, L, bins = 16, 32, 100.0, 12
    psi = _clustered(n, L, 8)
    mom = np.zeros_like(psi)
    pk_bar = np.random.default_rng(4).standard_normal(bins)
    with djb.PMSolver(djb.PMConfig(res_pm=res, n_part=n, boxsize=L)) as S:
        S.set_state(psi, mom)
        gb = S.state_power_spectrum_vjp(pk_bar, bins=bins)
    ref = oad.power_spectrum_vjp(res, n, L, psi.astype(np.float64), pk_bar, bins=bins)
    assert rel(gb, ref) < VJP_TOL


def test_pk_loss_gradient_through_a_run_vs_finite_differences(djb):
    """Adjoint stepper with checkpoints every 5 steps (BullFrog, 7 steps: two segments)
    against central differences of the same loss through the float64 oracle run."""
    from oracle import cosmology as cz
    from oracle import nbody as onb
    from oracle import pm as opm
    from oracle import power as opw
    from djb200 import adjoint as dad
    from djb200 import ics
    n, res, L, bins, steps = 16, 32, 200.0, 10, 7
    cl = djb.Cosmology(**COSMO)
    co = cz.compute_timetables(cz.Cosmology(**COSMO))
    psi, pi = ics.lpt_ics(cl, n, L, 0.05, n_order=2, seed=13, device="cpu")
    psi, pi = psi.numpy().astype(np.float64), pi.numpy().astype(np.float64)
    kw = dict(boxsize=L, a_ini=0.05, a_end=1.0, n_steps=steps, res_pm=res, stepper="bullfrog", worder=4,
              grad_kernel_order=4, antialias=1)

    def pk_of(P):
        mesh = opm.pm_scatter(np.zeros((res, res, res)), onb.add_q(P, L).reshape(-1, 3), res, L, 2)
        return opw.evaluate_power_spectrum(opw.density_contrast(mesh, n), L, bins=bins)[1]

    P_end, _, _ = onb.run_nbody(co, psi, pi, return_displacement=True, **kw)
    target = pk_of(P_end) * 0.8

    def loss(p, m):
        P, _, _ = onb.run_nbody(co, p, m, return_displacement=True, **kw)
        pk = pk_of(P)
        ok = (pk > 0) & (target > 0)
        return float(np.sum((np.log(pk[ok]) - np.log(target[ok])) ** 2))

    lg, gpsi, gpi = dad.pk_loss_and_gradient(cl, psi.astype(np.float32), pi.astype(np.float32), target,
                                             bins=bins, checkpoint_every=5, grad_kernel_order=4, **{
                                                 k: v for k, v in kw.items() if k != "grad_kernel_order"})
    assert abs(lg - loss(psi, pi)) < 1e-3 * abs(lg)
    rng = np.random.default_rng(3)
    for grad, which in ((gpsi, 0), (gpi, 1)):
        v = rng.standard_normal(psi.shape)
        eps = 1e-4 if which == 0 else 1e-4
        if which == 0:
            fd = (loss(psi + eps * v, pi) - loss(psi - eps * v, pi)) / (2 * eps)
        else:
            fd = (loss(psi, pi + eps * v) - loss(psi, pi - eps * v)) / (2 * eps)
        an = float(np.sum(grad.astype(np.float64) * v))
        assert abs(an - fd) < 2e-2 * abs(fd), (which, an, fd)


def _mode(n, m, phase, device):
    """A real Fourier mode of unit variance per voxel: √2 cos(2π m·x/n + phase)."""
    import torch
    i = torch.arange(n, device=device, dtype=torch.float64)
    arg = (2 * np.pi / n) * (m[0] * i[:, None, None] + m[1] * i[None, :, None] + m[2] * i[None, None, :]) + phase
    return (np.sqrt(2.0) * torch.cos(arg)).float()


def _white_noise_fd_check(djb, n, res, L, n_modes, capsys, label, eps=1e-3, seed=21, worder=2):
    """∂loss/∂(white noise) through 2LPT ICs and a checkpointed BullFrog run (CIC, grad 2,
    20 steps, checkpoints every 5), float32 on the GPU, against central differences
    (ε = 1e-3) of the same loss through the float64 oracle (2LPT ICs in float64, the
    float64 C port's steps, CIC P(k) with float64 shells), along random low-k Fourier
    modes of the white noise (|m| < n/8, random phases). The float64 differences are
    free of the float32 round-off that a 1e-3 step would otherwise amplify."""
    import torch

    from djb200 import adjoint as dad
    from djb200 import ics
    from oracle import cosmology as cz
    from oracle import cpm
    from oracle import nbody as onb
    from oracle import pm as opm
    from oracle import power as opw
    cl = djb.Cosmology(**COSMO)
    co = cz.compute_timetables(cz.Cosmology(**COSMO))
    steps, bins = 20, 32
    kw = dict(boxsize=L, a_ini=0.02, a_end=1.0, n_steps=steps, res_pm=res, stepper="bullfrog", worder=worder,
              grad_kernel_order=2, antialias=0, checkpoint_every=5, bins=bins)
    w = ics.white_noise(seed, n, device="cuda", dtype=torch.float32)
    _, pk0 = dad.white_noise_loss(cl, w, np.ones(bins), **dict(kw))
    target = 0.9 * pk0
    loss, gw = dad.white_noise_loss_and_gradient(cl, w, target, **dict(kw))
    coef = onb.stepper_coefficients(co, "bullfrog", 0.02, 1.0, steps)
    port = cpm.CPUPM(opm.PMConfig(res_pm=res, n_part=n, boxsize=L, worder=worder, grad_order=2), dtype=np.float64)
    w64 = w.double().cpu()

    def loss64(white):
        psi, pi = ics.lpt_ics(cl, n, L, 0.02, n_order=2, device="cpu", dtype=torch.float64, white=white)
        p, m = psi.numpy(), pi.numpy()
        for k in range(steps):
            p, m = port.step(p, m, coef["ddrift1"][k], coef["alpha"][k], coef["beta"][k], coef["ddrift2"][k])
        Xb = np.ascontiguousarray(np.moveaxis(onb.add_q(p, L), -1, 0).transpose(0, 3, 2, 1))
        mesh = np.zeros(res ** 3)
        cpm.lib().cpm_scatter_f64(cpm._ptr(Xb), n ** 3, res, float(L), 2, cpm._ptr(mesh))
        pk = opw.evaluate_power_spectrum(opw.density_contrast(mesh.reshape(res, res, res).T, n), L, bins=bins)[1]
        ok = (pk > 0) & (target > 0)
        return float(np.sum((np.log(pk[ok]) - np.log(target[ok])) ** 2))

    rng = np.random.default_rng(seed)
    an, fd = [], []
    for _ in range(n_modes):
        while True:
            m = rng.integers(-(n // 8) + 1, n // 8, size=3)
            if 0 < np.sum(m * m) < (n // 8) ** 2:
                break
        v = _mode(n, m, rng.uniform(0, 2 * np.pi), "cuda")
        an.append(float((gw.double() * v.double()).sum()))
        v64 = v.double().cpu()
        fd.append((loss64(w64 + eps * v64) - loss64(w64 - eps * v64)) / (2 * eps))
    an, fd = np.array(an), np.array(fd)
    err = np.abs(an - fd) / np.maximum(np.abs(fd), 1e-2 * np.max(np.abs(fd)))
    with capsys.disabled():
        print(f"\n[{label}] loss {loss:.4e}; {n_modes} modes: median rel err {np.median(err):.2e}, "
              f"max {np.max(err):.2e}, corr {np.corrcoef(an, fd)[0, 1]:.6f}")
    return an, fd, err


def test_white_noise_gradient_small_vs_finite_differences(djb, capsys):
    """32³/64³. The CIC weights are piecewise linear, so the loss has kinks wherever a
    particle crosses a cell face: a difference over ±ε averages the derivative's jumps
    of every crossing the step causes. The difference converges to the adjoint as ε
    shrinks (measured: median relative error 7.2e-2 at ε = 1e-3, 1.8e-2 at 1e-4, 2.3e-3
    at 1e-5); the check uses ε = 1e-5 (float64 differences) and reports ε = 1e-3."""
    an, fd, err = _white_noise_fd_check(djb, 32, 64, 62.5, 8, capsys, "white-noise gradient 32^3/64^3, eps 1e-5",
                                        eps=1e-5)
    assert np.median(err) < 1e-2
    assert np.corrcoef(an, fd)[0, 1] > 0.9999
    an3, fd3, _ = _white_noise_fd_check(djb, 32, 64, 62.5, 8, capsys, "white-noise gradient 32^3/64^3, eps 1e-3")
    assert np.corrcoef(an3, fd3)[0, 1] > 0.99


@pytest.mark.slow
def test_white_noise_gradient_c5_vs_finite_differences(djb, capsys):
    """The differentiable-run configuration: 128³ particles on a 256³ mesh, L = 250, at
    ε = 1e-5 (see above; at the configuration's ε = 1e-3 the CIC kinks leave a median
    relative error of 1.2e-1, correlation 0.82, over 16 modes). The float64 differences
    take ~10 s per run on 16 cores, so the default checks 8 modes; DJB_C5_MODES=64 and
    DJB_C5_EPS choose the configuration's full set and step."""
    import os
    modes = int(os.environ.get("DJB_C5_MODES", "8"))
    eps = float(os.environ.get("DJB_C5_EPS", "1e-5"))
    an, fd, err = _white_noise_fd_check(djb, 128, 256, 250.0, modes, capsys,
                                        f"white-noise gradient C5 128^3/256^3, eps {eps:g}", eps=eps)
    assert np.median(err) < 3e-2
    assert np.corrcoef(an, fd)[0, 1] > 0.9999
