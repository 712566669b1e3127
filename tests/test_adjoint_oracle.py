"""The float64 adjoint restatements (oracle/adjoint.py) against central finite differences
of the float64 forward restatements. The reference has no adjoint, so finite differences
are what pins it; the GPU VJPs are compared with these in test_gpu_adjoint.py."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import adjoint as oad
from oracle import pm as opm
from oracle import power as opw


def _psi(n, L, seed, amp=3.0):
    rng = np.random.default_rng(seed)
    return amp * rng.standard_normal((n, n, n, 3))


@pytest.mark.parametrize("W,g,aa", [(2, 2, 0), (3, 4, 1), (4, 6, 1), (4, 4, 2)])
def test_fd_force_equals_fourier_force(W, g, aa):
    """The real-space FD gradient equals the Fourier gradient kernel (pm.jl:309-311)."""
    cfg = opm.PMConfig(res_pm=16, n_part=8, boxsize=40.0, worder=W, grad_order=g, antialias=aa)
    psi = _psi(8, 40.0, 1)
    a = oad.pm_acceleration_fd(cfg, psi)
    b = opm.pm_acceleration(cfg, psi)
    assert np.max(np.abs(a - b)) < 1e-11 * np.max(np.abs(b))


@pytest.mark.parametrize("W,g,aa,lap,dec", [(2, 2, 0, 0, False), (3, 4, 1, 4, False), (4, 6, 1, 0, True),
                                            (4, 4, -1, 2, False), (3, 6, 2, 0, True)])
def test_force_vjp_matches_finite_differences(W, g, aa, lap, dec):
    n, res, L = 8, 16, 40.0
    cfg = opm.PMConfig(res_pm=res, n_part=n, boxsize=L, worder=W, grad_order=g, antialias=aa,
                       lap_order=lap, deconvolve=dec)
    rng = np.random.default_rng(11 + W + g)
    psi = _psi(n, L, 2 + W)
    abar = rng.standard_normal((n, n, n, 3))
    v = rng.standard_normal((n, n, n, 3))
    gbar = oad.pm_acceleration_vjp(cfg, psi, abar)
    eps = 1e-5
    lp = np.sum(abar * oad.pm_acceleration_fd(cfg, psi + eps * v))
    lm = np.sum(abar * oad.pm_acceleration_fd(cfg, psi - eps * v))
    fd = (lp - lm) / (2 * eps)
    an = np.sum(gbar * v)
    assert abs(an - fd) < 1e-6 * max(abs(fd), 1e-12) + 1e-9


def test_power_spectrum_vjp_matches_finite_differences():
    n, res, L, bins = 8, 16, 40.0, 8
    rng = np.random.default_rng(5)
    psi = _psi(n, L, 9)
    pbar = rng.standard_normal(bins)
    v = rng.standard_normal((n, n, n, 3))

    def loss(p):
        from oracle import nbody as onb
        X = onb.add_q(p, L).reshape(-1, 3)
        mesh = opm.pm_scatter(np.zeros((res, res, res)), X, res, L, 2)
        _, pk, _ = opw.evaluate_power_spectrum(opw.density_contrast(mesh, n), L, bins=bins)
        return np.sum(pbar * pk)

    gbar = oad.power_spectrum_vjp(res, n, L, psi, pbar, bins=bins)
    eps = 1e-5
    fd = (loss(psi + eps * v) - loss(psi - eps * v)) / (2 * eps)
    an = np.sum(gbar * v)
    assert abs(an - fd) < 1e-6 * abs(fd)
