"""Gradient of a P(k) loss through a whole PM run, with checkpoints.

No counterpart in the reference, which has no adjoint. The forward run is
`run_nbody` (run_nbody.jl:124-172) on the B200 solver; the loss is

    loss = Σ_b (ln P_b − ln P_target,b)²

over the bins where both are positive, with P the power spectrum of the final state
(CIC deposit on the PM mesh, as `PMSolver.state_power_spectrum`). The backward pass
runs the step adjoints (`djb_step_vjp`) in reverse. The state is saved every
`checkpoint_every` steps on the forward pass; each segment between checkpoints is run
forward again once, keeping its states on the device, before its steps are taken
back. Memory: (n_steps/checkpoint_every + checkpoint_every) states of 24·N_p bytes.
"""
from __future__ import annotations

import numpy as np

from .cosmology import Cosmology, stepper_coefficients
from .pm import PMConfig, PMSolver, logical_view, native_view


def _pk_loss(pk, pk_target):
    pt = np.asarray(pk_target, dtype=np.float64)
    ok = (pk > 0) & (pt > 0)
    r = np.where(ok, np.log(np.where(ok, pk, 1.0)) - np.log(np.where(ok, pt, 1.0)), 0.0)
    return float(np.sum(r * r)), np.where(ok, 2.0 * r / np.where(ok, pk, 1.0), 0.0)


def _config(n, boxsize, res_pm, worder, deconvolve, antialias, grad_kernel_order, laplace_kernel_order):
    return PMConfig(res_pm=res_pm, n_part=n, boxsize=float(boxsize), worder=worder, deconvolve=deconvolve,
                    antialias=antialias, grad_order=grad_kernel_order, lap_order=laplace_kernel_order)


def pk_loss_and_gradient_device(c: Cosmology, psi0, pi0, pk_target, *, boxsize, a_ini, a_end, n_steps, res_pm,
                                stepper="bullfrog", bins=32, logarithmic=True, checkpoint_every=5, antialias=0,
                                grad_kernel_order=4, laplace_kernel_order=0, worder=2, deconvolve=False, device=0):
    """-> (loss, ∂loss/∂psi0, ∂loss/∂pi0) for native (3,n,n,n) float32 device tensors
    psi0, pi0 (the gradients in the same layout, on the device)."""
    import torch
    n = int(psi0.shape[1])
    co = stepper_coefficients(c, stepper, a_ini, a_end, n_steps)
    cfg = _config(n, boxsize, res_pm, worder, deconvolve, antialias, grad_kernel_order, laplace_kernel_order)
    mom_scale = c.Fplus(a_ini) if stepper == "symplectic" else 1.0
    coef = [(co["ddrift1"][k], co["alpha"][k], co["beta"][k], co["ddrift2"][k]) for k in range(n_steps)]
    with PMSolver(cfg, device=device) as S:
        S.set_state(psi0, pi0, mom_scale=mom_scale)
        ckpt = {0: S.get_state(device=True)}
        for k in range(n_steps):
            S.step(*coef[k])
            if (k + 1) % checkpoint_every == 0 and k + 1 < n_steps:
                ckpt[k + 1] = S.get_state(device=True)
        _, pk, _ = S.state_power_spectrum(bins=bins, logarithmic=logarithmic)
        loss, pk_bar = _pk_loss(pk, pk_target)
        psi_bar = S.state_power_spectrum_vjp(pk_bar, bins=bins, logarithmic=logarithmic, device=True)
        mom_bar = torch.zeros_like(psi_bar)
        starts = sorted(ckpt)
        for si in range(len(starts) - 1, -1, -1):
            c0 = starts[si]
            c1 = starts[si + 1] if si + 1 < len(starts) else n_steps
            S.set_state(*ckpt[c0])
            states = [ckpt[c0]]
            for k in range(c0, c1 - 1):
                S.step(*coef[k])
                states.append(S.get_state(device=True))
            for k in range(c1 - 1, c0 - 1, -1):
                p_k, m_k = states[k - c0]
                psi_bar, mom_bar = S.step_vjp(*coef[k], p_k, m_k, psi_bar, mom_bar)
    return loss, psi_bar, mom_bar * float(mom_scale)


def pk_loss_and_gradient(c: Cosmology, psi_ini, pi_ini, pk_target, *, device=0, **kw):
    """-> (loss, ∂loss/∂psi_ini, ∂loss/∂pi_ini), the gradients as host (n,n,n,3) float32.

    psi_ini, pi_ini: (n,n,n,3) initial displacements and momenta as `run_nbody` takes
    them; pk_target: (bins,) target spectrum. Keywords as `pk_loss_and_gradient_device`."""
    import torch
    dev = f"cuda:{device}"
    psi0 = native_view(torch.as_tensor(np.asarray(psi_ini, dtype=np.float32), device=dev))
    pi0 = native_view(torch.as_tensor(np.asarray(pi_ini, dtype=np.float32), device=dev))
    loss, gp, gm = pk_loss_and_gradient_device(c, psi0, pi0, pk_target, device=device, **kw)
    gpsi = logical_view(gp).cpu().numpy()
    gpi = logical_view(gm).cpu().numpy()
    return loss, np.ascontiguousarray(gpsi), np.ascontiguousarray(gpi)


def white_noise_loss(c: Cosmology, white, pk_target, *, boxsize, a_ini, n_order=2, device=0, **kw):
    """The P(k) loss of the run from the LPT initial conditions of the white-noise field
    `white` ((n,n,n) float32 device tensor, [i,j,k]); keywords as
    `pk_loss_and_gradient_device`. Forward only."""
    from . import ics
    n = int(white.shape[0])
    psi, pi = ics.lpt_ics(c, n, float(boxsize), a_ini, n_order=n_order, device=white.device, dtype=white.dtype,
                          white=white)
    bins = kw.pop("bins", 32)
    logarithmic = kw.pop("logarithmic", True)
    co = stepper_coefficients(c, kw.pop("stepper", "bullfrog"), a_ini, kw.pop("a_end"), kw.pop("n_steps"))
    kw.pop("checkpoint_every", None)
    cfg = _config(n, boxsize, kw.pop("res_pm"), kw.pop("worder", 2), kw.pop("deconvolve", False),
                  kw.pop("antialias", 0), kw.pop("grad_kernel_order", 4), kw.pop("laplace_kernel_order", 0))
    with PMSolver(cfg, device=device) as S:
        S.set_state(native_view(psi.float().detach()), native_view(pi.float().detach()))
        S.run(co["ddrift1"], co["alpha"], co["beta"], co["ddrift2"])
        _, pk, _ = S.state_power_spectrum(bins=bins, logarithmic=logarithmic)
    return _pk_loss(pk, pk_target)[0], pk


def white_noise_loss_and_gradient(c: Cosmology, white, pk_target, *, boxsize, a_ini, n_order=2, device=0, **kw):
    """-> (loss, ∂loss/∂white) through the whole chain white noise → φ(k)
    (`white_noise_to_fphi`, src/ics/grf.jl:139-140) → nLPT shapes (`compute_core`,
    src/lpt/nlpt_core.jl:311) → (Ψ, Π) at a_ini → the checkpointed PM run → P(k) loss.

    The run's adjoint is the library's (djb_step_vjp, djb_state_power_spectrum_vjp); the
    initial-condition map is the torch FFT restatement in `ics`, differentiated by torch's
    autograd (its FFT transposes are the rrules of nlpt_core.jl:689-713). `white`:
    (n,n,n) float32 device tensor [i,j,k]; the gradient has the same shape."""
    import torch

    from . import ics
    n = int(white.shape[0])
    w = white.detach().clone().requires_grad_(True)
    with torch.enable_grad():
        psi, pi = ics.lpt_ics(c, n, float(boxsize), a_ini, n_order=n_order, device=w.device, dtype=w.dtype,
                              white=w)
        loss, gp, gm = pk_loss_and_gradient_device(c, native_view(psi.detach().float()),
                                                   native_view(pi.detach().float()), pk_target, boxsize=boxsize,
                                                   a_ini=a_ini, device=device, **kw)
        (gw,) = torch.autograd.grad((psi, pi), (w,), (logical_view(gp).to(psi.dtype),
                                                        logical_view(gm).to(pi.dtype)))
    return loss, gw.detach()
