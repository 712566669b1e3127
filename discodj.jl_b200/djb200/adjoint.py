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


def pk_loss_and_gradient(c: Cosmology, psi_ini, pi_ini, pk_target, *, boxsize, a_ini, a_end, n_steps, res_pm,
                         stepper="bullfrog", bins=32, logarithmic=True, checkpoint_every=5, antialias=0,
                         grad_kernel_order=4, laplace_kernel_order=0, worder=2, deconvolve=False, device=0):
    """-> (loss, ∂loss/∂psi_ini, ∂loss/∂pi_ini), the gradients as host (n,n,n,3) float32.

    psi_ini, pi_ini: (n,n,n,3) initial displacements and momenta as `run_nbody` takes
    them; pk_target: (bins,) target spectrum."""
    import torch
    n = int(np.shape(psi_ini)[0])
    co = stepper_coefficients(c, stepper, a_ini, a_end, n_steps)
    cfg = PMConfig(res_pm=res_pm, n_part=n, boxsize=float(boxsize), worder=worder, deconvolve=deconvolve,
                   antialias=antialias, grad_order=grad_kernel_order, lap_order=laplace_kernel_order)
    mom_scale = c.Fplus(a_ini) if stepper == "symplectic" else 1.0
    dev = f"cuda:{device}"
    coef = [(co["ddrift1"][k], co["alpha"][k], co["beta"][k], co["ddrift2"][k]) for k in range(n_steps)]
    with PMSolver(cfg, device=device) as S:
        psi0 = native_view(torch.as_tensor(np.asarray(psi_ini, dtype=np.float32), device=dev))
        pi0 = native_view(torch.as_tensor(np.asarray(pi_ini, dtype=np.float32), device=dev))
        S.set_state(psi0, pi0, mom_scale=mom_scale)
        ckpt = {0: S.get_state(device=True)}
        for k in range(n_steps):
            S.step(*coef[k])
            if (k + 1) % checkpoint_every == 0 and k + 1 < n_steps:
                ckpt[k + 1] = S.get_state(device=True)
        _, pk, _ = S.state_power_spectrum(bins=bins, logarithmic=logarithmic)
        pt = np.asarray(pk_target, dtype=np.float64)
        ok = (pk > 0) & (pt > 0)
        r = np.where(ok, np.log(np.where(ok, pk, 1.0)) - np.log(np.where(ok, pt, 1.0)), 0.0)
        loss = float(np.sum(r * r))
        pk_bar = np.where(ok, 2.0 * r / np.where(ok, pk, 1.0), 0.0)
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
        gpsi = logical_view(psi_bar).cpu().numpy()
        gpi = logical_view(mom_bar).cpu().numpy() * np.float32(mom_scale)
    return loss, np.ascontiguousarray(gpsi), np.ascontiguousarray(gpi)
