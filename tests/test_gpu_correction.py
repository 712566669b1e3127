"""The NN-corrected PM force on the B200, through the C ABI.

* The interpolation of three mesh fields to the particles (`djb_mesh_interp3`) against
  the float64 oracle's gather (pm.jl:344-364), and its transpose (`djb_mesh_deposit3`)
  by the adjoint identity <deposit(v), m> = <v, interp(m)>.
* `djb_nn_backward_output_grad` with dout = 2(out − target)/count gives the gradients
  of the network's own MSE backward.
* An attached network adds out_scale·interp(net(scaled [δ, F])) to the force, equal to
  the same chain assembled from the separate entry points.
* Training on (2× − 1×) force residuals of this PM code lowers the residual, and the
  corrected 1× run's P(k) at a = 1 is closer to the 2× run's than the plain 1× run's
  for k < k_Nyq/2 (what the trained network gains over the method without it).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def djb(cuda_device):
    import djb200
    return djb200


@pytest.fixture(scope="module")
def cosmo(djb):
    from djb200 import correction
    return djb.Cosmology(**correction.COSMO)


def _clustered(n, L, seed, amp=3.0):
    import torch
    rng = np.random.default_rng(seed)
    psi = (amp * rng.standard_normal((n, n, n, 3))).astype(np.float32)
    return psi, torch.from_numpy(np.ascontiguousarray(psi.transpose(3, 2, 1, 0))).cuda()


@pytest.mark.parametrize("W", [2, 3, 4])
def test_interp3_vs_oracle_and_deposit3_is_its_transpose(djb, W):
    import torch

    from oracle import nbody as onb
    from oracle import pm as opm
    n, res, L = 24, 48, 120.0
    psi, psi_d = _clustered(n, L, 5 + W)
    gen = torch.Generator(device="cuda").manual_seed(W)
    m = torch.randn((3, res, res, res), generator=gen, device="cuda")
    v = torch.randn((3, n, n, n), generator=gen, device="cuda")
    with djb.PMSolver(djb.PMConfig(res_pm=res, n_part=n, boxsize=L, worder=W, grad_order=2)) as S:
        out = S.mesh_interp3(psi_d, m)
        dep = S.mesh_deposit3(psi_d, v)
    X = onb.add_q(psi.astype(np.float64), L).reshape(-1, 3)
    mh = m.double().cpu().numpy()
    for c in range(3):
        ref = opm.pm_gather(mh[c].transpose(2, 1, 0), X, res, L, W).reshape(n, n, n)   # [i,j,k]
        got = out[c].double().cpu().numpy().transpose(2, 1, 0)
        assert rel(got, ref) < 1e-5
    lhs = float((dep.double() * m.double()).sum())
    rhs = float((v.double() * out.double()).sum())
    assert abs(lhs - rhs) < 1e-5 * abs(rhs) + 1e-6


def test_backward_output_grad_matches_mse_backward(djb):
    import torch

    from djb200.nn import ForceNet
    r = 20
    gen = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn((4, r, r, r), generator=gen, device="cuda")
    t = torch.randn((3, r, r, r), generator=gen, device="cuda")
    with ForceNet(seed=4) as net:
        net.backward(x, t)
        g_mse = net.grads()
        out = net.apply(x)
        net.backward_output_grad(x, (2.0 / out.numel()) * (out - t))
        g_out = net.grads()
    assert rel(g_out, g_mse) < 1e-6


def test_attached_network_adds_its_interpolated_correction(djb, cosmo):
    import torch

    from djb200 import correction
    from djb200.nn import ForceNet
    n, L = 32, 62.5
    p0, _ = correction.initial_state(cosmo, n, L, seed=3)
    psi = (p0 * float(cosmo.Dplus(1.0) / cosmo.Dplus(correction.A_INI))).contiguous()
    scales = (0.3, 2.0, 0.05)
    cfg = djb.PMConfig(res_pm=n, n_part=n, boxsize=L, **correction.OPTS)
    with ForceNet(seed=7) as net, djb.PMSolver(cfg) as S:
        plain = S.acceleration(psi)
        x = S.mesh_fields(psi)
        xs = x.clone()
        xs[0] *= scales[0]
        xs[1:] *= scales[1]
        manual = S.mesh_interp3(psi, net.apply(xs)) * scales[2]
        S.attach_nn(net, *scales)
        corrected = S.acceleration(psi)
        S.attach_nn(None)
        again = S.acceleration(psi)
    d = (corrected - plain).double()
    md = manual.double()
    assert float(md.abs().max()) > 0
    # the pipeline's δ comes from the brick deposit (fixed point), mesh_fields' from float
    # atomics: bf16 rounding of the network's input can flip in rare voxels
    assert float(torch.linalg.norm(d - md) / torch.linalg.norm(md)) < 2e-3
    assert rel(again.cpu().numpy(), plain.cpu().numpy()) < 1e-6      # detached: plain force again


def test_network_schedule(djb, cosmo):
    """djb_solver_nn_schedule: before `start` the steps are uncorrected (the plain run, up
    to the reordering of float reductions), from it on every step is corrected; with
    every = 2 the steps in between reuse the particles' last correction (and differ from
    both)."""
    import torch

    from djb200 import correction, stepper_coefficients
    from djb200.nn import ForceNet
    n, L, steps = 32, 62.5, 4
    p0, m0 = correction.initial_state(cosmo, n, L, seed=5)
    co = stepper_coefficients(cosmo, "bullfrog", correction.A_INI, 1.0, steps)
    cfg = djb.PMConfig(res_pm=n, n_part=n, boxsize=L, **correction.OPTS_LO)

    def run(net, every=1, start=0):
        with djb.PMSolver(cfg) as S:
            if net is not None:
                S.attach_nn(net, 0.3, 2.0, 0.05)
                S.nn_schedule(every, start)
            S.set_state(p0, m0)
            for k in range(steps):
                S.step(co["ddrift1"][k], co["alpha"][k], co["beta"][k], co["ddrift2"][k])
            p, _ = S.get_state(device=True)
        return p.cpu().numpy()

    with ForceNet(seed=11) as net:
        plain = run(None)
        late = run(net, 1, steps)         # never active within the run
        full = run(net, 1, 0)
        half = run(net, 2, 0)
        tail = run(net, 1, 2)
    # two runs of the same force agree to float-reduction reordering only
    noise = max(rel(late, plain), 1e-7)
    assert noise < 1e-5
    assert rel(full, plain) > 100 * noise
    for x in (half, tail):
        assert rel(x, plain) > 10 * noise and rel(x, full) > 10 * noise


@pytest.mark.slow
def test_training_gains_over_plain_pm(djb, cosmo, capsys):
    """64³ particles, L = 125 (the resolution of the 128³ / L = 250 training set):
    6 seeds × 20 states, 3 epochs; held-out states and seeds."""
    from djb200 import correction
    n, L = 64, 125.0
    T = correction.train(cosmo, n=n, boxsize=L, seeds=range(6), snapshots=20, epochs=3, lr=2e-3, lr_end=2e-4,
                         log=lambda *a: None)
    p0, m0 = correction.initial_state(cosmo, n, L, seed=500)
    _, _, held, _ = correction.run(cosmo, p0, m0, res=2 * n, boxsize=L, n_steps=20, keep_states=True)
    before = [T.loss(s)[1] for s in held[-5:]]
    after = [T.loss(s)[0] for s in held[-5:]]
    ev = correction.evaluate(cosmo, T.net, T.scales, n=n, boxsize=L, seeds=[501, 502])
    T.close()
    with capsys.disabled():
        print(f"\n[correction 64^3] held-out relative residual {np.mean(after):.3f} (plain 1.0); "
              f"P(k) max error k<kNyq/2: plain {ev['pk_max_err_plain']:.4f}, corrected {ev['pk_max_err_corrected']:.4f}")
    assert np.mean(after) < 0.8 * np.mean(before)
    assert ev["pk_max_err_corrected"] < ev["pk_max_err_plain"]
