"""NN-corrected PM force: training, the corrected run and its evaluation (no counterpart
in the reference).

The force-correction network (`ForceNet`, 4 → 32 → 32 → 32 → 3, 3³ periodic
convolutions on the tensor cores) maps the PM fields of a res³ mesh, [δ, F_x, F_y, F_z]
as `djb_mesh_fields` computes them, to a correction field on the same mesh. Attached to
a solver (`PMSolver.attach_nn`), every force adds the correction interpolated to the
particles with the solver's own assignment kernel.

Training uses only pairs that this PM code generates:
* states: BullFrog runs (2LPT ICs of seeded white noise at a = 0.02, `n_steps` steps to
  a = 1) of n³ particles on the 2× mesh ((2n)³, the finer force), one state per step;
* target at each state: the particle accelerations of the 2× mesh minus those of the
  1× mesh (n³), both from this library's PM force at the same positions;
* loss: mean squared error of the interpolated correction against that residual,
  relative to the residual's mean square. Its gradient with respect to the network's
  output mesh is the transpose of the interpolation (`djb_mesh_deposit3`), which the
  network back-propagates (`djb_nn_backward_output_grad`); Adam on float32 weights.
The plain PM step stays the fallback (detach) and the yardstick: evaluation runs plain 1×,
corrected 1× and plain 2× from the same held-out ICs and compares their P(k) at a = 1
(CIC deposit on the 1× mesh, float64 shells) for k < k_Nyq/2 of the 1× mesh.

    python -m djb200.correction --out DIR [--seeds 64 --snapshots 20 --eval-seeds 8 ...]
"""
from __future__ import annotations

import json
import math
import time

import numpy as np

from . import ics
from .cosmology import Cosmology, stepper_coefficients
from .nn import ForceNet
from .pm import PMConfig, PMSolver, native_view

COSMO = dict(Omega_c=0.31 - 0.049, Omega_b=0.049, h=0.677, n_s=0.965, sigma8=0.81)
# the 2x mesh runs the throughput configuration's options; the 1x mesh a cheaper PM (TSC,
# no interlacing, order-4 gradient, the assignment window divided out), whose remaining
# error the network corrects
OPTS = dict(worder=4, antialias=1, grad_order=6)
OPTS_LO = dict(worder=3, antialias=0, grad_order=4, deconvolve=True)
A_INI = 0.02


def initial_state(cosmo, n: int, boxsize: float, seed: int, device: int = 0):
    """2LPT (Ψ, Π) at a = 0.02 of seeded white noise, native (3,n,n,n) float32 device tensors."""
    import torch
    psi, pi = ics.lpt_ics(cosmo, n, boxsize, A_INI, n_order=2, seed=seed, device=f"cuda:{device}",
                          dtype=torch.float32)
    return native_view(psi.float()), native_view(pi.float())


def run(cosmo, psi, pi, *, res: int, boxsize: float, n_steps: int, opts=OPTS, device: int = 0, net=None,
        scales=None, keep_states: bool = False, timing: bool = False, every: int = 1, start: int = 0):
    """BullFrog run from (psi, pi) on a res³ mesh, optionally with an attached network
    (from step `start` on, on every `every`-th step: `PMSolver.nn_schedule`). Returns
    (final Ψ, final Π, [Ψ after each step] or None, device ms per step or None); the timing
    covers every step but the first two (one-time work-area allocations), which a run with
    a schedule repeats untimed first, so that the time is the mean over the whole run."""
    import torch
    n = int(psi.shape[1])
    co = stepper_coefficients(cosmo, "bullfrog", A_INI, 1.0, n_steps)
    states = [] if keep_states else None
    with PMSolver(PMConfig(res_pm=res, n_part=n, boxsize=boxsize, **opts), device=device) as S:
        stream = torch.cuda.Stream(device=device)
        S.set_stream(stream.cuda_stream)
        if net is not None:
            net.set_stream(stream.cuda_stream)
            S.attach_nn(net, *scales)
            S.nn_schedule(every, start)
        scheduled = net is not None and (every > 1 or start > 0)
        if timing and scheduled:
            # an untimed pass of the whole schedule takes the one-time allocations; the
            # timed pass below then averages over every step of the run
            S.set_state(psi, pi)
            for k in range(n_steps):
                S.step(co["ddrift1"][k], co["alpha"][k], co["beta"][k], co["ddrift2"][k])
        S.set_state(psi, pi)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        # the first steps carry one-time work-area allocations
        warm = (0 if scheduled else 2) if timing else 0
        for k in range(n_steps):
            if k == warm:
                torch.cuda.synchronize(device)
                e0.record(stream)
            S.step(co["ddrift1"][k], co["alpha"][k], co["beta"][k], co["ddrift2"][k])
            if keep_states:
                p, _ = S.get_state(device=True)
                states.append(p)
        e1.record(stream)
        torch.cuda.synchronize(device)
        ms = e0.elapsed_time(e1) / (n_steps - warm) if timing and not keep_states else None
        p, m = S.get_state(device=True)
        if net is not None:
            S.attach_nn(None)
    return p, m, states, ms


def state_pk(psi, *, res: int, boxsize: float, bins: int = 32, device: int = 0):
    """(k, P(k), modes) of particles Ψ: CIC deposit on a res³ mesh, δ = mesh·res³/n³ − 1,
    float64 shell sums (`djb_state_power_spectrum`)."""
    n = int(psi.shape[1])
    with PMSolver(PMConfig(res_pm=res, n_part=n, boxsize=boxsize, worder=2, grad_order=2), device=device) as S:
        S.set_state(psi, psi)
        return S.state_power_spectrum(bins=bins)


class CorrectionTrainer:
    """Training of a ForceNet on (2× − 1×) PM force residuals of n³ particles."""

    def __init__(self, cosmo, *, n: int = 128, boxsize: float = 250.0, opts_lo=OPTS_LO, opts_hi=OPTS, device: int = 0,
                 seed: int = 0):
        self.cosmo, self.n, self.L, self.device = cosmo, n, boxsize, device
        self.opts_lo, self.opts_hi = dict(opts_lo), dict(opts_hi)
        self.lo = PMSolver(PMConfig(res_pm=n, n_part=n, boxsize=boxsize, **opts_lo), device=device)
        self.hi = PMSolver(PMConfig(res_pm=2 * n, n_part=n, boxsize=boxsize, **opts_hi), device=device)
        self.net = ForceNet(layers=4, cin=4, hidden=32, cout=3, seed=seed, device=device)
        self.scales = (1.0, 1.0, 1.0)

    def close(self):
        self.lo.close()
        self.hi.close()

    def pair(self, psi):
        """Network input [δ, F] on the 1× mesh and the residual a_2× − a_1× at the particles."""
        x = self.lo.mesh_fields(psi)
        r = self.hi.acceleration(psi) - self.lo.acceleration(psi)
        return x, r

    def fit_scales(self, states):
        """delta_scale, force_scale: the inverse r.m.s. of δ and of F over `states`;
        out_scale: the r.m.s. of the residual."""
        sd = sf = sr = 0.0
        for psi in states:
            x, r = self.pair(psi)
            sd += float((x[0].double() ** 2).mean())
            sf += float((x[1:].double() ** 2).mean())
            sr += float((r.double() ** 2).mean())
        k = len(states)
        self.scales = (1.0 / math.sqrt(sd / k), 1.0 / math.sqrt(sf / k), math.sqrt(sr / k))
        return self.scales

    def _inputs(self, x):
        ds, fs, _ = self.scales
        xs = x.clone()
        xs[0] *= ds
        xs[1:] *= fs
        return xs

    def loss(self, psi) -> tuple[float, float]:
        """(loss of the corrected force, loss without correction = 1): mean |c − r|² / mean |r|²."""
        x, r = self.pair(psi)
        c = self.lo.mesh_interp3(psi, self.net.apply(self._inputs(x))) * self.scales[2]
        rr = float((r.double() ** 2).mean())
        return float(((c - r).double() ** 2).mean()) / rr, 1.0

    def step(self, psi, lr: float) -> float:
        """One Adam step on one state; returns the relative loss before the step. The
        gradient is that of mean |c − r|² / out_scale² (one normalisation for all states,
        so that the late, strongly clustered states, whose residuals are largest, weigh
        most)."""
        x, r = self.pair(psi)
        xs = self._inputs(x)
        os_ = self.scales[2]
        c = self.lo.mesh_interp3(psi, self.net.apply(xs)) * os_
        d = c - r
        rr = float((r.double() ** 2).mean())
        loss = float((d.double() ** 2).mean()) / rr
        g = (2.0 / (d.numel() * os_)) * d               # d loss / d(net output at the particles)
        dout = self.lo.mesh_deposit3(psi, g.contiguous())
        self.net.backward_output_grad(xs, dout)
        self.net.adam_step(lr)
        return loss


def train(cosmo, *, n=128, boxsize=250.0, seeds=range(64), snapshots=20, epochs=8, lr=1e-3, lr_end=1e-4,
          opts_lo=OPTS_LO, opts_hi=OPTS, device=0, log=print):
    """Trains a ForceNet on `snapshots` states of each training seed; returns the trainer."""
    import torch
    T = CorrectionTrainer(cosmo, n=n, boxsize=boxsize, opts_lo=opts_lo, opts_hi=opts_hi, device=device)
    states = []
    t0 = time.perf_counter()
    for s in seeds:
        p0, m0 = initial_state(cosmo, n, boxsize, s, device)
        _, _, st, _ = run(cosmo, p0, m0, res=2 * n, boxsize=boxsize, n_steps=snapshots, opts=opts_hi, device=device,
                          keep_states=True)
        states += st
    t_data = time.perf_counter() - t0
    T.fit_scales(states[snapshots - 1::snapshots])        # the a = 1 states set the scales
    rng = np.random.default_rng(1)
    nstep = epochs * len(states)
    t0 = time.perf_counter()
    hist = []
    for e in range(epochs):
        order = rng.permutation(len(states))
        acc = 0.0
        for i, j in enumerate(order):
            it = e * len(states) + i
            lr_t = lr * (lr_end / lr) ** (it / max(nstep - 1, 1))    # geometric decay
            acc += T.step(states[j], lr_t)
        hist.append(acc / len(states))
        log(f"epoch {e}: mean relative loss {hist[-1]:.4f}")
    torch.cuda.synchronize(device)
    T.info = dict(n_states=len(states), data_s=t_data, train_s=time.perf_counter() - t0, loss_history=hist,
                  scales=list(T.scales), epochs=epochs, lr=lr, lr_end=lr_end, opts_lo=dict(opts_lo),
                  opts_hi=dict(opts_hi))
    return T


def evaluate(cosmo, net, scales, *, n, boxsize, seeds, n_steps=20, opts_lo=OPTS_LO, opts_hi=OPTS, device=0,
             bins=32, timing=False, every=1, start=0):
    """Plain 1×, corrected 1× and plain 2× runs from each held-out seed. Returns per-bin
    P(k) ratios to the 2× run (mean over seeds) for k < k_Nyq/2 of the 1× mesh, their
    largest deviations, and (timing) device ms per step of the corrected 1× and plain 2×."""
    ratios = {"plain": [], "corrected": []}
    ms = {"corrected": [], "plain_2x": [], "plain_1x": []}
    k = None
    for s in seeds:
        p0, m0 = initial_state(cosmo, n, boxsize, s, device)
        p2, _, _, t2 = run(cosmo, p0, m0, res=2 * n, boxsize=boxsize, n_steps=n_steps, opts=opts_hi, device=device,
                           timing=timing)
        p1, _, _, t1 = run(cosmo, p0, m0, res=n, boxsize=boxsize, n_steps=n_steps, opts=opts_lo, device=device,
                           timing=timing)
        pc, _, _, tc = run(cosmo, p0, m0, res=n, boxsize=boxsize, n_steps=n_steps, opts=opts_lo, device=device,
                           net=net, scales=scales, timing=timing, every=every, start=start)
        k, P2, nm = state_pk(p2, res=n, boxsize=boxsize, bins=bins, device=device)
        _, P1, _ = state_pk(p1, res=n, boxsize=boxsize, bins=bins, device=device)
        _, Pc, _ = state_pk(pc, res=n, boxsize=boxsize, bins=bins, device=device)
        sel = (nm > 0) & (k < 0.5 * math.pi * n / boxsize)
        ratios["plain"].append(P1[sel] / P2[sel])
        ratios["corrected"].append(Pc[sel] / P2[sel])
        if timing:
            ms["corrected"].append(tc)
            ms["plain_2x"].append(t2)
            ms["plain_1x"].append(t1)
        ksel = k[sel]
    out = {"k": ksel.tolist(), "seeds": list(seeds), "n_part": n, "boxsize": boxsize, "res_1x": n, "res_2x": 2 * n}
    for key, v in ratios.items():
        r = np.mean(np.array(v), axis=0)
        out[f"pk_ratio_{key}"] = r.tolist()
        out[f"pk_max_err_{key}"] = float(np.max(np.abs(r - 1)))
    if timing:
        out["ms_per_step"] = {key: float(np.median(v)) for key, v in ms.items()}
        out["speedup_vs_2x"] = out["ms_per_step"]["plain_2x"] / out["ms_per_step"]["corrected"]
    return out


def save(path, net, scales, info):
    np.savez(path, params=net.get_params(), scales=np.asarray(scales, dtype=np.float64),
             info=np.array(json.dumps(info)))


def load(path, device: int = 0):
    """(ForceNet with the saved weights, scales, info dict)."""
    d = np.load(path)
    net = ForceNet(layers=4, cin=4, hidden=32, cout=3, seed=0, device=device)
    net.load(d["params"])
    return net, tuple(float(v) for v in d["scales"]), json.loads(str(d["info"]))


def _main(argv=None):
    import argparse
    import os
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory for the weights and the metrics JSON")
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--boxsize", type=float, default=250.0)
    ap.add_argument("--seeds", type=int, default=64)
    ap.add_argument("--snapshots", type=int, default=20)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--eval-seeds", type=int, default=8)
    ap.add_argument("--lr-end", type=float, default=1e-4)
    ap.add_argument("--eval-large", type=int, default=512, help="particles per side of the large evaluation (0: skip)")
    ap.add_argument("--opts-lo", default=json.dumps(OPTS_LO), help="PMConfig options of the 1x mesh (JSON)")
    ap.add_argument("--opts-hi", default=json.dumps(OPTS), help="PMConfig options of the 2x mesh (JSON)")
    args = ap.parse_args(argv)
    opts_lo, opts_hi = json.loads(args.opts_lo), json.loads(args.opts_hi)
    os.makedirs(args.out, exist_ok=True)
    cosmo = Cosmology(**COSMO)
    T = train(cosmo, n=args.n, boxsize=args.boxsize, seeds=range(args.seeds), snapshots=args.snapshots,
              epochs=args.epochs, lr=args.lr, lr_end=args.lr_end, opts_lo=opts_lo, opts_hi=opts_hi)
    info = dict(T.info, n=args.n, boxsize=args.boxsize, train_seeds=args.seeds, snapshots=args.snapshots)
    held = range(1000, 1000 + args.eval_seeds)
    info["eval_small"] = evaluate(cosmo, T.net, T.scales, n=args.n, boxsize=args.boxsize, seeds=held,
                                  opts_lo=opts_lo, opts_hi=opts_hi)
    if args.eval_large:
        nl = args.eval_large
        info["eval_large"] = evaluate(cosmo, T.net, T.scales, n=nl, boxsize=args.boxsize * nl / args.n,
                                      seeds=held, timing=True, opts_lo=opts_lo, opts_hi=opts_hi)
    save(os.path.join(args.out, "force_correction.npz"), T.net, T.scales, info)
    with open(os.path.join(args.out, "force_correction.json"), "w") as f:
        json.dump(info, f, indent=1)
    print(json.dumps({k: v for k, v in info.items() if not isinstance(v, (list, dict))}))
    for key in ("eval_small", "eval_large"):
        if key in info:
            e = info[key]
            print(key, {k: e[k] for k in e if k.startswith("pk_max") or k in ("speedup_vs_2x", "ms_per_step")})
    T.close()


if __name__ == "__main__":
    _main()
