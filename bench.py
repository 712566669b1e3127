"""Throughput of the B200 PM step (particle-steps/s) on the headline workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl djb|reference] [--size c3|c2|small]

Workload (default `c3`): 512³ particles, 1024³ mesh, L = 1000 Mpc/h, flat ΛCDM
(Ωm 0.31, Ωb 0.049, h 0.677, n_s 0.965, σ8 0.81, EH transfer), 3LPT initial
conditions at a = 0.02 from seeded white noise, PCS assignment, interlacing
(antialias = 1), order-6 gradient, BullFrog stepper over W+K steps from a = 0.02
to 1 (W + K = 20 by default). A step is one drift-kick-drift step of the whole
particle set. W warm-up steps run untimed, then exactly K steps are timed with CUDA
events on the solver's stream between a barrier + synchronize on both sides; the
meshes (4.3 GB each) exceed L2, so no flush is needed between steps.

Multi-GPU (torchrun): replicas only — every rank evolves its own box (seed + rank),
no collective on the data path; value = all ranks' particle-steps / max time.

`--impl reference` times the CPU restatement of the reference's algorithm (the
oracle's OpenMP/pocketfft port, float32, all host threads) on the same workload
(512³ particles / 1024³ mesh, same options), rank 0 only: 1 warm-up step and 2 timed
steps, a bounded sample of the schedule (a step takes about a minute on the host).
Nothing in that arm loads the B200 library: cosmology, stepper coefficients and ICs
come from `oracle/`.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "discodj.jl_b200"))

METRIC = "particle-steps/s at 512³/1024³ mesh"
UNIT = "particle-steps/s"
COSMO = dict(Omega_c=0.31 - 0.049, Omega_b=0.049, h=0.677, n_s=0.965, sigma8=0.81)
SIZES = {
    # name: n, res, L, lpt order
    "c3": (512, 1024, 1000.0, 3),
    "c2": (256, 512, 500.0, 3),
    "small": (64, 128, 125.0, 2),
}
OPTIONS = dict(worder=4, antialias=1, grad_order=6, lap_order=0, deconvolve=False)
A_INI, A_END = 0.02, 1.0


def algorithmic_bytes(n, res, nshift=2):
    """Per-step and per-kernel algorithmic HBM bytes (float32).

    step: n_shift·(24·N_m + 24·N_p) + 48·N_p (one compulsory pass per array).
    kernels, per launch (one launch covers the 2 interlacing meshes):
      scatter: read Ψ (12 B/particle) and the sort order (4), write each mesh (4 B/cell);
               the first drift is applied by the binning pass
      gather:  read Ψ, Mom (24), write Ψ, Mom (24), read each potential mesh (4 B/cell)
      kspace:  read + write the half spectrum of one mesh (16 B/complex mode); the same
               for the fused z pass (forward z DFT, Kφ, inverse z DFT) at 1024³"""
    Np, Nm = n ** 3, res ** 3
    modes = res * res * (res // 2 + 1)
    return dict(
        step=nshift * (24 * Nm + 24 * Np) + 48 * Np,
        scatter=16 * Np + 4 * Nm * nshift,
        gather=48 * Np + 4 * Nm * nshift,
        kspace=16 * modes,
    )


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self._t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.dev)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()
        time.sleep(0.25)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks(key="hbm_gbs"):
    """(peak, "measured" | "fallback") from MEASURED_PEAKS.json: HBM GB/s or bf16 TFLOP/s."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        if key in d:
            return float(d[key]), "measured"
    return (6650.0 if key == "hbm_gbs" else 1590.0), "fallback"


def profile_traffic():
    """dram bytes per launch of the top kernel from the committed ncu summary, or None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        return json.load(open(p))
    return None


def dist_setup(backend: str | None = None):
    """One process per GPU (torchrun env); NCCL on GPUs, gloo on CPU-only hosts."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def replica_seed(rank: int, base: int = 42) -> int:
    """Replicas only: every rank evolves an independent box."""
    return base + rank


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(world, x: float) -> float:
    """Max over ranks (the timing rule: the slowest rank defines the step time)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_value(world: int, n_part: int, steps: int, ms_max: float) -> float:
    """Whole-job particle-steps/s: all ranks' particles over the slowest rank's time."""
    return world * n_part ** 3 * steps / (ms_max / 1e3)


def make_ics(cosmo, n, L, lpt, seed, device):
    """nLPT (Ψ, Π) at A_INI as native (3,n,n,n) float32 tensors on `device`: the library's
    CUDA generator (`djb_lpt_ics`) at n >= 256, the float64 torch restatement below."""
    import torch

    import djb200
    from djb200 import ics
    if n >= 256 and str(device).startswith("cuda"):
        return ics.lpt_ics_native(cosmo, n, L, A_INI, n_order=lpt, seed=seed, device=torch.device(device).index or 0)
    psi, pi = ics.lpt_ics(cosmo, n, L, A_INI, n_order=lpt, seed=seed, device=device, dtype=torch.float64)
    return djb200.native_view(psi.float()), djb200.native_view(pi.float())


def cpu_sample(n: int, res: int, L: float, steps: int, warmup: int, seed: int = 42):
    """The oracle's CPU port (float32 OpenMP scatter/gather + pocketfft on all host
    threads) stepping n³ particles on a res³ mesh with the headline options. Everything
    here comes from `oracle/` (cosmology, stepper coefficients, ICs): the B200 library
    is not loaded. ICs are 1LPT (Zel'dovich) of seeded white noise at a = 0.02; at that
    time the higher LPT orders move particles by ~1% of their displacement, which does
    not change the cost of a step."""
    import numpy as np

    from oracle import cosmology as cz
    from oracle import cpm, ics as oi, nbody as onb
    from oracle import pm as opm
    c = cz.compute_timetables(cz.Cosmology(**COSMO))
    psi, pi = oi.zeldovich_ics(n, L, cz.Dplus(c, A_INI), seed=seed, **COSMO)
    psi = psi.astype(np.float32)
    mom = pi.astype(np.float32)
    co = onb.stepper_coefficients(c, "bullfrog", A_INI, A_END, steps + warmup)
    cfg = opm.PMConfig(res_pm=res, n_part=n, boxsize=L, **OPTIONS)
    P = cpm.CPUPM(cfg, dtype=np.float32)
    for k in range(warmup):
        psi, mom = P.step(psi, mom, co["ddrift1"][k], co["alpha"][k], co["beta"][k], co["ddrift2"][k])
    t0 = time.perf_counter()
    for k in range(warmup, warmup + steps):
        psi, mom = P.step(psi, mom, co["ddrift1"][k], co["alpha"][k], co["beta"][k], co["ddrift2"][k])
    dt = time.perf_counter() - t0
    return dict(value=n ** 3 * steps / dt, unit=UNIT, cores=cpm.threads(), kind="port",
                sample=f"{n}^3 particles / {res}^3 mesh (L={L:g}), PCS, antialias=1, grad 6, BullFrog from a=0.02, "
                       f"1LPT ICs; {steps} timed steps after {warmup} warm-up; the oracle's float32 OpenMP "
                       f"scatter/gather + pocketfft port of the reference's PMSolver path (Julia is not installed)",
                ms_per_step=1e3 * dt / steps)


# The reference arm times full steps of the workload on the host cores; a step at
# 512³/1024³ takes about a minute there, so it runs a fixed, bounded sample of the
# requested schedule: 1 untimed warm-up step, then 2 timed steps.
REF_WARMUP, REF_STEPS = 1, 2


def run_reference(args, world, rank):
    if rank != 0:
        return
    n, res, L, lpt = SIZES[args.size]
    cb = cpu_sample(n, res, L, REF_STEPS, REF_WARMUP)
    cb["sample"] += f" (bounded sample of the requested {args.warmup}+{args.steps}-step schedule)"
    line = dict(metric=METRIC, value=cb["value"], unit=UNIT, n_gpus=args.gpus, steps=REF_STEPS,
                warmup=REF_WARMUP, ms_per_step=cb["ms_per_step"], higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype="f32", data="synthetic (seeded white noise -> EH P(k) -> 1LPT)",
                config=dict(config_block(args.size, n, res, L, lpt, world),
                            ics_of_sample="1LPT at a=0.02 from the oracle (the cost of a step does not depend on "
                                          "the IC order; the GPU arm starts from 3LPT)"),
                impl="reference",
                cpu_baseline={k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
                e2e=dict(value=cb["value"], unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)


def config_block(size, n, res, L, lpt, world):
    return dict(workload=f"PM step {n}^3 particles / {res}^3 mesh, L={L:g} Mpc/h, {lpt}LPT ICs at a={A_INI}, "
                         f"PCS + interlacing (antialias=1), order-6 gradient, BullFrog to a=1",
                size=size, n_part=n, res_pm=res, boxsize=L, worder=4, antialias=1, grad_order=6,
                stepper="bullfrog", parallelism=f"replicas{world}" if world > 1 else "single",
                l2="inputs larger than L2 (each mesh exceeds 126 MB); no flush")


def nn_flops_per_voxel(layers=4, cin=4, hidden=32, cout=3):
    """Algorithmic FLOPs per voxel of one forward pass: 2·27·cin·cout per layer with the
    real channel counts (the kernels pad K and N; the padding is not counted)."""
    f = 0
    for l in range(layers):
        ci = cin if l == 0 else hidden
        co = cout if l == layers - 1 else hidden
        f += 2 * 27 * ci * co
    return f


def nn_timing(dev, stream, world):
    """Adam steps of the 4-layer, 32-channel network at 128³ and one forward at 512³."""
    import torch

    from djb200.nn import ForceNet
    gen = torch.Generator(device=dev).manual_seed(11)
    out = {}
    with ForceNet(layers=4, cin=4, hidden=32, cout=3, seed=0) as net:
        net.set_stream(stream.cuda_stream)
        x = torch.randn((4, 128, 128, 128), generator=gen, device=dev)
        t = torch.randn((3, 128, 128, 128), generator=gen, device=dev)
        for _ in range(2):
            net.train_step(x, t, lr=1e-4)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(5):
            net.train_step(x, t, lr=1e-4)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_train = allmax(world, e0.elapsed_time(e1) / 5)
        del x, t
        x = torch.randn((4, 512, 512, 512), generator=gen, device=dev)
        net.apply(x)
        torch.cuda.synchronize()
        e0.record(stream)
        net.apply(x)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_eval = allmax(world, e0.elapsed_time(e1))
        del x
    peak, kind = measured_peaks(key="bf16_tflops")
    f = nn_flops_per_voxel()
    v128, v512 = 128 ** 3, 512 ** 3
    train_tflops = 3 * f * v128 / (ms_train / 1e3) / 1e12   # forward + two GEMMs per layer backward
    eval_tflops = f * v512 / (ms_eval / 1e3) / 1e12
    out.update(train_ms_per_step=ms_train, train_voxels_per_s=world * v128 / (ms_train / 1e3),
               eval_ms_512=ms_eval, eval_voxels_per_s=world * v512 / (ms_eval / 1e3),
               flops_per_voxel_forward=f,
               roofline=dict(bound="tensor", unit="TFLOP/s", achieved_train=train_tflops,
                             achieved_eval=eval_tflops, peak=peak, frac_train=train_tflops / peak,
                             frac_eval=eval_tflops / peak, peak_source=f"{kind} bf16_tflops"),
               note="4 layers 4->32->32->32->3, 3^3 kernels, periodic; forward, data-gradient and weight-"
                    "gradient convolutions as implicit GEMMs on the tcgen05 tensor cores (bf16 operands, float32 "
                    "accumulation in tensor memory; narrow inputs zero-widened for the weight gradient); "
                    "train = forward + backward + Adam at 128^3 (FLOPs counted as 3x forward); eval = one "
                    "forward at 512^3; FLOPs with the real channel counts")
    return out


def nn_corrected(world):
    """NN-corrected 1x-mesh PM against the plain 2x-mesh PM, 512³ particles in L = 1000
    (1x mesh 512³, 2x mesh 1024³ with this workload's options), one held-out seed, with
    the network trained by `python -m djb200.correction` and shipped with the package:
    P(k) at a = 1 against the 2x run for k < k_Nyq/2 of the 1x mesh, and device ms per
    step (CUDA events, after 2 steps) of the corrected 1x and the plain 2x runs."""
    import djb200
    from djb200 import correction
    path = os.path.join(ROOT, "discodj.jl_b200", "djb200", "data", "force_correction.npz")
    if not os.path.exists(path):
        return None
    net, scales, info = correction.load(path)
    cosmo = djb200.Cosmology(**correction.COSMO)
    ev = correction.evaluate(cosmo, net, scales, n=512, boxsize=1000.0, seeds=[1000], timing=True,
                             opts_lo=info.get("opts_lo", correction.OPTS_LO), opts_hi=info.get("opts_hi", correction.OPTS))
    net.close()
    ms = ev["ms_per_step"]
    return dict(pk_max_err_lt_kNyq2=ev["pk_max_err_corrected"], pk_max_err_plain_1x=ev["pk_max_err_plain"],
                speedup_vs_2x=ev["speedup_vs_2x"], ms_per_step=ms,
                value=world * 512 ** 3 / (ms["corrected"] / 1e3), unit=UNIT,
                # the 8-seed held-out P(k) errors recorded when the shipped network was evaluated
                # (its timing then is superseded by this run's)
                held_out={k: {kk: info[k][kk] for kk in ("n_part", "seeds", "pk_max_err_plain", "pk_max_err_corrected")
                              if kk in info[k]}
                          for k in ("eval_small", "eval_large") if k in info},
                note="1x: " + json.dumps(info.get("opts_lo")) + " + network; 2x: " + json.dumps(info.get("opts_hi")) +
                     "; trained on 64 seeds x 20 states of 128^3 particles (L=250) by this library's kernels")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=17)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="djb", choices=["djb", "reference"])
    ap.add_argument("--size", default="c3", choices=sorted(SIZES))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-nn", action="store_true")
    ap.add_argument("--only-nn-corrected", action="store_true",
                    help="run only the NN-corrected comparison at 512^3 and print it (profiling)")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("warm-up must be >= 3 steps")
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.only_nn_corrected:
        import torch
        torch.cuda.set_device(local)
        print(json.dumps(nn_corrected(world)), flush=True)
        return
    import numpy as np
    import torch

    import djb200
    dev = f"cuda:{local}"
    torch.cuda.set_device(local)
    n, res, L, lpt = SIZES[args.size]
    cosmo = djb200.Cosmology(**COSMO)
    psi_d, pi_d = make_ics(cosmo, n, L, lpt, replica_seed(rank), dev)
    # pinned host copies for the end-to-end leg
    psi_h = torch.empty((3, n, n, n), dtype=torch.float32, pin_memory=True)
    pi_h = torch.empty_like(psi_h, pin_memory=True)
    psi_h.copy_(psi_d)
    pi_h.copy_(pi_d)
    torch.cuda.empty_cache()
    nsteps = args.warmup + args.steps
    co = djb200.stepper_coefficients(cosmo, "bullfrog", A_INI, A_END, nsteps)
    cfg = djb200.PMConfig(res_pm=res, n_part=n, boxsize=L, **OPTIONS)
    S = djb200.PMSolver(cfg, device=local)
    stream = torch.cuda.Stream()          # a real stream: events and the solver share it
    torch.cuda.set_stream(stream)
    S.set_stream(stream.cuda_stream)
    S.set_state(psi_d, pi_d)
    del psi_d, pi_d
    for k in range(args.warmup):
        S.step(co["ddrift1"][k], co["alpha"][k], co["beta"][k], co["ddrift2"][k])
    S.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    S.profile(True)
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.warmup, nsteps):
        S.step(co["ddrift1"][k], co["alpha"][k], co["beta"][k], co["ddrift2"][k])
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms_local = e0.elapsed_time(e1)
    prof = S.profile_read()
    clk = clocks.stop()
    S.synchronize()
    ms = allmax(world, ms_local)
    device_bytes = S.device_bytes
    Np = n ** 3
    value = aggregate_value(world, n, args.steps, ms)

    # end to end through the C ABI with host buffers: H2D of (Ψ, Π) from pinned memory,
    # K fused steps, D2H of (X, P) into pinned memory, all inside the timed region
    e2e = None
    if not args.no_e2e:
        xo = torch.empty((3, n, n, n), dtype=torch.float32, pin_memory=True)
        po = torch.empty_like(xo, pin_memory=True)
        from djb200 import _lib
        import ctypes as C
        co2 = djb200.stepper_coefficients(cosmo, "bullfrog", A_INI, A_END, args.steps)
        arrs = [np.ascontiguousarray(co2[k]) for k in ("ddrift1", "alpha", "beta", "ddrift2")]
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _lib.check(_lib.lib.djb_set_state(S.handle, C.c_void_p(psi_h.data_ptr()), C.c_void_p(pi_h.data_ptr()),
                                          1.0, _lib.MEM_HOST))
        _lib.check(_lib.lib.djb_run(S.handle, args.steps, *[_lib.dptr(a) for a in arrs]))
        _lib.check(_lib.lib.djb_get_output(S.handle, C.c_void_p(xo.data_ptr()), C.c_void_p(po.data_ptr()), 1,
                                           1.0, cosmo.Fplus(A_END), _lib.MEM_HOST))
        t_e2e = time.perf_counter() - t0
        barrier(world)
        t_e2e = allmax(world, t_e2e)
        e2e = dict(value=world * Np * args.steps / t_e2e, unit=UNIT,
                   h2d_bytes_per_step=int(2 * 12 * Np / args.steps),
                   d2h_bytes_per_step=int(2 * 12 * Np / args.steps),
                   note=f"one run of {args.steps} steps through djb_set_state/djb_run/djb_get_output with "
                        f"pinned host buffers; bytes per step = state in + (X, P) out over the run")

    # adjoint of a step (djb_step_vjp) on the resident final state, device arrays, CUDA
    # events on the solver's stream: one untimed call, then two timed
    adjoint = None
    if not args.no_adjoint:
        p_s, m_s = S.get_state(device=True)
        gen = torch.Generator(device=dev).manual_seed(5)
        pb = torch.randn(p_s.shape, generator=gen, device=dev)
        mb = torch.randn(p_s.shape, generator=gen, device=dev)
        k_last = nsteps - 1
        cargs = (co["ddrift1"][k_last], co["alpha"][k_last], co["beta"][k_last], co["ddrift2"][k_last])
        torch.cuda.nvtx.range_push("step_vjp")   # the untimed call, for `ncu --nvtx-include step_vjp/`
        S.step_vjp(*cargs, p_s, m_s, pb, mb)
        torch.cuda.nvtx.range_pop()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a0.record(stream)
        for _ in range(2):
            S.step_vjp(*cargs, p_s, m_s, pb, mb)
        a1.record(stream)
        torch.cuda.synchronize()
        ms_vjp = allmax(world, a0.elapsed_time(a1) / 2)
        adjoint = dict(ms_per_step_vjp=ms_vjp, value=world * Np / (ms_vjp / 1e3), unit=UNIT,
                       note="djb_step_vjp at the last step's coefficients on the final state: drift, force VJP "
                            "over both shifts (deposit, Poisson, FD gradient, weight-derivative gathers, "
                            "cotangent deposit, transposed stencil, Poisson), kick and drift adjoints")
        del p_s, m_s, pb, mb

    # force-correction network: Adam steps at 128³ and one application at 512³ (random
    # inputs of the network's shape; the timing does not depend on the values)
    nn = None
    if not args.no_nn:
        nn = nn_timing(dev, stream, world)
    nnc = None
    if not args.no_nn and args.size == "c3":
        S.close()      # the corrected and 2x runs hold their own meshes
        torch.cuda.empty_cache()
        nnc = nn_corrected(world)

    # roofline of the dominant kernel of this library (CUDA-event time per launch)
    ab = algorithmic_bytes(n, res)
    peak, peak_kind = measured_peaks()
    mine = {k: prof[k] for k in ("scatter", "kspace", "gather")}
    top = max(mine, key=lambda k: mine[k][0])
    t_ms, launches, calls = mine[top]
    per_launch_ms = t_ms / max(calls, 1)
    per_launch_bytes = ab[top] if top != "kspace" else ab["kspace"]
    achieved = per_launch_bytes / (per_launch_ms / 1e3) / 1e9
    tr = profile_traffic()
    traffic = None
    if tr and tr.get("kernel") == top and tr.get("size") == args.size:
        traffic = tr.get("dram_bytes_per_launch")
    step_bytes = ab["step"]
    step_ms = ms / args.steps
    roof = dict(bound="hbm", kernel=top, achieved=achieved, peak=peak, unit="GB/s", frac=achieved / peak,
                traffic=traffic, peak_source=f"{peak_kind} hbm_gbs",
                algorithmic_bytes_per_launch=per_launch_bytes, ms_per_launch=per_launch_ms)
    # the pipe that does bound the brick interpolation: shared-memory wavefronts (one per SM
    # clock at most), from the committed ncu count per particle-shift and this run's time
    pipe = None
    if top == "gather" and tr and tr.get("smem_wavefronts_per_particle_shift"):
        wf = tr["smem_wavefronts_per_particle_shift"] * n ** 3 * 2
        sm_hz = float((clk or {}).get("sm_mhz") or 0) * 1e6
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        if sm_hz > 0:
            ach = wf / (per_launch_ms / 1e3)
            pipe = dict(kernel="gather", unit="shared-memory wavefronts/s", wavefronts_per_launch=wf, achieved=ach,
                        peak=sms * sm_hz, frac=ach / (sms * sm_hz),
                        source="wavefronts per particle-shift from profiles/traffic.json; peak = SMs x median SM "
                               "clock of this run (one 128-byte wavefront per clock per SM)")
    phases = {k: dict(ms_per_step=v[0] / args.steps, launches=v[1]) for k, v in prof.items() if v[2]}
    step_roof = dict(algorithmic_bytes=step_bytes, achieved=step_bytes / (step_ms / 1e3) / 1e9, peak=peak,
                     frac=step_bytes / (step_ms / 1e3) / 1e9 / peak, unit="GB/s")
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # a 1/64-volume sub-box of the workload at the same resolution (cell and particle
        # spacing, options): 128³ particles on a 256³ mesh in L = 250 Mpc/h
        cb = cpu_sample(n // 4, res // 4, L / 4, 2, 1)
        cpu = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    if rank == 0:
        line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup,
                    ms_per_step=step_ms, higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32",
                    data="synthetic (seeded white noise -> EH P(k) -> 3LPT)",
                    config=config_block(args.size, n, res, L, lpt, world), roofline=roof, pipe_roofline=pipe,
                    step_roofline=step_roof, phases=phases, cpu_baseline=cpu, e2e=e2e, adjoint=adjoint, nn=nn,
                    nn_corrected=nnc, clocks=clk,
                    gpu_launches=int(sum(v[1] for v in prof.values())),
                    device_bytes=device_bytes)
        print(json.dumps(line), flush=True)
    S.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
