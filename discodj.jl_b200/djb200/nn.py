"""Force-correction network on the PM mesh (no counterpart in the reference).

A 3-D CNN with 3³ kernels and periodic boundaries over libdjb200's `djb_nn_*`
entry points: implicit GEMMs on the tcgen05 tensor cores (bf16 operands, float32
accumulation in tensor memory), float32 master weights, Adam. Meshes are (channels, res, res, res) float32 in the library's memory
order [c][z][y][x]: numpy arrays on the host, or torch CUDA tensors.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import MEM_DEVICE, MEM_HOST, check, lib


def _pad8(c: int) -> int:
    return (c + 7) // 8 * 8


class ForceNet:
    """`layers` convolutions cin → hidden → … → cout, ReLU between them."""

    def __init__(self, layers: int = 4, cin: int = 4, hidden: int = 32, cout: int = 3, seed: int = 0,
                 device: int = 0):
        self.layers, self.cin, self.hidden, self.cout, self.device = layers, cin, hidden, cout, device
        h = C.c_void_p()
        check(lib.djb_nn_create(layers, cin, hidden, cout, C.c_uint64(seed), device, C.byref(h)))
        self._h = h
        n = C.c_int64()
        check(lib.djb_nn_param_count(self._h, C.byref(n)))
        self.n_params = n.value

    def close(self):
        if getattr(self, "_h", None):
            lib.djb_nn_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def layout(self):
        """[(W: (27, cin_pad, cout_pad), b: (cout_pad,), cin, cout)] offsets into params."""
        out, off = [], 0
        for l in range(self.layers):
            ci = self.cin if l == 0 else self.hidden
            co = self.cout if l == self.layers - 1 else self.hidden
            cp, op = _pad8(ci), _pad8(co)
            out.append((off, (27, cp, op), off + 27 * cp * op, op, ci, co))
            off += 27 * cp * op + op
        return out

    def set_stream(self, stream_ptr: int | None):
        check(lib.djb_nn_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def set_conv(self, mode: str):
        """"tensor" (default): convolutions, forward and backward, as implicit GEMMs on
        the tcgen05 tensor cores where the padded channel counts are at most 32;
        "im2col": im2col + cuBLAS GEMMs for every layer."""
        modes = {"tensor": 0, "im2col": 1}
        if mode not in modes:
            raise ValueError(f"conv mode must be one of {sorted(modes)}")
        check(lib.djb_nn_set_conv(self._h, modes[mode]))

    def conv_info(self) -> dict:
        """{"mode": "tensor" | "im2col", "tma": bool}: the convolution path and whether
        the tensor-core kernel has staged planes by bulk tensor copies."""
        mode, tma = C.c_int32(), C.c_int32()
        check(lib.djb_nn_get_conv(self._h, C.byref(mode), C.byref(tma)))
        return {"mode": "im2col" if mode.value else "tensor", "tma": bool(tma.value)}

    def get_params(self) -> np.ndarray:
        p = np.empty(self.n_params, dtype=np.float32)
        check(lib.djb_nn_get_params(self._h, C.c_void_p(p.ctypes.data)))
        return p

    def load(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.shape != (self.n_params,):
            raise ValueError(f"expected {self.n_params} parameters")
        check(lib.djb_nn_load(self._h, C.c_void_p(p.ctypes.data)))

    def _mesh(self, x, channels):
        if type(x).__module__.startswith("torch") and x.is_cuda:
            if tuple(x.shape[:1]) != (channels,) or x.dim() != 4 or not x.is_contiguous():
                raise ValueError(f"expected a contiguous ({channels}, res, res, res) tensor")
            return C.c_void_p(x.data_ptr()), MEM_DEVICE, x, int(x.shape[1])
        a = np.ascontiguousarray(x, dtype=np.float32)
        if a.ndim != 4 or a.shape[0] != channels:
            raise ValueError(f"expected a ({channels}, res, res, res) array")
        return C.c_void_p(a.ctypes.data), MEM_HOST, a, int(a.shape[1])

    def apply(self, x):
        p, mem, keep, res = self._mesh(x, self.cin)
        if mem == MEM_DEVICE:
            import torch
            out = torch.empty((self.cout, res, res, res), dtype=torch.float32, device=x.device)
            check(lib.djb_nn_apply(self._h, p, res, C.c_void_p(out.data_ptr()), mem))
        else:
            out = np.empty((self.cout, res, res, res), dtype=np.float32)
            check(lib.djb_nn_apply(self._h, p, res, C.c_void_p(out.ctypes.data), mem))
        del keep
        return out

    def train_step(self, x, target, lr: float = 1e-3) -> float:
        p, mem, k1, res = self._mesh(x, self.cin)
        t, mem2, k2, res2 = self._mesh(target, self.cout)
        if mem != mem2 or res != res2:
            raise ValueError("x and target must live in the same memory and have the same size")
        loss = C.c_double()
        check(lib.djb_nn_train_step(self._h, p, t, res, float(lr), C.byref(loss), mem))
        del k1, k2
        return loss.value

    def backward(self, x, target) -> float:
        """Gradients of the MSE into the network's buffer; returns the loss."""
        p, mem, k1, res = self._mesh(x, self.cin)
        t, mem2, k2, res2 = self._mesh(target, self.cout)
        if mem != mem2 or res != res2:
            raise ValueError("x and target must live in the same memory and have the same size")
        loss = C.c_double()
        check(lib.djb_nn_backward(self._h, p, t, res, C.byref(loss), mem))
        del k1, k2
        return loss.value

    def backward_output_grad(self, x, dout):
        """Gradients of Σ dout·net(x) into the network's buffer (dout: the loss gradient
        with respect to the output mesh, same memory and size as x)."""
        p, mem, k1, res = self._mesh(x, self.cin)
        d, mem2, k2, res2 = self._mesh(dout, self.cout)
        if mem != mem2 or res != res2:
            raise ValueError("x and dout must live in the same memory and have the same size")
        check(lib.djb_nn_backward_output_grad(self._h, p, d, res, mem))
        del k1, k2

    def grads(self) -> np.ndarray:
        g = np.empty(self.n_params, dtype=np.float32)
        check(lib.djb_nn_grads(self._h, C.c_void_p(g.ctypes.data), MEM_HOST))
        return g

    def set_grads(self, g):
        g = np.ascontiguousarray(g, dtype=np.float32)
        check(lib.djb_nn_set_grads(self._h, C.c_void_p(g.ctypes.data), MEM_HOST))

    def adam_step(self, lr: float = 1e-3):
        check(lib.djb_nn_adam_step(self._h, float(lr)))


def allreduce_gradients(net, group=None):
    """Data-parallel training over seeds, one replica per GPU: every replica's gradient
    buffer is replaced by the mean over the replicas (djb_nn_grads, all_reduce,
    djb_nn_set_grads) before its Adam step, so that the replicas' weights stay equal."""
    import torch
    import torch.distributed as dist
    g = torch.from_numpy(net.grads())
    if dist.get_backend(group) == "nccl":
        g = g.cuda()
    dist.all_reduce(g, group=group)
    g /= dist.get_world_size(group)
    net.set_grads(g.cpu().numpy())


def force_correction_pair(cosmo, *, n=64, boxsize=250.0, res=128, a=1.0, seed=0, worder=4, grad_order=6,
                          device=0):
    """One training pair for the force-correction network on device tensors.

    Particles: 2LPT initial conditions (seeded white noise) moved to scale factor `a`
    with the linear growth ratio. Input: [δ, F] on the res³ mesh (djb_mesh_fields);
    target: ΔF = F at twice the resolution, sampled at the res³ nodes, minus F."""
    import torch

    from . import ics
    from .pm import PMConfig, PMSolver, native_view
    psi, _ = ics.lpt_ics(cosmo, n, boxsize, 0.02, n_order=2, seed=seed, device=f"cuda:{device}",
                         dtype=torch.float32)
    psi = native_view(psi * float(cosmo.Dplus(a) / cosmo.Dplus(0.02)))
    with PMSolver(PMConfig(res_pm=res, n_part=n, boxsize=boxsize, worder=worder, grad_order=grad_order),
                  device=device) as lo:
        x = lo.mesh_fields(psi)
    with PMSolver(PMConfig(res_pm=2 * res, n_part=n, boxsize=boxsize, worder=worder, grad_order=grad_order),
                  device=device) as hi:
        fh = hi.mesh_fields(psi)[1:, ::2, ::2, ::2].contiguous()
    return x, (fh - x[1:]).contiguous()


def _main(argv=None):
    """Forward passes (and optionally Adam steps) of the 4-layer, 32-channel network on
    a seeded random res³ input, for profiling: python -m djb200.nn --res 256."""
    import argparse

    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--res", type=int, default=256)
    ap.add_argument("--repeat", type=int, default=2)
    ap.add_argument("--conv", default="tensor", choices=["tensor", "im2col"])
    ap.add_argument("--train", action="store_true", help="Adam steps instead of forward passes")
    args = ap.parse_args(argv)
    gen = torch.Generator(device="cuda:0").manual_seed(11)
    r = args.res
    with ForceNet(layers=4, cin=4, hidden=32, cout=3, seed=0) as net:
        net.set_conv(args.conv)
        x = torch.randn((4, r, r, r), generator=gen, device="cuda:0")
        t = torch.randn((3, r, r, r), generator=gen, device="cuda:0") if args.train else None
        for _ in range(args.repeat):
            if args.train:
                net.train_step(x, t, lr=1e-4)
            else:
                net.apply(x)
        torch.cuda.synchronize()
        print(net.conv_info())


if __name__ == "__main__":
    _main()
