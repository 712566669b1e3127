"""PM force on the B200: `PMConfig`, `PMSolver`, `pm_acceleration`.

Mirrors native/DiscoDJNative/src/nbody/pm.jl:28-46,366-414,503-529,545-585 on top
of libdjb200's C ABI. Arrays follow the reference's logical layout: particle
fields are (n,n,n,3) indexed [i,j,k,c]. Host arrays are numpy (any order; they
are converted to the column-major float32 memory the C ABI takes). Device arrays
are torch CUDA tensors in that memory layout, i.e. shape (3,n,n,n) contiguous
indexed [c,k,j,i] (`native_view`/`logical_view` convert).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import MEM_DEVICE, MEM_HOST, check, lib


@dataclass
class PMConfig:
    """pm.jl:35-46 (keyword names and defaults as there)."""
    res_pm: int
    n_part: int
    boxsize: float
    worder: int = 2
    deconvolve: bool = False
    antialias: int = 0
    grad_order: int = 4
    lap_order: int = 0
    n_resample: int = 1
    resampling: str = "fourier"

    def to_c(self, lean: bool = False, device: int = 0) -> _lib.PMConfigC:
        if self.resampling not in _lib.RESAMPLING:
            raise _lib.DJBInvalidOption(_lib.DJB_ERR_INVALID, "resampling must be :fourier or :linear")
        return _lib.PMConfigC(int(self.res_pm), int(self.n_part), float(self.boxsize), int(self.worder),
                              int(bool(self.deconvolve)), int(self.antialias), int(self.grad_order),
                              int(self.lap_order), int(self.n_resample), _lib.RESAMPLING[self.resampling],
                              int(bool(lean)), int(device))


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def native_host(a, n: int) -> np.ndarray:
    """(n,n,n,3) logical array -> float32 numpy in the C ABI's memory order."""
    a = np.asarray(a)
    if a.shape != (n, n, n, 3):
        raise ValueError(f"expected a ({n},{n},{n},3) particle array, got {a.shape}")
    return np.asfortranarray(a, dtype=np.float32)


def native_view(t):
    """(n,n,n,3) torch tensor -> contiguous (3,n,n,n) tensor with the C ABI's memory order."""
    return t.permute(3, 2, 1, 0).contiguous()


def logical_view(t):
    """Inverse of `native_view`: (3,n,n,n) -> (n,n,n,3) view."""
    return t.permute(3, 2, 1, 0)


def _ptr_mem(x, n: int):
    """(pointer, mem kind, keep-alive) for a particle array argument."""
    if _is_torch(x):
        if x.dtype.__repr__() != "torch.float32" or not x.is_contiguous() or tuple(x.shape) != (3, n, n, n):
            raise ValueError("device particle arrays must be contiguous float32 (3,n,n,n) tensors "
                             "(use djb200.native_view)")
        if x.is_cuda:
            return C.c_void_p(x.data_ptr()), MEM_DEVICE, x
        x = x.numpy()
        return C.c_void_p(x.ctypes.data), MEM_HOST, x
    h = native_host(x, n)
    return C.c_void_p(h.ctypes.data), MEM_HOST, h


def _empty_like_mem(x, n: int, mem: int):
    if mem == MEM_DEVICE:
        import torch
        return torch.empty((3, n, n, n), dtype=torch.float32, device=x.device)
    return np.empty((n, n, n, 3), dtype=np.float32, order="F")


def _copy_mem(x, n: int, mem: int):
    """A writable copy of a particle array in the C ABI's layout and memory kind."""
    if mem == MEM_DEVICE:
        if not _is_torch(x) or not x.is_cuda:
            raise ValueError("all arrays must live in the same memory")
        return x.contiguous().clone()
    return np.array(native_host(x.numpy() if _is_torch(x) else x, n), order="F", copy=True)


def _out_ptr(x):
    return C.c_void_p(x.data_ptr()) if _is_torch(x) else C.c_void_p(x.ctypes.data)


class PMSolver:
    """B200 PM workspace (`PMSolver` / `PMSolverLean`, pm.jl:371-414,547-585).

    Owns the device meshes, cuFFT plans and the resident particle state."""

    def __init__(self, cfg: PMConfig, like=None, *, lean: bool = False, device: int = 0):
        self.cfg = cfg
        self.lean = lean
        self.device = device
        self.n = int(cfg.n_part)
        c = cfg.to_c(lean=lean, device=device)
        h = C.c_void_p()
        check(lib.djb_solver_create(C.byref(c), C.byref(h)))
        self._h = h

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            lib.djb_solver_destroy(h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    @property
    def device_bytes(self) -> int:
        v = C.c_int64()
        check(lib.djb_solver_device_bytes(self._h, C.byref(v)))
        return v.value

    def set_stream(self, stream_ptr: int | None):
        check(lib.djb_solver_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    # pm_acceleration!(S, psi)
    def acceleration(self, psi, out=None):
        n = self.n
        p, mem, keep = _ptr_mem(psi, n)
        if out is None:
            if mem == MEM_DEVICE:
                import torch
                out = torch.empty((3, n, n, n), dtype=torch.float32, device=psi.device)
            else:
                out = np.empty((n, n, n, 3), dtype=np.float32, order="F")
        optr = C.c_void_p(out.data_ptr()) if _is_torch(out) else C.c_void_p(out.ctypes.data)
        if _is_torch(out) != (mem == MEM_DEVICE) or (not _is_torch(out) and not out.flags.f_contiguous):
            raise ValueError("out must match psi's memory kind and layout")
        check(lib.djb_pm_acceleration(self._h, p, optr, mem))
        del keep
        return out

    def acceleration_vjp(self, psi, acc_bar):
        """ψ̄ = (∂acc/∂ψ)ᵀ ā at displacements psi (no reference counterpart). Host arrays
        give a host (n,n,n,3) array; device (3,n,n,n) tensors give a device tensor."""
        n = self.n
        p, mem, k1 = _ptr_mem(psi, n)
        a, mem2, k2 = _ptr_mem(acc_bar, n)
        if mem != mem2:
            raise ValueError("psi and acc_bar must live in the same memory")
        out = _empty_like_mem(psi, n, mem)
        check(lib.djb_pm_acceleration_vjp(self._h, p, a, _out_ptr(out), mem))
        del k1, k2
        return out

    def step_vjp(self, dd1, alpha, beta, dd2, psi0, mom0, psi_bar, mom_bar):
        """Cotangents (ψ̄₀, M̄₀) of the state (psi0, mom0) a step started from, given those
        after the step (psi_bar, mom_bar; not modified)."""
        n = self.n
        p, mem, k1 = _ptr_mem(psi0, n)
        m, _, k2 = _ptr_mem(mom0, n)
        pb = _copy_mem(psi_bar, n, mem)
        mb = _copy_mem(mom_bar, n, mem)
        check(lib.djb_step_vjp(self._h, float(dd1), float(alpha), float(beta), float(dd2), p, m, _out_ptr(pb),
                               _out_ptr(mb), mem))
        del k1, k2
        return pb, mb

    def state_power_spectrum_vjp(self, pk_bar, bins: int = 32, logarithmic: bool = True, device: bool = False):
        """ψ̄ of Σ_b pk_bar[b]·P_b for P(k) of the resident state (state_power_spectrum)."""
        n = self.n
        pb = np.ascontiguousarray(pk_bar, dtype=np.float64)
        if pb.shape != (bins,):
            raise ValueError("pk_bar must have one entry per bin")
        if device:
            import torch
            out = torch.empty((3, n, n, n), dtype=torch.float32, device=f"cuda:{self.device}")
            check(lib.djb_state_power_spectrum_vjp(self._h, int(bins), int(bool(logarithmic)), _lib.dptr(pb),
                                                   C.c_void_p(out.data_ptr()), MEM_DEVICE))
            return out
        out = np.empty((n, n, n, 3), dtype=np.float32, order="F")
        check(lib.djb_state_power_spectrum_vjp(self._h, int(bins), int(bool(logarithmic)), _lib.dptr(pb),
                                               C.c_void_p(out.ctypes.data), MEM_HOST))
        return out

    def mesh_fields(self, psi):
        """[δ, F_x, F_y, F_z] on the mesh for displacements psi: (4, res, res, res) float32
        [c][z][y][x] (host numpy for host psi, a device tensor for a device psi)."""
        n, res = self.n, int(self.cfg.res_pm)
        p, mem, keep = _ptr_mem(psi, n)
        if mem == MEM_DEVICE:
            import torch
            out = torch.empty((4, res, res, res), dtype=torch.float32, device=psi.device)
        else:
            out = np.empty((4, res, res, res), dtype=np.float32)
        check(lib.djb_mesh_fields(self._h, p, _out_ptr(out), mem))
        del keep
        return out

    def attach_nn(self, net, delta_scale: float = 1.0, force_scale: float = 1.0, out_scale: float = 1.0):
        """Adds out_scale·interp(net([delta_scale·δ, force_scale·F])) to every force of this
        solver (`djb_solver_attach_nn`); net = None detaches."""
        check(lib.djb_solver_attach_nn(self._h, net._h if net is not None else None, float(delta_scale),
                                       float(force_scale), float(out_scale)))
        self._net = net   # the network must outlive its attachment

    def nn_schedule(self, every: int = 1, start: int = 0):
        """The attached network corrects the force from step `start` on, running on every
        `every`-th of those steps; in between, each particle keeps the correction it was
        last given (`djb_solver_nn_schedule`)."""
        check(lib.djb_solver_nn_schedule(self._h, int(every), int(start)))

    def mesh_interp3(self, psi, mesh3):
        """(3,n,n,n) device tensor of the W-order interpolation of three res³ meshes
        ((3,res,res,res) device tensor [c][z][y][x]) at X = q + psi (device, native layout)."""
        import torch
        p, mem, keep = _ptr_mem(psi, self.n)
        if mem != MEM_DEVICE or not mesh3.is_cuda or not mesh3.is_contiguous():
            raise ValueError("mesh_interp3 takes device tensors")
        out = torch.empty((3, self.n, self.n, self.n), dtype=torch.float32, device=psi.device)
        check(lib.djb_mesh_interp3(self._h, p, C.c_void_p(mesh3.data_ptr()), C.c_void_p(out.data_ptr()), mem))
        del keep
        return out

    def mesh_deposit3(self, psi, vec):
        """The transpose of `mesh_interp3`: (3,res,res,res) device tensor."""
        import torch
        p, mem, keep = _ptr_mem(psi, self.n)
        v, mem2, keep2 = _ptr_mem(vec, self.n)
        if mem != MEM_DEVICE or mem2 != MEM_DEVICE:
            raise ValueError("mesh_deposit3 takes device tensors")
        r = int(self.cfg.res_pm)
        out = torch.empty((3, r, r, r), dtype=torch.float32, device=psi.device)
        check(lib.djb_mesh_deposit3(self._h, p, v, C.c_void_p(out.data_ptr()), mem))
        del keep, keep2
        return out

    def set_state(self, psi, mom, mom_scale: float = 1.0):
        n = self.n
        p, mem, k1 = _ptr_mem(psi, n)
        m, mem2, k2 = _ptr_mem(mom, n)
        if mem != mem2:
            raise ValueError("psi and mom must live in the same memory")
        check(lib.djb_set_state(self._h, p, m, float(mom_scale), mem))
        del k1, k2

    def get_state(self, device: bool = False):
        n = self.n
        if device:
            import torch
            psi = torch.empty((3, n, n, n), dtype=torch.float32, device=f"cuda:{self.device}")
            mom = torch.empty_like(psi)
            check(lib.djb_get_state(self._h, C.c_void_p(psi.data_ptr()), C.c_void_p(mom.data_ptr()), MEM_DEVICE))
            return psi, mom
        psi = np.empty((n, n, n, 3), dtype=np.float32, order="F")
        mom = np.empty((n, n, n, 3), dtype=np.float32, order="F")
        check(lib.djb_get_state(self._h, C.c_void_p(psi.ctypes.data), C.c_void_p(mom.ctypes.data), MEM_HOST))
        return psi, mom

    def step(self, dd1: float, alpha: float, beta: float, dd2: float):
        check(lib.djb_step(self._h, float(dd1), float(alpha), float(beta), float(dd2)))

    def run(self, dd1, alpha, beta, dd2):
        arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (dd1, alpha, beta, dd2)]
        check(lib.djb_run(self._h, len(arrs[0]), *[_lib.dptr(a) for a in arrs]))

    def synchronize(self):
        check(lib.djb_synchronize(self._h))

    PHASES = ("clear", "scatter", "resample", "r2c", "kspace", "c2r", "gather", "sort", "nn")

    def profile(self, enable: bool = True):
        """Start (or stop) per-phase CUDA-event timing; resets the sums."""
        check(lib.djb_solver_profile(self._h, int(bool(enable))))

    def profile_read(self) -> dict:
        """{phase: (ms, kernel launches, executions)} since the last read; resets."""
        n = len(self.PHASES)
        ms = np.zeros(n)
        la = np.zeros(n, dtype=np.int64)
        ca = np.zeros(n, dtype=np.int64)
        check(lib.djb_solver_profile_read(self._h, _lib.dptr(ms), _lib.i64ptr(la), _lib.i64ptr(ca), n))
        return {name: (float(ms[i]), int(la[i]), int(ca[i])) for i, name in enumerate(self.PHASES)}

    def output(self, wrap: bool, p_div: float = 1.0, p_mul: float = 1.0, x=True, p=True):
        n = self.n
        xo = np.empty((n, n, n, 3), dtype=np.float32, order="F") if x else None
        po = np.empty((n, n, n, 3), dtype=np.float32, order="F") if p else None
        check(lib.djb_get_output(self._h, C.c_void_p(xo.ctypes.data) if x else None,
                                 C.c_void_p(po.ctypes.data) if p else None, int(wrap),
                                 float(p_div), float(p_mul), MEM_HOST))
        return xo, po

    def write_snapshot(self, path, D: float, L: float, p_div: float = 1.0, p_mul: float = 1.0):
        """HDF5 snapshot of the resident state: "Psi" (the displacement) and
        "Pi" = Mom / p_div * p_mul, root attributes "D" and "L" (the study driver's
        `snap_writer`, run_jobs.jl:41-48; the reference passes Pi = P / Fplus(a)).
        Streams from HBM through pinned buffers (`djb_state_write_snapshot`)."""
        check(lib.djb_state_write_snapshot(self._h, os.fsencode(path), float(D), float(L), float(p_div),
                                           float(p_mul)))

    def state_density_modes(self, modes) -> np.ndarray:
        """Complex δ(m)/res³ / W_CIC(m) of the resident state at integer modes (k, 3)
        (`djb_state_density_modes`; measure.jl:80-91 `density_modes`)."""
        m = np.ascontiguousarray(np.asarray(modes, dtype=np.int32).reshape(-1, 3))
        out = np.empty(2 * len(m), dtype=np.float64)
        check(lib.djb_state_density_modes(self._h, len(m), m.ctypes.data_as(C.POINTER(C.c_int32)), _lib.dptr(out)))
        return out[0::2] + 1j * out[1::2]

    def state_power_spectrum(self, bins: int = 32, logarithmic: bool = True):
        k = np.empty(bins)
        pk = np.empty(bins)
        nm = np.empty(bins, dtype=np.int64)
        check(lib.djb_state_power_spectrum(self._h, int(bins), int(bool(logarithmic)), _lib.dptr(k),
                                           _lib.dptr(pk), _lib.i64ptr(nm)))
        return k, pk, nm


def pm_acceleration(psi, cfg: PMConfig, solver: PMSolver | None = None):
    """pm.jl:528-529: −∇φ at X = q + ψ (a fresh array)."""
    if solver is None:
        with PMSolver(cfg) as s:
            return s.acceleration(psi)
    return solver.acceleration(psi)


def pm_acceleration_(solver: PMSolver, psi, out=None):
    """pm.jl:507 `pm_acceleration!(S, psi)` (writes into `out` when given)."""
    return solver.acceleration(psi, out=out)
