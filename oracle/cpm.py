"""ctypes binding of cpm.c and a threaded CPU PM step built on it.

TEST INFRASTRUCTURE ONLY (see `oracle/__init__.py`). `CPUPM` restates the
reference's optimised `PMSolver` path (pm.jl:466-521): OpenMP atomic scatter,
pocketfft (scipy.fft, all cores) R2C, multiplier Kφ, unnormalised C2R, the
finite-difference stencil into a 3-component force mesh and the fused gather;
the DKD step of run_nbody.jl:156-158 in numpy. float32 or float64. It is the
CPU baseline that bench.py times and the checker for the larger parity cases.
Sheet resampling is not supported here (use `oracle.pm`).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from . import pm as opm

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cpm.c")
LIB = os.path.join(HERE, "libcpm.so")


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        cmd = ["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-shared", "-fPIC", SRC, "-o", LIB + ".tmp", "-lm"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"gcc failed:\n{r.stderr}")
        os.replace(LIB + ".tmp", LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        for suf, ct in (("f32", C.c_float), ("f64", C.c_double)):
            P = C.c_void_p
            getattr(L, f"cpm_scatter_{suf}").argtypes = [P, C.c_int64, C.c_int, ct, C.c_int, P]
            getattr(L, f"cpm_fdgrad_{suf}").argtypes = [P, C.c_int, ct, ct, ct, P]
            getattr(L, f"cpm_gather3_{suf}").argtypes = [P, P, C.c_int64, C.c_int, ct, C.c_int, P]
            getattr(L, f"cpm_gather1_{suf}").argtypes = [P, P, C.c_int64, C.c_int, ct, C.c_int, P]
        L.cpm_threads.restype = C.c_int
        _lib = L
    return _lib


def threads() -> int:
    return int(lib().cpm_threads())


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


class CPUPM:
    """PM force/step on the CPU. Particle arrays are (n,n,n,3) logical [i,j,k,c]."""

    def __init__(self, cfg: opm.PMConfig, dtype=np.float32, workers: int | None = None):
        if cfg.n_resample != 1:
            raise ValueError("CPUPM does not implement sheet resampling")
        opm.validate(cfg)
        self.cfg = cfg
        self.dt = np.dtype(dtype)
        self.suf = "f32" if self.dt == np.float32 else "f64"
        self.workers = workers or os.cpu_count()
        res, n, L = cfg.res_pm, cfg.n_part, cfg.boxsize
        self.kphi = opm.k_phi(cfg).astype(self.dt)          # [ix,iy,kz], z halved
        if cfg.grad_order == 0:
            K = opm.PMKernels(cfg)
            self.g = [K.gx.astype(np.complex128), K.gy.astype(np.complex128), K.gz.astype(np.complex128)]
        else:
            self.c = tuple(self.dt.type(v) for v in opm.fd_coeffs(cfg.grad_order, L / res))
        self.shifts = opm.aa_shifts(cfg.antialias, 0.5 * L / res)
        q = np.array([i * (L / n) for i in range(n)]).astype(self.dt)
        self.q = (q[:, None, None], q[None, :, None], q[None, None, :])
        self.mesh = np.zeros(res ** 3, dtype=self.dt)
        self.F = np.zeros(3 * res ** 3, dtype=self.dt)

    def _fft(self, mesh_xfast):
        import scipy.fft as sf
        res = self.cfg.res_pm
        logical = mesh_xfast.reshape(res, res, res).T          # [ix,iy,iz] view
        return sf.rfftn(logical, axes=(0, 1, 2), workers=self.workers)

    def _ifft(self, spec):
        import scipy.fft as sf
        res = self.cfg.res_pm
        out = sf.irfftn(spec, s=(res, res, res), axes=(0, 1, 2), workers=self.workers)
        return np.asfortranarray(out, dtype=self.dt) * self.dt.type(res ** 3)  # brfft (unnormalised)

    def acceleration(self, psi):
        cfg = self.cfg
        n, res, W = cfg.n_part, cfg.res_pm, cfg.worder
        L = self.dt.type(cfg.boxsize)
        L_lib = cfg.boxsize
        np_ = n ** 3
        f = getattr(lib(), f"cpm_scatter_{self.suf}")
        g3 = getattr(lib(), f"cpm_gather3_{self.suf}")
        psi = np.asarray(psi, dtype=self.dt)
        X = np.empty((3, n, n, n), dtype=self.dt)  # [c][k][j][i] = component blocks, x fastest
        for c in range(3):
            X[c] = (psi[..., c] + self.q[c]).T
        acc = np.zeros((3, n, n, n), dtype=self.dt)
        Xs = np.empty_like(X)
        for s in self.shifts:
            for c in range(3):
                Xs[c] = X[c] + self.dt.type(s[c])
            self.mesh[:] = 0
            f(_ptr(Xs), np_, res, L, W, _ptr(self.mesh))
            fd = self._fft(self.mesh)
            if cfg.grad_order == 0:
                for ax in range(3):
                    phi = self._ifft(-(self.g[ax] * self.kphi * fd))
                    self.F[ax * res ** 3:(ax + 1) * res ** 3] = phi.reshape(-1, order="F")
            else:
                phi = self._ifft(fd * self.kphi)
                getattr(lib(), f"cpm_fdgrad_{self.suf}")(_ptr(phi), res, *self.c, _ptr(self.F))
            g3(_ptr(self.F), _ptr(Xs), np_, res, L, W, _ptr(acc))
        if len(self.shifts) > 1:
            acc /= self.dt.type(len(self.shifts))
        del L_lib
        return np.moveaxis(acc, 0, -1).transpose(2, 1, 0, 3)  # -> [i,j,k,c]

    def step(self, psi, mom, dd1, alpha, beta, dd2):
        T = self.dt.type
        psi = psi + T(dd1) * mom
        mom = T(alpha) * mom + T(beta) * self.acceleration(psi)
        psi = psi + T(dd2) * mom
        return psi, mom
