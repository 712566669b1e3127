"""Particle-mesh acceleration (float64 numpy), every option of `PMConfig`.

Restates `native/DiscoDJNative/src/nbody/pm.jl`. The main entry point,
`pm_acceleration`, follows the straightforward transcription
`pm_acceleration_reference` (pm.jl:253-298): one inverse FFT per force component,
gradient kernels applied in Fourier space. The CUDA library instead applies the
finite-difference gradient as a real-space stencil on the potential (pm.jl:330-342),
which equals the Fourier kernel exactly (circulant identity, pm.jl:309-311), so
comparing the two is a real check of that identity.

Layouts: particle arrays (n,n,n,3) indexed [i,j,k,c]; meshes (res,res,res)
indexed [ix,iy,iz]; half spectra (res,res,res//2+1) with the z axis halved, the
reference's `rfft(x, [3,1,2])` convention (numpy `rfftn(axes=(0,1,2))`).
Test infrastructure only (see `oracle/__init__.py`).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

try:  # scipy's pocketfft with threads when available; numpy otherwise
    import scipy.fft as _fft

    def rfftn(x):
        return _fft.rfftn(x, axes=(0, 1, 2), workers=-1)

    def irfftn(f, n):
        return _fft.irfftn(f, s=(n, n, n), axes=(0, 1, 2), workers=-1)
except ImportError:  # pragma: no cover
    def rfftn(x):
        return np.fft.rfftn(x, axes=(0, 1, 2))

    def irfftn(f, n):
        return np.fft.irfftn(f, s=(n, n, n), axes=(0, 1, 2))


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


# ── mass-assignment kernels, pm.jl:49-55 ──────────────────────────────────────
def wk(W: int, d):
    d = np.asarray(d)
    if W == 2:
        return np.where(d > 1, 0.0, 1 - d)
    if W == 3:
        return np.where(d > 1.5, 0.0, np.where(d > 0.5, 0.5 * (1.5 - d) ** 2, 0.75 - d ** 2))
    if W == 4:
        return np.where(d > 2, 0.0, np.where(d > 1, (2 - d) ** 3 / 6, (4 - 6 * d ** 2 + 3 * d ** 3) / 6))
    raise ValueError("worder must be 2, 3 or 4")


def wbase(W: int, g):
    """Even orders floor, odd orders round half to even (Julia `round`)."""
    return (np.floor(g) if W % 2 == 0 else np.rint(g)).astype(np.int64)


def woffsets(W: int):
    return {2: range(0, 2), 3: range(-1, 2), 4: range(-1, 3)}[W]


def _grid_coords(X, res, L):
    """pm.jl:61: g = mod(X, L)/L·res (Julia `mod` == numpy `mod` for floats)."""
    L = float(L)
    return [np.mod(X[:, c], L) / L * res for c in range(3)]


def pm_scatter(mesh, X, res, L, W):
    """pm.jl:57-74,102-106: mesh[node] += Π w over the W³ nodes (unit masses)."""
    gx, gy, gz = _grid_coords(X, res, L)
    bx, by, bz = wbase(W, gx), wbase(W, gy), wbase(W, gz)
    flat = mesh.reshape(-1)
    for oz in woffsets(W):
        wz = wk(W, np.abs(gz - (bz + oz)))
        kz = np.mod(bz + oz, res)
        for oy in woffsets(W):
            wy = wk(W, np.abs(gy - (by + oy)))
            ky = np.mod(by + oy, res)
            for ox in woffsets(W):
                wx = wk(W, np.abs(gx - (bx + ox)))
                kx = np.mod(bx + ox, res)
                idx = (kx * res + ky) * res + kz
                flat += np.bincount(idx, weights=wx * wy * wz, minlength=res ** 3)
    return mesh


def pm_gather(mesh, X, res, L, W):
    """pm.jl:76-95,109-114: Σ w·mesh[node] at each particle."""
    gx, gy, gz = _grid_coords(X, res, L)
    bx, by, bz = wbase(W, gx), wbase(W, gy), wbase(W, gz)
    s = np.zeros(X.shape[0])
    for oz in woffsets(W):
        wz = wk(W, np.abs(gz - (bz + oz)))
        kz = np.mod(bz + oz, res)
        for oy in woffsets(W):
            wy = wk(W, np.abs(gy - (by + oy)))
            ky = np.mod(by + oy, res)
            for ox in woffsets(W):
                wx = wk(W, np.abs(gx - (bx + ox)))
                kx = np.mod(bx + ox, res)
                s += mesh[kx, ky, kz] * (wx * wy * wz)
    return s


# ── Fourier kernels, pm.jl:119-183 ────────────────────────────────────────────
def pm_kvecs(res, L):
    """pm.jl:119-123 (full axis: index res/2 holds −res/2)."""
    kf = np.array([(m if m < res // 2 else m - res) * 2 * math.pi / L for m in range(res)])
    kh = np.array([m * 2 * math.pi / L for m in range(res // 2 + 1)])
    return kf, kh


def grad1d(k, order, half):
    """pm.jl:125-138"""
    if order == 0:
        g = 1j * k
        if half:
            g[-1] = 0
        else:
            g[len(k) // 2] = 0
        return g
    m = np.max(np.abs(k)) / math.pi
    s = lambda j: np.sin(j * k / m)
    if order == 2:
        kern = s(1)
    elif order == 4:
        kern = (8 * s(1) - s(2)) / 6
    elif order == 6:
        kern = (45 * s(1) - 9 * s(2) + s(3)) / 30
    else:
        raise ValueError("grad_order must be 0, 2, 4 or 6")
    return 1j * m * kern


def invlap1d_terms(k, order):
    """pm.jl:140-147"""
    m = np.max(np.abs(k)) / math.pi
    c = lambda j: np.cos(j * k / m)
    if order == 2:
        return -2 * (1 - c(1)) * m ** 2
    if order == 4:
        return -(c(2) - 16 * c(1) + 15) / 6 * m ** 2
    if order == 6:
        return -(-2 * c(3) + 27 * c(2) - 270 * c(1) + 245) / 90 * m ** 2
    raise ValueError("lap_order must be 0, 2, 4 or 6")


def invmak1d(k, worder):
    """pm.jl:150-151: sinc(π x)^(−2·worder), x = k/(2π m), DC 1."""
    m = np.max(np.abs(k)) / math.pi
    x = k / (2 * math.pi) / m
    out = np.ones_like(x)
    nz = x != 0
    out[nz] = np.sin(math.pi * x[nz]) / (math.pi * x[nz])
    return out ** (-2 * worder)


class PMKernels:
    """pm.jl:153-183"""

    def __init__(self, cfg: PMConfig):
        res = cfg.res_pm
        kf, kh = pm_kvecs(res, cfg.boxsize)
        self.gx = grad1d(kf, cfg.grad_order, False)[:, None, None]
        self.gy = grad1d(kf, cfg.grad_order, False)[None, :, None]
        self.gz = grad1d(kh, cfg.grad_order, True)[None, None, :]
        KX, KY, KZ = kf[:, None, None], kf[None, :, None], kh[None, None, :]
        if cfg.lap_order == 0:
            k2 = KX ** 2 + KY ** 2 + KZ ** 2
            k2[0, 0, 0] = 1.0
            il = -1.0 / k2
            il[0, 0, 0] = 0.0
        else:
            inv = (invlap1d_terms(kf, cfg.lap_order)[:, None, None]
                   + invlap1d_terms(kf, cfg.lap_order)[None, :, None]
                   + invlap1d_terms(kh, cfg.lap_order)[None, None, :])
            inv[0, 0, 0] = -1.0
            il = 1.0 / inv
        self.invlap = il
        self.mak = None
        if cfg.deconvolve:
            self.mak = (invmak1d(kf, cfg.worder)[:, None, None] * invmak1d(kf, cfg.worder)[None, :, None]
                        * invmak1d(kh, cfg.worder)[None, None, :])


# ── sheet resampling, pm.jl:186-234 ───────────────────────────────────────────
def _lagr1d(n, L):
    return np.array([i * (L / n) for i in range(n)])


def _trilinear_shift(f, d):
    """pm.jl:220-231 periodic trilinear interpolation at (i+d1, j+d2, k+d3)."""
    dx, dy, dz = d
    r = lambda a, ax: np.roll(a, -1, axis=ax)
    f1 = r(f, 0)
    f2 = r(f, 1)
    f3 = r(f, 2)
    f12 = r(f1, 1)
    f13 = r(f1, 2)
    f23 = r(f2, 2)
    f123 = r(f12, 2)
    return (f * (1 - dx) * (1 - dy) * (1 - dz) + f1 * dx * (1 - dy) * (1 - dz)
            + f2 * (1 - dx) * dy * (1 - dz) + f3 * (1 - dx) * (1 - dy) * dz
            + f12 * dx * dy * (1 - dz) + f13 * dx * (1 - dy) * dz
            + f23 * (1 - dx) * dy * dz + f123 * dx * dy * dz)


def resample_shifts(nr):
    """pm.jl:233-234 (last coordinate fastest; the zero offset dropped)."""
    if nr == 1:
        return []
    v = [i / nr for i in range(nr)]
    return [(a, b, c) for a in v for b in v for c in v][1:]


def aa_shifts(aa, dhalf):
    """pm.jl:237-246 interlacing shift list."""
    if aa == 0:
        return [(0.0, 0.0, 0.0)]
    if aa == -1:
        return [(dhalf, dhalf, dhalf)]
    base = [(a, b, c) for a in (0.0, dhalf) for b in (0.0, dhalf) for c in (0.0, dhalf)]
    if aa == 1:
        return [(0.0, 0.0, 0.0), (dhalf, dhalf, dhalf)]
    if aa == 2:
        return base
    q = dhalf / 2
    if aa == 3:
        return base + [(a, b, c) for a in (-q, q) for b in (-q, q) for c in (-q, q)]
    raise ValueError("antialias must be -1, 0, 1, 2 or 3")


def spawn(X4, d, cfg: PMConfig):
    """pm.jl:189-217: resampled positions at Lagrangian offset d (cells), wrapped to [0, L)."""
    n = X4.shape[0]
    L = float(cfg.boxsize)
    q1 = _lagr1d(n, cfg.boxsize)
    qs = (q1[:, None, None], q1[None, :, None], q1[None, None, :])
    out = np.empty_like(X4)
    if cfg.resampling == "fourier":
        mf = np.array([(m if m < n // 2 else m - n) / n for m in range(n)])
        mh = np.array([m / n for m in range(n // 2 + 1)])
        kd = mf[:, None, None] * d[0] + mf[None, :, None] * d[1] + mh[None, None, :] * d[2]
        ph = np.exp(1j * 2 * math.pi * kd)
        for c in range(3):
            psi = np.mod(X4[..., c] - qs[c] + L / 2, L) - L / 2
            npsi = irfftn(rfftn(psi) * ph, n)
            out[..., c] = np.mod(qs[c] + npsi + d[c] * cfg.boxsize / n + L, L)
    elif cfg.resampling == "linear":
        for c in range(3):
            psi = np.mod(X4[..., c] - qs[c] + L / 2, L) - L / 2
            npsi = _trilinear_shift(psi, d)
            out[..., c] = np.mod(qs[c] + npsi + d[c] * cfg.boxsize / n + L, L)
    else:
        raise ValueError("resampling must be :fourier or :linear")
    return out


def validate(cfg: PMConfig):
    """The option checks the reference raises on (pm.jl:136,146,214,245,423)."""
    if cfg.worder not in (2, 3, 4):
        raise ValueError("worder must be 2, 3 or 4")
    if cfg.grad_order not in (0, 2, 4, 6):
        raise ValueError("grad_order must be 0, 2, 4 or 6")
    if cfg.lap_order not in (0, 2, 4, 6):
        raise ValueError("lap_order must be 0, 2, 4 or 6")
    if cfg.antialias not in (-1, 0, 1, 2, 3):
        raise ValueError("antialias must be -1, 0, 1, 2 or 3")
    if cfg.resampling not in ("fourier", "linear"):
        raise ValueError("resampling must be :fourier or :linear")


def _acc_pm_single(X4, cfg: PMConfig, K: PMKernels):
    """pm.jl:273-298"""
    n = cfg.n_part
    res = cfg.res_pm
    L = cfg.boxsize
    W = cfg.worder
    Xf = X4.reshape(n ** 3, 3)
    mesh = np.zeros((res, res, res))
    rhomean = n ** 3 / res ** 3
    pm_scatter(mesh, Xf, res, L, W)
    delta = mesh / rhomean - 1.0
    if cfg.n_resample > 1:
        for d in resample_shifts(cfg.n_resample):
            m2 = np.zeros_like(mesh)
            pm_scatter(m2, spawn(X4, d, cfg).reshape(n ** 3, 3), res, L, W)
            delta += m2 / rhomean - 1.0
        delta /= cfg.n_resample ** 3
    fd = rfftn(delta)
    if K.mak is not None:
        fd *= K.mak
    fd[0, 0, 0] = 0
    acc = np.empty_like(X4)
    for c, g in enumerate((K.gx, K.gy, K.gz)):
        fa = -(g * K.invlap * fd)
        field = irfftn(fa, res)
        acc[..., c] = pm_gather(field, Xf, res, L, W).reshape(n, n, n)
    return acc


def pm_acceleration(cfg: PMConfig, psi):
    """pm.jl:253-271 `pm_acceleration_reference`: −∇φ at X = q + ψ (∇²φ = δ)."""
    validate(cfg)
    n = cfg.n_part
    if psi.shape[0] != n:
        raise ValueError("psi does not match n_part")
    L = cfg.boxsize
    res = cfg.res_pm
    K = PMKernels(cfg)
    q1 = _lagr1d(n, L)
    X = np.empty_like(psi, dtype=np.float64)
    X[..., 0] = psi[..., 0] + q1[:, None, None]
    X[..., 1] = psi[..., 1] + q1[None, :, None]
    X[..., 2] = psi[..., 2] + q1[None, None, :]
    shifts = aa_shifts(cfg.antialias, 0.5 * L / res)
    acc = np.zeros_like(X)
    for s in shifts:
        Xs = X + np.asarray(s)[None, None, None, :]
        acc += _acc_pm_single(Xs, cfg, K)
    if len(shifts) > 1:
        acc /= len(shifts)
    return acc


# ── optimised-solver building blocks (pm.jl:386-424) ─────────────────────────
def fd_coeffs(order, h):
    """pm.jl:419-424"""
    if order == 2:
        return (1 / (2 * h), 0.0, 0.0)
    if order == 4:
        return (8 / (12 * h), -1 / (12 * h), 0.0)
    if order == 6:
        return (45 / (60 * h), -9 / (60 * h), 1 / (60 * h))
    raise ValueError("grad_order must be 0, 2, 4 or 6")


def k_phi(cfg: PMConfig):
    """pm.jl:389-391 combined multiplier Kφ = invlap·mak/(ρ̄·n_sets·res³), DC 0."""
    K = PMKernels(cfg)
    res, n = cfg.res_pm, cfg.n_part
    kp = K.invlap * (1.0 if K.mak is None else K.mak) / (n ** 3 / res ** 3) / (cfg.n_resample ** 3) / res ** 3
    kp[0, 0, 0] = 0.0
    return kp


def potential(cfg: PMConfig, X4):
    """Unnormalised potential mesh φ = brfft(Kφ·rfft(mesh)) of one shift (pm.jl:494-495)."""
    n, res = cfg.n_part, cfg.res_pm
    mesh = np.zeros((res, res, res))
    pm_scatter(mesh, X4.reshape(n ** 3, 3), res, cfg.boxsize, cfg.worder)
    return irfftn(rfftn(mesh) * k_phi(cfg), res) * res ** 3
