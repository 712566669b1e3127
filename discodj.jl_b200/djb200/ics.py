"""Initial conditions for the PM step (input generation, not the hot path).

Restates, with torch FFTs so it runs on the GPU or the CPU:
* the Eisenstein & Hu (1998) transfer function and σ8-normalised linear P(k)
  (native/DiscoDJNative/src/cosmology/transfer.jl:24-77,121-153),
* the IC map φ(k) = rfft(ω)·(−√(P·(res/L)³)/k²) (src/ics/grf.jl:118-144,218-240),
* EdS nLPT displacement shapes ψ₁..ψ₃ from φ with 3/2-rule de-aliasing
  (`compute_core`, src/lpt/nlpt_core.jl:44-311),
* Ψ, Π = dΨ/dD at a (`nbody_ics_lpt`, src/nbody/run_nbody.jl:180-208).

White noise is a seeded standard-normal field from torch's generator; the
reference's bit-exact N-GenIC/GSL noise is not restated (the PM step takes the
resulting displacements as input, and the oracle receives the same ones).
Arrays are logical [i,j,k] (real) and [i,j,kz] with the z axis halved (spectra);
particle fields are (n,n,n,3) [i,j,k,c].
"""
from __future__ import annotations

import math

import numpy as np
import torch

# ── linear power spectrum (host float64) ──────────────────────────────────────


def eisenstein_hu(p: dict, k: np.ndarray, Tcmb: float = 2.72548) -> np.ndarray:
    """transfer.jl:24-77: EH98 transfer function with baryons, k in h/Mpc."""
    Om = p["Omega_c"] + p["Omega_b"]
    h = p["h"]
    th = Tcmb / 2.7
    th2 = th * th
    th4 = th2 * th2
    omh2 = Om * h * h
    f_b = p["Omega_b"] / Om
    obh2 = omh2 * f_b
    z_eq = 2.50e4 * omh2 / th4
    k_eq = 0.0746 * omh2 / th2 / h
    z_d1 = 0.313 * omh2 ** (-0.419) * (1 + 0.607 * omh2 ** 0.674)
    z_d2 = 0.238 * omh2 ** 0.223
    z_d = 1291.0 * omh2 ** 0.251 / (1 + 0.659 * omh2 ** 0.828) * (1 + z_d1 * obh2 ** z_d2)
    R_d = 31.5 * obh2 / th4 * (1000 / (1 + z_d))
    R_eq = 31.5 * obh2 / th4 * (1000 / z_eq)
    s = 2 / 3 / k_eq * math.sqrt(6 / R_eq) * math.log(
        (math.sqrt(1 + R_d) + math.sqrt(R_d + R_eq)) / (1 + math.sqrt(R_eq)))
    k_silk = 1.6 * obh2 ** 0.52 * omh2 ** 0.73 * (1 + (10.4 * omh2) ** (-0.95)) / h
    a1 = (46.9 * omh2) ** 0.670 * (1 + (32.1 * omh2) ** (-0.532))
    a2 = (12.0 * omh2) ** 0.424 * (1 + (45.0 * omh2) ** (-0.582))
    alpha_c = a1 ** (-f_b) * a2 ** (-f_b ** 3)
    b1 = 0.944 / (1 + (458 * omh2) ** (-0.708))
    b2 = (0.395 * omh2) ** (-0.0266)
    beta_c = 1 / (1 + b1 * ((1 - f_b) ** b2 - 1))
    yG = (1 + z_eq) / (1 + z_d)
    Gy = yG * (-6 * math.sqrt(1 + yG) + (2 + 3 * yG) * math.log((math.sqrt(1 + yG) + 1) / (math.sqrt(1 + yG) - 1)))
    alpha_b = 2.07 * k_eq * s * (1 + R_d) ** (-0.75) * Gy
    beta_b = 0.5 + f_b + (3 - 2 * f_b) * math.sqrt((17.2 * omh2) ** 2 + 1)
    beta_node = 8.41 * omh2 ** 0.435
    kk = np.asarray(k, dtype=np.float64)
    q = kk / (13.41 * k_eq)
    ks = kk * s
    Cf = lambda ac: 14.2 / ac + 386 / (1 + 69.9 * q ** 1.08)
    lt = lambda b: np.log(math.e + 1.8 * b * q)
    T0t = lambda ac, bc: lt(bc) / (lt(bc) + Cf(ac) * q ** 2)
    f = 1 / (1 + (ks / 5.4) ** 4)
    T_c = f * T0t(1.0, beta_c) + (1 - f) * T0t(alpha_c, beta_c)
    s_tilde = s / (1 + (beta_node / ks) ** 3) ** (1 / 3)
    Tb1 = T0t(1.0, 1.0) / (1 + (ks / 5.2) ** 2)
    Tb2 = alpha_b / (1 + (beta_b / ks) ** 3) * np.exp(-(kk / k_silk) ** 1.4)
    T_b = np.sinc(kk * s_tilde / math.pi) * (Tb1 + Tb2)
    return f_b * T_b + (1 - f_b) * T_c


def _julia_linrange(a, b, n):
    j = np.arange(n, dtype=np.float64)
    t = j / (n - 1)
    out = (1 - t) * a + t * b
    out[0], out[-1] = a, b
    return out


def linear_power_spectrum(p: dict, kmin=1e-4, kmax=50.0, n_modes=512):
    """transfer.jl:121-153: P(k) = k^n_s T(k)², σ8-normalised (trapezoid in ln k)."""
    k = 10.0 ** _julia_linrange(math.log10(kmin), math.log10(kmax), n_modes)
    Tk = eisenstein_hu(p, k)
    Pk = k ** p["n_s"] * Tk ** 2
    x = k * 8.0
    W = 3 * (np.sin(x) - x * np.cos(x)) / x ** 3
    integrand = k ** 3 * Pk * W ** 2
    logk = np.log(k)
    s8sq = np.sum(0.5 * (integrand[:-1] + integrand[1:]) * np.diff(logk)) / (2 * math.pi ** 2)
    return k, Pk * (p["sigma8"] ** 2 / s8sq)


# ── Fourier grids ──────────────────────────────────────────────────────────────
def _kfull(n, L, dev, dt):
    dk = 2 * math.pi / L
    m = torch.arange(n, device=dev, dtype=dt)
    return torch.where(m < n // 2, m, m - n) * dk


def _khalf(n, L, dev, dt):
    return torch.arange(n // 2 + 1, device=dev, dtype=dt) * (2 * math.pi / L)


def _grad_kernels(n, L, dev, dt):
    """nlpt_core.jl:56-67: i·k per axis, Nyquist zeroed; broadcastable to (n,n,n//2+1)."""
    cdt = torch.complex128 if dt == torch.float64 else torch.complex64
    kf = _kfull(n, L, dev, dt).clone()
    kf[n // 2] = 0
    kh = _khalf(n, L, dev, dt).clone()
    kh[-1] = 0
    return ((1j * kf.to(cdt)).reshape(n, 1, 1), (1j * kf.to(cdt)).reshape(1, n, 1),
            (1j * kh.to(cdt)).reshape(1, 1, n // 2 + 1))


def _inv_lap(n, L, dev, dt):
    """nlpt_core.jl:71-78: −1/k² with the DC entry finite."""
    kx = _kfull(n, L, dev, dt).reshape(n, 1, 1)
    ky = _kfull(n, L, dev, dt).reshape(1, n, 1)
    kz = _khalf(n, L, dev, dt).reshape(1, 1, n // 2 + 1)
    k2 = kx ** 2 + ky ** 2 + kz ** 2
    k2[0, 0, 0] = 1
    return -1.0 / k2


def white_noise(seed: int, n: int, device="cpu", dtype=torch.float64):
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    return torch.randn((n, n, n), generator=g, device=device, dtype=dtype)


def white_noise_to_fphi(white, boxsize: float, pk_table):
    """grf.jl:118-144: φ(k) = rfft(ω)·(−√(P(k)·(res/L)³)/k²), 0 at k = 0 (P by np.interp)."""
    n = white.shape[0]
    dev, dt = white.device, white.dtype
    k_tab, P_tab = pk_table
    kx = (torch.arange(n, dtype=torch.float64) - n * (torch.arange(n) > n // 2)).reshape(n, 1, 1)
    kz = torch.arange(n // 2 + 1, dtype=torch.float64).reshape(1, 1, n // 2 + 1)
    dk = 2 * math.pi / boxsize
    k2 = (kx * dk) ** 2 + (kx.reshape(1, n, 1) * dk) ** 2 + (kz * dk) ** 2
    kk = torch.sqrt(k2)
    P = torch.from_numpy(np.interp(kk.numpy().ravel(), k_tab, P_tab).reshape(kk.shape))
    scale = torch.where(k2 == 0, torch.zeros_like(k2), -torch.sqrt(P * (n / boxsize) ** 3) / torch.where(k2 == 0, torch.ones_like(k2), k2))
    return torch.fft.rfftn(white, dim=(0, 1, 2)) * scale.to(dev, dt)


# ── de-aliased nLPT (nlpt_core.jl:95-311) ────────────────────────────────────
class _K:
    def __init__(self, n, L, dev, dt):
        self.n, self.ext = n, 3 * n // 2
        self.d = _grad_kernels(n, L, dev, dt)
        self.il = _inv_lap(n, L, dev, dt)
        self.de = _grad_kernels(self.ext, L, dev, dt)


def _pad3(ff, orig, ext):
    """nlpt_core.jl:132-142: embed the (orig) half spectrum in the (ext) one, Nyquist planes dropped."""
    h = orig // 2
    out = torch.zeros((ext, ext, ext // 2 + 1), dtype=ff.dtype, device=ff.device)
    lo, hs, hd = slice(0, h), slice(h + 1, orig), slice(ext - h + 1, ext)
    for xs, xd in ((lo, lo), (hs, hd)):
        for ys, yd in ((lo, lo), (hs, hd)):
            out[xd, yd, :h] = ff[xs, ys, :h]
    return out * ((ext / orig) ** 3)


def _crop3(ff, orig, ext):
    """nlpt_core.jl:146-156"""
    h = orig // 2
    out = torch.zeros((orig, orig, orig // 2 + 1), dtype=ff.dtype, device=ff.device)
    lo, hs, hd = slice(0, h), slice(ext - h + 1, ext), slice(h + 1, orig)
    for xs, xd in ((lo, lo), (hs, hd)):
        for ys, yd in ((lo, lo), (hs, hd)):
            out[xd, yd, :h] = ff[xs, ys, :h]
    return out * ((orig / ext) ** 3)


def _conv2(a, b, K: _K, crop=True):
    """nlpt_core.jl:174-179: rfft(irfft(a)·irfft(b)) on the extended grid."""
    e = K.ext
    prod = torch.fft.irfftn(a, s=(e, e, e), dim=(0, 1, 2)) * torch.fft.irfftn(b, s=(e, e, e), dim=(0, 1, 2))
    f = torch.fft.rfftn(prod, dim=(0, 1, 2))
    return _crop3(f, K.n, e) if crop else f


def _dext(K: _K, X, m, axis):
    """nlpt_core.jl:183-186 (1-based component m and axis)."""
    return K.de[axis - 1] * _pad3(X[m - 1], K.n, K.ext)


_MU2_SYM = ((1, 2, 1, 2, 1), (1, 3, 1, 3, 1), (2, 3, 2, 3, 1), (1, 2, 2, 1, -1), (1, 3, 3, 1, -1), (2, 3, 3, 2, -1))
_MU2_I = (1, 1, 2, 3, 2, 2, 3, 1, 3, 3, 1, 2)
_MU2_J = (2, 3, 1, 1, 3, 1, 2, 2, 1, 2, 3, 3)
_MU2_K = (1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3)
_MU2_L = (2, 3, 2, 3, 3, 1, 3, 1, 1, 2, 1, 2)
_MU2_S = (1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1)
_C_I = (1, 1, 2, 2, 3, 3)
_C_J = (1, 1, 2, 2, 3, 3)
_C_K = (2, 3, 2, 3, 2, 3)
_C_L = (3, 2, 3, 2, 3, 2)
_C_S = (1, -1, 1, -1, 1, -1)
_MU3_K = (1, 1, 2, 2, 3, 3)
_MU3_L = (2, 3, 3, 1, 1, 2)
_MU3_M = (3, 2, 1, 3, 2, 1)
_MU3_S = (1, -1, 1, -1, 1, -1)


def _cyc(x, n):
    return (x - 1 + n) % 3 + 1


def _fmu2_sym(K, f1):
    """nlpt_core.jl:195-204"""
    acc = 0
    for i, j, k, l, s in _MU2_SYM:
        acc = acc + s * _conv2(_dext(K, f1, i, k), _dext(K, f1, j, l), K)
    return acc


def _fmu2_and_C(K, f1, f2):
    """nlpt_core.jl:223-245"""
    mu2 = 0
    for t in range(12):
        mu2 = mu2 + _MU2_S[t] * _conv2(_dext(K, f1, _MU2_I[t], _MU2_K[t]), _dext(K, f2, _MU2_J[t], _MU2_L[t]), K)
    C = []
    for shift in range(3):
        acc = 0
        for t in range(6):
            i, j = _cyc(_C_I[t], shift), _cyc(_C_J[t], shift)
            k, l = _cyc(_C_K[t], shift), _cyc(_C_L[t], shift)
            acc = acc + _C_S[t] * _conv2(_dext(K, f1, i, k), _dext(K, f2, j, l), K)
        C.append(acc)
    return mu2, C


def _fmu3(K, f1, f2, f3):
    """nlpt_core.jl:251-263"""
    acc = 0
    for t in range(6):
        termA = _dext(K, f1, 1, _MU3_K[t])
        inner = _conv2(_dext(K, f2, 2, _MU3_L[t]), _dext(K, f3, 3, _MU3_M[t]), K, crop=False)
        acc = acc + _MU3_S[t] * _conv2(termA, inner, K)
    return acc


def _assemble(K, fL, fT):
    """nlpt_core.jl:267-280"""
    dx, dy, dz = K.d
    il = K.il
    if fT is None:
        return [il * (dx * fL), il * (dy * fL), il * (dz * fL)]
    Cx, Cy, Cz = fT
    return [il * (dx * fL - (dy * Cz - dz * Cy)), il * (dy * fL - (dz * Cx - dx * Cz)),
            il * (dz * fL - (dx * Cy - dy * Cx))]


def compute_core(fphi, boxsize: float, n_order: int = 2):
    """nlpt_core.jl:311-365 (EdS growth, longitudinal + transverse, de-aliased).
    Returns {"psi_1": (n,n,n,3), ...} real fields in fphi's real dtype and device."""
    n = fphi.shape[0]
    dt = torch.float64 if fphi.dtype == torch.complex128 else torch.float32
    K = _K(n, boxsize, fphi.device, dt)
    dx, dy, dz = K.d
    psi = [[-(dx * fphi), -(dy * fphi), -(dz * fphi)]]
    for i in range(2, n_order + 1):
        fL = 0
        fT = None
        if i % 2 == 0:
            h = i // 2
            fac = ((3 - i) / 2 - h ** 2 - h ** 2) / ((i + 1.5) * (i - 1))
            fL = fL + fac * _fmu2_sym(K, psi[h - 1])
        if i > 2:
            fT = [0, 0, 0]
            for j in range(1, (i + 1) // 2):
                imj = i - j
                fac_mu2 = ((3 - i) / 2 - j ** 2 - imj ** 2) / ((i + 1.5) * (i - 1))
                fac_C = 1 - 2 * j / i
                mu2, C = _fmu2_and_C(K, psi[j - 1], psi[imj - 1])
                fL = fL + fac_mu2 * mu2
                fT = [fT[c] + fac_C * C[c] for c in range(3)]
            for k in range(1, i - 1):
                for l in range(1, i - k):
                    m = i - k - l
                    fac = ((3 - i) / 2 - k ** 2 - l ** 2 - m ** 2) / ((i + 1.5) * (i - 1))
                    fL = fL + fac * _fmu3(K, psi[k - 1], psi[l - 1], psi[m - 1])
            fT = [t if torch.is_tensor(t) else torch.zeros_like(fphi) for t in fT]
        psi.append(_assemble(K, fL, fT))
    out = {}
    for i, comps in enumerate(psi, start=1):
        out[f"psi_{i}"] = torch.stack([torch.fft.irfftn(c, s=(n, n, n), dim=(0, 1, 2)) for c in comps], dim=-1)
    return out


def lpt_ics(cosmo, n: int, boxsize: float, a: float, *, n_order: int = 2, seed: int = 42,
            device="cpu", dtype=torch.float64, white=None):
    """White noise -> φ -> nLPT shapes -> (Ψ, Π = dΨ/dD) at a, as (n,n,n,3) tensors on `device`."""
    p = cosmo.params
    pk = linear_power_spectrum(p)
    w = white if white is not None else white_noise(seed, n, device=device, dtype=dtype)
    fphi = white_noise_to_fphi(w.to(device, dtype), boxsize, pk)
    shapes = compute_core(fphi, boxsize, n_order=n_order)
    D = cosmo.Dplus(a)
    Psi = torch.zeros_like(shapes["psi_1"])
    Pi = torch.zeros_like(Psi)
    for m in range(1, n_order + 1):
        Psi += (D ** m) * shapes[f"psi_{m}"]
        Pi += (m * D ** (m - 1)) * shapes[f"psi_{m}"]
    return Psi, Pi


def lpt_ics_native(cosmo, n: int, boxsize: float, a: float, *, n_order: int = 2, seed: int = 42, white=None,
                   device: int = 0):
    """nLPT (Ψ, Π = dΨ/dD) at scale factor a from the library's CUDA kernels
    (`djb_lpt_ics`, n_order 2 or 3): the same white noise → φ → ψ₁, ψ₂ (, ψ₃) chain as
    `lpt_ics(n_order=...)`, with the fields and products in float32 on the GPU. `white`:
    (n,n,n) [i,j,k] tensor (default: `white_noise(seed, n)` on the device). Returns native
    (3,n,n,n) float32 device tensors (the library's particle layout, `pm.native_view`)."""
    import ctypes as C

    from . import _lib
    dev = f"cuda:{device}"
    w = white if white is not None else white_noise(seed, n, device=dev, dtype=torch.float32)
    w_native = w.to(dev, torch.float32).permute(2, 1, 0).contiguous()   # x fastest
    k_tab, p_tab = linear_power_spectrum(cosmo.params)
    k_tab = np.ascontiguousarray(k_tab, dtype=np.float64)
    p_tab = np.ascontiguousarray(p_tab, dtype=np.float64)
    psi = torch.empty((3, n, n, n), dtype=torch.float32, device=dev)
    pi = torch.empty_like(psi)
    nb = np.zeros(1, dtype=np.int64)
    _lib.check(_lib.lib.djb_lpt_ics_work_bytes(int(n), int(n_order), len(k_tab), _lib.i64ptr(nb)))
    work = torch.empty(int(nb[0]), dtype=torch.uint8, device=dev)   # torch's cache keeps it between calls
    stream = torch.cuda.current_stream(dev).cuda_stream
    _lib.check(_lib.lib.djb_lpt_ics(C.c_void_p(w_native.data_ptr()), int(n), float(boxsize), _lib.dptr(k_tab),
                                    _lib.dptr(p_tab), len(k_tab), int(n_order), float(cosmo.Dplus(a)),
                                    C.c_void_p(psi.data_ptr()), C.c_void_p(pi.data_ptr()),
                                    C.c_void_p(work.data_ptr()), int(nb[0]), int(device), C.c_void_p(stream)))
    del work
    return psi, pi


def lpt2_ics_native(cosmo, n: int, boxsize: float, a: float, *, seed: int = 42, white=None, device: int = 0):
    """`lpt_ics_native` at n_order = 2 (`djb_lpt2_ics`)."""
    return lpt_ics_native(cosmo, n, boxsize, a, n_order=2, seed=seed, white=white, device=device)
