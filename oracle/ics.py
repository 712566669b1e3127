"""Initial conditions for the CPU side: seeded white noise -> EH98 linear P(k) -> φ(k)
-> Zel'dovich (1LPT) displacements, in numpy float64.

TEST INFRASTRUCTURE ONLY (see `oracle/__init__.py`). bench.py's reference arm and CPU
baseline take their particle state from here, so that neither loads the B200
library. Restates:
* the Eisenstein & Hu (1998) transfer function with baryons (astro-ph/9709112,
  eqs. 2-24; the reference's native/DiscoDJNative/src/cosmology/transfer.jl:24-77),
* the σ8-normalised linear spectrum P(k) = k^n_s T(k)^2 (transfer.jl:121-153,
  trapezoid in ln k over 512 log-spaced k from 1e-4 to 50 h/Mpc),
* the IC map φ(k) = rfft(ω)·(−√(P(k)·(res/L)^3)/k^2), zero at k = 0
  (src/ics/grf.jl:118-144),
* the first-order LPT shape ψ₁ = −∇φ with the Nyquist derivative zeroed
  (src/lpt/nlpt_core.jl:56-67), Ψ = D(a)·ψ₁ and Π = dΨ/dD = ψ₁
  (src/nbody/run_nbody.jl:180-208 at n_order = 1),
* the second- and third-order shapes of `compute_core` (src/lpt/nlpt_core.jl:95-311,
  EdS growth) with its 3/2-padded products, written here through the invariants of the
  displacement-gradient matrices A = ∂ψ₁ and B = ∂ψ₂ (μ₂(A,B) = tr A tr B − Σ A_ab B_ab,
  μ₃ = det A, the transverse vector from the antisymmetric part of A·B) rather than the
  reference's index tables, as an independent check of the restatements that use them.
White noise comes from numpy's PCG64 generator (the reference's N-GenIC/GSL noise
is not restated). Particle fields are (n,n,n,3) indexed [i,j,k,c].
"""
from __future__ import annotations

import math

import numpy as np


def eisenstein_hu(Omega_c: float, Omega_b: float, h: float, k: np.ndarray, Tcmb: float = 2.72548) -> np.ndarray:
    """EH98 transfer function (CDM + baryons), k in h/Mpc."""
    Om = Omega_c + Omega_b
    fb = Omega_b / Om
    t27 = Tcmb / 2.7
    w_m = Om * h * h                     # Ω_m h²
    w_b = w_m * fb                       # Ω_b h²
    zeq = 2.50e4 * w_m * t27 ** -4       # eq. 2
    keq = 7.46e-2 * w_m * t27 ** -2      # eq. 3, 1/Mpc
    b1 = 0.313 * w_m ** -0.419 * (1 + 0.607 * w_m ** 0.674)
    b2 = 0.238 * w_m ** 0.223
    zd = 1291 * w_m ** 0.251 / (1 + 0.659 * w_m ** 0.828) * (1 + b1 * w_b ** b2)  # eq. 4
    Rf = lambda z: 31.5 * w_b * t27 ** -4 * (1e3 / z)                              # eq. 5
    Req, Rd = Rf(zeq), Rf(1 + zd)
    s = 2 / (3 * keq) * math.sqrt(6 / Req) * math.log((math.sqrt(1 + Rd) + math.sqrt(Rd + Req)) /
                                                      (1 + math.sqrt(Req)))       # eq. 6
    ksilk = 1.6 * w_b ** 0.52 * w_m ** 0.73 * (1 + (10.4 * w_m) ** -0.95)          # eq. 7
    a1 = (46.9 * w_m) ** 0.670 * (1 + (32.1 * w_m) ** -0.532)
    a2 = (12.0 * w_m) ** 0.424 * (1 + (45.0 * w_m) ** -0.582)
    ac = a1 ** -fb * a2 ** -(fb ** 3)                                              # eq. 11
    bb1 = 0.944 / (1 + (458 * w_m) ** -0.708)
    bb2 = (0.395 * w_m) ** -0.0266
    bc = 1 / (1 + bb1 * ((1 - fb) ** bb2 - 1))                                     # eq. 12
    y = (1 + zeq) / (1 + zd)
    G = y * (-6 * math.sqrt(1 + y) + (2 + 3 * y) * math.log((math.sqrt(1 + y) + 1) / (math.sqrt(1 + y) - 1)))
    ab = 2.07 * keq * s * (1 + Rd) ** -0.75 * G                                    # eq. 14
    bnode = 8.41 * w_m ** 0.435                                                    # eq. 23
    bb = 0.5 + fb + (3 - 2 * fb) * math.sqrt((17.2 * w_m) ** 2 + 1)                # eq. 24
    kM = np.asarray(k, dtype=np.float64) * h                                       # 1/Mpc
    q = kM / (13.41 * keq)                                                         # eq. 10

    def T0(alpha, beta):                                                           # eq. 19-20
        L0 = np.log(math.e + 1.8 * beta * q)
        C = 14.2 / alpha + 386 / (1 + 69.9 * q ** 1.08)
        return L0 / (L0 + C * q * q)

    ks = kM * s
    f = 1 / (1 + (ks / 5.4) ** 4)                                                  # eq. 18
    Tc = f * T0(1, bc) + (1 - f) * T0(ac, bc)                                      # eq. 17
    st = s / (1 + (bnode / ks) ** 3) ** (1 / 3)                                    # eq. 22
    Tb = (T0(1, 1) / (1 + (ks / 5.2) ** 2) + ab / (1 + (bb / ks) ** 3) * np.exp(-(kM / ksilk) ** 1.4)) \
        * np.sinc(kM * st / math.pi)                                               # eq. 21
    return fb * Tb + (1 - fb) * Tc                                                 # eq. 16


def linear_power_spectrum(Omega_c, Omega_b, h, n_s, sigma8, n_modes: int = 512, kmin=1e-4, kmax=50.0):
    """(k, P(k)) with P ∝ k^n_s T², normalised to σ8 with a top hat of 8 Mpc/h."""
    t = np.arange(n_modes, dtype=np.float64) / (n_modes - 1)
    lk = (1 - t) * math.log10(kmin) + t * math.log10(kmax)
    k = 10.0 ** lk
    k[0], k[-1] = kmin, kmax
    P = k ** n_s * eisenstein_hu(Omega_c, Omega_b, h, k) ** 2
    x = 8.0 * k
    w = 3 * (np.sin(x) - x * np.cos(x)) / x ** 3
    y = k ** 3 * P * w * w
    s2 = np.sum(0.5 * (y[1:] + y[:-1]) * np.diff(np.log(k))) / (2 * math.pi ** 2)
    return k, P * sigma8 ** 2 / s2


def fphi_from_white(white: np.ndarray, boxsize: float, pk) -> np.ndarray:
    """φ(k) on the half spectrum [i, j, kz] of a real (n,n,n) white-noise field."""
    n = white.shape[0]
    m = np.fft.fftfreq(n, d=1.0 / n)
    mz = np.arange(n // 2 + 1, dtype=np.float64)
    dk = 2 * math.pi / boxsize
    k2 = (dk * m[:, None, None]) ** 2 + (dk * m[None, :, None]) ** 2 + (dk * mz[None, None, :]) ** 2
    P = np.interp(np.sqrt(k2), pk[0], pk[1])
    with np.errstate(divide="ignore", invalid="ignore"):
        scale = np.where(k2 > 0, -np.sqrt(P * (n / boxsize) ** 3) / k2, 0.0)
    return np.fft.rfftn(white) * scale


def zeldovich_shape(fphi: np.ndarray, boxsize: float) -> np.ndarray:
    """ψ₁ = −∇φ (ik derivative, Nyquist entries zeroed), (n,n,n,3) float64."""
    n = fphi.shape[0]
    dk = 2 * math.pi / boxsize
    kf = np.fft.fftfreq(n, d=1.0 / n) * dk
    kf[n // 2] = 0.0
    kh = np.arange(n // 2 + 1, dtype=np.float64) * dk
    kh[-1] = 0.0
    ks = (kf[:, None, None], kf[None, :, None], kh[None, None, :])
    out = np.empty((n, n, n, 3))
    for c in range(3):
        out[..., c] = np.fft.irfftn(-(1j * ks[c]) * fphi, s=(n, n, n), axes=(0, 1, 2))
    return out


def zeldovich_ics(n: int, boxsize: float, D: float, *, Omega_c, Omega_b, h, n_s, sigma8, seed: int = 42):
    """(Ψ, Π) at growth factor D from 1LPT of seeded white noise, float64 (n,n,n,3)."""
    white = np.random.default_rng(seed).standard_normal((n, n, n))
    pk = linear_power_spectrum(Omega_c, Omega_b, h, n_s, sigma8)
    psi1 = zeldovich_shape(fphi_from_white(white, boxsize, pk), boxsize)
    return D * psi1, psi1


# ── second and third order (compute_core, nlpt_core.jl:95-311) ─────────────────────
def _axes_k(n: int, boxsize: float):
    """ik derivative factors (Nyquist zeroed) of the full, full and half axes, and k²."""
    dk = 2 * math.pi / boxsize
    kf = np.fft.fftfreq(n, d=1.0 / n) * dk
    kh = np.arange(n // 2 + 1, dtype=np.float64) * dk
    k2 = kf[:, None, None] ** 2 + kf[None, :, None] ** 2 + kh[None, None, :] ** 2
    kfz, khz = kf.copy(), kh.copy()
    kfz[n // 2] = 0.0
    khz[-1] = 0.0
    return (kfz[:, None, None], kfz[None, :, None], khz[None, None, :]), k2


def _embed(f: np.ndarray, n: int, e: int) -> np.ndarray:
    """Half spectrum of the n grid into the e grid (Nyquist planes dropped), × (e/n)³."""
    h = n // 2
    out = np.zeros((e, e, e // 2 + 1), dtype=complex)
    src = np.r_[0:h, h + 1:n]
    dst = np.r_[0:h, e - h + 1:e]
    out[np.ix_(dst, dst, np.arange(h))] = f[np.ix_(src, src, np.arange(h))]
    return out * (e / n) ** 3


def _crop(f: np.ndarray, n: int, e: int) -> np.ndarray:
    """The inverse of _embed on the kept modes (× (n/e)³), zero on the Nyquist planes."""
    h = n // 2
    out = np.zeros((n, n, n // 2 + 1), dtype=complex)
    src = np.r_[0:h, e - h + 1:e]
    dst = np.r_[0:h, h + 1:n]
    out[np.ix_(dst, dst, np.arange(h))] = f[np.ix_(src, src, np.arange(h))]
    return out * (n / e) ** 3


def lpt_shapes(fphi: np.ndarray, boxsize: float, order: int = 3):
    """[ψ₁, ψ₂(, ψ₃)] as (n,n,n,3) float64 fields for φ(k) on the half spectrum."""
    n = fphi.shape[0]
    e = 3 * n // 2
    d, k2 = _axes_k(n, boxsize)
    with np.errstate(divide="ignore"):
        il = np.where(k2 > 0, -1.0 / np.where(k2 > 0, k2, 1.0), -1.0)
    real = lambda f: np.fft.irfftn(f, s=(e, e, e), axes=(0, 1, 2))
    spec = lambda x: _crop(np.fft.rfftn(x), n, e)
    psi1 = [-(1j * d[a]) * fphi for a in range(3)]
    # A[a][b] = ∂_b ψ₁_a on the padded grid
    A = [[real(_embed((1j * d[b]) * psi1[a], n, e)) for b in range(3)] for a in range(3)]
    trA = A[0][0] + A[1][1] + A[2][2]
    mu2 = 0.5 * (trA * trA - sum(A[a][b] * A[b][a] for a in range(3) for b in range(3)))
    fl2 = (-3.0 / 7.0) * spec(mu2)
    psi2 = [il * (1j * d[a]) * fl2 for a in range(3)]
    shapes = [psi1, psi2]
    if order >= 3:
        B = [[real(_embed((1j * d[b]) * psi2[a], n, e)) for b in range(3)] for a in range(3)]
        trB = B[0][0] + B[1][1] + B[2][2]
        mu2ab = trA * trB - sum(A[b][a] * B[a][b] for a in range(3) for b in range(3))
        det = (A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0])
               + A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]))
        AB = [[sum(A[i][r] * B[i][c] for i in range(3)) for c in range(3)] for r in range(3)]
        fl3 = spec((-5.0 / 9.0) * mu2ab - (1.0 / 3.0) * det)
        ct = [spec((1.0 / 3.0) * (AB[(c + 1) % 3][(c + 2) % 3] - AB[(c + 2) % 3][(c + 1) % 3])) for c in range(3)]
        psi3 = [il * ((1j * d[a]) * fl3 - ((1j * d[(a + 1) % 3]) * ct[(a + 2) % 3] - (1j * d[(a + 2) % 3]) * ct[(a + 1) % 3]))
                for a in range(3)]
        shapes.append(psi3)
    return [np.stack([np.fft.irfftn(c, s=(n, n, n), axes=(0, 1, 2)) for c in comps], axis=-1) for comps in shapes]
