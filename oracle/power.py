"""Isotropic power spectrum (float64 shell sums).

Restates `native/DiscoDJNative/src/analysis/power_spectrum.jl:25-79`.
Test infrastructure only (see `oracle/__init__.py`).
"""
from __future__ import annotations

import math

import numpy as np

from .cosmology import _julia_linrange
from .pm import rfftn


def bin_edges(res, boxsize, bins, logarithmic=True):
    """power_spectrum.jl:47-52"""
    dk = 2 * math.pi / boxsize
    k_ny = math.pi * res / boxsize
    k_min, k_max = dk, k_ny * math.sqrt(3)
    if logarithmic:
        return 10.0 ** _julia_linrange(math.log10(k_min), math.log10(k_max), bins + 1)
    return _julia_linrange(k_min, k_max, bins + 1)


def evaluate_power_spectrum(field, boxsize, bins=20, logarithmic=True):
    """power_spectrum.jl:25-79 -> (k, Pk, N_modes). `field` is (res,res,res) [ix,iy,iz]."""
    res = field.shape[0]
    if field.shape != (res, res, res):
        raise ValueError("field must be cubic")
    V = boxsize ** 3
    dk = 2 * math.pi / boxsize
    f = rfftn(np.asarray(field, dtype=np.float64))
    fft_norm = np.abs(f) ** 2 * (V / res ** 6)
    kfull = np.array([i if i <= res // 2 else i - res for i in range(res)]) * dk
    khalf = np.arange(res // 2 + 1) * dk
    k_arr = np.sqrt(kfull[:, None, None] ** 2 + kfull[None, :, None] ** 2 + khalf[None, None, :] ** 2)
    edges = bin_edges(res, boxsize, bins, logarithmic)
    w = np.ones((res, res, res // 2 + 1))
    w[:, :, 0] = 0.5
    w[:, :, -1] = 0.5
    k_cen = np.empty(bins)
    pk = np.empty(bins)
    nm = np.empty(bins, dtype=np.int64)
    for b in range(bins):
        lo, hi = edges[b], edges[b + 1]
        mask = (k_arr >= lo) & (k_arr < hi)
        n_k = int(mask.sum())
        if n_k == 0:
            k_cen[b] = math.sqrt(lo * hi)
            pk[b] = 0.0
            nm[b] = 0
        else:
            k_cen[b] = k_arr[mask].sum() / n_k
            pk[b] = (fft_norm[mask] * w[mask]).sum() / w[mask].sum()
            nm[b] = n_k
    return k_cen, pk, nm


def density_contrast(mesh, n_part):
    """δ = mesh·res³/n³ − 1 for a CIC mesh of unit masses (the P(k) measurement of
    `studies/eft_shell_crossing/src/measure.jl:430-447`)."""
    res = mesh.shape[0]
    return mesh * (res ** 3 / n_part ** 3) - 1.0
