"""Snapshot files of the particle state, (Psi, Pi = dPsi/dD) as HDF5.

The study driver's `snap_writer` (studies/eft_shell_crossing/scripts/run_jobs.jl:41-48,
called from studies/eft_shell_crossing/src/runners.jl:154-156) writes one file per
snapshot epoch: datasets "Psi" and "Pi", each the (n,n,n,3) Float32 column-major array,
and the float64 root attributes "D" and "L". `write_snapshot` writes the same file from
host arrays through `djb_write_snapshot_h5`; `PMSolver.write_snapshot` writes it from the
resident device state. h5py is not needed: the library writes the HDF5 structures itself
(superblock version 0, the format every HDF5 library reads).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import check, lib


def _julia_layout(a, n):
    """(n,n,n,3) Fortran-ordered float32 view (the reference's array), copying if needed."""
    a = np.asarray(a, dtype=np.float32)
    if a.shape != (n, n, n, 3):
        raise ValueError(f"expected shape {(n, n, n, 3)}, got {a.shape}")
    return np.asfortranarray(a)


def write_snapshot(path, psi, pi, D: float, L: float):
    """Write `psi` and `pi` ((n,n,n,3) arrays in the reference's layout) with the
    attributes D and L. Raises DJBError (code DJB_ERR_IO) when the file cannot be
    written; no partial file is left behind."""
    n = int(np.shape(psi)[0])
    ps = _julia_layout(psi, n)
    pv = _julia_layout(pi, n)
    check(lib.djb_write_snapshot_h5(os.fsencode(path), C.c_void_p(ps.ctypes.data), C.c_void_p(pv.ctypes.data), n,
                                    float(D), float(L)))


def snapshot_name(prefix: str, D: float) -> str:
    """File name of the study driver's snapshots: `<prefix>_D%.3f.h5`, the tag part of `snapname` (run_jobs.jl:39-44)."""
    return f"{prefix}_D{D:.3f}.h5"
