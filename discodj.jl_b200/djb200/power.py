"""P(k) on the B200 with float64 shell sums (power_spectrum.jl:25-79)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import MEM_DEVICE, MEM_HOST, check, dptr, i64ptr, lib


def evaluate_power_spectrum(field, boxsize: float, bins: int = 20, logarithmic: bool = True,
                            deconvolve: bool = False, device: int = 0):
    """(k, Pk, N_modes) of a (res,res,res) field indexed [ix,iy,iz] (a numpy array, or a
    torch CUDA tensor of shape (res,res,res) in column-major memory, i.e. a contiguous
    tensor indexed [iz,iy,ix]). `deconvolve` is accepted and unused, as in the reference."""
    del deconvolve
    if type(field).__module__.startswith("torch") and field.is_cuda:
        res = int(field.shape[0])
        if not field.is_contiguous() or tuple(field.shape) != (res, res, res):
            raise ValueError("device field must be a contiguous cubic float32 tensor")
        ptr, mem, keep = C.c_void_p(field.data_ptr()), MEM_DEVICE, field
        device = field.device.index or 0
    else:
        a = np.asarray(field)
        res = a.shape[0]
        if a.shape != (res, res, res):
            raise ValueError("field must be cubic")
        keep = np.asfortranarray(a, dtype=np.float32)
        ptr, mem = C.c_void_p(keep.ctypes.data), MEM_HOST
    k = np.empty(bins)
    pk = np.empty(bins)
    nm = np.empty(bins, dtype=np.int64)
    check(lib.djb_power_spectrum(ptr, int(res), float(boxsize), int(bins), int(bool(logarithmic)), dptr(k),
                                 dptr(pk), i64ptr(nm), mem, int(device)))
    del keep
    return k, pk, nm


def power_spectrum_shells_noalloc(spectrum, boxsize: float, bins: int = 20, logarithmic: bool = True,
                                  scale2: float = 1.0, stream: int | None = None):
    """Shell sums of a device half spectrum without any device allocation
    (`djb_power_spectrum_shells_noalloc`). `spectrum` is a contiguous complex64 CUDA
    tensor of shape (res, res, res//2+1) indexed [kz, ky, kx], e.g.
    `torch.fft.rfftn(field_zyx, dim=(0, 1, 2))` of a field stored [iz, iy, ix].
    `stream` (a cudaStream_t as an int) defaults to torch's current stream on the
    spectrum's device, so a spectrum still being written there is read after it is done."""
    import torch

    if not (isinstance(spectrum, torch.Tensor) and spectrum.is_cuda and spectrum.dtype == torch.complex64):
        raise ValueError("spectrum must be a complex64 CUDA tensor")
    res = int(spectrum.shape[0])
    if tuple(spectrum.shape) != (res, res, res // 2 + 1) or not spectrum.is_contiguous():
        raise ValueError("spectrum must be a contiguous (res, res, res//2+1) complex64 tensor")
    if stream is None:
        stream = torch.cuda.current_stream(spectrum.device).cuda_stream
    k = np.empty(bins)
    pk = np.empty(bins)
    nm = np.empty(bins, dtype=np.int64)
    check(lib.djb_power_spectrum_shells_noalloc(C.c_void_p(spectrum.data_ptr()), res, float(boxsize), int(bins),
                                                int(bool(logarithmic)), float(scale2), dptr(k), dptr(pk),
                                                i64ptr(nm), C.c_void_p(stream or 0),
                                                int(spectrum.device.index or 0)))
    return k, pk, nm
