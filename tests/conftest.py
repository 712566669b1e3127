"""Shared fixtures. `-m "not gpu"` runs on any machine; `-m gpu` needs a CUDA device."""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "discodj.jl_b200"))

GOLDEN = os.path.join(ROOT, "tests", "golden", "jax_nbody_reference.npz")
# The reference checkout (yipihey/DiscoDJ.jl), when one is present: its root directory is
# named by DISCODJ_REFERENCE. Tests that read it skip when it is unset or missing.
REFERENCE_ROOT = os.environ.get("DISCODJ_REFERENCE", "")
REFERENCE_H5 = os.path.join(REFERENCE_ROOT, "native", "DiscoDJNative", "test", "reference",
                            "jax_nbody_reference.h5") if REFERENCE_ROOT else ""


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: larger parity cases")


def rel(x, y) -> float:
    """The reference's parity metric max|x − y| / max|y| (nbody_parity_tests.jl:11)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    return float(np.max(np.abs(x - y)) / np.max(np.abs(y)))


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


def config_names(d):
    return json.loads(str(d["configs"]))


def config_attrs(d, name):
    return json.loads(str(d[f"{name}/attrs"]))


def run_kwargs(d, name):
    a = config_attrs(d, name)
    tv = a["time_var"]
    tv = d[f"{name}/time_var_array"] if tv == "array" else tv
    return dict(boxsize=100.0, a_ini=a["a_ini"], a_end=a["a_end"], n_steps=a["n_steps"], res_pm=a["res_pm"],
                time_var=tv, stepper=a["stepper"], antialias=a["antialias"],
                grad_kernel_order=a["grad_kernel_order"], laplace_kernel_order=a["laplace_kernel_order"],
                worder=a["worder"], deconvolve=bool(a["deconvolve"]), n_resample=a["n_resample"],
                resampling_method=a["resampling_method"])


# parity targets: every configuration except the upstream-bug evidence group
# (nbody_parity_tests.jl:38)
PARITY_CONFIGS = [
    "bullfrog_D_cic", "fastpm_D_tsc", "symplectic_a_pcs_deconv", "symplectic_superconft",
    "bullfrog_loga_ik_aa1", "bullfrog_D_aa2_lap2", "bullfrog_D_aa3_grad6_lap4", "bullfrog_D_aam1_lap6",
    "bullfrog_resample_fourier", "bullfrog_resample_linear_fixed", "bullfrog_ic_bullfrog",
    "bullfrog_explicit_a",
]


@pytest.fixture(scope="session")
def cuda_device():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return 0
