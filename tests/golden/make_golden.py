"""Convert the reference's JAX parity fixture into a numpy archive for the tests.

    python tests/golden/make_golden.py [path/to/jax_nbody_reference.h5]

Reads `native/DiscoDJNative/test/reference/jax_nbody_reference.h5` (written by the
reference's `export_jax_nbody_reference.py` from JAX DISCO-DJ in float64) with the
pure-Python reader in `h5lite.py` and writes `jax_nbody_reference.npz` beside this
script. Arrays keep the fixture's C-order layout: particle fields are (n,n,n,3)
indexed [i,j,k,c]; `fphi` is (n,n,n//2+1) complex indexed [i,j,k] with the z axis
halved. Per-configuration run keywords are stored as JSON strings under
`<config>/kwargs`. The archive is what the tests read, so the GPU box (which has
no copy of the reference) sees the same golden vectors.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from h5lite import H5File  # noqa: E402

DEFAULT_SRC = os.path.join(os.environ.get("DISCODJ_REFERENCE", "/root/reference"), "native", "DiscoDJNative",
                           "test", "reference", "jax_nbody_reference.h5")
OUT = os.path.join(HERE, "jax_nbody_reference.npz")


def extract(src: str) -> dict:
    f = H5File(src)
    out = {}
    for k in f.keys("cosmo"):
        out[f"cosmo/{k}"] = np.asarray(f[f"cosmo/{k}"], dtype=np.float64)
    out["cosmo/attrs"] = np.array(json.dumps(f.attrs("cosmo")))
    for k in f.keys("ics"):
        out[f"ics/{k}"] = np.asarray(f[f"ics/{k}"], dtype=np.float64)
    configs = [g for g in f.keys() if g not in ("cosmo", "ics")]
    out["configs"] = np.array(json.dumps(configs))
    for g in configs:
        for k in f.keys(g):
            out[f"{g}/{k}"] = np.asarray(f[f"{g}/{k}"], dtype=np.float64)
        attrs = f.attrs(g)
        out[f"{g}/kwargs"] = np.array(attrs["kwargs"])
        out[f"{g}/attrs"] = np.array(json.dumps(attrs, default=float))
    return out


def main(argv):
    src = argv[1] if len(argv) > 1 else DEFAULT_SRC
    data = extract(src)
    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT}: {len(data)} arrays, {os.path.getsize(OUT) / 1e6:.2f} MB")


if __name__ == "__main__":
    main(sys.argv)
