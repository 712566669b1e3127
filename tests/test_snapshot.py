"""Snapshot files (Psi, Pi) in HDF5: the layout the study driver's `snap_writer` writes
(studies/eft_shell_crossing/scripts/run_jobs.jl:41-48), read back with the test suite's
own HDF5 reader, and the format structures checked field by field. The host writer runs
on CPU; the resident-state writer is a GPU test."""
from __future__ import annotations

import os
import struct
import sys

import numpy as np
import pytest

from conftest import REFERENCE_H5, ROOT

djb200 = pytest.importorskip("djb200")
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
from h5lite import H5File  # noqa: E402

from djb200.snapshot import snapshot_name, write_snapshot  # noqa: E402


def _arrays(n, seed=0):
    rng = np.random.default_rng(seed)
    psi = np.asfortranarray(rng.standard_normal((n, n, n, 3)).astype(np.float32))
    pi = np.asfortranarray(rng.standard_normal((n, n, n, 3)).astype(np.float32))
    return psi, pi


def _as_julia(a):
    """A C-order (3,n,n,n) dataset as the (n,n,n,3) array a Julia reader returns."""
    return np.transpose(a, (3, 2, 1, 0))


def _object_messages(buf, addr):
    """(type, flags, body) of a version-1 object header, checking its prefix."""
    assert buf[addr] == 1                                  # object header version 1
    nmsg, refc, chunk = struct.unpack_from("<HII", buf, addr + 2)
    assert refc == 1
    out, p = [], addr + 16
    while p < addr + 16 + chunk:
        t, size, flags = struct.unpack_from("<HHB", buf, p)
        assert size % 8 == 0                               # bodies are 8-byte aligned
        out.append((t, flags, buf[p + 8:p + 8 + size]))
        p += 8 + size
    assert p == addr + 16 + chunk and len(out) == nmsg     # the chunk is filled exactly
    return out


@pytest.mark.parametrize("n", [1, 4, 13])
def test_host_snapshot_round_trip(tmp_path, n):
    psi, pi = _arrays(n, seed=n)
    path = tmp_path / snapshot_name("run", 0.25)
    write_snapshot(path, psi, pi, D=0.25, L=250.0)
    f = H5File(path)
    assert f.keys("/") == ["Pi", "Psi"]                    # symbol-table order (by name)
    assert f.attrs("/") == {"D": 0.25, "L": 250.0}
    for name, ref in (("Psi", psi), ("Pi", pi)):
        a = f[name]
        assert a.shape == (3, n, n, n) and a.dtype == np.float32
        assert np.array_equal(_as_julia(a), ref)          # bit-exact


def test_snapshot_name_matches_the_study_driver():
    assert snapshot_name("cfg_j1", 0.5) == "cfg_j1_D0.500.h5"


def test_snapshot_format_structures(tmp_path):
    """Superblock 0, root symbol table, heap, B-tree and symbol-table node as the HDF5
    File Format Specification 2.0 lays them out; end-of-file address = file size."""
    n = 5
    psi, pi = _arrays(n)
    path = tmp_path / "s.h5"
    write_snapshot(path, psi, pi, D=1.0, L=100.0)
    b = open(path, "rb").read()
    assert b[:8] == b"\x89HDF\r\n\x1a\n"
    assert tuple(b[8:16]) == (0, 0, 0, 0, 0, 8, 8, 0)     # versions 0, 8-byte offsets and lengths
    leaf_k, internal_k, flags = struct.unpack_from("<HHI", b, 16)
    assert (leaf_k, internal_k, flags) == (4, 16, 0)
    base, freesp, eof, drv = struct.unpack_from("<QQQQ", b, 24)
    assert base == 0 and freesp == drv == 2 ** 64 - 1 and eof == len(b)
    name_off, root, cache, _r, btree, heap = struct.unpack_from("<QQIIQQ", b, 56)
    assert name_off == 0 and root == 96 and cache == 1
    msgs = _object_messages(b, root)
    assert msgs[0][0] == 0x11 and struct.unpack_from("<QQ", msgs[0][2]) == (btree, heap)
    assert [m[0] for m in msgs[1:]] == [0x0C, 0x0C]        # attributes D and L
    assert all(m[2][0] == 1 for m in msgs[1:])             # attribute message version 1
    # local heap: empty name at offset 0, "no free block" marker
    assert b[heap:heap + 4] == b"HEAP" and b[heap + 4] == 0
    dsize, free, daddr = struct.unpack_from("<QQQ", b, heap + 8)
    assert free == 1 and b[daddr:daddr + 8] == bytes(8)
    # B-tree: one leaf-level group node over one symbol-table node, full node size allocated
    assert b[btree:btree + 4] == b"TREE" and (b[btree + 4], b[btree + 5]) == (0, 0)
    used, left, right, k0, child, k1 = struct.unpack_from("<HQQQQQ", b, btree + 6)
    assert used == 1 and left == right == 2 ** 64 - 1 and k0 == 0
    assert b[daddr + k1:daddr + k1 + 4] == b"Psi\x00"     # right key: the last name in the child
    assert child - btree >= 24 + 32 * 8 + 33 * 8
    assert b[child:child + 4] == b"SNOD" and b[child + 4] == 1
    nsym, = struct.unpack_from("<H", b, child + 6)
    assert nsym == 2
    names = []
    for i in range(nsym):
        off, ohdr, ctype = struct.unpack_from("<QQI", b, child + 8 + 40 * i)
        names.append(b[daddr + off:b.index(b"\x00", daddr + off)].decode())
        assert ctype == 0
        types = [(t, fl, body[0]) for t, fl, body in _object_messages(b, ohdr)]
        # dataspace 1, datatype (constant) class 1 version 1, fill value 2 (constant), layout 3
        assert types == [(0x01, 0, 1), (0x03, 1, 0x11), (0x05, 1, 2), (0x08, 0, 3)]
    assert names == ["Pi", "Psi"]


@pytest.mark.skipif(not (REFERENCE_H5 and os.path.exists(REFERENCE_H5)), reason="reference checkout not present")
def test_dataset_headers_carry_the_messages_the_hdf5_library_writes(tmp_path):
    """The fixture was written by the HDF5 library in the same file-format version: its
    datasets carry the same message types, flags and versions as ours (the library pads
    its headers with a null message, which the comparison drops)."""
    ref = H5File(REFERENCE_H5)
    e = ref._resolve("ics/psi_ini")
    b = ref.buf
    theirs = [(t, fl, body[0]) for t, fl, body in _object_messages(b, e["ohdr"]) if t != 0]
    path = tmp_path / "s.h5"
    write_snapshot(path, *_arrays(2), D=1.0, L=1.0)
    ours_file = H5File(path)
    ours = [(t, fl, body[0]) for t, fl, body in
            _object_messages(ours_file.buf, ours_file._resolve("Psi")["ohdr"])]
    assert ours == theirs
    fill_theirs = [body for t, _f, body in _object_messages(b, e["ohdr"]) if t == 0x05][0]
    fill_ours = [body for t, _f, body in _object_messages(ours_file.buf, ours_file._resolve("Psi")["ohdr"])
                 if t == 0x05][0]
    assert fill_ours == fill_theirs
    # a float64 scalar attribute: same datatype and dataspace bytes as the library's
    a_theirs = [body for t, body in ref._read_object(ref._resolve("bullfrog_D_cic")["ohdr"]).messages
                if t == 0x0C and body[8:14] == b"a_ini\x00"][0]
    a_ours = [body for t, _f, body in _object_messages(ours_file.buf, 96) if t == 0x0C][0]
    assert a_ours[4:8] == a_theirs[4:8]                    # datatype and dataspace sizes
    assert a_ours[16:48] == a_theirs[16:48]                # the float64 datatype, the scalar dataspace


def test_unwritable_path_raises_and_leaves_nothing(tmp_path):
    psi, pi = _arrays(2)
    bad = tmp_path / "missing_dir" / "s.h5"
    with pytest.raises(djb200.DJBError) as ei:
        write_snapshot(bad, psi, pi, D=1.0, L=1.0)
    assert ei.value.code == djb200._lib.DJB_ERR_IO
    assert not bad.exists()


def test_wrong_shape_is_rejected(tmp_path):
    psi, pi = _arrays(3)
    with pytest.raises(ValueError):
        write_snapshot(tmp_path / "s.h5", psi, pi[:2], D=1.0, L=1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [64, 192])
def test_state_snapshot_equals_the_output(tmp_path, n):
    """djb_state_write_snapshot streams the resident state; the file holds exactly what
    djb_get_output returns (Psi unwrapped, Pi = Mom / p_div). At n = 192 each array
    (21.2 M floats) crosses in two 16 M-float pieces."""
    from djb200.pm import PMConfig, PMSolver
    rng = np.random.default_rng(3)
    psi = np.asfortranarray((rng.standard_normal((n, n, n, 3)) * 2.0).astype(np.float32))
    mom = np.asfortranarray(rng.standard_normal((n, n, n, 3)).astype(np.float32))
    cfg = PMConfig(res_pm=n, n_part=n, boxsize=100.0)
    with PMSolver(cfg) as s:
        s.set_state(psi, mom)
        path = tmp_path / "state.h5"
        s.write_snapshot(path, D=0.7, L=100.0, p_div=1.3)
        x, p = s.output(wrap=False, p_div=1.3)
    f = H5File(path)
    assert f.attrs("/") == {"D": 0.7, "L": 100.0}
    assert np.array_equal(_as_julia(f["Psi"]), x)
    assert np.array_equal(_as_julia(f["Pi"]), p)
    assert np.array_equal(x, psi)
