"""Minimal read-only HDF5 reader for the reference's parity fixture.

Test infrastructure only. h5py is not installed in this image, so this module
reads the subset of the HDF5 file format that the fixture
`native/DiscoDJNative/test/reference/jax_nbody_reference.h5` uses (written by
h5py with the earliest file-format version):

* superblock version 0 with 8-byte offsets and lengths,
* version-1 object headers with continuation blocks,
* old-style groups (symbol-table message -> v1 B-tree of SNOD nodes + local heap),
* datasets with contiguous or compact layout (layout message version 3),
* fixed-point, floating-point, enum (numpy bool), fixed and variable-length
  string datatypes; scalar and simple dataspaces (versions 1 and 2),
* attributes stored in the object header (attribute message version 1),
  variable-length string data in global heap collections.

The layouts follow the published HDF5 File Format Specification, version 2.0
(sections II-IV); nothing else is supported and unsupported features raise.
"""
from __future__ import annotations

import struct

import numpy as np

_SIG = b"\x89HDF\r\n\x1a\n"
_UNDEF = 0xFFFFFFFFFFFFFFFF


class H5Error(RuntimeError):
    pass


class _Datatype:
    def __init__(self, cls, size, dtype=None, vlen_string=False, str_len=None):
        self.cls = cls
        self.size = size
        self.dtype = dtype
        self.vlen_string = vlen_string
        self.str_len = str_len


class _Object:
    def __init__(self):
        self.messages = []  # list of (type, bytes)


class H5File:
    """Read-only view of an HDF5 file: `f["group/dataset"]` returns numpy arrays,
    `f.attrs("group")` returns a dict of attribute values, `f.keys("group")` the
    member names in the order the symbol table stores them (sorted by name)."""

    def __init__(self, path):
        with open(path, "rb") as fh:
            self.buf = fh.read()
        b = self.buf
        if b[:8] != _SIG:
            raise H5Error("not an HDF5 file")
        sb_ver = b[8]
        if sb_ver != 0:
            raise H5Error(f"superblock version {sb_ver} unsupported")
        so, sl = b[13], b[14]
        if so != 8 or sl != 8:
            raise H5Error("only 8-byte offsets/lengths supported")
        # root group symbol table entry at 24 + 4*8 = 56
        self.root = self._symbol_entry(56)
        self._gheap_cache = {}

    # ── low-level helpers ────────────────────────────────────────────────
    def _u(self, fmt, off):
        return struct.unpack_from("<" + fmt, self.buf, off)

    def _symbol_entry(self, off):
        name_off, ohdr, cache = self._u("QQI", off)
        scratch = self.buf[off + 24: off + 40]
        return dict(name_off=name_off, ohdr=ohdr, cache=cache, scratch=scratch)

    def _read_object(self, addr):
        b = self.buf
        ver = b[addr]
        if ver != 1:
            raise H5Error(f"object header version {ver} unsupported at {addr}")
        nmsg, = self._u("H", addr + 2)
        hsize, = self._u("I", addr + 8)
        obj = _Object()
        blocks = [(addr + 16, hsize)]
        count = 0
        while blocks and count < nmsg:
            start, size = blocks.pop(0)
            p = start
            end = start + size
            while p + 8 <= end and count < nmsg:
                mtype, msize, _flags = self._u("HHB", p)
                data = b[p + 8: p + 8 + msize]
                count += 1
                if mtype == 0x10:  # continuation
                    coff, clen = struct.unpack_from("<QQ", data, 0)
                    blocks.append((coff, clen))
                else:
                    obj.messages.append((mtype, data))
                p += 8 + msize
        return obj

    def _local_heap(self, addr):
        if self.buf[addr: addr + 4] != b"HEAP":
            raise H5Error("bad local heap signature")
        _dsize, _free, daddr = self._u("QQQ", addr + 8)
        return daddr

    def _heap_string(self, daddr, off):
        s = daddr + off
        e = self.buf.index(b"\x00", s)
        return self.buf[s:e].decode()

    def _btree_group_children(self, addr):
        """All symbol-table entries reachable from a v1 group B-tree node."""
        b = self.buf
        if b[addr: addr + 4] != b"TREE":
            raise H5Error("bad B-tree signature")
        ntype, level = b[addr + 4], b[addr + 5]
        used, = self._u("H", addr + 6)
        if ntype != 0:
            raise H5Error("expected a group B-tree node")
        p = addr + 24  # after signature, type, level, used, left, right
        out = []
        # keys and children interleaved: key0 child0 key1 child1 ... key_used
        for i in range(used):
            p += 8  # key (heap offset)
            child, = self._u("Q", p)
            p += 8
            if level > 0:
                out.extend(self._btree_group_children(child))
            else:
                out.extend(self._snod_entries(child))
        return out

    def _snod_entries(self, addr):
        b = self.buf
        if b[addr: addr + 4] != b"SNOD":
            raise H5Error("bad symbol-table node signature")
        nsym, = self._u("H", addr + 6)
        return [self._symbol_entry(addr + 8 + 40 * i) for i in range(nsym)]

    # ── message decoders ─────────────────────────────────────────────────
    @staticmethod
    def _dataspace(data):
        ver = data[0]
        ndim = data[1]
        flags = data[2]
        if ver == 1:
            p = 8
            if ndim == 0:
                return ()
        elif ver == 2:
            p = 4
            stype = data[3]
            if stype == 0:  # scalar
                return ()
            if stype == 2:
                return None  # null dataspace
        else:
            raise H5Error(f"dataspace version {ver} unsupported")
        dims = struct.unpack_from("<" + "Q" * ndim, data, p)
        _ = flags
        return tuple(int(d) for d in dims)

    def _datatype(self, data):
        cv = data[0]
        cls = cv & 0x0F
        bits = data[1] | (data[2] << 8) | (data[3] << 16)
        size, = struct.unpack_from("<I", data, 4)
        if cls == 0:  # fixed point
            signed = bool(bits & 0x08)
            big = bool(bits & 0x01)
            dt = np.dtype(("i" if signed else "u") + str(size)).newbyteorder(">" if big else "<")
            return _Datatype(cls, size, dt)
        if cls == 1:  # floating point
            big = bool(bits & 0x01)
            dt = np.dtype("f" + str(size)).newbyteorder(">" if big else "<")
            return _Datatype(cls, size, dt)
        if cls == 3:  # fixed-length string
            return _Datatype(cls, size, None, str_len=size)
        if cls == 8:  # enum: base type follows the 8-byte header
            base = self._datatype(data[8:])
            return _Datatype(cls, size, base.dtype)
        if cls == 9:  # variable length
            vtype = bits & 0x0F
            if vtype == 1:
                return _Datatype(cls, size, None, vlen_string=True)
            raise H5Error("variable-length sequences unsupported")
        raise H5Error(f"datatype class {cls} unsupported")

    def _global_heap_object(self, coll_addr, index):
        key = coll_addr
        if key not in self._gheap_cache:
            b = self.buf
            if b[coll_addr: coll_addr + 4] != b"GCOL":
                raise H5Error("bad global heap signature")
            csize, = self._u("Q", coll_addr + 8)
            objs = {}
            p = coll_addr + 16
            end = coll_addr + csize
            while p + 16 <= end:
                idx, _ref = self._u("HH", p)
                osize, = self._u("Q", p + 8)
                if idx == 0:
                    break
                objs[idx] = b[p + 16: p + 16 + osize]
                p += 16 + ((osize + 7) // 8) * 8
            self._gheap_cache[key] = objs
        return self._gheap_cache[key][index]

    def _decode_values(self, dt, shape, raw):
        if shape is None:
            return None
        count = int(np.prod(shape)) if shape else 1
        if dt.vlen_string:
            vals = []
            for i in range(count):
                ln, caddr, idx = struct.unpack_from("<IQI", raw, 16 * i)
                vals.append(self._global_heap_object(caddr, idx)[:ln].decode())
            return vals[0] if shape == () else np.array(vals, dtype=object).reshape(shape)
        if dt.str_len is not None:
            vals = [raw[i * dt.str_len:(i + 1) * dt.str_len].split(b"\x00")[0].decode()
                    for i in range(count)]
            return vals[0] if shape == () else np.array(vals, dtype=object).reshape(shape)
        arr = np.frombuffer(raw, dtype=dt.dtype, count=count).astype(dt.dtype.newbyteorder("="))
        if shape == ():
            return arr[0].item()
        return arr.reshape(shape)

    def _attributes(self, obj):
        out = {}
        for mtype, data in obj.messages:
            if mtype != 0x0C:
                continue
            ver = data[0]
            if ver != 1:
                raise H5Error(f"attribute message version {ver} unsupported")
            nsz, tsz, ssz = struct.unpack_from("<HHH", data, 2)
            pad = lambda n: ((n + 7) // 8) * 8
            p = 8
            name = data[p: p + nsz].split(b"\x00")[0].decode()
            p += pad(nsz)
            dt = self._datatype(data[p: p + tsz])
            p += pad(tsz)
            shape = self._dataspace(data[p: p + ssz])
            p += pad(ssz)
            out[name] = self._decode_values(dt, shape, data[p:])
        return out

    def _dataset(self, obj):
        shape = dt = layout = None
        for mtype, data in obj.messages:
            if mtype == 0x01:
                shape = self._dataspace(data)
            elif mtype == 0x03:
                dt = self._datatype(data)
            elif mtype == 0x08:
                layout = data
        if shape is None or dt is None or layout is None:
            raise H5Error("object is not a dataset")
        ver = layout[0]
        if ver != 3:
            raise H5Error(f"layout message version {ver} unsupported")
        lclass = layout[1]
        count = int(np.prod(shape)) if shape else 1
        nbytes = count * (16 if dt.vlen_string else dt.size)
        if lclass == 0:  # compact
            sz, = struct.unpack_from("<H", layout, 2)
            raw = layout[4: 4 + sz]
        elif lclass == 1:  # contiguous
            addr, sz = struct.unpack_from("<QQ", layout, 2)
            raw = self.buf[addr: addr + nbytes] if addr != _UNDEF else bytes(nbytes)
        else:
            raise H5Error("chunked datasets unsupported")
        return self._decode_values(dt, shape, raw)

    # ── navigation ───────────────────────────────────────────────────────
    def _group_members(self, entry):
        obj = self._read_object(entry["ohdr"])
        for mtype, data in obj.messages:
            if mtype == 0x11:
                btree, heap = struct.unpack_from("<QQ", data, 0)
                daddr = self._local_heap(heap)
                return {self._heap_string(daddr, e["name_off"]): e
                        for e in self._btree_group_children(btree)}
        raise H5Error("object is not a group")

    def _resolve(self, path):
        entry = self.root
        for part in [p for p in path.split("/") if p]:
            members = self._group_members(entry)
            if part not in members:
                raise KeyError(path)
            entry = members[part]
        return entry

    def keys(self, path="/"):
        return list(self._group_members(self._resolve(path)).keys())

    def attrs(self, path="/"):
        return self._attributes(self._read_object(self._resolve(path)["ohdr"]))

    def __getitem__(self, path):
        return self._dataset(self._read_object(self._resolve(path)["ohdr"]))

    def __contains__(self, path):
        try:
            self._resolve(path)
            return True
        except KeyError:
            return False
