"""Minimal HDF5 reader/writer for the reference's file formats (no libhdf5).

The reference reads its input from an HDF5 ``config`` file written by h5py
(wrapper_python/DemystiFicatioN.py:330-422, read by src/configuration.f90:70-379)
and writes ``output%07d`` snapshot files (src/solver.f90:227-317). Neither
h5py nor libhdf5 is installed here, so this module implements the subset of
the HDF5 file format those files use:

* superblock version 0, 8-byte offsets and lengths;
* version-1 object headers (with continuation blocks);
* groups as symbol tables: version-1 B-tree (type 0) + symbol-table nodes +
  local heap for the link names;
* datasets: dataspace (scalar or simple), fixed-point / floating-point /
  variable-length string datatypes, compact or contiguous layout;
* variable-length strings stored in a global heap collection.

Reading is checked against the two config files the reference ships
(problems/BP6QD_A_4000/config, problems/network_rate_strengthening/config).
"""
from __future__ import annotations

import os
import struct

import numpy as np

SIG = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class HDF5Error(ValueError):
    pass


# ---------------------------------------------------------------------------
# reader

class _Reader:
    def __init__(self, data: bytes):
        self.d = data
        off = 0
        while off < len(data) and data[off:off + 8] != SIG:
            off = 512 if off == 0 else off * 2
        if off >= len(data):
            raise HDF5Error("not an HDF5 file")
        self.base = off
        ver = data[off + 8]
        if ver not in (0, 1):
            raise HDF5Error(f"superblock version {ver} not supported")
        self.so, self.sl = data[off + 13], data[off + 14]
        if self.so != 8 or self.sl != 8:
            raise HDF5Error("only 8-byte offsets/lengths are supported")
        p = off + 24 + (4 if ver == 1 else 0)
        self.base_addr = self.u(p, 8)
        p += 32  # base, free-space, eof, driver
        # root group symbol table entry
        self.root = self._entry(p)

    def u(self, p, n):
        return int.from_bytes(self.d[p:p + n], "little")

    def _entry(self, p):
        return {"name_off": self.u(p, 8), "ohdr": self.u(p + 8, 8), "cache": self.u(p + 16, 4),
                "btree": self.u(p + 24, 8), "heap": self.u(p + 32, 8)}

    # object header v1 -> list of (type, data bytes)
    def messages(self, addr):
        d = self.d
        if d[addr] != 1:
            raise HDF5Error(f"object header version {d[addr]} at {addr} not supported")
        nmsg = self.u(addr + 2, 2)
        size = self.u(addr + 8, 4)
        blocks = [(addr + 16, size)]
        out = []
        while blocks and len(out) < nmsg:
            start, length = blocks.pop(0)
            p = start
            while p + 8 <= start + length and len(out) < nmsg:
                mtype, msize = self.u(p, 2), self.u(p + 2, 2)
                body = d[p + 8:p + 8 + msize]
                if mtype == 0x10:
                    blocks.append((self.u(p + 8, 8), self.u(p + 16, 8)))
                out.append((mtype, body))
                p += 8 + msize
        return out

    def _heap_name(self, heap_addr, off):
        if self.d[heap_addr:heap_addr + 4] != b"HEAP":
            raise HDF5Error("bad local heap")
        seg = self.u(heap_addr + 24, 8)
        s = seg + off
        e = self.d.index(b"\0", s)
        return self.d[s:e].decode()

    def _btree_entries(self, addr, heap):
        d = self.d
        if d[addr:addr + 4] != b"TREE":
            raise HDF5Error("bad B-tree node")
        level = d[addr + 5]
        used = self.u(addr + 6, 2)
        p = addr + 24
        ents = []
        for i in range(used):
            child = self.u(p + 8, 8)   # key (8) then child (8)
            p += 16
            if level > 0:
                ents += self._btree_entries(child, heap)
            else:
                if d[child:child + 4] != b"SNOD":
                    raise HDF5Error("bad symbol table node")
                n = self.u(child + 6, 2)
                q = child + 8
                for _ in range(n):
                    e = self._entry(q)
                    e["name"] = self._heap_name(heap, e["name_off"])
                    ents.append(e)
                    q += 40
        return ents

    def group_children(self, ohdr, entry=None):
        bt = heap = None
        for t, body in self.messages(ohdr):
            if t == 0x11:
                bt, heap = struct.unpack_from("<QQ", body, 0)
        if bt is None:
            raise HDF5Error("object is not a group")
        return {e["name"]: e["ohdr"] for e in self._btree_entries(bt, heap)}

    def is_group(self, ohdr):
        return any(t == 0x11 for t, _ in self.messages(ohdr))

    def dataset(self, ohdr):
        shape, dtype, raw = None, None, None
        for t, b in self.messages(ohdr):
            if t == 0x01:
                shape = self._dataspace(b)
            elif t == 0x03:
                dtype = self._datatype(b)
            elif t == 0x08:
                raw = self._layout(b)
        if shape is None or dtype is None or raw is None:
            raise HDF5Error("incomplete dataset header")
        count = int(np.prod(shape)) if shape else 1
        if dtype[0] == "vlen_str":
            vals = []
            for i in range(count):
                ln, coll, idx = struct.unpack_from("<IQI", raw, 16 * i)
                vals.append(self._gheap(coll, idx)[:ln].decode("utf-8"))
            return vals[0] if not shape else np.array(vals, dtype=object).reshape(shape)
        arr = np.frombuffer(raw[:count * dtype[1].itemsize], dtype=dtype[1]).copy()
        return arr.reshape(shape) if shape else arr[0]

    def _dataspace(self, b):
        ver, rank, flags = b[0], b[1], b[2]
        if ver == 1:
            p = 8
        elif ver == 2:
            p = 4
            if b[3] == 0:
                return ()
        else:
            raise HDF5Error("dataspace version")
        return tuple(struct.unpack_from("<%dQ" % rank, b, p)) if rank else ()

    def _datatype(self, b):
        cls, ver = b[0] & 0x0F, b[0] >> 4
        bits = b[1] | (b[2] << 8) | (b[3] << 16)
        size = struct.unpack_from("<I", b, 4)[0]
        big = bits & 1
        if cls == 0:
            signed = (bits >> 3) & 1
            dt = np.dtype(("<" if not big else ">") + ("i" if signed else "u") + str(size))
            return ("int", dt)
        if cls == 1:
            dt = np.dtype(("<" if not big else ">") + "f" + str(size))
            return ("float", dt)
        if cls == 9 and (bits & 0x0F) == 1:
            return ("vlen_str", None)
        if cls == 3:
            return ("str", np.dtype("S%d" % size))
        raise HDF5Error(f"datatype class {cls} not supported")

    def _layout(self, b):
        ver = b[0]
        if ver == 3:
            cls = b[1]
            if cls == 0:
                n = struct.unpack_from("<H", b, 2)[0]
                return bytes(b[4:4 + n])
            if cls == 1:
                addr, size = struct.unpack_from("<QQ", b, 2)
                if addr == UNDEF:
                    return b"\0" * size
                return self.d[addr:addr + size]
            raise HDF5Error("chunked layout not supported")
        if ver in (1, 2):
            rank, cls = b[1], b[2]
            p = 8
            if cls == 1:
                addr = struct.unpack_from("<Q", b, p)[0]
                dims = struct.unpack_from("<%dI" % rank, b, p + 8)
                size = int(np.prod(dims))
                return self.d[addr:addr + size]
            if cls == 0:
                dims = struct.unpack_from("<%dI" % rank, b, p)
                q = p + 4 * rank
                n = struct.unpack_from("<I", b, q)[0]
                return bytes(b[q + 4:q + 4 + n])
        raise HDF5Error("layout version")

    def _gheap(self, coll, idx):
        d = self.d
        if d[coll:coll + 4] != b"GCOL":
            raise HDF5Error("bad global heap")
        size = self.u(coll + 8, 8)
        p, end = coll + 16, coll + size
        while p + 16 <= end:
            oi, osz = self.u(p, 2), self.u(p + 8, 8)
            if oi == 0:
                break
            if oi == idx:
                return d[p + 16:p + 16 + osz]
            p += 16 + ((osz + 7) & ~7)
        raise HDF5Error("global heap object not found")


def read_file(path):
    """Read an HDF5 file into nested dicts {name: value or dict}."""
    with open(path, "rb") as f:
        r = _Reader(f.read())

    def walk(ohdr):
        out = {}
        for name, child in r.group_children(ohdr).items():
            out[name] = walk(child) if r.is_group(child) else r.dataset(child)
        return out

    return walk(r.root["ohdr"])


def read_config(path):
    """Build a :class:`DemystiFicatioN` problem from a reference ``config`` file."""
    if os.path.isdir(path):
        path = os.path.join(path, "config")
    return problem_from_tree(read_file(path))


def problem_from_tree(t):
    """Build a problem from the nested dict of a ``config`` file's datasets
    (the reader of src/configuration.f90:70-379, same dataset names)."""
    from .problem import DemystiFicatioN

    hp = t["hyperparameter"]
    nf = int(hp["nb_fault"])
    p = DemystiFicatioN(nf)
    for k in ("simulation_name", "fracture_mode", "static_kernel", "friction_law"):
        setattr(p.hyperparameter, k, str(hp[k]))
    p.hyperparameter.tol_solver = float(hp["tol_solver"])
    for k in ("freq_writing_file", "max_it", "stride_time", "iprec", "permeability_coupling"):
        setattr(p.hyperparameter, k, int(hp[k]))
    ml = t["material_loading"]
    for k, v in ml.items():
        setattr(p.material_loading, k, float(v))
    for i in range(nf):
        g = t[f"fault{i + 1}"]
        f = p.faults[i]
        f.nb_element = int(g["nb_element"])
        for k in ("a", "b", "Dc", "f0", "V0", "sigmaN", "V", "theta", "P", "normal_loading_dot",
                  "shear_loading_dot", "permeability", "Lk", "Tk", "kmin", "kmax", "Snk"):
            if k in g:
                setattr(f, k, np.array(g[k], dtype=np.float64).reshape(-1) * np.ones(f.nb_element))
        f.node = np.array(g["node"], dtype=np.float64).reshape(f.nb_element + 1, 2).T.copy()
        ns = int(g.get("nb_source", 0))
        if ns >= 1:
            f.nb_source = ns
            f.Q = np.array(g["Q"], dtype=np.float64).reshape(-1)
            f.t_injection_beg = np.array(g["t_injection_beg"], dtype=np.float64).reshape(-1)
            f.t_injection_end = np.array(g["t_injection_end"], dtype=np.float64).reshape(-1)
            f.index_injection = np.array(g["index_injection"], dtype=np.int64).reshape(-1)
    return p
