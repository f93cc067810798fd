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


# ---------------------------------------------------------------------------
# writer
#
# Files are laid out as libhdf5 1.8-era tools (h5py, the HDF5 Fortran API)
# lay out the reference's files: superblock version 0 with the default
# B-tree widths (group leaf K = 4, internal K = 16), version-1 object headers,
# symbol-table groups whose links are sorted by name in symbol-table nodes of
# at most 2K entries under a version-1 B-tree (more levels when a group has
# more than 32 nodes), version-1 dataspaces with maximum dimensions, version-1
# datatypes (little-endian IEEE double, signed 64-bit integer, UTF-8
# variable-length string), a version-2 fill-value message, version-3
# contiguous layouts, and one global heap collection for the strings.

_LEAF_K, _NODE_K = 4, 16
_DT_F64 = bytes.fromhex("11203f000800000000004000340b0034ff030000")
_DT_I64 = bytes.fromhex("1008000008000000" "00004000")
_DT_VSTR = bytes.fromhex("1901010010000000" "1000000001000000" "00000800")
_FILL_NUM = bytes.fromhex("0202020100000000")
_FILL_STR = bytes.fromhex("0202000100000000")


def _pad8(b):
    return b + b"\0" * ((-len(b)) % 8)


class _Writer:
    def __init__(self):
        self.buf = bytearray(96)          # superblock, patched at the end
        self.strings = []                 # vlen string payloads (global heap)
        self.str_refs = []                # (address of the 16-byte reference, object index)

    def alloc(self, data, align=8):
        pad = (-len(self.buf)) % align
        self.buf += b"\0" * pad
        addr = len(self.buf)
        self.buf += data
        return addr

    @staticmethod
    def _msg(mtype, body, flags=0):
        body = _pad8(body)
        return struct.pack("<HHB3x", mtype, len(body), flags) + body

    def object_header(self, msgs):
        block = b"".join(msgs)
        hdr = struct.pack("<BBHII4x", 1, 0, len(msgs), 1, len(block))
        return self.alloc(hdr + block)

    def dataset(self, value):
        if isinstance(value, str):
            dt, fill, shape = _DT_VSTR, _FILL_STR, ()
            idx = len(self.strings) + 1
            self.strings.append(value.encode("utf-8"))
            raw = bytearray(16)
            data_addr = self.alloc(bytes(raw))
            self.str_refs.append((data_addr, idx))
            size = 16
        else:
            a = np.asarray(value)
            if a.dtype.kind in "iub":
                a = a.astype("<i8")
                dt = _DT_I64
            elif a.dtype.kind == "f":
                a = a.astype("<f8")
                dt = _DT_F64
            else:
                raise HDF5Error(f"cannot write dtype {a.dtype}")
            fill, shape = _FILL_NUM, a.shape
            raw = np.ascontiguousarray(a).tobytes()
            data_addr = self.alloc(raw) if raw else UNDEF
            size = len(raw)
        rank = len(shape)
        space = struct.pack("<BBB5x", 1, rank, 1 if rank else 0)
        if rank:
            space += struct.pack("<%dQ" % rank, *shape) + struct.pack("<%dQ" % rank, *shape)
        layout = struct.pack("<BBQQ", 3, 1, data_addr, size)
        return self.object_header([self._msg(0x01, space), self._msg(0x03, dt, 1), self._msg(0x05, fill, 1),
                                   self._msg(0x08, layout)])

    def group(self, children):
        """children: dict name -> value (dict for a subgroup)."""
        addrs = {}
        for name in sorted(children):
            v = children[name]
            addrs[name] = self.group(v) if isinstance(v, dict) else self.dataset(v)
        names = sorted(addrs)
        # local heap: offset 0 is the empty string
        heap = bytearray(b"\0" * 8)
        off = {}
        for n in names:
            off[n] = len(heap)
            heap += _pad8(n.encode() + b"\0")
        heap_data = self.alloc(bytes(heap))
        heap_addr = self.alloc(b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap), UNDEF, heap_data))
        # symbol-table nodes of at most 2K entries, filled evenly
        n = len(names)
        nsnod = max(1, -(-n // (2 * _LEAF_K)))
        snods = []   # (address, heap offset of its last name)
        start = 0
        for i in range(nsnod):
            cnt = n // nsnod + (1 if i < n % nsnod else 0)
            part = names[start:start + cnt]
            start += cnt
            body = b"SNOD" + struct.pack("<BBH", 1, 0, len(part))
            for nm in part:
                body += struct.pack("<QQI4x16x", off[nm], addrs[nm], 0)
            body += b"\0" * (40 * (2 * _LEAF_K - len(part)))
            snods.append((self.alloc(body), off[part[-1]] if part else 0))
        # B-tree levels of at most 2K children per node
        level, children_ = 0, snods
        lo_key = 0
        while True:
            nn = max(1, -(-len(children_) // (2 * _NODE_K)))
            nodes, s = [], 0
            prev_key = lo_key
            for i in range(nn):
                cnt = len(children_) // nn + (1 if i < len(children_) % nn else 0)
                part = children_[s:s + cnt]
                s += cnt
                body = b"TREE" + struct.pack("<BBHQQ", 0, level, len(part), UNDEF, UNDEF)
                body += struct.pack("<Q", prev_key)
                for caddr, ckey in part:
                    body += struct.pack("<QQ", caddr, ckey)
                body += b"\0" * (16 * (2 * _NODE_K - len(part)))
                nodes.append((self.alloc(body), part[-1][1]))
                prev_key = part[-1][1]
            if len(nodes) == 1:
                root_bt = nodes[0][0]
                break
            children_, level = nodes, level + 1
        return self.object_header([self._msg(0x11, struct.pack("<QQ", root_bt, heap_addr))])

    def finish(self, root_ohdr, root_btree_heap):
        # global heap collection with the strings (at least 4096 bytes)
        if self.strings:
            objs = b""
            for i, s in enumerate(self.strings):
                objs += struct.pack("<HH4xQ", i + 1, 0, len(s)) + _pad8(s)
            size = max(4096, 16 + len(objs) + 16)
            free = size - 16 - len(objs)
            coll = b"GCOL" + struct.pack("<B3xQ", 1, size) + objs + struct.pack("<HH4xQ", 0, 0, free)
            coll += b"\0" * (size - len(coll))
            gaddr = self.alloc(coll)
            for (addr, idx), s in zip(self.str_refs, self.strings):
                struct.pack_into("<IQI", self.buf, addr, len(s), gaddr, idx)
        eof = len(self.buf)
        sb = SIG + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", _LEAF_K, _NODE_K, 0)
        sb += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
        sb += struct.pack("<QQI4xQQ", 0, root_ohdr, 1, *root_btree_heap)
        self.buf[0:96] = sb
        return bytes(self.buf)


def write_file(path, tree):
    """Write nested dicts {name: value or dict} as an HDF5 file (values: str,
    int, float or numpy arrays of integers / floats)."""
    w = _Writer()
    root = w.group(tree)
    # the root symbol-table entry caches the root group's B-tree and heap
    r = _Reader.__new__(_Reader)
    r.d = bytes(w.buf)
    bt_heap = None
    for t, body in r.messages(root):
        if t == 0x11:
            bt_heap = struct.unpack_from("<QQ", body, 0)
    data = w.finish(root, bt_heap)
    with open(path, "wb") as f:
        f.write(data)


def config_tree(problem):
    """The datasets of the reference's ``config`` file for a problem
    (wrapper_python/DemystiFicatioN.py:340-418: same names, groups and types;
    ``node`` stored transposed as (nb_node, 2))."""
    hp, ml = problem.hyperparameter, problem.material_loading
    t = {"hyperparameter": {
        "tol_solver": float(hp.tol_solver), "freq_writing_file": int(hp.freq_writing_file),
        "max_it": int(hp.max_it), "stride_time": int(hp.stride_time), "iprec": int(hp.iprec),
        "nb_fault": int(hp.nb_fault), "simulation_name": str(hp.simulation_name),
        "fracture_mode": str(hp.fracture_mode), "static_kernel": str(hp.static_kernel),
        "friction_law": str(hp.friction_law), "permeability_coupling": int(hp.permeability_coupling)}}
    for i, f in enumerate(problem.faults[:int(hp.nb_fault)]):
        g = {"nb_element": int(f.nb_element)}
        for k in ("a", "b", "Dc", "f0", "V0", "sigmaN", "V", "theta", "P"):
            g[k] = np.asarray(getattr(f, k), dtype=np.float64)
        g["node"] = np.ascontiguousarray(np.asarray(f.node, dtype=np.float64).T).reshape(f.nb_node, 2)
        for k in ("normal_loading_dot", "shear_loading_dot", "permeability", "Lk", "Tk", "kmin", "kmax", "Snk"):
            g[k] = np.asarray(getattr(f, k), dtype=np.float64)
        g["nb_source"] = int(f.nb_source)
        if f.nb_source >= 1:
            g["Q"] = np.asarray(f.Q, dtype=np.float64)
            g["t_injection_beg"] = np.asarray(f.t_injection_beg, dtype=np.float64)
            g["t_injection_end"] = np.asarray(f.t_injection_end, dtype=np.float64)
            g["index_injection"] = np.asarray(f.index_injection, dtype=np.int64)
        t[f"fault{i + 1}"] = g
    t["material_loading"] = {k: float(getattr(ml, k)) for k in (
        "mu", "cp", "cs", "Sigma31_dot", "Sigma32_dot", "Sigma11_dot", "Sigma12_dot", "Sigma22_dot",
        "rock_comp", "fluid_comp", "dyn_viscosity", "porosity", "fluid_density")}
    return t


def write_config(problem, path_problem):
    """``DemystiFicatioN.write``: ``path_problem + 'config'`` (the path is
    concatenated as in the reference, so it normally ends with a separator);
    the directory is created when missing. Returns the file path."""
    d = os.path.dirname(path_problem + "config")
    if d and not os.path.exists(d):
        os.makedirs(d)
    path = path_problem + "config"
    write_file(path, config_tree(problem))
    return path


OUTPUT_FIELDS = ("V", "theta", "P", "tractionTel", "tractionNel", "permeability")


def write_output(path, rows, freq_writing_file, nb_element, stale=None):
    """One ``output%07d`` file of write_data (src/solver.f90:227-317).

    ``rows`` are saved snapshots (dicts with the six fields and ``time``). The
    file always holds ``freq_writing_file`` rows: the datasets are
    V/theta/P/tractionTel/tractionNel/permeability of shape
    (nb_element, freq_writing_file) (the Fortran (freq, nb_element) array as
    C-ordered readers see it) and time of shape (freq_writing_file,). Rows
    past ``len(rows)`` hold what the reference's save arrays hold there: the
    rows of the previous file (``stale``, the dict this function returns), or
    zeros for the first file."""
    F, N = int(freq_writing_file), int(nb_element)
    if len(rows) > F:
        raise HDF5Error("more rows than freq_writing_file")
    ring = {k: np.zeros((F, N)) for k in OUTPUT_FIELDS}
    ring["time"] = np.zeros(F)
    if stale is not None:
        for k in ring:
            ring[k][:] = stale[k]
    for r, snap in enumerate(rows):
        for k in OUTPUT_FIELDS:
            ring[k][r] = snap[k]
        ring["time"][r] = snap["time"]
    tree = {k: np.ascontiguousarray(ring[k].T) for k in OUTPUT_FIELDS}
    tree["time"] = ring["time"].copy()
    write_file(path, tree)
    return ring


def read_output(path):
    """An ``output%07d`` file as {field: array}; the six fields are returned
    as (freq_writing_file, nb_element), rows in saving order."""
    t = read_file(path)
    out = {k: np.asarray(t[k]).T.copy() for k in OUTPUT_FIELDS if k in t}
    out["time"] = np.asarray(t["time"])
    return out
