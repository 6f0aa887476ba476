"""Reader and writer for the subset of HDF5 that HOPR mesh files and FLUXO State files use.

The reference opens its mesh (src/mesh/mesh_readin.f90:168-716, ReadMesh) and its restart
state (src/restart/restart.f90) through the HDF5 library (src/io_hdf5/hdf5_input.f90:
ReadArray, ReadAttribute, GetDataSize).  No HDF5 library is part of this package, so this
module implements the file format directly, restricted to what those files hold:

* superblock version 0 or 1, 8-byte offsets and lengths;
* version-1 object headers (with continuation blocks) for groups and datasets;
* symbol-table groups (v1 B-tree of group nodes, symbol-table nodes, local heap);
* fixed-point and floating-point datatypes of 1-8 bytes, fixed-length strings;
* simple dataspaces; contiguous and compact data layouts; unfiltered chunked layouts;
* attributes (message versions 1-3) on the root group and on datasets.

Compressed (filtered) data, variable-length strings and the dense link storage of newer
library versions raise H5FormatError: HOPR and FLUXO write none of them.

Arrays come back in the file's (C) dimension order, so a Fortran array written as
A(3, nNodes) is read as shape (nNodes, 3), which is the Fortran array's transpose.

The writer (write_h5) emits the same subset: superblock 0, one level of datasets under the
root group, contiguous little-endian data, and scalar, array and string attributes.
"""

from __future__ import annotations

import struct

import numpy as np

__all__ = ["H5File", "H5FormatError", "write_h5"]

_SIG = b"\x89HDF\r\n\x1a\n"
_UNDEF = 0xFFFFFFFFFFFFFFFF


class H5FormatError(ValueError):
    pass


class _Dataset:
    def __init__(self, f, name, msgs):
        self._f = f
        self.name = name
        self.shape = None
        self.dtype = None
        self.attrs = {}
        self._layout = None
        self._filters = False
        for mtype, body in msgs:
            if mtype == 0x0001:
                self.shape = f._dataspace(body)
            elif mtype == 0x0003:
                self.dtype, _ = f._datatype(body, 0)
            elif mtype == 0x0008:
                self._layout = body
            elif mtype == 0x000B:
                self._filters = True
            elif mtype == 0x000C:
                k, v = f._attribute(body)
                self.attrs[k] = v

    def read(self):
        if self._filters:
            raise H5FormatError(f"dataset {self.name}: filtered (compressed) data is not supported")
        if self.shape is None or self.dtype is None or self._layout is None:
            raise H5FormatError(f"dataset {self.name}: missing dataspace, datatype or layout")
        return self._f._read_layout(self._layout, self.shape, self.dtype, self.name)


class H5File:
    """Read-only view of an HDF5 file: ``datasets`` (name -> dataset), ``attrs`` (root attributes).

    ``read(name)`` returns a dataset as a numpy array; ``attr(name)`` a root attribute
    (strings decoded, one-element arrays returned as scalars)."""

    def __init__(self, path):
        with open(path, "rb") as fh:
            self._d = fh.read()
        self.path = str(path)
        d = self._d
        if d[:8] != _SIG:
            raise H5FormatError(f"{path}: not an HDF5 file")
        ver = d[8]
        if ver not in (0, 1):
            raise H5FormatError(f"{path}: superblock version {ver} is not supported")
        so, sl = d[13], d[14]
        if so != 8 or sl != 8:
            raise H5FormatError(f"{path}: only 8-byte offsets and lengths are supported")
        p = 24 if ver == 0 else 28  # v1 adds indexed-storage K (2) + reserved (2)
        base = struct.unpack_from("<Q", d, p)[0]
        if base != 0:
            raise H5FormatError(f"{path}: a nonzero base address is not supported")
        p += 32  # base, free-space, end-of-file, driver-info addresses
        root_oh = struct.unpack_from("<Q", d, p + 8)[0]
        self.datasets = {}
        self.attrs = {}
        self._walk_group(root_oh, "")

    # -- low-level structures ------------------------------------------------------------
    def _u(self, fmt, p):
        return struct.unpack_from("<" + fmt, self._d, p)

    def _header_messages(self, addr):
        d = self._d
        if d[addr:addr + 4] == b"OHDR":
            raise H5FormatError("version-2 object headers are not supported")
        ver, _, nmsg = self._u("BBH", addr)
        if ver != 1:
            raise H5FormatError(f"object header version {ver} is not supported")
        hsize = self._u("I", addr + 8)[0]
        blocks = [(addr + 16, hsize)]
        msgs = []
        while blocks:
            start, size = blocks.pop(0)
            p, end = start, start + size
            while p + 8 <= end and len(msgs) < nmsg:
                mtype, msize, _flags = self._u("HHB", p)
                body = d[p + 8:p + 8 + msize]
                if mtype == 0x0010:  # continuation
                    caddr, clen = self._u("QQ", p + 8)
                    blocks.append((caddr, clen))
                msgs.append((mtype, body))
                p += 8 + msize
        return msgs

    def _local_heap(self, addr):
        if self._d[addr:addr + 4] != b"HEAP":
            raise H5FormatError("local heap signature missing")
        size, _free, data = self._u("QQQ", addr + 8)
        return self._d[data:data + size]

    def _heap_str(self, heap, off):
        end = heap.index(b"\0", off)
        return heap[off:end].decode("ascii")

    def _btree_group_leaves(self, addr, out):
        d = self._d
        if d[addr:addr + 4] != b"TREE":
            raise H5FormatError("B-tree signature missing")
        ntype, level, nused = self._u("BBH", addr + 4)
        if ntype != 0:
            raise H5FormatError("expected a group B-tree")
        p = addr + 24  # signature, type, level, entries, left and right siblings
        for i in range(nused):
            child = self._u("Q", p + 8 + 16 * i)[0]
            if level == 0:
                out.append(child)
            else:
                self._btree_group_leaves(child, out)

    def _walk_group(self, oh_addr, prefix):
        msgs = self._header_messages(oh_addr)
        stab = None
        for mtype, body in msgs:
            if mtype == 0x0011:
                stab = struct.unpack_from("<QQ", body, 0)
            elif mtype == 0x000C:
                k, v = self._attribute(body)
                if not prefix:
                    self.attrs[k] = v
            elif mtype in (0x0002, 0x0006, 0x000A):
                raise H5FormatError("link-message (new-style) groups are not supported")
        if stab is None:
            return
        btree, heap_addr = stab
        heap = self._local_heap(heap_addr)
        leaves = []
        self._btree_group_leaves(btree, leaves)
        for snod in leaves:
            if self._d[snod:snod + 4] != b"SNOD":
                raise H5FormatError("symbol-table node signature missing")
            nsym = self._u("H", snod + 6)[0]
            for i in range(nsym):
                e = snod + 8 + 40 * i
                name_off, oh = self._u("QQ", e)
                name = prefix + self._heap_str(heap, name_off)
                sub = self._header_messages(oh)
                if any(t == 0x0011 for t, _ in sub):
                    self._walk_group(oh, name + "/")
                else:
                    self.datasets[name] = _Dataset(self, name, sub)

    def _dataspace(self, b):
        ver = b[0]
        if ver == 1:
            rank, flags = b[1], b[2]
            p = 8
        elif ver == 2:
            rank, flags, stype = b[1], b[2], b[3]
            if stype == 2:
                return None  # null dataspace
            p = 4
        else:
            raise H5FormatError(f"dataspace version {ver} is not supported")
        return tuple(struct.unpack_from("<Q", b, p + 8 * i)[0] for i in range(rank))

    def _datatype(self, b, p):
        cv = b[p]
        cls, ver = cv & 0x0F, cv >> 4
        bits = b[p + 1] | (b[p + 2] << 8) | (b[p + 3] << 16)
        size = struct.unpack_from("<I", b, p + 4)[0]
        if cls == 0:  # fixed point
            order = ">" if bits & 1 else "<"
            kind = "i" if bits & 8 else "u"
            return np.dtype(f"{order}{kind}{size}"), p + 8 + 4
        if cls == 1:  # floating point
            order = ">" if bits & 1 else "<"
            if size not in (4, 8):
                raise H5FormatError(f"float of {size} bytes is not supported")
            return np.dtype(f"{order}f{size}"), p + 8 + 12
        if cls == 3:  # fixed-length string
            return np.dtype(f"S{size}"), p + 8
        raise H5FormatError(f"datatype class {cls} (version {ver}) is not supported")

    def _attribute(self, b):
        ver = b[0]
        if ver not in (1, 2, 3):
            raise H5FormatError(f"attribute message version {ver} is not supported")
        nsize, tsize, ssize = struct.unpack_from("<HHH", b, 2)
        p = 8 if ver < 3 else 9
        pad = (lambda n: (n + 7) & ~7) if ver == 1 else (lambda n: n)
        name = b[p:p + nsize].split(b"\0", 1)[0].decode("ascii")
        p += pad(nsize)
        dt, _ = self._datatype(b, p)
        p += pad(tsize)
        shape = self._dataspace(b[p:p + ssize])
        p += pad(ssize)
        if shape is None:
            return name, None
        count = int(np.prod(shape)) if shape else 1
        arr = np.frombuffer(b, dtype=dt, count=count, offset=p).reshape(shape if shape else ())
        return name, _decode(arr)

    def _read_layout(self, body, shape, dt, name):
        ver = body[0]
        if ver != 3:
            raise H5FormatError(f"dataset {name}: layout message version {ver} is not supported")
        cls = body[1]
        count = int(np.prod(shape)) if shape else 1
        if cls == 0:  # compact
            size = struct.unpack_from("<H", body, 2)[0]
            raw = body[4:4 + size]
            return np.frombuffer(raw, dtype=dt, count=count).reshape(shape).copy()
        if cls == 1:  # contiguous
            addr, size = struct.unpack_from("<QQ", body, 2)
            if addr == _UNDEF:
                return np.zeros(shape, dtype=dt)
            if size < count * dt.itemsize:
                raise H5FormatError(f"dataset {name}: contiguous storage is too small")
            return np.frombuffer(self._d, dtype=dt, count=count, offset=addr).reshape(shape).copy()
        if cls == 2:  # chunked, no filters
            rank = body[2] - 1
            btree = struct.unpack_from("<Q", body, 3)[0]
            cdims = struct.unpack_from("<" + "I" * rank, body, 11)
            out = np.zeros(shape, dtype=dt)
            if btree != _UNDEF:
                self._read_chunks(btree, rank, cdims, out, dt)
            return out
        raise H5FormatError(f"dataset {name}: layout class {cls} is not supported")

    def _read_chunks(self, addr, rank, cdims, out, dt):
        d = self._d
        if d[addr:addr + 4] != b"TREE":
            raise H5FormatError("chunk B-tree signature missing")
        ntype, level, nused = self._u("BBH", addr + 4)
        if ntype != 1:
            raise H5FormatError("expected a raw-data chunk B-tree")
        ksize = 8 + 8 * (rank + 1)
        p = addr + 24
        for i in range(nused):
            kp = p + i * (ksize + 8)
            csize, fmask = self._u("II", kp)
            offs = self._u("Q" * rank, kp + 8)
            child = self._u("Q", kp + ksize)[0]
            if level > 0:
                self._read_chunks(child, rank, cdims, out, dt)
                continue
            if fmask != 0:
                raise H5FormatError("filtered chunks are not supported")
            chunk = np.frombuffer(d, dtype=dt, count=int(np.prod(cdims)), offset=child).reshape(cdims)
            sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, cdims, out.shape))
            out[sl] = chunk[tuple(slice(0, s.stop - s.start) for s in sl)]

    # -- public --------------------------------------------------------------------------
    def read(self, name):
        if name not in self.datasets:
            raise KeyError(f"{self.path}: no dataset {name!r}")
        return self.datasets[name].read()

    def attr(self, name, default=KeyError):
        if name not in self.attrs:
            if default is KeyError:
                raise KeyError(f"{self.path}: no attribute {name!r}")
            return default
        return self.attrs[name]

    def __contains__(self, name):
        return name in self.datasets


def _decode(arr):
    if arr.dtype.kind == "S":
        vals = [x.split(b"\0", 1)[0].decode("ascii").rstrip() for x in arr.reshape(-1)]
        return vals[0] if arr.size == 1 else vals
    if arr.size == 1:
        return arr.reshape(-1)[0].item()
    return arr.copy()


# ---------------------------------------------------------------------------------------------
# writer
# ---------------------------------------------------------------------------------------------
def _dt_msg(dt):
    dt = np.dtype(dt)
    if dt.kind in "iu":
        bits = (8 if dt.kind == "i" else 0)
        return struct.pack("<BBBBI", 0x10 | 0, bits, 0, 0, dt.itemsize) + struct.pack("<HH", 0, 8 * dt.itemsize)
    if dt.kind == "f":
        if dt.itemsize == 8:
            bits0, sign, epos, esz, mpos, msz, bias = 0x20, 63, 52, 11, 0, 52, 1023
        else:
            bits0, sign, epos, esz, mpos, msz, bias = 0x20, 31, 23, 8, 0, 23, 127
        return (struct.pack("<BBBBI", 0x10 | 1, bits0, sign, 0, dt.itemsize)
                + struct.pack("<HHBBBBI", 0, 8 * dt.itemsize, epos, esz, mpos, msz, bias))
    if dt.kind == "S":
        return struct.pack("<BBBBI", 0x10 | 3, 0, 0, 0, dt.itemsize)  # null-terminated, ASCII
    raise H5FormatError(f"cannot write dtype {dt}")


def _ds_msg(shape):
    b = struct.pack("<BBBB I", 1, len(shape), 0, 0, 0)
    for s in shape:
        b += struct.pack("<Q", s)
    return b


def _pad8(b):
    return b + b"\0" * ((-len(b)) % 8)


def _attr_msg(name, value):
    if isinstance(value, str):
        raw = value.encode("ascii")
        arr = np.array([raw], dtype=f"S{max(len(raw), 1)}")
    elif isinstance(value, (list, tuple)) and value and isinstance(value[0], str):
        n = max(len(v) for v in value)
        arr = np.array([v.encode("ascii") for v in value], dtype=f"S{max(n, 1)}")
    else:
        arr = np.asarray(value)
        if arr.dtype.kind == "f":
            arr = arr.astype("<f8")
        elif arr.dtype.kind in "iub":
            arr = arr.astype("<i4")
        if arr.ndim == 0:
            arr = arr.reshape(1)
    nb = name.encode("ascii") + b"\0"
    tm, sm = _dt_msg(arr.dtype), _ds_msg(arr.shape)
    head = struct.pack("<BBHHH", 1, 0, len(nb), len(tm), len(sm))
    return _pad8(head + _pad8(nb) + _pad8(tm) + _pad8(sm) + arr.tobytes())


def _msg(mtype, body, flags=0):
    body = _pad8(body)
    return struct.pack("<HHB3x", mtype, len(body), flags) + body


def _ohdr(msgs):
    blob = b"".join(msgs)
    return struct.pack("<BBHII", 1, 0, len(msgs), 1, len(blob)) + b"\0" * 4 + blob


def write_h5(path, datasets, attrs=None):
    """Write ``datasets`` (name -> numpy array, C order) and root ``attrs`` to an HDF5 file.

    Attribute values may be numbers, numpy arrays, strings or lists of strings; integers
    are stored as 32-bit and floats as 64-bit, as the reference's HDF5 output does."""
    attrs = attrs or {}
    names = sorted(datasets)
    # layout: superblock | root OH | B-tree | SNOD | local heap (+data) | dataset OHs | raw data
    sb_size = 56 + 40
    out = bytearray()
    # heap data: "" at 0, then names
    heap = bytearray(b"\0" * 8)
    offs = {}
    for n in names:
        offs[n] = len(heap)
        heap += _pad8(n.encode("ascii") + b"\0")
    # sizes of fixed parts
    root_msgs_attr = [_msg(0x000C, _attr_msg(k, v)) for k, v in attrs.items()]
    root_size = len(_ohdr([_msg(0x0011, b"\0" * 16)] + root_msgs_attr))
    # group B-tree node allocated for 2K children (internal K = 16), holding one leaf child
    btree_K = 16
    btree_size = 24 + (2 * btree_K + 1) * 8 + 2 * btree_K * 8
    # one symbol-table node: leaf K with 2K >= number of datasets
    leaf_K = max(4, (len(names) + 1) // 2)
    snod_size = 8 + 40 * 2 * leaf_K
    heap_hdr = 32
    root_addr = sb_size
    btree_addr = root_addr + root_size
    snod_addr = btree_addr + btree_size
    heap_addr = snod_addr + snod_size
    heap_data_addr = heap_addr + heap_hdr
    p = heap_data_addr + len(heap)
    arrays = {n: np.ascontiguousarray(datasets[n]) for n in names}
    for n, a in arrays.items():
        if a.dtype.kind == "f":
            arrays[n] = a.astype("<f8")
        elif a.dtype.kind in "iub":
            arrays[n] = a.astype("<i4") if a.dtype.itemsize <= 4 else a.astype("<i8")
    oh_addr = {}
    oh_blobs = {}
    data_addr = {}
    # dataset object headers (layout address patched after sizes are known)
    for n in names:
        oh_addr[n] = p
        a = arrays[n]
        blob = _ohdr([_msg(0x0001, _ds_msg(a.shape)), _msg(0x0003, _dt_msg(a.dtype), 1),
                      _msg(0x0008, struct.pack("<BBQQ", 3, 1, 0, 0))])
        oh_blobs[n] = blob
        p += len(blob)
    for n in names:
        p = (p + 7) & ~7
        data_addr[n] = p
        p += arrays[n].nbytes
    eof = p
    # superblock
    out += _SIG + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", leaf_K, btree_K, 0)
    out += struct.pack("<QQQQ", 0, _UNDEF, eof, _UNDEF)
    out += struct.pack("<QQII", 0, root_addr, 1, 0) + struct.pack("<QQ", btree_addr, heap_addr)
    # root object header
    out += _ohdr([_msg(0x0011, struct.pack("<QQ", btree_addr, heap_addr))] + root_msgs_attr)
    # B-tree (one leaf child); keys: heap offsets of "" and of the last name
    last = offs[names[-1]] if names else 0
    out += b"TREE" + struct.pack("<BBH", 0, 0, 1 if names else 0) + struct.pack("<QQ", _UNDEF, _UNDEF)
    out += struct.pack("<QQQ", 0, snod_addr, last)
    out += b"\0" * (btree_addr + btree_size - len(out))
    # SNOD
    snod = bytearray(b"SNOD" + struct.pack("<BBH", 1, 0, len(names)))
    for n in names:
        snod += struct.pack("<QQII", offs[n], oh_addr[n], 0, 0) + b"\0" * 16
    snod += b"\0" * (snod_size - len(snod))
    out += snod
    # local heap
    out += b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap), _UNDEF, heap_data_addr)
    out += heap
    for n in names:
        blob = bytearray(oh_blobs[n])
        # patch the layout message (last message): address and size
        lay = blob.rfind(struct.pack("<BBQQ", 3, 1, 0, 0))
        blob[lay:lay + 18] = struct.pack("<BBQQ", 3, 1, data_addr[n], arrays[n].nbytes)
        assert len(out) == oh_addr[n]
        out += blob
    for n in names:
        out += b"\0" * (data_addr[n] - len(out))
        out += arrays[n].tobytes()
    with open(path, "wb") as fh:
        fh.write(bytes(out))
