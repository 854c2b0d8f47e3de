"""Strict reader of the HDF5 subset the solver's output files use (test
infrastructure; no libhdf5 or h5py exists in this image).

Written independently of 2d-navier-stokes_b200/h5/ns2d_h5.c from the HDF5
file-format specification, and strict: every structure is checked against
the specification's constraints (signatures, versions, sizes, node
capacities, name order inside symbol-table nodes and against the B-tree keys,
message alignment and counts, extents inside the end-of-file address) and any
violation raises H5FormatError.

Supported: superblock v0/v1 with 8-byte offsets and lengths; version-1 object
headers (with continuation messages); symbol-table groups (v1 B-tree type 0,
local heap, SNOD); dataspace v1/v2; datatypes v1 fixed-point, IEEE floating
point and compound, v3 compound; layout v3 (contiguous, compact); attribute v1.
"""
import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIGNATURE = b"\x89HDF\r\n\x1a\n"


class H5FormatError(ValueError):
    pass


def _need(cond, msg):
    if not cond:
        raise H5FormatError(msg)


class Node:
    def __init__(self, name, kind):
        self.name = name
        self.kind = kind  # "group" or "dataset"
        self.children = {}
        self.attrs = {}
        self.data = None


class Reader:
    def __init__(self, path):
        with open(path, "rb") as fh:
            self.b = fh.read()
        self._superblock()

    def u(self, at, n):
        _need(at + n <= len(self.b), f"read past end of file at {at}+{n}")
        return int.from_bytes(self.b[at:at + n], "little")

    def bytes_at(self, at, n):
        _need(0 <= at and at + n <= self.eof, f"extent {at}+{n} beyond eof {self.eof}")
        return self.b[at:at + n]

    # -- superblock ----------------------------------------------------------
    def _superblock(self):
        b = self.b
        _need(b[:8] == SIGNATURE, "bad signature")
        ver = b[8]
        _need(ver in (0, 1), f"superblock version {ver}")
        _need(b[9] == 0 and b[10] == 0 and b[12] == 0, "free-space / root entry / shared header versions must be 0")
        _need(b[13] == 8 and b[14] == 8, "only 8-byte offsets and lengths")
        self.leaf_k = self.u(16, 2)
        self.node_k = self.u(18, 2)
        _need(self.leaf_k > 0 and self.node_k > 0, "group K values must be > 0")
        at = 24 if ver == 0 else 28
        _need(self.u(at, 8) == 0, "base address must be 0")
        self.eof = self.u(at + 16, 8)
        _need(self.eof <= len(b), f"truncated file: eof {self.eof} > size {len(b)}")
        _need(self.u(at + 8, 8) == UNDEF, "free-space info address must be undefined")
        _need(self.u(at + 24, 8) == UNDEF, "driver info block must be undefined")
        e = at + 32
        self.root_oh = self.u(e + 8, 8)
        cache = self.u(e + 16, 4)
        self.root_cache = (self.u(e + 24, 8), self.u(e + 32, 8)) if cache == 1 else None

    # -- local heap -------------------------------------------------------------
    def heap(self, addr):
        _need(self.bytes_at(addr, 4) == b"HEAP", f"no HEAP at {addr}")
        _need(self.b[addr + 4] == 0, "local heap version must be 0")
        size = self.u(addr + 8, 8)
        free = self.u(addr + 16, 8)
        data = self.u(addr + 24, 8)
        _need(size > 0, "empty heap data segment")
        _need(free == 1 or free < size, "bad heap free-list offset")
        seg = self.bytes_at(data, size)
        _need(seg[0] == 0, "heap offset 0 must hold the empty name")
        return seg

    @staticmethod
    def heap_name(seg, off):
        _need(off < len(seg), f"heap offset {off} beyond data segment")
        end = seg.find(b"\0", off)
        _need(end >= 0, "unterminated heap name")
        return seg[off:end].decode()

    # -- B-tree (type 0) + symbol-table nodes -----------------------------------
    def group_entries(self, btree, heapaddr):
        seg = self.heap(heapaddr)
        entries = []
        self._btree(btree, seg, entries, None, None, set())
        names = [n for n, _ in entries]
        _need(names == sorted(names) and len(set(names)) == len(names), "group entries out of order or repeated")
        return entries

    def _btree(self, addr, seg, out, lo, hi, seen):
        _need(addr not in seen, "B-tree cycle")
        seen.add(addr)
        two_k = 2 * self.node_k
        size = 24 + (two_k + 1) * 8 + two_k * 8
        self.bytes_at(addr, size)
        _need(self.b[addr:addr + 4] == b"TREE", f"no TREE at {addr}")
        _need(self.b[addr + 4] == 0, "B-tree node type must be 0 (group)")
        level = self.b[addr + 5]
        n = self.u(addr + 6, 2)
        _need(n <= two_k, f"B-tree node holds {n} > 2K children")
        at = addr + 24
        keys, kids = [self.u(at, 8)], []
        at += 8
        for _ in range(n):
            kids.append(self.u(at, 8))
            keys.append(self.u(at + 8, 8))
            at += 16
        knames = [self.heap_name(seg, k) for k in keys]
        for a, c in zip(knames, knames[1:]):
            _need(a < c, "B-tree keys not increasing")
        if lo is not None:
            _need(knames[0] == lo, "left key differs from the parent's key")
        if hi is not None and n:
            _need(knames[-1] == hi, "right key differs from the parent's key")
        for c in range(n):
            left, right = knames[c], knames[c + 1]
            if level > 0:
                self._btree(kids[c], seg, out, left, right, seen)
            else:
                self._snod(kids[c], seg, out, left, right)

    def _snod(self, addr, seg, out, left, right):
        size = 8 + 2 * self.leaf_k * 40
        self.bytes_at(addr, size)
        _need(self.b[addr:addr + 4] == b"SNOD", f"no SNOD at {addr}")
        _need(self.b[addr + 4] == 1, "SNOD version must be 1")
        n = self.u(addr + 6, 2)
        _need(0 < n <= 2 * self.leaf_k, f"SNOD holds {n} entries")
        prev = None
        for k in range(n):
            e = addr + 8 + 40 * k
            name = self.heap_name(seg, self.u(e, 8))
            _need(left < name <= right, f"entry {name!r} outside ({left!r}, {right!r}]")
            _need(prev is None or name > prev, "SNOD entries not sorted")
            prev = name
            out.append((name, self.u(e + 8, 8)))
        _need(prev == right, "B-tree right key is not the SNOD's last name")

    # -- object headers ---------------------------------------------------------------
    def messages(self, addr):
        _need(self.b[addr] == 1, f"object header version {self.b[addr]} at {addr}")
        nmsg = self.u(addr + 2, 2)
        _need(self.u(addr + 4, 4) >= 1, "reference count 0")
        chunks = [(addr + 16, self.u(addr + 8, 4))]
        msgs = []
        while chunks:
            start, size = chunks.pop(0)
            self.bytes_at(start, size)
            at, end = start, start + size
            while at < end:
                _need(end - at >= 8, "truncated message header")
                mtype, msize, flags = self.u(at, 2), self.u(at + 2, 2), self.b[at + 4]
                _need(msize % 8 == 0, "v1 message size not a multiple of 8")
                _need(at + 8 + msize <= end, "message overruns its chunk")
                body = self.b[at + 8:at + 8 + msize]
                if mtype == 0x10:
                    chunks.append(struct.unpack_from("<QQ", body))
                msgs.append((mtype, flags, body))
                at += 8 + msize
        _need(len(msgs) == nmsg, f"header says {nmsg} messages, found {len(msgs)}")
        return msgs

    @staticmethod
    def dataspace(body):
        ver, rank, flags = body[0], body[1], body[2]
        if ver == 1:
            _need(not (flags & 2), "permutation indices unsupported")
            at = 8
        else:
            _need(ver == 2, f"dataspace version {ver}")
            at = 4
        dims = [struct.unpack_from("<Q", body, at + 8 * i)[0] for i in range(rank)]
        if flags & 1:
            maxd = [struct.unpack_from("<Q", body, at + 8 * (rank + i))[0] for i in range(rank)]
            for d, m in zip(dims, maxd):
                _need(m == UNDEF or m >= d, "max dimension below current")
        return tuple(dims)

    def datatype(self, body, at=0):
        """(numpy dtype, encoded length) of the datatype at body[at:]."""
        cv = body[at]
        cls, ver = cv & 0x0F, cv >> 4
        bits = body[at + 1] | (body[at + 2] << 8) | (body[at + 3] << 16)
        size = struct.unpack_from("<I", body, at + 4)[0]
        if cls == 0:
            _need(ver == 1, "fixed-point datatype version")
            _need(not (bits & 1), "big-endian unsupported")
            off, prec = struct.unpack_from("<HH", body, at + 8)
            _need(off == 0 and prec == 8 * size, "bit offset/precision")
            return np.dtype(f"<{'i' if bits & 8 else 'u'}{size}"), 12
        if cls == 1:
            _need(ver == 1, "floating-point datatype version")
            _need(not (bits & 1) and not (bits & 0x40), "big-endian unsupported")
            props = struct.unpack_from("<HHBBBBI", body, at + 8)
            if size == 8:
                _need(props == (0, 64, 52, 11, 0, 52, 1023), "not IEEE double")
                _need(((bits >> 4) & 3) == 2 and ((bits >> 8) & 0xFF) == 63, "not IEEE double")
                return np.dtype("<f8"), 20
            _need(size == 4 and props == (0, 32, 23, 8, 0, 23, 127), "float format")
            return np.dtype("<f4"), 20
        if cls == 6:
            nmemb = bits & 0xFFFF
            p = at + 8
            fields = []
            for _ in range(nmemb):
                end = body.index(b"\0", p)
                name = body[p:end].decode()
                if ver == 1:
                    p += ((end - p + 1 + 7) // 8) * 8
                    off = struct.unpack_from("<I", body, p)[0]
                    _need(body[p + 4] == 0, "array members unsupported")
                    p += 32  # offset, dimensionality + 3 reserved, permutation, reserved, 4 dims
                else:
                    _need(ver == 3, f"compound version {ver}")
                    p = end + 1
                    nb = max(1, (size.bit_length() + 7) // 8)
                    off = int.from_bytes(body[p:p + nb], "little")
                    p += nb
                dt, n = self.datatype(body, p)
                p += n
                fields.append((name, dt, off))
            dtype = np.dtype({"names": [f[0] for f in fields], "formats": [f[1] for f in fields],
                              "offsets": [f[2] for f in fields], "itemsize": size})
            return dtype, p - at
        raise H5FormatError(f"datatype class {cls} unsupported")

    def attribute(self, body):
        _need(body[0] == 1, f"attribute message version {body[0]}")
        nl, dtl, dsl = struct.unpack_from("<HHH", body, 2)
        p = 8
        _need(body[p + nl - 1] == 0, "attribute name not terminated")
        name = body[p:p + nl - 1].decode()
        p += (nl + 7) // 8 * 8
        dt, n = self.datatype(body, p)
        _need(n == dtl, f"attribute datatype length {dtl} != {n}")
        p += (dtl + 7) // 8 * 8
        dims = self.dataspace(body[p:p + dsl])
        p += (dsl + 7) // 8 * 8
        count = int(np.prod(dims)) if dims else 1
        _need(p + count * dt.itemsize <= len(body), "attribute data overruns its message")
        return name, np.frombuffer(body, dtype=dt, count=count, offset=p).reshape(dims)

    def object(self, name, addr):
        msgs = self.messages(addr)
        types = [m[0] for m in msgs]
        attrs = {}
        for t, _, body in msgs:
            if t == 0x0C:
                k, v = self.attribute(body)
                _need(k not in attrs, f"repeated attribute {k}")
                attrs[k] = v
        if 0x11 in types:
            btree, heap = struct.unpack_from("<QQ", msgs[types.index(0x11)][2])
            node = Node(name, "group")
            for child, caddr in self.group_entries(btree, heap):
                node.children[child] = self.object(child, caddr)[0]
            node.attrs = attrs
            return node, (btree, heap)
        _need(0x01 in types and 0x03 in types and 0x08 in types, f"{name}: neither a group nor a dataset")
        dims = self.dataspace(msgs[types.index(0x01)][2])
        dtype, _ = self.datatype(msgs[types.index(0x03)][2])
        lay = msgs[types.index(0x08)][2]
        _need(lay[0] == 3, f"layout version {lay[0]}")
        count = int(np.prod(dims)) if dims else 1
        nbytes = count * dtype.itemsize
        if lay[1] == 1:
            daddr, dsize = struct.unpack_from("<QQ", lay, 2)
            if daddr == UNDEF:
                raw = bytes(nbytes)
            else:
                _need(dsize == nbytes, f"{name}: layout size {dsize} != {nbytes}")
                raw = self.bytes_at(daddr, dsize)
        else:
            _need(lay[1] == 0, f"layout class {lay[1]} unsupported")
            csize = struct.unpack_from("<H", lay, 2)[0]
            _need(csize == nbytes, "compact size")
            raw = lay[4:4 + csize]
        node = Node(name, "dataset")
        node.data = np.frombuffer(raw, dtype=dtype, count=count).reshape(dims)
        node.attrs = attrs
        return node, None

    def root(self):
        node, stab = self.object("", self.root_oh)
        _need(node.kind == "group", "root is not a group")
        if self.root_cache is not None:
            _need(self.root_cache == stab, "superblock's cached root symbol table differs from the root header")
        return node


def read(path):
    """Root Node of the file at `path` (groups: .children, .attrs; datasets: .data)."""
    return Reader(path).root()


def as_complex(a):
    """Compound {r, i} doubles as complex128."""
    if a.dtype.names and set(a.dtype.names) == {"r", "i"}:
        out = np.empty(a.shape, np.complex128)  # part by part: keeps the sign of zero parts
        out.real = a["r"]
        out.imag = a["i"]
        return out
    return a


def flatten(node, prefix=""):
    """{path: dataset array} and {path: {attr: value}} over the whole file."""
    data, attrs = {}, {}
    path = prefix + ("/" + node.name if node.name else "")
    if node.attrs:
        attrs[path or "/"] = dict(node.attrs)
    if node.kind == "dataset":
        data[path] = as_complex(node.data)
        return data, attrs
    for child in node.children.values():
        d, a = flatten(child, path)
        data.update(d)
        attrs.update(a)
    return data, attrs
