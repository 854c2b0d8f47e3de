"""Reader of the logs that the reference program writes when it is built with
the oracle's HDF5 stand-in (oracle/shim/h5log.c): test infrastructure.

Returns the same shapes as h5read.flatten: {path: array} and
{group path: {attribute: value}}, later records replacing earlier ones.
"""
import struct

import numpy as np

_DT = {0: np.dtype("<f8"), 1: np.dtype("<i4"), 2: np.dtype("<c16")}


def read(path):
    with open(path, "rb") as fh:
        b = fh.read()
    if b[:8] != b"NS2DLOG1":
        raise ValueError(f"{path}: not a reference output log")
    at = 8
    data, attrs, groups = {}, {}, []

    def u32():
        nonlocal at
        v = struct.unpack_from("<I", b, at)[0]
        at += 4
        return v

    def string():
        nonlocal at
        n = u32()
        s = b[at:at + n].decode()
        at += n
        return s

    while at < len(b):
        kind = u32()
        p = string()
        if kind == 1:
            groups.append(p)
        elif kind == 2:
            name = string()
            (v,) = struct.unpack_from("<d", b, at)
            at += 8
            attrs.setdefault(p, {})[name] = v
        elif kind == 3:
            t, rank = u32(), u32()
            dims = struct.unpack_from(f"<{rank}Q", b, at)
            at += 8 * rank
            (nbytes,) = struct.unpack_from("<Q", b, at)
            at += 8
            data["/" + p.lstrip("/")] = np.frombuffer(b[at:at + nbytes], dtype=_DT[t]).reshape(dims)
            at += nbytes
        else:
            raise ValueError(f"{path}: bad record kind {kind}")
    return data, attrs, groups
