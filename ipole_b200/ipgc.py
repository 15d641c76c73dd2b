"""IPGC keyed container: the on-disk format used for fluid dumps and images.

The reference ipole reads iharm dumps and writes images through its HDF5
wrapper (src/hdf5_utils.h).  libhdf5 is not available on this platform, so
dumps and images keep the HDF5 *schema* (same paths, dtypes, shapes and C
element order) inside a flat container:

    char   magic[8] = "IPGC0001"
    uint32 n_entries
    n_entries x {
      uint16 path_len; char path[path_len]     absolute path, e.g. "/header/n1"
      uint8  kind                               0 group, 1 f64, 2 i32, 3 fixed string
      uint8  rank
      uint64 dims[rank]
      uint64 nbytes; uint8 data[nbytes]
    }

Attributes are entries named "<object path>@<attribute>".  The C reader and
writer of the host library (ipole_b200/csrc/host/ipgc.c) implement the same
layout.  The host library also reads and writes the same entries as HDF5
files (ipole_b200/csrc/host/h5lite.c); ``read`` accepts either format and
``write_hdf5`` writes HDF5 through the library.
"""
from __future__ import annotations

import os
import struct
import tempfile
from typing import Dict, Union

import numpy as np

MAGIC = b"IPGC0001"
HDF5_MAGIC = b"\x89HDF\r\n\x1a\n"
GROUP, F64, I32, STR = 0, 1, 2, 3

Value = Union[None, np.ndarray, str, float, int]


def _kind_of(v) -> int:
    if v is None:
        return GROUP
    if isinstance(v, str):
        return STR
    a = np.asarray(v)
    if a.dtype.kind == "f":
        return F64
    if a.dtype.kind in "iu":
        return I32
    raise TypeError(f"unsupported value type {a.dtype}")


def write(path: str, entries: Dict[str, Value], strlen: Dict[str, int] | None = None) -> None:
    """Write ``entries`` (path -> value) to ``path``.

    Floats become f64, integers i32, ``str`` a fixed-length string (length
    from ``strlen`` or len+1), ``None`` a group.  Parent groups are added.
    """
    strlen = strlen or {}
    full: Dict[str, Value] = {}
    for k in entries:
        parts = k.split("@")[0].strip("/").split("/")
        for i in range(1, len(parts)):
            g = "/" + "/".join(parts[:i])
            full.setdefault(g, None)
        full[k] = entries[k]
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<I", len(full)))
        for k, v in full.items():
            kind = _kind_of(v)
            kb = k.encode()
            f.write(struct.pack("<H", len(kb)))
            f.write(kb)
            if kind == GROUP:
                f.write(struct.pack("<BBQ", GROUP, 0, 0))
                continue
            if kind == STR:
                n = strlen.get(k, len(v) + 1)
                data = v.encode()[:n].ljust(n, b"\0")
                f.write(struct.pack("<BBQ", STR, 0, len(data)))
                f.write(data)
                continue
            a = np.array(v, dtype="<f8" if kind == F64 else "<i4", order="C")  # keeps rank 0 for scalars
            f.write(struct.pack("<BB", kind, a.ndim))
            for d in a.shape:
                f.write(struct.pack("<Q", d))
            data = a.tobytes()
            f.write(struct.pack("<Q", len(data)))
            f.write(data)


def _via_library(src: str, dst: str) -> None:
    from . import convert_container
    convert_container(src, dst)


def write_hdf5(path: str, entries: Dict[str, Value], strlen: Dict[str, int] | None = None) -> None:
    """``write`` to an HDF5 file (same entries, same types) through the host
    library's HDF5 writer."""
    with tempfile.TemporaryDirectory() as d:
        tmp = os.path.join(d, "x.ipgc")
        write(tmp, entries, strlen)
        _via_library(tmp, path)


def read(path: str) -> Dict[str, Value]:
    """Read a container or an HDF5 file into a dict path -> value (arrays
    keep their shape; rank-0 numbers come back as 0-d arrays, strings as
    ``str``).  HDF5 files are read by the host library."""
    out: Dict[str, Value] = {}
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:8] != MAGIC and any(buf[o:o + 8] == HDF5_MAGIC for o in (0, 512, 1024, 2048, 4096)):
        with tempfile.TemporaryDirectory() as d:
            tmp = os.path.join(d, "x.ipgc")
            _via_library(path, tmp)
            return read(tmp)
    if buf[:8] != MAGIC:
        raise ValueError(f"{path}: not an IPGC container")
    (n,) = struct.unpack_from("<I", buf, 8)
    off = 12
    for _ in range(n):
        (pl,) = struct.unpack_from("<H", buf, off)
        off += 2
        key = buf[off:off + pl].decode()
        off += pl
        kind, rank = struct.unpack_from("<BB", buf, off)
        off += 2
        dims = struct.unpack_from("<" + "Q" * rank, buf, off)
        off += 8 * rank
        (nb,) = struct.unpack_from("<Q", buf, off)
        off += 8
        raw = buf[off:off + nb]
        off += nb
        if kind == GROUP:
            out[key] = None
        elif kind == STR:
            out[key] = raw.split(b"\0")[0].decode(errors="replace")
        else:
            dt = "<f8" if kind == F64 else "<i4"
            out[key] = np.frombuffer(raw, dtype=dt).reshape(dims).copy()
    return out
