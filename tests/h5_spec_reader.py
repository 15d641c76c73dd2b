"""An independent HDF5 decoder for the tests: reads the file layout the
HDF5 File Format Specification (version 3) describes for superblock
version 0, version-1 object headers, symbol-table groups (version-1 B-tree
group nodes, symbol-table nodes, local heaps), contiguous and compact
layouts, fixed-point, floating-point and fixed-length string types, and
version-1 attribute messages.  Written in Python from the specification,
separately from the library's C reader and writer (h5lite.c), so that a
file the library writes can be checked by a second implementation (libhdf5
and h5py are not installed here).

    read(path) -> {"/path/to/dataset": ndarray or bytes, "/path@attr": ...,
                   "/path/to/group": None}
"""
from __future__ import annotations

import struct

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class H5Error(Exception):
    pass


class _File:
    def __init__(self, data: bytes):
        self.d = data
        self.base = 0
        for off in (0, 512, 1024, 2048, 4096):
            if data[off:off + 8] == SIGNATURE:
                self.base = off
                break
        else:
            raise H5Error("no superblock signature")
        p = self.base + 8
        ver = data[p]
        if ver != 0:
            raise H5Error(f"superblock version {ver}")
        # version 0: free-space, root symtab, reserved, shared header versions
        self.so = data[p + 5]  # size of offsets
        self.sl = data[p + 6]  # size of lengths
        if self.so != 8 or self.sl != 8:
            raise H5Error("only 8-byte offsets and lengths")
        p += 8
        self.leaf_k, self.internal_k = struct.unpack_from("<HH", data, p)
        p += 4
        p += 4  # file consistency flags
        base_addr, _ext, eof, _drv = struct.unpack_from("<QQQQ", data, p)
        p += 32
        if eof > len(data) - self.base:
            raise H5Error("end-of-file address past the file")
        # root group symbol table entry
        self.root = self.symtab_entry(p)

    def symtab_entry(self, p):
        """symbol table entry at absolute position p: (name offset, header
        address, cache type, scratch b-tree address, scratch heap address)"""
        name_off, ohdr, cache = struct.unpack_from("<QQI", self.d, p)
        btree = heap = None
        if cache == 1:
            btree, heap = struct.unpack_from("<QQ", self.d, p + 24)
        return name_off, ohdr, cache, btree, heap

    # -- object headers (version 1) --
    def messages(self, addr):
        d = self.d
        p = self.base + addr
        if d[p] != 1:
            raise H5Error(f"object header version {d[p]} at {addr}")
        nmsg = struct.unpack_from("<H", d, p + 2)[0]
        size = struct.unpack_from("<I", d, p + 8)[0]
        out = []
        blocks = [(p + 16, size)]
        while blocks and len(out) < nmsg:
            q, n = blocks.pop(0)
            end = q + n
            while q + 8 <= end and len(out) < nmsg:
                mtype, msize, flags = struct.unpack_from("<HHB", d, q)
                body = d[q + 8:q + 8 + msize]
                if mtype == 0x10:  # continuation
                    caddr, clen = struct.unpack_from("<QQ", body, 0)
                    blocks.append((self.base + caddr, clen))
                out.append((mtype, flags, body))
                q += 8 + msize
        return out

    # -- groups --
    def group_members(self, btree, heap):
        d = self.d
        # local heap: "HEAP", version, reserved, data size, free list, data address
        hp = self.base + heap
        if d[hp:hp + 4] != b"HEAP":
            raise H5Error("local heap signature")
        data_addr = struct.unpack_from("<Q", d, hp + 24)[0]

        def name_at(off):
            s = self.base + data_addr + off
            e = d.index(b"\0", s)
            return d[s:e].decode()

        members = []

        def walk(node):
            p = self.base + node
            if d[p:p + 4] != b"TREE":
                raise H5Error("b-tree signature")
            ntype, level, used = d[p + 4], d[p + 5], struct.unpack_from("<H", d, p + 6)[0]
            if ntype != 0:
                raise H5Error("not a group node")
            q = p + 8 + 16  # left and right siblings
            q += 8  # key 0
            for _ in range(used):
                child = struct.unpack_from("<Q", d, q)[0]
                q += 16  # child, next key
                if level > 0:
                    walk(child)
                else:
                    sp = self.base + child
                    if d[sp:sp + 4] != b"SNOD":
                        raise H5Error("symbol table node signature")
                    nsym = struct.unpack_from("<H", d, sp + 6)[0]
                    for k in range(nsym):
                        e = self.symtab_entry(sp + 8 + 40 * k)
                        members.append((name_at(e[0]), e[1]))

        walk(btree)
        return members

    # -- datatypes, dataspaces --
    @staticmethod
    def dtype(body):
        cls_ver = body[0]
        cls = cls_ver & 0x0F
        bits0 = body[1]
        size = struct.unpack_from("<I", body, 4)[0]
        order = ">" if bits0 & 1 else "<"
        if cls == 0:  # fixed point
            signed = bool(bits0 & 0x08)
            return np.dtype(f"{order}{'i' if signed else 'u'}{size}")
        if cls == 1:  # floating point
            return np.dtype(f"{order}f{size}")
        if cls == 3:  # fixed-length string
            return ("S", size)
        raise H5Error(f"datatype class {cls}")

    @staticmethod
    def dspace(body):
        ver, rank = body[0], body[1]
        if ver != 1:
            raise H5Error(f"dataspace version {ver}")
        return tuple(struct.unpack_from("<Q", body, 8 + 8 * i)[0] for i in range(rank))

    def values(self, dt, shape, raw):
        if isinstance(dt, tuple):
            return raw  # string bytes as stored
        n = int(np.prod(shape)) if shape else 1
        return np.frombuffer(raw, dtype=dt, count=n).reshape(shape).astype(dt.newbyteorder("="))

    def dataset(self, msgs):
        dt = shape = None
        raw = None
        for mtype, _f, body in msgs:
            if mtype == 0x01:
                shape = self.dspace(body)
            elif mtype == 0x03:
                dt = self.dtype(body)
        for mtype, _f, body in msgs:
            if mtype == 0x08:
                ver, cls = body[0], body[1]
                if ver != 3:
                    raise H5Error(f"layout version {ver}")
                if cls == 1:  # contiguous
                    addr, size = struct.unpack_from("<QQ", body, 2)
                    raw = b"" if addr == UNDEF else self.d[self.base + addr:self.base + addr + size]
                elif cls == 0:  # compact
                    size = struct.unpack_from("<H", body, 2)[0]
                    raw = body[4:4 + size]
                else:
                    raise H5Error(f"layout class {cls}")
        return self.values(dt, shape, raw)

    def attributes(self, msgs):
        out = {}
        for mtype, _f, body in msgs:
            if mtype != 0x0C:
                continue
            if body[0] != 1:
                raise H5Error(f"attribute version {body[0]}")
            nsz, dsz, ssz = struct.unpack_from("<HHH", body, 2)
            p = 8
            name = body[p:p + nsz].split(b"\0")[0].decode()
            p += (nsz + 7) & ~7
            dt = self.dtype(body[p:p + dsz])
            p += (dsz + 7) & ~7
            shape = self.dspace(body[p:p + ssz])
            p += (ssz + 7) & ~7
            out[name] = self.values(dt, shape, body[p:])
        return out


def read(path: str) -> dict:
    with open(path, "rb") as f:
        F = _File(f.read())
    out = {}

    def visit(ohdr, prefix):
        msgs = F.messages(ohdr)
        stab = [b for t, _f, b in msgs if t == 0x11]
        for k, v in F.attributes(msgs).items():
            out[f"{prefix or '/'}@{k}" if prefix else f"/@{k}"] = v
        if stab:
            if prefix:
                out[prefix] = None  # a group
            btree, heap = struct.unpack_from("<QQ", stab[0], 0)
            for name, child in F.group_members(btree, heap):
                visit(child, f"{prefix}/{name}")
        else:
            out[prefix] = F.dataset(msgs)

    visit(F.root[1], "")
    return out
