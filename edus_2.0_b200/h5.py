"""Minimal HDF5 writer (and reader) for output.h5.

The reference writes output.h5 through the HDF5 library (core/hdf5/hdf5_tree.hpp):
groups, and one-dimensional contiguous datasets of little-endian double, int32
or uint8 (strings are written as uint8 arrays, scalars as one-element arrays),
no attributes.  No HDF5 library exists beside this package, so this module
writes that subset of the HDF5 file format itself:

  * superblock version 0 (8-byte offsets and lengths);
  * every object header version 1;
  * groups as "old-style" symbol-table groups: a symbol-table message pointing
    at a version-1 B-tree (one level-0 node) and a local heap of member names,
    members in symbol-table nodes sorted by name;
  * datasets with dataspace (version 1, rank 1), datatype (fixed-point or IEEE
    floating point, version 1), fill-value (version 2, undefined) and layout
    (version 3, contiguous) messages, data right after the header.

The tree is built in memory (H5Tree) and written in one pass (H5Tree.save), so
a file is always complete.  read_h5 parses the same subset back, checking
signatures, versions and sizes; it is the test-side check of the writer.
"""
from __future__ import annotations

import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIGNATURE = b"\x89HDF\r\n\x1a\n"
LEAF_K = 64        # symbols per symbol-table node: 2 * LEAF_K
INTERNAL_K = 256   # children of a B-tree node: 2 * INTERNAL_K
_ENTRY = 40        # symbol-table entry bytes


def _pad8(b: bytes) -> bytes:
    return b + b"\0" * (-len(b) % 8)


class H5Tree:
    """A group: members are H5Tree (subgroups) or numpy 1-D arrays (datasets)."""

    def __init__(self):
        self.members: dict[str, object] = {}

    def group(self, name: str) -> "H5Tree":
        """The subgroup `name` (created if absent), as HDF5_tree::create_node."""
        name = str(name)
        g = self.members.get(name)
        if g is None:
            g = self.members[name] = H5Tree()
        if not isinstance(g, H5Tree):
            raise ValueError(f"{name} is a dataset")
        return g

    def __getitem__(self, name):
        return self.members[str(name)]

    def write(self, name: str, value):
        """A dataset as HDF5_tree::write does: str -> uint8 array, Python int ->
        int32[1], float -> double[1], sequences and arrays flattened."""
        name = str(name)
        if name in self.members:
            raise ValueError(f"{name} exists")
        if isinstance(value, str):
            arr = np.frombuffer(value.encode(), dtype=np.uint8).copy()
        elif isinstance(value, (bool, int, np.integer)):
            arr = np.array([int(value)], dtype=np.int32)
        elif isinstance(value, (float, np.floating)):
            arr = np.array([float(value)], dtype=np.float64)
        else:
            arr = np.asarray(value)
            if np.iscomplexobj(arr):
                arr = np.ascontiguousarray(arr).view(np.float64)
            arr = arr.reshape(-1)
            if arr.dtype.kind == "f":
                arr = arr.astype(np.float64)
            elif arr.dtype == np.uint8:
                pass
            elif arr.dtype.kind in "iub":
                arr = arr.astype(np.int32)
            else:
                raise TypeError(f"unsupported dataset type {arr.dtype}")
        if arr.size == 0:
            raise ValueError("empty datasets are not written")
        self.members[name] = np.ascontiguousarray(arr)

    # ---- file writing ----
    def save(self, path: str):
        w = _Writer()
        root_hdr = w.group(self)
        eof = len(w.buf)
        sb = bytearray()
        sb += SIGNATURE
        sb += bytes([0, 0, 0, 0, 0, 8, 8, 0])
        sb += struct.pack("<HHI", LEAF_K, INTERNAL_K, 0)
        sb += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
        btree, heap = w.group_tables[root_hdr]
        sb += struct.pack("<QQII", 0, root_hdr, 1, 0) + struct.pack("<QQ", btree, heap)
        assert len(sb) == 96
        w.buf[0:96] = sb
        with open(path, "wb") as f:
            f.write(bytes(w.buf))


class _Writer:
    def __init__(self):
        self.buf = bytearray(96)  # superblock, filled last
        self.group_tables = {}

    def alloc(self, data: bytes) -> int:
        addr = len(self.buf)
        self.buf += data
        self.buf += b"\0" * (-len(self.buf) % 8)
        return addr

    @staticmethod
    def object_header(messages) -> bytes:
        body = bytearray()
        for mtype, data in messages:
            data = _pad8(data)
            body += struct.pack("<HHB3x", mtype, len(data), 0) + data
        return struct.pack("<BBHII", 1, 0, len(messages), 1, len(body)) + b"\0" * 4 + bytes(body)

    def dataset(self, arr: np.ndarray) -> int:
        n = arr.size
        if arr.dtype == np.float64:
            dtype = bytes([0x11, 0x20, 63, 0]) + struct.pack("<I", 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
        elif arr.dtype == np.int32:
            dtype = bytes([0x10, 0x08, 0, 0]) + struct.pack("<I", 4) + struct.pack("<HH", 0, 32)
        else:  # uint8
            dtype = bytes([0x10, 0x00, 0, 0]) + struct.pack("<I", 1) + struct.pack("<HH", 0, 8)
        space = struct.pack("<BBBB4x", 1, 1, 0, 0) + struct.pack("<Q", n)
        fill = bytes([2, 2, 2, 0])  # version 2, late allocation, write if set, undefined
        nbytes = arr.nbytes
        # the data follow the header: its size is known before the address
        probe = self.object_header([(0x0001, space), (0x0003, dtype), (0x0005, fill),
                                    (0x0008, struct.pack("<BBQQ", 3, 1, 0, nbytes))])
        hdr_addr = len(self.buf)
        data_addr = hdr_addr + len(probe) + (-len(probe) % 8)
        hdr = self.object_header([(0x0001, space), (0x0003, dtype), (0x0005, fill),
                                  (0x0008, struct.pack("<BBQQ", 3, 1, data_addr, nbytes))])
        assert len(hdr) == len(probe)
        assert self.alloc(hdr) == hdr_addr
        assert self.alloc(arr.astype(arr.dtype.newbyteorder("<"), copy=False).tobytes()) == data_addr
        return hdr_addr

    def group(self, g: H5Tree) -> int:
        names = sorted(g.members)
        kids = {}
        for nm in names:
            m = g.members[nm]
            kids[nm] = self.group(m) if isinstance(m, H5Tree) else self.dataset(m)
        # local heap: "" at 0, then the names, each padded to 8 bytes
        data = bytearray(8)
        off = {}
        for nm in names:
            off[nm] = len(data)
            data += _pad8(nm.encode() + b"\0")
        data += b"\0" * 8  # room that is not a free block: the free list stays empty
        heap_data = self.alloc(bytes(data))
        heap = self.alloc(b"HEAP" + bytes([0, 0, 0, 0]) + struct.pack("<QQQ", len(data), UNDEF, heap_data))
        # symbol-table nodes of at most 2 * LEAF_K sorted entries
        per = 2 * LEAF_K
        chunks = [names[i:i + per] for i in range(0, len(names), per)] or [[]]
        if len(chunks) > 2 * INTERNAL_K:
            raise ValueError("group too large for a one-level B-tree")
        snods = []
        for ch in chunks:
            node = bytearray(b"SNOD" + bytes([1, 0]) + struct.pack("<H", len(ch)))
            for nm in ch:
                node += struct.pack("<QQII", off[nm], kids[nm], 0, 0) + b"\0" * 16
            node += b"\0" * (_ENTRY * per - _ENTRY * len(ch))
            snods.append(self.alloc(bytes(node)))
        # one level-0 B-tree node: key0 = "" and key i = the last name of child i-1
        tree = bytearray(b"TREE" + bytes([0, 0]) + struct.pack("<H", len(snods)) + struct.pack("<QQ", UNDEF, UNDEF))
        tree += struct.pack("<Q", 0)
        for ch, addr in zip(chunks, snods):
            tree += struct.pack("<QQ", addr, off[ch[-1]] if ch else 0)
        tree += b"\0" * (8 * (4 * INTERNAL_K + 1) - 8 * (2 * len(snods) + 1))
        btree = self.alloc(bytes(tree))
        hdr = self.alloc(self.object_header([(0x0011, struct.pack("<QQ", btree, heap))]))
        self.group_tables[hdr] = (btree, heap)
        return hdr


# ---- reading (the subset written above) ----
def read_h5(path: str) -> dict:
    """Nested dict of the file: groups as dicts, datasets as numpy arrays."""
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:8] != SIGNATURE:
        raise ValueError("not an HDF5 file")
    if buf[8] != 0 or buf[13] != 8 or buf[14] != 8:
        raise ValueError("unsupported superblock")
    leaf_k, int_k = struct.unpack_from("<HH", buf, 16)
    base, _, eof, _ = struct.unpack_from("<QQQQ", buf, 24)
    if base != 0 or eof != len(buf):
        raise ValueError("end-of-file address does not match the file size")
    _, root_hdr, cache, _ = struct.unpack_from("<QQII", buf, 56)

    def messages(addr):
        ver, _, nmsg, _, size = struct.unpack_from("<BBHII", buf, addr)
        if ver != 1:
            raise ValueError("object header version")
        pos, end, out = addr + 16, addr + 16 + size, []
        for _ in range(nmsg):
            mtype, msize, _ = struct.unpack_from("<HHB", buf, pos)
            out.append((mtype, buf[pos + 8:pos + 8 + msize]))
            pos += 8 + msize
        if pos != end:
            raise ValueError("object header size")
        return dict(out)

    def read_obj(addr):
        msgs = messages(addr)
        if 0x0011 in msgs:
            btree, heap = struct.unpack_from("<QQ", msgs[0x0011])
            if buf[heap:heap + 4] != b"HEAP":
                raise ValueError("local heap signature")
            hsize, _, hdata = struct.unpack_from("<QQQ", buf, heap + 8)
            if buf[btree:btree + 4] != b"TREE" or buf[btree + 4] != 0 or buf[btree + 5] != 0:
                raise ValueError("B-tree node")
            nchild = struct.unpack_from("<H", buf, btree + 6)[0]
            out = {}
            last = ""
            for c in range(nchild):
                child = struct.unpack_from("<Q", buf, btree + 24 + 8 + 16 * c)[0]
                if buf[child:child + 4] != b"SNOD":
                    raise ValueError("symbol-table node")
                nsym = struct.unpack_from("<H", buf, child + 6)[0]
                for e in range(nsym):
                    noff, oaddr = struct.unpack_from("<QQ", buf, child + 8 + _ENTRY * e)
                    if noff >= hsize:
                        raise ValueError("name outside the heap")
                    nm = buf[hdata + noff:buf.index(b"\0", hdata + noff)].decode()
                    if nm <= last:
                        raise ValueError("symbols out of order")
                    last = nm
                    out[nm] = read_obj(oaddr)
            return out
        space, dtype, layout = msgs[0x0001], msgs[0x0003], msgs[0x0008]
        if space[0] != 1 or space[1] != 1:
            raise ValueError("dataspace")
        n = struct.unpack_from("<Q", space, 8)[0]
        cls = dtype[0] & 0x0F
        size = struct.unpack_from("<I", dtype, 4)[0]
        if cls == 1 and size == 8:
            dt = np.dtype("<f8")
        elif cls == 0 and size == 4 and dtype[1] & 0x08:
            dt = np.dtype("<i4")
        elif cls == 0 and size == 1:
            dt = np.dtype("u1")
        else:
            raise ValueError("datatype")
        if layout[0] != 3 or layout[1] != 1:
            raise ValueError("layout")
        daddr, dsize = struct.unpack_from("<QQ", layout, 2)
        if dsize != n * dt.itemsize or daddr + dsize > len(buf):
            raise ValueError("dataset storage")
        return np.frombuffer(buf, dtype=dt, count=n, offset=daddr).copy()

    return read_obj(root_hdr)
