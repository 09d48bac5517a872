"""Test-side HDF5 subset decoder and encoder, written independently of the
library's C++ reader/writer (dg-mpi_b200/host/h5file.cpp) so each checks the
other: version 0 superblock, symbol-table root group, version 1 object
headers, contiguous or compact datasets of little-endian integers / IEEE
binary64, version 1 attribute messages.

The decoder is strict about the structure the HDF5 library itself relies on
(symbol-node entries sorted by name, B-tree keys equal to the last name of
the child on their left, 8-byte aligned messages that exactly fill their
header, the local heap's free-list end marker, the end-of-file address), so
that a file the library would refuse fails here too.
"""
from __future__ import annotations

import struct

import numpy as np

SIG = b"\x89HDF\r\n\x1a\n"
UNDEF = (1 << 64) - 1


class Format(ValueError):
    pass


def _u(b, off, n):
    return int.from_bytes(b[off:off + n], "little")


def _dtype(msg):
    cls, size = msg[0] & 15, _u(msg, 4, 4)
    if cls == 0:
        if msg[1] & 1:
            raise Format("big-endian integer")
        return np.dtype(("<i%d" if msg[1] & 8 else "<u%d") % size)
    if cls == 1 and size == 8 and msg[1] == 0x20 and msg[2] == 63 and tuple(msg[12:16]) == (52, 11, 0, 52) \
            and _u(msg, 16, 4) == 1023:
        return np.dtype("<f8")
    raise Format("datatype class %d size %d" % (cls, size))


def _space(msg):
    ver, rank = msg[0], msg[1]
    off = 8 if ver == 1 else 4
    if ver not in (1, 2):
        raise Format("dataspace version %d" % ver)
    return tuple(_u(msg, off + 8 * i, 8) for i in range(rank))


def _messages(b, addr):
    if b[addr] != 1:
        raise Format("object header version %d" % b[addr])
    nmsg, hsize = _u(b, addr + 2, 2), _u(b, addr + 8, 4)
    blocks, out = [(addr + 16, hsize)], []
    while blocks:
        start, size = blocks.pop(0)
        pos = start
        while pos < start + size:
            t, s = _u(b, pos, 2), _u(b, pos + 2, 2)
            if s % 8:
                raise Format("message size %d not a multiple of 8" % s)
            data = b[pos + 8:pos + 8 + s]
            if t == 0x10:
                blocks.append((_u(data, 0, 8), _u(data, 8, 8)))
            out.append((t, data))
            pos += 8 + s
        if pos != start + size:
            raise Format("messages do not fill their header block")
    if len(out) != nmsg:
        raise Format("header says %d messages, holds %d" % (nmsg, len(out)))
    return out


def _attributes(msgs):
    out = {}
    for t, m in msgs:
        if t != 0x0C:
            continue
        if m[0] != 1:
            raise Format("attribute message version %d" % m[0])
        nsz, tsz, ssz = _u(m, 2, 2), _u(m, 4, 2), _u(m, 6, 2)
        p8 = lambda n: (n + 7) & ~7
        name = m[8:8 + nsz].split(b"\0")[0].decode()
        pos = 8 + p8(nsz)
        dt = _dtype(m[pos:pos + tsz])
        pos += p8(tsz)
        shape = _space(m[pos:pos + ssz])
        pos += p8(ssz)
        n = int(np.prod(shape)) if shape else 1
        out[name] = np.frombuffer(m[pos:pos + n * dt.itemsize], dt).reshape(shape)
    return out


def read(path):
    """{'datasets': {name: array}, 'attrs': {obj: {name: array}}} (obj '' = the root group)."""
    with open(path, "rb") as f:
        b = f.read()
    if b[:8] != SIG:
        raise Format("no signature at 0")
    if b[8] != 0 or b[13] != 8 or b[14] != 8:
        raise Format("superblock version / sizes")
    leaf_k, int_k = _u(b, 16, 2), _u(b, 18, 2)
    if _u(b, 24, 8) != 0 or _u(b, 40, 8) != len(b):
        raise Format("base address or end-of-file address")
    root = _u(b, 56 + 8, 8)
    msgs = _messages(b, root)
    stab = [m for t, m in msgs if t == 0x11]
    if len(stab) != 1:
        raise Format("root group without one symbol table message")
    btree, heap = _u(stab[0], 0, 8), _u(stab[0], 8, 8)
    if b[heap:heap + 4] != b"HEAP" or b[heap + 4] != 0:
        raise Format("local heap")
    hsize, free, hdata = _u(b, heap + 8, 8), _u(b, heap + 16, 8), _u(b, heap + 24, 8)
    if free != 1 and not (free % 8 == 0 and free < hsize):
        raise Format("local heap free list head %d" % free)
    hbytes = b[hdata:hdata + hsize]
    name_at = lambda off: hbytes[off:hbytes.index(b"\0", off)].decode()
    if b[btree:btree + 4] != b"TREE" or b[btree + 4] != 0 or b[btree + 5] != 0:
        raise Format("root B-tree (a single leaf expected)")
    used = _u(b, btree + 6, 2)
    if used > 2 * int_k:
        raise Format("B-tree entries exceed 2K")
    entries = []
    for i in range(used):
        child = _u(b, btree + 24 + 8 + 16 * i, 8)
        right_key = _u(b, btree + 24 + 16 + 16 * i, 8)
        if b[child:child + 4] != b"SNOD" or b[child + 4] != 1:
            raise Format("symbol node")
        nsym = _u(b, child + 6, 2)
        if nsym > 2 * leaf_k:
            raise Format("symbol node entries exceed 2K")
        names = [(name_at(_u(b, child + 8 + 40 * k, 8)), _u(b, child + 16 + 40 * k, 8)) for k in range(nsym)]
        if names and name_at(right_key) != names[-1][0]:
            raise Format("B-tree key is not the last name of its child")
        entries += names
    if [n for n, _ in entries] != sorted(n for n, _ in entries):
        raise Format("symbol table entries not sorted by name")
    out = {"datasets": {}, "attrs": {"": _attributes(msgs)}}
    for name, addr in entries:
        m = _messages(b, addr)
        kinds = {t: d for t, d in m}
        shape, dt, lay = _space(kinds[0x01]), _dtype(kinds[0x03]), kinds[0x08]
        if lay[0] != 3:
            raise Format("layout version %d" % lay[0])
        n = int(np.prod(shape)) if shape else 1
        if lay[1] == 1:
            a, size = _u(lay, 2, 8), _u(lay, 10, 8)
            raw = bytes(n * dt.itemsize) if a == UNDEF else b[a:a + n * dt.itemsize]
            if a != UNDEF and size != n * dt.itemsize:
                raise Format("contiguous size of %s" % name)
        elif lay[1] == 0:
            raw = lay[4:4 + _u(lay, 2, 2)]
        else:
            raise Format("layout class %d" % lay[1])
        out["datasets"][name] = np.frombuffer(raw, dt).reshape(shape).copy()
        out["attrs"][name] = _attributes(m)
    return out


# ---------------- encoder ----------------

def _dt_msg(dt: np.dtype):
    if dt.kind in "iu":
        return bytes([0x10, 0x08 if dt.kind == "i" else 0, 0, 0]) + struct.pack("<IHH", dt.itemsize, 0, 8 * dt.itemsize)
    assert dt == np.dtype("<f8")
    return bytes([0x11, 0x20, 63, 0]) + struct.pack("<IHHBBBBI", 8, 0, 64, 52, 11, 0, 52, 1023)


def _sp_msg(shape):
    return bytes([1, len(shape), 1 if shape else 0, 0, 0, 0, 0, 0]) + b"".join(
        struct.pack("<Q", d) for d in tuple(shape) * 2)


def _pad(x):
    return x + bytes(-len(x) % 8)


def _attr_msg(name, value):
    v = np.asarray(value)
    n = name.encode() + b"\0"
    dt, sp = _dt_msg(v.dtype), _sp_msg(())
    return _pad(bytes([1, 0]) + struct.pack("<HHH", len(n), len(dt), len(sp)) + _pad(n) + _pad(dt) + _pad(sp)
                + v.tobytes())


def _header(msgs):
    body = b"".join(struct.pack("<HHB3x", t, len(_pad(d)), fl) + _pad(d) for t, d, fl in msgs)
    return struct.pack("<BBHII4x", 1, 0, len(msgs), 1, len(body)) + body


def write(path, datasets: dict, attrs: dict | None = None):
    """datasets {name: array}; attrs {obj ('' = root): {name: scalar array}}.
    Entries go into symbol nodes of at most 8 (leaf K = 4)."""
    attrs = attrs or {}
    names = sorted(datasets)
    heap, offs = bytearray(8), {}
    for n in names:
        offs[n] = len(heap)
        heap += _pad(n.encode() + b"\0")
    nsn = max(1, -(-len(names) // 8))
    root_msgs = [(0x11, bytes(16), 0)] + [(0x0C, _attr_msg(k, v), 0) for k, v in attrs.get("", {}).items()]
    a_root = 96
    a_bt = a_root + len(_header(root_msgs))
    a_heap = a_bt + 24 + 32 * 8 + 33 * 8
    a_sn = a_heap + 32 + len(heap)
    at = a_sn + nsn * (8 + 8 * 40)
    hdrs, datas = [], []
    for n in names:
        arr = np.ascontiguousarray(datasets[n])
        msgs = [(0x01, _sp_msg(arr.shape), 0), (0x03, _dt_msg(arr.dtype), 1), (0x05, bytes([2, 2, 2, 1, 0, 0, 0, 0]), 1),
                (0x08, bytes(18), 0)] + [(0x0C, _attr_msg(k, v), 0) for k, v in attrs.get(n, {}).items()]
        hdrs.append([at, msgs, arr])
        at += len(_header(msgs))
    for h in hdrs:
        raw = h[2].tobytes()
        h[1][3] = (0x08, bytes([3, 1]) + struct.pack("<QQ", at, len(raw)), 0)
        datas.append(_pad(raw))
        at += len(_pad(raw))
    eof = at
    root_msgs[0] = (0x11, struct.pack("<QQ", a_bt, a_heap), 0)
    out = bytearray(SIG + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", 4, 16, 0)
                    + struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF) + struct.pack("<QQII", 0, a_root, 1, 0)
                    + struct.pack("<QQ", a_bt, a_heap))
    out += _header(root_msgs)
    bt = bytearray(b"TREE" + bytes([0, 0]) + struct.pack("<HQQ", nsn if names else 0, UNDEF, UNDEF) + bytes(8))
    for s in range(nsn if names else 0):
        last = names[min(len(names), 8 * (s + 1)) - 1]
        bt += struct.pack("<QQ", a_sn + s * 328, offs[last])
    out += bt + bytes(24 + 32 * 8 + 33 * 8 - len(bt))
    out += b"HEAP" + bytes(4) + struct.pack("<QQQ", len(heap), 1, a_heap + 32) + heap
    for s in range(nsn):
        grp = names[8 * s:8 * s + 8]
        sn = bytearray(b"SNOD" + bytes([1, 0]) + struct.pack("<H", len(grp)))
        for n in grp:
            sn += struct.pack("<QQII16x", offs[n], hdrs[names.index(n)][0], 0, 0)
        out += sn + bytes(328 - len(sn))
    for h in hdrs:
        assert len(out) == h[0]
        out += _header(h[1])
    for d in datas:
        out += d
    assert len(out) == eof
    with open(path, "wb") as f:
        f.write(out)
