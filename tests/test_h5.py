"""The HDF5 reader/writer (csrc/h5mini.cpp via gjx_h5_read/gjx_h5_write):
round trips, the file structure checked by an independent parser written
here from the format specification, a hand-built file in the newer format
(superblock v2, v2 object headers, link messages, compact layout) read back,
and the error paths.  CPU only (no libhdf5 or h5py on these hosts)."""

import os
import struct

import numpy as np
import pytest

from gpujachx_b200 import GjxError, h5

UNDEF = 0xFFFFFFFFFFFFFFFF


def test_round_trip_modes(built, tmp_path):
    f = str(tmp_path / "a.h5")
    G = np.random.default_rng(0).standard_normal((64, 96))
    ida = np.array([96, 96, 64, 64], np.int32)
    h5.write(f, "64", {"IDADIM": ida, "G": G}, mode=0)
    assert np.array_equal(h5.read(f, "64/IDADIM", as_float=False), ida)
    assert np.array_equal(h5.read(f, "64/G"), G) and h5.shape(f, "64/G") == (64, 96)
    h5.write(f, "128", {"X": np.arange(5.0)}, mode=1)            # second group
    assert np.array_equal(h5.read(f, "128/X"), np.arange(5.0))
    h5.write(f, "64", {f"D{i:02d}": np.full(3, float(i)) for i in range(20)}, mode=2)  # 3 symbol nodes
    for i in range(20):
        assert h5.read(f, f"64/D{i:02d}")[1] == i
    h5.write(f, "64", {"G": 2 * G}, mode=2)                       # in place
    assert np.array_equal(h5.read(f, "64/G"), 2 * G)
    assert np.array_equal(h5.read(f, "64/IDADIM", as_float=False), ida)
    assert h5.read(f, "64/IDADIM").dtype == np.float64            # ints convert to float on request


def test_errors(built, tmp_path):
    f = str(tmp_path / "b.h5")
    h5.write(f, "g", {"A": np.ones(4)}, mode=0)
    with pytest.raises(GjxError, match="exists"):
        h5.write(f, "g", {"B": np.ones(4)}, mode=0)               # new file over an old one
    with pytest.raises(GjxError, match="group g exists"):
        h5.write(f, "g", {"B": np.ones(4)}, mode=1)
    with pytest.raises(GjxError, match="another type or shape"):
        h5.write(f, "g", {"A": np.ones(5)}, mode=2)
    with pytest.raises(GjxError, match="no object named"):
        h5.read(f, "g/nothing")
    with pytest.raises(GjxError, match="does not exist"):
        h5.write(str(tmp_path / "none.h5"), "g", {"A": np.ones(1)}, mode=1)
    bad = tmp_path / "bad.h5"
    bad.write_bytes(b"not an hdf5 file at all" * 10)
    with pytest.raises(GjxError, match="signature"):
        h5.read(str(bad), "g/A")


# ---- an independent reader of the classic format ---------------------------
def _u(b, o, n=8):
    return int.from_bytes(b[o:o + n], "little")


def _messages_v1(b, oh):
    assert b[oh] == 1
    n, size = _u(b, oh + 2, 2), _u(b, oh + 8, 4)
    out, p = [], oh + 16
    for _ in range(n):
        t, sz = _u(b, p, 2), _u(b, p + 2, 2)
        assert sz % 8 == 0 and p + 8 + sz <= oh + 16 + size
        out.append((t, p + 8, sz))
        p += 8 + sz
    return out


def _group(b, oh):
    ms = {t: (o, sz) for t, o, sz in _messages_v1(b, oh)}
    o, _ = ms[0x11]
    bt, hp = _u(b, o), _u(b, o + 8)
    assert b[hp:hp + 4] == b"HEAP" and b[hp + 4] == 0
    hsize, hfree, hdata = _u(b, hp + 8), _u(b, hp + 16), _u(b, hp + 24)
    assert hfree == UNDEF and b[hdata] == 0
    assert b[bt:bt + 4] == b"TREE" and b[bt + 4] == 0 and b[bt + 5] == 0
    used = _u(b, bt + 6, 2)
    assert _u(b, bt + 8) == UNDEF and _u(b, bt + 16) == UNDEF
    name = lambda off: b[hdata + off:b.index(b"\0", hdata + off)].decode()  # noqa: E731
    keys = [_u(b, bt + 24 + 16 * i) for i in range(used + 1)]
    kids = [_u(b, bt + 32 + 16 * i) for i in range(used)]
    assert keys[0] == 0
    entries = []
    for i, k in enumerate(kids):
        assert b[k:k + 4] == b"SNOD" and b[k + 4] == 1
        ns = _u(b, k + 6, 2)
        assert 1 <= ns <= 8
        names = [name(_u(b, k + 8 + 40 * j)) for j in range(ns)]
        assert names == sorted(names) and names[-1] == name(keys[i + 1])
        entries += [(nm, _u(b, k + 16 + 40 * j)) for j, nm in enumerate(names)]
    assert [e[0] for e in entries] == sorted(e[0] for e in entries)
    return dict(entries), bt, hp


def _dataset(b, oh):
    ms = {t: (o, sz) for t, o, sz in _messages_v1(b, oh)}
    o, _ = ms[0x01]
    assert b[o] == 1
    rank = b[o + 1]
    dims = [_u(b, o + 8 + 8 * i) for i in range(rank)]
    o, _ = ms[0x03]
    cls, size = b[o] & 15, _u(b, o + 4, 4)
    o, _ = ms[0x08]
    assert b[o] == 3 and b[o + 1] == 1
    addr, nbytes = _u(b, o + 2), _u(b, o + 10)
    assert 0x05 in ms                                   # a fill value message
    dt = {(1, 8): "<f8", (0, 4): "<i4"}[(cls, size)]
    assert nbytes == int(np.prod(dims)) * size
    return np.frombuffer(b[addr:addr + nbytes], dtype=dt).reshape(dims)


def test_classic_structure_by_independent_parser(built, tmp_path):
    f = str(tmp_path / "c.h5")
    G = np.arange(24.0).reshape(4, 6)
    h5.write(f, "2048", {"IDADIM": np.array([6, 6, 4, 4], np.int32), "G": G, "D": np.ones(4)}, mode=0)
    h5.write(f, "extra", {f"x{i}": np.full(2, i * 1.0) for i in range(10)}, mode=1)
    b = open(f, "rb").read()
    assert b[:8] == b"\x89HDF\r\n\x1a\n" and b[8] == 0 and b[13] == 8 and b[14] == 8
    assert _u(b, 16, 2) == 4 and _u(b, 18, 2) == 16
    assert _u(b, 24) == 0 and _u(b, 32) == UNDEF and _u(b, 40) == len(b) and _u(b, 48) == UNDEF
    root = _u(b, 64)
    assert _u(b, 72, 4) == 1                             # cached B-tree and heap
    top, bt, hp = _group(b, root)
    assert (bt, hp) == (_u(b, 80), _u(b, 88))
    assert sorted(top) == ["2048", "extra"]
    g, _, _ = _group(b, top["2048"])
    assert np.array_equal(_dataset(b, g["G"]), G)
    assert np.array_equal(_dataset(b, g["IDADIM"]), [6, 6, 4, 4])
    x, _, _ = _group(b, top["extra"])
    assert len(x) == 10 and _dataset(b, x["x7"])[0] == 7.0


# ---- a file in the newer format, built here --------------------------------
def _ohdr_v2(msgs):
    body = b"".join(struct.pack("<BHB", t, len(d), 0) + d for t, d in msgs)
    head = b"OHDR" + bytes([2, 0x02]) + struct.pack("<I", len(body))   # 4-byte chunk size
    return head + body + b"\0\0\0\0"                                  # checksum (not verified)


def test_reader_newer_format(built, tmp_path):
    vals = np.array([1.5, -2.25, 3.0])
    ints = np.array([[1, 2], [3, 4], [5, 6]], dtype=np.int64)
    f64 = bytes([0x11, 0x20, 63, 0]) + struct.pack("<I", 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
    i64 = bytes([0x10, 0x08, 0, 0]) + struct.pack("<I", 8) + struct.pack("<HH", 0, 64)
    space = lambda dims: bytes([2, len(dims), 0, 1]) + b"".join(struct.pack("<Q", d) for d in dims)  # noqa: E731
    # layout: file = superblock v2 (48 bytes) | root OHDR | dataset A | dataset B | raw data of B
    sb_len = 8 + 4 + 8 * 4 + 4
    dsA = _ohdr_v2([(0x01, space([3])), (0x03, f64),
                    (0x08, bytes([3, 0]) + struct.pack("<H", 24) + vals.tobytes())])      # compact
    link = lambda name, addr: bytes([1, 0]) + bytes([len(name)]) + name + struct.pack("<Q", addr)  # noqa: E731
    root_len = len(_ohdr_v2([(0x06, link(b"A", 0)), (0x06, link(b"sub", 0))]))
    a_addr = sb_len + root_len
    b_addr = a_addr + len(dsA)
    dsB_tmp = _ohdr_v2([(0x01, space([3, 2])), (0x03, i64),
                        (0x08, bytes([3, 1]) + struct.pack("<QQ", 0, 48))])
    raw_addr = b_addr + len(dsB_tmp)
    dsB = _ohdr_v2([(0x01, space([3, 2])), (0x03, i64),
                    (0x08, bytes([3, 1]) + struct.pack("<QQ", raw_addr, 48))])
    sub_addr = raw_addr + 48
    sub = _ohdr_v2([(0x06, link(b"B", b_addr))])
    root = _ohdr_v2([(0x06, link(b"A", a_addr)), (0x06, link(b"sub", sub_addr))])
    eof = sub_addr + len(sub)
    sb = b"\x89HDF\r\n\x1a\n" + bytes([2, 8, 8, 0]) + struct.pack("<QQQQ", 0, UNDEF, eof, sb_len) + b"\0" * 4
    data = sb + root + dsA + dsB + ints.tobytes() + sub
    assert len(data) == eof
    f = tmp_path / "v2.h5"
    f.write_bytes(data)
    assert np.array_equal(h5.read(str(f), "A"), vals)
    assert np.array_equal(h5.read(str(f), "sub/B", as_float=False), ints.astype(np.int32))
    with pytest.raises(GjxError, match="classic-format"):
        h5.write(str(f), "g", {"A": np.ones(1)}, mode=2)


def test_dataset_extents_that_overflow_are_refused(built, tmp_path):
    """A file whose dataspace claims extents whose byte count wraps around 2^64
    (here 2^62 x 2^4 doubles) is refused with a message, not read."""
    f = tmp_path / "wrap.h5"
    h5.write(str(f), "g", {"A": np.ones((3, 7))}, mode=0)
    raw = bytearray(f.read_bytes())
    dims = struct.pack("<QQ", 3, 7)
    at = raw.find(dims)
    assert at > 0
    raw[at:at + 16] = struct.pack("<QQ", 1 << 62, 1 << 4)
    f.write_bytes(bytes(raw))
    with pytest.raises(GjxError, match="larger than the file"):
        h5.read(str(f), "g/A")
