"""Snapshot files in the reference's HDF5 layout (savedata, IOmanager.jl:
17-114), written and read without an HDF5 library: round trips, the
structures compared with what libhdf5 writes, and the reader on the HDF5
files the reference ships (when that tree is at hand)."""
import os
import struct

import numpy as np
import pytest

from dimspers_b200 import snapshot as S

# the reference's source tree, named by the caller (unset: those comparisons skip)
REFERENCE = os.environ.get("DIMSPERS_REFERENCE")
DEM_H5 = os.path.join(REFERENCE, "newDEM", "DEM_1e-3_vol30.h5") if REFERENCE else None

# message bodies as libhdf5 wrote them in the reference's DEM files: the
# float64 datatype (class 1, version 1, IEEE little-endian) and the fill value
LIBHDF5_F64 = bytes.fromhex("11203f000800000000004000340b0034ff03000000000000")
LIBHDF5_FILL = bytes.fromhex("0202020100000000")


def _messages(b, oh):
    n = struct.unpack_from("<H", b, oh + 2)[0]
    size = struct.unpack_from("<I", b, oh + 8)[0]
    p, out = oh + 16, []
    while p < oh + 16 + size and len(out) < n:
        t, sz, fl = struct.unpack_from("<HHB", b, p)
        out.append((t, fl, b[p + 8:p + 8 + sz]))
        p += 8 + sz
    return out


def _fields(nel, nnod, rng):
    return dict(Upolar=rng.standard_normal(2 * nnod), Ucartesian=rng.standard_normal(2 * nnod),
                T=rng.random(nnod), eta_node=rng.random(nnod), eta_ip=rng.random((nel, 7)),
                strain={k: rng.standard_normal((nel, 7)) for k in ("xx", "zz", "xz")}, rho=rng.random(nnod),
                F=rng.standard_normal((nel, 6, 2, 2)),
                fse={k: rng.random((nel, 6)) for k in ("x1", "x2", "y1", "y2", "a1", "a2")})


def test_savedata_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    nel, nnod = 64, 2 * 5 * 16
    f = _fields(nel, nnod, rng)
    p = str(tmp_path / "file_0.h5")
    S.savedata(p, ntheta=16, nr=3, time2save=2.5e13, **f)
    r = S.read(p)
    assert sorted(r) == ["MESH", "PART", "Time", "VAR"] and r["PART"] == {}
    assert r["MESH"]["nθ"] == 16 and r["MESH"]["nr"] == 3 and r["Time"]["t"] == 2.5e13
    assert list(r["VAR"]) == list(S.VAR_NAMES)
    v = r["VAR"]
    assert np.array_equal(v["nu_ip"], f["eta_ip"]) and v["nu_ip"].shape == (nel, 7)
    assert np.array_equal(v["Utheta"], f["Upolar"][0::2]) and np.array_equal(v["Ur"], f["Upolar"][1::2])
    assert np.array_equal(v["Ux"], f["Ucartesian"][0::2]) and np.array_equal(v["Uz"], f["Ucartesian"][1::2])
    assert np.array_equal(v["Fxz"], f["F"][..., 0, 1]) and np.array_equal(v["Fzx"], f["F"][..., 1, 0])
    assert np.array_equal(v["strain_xz"], f["strain"]["xz"]) and np.array_equal(v["y2"], f["fse"]["y2"])


def test_layout_matches_libhdf5_structures(tmp_path):
    """Superblock version 0 with 8-byte offsets, an (nel, 7) array stored as
    dimensions (7, nel) over its column-major bytes, and dataset headers with
    libhdf5's message types, versions, flags and encodings."""
    a = np.arange(21.0).reshape(3, 7)
    p = str(tmp_path / "x.h5")
    S.write(p, {"g": {"a": a, "n": np.int64(5)}})
    b = open(p, "rb").read()
    assert b[:8] == S.SIGNATURE and b[8:16] == bytes([0, 0, 0, 0, 0, 8, 8, 0])
    assert struct.unpack_from("<Q", b, 40)[0] == len(b)                    # end-of-file address
    root = struct.unpack_from("<Q", b, 64)[0]
    rm = _messages(b, root)
    assert [m[0] for m in rm] == [0x2, 0xA, 0x6]
    g = struct.unpack_from("<Q", rm[2][2], 4 + 1)[0]                       # link "g" -> its header
    gm = _messages(b, g)
    assert [m[0] for m in gm] == [0x2, 0xA, 0x6, 0x6]
    link_a = gm[2][2]
    assert link_a[:5] == bytes([1, 0x10, 1, 1]) + b"a"
    dm = _messages(b, struct.unpack_from("<Q", link_a, 5)[0])
    assert [(t, fl) for t, fl, _ in dm] == [(0x1, 0), (0x3, 1), (0x5, 1), (0x8, 0)]
    assert dm[0][2] == struct.pack("<BBB5xQQQQ", 1, 2, 1, 7, 3, 7, 3)
    assert dm[1][2] == LIBHDF5_F64 and dm[2][2] == LIBHDF5_FILL
    assert dm[3][2][:2] == bytes([3, 1])
    addr, size = struct.unpack_from("<QQ", dm[3][2], 2)
    assert size == a.nbytes and b[addr:addr + size] == np.asfortranarray(a).tobytes(order="F")


@pytest.mark.skipif(DEM_H5 is None or not os.path.exists(DEM_H5),
                    reason="DIMSPERS_REFERENCE does not name the reference tree")
def test_reader_reads_files_libhdf5_wrote():
    """The reference's DEM tables, written by Julia through libhdf5: the same
    values as the committed fixture, and dataset headers whose messages ours
    reproduce (datatype and fill value bodies, flags)."""
    r = S.read(DEM_H5)
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "dem_1e-3_vol30.npz"))
    assert np.array_equal(r["C"], d["C"]) and np.array_equal(r["ax"], d["ax"]) and r["vol"] == 0.3
    b = open(DEM_H5, "rb").read()
    root = struct.unpack_from("<Q", b, 64)[0]
    oh = None
    for t, d_off, _ in S._read_messages(b, root):
        if t == 0x6 and b[d_off + 4:d_off + 6] == b"ax":
            oh = struct.unpack_from("<Q", b, d_off + 6)[0]
    ms = _messages(b, oh)
    kinds = {t: (fl, body) for t, fl, body in ms}
    assert kinds[0x3] == (1, LIBHDF5_F64) and kinds[0x5] == (1, LIBHDF5_FILL)
    assert kinds[0x1][1][:3] == bytes([1, 2, 1]) and kinds[0x8][1][:2] == bytes([3, 1])
