"""Extract the reference's DEM viscous-tensor tables into a numpy fixture
(test infrastructure).

The reference reads `DEM/DEM_1e-3_vol{10,20,30}.h5` with HDF5.jl
(DEMloader, src/Rheology/anisotropy.jl:48-54: datasets "C", "ax", "vol").
Neither h5py nor libhdf5 is available here, so this script carries a minimal
reader for exactly what those files hold: superblock version 0, a root group
with compact link messages, and contiguous little-endian float64 datasets
(object headers of version 1 or 2).  Anything else raises.  HDF5 stores the
dimensions slowest-first; Julia writes column-major, so a Julia (100, 9)
matrix appears as (9, 100) and is transposed back here.

Run from the repository root with the reference tree at hand:
    python tests/golden/make_dem_fixture.py /path/to/reference/newDEM
Writes tests/golden/dem_1e-3_vol{10,20,30}.npz with C (n, 9), ax (n, 3), vol.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SIG = b"\x89HDF\r\n\x1a\n"


def _messages(b, oh):
    """(type, data offset, size) of every header message of the object at oh,
    following continuation blocks."""
    u = lambda off, n: int.from_bytes(b[off:off + n], "little")  # noqa: E731
    out = []
    if b[oh:oh + 4] == b"OHDR":                     # version-2 object header
        fl = b[oh + 5]
        p = oh + 6 + (16 if fl & 0x20 else 0) + (4 if fl & 0x10 else 0)
        nsz = 1 << (fl & 3)
        size = u(p, nsz)
        p += nsz
        blocks = [(p, p + size)]
        while blocks:
            p, end = blocks.pop(0)
            while p + 4 <= end:
                t, sz = b[p], u(p + 1, 2)
                p += 4 + (2 if fl & 0x04 else 0)
                out.append((t, p, sz))
                if t == 0x10:
                    a, ln = u(p, 8), u(p + 8, 8)
                    if b[a:a + 4] != b"OCHK":
                        raise ValueError("bad continuation block")
                    blocks.append((a + 4, a + ln - 4))
                p += sz
        return out
    if b[oh] != 1:
        raise ValueError("unsupported object header version %d" % b[oh])
    blocks = [(oh + 16, oh + 16 + u(oh + 8, 4))]
    while blocks:
        p, end = blocks.pop(0)
        while p + 8 <= end:
            t, sz = u(p, 2), u(p + 2, 2)
            out.append((t, p + 8, sz))
            if t == 0x10:
                blocks.append((u(p + 8, 8), u(p + 8, 8) + u(p + 16, 8)))
            p += 8 + sz
    return out


def read_h5(path):
    """{dataset name: array} of the root group's datasets."""
    b = open(path, "rb").read()
    if b[:8] != SIG or b[8] != 0 or b[13] != 8 or b[14] != 8:
        raise ValueError("expected an HDF5 superblock v0 with 8-byte offsets and lengths")
    u = lambda off, n: int.from_bytes(b[off:off + n], "little")  # noqa: E731
    root = u(24 + 4 * 8 + 8, 8)                       # root symbol-table entry: object header address
    links = []
    for t, d, _ in _messages(b, root):
        if t == 0x06:                                  # link message
            fl = b[d + 1]
            p = d + 2
            ltype = 0
            if fl & 8:
                ltype = b[p]
                p += 1
            if fl & 4:
                p += 8
            if fl & 16:
                p += 1
            nl = 1 << (fl & 3)
            ln = u(p, nl)
            p += nl
            name = b[p:p + ln].decode()
            p += ln
            if ltype != 0:
                raise ValueError("only hard links are supported")
            links.append((name, u(p, 8)))
    out = {}
    for name, oh in links:
        dims, dt, raw = None, None, None
        for t, d, _ in _messages(b, oh):
            if t == 0x01:                              # dataspace
                v, nd = b[d], b[d + 1]
                off = d + 8 if v == 1 else d + 4
                dims = [u(off + 8 * k, 8) for k in range(nd)]
            elif t == 0x03:                            # datatype
                cls, size = b[d] & 15, u(d + 4, 4)
                if b[d + 1] & 1:
                    raise ValueError("big-endian data")
                dt = {(1, 8): "<f8", (1, 4): "<f4", (0, 8): "<i8", (0, 4): "<i4"}[(cls, size)]
            elif t == 0x08:                            # data layout
                if b[d] != 3:
                    raise ValueError("layout message version %d" % b[d])
                if b[d + 1] == 1:
                    raw = b[u(d + 2, 8):u(d + 2, 8) + u(d + 10, 8)]
                elif b[d + 1] == 0:
                    raw = b[d + 4:d + 4 + u(d + 2, 2)]
                else:
                    raise ValueError("chunked dataset")
            elif t == 0x0B:
                raise ValueError("filtered dataset")
        a = np.frombuffer(raw, dtype=dt).copy()
        out[name] = a.reshape(dims) if dims else a
    return out


def main(src):
    for vol in (10, 20, 30):
        d = read_h5(os.path.join(src, "DEM_1e-3_vol%d.h5" % vol))
        C, ax = d["C"].T, d["ax"].T                     # back to the Julia (n, 9) and (n, 3)
        assert C.shape[1] == 9 and ax.shape[1] == 3 and C.shape[0] == ax.shape[0]
        np.savez(os.path.join(HERE, "dem_1e-3_vol%d.npz" % vol), C=C, ax=ax, vol=d["vol"])
        print("vol%d: %d rows" % (vol, C.shape[0]))


if __name__ == "__main__":
    main(sys.argv[1])
