"""Snapshot files in the reference's HDF5 layout, without an HDF5 library.

savedata (src/IO/IOmanager.jl:17-114) writes one HDF5 file per output step
with four groups: MESH (scalars "nθ", "nr"), VAR (the fields: "nu_node",
"nu_ip", "strain_xx", "strain_zz", "strain_xz", "Ux", "Uz", "Utheta", "Ur",
"T", "density", "Fxx", "Fzz", "Fxz", "Fzx", "a1", "a2", "x1", "x2", "y1",
"y2"), PART (empty: its writes are commented out) and Time (scalar "t").
No HDF5 library exists in this image, so this module writes the subset of
the format such a file needs, with the structures libhdf5 itself writes for
that subset (as seen in the HDF5 files shipped with the reference):

* superblock version 0, 8-byte offsets and lengths, the root symbol-table
  entry caching an empty version-1 group B-tree and local heap;
* every group a version-1 object header holding a Link Info message (no
  fractal heap, no name index), a Group Info message and one compact hard
  Link message (UTF-8 name) per member;
* every dataset a version-1 object header with a version-1 dataspace (rank
  0 for scalars; for arrays the dimensions and equal maximum dimensions),
  a version-1 datatype (IEEE little-endian float64 or signed little-endian
  int64, flagged constant), a version-2 fill-value message and a version-3
  contiguous layout, the raw data stored after the metadata.

Julia writes arrays column-major and HDF5 lists dimensions slowest first, so
an (nel, 7) matrix is stored with dimensions (7, nel) over its column-major
bytes; `write` and `read` apply that convention to numpy arrays, so a
round trip returns the shapes the reference uses.
"""
import struct

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF
_GROUP_K_LEAF, _GROUP_K_INTERNAL = 4, 16
_BTREE_SIZE = 24 + (2 * _GROUP_K_INTERNAL + 1) * 8 + 2 * _GROUP_K_INTERNAL * 8   # empty group node
_HEAP_DATA = 88                                                                   # empty name + one free block

VAR_NAMES = ("nu_node", "nu_ip", "strain_xx", "strain_zz", "strain_xz", "Ux", "Uz", "Utheta", "Ur", "T",
             "density", "Fxx", "Fzz", "Fxz", "Fzx", "a1", "a2", "x1", "x2", "y1", "y2")


def _pad8(n):
    return (n + 7) & ~7


def _msg(mtype, body, flags=0):
    body = body + b"\0" * (_pad8(len(body)) - len(body))
    return struct.pack("<HHB3x", mtype, len(body), flags) + body


def _header(messages):
    """Version-1 object header: prefix (12 bytes + 4 of alignment) and messages."""
    blob = b"".join(messages)
    return struct.pack("<BBHII4x", 1, 0, len(messages), 1, len(blob)) + blob


def _dataspace(shape):
    rank = len(shape)
    flags = 1 if rank else 0                  # maximum dimensions present (equal to the dimensions)
    body = struct.pack("<BBB5x", 1, rank, flags)
    body += b"".join(struct.pack("<Q", d) for d in shape)
    if rank:
        body += b"".join(struct.pack("<Q", d) for d in shape)
    return _msg(0x0001, body)


def _datatype(dtype):
    if dtype == np.float64:
        # class 1 (floating point) version 1; little-endian, implied mantissa
        # bit, sign at bit 63; exponent at 52 (11 bits, bias 1023), mantissa
        # at 0 (52 bits)
        body = bytes([0x11, 0x20, 0x3F, 0x00]) + struct.pack("<I", 8)
        body += struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
    elif dtype == np.int64:
        # class 0 (fixed point) version 1; little-endian, signed
        body = bytes([0x10, 0x08, 0x00, 0x00]) + struct.pack("<I", 8) + struct.pack("<HH", 0, 64)
    else:
        raise TypeError("only float64 and int64 datasets are written")
    return _msg(0x0003, body, flags=1)


def _fill_value():
    return _msg(0x0005, bytes([2, 2, 2, 1]) + struct.pack("<I", 0), flags=1)


def _layout(addr, size):
    return _msg(0x0008, struct.pack("<BBQQ", 3, 1, addr, size))


def _link(name, addr):
    nb = name.encode("utf-8")
    if len(nb) > 255:
        raise ValueError("link names are limited to 255 bytes")
    return _msg(0x0006, bytes([1, 0x10, 1, len(nb)]) + nb + struct.pack("<Q", addr))


def _group_header(links):
    msgs = [_msg(0x0002, struct.pack("<BBQQ", 0, 0, UNDEF, UNDEF)), _msg(0x000A, struct.pack("<BB", 0, 0))]
    msgs += [_link(n, a) for n, a in links]
    return _header(msgs)


def _as_data(v):
    """(stored dims, dtype, raw bytes) of a value: reference-orientation
    arrays are stored column-major with their dimensions reversed."""
    a = np.asarray(v)
    if a.dtype.kind == "f":
        a = a.astype(np.float64, copy=False)
    elif a.dtype.kind in "iub":
        a = a.astype(np.int64, copy=False)
    else:
        raise TypeError("datasets hold float64 or int64 values")
    if a.ndim == 0:
        return (), a.dtype, a.tobytes()
    return tuple(reversed(a.shape)), a.dtype, np.asfortranarray(a).tobytes(order="F")


def write(path, tree):
    """Write a nested dict (group name -> dict, dataset name -> array or
    scalar) as an HDF5 file."""
    # pass 1: flatten the objects in depth-first order and size their headers
    objs = []                                  # (kind, payload, header size)

    def visit(node):
        idx = len(objs)
        if isinstance(node, dict):
            objs.append(["group", node, len(_group_header([(n, 0) for n in node]))])
            kids = [visit(child) for child in node.values()]
            objs[idx].append(kids)
        else:
            dims, dt, raw = _as_data(node)
            hdr = _header([_dataspace(dims), _datatype(dt), _fill_value(), _layout(0, 0)])
            objs.append(["data", (dims, dt, raw), len(hdr), None])
        return idx

    visit(tree)
    btree = 96
    heap = btree + _BTREE_SIZE
    heap_data = heap + 32
    addr = heap_data + _HEAP_DATA
    for o in objs:
        o.append(addr)
        addr += o[2]
    for o in objs:                              # raw data after all metadata, 8-byte aligned
        if o[0] == "data":
            addr = _pad8(addr)
            o.append(addr if len(o[1][2]) else UNDEF)
            addr += len(o[1][2])
    eof = _pad8(addr)

    # pass 2: emit
    out = bytearray(eof)
    out[0:96] = (SIGNATURE + bytes([0, 0, 0, 0, 0, 8, 8, 0])
                 + struct.pack("<HHI", _GROUP_K_LEAF, _GROUP_K_INTERNAL, 0)
                 + struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
                 + struct.pack("<QQI4xQQ", 0, objs[0][4], 1, btree, heap))
    out[btree:btree + 24] = b"TREE" + struct.pack("<BBHQQ", 0, 0, 0, UNDEF, UNDEF)
    out[heap:heap + 32] = b"HEAP" + struct.pack("<B3xQQQ", 0, _HEAP_DATA, 8, heap_data)
    out[heap_data + 8:heap_data + 24] = struct.pack("<QQ", 1, _HEAP_DATA - 8)
    for o in objs:
        if o[0] == "group":
            names = list(o[1].keys())
            hdr = _group_header([(n, objs[k][4]) for n, k in zip(names, o[3])])
            at = o[4]
        else:
            dims, dt, raw = o[1]
            hdr = _header([_dataspace(dims), _datatype(dt), _fill_value(), _layout(o[5], len(raw))])
            at = o[4]
            if raw:
                out[o[5]:o[5] + len(raw)] = raw
        assert len(hdr) == o[2]
        out[at:at + len(hdr)] = hdr
    with open(path, "wb") as f:
        f.write(bytes(out))


def _read_messages(b, oh):
    """(type, data offset, size) of a version-1 object header's messages,
    following continuation blocks."""
    if b[oh] != 1:
        raise ValueError("only version-1 object headers are read")
    nmsg = struct.unpack_from("<H", b, oh + 2)[0]
    blocks = [(oh + 16, oh + 16 + struct.unpack_from("<I", b, oh + 8)[0])]
    out = []
    while blocks and len(out) < nmsg:
        p, end = blocks.pop(0)
        while p + 8 <= end and len(out) < nmsg:
            t, sz = struct.unpack_from("<HH", b, p)
            out.append((t, p + 8, sz))
            if t == 0x0010:
                a, ln = struct.unpack_from("<QQ", b, p + 8)
                blocks.append((a, a + ln))
            p += 8 + sz
    return out


def _read_object(b, oh):
    msgs = _read_messages(b, oh)
    links = []
    dims = dt = raw = None
    for t, d, _ in msgs:
        if t == 0x0006:                              # link: version, flags, [type], [order], [charset], name, address
            fl = b[d + 1]
            p = d + 2 + (1 if fl & 8 else 0) + (8 if fl & 4 else 0) + (1 if fl & 16 else 0)
            if fl & 8 and b[d + 2] != 0:
                raise ValueError("only hard links are read")
            nlen_size = 1 << (fl & 3)
            nlen = int.from_bytes(b[p:p + nlen_size], "little")
            p += nlen_size
            links.append((b[p:p + nlen].decode("utf-8"), struct.unpack_from("<Q", b, p + nlen)[0]))
        elif t == 0x0001:
            rank = b[d + 1]
            off = d + 8 if b[d] == 1 else d + 4
            dims = struct.unpack_from("<%dQ" % rank, b, off)
        elif t == 0x0003:
            cls, size = b[d] & 15, struct.unpack_from("<I", b, d + 4)[0]
            if b[d + 1] & 1:
                raise ValueError("big-endian data")
            dt = {(1, 8): "<f8", (1, 4): "<f4", (0, 8): "<i8", (0, 4): "<i4"}[(cls, size)]
        elif t == 0x0008:
            if b[d] != 3:
                raise ValueError("layout message version %d" % b[d])
            if b[d + 1] == 1:
                a, n = struct.unpack_from("<QQ", b, d + 2)
                raw = b"" if a == UNDEF else b[a:a + n]
            elif b[d + 1] == 0:
                n = struct.unpack_from("<H", b, d + 2)[0]
                raw = b[d + 4:d + 4 + n]
            else:
                raise ValueError("chunked datasets are not read")
        elif t == 0x000B:
            raise ValueError("filtered datasets are not read")
    if dt is None:
        return {name: _read_object(b, a) for name, a in links}
    a = np.frombuffer(raw, dtype=dt).copy()
    if not dims:
        return a[0] if a.size else a
    return a.reshape(dims).T                         # back to the column-major (reference) orientation


def read(path):
    """Read a file written by `write` (or any file made of the structures it
    writes) into the nested dict it came from."""
    b = open(path, "rb").read()
    if b[:8] != SIGNATURE or b[8] != 0 or b[13] != 8 or b[14] != 8:
        raise ValueError("expected an HDF5 superblock version 0 with 8-byte offsets and lengths")
    root = struct.unpack_from("<Q", b, 24 + 4 * 8 + 8)[0]
    return _read_object(b, root)


def savedata(path, Upolar, Ucartesian, T, eta_node, eta_ip, strain, rho, F, fse, ntheta, nr, time2save):
    """savedata(OUT, Upolar, Ucartesian, T, η, 𝓒, ρ, ε, F, FSE, nθ, nr, ...,
    time2save, ::Val{Isotropic}) (IOmanager.jl:17-114): U vectors interleaved
    per node (u_theta, u_r) and (u_x, u_z); T, rho, eta_node nodal; eta_ip and
    strain["xx"|"zz"|"xz"] (nel, 7); F (nel, 6, 2, 2); fse["x1"|"x2"|"y1"|
    "y2"|"a1"|"a2"] (nel, 6)."""
    F = np.asarray(F, dtype=np.float64)
    var = {"nu_node": eta_node, "nu_ip": eta_ip, "strain_xx": strain["xx"], "strain_zz": strain["zz"],
           "strain_xz": strain["xz"], "Ux": np.asarray(Ucartesian)[0::2], "Uz": np.asarray(Ucartesian)[1::2],
           "Utheta": np.asarray(Upolar)[0::2], "Ur": np.asarray(Upolar)[1::2], "T": T, "density": rho,
           "Fxx": F[..., 0, 0], "Fzz": F[..., 1, 1], "Fxz": F[..., 0, 1], "Fzx": F[..., 1, 0],
           "a1": fse["a1"], "a2": fse["a2"], "x1": fse["x1"], "x2": fse["x2"], "y1": fse["y1"], "y2": fse["y2"]}
    tree = {"MESH": {"nθ": np.int64(ntheta), "nr": np.int64(nr)},
            "VAR": {k: var[k] for k in VAR_NAMES},
            "PART": {},
            "Time": {"t": np.float64(time2save)}}
    write(path, tree)
