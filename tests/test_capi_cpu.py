"""C-ABI library checks that need no GPU: it loads, exports every symbol
declared in include/dimspers_b200.h, and its host mesh builder reproduces the
oracle's literal restatement of Grid_split1 / edge_connectivity / color_mesh
bit-exactly."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from dimspers_b200 import _lib, build_mesh
from oracle import mesh as OM


def header_symbols():
    src = open(os.path.join(ROOT, "include", "dimspers_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dp_[A-Za-z_0-9]+)\s*\(", src)))


def test_library_loads_and_exports_header_symbols():
    L = _lib.lib()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(_lib.SIGNATURES), set(syms) ^ set(_lib.SIGNATURES)


def test_status_strings():
    L = _lib.lib()
    assert L.dp_status_string(0) == b"OK"
    assert L.dp_status_string(2) == b"BREAKDOWN"
    assert L.dp_status_string(99) == b"UNKNOWN"


@pytest.mark.parametrize("ncr,nct", [(1, 3), (2, 5), (3, 17), (4, 32), (8, 64)])
def test_mesh_bit_exact_vs_literal_oracle(ncr, nct):
    g = OM.grid_cells(ncr, nct, literal=True)
    colors, color_list = OM.color_mesh(g.e2n)
    m = build_mesh(ncr, nct, pin_rotation=False)
    assert np.array_equal(m.e2n, g.e2n)
    assert np.array_equal(m.theta, g.theta)
    assert np.array_equal(m.r, g.r)
    assert np.array_equal(m.colors, colors)
    assert m.ncolors == len(color_list)
    om, _ = OM.free_slip(g)
    assert np.array_equal(m.omega, om)


def test_mesh_bit_exact_config1_size():
    g = OM.grid_cells(32, 256)          # vectorised first-seen numbering
    m = build_mesh(32, 256, pin_rotation=True)
    assert np.array_equal(m.e2n, g.e2n)
    assert np.array_equal(m.theta, g.theta) and np.array_equal(m.r, g.r)
    om, _ = OM.free_slip(g, pin_rotation=True)
    assert np.array_equal(m.omega, om)
    assert m.nel == 16384 and m.nnod == 33280


def test_colouring_is_valid():
    m = build_mesh(16, 128)
    els = m.e2n[:3]
    for c in range(1, m.ncolors + 1):
        ids = np.flatnonzero(m.colors == c)
        nodes = els[:, ids].ravel()
        assert np.unique(nodes).size == nodes.size, c


def test_bad_arguments_are_reported():
    with pytest.raises(_lib.DPError) as e:
        build_mesh(0, 8)
    assert e.value.status == _lib.DP_BAD_ARG
    with pytest.raises(_lib.DPError):
        build_mesh(4, 2)


def test_sizes_match_the_split1_formulas():
    for (ncr, nct), (nel, nnod, npd) in {(32, 256): (16384, 33280, 49152),
                                         (128, 1024): (262144, 526336, 786432)}.items():
        d = _lib.MeshDesc(ncr, nct, 1.22, 2.22, 1, 0, 1)
        import ctypes as C
        a, b, c_, f = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        assert _lib.lib().dp_mesh_sizes(C.byref(d), C.byref(a), C.byref(b), C.byref(c_), C.byref(f)) == 0
        assert (a.value, b.value, c_.value) == (nel, nnod, npd)
        assert f.value == 2 * 2 * nct + 1


def _header_struct_fields(name):
    """Field names of a typedef struct { ... } name; in the C header, in order."""
    hdr = open(os.path.join(ROOT, "include", "dimspers_b200.h")).read()
    end = hdr.index("} " + name + ";")
    start = hdr.rindex("typedef struct {", 0, end) + len("typedef struct {")
    body = hdr[start:end]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        parts = decl.split(",")
        fields += [parts[0].split()[-1].lstrip("*")] + [p.strip().lstrip("*") for p in parts[1:]]
    return fields


@pytest.mark.parametrize("cname,pystruct", [("dp_solve_opts", "SolveOpts"), ("dp_solve_report", "SolveReport"),
                                            ("dp_mesh_desc", "MeshDesc"), ("dp_arrhenius", "Arrhenius"),
                                            ("dp_dem", "Dem"),
                                            ("dp_thermal_opts", "ThermalOpts")])
def test_ctypes_structs_mirror_the_header(cname, pystruct):
    """The ctypes mirrors list the header's fields in the header's order."""
    py = [f for f, _ in getattr(_lib, pystruct)._fields_]
    assert py == _header_struct_fields(cname)


def test_default_opts_fill_exactly_the_struct():
    """dp_default_opts writes the whole options struct and nothing beyond it
    (a shorter mirror would let the library write past the caller's buffer)."""
    import ctypes as C
    n = C.sizeof(_lib.SolveOpts)
    buf = (C.c_ubyte * (n + 64))(*([0xAB] * (n + 64)))
    _lib.lib().dp_default_opts(C.cast(buf, C.POINTER(_lib.SolveOpts)))
    assert bytes(buf[n:]) == bytes([0xAB] * 64)
    o = _lib.SolveOpts.from_buffer(buf)
    assert (o.rtol, o.itmax, o.itmin, o.cheb_degree, o.coarse_max) == (1e-8, 200, 10, 3, 1536)
    assert (o.launch_overlap, o.true_residual, o.matrix_free, o.mg_tail, o.relax_base) == (1, 1, 0, 0, 0.0)


def test_default_thermal_opts():
    """dp_default_thermal_opts fills exactly the struct: MAIN.jl's thermal
    parameters (K = 3.3, Cp = 1.2e3, walls 300 / 4000, heated) and Krylov.jl's
    default tolerances sqrt(eps)."""
    import ctypes as C
    n = C.sizeof(_lib.ThermalOpts)
    buf = (C.c_ubyte * (n + 32))(*([0xCD] * (n + 32)))
    _lib.lib().dp_default_thermal_opts(C.cast(buf, C.POINTER(_lib.ThermalOpts)))
    assert bytes(buf[n:]) == bytes([0xCD] * 32)
    o = _lib.ThermalOpts.from_buffer(buf)
    assert (o.K, o.Cp, o.Ttop, o.Tbot, o.heated, o.itmax) == (3.3, 1.2e3, 300.0, 4000.0, 1, 0)
    assert o.rtol == o.atol == np.sqrt(np.finfo(np.float64).eps)
