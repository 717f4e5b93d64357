"""dp_apply_K_noalloc: the K-apply for callers that cannot allocate device
memory (a host whose own allocator owns the device memory, a real-time loop
that forbids allocation after start-up).  Its staging vectors live in a
static device array of the library instead of context work buffers; this
file checks it against dp_apply_K through the C ABI on two calls in a row (the
shared array keeps the previous call's contents), and that meshes beyond the
array's size are refused.  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel
from dimspers_b200 import StokesContext, _lib, build_mesh, inputs

pytestmark = pytest.mark.gpu


def test_apply_K_noalloc_matches_apply_K_twice():
    import torch
    mesh = build_mesh(32, 256, "discontinuous")
    mat = inputs.make_material(mesh, "aniso", seed=21)
    rng = np.random.default_rng(3)
    with StokesContext(32, 256, "discontinuous") as ctx:
        ctx.set_material(mat.eta_ip, mat.rho, mat.g, mat.C6)
        ctx.assemble(0)
        for call in range(2):
            x = rng.standard_normal(2 * ctx.nnod)
            y_ref = ctx.apply_K(x)
            xd = torch.from_numpy(x).cuda()
            yd = torch.full_like(xd, float("nan"))
            torch.cuda.synchronize()
            st = _lib.lib().dp_apply_K_noalloc(ctx.h, C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr()))
            assert st == 0, _lib.lib().dp_last_error(ctx.h)
            y = yd.cpu().numpy()
            assert np.all(np.isfinite(y))
            assert rel(y, y_ref) < 1e-13, (call, rel(y, y_ref))


def test_apply_K_noalloc_rejects_meshes_beyond_the_scratch():
    import torch
    with StokesContext(256, 2048, "discontinuous") as ctx:   # 2,101,248 nodes > 1,048,576
        xd = torch.zeros(2 * ctx.nnod, dtype=torch.float64, device="cuda")
        yd = torch.zeros_like(xd)
        st = _lib.lib().dp_apply_K_noalloc(ctx.h, C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr()))
        assert st == _lib.DP_BAD_ARG
        assert b"static scratch" in _lib.lib().dp_last_error(ctx.h)
