"""Learned initial guess for the Schur PCG (host side of the dp_cnn C ABI).

The network maps the material of a context, sampled on the half-resolution
vertex grid (dp_cnn_inputs: rho, log10 eta, cos 2phi, sin 2phi), to P/g on
that grid; dp_guess_from_grid prolongates it to the pressure DOFs, and
dp_solve(use_guess=2) keeps it only if its initial Schur residual is below
the zero guess's, stopping at rtol relative to the zero-guess residual.
Training, forward and backward run in the library's own kernels.
"""
import ctypes as C
import json
import os

import numpy as np

from . import _lib
from ._lib import DP_MEM_DEVICE, check, lib

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "weights")
DEFAULT_ARCH = dict(channels=32, layers=6, dilations=(1, 2, 4, 8, 16, 1))


def grid_shape(nr_cells, ntheta_cells):
    return nr_cells // 2 + 1, ntheta_cells // 2


class GuessNet:
    def __init__(self, nrg, ntg, channels=16, layers=6, dilations=(1, 2, 4, 8, 16, 1), max_batch=8, device=0):
        self.nrg, self.ntg, self.channels, self.layers = nrg, ntg, channels, layers
        self.dilations = tuple(dilations)
        self.max_batch = max_batch
        self.h = C.c_void_p()
        dil = (C.c_int32 * layers)(*self.dilations)
        check(lib().dp_cnn_create(nrg, ntg, channels, layers, dil, max_batch, device, C.byref(self.h)))
        self.n = int(lib().dp_cnn_num_params(self.h))
        self.bf16 = True
        self.x_mean = np.zeros(4, np.float32)
        self.x_std = np.ones(4, np.float32)
        self.y_mean, self.y_std = 0.0, 1.0

    def set_math(self, bf16=True):
        """BF16 tensor-core convolutions (FP32 accumulation; the default) or
        FP32 CUDA-core convolutions."""
        check(lib().dp_cnn_set_math(self.h, 1 if bf16 else 0))
        self.bf16 = bool(bf16)

    def close(self):
        if self.h:
            lib().dp_cnn_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- parameters ----------------------------------------------------------
    def init_params(self, seed=0):
        """He-uniform weights, zero biases (layer layout: W[cout][cin][3][3], b[cout])."""
        rng = np.random.default_rng(seed)
        p = np.zeros(self.n, np.float32)
        off = 0
        for l in range(self.layers):
            cin = 4 if l == 0 else self.channels
            cout = 1 if l == self.layers - 1 else self.channels
            nw = cout * cin * 9
            lim = np.sqrt(6.0 / (cin * 9))
            p[off:off + nw] = rng.uniform(-lim, lim, nw) * (0.1 if l == self.layers - 1 else 1.0)
            off += nw + cout
        self.set_params(p)

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        check(lib().dp_cnn_set_params(self.h, C.c_void_p(p.ctypes.data), p.size))

    def get_params(self, grads=False):
        p = np.empty(self.n, np.float32)
        g = np.empty(self.n, np.float32) if grads else None
        check(lib().dp_cnn_get_params(self.h, C.c_void_p(p.ctypes.data),
                                      C.c_void_p(g.ctypes.data) if grads else None, self.n))
        return (p, g) if grads else p

    # ---- compute (device pointers of float32 torch tensors) -------------------------
    def forward(self, x, y):
        check(lib().dp_cnn_forward(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), x.shape[0]))

    def gradients(self, x, t):
        loss = C.c_double(0.0)
        check(lib().dp_cnn_gradients(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(t.data_ptr()), x.shape[0],
                                     C.byref(loss)))
        return loss.value

    def train_step(self, x, t, lr):
        loss = C.c_double(0.0)
        check(lib().dp_cnn_train_step(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(t.data_ptr()), x.shape[0],
                                      C.c_float(lr), C.byref(loss)))
        return loss.value

    def for_grid(self, nrg, ntg, max_batch=1, device=0):
        """The same network (weights and normalisation) on another grid: the
        layers are convolutions, so they apply unchanged at any resolution."""
        net = GuessNet(nrg, ntg, self.channels, self.layers, self.dilations, max_batch, device)
        net.set_params(self.get_params())
        net.x_mean, net.x_std = self.x_mean, self.x_std
        net.y_mean, net.y_std = self.y_mean, self.y_std
        net.meta = dict(getattr(self, "meta", {}), nrg=nrg, ntg=ntg)
        return net

    # ---- persistence -------------------------------------------------------------
    def save(self, path, extra=None):
        meta = dict(nrg=self.nrg, ntg=self.ntg, channels=self.channels, layers=self.layers,
                    dilations=list(self.dilations), y_mean=self.y_mean, y_std=self.y_std)
        if extra:
            meta.update(extra)
        np.savez_compressed(path, params=self.get_params(), x_mean=self.x_mean, x_std=self.x_std,
                            meta=json.dumps(meta))

    @classmethod
    def load(cls, path, max_batch=8, device=0):
        d = np.load(path)
        meta = json.loads(str(d["meta"]))
        net = cls(meta["nrg"], meta["ntg"], meta["channels"], meta["layers"], meta["dilations"], max_batch, device)
        net.set_params(d["params"])
        net.x_mean, net.x_std = d["x_mean"], d["x_std"]
        net.y_mean, net.y_std = float(meta["y_mean"]), float(meta["y_std"])
        net.meta = meta
        return net


def weights_path(nr_cells, ntheta_cells):
    return os.path.join(WEIGHTS, f"guess_{nr_cells}x{ntheta_cells}.npz")


def features(ctx, out):
    """Raw network inputs of a context into the (1, 4, nrg, ntg) float32 device tensor `out`."""
    nrg, ntg = grid_shape(ctx.desc.nr_cells, ctx.desc.ntheta_cells)
    ctx._chk(lib().dp_cnn_inputs(ctx.h, C.c_void_p(out.data_ptr()), nrg, ntg))


def vertex_target(mesh, P, g):
    """Training target: P/g averaged to the mesh vertices, sampled at the
    half-resolution vertex grid -> (nrg, ntg)."""
    ncr, nct = mesh.nr_cells, mesh.ntheta_cells
    nv = (ncr + 1) * nct
    if mesh.pressure == "discontinuous":
        v = mesh.e2n[:3].T.ravel()
        pv = np.bincount(v, weights=P, minlength=nv) / np.bincount(v, minlength=nv)
    else:
        pv = P.copy()
    pv = pv.reshape(nct, ncr + 1)            # vertex = ir + (ncr+1) * it
    return (pv[::2, ::2].T / g).astype(np.float32)


class LearnedGuess:
    """Device pipeline: features -> normalised CNN forward -> prolongation."""

    def __init__(self, net, ctx):
        import torch
        self.net, self.ctx = net, ctx
        dev = torch.device("cuda", ctx.desc.device)
        self.x = torch.empty((1, 4, net.nrg, net.ntg), dtype=torch.float32, device=dev)
        self.y = torch.empty((1, 1, net.nrg, net.ntg), dtype=torch.float32, device=dev)
        self.xm = torch.tensor(net.x_mean, device=dev).view(1, 4, 1, 1)
        self.xs = torch.tensor(net.x_std, device=dev).view(1, 4, 1, 1)

    def predict(self, g, P_out_ptr, mem=DP_MEM_DEVICE):
        """Write the guess for the context's current material into P (device
        pointer by default)."""
        features(self.ctx, self.x)
        self.x.sub_(self.xm).div_(self.xs)
        self.net.forward(self.x, self.y)
        self.y.mul_(self.net.y_std).add_(self.net.y_mean)
        self.ctx._chk(lib().dp_guess_from_grid(self.ctx.h, C.c_void_p(self.y.data_ptr()), self.net.nrg, self.net.ntg,
                                               float(g), C.c_void_p(P_out_ptr), mem))
