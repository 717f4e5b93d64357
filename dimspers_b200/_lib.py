"""ctypes binding of libdimspers_b200.so (the C ABI in include/dimspers_b200.h).

The library is built in-tree (``python -m dimspers_b200.build``).  There is
no CPU fallback: if the shared library is missing, importing the solver API
raises immediately.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdimspers_b200.so")

DP_OK, DP_NOT_CONVERGED, DP_BREAKDOWN, DP_BAD_ARG, DP_CUDA_ERROR, DP_DEVICE_TIMEOUT = range(6)
DP_PRESSURE_CONTINUOUS, DP_PRESSURE_DISCONTINUOUS = 0, 1
DP_PREC_FP64, DP_PREC_FP32_REFINED, DP_PREC_FP32_IR = 0, 1, 2
DP_MEM_HOST, DP_MEM_DEVICE = 0, 1
DP_INNER_MG, DP_INNER_JACOBI = 0, 1


class MeshDesc(C.Structure):
    _fields_ = [("nr_cells", C.c_int32), ("ntheta_cells", C.c_int32), ("r_in", C.c_double),
                ("r_out", C.c_double), ("pressure_space", C.c_int32), ("device", C.c_int32),
                ("pin_rotation", C.c_int32)]


class SolveOpts(C.Structure):
    _fields_ = [("rtol", C.c_double), ("itmax", C.c_int32), ("itmin", C.c_int32),
                ("precision", C.c_int32), ("inner_pc", C.c_int32), ("inner_rtol", C.c_double),
                ("inner_itmax", C.c_int32), ("remove_rotation", C.c_int32), ("use_guess", C.c_int32),
                ("verbose", C.c_int32), ("cheb_degree", C.c_int32), ("inner_rtol32", C.c_double),
                ("max_refine", C.c_int32), ("host_loop", C.c_int32), ("block_jacobi", C.c_int32),
                ("cheb_lo", C.c_double), ("cheb_hi", C.c_double), ("inner_relax", C.c_double),
                ("coarse_max", C.c_int32), ("schur_pc", C.c_int32),
                ("apply_warps", C.c_int32), ("apply_warps_t", C.c_int32),
                ("launch_overlap", C.c_int32), ("mg_tail", C.c_int32),
                ("matrix_free", C.c_int32), ("cheb_degree_coarse", C.c_int32), ("true_residual", C.c_int32),
                ("relax_base", C.c_double)]


class Arrhenius(C.Structure):
    _fields_ = [("eta0", C.c_double), ("R", C.c_double), ("Ea", C.c_double), ("Va", C.c_double),
                ("T0", C.c_double), ("phi_deg", C.c_double)]


class ThermalOpts(C.Structure):
    _fields_ = [("K", C.c_double), ("Cp", C.c_double), ("dt", C.c_double), ("Ttop", C.c_double),
                ("Tbot", C.c_double), ("rtol", C.c_double), ("atol", C.c_double), ("heated", C.c_int32),
                ("itmax", C.c_int32)]


class Dem(C.Structure):
    _fields_ = [("C", C.c_void_p), ("nrows", C.c_int64), ("a1a2_blk", C.c_void_p), ("n_a1a2", C.c_int64),
                ("a2a3_blk", C.c_void_p), ("permutation_blk", C.c_void_p), ("sblk", C.c_int64), ("w", C.c_double)]


class SolveReport(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("inner_iterations", C.c_int64),
                ("relres", C.c_double), ("r0", C.c_double), ("omega", C.c_double),
                ("div_residual", C.c_double), ("mom_residual", C.c_double),
                ("t_assemble_ms", C.c_double), ("t_setup_ms", C.c_double), ("t_solve_ms", C.c_double),
                ("fallback_used", C.c_int32), ("mg_levels", C.c_int32), ("kernel_launches", C.c_int64),
                ("refinements", C.c_int64), ("r0_guess", C.c_double), ("restarts", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)
_I32 = C.POINTER(C.c_int32)

# name -> (restype, argtypes); every entry of include/dimspers_b200.h
SIGNATURES = {
    "dp_mesh_sizes": (C.c_int, [C.POINTER(MeshDesc), _I64, _I64, _I64, _I64]),
    "dp_mesh_build": (C.c_int, [C.POINTER(MeshDesc), _I64, _D, _D, _I32, _I32]),
    "dp_mesh_free_slip": (C.c_int, [C.POINTER(MeshDesc), _I64, _I64]),
    "dp_status_string": (C.c_char_p, [C.c_int]),
    "dp_ctx_create": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(_P)]),
    "dp_ctx_destroy": (None, [_P]),
    "dp_last_error": (C.c_char_p, [_P]),
    "dp_ctx_stream": (_P, [_P]),
    "dp_get_connectivity": (C.c_int, [_P, _I64, _I32]),
    "dp_set_material": (C.c_int, [_P, _P, C.c_int64, C.POINTER(_P), C.c_int64, _P, C.c_double, C.c_int32]),
    "dp_set_material_ti": (C.c_int, [_P, _P, C.c_int64, _P, _P, _P, _P, C.c_double, C.c_int32]),
    "dp_fse_director": (C.c_int, [_P, _P, _P, _P, C.c_int32]),
    "dp_assemble": (C.c_int, [_P, C.c_int32]),
    "dp_set_deterministic": (C.c_int, [_P, C.c_int32]),
    "dp_get_element_matrices": (C.c_int, [_P, _P, _P, _P, _P]),
    "dp_solve": (C.c_int, [_P, _P, _P, _P, C.POINTER(SolveOpts), C.POINTER(SolveReport), C.c_int32]),
    "dp_apply_K": (C.c_int, [_P, _P, _P, C.c_int32]),
    "dp_apply_G": (C.c_int, [_P, _P, _P, C.c_int32]),
    "dp_apply_GT": (C.c_int, [_P, _P, _P, C.c_int32]),
    "dp_apply_K_noalloc": (C.c_int, [_P, _P, _P]),
    "dp_get_rhs": (C.c_int, [_P, _P, _P]),
    "dp_reduce": (C.c_int, [_P, _P, _P, C.c_int64, C.c_int32, _P, C.c_int32]),
    "dp_default_opts": (None, [C.POINTER(SolveOpts)]),
    "dp_profile_kernel": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_double)]),
    "dp_stress": (C.c_int, [_P, _P, _P, C.c_int64, C.POINTER(_P), C.c_int64, _P, C.c_int32]),
    "dp_viscosity_arrhenius": (C.c_int, [_P, C.POINTER(Arrhenius), _P, _P, C.c_int64, _P, _P, _P, _P, _P, C.c_int32]),
    "dp_default_thermal_opts": (None, [C.POINTER(ThermalOpts)]),
    "dp_thermal_step": (C.c_int, [_P, C.POINTER(ThermalOpts), _P, _P, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                  C.c_int32]),
    "dp_fse": (C.c_int, [_P, _P, C.POINTER(_P), C.c_int64, C.c_int32]),
    "dp_anisotropic_tensor": (C.c_int, [_P, C.POINTER(Dem), _P, _P, _P, _P, C.c_int64, C.POINTER(_P), C.c_int64,
                                        C.c_int32]),
    "dp_batch_create": (C.c_int, [C.POINTER(_P), C.c_int32, _P, C.POINTER(_P)]),
    "dp_batch_run": (C.c_int, [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P), C.c_int32, _P,
                               C.POINTER(C.c_double)]),
    "dp_batch_destroy": (None, [_P]),
    "dp_cnn_create": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, _I32, C.c_int32, C.c_int32,
                                C.POINTER(_P)]),
    "dp_cnn_destroy": (None, [_P]),
    "dp_cnn_num_params": (C.c_int64, [_P]),
    "dp_cnn_set_math": (C.c_int, [_P, C.c_int32]),
    "dp_cnn_set_params": (C.c_int, [_P, _P, C.c_int64]),
    "dp_cnn_get_params": (C.c_int, [_P, _P, _P, C.c_int64]),
    "dp_cnn_forward": (C.c_int, [_P, _P, _P, C.c_int32]),
    "dp_cnn_gradients": (C.c_int, [_P, _P, _P, C.c_int32, C.POINTER(C.c_double)]),
    "dp_cnn_train_step": (C.c_int, [_P, _P, _P, C.c_int32, C.c_float, C.POINTER(C.c_double)]),
    "dp_cnn_inputs": (C.c_int, [_P, _P, C.c_int32, C.c_int32]),
    "dp_guess_from_grid": (C.c_int, [_P, _P, C.c_int32, C.c_int32, C.c_double, _P, C.c_int32]),
}

_lib = None


def lib():
    """Load (once) and return the shared library; raises if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m dimspers_b200.build` "
                               "(the Stokes path has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class DPError(RuntimeError):
    def __init__(self, status, msg):
        self.status = status
        super().__init__(f"{lib().dp_status_string(status).decode()}: {msg}")


def check(status, ctx=None):
    if status != DP_OK:
        msg = lib().dp_last_error(ctx).decode(errors="replace")
        raise DPError(status, msg)
