"""ctypes binding of ``_lib/libdwfb200.so`` (the C ABI in include/dwf_b200.h).

The library is required: importing a compute entry point without it raises,
there is no CPU fallback.
"""
import ctypes as C
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
# DWF_B200_LIB selects another build of the same library (e.g. a tuning variant).
LIB_PATH = Path(os.environ.get("DWF_B200_LIB", _PKG / "_lib" / "libdwfb200.so"))

DWF_OK, DWF_NOT_CONVERGED, DWF_ZERO_DENOM, DWF_NONFINITE = 0, 1, 2, 3
DWF_CUDA_ERROR, DWF_TIMEOUT, DWF_BAD_ARG = 4, 5, 6
OP_D, OP_DDAG, OP_DDDAG, OP_DDAGD = 0, 1, 2, 3
SOLVER_CG64, SOLVER_MIXED, SOLVER_EO_MIXED, SOLVER_LEARNED = 0, 1, 2, 3
LP_GCR, LP_BICGSTAB = 0, 1


class DwfParams(C.Structure):
    _fields_ = [("Nt", C.c_int), ("Nx", C.c_int), ("Ls", C.c_int),
                ("M5", C.c_double), ("mf", C.c_double), ("beta", C.c_double),
                ("device", C.c_int)]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("status", C.c_int),
                ("solver", C.c_int), ("relres", C.c_double), ("true_relres", C.c_double),
                ("reliable_updates", C.c_int), ("fallback", C.c_int),
                ("dirac_relres", C.c_double), ("schur_iterations", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class HmcParams(C.Structure):
    _fields_ = [("epsilon", C.c_double), ("steps", C.c_int), ("rtol", C.c_double),
                ("maxiter", C.c_int), ("solver", C.c_int)]


class TrajInfo(C.Structure):
    _fields_ = [("dH", C.c_double), ("H0", C.c_double), ("H", C.c_double),
                ("S_gauge", C.c_double), ("S_pf", C.c_double), ("kinetic0", C.c_double),
                ("kinetic", C.c_double), ("plaquette", C.c_double),
                ("acceptance_probability", C.c_double), ("accepted", C.c_int),
                ("solves", C.c_int), ("cg_iterations", C.c_long), ("status", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class WilParams(C.Structure):
    _fields_ = [("Nt", C.c_int), ("Nx", C.c_int), ("m0", C.c_double), ("beta", C.c_double),
                ("bc_t", C.c_double), ("bc_x", C.c_double), ("device", C.c_int)]


class MeasureParams(C.Structure):
    _fields_ = [("n_point_times", C.c_int), ("n_wall_times", C.c_int), ("n_noise", C.c_int),
                ("max_momentum", C.c_int), ("rtol", C.c_double), ("maxiter", C.c_int),
                ("solver", C.c_int)]


class LpTrainParams(C.Structure):
    _fields_ = [("steps", C.c_int), ("batch", C.c_int), ("lr", C.c_double),
                ("lr_decay_steps", C.c_int), ("pairs_per_conf", C.c_int),
                ("solver_iters", C.c_int), ("solver_every", C.c_int),
                ("solver_maxiter", C.c_int), ("seed", C.c_uint64)]


class LpTrainInfo(C.Structure):
    _fields_ = [("loss_first", C.c_double), ("loss_last", C.c_double), ("steps", C.c_int),
                ("npairs", C.c_int), ("solver_pairs", C.c_int), ("seconds_pairs", C.c_double),
                ("seconds_train", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_DP = C.POINTER(C.c_double)

# name -> (restype, argtypes)
SIGNATURES = {
    "dwf_ctx_create": (_I, [C.POINTER(DwfParams), C.POINTER(_P)]),
    "dwf_ctx_destroy": (_I, [_P]),
    "dwf_status_string": (C.c_char_p, [_I]),
    "dwf_last_error": (C.c_char_p, [_P]),
    "dwf_set_wait_limit": (_I, [_P, C.c_uint64]),
    "dwf_sync": (_I, [_P]),
    "dwf_stream": (_P, [_P]),
    "dwf_set_gauge": (_I, [_P, _I, _P]),
    "dwf_set_gauge_dev": (_I, [_P, _I, _P]),
    "dwf_apply": (_I, [_P, _I, _I, _P, _P, _I]),
    "dwf_apply_dev": (_I, [_P, _I, _I, _P, _P, _I, _I]),
    "dwf_cg": (_I, [_P, _I, _I, _P, _P, _I, _D, _I, _I, C.POINTER(SolveInfo)]),
    "dwf_cg_batch_dev": (_I, [_P, _I, _I, _P, _P, _P, _I, _D, _I, _I, C.POINTER(SolveInfo)]),
    "dwf_cg_batch": (_I, [_P, _I, _I, _P, _P, _P, _I, _D, _I, _I, C.POINTER(SolveInfo)]),
    "dwf_propagators": (_I, [_P, _I, _P, _P, _P, _D, _I, _I, C.POINTER(SolveInfo)]),
    "dwf_propagators_dev": (_I, [_P, _I, _P, _P, _P, _D, _I, _I, C.POINTER(SolveInfo)]),
    "dwf_launch_count": (C.c_uint64, [_P]),
    "dwf_device_count": (_I, [C.POINTER(_I)]),
    "dwf_set_eo_kernel": (_I, [_P, _I]),
    "dwf_round_robin_device": (_I, [_I, C.c_char_p, C.POINTER(_I)]),
    "dwf_set_dslash_variant": (_I, [_P, _I]),
    "dwf_dslash_variant": (_I, [_P, _I, _I]),
    "dwf_set_dslash_chunk": (_I, [_P, _I]),
    "dwf_barrier_selftest": (_I, [_P, _I, C.c_uint64]),
    "dwf_cg_noalloc": (_I, [C.POINTER(DwfParams), _I, _P, _P, _P, _I, _D, _I, _P,
                            C.POINTER(SolveInfo)]),
    "dwf_measure": (_I, [_P, C.POINTER(MeasureParams), _I, _P, _P, _P, _P, _P, _P,
                         C.POINTER(SolveInfo)]),
    "wil_pseudoscalar_correlator": (_I, [_P, _I, _P, _I, _I, _D, _I, _I, _P,
                                         C.POINTER(SolveInfo)]),
    "dwf_rng_create": (_I, [C.c_uint64, C.POINTER(_P)]),
    "dwf_rng_destroy": (_I, [_P]),
    "dwf_rng_normals": (_I, [_P, C.c_long, _P]),
    "dwf_rng_uniform": (_I, [_P, C.POINTER(C.c_double)]),
    "dwf_rng_pseudofermion": (_I, [_P, C.c_long, _P]),
    "dwf_z4_digits": (_I, [C.c_uint64, C.c_long, _P]),
    "dwf_gauge_action_force": (_I, [_P, _P, _P, _P]),
    "dwf_average_plaquette": (_I, [_P, _P, _P]),
    "dwf_pf_action_force": (_I, [_P, _P, _P, _P, _D, _I, _I, _P, _P, _P, C.POINTER(SolveInfo)]),
    "dwf_hmc_trajectory": (_I, [_P, C.POINTER(HmcParams), _P, _P, _P, _P, C.POINTER(TrajInfo)]),
    "wil_ctx_create": (_I, [C.POINTER(WilParams), C.POINTER(_P)]),
    "wil_solve_cgnr": (_I, [_P, _P, _P, _D, _I, _I, _P, _P]),
    "wil_solve_dddag": (_I, [_P, _P, _P, _D, _I, _I, _P, _P]),
    "wil_hmc_step": (_I, [_P, C.POINTER(HmcParams), _P, _P, _P, _D, _P, C.POINTER(TrajInfo)]),
    "dwf_solver_kernel_ms": (C.c_double, [_P, _I, C.POINTER(C.c_uint64)]),
    "dwf_graph_replays": (C.c_uint64, [_P, C.POINTER(C.c_int)]),
    "dwf_eo_phase_profile": (_I, [_P, _I]),
    "dwf_eo_phase_times": (_I, [_P, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
    "dwf_lp_init": (_I, [_P, _I, C.c_uint64]),
    "dwf_lp_weights_size": (_I, [_P, C.POINTER(C.c_long)]),
    "dwf_lp_get_weights": (_I, [_P, _P]),
    "dwf_lp_set_weights": (_I, [_P, _P]),
    "dwf_lp_transports": (_I, [_P, _I, _P]),
    "dwf_lp_apply_dev": (_I, [_P, _I, _I, _P, _P, _P]),
    "dwf_lp_layer_dev": (_I, [_P, _I, _I, _I, _P, _P, _P]),
    "dwf_lp_loss_grad_dev": (_I, [_P, _I, _P, _P, _P, C.POINTER(C.c_double), _P]),
    "dwf_lp_train": (_I, [_P, C.POINTER(LpTrainParams), C.POINTER(LpTrainInfo), _P]),
    "dwf_lp_set_solver": (_I, [_P, _D, _I, _I]),
    "dwf_lp_set_krylov": (_I, [_P, _I, _I]),
    "dwf_lp_set_variant": (_I, [_P, _I]),
    "dwf_lp_time_network": (_I, [_P, _I, _I, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
}

_lib = None


class DwfError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__(f"{status_string(status)}{': ' + msg if msg else ''}")


def lib():
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with "
                "`python -m three_part_dwf_study_b200.build` (no CPU fallback exists)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def status_string(status):
    return lib().dwf_status_string(int(status)).decode()


def check(status, ctx=None):
    if status != DWF_OK:
        msg = lib().dwf_last_error(ctx).decode() if ctx else ""
        raise DwfError(status, msg)
