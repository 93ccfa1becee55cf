"""ctypes declarations of the C ABI in include/ddamg.h (libddamg.so, built in-tree)."""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libddamg.so")
MAX_LEVELS = 6

OK, ERR_BAD_PARAM, ERR_IO, NOT_CONVERGED, ERR_NAN, ERR_DEVICE_TIMEOUT, ERR_CUDA, ERR_STATE = range(8)
STATUS_NAMES = {0: "OK", 1: "BAD_PARAM", 2: "IO", 3: "NOT_CONVERGED", 4: "NAN", 5: "DEVICE_TIMEOUT", 6: "CUDA_ERROR",
                7: "STATE"}
PREC_DOUBLE, PREC_MIXED = 0, 1
CYCLE_V, CYCLE_K = 0, 1


class Params(ctypes.Structure):
    _fields_ = [
        ("Nx", ctypes.c_int), ("Nt", ctypes.c_int), ("levels", ctypes.c_int), ("m0", ctypes.c_double),
        ("rows", (ctypes.c_int * 6) * (MAX_LEVELS - 1)),
        ("sap_gmres_restart_length", ctypes.c_int), ("sap_gmres_restarts", ctypes.c_int),
        ("sap_gmres_tolerance", ctypes.c_double), ("sap_test_vectors_iterations", ctypes.c_int),
        ("coarse_gmres_restart_length", ctypes.c_int), ("coarse_gmres_restarts", ctypes.c_int),
        ("coarse_gmres_tolerance", ctypes.c_double), ("nu1", ctypes.c_int), ("nu2", ctypes.c_int),
        ("kcycle_restart_length", ctypes.c_int), ("kcycle_restarts", ctypes.c_int),
        ("kcycle_tolerance", ctypes.c_double), ("fgmres_restart_length", ctypes.c_int),
        ("fgmres_restarts", ctypes.c_int), ("fgmres_tolerance", ctypes.c_double),
        ("smoother_tolerance", ctypes.c_double), ("cycle", ctypes.c_int), ("precision", ctypes.c_int),
        ("max_rhs", ctypes.c_int), ("device", ctypes.c_int), ("tensor_cores", ctypes.c_int),
        ("cuda_graphs", ctypes.c_int), ("coarse_barrier_polls", ctypes.c_int),
        ("coarse_kernel", ctypes.c_int),
    ]


class SolveInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("converged", ctypes.c_int), ("rel_residual", ctypes.c_double),
                ("setup_seconds", ctypes.c_double), ("solve_seconds", ctypes.c_double)]


# every symbol the header declares, with (restype, argtypes)
_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p
_h = ctypes.c_void_p
_st = ctypes.c_int
_i = ctypes.c_int
class HmcInfo(ctypes.Structure):
    _fields_ = [("accepted", ctypes.c_int), ("dH", ctypes.c_double), ("plaquette", ctypes.c_double),
                ("cg_iterations", ctypes.c_int), ("seconds", ctypes.c_double)]


SIGNATURES = {
    "ddamg_params_default": (_st, [ctypes.POINTER(Params)]),
    "ddamg_parse_params_file": (_st, [ctypes.c_char_p, _i, ctypes.POINTER(Params)]),
    "ddamg_create": (_st, [ctypes.POINTER(Params), ctypes.POINTER(_vp)]),
    "ddamg_destroy": (_st, [_h]),
    "ddamg_last_error": (ctypes.c_char_p, []),
    "ddamg_get_stream": (_st, [_h, ctypes.POINTER(_vp)]),
    "ddamg_launch_count": (_st, [_h, ctypes.POINTER(ctypes.c_longlong)]),
    "ddamg_profile": (_st, [_h, _i]),
    "ddamg_profile_query": (_st, [_h, _i, _i, _dp, ctypes.POINTER(ctypes.c_longlong)]),
    "ddamg_autotune_report": (_st, [_h, ctypes.c_char_p, _i]),
    "ddamg_read_binary": (_st, [ctypes.c_char_p, _i, _i, _dp]),
    "ddamg_write_binary": (_st, [ctypes.c_char_p, _i, _i, _dp]),
    "ddamg_load_gauge": (_st, [_h, _dp]),
    "ddamg_apply_dirac": (_st, [_h, _i, _dp, _dp, _i]),
    "ddamg_apply_dirac_device": (_st, [_h, _i, _vp, _vp, _i]),
    "ddamg_apply_dirac_f32_device": (_st, [_h, _i, _vp, _vp, _i]),
    "ddamg_apply_level_op": (_st, [_h, _i, _dp, _dp]),
    "ddamg_apply_level_op_device": (_st, [_h, _i, _i, _vp, _vp, _i]),
    "ddamg_restrict": (_st, [_h, _i, _dp, _dp]),
    "ddamg_prolong": (_st, [_h, _i, _dp, _dp]),
    "ddamg_sap": (_st, [_h, _i, _dp, _dp, _i, ctypes.c_double, ctypes.POINTER(_i)]),
    "ddamg_sap_batched": (_st, [_h, _i, _dp, _dp, _i, _i, ctypes.c_double]),
    "ddamg_setup": (_st, [_h, ctypes.c_uint64]),
    "ddamg_setup_with_vectors": (_st, [_h, _dp, ctypes.c_int64]),
    "ddamg_setup_random_count": (_st, [_h, ctypes.POINTER(ctypes.c_int64)]),
    "ddamg_get_test_vectors": (_st, [_h, _i, _dp]),
    "ddamg_set_test_vectors": (_st, [_h, _i, _dp]),
    "ddamg_orthonormalize": (_st, [_h, _i]),
    "ddamg_build_coarse_links": (_st, [_h, _i]),
    "ddamg_get_coarse_links": (_st, [_h, _i, _i, _dp]),
    "ddamg_coarse_solve": (_st, [_h, _dp, _dp, ctypes.POINTER(_i)]),
    "ddamg_coarse_gmres_noalloc": (_st, [_vp, _vp, _vp, _i, _i, _i, ctypes.c_double, _i, _i, ctypes.c_double, _vp,
                                         ctypes.POINTER(_i)]),
    "ddamg_set_coarse_barrier_polls": (_st, [_h, _i]),
    "ddamg_get_counters": (_st, [_h, ctypes.POINTER(ctypes.c_longlong)]),
    "ddamg_set_stencil_kernel": (_st, [_i]),
    "ddamg_get_stencil_kernel": (_st, [ctypes.POINTER(_i)]),
    "ddamg_write_metadata": (_st, [_h, ctypes.c_char_p, _i, ctypes.c_double]),
    "ddamg_write_metadata_params": (_st, [ctypes.POINTER(Params), ctypes.POINTER(ctypes.c_longlong), _i,
                                          ctypes.c_double, ctypes.c_char_p]),
    "ddamg_apply_multilevel": (_st, [_h, _dp, _dp, _i, ctypes.c_double, ctypes.POINTER(_i), _dp]),
    "ddamg_fgmres_sap": (_st, [_h, _dp, _dp, _i, _i, _i, _i, ctypes.c_double, ctypes.POINTER(SolveInfo)]),
    "ddamg_sap_fine": (_st, [_h, _dp, _dp, _i, _i, _i, ctypes.c_double, ctypes.POINTER(_i)]),
    "ddamg_vcycle": (_st, [_h, _dp, _dp]),
    "ddamg_kcycle": (_st, [_h, _dp, _dp]),
    "ddamg_solve": (_st, [_h, _dp, _dp, _i, ctypes.POINTER(SolveInfo)]),
    "ddamg_solve_device": (_st, [_h, _vp, _vp, _i, ctypes.POINTER(SolveInfo)]),
    "ddamg_gmres_plain": (_st, [_h, _dp, _dp, _i, _i, ctypes.c_double, ctypes.POINTER(SolveInfo)]),
    "ddamg_bicgstab": (_st, [_h, _dp, _dp, _dp, _i, ctypes.c_double, ctypes.POINTER(SolveInfo)]),
    "ddamg_cg_normal": (_st, [_h, _dp, _dp, _i, ctypes.c_double, ctypes.POINTER(SolveInfo)]),
    "ddamg_gradient": (_st, [_h, _dp, _dp, _dp, ctypes.POINTER(SolveInfo)]),
    "ddamg_link_derivative": (_st, [_h, _dp, _dp, _dp]),
    "ddamg_gauge_metropolis": (_st, [_i, _i, ctypes.c_double, _i, ctypes.c_uint64, ctypes.c_double, _dp, _dp, _i]),
    "ddamg_gaussian_field": (_st, [ctypes.c_int64, ctypes.c_uint64, _dp]),
    "ddamg_from_halo": (_st, [_dp, _i, _i, _i, _dp]),
    "ddamg_hmc_trajectory": (_st, [_h, _dp, ctypes.c_double, _i, ctypes.c_double, ctypes.c_uint64, ctypes.c_double,
                                   ctypes.POINTER(HmcInfo)]),
    "ddamg_hmc_force": (_st, [_h, _dp, _dp, ctypes.c_double, ctypes.c_double, _dp]),
    "ddamg_to_halo": (_st, [_dp, _i, _i, _i, _dp]),
}

_lib = None


def load(path=LIB_PATH):
    """Load libddamg.so; raises if it is missing (there is no fallback implementation)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise OSError(f"{path} not found: build it with `python ddalphaamg-sm_b200/ddamg/build.py`")
        L = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class DDAMGError(RuntimeError):
    def __init__(self, status, msg):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")


def check(status, allow=()):
    if status != OK and status not in allow:
        raise DDAMGError(status, load().ddamg_last_error().decode(errors="replace"))
    return status
