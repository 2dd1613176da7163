"""ctypes binding of liblaph_gpu.so (the C ABI declared in include/laph_gpu.h).

The shared library is built in-tree (laph_eigsys_b200/liblaph_gpu.so).  There
is no fallback: if the library is missing, importing this module raises.
LAPH_GPU_LIB=check selects the bounds-checked build of the same sources
(liblaph_gpu_check.so, -DLAPH_CHECK) instead.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
_VARIANTS = {"": "liblaph_gpu.so", "check": "liblaph_gpu_check.so"}
_variant = os.environ.get("LAPH_GPU_LIB", "")
if _variant not in _VARIANTS:
    raise ImportError(f"LAPH_GPU_LIB={_variant!r}: expected one of {sorted(_VARIANTS)}")
LIB_PATH = os.path.join(_HERE, _VARIANTS[_variant])

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `make -C laph_eigsys_b200/csrc all check` "
        "(or __graft_entry__.build()); there is no CPU fallback")

lib = ctypes.CDLL(LIB_PATH)

c_int, c_double, c_void_p, c_char_p = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_char_p
c_u64, c_ll = ctypes.c_uint64, ctypes.c_longlong
P = ctypes.POINTER

LAPH_OK, LAPH_EINVAL, LAPH_ECUDA, LAPH_ENOMEM, LAPH_EIO, LAPH_ENORECORD, LAPH_ESIZE, \
    LAPH_ESINGLE, LAPH_ENOTCONV, LAPH_ETIMEOUT, LAPH_ETRACE, LAPH_EPARSE, LAPH_ENODEV = range(13)
LAYOUT_ROWMAJOR, LAYOUT_EIGEN, LAYOUT_CONF = 0, 1, 2
SMEAR_NONE, SMEAR_HYP, SMEAR_STOUT, SMEAR_APE = 0, 1, 2, 3
WINDOW_FIXED, WINDOW_LANCZOS, WINDOW_MLP = 0, 1, 2
LINKS_FP32, LINKS_BF16 = 0, 1


class laph_params(ctypes.Structure):
    _fields_ = [("L", c_int), ("lam_l", c_double), ("lam_c", c_double), ("deg", c_int), ("device", c_int)]


class laph_problem(ctypes.Structure):
    _fields_ = [("L", c_int), ("nev", c_int)]


class laph_solve_opts(ctypes.Structure):
    _fields_ = [("smear_kind", c_int), ("smear_p1", c_double), ("smear_p2", c_double), ("smear_iters", c_int),
                ("smear_compat", c_int), ("guard", c_int), ("link_prec", c_int), ("tol", c_double),
                ("max_it", c_int), ("window", c_int), ("lam_cut", c_double), ("lam_max", c_double),
                ("deg", c_int), ("phase_fix", c_int), ("seed", c_u64), ("block", c_int), ("filter_kernel", c_int),
                ("jacobi_sweeps", c_int), ("window_margin", c_double),
                ("host_loop", c_int), ("filter_tile", c_int),
                ("direct_resid", c_double)]


class laph_result(ctypes.Structure):
    _fields_ = [("status", c_int), ("iters", c_int), ("nconv", c_int), ("deg", c_int), ("lam_cut0", c_double),
                ("lam_max", c_double), ("max_resid", c_double), ("trace_vdv", c_double), ("window_fallback", c_int)]


class laph_tune_result(ctypes.Structure):
    _fields_ = [("deg", c_int), ("block", c_int), ("guard", c_int), ("ms_per_problem", c_double),
                ("trials", c_int), ("from_cache", c_int), ("tile", c_int)]


TUNE_TRIAL = ctypes.CFUNCTYPE(c_double, c_void_p, c_int, c_int, c_int)


class laph_config(ctypes.Structure):
    _fields_ = [("config_path", ctypes.c_char * 512), ("result_path", ctypes.c_char * 512),
                ("in_path", ctypes.c_char * 512), ("phase_path", ctypes.c_char * 512),
                ("LT", c_int), ("LX", c_int), ("NEV", c_int), ("iter", c_int), ("DEG", c_int),
                ("OMP_THRDS", c_int), ("alpha_1", c_double), ("alpha_2", c_double), ("LAM_L", c_double),
                ("LAM_C", c_double), ("smear", c_int), ("rho", c_double), ("alpha", c_double),
                ("tol", c_double), ("guard", c_int), ("block", c_int), ("window", c_int), ("solver", c_int),
                ("V3", c_int), ("MAT_ENTRIES", c_int), ("V_TS", c_int), ("alpha_1_i", c_double),
                ("alpha_1_f", c_double), ("alpha_2_i", c_double), ("alpha_2_f", c_double), ("autotune", c_int),
                ("filter_deg", c_int)]


def _sig(name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_sig("laph_strerror", c_char_p, c_int)
_sig("laph_last_error", c_char_p)
_sig("laph_version", c_int)
_sig("laph_ctx_create", c_int, P(c_void_p), P(laph_params))
_sig("laph_ctx_destroy", c_int, c_void_p)
_sig("laph_ctx_set_window", c_int, c_void_p, c_double, c_double, c_int)
_sig("laph_set_links", c_int, c_void_p, c_void_p, c_int)
_sig("laph_get_links", c_int, c_void_p, c_void_p, c_int)
_sig("laph_smear", c_int, c_void_p, c_int, c_double, c_double, c_int, c_int)
_sig("laph_matmult", c_int, c_void_p, c_void_p, c_void_p, c_int, c_int)
_sig("laph_matmult_noalloc", c_int, c_void_p, c_int, c_double, c_double, c_int, c_void_p, c_void_p, c_void_p)
_sig("laph_apply_neglap", c_int, c_void_p, c_void_p, c_void_p, c_int)
_sig("laph_get_diagonal", c_int, c_void_p, c_void_p, c_int)
_sig("laph_plaquette", c_int, c_void_p, P(c_double))
_sig("laph_eps_solve", c_int, c_void_p, c_int, c_int, c_double, c_int, c_int, c_u64, c_void_p, c_void_p, P(c_int),
     P(c_int), P(c_ll))
_sig("laph_solve_opts_default", None, P(laph_solve_opts))
_sig("laph_solver_create", c_int, P(c_void_p), P(laph_problem), c_int, P(laph_solve_opts), c_int)
_sig("laph_solver_destroy", c_int, c_void_p)
_sig("laph_solver_set_links", c_int, c_void_p, c_int, c_void_p, c_int, c_int)
_sig("laph_solver_run", c_int, c_void_p, P(laph_result))
_sig("laph_solver_get", c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_int)
_sig("laph_solver_stream", c_int, c_void_p, P(c_void_p))
_sig("laph_solver_get_async", c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p)
_sig("laph_solver_wait", c_int, c_void_p)
_sig("laph_solver_filter_bytes", c_int, c_void_p, P(c_double))
_sig("laph_solver_loop_info", c_int, c_void_p, P(c_int), P(ctypes.c_longlong))
_sig("laph_ctx_stream", c_int, c_void_p, P(c_void_p))
_sig("laph_binary_version", c_int, P(c_int))
_sig("laph_probe_fp64", c_int, c_int, P(c_double), P(c_double))
_sig("laph_check_enabled", c_int)
_sig("laph_check_report", c_int, P(c_u64), P(c_ll), P(c_ll), P(c_int), c_char_p, c_int, c_int)
_sig("laph_check_selftest", c_int, c_int)
_sig("laph_solver_set_window_model", c_int, c_void_p, c_void_p, c_int)
_sig("laph_solver_features", c_int, c_void_p, c_void_p, c_void_p)
_sig("laph_solver_ritz", c_int, c_void_p, c_int, c_void_p, P(c_int))
_sig("laph_mlp_nparams", c_int)
_sig("laph_mlp_forward", c_int, c_void_p, c_void_p, c_int, c_void_p, c_int)
_sig("laph_mlp_grad", c_int, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int)
_sig("laph_mlp_train", c_int, c_void_p, c_void_p, c_void_p, c_int, c_int, ctypes.c_float, c_void_p, c_int)
_sig("laph_solver_timings", c_int, c_void_p, P(c_double))
_sig("laph_solver_counters", c_int, c_void_p, P(c_ll))
_sig("laph_solver_footprint", c_int, P(laph_problem), c_int, P(laph_solve_opts), P(c_ll))
_sig("laph_solver_max_batch", c_int, P(laph_problem), c_int, P(laph_solve_opts), c_int, c_double, P(c_int))
_sig("laph_autotune_search", c_int, P(c_int), c_int, P(c_int), c_int, P(c_int), c_int, c_int, c_int, c_int, TUNE_TRIAL,
     c_void_p, P(laph_tune_result))
_sig("laph_solver_autotune", c_int, P(laph_problem), c_int, P(c_void_p), c_int, c_int, P(laph_solve_opts), c_void_p,
     c_int, c_int, ctypes.c_char_p, P(laph_tune_result))
_sig("laph_gauge_random", c_int, c_void_p, c_int, c_int, c_double, c_u64)
_sig("laph_lime_write_gauge", c_int, c_char_p, c_void_p, c_int, c_int)
_sig("laph_lime_read_gauge", c_int, c_char_p, c_int, c_int, c_int, c_int, c_void_p)
_sig("laph_lime_read_gauge_any", c_int, c_char_p, c_int, c_int, c_int, c_int, c_void_p, P(c_int))
_sig("laph_lime_info", c_int, c_char_p, P(c_int), P(c_int), P(c_int), P(c_int), P(c_int))
_sig("laph_lime_write_gauge_prec", c_int, c_char_p, c_void_p, c_int, c_int, c_int)
_sig("laph_sourceshape", c_int, c_void_p, c_int, c_int, c_void_p, c_int, c_void_p, c_int)
_sig("laph_solver_sourceshape", c_int, c_void_p, c_int, c_int, c_void_p)
_sig("laph_solver_set_smear", c_int, c_void_p, c_int, c_double, c_double)
_sig("laph_displace", c_int, c_void_p, c_int, c_void_p, c_void_p, c_int, c_int)
_sig("laph_solver_displace", c_int, c_void_p, c_int, c_int, c_void_p, c_int)
_sig("laph_sourceshape_avg", c_int, c_int, c_void_p, c_void_p, c_void_p, P(c_int))
_sig("laph_write_sourceshape", c_int, c_char_p, c_int, c_int, c_int, c_int, c_void_p, c_void_p)
_sig("laph_write_eigsys_bin", c_int, c_char_p, c_char_p, c_int, c_int, c_int, c_int, c_void_p)
_sig("laph_write_eigenvalues_bin", c_int, c_char_p, c_char_p, c_int, c_int, c_int, c_void_p)
_sig("laph_read_eigsys_bin", c_int, c_char_p, c_char_p, c_int, c_int, c_int, c_int, c_void_p)
_sig("laph_read_eigenvalues_bin", c_int, c_char_p, c_char_p, c_int, c_int, c_int, c_void_p)
_sig("laph_check_trace", c_int, c_int, c_int, c_void_p, P(c_double), P(c_double))
_sig("laph_fix_phase_host", c_int, c_int, c_int, c_void_p, c_void_p, c_void_p)
_sig("laph_reset_phase_host", c_int, c_int, c_int, c_void_p, c_void_p, c_void_p)
_sig("laph_read_eigenvalues_ascii", c_int, c_char_p, c_int, c_int, c_int, c_void_p)
_sig("laph_write_gauge_matrices", c_int, c_char_p, c_int, c_void_p)
_sig("laph_read_gauge_matrices", c_int, c_char_p, c_int, c_void_p)
_sig("laph_recover_spectrum", c_int, c_int, c_void_p, c_int, c_double, c_double, c_void_p)
_sig("laph_parse_parameters", c_int, c_char_p, P(laph_config))
_sig("laph_timeslice_split", c_int, c_int, c_int, c_int, P(c_int), P(c_int))


class LaphError(RuntimeError):
    """A LAPH_E* status from the library: .status is the code, the message carries laph_last_error()."""
    def __init__(self, status, where):
        self.status = status
        msg = lib.laph_last_error().decode(errors="replace")
        super().__init__(f"{where}: {lib.laph_strerror(status).decode()} ({status}): {msg}")


def check(status, where):
    if status != LAPH_OK:
        raise LaphError(status, where)
    return status
