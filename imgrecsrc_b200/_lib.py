"""ctypes binding of libctprj.so, the engine's C ABI (include/ctprj.h).

The library is built in-tree by imgrecsrc_b200/build.py.  There is no CPU
fallback: importing a compute entry point without the library raises.
"""
import ctypes
import os

from .build import LIB

CTPRJ_OK, CTPRJ_EINVAL, CTPRJ_ENOTSETUP, CTPRJ_ENOMEM, CTPRJ_ECUDA, CTPRJ_ERANGE, CTPRJ_ETIMEOUT = range(7)
FWD_BIT, BWD_BIT, FBP_BIT = 1 << 1, 1 << 2, 1 << 3


class CtprjError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("ctprj status %d: %s" % (status, message))
        self.status = status


class ParConf(ctypes.Structure):
    """parConf of include/parprj.h (prj/parPrj.h:9-16)."""
    _fields_ = [("bw", ctypes.c_double), ("nc", ctypes.c_int), ("nr", ctypes.c_int),
                ("np", ctypes.c_int), ("prjWidth", ctypes.c_int),
                ("theta", ctypes.POINTER(ctypes.c_double)), ("fwd", ctypes.c_int)]


MAX_TRACE = 256


class LoopOpts(ctypes.Structure):
    """ctprj_bhc_loop_opts of include/ctprj_bhc_loop.h."""
    _fields_ = [("iterations", ctypes.c_int), ("x_step", ctypes.c_double),
                ("spectrum_newton_steps", ctypes.c_int), ("skip_spectrum", ctypes.c_int),
                ("unfused", ctypes.c_int), ("init_step", ctypes.c_int),
                ("density_method", ctypes.c_int), ("thresh", ctypes.c_double),
                ("min_iterations", ctypes.c_int), ("proximal", ctypes.c_int),
                ("u", ctypes.c_double), ("max_inner", ctypes.c_int), ("admm_tol", ctypes.c_double),
                ("no_restart", ctypes.c_int), ("no_adaptive_step", ctypes.c_int), ("cumu_tol", ctypes.c_int),
                ("wvlt_filter_len", ctypes.c_int), ("wvlt_filter", ctypes.c_double * 20),
                ("wvlt_levels", ctypes.c_int), ("mask", ctypes.c_void_p), ("wvlt_mask", ctypes.c_void_p),
                ("pre_steps", ctypes.c_int)]


class LoopStats(ctypes.Structure):
    """ctprj_bhc_loop_stats of include/ctprj_bhc_loop.h."""
    _fields_ = [("iterations", ctypes.c_int), ("final_cost", ctypes.c_double),
                ("final_x_step", ctypes.c_double), ("cost", ctypes.c_double * MAX_TRACE),
                ("x_step", ctypes.c_double * MAX_TRACE), ("ms", ctypes.c_float),
                ("ms_spectrum", ctypes.c_float), ("evaluations", ctypes.c_int),
                ("restarts", ctypes.c_int), ("newton_steps", ctypes.c_int),
                ("converged", ctypes.c_int), ("x_change", ctypes.c_double * MAX_TRACE),
                ("inner_iterations", ctypes.c_int), ("prox_retries", ctypes.c_int),
                ("penalty", ctypes.c_double)]


class ParDevConf(ctypes.Structure):
    """ctprj_par_conf of include/parprj.h (device-pointer form)."""
    _fields_ = [("bw", ctypes.c_double), ("nc", ctypes.c_int), ("nr", ctypes.c_int),
                ("np", ctypes.c_int), ("prjWidth", ctypes.c_int)]


class Geometry(ctypes.Structure):
    """struct ctprj_geometry -- the reference's projector configuration
    (prj/prj.h:42-57): n, prjWidth, np, prjFull, dSize, effectiveRate, d."""
    _fields_ = [("n", ctypes.c_int), ("prjWidth", ctypes.c_int), ("np", ctypes.c_int),
                ("prjFull", ctypes.c_int), ("dSize", ctypes.c_float),
                ("effectiveRate", ctypes.c_float), ("d", ctypes.c_float)]

    def __init__(self, n, prjWidth, np, prjFull, dSize=1.0, effectiveRate=1.0, d=0.0):
        super().__init__(int(n), int(prjWidth), int(np), int(prjFull), float(dSize),
                         float(effectiveRate), float(d))

    @property
    def fan(self):
        return self.d > 0

    def as_tuple(self):
        return (self.n, self.prjWidth, self.np, self.prjFull, self.dSize, self.effectiveRate, self.d)

    def __repr__(self):
        return ("Geometry(n=%d, prjWidth=%d, np=%d, prjFull=%d, dSize=%g, effectiveRate=%g, d=%g)"
                % self.as_tuple())


_lib = None
VP = ctypes.c_void_p


def lib():
    """The loaded libctprj.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = os.environ.get("CTPRJ_LIB") or LIB    # another build of the same library
    if not os.path.exists(path):
        raise RuntimeError("libctprj.so is missing: build it with `python -m imgrecsrc_b200.build`")
    L = ctypes.CDLL(path)
    GP = ctypes.POINTER(Geometry)
    sig = {
        "setup": ([ctypes.c_int] * 4 + [ctypes.c_float] * 3, None),
        "showSetup": ([], None),
        "gpuPrj": ([VP, VP, ctypes.c_char], ctypes.c_int),
        "ctprj_plan_create": ([GP, ctypes.c_int, ctypes.POINTER(VP)], ctypes.c_int),
        "ctprj_plan_destroy": ([VP], None),
        "ctprj_forward": ([VP, VP, VP, VP], ctypes.c_int),
        "ctprj_backward": ([VP, VP, VP, VP], ctypes.c_int),
        "ctprj_fbp": ([VP, VP, VP, VP], ctypes.c_int),
        "ctprj_count_updates": ([VP, ctypes.POINTER(ctypes.c_longlong),
                                 ctypes.POINTER(ctypes.c_longlong), VP], ctypes.c_int),
        "ctprj_bhc_create": ([VP, ctypes.c_int, VP, ctypes.c_double, ctypes.POINTER(VP)], ctypes.c_int),
        "ctprj_bhc_destroy": ([VP], None),
        "ctprj_bhc_forward": ([VP, VP, VP, VP, VP, ctypes.c_int, VP], ctypes.c_int),
        "ctprj_bhc_backward": ([VP, VP, VP, VP, VP, VP, VP], ctypes.c_int),
        "ctprj_bhc_terms": ([VP, VP, VP, VP, VP, ctypes.c_int, VP], ctypes.c_int),
        "ctprj_bhc_basis": ([VP, VP, VP, VP], ctypes.c_int),
        "ctprj_bhc_state": ([VP, ctypes.POINTER(VP), ctypes.POINTER(VP), ctypes.POINTER(VP)], ctypes.c_int),
        "ctprj_bhc_set_noise": ([VP, ctypes.c_int], ctypes.c_int),
        "ctprj_bhc_hessian": ([VP, VP, VP, VP, VP, VP, VP], ctypes.c_int),
        "parPrjConf": ([VP, VP, VP, ctypes.POINTER(ParConf), ctypes.c_size_t], ctypes.c_int),
        "ctprj_par_forward": ([ctypes.POINTER(ParDevConf), VP, VP, ctypes.c_longlong, VP, VP, VP], ctypes.c_int),
        "ctprj_par_backward": ([ctypes.POINTER(ParDevConf), VP, VP, ctypes.c_longlong, VP, VP, VP], ctypes.c_int),
        "parPrjThread": ([], ctypes.c_int),
        "parPrjRun": ([], ctypes.c_int),
        "ctprj_batch_create": ([GP, ctypes.c_int, ctypes.c_int, ctypes.POINTER(VP)], ctypes.c_int),
        "ctprj_batch_destroy": ([VP], None),
        "ctprj_batch_bind": ([VP, VP, VP, VP, VP], ctypes.c_int),
        "ctprj_batch_forward": ([VP, VP], ctypes.c_int),
        "ctprj_batch_backward": ([VP, VP], ctypes.c_int),
        "ctprj_batch_capture": ([VP, VP], ctypes.c_int),
        "ctprj_batch_autotune": ([VP, VP, ctypes.c_char_p], ctypes.c_int),
        "ctprj_batch_config": ([VP, ctypes.c_char_p, ctypes.c_int], ctypes.c_int),
        "ctprj_bhc_spectrum_step": ([VP, VP, VP, ctypes.c_int, ctypes.POINTER(ctypes.c_double), VP], ctypes.c_int),
        "ctprj_bhc_reconstruct": ([VP, VP, VP, VP, ctypes.POINTER(LoopOpts), ctypes.POINTER(LoopStats), VP], ctypes.c_int),
        "ctprj_stream_flags_create": ([ctypes.c_int, ctypes.POINTER(VP), ctypes.POINTER(VP)], ctypes.c_int),
        "ctprj_stream_flags_destroy": ([VP], None),
        "ctprj_batch_stream_backward": ([VP, VP, ctypes.c_double, VP, VP], ctypes.c_int),
        "ctprj_masked_forward": ([VP, VP, ctypes.c_longlong, VP, ctypes.c_double, VP, VP], ctypes.c_int),
        "ctprj_masked_backward": ([VP, VP, ctypes.c_longlong, VP, ctypes.c_double, VP, VP], ctypes.c_int),
        "ctprj_masked_fbp": ([VP, VP, ctypes.c_longlong, VP, ctypes.c_double, VP, VP], ctypes.c_int),
        "ctprj_tv_denoise": ([VP, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                              ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double, VP,
                              ctypes.POINTER(ctypes.c_int), VP], ctypes.c_int),
        "ctprj_tv_value": ([VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, VP, VP], ctypes.c_int),
        "ctprj_dwt": ([VP, ctypes.c_int, ctypes.c_int, VP, ctypes.c_int, ctypes.c_int, VP, VP], ctypes.c_int),
        "ctprj_idwt": ([VP, ctypes.c_int, ctypes.c_int, VP, ctypes.c_int, ctypes.c_int, VP, VP], ctypes.c_int),
        "ctprj_wvlt_l1": ([VP, ctypes.c_int, ctypes.c_int, VP, ctypes.c_int, ctypes.c_int, VP, VP], ctypes.c_int),
        "ctprj_wvlt_admm": ([VP, ctypes.c_int, ctypes.c_int, VP, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                             ctypes.c_double, ctypes.c_int, VP, VP, ctypes.POINTER(ctypes.c_int), VP], ctypes.c_int),
        "ctprj_wvlt_mask": ([VP, ctypes.c_int, ctypes.c_int, VP, ctypes.c_int, ctypes.c_int, VP, VP], ctypes.c_int),
        "ctprj_error_string": ([ctypes.c_int], ctypes.c_char_p),
        "ctprj_last_error": ([], ctypes.c_char_p),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def check(status):
    if status != CTPRJ_OK:
        L = lib()
        raise CtprjError(status, (L.ctprj_last_error() or L.ctprj_error_string(status)).decode())
    return status
