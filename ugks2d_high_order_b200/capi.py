"""ctypes binding of libugks_b200.so (include/ugks_b200.h).

The binding loads the in-tree library only.  There is no CPU fallback: if the library is missing
or no CUDA device is present, constructing a Solver raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libugks_b200.so")

UGKS_OK = 0
UGKS_EINVAL = 1
UGKS_ECUDA = 2
UGKS_ENUMERIC = 3
UGKS_ETIMEOUT = 4
UGKS_ENOMEM = 5
UGKS_EUNSUPPORTED = 6
UGKS_METHOD_EXPLICIT = 0
UGKS_METHOD_IMPLICIT_STEADY = 1
UGKS_METHOD_HIGH_ORDER_IMPLICIT = 2
UGKS_METHOD_S2CN2 = 3

# every symbol include/ugks_b200.h declares (checked by the CPU test suite)
EXPORTS = [
    "ugks_ctx_create", "ugks_ctx_destroy", "ugks_upload_state", "ugks_download_state", "ugks_init_freestream",
    "ugks_timestep", "ugks_evolution", "ugks_compute_residual", "ugks_apply_explicit_update",
    "ugks_step_explicit", "ugks_wall_aero", "ugks_macro_fields", "ugks_copy_array", "ugks_last_status", "ugks_status_reference_code",
    "ugks_error_string", "ugks_stream", "ugks_synchronize", "ugks_profile_enable", "ugks_profile_read",
    "ugks_launch_count", "ugks_step_explicit_noalloc", "ugks_implicit_init", "ugks_implicit_restore", "ugks_implicit_steps",
    "ugks_implicit_state", "ugks_s2cn2_init", "ugks_s2cn2_steps",
    "ugks_s2cn2_test_reject", "ugks_batch_create", "ugks_batch_destroy", "ugks_batch_init_freestream",
    "ugks_batch_run", "ugks_batch_tune", "ugks_batch_set_streams", "ugks_batch_upload", "ugks_batch_download",
    "ugks_batch_report", "ugks_batch_wall_aero", "ugks_batch_launch_count", "ugks_batch_stream",
    "ugks_evolution_s2", "ugks_upload_state_halo", "ugks_download_state_halo", "ugks_s2cn2_report",
    "ugks_s2cn2_forward_checkpointed", "ugks_s2cn2_backward", "ugks_s2cn2_step_vjp",
]
REPORT_LEN = 80
CN_REPORT_LEN = 24
# stages of one ImplicitSteady pseudo-step timed by the profile mode (kImStageNames in ugks_implicit.cuh)
IMPLICIT_STAGES = ("timestep", "pre_evaluation", "pr2_sweep", "equilibrium", "lusgs_forward", "wall_closure",
                   "lusgs_backward", "micro_alpha", "apply", "rescale", "post_fluxes", "post_residual")


class UgksParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nvel", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("ck", ctypes.c_int),
        ("pr", ctypes.c_double), ("omega", ctypes.c_double), ("mu_ref", ctypes.c_double), ("cfl", ctypes.c_double),
        ("wall_ux", ctypes.c_double * 2), ("wall_tnative", ctypes.c_double * 2),
        ("fixed_dt", ctypes.c_double),
        ("method", ctypes.c_int),
        ("ncfl", ctypes.c_double), ("nslab", ctypes.c_int), ("mass_rescale", ctypes.c_int),
        ("macro_sweeps", ctypes.c_int),
        ("residual_tol", ctypes.c_double), ("moment_tol", ctypes.c_double), ("min_alpha", ctypes.c_double),
        ("s2_kinetic_wall", ctypes.c_int), ("s2_time_centered", ctypes.c_int), ("s2_face_time", ctypes.c_int),
        ("s2_shared_predictor", ctypes.c_int),
    ]


class UgksInstanceDesc(ctypes.Structure):
    _fields_ = [("params", UgksParams), ("u", ctypes.c_void_p), ("v", ctypes.c_void_p), ("w", ctypes.c_void_p)]


class UgksError(RuntimeError):
    def __init__(self, code, msg, status=0, reference_code=0):
        super().__init__(f"{msg} (ugks code {code}, device status 0x{status:x}, reference abort {reference_code})")
        self.code = code
        self.status = status
        self.reference_code = reference_code


_lib = None


def load(path=LIB_PATH):
    """Load the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} not found: build it with `python -m ugks2d_high_order_b200.build`")
    L = ctypes.CDLL(path)
    dp = ctypes.POINTER(ctypes.c_double)
    vp = ctypes.c_void_p
    L.ugks_ctx_create.argtypes = [ctypes.POINTER(UgksParams), dp, dp, dp, ctypes.c_int, ctypes.POINTER(vp)]
    L.ugks_ctx_destroy.argtypes = [vp]
    L.ugks_upload_state.argtypes = [vp, dp, dp, dp]
    L.ugks_download_state.argtypes = [vp, dp, dp, dp]
    L.ugks_init_freestream.argtypes = [vp] + [ctypes.c_double] * 4
    L.ugks_timestep.argtypes = [vp, dp]
    L.ugks_evolution.argtypes = [vp]
    L.ugks_evolution_s2.argtypes = [vp, ctypes.c_int]
    L.ugks_upload_state_halo.argtypes = [vp, dp, dp, dp, ctypes.c_int]
    L.ugks_download_state_halo.argtypes = [vp, dp, dp, dp, ctypes.c_int]
    L.ugks_s2cn2_report.argtypes = [vp, dp]
    L.ugks_s2cn2_forward_checkpointed.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
    L.ugks_s2cn2_backward.argtypes = [vp, dp, dp, dp, dp, dp]
    L.ugks_s2cn2_step_vjp.argtypes = [vp, dp, dp, dp, dp, dp, dp, dp, dp]
    L.ugks_compute_residual.argtypes = [vp, ctypes.c_int]
    L.ugks_apply_explicit_update.argtypes = [vp, dp]
    L.ugks_step_explicit.argtypes = [vp, ctypes.c_int, dp, dp]
    L.ugks_wall_aero.argtypes = [vp, dp]
    L.ugks_macro_fields.argtypes = [vp, dp]
    L.ugks_copy_array.argtypes = [vp, ctypes.c_char_p, dp, ctypes.c_size_t]
    L.ugks_last_status.argtypes = [vp]
    L.ugks_last_status.restype = ctypes.c_uint
    L.ugks_status_reference_code.argtypes = [ctypes.c_uint]
    L.ugks_error_string.argtypes = [ctypes.c_int]
    L.ugks_error_string.restype = ctypes.c_char_p
    L.ugks_stream.argtypes = [vp]
    L.ugks_stream.restype = vp
    L.ugks_synchronize.argtypes = [vp]
    L.ugks_profile_enable.argtypes = [vp, ctypes.c_int]
    L.ugks_profile_read.argtypes = [vp, ctypes.c_char_p, dp, ctypes.POINTER(ctypes.c_longlong)]
    L.ugks_launch_count.argtypes = [vp]
    L.ugks_launch_count.restype = ctypes.c_longlong
    L.ugks_step_explicit_noalloc.argtypes = [ctypes.POINTER(UgksParams), vp, vp, vp, vp, vp, vp, ctypes.c_int, vp,
                                             dp, dp]
    L.ugks_implicit_init.argtypes = [vp]
    L.ugks_implicit_restore.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int]
    L.ugks_implicit_steps.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), dp]
    L.ugks_implicit_state.argtypes = [vp, dp, dp]
    L.ugks_s2cn2_init.argtypes = [vp]
    L.ugks_s2cn2_steps.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), dp]
    L.ugks_s2cn2_test_reject.argtypes = [vp, ctypes.c_int]
    ip = ctypes.POINTER(ctypes.c_int)
    L.ugks_batch_create.argtypes = [ctypes.c_int, ctypes.POINTER(UgksInstanceDesc), ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(vp)]
    L.ugks_batch_destroy.argtypes = [vp]
    L.ugks_batch_init_freestream.argtypes = [vp] + [ctypes.c_double] * 4
    L.ugks_batch_run.argtypes = [vp, ctypes.c_int, ip, ctypes.POINTER(ctypes.c_uint)]
    L.ugks_batch_tune.argtypes = [vp, ctypes.c_int, ip, dp]
    L.ugks_batch_set_streams.argtypes = [vp, ctypes.c_int]
    L.ugks_batch_upload.argtypes = [vp, ctypes.c_int, dp, dp, dp]
    L.ugks_batch_download.argtypes = [vp, ctypes.c_int, dp, dp, dp]
    L.ugks_batch_report.argtypes = [vp, ctypes.c_int, dp]
    L.ugks_batch_wall_aero.argtypes = [vp, ctypes.c_int, dp]
    L.ugks_batch_launch_count.argtypes = [vp]
    L.ugks_batch_launch_count.restype = ctypes.c_longlong
    L.ugks_batch_stream.argtypes = [vp]
    L.ugks_batch_stream.restype = vp
    _lib = L
    return L


def check(L, ctx, code, what):
    if code != UGKS_OK:
        st = L.ugks_last_status(ctx) if ctx else 0
        raise UgksError(code, f"{what}: {L.ugks_error_string(code).decode()}", st, L.ugks_status_reference_code(st))
