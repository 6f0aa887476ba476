"""ctypes binding of ``libfluxo_gpu.so`` (the C ABI declared in ``include/fluxo_gpu.h``).

The library is built in-tree by ``fluxo_b200/build.py``.  There is no fallback: if the
library is missing or fails to load, importing this module raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfluxo_gpu.so")

FLUXO_OK = 0
ERRORS = {
    -1: "FLUXO_EINVAL_CFG",
    -2: "FLUXO_ENOMEM_HBM",
    -3: "FLUXO_ECUDA",
    -4: "FLUXO_ENAN_STATE",
    -5: "FLUXO_ETIMEOUT",
    -6: "FLUXO_ENOTREADY",
    -7: "FLUXO_EXCHANGE",
}
FLUXO_XCHG_STATE, FLUXO_XCHG_GTRACE, FLUXO_XCHG_DT, FLUXO_XCHG_ALPHA = 1, 2, 3, 4
# fluxo_exchange_fn of include/fluxo_gpu.h: (ctx, what, stream, a, b) -> 0 or a failure
EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_void_p)


class FluxoError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "FLUXO_E?"), code, msg))
        self.code = code


class FluxoExact(ctypes.Structure):
    _fields_ = [
        ("func", ctypes.c_int),
        ("adv_vel", ctypes.c_double * 3),
        ("ini_wavenumber", ctypes.c_double * 3),
        ("ini_amplitude", ctypes.c_double),
        ("ini_frequency", ctypes.c_double),
        ("ref_state_prim", ctypes.c_double * 5),
        ("ini_center", ctypes.c_double * 3),
    ]


class FluxoCfg(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int),
        ("N", ctypes.c_int),
        ("eqn", ctypes.c_int),
        ("riemann", ctypes.c_int),
        ("volume_flux", ctypes.c_int),
        ("lifting", ctypes.c_int),
        ("lifting_var", ctypes.c_int),
        ("visc", ctypes.c_int),
        ("kappa", ctypes.c_double),
        ("R", ctypes.c_double),
        ("Pr", ctypes.c_double),
        ("mu0", ctypes.c_double),
        ("Ts", ctypes.c_double),
        ("Tref", ctypes.c_double),
        ("ExpoSuth", ctypes.c_double),
        ("ExpoPow", ctypes.c_double),
        ("etaBR2", ctypes.c_double),
        ("time_disc", ctypes.c_int),
        ("cfl_scale", ctypes.c_double),
        ("dfl_scale", ctypes.c_double),
        ("ini_exact_func", ctypes.c_int),
        ("ini_frequency", ctypes.c_double),
        ("ini_amplitude", ctypes.c_double),
        ("device", ctypes.c_int),
        ("mu_0", ctypes.c_double),
        ("eta", ctypes.c_double),
        ("glm_scale", ctypes.c_double),
        ("glm_scr", ctypes.c_double),
        ("noncons", ctypes.c_int),
        ("nc_glm", ctypes.c_int),
        ("nfvse", ctypes.c_int),
        ("compute_alpha", ctypes.c_int),
        ("shock_blend_coef", ctypes.c_double),
        ("modal_threshold", ctypes.c_int),
        ("alpha_max", ctypes.c_double),
        ("alpha_min", ctypes.c_double),
        ("space_prop_factor", ctypes.c_double),
        ("space_prop_sweeps", ctypes.c_int),
        ("time_rel_factor", ctypes.c_double),
        ("indicator_quantity", ctypes.c_int),
        ("sub_fv_method", ctypes.c_int),
        ("recons_boundaries", ctypes.c_int),
        ("nfvse_corr", ctypes.c_int),
        ("posit_corr_factor", ctypes.c_double),
        ("posit_max_iter", ctypes.c_int),
        ("node_type", ctypes.c_int),
    ]


EXPORTS = [
    "fluxo_gpu_create", "fluxo_gpu_set_mesh", "fluxo_gpu_set_state", "fluxo_gpu_get_state", "fluxo_gpu_get_ut",
    "fluxo_gpu_get_gradients", "fluxo_gpu_dg_time_derivative", "fluxo_gpu_calc_timestep", "fluxo_gpu_timestep",
    "fluxo_gpu_time_disc", "fluxo_gpu_device_buffers", "fluxo_gpu_launch_count", "fluxo_gpu_destroy",
    "fluxo_gpu_last_error", "fluxo_gpu_set_profiling", "fluxo_gpu_get_profile", "fluxo_gpu_fp64_peak",
    "fluxo_host_box_sizes", "fluxo_host_box_mesh", "fluxo_host_box_mesh_gauss", "fluxo_host_hopr_mesh",
    "fluxo_host_nodes",
    "fluxo_host_exact_func", "fluxo_gpu_dg_time_derivative_noalloc",
    "fluxo_gpu_set_glm_ch", "fluxo_gpu_get_glm_ch", "fluxo_gpu_get_alpha", "fluxo_gpu_set_alpha",
    "fluxo_gpu_set_partition", "fluxo_gpu_exchange_buffers", "fluxo_gpu_volume_shape",
    "fluxo_gpu_set_volume_shape", "fluxo_gpu_analyze", "fluxo_gpu_set_surf_metrics",
    "fluxo_batch_create", "fluxo_batch_add", "fluxo_batch_run", "fluxo_batch_status", "fluxo_batch_get_state",
    "fluxo_batch_set_state",
    "fluxo_batch_remove", "fluxo_batch_info", "fluxo_batch_stream", "fluxo_batch_instance_bytes",
    "fluxo_batch_last_error",
    "fluxo_batch_destroy", "fluxo_batch_loop_start", "fluxo_batch_loop_wake", "fluxo_batch_loop_poll",
    "fluxo_batch_loop_wait", "fluxo_batch_prepare", "fluxo_batch_add_prepared", "fluxo_batch_prepared_free",
]

# fluxo_batch_loop_* end reasons (FLUXO_LOOP_* of fluxo_gpu.h)
LOOP_IDLE, LOOP_FINISHED, LOOP_WOKEN, LOOP_STEP_LIMIT = 0, 1, 2, 3

# FLUXO_NOALLOC_SCRATCH_BYTES of fluxo_gpu.h: the static scratch of fluxo_gpu_dg_time_derivative_noalloc
NOALLOC_SCRATCH_BYTES = 8 * 1024 * 1024

_lib = None


def load():
    """Loads the library once and declares the argument types of every export."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libfluxo_gpu.so not built (run fluxo_b200/build.py): " + LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    vp, i, d, P = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.POINTER
    lib.fluxo_gpu_create.argtypes = [P(FluxoCfg), P(vp)]
    lib.fluxo_gpu_set_mesh.argtypes = [vp, i, i] + [vp] * 11
    lib.fluxo_gpu_set_surf_metrics.argtypes = [vp, vp]
    lib.fluxo_gpu_set_state.argtypes = [vp, vp]
    lib.fluxo_gpu_get_state.argtypes = [vp, vp]
    lib.fluxo_gpu_get_ut.argtypes = [vp, vp]
    lib.fluxo_gpu_get_gradients.argtypes = [vp, vp, vp, vp]
    lib.fluxo_gpu_dg_time_derivative.argtypes = [vp, d]
    lib.fluxo_gpu_calc_timestep.argtypes = [vp, P(d), P(i)]
    lib.fluxo_gpu_timestep.argtypes = [vp, d, d]
    lib.fluxo_gpu_time_disc.argtypes = [vp, d, d, i, P(d), P(i), P(i)]
    lib.fluxo_gpu_device_buffers.argtypes = [vp, P(vp), P(vp), P(vp)]
    lib.fluxo_gpu_launch_count.argtypes = [vp, P(ctypes.c_uint64)]
    lib.fluxo_gpu_destroy.argtypes = [vp]
    lib.fluxo_gpu_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
    lib.fluxo_gpu_set_profiling.argtypes = [vp, i]
    lib.fluxo_gpu_get_profile.argtypes = [vp, i, P(d), P(ctypes.c_uint64)]
    lib.fluxo_gpu_fp64_peak.argtypes = [i, P(d)]
    lib.fluxo_host_box_sizes.argtypes = [vp, P(i), P(i)]
    lib.fluxo_host_box_mesh.argtypes = [i, vp, vp, vp, i, d] + [vp] * 11
    lib.fluxo_host_box_mesh_gauss.argtypes = [i, vp, vp, vp, i, d] + [vp] * 12
    lib.fluxo_host_hopr_mesh.argtypes = [i, i, i, vp, i, vp, i, vp, i, i, vp, d, i] + [vp] * 12
    lib.fluxo_host_nodes.argtypes = [i, i, vp, vp]
    lib.fluxo_host_exact_func.argtypes = [i, d, ctypes.c_size_t, vp, d, vp, d, vp, d, vp, vp]
    lib.fluxo_gpu_dg_time_derivative_noalloc.argtypes = [P(FluxoCfg), i, i] + [vp] * 8
    lib.fluxo_gpu_set_glm_ch.argtypes = [vp, d]
    lib.fluxo_gpu_get_glm_ch.argtypes = [vp, P(d)]
    lib.fluxo_gpu_get_alpha.argtypes = [vp, vp]
    lib.fluxo_gpu_set_alpha.argtypes = [vp, vp]
    lib.fluxo_gpu_set_partition.argtypes = [vp, i, EXCHANGE_FN, vp]
    lib.fluxo_gpu_exchange_buffers.argtypes = [vp, P(vp)]
    lib.fluxo_gpu_volume_shape.argtypes = [i, i, i, P(i), P(i), P(i), P(i)]
    lib.fluxo_gpu_set_volume_shape.argtypes = [i, i, i, i]
    lib.fluxo_gpu_analyze.argtypes = [vp, d, P(FluxoExact), vp, vp, vp, vp]
    sz = ctypes.c_size_t
    lib.fluxo_batch_create.argtypes = [i, P(vp)]
    lib.fluxo_batch_add.argtypes = [vp, P(FluxoCfg), i, i] + [vp] * 11 + [d, d, i, P(i)]
    lib.fluxo_batch_run.argtypes = [vp, i, P(i)]
    lib.fluxo_batch_status.argtypes = [vp, i, P(d), P(i), P(i), P(i)]
    lib.fluxo_batch_get_state.argtypes = [vp, i, vp]
    lib.fluxo_batch_set_state.argtypes = [vp, i, vp]
    lib.fluxo_batch_remove.argtypes = [vp, i]
    lib.fluxo_batch_info.argtypes = [vp, P(i), P(i), P(sz)]
    lib.fluxo_batch_stream.argtypes = [vp, P(vp)]
    lib.fluxo_batch_instance_bytes.argtypes = [P(FluxoCfg), i, i, P(sz)]
    lib.fluxo_batch_last_error.argtypes = [vp, ctypes.c_char_p, sz]
    lib.fluxo_batch_destroy.argtypes = [vp]
    lib.fluxo_batch_prepare.argtypes = [P(FluxoCfg), i, i] + [vp] * 11 + [d, d, i, P(vp)]
    lib.fluxo_batch_add_prepared.argtypes = [vp, vp, P(i)]
    lib.fluxo_batch_prepared_free.argtypes = [vp]
    lib.fluxo_batch_loop_start.argtypes = [vp, i]
    lib.fluxo_batch_loop_wake.argtypes = [vp]
    lib.fluxo_batch_loop_poll.argtypes = [vp, P(i), P(i), P(i), P(i)]
    lib.fluxo_batch_loop_wait.argtypes = [vp, P(i), P(i), P(i)]
    for name in EXPORTS:
        getattr(lib, name).restype = ctypes.c_int
    _lib = lib
    return lib


def last_error(h):
    buf = ctypes.create_string_buffer(1024)
    load().fluxo_gpu_last_error(h, buf, 1024)
    return buf.value.decode(errors="replace")


def check(code, h=None):
    if code != FLUXO_OK:
        raise FluxoError(code, last_error(h))
