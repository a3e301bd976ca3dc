"""ctypes binding of libncs_b200.so (C ABI in include/ncs_b200.h).

The library is the only compute path: importing the package raises if it is
not built (require), and the first call that needs it loads it (load), which
raises if it fails to load -- there is no CPU fallback.  Loading on first use
keeps processes that only use the package's host-side helpers (the seeded
workload generators) from mapping the library.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libncs_b200.so")

NCSB_OK = 0
NCSB_EINVAL = -1
NCSB_ECUDA = -2
NCSB_ENOMASK = -3
NCSB_ESIZE = -4
NCSB_ESCRATCH = -5

MODE_PLAIN = 0
MODE_PLAIN_WG = 1
MODE_SPECTRAL = 2
MODE_TC_TF32 = 3
MODE_TC_BF16X3 = 4

# raw-frame element types (NCSB_ADU_*)
ADU_F32 = 0
ADU_U16 = 1
ADU_U8 = 2

# Per-tile status codes (cuda/ncs.cu:61-67).
SUCCESS = 0
UNSTARTED = -1
REACHED_MAXITERS = -2
INCREASING_GRADIENT = -3
MINIMUM_STEP = -4
REACHED_MAXPRECISION = -5
STATUS_NAMES = {
    UNSTARTED: "Unstarted",
    REACHED_MAXITERS: "Reached maximum iterations",
    INCREASING_GRADIENT: "Increasing gradient",
    MINIMUM_STEP: "Reached minimum step size",
    REACHED_MAXPRECISION: "Reached machine precision",
}


class NcsbParams(ctypes.Structure):
    _fields_ = [
        ("alpha", ctypes.c_double),
        ("max_iters", ctypes.c_int32),
        ("m", ctypes.c_int32),
        ("epsilon", ctypes.c_double),
        ("c1", ctypes.c_double),
        ("min_step", ctypes.c_double),
        ("mode", ctypes.c_int32),
        ("ctas_per_sm", ctypes.c_int32),
    ]


MASK_TYPES = {"OTFweighted": 0, "pureN": 1, "adjustable": 2, "incoherent": 3}


class NcsbOptics(ctypes.Structure):
    """ncsb_optics: parameters of a mask built on the device."""
    _fields_ = [
        ("type", ctypes.c_int32),
        ("pixel_size", ctypes.c_double),
        ("na", ctypes.c_double),
        ("wavelength", ctypes.c_double),
        ("w", ctypes.c_double),
        ("h", ctypes.c_double),
    ]


def optics(type="OTFweighted", pixel_size=0.1, NA=1.4, wavelength=0.7, w=1.0, h=0.7):
    o = NcsbOptics()
    o.type = MASK_TYPES[type]
    o.pixel_size, o.na, o.wavelength, o.w, o.h = pixel_size, NA, wavelength, w, h
    return o


class NcsbStack(ctypes.Structure):
    """ncsb_stack: one stack of a batched launch."""
    _fields_ = [
        ("images", ctypes.c_void_p),
        ("gamma", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
        ("n_frames", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("width", ctypes.c_int32),
        ("gamma_per_frame", ctypes.c_int32),
        ("alpha", ctypes.c_double),
        ("mask_shifted", ctypes.c_float * 256),
        ("mask_from_optics", ctypes.c_int32),
        ("optics", NcsbOptics),
    ]


class NcsbCalibration(ctypes.Structure):
    """ncsb_calibration: camera maps for raw-ADU input."""
    _fields_ = [
        ("offset", ctypes.c_void_p),
        ("gain", ctypes.c_void_p),
        ("variance", ctypes.c_void_p),
        ("n_levels", ctypes.c_int32),
        ("levels", ctypes.c_float * 3),
    ]


MAX_STACKS = 65536

# Every symbol include/ncs_b200.h declares (checked by the tests).
EXPORTS = [
    "ncsb_default_params", "ncsb_create", "ncsb_set_params", "ncsb_destroy", "ncsb_last_error",
    "ncsb_set_otf_mask", "ncsb_num_tiles", "ncsb_reduce_noise", "ncsb_solve_tiles",
    "ncsb_reduce_noise_noalloc", "ncsb_reduce_noise_start",
    "ncsb_net_param_count", "ncsb_net_conv_fwd", "ncsb_net_conv_wgrad", "ncsb_net_flip",
    "ncsb_net_relu_bwd", "ncsb_net_mse_grad", "ncsb_net_adam", "ncsb_net_features",
    "ncsb_net_infer_stack", "ncsb_net_infer_tiles", "ncsb_net_infer_batch",
    "ncsb_batch_set", "ncsb_batch_num_tiles", "ncsb_batch_reduce_noise",
    "ncsb_reduce_noise_adu", "ncsb_genfilter",
    "ncsb_sim_render", "ncsb_sim_camera", "ncsb_sim_uniforms", "ncsb_reduce_noise_normalized",
    "ncsb_net_infer_stack_tc", "ncsb_net_infer_tiles_tc", "ncsb_genpsfparam",
    "ncsb_net_infer_batch_tc", "ncsb_reduce_noise_host",
    "ncsb_net_infer_stack_tc_fp8", "ncsb_net_infer_tiles_tc_fp8", "ncsb_net_infer_batch_tc_fp8",
    "ncsb_reduce_noise_adu_typed", "ncsb_reduce_noise_adu_host", "ncsb_sim_ideal_image",
]

_lib = None


def require():
    """Raise OSError unless the library has been built."""
    if not os.path.exists(LIB_PATH):
        raise OSError("libncs_b200.so is not built; run `python ncs_b200/build.py`")


def load():
    """Load and type the library (raises OSError if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError("libncs_b200.so is not built; run `python ncs_b200/build.py`")
    lib = ctypes.CDLL(LIB_PATH)
    vp, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
    P = ctypes.POINTER
    lib.ncsb_default_params.argtypes = [P(NcsbParams)]
    lib.ncsb_default_params.restype = None
    lib.ncsb_create.argtypes = [P(vp), P(NcsbParams)]
    lib.ncsb_create.restype = ctypes.c_int
    lib.ncsb_set_params.argtypes = [vp, P(NcsbParams)]
    lib.ncsb_set_params.restype = ctypes.c_int
    lib.ncsb_destroy.argtypes = [vp]
    lib.ncsb_destroy.restype = ctypes.c_int
    lib.ncsb_last_error.argtypes = [vp]
    lib.ncsb_last_error.restype = ctypes.c_char_p
    lib.ncsb_set_otf_mask.argtypes = [vp, P(ctypes.c_float)]
    lib.ncsb_set_otf_mask.restype = ctypes.c_int
    lib.ncsb_num_tiles.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, P(i64)]
    lib.ncsb_num_tiles.restype = ctypes.c_int
    lib.ncsb_reduce_noise.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp,
                                      ctypes.c_int, vp, vp, vp, vp, vp, vp]
    lib.ncsb_reduce_noise.restype = ctypes.c_int
    lib.ncsb_solve_tiles.argtypes = [vp, vp, vp, vp, i64, vp, vp, vp, vp, vp, vp]
    lib.ncsb_solve_tiles.restype = ctypes.c_int
    lib.ncsb_reduce_noise_noalloc.argtypes = [P(NcsbParams), P(ctypes.c_float), vp, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, vp,
                                              vp, vp, vp, vp, vp]
    lib.ncsb_reduce_noise_noalloc.restype = ctypes.c_int
    lib.ncsb_reduce_noise_start.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp,
                                            ctypes.c_int, vp, vp, vp, vp, vp, vp, vp, vp]
    lib.ncsb_reduce_noise_start.restype = ctypes.c_int
    ci, f32 = ctypes.c_int, ctypes.c_float
    lib.ncsb_net_param_count.argtypes = []
    lib.ncsb_net_conv_fwd.argtypes = [vp, vp, vp, vp, ci, ci, ci, ci, vp]
    lib.ncsb_net_conv_wgrad.argtypes = [vp, vp, vp, vp, ci, ci, ci, vp]
    lib.ncsb_net_flip.argtypes = [vp, vp, ci, ci, vp]
    lib.ncsb_net_relu_bwd.argtypes = [vp, vp, i64, vp]
    lib.ncsb_net_mse_grad.argtypes = [vp, vp, vp, vp, i64, vp]
    lib.ncsb_net_adam.argtypes = [vp, vp, vp, vp, i64, f32, f32, f32, f32, ci, vp]
    lib.ncsb_net_features.argtypes = [vp, vp, vp, vp, ci, vp]
    lib.ncsb_net_infer_stack.argtypes = [vp, vp, ci, ci, ci, vp, ci, vp, vp]
    lib.ncsb_net_infer_tiles.argtypes = [vp, vp, vp, i64, vp, vp]
    lib.ncsb_reduce_noise_adu.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          P(NcsbCalibration), vp, vp, vp, vp, vp, vp]
    lib.ncsb_reduce_noise_adu.restype = ctypes.c_int
    lib.ncsb_reduce_noise_adu_typed.argtypes = [vp, vp, ci, ci, ci, ci, P(NcsbCalibration), vp,
                                                vp, vp, vp, vp, vp]
    lib.ncsb_reduce_noise_adu_typed.restype = ctypes.c_int
    lib.ncsb_reduce_noise_adu_host.argtypes = [vp, vp, ci, ci, ci, ci, P(NcsbCalibration), vp,
                                               ci, ci, vp]
    lib.ncsb_reduce_noise_adu_host.restype = ctypes.c_int
    lib.ncsb_sim_render.argtypes = [vp, vp, ci, ci, ctypes.c_double, ci, f32, vp, vp]
    lib.ncsb_sim_render.restype = ctypes.c_int
    lib.ncsb_sim_camera.argtypes = [vp, ci, ci, ci, vp, vp, vp, ctypes.c_uint64, vp, vp, vp]
    lib.ncsb_sim_camera.restype = ctypes.c_int
    lib.ncsb_sim_ideal_image.argtypes = [vp, vp, ci, ci, ci, vp, ci, vp, vp, vp]
    lib.ncsb_sim_ideal_image.restype = ctypes.c_int
    lib.ncsb_sim_uniforms.argtypes = [i64, ctypes.c_uint32, ctypes.c_uint64, vp, vp]
    lib.ncsb_sim_uniforms.restype = ctypes.c_int
    lib.ncsb_reduce_noise_normalized.argtypes = [vp, ci, ci, ci, vp, ci, P(ctypes.c_float),
                                                 ctypes.c_double, ci, ctypes.c_double, vp, vp,
                                                 vp, vp, vp]
    lib.ncsb_reduce_noise_normalized.restype = ctypes.c_int
    lib.ncsb_genpsfparam.argtypes = [ci, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                     vp, vp, vp, vp]
    lib.ncsb_genpsfparam.restype = ctypes.c_int
    lib.ncsb_genfilter.argtypes = [P(NcsbOptics), ctypes.c_int, vp, vp]
    lib.ncsb_genfilter.restype = ctypes.c_int
    lib.ncsb_net_infer_stack_tc.argtypes = [vp, vp, ci, ci, ci, vp, ci, vp, vp, vp]
    lib.ncsb_net_infer_stack_tc.restype = ctypes.c_int
    lib.ncsb_net_infer_tiles_tc.argtypes = [vp, vp, vp, i64, vp, vp, vp]
    lib.ncsb_net_infer_tiles_tc.restype = ctypes.c_int
    lib.ncsb_net_infer_batch_tc.argtypes = [vp, vp, vp, vp, vp]
    lib.ncsb_net_infer_batch_tc.restype = ctypes.c_int
    lib.ncsb_net_infer_stack_tc_fp8.argtypes = [vp, vp, ci, ci, ci, vp, ci, vp, vp, vp]
    lib.ncsb_net_infer_stack_tc_fp8.restype = ctypes.c_int
    lib.ncsb_net_infer_tiles_tc_fp8.argtypes = [vp, vp, vp, i64, vp, vp, vp]
    lib.ncsb_net_infer_tiles_tc_fp8.restype = ctypes.c_int
    lib.ncsb_net_infer_batch_tc_fp8.argtypes = [vp, vp, vp, vp, vp]
    lib.ncsb_net_infer_batch_tc_fp8.restype = ctypes.c_int
    lib.ncsb_reduce_noise_host.argtypes = [vp, vp, i32, i32, i32, vp, i32, vp, i32, i32, vp]
    lib.ncsb_reduce_noise_host.restype = ctypes.c_int
    lib.ncsb_net_infer_batch.argtypes = [vp, vp, vp, vp]
    lib.ncsb_batch_set.argtypes = [vp, P(NcsbStack), ctypes.c_int]
    lib.ncsb_batch_set.restype = ctypes.c_int
    lib.ncsb_batch_num_tiles.argtypes = [vp, P(i64)]
    lib.ncsb_batch_num_tiles.restype = ctypes.c_int
    lib.ncsb_batch_reduce_noise.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
    lib.ncsb_batch_reduce_noise.restype = ctypes.c_int
    for name in ("ncsb_net_infer_batch", "ncsb_net_param_count", "ncsb_net_conv_fwd", "ncsb_net_conv_wgrad",
                 "ncsb_net_flip", "ncsb_net_relu_bwd", "ncsb_net_mse_grad", "ncsb_net_adam",
                 "ncsb_net_features", "ncsb_net_infer_stack", "ncsb_net_infer_tiles"):
        getattr(lib, name).restype = ctypes.c_int
    _lib = lib
    return lib


def default_params():
    p = NcsbParams()
    load().ncsb_default_params(ctypes.byref(p))
    return p


def num_tiles(n_frames, height, width):
    n = ctypes.c_int64(0)
    rc = load().ncsb_num_tiles(int(n_frames), int(height), int(width), ctypes.byref(n))
    if rc != NCSB_OK:
        raise ValueError("frames of %dx%d cannot be tiled (need >= 14 on each axis)"
                         % (height, width))
    return n.value
