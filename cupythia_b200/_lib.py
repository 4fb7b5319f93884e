"""ctypes binding of the C ABI declared in include/cupythia_b200.h.

The product path is the CUDA library only: if ``libcupythia_b200.so`` cannot be loaded the
import raises, there is no CPU fallback.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("CUPYTHIA_B200_LIB") or os.path.join(HERE, "libcupythia_b200.so")

CP_OK = 0
CP_ERR_INVALID = 1
CP_ERR_CUDA = 2
CP_ERR_NUMERIC = 3
CP_ERR_TIMEOUT = 4
CP_ERR_CAPACITY = 5
CP_ERR_NOMEM = 6

CP_PROC_GG2GG = 1
CP_PROC_GG2QQBAR = 2
CP_PROC_QG2QG = 4
CP_PROC_QQ2QQ = 8
CP_PROC_QQBAR2GG = 16
CP_PROC_ALL = 31
CP_MAX_BINS = 128


class cp_config(C.Structure):
    _fields_ = [
        ("sqrt_s", C.c_double), ("pt_hat_min", C.c_double), ("alphas_mz", C.c_double),
        ("k_ren", C.c_double), ("k_fac", C.c_double), ("convert2mb", C.c_double),
        ("n_quark_in", C.c_int), ("n_quark_new", C.c_int), ("proc_mask", C.c_int),
        ("n_bins", C.c_int), ("device", C.c_int), ("reserved", C.c_int), ("seed", C.c_uint64),
    ]


class cp_result(C.Structure):
    _fields_ = [
        ("sigma", C.c_double), ("sigma_err", C.c_double), ("sum_w", C.c_double),
        ("sum_w2", C.c_double), ("w_max", C.c_double), ("n_points", C.c_uint64),
        ("n_bad", C.c_uint64), ("eta", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class cp_event(C.Structure):
    _fields_ = [
        ("id", C.c_int16 * 4), ("pz_in", C.c_float * 2), ("p3", C.c_float * 4),
        ("p4", C.c_float * 4), ("weight", C.c_float), ("pt_hat", C.c_float),
        ("process", C.c_uint16), ("colour", C.c_uint16), ("point", C.c_uint32),
    ]


class cp_unweight_result(C.Structure):
    _fields_ = [
        ("sigma", C.c_double), ("sigma_err", C.c_double), ("sigma_unweighted", C.c_double),
        ("w_max", C.c_double), ("w_max_seen", C.c_double), ("eta", C.c_double),
        ("n_points", C.c_uint64), ("n_accepted", C.c_uint64), ("n_overweight", C.c_uint64),
        ("n_bad", C.c_uint64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class cp_grad(C.Structure):
    _fields_ = [
        ("sigma", C.c_double), ("var", C.c_double), ("dsigma", C.c_double * 3),
        ("dvar", C.c_double * 3), ("n_points", C.c_uint64), ("n_bad", C.c_uint64),
    ]


class cp_device_events(C.Structure):
    """The reference pipeline's DeviceEvents (cuPythia/pipeline/event.cuh:20-31), member for member."""
    _fields_ = [("nEvents", C.c_int), ("maxPart", C.c_int), ("nVar", C.c_int)] + [
        (f, C.c_void_p) for f in ("px", "py", "pz", "e", "m", "pdg", "status", "col", "acol", "mo1", "mo2",
                                  "d1", "d2", "nPart", "seed", "scale", "x1", "x2", "flavA", "flavB",
                                  "active", "weight")]


_P = C.c_void_p
_u64 = C.c_uint64
_u32 = C.c_uint32
_i64 = C.c_int64
_d = C.c_double
_i = C.c_int

# name -> argtypes; every function returns int status except where noted
SIGNATURES = {
    "cp_abi_version": [],
    "cp_config_default": [C.POINTER(cp_config)],
    "cp_create": [C.POINTER(cp_config), C.POINTER(_P)],
    "cp_destroy": [_P],
    "cp_set_stream": [_P, _P],
    "cp_set_point_offset": [_P, _u64],
    "cp_pick_state_batch": [_P, _i, _P, _P, _P],
    "cp_set_scale_weights": [_P, _P, _u64],
    "cp_vegas_accumulate": [_P, _u64, _u32, _P],
    "cp_vegas_refine_sums": [_P, _P, _d, _d, C.POINTER(cp_result)],
    "cp_weight_histogram": [_P, _P],
    "cp_weight_quantile_hist": [_P, _P, _d, C.POINTER(_d)],
    "cp_synchronize": [_P],
    "cp_device_sm_count": [_P, C.POINTER(_i)],
    "cp_philox_words": [_P, _u64, _u64, _u64, _u32, _u32, _P],
    "cp_splitmix_uniforms": [_P, _u64, _u64, _u64, _P],
    "cp_event_keys": [_P, _u64, _u64, _u64, _P],
    "cp_set2kin_batch": [_P, _P, _P, _P, _P, _i64],
    "cp_set2kin_batch_f64": [_P, _P, _P, _P, _P, _i64],
    "cp_sigma_kin_batch": [_P, _i, _P],
    "cp_sigma_hat_batch": [_P, _i, _i, _i, _P],
    "cp_sigma_pdf_batch": [_P, _i, _P],
    "cp_scales_batch": [_P, _P, _P, _P],
    "cp_pdf_batch": [_P, _P, _P, _i64, _P],
    "cp_grid_reset": [_P],
    "cp_grid_set": [_P, C.POINTER(_d)],
    "cp_grid_get": [_P, C.POINTER(_d)],
    "cp_vegas_iteration": [_P, _u64, _u32, _d, C.POINTER(cp_result)],
    "cp_integrate": [_P, _i, _u64, _d, _i, C.POINTER(cp_result), C.POINTER(cp_result)],
    "cp_point_weights": [_P, _u64, _u64, _u32, _P, _P],
    "cp_weight_at": [_P, _P, _i64, _P],
    "cp_last_histogram": [_P, C.POINTER(_d)],
    "cp_weight_quantile": [_P, _d, C.POINTER(_d)],
    "cp_set_wmax": [_P, _d],
    "cp_unweight": [_P, _u64, _u32, _P, _u64, C.POINTER(cp_unweight_result)],
    "cp_generate_host": [_P, _u64, _u32, _u64, _P, _u64, C.POINTER(cp_unweight_result)],
    "cp_adjoint": [_P, _u64, _u32, _u32, C.POINTER(cp_grad), _P, _P],
    "cp_vegas_gradient_step": [_P, _u64, _u32, _d, C.POINTER(cp_grad)],
    "cp_adjoint_sums_size": [_P, C.POINTER(_i)],
    "cp_vegas_gradient_objective": [_P, _d],
    "cp_adjoint_parameter_tangents": [_P, _i],
    "cp_adjoint_accumulate": [_P, _u64, _u32, _u32, _P],
    "cp_vegas_gradient_apply": [_P, _P, _u64, _d, C.POINTER(cp_grad)],
    "cp_flow_step_moments": [_P, _u64, _u64, _P],
    "cp_flow_step_gradient": [_P, _P, _u64, _P, _P],
    "cp_flow_step_update": [_P, _P, _d],
    "cp_records_to_device_events": [_P, _P, _u64, _P, C.POINTER(cp_device_events), _u64],
    "cp_flow_num_params": [],
    "cp_flow_init": [_P, _u64],
    "cp_flow_get_params": [_P, _P, _i],
    "cp_flow_set_params": [_P, _P, _i],
    "cp_flow_state_size": [],
    "cp_flow_get_state": [_P, _P, _i, C.POINTER(_i64)],
    "cp_flow_set_state": [_P, _P, _i, _i64],
    "cp_flow_sample": [_P, _u64, _u64, _u32, _u32, _P],
    "cp_flow_enable": [_P, _i],
    "cp_flow_select_kernel": [_P, _i],
    "cp_flow_fuse_production": [_P, _i],
    "cp_flow_test_stall": [_P, _i],
    "cp_colour_tags": [C.c_uint16, C.c_uint16, _P, _P],
    "cp_set_id_col_acol": [_i, _i, _i, _d, _d, _i, _d, _d, _d, _P, _P, _P],
    "cp_write_lhef": [C.POINTER(cp_config), _P, _u64, _d, _d, C.c_char_p],
    "cp_flow_train": [_P, _i, _u64, _d, _P],
    "cp_flow_set_objective": [_P, _d],
    "cp_flow_loss_grad": [_P, _u64, _u32, _P, _P],
    "cp_set_kernel_timing": [_P, _i],
    "cp_kernel_times": [_P, _P, _P, _i],
    "cp_measure_peaks": [_P, C.POINTER(_d), C.POINTER(_d)],
    "cp_vegas_pass_noalloc": [C.POINTER(cp_config), _u64, _u32, _P, _P, _P],
    "cp_partonic_integrate": [_P, _d, _d, _d, _d, _u64, _u64, C.POINTER(cp_result)],
    "cp_partonic_splitmix": [_P, _d, _d, _d, _d, _u64, _u64, _u64, C.POINTER(cp_result)],
    "cp_partonic_weights": [_P, _d, _d, _d, _d, _u64, _u64, _u64, _P],
}
OPTIONAL = {}
EXTRA_RESTYPES = {"cp_last_error": C.c_char_p}

CP_SLOT_HEAD = 4
CP_QBINS = 4096

_lib = None


def load():
    """Load the CUDA library (raises OSError when it is missing: no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing; build it with `python -m cupythia_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, args in list(SIGNATURES.items()) + list(OPTIONAL.items()):
        if not hasattr(lib, name):
            if name in OPTIONAL:
                continue
            raise OSError(f"{LIB_PATH} does not export {name}")
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    lib.cp_last_error.argtypes = [_P]
    lib.cp_last_error.restype = C.c_char_p
    _lib = lib
    return lib


class CpError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cupythia_b200 error {code}: {msg}")
        self.code = code


def check(lib, handle, rc):
    if rc != CP_OK:
        msg = lib.cp_last_error(handle).decode() if handle else ""
        raise CpError(rc, msg)
    return rc
