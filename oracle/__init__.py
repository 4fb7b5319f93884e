"""Python loader of the CPU oracle (oracle/libcp_oracle.so) and of the reference builds.

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module as the checker.  The product (cupythia_b200) never imports it.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libcp_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")
PYTHIA_REF = os.path.join(REF_DIR, "pythia_ref")
CUPYTHIA_REF = os.path.join(REF_DIR, "libcupythia_ref.so")

CPO_GG2GG, CPO_GG2QQBAR, CPO_QG2QG, CPO_QQ2QQ, CPO_QQBAR2GG, CPO_ALLQCD = 1, 2, 4, 8, 16, 31


class HadCfg(C.Structure):
    _fields_ = [("sqrtS", C.c_double), ("pTmin", C.c_double), ("aSmZ", C.c_double),
                ("kR", C.c_double), ("kF", C.c_double), ("convert2mb", C.c_double),
                ("nQuarkIn", C.c_int), ("nQuarkNew", C.c_int), ("procMask", C.c_int)]


_D = C.c_double
_PD = C.POINTER(C.c_double)
_U64 = C.c_uint64
_U32 = C.c_uint32
_SIG = {
    "cpo_splitmix64": (_U64, [_U64]),
    "cpo_u01": (_D, [_U64]),
    "cpo_thread_counter": (_U64, [_U64, _U64]),
    "cpo_event_key": (_U64, [_U64, _U64]),
    "cpo_philox4x32_10": (None, [C.POINTER(_U32), C.POINTER(_U32), C.POINTER(_U32)]),
    "cpo_point_words": (None, [_U64, _U64, _U32, _U32, C.POINTER(_U32)]),
    "cpo_sigma_gg2gg": (_D, [_D] * 4),
    "cpo_gg2gg_recip": (_D, [_D] * 4),
    "cpo_sigma_qq2qq": (_D, [_D] * 4 + [C.c_int, C.c_int]),
    "cpo_cteq5l_raw": (None, [_D, _D, _PD]),
    "cpo_pdf_xf": (_D, [C.c_int, _D, _D]),
    "cpo_had_default": (None, [C.c_void_p]),
    "cpo_had_sigma_pdf": (None, [C.c_void_p, _D, _D, _D, _D, C.c_int, _PD]),
    "cpo_had_weight_x": (_D, [C.c_void_p, _PD, _PD]),
    "cpo_opcount_weight": (_D, [C.c_void_p, _PD]),
    "cpo_opcount_counts": (None, [C.c_void_p, C.c_void_p, C.c_int64, _PD]),
    "cpo_had_weight_x_batch": (None, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int]),
    "cpo_vegas_map": (_D, [_PD, C.c_int, C.POINTER(_U32), _PD, C.POINTER(C.c_int)]),
    "cpo_had_point_weight": (_D, [C.c_void_p, _PD, C.c_int, _U64, _U32, _U64, C.POINTER(C.c_int), _PD]),
    "cpo_had_accumulate": (None, [C.c_void_p, _PD, C.c_int, _U64, _U32, _U64, _U64, _PD, _PD, C.c_int]),
    "cpo_vegas_refine": (None, [_PD, _PD, C.c_int, C.c_int, _D]),
    "cpo_vegas_uniform": (None, [_PD, C.c_int, C.c_int]),
    "cpo_partonic_weight": (_D, [_D] * 5),
    "cpo_partonic_philox": (None, [_D, _D, _D, _D, _U64, _U64, _U64, _PD, C.c_int]),
    "cpo_partonic_splitmix": (None, [_D, _D, _D, _D, _U64, _U64, _U64, _PD, C.c_int]),
    "cpo_simpson_gg2gg": (_D, [C.c_int, _D, _D, _D, _D]),
    "cpo_had_weight_grad": (None, [C.c_void_p, _PD, _PD]),
    "cpo_had_adjoint_sums": (None, [C.c_void_p, _PD, C.c_int, _U64, _U32, _U32, _U64, _U64, _PD, C.c_int]),
    "cpo_accept": (C.c_int, [_D, _D, _U32]),
    "cpo_pick_state": (C.c_int, [C.c_void_p, C.c_int, _D, _D, _D, _D, _D, _D, _D, _D, C.POINTER(C.c_int),
                                 C.POINTER(C.c_int)]),
    "cpo_pick_record": (C.c_int, [C.c_void_p, _PD, _D, _D, _D, _D, _D, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "cpo_pick_state_margin": (C.c_int, [C.c_void_p, C.c_int, _D, _D, _D, _D, _D, _D, _D, _D, C.POINTER(C.c_int),
                                        C.POINTER(C.c_int), _PD]),
    "cpo_pick_record_margin": (C.c_int, [C.c_void_p, _PD, _D, _D, _D, _D, _D, C.POINTER(C.c_int),
                                         C.POINTER(C.c_int), _PD]),
    "cpo_flow_forward": (None, [C.c_void_p, _PD, _PD, _PD]),
    "cpo_flow_set_rounding": (None, [C.c_int]),
    "cpo_flow_backward_batch": (None, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise OSError(f"{LIB} missing: run `make -f oracle/Makefile`")
        L = C.CDLL(LIB)
        for name, (res, args) in _SIG.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def had_cfg(**kw):
    c = HadCfg()
    lib().cpo_had_default(C.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def dptr(a):
    return a.ctypes.data_as(_PD)


def weight_x_batch(cfg, x, nthreads=None):
    x = np.ascontiguousarray(np.asarray(x, np.float32).reshape(-1, 3))
    out = np.zeros(x.shape[0])
    lib().cpo_had_weight_x_batch(C.byref(cfg), x.ctypes.data, x.shape[0], out.ctypes.data,
                                 nthreads or os.cpu_count() or 1)
    return out


def vegas_uniform(nb, ndim=3):
    e = np.zeros(ndim * (nb + 1))
    lib().cpo_vegas_uniform(dptr(e), ndim, nb)
    return e


def point_words(seed, points, iteration=0, stream=0):
    out = np.zeros((len(points), 4), np.uint32)
    w = (C.c_uint32 * 4)()
    for i, p in enumerate(points):
        lib().cpo_point_words(seed, int(p), iteration, stream, w)
        out[i] = w[:]
    return out


def cupythia_ref():
    """The reference's own rng.cuh / physics.cuh compiled as C++ (only where the reference
    was present at build time)."""
    L = C.CDLL(CUPYTHIA_REF)
    L.ref_splitmix64.restype = _U64
    L.ref_splitmix64.argtypes = [_U64]
    L.ref_u01.restype = _D
    L.ref_u01.argtypes = [_U64]
    L.ref_gg2gg_sigma.restype = _D
    L.ref_gg2gg_sigma.argtypes = [_D] * 4
    L.ref_fused_cpu_sum.restype = _D
    L.ref_fused_cpu_sum.argtypes = [_U64, _U64, _U64, _D, _D, _D, C.c_int]
    L.ref_cpuMC.restype = _D
    L.ref_cpuMC.argtypes = [_U64, _U64, _D, _D, _D]
    return L


def pick_record(cfg, x, r0, r1, r3, rc, rs, with_margin=False):
    """(code, ids[4], colour) of the oracle's record picks at the point x (cpo_pick_record); with
    with_margin also the draws' smallest relative distance from a selection boundary."""
    ids = (C.c_int * 4)()
    col = C.c_int()
    m = C.c_double()
    xx = np.ascontiguousarray(np.asarray(x, np.float64))
    code = lib().cpo_pick_record_margin(C.byref(cfg), dptr(xx), r0, r1, r3, rc, rs, ids, C.byref(col), C.byref(m))
    return (code, list(ids), col.value, m.value) if with_margin else (code, list(ids), col.value)


def pick_state(cfg, code, x1, x2, sH, tH, r1, r3, rc, rs, with_margin=False):
    """(code or 0, ids[4], colour) of the oracle's pickInState + setIdColAcol at given kinematics;
    with with_margin also the draws' smallest relative distance from a selection boundary."""
    ids = (C.c_int * 4)()
    col = C.c_int()
    m = C.c_double()
    got = lib().cpo_pick_state_margin(C.byref(cfg), code, x1, x2, sH, tH, r1, r3, rc, rs, ids, C.byref(col),
                                      C.byref(m))
    return (got, list(ids), col.value, m.value) if with_margin else (got, list(ids), col.value)

