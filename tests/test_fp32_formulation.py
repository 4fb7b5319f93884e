"""The FP32 integrand of the CUDA kernels (cupythia_b200/csrc/cp_integrand.cuh), compiled for the
host, against the FP64 oracle: the FP32 formulation alone must hold 1e-5 relative per point."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))

REL_TOL = 1e-5      # per-point weight tolerance in FP32
TINY = 1e-12        # weights below TINY * mean underflow FP32 and carry no cross section


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    so = str(tmp_path_factory.mktemp("probe") / "fp32_probe.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", os.path.join(HERE, "fp32_probe.cc"),
                    "-o", so], check=True)
    return C.CDLL(so)


def _weights(probe, x, **kw):
    out = np.zeros(len(x), np.float32)
    args = dict(sqrtS=13000., pTmin=20., aSmZ=.13, kR=1., kF=1., conv=.389380)
    args.update(kw)
    rc = probe.probe_had_weights(*[C.c_double(args[k]) for k in ("sqrtS", "pTmin", "aSmZ", "kR", "kF", "conv")],
                                 31, x.ctypes.data_as(C.c_void_p), len(x), out.ctypes.data_as(C.c_void_p))
    assert rc == 0
    return out


@pytest.mark.parametrize("pTmin,aSmZ,kR", [(20., .13, 1.), (10., .11, .5), (50., .14, 2.)])
def test_fp32_weights_within_tolerance(probe, orc, pTmin, aSmZ, kR):
    rng = np.random.default_rng(7)
    n = 40000
    x = rng.random((n, 3)).astype(np.float32)
    # edges of the cube, where the poles and the PDF endpoints sit
    x[:2000, 2] = (1 - rng.random(2000) * 1e-4).astype(np.float32)
    x[2000:4000, 2] = (rng.random(2000) * 1e-4).astype(np.float32)
    x[4000:6000, 1] = (1 - rng.random(2000) * 1e-4).astype(np.float32)
    x[6000:8000, 0] = (rng.random(2000) * 1e-4).astype(np.float32)
    got = _weights(probe, x, pTmin=pTmin, aSmZ=aSmZ, kR=kR)
    ref = orc.weight_x_batch(orc.had_cfg(pTmin=pTmin, aSmZ=aSmZ, kR=kR), x)
    keep = ref > TINY * ref.mean()
    rel = np.abs(got[keep] - ref[keep]) / ref[keep]
    assert rel.max() < REL_TOL, (rel.max(), np.percentile(rel, 99))
    assert np.all(np.isfinite(got))


def test_probe_philox_matches_oracle(probe, orc):
    out = (C.c_uint32 * 4)()
    rng = np.random.default_rng(1)
    for _ in range(100):
        c = [int(v) for v in rng.integers(0, 2 ** 32, 6)]
        probe.probe_philox(*[C.c_uint32(v) for v in c], out)
        ref = (C.c_uint32 * 4)()
        orc.lib().cpo_philox4x32_10((C.c_uint32 * 4)(*c[:4]), (C.c_uint32 * 2)(*c[4:]), ref)
        assert list(out) == list(ref)


def test_dual_number_gradients_match_complex_step(probe, orc):
    """The adjoint kernel's forward-mode integrand (cp_dual.cuh) against the FP64 complex-step
    derivatives of the oracle, at the same FP32 points."""
    L = orc.lib()
    probe.probe_had_grad.argtypes = [C.c_double] * 4 + [C.c_void_p, C.c_void_p]
    rng = np.random.default_rng(9)
    cfg = orc.had_cfg()
    worst = 0.0
    for _ in range(400):
        x = rng.uniform(0.02, 0.98, 3).astype(np.float32)
        got = np.zeros(7)
        assert probe.probe_had_grad(13000., 20., .13, 1., x.ctypes.data, got.ctypes.data) == 0
        ref = (C.c_double * 7)()
        L.cpo_had_weight_grad(C.byref(cfg), orc.dptr(x.astype(np.float64)), ref)
        ref = np.array(ref[:])
        assert abs(got[0] / ref[0] - 1) < 1e-4
        # derivative scale: |w| per unit of each variable (x in [0,1], alpha_s ~ 0.1, k ~ 1, pT ~ 20)
        scale = np.abs(ref[0]) * np.array([1, 1, 1, 1 / 0.13, 1.0, 1 / 20.0])
        err = np.abs(got[1:] - ref[1:]) / (np.abs(ref[1:]) + 1e-3 * scale)
        worst = max(worst, err.max())
    assert worst < 2e-3, worst


@pytest.mark.parametrize("lo,hi", [(-32.1, 3.7), (-13.9, 0.0), (-80.0, 0.0), (-0.35, 0.35)])
def test_exp_reduction_within_its_bound(probe, lo, hi):
    """cp_exp_reduce2 (e^a = 2^k e^r, Taylor e^r - 1 to r^7) over the argument ranges its callers
    pass (CTEQ5L's p ln y, the beams' ln x, x0 ln tauMin, and the k = 0 band around zero) against
    FP64, in units u = 2^-24: e^a within 2.5 u relative, e^a - 1 within 2.5 u of max(|e^a - 1|, 1)
    and, for |a| < ln 2 / 2, within 2.5 u relative."""
    rng = np.random.default_rng(3)
    a = rng.uniform(lo, hi, 400000).astype(np.float32)
    a[:4] = np.array([lo, hi, 0.0, -1e-30], np.float32)
    e = np.zeros_like(a)
    m = np.zeros_like(a)
    fp = C.POINTER(C.c_float)
    probe.probe_exp_reduce(a.ctypes.data_as(fp), len(a), e.ctypes.data_as(fp), m.ctypes.data_as(fp))
    ad = a.astype(np.float64)
    ulp = 2.0 ** -24
    ref_e, ref_m = np.exp(ad), np.expm1(ad)
    assert np.max(np.abs(e - ref_e) / ref_e) < 2.5 * ulp
    assert np.max(np.abs(m - ref_m) / np.maximum(np.abs(ref_m), 1.0)) < 2.5 * ulp
    small = (np.abs(ad) < 0.3465) & (ad != 0)
    if small.any():
        assert np.max(np.abs(m[small] - ref_m[small]) / np.abs(ref_m[small])) < 2.5 * ulp
    assert m[2] == 0.0 and m[3] == np.float32(-1e-30)


def test_parameter_builder_keeps_the_exp_reduction_in_range(probe):
    """x0 ln tauMin enters the kernels' exp reduction, whose 2^k scale is valid for arguments above
    -87: configurations with ln tauMin <= -80 are refused, ordinary ones accepted."""
    f = probe.probe_build_params
    f.argtypes = [C.c_double, C.c_double, C.c_double]
    assert f(13000.0, 20.0, 0.13) == 0
    assert f(1.0e6, 2.0, 0.13) == 0              # ln tauMin = ln(16 / 1e12) = -27.2
    assert f(1.0e18, 2.0, 0.13) != 0             # ln tauMin = -80.1
