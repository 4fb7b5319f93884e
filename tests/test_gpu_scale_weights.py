"""Scale-variation weights of the production pass (cp_set_scale_weights): the 7-point mu_R / mu_F
variation of every event's weight, against the FP64 oracle at the event's own point (the ratio of
oracle weights at the varied and nominal k_ren, k_fac), and the reweighted cross sections of the
unweighted sample against direct integrations at the varied scales.  Tolerances: 5e-5 relative
per ratio (FP32 weights carry ~6e-6 each); the reweighted cross sections within five combined
standard errors."""
import ctypes as C

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

N = 1 << 23
FACTORS = [(2, 1), (0.5, 1), (1, 2), (1, 0.5), (2, 2), (0.5, 0.5)]   # (muR, muF) multipliers


@pytest.fixture(scope="module")
def sample():
    import cupythia_b200 as cp
    it = cp.Integrator()
    it.integrate(8, 1 << 22, alpha=1.5)
    it.iteration(N, 70, alpha=0.0)
    it.weight_quantile(0.999)
    rec, w, st = it.unweight_scale_weights(N, iteration=71)
    yield it, cp.events_view(rec), w.cpu().numpy().astype(np.float64), st
    it.close()


def test_ratios_match_the_fp64_oracle(sample):
    it, ev, w, st = sample
    sub = slice(0, 3000)
    pts = ev["point"][sub].astype(np.int64)
    _, x = it.point_weights(0, N, 71, with_x=True)
    x = x.cpu().numpy()[pts].astype(np.float64)
    L = oracle.lib()
    base = oracle.had_cfg()
    cfgs = [oracle.had_cfg(kR=base.kR * fr ** 2, kF=base.kF * ff ** 2) for fr, ff in FACTORS]
    ref = np.zeros((len(pts), 6))
    for i in range(len(pts)):
        xi = np.ascontiguousarray(x[i])
        w0 = L.cpo_had_weight_x(C.byref(base), oracle.dptr(xi), None)
        for j, c in enumerate(cfgs):
            ref[i, j] = L.cpo_had_weight_x(C.byref(c), oracle.dptr(xi), None) / w0
    got = w[sub]
    assert np.all(np.isfinite(got))
    assert np.max(np.abs(got / ref - 1)) < 5e-5, np.max(np.abs(got / ref - 1))
    # mu_R up lowers alpha_s, mu_R down raises it
    assert np.all(got[:, 0] < 1) and np.all(got[:, 1] > 1)


def test_reweighted_sample_matches_direct_integration(sample):
    import cupythia_b200 as cp
    it, ev, w, st = sample
    grid = it.grid
    ew = ev["weight"].astype(np.float64)
    for j, (fr, ff) in enumerate(FACTORS):
        contrib = ew * w[:, j] * st["w_max"] / N
        sig_rw = contrib.sum()
        err_rw = np.sqrt((contrib ** 2).sum())
        with cp.Integrator(k_ren=fr ** 2, k_fac=ff ** 2) as jt:
            jt.grid = grid
            r = jt.iteration(1 << 24, 72, alpha=0.0)
        pull = (sig_rw - r["sigma"]) / np.hypot(err_rw, r["sigma_err"])
        assert abs(pull) < 5, ((fr, ff), sig_rw, r["sigma"], pull)


def test_weights_off_by_default(sample):
    it, _, _, _ = sample
    rec, st = it.unweight(1 << 20, iteration=73)   # no buffer set: plain production pass
    assert st["n_accepted"] > 0
