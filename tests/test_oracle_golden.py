"""The CPU oracle against the reference's own code (fixtures made by tests/golden/make_golden.py
from stock Pythia 8.317 and cuPythia's rng.cuh / physics.cuh) and against published vectors."""
import ctypes as C

import numpy as np
import pytest


def test_philox_known_answers(orc):
    # known-answer vectors of philox4x32_10 distributed with Random123 (Salmon et al., SC'11)
    kat = [([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
           ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
           ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
            [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1])]
    out = (C.c_uint32 * 4)()
    for ctr, key, want in kat:
        orc.lib().cpo_philox4x32_10((C.c_uint32 * 4)(*ctr), (C.c_uint32 * 2)(*key), out)
        assert list(out) == want


def test_splitmix_and_u01_match_reference(orc, golden):
    g = golden("cupythia_ref.json")
    L = orc.lib()
    for x, want, u in g["splitmix"]:
        assert L.cpo_splitmix64(x) == want
        assert L.cpo_u01(want) == u


def test_gg2gg_matches_reference_header(orc, golden):
    L = orc.lib()
    for s, t, u, a, want in golden("cupythia_ref.json")["gg2gg"]:
        assert L.cpo_gg2gg_recip(s, t, u, a) == want
        assert abs(L.cpo_sigma_gg2gg(s, t, u, a) / want - 1) < 1e-14


def test_fused_stage_sums_match_reference(orc, golden):
    """SplitMix64 per-thread streams (fused_gg2gg.cu:43-46) summed like the reference CPU loop."""
    L = orc.lib()
    for f in golden("cupythia_ref.json")["fused_sums"]:
        sums = (C.c_double * 2)()
        conv = 1.0
        s = f["s"]
        L.cpo_partonic_splitmix(np.sqrt(s), f["alphas"], f["cmax"], conv, f["seed"], f["n_threads"],
                                f["k_per"], sums, 1)
        scale = 2 * f["cmax"] * s / 2
        assert abs(sums[0] / scale / f["sum"] - 1) < 1e-13


def test_pdf_matches_pythia(orc, golden):
    g = golden("pythia_pdf.json")
    L = orc.lib()
    for row in g["rows"]:
        x, q2, vals = row[0], row[1], row[2:]
        for pid, want in zip(g["ids"], vals):
            got = L.cpo_pdf_xf(pid, x, q2)
            assert got == pytest.approx(want, rel=1e-14, abs=1e-300)


def test_alphas_matches_pythia(orc, golden):
    L = orc.lib()

    class A(C.Structure):
        _fields_ = [("a", C.c_double * 10), ("nf", C.c_int)]
    L.cpo_alphas_init.argtypes = [C.c_void_p, C.c_double]
    L.cpo_alphas_eval.argtypes = [C.c_void_p, C.c_double]
    L.cpo_alphas_eval.restype = C.c_double
    for a, rows in golden("pythia_alphas.json").items():
        st = A()
        L.cpo_alphas_init(C.byref(st), float(a))
        for q2, want in rows:
            assert L.cpo_alphas_eval(C.byref(st), q2) == pytest.approx(want, rel=1e-14)


@pytest.mark.parametrize("k,bit", list(enumerate([1, 2, 4, 8, 16])))
def test_sigma_pdf_matches_pythia(orc, golden, k, bit):
    g = golden("pythia_sigma.json")
    cfg = orc.had_cfg()
    out = (C.c_double * 6)()
    for r in g["rows"]:
        orc.lib().cpo_had_sigma_pdf(C.byref(cfg), r[0], r[1], r[2], r[3], bit, out)
        assert out[0] == pytest.approx(r[4 + k], rel=1e-13, abs=1e-300)
        assert out[1] == pytest.approx(r[9], rel=1e-14)
        assert out[2] == pytest.approx(r[10], rel=1e-14)


def test_simpson_and_partonic_mc(orc):
    L = orc.lib()
    simp = L.cpo_simpson_gg2gg(100000, 100.0, 0.13, 0.9, 0.3893793721)
    assert simp == pytest.approx(1.606699e-4, rel=1e-6)
    sums = (C.c_double * 2)()
    n = 1 << 18
    L.cpo_partonic_philox(100.0, 0.13, 0.9, 0.3893793721, 42, 0, n, sums, 4)
    m = sums[0] / n
    err = np.sqrt((sums[1] / n - m * m) / (n - 1))
    assert abs(m - simp) < 4 * err


def test_gg2gg_closed_form_matches_the_bracket_form(orc):
    """The partonic kernel evaluates gg -> gg as (9/2)(3 - tu/s^2 - su/t^2 - st/u^2) with one
    reciprocal of t u; with u = -s - t rounded as the reference rounds it, that form agrees with
    the oracle's bracket form (Sigma2gg2gg::sigmaKin, the reference's gg2gg_sigma) to 2e-15 over
    |cos theta| < 0.9, at the ends of the range included."""
    L = orc.lib()
    s, aS, cmax, conv = 1e4, 0.118, 0.9, 0.3893793721
    u01 = np.concatenate([np.random.default_rng(5).random(20000), [0.0, 1e-12, 0.5, 1.0 - 2 ** -53]])
    is_ = 1.0 / s
    pre = np.pi * is_ * is_ * (aS * aS) * 0.5 * 4.5
    c = (2.0 * u01 - 1.0) * cmax
    t = -0.5 * s * (1.0 - c)
    u = -s - t
    tu = t * u
    itu = 1.0 / tu
    it, iu = u * itu, t * itu
    closed = pre * (3.0 - tu * (is_ * is_) - (s * u) * (it * it) - (s * t) * (iu * iu))
    closed *= (2.0 * cmax) * (s / 2.0) * conv
    ref = np.array([L.cpo_partonic_weight(100.0, aS, cmax, conv, float(v)) for v in u01])
    assert np.max(np.abs(closed / ref - 1)) < 2e-15


def test_oracle_vegas_matches_pythia_sigma_gen(orc, golden):
    """FP64 oracle VEGAS (3 x 50 bins) against stock Pythia's sigmaGen for the dijet config."""
    L = orc.lib()
    cfg = orc.had_cfg()
    nb = 50
    e = orc.vegas_uniform(nb)
    est = []
    for it in range(6):
        sums = np.zeros(2)
        hist = np.zeros(3 * nb)
        n = 100000
        L.cpo_had_accumulate(C.byref(cfg), orc.dptr(e), nb, 42, it, 0, n, orc.dptr(sums), orc.dptr(hist), 8)
        m = sums[0] / n
        est.append((m, np.sqrt((sums[1] / n - m * m) / (n - 1))))
        L.cpo_vegas_refine(orc.dptr(e), orc.dptr(hist), 3, nb, 1.5)
    w = np.array([1 / s ** 2 for _, s in est[2:]])
    sig = sum(m / s ** 2 for m, s in est[2:]) / w.sum()
    err = 1 / np.sqrt(w.sum())
    g = golden("pythia_sigma_gen.json")
    pull = (sig - g["sigma_mb"]) / np.hypot(err, g["sigma_err_mb"])
    assert abs(pull) < 4, (sig, err, g["sigma_mb"])


def test_complex_step_gradient_matches_finite_differences(orc):
    L = orc.lib()
    cfg = orc.had_cfg()
    rng = np.random.default_rng(3)
    for _ in range(20):
        x = rng.uniform(0.05, 0.95, 3)
        g = (C.c_double * 7)()
        L.cpo_had_weight_grad(C.byref(cfg), orc.dptr(x), g)
        for d in range(3):
            h = 1e-6
            xp, xm = x.copy(), x.copy()
            xp[d] += h
            xm[d] -= h
            fd = (L.cpo_had_weight_x(C.byref(cfg), orc.dptr(xp), None) -
                  L.cpo_had_weight_x(C.byref(cfg), orc.dptr(xm), None)) / (2 * h)
            assert g[1 + d] == pytest.approx(fd, rel=1e-5, abs=1e-9 * abs(g[0]))
        for k, (name, h) in enumerate([("aSmZ", 1e-7), ("kR", 1e-6), ("pTmin", 1e-5)]):
            cp_, cm_ = orc.had_cfg(), orc.had_cfg()
            setattr(cp_, name, getattr(cfg, name) + h)
            setattr(cm_, name, getattr(cfg, name) - h)
            fd = (L.cpo_had_weight_x(C.byref(cp_), orc.dptr(x), None) -
                  L.cpo_had_weight_x(C.byref(cm_), orc.dptr(x), None)) / (2 * h)
            assert g[4 + k] == pytest.approx(fd, rel=1e-5, abs=1e-9 * abs(g[0]))


def test_flow_oracle_backprop_matches_finite_differences(orc):
    """The FP64 reference backprop of the flow against central differences of its forward."""
    L = orc.lib()
    L.cpo_flow_set_rounding(0)
    try:
        rng = np.random.default_rng(4)
        npar = 4 * 5768
        P = (rng.normal(0, 0.2, npar)).astype(np.float32)
        n = 6
        u = rng.uniform(0.05, 0.95, (n, 3))
        cv = rng.normal(0, 1, (n, 3))
        cJ = rng.normal(0, 1, n)
        G = np.zeros(npar)
        L.cpo_flow_backward_batch(P.ctypes.data, n, u.ctypes.data, cv.ctypes.data, cJ.ctypes.data, G.ctypes.data, 2)

        def objective(Pp):
            tot = 0.0
            for i in range(n):
                v = np.zeros(3)
                lj = C.c_double()
                L.cpo_flow_forward(Pp.ctypes.data, orc.dptr(u[i].copy()), orc.dptr(v), C.byref(lj))
                tot += float(cv[i] @ v) + cJ[i] * lj.value
            return tot
        # parameters that the architecture uses: W1 row 0, b1, W2, b2, W3 cols < 2 nt, b3
        idx = [0 * 5768 + 5, 0 * 5768 + 1024 + 7, 1 * 5768 + 1088 + 300, 2 * 5768 + 5184 + 9,
               3 * 5768 + 5248 + 8 * 10 + 1, 0 * 5768 + 5760 + 3, 1 * 5768 + 64 + 2, 2 * 5768 + 1088 + 4000]
        for k in idx:
            h = 1e-4
            Pp, Pm = P.astype(np.float64).copy(), P.astype(np.float64).copy()
            Pp[k] += h
            Pm[k] -= h
            fd = (objective(Pp.astype(np.float32)) - objective(Pm.astype(np.float32))) / (
                float(np.float32(Pp[k])) - float(np.float32(Pm[k])))
            assert G[k] == pytest.approx(fd, rel=2e-3, abs=1e-6), (k, G[k], fd)
    finally:
        L.cpo_flow_set_rounding(1)
