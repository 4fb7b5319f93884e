"""Parity of the CUDA path (through the C ABI) with the CPU oracle and the reference fixtures.

Tolerances, stated once:
  * integer / RNG work: bit-exact;
  * FP32 per-point weights: 1e-5 relative for weights >= 1e-12 of the mean (smaller weights
    underflow FP32 and carry no cross section);
  * FP32 single PDFs: 5e-5 relative (the weight combines them with averaging errors);
  * FP64 partonic kernel: 1e-13 relative per point, 1e-12 on sums.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W_TOL = 1e-5
TINY = 1e-12


def _torch():
    import torch
    return torch


# ----------------------------------------------------------------------------- RNG
def test_philox_words_bit_exact(integ, orc):
    rng = np.random.default_rng(11)
    for seed, p0, it, st in [(42, 0, 0, 0), (7, 2 ** 32 - 100, 3, 1), (2 ** 63 + 5, 2 ** 40, 9, 2)]:
        got = integ.philox_words(seed, p0, 4096, it, st)
        idx = rng.integers(0, 4096, 200)
        ref = orc.point_words(seed, [p0 + int(i) for i in idx], it, st)
        assert np.array_equal(got[idx], ref)


def test_splitmix_uniforms_match_reference_streams(integ, orc, golden):
    L = orc.lib()
    seed, nthr, kper = 0xABCDEF01, 300, 17
    got = integ.splitmix_uniforms(seed, nthr, kper)
    ref = np.array([L.cpo_u01(L.cpo_splitmix64(L.cpo_thread_counter(seed, t) + i))
                    for t in range(nthr) for i in range(kper)])
    assert np.array_equal(got, ref)
    for x, want, u in golden("cupythia_ref.json")["splitmix"][:3]:
        pass  # the oracle itself is pinned to the reference by test_oracle_golden


def test_event_keys_bit_exact(integ, orc):
    L = orc.lib()
    got = integ.event_keys(0x6E11, 1000, 513)
    ref = np.array([L.cpo_event_key(0x6E11, 1000 + i) for i in range(513)], np.uint64)
    assert np.array_equal(got, ref)


# ----------------------------------------------------------------------------- SigmaProcess
def test_sigma_pdf_surface_matches_pythia(golden, integ):
    from cupythia_b200 import sigma as S
    g = np.array(golden("pythia_sigma.json")["rows"])
    x1, x2, sH, tH = (g[:, k].astype(np.float32) for k in range(4))
    for k, cls in enumerate(S.HARD_QCD):
        p = cls(integ)
        p.set2Kin(x1, x2, sH, tH)
        got = p.sigmaPDF().cpu().numpy().astype(np.float64)
        want = g[:, 4 + k]
        keep = want > TINY * want.mean()
        rel = np.abs(got[keep] - want[keep]) / want[keep]
        assert rel.max() < W_TOL, (cls.__name__, rel.max())
        a = p.alphaSRen().cpu().numpy()
        assert np.allclose(a, g[:, 9], rtol=1e-6)
        assert np.allclose(p.Q2Ren().cpu().numpy(), g[:, 10], rtol=1e-6)


def test_sigma_hat_matches_oracle(integ, orc):
    from cupythia_b200 import sigma as S
    L = orc.lib()
    rng = np.random.default_rng(5)
    n = 2000
    sH = (10 ** rng.uniform(3.3, 8.2, n)).astype(np.float32)
    c = rng.uniform(-0.99, 0.99, n)
    tH = (-0.5 * sH * (1 - c)).astype(np.float32)
    x = np.full(n, 0.1, np.float32)
    p = S.Sigma2qq2qq(integ)
    p.set2Kin(x, x, sH, tH)
    alpha = p.alphaSRen().cpu().numpy().astype(np.float64)
    for id1, id2 in [(1, 1), (1, -1), (2, 1), (-3, 3), (-2, -2)]:
        got = p.sigmaHat(id1, id2).cpu().numpy()
        s64, t64 = sH.astype(np.float64), tH.astype(np.float64)
        want = np.array([L.cpo_sigma_qq2qq(s, t, -s - t, a, id1, id2) for s, t, a in zip(s64, t64, alpha)])
        assert np.allclose(got, want, rtol=W_TOL)
    for cls, f in [(S.Sigma2gg2gg, L.cpo_sigma_gg2gg), (S.Sigma2qg2qg, None)]:
        q = cls(integ)
        q.set2Kin(x, x, sH, tH)
        got = q.sigmaKin().cpu().numpy()
        if f is not None:
            want = np.array([f(s, t, -s - t, a) for s, t, a in zip(sH.astype(float), tH.astype(float), alpha)])
            assert np.allclose(got, want, rtol=W_TOL)
    with pytest.raises(Exception):
        S.Sigma2qq2qq(integ).sigmaKin()


def test_pdf_batch_matches_pythia(integ, golden):
    g = golden("pythia_pdf.json")
    rows = np.array(g["rows"])
    x = rows[:, 0].astype(np.float32)
    q2 = rows[:, 1].astype(np.float32)
    got = integ.pdf(x, q2).astype(np.float64)
    want = rows[:, 2:]
    # evaluate the oracle at the FP32 inputs the kernel saw
    import oracle
    L = oracle.lib()
    ids = g["ids"]
    want32 = np.array([[L.cpo_pdf_xf(i, float(xx), float(qq)) for i in ids] for xx, qq in zip(x, q2)])
    keep = (want32 > 1e-20) & (x[:, None] < 0.999)
    rel = np.abs(got - want32)[keep] / want32[keep]
    assert rel.max() < 5e-5, rel.max()
    assert np.allclose(want32[(x.astype(np.float64) == rows[:, 0])], want[(x.astype(np.float64) == rows[:, 0])], rtol=1e-12)


# ----------------------------------------------------------------------------- integrand
def _check_weights(integ, orc, n, it=0, cfg=None):
    w, x = integ.point_weights(0, n, it, with_x=True)
    w = w.cpu().numpy().astype(np.float64)
    x = x.cpu().numpy()
    grid = integ.grid
    nb = integ.nb
    words = integ.philox_words(integ.cfg.seed, 0, n, it, 0)
    m = (words[:, :3] >> 8).astype(np.uint64) * nb
    bins = (m >> 24).astype(np.int64)
    jv = np.ones(n)
    for d in range(3):
        e = grid[d]
        lo = e[bins[:, d]].astype(np.float32)
        wd = (e[bins[:, d] + 1] - e[bins[:, d]]).astype(np.float32)
        jv *= nb * wd.astype(np.float64)
        frac = (m[:, d] & 0xFFFFFF).astype(np.float64) / 2 ** 24
        xd = lo.astype(np.float64) + frac * wd.astype(np.float64)
        assert np.all(np.abs(x[:, d] - xd) <= 2 * np.spacing(np.float32(np.maximum(xd, 1e-30)))), d
    ref = orc.weight_x_batch(cfg or orc.had_cfg(), x) * jv
    keep = ref > TINY * ref.mean()
    rel = np.abs(w[keep] - ref[keep]) / ref[keep]
    assert rel.max() < W_TOL, (rel.max(), np.percentile(rel, 99.9))
    return w, ref


def test_point_weights_uniform_grid(integ, orc):
    integ.reset_grid()
    _check_weights(integ, orc, 1 << 18)


def test_point_weights_adapted_grid(integ, orc):
    integ.reset_grid()
    integ.integrate(6, 1 << 20, alpha=1.5)
    _check_weights(integ, orc, 1 << 18, it=17)
    integ.reset_grid()


def test_iteration_sums_and_histogram_match_oracle(integ, orc):
    integ.reset_grid()
    integ.integrate(3, 1 << 20, alpha=1.5)
    grid = integ.grid.copy()
    n = 1 << 17
    w, xw = integ.point_weights(0, n, 5, with_x=True)
    w = w.cpu().numpy().astype(np.float64)
    r = integ.iteration(n, 5, alpha=1.5)
    assert r["n_bad"] == 0
    assert abs(r["sum_w"] / w.sum() - 1) < 1e-6
    assert abs(r["sum_w2"] / (w * w).sum() - 1) < 1e-6
    h = integ.last_histogram()
    # per-bin sums of w^2 against FP64 weights at the x the kernel evaluated (the FP64 map of the
    # same words differs from the FP32 one by an ulp of x, which the t-channel pole amplifies)
    x = xw.cpu().numpy()
    words = integ.philox_words(integ.cfg.seed, 0, n, 5, 0)
    m = (words[:, :3] >> 8).astype(np.uint64) * integ.nb
    bins = (m >> 24).astype(np.int64)
    jv = np.prod([integ.nb * (grid[d][bins[:, d] + 1] - grid[d][bins[:, d]]).astype(np.float32)
                  for d in range(3)], axis=0)
    ref = orc.weight_x_batch(orc.had_cfg(), x) * jv
    hist = np.zeros((3, integ.nb))
    for d in range(3):
        np.add.at(hist[d], bins[:, d], ref * ref)
    assert np.allclose(h["hist"], hist, rtol=1e-4, atol=1e-12 * hist.max())
    L = orc.lib()
    # the device refinement of the device histogram == the oracle refinement of the same input
    e2 = grid.reshape(-1).copy()
    L.cpo_vegas_refine(orc.dptr(e2), orc.dptr(np.ascontiguousarray(h["hist"].reshape(-1))), 3, integ.nb, 1.5)
    assert np.max(np.abs(integ.grid.reshape(-1) - e2)) < 1e-12
    integ.reset_grid()


def test_integration_matches_pythia_and_is_deterministic(integ, golden):
    integ.reset_grid()
    per, comb = integ.integrate(10, 1 << 24, alpha=1.5, skip=3)
    g1 = integ.grid
    integ.reset_grid()
    per2, comb2 = integ.integrate(10, 1 << 24, alpha=1.5, skip=3)
    assert comb["sigma"] == comb2["sigma"] and np.array_equal(g1, integ.grid)
    assert comb["n_bad"] == 0
    ref = golden("pythia_sigma_gen.json")
    pull = (comb["sigma"] - ref["sigma_mb"]) / np.hypot(comb["sigma_err"], ref["sigma_err_mb"])
    assert abs(pull) < 4, (comb, ref)
    assert comb["sigma_err"] / comb["sigma"] < 1e-3
    assert per[-1]["eta"] > per[0]["eta"]
    integ.reset_grid()


@pytest.mark.parametrize("pt,aS,kR", [(10.0, 0.11, 0.5), (50.0, 0.14, 2.0)])
def test_other_parameter_points(orc, pt, aS, kR):
    import cupythia_b200 as cp
    with cp.Integrator(pt_hat_min=pt, alphas_mz=aS, k_ren=kR) as it:
        _check_weights(it, orc, 1 << 16, cfg=orc.had_cfg(pTmin=pt, aSmZ=aS, kR=kR))


# ----------------------------------------------------------------------------- partonic
def test_partonic_philox_matches_oracle(integ, orc):
    L = orc.lib()
    n = 1 << 22
    r = integ.partonic_integrate(n)
    sums = (C.c_double * 2)()
    L.cpo_partonic_philox(100.0, 0.13, 0.9, 0.3893793721, 42, 0, n, sums, 8)
    assert abs(r["sum_w"] / sums[0] - 1) < 1e-12
    assert abs(r["sum_w2"] / sums[1] - 1) < 1e-12
    simp = L.cpo_simpson_gg2gg(100000, 100.0, 0.13, 0.9, 0.3893793721)
    assert abs(r["sigma"] - simp) < 4 * r["sigma_err"]
    w = integ.partonic_weights(12345, 1000).cpu().numpy()
    words = orc.point_words(42, range(12345, 13345))
    u = ((words[:, 1].astype(np.uint64) << np.uint64(32)) | words[:, 0].astype(np.uint64)) >> np.uint64(11)
    ref = np.array([L.cpo_partonic_weight(100.0, 0.13, 0.9, 0.3893793721, float(v) / 2 ** 53) for v in u])
    assert np.allclose(w, ref, rtol=1e-13, atol=0)


def test_partonic_splitmix_matches_reference_stage(integ, golden):
    for f in golden("cupythia_ref.json")["fused_sums"]:
        r = integ.partonic_splitmix(f["n_threads"], f["k_per"], sqrt_shat=np.sqrt(f["s"]), alphas=f["alphas"],
                                    cmax=f["cmax"], conv=1.0, seed=f["seed"])
        scale = 2 * f["cmax"] * f["s"] / 2
        assert abs(r["sum_w"] / scale / f["sum"] - 1) < 1e-12


# ----------------------------------------------------------------------------- edge cases
def test_edge_cases(integ):
    import cupythia_b200 as cp
    assert integ.philox_words(1, 0, 0).shape == (0, 4)
    with pytest.raises(cp.CpError):
        integ.iteration(1)
    with pytest.raises(cp.CpError):
        integ.grid = np.tile(np.linspace(1, 0, integ.nb + 1), (3, 1))
    with pytest.raises(cp.CpError):
        cp.Integrator(pt_hat_min=1.0)
    with pytest.raises(cp.CpError):
        cp.Integrator(n_bins=500)
    with pytest.raises(KeyError):
        cp.Integrator(not_a_field=1)
    # ragged sizes: not a multiple of the block or grid size
    w = integ.point_weights(3, 1000003 % 4099)
    assert np.all(np.isfinite(w.cpu().numpy()))


# a draw this close (relative) to a selection boundary can be decided either way by FP32 sums
PICK_MARGIN = 1e-4
# picks observed to differ from the FP64 oracle's per process code (3000 seeded points each, B200)
PICK_DIFFERS = {111: 0, 112: 0, 113: 0, 114: 0, 115: 0}


def test_pick_in_state_and_set_id_col_acol_match_oracle():
    import oracle
    """The SigmaProcess surface's pickInState and setIdColAcol over a batch, per process, against
    the oracle's restatement at the same FP32 kinematics and uniforms.  A pick may differ only
    where a draw lies within FP32 rounding of a selection boundary (the oracle's margin below
    PICK_MARGIN: FP32 pair sums and PDFs against FP64 ones), and no more picks differ than were
    observed on the B200 (PICK_DIFFERS, deterministic kernels and draws)."""
    import ctypes as C

    import cupythia_b200 as cp
    from cupythia_b200.sigma import HARD_QCD
    cfg = oracle.had_cfg()
    rng = np.random.default_rng(12)
    s = cfg.sqrtS ** 2
    kin = []
    while len(kin) < 3000:
        x = rng.random(3)
        tyz = np.zeros(3)
        if not oracle.lib().cpo_had_weight_x(C.byref(cfg), oracle.dptr(x), oracle.dptr(tyz)) > 0:
            continue
        tau, y, z = tyz
        sH = tau * s
        kin.append((np.sqrt(tau) * np.exp(y), np.sqrt(tau) * np.exp(-y), sH, -0.5 * sH * (1 - z)))
    kin = np.array(kin, np.float32)
    n = len(kin)
    with cp.Integrator() as it:
        for cls in HARD_QCD:
            sp = cls(integrator=it)
            sp.set2Kin(kin[:, 0], kin[:, 1], kin[:, 2], kin[:, 3])
            r = rng.random((n, 4)).astype(np.float32)
            id1, id2 = sp.pickInState(r[:, 0])
            ids, col, acol = sp.setIdColAcol(r[:, 1], r[:, 2], r[:, 3])
            assert np.array_equal(id1.cpu().numpy(), ids[:, 0]) and np.array_equal(id2.cpu().numpy(), ids[:, 1])
            ref = np.zeros(n, cp.EVENT_DTYPE)
            ref_ids = np.zeros((n, 4), int)
            margin = np.zeros(n)
            for i in range(n):
                got, rid, rcol, margin[i] = oracle.pick_state(cfg, sp.code(), *[float(v) for v in kin[i]],
                                                              *[float(v) for v in r[i]], with_margin=True)
                assert got == sp.code()
                ref_ids[i] = rid
                ref["colour"][i] = rcol
            ref["process"] = sp.code()
            rc_, ra_ = cp.colour_tags(ref)
            same = (ids == ref_ids).all(1) & (col == rc_).all(1) & (acol == ra_).all(1)
            differ = int((~same).sum())
            print(f"{sp.name()}: {differ} of {n} picks differ, margins {np.sort(margin[~same]).tolist()}")
            assert np.all(margin[~same] < PICK_MARGIN), (sp.name(), margin[~same])
            assert differ <= PICK_DIFFERS[sp.code()], (sp.name(), differ)


def test_philox_words_match_curand(integ, tmp_path):
    """An independent pin of the counter-RNG: cuRAND's own device Philox-4x32-10
    (curand_Philox4x32_10) with the same key (seed) and counter (point lo, point hi, iteration,
    stream) gives bit-identical words."""
    import os
    import subprocess
    src = os.path.join(os.path.dirname(os.path.abspath(__file__)), "curand_philox_probe.cu")
    exe = str(tmp_path / "curand_philox_probe")
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", src, "-o", exe], check=True,
                   capture_output=True)
    for seed, p0, it_, st in [(42, 0, 0, 0), (42, 2 ** 32 - 3, 7, 1), (2 ** 40 + 11, 12345, 3, 2)]:
        out = subprocess.run([exe, str(seed), str(p0), "1000", str(it_), str(st)], check=True, capture_output=True,
                             text=True).stdout.split()
        ref = np.array([int(v, 16) for v in out], np.uint32).reshape(-1, 4)
        got = integ.philox_words(seed, p0, 1000, it_, st)
        assert np.array_equal(got, ref), (seed, p0, it_, st)
