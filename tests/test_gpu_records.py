"""Event records on the GPU against the oracle: the record builder's process, incoming pair,
new flavour and colour flow (pickInState + setIdColAcol restated in cpo_pick_record) at the
kernel's own points and random numbers, and the LHE file of device records read back by Pythia.
The kernel evaluates the pair sums in FP32 and the oracle in FP64, so a pick can differ when a
random number falls within rounding of a boundary: every differing record must have a draw within
RECORD_MARGIN (relative) of a selection boundary by the oracle's own sums, and no more records
may differ than were observed on the B200 (RECORD_DIFFERS; kernels and draws are deterministic)."""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

N = 1 << 20
RECORD_MARGIN = 1e-4
RECORD_DIFFERS = 0        # observed on the B200 for these 20,000 records


@pytest.fixture(scope="module")
def production():
    import cupythia_b200 as cp
    it = cp.Integrator()
    it.integrate(6, 1 << 21, alpha=1.5)
    it.iteration(N, 60, alpha=0.0)
    it.weight_quantile(0.999)
    rec, st = it.unweight(N, iteration=61)
    yield it, cp.events_view(rec), st
    it.close()


def _u24(w):
    return (w >> 8).astype(np.float32) * np.float32(1.0 / 16777216.0)


def test_record_picks_match_oracle(production):
    it, ev, st = production
    sub = ev[:20000]
    pts = sub["point"].astype(np.int64)
    _, x = it.point_weights(0, N, 61, with_x=True)
    x = x.cpu().numpy()[pts].astype(np.float64)
    w1 = it.philox_words(it.cfg.seed, 0, N, 61, 1)[pts]
    cfg = oracle.had_cfg()
    bad = 0
    bad_margins = []
    codes = np.zeros(len(sub), int)
    for i in range(len(sub)):
        w = [int(v) for v in w1[i]]
        rc = ((w[0] & 0xFF) | ((w[1] & 0xFF) << 8) | ((w[2] & 0xFF) << 16)) / 16777216.0
        rs = (w[3] & 0xFF) / 256.0
        r = [float(_u24(w1[i, 0])), float(_u24(w1[i, 1])), float(_u24(w1[i, 3])), rc, rs]
        code, ids, colour, margin = oracle.pick_record(cfg, x[i], *r, with_margin=True)
        codes[i] = code
        if (code, ids, colour) != (int(sub["process"][i]), sub["id"][i].tolist(), int(sub["colour"][i])):
            bad += 1
            bad_margins.append(margin)
    print(f"records: {bad} of {len(sub)} differ from the oracle's picks, margins {sorted(bad_margins)}")
    assert all(m < RECORD_MARGIN for m in bad_margins), bad_margins
    assert bad <= RECORD_DIFFERS, bad
    assert set(np.unique(codes)) == {111, 112, 113, 114, 115}


def test_device_colour_flows_are_valid(production):
    import cupythia_b200 as cp
    from test_records import _valid_flow
    _, ev, _ = production
    sub = ev[:50000]
    col, acol = cp.colour_tags(sub)
    ok = [_valid_flow(e.tolist(), c.tolist(), a.tolist()) for e, c, a in zip(sub["id"], col, acol)]
    assert all(ok)


@pytest.mark.skipif(not os.path.exists(oracle.PYTHIA_REF), reason="oracle/_ref not built")
def test_lhef_of_device_records_reads_back_in_pythia(production, tmp_path):
    import cupythia_b200 as cp
    it, ev, st = production
    n = 2000
    path = tmp_path / "gpu.lhe"
    cp.write_lhef(path, ev[:n], st["sigma"], st["sigma_err"], cfg=it.cfg)
    r = subprocess.run([oracle.PYTHIA_REF, "lhef", str(path), "1"], capture_output=True, text=True, timeout=600)
    out = json.loads(r.stdout.strip().split("\n")[-1])
    assert out["init"] and out["read"] == n and out["aborted"] == 0, out
    assert out["max_imbalance_gev"] < 0.05, out
    assert out["by_code"] == [int((ev[:n]["process"] == c).sum()) for c in range(111, 116)]
    assert abs(out["sigma_gen_mb"] / st["sigma"] - 1) < 1e-6


def _splitmix64(x):
    x = (x + np.uint64(0x9E3779B97F4A7C15))
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def test_device_event_hand_off():
    """Records (with the 7-point scale ratios) handed over to the reference pipeline's device
    event record: every member equals the host-side expansion of the same records bit for bit
    (incoming status -21 with mothers -1, outgoing 23 with mothers 0 and 1, colour tags 500 + the
    record's setIdColAcol tags, the event key, scale, x1, x2, flavours, weight vector); events
    outside [e0, e0 + n) stay untouched; bad shapes are refused."""
    import ctypes as C

    import torch

    import cupythia_b200 as cp
    n_pts = 1 << 20
    with cp.Integrator() as it:
        it.integrate(5, 1 << 20, alpha=1.5)
        it.iteration(n_pts, 80, alpha=0.0)
        it.weight_quantile(0.999)
        rec, ratios, st = it.unweight_scale_weights(n_pts, iteration=81)
        n = rec.shape[0]
        e0 = 3
        ev = it.to_device_events(rec, n_events=n + 5, n_var=7, scale_ratios=ratios.contiguous(), e0=e0)
        # refused: more than one weight without ratios, too few particle slots, too many events
        res = []
        for kw in ({"n_var": 2}, {"max_part": 3}, {"n_events": n - 1}):
            try:
                it.to_device_events(rec, **kw)
                res.append(0)
            except cp.CpError as err:
                res.append(1 if err.code == cp._lib.CP_ERR_INVALID else 2)
        cfg = it.cfg
        host = {k: (v.cpu().numpy() if hasattr(v, "cpu") else v) for k, v in ev.items()}
        r = cp.events_view(rec)
        rt = ratios.cpu().numpy()
    assert res == [1, 1, 1]
    mp = 4
    idx = (e0 + np.arange(n))[:, None] * mp + np.arange(4)[None, :]
    pz_in = r["pz_in"].astype(np.float64)
    px = np.zeros((n, 4)); py = np.zeros((n, 4)); pz = np.zeros((n, 4)); en = np.zeros((n, 4))
    pz[:, :2] = pz_in
    en[:, :2] = np.abs(pz_in)
    for k, key in ((2, "p3"), (3, "p4")):
        p = r[key].astype(np.float64)
        px[:, k], py[:, k], pz[:, k], en[:, k] = p[:, 0], p[:, 1], p[:, 2], p[:, 3]
    c, a = cp.colour_tags(r)
    col = np.where(c > 0, 500 + c, 0).astype(np.int32)
    acol = np.where(a > 0, 500 + a, 0).astype(np.int32)
    assert np.array_equal(host["px"][idx], px) and np.array_equal(host["py"][idx], py)
    assert np.array_equal(host["pz"][idx], pz) and np.array_equal(host["e"][idx], en)
    assert np.all(host["m"][idx] == 0)
    assert np.array_equal(host["pdg"][idx], r["id"].astype(np.int32))
    assert np.array_equal(host["status"][idx], np.tile([-21, -21, 23, 23], (n, 1)))
    assert np.array_equal(host["mo1"][idx], np.tile([-1, -1, 0, 0], (n, 1)))
    assert np.array_equal(host["mo2"][idx], np.tile([-1, -1, 1, 1], (n, 1)))
    assert np.all(host["d1"][idx] == -1) and np.all(host["d2"][idx] == -1)
    assert np.array_equal(host["col"][idx], col) and np.array_equal(host["acol"][idx], acol)
    e = e0 + np.arange(n)
    assert np.all(host["nPart"][e] == 4) and np.all(host["active"][e] == 1)
    key = _splitmix64(np.uint64(cfg.seed) ^ (r["point"].astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15)))
    assert np.array_equal(host["seed"][e].view(np.uint64), key)
    assert np.array_equal(host["scale"][e], np.sqrt(cfg.k_fac) * r["pt_hat"].astype(np.float64))
    assert np.array_equal(host["x1"][e], np.abs(pz_in[:, 0]) * (2.0 / cfg.sqrt_s))
    assert np.array_equal(host["x2"][e], np.abs(pz_in[:, 1]) * (2.0 / cfg.sqrt_s))
    assert np.array_equal(host["flavA"][e], r["id"][:, 0].astype(np.int32))
    assert np.array_equal(host["flavB"][e], r["id"][:, 1].astype(np.int32))
    w = host["weight"].reshape(-1, 7)[e]
    wt = r["weight"].astype(np.float64)
    assert np.array_equal(w[:, 0], wt)
    assert np.array_equal(w[:, 1:], wt[:, None] * rt.astype(np.float64))
    # events before e0 and after e0 + n are as allocated
    out = np.r_[0:e0, e0 + n:n + 5]
    assert np.all(host["nPart"][out] == 0) and np.all(host["weight"].reshape(-1, 7)[out] == 0)
