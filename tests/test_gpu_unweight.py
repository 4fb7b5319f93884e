"""Unweighting and on-device compaction into 64-byte records (the production pass)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 1 << 22


@pytest.fixture(scope="module")
def adapted():
    import cupythia_b200 as cp
    it = cp.Integrator()
    it.integrate(6, 1 << 22, alpha=1.5)
    yield it
    it.close()


def test_quantile_threshold(adapted):
    it = adapted
    it.iteration(N, 40, alpha=0.0)
    wq = it.weight_quantile(0.999)
    w = np.sort(it.point_weights(0, N, 40).cpu().numpy())
    exact = w[int(0.999 * N)]
    assert exact <= wq <= exact * 1.045
    frac_above = (w > wq).mean()
    assert 0.0 < frac_above <= 1e-3


def test_records_physics_and_accounting(adapted):
    import cupythia_b200 as cp
    it = adapted
    it.iteration(N, 41, alpha=0.0)
    wq = it.weight_quantile(0.999)
    rec, st = it.unweight(N, iteration=42)
    ev = cp.events_view(rec)
    assert st["n_bad"] == 0 and len(ev) == st["n_accepted"] > 0
    # acceptance: the accepted set is exactly {p : u(p) w_max < w(p)} on the same FP32 weights
    w = it.point_weights(0, N, 42).cpu().numpy()
    words = it.philox_words(it.cfg.seed, 0, N, 42, 0)
    u = (words[:, 3] >> 8).astype(np.float32) * np.float32(1.0 / 16777216.0)
    expect = np.nonzero(u * np.float32(wq) < w)[0]
    got = ev["point"].astype(np.int64)
    # point order, as the reference's library compaction (DeviceSelect::Flagged) leaves it
    assert np.all(np.diff(got) > 0)
    assert len(np.setxor1d(expect, got)) <= max(2, len(expect) // 100000)
    # weights: 1, or w / w_max for overweight events
    over = w[got] > wq
    assert np.allclose(ev["weight"][over], (w[got][over] / np.float32(wq)), rtol=1e-6)
    assert np.all(ev["weight"][~over] == 1.0)
    assert st["n_overweight"] == int(over.sum())
    # sigma from the unweighted sample agrees with the weighted estimate
    assert abs(st["sigma_unweighted"] - st["sigma"]) < 5 * st["sigma_err"] + 3e-3 * st["sigma"]
    # four-momentum conservation and masslessness
    e_in = np.abs(ev["pz_in"]).sum(1)
    pz_in = ev["pz_in"].sum(1)
    p3, p4 = ev["p3"].astype(np.float64), ev["p4"].astype(np.float64)
    assert np.allclose(p3[:, 0] + p4[:, 0], 0, atol=1e-3 * e_in.max())
    assert np.allclose(p3[:, 3] + p4[:, 3], e_in, rtol=1e-5)
    assert np.allclose(p3[:, 2] + p4[:, 2], pz_in, atol=2e-5 * e_in.max())
    m3 = p3[:, 3] ** 2 - (p3[:, :3] ** 2).sum(1)
    assert np.all(np.abs(m3) < 1e-4 * p3[:, 3] ** 2)
    pt = np.hypot(p3[:, 0], p3[:, 1])
    assert np.all(pt >= 20.0 * (1 - 1e-4)) and np.allclose(pt, ev["pt_hat"], rtol=1e-4)
    # flavours consistent with the process
    ids = ev["id"].astype(int)
    code = ev["process"]
    assert set(np.unique(code)) <= {111, 112, 113, 114, 115}
    g = ids == 21
    assert np.all(g[code == 111].all(1)) and np.all(g[code == 115][:, 2:].all(1))
    assert np.all(g[code == 112][:, :2].all(1))
    assert np.all(ids[code == 112][:, 2] == -ids[code == 112][:, 3])
    assert np.all((np.abs(ids[code == 112][:, 2]) >= 1) & (np.abs(ids[code == 112][:, 2]) <= 3))
    qg = code == 113
    assert np.all(g[qg][:, :2].sum(1) == 1) and np.all(ids[qg][:, :2] == ids[qg][:, 2:])
    qq = code == 114
    assert np.all(~g[qq].any(1)) and np.all(ids[qq][:, :2] == ids[qq][:, 2:])
    qb = code == 115
    assert np.all(ids[qb][:, 0] == -ids[qb][:, 1])


def test_process_fractions_match_per_process_cross_sections():
    import cupythia_b200 as cp
    sig = {}
    for k, bit in enumerate([1, 2, 4, 8, 16]):
        with cp.Integrator(proc_mask=bit) as it:
            _, c = it.integrate(6, 1 << 21, alpha=1.5, skip=2)
            sig[111 + k] = c["sigma"]
    with cp.Integrator() as it:
        it.integrate(6, 1 << 22, alpha=1.5)
        it.iteration(N, 50, alpha=0.0)
        it.weight_quantile(0.999)
        rec, st = it.unweight(N, iteration=51)
        ev = cp.events_view(rec)
    tot = sum(sig.values())
    for code, s in sig.items():
        f = (ev["weight"] * (ev["process"] == code)).sum() / ev["weight"].sum()
        err = np.sqrt(f * (1 - f) / len(ev)) + 1e-3
        assert abs(f - s / tot) < 5 * err, (code, f, s / tot)


def test_capacity_overflow_is_reported(adapted):
    import cupythia_b200 as cp
    it = adapted
    import torch
    small = torch.empty((100, 64), dtype=torch.uint8, device="cuda:0")
    with pytest.raises(cp.CpError) as e:
        it.unweight(N, iteration=43, records=small)
    assert e.value.code == 5


def test_host_generation_matches_device_pass(adapted):
    import torch

    import cupythia_b200 as cp
    it = adapted
    it.iteration(N, 44, alpha=0.0)
    it.weight_quantile(0.999)
    rec, st = it.unweight(N, iteration=45)
    dev = cp.events_view(rec)
    host = torch.empty((st["n_accepted"] + 16, 64), dtype=torch.uint8, pin_memory=True)
    st2 = it.generate_host(N, host, iteration=45, chunk=1 << 20)
    assert st2["n_accepted"] == st["n_accepted"]
    h = cp.events_view(host[:st2["n_accepted"]])
    a, b = dev, h   # both in point order: byte-identical without sorting
    assert a.tobytes() == b.tobytes()
