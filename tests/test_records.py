"""Record consumers on the CPU: colour tags of the encoded colour flows (cp_colour_tags) and the
Les Houches Event File writer (cp_write_lhef), read back by stock Pythia 8.317
(Beams:frameType = 4, showered and hadronized, which needs a valid colour flow) -- the
reference's own LHE validation (cuPythia/pipeline/lhe_validate.cc)."""
import ctypes as C
import json
import os
import subprocess

import numpy as np
import pytest

import oracle


def _valid_flow(ids, col, acol):
    """Colour conservation of a 2 -> 2 record and colour-charge rules of each parton."""
    inflow = [col[0], col[1], acol[2], acol[3]]
    outflow = [acol[0], acol[1], col[2], col[3]]
    if sorted(t for t in inflow if t) != sorted(t for t in outflow if t):
        return False
    for i, c, a in zip(ids, col, acol):
        if i == 21 and not (c and a and c != a):
            return False
        if 1 <= i <= 6 and not (c and not a):
            return False
        if -6 <= i <= -1 and not (a and not c):
            return False
    return True


def _oracle_records(n, seed=1):
    """n records (EVENT_DTYPE) from oracle picks at random points, kinematics from the base map."""
    import cupythia_b200 as cp
    cfg = oracle.had_cfg()
    rng = np.random.default_rng(seed)
    ev = np.zeros(n, cp.EVENT_DTYPE)
    s = cfg.sqrtS ** 2
    eb = 0.5 * cfg.sqrtS
    k = 0
    while k < n:
        x = rng.random(3)
        tyz = np.zeros(3)
        if not oracle.lib().cpo_had_weight_x(C.byref(cfg), oracle.dptr(x), oracle.dptr(tyz)) > 0:
            continue
        code, ids, colour = oracle.pick_record(cfg, x, *rng.random(5))
        tau, y, z = tyz
        sH = tau * s
        pst, st, phi = 0.5 * np.sqrt(sH), np.sqrt(1 - z * z), 2 * np.pi * rng.random()
        ch, sh = np.cosh(y), np.sinh(y)
        p3 = [pst * st * np.cos(phi), pst * st * np.sin(phi), pst * (z * ch + sh), pst * (ch + z * sh)]
        p4 = [-p3[0], -p3[1], pst * (sh - z * ch), pst * (ch - z * sh)]
        ev[k] = (ids, [eb * np.sqrt(tau) * np.exp(y), -eb * np.sqrt(tau) * np.exp(-y)], p3, p4, 1.0, pst * st,
                 code, colour, k)
        k += 1
    return ev


def test_colour_tags_of_every_flow_are_valid():
    import cupythia_b200 as cp
    ev = _oracle_records(3000, seed=2)
    col, acol = cp.colour_tags(ev)
    for e, c, a in zip(ev, col, acol):
        assert _valid_flow(e["id"].tolist(), c.tolist(), a.tolist()), (e["process"], e["id"], e["colour"], c, a)
    # every topology of every process occurs
    seen = {(int(p), int(c) & 3) for p, c in zip(ev["process"], ev["colour"])}
    assert {(111, 0), (111, 1), (111, 2), (113, 0), (113, 1), (114, 0), (114, 1)} <= seen


def test_invalid_colour_codes_are_rejected():
    import cupythia_b200 as cp
    lib = cp._lib.load()
    a, b = (C.c_int * 4)(), (C.c_int * 4)()
    assert lib.cp_colour_tags(110, 0, a, b) == 1
    assert lib.cp_colour_tags(113, 2, a, b) == 1
    assert lib.cp_colour_tags(111, 3, a, b) == 1
    assert lib.cp_colour_tags(111, 2, a, b) == 0


@pytest.mark.skipif(not os.path.exists(oracle.PYTHIA_REF), reason="oracle/_ref not built")
def test_lhef_reads_back_in_pythia(tmp_path):
    import cupythia_b200 as cp
    n = 300
    ev = _oracle_records(n, seed=3)
    path = tmp_path / "events.lhe"
    cp.write_lhef(path, ev, 0.7674, 0.0009)
    text = path.read_text()
    assert text.count("<event>") == n and text.startswith('<LesHouchesEvents version="3.0">')
    r = subprocess.run([oracle.PYTHIA_REF, "lhef", str(path), "1"], capture_output=True, text=True, timeout=300)
    out = json.loads(r.stdout.strip().split("\n")[-1])
    assert out["init"] and out["read"] == n and out["aborted"] == 0, out
    assert out["max_imbalance_gev"] < 1e-2, out
    assert out["by_code"] == [int((ev["process"] == c).sum()) for c in range(111, 116)]
    assert abs(out["sigma_gen_mb"] / 0.7674 - 1) < 1e-6
    assert abs(out["e_cm"] - 13000.0) < 1e-6
