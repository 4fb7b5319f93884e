"""The host-side setIdColAcol of one event (cp_set_id_col_acol, the Pythia plug-in's
setIdColAcol) against Sigma2*::setIdColAcol as pythia8317/src/SigmaQCD.cc:135-342 writes it,
restated here in FP64 on the same incoming pairs, kinematics and draws.  No GPU needed.  A draw
within FP32 rounding of a topology boundary may be decided either way (the library evaluates the
topology terms in FP32); every other event must match exactly, and every flow must conserve
colour."""
import ctypes as C

import numpy as np

from test_records import _valid_flow

MARGIN = 1e-5


def _swap_ca(col, acol):
    return acol[:], col[:]


def _ref(code, id1, id2, tp, up, nqn, rf, rc, rs):
    """(ids, col, acol, margin) of the stock setIdColAcol; tp = tHat/sHat, up = uHat/sHat."""
    margin = 1.0
    if code == 111:
        ids = [id1, id2, 21, 21]
        a = (9 / 4) * (tp * tp + 2 * tp + 3 + 2 / tp + 1 / (tp * tp))
        b = (9 / 4) * (up * up + 2 * up + 3 + 2 / up + 1 / (up * up))
        c = (9 / 4) * ((tp / up) ** 2 + 2 * tp / up + 3 + 2 * up / tp + (up / tp) ** 2)
        r = (a + b + c) * rc
        flows = [(1, 2, 2, 3, 1, 4, 4, 3), (1, 2, 3, 1, 3, 4, 4, 2), (1, 2, 3, 4, 1, 4, 3, 2)]
        f = flows[0] if r < a else (flows[1] if r < a + b else flows[2])
        margin = min(abs(r - a), abs(r - a - b)) / (a + b + c)
        col, acol = list(f[0::2]), list(f[1::2])
        if rs > 0.5:
            col, acol = _swap_ca(col, acol)
        margin = min(margin, abs(rs - 0.5))
    elif code == 112:
        qn = min(1 + int(nqn * rf), nqn)
        ids = [id1, id2, qn, -qn]
        a = (1 / 6) * up / tp - (3 / 8) * up * up
        b = (1 / 6) * tp / up - (3 / 8) * tp * tp
        f = (1, 2, 2, 3, 1, 0, 0, 3) if (a + b) * rc < a else (1, 2, 3, 1, 3, 0, 0, 2)
        margin = abs((a + b) * rc - a) / (a + b)
        margin = min(margin, min(abs(nqn * rf - j) for j in range(1, nqn)) / nqn) if nqn > 1 else margin
        col, acol = list(f[0::2]), list(f[1::2])
    elif code == 113:
        ids = [id1, id2, id1, id2]
        a = (up / tp) ** 2 - (4 / 9) * up
        b = 1 / (tp * tp) - (4 / 9) / up
        f = (1, 0, 2, 1, 3, 0, 2, 3) if (a + b) * rc < a else (1, 0, 2, 3, 2, 0, 1, 3)
        margin = abs((a + b) * rc - a) / (a + b)
        col, acol = list(f[0::2]), list(f[1::2])
        if id1 == 21:   # swapCol1234
            col = [col[1], col[0], col[3], col[2]]
            acol = [acol[1], acol[0], acol[3], acol[2]]
        if id1 < 0 or id2 < 0:
            col, acol = _swap_ca(col, acol)
    elif code == 114:
        ids = [id1, id2, id1, id2]
        f = (1, 0, 2, 0, 2, 0, 1, 0) if id1 * id2 > 0 else (1, 0, 0, 1, 2, 0, 0, 2)
        if id2 == id1:
            T = (4 / 9) * (1 + up * up) / (tp * tp)
            U = (4 / 9) * (1 + tp * tp) / (up * up)
            if (T + U) * rc > T:
                f = (1, 0, 2, 0, 1, 0, 2, 0)
            margin = abs((T + U) * rc - T) / (T + U)
        col, acol = list(f[0::2]), list(f[1::2])
        if id1 < 0:
            col, acol = _swap_ca(col, acol)
    else:
        ids = [id1, id2, 21, 21]
        a = (32 / 27) * up / tp - (8 / 3) * up * up
        b = (32 / 27) * tp / up - (8 / 3) * tp * tp
        f = (1, 0, 0, 2, 1, 3, 3, 2) if (a + b) * rc < a else (1, 0, 0, 2, 3, 2, 1, 3)
        margin = abs((a + b) * rc - a) / (a + b)
        col, acol = list(f[0::2]), list(f[1::2])
        if id1 < 0:
            col, acol = _swap_ca(col, acol)
    return ids, col, acol, margin


def _pairs(code, rng):
    q = [i for i in range(-5, 6) if i]
    if code in (111, 112):
        return 21, 21
    if code == 113:
        a = int(rng.choice(q))
        return (a, 21) if rng.random() < 0.5 else (21, a)
    if code == 114:
        a = int(rng.choice(q))
        r = rng.random()
        return (a, a) if r < 0.3 else ((a, -a) if r < 0.5 else (a, int(rng.choice(q))))
    a = int(rng.choice(q))
    return a, -a


def test_set_id_col_acol_matches_pythia_logic():
    import cupythia_b200 as cp
    lib = cp._lib.load()
    rng = np.random.default_rng(21)
    ids = (C.c_int * 4)()
    col = (C.c_int * 4)()
    acol = (C.c_int * 4)()
    differ = 0
    for code in (111, 112, 113, 114, 115):
        for _ in range(4000):
            id1, id2 = _pairs(code, rng)
            z = rng.uniform(-0.999, 0.999)
            tp, up = -0.5 * (1 - z), -0.5 * (1 + z)
            rf, rc, rs = rng.random(3)
            assert lib.cp_set_id_col_acol(code, id1, id2, tp, up, 3, rf, rc, rs, ids, col, acol) == 0
            got = (list(ids), list(col), list(acol))
            r_ids, r_col, r_acol, margin = _ref(code, id1, id2, tp, up, 3, rf, rc, rs)
            assert _valid_flow(got[0], got[1], got[2]), (code, id1, id2, got)
            if got != (r_ids, r_col, r_acol):
                differ += 1
                assert margin < MARGIN, (code, id1, id2, z, rc, got, (r_ids, r_col, r_acol), margin)
    assert differ <= 5


def test_set_id_col_acol_rejects_pairs_the_process_does_not_take():
    import cupythia_b200 as cp
    lib = cp._lib.load()
    v = (C.c_int * 4)()
    bad = [(111, 1, 21), (112, 21, 2), (113, 21, 21), (113, 1, 2), (114, 21, 1), (115, 1, 1), (115, 2, -1),
           (110, 21, 21), (116, 1, -1)]
    for code, a, b in bad:
        assert lib.cp_set_id_col_acol(code, a, b, -0.5, -0.5, 3, 0.5, 0.5, 0.5, v, v, v) == cp._lib.CP_ERR_INVALID
    assert lib.cp_set_id_col_acol(111, 21, 21, 0.1, -1.1, 3, 0.5, 0.5, 0.5, v, v, v) == cp._lib.CP_ERR_INVALID
