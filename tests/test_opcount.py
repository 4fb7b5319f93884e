"""The integrand's algorithmic operation count per point (oracle/cp_opcount.cc), pinned.

The counted restatement evaluates the same weight as the literal FP64 oracle (cpo_had_weight_x)
in the form with the least arithmetic (Q-only CTEQ5L terms once per point, factorised channel
sums, shared reciprocals); the tally of its +, -, x, / and exp, log, sqrt is the per-point work
the integrand kernels' roofline is quoted on, and bench.py carries the same numbers.
"""
import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

# per point: add/sub, mul, div, exp, log, sqrt (the VEGAS map included)
PINNED = {"add": 364, "mul": 422, "div": 9, "exp": 35, "log": 26, "sqrt": 2}


def _points(n, seed):
    return np.random.default_rng(seed).random((n, 3))


def test_counted_form_is_the_oracle_integrand():
    import oracle
    L = oracle.lib()
    cfg = oracle.had_cfg()
    x = _points(4000, 11)
    a = np.array([L.cpo_opcount_weight(C.byref(cfg), oracle.dptr(np.ascontiguousarray(p))) for p in x])
    b = np.array([L.cpo_had_weight_x(C.byref(cfg), oracle.dptr(np.ascontiguousarray(p)), None) for p in x])
    assert np.array_equal(a == 0, b == 0)
    keep = b > 1e-6 * b.mean()      # the exponent sums of CTEQ5L cancel at x -> 1, where w -> 0
    rel = np.abs(a[keep] - b[keep]) / b[keep]
    assert rel.max() < 1e-12, rel.max()
    assert abs(a.sum() / b.sum() - 1) < 1e-14


def test_operation_count_is_pinned_and_in_bench():
    import oracle
    L = oracle.lib()
    cfg = oracle.had_cfg()
    for seed in (1, 2):
        x = _points(20000, seed)
        out = np.zeros(7)
        L.cpo_opcount_counts(C.byref(cfg), x.ctypes.data_as(C.c_void_p), len(x), oracle.dptr(out))
        got = dict(zip(["add", "mul", "div", "exp", "log", "sqrt"], out[:6]))
        assert got == {k: float(v) for k, v in PINNED.items()}, got
        assert out[6] < 1e-9      # the counted evaluations are the oracle's weights
    import bench
    assert bench.ALG_FP32_OPS_PER_POINT == PINNED["add"] + PINNED["mul"] + PINNED["div"]
    assert bench.ALG_MUFU_OPS_PER_POINT == PINNED["exp"] + PINNED["log"] + PINNED["sqrt"] + PINNED["div"]
