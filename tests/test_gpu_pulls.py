"""Multi-seed pull distribution of sigma for both forms of the dijet integrator.

One seed is one full run: the config-2 adaptation (10 x 2^24 points, classic refinement), then,
for the flow+adjoint form, the bench's recipe: 12 variance-gradient steps (backtracking) and the
flow trained on 200 x 65,536 points (moment orders 3 then 4), then one fresh production-sized
pass of 2^24 points on counter points disjoint from everything the adaptation saw.  Across seeds (the Philox key of the whole run):
  * the error estimate is honest: the spread of sigma_i about the seeds' mean, in units of each
    run's own sigma_err, has a standard deviation between 0.7 and 1.4;
  * the estimate is unbiased against the FP64 oracle (tests/golden/sigma_oracle.json, 2^28 points):
    the seeds' mean is within 3 combined standard deviations of it (the oracle's error enters once,
    being common to all seeds).
One seed's pull against a 1-sigma window would fail for about a third of correct seeds; the
distribution is the test (ProcessContainer::sigmaDelta, pythia8317/src/ProcessContainer.cc:
1416-1470, for the sigma / delta-sigma definition).
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SEEDS = list(range(101, 149))     # 48 runs
N = 1 << 24


def _oracle():
    with open(os.path.join(ROOT, "tests", "golden", "sigma_oracle.json")) as f:
        g = json.load(f)
    return g["sigma_mb"], g["sigma_err_mb"]


def _runs(flow):
    import cupythia_b200 as cp
    out = []
    for seed in SEEDS:
        with cp.Integrator(seed=seed) as it:
            it.integrate(10, N, alpha=1.5, skip=3)
            if flow:
                it.adapt_gradient(12, 1 << 22, lr=0.2, iteration0=200)
                it.flow_init(7)
                for steps, p in ((100, 3.0), (100, 4.0)):
                    it.flow_objective(p)
                    it.flow_train(steps, 65536, lr=8e-3)
                it.flow_objective(2.0)
                it.flow_enable(True)
            r = it.iteration(N, 7000, alpha=0.0)
            assert r["n_bad"] == 0
            out.append((r["sigma"], r["sigma_err"]))
    return np.array(out)


def _check(res, label):
    so, eo = _oracle()
    s, e = res[:, 0], res[:, 1]
    n = len(s)
    mean = s.mean()
    self_pull = (s - mean) / e * np.sqrt(n / (n - 1.0))
    sd = self_pull.std(ddof=0)
    mean_err = np.sqrt((e ** 2).sum()) / n
    bias_pull = (mean - so) / np.sqrt(mean_err ** 2 + eo ** 2)
    pulls = (s - so) / np.sqrt(e ** 2 + eo ** 2)
    print(f"{label}: seeds {n}, mean pull vs oracle {pulls.mean():+.3f}, sd of pulls {pulls.std():.3f}, "
          f"self-pull sd {sd:.3f}, bias pull of the mean {bias_pull:+.3f}, "
          f"|pull| < 1 for {np.mean(np.abs(pulls) < 1):.2f} of the seeds")
    assert 0.7 < sd < 1.4, (label, sd)
    assert abs(bias_pull) < 3.0, (label, bias_pull)


def test_pull_distribution_plain_vegas():
    _check(_runs(False), "plain VEGAS")


def test_pull_distribution_flow_adjoint():
    _check(_runs(True), "flow+adjoint")
