"""Generates tests/golden/sigma_oracle.json: the FP64 oracle's cross section of the dijet
configuration (pp 13 TeV, pT_hat > 20 GeV, CTEQ5L, alpha_s(mZ) = 0.13 first order, the five
HardQCD processes): 10 classic VEGAS iterations of 2^22 points (alpha 1.5, 3 x 50 bins) on the
oracle, then one pass of 2^28 points on the adapted grid (Philox seed 42, counter iteration 1000).
bench.py reports the pull of its estimate against this value.  Runtime: about two minutes on 8 cores.

    python tests/golden/make_sigma_oracle.py
"""
import ctypes as C
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

NB, SEED = 50, 42


def main():
    L = oracle.lib()
    cfg = oracle.had_cfg()
    edges = np.zeros(3 * (NB + 1))
    L.cpo_vegas_uniform(oracle.dptr(edges), 3, NB)
    threads = os.cpu_count() or 1
    t0 = time.time()
    for it in range(10):
        sums, hist = np.zeros(2), np.zeros(3 * NB)
        L.cpo_had_accumulate(C.byref(cfg), oracle.dptr(edges), NB, SEED, it, 0, 1 << 22, oracle.dptr(sums),
                             oracle.dptr(hist), threads)
        L.cpo_vegas_refine(oracle.dptr(edges), oracle.dptr(hist), 3, NB, 1.5)
    n = 1 << 28
    sums = np.zeros(2)
    L.cpo_had_accumulate(C.byref(cfg), oracle.dptr(edges), NB, SEED, 1000, 0, n, oracle.dptr(sums), None, threads)
    mean = sums[0] / n
    err = float(np.sqrt((sums[1] / n - mean * mean) / (n - 1)))
    out = {"sigma_mb": mean, "sigma_err_mb": err, "n_points": n, "adapt": "10 x 2^22 classic VEGAS, alpha 1.5",
           "config": "pp 13 TeV, pT_hat > 20 GeV, CTEQ5L, alpha_s(mZ) = 0.13 first order, 5 HardQCD processes",
           "seconds": round(time.time() - t0, 1)}
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "sigma_oracle.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(out)


if __name__ == "__main__":
    main()
