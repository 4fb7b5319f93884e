"""Generate the golden fixtures of tests/golden/ from the reference's own code.

Runs only where the reference sources were present to build oracle/_ref/ (make -f oracle/ref.mk):
  * oracle/_ref/pythia_ref        stock Pythia 8.317 (CTEQ5L, AlphaStrong, Sigma2* sigmaPDF, and
                                  ProcessLevel generation for sigma_gen)
  * oracle/_ref/libcupythia_ref.so  cuPythia's rng.cuh / physics.cuh compiled as C++
and writes small JSON files that the test suite reads on any machine.

Usage: python tests/golden/make_golden.py [--gen-events N]
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def run(args):
    return subprocess.run([oracle.PYTHIA_REF] + [str(a) for a in args], capture_output=True,
                          text=True, check=True).stdout


def pdf_fixture(rng):
    xs = np.concatenate([10 ** rng.uniform(-5.9, -0.01, 60), [1e-6, 1e-5, 0.5, 0.9, 0.999, 0.9999]])
    q2 = np.concatenate([10 ** rng.uniform(0.1, 7.9, 60), [2.0, 400.0, 1e4, 4.2e7, 1.5, 1e8]])
    args = []
    for x, q in zip(xs, q2):
        args += [repr(float(x)), repr(float(q))]
    rows = [list(map(float, l.split())) for l in run(["pdf"] + args).strip().split("\n")]
    return {"ids": [-5, -4, -3, -2, -1, 1, 2, 3, 4, 5, 21], "rows": rows}


def alphas_fixture():
    out = {}
    q2 = [1.0, 2.0, 5.0, 30.0, 400.0, 8315.2, 1e4, 3e4, 29241.0, 29242.0, 1e6, 4.2e7]
    for a in (0.11, 0.118, 0.13, 0.14):
        rows = [list(map(float, l.split())) for l in run(["alphas", a] + q2).strip().split("\n")]
        out[repr(a)] = rows
    return out


def sigma_fixture(rng, n=400):
    s = 13000.0 ** 2
    rows = []
    for _ in range(n):
        tau = np.exp(np.log(1600 / s) * rng.random())
        y = np.log(tau) * (rng.random() - 0.5)
        x1, x2 = np.sqrt(tau) * np.exp(y), np.sqrt(tau) * np.exp(-y)
        sH = tau * s
        zmax = np.sqrt(1 - 400 / (sH / 4))
        z = zmax * (2 * rng.random() - 1)
        rows.append((x1, x2, sH, -0.5 * sH * (1 - z)))
    # the kernels take FP32 inputs: store FP32-representable values
    rows = [tuple(float(np.float32(v)) for v in r) for r in rows]
    path = os.path.join(OUT, "_kin.txt")
    with open(path, "w") as f:
        f.write("\n".join("%.17g %.17g %.17g %.17g" % r for r in rows))
    lines = run(["sigma", path]).strip().split("\n")
    os.remove(path)
    table = [list(map(float, l.split())) for l in lines if l and l[0] in "0123456789-."]
    return {"columns": ["x1", "x2", "sH", "tH", "gg2gg", "gg2qqbar", "qg2qg", "qq2qq", "qqbar2gg",
                        "alphaSRen", "Q2Ren"], "rows": table}


def cupythia_fixture():
    L = oracle.cupythia_ref()
    xs = [0, 1, 42, 0xABCDEF01, 0x9E3779B97F4A7C15, 2 ** 64 - 1, 0x100000001B3 * 12345]
    sm = [[x, L.ref_splitmix64(x), L.ref_u01(L.ref_splitmix64(x))] for x in xs]
    me = []
    for s, c, a in [(1e4, 0.3, 0.13), (1e4, -0.89, 0.118), (1e4, 0.0, 0.13), (2.5e5, 0.7, 0.1)]:
        t = -0.5 * s * (1 - c)
        me.append([s, t, -s - t, a, L.ref_gg2gg_sigma(s, t, -s - t, a)])
    fused = []
    for seed, nthr, kper, aS in [(0xABCDEF01, 256, 64, 0.118), (42, 1000, 7, 0.13)]:
        fused.append({"seed": seed, "n_threads": nthr, "k_per": kper, "alphas": aS, "s": 1e4, "cmax": 0.9,
                      "sum": L.ref_fused_cpu_sum(seed, nthr, kper, 1e4, aS, 0.9, 1)})
    cpumc = {"seed": 0xABCDEF01, "n": 100000, "s": 1e4, "alphas": 0.118, "cmax": 0.9,
             "value_gev2": L.ref_cpuMC(0xABCDEF01, 100000, 1e4, 0.118, 0.9)}
    return {"splitmix": sm, "gg2gg": me, "fused_sums": fused, "cpuMC": cpumc}


def sigma_gen_fixture(n_events, threads):
    out = json.loads(run(["gen", n_events, 1, threads]).strip().split("\n")[-1])
    out.update({"pTHatMin": 20.0, "alphaSvalue": 0.13, "eCM": 13000.0, "PDF:pSet": 2,
                "processes": ["gg2gg", "qg2qg", "qqbar2gg", "gg2qqbar", "qq2qq"]})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gen-events", type=int, default=2000000)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--skip-gen", action="store_true")
    a = ap.parse_args()
    rng = np.random.default_rng(20261203)
    fixtures = {
        "pythia_pdf.json": pdf_fixture(rng),
        "pythia_alphas.json": alphas_fixture(),
        "pythia_sigma.json": sigma_fixture(rng),
        "cupythia_ref.json": cupythia_fixture(),
    }
    if not a.skip_gen:
        fixtures["pythia_sigma_gen.json"] = sigma_gen_fixture(a.gen_events, a.threads)
    for name, obj in fixtures.items():
        with open(os.path.join(OUT, name), "w") as f:
            json.dump(obj, f, indent=1)
        print("wrote", name)


if __name__ == "__main__":
    main()
