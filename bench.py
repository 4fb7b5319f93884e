"""Benchmark: unweighted events/s of pp -> 2 jets (13 TeV, pT_hat > 20 GeV, CTEQ5L, first-order
alpha_s(mZ) = 0.13, the five HardQCD 2 -> 2 processes) on B200, at a relative sigma error
<= 1% per step.

One step = one production pass over a batch of counter-RNG points: draw -> (flow) -> VEGAS map
-> (tau, y, cos theta) -> matrix elements x PDFs x alpha_s -> weights -> unweighting against
w_max (99.9th percentile) -> on-device compaction into 64-byte event records.  Grid adaptation
(and flow training) run before the timed region and are reported separately.

  value   steady-state events/s, inputs resident, CUDA events on the library's stream, max over
          ranks; every rank produces a disjoint range of counter points (weak scaling, no
          data-path collective)
  e2e     the same through the host-buffer C-ABI call cp_generate_host: the step's inputs
          (VEGAS grid) copied host -> device and every event record copied device -> pinned
          host memory inside the timed region
  --impl reference   stock Pythia 8.317 (ProcessLevel, the same settings) on all host cores

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "unweighted events/s at 1% sigma error (pp->2 jets, pT_hat>20 GeV, 13 TeV)"
UNIT = "events/s"
WORKLOAD = ("pp->2 jets 13 TeV, 5 HardQCD processes, CTEQ5L, alpha_s(mZ)=0.13 first order, "
            "mu^2=pT^2, pT_hat>20 GeV: VEGAS 3x50 adapted 10x2^24 points, unweighting at the "
            "99.9th-percentile w_max, 64-byte event records")
ADAPT_ITERS = 10
ADAPT_POINTS = 1 << 24
RECORD_BYTES = 64
GRID_BYTES = 3 * 51 * 8


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--points", type=int, default=1 << 27, help="points per step and rank")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample length")
    return ap.parse_args()


# --------------------------------------------------------------------------- distributed
def dist_init(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world != n:
        raise SystemExit(f"--gpus {n} but WORLD_SIZE={world}: launch with torch.distributed.run")
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return rank, world, pg


def barrier(pg, dev):
    import torch
    if pg is not None:
        pg.barrier(device_ids=[dev])
    torch.cuda.synchronize()


def allmax(pg, v, dev):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{dev}")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def allsum(pg, v, dev):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{dev}")
    pg.all_reduce(t)
    return float(t.item())


# --------------------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi sampling during the timed region (SM clock, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        self.rows = []
        if self.p is None:
            return
        time.sleep(0.25)
        self.p.terminate()
        out, _ = self.p.communicate(timeout=10)
        for line in out.strip().split("\n"):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                self.rows.append(f)

    def summary(self):
        if not getattr(self, "rows", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit())
        mx = max(float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(self.rows)}


# --------------------------------------------------------------------------- peaks
def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


# --------------------------------------------------------------------------- our arm
def run_ours(a):
    import numpy as np
    import torch

    import cupythia_b200 as cp
    rank, world, pg = dist_init(a.gpus)
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    it = cp.Integrator(device=dev)
    stream = torch.cuda.Stream(device=dev)
    it.set_stream(stream.cuda_stream)
    n = a.points

    # ---- adaptation (untimed in `value`, reported): classic VEGAS refinement, then w_max
    t0 = time.perf_counter()
    per, comb = it.integrate(ADAPT_ITERS, ADAPT_POINTS, alpha=1.5, skip=3)
    wmax = it.weight_quantile(0.999)
    torch.cuda.synchronize()
    adapt_s = time.perf_counter() - t0

    cap = n
    records = torch.empty((cap, RECORD_BYTES), dtype=torch.uint8, device=f"cuda:{dev}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")   # > 126 MB L2
    r0 = rank * (a.steps + a.warmup + 1)     # disjoint counter iterations per rank

    def step(k):
        return it.unweight(n, iteration=1000 + r0 + k, records=records)[1]

    with torch.cuda.stream(stream):
        for k in range(a.warmup):
            step(k)
        barrier(pg, dev)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(a.steps)]
        stats = []
        with Clocks(dev) as clk:
            for k in range(a.steps):
                flush.zero_()
                evs[k][0].record(stream)
                stats.append(step(a.warmup + k))
                evs[k][1].record(stream)
            stream.synchronize()
        barrier(pg, dev)
    ms = sum(s.elapsed_time(e) for s, e in evs)
    events = sum(s["n_accepted"] for s in stats)
    sec = allmax(pg, ms / 1e3, dev)
    events_all = allsum(pg, events, dev)
    rel_err = max(s["sigma_err"] / s["sigma"] for s in stats)

    # ---- e2e through the host-buffer C-ABI call (grid H2D + records D2H inside the region)
    eta_max = max(s_["eta"] for s_ in stats)
    host = torch.empty((int(n * min(1.0, 1.2 * eta_max)) + 4096, RECORD_BYTES), dtype=torch.uint8,
                       pin_memory=True)
    grid = it.grid
    e2e_events = 0
    for k in range(2):   # warm-up of the host path
        it.grid = grid
        it.generate_host(n, host, iteration=5000 + r0 + k, chunk=1 << 24)
    barrier(pg, dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e2e_steps = max(1, a.steps // 2)
    e0.record(stream)
    w0 = time.perf_counter()
    d2h = 0
    for k in range(e2e_steps):
        it.grid = grid
        s = it.generate_host(n, host, iteration=6000 + r0 + k, chunk=1 << 24)
        e2e_events += s["n_accepted"]
        d2h += s["n_accepted"] * RECORD_BYTES
    e1.record(stream)
    stream.synchronize()
    wall = time.perf_counter() - w0
    e2e_sec = allmax(pg, max(e0.elapsed_time(e1) / 1e3, wall), dev)
    e2e_all = allsum(pg, e2e_events, dev)

    # ---- roofline of the dominant kernel (k_unw_accept): FP32-pipe work per point
    peaks, src = measured_peaks()
    fp32_peak = fp32_peak_tflops(it, stream)
    ops = FP32_FLOP_PER_POINT
    achieved = ops * n * a.steps / (ms / 1e3) / 1e12
    unit_ms = ms / a.steps

    line = {
        "metric": METRIC, "value": events_all / sec, "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * sec / a.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (counter-based Philox draws, seed 42)",
        "config": {"workload": WORKLOAD, "form": "plain VEGAS (classic refinement)",
                   "points_per_step_per_gpu": n, "adapt_points": ADAPT_ITERS * ADAPT_POINTS,
                   "l2": "256 MB buffer written between timed steps; records written per step exceed L2",
                   "parallelism": f"dp{world} (disjoint counter ranges)"},
        "sigma_mb": comb["sigma"], "sigma_err_mb": comb["sigma_err"], "step_sigma_rel_err_max": rel_err,
        "eta": float(np.mean([s["eta"] for s in stats])), "w_max": wmax,
        "weighted_points_per_s": n * a.steps * world / sec,
        "adapt_seconds": adapt_s,
        "e2e": {"value": e2e_all / e2e_sec, "unit": UNIT, "h2d_bytes_per_step": GRID_BYTES,
                "d2h_bytes_per_step": int(d2h / e2e_steps)},
        "gpu_launches": 3 * a.steps,
        "roofline": {"bound": "fp32", "kernel": "k_unw_accept", "achieved": achieved,
                     "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                     "peak_source": "measured: FMA-chain microbenchmark on this GPU (cp_measure_peaks)",
                     "flop_per_point": ops, "traffic": None, "ms_per_launch": unit_ms,
                     "hbm_peak_gbs": peaks.get("hbm_gbs"), "hbm_peak_source": src},
        "clocks": clk.summary(),
    }
    if rank == 0:
        line["cpu_baseline"] = cpu_baseline(a.cpu_seconds)
        print(json.dumps(line), flush=True)
    it.close()
    if pg is not None:
        pg.destroy_process_group()


# FP32 FLOP per point of the fused integrand (FADD + FMUL + 2 FFMA, thread level), from the ncu
# SASS counters of k_unw_accept on a 2^22-point pass; see profiles/.
FP32_FLOP_PER_POINT = 3278.0


def fp32_peak_tflops(it, stream):
    return it.measure_peaks()[0]


# --------------------------------------------------------------------------- CPU baselines
def pythia_gen(n_events, threads):
    import oracle
    out = subprocess.run([oracle.PYTHIA_REF, "gen", str(n_events), "1", str(threads)],
                         capture_output=True, text=True, check=True).stdout
    return json.loads(out.strip().split("\n")[-1])


def cpu_baseline(seconds):
    """Stock Pythia 8.317 (ProcessLevel, same settings) on all host cores, bounded sample."""
    import oracle
    threads = os.cpu_count() or 1
    if not os.path.exists(oracle.PYTHIA_REF):
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "oracle/_ref/pythia_ref missing (reference not built)"}
    probe = pythia_gen(20000 * threads, threads)
    rate = probe["accepted"] / probe["seconds"]
    n = max(int(rate * seconds), 20000 * threads)
    r = pythia_gen(n, threads)
    return {"value": r["accepted"] / r["seconds"], "unit": UNIT, "cores": threads,
            "kind": "reference",
            "sample": f"{r['accepted']} unweighted events ({r['tried']} tried) of stock Pythia 8.317 "
                      f"ProcessLevel, {threads} threads x 1 Pythia instance, sigma_gen "
                      f"{r['sigma_mb']:.5g} +- {r['sigma_err_mb']:.2g} mb"}


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    if not os.path.exists(oracle.PYTHIA_REF):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/pythia_ref not built"}))
        return
    threads = os.cpu_count() or 1
    probe = pythia_gen(10000 * threads, threads)
    rate = probe["accepted"] / probe["seconds"]
    per_step = max(int(rate * 2.0), 10000 * threads)     # ~2 s per step
    for _ in range(a.warmup):
        pythia_gen(per_step // 4, threads)
    tot_ev, tot_s, last = 0, 0.0, None
    for _ in range(a.steps):
        last = pythia_gen(per_step, threads)
        tot_ev += last["accepted"]
        tot_s += last["seconds"]
    v = tot_ev / tot_s
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * tot_s / a.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (Pythia RANMAR, seed 1..threads)",
        "config": {"workload": WORKLOAD.replace("VEGAS 3x50 adapted 10x2^24 points, unweighting at the "
                                                "99.9th-percentile w_max, 64-byte event records",
                                                "Pythia multichannel sampling and sigma_max unweighting"),
                   "events_per_step": per_step, "threads": threads},
        "sigma_mb": last["sigma_mb"], "sigma_err_mb": last["sigma_err_mb"],
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{per_step} events per step, stock Pythia 8.317 ProcessLevel"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
