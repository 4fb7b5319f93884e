"""Benchmark: unweighted events/s of pp -> 2 jets (13 TeV, pT_hat > 20 GeV, CTEQ5L, first-order
alpha_s(mZ) = 0.13, the five HardQCD 2 -> 2 processes) on B200, at a relative sigma error
<= 1% per step, for two forms of the integrator on the same workload:

  plain VEGAS    classic Lepage refinement (10 x 2^24 points, alpha 1.5), w_max = q99.9
  flow+adjoint   variance-gradient grid refinement (adjoint kernel, 12 x 2^22 points), then a
                 BF16 coupling flow after the VEGAS map trained on 200 x 65536 points by the
                 pathwise gradient of the relative moments <w^3>/<w>^3 (100 batches), then
                 <w^4>/<w>^4 (100 batches), w_max = q99.9 through the flow
and, reported beside them, VEGAS alone on the adjoint's tail grid: the classic grid refined by
12 gradient steps of <w^4>/<w>^4 (the adjoint kernel with moment order 4), w_max = q99.9.

One step = one production pass over a batch of counter-RNG points: draw -> (flow) -> VEGAS map
-> (tau, y, cos theta) -> matrix elements x PDFs x alpha_s -> weights -> unweighting against
w_max -> on-device compaction into 64-byte event records.  Grid adaptation and flow training
run before the timed region and are reported separately (adapt_seconds).

  value        flow+adjoint events/s, inputs resident, CUDA events on the library's stream,
               max over ranks; every rank produces a disjoint range of counter points (weak
               scaling, no data-path collective; the adaptation sums are all-reduced once per
               iteration); plain_vegas holds the same for the plain form; quality: the pull
               against the FP64 oracle sigma and the points / time the 1% error needs
  e2e          the flow+adjoint form through the host-buffer C-ABI call cp_generate_host: the
               step's inputs (VEGAS grid) copied host -> device and every event record copied
               device -> pinned host memory inside the timed region; d2h_copy_gbs is the
               box's plain device -> host copy rate, the bound of this path at 64 B per event
  roofline     the dominant kernel of the timed step from live per-kernel CUDA-event durations
               (cp_set_kernel_timing); roofline_secondary the other one
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
# flow training plan of the flow+adjoint form: (batches of 65536 points, moment order p of the
# objective <w^p>/<w>^p), Adam at learning rate 8e-3.  The higher moments weigh the tail of the
# weights, which sets eta at the 99.9th-percentile w_max (mean eta over 4 seeds on the adjoint
# grid: 0.52 against 0.46 for the variance alone, <w^2>/<w>^2, at the same 200 batches).
TRAIN_PLAN = [(100, 3.0), (100, 4.0)]
TRAIN_LR = 8e-3
TAIL_GRID_MOMENT = 4.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--points", type=int, default=1 << 27, help="points per step and rank")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample length")
    ap.add_argument("--fused-production", action="store_true",
                    help="flow form through the fused flow + accept kernel (cp_flow_fuse_production) "
                         "instead of the forward followed by the accept kernel")
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
    """The pool's measured peaks (MEASURED_PEAKS.json beside this file), else the fallback of an
    earlier measurement on the same B200s: 6.65 TB/s copy, 1.59 PFLOP/s bf16 burst, about
    1.4 PFLOP/s sustained under the 1 kW power cap."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "of measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, \
        "of fallback (no MEASURED_PEAKS.json on this box)"


# --------------------------------------------------------------------------- our arm
# algorithmic work per point of the two dominant kernels
UNW_CHUNK = 1 << 24               # points per production chunk of the library (accept/scan/build launches)
# k_unw_accept, algorithmic: the integrand's operations per point counted on its least-arithmetic
# FP64 restatement (oracle/cp_opcount.cc, pinned by tests/test_opcount.py): 364 add + 422 mul + 9
# div FP32 ops, 35 exp + 26 log + 2 sqrt + 9 reciprocals on the MUFU
ALG_FP32_OPS_PER_POINT = 795
ALG_MUFU_OPS_PER_POINT = 72
# k_unw_accept, executed: FADD + FMUL + 2 FFMA lane operations per point from the ncu per-opcode
# counters of a flow-form launch (profiles/k_unw_accept_production_2e24.md; packed two-lane
# forms counted per lane), i.e. the algorithm plus the FP32 precision bookkeeping (FMA residuals,
# (hi, lo) logarithms) and the transcendentals' own arithmetic (the exp reduction's polynomial)
EXEC_FLOP_PER_POINT = 1866.7
FLOW_FLOP_PER_POINT = 35072.0     # k_flow_fwd: 2 x sum over couplings of (n_in*64 + 64*64 + 64*n_out) MACs
# DRAM bytes (read + write) per point of the flow-form launches, from ncu captures of 2^24-point
# launches of the same workload (profiles/traffic_flow_form_2e24.md); scaled to a launch's points
TRAFFIC_PER_POINT = {"k_unw_accept": (343450880 + 688227584) / 2 ** 24,
                     "k_flow_fwd_tc": (158976 + 275642624) / 2 ** 24}


def production(it, n, records, k0, warmup, steps, pg, dev, stream, clocks=None):
    """warmup + steps production passes (unweighting + compaction), device-timed per step."""
    import torch
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")   # > 126 MB L2
    for k in range(warmup):
        it.unweight(n, iteration=k0 + k, records=records)
    barrier(pg, dev)
    it.set_kernel_timing(True)
    it.kernel_times(reset=True)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    stats = []
    ctx = clocks if clocks is not None else _Null()
    with ctx:
        for k in range(steps):
            flush.zero_()
            evs[k][0].record(stream)
            stats.append(it.unweight(n, iteration=k0 + warmup + k, records=records)[1])
            evs[k][1].record(stream)
        stream.synchronize()
    barrier(pg, dev)
    it.set_kernel_timing(False)
    ktimes = it.kernel_times(reset=True)
    ms = sum(s_.elapsed_time(e_) for s_, e_ in evs)
    return stats, ms, ktimes


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def d2h_bandwidth(host, dev):
    """Plain device -> pinned host copy rate of this box (GB/s) over the e2e record buffer: the
    bound of the host-buffer path, which moves 64 bytes per event."""
    import torch
    nbytes = min(host.numel(), 1 << 30)
    src = torch.empty(nbytes, dtype=torch.uint8, device=f"cuda:{dev}")
    dst = host.view(-1)[:nbytes]
    dst.copy_(src, non_blocking=True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        dst.copy_(src, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    return 3 * nbytes / (e0.elapsed_time(e1) / 1e3) / 1e9


def oracle_sigma():
    with open(os.path.join(ROOT, "tests", "golden", "sigma_oracle.json")) as f:
        g = json.load(f)
    return g["sigma_mb"], g["sigma_err_mb"]


def quality(stats, n, sec_per_step, adapt_s):
    """The 1%-error gate and the pull against the FP64 oracle (tests/golden/sigma_oracle.json):
    inverse-variance combination of the timed steps, the points (and time) one step's throughput
    needs for delta sigma / sigma = 1%, with and without the adaptation in front."""
    import math
    w = [1.0 / s_["sigma_err"] ** 2 for s_ in stats]
    sig = sum(wi * s_["sigma"] for wi, s_ in zip(w, stats)) / sum(w)
    err = 1.0 / math.sqrt(sum(w))
    so, eo = oracle_sigma()
    rel_point = max(s_["sigma_err"] / s_["sigma"] for s_ in stats) * math.sqrt(n)   # per-point relative std
    n_1pct = math.ceil((rel_point / 0.01) ** 2)
    t_1pct = sec_per_step * n_1pct / n
    return {"sigma_mb": sig, "sigma_err_mb": err, "oracle_sigma_mb": so, "oracle_sigma_err_mb": eo,
            "pull_vs_oracle": (sig - so) / math.sqrt(err ** 2 + eo ** 2),
            "points_to_1pct": n_1pct, "time_to_1pct_s": {"steady": t_1pct, "with_adaptation": adapt_s + t_1pct}}


def run_ours(a):
    import numpy as np
    import torch

    import cupythia_b200 as cp
    from cupythia_b200.distributed import ShardedIntegrator
    rank, world, pg = dist_init(a.gpus)
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    it = cp.Integrator(device=dev)
    stream = torch.cuda.Stream(device=dev)
    it.set_stream(stream.cuda_stream)
    n = a.points
    r0 = 1000
    si = ShardedIntegrator(it)           # adaptation: shared points, one exchange per iteration
    it.adjoint_parameter_tangents(False)   # the gradient steps use only the edge gradients
    records = torch.empty((n, RECORD_BYTES), dtype=torch.uint8, device=f"cuda:{dev}")

    with torch.cuda.stream(stream):
        # ---- plain VEGAS form: classic refinement (config 2), w_max = q99.9, production
        t0 = time.perf_counter()
        per, comb = si.integrate(ADAPT_ITERS, ADAPT_POINTS, alpha=1.5, skip=3)
        wmax_plain = si.weight_quantile(0.999)
        torch.cuda.synchronize()
        adapt_plain = time.perf_counter() - t0
        it.set_point_offset(rank * n)    # production: this rank's own points, no exchange
        st_p, ms_p, kt_p = production(it, n, records, r0, a.warmup, a.steps, pg, dev, stream)
        grid_classic = it.grid

        # ---- VEGAS alone on the adjoint's tail grid: the classic grid refined by gradient steps of
        # <w^4>/<w>^4 (moment order 4 of the adjoint pass), which classic refinement cannot target
        t0 = time.perf_counter()
        it.gradient_objective(TAIL_GRID_MOMENT)
        thist = si.adapt_gradient(12, 1 << 22, lr=0.2, iteration0=400)
        it.gradient_objective(2.0)
        r_tail = si.iteration(ADAPT_POINTS, 301, alpha=0.0)
        wmax_tail = si.weight_quantile(0.999)
        torch.cuda.synchronize()
        adapt_tail = time.perf_counter() - t0
        it.set_point_offset(rank * n)
        st_t, ms_t, _ = production(it, n, records, r0 + 30000, a.warmup, a.steps, pg, dev, stream)
        it.grid = grid_classic

        # ---- flow + adjoint form: variance-gradient grid refinement (adjoint), flow trained on
        # the integrator's weights (200 x 65536 points), w_max = q99.9 through the flow
        t0 = time.perf_counter()
        # variance-gradient steps with their adjoint sums exchanged, then data-parallel flow
        # training (batch moments and gradients exchanged every step)
        ghist = si.adapt_gradient(12, 1 << 22, lr=0.2, iteration0=200)
        it.flow_init(7)
        losses = []
        for steps_, p_ in TRAIN_PLAN:
            it.flow_objective(p_)
            losses += list(si.flow_train(steps_, 65536, lr=TRAIN_LR))
        it.flow_objective(2.0)
        # proposal choice (config 5): the flow only where its weight variance beats VEGAS alone
        # on the same grid at equal points, else VEGAS is the fallback
        it.flow_enable(False)
        r_vegas = si.iteration(ADAPT_POINTS, 300, alpha=0.0)
        it.flow_enable(True)
        r_flowp = si.iteration(ADAPT_POINTS, 300, alpha=0.0)
        relvar = {k: (r["sigma_err"] / r["sigma"]) ** 2 * ADAPT_POINTS for k, r in
                  (("vegas", r_vegas), ("flow", r_flowp))}
        use_flow = relvar["flow"] < relvar["vegas"]
        it.flow_fuse_production(a.fused_production)
        if not use_flow:
            it.flow_enable(False)
            si.iteration(ADAPT_POINTS, 300, alpha=0.0)
        wmax_flow = si.weight_quantile(0.999)
        torch.cuda.synchronize()
        adapt_flow = time.perf_counter() - t0
        it.set_point_offset(rank * n)
        clk = Clocks(dev)
        st_f, ms_f, kt_f = production(it, n, records, r0 + 50000, a.warmup, a.steps, pg, dev, stream, clk)

    ev_f = sum(s_["n_accepted"] for s_ in st_f)
    ev_p = sum(s_["n_accepted"] for s_ in st_p)
    sec_f = allmax(pg, ms_f / 1e3, dev)
    sec_p = allmax(pg, ms_p / 1e3, dev)
    value = allsum(pg, ev_f, dev) / sec_f
    value_plain = allsum(pg, ev_p, dev) / sec_p
    sec_t = allmax(pg, ms_t / 1e3, dev)
    value_tail = allsum(pg, sum(s_["n_accepted"] for s_ in st_t), dev) / sec_t
    rel_err = max(s_["sigma_err"] / s_["sigma"] for s_ in st_f)
    q_f, q_p = quality(st_f, n, sec_f / a.steps, adapt_plain + adapt_flow), quality(st_p, n, sec_p / a.steps, adapt_plain)

    # ---- e2e through the host-buffer C-ABI call (grid H2D + records D2H inside the region)
    eta_max = max(s_["eta"] for s_ in st_f)
    host = torch.empty((int(n * min(1.0, 1.2 * eta_max)) + 4096, RECORD_BYTES), dtype=torch.uint8,
                       pin_memory=True)
    grid = it.grid
    for k in range(2):
        it.grid = grid
        it.generate_host(n, host, iteration=r0 + 90000 + k, chunk=1 << 21)
    barrier(pg, dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e2e_steps = max(1, a.steps // 2)
    e0.record(stream)
    w0 = time.perf_counter()
    d2h, e2e_events = 0, 0
    for k in range(e2e_steps):
        it.grid = grid
        s_ = it.generate_host(n, host, iteration=r0 + 91000 + k, chunk=1 << 21)
        e2e_events += s_["n_accepted"]
        d2h += s_["n_accepted"] * RECORD_BYTES
    e1.record(stream)
    stream.synchronize()
    wall = time.perf_counter() - w0
    e2e_sec = allmax(pg, max(e0.elapsed_time(e1) / 1e3, wall), dev)
    d2h_gbs = d2h_bandwidth(host, dev)
    e2e_all = allsum(pg, e2e_events, dev)

    # ---- rooflines of the two dominant kernels from their live CUDA-event durations
    peaks, src = measured_peaks()
    fp32_peak, mufu_peak = it.measure_peaks()
    acc_ms, acc_n = kt_f["accept"]
    flow_ms, flow_n = kt_f["flow_forward"]
    # the flow form's production kernel: the fused tcgen05 kernel (flow forward, integrand and
    # accept step in one launch per chunk) unless the forward ran as its own launch
    fused = use_flow and flow_n == 0
    bf16_peak = peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops"))
    # the integrand's bound (SIMT FP32 and MUFU co-limited): algorithmic FP32 operations per second
    # against the FP32 issue peak (one operation per lane and cycle = half the FMA-chain TFLOP/s,
    # which counts an FMA as two), and MUFU operations against the measured MUFU peak; the larger
    # fraction is the roofline
    fp32_op_peak = fp32_peak / 2.0

    chunks = (n + UNW_CHUNK - 1) // UNW_CHUNK    # launches of the accept kernel per pass

    def integrand_roof(kernel, ms, launches, with_flow):
        pts_per_s = n / (ms / max(1, launches) / 1e3)
        ops = ALG_FP32_OPS_PER_POINT * pts_per_s / 1e12
        mufu = ALG_MUFU_OPS_PER_POINT * pts_per_s / 1e12
        traffic = TRAFFIC_PER_POINT.get(kernel)
        r = {"bound": "fp32", "kernel": kernel, "achieved": ops, "peak": fp32_op_peak,
             "unit": "TFLOP/s", "frac": max(ops / fp32_op_peak, mufu / mufu_peak),
             "basis": "algorithmic FP32 operations per point (add + mul + div = %d, oracle/cp_opcount.cc) "
                      "per second against the FP32 issue peak (one op per lane-cycle); frac = max of that "
                      "and the MUFU fraction" % ALG_FP32_OPS_PER_POINT,
             "peak_source": "measured: FMA-chain microbenchmark on this GPU (cp_measure_peaks), "
                            "%.1f TFLOP/s at 2 per FMA" % fp32_peak,
             "fp32_frac": ops / fp32_op_peak, "mufu_frac": mufu / mufu_peak,
             "mufu_achieved_tops": mufu, "mufu_ops_per_point": ALG_MUFU_OPS_PER_POINT,
             "flop_per_point": ALG_FP32_OPS_PER_POINT, "traffic": traffic * n / chunks if traffic else None,
             "ms_per_launch": ms / max(1, launches) / chunks, "points_per_launch": n / chunks}
        if not with_flow:
            # executed FP32 FLOPs of k_unw_accept from its SASS counters
            r.update({"executed_flop_per_point": EXEC_FLOP_PER_POINT,
                      "executed_frac": EXEC_FLOP_PER_POINT * pts_per_s / 1e12 / fp32_peak})
        if with_flow:
            # the same launch also runs the flow's dense layers on the tensor cores
            tens = FLOW_FLOP_PER_POINT * pts_per_s / 1e12
            r.update({"basis": r["basis"] + "; and the flow's BF16 MMA FLOPs (%d per point) against the "
                      "sustained bf16 peak (%s), the largest of the three fractions" % (FLOW_FLOP_PER_POINT, src),
                      "tensor_achieved_tflops": tens, "tensor_frac": tens / bf16_peak,
                      "frac": max(r["frac"], tens / bf16_peak)})
        return r

    if fused:
        roof = integrand_roof("k_flow_accept_tc", acc_ms, acc_n, True)
        # the integrand alone: the plain VEGAS form's accept kernel
        roof2 = integrand_roof("k_unw_accept", kt_p["accept"][0], kt_p["accept"][1], False)
    else:
        r_acc = integrand_roof("k_unw_accept", acc_ms, acc_n, False)
        roof_flow = FLOW_FLOP_PER_POINT * n / (flow_ms / max(1, flow_n) / 1e3) / 1e12
        r_flow = {"bound": "tensor", "kernel": "k_flow_fwd_tc", "achieved": roof_flow, "peak": bf16_peak,
                  "unit": "TFLOP/s", "frac": roof_flow / bf16_peak,
                  "peak_source": "bf16 sustained, %s" % src,
                  "flop_per_point": FLOW_FLOP_PER_POINT, "traffic": TRAFFIC_PER_POINT["k_flow_fwd_tc"] * n,
                  "ms_per_launch": flow_ms / max(1, flow_n), "points_per_launch": n}
        roof, roof2 = (r_acc, r_flow) if acc_ms >= flow_ms else (r_flow, r_acc)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * sec_f / a.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (counter-based Philox draws, seed 42)",
        "config": {"workload": WORKLOAD, "production": "fused flow + accept kernel" if fused else "flow forward, then accept kernel",
                   "form": "flow+adjoint: classic VEGAS, variance-gradient (adjoint) grid "
                   "refinement, BF16 coupling flow trained 200 x 65536 points (moment orders 3 then 4), "
                   "unweighting at q99.9",
                   "points_per_step_per_gpu": n, "adapt_points": ADAPT_ITERS * ADAPT_POINTS,
                   "l2": "256 MB buffer written between timed steps; records written per step exceed L2",
                   "parallelism": f"dp{world}: contiguous point shards per rank; VEGAS and adjoint "
                                  "sums all-reduced once per adaptation step, flow training data-parallel "
                                  "(moments and gradients all-reduced per step), production without exchange"},
        "sigma_mb": comb["sigma"], "sigma_err_mb": comb["sigma_err"], "step_sigma_rel_err_max": rel_err,
        "eta": float(np.mean([s_["eta"] for s_ in st_f])), "w_max": wmax_flow,
        "weighted_points_per_s": n * a.steps * world / sec_f,
        "plain_vegas": {"value": value_plain, "unit": UNIT, "ms_per_step": 1e3 * sec_p / a.steps,
                        "eta": float(np.mean([s_["eta"] for s_ in st_p])), "w_max": wmax_plain,
                        "weighted_points_per_s": n * a.steps * world / sec_p,
                        "step_sigma_rel_err_max": max(s_["sigma_err"] / s_["sigma"] for s_ in st_p),
                        "adapt_seconds": adapt_plain, "quality": q_p},
        "vegas_adjoint_tail": {"value": value_tail, "unit": UNIT, "ms_per_step": 1e3 * sec_t / a.steps,
                               "eta": float(np.mean([s_["eta"] for s_ in st_t])), "w_max": wmax_tail,
                               "relative_variance_per_point": (r_tail["sigma_err"] / r_tail["sigma"]) ** 2 * ADAPT_POINTS,
                               "moment_order": TAIL_GRID_MOMENT, "adapt_seconds": adapt_tail,
                               "vs_plain": value_tail / value_plain,
                               "quality": quality(st_t, n, sec_t / a.steps, adapt_plain + adapt_tail)},
        "flow_vs_plain": value / value_plain,
        "eta_flow_over_eta_plain": float(np.mean([s_["eta"] for s_ in st_f]) / np.mean([s_["eta"] for s_ in st_p])),
        "quality": q_f,
        "adapt_seconds": adapt_plain + adapt_flow,
        "value_with_adaptation": allsum(pg, ev_f, dev) / (sec_f + adapt_flow),
        "proposal": {"used": "flow" if use_flow else "vegas (fallback)",
                     "relative_variance_per_point": relvar},
        "flow_training": {"steps": 200, "batch": 65536, "plan": [{"batches": k, "moment_order": p_} for k, p_ in TRAIN_PLAN],
                          "lr": TRAIN_LR, "loss_first": float(losses[0]),
                          "loss_last20": float(np.mean(losses[-20:])), "adjoint_rel_var": ghist[-1]["rel_var"]},
        "kernel_ms_per_step": {k: v[0] / max(1, v[1]) for k, v in kt_f.items()},
        "e2e": {"value": e2e_all / e2e_sec, "unit": UNIT, "h2d_bytes_per_step": GRID_BYTES,
                "d2h_bytes_per_step": int(d2h / e2e_steps),
                "d2h_copy_gbs": d2h_gbs, "events_per_s_at_copy_rate": d2h_gbs * 1e9 / RECORD_BYTES,
                "d2h_seconds_per_step": d2h / e2e_steps / (d2h_gbs * 1e9)},
        # per step and 2^24-point chunk: the accept kernel (fused: flow forward + accept), the slot
        # reduction, the output-offset scan and the record builder; unfused, the flow forward once
        "gpu_launches": a.steps * ((1 if use_flow and not fused else 0) + 4 * ((n + UNW_CHUNK - 1) // UNW_CHUNK)),
        "roofline": roof, "roofline_secondary": roof2,
        "mufu_peak_tops": mufu_peak,
        "clocks": clk.summary(),
    }
    if rank == 0:
        if world == 1:      # the host-core baseline is timed at N = 1 only
            line["cpu_baseline"] = cpu_baseline(a.cpu_seconds, line["plain_vegas"]["eta"])
        print(json.dumps(line), flush=True)
    it.close()
    if pg is not None:
        pg.destroy_process_group()


# --------------------------------------------------------------------------- CPU baselines
def pythia_gen(n_events, threads):
    import oracle
    out = subprocess.run([oracle.PYTHIA_REF, "gen", str(n_events), "1", str(threads)],
                         capture_output=True, text=True, check=True).stdout
    return json.loads(out.strip().split("\n")[-1])


def oracle_rate(seconds, threads, eta):
    """The FP64 C restatement of the integrand (oracle/cp_oracle.c, cpo_had_accumulate: Philox
    draw, map, tau-y-z phase space, CTEQ5L, alpha_s, the five processes' channel sum) on all host
    cores over a bounded sample; the unweighted rate it implies at the GPU arm's plain-VEGAS eta."""
    import ctypes as C

    import numpy as np

    import oracle
    L = oracle.lib()
    cfg = oracle.had_cfg()
    edges = oracle.vegas_uniform(50)
    hist = np.zeros(3 * 50)
    sums = (C.c_double * 2)()

    def run(n):
        t0 = time.perf_counter()
        L.cpo_had_accumulate(C.byref(cfg), oracle.dptr(edges), 50, 42, 0, 0, n, sums, oracle.dptr(hist), threads)
        return time.perf_counter() - t0
    probe = 1 << 16
    n = max(int(probe / run(probe) * seconds), probe)
    rate = n / run(n)
    return {"weighted_points_per_s": rate, "unweighted_events_per_s_at_plain_eta": rate * eta,
            "cores": threads, "kind": "port",
            "sample": f"{n} points of the FP64 restatement on a uniform 3x50 grid (the cost per point "
                      f"does not depend on the grid), eta {eta:.3f} of the plain-VEGAS form"}


def cpu_baseline(seconds, eta_plain):
    """Stock Pythia 8.317 (ProcessLevel, same settings) on all host cores, bounded sample; beside
    it the FP64 restatement of the integrand (the oracle) on the same cores."""
    import oracle
    threads = os.cpu_count() or 1
    if not os.path.exists(oracle.PYTHIA_REF):
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "oracle/_ref/pythia_ref missing (reference not built)",
                "port": oracle_rate(seconds / 5, threads, eta_plain)}
    probe = pythia_gen(20000 * threads, threads)
    rate = probe["accepted"] / probe["seconds"]
    n = max(int(rate * seconds), 20000 * threads)
    r = pythia_gen(n, threads)
    return {"value": r["accepted"] / r["seconds"], "unit": UNIT, "cores": threads,
            "kind": "reference",
            "sample": f"{r['accepted']} unweighted events ({r['tried']} tried) of stock Pythia 8.317 "
                      f"ProcessLevel, {threads} threads x 1 Pythia instance, sigma_gen "
                      f"{r['sigma_mb']:.5g} +- {r['sigma_err_mb']:.2g} mb; event generation timed, "
                      f"init ({r.get('init_seconds', 0.0):.2f} s) before the clock",
            "port": oracle_rate(seconds / 5, threads, eta_plain)}


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
    tot_ev, tot_s, tot_init, last = 0, 0.0, 0.0, None
    for _ in range(a.steps):
        last = pythia_gen(per_step, threads)
        tot_ev += last["accepted"]
        tot_s += last["seconds"]            # event generation only (after every thread's init)
        tot_init += last.get("init_seconds", 0.0)
    v = tot_ev / tot_s
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * tot_s / a.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (Pythia RANMAR, seed 1..threads)",
        "config": {"workload": WORKLOAD.replace("VEGAS 3x50 adapted 10x2^24 points, unweighting at the "
                                                "99.9th-percentile w_max, 64-byte event records",
                                                "Pythia multichannel sampling and sigma_max unweighting"),
                   "events_per_step": per_step, "threads": threads},
        "sigma_mb": last["sigma_mb"], "sigma_err_mb": last["sigma_err_mb"],
        "init_seconds_per_step": tot_init / a.steps,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{per_step} events per step, stock Pythia 8.317 ProcessLevel; the "
                                   f"clock covers event generation only, each thread's Pythia::init "
                                   f"(with the sigma_max scan) runs before it"},
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
