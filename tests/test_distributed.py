"""Multi-GPU logic on the CPU: contiguous point shards and the per-iteration exchange of
``cupythia_b200.distributed.ShardedIntegrator``, run as world_size-2 gloo process groups with the
oracle as the compute backend.  Two ranks must produce exactly the grid and cross section of
one process over all points (the reduction is a sum of two partial sums, order-independent)."""
import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from cupythia_b200.distributed import ShardedIntegrator, shard

NB = 50
SEED = 42


class OracleBackend:
    """The Integrator's pass/refine surface on the FP64 oracle (CPU tensors)."""

    def __init__(self):
        self.cfg = oracle.had_cfg()
        self.edges = np.zeros(3 * (NB + 1))
        oracle.lib().cpo_vegas_uniform(oracle.dptr(self.edges), 3, NB)
        self.offset = 0

    def set_point_offset(self, offset):
        self.offset = offset

    def accumulate(self, n, iteration):
        sums = np.zeros(2)
        hist = np.zeros(3 * NB)
        oracle.lib().cpo_had_accumulate(C.byref(self.cfg), oracle.dptr(self.edges), NB, SEED, iteration,
                                        self.offset, n, oracle.dptr(sums), oracle.dptr(hist), 2)
        return torch.tensor(np.concatenate([sums, [0.0, 0.0], hist]), dtype=torch.float64)

    def refine(self, sums, n_total, alpha):
        s = sums.numpy()
        mean = s[0] / n_total
        var = (s[1] / n_total - mean * mean) / (n_total - 1)
        oracle.lib().cpo_vegas_refine(oracle.dptr(self.edges), oracle.dptr(np.ascontiguousarray(s[4:])), 3, NB, alpha)
        return {"sigma": mean, "sigma_err": float(np.sqrt(max(var, 0.0))), "grid": self.edges.copy()}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, n_total, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        si = ShardedIntegrator(OracleBackend())
        per, comb = si.integrate(3, n_total, alpha=1.5)
        out[rank] = (per[-1]["grid"], [r["sigma"] for r in per], [r["sigma_err"] for r in per])
    finally:
        dist.destroy_process_group()


def test_shards_cover_the_points_once():
    for n, w in [(10, 3), (1 << 20, 8), (7, 7), (5, 8)]:
        got = []
        for r in range(w):
            off, cnt = shard(n, r, w)
            got.extend(range(off, off + cnt))
        assert got == list(range(n))
    with pytest.raises(ValueError):
        shard(10, 2, 2)


def test_two_gloo_ranks_equal_one_process():
    n_total = 1 << 14
    single = ShardedIntegrator(OracleBackend())
    assert single.world == 1
    per, _ = single.integrate(3, n_total, alpha=1.5)
    ref_grid, ref_sig = per[-1]["grid"], [r["sigma"] for r in per]
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank_main, args=(r, 2, port, n_total, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    for r in range(2):
        grid, sig, err = res[r]
        assert np.allclose(grid, ref_grid, rtol=0, atol=1e-12)
        assert np.allclose(sig, ref_sig, rtol=1e-12)
    assert np.array_equal(res[0][0], res[1][0])   # both ranks hold the same grid


class CountingBackend:
    """Production surface only: a rank's pass over count points accepts count // 3 + offset % 5
    of them (any deterministic, rank-dependent number does)."""

    def __init__(self):
        self.offset = 0

    def set_point_offset(self, offset):
        self.offset = offset

    def unweight(self, count, iteration=0, records=None):
        k = count // 3 + self.offset % 5
        return torch.zeros((k, 64), dtype=torch.uint8), {
            "n_accepted": k, "n_overweight": 1, "n_bad": 0, "sigma": 0.75, "sigma_err": 0.01, "eta": k / count}


def _unweight_rank_main(rank, world, port, n_total, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rec, st, glob = ShardedIntegrator(CountingBackend()).unweight(n_total, iteration=5)
        out[rank] = (len(rec), glob["record_offset"], glob["records_per_rank"], glob["n_accepted"],
                     glob["n_overweight"])
    finally:
        dist.destroy_process_group()


def test_record_offsets_are_the_exclusive_scan_of_accepted_counts():
    n_total, world = 1000003, 3
    expect = []
    for r in range(world):
        off, cnt = shard(n_total, r, world)
        expect.append(cnt // 3 + off % 5)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_unweight_rank_main, args=(r, world, port, n_total, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    for r in range(world):
        n_rec, rec_off, per_rank, n_acc, n_over = res[r]
        assert n_rec == expect[r]
        assert per_rank == expect
        assert rec_off == sum(expect[:r])
        assert n_acc == sum(expect) and n_over == world

