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



class ToyStepBackend:
    """Adjoint-sum and flow-training surfaces with deterministic per-point contributions, so that
    the sharded schedules can be compared with one process exactly (up to FP64 rounding)."""

    def __init__(self):
        self.offset = 0
        self.grid = np.linspace(0.0, 1.0, 6)
        self.theta = np.array([0.3, -0.2, 0.1])
        self.t = 0
        self.points = None

    def set_point_offset(self, offset):
        self.offset = offset

    # per-point values of global point p: a feature vector and a weight
    def _phi(self, p, salt):
        p = np.asarray(p, np.float64)
        return np.stack([np.sin(0.37 * p + salt), np.cos(0.11 * p + 2 * salt), np.sin(0.05 * p) ** 2], 1)

    def adjoint_accumulate(self, count, iteration):
        p = self.offset + np.arange(count)
        w = 1.0 + 0.5 * np.sin(0.13 * p + iteration) * self.grid[1]
        v = np.zeros(20)
        v[0], v[1] = w.sum(), (w * w).sum()
        v[2:8] = self._phi(p, iteration).sum(0).repeat(2)
        v[8] = w.max()
        v[9:] = (w[:, None] * self._phi(p, 1.0)).sum(0).repeat(4)[:11]
        return torch.tensor(v, dtype=torch.float64)

    def gradient_apply(self, sums, n_total, lr):
        s = sums.numpy()
        mean = s[0] / n_total
        var = s[1] / n_total - mean * mean
        self.grid[1:5] += lr * 1e-3 * np.tanh(s[9:13] / n_total) * (1 + s[8])
        return {"sigma": mean, "var": var}

    def flow_step_moments(self, point0, count):
        p = point0 + np.arange(count)
        self.points = p
        w = np.exp(self._phi(p, self.t) @ self.theta)
        return torch.tensor([w.sum(), (w * w).sum()], dtype=torch.float64)

    def flow_step_gradient(self, m, batch):
        a, b = m.numpy()
        sig = a / batch
        phi = self._phi(self.points, self.t)
        w = np.exp(phi @ self.theta)
        g = (2.0 * (w * w)[:, None] * phi).sum(0) / (batch * sig * sig)
        return torch.tensor(g, dtype=torch.float64), (b / batch) / (sig * sig)

    def flow_step_update(self, g, lr):
        self.theta = self.theta - lr * g.numpy()
        self.t += 1


def _toy_schedule(si):
    hist = si.adapt_gradient(5, 1001, lr=0.4, iteration0=3)
    losses = si.flow_train(4, 777, lr=0.05)
    return hist, list(losses), si.b.grid.copy(), si.b.theta.copy()


def _toy_rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = _toy_schedule(ShardedIntegrator(ToyStepBackend()))
    finally:
        dist.destroy_process_group()


def test_sharded_gradient_steps_and_data_parallel_training_equal_one_process():
    """The variance-gradient schedule with sharded adjoint sums (largest weight by max) and the
    data-parallel flow training (moments, then gradients, all-reduced) take the same steps on two
    gloo ranks as in one process."""
    ref_hist, ref_loss, ref_grid, ref_theta = _toy_schedule(ShardedIntegrator(ToyStepBackend()))
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_toy_rank_main, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    for r in range(2):
        hist, loss, grid, theta = res[r]
        assert [h["lr"] for h in hist] == [h["lr"] for h in ref_hist]
        assert np.allclose([h["rel_var"] for h in hist], [h["rel_var"] for h in ref_hist], rtol=1e-12)
        assert np.allclose(loss, ref_loss, rtol=1e-12)
        assert np.allclose(grid, ref_grid, rtol=0, atol=1e-14)
        assert np.allclose(theta, ref_theta, rtol=1e-12, atol=1e-15)
    assert np.array_equal(res[0][3], res[1][3])   # every rank holds the same parameters
