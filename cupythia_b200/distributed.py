"""Multi-GPU integration: one process per GPU (``torch.distributed``), contiguous point shards.

Rank r of W owns the points [offset_r, offset_r + count_r) of every pass (``shard``), the
reference's shard layout (cuPythia/common/rng.cuh:5-19: shard i covers global events
[i M, i M + count)); its handle draws the Philox block of global point offset_r + p, so the
union of the shards is exactly the single-device run.  The path has one exchange per VEGAS
iteration: the pass sums (sum w, sum w^2, n_bad, 3 x n_bins per-bin sums of w^2; about 1.2 KB)
are all-reduced by sum, the largest weight by max, and every rank then refines the same grid
from the same numbers.  The unweighting threshold comes from the weight histogram summed over
ranks, so every rank accepts against the same w_max.  A variance-gradient step exchanges the
adjoint sums of its pass the same way (entry 8, the largest weight, by max).  Flow training is
data-parallel: each step's batch is shared out, the batch moments (2 doubles) and then the
gradient (one float per parameter) are all-reduced, and every rank takes the same Adam step.
Production passes need no exchange on their data path: each rank compacts its own events; the
per-pass counts are summed for reporting and exclusive-scanned into record offsets.

The compute backend is any object with the ``Integrator`` methods the calls use:
``set_point_offset``, ``accumulate``, ``refine``, ``weight_histogram``,
``quantile_from_histogram``, ``unweight``, ``adjoint_accumulate``, ``gradient_apply`` and
``flow_step_moments`` / ``flow_step_gradient`` / ``flow_step_update``; the reductions run on
whatever device its tensors live on (NCCL for CUDA tensors, gloo for CPU).
"""
import math

import numpy as np

__all__ = ["shard", "ShardedIntegrator"]


def shard(n_total, rank, world):
    """(offset, count) of rank's contiguous share of n_total points; the first n_total % world
    ranks take one point more."""
    if not (0 <= rank < world):
        raise ValueError("rank out of range")
    base, rem = divmod(int(n_total), int(world))
    return rank * base + min(rank, rem), base + (1 if rank < rem else 0)


class ShardedIntegrator:
    def __init__(self, backend, group=None):
        import torch.distributed as dist
        self.b = backend
        self.group = group
        self.dist = dist if dist.is_available() and dist.is_initialized() else None
        self.rank = self.dist.get_rank(group) if self.dist else 0
        self.world = self.dist.get_world_size(group) if self.dist else 1

    # ---------------------------------------------------------------- reductions
    def _reduce_sums(self, sums, max_index=2):
        """sum over ranks, except entry max_index (the largest weight): max"""
        if self.world == 1:
            return sums
        wmax = sums[max_index:max_index + 1].clone()
        sums[max_index] = 0
        self.dist.all_reduce(sums, group=self.group)
        self.dist.all_reduce(wmax, op=self.dist.ReduceOp.MAX, group=self.group)
        sums[max_index:max_index + 1] = wmax
        return sums

    def _sum(self, values, like):
        if self.world == 1:
            return [float(v) for v in values]
        import torch
        t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=like.device)
        self.dist.all_reduce(t, group=self.group)
        return t.tolist()

    def _gather(self, value, like):
        """value of every rank, in rank order (one all-reduce of a one-hot vector; exact for
        integers below 2^53)"""
        if self.world == 1:
            return [float(value)]
        import torch
        t = torch.zeros(self.world, dtype=torch.float64, device=like.device)
        t[self.rank] = float(value)
        self.dist.all_reduce(t, group=self.group)
        return t.tolist()

    # ---------------------------------------------------------------- VEGAS
    def iteration(self, n_total, iteration=0, alpha=1.5):
        offset, count = shard(n_total, self.rank, self.world)
        self.b.set_point_offset(offset)
        sums = self._reduce_sums(self.b.accumulate(count, iteration))
        return self.b.refine(sums, n_total, alpha)

    def integrate(self, n_iter, n_total, alpha=1.5, skip=0):
        """n_iter iterations; (per-iteration results, inverse-variance combination of those with
        index >= skip), as ``Integrator.integrate``."""
        per = [self.iteration(n_total, it, alpha) for it in range(n_iter)]
        ws = [(r["sigma"], r["sigma_err"]) for r in per[skip:] if r["sigma_err"] > 0]
        w = sum(1.0 / e ** 2 for _, e in ws)
        comb = {"sigma": sum(s / e ** 2 for s, e in ws) / w if w else 0.0,
                "sigma_err": 1.0 / math.sqrt(w) if w else 0.0, "n_points": n_total * n_iter}
        return per, comb

    def weight_quantile(self, q=0.999):
        hist = self.b.weight_histogram()
        if self.world > 1:
            self.dist.all_reduce(hist, group=self.group)
        return self.b.quantile_from_histogram(hist, q)

    # ---------------------------------------------------------------- variance-gradient steps
    def gradient_step(self, n_total, iteration=0, lr=0.5):
        """One variance-gradient step with its adjoint pass sharded: one exchange of the adjoint
        sums (10 + 12 n_bins doubles), then every rank takes the same step on its grid."""
        offset, count = shard(n_total, self.rank, self.world)
        self.b.set_point_offset(offset)
        sums = self._reduce_sums(self.b.adjoint_accumulate(count, iteration), max_index=8)
        return self.b.gradient_apply(sums, n_total, lr)

    def adapt_gradient(self, steps, n_points, lr=0.4, iteration0=0):
        """Integrator.adapt_gradient with every step sharded."""
        from . import adapt_gradient_loop
        return adapt_gradient_loop(self.gradient_step, steps, n_points, lr, iteration0)

    # ---------------------------------------------------------------- flow training
    def flow_train(self, steps, batch=65536, lr=1e-3, phases=False):
        """Integrator.flow_train data-parallel: each step's batch [0, batch) is shared out in
        contiguous ranges; two exchanges per step (the batch moments, 2 doubles, then the gradient,
        one float per parameter) and every rank takes the same Adam step.  One rank reproduces
        Integrator.flow_train bit for bit, and with one rank the backend's own training loop runs
        unless phases is set."""
        if batch < self.world:
            raise ValueError("flow_train: fewer batch points than ranks")
        if self.world == 1 and not phases and hasattr(self.b, "flow_train"):
            # nothing to exchange: the handle's own loop, with no host round trip per step
            return self.b.flow_train(steps, batch, lr)
        offset, count = shard(batch, self.rank, self.world)
        losses = np.zeros(steps)
        for s in range(steps):
            m = self.b.flow_step_moments(offset, count)
            if self.world > 1:
                self.dist.all_reduce(m, group=self.group)
            g, losses[s] = self.b.flow_step_gradient(m, batch)
            if self.world > 1:
                self.dist.all_reduce(g, group=self.group)
            self.b.flow_step_update(g, lr)
        return losses

    # ---------------------------------------------------------------- production
    def unweight(self, n_total, iteration=0, records=None):
        """Production pass over the global points [0, n_total): this rank's records (device) and
        the pass statistics summed over ranks (accepted, overweight, n_bad; sigma combined).
        ``record_offset`` is the exclusive scan of the ranks' accepted counts, the index of this
        rank's first record in the concatenation of all ranks' records in rank order (the global
        record offsets of the reference's merged output); ``records_per_rank`` the counts."""
        offset, count = shard(n_total, self.rank, self.world)
        self.b.set_point_offset(offset)
        rec, st = self.b.unweight(count, iteration=iteration, records=records)
        acc, over, bad, sw, var = self._sum(
            [st["n_accepted"], st["n_overweight"], st["n_bad"], st["sigma"] * count,
             (st["sigma_err"] * count) ** 2], like=rec)
        per_rank = [int(c) for c in self._gather(st["n_accepted"], like=rec)]
        glob = dict(st, n_points=n_total, n_accepted=int(acc), n_overweight=int(over), n_bad=int(bad),
                    sigma=sw / n_total, sigma_err=math.sqrt(var) / n_total, eta=acc / n_total,
                    record_offset=sum(per_rank[:self.rank]), records_per_rank=per_rank)
        return rec, st, glob
