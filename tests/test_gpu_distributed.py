"""The multi-GPU pieces on one GPU: a pass split into accumulate + refine_sums reproduces
cp_vegas_iteration exactly, shards through point offsets reproduce the unsharded sums, and the
quantile of an exported histogram equals cp_weight_quantile.""" 
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 1 << 22


def test_accumulate_refine_equals_iteration():
    import cupythia_b200 as cp
    with cp.Integrator() as a, cp.Integrator() as b:
        a.integrate(2, 1 << 20, alpha=1.5)
        b.grid = a.grid
        ra = a.iteration(N, 7, alpha=1.5)
        rb = b.refine(b.accumulate(N, 7), N, alpha=1.5)
        assert rb["sigma"] == ra["sigma"] and rb["sigma_err"] == ra["sigma_err"]
        assert np.array_equal(a.grid, b.grid)


def test_two_shards_sum_to_the_whole():
    import cupythia_b200 as cp
    from cupythia_b200.distributed import shard
    with cp.Integrator() as it:
        it.integrate(2, 1 << 20, alpha=1.5)
        whole = it.accumulate(N, 9).cpu().numpy()
        parts = []
        for r in range(2):
            off, cnt = shard(N, r, 2)
            it.set_point_offset(off)
            parts.append(it.accumulate(cnt, 9).cpu().numpy())
        it.set_point_offset(0)
    tot = parts[0] + parts[1]
    # the same points in other thread / block groupings: FP32 compensated partial sums agree
    # with the whole pass to rounding of the grouping (1e-9 relative)
    assert np.allclose(tot[[0, 1, 3]], whole[[0, 1, 3]], rtol=1e-9)
    assert max(parts[0][2], parts[1][2]) == whole[2]
    # per-bin sums are FP32 per warp before the FP64 block sums: agreement to FP32 rounding
    assert np.allclose(tot[4:], whole[4:], rtol=1e-6, atol=1e-300)


def test_histogram_quantile_equals_local_quantile():
    import cupythia_b200 as cp
    with cp.Integrator() as it:
        it.integrate(3, 1 << 21, alpha=1.5)
        it.iteration(N, 11, alpha=0.0)
        q_local = it.weight_quantile(0.999)
        q_hist = it.quantile_from_histogram(it.weight_histogram(), 0.999)
    assert q_hist == q_local
