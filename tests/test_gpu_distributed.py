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


def test_sharded_gradient_steps_equal_the_single_handle_steps():
    """One rank: the accumulate + apply pair of every variance-gradient step reproduces
    cp_vegas_gradient_step bit for bit (grid and history)."""
    import cupythia_b200 as cp
    from cupythia_b200.distributed import ShardedIntegrator
    with cp.Integrator() as a, cp.Integrator() as b:
        a.integrate(3, 1 << 20, alpha=1.5)
        b.grid = a.grid
        ha = a.adapt_gradient(4, 1 << 20, lr=0.2, iteration0=200)
        hb = ShardedIntegrator(b).adapt_gradient(4, 1 << 20, lr=0.2, iteration0=200)
        assert ha == hb
        assert np.array_equal(a.grid, b.grid)


def test_adjoint_shards_sum_to_the_whole():
    import cupythia_b200 as cp
    from cupythia_b200.distributed import shard
    n = 1 << 21
    with cp.Integrator() as it:
        it.integrate(3, 1 << 20, alpha=1.5)
        whole = it.adjoint_accumulate(n, 5).cpu().numpy()
        parts = []
        for r in range(2):
            off, cnt = shard(n, r, 2)
            it.set_point_offset(off)
            parts.append(it.adjoint_accumulate(cnt, 5).cpu().numpy())
        it.set_point_offset(0)
    tot = parts[0] + parts[1]
    assert max(parts[0][8], parts[1][8]) == whole[8]
    rest = np.r_[0:8, 9:len(whole)]
    # FP32 per-thread duals, FP64 block slots: the two groupings agree to FP32 rounding
    assert np.allclose(tot[rest], whole[rest], rtol=2e-6, atol=1e-12 * np.abs(whole[rest]).max())


def test_data_parallel_training_equals_flow_train():
    """One rank: the three phases of every step reproduce cp_flow_train bit for bit; two shards
    of a batch (run one after the other on this GPU) sum to the whole batch's moments and
    gradient."""
    import cupythia_b200 as cp
    from cupythia_b200.distributed import ShardedIntegrator, shard
    with cp.Integrator() as a, cp.Integrator() as b:
        a.integrate(3, 1 << 20, alpha=1.5)
        b.grid = a.grid
        for it in (a, b):
            it.flow_init(7)
        la = a.flow_train(6, 65536, lr=8e-3)
        lb = ShardedIntegrator(b).flow_train(6, 65536, lr=8e-3, phases=True)
        assert np.array_equal(la, lb)
        assert np.array_equal(a.flow_params, b.flow_params)
        # the next step, whole batch vs two shards
        batch = 65536
        m_whole = b.flow_step_moments(0, batch)
        g_whole, loss_whole = b.flow_step_gradient(m_whole, batch)
        m_parts, g_parts = [], []
        for r in range(2):
            off, cnt = shard(batch, r, 2)
            m_parts.append(b.flow_step_moments(off, cnt).clone())
        m_sum = m_parts[0] + m_parts[1]
        for r in range(2):
            off, cnt = shard(batch, r, 2)
            b.flow_step_moments(off, cnt)
            g, loss = b.flow_step_gradient(m_sum, batch)
            g_parts.append(g.clone())
        g_sum = (g_parts[0] + g_parts[1]).cpu().numpy().astype(np.float64)
        gw = g_whole.cpu().numpy().astype(np.float64)
    assert np.allclose(m_sum.cpu().numpy(), m_whole.cpu().numpy(), rtol=1e-12)
    assert abs(loss / loss_whole - 1) < 1e-12
    # FP32 block partial sums in other groupings: cosine 1 - 1e-9, norm to 1e-5
    cos = g_sum @ gw / np.linalg.norm(g_sum) / np.linalg.norm(gw)
    assert cos > 1 - 1e-9 and abs(np.linalg.norm(g_sum) / np.linalg.norm(gw) - 1) < 1e-5, cos
