"""The learned proposal: BF16 tensor-core flow kernels against the FP64 CPU oracle.

Tolerances: the forward runs in BF16 (weights, MLP inputs, activations) with FP32 accumulation,
the oracle in FP64 with the same rounding points, so single BF16 rounding flips near ties move a
few points: forward |dv| <= 2e-3 and |d ln J| <= 2e-2 for 99.9% of points.  The training
gradient (tensor-core backward, BF16 operands) must agree with the FP64 backprop of the same
cotangents to cosine similarity 0.999 and 5% in L2 norm."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NPAR = 4 * 5768
PER = 5768


def _used_mask():
    m = np.zeros(NPAR, bool)
    nin = [1, 2, 1, 2]
    nout = [4, 2, 4, 2]
    for c in range(4):
        b = c * PER
        for r in range(nin[c]):
            m[b + r * 64:b + r * 64 + 64] = True
        m[b + 1024:b + 5248] = True
        for k in range(64):
            m[b + 5248 + k * 8:b + 5248 + k * 8 + nout[c]] = True
        m[b + 5760:b + 5760 + nout[c]] = True
    return m


def _random_flow(it, seed=3, scale=0.08):
    it.flow_init(7)
    P = it.flow_params.copy()
    rng = np.random.default_rng(seed)
    m = _used_mask()
    for c in range(4):
        b = c * PER
        sl = slice(b + 5248, b + 5768)
        P[sl] = np.where(m[sl], rng.normal(0, scale, 520), 0).astype(np.float32)
        P[b + 1024:b + 1088] = rng.normal(0, 0.05, 64)
        P[b + 5184:b + 5248] = rng.normal(0, 0.05, 64)
    it.flow_params = P
    return P


def _xv(it, words):
    """The flow's input: the VEGAS map of the words with a half-step offset (x_v strictly inside
    (0, 1)), in FP32 as the kernel forms it, and ln of the VEGAS Jacobian."""
    nb = it.nb
    grid = it.grid
    m = (words[:, :3] >> 8).astype(np.uint64) * nb
    b = (m >> 24).astype(np.int64)
    frac = (((m & 0xFFFFFF).astype(np.float64) + 0.5) / 2 ** 24).astype(np.float32)
    lo = np.stack([grid[d][b[:, d]] for d in range(3)], 1).astype(np.float32)
    wd = np.stack([grid[d][b[:, d] + 1] - grid[d][b[:, d]] for d in range(3)], 1).astype(np.float32)
    x = (lo.astype(np.float64) + frac.astype(np.float64) * wd.astype(np.float64)).astype(np.float32)
    x = np.clip(x, np.float32(5.9604645e-8), np.float32(0.99999994)).astype(np.float64)
    lnjv = np.log(np.prod(nb * wd.astype(np.float64), 1))
    return x, lnjv


def test_untrained_flow_is_identity(integ):
    integ.reset_grid()
    integ.integrate(3, 1 << 20, alpha=1.5)
    integ.flow_init(7)
    out = integ.flow_sample(0, 4096, 3, 0).cpu().numpy()
    xv, lnjv = _xv(integ, integ.philox_words(integ.cfg.seed, 0, 4096, 3, 0))
    assert np.max(np.abs(out[:, :3] - xv)) < 2e-6
    assert np.max(np.abs(out[:, 3] - lnjv)) < 2e-4 * np.maximum(1, np.abs(lnjv)).max()
    integ.reset_grid()


def test_flow_forward_matches_fp64_oracle(integ, orc):
    P = _random_flow(integ)
    n = 4096
    out = integ.flow_sample(0, n, 3, 0).cpu().numpy().astype(np.float64)
    u, lnjv = _xv(integ, integ.philox_words(integ.cfg.seed, 0, n, 3, 0))
    out[:, 3] -= lnjv
    L = orc.lib()
    ref = np.zeros((n, 4))
    v = np.zeros(3)
    lj = C.c_double()
    for i in range(n):
        L.cpo_flow_forward(P.ctypes.data, orc.dptr(u[i].copy()), orc.dptr(v), C.byref(lj))
        ref[i, :3] = v
        ref[i, 3] = lj.value
    dv = np.abs(out[:, :3] - ref[:, :3]).max(1)
    dj = np.abs(out[:, 3] - ref[:, 3])
    assert np.percentile(dv, 99.9) < 2e-3 and np.median(dv) < 1e-4, (np.median(dv), np.percentile(dv, 99.9))
    assert np.percentile(dj, 99.9) < 2e-2 and np.median(dj) < 1e-3, (np.median(dj), np.percentile(dj, 99.9))
    # the map is non-trivial: it moved the points
    assert np.median(np.abs(ref[:, :3] - u)) > 1e-3


def test_tcgen05_forward_matches_mma_forward(integ):
    """The tcgen05 kernel (TMEM accumulators, biases inside the MMAs as BF16 hi/lo pairs) and the
    warp-level mma.sync kernel compute the same map; they differ by FP32 accumulation order and
    the ~2^-17 bias split, which moves a BF16 rounding of a hidden unit now and then."""
    integ.reset_grid()
    integ.integrate(3, 1 << 20, alpha=1.5)
    _random_flow(integ, seed=11)
    n = 100_003                                    # ragged: not a multiple of the 256-point tile pair
    integ.flow_kernel("mma")
    ref = integ.flow_sample(17, n, 5, 0).cpu().numpy().astype(np.float64)
    integ.flow_kernel("tcgen05")
    out = integ.flow_sample(17, n, 5, 0).cpu().numpy().astype(np.float64)
    assert np.all(np.isfinite(out))
    dv = np.abs(out[:, :3] - ref[:, :3]).max(1)
    dj = np.abs(out[:, 3] - ref[:, 3])
    assert np.percentile(dv, 99.9) < 2e-3 and np.median(dv) < 1e-5, (np.median(dv), np.percentile(dv, 99.9))
    assert np.percentile(dj, 99.9) < 2e-2 and np.median(dj) < 1e-4, (np.median(dj), np.percentile(dj, 99.9))
    integ.reset_grid()


def _cpu_cotangents(it, orc, flow_out, n):
    """(w, d ln f/dx) at the flow's points from the FP64 oracle (complex step), as the GPU forms them."""
    L = orc.lib()
    cfg = orc.had_cfg()
    x = flow_out[:, :3].astype(np.float64)
    g = np.zeros((n, 7))
    out = (C.c_double * 7)()
    for i in range(n):
        L.cpo_had_weight_grad(C.byref(cfg), orc.dptr(x[i].copy()), out)
        g[i] = out[:]
    f = g[:, 0]
    w = f * np.exp(flow_out[:, 3].astype(np.float64))
    dlnf = np.where(f[:, None] > 0, g[:, 1:4] / np.where(f > 0, f, 1)[:, None], 0)
    return w, dlnf


def test_training_gradient_matches_fp64_backprop(integ, orc):
    integ.reset_grid()
    integ.integrate(4, 1 << 20, alpha=1.5)
    P = _random_flow(integ, seed=5, scale=0.05)
    B = 8192
    it_idx = 11
    g_gpu, loss_gpu = integ.flow_loss_grad(B, it_idx)
    flow_out = integ.flow_sample(0, B, it_idx, 2).cpu().numpy()
    w, dlnF = _cpu_cotangents(integ, orc, flow_out, B)
    sig = w.mean()
    loss_cpu = (w * w).mean() / sig ** 2
    assert abs(loss_gpu / loss_cpu - 1) < 2e-3, (loss_gpu, loss_cpu)
    cJ = 2 * w * w / (B * sig ** 2)
    cv = cJ[:, None] * dlnF
    u, _ = _xv(integ, integ.philox_words(integ.cfg.seed, 0, B, it_idx, 2))
    G = np.zeros(NPAR)
    orc.lib().cpo_flow_backward_batch(P.ctypes.data, B, np.ascontiguousarray(u).ctypes.data,
                                      np.ascontiguousarray(cv).ctypes.data, np.ascontiguousarray(cJ).ctypes.data,
                                      G.ctypes.data, 8)
    m = _used_mask()
    a, b = g_gpu[m].astype(np.float64), G[m]
    cos = a @ b / np.linalg.norm(a) / np.linalg.norm(b)
    rel = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert cos > 0.999 and rel < 5e-2, (cos, rel)
    assert np.all(g_gpu[~m] == 0)
    integ.reset_grid()


def test_tcgen05_weight_gradients_match_mma_sync(integ):
    """The training step's weight and bias gradients from the tcgen05 GEMMs (TMEM accumulators,
    MN-major shared-memory operands) equal those of the warp-level mma.sync GEMMs on the same
    activations and output gradients, up to FP32 summation order: the same BF16 products, FP32
    accumulation, block slots added in the same order."""
    integ.reset_grid()
    integ.integrate(4, 1 << 20, alpha=1.5)
    _random_flow(integ, seed=9, scale=0.05)
    m = _used_mask()
    for batch in (65536, 65536 - 96, 4096):
        integ.flow_kernel("tcgen05")
        g_tc, l_tc = integ.flow_loss_grad(batch, 17)
        integ.flow_kernel("mma")
        g_mma, l_mma = integ.flow_loss_grad(batch, 17)
        integ.flow_kernel("tcgen05")
        assert l_tc == l_mma
        a, b = g_tc[m].astype(np.float64), g_mma[m].astype(np.float64)
        assert np.all(g_tc[~m] == 0)
        assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b), (batch, np.linalg.norm(a - b) / np.linalg.norm(b))
        big = np.abs(b) > 1e-3 * np.abs(b).max()
        assert np.max(np.abs(a[big] - b[big]) / np.abs(b[big])) < 1e-3, batch
    integ.reset_grid()


def test_training_lowers_the_weight_variance():
    import cupythia_b200 as cp
    n = 1 << 22
    with cp.Integrator() as it:
        it.integrate(8, 1 << 22, alpha=1.5)
        base = it.iteration(n, 500, alpha=0.0)
        it.flow_init(7)
        loss = it.flow_train(120, 65536, lr=1e-3)
        it.flow_enable(True)
        flow = it.iteration(n, 500, alpha=0.0)
        it.flow_enable(False)
    assert np.all(np.isfinite(loss))
    assert loss[-10:].mean() < loss[:5].mean()
    rv_base = (base["sigma_err"] / base["sigma"]) ** 2
    rv_flow = (flow["sigma_err"] / flow["sigma"]) ** 2
    print("relative variance VEGAS %.3e  flow+VEGAS %.3e  loss %.4f -> %.4f" % (rv_base, rv_flow, loss[0], loss[-1]))
    assert rv_flow < rv_base
    assert abs(flow["sigma"] - base["sigma"]) < 5 * np.hypot(flow["sigma_err"], base["sigma_err"])


def test_training_is_reproducible():
    """Two trainings from the same initialisation on the same grid end with bit-identical
    parameters and losses: every reduction of the training step (batch moments, weight and bias
    gradients) sums in a fixed order."""
    import cupythia_b200 as cp
    runs = []
    for _ in range(2):
        with cp.Integrator() as it:
            it.integrate(3, 1 << 20, alpha=1.5)
            it.flow_init(7)
            loss = it.flow_train(10, 65536, lr=8e-3)
            runs.append((it.flow_params.copy(), np.asarray(loss).copy()))
    assert np.array_equal(runs[0][1], runs[1][1])
    assert np.array_equal(runs[0][0], runs[1][0])


def test_training_resumes_from_a_checkpoint_bit_for_bit():
    """A training interrupted after k updates, checkpointed (parameters, Adam moments, update
    count), restored into a fresh handle on the same grid and trained for m more updates ends
    with the parameters and losses of k + m uninterrupted updates, bit for bit."""
    import cupythia_b200 as cp
    k, m = 12, 9
    with cp.Integrator() as it:
        it.integrate(3, 1 << 20, alpha=1.5)
        grid = it.grid
        it.flow_init(7)
        loss_all = np.asarray(it.flow_train(k + m, 65536, lr=8e-3)).copy()
        p_all = it.flow_params.copy()
    with cp.Integrator() as it:
        it.grid = grid
        it.flow_init(7)
        loss_a = np.asarray(it.flow_train(k, 65536, lr=8e-3)).copy()
        state, updates = it.flow_state()
    assert updates == k and state.size == 3 * p_all.size
    with cp.Integrator() as it:
        it.grid = grid
        it.flow_restore(state, updates)
        assert np.array_equal(it.flow_params, state[:p_all.size])
        loss_b = np.asarray(it.flow_train(m, 65536, lr=8e-3)).copy()
        again, n_up = it.flow_state()
        assert n_up == k + m
        assert np.array_equal(np.concatenate([loss_a, loss_b]), loss_all)
        assert np.array_equal(it.flow_params, p_all)


def test_expired_tensor_core_wait_is_reported_and_recoverable(integ):
    """Failure detection without a GPU fault: the test hook stops MMA issue, so the epilogue's
    bounded waits expire (about 1 s); the call must return CP_ERR_TIMEOUT (4), and the next call
    on the same handle must succeed with the normal result."""
    import cupythia_b200 as cp
    integ.reset_grid()
    integ.flow_init(7)
    integ.flow_kernel("tcgen05")
    ref = integ.flow_sample(0, 4096, 3, 0).cpu().numpy()
    integ.lib.cp_flow_test_stall(integ.h, 1)
    try:
        with pytest.raises(cp.CpError) as e:
            integ.flow_sample(0, 4096, 3, 0)
        assert e.value.code == 4
    finally:
        integ.lib.cp_flow_test_stall(integ.h, 0)
    again = integ.flow_sample(0, 4096, 3, 0).cpu().numpy()
    assert np.array_equal(again, ref)


def test_fused_production_matches_forward_then_accept():
    """The flow form's production pass as one tcgen05 kernel per chunk (flow forward, integrand and
    accept step, the flow output never stored) gives the records of the forward-then-accept path
    byte for byte, with the same counts, over a pass of two staging chunks (the second ragged),
    with scale weights, and through the host-delivery call; the sums of w differ only by their
    addition order (relative 1e-6)."""
    import torch

    import cupythia_b200 as cp
    n = (1 << 24) + 4099
    with cp.Integrator() as it:
        it.integrate(4, 1 << 20, alpha=1.5)
        it.flow_init(7)
        it.flow_train(20, 65536, lr=8e-3)
        it.flow_enable(True)
        it.iteration(1 << 20, 70, alpha=0.0)
        it.weight_quantile(0.999)
        got = {}
        for fused in (True, False):
            it.flow_fuse_production(fused)
            rec, st = it.unweight(n, iteration=71)
            r2, sw, st2 = it.unweight_scale_weights(1 << 20, iteration=72)
            host = torch.empty((st["n_accepted"] + 8, 64), dtype=torch.uint8, pin_memory=True)
            st3 = it.generate_host(n, host, iteration=71, chunk=3 * (1 << 22) + 1)
            got[fused] = (cp.events_view(rec).tobytes(), st, cp.events_view(r2).tobytes(), sw.cpu().numpy(), st2,
                          cp.events_view(host[:st3["n_accepted"]]).tobytes(), st3)
        it.flow_fuse_production(False)
    a, b = got[True], got[False]
    assert a[1]["n_accepted"] > 1000 and a[1]["n_bad"] == 0
    for k in ("n_accepted", "n_overweight", "n_bad", "n_points"):
        assert a[1][k] == b[1][k] and a[4][k] == b[4][k] and a[6][k] == b[6][k], k
    assert a[0] == b[0]
    assert a[2] == b[2] and np.array_equal(a[3], b[3])
    assert a[5] == a[0] and b[5] == b[0]
    for st_a, st_b in ((a[1], b[1]), (a[4], b[4]), (a[6], b[6])):
        for k in ("sigma", "sigma_err", "sigma_unweighted", "w_max_seen"):
            assert st_a[k] == pytest.approx(st_b[k], rel=1e-6), k


def test_expired_wait_in_fused_production_is_reported_and_recoverable():
    """Failure detection of the fused production kernel without a GPU fault: with MMA issue
    stopped by the test hook, its bounded waits expire, cp_unweight returns CP_ERR_TIMEOUT (4),
    and the next pass on the same handle returns the records of an undisturbed pass."""
    import cupythia_b200 as cp
    with cp.Integrator() as it:
        it.integrate(2, 1 << 18, alpha=1.5)
        it.flow_init(7)
        it.flow_enable(True)
        it.flow_fuse_production(True)
        it.iteration(1 << 18, 80, alpha=0.0)
        it.weight_quantile(0.999)
        rec, st = it.unweight(1 << 18, iteration=81)
        ref = cp.events_view(rec).tobytes()
        it.lib.cp_flow_test_stall(it.h, 1)
        try:
            with pytest.raises(cp.CpError) as e:
                it.unweight(1 << 18, iteration=81)
            assert e.value.code == 4
        finally:
            it.lib.cp_flow_test_stall(it.h, 0)
        rec2, st2 = it.unweight(1 << 18, iteration=81)
        assert st2["n_accepted"] == st["n_accepted"]
        assert cp.events_view(rec2).tobytes() == ref


def test_diverged_flow_is_reported_as_numeric_fault():
    """A flow with non-finite parameters (what a diverged training leaves) makes the next pass report
    CP_ERR_NUMERIC (3) with the bad weights zeroed and counted; with the flow switched off the
    same handle integrates normally again (VEGAS is the fallback)."""
    import cupythia_b200 as cp
    with cp.Integrator() as it:
        it.integrate(3, 1 << 20, alpha=1.5)
        it.flow_init(7)
        it.flow_params = np.where(_used_mask(), np.float32(np.nan), np.float32(0))
        it.flow_enable(True)
        with pytest.raises(cp.CpError) as e:
            it.iteration(1 << 20, 40, alpha=0.0)
        assert e.value.code == 3
        it.flow_enable(False)
        r = it.iteration(1 << 20, 41, alpha=0.0)
        assert r["n_bad"] == 0 and np.isfinite(r["sigma"]) and r["sigma"] > 0

