"""Edge cases of the GPU path through the C ABI: empty, tiny and ragged sizes (not multiples of
a warp, block, tile or chunk), the largest and smallest grids, 64-bit seeds and point indices,
and the size limits, each checked against the oracle or against the regular-size path."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def test_empty_batches_are_no_ops(integ):
    import torch
    assert integ.philox_words(42, 0, 0).shape == (0, 4)
    from cupythia_b200.sigma import Sigma2qg2qg
    sp = Sigma2qg2qg(integrator=integ)
    sp.set2Kin([], [], [], [])
    assert sp.sigmaPDF().numel() == 0 and sp.sigmaKin().numel() == 0
    integ.flow_init(7)
    out = torch.empty((1, 4), dtype=torch.float32, device="cuda")
    import ctypes as C
    assert integ.lib.cp_flow_sample(integ.h, 0, 0, 0, 0, C.c_void_p(out.data_ptr())) == 0


def test_64_bit_seeds_and_point_indices_are_bit_exact(integ):
    for seed, p0 in [(2 ** 40 + 5, 0), (42, 2 ** 33 + 7), (2 ** 64 - 1, 2 ** 63)]:
        got = integ.philox_words(seed, p0, 37, 3, 1)
        ref = oracle.point_words(seed, [p0 + i for i in range(37)], 3, 1)
        assert np.array_equal(got, ref), (seed, p0)


@pytest.mark.parametrize("n_bins", [2, 128])
def test_smallest_and_largest_grids(n_bins):
    """Point weights on an adapted grid of n_bins bins per dimension against the FP64 oracle."""
    import cupythia_b200 as cp
    with cp.Integrator(n_bins=n_bins) as it:
        it.integrate(3, 1 << 20, alpha=1.5)
        n = 4097                                   # ragged
        w, x = it.point_weights(5, n, 9, with_x=True)
        grid = it.grid
        words = it.philox_words(it.cfg.seed, 5, n, 9, 0)
    m = (words[:, :3] >> 8).astype(np.uint64) * n_bins
    b = (m >> 24).astype(np.int64)
    jv = np.prod([n_bins * (grid[d][b[:, d] + 1] - grid[d][b[:, d]]).astype(np.float32) for d in range(3)], 0)
    ref = oracle.weight_x_batch(oracle.had_cfg(), x.cpu().numpy()) * jv
    w = w.cpu().numpy().astype(np.float64)
    keep = ref > 1e-12 * ref.mean()
    assert np.max(np.abs(w[keep] - ref[keep]) / ref[keep]) < 1e-5


def test_ragged_production_matches_its_recount():
    """A production pass of a prime number of points: every record is a distinct accepted point
    and the count equals the recount u w_max < w on the same FP32 weights."""
    import cupythia_b200 as cp
    n = 1000003
    with cp.Integrator() as it:
        it.integrate(4, 1 << 20, alpha=1.5)
        it.iteration(1 << 20, 30, alpha=0.0)
        wq = it.weight_quantile(0.999)
        rec, st = it.unweight(n, iteration=31)
        w = it.point_weights(0, n, 31).cpu().numpy()
        words = it.philox_words(it.cfg.seed, 0, n, 31, 0)
    ev = cp.events_view(rec)
    u = (words[:, 3] >> 8).astype(np.float32) * np.float32(1.0 / 16777216.0)
    expect = np.nonzero(u * np.float32(wq) < w)[0]
    pts = ev["point"].astype(np.int64)
    assert np.all(np.diff(pts) > 0)   # point order
    assert len(pts) == st["n_accepted"]
    assert pts.max() < n
    assert len(np.setxor1d(expect, pts)) <= 2


def test_ragged_host_chunks_match_the_device_pass():
    import torch

    import cupythia_b200 as cp
    n = 300007
    with cp.Integrator() as it:
        it.integrate(4, 1 << 20, alpha=1.5)
        it.iteration(1 << 20, 32, alpha=0.0)
        it.weight_quantile(0.999)
        rec, st = it.unweight(n, iteration=33)
        host = torch.empty((st["n_accepted"] + 8, 64), dtype=torch.uint8, pin_memory=True)
        st2 = it.generate_host(n, host, iteration=33, chunk=65537)   # does not divide n
    assert st2["n_accepted"] == st["n_accepted"]
    a = cp.events_view(rec)
    b = cp.events_view(host[:st2["n_accepted"]])
    assert a.tobytes() == b.tobytes()   # the same records in the same (point) order


def test_tiny_passes_and_size_limits(integ):
    import ctypes as C

    import torch

    import cupythia_b200 as cp
    r = integ.iteration(2, 40, alpha=0.0)
    assert r["n_points"] == 2
    integ.weight_quantile(0.999)
    rec, st = integ.unweight(2, iteration=41)
    assert st["n_points"] == 2 and st["n_accepted"] <= 2
    # more than 2^32 points in one production call is refused before any launch
    res = cp._lib.cp_unweight_result()
    recs = torch.empty((1, 64), dtype=torch.uint8, device="cuda")
    rc = integ.lib.cp_unweight(integ.h, (1 << 32) + 1, 0, C.c_void_p(recs.data_ptr()), 1, C.byref(res))
    assert rc == cp._lib.CP_ERR_INVALID
    # a misaligned record buffer is refused
    rc = integ.lib.cp_unweight(integ.h, 1024, 0, C.c_void_p(recs.data_ptr() + 4), 1, C.byref(res))
    assert rc == cp._lib.CP_ERR_INVALID
    # a production pass needs a threshold (cp_weight_quantile or cp_set_wmax); cp_set_wmax sets it
    with cp.Integrator() as fresh:
        rc = fresh.lib.cp_unweight(fresh.h, 1024, 0, C.c_void_p(recs.data_ptr()), 1, C.byref(res))
        assert rc == cp._lib.CP_ERR_INVALID
        hrec = torch.empty((1, 64), dtype=torch.uint8, pin_memory=True)
        rc = fresh.lib.cp_generate_host(fresh.h, 1024, 0, 512, C.c_void_p(hrec.data_ptr()), 1, C.byref(res))
        assert rc == cp._lib.CP_ERR_INVALID
        fresh.set_wmax(1e30)   # nothing is accepted against an unreachable threshold
        _, st0 = fresh.unweight(1024, iteration=42)
        assert st0["n_accepted"] == 0 and st0["w_max"] == 1e30
    # the flow forward of a single point (far below one 128-point tile)
    integ.flow_init(7)
    out = integ.flow_sample(11, 1, 3, 0).cpu().numpy()
    assert np.all(np.isfinite(out)) and np.all((out[0, :3] > 0) & (out[0, :3] < 1))


def test_host_generation_capacity_and_staging_reuse():
    """The host-delivery call (three staging buffers kept in the handle, counts through mapped
    pinned memory): with a record buffer smaller than the accepted count it fills the buffer with
    real records and reports CP_ERR_CAPACITY; afterwards the handle still works, and calls that
    grow and then shrink the chunk, with VEGAS and with the flow as proposal, deliver exactly the
    device pass's records."""
    import ctypes as C

    import torch

    import cupythia_b200 as cp
    n = 200003
    with cp.Integrator() as it:
        it.integrate(4, 1 << 20, alpha=1.5)
        it.iteration(1 << 20, 50, alpha=0.0)
        it.weight_quantile(0.999)
        rec, st = it.unweight(n, iteration=51)
        dev = cp.events_view(rec)
        k = st["n_accepted"]
        small = torch.zeros((k // 3, 64), dtype=torch.uint8, pin_memory=True)
        res = cp._lib.cp_unweight_result()
        rc = it.lib.cp_generate_host(it.h, n, 51, 1 << 14, C.c_void_p(small.data_ptr()), small.shape[0], C.byref(res))
        assert rc == cp._lib.CP_ERR_CAPACITY and res.n_accepted == k
        got = cp.events_view(small)
        assert got.tobytes() == dev[:len(got)].tobytes()   # the first records in point order
        full = torch.empty((k + 8, 64), dtype=torch.uint8, pin_memory=True)
        for chunk in (1 << 17, 1 << 12, 100001):
            full.zero_()
            st2 = it.generate_host(n, full, iteration=51, chunk=chunk)
            assert st2["n_accepted"] == k
            h = cp.events_view(full[:k])
            assert dev.tobytes() == h.tobytes(), chunk
        # the flow as proposal: its forward pass runs per chunk on the same handle
        it.flow_init(7)
        it.flow_train(10, 65536, lr=8e-3)
        it.flow_enable(True)
        it.iteration(1 << 20, 52, alpha=0.0)
        it.weight_quantile(0.999)
        rec_f, st_f = it.unweight(n, iteration=53)
        host_f = torch.empty((st_f["n_accepted"] + 8, 64), dtype=torch.uint8, pin_memory=True)
        st3 = it.generate_host(n, host_f, iteration=53, chunk=50000)
        it.flow_enable(False)
    assert st3["n_accepted"] == st_f["n_accepted"]
    a = cp.events_view(rec_f)
    b = cp.events_view(host_f[:st3["n_accepted"]])
    assert a.tobytes() == b.tobytes()


def test_pass_across_staging_chunks_is_one_pass():
    """A production pass of 2^24 + 4099 points runs as two staging chunks (the second ragged): its
    records are the accepted points of the whole pass in strictly increasing point order, their
    count is the recount u w_max < w, and the host-delivery call with chunks that divide neither
    the pass nor 2^24 delivers the same bytes; with the flow as proposal (one forward pass for the
    whole call, read chunk by chunk) the two calls agree as well."""
    import torch

    import cupythia_b200 as cp
    n = (1 << 24) + 4099
    with cp.Integrator() as it:
        it.integrate(4, 1 << 20, alpha=1.5)
        it.iteration(1 << 20, 60, alpha=0.0)
        wq = it.weight_quantile(0.999)
        rec, st = it.unweight(n, iteration=61)
        w = it.point_weights(0, n, 61).cpu().numpy()
        u = (it.philox_words(it.cfg.seed, 0, n, 61, 0)[:, 3] >> 8).astype(np.float32) * np.float32(1.0 / 16777216.0)
        ev = cp.events_view(rec)
        pts = ev["point"].astype(np.int64)
        assert np.all(np.diff(pts) > 0) and pts.max() < n
        assert len(pts) == st["n_accepted"]
        assert (pts >= 1 << 24).any()                     # the second chunk delivered records
        expect = np.nonzero(u * np.float32(wq) < w)[0]
        assert len(np.setxor1d(expect, pts)) <= 2
        host = torch.empty((st["n_accepted"] + 8, 64), dtype=torch.uint8, pin_memory=True)
        st2 = it.generate_host(n, host, iteration=61, chunk=3 * (1 << 22) + 1)
        assert st2["n_accepted"] == st["n_accepted"]
        assert cp.events_view(host[:st2["n_accepted"]]).tobytes() == ev.tobytes()
        it.flow_init(7)
        it.flow_train(10, 65536, lr=8e-3)
        it.flow_enable(True)
        it.iteration(1 << 20, 62, alpha=0.0)
        it.weight_quantile(0.999)
        rec_f, st_f = it.unweight(n, iteration=63)
        host_f = torch.empty((st_f["n_accepted"] + 8, 64), dtype=torch.uint8, pin_memory=True)
        st3 = it.generate_host(n, host_f, iteration=63, chunk=5000011)
        it.flow_enable(False)
    a = cp.events_view(rec_f)
    pf = a["point"].astype(np.int64)
    assert np.all(np.diff(pf) > 0) and (pf >= 1 << 24).any()
    assert st3["n_accepted"] == st_f["n_accepted"]
    assert cp.events_view(host_f[:st3["n_accepted"]]).tobytes() == a.tobytes()
