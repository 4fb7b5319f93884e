"""The allocation-free VEGAS pass (cp_vegas_pass_noalloc) against the handle's pass.

Some callers cannot allocate device memory (a host program that owns every device allocation, a
process under a fixed memory budget, a plugin inside another program's event loop);
cp_vegas_pass_noalloc serves them from a file-scope device array.  Its sums and histograms must equal those of
cp_vegas_iteration on the same grid and counter iteration, on consecutive calls (the array keeps
the previous call's contents, so a second call checks that nothing leaks between calls).
Collected last on purpose: a run that stops at the first failure has run everything else first.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-12   # same kernel, same launch shape: equal up to FP64 reduction rounding


def test_noalloc_pass_matches_handle_pass_on_consecutive_calls():
    import torch

    import cupythia_b200 as cp
    lib = cp._lib.load()
    n = 1 << 20
    with cp.Integrator() as it:
        it.integrate(3, n, alpha=1.5)
        grid = it.grid
        nb = it.nb
        edges = torch.tensor(grid.reshape(-1), dtype=torch.float64, device="cuda:0")
        for iteration in (7, 8):
            out = torch.full((4 + 3 * nb,), -1.0, dtype=torch.float64, device="cuda:0")
            rc = lib.cp_vegas_pass_noalloc(C.byref(it.cfg), n, iteration, C.c_void_p(edges.data_ptr()),
                                           C.c_void_p(out.data_ptr()), None)
            assert rc == 0
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            r = it.iteration(n, iteration, alpha=0.0)          # the handle's pass, grid unchanged
            ref = it.last_histogram()
            assert np.array_equal(it.grid, grid)
            assert abs(got[0] / ref["sum_w"] - 1) < REL and abs(got[1] / ref["sum_w2"] - 1) < REL
            assert got[2] == ref["w_max"] and got[3] == ref["n_bad"] == 0
            assert np.allclose(got[4:].reshape(3, nb), ref["hist"], rtol=REL, atol=0)
            assert abs(got[0] / n - r["sigma"]) < REL * r["sigma"]


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    import cupythia_b200 as cp
    lib = cp._lib.load()
    cfg = cp.default_config(n_bins=cp._lib.CP_MAX_BINS + 1)
    edges = torch.zeros(3 * (cfg.n_bins + 1), dtype=torch.float64, device="cuda:0")
    out = torch.zeros(4 + 3 * cfg.n_bins, dtype=torch.float64, device="cuda:0")
    rc = lib.cp_vegas_pass_noalloc(C.byref(cfg), 1 << 10, 0, C.c_void_p(edges.data_ptr()),
                                   C.c_void_p(out.data_ptr()), None)
    assert rc == cp._lib.CP_ERR_INVALID
