"""cupythia_b200 -- B200-native (sm_100a) batched QCD 2->2 hard-process Monte-Carlo integrator.

Host-side mirror of the reference's interfaces for this path:
  * :class:`Integrator` -- the stage-driver surface (fused partonic MC, VEGAS iterations,
    unweighting, adjoint, flow), one CUDA handle of the C ABI (include/cupythia_b200.h);
  * :mod:`cupythia_b200.sigma` -- Pythia's ``SigmaProcess`` surface (set2Kin / sigmaKin /
    sigmaHat / sigmaPDF) over batches.
Device buffers are torch CUDA tensors; torch is only the allocator here, every number is
computed by the library's own kernels.
"""
import ctypes as C
import os

import numpy as np

from . import _lib
from ._lib import (CP_PROC_ALL, CP_PROC_GG2GG, CP_PROC_GG2QQBAR, CP_PROC_QG2QG,  # noqa: F401
                   CP_PROC_QQ2QQ, CP_PROC_QQBAR2GG, CpError, cp_config, cp_event, cp_grad,
                   cp_result, cp_unweight_result)

__all__ = ["Integrator", "CpError", "default_config", "CP_PROC_ALL", "events_view", "colour_tags", "write_lhef"]


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise CpError(_lib.CP_ERR_CUDA, "no CUDA device available")
    return torch


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def default_config(**overrides):
    lib = _lib.load()
    cfg = cp_config()
    lib.cp_config_default(C.byref(cfg))
    for k, v in overrides.items():
        if not hasattr(cfg, k):
            raise KeyError(f"unknown config field {k}")
        setattr(cfg, k, v)
    return cfg


class Integrator:
    """One handle of the CUDA integrator (pp -> 2 jets at 13 TeV by default)."""

    def __init__(self, **cfg):
        self.lib = _lib.load()
        self.cfg = default_config(**cfg)
        h = C.c_void_p()
        rc = self.lib.cp_create(C.byref(self.cfg), C.byref(h))
        if rc != 0:
            raise CpError(rc, "cp_create failed (no device, bad configuration or out of memory)")
        self.h = h
        self.nb = self.cfg.n_bins
        self.device = f"cuda:{self.cfg.device}"

    # ------------------------------------------------------------------ lifecycle
    def close(self):
        if getattr(self, "h", None):
            self.lib.cp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        return _lib.check(self.lib, self.h, rc)

    def set_point_offset(self, offset):
        """Shard offset added to every pass's point indices (cp_set_point_offset)."""
        self._check(self.lib.cp_set_point_offset(self.h, int(offset)))

    def set_stream(self, stream):
        self._check(self.lib.cp_set_stream(self.h, C.c_void_p(stream)))

    def measure_peaks(self):
        """(FP32 TFLOP/s, MUFU Tops/s) of the device from the library's microbenchmarks."""
        f, m = C.c_double(), C.c_double()
        self._check(self.lib.cp_measure_peaks(self.h, C.byref(f), C.byref(m)))
        return f.value, m.value

    def set_kernel_timing(self, on=True):
        self._check(self.lib.cp_set_kernel_timing(self.h, 1 if on else 0))

    def kernel_times(self, reset=True):
        """{kernel: (total ms, launches)} of the production pass since the last reset."""
        ms = np.zeros(3)
        n = np.zeros(3, np.uint64)
        self._check(self.lib.cp_kernel_times(self.h, ms.ctypes.data_as(C.c_void_p), n.ctypes.data_as(C.c_void_p),
                                             1 if reset else 0))
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(["flow_forward", "accept", "build"])}

    def sm_count(self):
        n = C.c_int()
        self._check(self.lib.cp_device_sm_count(self.h, C.byref(n)))
        return n.value

    # ------------------------------------------------------------------ RNG surface
    def philox_words(self, seed, point0, n, iteration=0, stream=0):
        torch = _torch()
        out = torch.empty((n, 4), dtype=torch.int32, device=self.device)
        self._check(self.lib.cp_philox_words(self.h, seed, point0, n, iteration, stream, _ptr(out)))
        return out.cpu().numpy().view(np.uint32)

    def splitmix_uniforms(self, seed, n_threads, k_per):
        torch = _torch()
        out = torch.empty(n_threads * k_per, dtype=torch.float64, device=self.device)
        self._check(self.lib.cp_splitmix_uniforms(self.h, seed, n_threads, k_per, _ptr(out)))
        return out.cpu().numpy()

    def event_keys(self, base, e0, n):
        torch = _torch()
        out = torch.empty(n, dtype=torch.int64, device=self.device)
        self._check(self.lib.cp_event_keys(self.h, base, e0, n, _ptr(out)))
        return out.cpu().numpy().view(np.uint64)

    # ------------------------------------------------------------------ PDFs
    def pdf(self, x, q2):
        """CTEQ5L x f for ids -5..-1, 1..5, 21 at (x, Q2); returns (n, 11) float32."""
        torch = _torch()
        x = torch.as_tensor(np.asarray(x, np.float32), device=self.device)
        q2 = torch.as_tensor(np.asarray(q2, np.float32), device=self.device)
        out = torch.empty((x.numel(), 11), dtype=torch.float32, device=self.device)
        self._check(self.lib.cp_pdf_batch(self.h, _ptr(x), _ptr(q2), x.numel(), _ptr(out)))
        return out.cpu().numpy()

    # ------------------------------------------------------------------ VEGAS grid
    @property
    def grid(self):
        e = (C.c_double * (3 * (self.nb + 1)))()
        self._check(self.lib.cp_grid_get(self.h, e))
        return np.array(e[:]).reshape(3, self.nb + 1)

    @grid.setter
    def grid(self, edges):
        e = np.ascontiguousarray(np.asarray(edges, np.float64).reshape(-1))
        self._check(self.lib.cp_grid_set(self.h, e.ctypes.data_as(C.POINTER(C.c_double))))

    def reset_grid(self):
        self._check(self.lib.cp_grid_reset(self.h))

    def iteration(self, n_points, iteration=0, alpha=1.5):
        r = cp_result()
        self._check(self.lib.cp_vegas_iteration(self.h, n_points, iteration, alpha, C.byref(r)))
        return r.as_dict()

    def integrate(self, n_iter, n_points, alpha=1.5, skip=0):
        per = (cp_result * n_iter)()
        comb = cp_result()
        self._check(self.lib.cp_integrate(self.h, n_iter, n_points, alpha, skip, per, C.byref(comb)))
        return [p.as_dict() for p in per], comb.as_dict()

    # ------------------------------------------------------------------ multi-GPU pieces
    def accumulate(self, n_points, iteration=0):
        """One pass over this handle's points; returns its sums as a device float64 tensor of
        CP_SLOT_HEAD + 3 n_bins entries (sum w, sum w^2, max w, n_bad, per-bin sums of w^2)."""
        torch = _torch()
        out = torch.empty(_lib.CP_SLOT_HEAD + 3 * self.nb, dtype=torch.float64, device=self.device)
        self._check(self.lib.cp_vegas_accumulate(self.h, n_points, iteration, _ptr(out)))
        return out

    def refine(self, sums, n_total, alpha=1.5):
        """Iteration result and grid refinement from (rank-reduced) sums."""
        r = cp_result()
        self._check(self.lib.cp_vegas_refine_sums(self.h, _ptr(sums), float(n_total), alpha, C.byref(r)))
        return r.as_dict()

    def weight_histogram(self):
        torch = _torch()
        out = torch.empty(_lib.CP_QBINS, dtype=torch.int64, device=self.device)
        self._check(self.lib.cp_weight_histogram(self.h, _ptr(out)))
        return out

    def quantile_from_histogram(self, hist, q=0.999):
        v = C.c_double()
        self._check(self.lib.cp_weight_quantile_hist(self.h, _ptr(hist), q, C.byref(v)))
        return v.value

    def point_weights(self, point0, n, iteration=0, with_x=False):
        torch = _torch()
        w = torch.empty(n, dtype=torch.float32, device=self.device)
        x = torch.empty((n, 3), dtype=torch.float32, device=self.device) if with_x else None
        self._check(self.lib.cp_point_weights(self.h, point0, n, iteration, _ptr(w),
                                              _ptr(x) if with_x else None))
        return (w, x) if with_x else w

    def weight_at(self, x):
        torch = _torch()
        x = torch.as_tensor(np.asarray(x, np.float32).reshape(-1, 3), device=self.device).contiguous()
        w = torch.empty(x.shape[0], dtype=torch.float32, device=self.device)
        self._check(self.lib.cp_weight_at(self.h, _ptr(x), x.shape[0], _ptr(w)))
        return w

    def last_histogram(self):
        out = (C.c_double * (4 + 3 * self.nb))()
        self._check(self.lib.cp_last_histogram(self.h, out))
        a = np.array(out[:])
        return {"sum_w": a[0], "sum_w2": a[1], "w_max": a[2], "n_bad": a[3],
                "hist": a[4:].reshape(3, self.nb)}

    # ------------------------------------------------------------------ adjoint
    def adjoint(self, n_points, iteration=0, stream=0):
        """Gradients of sigma and Var[w] (see cp_adjoint); edge gradients as (3, nb+1) arrays."""
        g = cp_grad()
        ne = 3 * (self.nb + 1)
        ds = np.zeros(ne)
        dv = np.zeros(ne)
        self._check(self.lib.cp_adjoint(self.h, n_points, iteration, stream, C.byref(g),
                                        ds.ctypes.data_as(C.c_void_p), dv.ctypes.data_as(C.c_void_p)))
        return {"sigma": g.sigma, "var": g.var, "dsigma": list(g.dsigma), "dvar": list(g.dvar),
                "params": ["alphas_mz", "k_ren", "pt_hat_min"], "n_bad": g.n_bad,
                "dsigma_dedges": ds.reshape(3, -1), "dvar_dedges": dv.reshape(3, -1)}

    def adapt_gradient(self, steps, n_points, lr=0.4, iteration0=0):
        """Variance-gradient adaptation: `steps` device gradient steps, halving lr whenever the
        batch variance (measured at the pre-step grid of each step) rises. Returns the history."""
        return adapt_gradient_loop(self.gradient_step, steps, n_points, lr, iteration0)

    def gradient_objective(self, p=2.0):
        """Moment order of the adjoint passes: <w^p>/<w>^p instead of the variance (p = 2)."""
        self._check(self.lib.cp_vegas_gradient_objective(self.h, float(p)))

    def adjoint_parameter_tangents(self, on=True):
        """Adjoint passes with or without the alpha_s(mZ), k_ren and pT-cut tangents; without
        them the edge gradients and grid steps are the same bit for bit and the passes faster."""
        self._check(self.lib.cp_adjoint_parameter_tangents(self.h, 1 if on else 0))

    def gradient_step(self, n_points, iteration=0, lr=0.5):
        g = cp_grad()
        self._check(self.lib.cp_vegas_gradient_step(self.h, n_points, iteration, lr, C.byref(g)))
        return {"sigma": g.sigma, "var": g.var}

    def adjoint_accumulate(self, n_points, iteration=0, stream=0):
        """Adjoint sums of this handle's points as a device float64 tensor (entry 8 reduces by max
        over ranks, every other entry by sum)."""
        torch = _torch()
        k = C.c_int()
        self._check(self.lib.cp_adjoint_sums_size(self.h, C.byref(k)))
        out = torch.empty(k.value, dtype=torch.float64, device=self.device)
        self._check(self.lib.cp_adjoint_accumulate(self.h, n_points, iteration, stream, _ptr(out)))
        return out

    def gradient_apply(self, sums, n_total, lr=0.5):
        """Gradient record of n_total points from (rank-reduced) adjoint sums; lr > 0 also takes
        the variance-gradient step on the grid."""
        g = cp_grad()
        self._check(self.lib.cp_vegas_gradient_apply(self.h, _ptr(sums), int(n_total), lr, C.byref(g)))
        return {"sigma": g.sigma, "var": g.var}

    # ------------------------------------------------------------------ learned proposal
    def flow_init(self, seed=7):
        self._check(self.lib.cp_flow_init(self.h, seed))

    @property
    def flow_params(self):
        n = self.lib.cp_flow_num_params()
        out = np.zeros(n, np.float32)
        self._check(self.lib.cp_flow_get_params(self.h, out.ctypes.data_as(C.c_void_p), n))
        return out

    @flow_params.setter
    def flow_params(self, p):
        p = np.ascontiguousarray(np.asarray(p, np.float32))
        self._check(self.lib.cp_flow_set_params(self.h, p.ctypes.data_as(C.c_void_p), p.size))

    def flow_state(self):
        """Training checkpoint: (FP32 master parameters + Adam moments, updates taken)."""
        n = self.lib.cp_flow_state_size()
        out = np.zeros(n, np.float32)
        k = C.c_int64()
        self._check(self.lib.cp_flow_get_state(self.h, out.ctypes.data_as(C.c_void_p), n, C.byref(k)))
        return out, k.value

    def flow_restore(self, state, updates):
        """Resumes training from a flow_state() checkpoint."""
        state = np.ascontiguousarray(np.asarray(state, np.float32))
        self._check(self.lib.cp_flow_set_state(self.h, state.ctypes.data_as(C.c_void_p), state.size, int(updates)))

    def flow_sample(self, point0, n, iteration=0, stream=0):
        torch = _torch()
        out = torch.empty((n, 4), dtype=torch.float32, device=self.device)
        self._check(self.lib.cp_flow_sample(self.h, point0, n, iteration, stream, _ptr(out)))
        return out

    def flow_enable(self, on=True):
        self._check(self.lib.cp_flow_enable(self.h, 1 if on else 0))

    def flow_kernel(self, which):
        """Forward kernel: "tcgen05" (TMEM accumulators, default) or "mma" (warp-level mma.sync)."""
        self._check(self.lib.cp_flow_select_kernel(self.h, {"tcgen05": 0, "mma": 1}[which]))

    def flow_fuse_production(self, on=True):
        """Production passes in the flow form: flow forward, integrand and accept step in one
        tcgen05 kernel (on), or the forward over the pass followed by the accept kernel (off, the
        default and the faster of the two)."""
        self._check(self.lib.cp_flow_fuse_production(self.h, 1 if on else 0))

    def flow_objective(self, p=2.0):
        """Training objective <w^p>/<w>^p (p = 2: the weight variance)."""
        self._check(self.lib.cp_flow_set_objective(self.h, float(p)))

    def flow_train(self, steps, batch=65536, lr=1e-3):
        loss = np.zeros(steps)
        self._check(self.lib.cp_flow_train(self.h, steps, batch, lr, loss.ctypes.data_as(C.c_void_p)))
        return loss

    def flow_step_moments(self, point0, count):
        """Phase 1 of a data-parallel training step: (sum w, sum w^2) of the batch points
        [point0, point0 + count) as a device float64 tensor."""
        torch = _torch()
        out = torch.empty(2, dtype=torch.float64, device=self.device)
        self._check(self.lib.cp_flow_step_moments(self.h, point0, count, _ptr(out)))
        return out

    def flow_step_gradient(self, moments, batch_total):
        """Phase 2: these points' part of the batch-loss gradient (device float32 tensor) from the
        rank-summed moments, and the batch loss."""
        torch = _torch()
        g = torch.empty(self.lib.cp_flow_num_params(), dtype=torch.float32, device=self.device)
        loss = C.c_double()
        self._check(self.lib.cp_flow_step_gradient(self.h, _ptr(moments), int(batch_total), _ptr(g), C.byref(loss)))
        return g, loss.value

    def flow_step_update(self, grad, lr):
        """Phase 3: Adam step with the rank-summed gradient."""
        self._check(self.lib.cp_flow_step_update(self.h, _ptr(grad), lr))

    def flow_loss_grad(self, batch, iteration):
        n = self.lib.cp_flow_num_params()
        g = np.zeros(n, np.float32)
        loss = C.c_double()
        self._check(self.lib.cp_flow_loss_grad(self.h, batch, iteration, g.ctypes.data_as(C.c_void_p), C.byref(loss)))
        return g, loss.value

    # ------------------------------------------------------------------ unweighting
    def weight_quantile(self, q=0.999):
        v = C.c_double()
        self._check(self.lib.cp_weight_quantile(self.h, q, C.byref(v)))
        return v.value

    def set_wmax(self, w_max):
        self._check(self.lib.cp_set_wmax(self.h, w_max))

    def unweight(self, n_points, iteration=0, capacity=None, records=None):
        """Production pass into a device buffer; returns (records tensor [n_acc, 64] uint8, stats)."""
        torch = _torch()
        if records is None:
            capacity = capacity if capacity is not None else n_points
            records = torch.empty((capacity, 64), dtype=torch.uint8, device=self.device)
        capacity = records.shape[0]
        r = cp_unweight_result()
        rc = self.lib.cp_unweight(self.h, n_points, iteration, _ptr(records), capacity, C.byref(r))
        self._check(rc)
        return records[:min(r.n_accepted, capacity)], r.as_dict()

    def to_device_events(self, records, n_events=None, max_part=4, n_var=1, scale_ratios=None, events=None, e0=0):
        """Hand records (device uint8 [n, 64]) over to the reference pipeline's device event
        record (DeviceEvents): a dict of device tensors, one per member, allocated like the
        reference's allocEvents for n_events events (default: the records) unless `events` (such
        a dict) is given; events e0 .. e0 + n - 1 are filled."""
        torch = _torch()
        n = records.shape[0]
        if events is None:
            ne = n_events if n_events is not None else n
            npart = ne * max_part
            dev = self.device
            events = {"nEvents": ne, "maxPart": max_part, "nVar": n_var}
            for f in ("px", "py", "pz", "e", "m"):
                events[f] = torch.zeros(npart, dtype=torch.float64, device=dev)
            for f in ("pdg", "status", "col", "acol", "mo1", "mo2", "d1", "d2"):
                events[f] = torch.zeros(npart, dtype=torch.int32, device=dev)
            events["nPart"] = torch.zeros(ne, dtype=torch.int32, device=dev)
            events["seed"] = torch.zeros(ne, dtype=torch.int64, device=dev)
            for f in ("scale", "x1", "x2"):
                events[f] = torch.zeros(ne, dtype=torch.float64, device=dev)
            for f in ("flavA", "flavB"):
                events[f] = torch.zeros(ne, dtype=torch.int32, device=dev)
            events["active"] = torch.ones(ne, dtype=torch.uint8, device=dev)
            events["weight"] = torch.zeros(ne * n_var, dtype=torch.float64, device=dev)
        ev = _lib.cp_device_events(events["nEvents"], events["maxPart"], events["nVar"],
                                   *[_ptr(events[f]) for f, _ in _lib.cp_device_events._fields_[3:]])
        self._check(self.lib.cp_records_to_device_events(
            self.h, _ptr(records), n, _ptr(scale_ratios) if scale_ratios is not None else None, C.byref(ev), e0))
        return events

    def unweight_scale_weights(self, n_points, iteration=0, records=None):
        """cp_unweight with the 7-point scale variation: (records, weights [n_acc, 6], stats); the
        weight columns are the ratios for (muR, muF) factors (2,1), (1/2,1), (1,2), (1,1/2),
        (2,2), (1/2,1/2)."""
        torch = _torch()
        if records is None:
            records = torch.empty((n_points, 64), dtype=torch.uint8, device=self.device)
        w = torch.empty((records.shape[0], 6), dtype=torch.float32, device=self.device)
        self._check(self.lib.cp_set_scale_weights(self.h, _ptr(w), records.shape[0]))
        try:
            rec, st = self.unweight(n_points, iteration=iteration, records=records)
        finally:
            self._check(self.lib.cp_set_scale_weights(self.h, None, 0))
        return rec, w[:rec.shape[0]], st

    def generate_host(self, n_points, records_host, iteration=0, chunk=1 << 21):
        """Production pass into a host uint8 tensor/array of shape [capacity, 64]."""
        r = cp_unweight_result()
        ptr = records_host.data_ptr() if hasattr(records_host, "data_ptr") else records_host.ctypes.data
        self._check(self.lib.cp_generate_host(self.h, n_points, iteration, chunk, C.c_void_p(ptr),
                                              records_host.shape[0], C.byref(r)))
        return r.as_dict()

    # ------------------------------------------------------------------ partonic gg -> gg
    def partonic_integrate(self, n_points, sqrt_shat=100.0, alphas=0.13, cmax=0.9,
                           conv=0.3893793721, seed=42):
        r = cp_result()
        self._check(self.lib.cp_partonic_integrate(self.h, sqrt_shat, alphas, cmax, conv, seed,
                                                   n_points, C.byref(r)))
        return r.as_dict()

    def partonic_splitmix(self, n_threads, k_per, sqrt_shat=100.0, alphas=0.118, cmax=0.9,
                          conv=0.3893793721, seed=0xABCDEF01):
        r = cp_result()
        self._check(self.lib.cp_partonic_splitmix(self.h, sqrt_shat, alphas, cmax, conv, seed,
                                                  n_threads, k_per, C.byref(r)))
        return r.as_dict()

    def partonic_weights(self, point0, n, sqrt_shat=100.0, alphas=0.13, cmax=0.9,
                         conv=0.3893793721, seed=42):
        torch = _torch()
        w = torch.empty(n, dtype=torch.float64, device=self.device)
        self._check(self.lib.cp_partonic_weights(self.h, sqrt_shat, alphas, cmax, conv, seed,
                                                 point0, n, _ptr(w)))
        return w


def adapt_gradient_loop(step, steps, n_points, lr, iteration0):
    """The variance-gradient schedule over any gradient-step function step(n, iteration=, lr=)
    (one handle, or the sharded form of cupythia_b200.distributed)."""
    hist = []
    prev = None
    for s in range(steps):
        r = step(n_points, iteration=iteration0 + s, lr=lr)
        rel = r["var"] / r["sigma"] ** 2
        if prev is not None and rel > prev:
            lr *= 0.5
        prev = rel
        hist.append({"step": s, "lr": lr, "rel_var": rel, "sigma": r["sigma"]})
    return hist


EVENT_DTYPE = np.dtype([("id", "<i2", 4), ("pz_in", "<f4", 2), ("p3", "<f4", 4), ("p4", "<f4", 4),
                        ("weight", "<f4"), ("pt_hat", "<f4"), ("process", "<u2"), ("colour", "<u2"),
                        ("point", "<u4")])


def events_view(records):
    """Structured numpy view (cp_event layout) of a [n, 64] uint8 record array or tensor."""
    a = records.cpu().numpy() if hasattr(records, "cpu") else np.asarray(records)
    return np.ascontiguousarray(a).view(EVENT_DTYPE).reshape(-1)


def colour_tags(events):
    """(col, acol) int arrays [n, 4] of structured records (EVENT_DTYPE): colour indices 1..4 of
    the flow each record's process chose (cp_colour_tags), 0 = no colour."""
    lib = _lib.load()
    ev = np.asarray(events)
    col = np.zeros((len(ev), 4), np.int32)
    acol = np.zeros((len(ev), 4), np.int32)
    cache = {}
    for i, (p, c) in enumerate(zip(ev["process"].tolist(), ev["colour"].tolist())):
        key = (p, c)
        if key not in cache:
            a = (C.c_int * 4)()
            b = (C.c_int * 4)()
            rc = lib.cp_colour_tags(p, c, a, b)
            if rc:
                raise CpError(rc, f"invalid colour flow {c} for process {p}")
            cache[key] = (list(a), list(b))
        col[i], acol[i] = cache[key]
    return col, acol


def write_lhef(path, records, sigma_mb, sigma_err_mb, cfg=None):
    """Les Houches Event File 3.0 of host or device records (cp_write_lhef); cfg defaults to the
    library's default configuration."""
    lib = _lib.load()
    if cfg is None:
        cfg = cp_config()
        lib.cp_config_default(C.byref(cfg))
    a = records.cpu().numpy() if hasattr(records, "cpu") else np.asarray(records)
    a = np.ascontiguousarray(a)
    n = a.nbytes // 64
    rc = lib.cp_write_lhef(C.byref(cfg), a.ctypes.data_as(C.c_void_p), n, sigma_mb, sigma_err_mb,
                           os.fsencode(str(path)))
    if rc:
        raise CpError(rc, "cp_write_lhef failed")

