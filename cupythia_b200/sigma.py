"""Pythia ``SigmaProcess`` surface over batches (pythia8317/include/Pythia8/SigmaProcess.h).

Each class mirrors one Pythia 2 -> 2 QCD process (pythia8317/include/Pythia8/SigmaQCD.h:188-352)
with the same ``name()``, ``code()`` and ``inFlux()``; the per-point methods of Pythia become
batch methods over device arrays:

    Pythia (one point)                          here (n points, CUDA)
    set2Kin(x1, x2, sH, tH, m3, m4, bw3, bw4)   set2Kin(x1, x2, sH, tH)     (massless)
    sigmaKin(); sigmaHat()                       sigmaHat(id1=0, id2=0)      GeV^-4
    sigmaPDF()                                   sigmaPDF()                  mb GeV^-2
    alphaSRen(), Q2Ren(), Q2Fac()                same names, arrays
    pickInState()                                pickInState(r_pair) -> (id1, id2)
    setIdColAcol()                               setIdColAcol(r_flavour, r_colour, r_orient)
                                                 -> (ids [n, 4], col [n, 4], acol [n, 4])

As in Pythia, ``sigmaHat`` of ``Sigma2qq2qq`` needs the incoming flavour pair; the others are
flavour independent.  Pythia draws its own random numbers in ``pickInState`` and
``setIdColAcol``; here the caller passes the uniforms (one per point per draw), so a batch is
reproducible.  Errors raise :class:`cupythia_b200.CpError` with Pythia's meaning of
"invalid input"; there is no CPU path.
"""
import numpy as np

from . import Integrator, _lib
from ._lib import CP_PROC_GG2GG, CP_PROC_GG2QQBAR, CP_PROC_QG2QG, CP_PROC_QQ2QQ, CP_PROC_QQBAR2GG


class Sigma2Process:
    """Base class: one handle, one stored batch."""

    _name = ""
    _code = 0
    _flux = ""
    _bit = 0

    def __init__(self, integrator=None, **cfg):
        self.it = integrator if integrator is not None else Integrator(**cfg)
        self.n = 0

    def name(self):
        return self._name

    def code(self):
        return self._code

    def inFlux(self):
        return self._flux

    def _dev(self, a):
        import torch
        return torch.as_tensor(np.asarray(a, np.float32), device=self.it.device).contiguous()

    def set2Kin(self, x1, x2, sH, tH):
        t = [self._dev(v) for v in (x1, x2, sH, tH)]
        n = t[0].numel()
        if any(v.numel() != n for v in t):
            raise _lib.CpError(_lib.CP_ERR_INVALID, "set2Kin: arrays of different length")
        self._keep = t
        self.n = n
        self.it._check(self.it.lib.cp_set2kin_batch(self.it.h, *[_ptr(v) for v in t], n))

    def _out(self):
        import torch
        return torch.empty(self.n, dtype=torch.float32, device=self.it.device)

    def sigmaHat(self, id1=0, id2=0):
        out = self._out()
        self.it._check(self.it.lib.cp_sigma_hat_batch(self.it.h, self._code, id1, id2, _ptr(out)))
        return out

    def sigmaKin(self):
        out = self._out()
        self.it._check(self.it.lib.cp_sigma_kin_batch(self.it.h, self._code, _ptr(out)))
        return out

    def sigmaPDF(self):
        out = self._out()
        self.it._check(self.it.lib.cp_sigma_pdf_batch(self.it.h, self._bit, _ptr(out)))
        return out

    def _scales(self):
        a, r, f = self._out(), self._out(), self._out()
        self.it._check(self.it.lib.cp_scales_batch(self.it.h, _ptr(a), _ptr(r), _ptr(f)))
        return a, r, f

    def _pick(self, r_pair, r_flavour, r_colour, r_orient):
        import torch
        r = torch.stack([self._dev(np.array(np.broadcast_to(v, (self.n,)))) for v in (r_pair, r_flavour, r_colour, r_orient)],
                        1).contiguous()
        ids = torch.empty((self.n, 4), dtype=torch.int16, device=self.it.device)
        colour = torch.empty(self.n, dtype=torch.int16, device=self.it.device)
        self.it._check(self.it.lib.cp_pick_state_batch(self.it.h, self._code, _ptr(r), _ptr(ids), _ptr(colour)))
        return ids, colour

    def pickInState(self, r_pair):
        """Incoming flavour pair of every point of the batch (SigmaProcess::pickInState)."""
        self._r_pair = np.asarray(r_pair, np.float32)
        ids, _ = self._pick(self._r_pair, 0.5, 0.5, 0.5)
        return ids[:, 0], ids[:, 1]

    def setIdColAcol(self, r_flavour=0.5, r_colour=0.5, r_orient=0.5):
        """Outgoing flavours and colour tags (the process's setIdColAcol) for the pairs of the last
        pickInState; returns (ids [n, 4], col [n, 4], acol [n, 4]) as numpy arrays."""
        from . import colour_tags, EVENT_DTYPE
        ids, colour = self._pick(self._r_pair, r_flavour, r_colour, r_orient)
        ev = np.zeros(self.n, EVENT_DTYPE)
        ev["process"] = self._code
        ev["colour"] = colour.cpu().numpy().view(np.uint16)
        col, acol = colour_tags(ev)
        return ids.cpu().numpy(), col, acol

    def alphaSRen(self):
        return self._scales()[0]

    def Q2Ren(self):
        return self._scales()[1]

    def Q2Fac(self):
        return self._scales()[2]


def _ptr(t):
    import ctypes as C
    return C.c_void_p(t.data_ptr())


class Sigma2gg2gg(Sigma2Process):
    _name, _code, _flux, _bit = "g g -> g g", 111, "gg", CP_PROC_GG2GG


class Sigma2gg2qqbar(Sigma2Process):
    _name, _code, _flux, _bit = "g g -> q qbar (uds)", 112, "gg", CP_PROC_GG2QQBAR


class Sigma2qg2qg(Sigma2Process):
    _name, _code, _flux, _bit = "q g -> q g", 113, "qg", CP_PROC_QG2QG


class Sigma2qq2qq(Sigma2Process):
    _name, _code, _flux, _bit = "q q(bar)' -> q q(bar)'", 114, "qq", CP_PROC_QQ2QQ

    def sigmaKin(self):
        raise _lib.CpError(_lib.CP_ERR_INVALID,
                           "Sigma2qq2qq: the cross section depends on the flavour pair; use sigmaHat(id1, id2)")


class Sigma2qqbar2gg(Sigma2Process):
    _name, _code, _flux, _bit = "q qbar -> g g", 115, "qqbarSame", CP_PROC_QQBAR2GG


HARD_QCD = [Sigma2gg2gg, Sigma2gg2qqbar, Sigma2qg2qg, Sigma2qq2qq, Sigma2qqbar2gg]
