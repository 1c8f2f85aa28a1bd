"""Differentiable distortion energies on the device.

``DistortionEnergy`` is a ``torch.autograd.Function`` over the hand-written
forward / backward kernels of csrc/energy.cu: the ARAP (kind 0) and
symmetric-Dirichlet (kind 1) energies of engine/param.py:294-319, per island,
differentiated with respect to the UVs and to the 3D positions (through each
triangle's isometric frame). ``sd_refine`` drives the p95-stretch refinement:
Jacobi-preconditioned, flip-safe, monotone descent on the symmetric Dirichlet
energy of every island at once.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib

vp = C.c_void_p
ARAP, SYMMETRIC_DIRICHLET = 0, 1


def _sig():
    L = _lib.lib()
    if not getattr(L, "_uva_energy_sig", False):
        L.uva_energy_fwd.argtypes = [vp, vp, vp, C.c_int32, vp, vp, vp]
        L.uva_energy_fwd.restype = C.c_int32
        L.uva_energy_bwd.argtypes = [vp, vp, vp, C.c_int32, vp, vp, vp, vp]
        L.uva_energy_bwd.restype = C.c_int32
        L.uva_sd_refine.argtypes = [vp, C.c_int32, C.c_int32, C.c_double, vp, vp, vp]
        L.uva_sd_refine.restype = C.c_int32
        L._uva_energy_sig = True
    return L


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class DistortionEnergy(torch.autograd.Function):
    """Per-island energy E_i(U, P) of a device batch (topology from ``db``).

    forward(U (n,2) f64, P (n,3) f64, db, kind) -> (nc,) f64
    backward: dE/dU (n,2) and dE/dP (n,3), scaled by the incoming gradient
    of each island's energy."""

    @staticmethod
    def forward(ctx, U, P, db, kind):
        L = _sig()
        U = U.contiguous()
        P = P.contiguous()
        e = torch.empty(max(db.nc, 1), dtype=torch.float64, device=U.device)
        s = C.c_void_p(torch.cuda.current_stream(U.device).cuda_stream)
        _lib.check(L.uva_energy_fwd(C.byref(db.desc), _p(P), _p(U), int(kind), _p(e), None, s), "uva_energy_fwd")
        ctx.save_for_backward(U, P)
        ctx.db = db
        ctx.kind = int(kind)
        return e[:db.nc]

    @staticmethod
    def backward(ctx, g):
        L = _sig()
        U, P = ctx.saved_tensors
        db = ctx.db
        gs = g.contiguous().to(torch.float64)
        gU = torch.empty_like(U)
        gP = torch.empty_like(P) if ctx.needs_input_grad[1] else None
        s = C.c_void_p(torch.cuda.current_stream(U.device).cuda_stream)
        _lib.check(L.uva_energy_bwd(C.byref(db.desc), _p(P), _p(U), ctx.kind, _p(gs), _p(gU), _p(gP), s),
                   "uva_energy_bwd")
        return gU, gP, None, None


def distortion_energy(db, U=None, P=None, kind=ARAP):
    """Differentiable per-island energies of the batch ``db`` (defaults: its
    own UVs and positions)."""
    U = db.U[:db.n] if U is None else U
    P = db.P[:db.n] if P is None else P
    return DistortionEnergy.apply(U, P, db, kind)


def sd_refine(db, steps=50, halvings=8, cap=1.0):
    """``steps`` flip-safe descent steps on the symmetric Dirichlet energy of
    every island of ``db`` (a batch set up with param semantics); updates
    ``db.U`` in place and returns the final per-island energies."""
    L = _sig()
    n, nc = max(db.n, 1), max(db.nc, 1)
    scratch = torch.empty(8 * n + 8 * nc + n + 2, dtype=torch.float64, device=db.dev)
    e = torch.empty(nc, dtype=torch.float64, device=db.dev)
    s = C.c_void_p(torch.cuda.current_stream(db.dev).cuda_stream)
    _lib.check(L.uva_sd_refine(C.byref(db.desc), int(steps), int(halvings), float(cap), _p(e), _p(scratch), s),
               "uva_sd_refine")
    return e[:db.nc]
