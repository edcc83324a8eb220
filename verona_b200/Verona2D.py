"""Mirror of the reference's Verona2D module (src/2dim/) over the B200 library.

ParVector2D / CuParVector2D hold P as (4, Nx+6, Ny+6) FP64 column-major
arrays; HARM_HLL runs the time loop of src/2dim/algos.jl:192-324 on the
device. Single GPU only (XMPI = YMPI = 1); SizeX/SizeY are ignored.
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from ._harm import run_loop
from .solver import Solver

NVAR = 4


class ParVector2D:
    """src/2dim/structs.jl:34-46 (host)."""

    def __init__(self, Nx, Ny=None):
        if isinstance(Nx, (ParVector2D, CuParVector2D)):
            src = Nx
            self.arr = np.asfortranarray(src.arr if isinstance(src, ParVector2D) else src.to_host())
        else:
            self.arr = np.zeros((NVAR, Nx + 6, Ny + 6), order="F")
        self.size_X, self.size_Y = self.arr.shape[1:]


class CuParVector2D:
    """src/2dim/structs.jl:48-60 (device): torch tensor of shape (Ny+6, Nx+6, 4)."""

    def __init__(self, P):
        import torch

        if isinstance(P, ParVector2D):
            a = np.asfortranarray(P.arr)
        else:
            a = np.zeros((NVAR, P[0] + 6, P[1] + 6), order="F")
        self.size_X, self.size_Y = a.shape[1:]
        self.arr = torch.from_numpy(np.ascontiguousarray(a.transpose(2, 1, 0))).cuda()

    def to_host(self) -> np.ndarray:
        return np.asfortranarray(self.arr.cpu().numpy().transpose(2, 1, 0))


def VectorLike(X):
    """src/2dim/structs.jl:62-68"""
    if isinstance(X, CuParVector2D):
        return CuParVector2D((X.size_X - 6, X.size_Y - 6))
    return ParVector2D(X.size_X - 6, X.size_Y - 6)


def turnoff_boundary(dt, T_exp, box_X):
    """Built-in equivalent of examples/Jet2D/HARM_jet_breakout.jl:84-99: x-lo
    ghosts fixed with the decay of P[4] (u^y, as that example does) for
    box_X/3 < t < box_X, zero-gradient on y-lo, y-hi and x-hi."""
    return [(L.FACE["xlo"], L.BC_FIXED, (3, box_X / 3, box_X, 1 - dt / T_exp))] + [
        (f, L.BC_OUTFLOW, ()) for f in (1, 2, 3)
    ]


def HARM_HLL(comm, P, XMPI, YMPI, SizeX, SizeY, dt, dx, dy, Tmax, eos, drops, floor=1e-7, out_dir=".", *kwargs,
             dump=None, verbose=False, **options):
    """Verona2D.HARM_HLL, src/2dim/algos.jl:192-324. kwargs = (n_iter, tol[, fun_bound])."""
    if (XMPI, YMPI) != (1, 1):
        raise NotImplementedError("single GPU: XMPI = YMPI = 1")
    n_iter, tol = int(kwargs[0]), float(kwargs[1])
    boundary = kwargs[2] if len(kwargs) > 2 else None
    gamma = eos.gamma if hasattr(eos, "gamma") else float(eos)
    s = Solver(2, (P.size_X - 6, P.size_Y - 6), gamma, (dx, dy), n_iter=n_iter, tol=tol, floor=floor, **options)
    try:
        for face, kind, par in boundary or []:
            s.set_boundary(face, kind, par)
        s.load_prims(P.arr)
        i = run_loop(s, dt, Tmax, drops, dump, verbose)
        if isinstance(P, CuParVector2D):
            s.store_prims(P.arr)
        else:
            s.prims_into(P.arr)
    finally:
        s.close()
    return i
