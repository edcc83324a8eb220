"""Mirror of the reference's Verona3D module (src/3dim/) over the B200 library.

Same names and argument meaning as the Julia API: ParVector3D / CuParVector3D
hold P as (5, Nx+6, Ny+6, Nz+6) FP64 column-major arrays and HARM_HLL runs the
time loop (src/3dim/algos.jl:203-362), now on the device through the C ABI.
Differences: no MPI (single GPU, MPI_dims must be (1,1,1)); `Size` (the
KernelAbstractions group size) is ignored because the library picks its own
tiles; `fun_bound` is a boundary spec (see `boundary`), and dumps go to an
optional `dump(i, t, solver)` callback instead of HDF5.
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from ._harm import run_loop
from .solver import Solver

NVAR = 5


class ParVector3D:
    """src/3dim/structs.jl:28-41 (host)."""

    def __init__(self, Nx, Ny=None, Nz=None):
        if isinstance(Nx, (ParVector3D, CuParVector3D)):
            src = Nx
            self.arr = np.asfortranarray(src.arr if isinstance(src, ParVector3D) else src.to_host())
        else:
            self.arr = np.zeros((NVAR, Nx + 6, Ny + 6, Nz + 6), order="F")
        self.size_X, self.size_Y, self.size_Z = self.arr.shape[1:]


class CuParVector3D:
    """src/3dim/structs.jl:43-56 (device): the same memory as a contiguous
    torch tensor of shape (Nz+6, Ny+6, Nx+6, 5)."""

    def __init__(self, P):
        import torch

        if isinstance(P, ParVector3D):
            a = np.asfortranarray(P.arr)
        else:
            a = np.zeros((NVAR, P[0] + 6, P[1] + 6, P[2] + 6), order="F")
        self.size_X, self.size_Y, self.size_Z = a.shape[1:]
        self.arr = torch.from_numpy(np.ascontiguousarray(a.transpose(3, 2, 1, 0))).cuda()

    def to_host(self) -> np.ndarray:
        return np.asfortranarray(self.arr.cpu().numpy().transpose(3, 2, 1, 0))


def VectorLike(X):
    """src/3dim/structs.jl:58-64"""
    if isinstance(X, CuParVector3D):
        return CuParVector3D((X.size_X - 6, X.size_Y - 6, X.size_Z - 6))
    return ParVector3D(X.size_X - 6, X.size_Y - 6, X.size_Z - 6)


def turnoff_boundary(dt, T_exp, box_X):
    """The built-in equivalent of the jet example's TurnOff callback
    (examples/Jet3D/HARM_jet_breakout.jl:131-158): x-lo ghosts fixed with the
    u^x decay (1 - dt/T_exp) for box_X/3 < t < box_X, zero-gradient elsewhere."""
    return [(L.FACE["xlo"], L.BC_FIXED, (2, box_X / 3, box_X, 1 - dt / T_exp))] + [
        (f, L.BC_OUTFLOW, ()) for f in (1, 2, 3, 4, 5)
    ]


def make_solver(P, dx, dy, dz, eos, floor, n_iter, tol, boundary=None, **options) -> Solver:
    gamma = eos.gamma if hasattr(eos, "gamma") else float(eos)
    s = Solver(3, (P.size_X - 6, P.size_Y - 6, P.size_Z - 6), gamma, (dx, dy, dz), n_iter=n_iter, tol=tol,
               floor=floor, **options)
    for face, kind, par in boundary or []:
        s.set_boundary(face, kind, par)
    if isinstance(P, CuParVector3D):
        s.load_prims(P.arr)
    else:
        s.load_prims(P.arr)
    return s


def HARM_HLL(comm, P, MPI_dims, Size, dt, dx, dy, dz, Tmax, eos, drops, floor=1e-7, out_dir=".", verbose=False,
             *kwargs, dump=None, **options):
    """Verona3D.HARM_HLL, src/3dim/algos.jl:203-362. kwargs = (n_iter, tol[, fun_bound]);
    fun_bound is a list of (face, kind, params) boundary specs. P is updated in place;
    returns the number of dumps, as the reference does."""
    if tuple(MPI_dims) != (1, 1, 1):
        raise NotImplementedError("single GPU: MPI_dims must be (1, 1, 1)")
    n_iter, tol = int(kwargs[0]), float(kwargs[1])
    boundary = kwargs[2] if len(kwargs) > 2 else None
    s = make_solver(P, dx, dy, dz, eos, floor, n_iter, tol, boundary, **options)
    try:
        i = run_loop(s, dt, Tmax, drops, dump, verbose)
        if isinstance(P, CuParVector3D):
            s.store_prims(P.arr)
        else:
            s.prims_into(P.arr)
    finally:
        s.close()
    return i
