"""Mirror of the reference's Verona1D module (src/1dim/) over the B200 library.

ParVector1D keeps arr1/arr2/arr3 (rho, u, u^x) on N cells with no ghosts;
HARM_HLL (src/1dim/algos.jl:58-315) runs the reference's 1D scheme -- its
frozen end cells and persistent face arrays included -- in one persistent
CTA on the device and returns the list of snapshots taken every `drops`.
"""
from __future__ import annotations

import copy

import numpy as np

from ._harm import steps_until_dump
from .solver import Solver

_REC = {"minmod": "minmod", "ppm": "ppm", "wenoz": "wenoz"}


class ParVector1D:
    """src/1dim/structs.jl:22-34"""

    def __init__(self, N, arr1=None, arr2=None, arr3=None):
        self.size = int(N)
        self.arr1 = np.zeros(N) if arr1 is None else np.array(arr1, dtype=np.float64)
        self.arr2 = np.zeros(N) if arr2 is None else np.array(arr2, dtype=np.float64)
        self.arr3 = np.zeros(N) if arr3 is None else np.array(arr3, dtype=np.float64)

    def aos(self) -> np.ndarray:
        return np.asfortranarray(np.stack([self.arr1, self.arr2, self.arr3]))


def HARM_HLL(P: ParVector1D, N: int, dt: float, dx: float, T: float, eos, drops: float, rec: str, *kwargs):
    """Verona1D.HARM_HLL(P, N, dt, dx, T, eos, drops, rec, n_iter, tol)."""
    if rec not in _REC:
        raise ValueError("reconstruction not supported!")  # src/1dim/algos.jl:115-116
    n_iter = int(kwargs[0]) if len(kwargs) > 0 else 50
    tol = float(kwargs[1]) if len(kwargs) > 1 else 1e-10  # UtoP's default, src/1dim/structs.jl:78
    gamma = eos.gamma if hasattr(eos, "gamma") else float(eos)
    s = Solver(1, (N,), gamma, (dx,), nghost=0, recon=_REC[rec], n_iter=n_iter, tol=tol)
    out = [copy.deepcopy(P)]
    try:
        s.load_prims(P.aos())
        t, thres = 0.0, drops
        while t < T:
            n, t = steps_until_dump(t, dt, T, thres)
            s.step(dt, n)
            if t > thres:
                a = s.prims()
                out.append(ParVector1D(N, a[0], a[1], a[2]))
                thres += drops
        a = s.prims()
        P.arr1[:], P.arr2[:], P.arr3[:] = a[0], a[1], a[2]
    finally:
        s.close()
    return out
