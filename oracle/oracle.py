"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm import this module, and only to check or time against. The product (verona_b200)
never imports it.

The oracle is a C FP64 restatement of Wesenheit/Verona's SRHD update
(src/fluxlimiter.jl, src/eos.jl, src/{1,2,3}dim/{structs,algos}.jl). Parity
with the Julia reference itself is unpinned (no Julia here, no reference
tests); it is pinned to published known answers in tests/test_oracle_*.py.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libveronaoracle.so")

MINMOD, PPM, WENOZ = 0, 1, 2
HLL, HLLC = 0, 1
BC_OUTFLOW, BC_FIXED, BC_NOZZLE = 0, 1, 2
RECON = {"minmod": MINMOD, "ppm": PPM, "wenoz": WENOZ}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    src = os.path.join(HERE, "verona_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE], stdout=subprocess.DEVNULL)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        L.or_recon.argtypes = [C.c_int, _dp, _dp]
        L.or_sound_speed.argtypes = [C.c_double] * 3
        L.or_sound_speed.restype = C.c_double
        L.or_face_flux.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, _dp, _dp, _dp]
        L.or_prim2con.argtypes = [C.c_int, C.c_double, _dp, _dp]
        L.or_con2prim.argtypes = [C.c_int, C.c_double, C.c_int, C.c_double, _dp, _dp]
        L.or_con2prim.restype = C.c_int
        L.or_lu4_swaps_take.argtypes = []
        L.or_lu4_swaps_take.restype = C.c_longlong
        L.or1d_create.argtypes = [C.c_int, _dp, _dp, _dp, C.c_double, C.c_int, C.c_int, C.c_double]
        L.or1d_create.restype = C.c_void_p
        L.or1d_step.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int]
        L.or1d_get.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.or1d_get_cons.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.or1d_destroy.argtypes = [C.c_void_p]
        L.ornd_create.argtypes = [C.c_int, _ip, _dp, C.c_double, C.c_double, C.c_int, C.c_double,
                                  C.c_int, C.c_int, C.c_int]
        L.ornd_create.restype = C.c_void_p
        L.ornd_set_grid.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double]
        L.ornd_set_boundary.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, C.c_int]
        L.ornd_step.argtypes = [C.c_void_p, C.c_double, C.c_int]
        L.ornd_get_prims.argtypes = [C.c_void_p, _dp]
        L.ornd_get_cons.argtypes = [C.c_void_p, _dp]
        L.ornd_time.argtypes = [C.c_void_p]
        L.ornd_time.restype = C.c_double
        L.ornd_c2p_failures.argtypes = [C.c_void_p]
        L.ornd_c2p_failures.restype = C.c_int64
        L.ornd_destroy.argtypes = [C.c_void_p]
        for name in ("ornd_k_fluxes",):
            getattr(L, name).argtypes = [C.c_int, _ip, _dp, C.c_double, C.c_double, _dp, C.c_int,
                                         C.c_int, C.c_int]
        L.ornd_k_update.argtypes = [C.c_int, _ip, _dp, _dp, C.c_double, _dp, _dp, _dp, _dp]
        L.ornd_k_utop.argtypes = [C.c_int, _ip, _dp, _dp, C.c_double, C.c_int, C.c_double]
        L.ornd_k_ptou.argtypes = [C.c_int, _ip, _dp, _dp, C.c_double]
        L.ornd_k_limit.argtypes = [C.c_int, _ip, _dp, C.c_double]
        L.or_num_threads.restype = C.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"])
    return a.ctypes.data_as(_dp)


def num_threads() -> int:
    return lib().or_num_threads()


def recon(method: int, q) -> tuple[float, float]:
    q = np.ascontiguousarray(q, dtype=np.float64)
    out = np.zeros(2)
    lib().or_recon(method, _p(q), _p(out))
    return float(out[0]), float(out[1])


def prim2con(dims: int, gamma: float, P) -> np.ndarray:
    P = np.ascontiguousarray(P, dtype=np.float64)
    U = np.zeros(2 + dims)
    lib().or_prim2con(dims, gamma, _p(P), _p(U))
    return U


def con2prim(dims: int, gamma: float, n_iter: int, tol: float, U, guess) -> tuple[np.ndarray, int]:
    U = np.ascontiguousarray(U, dtype=np.float64)
    P = np.array(guess, dtype=np.float64)
    r = lib().or_con2prim(dims, gamma, n_iter, tol, _p(U), _p(P))
    return P, r


def lu4_swaps_take() -> int:
    """Row swaps of the 2D con2prim's pivoted LU on this thread since the last call."""
    return int(lib().or_lu4_swaps_take())


def face_flux(dims: int, axis: int, riemann: int, gamma: float, PL, PR) -> np.ndarray:
    PL = np.ascontiguousarray(PL, dtype=np.float64)
    PR = np.ascontiguousarray(PR, dtype=np.float64)
    F = np.zeros(2 + dims)
    lib().or_face_flux(dims, axis, riemann, gamma, _p(PL), _p(PR), _p(F))
    return F


class Solver1DRef:
    """Verona1D.HARM_HLL (src/1dim/algos.jl:58-315): N cells, no ghosts."""

    def __init__(self, rho, u, ux, gamma, rec, n_iter, tol):
        self.N = len(rho)
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (rho, u, ux)]
        self._h = lib().or1d_create(self.N, _p(a[0]), _p(a[1]), _p(a[2]), gamma,
                                    RECON.get(rec, rec) if isinstance(rec, str) else rec, n_iter, tol)

    def step(self, dt, dx, nsteps=1):
        lib().or1d_step(self._h, dt, dx, nsteps)

    def prims(self):
        out = [np.zeros(self.N) for _ in range(3)]
        lib().or1d_get(self._h, *[_p(o) for o in out])
        return np.stack(out)

    def cons(self):
        out = [np.zeros(self.N) for _ in range(3)]
        lib().or1d_get_cons(self._h, *[_p(o) for o in out])
        return np.stack(out)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().or1d_destroy(self._h)
            self._h = None


class SolverND:
    """Verona2D/3D.HARM_HLL time loop (src/{2,3}dim/algos.jl) on padded AoS
    arrays (nv, n0+6, n1+6, n2+6) in Julia's column-major order, plus the
    HLLC / SSP-RK3 / reconstruction-choice extensions."""

    def __init__(self, dims, n, P_aos, gamma, floor, n_iter, tol, recon=WENOZ, riemann=HLL, rk=2):
        self.dims = dims
        self.n = tuple(int(x) for x in n) + (1,) * (3 - len(n))
        self.nv = 2 + dims
        self.shape = (self.nv,) + tuple(self.n[a] + 6 for a in range(dims))
        P = np.asfortranarray(P_aos, dtype=np.float64)
        assert P.shape == self.shape, (P.shape, self.shape)
        narr = (C.c_int * 3)(*self.n)
        self._h = lib().ornd_create(dims, narr, _p(P), gamma, floor, n_iter, tol, recon, riemann, rk)

    def set_grid(self, dx, dy=1.0, dz=1.0):
        lib().ornd_set_grid(self._h, dx, dy, dz)

    def set_boundary(self, face, kind, params=()):
        par = np.zeros(16)
        par[: len(params)] = params
        lib().ornd_set_boundary(self._h, face, kind, _p(par), len(params))

    def step(self, dt, nsteps=1):
        lib().ornd_step(self._h, dt, nsteps)

    @property
    def t(self):
        return lib().ornd_time(self._h)

    @property
    def c2p_failures(self):
        return lib().ornd_c2p_failures(self._h)

    def prims(self):
        out = np.zeros(self.shape, order="F")
        lib().ornd_get_prims(self._h, _p(out))
        return out

    def cons(self):
        out = np.zeros(self.shape, order="F")
        lib().ornd_get_cons(self._h, _p(out))
        return out

    def __del__(self):
        if getattr(self, "_h", None):
            lib().ornd_destroy(self._h)
            self._h = None


def _npad(shape):
    d = len(shape) - 1
    return (C.c_int * 3)(*(list(shape[1:]) + [1] * (3 - d)))


def k_fluxes(P, gamma, floor, axis, recon=WENOZ, riemann=HLL):
    """function_Fluxes of one axis on a padded AoS array (column-major)."""
    P = np.asfortranarray(P, dtype=np.float64)
    F = np.zeros_like(P, order="F")
    lib().ornd_k_fluxes(P.ndim - 1, _npad(P.shape), _p(P), gamma, floor, _p(F), axis, recon, riemann)
    return F


def k_update(U, dt, dxs, Fs):
    U = np.asfortranarray(U, dtype=np.float64)
    Ub = np.zeros_like(U, order="F")
    Fs = [np.asfortranarray(f) for f in Fs] + [U] * (3 - len(Fs))
    d = np.asarray(list(dxs) + [1.0] * (3 - len(dxs)), dtype=np.float64)
    lib().ornd_k_update(U.ndim - 1, _npad(U.shape), _p(U), _p(Ub), dt, _p(d), *[_p(f) for f in Fs])
    return Ub


def k_utop(U, Pguess, gamma, n_iter, tol):
    U = np.asfortranarray(U, dtype=np.float64)
    P = np.array(Pguess, dtype=np.float64, order="F")
    lib().ornd_k_utop(U.ndim - 1, _npad(U.shape), _p(U), _p(P), gamma, n_iter, tol)
    return P


def k_ptou(P, gamma):
    P = np.asfortranarray(P, dtype=np.float64)
    U = np.zeros_like(P, order="F")
    lib().ornd_k_ptou(P.ndim - 1, _npad(P.shape), _p(P), _p(U), gamma)
    return U


def k_limit(P, floor):
    P = np.array(P, dtype=np.float64, order="F")
    lib().ornd_k_limit(P.ndim - 1, _npad(P.shape), _p(P), floor)
    return P
