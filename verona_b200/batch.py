"""Batch of independent 1D/2D problems on one GPU (vb_batch_*, include/verona_b200.h).

Each problem evolves as a single-grid `Solver` of the same dims and options
with outflow on every face; `Batch.step(n)` advances all of them by n steps in
one persistent kernel launch replayed from a CUDA graph. The tile variant and
CTAs per SM come from `verona_b200.autotune.tune_batch`.

Arrays use the reference layout of `Solver`: FP64, column-major (nvar, nx+6
[, ny+6]) on the host, the reversed-shape contiguous tensor on the device.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib as L
from .solver import _stream_ptr


class BatchProblem(C.Structure):
    _fields_ = [("dims", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("recon", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dt", C.c_double)]


def _sig():
    lib = L.lib()
    vp = C.c_void_p
    i64 = C.POINTER(C.c_int64)
    ip = C.POINTER(C.c_int)
    sigs = {
        "vb_batch_create": [C.POINTER(vp), C.c_int, C.POINTER(BatchProblem), C.c_double, C.POINTER(L.VBOptions)],
        "vb_batch_destroy": [vp],
        "vb_batch_load_prims": [vp, C.c_int, vp, vp],
        "vb_batch_store_prims": [vp, C.c_int, vp, vp],
        "vb_batch_step": [vp, C.c_int, vp],
        "vb_batch_get_time": [vp, C.c_int, C.POINTER(C.c_double)],
        "vb_batch_get_counters": [vp, C.POINTER(C.c_uint64), vp],
        "vb_batch_reset_counters": [vp, vp],
        "vb_batch_check": [vp, vp],
        "vb_batch_set_boundary": [vp, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_int],
        "vb_batch_set_wait_limit": [vp, C.c_uint32],
        "vb_batch_num_variants": [C.c_int],
        "vb_batch_variant_shape": [C.c_int, C.c_int, ip, ip, ip],
        "vb_batch_set_tuning": [vp, C.c_int, C.c_int],
        "vb_batch_get_tuning": [vp, ip, ip, ip],
        "vb_batch_info": [vp, i64, i64, i64],
        "vb_batch_checkpoint": [vp, vp],
        "vb_batch_rollback": [vp, vp],
    }
    for k, a in sigs.items():
        f = getattr(lib, k)
        f.argtypes = a
        f.restype = C.c_int
    lib.vb_batch_last_error.argtypes = [vp]
    lib.vb_batch_last_error.restype = C.c_char_p
    return lib


def _chk(rc, h=None):
    if rc != 0:
        msg = _sig().vb_batch_last_error(h)
        raise L.VBError(rc, (msg or b"").decode())
    return rc


def variants(precision="fp32"):
    """Tile shapes [(TX2, TY2, L1), ...] of the batch kernel variants of a precision."""
    lib = _sig()
    p = L.PRECISION[precision] if isinstance(precision, str) else precision
    out = []
    for v in range(lib.vb_batch_num_variants(p)):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        _chk(lib.vb_batch_variant_shape(p, v, C.byref(a), C.byref(b), C.byref(c)))
        out.append((a.value, b.value, c.value))
    return out


class Batch:
    """problems: sequence of dicts {dims, n: (nx,) or (nx, ny), recon, dx[, dy], dt}.
    Options as `Solver`: riemann, rk, precision, n_iter, tol, floor, stats."""

    def __init__(self, problems, gamma: float, **options):
        self.lib = _sig()
        arr = (BatchProblem * len(problems))()
        self.specs = []
        for i, q in enumerate(problems):
            n = tuple(int(x) for x in q["n"])
            dims = int(q["dims"])
            rec = q.get("recon", "wenoz")
            arr[i] = BatchProblem(dims, n[0], n[1] if dims == 2 else 1, L.RECON[rec] if isinstance(rec, str) else rec,
                                  float(q["dx"]), float(q.get("dy", q["dx"])), float(q["dt"]))
            self.specs.append(dict(q, n=n, dims=dims))
        self.opts = L.default_options(**options)
        h = C.c_void_p()
        _chk(self.lib.vb_batch_create(C.byref(h), len(problems), arr, gamma, C.byref(self.opts)))
        self._h = h
        self.gamma = gamma
        self.nprob = len(problems)

    # -- geometry ---------------------------------------------------------------------
    def shape(self, i):
        q = self.specs[i]
        return (2 + q["dims"],) + tuple(x + 6 for x in q["n"][: q["dims"]])

    def device_shape(self, i):
        return tuple(reversed(self.shape(i)))

    # -- state --------------------------------------------------------------------------
    def load_prims(self, i, P, stream=None):
        """P: host numpy array (Fortran order, shape(i)) or device tensor (device_shape(i))."""
        import torch

        if isinstance(P, np.ndarray):
            a = np.asfortranarray(P, dtype=np.float64)
            assert a.shape == self.shape(i), (a.shape, self.shape(i))
            P = torch.from_numpy(np.ascontiguousarray(a.transpose(tuple(range(a.ndim - 1, -1, -1))))).cuda()
        assert P.is_cuda and P.dtype == torch.float64 and P.is_contiguous() and tuple(P.shape) == self.device_shape(i)
        _chk(self.lib.vb_batch_load_prims(self._h, i, C.c_void_p(P.data_ptr()), _stream_ptr(stream)), self._h)
        torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()

    def store_prims(self, i, out=None, stream=None):
        import torch

        if out is None:
            out = torch.empty(self.device_shape(i), dtype=torch.float64, device="cuda")
        _chk(self.lib.vb_batch_store_prims(self._h, i, C.c_void_p(out.data_ptr()), _stream_ptr(stream)), self._h)
        return out

    def prims(self, i) -> np.ndarray:
        import torch

        d = self.store_prims(i)
        torch.cuda.current_stream().synchronize()
        return np.asfortranarray(d.cpu().numpy().transpose(tuple(range(d.dim() - 1, -1, -1))))

    def step(self, nsteps=1, stream=None):
        _chk(self.lib.vb_batch_step(self._h, int(nsteps), _stream_ptr(stream)), self._h)

    def time(self, i) -> float:
        t = C.c_double()
        _chk(self.lib.vb_batch_get_time(self._h, i, C.byref(t)), self._h)
        return t.value

    def counters(self, stream=None) -> np.ndarray:
        out = (C.c_uint64 * L.CNT_N)()
        _chk(self.lib.vb_batch_get_counters(self._h, out, _stream_ptr(stream)), self._h)
        return np.array(out[:], dtype=np.uint64)

    def reset_counters(self, stream=None):
        _chk(self.lib.vb_batch_reset_counters(self._h, _stream_ptr(stream)), self._h)

    def set_boundary(self, i: int, face, kind: int, params=()):
        """vb_batch_set_boundary: face (0 x-lo, 1 x-hi, 2 y-lo, 3 y-hi or a name
        of verona_b200._lib.FACE) of problem i gets kind OUTFLOW (0), FIXED (1,
        params: none or {var, t_on, t_off, factor}) or NOZZLE (2, params:
        {radius, c1, c2, rho, u, u1[, u2]})."""
        face = L.FACE[face] if isinstance(face, str) else face
        par = (C.c_double * 8)(*[float(x) for x in params])
        _chk(self.lib.vb_batch_set_boundary(self._h, int(i), int(face), int(kind), par, len(params)), self._h)

    def check(self, stream=None) -> int:
        """vb_batch_check: synchronises and returns its status code (0, or
        VB_ERR_TIMEOUT when a bounded wait of the batch kernel gave up) with
        the message in self.last_error."""
        rc = self.lib.vb_batch_check(self._h, _stream_ptr(stream))
        self.last_error = self.lib.vb_batch_last_error(self._h).decode() if rc else ""
        return rc

    def set_wait_limit(self, max_polls: int = 0):
        """Bound of a tile's wait for the previous stage, in polls of about
        128 ns (0: the default, 2^24)."""
        _chk(self.lib.vb_batch_set_wait_limit(self._h, int(max_polls)), self._h)

    def checkpoint(self, stream=None):
        _chk(self.lib.vb_batch_checkpoint(self._h, _stream_ptr(stream)), self._h)

    def rollback(self, stream=None):
        _chk(self.lib.vb_batch_rollback(self._h, _stream_ptr(stream)), self._h)

    # -- tuning ---------------------------------------------------------------------------
    def set_tuning(self, variant: int, ctas_per_sm: int = 0):
        _chk(self.lib.vb_batch_set_tuning(self._h, int(variant), int(ctas_per_sm)), self._h)

    @property
    def tuning(self):
        v, c, g = C.c_int(), C.c_int(), C.c_int()
        _chk(self.lib.vb_batch_get_tuning(self._h, C.byref(v), C.byref(c), C.byref(g)), self._h)
        return {"variant": v.value, "ctas_per_sm": c.value, "grid": g.value}

    def info(self):
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        _chk(self.lib.vb_batch_info(self._h, C.byref(a), C.byref(b), C.byref(c)), self._h)
        return {"interior_cells": a.value, "tiles_per_stage": b.value, "device_bytes": c.value}

    @property
    def precision(self) -> int:
        return int(self.opts.precision)

    def signature(self) -> str:
        """Key of the batch's shape for the tuning cache: sizes, reconstructions, options."""
        import hashlib

        h = hashlib.sha1()
        for q in self.specs:
            h.update(f"{q['dims']}:{q['n']}:{q.get('recon', 'wenoz')};".encode())
        o = self.opts
        h.update(f"r{o.riemann}k{o.rk}p{o.precision}".encode())
        return h.hexdigest()[:16]

    def close(self):
        if getattr(self, "_h", None):
            self.lib.vb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- the uneven Riemann / quadrant workload ---------------------------------------------
def _state(rng, gamma, dims):
    """(rho, u, u^x[, u^y]): rho log-uniform in [0.1, 10], p log-uniform in
    [1e-4, 20], |v| uniform in [0, 0.9] in a random direction."""
    rho = 10 ** rng.uniform(-1.0, 1.0)
    p = 10 ** rng.uniform(-4.0, math.log10(20.0))
    v = rng.uniform(0.0, 0.9)
    if dims == 1:
        d = np.array([rng.choice([-1.0, 1.0])])
    else:
        a = rng.uniform(0.0, 2 * math.pi)
        d = np.array([math.cos(a), math.sin(a)])
    lor = 1.0 / math.sqrt(1.0 - v * v)
    return np.concatenate([[rho, p / (gamma - 1.0)], lor * v * d])


def riemann_problems(seed=0, n1d=192, n2d=64, n1d_range=(256, 8192), n2d_range=(128, 1024), gamma=5.0 / 3.0,
                     cfl=0.4):
    """Seeded batch of 1D shock tubes (interface at x = 0.5) and 2D four-quadrant
    problems (quadrants meeting at the centre) on the unit interval / square:
    returns (problem specs, host primitive arrays). Reconstruction is drawn per
    problem from MINMOD / PPM / WENOZ; dt = cfl / (sum of 1/dx)."""
    rng = np.random.default_rng(seed)
    recs = ("minmod", "ppm", "wenoz")
    specs, prims = [], []
    for _ in range(n1d):
        N = int(rng.integers(n1d_range[0], n1d_range[1] + 1))
        dx = 1.0 / N
        L_, R_ = _state(rng, gamma, 1), _state(rng, gamma, 1)
        P = np.zeros((3, N + 6), order="F")
        x = (np.arange(N + 6) - 3 + 0.5) * dx
        P[:, x < 0.5] = L_[:, None]
        P[:, x >= 0.5] = R_[:, None]
        specs.append({"dims": 1, "n": (N,), "recon": recs[int(rng.integers(3))], "dx": dx, "dt": cfl * dx})
        prims.append(P)
    for _ in range(n2d):
        S = int(rng.integers(n2d_range[0], n2d_range[1] + 1))
        dx = 1.0 / S
        Q = [_state(rng, gamma, 2) for _ in range(4)]
        P = np.zeros((4, S + 6, S + 6), order="F")
        x = (np.arange(S + 6) - 3 + 0.5) * dx
        X, Y = np.meshgrid(x, x, indexing="ij")
        for k, (mx, my) in enumerate(((X >= 0.5, Y >= 0.5), (X < 0.5, Y >= 0.5), (X < 0.5, Y < 0.5),
                                      (X >= 0.5, Y < 0.5))):
            m = mx & my
            for v in range(4):
                P[v][m] = Q[k][v]
        specs.append({"dims": 2, "n": (S, S), "recon": recs[int(rng.integers(3))], "dx": dx, "dy": dx,
                      "dt": cfl / (2.0 / dx)})
        prims.append(P)
    return specs, prims
