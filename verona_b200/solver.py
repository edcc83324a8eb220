"""Python handle over the C ABI: one SRHD solver state resident on a GPU.

Arrays at this boundary use the reference's layout: FP64, column-major
(nvar, Nx+6, Ny+6[, Nz+6]) with the variable index fastest
(src/3dim/structs.jl:28-64). On the host that is a numpy array in Fortran
order of that shape; on the device a contiguous torch tensor of the reversed
shape (Nz+6, Ny+6, Nx+6, nvar), which is the same memory.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


def _stream_ptr(stream):
    if stream is None:
        import torch

        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)


class Solver:
    """A 1D/2D/3D grid of interior size `n` (3 ghosts per side), or the 1D
    reference layout (nghost=0, N cells). Options: recon, riemann, rk,
    precision, guess, n_iter, tol, floor, stats, w_rtol, w_max_newton."""

    def __init__(self, dims: int, n, gamma: float, dx=(1.0, 1.0, 1.0), nghost: int = 3, **options):
        n = tuple(int(x) for x in (n if hasattr(n, "__len__") else (n,)))
        self.dims = dims
        self.nghost = nghost
        self.n = n + (1,) * (3 - len(n))
        self.nv = 2 + dims
        self.opts = L.default_options(**options)
        h = C.c_void_p()
        L.check(L.lib().vb_create(C.byref(h), dims, self.n[0], self.n[1], self.n[2], nghost, C.byref(self.opts)))
        self._h = h
        L.check(L.lib().vb_set_eos(h, gamma), h)
        dx = tuple(dx) + (1.0,) * (3 - len(tuple(dx)))
        L.check(L.lib().vb_set_grid(h, *dx), h)
        self.gamma = gamma
        self.dx = dx

    # -- geometry -----------------------------------------------------------------
    @property
    def shape(self):
        """Fortran-order host shape (nvar, Nx+6, ...) of a primitive array."""
        if self.nghost == 0:
            return (self.nv, self.n[0])
        return (self.nv,) + tuple(self.n[a] + 2 * self.nghost for a in range(self.dims))

    @property
    def device_shape(self):
        return tuple(reversed(self.shape))

    # -- configuration --------------------------------------------------------------
    def set_boundary(self, face, kind, params=()):
        face = L.FACE[face] if isinstance(face, str) else face
        par = (C.c_double * 16)(*[float(x) for x in params])
        L.check(L.lib().vb_set_boundary(self._h, face, kind, par, len(params)), self._h)

    # -- state ------------------------------------------------------------------------
    def load_prims(self, P, stream=None):
        """P: host numpy array (Fortran order, self.shape) or device torch tensor."""
        if isinstance(P, np.ndarray):
            a = np.asfortranarray(P, dtype=np.float64)
            assert a.shape == self.shape, (a.shape, self.shape)
            L.check(L.lib().vb_load_prims_host(self._h, a.ctypes.data_as(C.c_void_p), _stream_ptr(stream)), self._h)
        else:
            self._check_dev(P)
            L.check(L.lib().vb_load_prims(self._h, C.c_void_p(P.data_ptr()), _stream_ptr(stream)), self._h)

    def init_prims(self, kind: str = "star_jet", stream=None, **params):
        """Generate the initial condition on the device (vb_init_prims): the
        examples' star + jet engine ("star_jet", 2D/3D) or an ambient medium
        ("ambient"); keyword arguments override the example values
        (seed, noise, rho, u, box, r_max, r_eng, rho0, temp, outer, gamma0,
        engine_rho, engine_temp). Returns the parameters used."""
        ic = L.VBIcParams()
        L.check(L.lib().vb_default_ic(self.dims, L.IC_KINDS[kind], C.byref(ic)))
        for k, v in params.items():
            if k == "box":
                for a, x in enumerate(v):
                    ic.box[a] = float(x)
            else:
                setattr(ic, k, v)
        L.check(L.lib().vb_init_prims(self._h, C.byref(ic), _stream_ptr(stream)), self._h)
        return ic

    @property
    def interior_shape(self):
        """Fortran-order host shape (nvar, Nx, ...) of a dump."""
        return (self.nv,) + tuple(self.n[a] for a in range(self.dims))

    def dump_begin(self, out: np.ndarray, stream=None) -> np.ndarray:
        """Start an asynchronous dump of the interior P into `out` (float64,
        Fortran order, interior_shape; pinned memory for the copy to overlap
        later steps). Keep `out` alive until dump_wait."""
        assert out.dtype == np.float64 and out.flags["F_CONTIGUOUS"] and out.shape == self.interior_shape
        L.check(L.lib().vb_dump_begin(self._h, out.ctypes.data_as(C.c_void_p), _stream_ptr(stream)), self._h)
        self._dump_out = out
        return out

    def dump_wait(self) -> int:
        """Wait for the dump in flight; returns the number of NaN values in it."""
        n = C.c_uint64()
        L.check(L.lib().vb_dump_wait(self._h, C.byref(n)), self._h)
        self._dump_out = None
        return int(n.value)

    def store_prims(self, out=None, stream=None):
        """Device tensor `out` (or a new one) filled with the current P."""
        import torch

        if out is None:
            out = torch.empty(self.device_shape, dtype=torch.float64, device="cuda")
        self._check_dev(out)
        L.check(L.lib().vb_store_prims(self._h, C.c_void_p(out.data_ptr()), _stream_ptr(stream)), self._h)
        return out

    def prims(self, stream=None) -> np.ndarray:
        """Current P copied to the host (Fortran order, self.shape)."""
        out = np.zeros(self.shape, dtype=np.float64, order="F")
        L.check(L.lib().vb_store_prims_host(self._h, out.ctypes.data_as(C.c_void_p), _stream_ptr(stream)), self._h)
        return out

    def prims_into(self, out: np.ndarray, stream=None) -> np.ndarray:
        assert out.dtype == np.float64 and out.flags["F_CONTIGUOUS"] and out.shape == self.shape
        L.check(L.lib().vb_store_prims_host(self._h, out.ctypes.data_as(C.c_void_p), _stream_ptr(stream)), self._h)
        return out

    def cons(self, stream=None) -> np.ndarray:
        import torch

        d = torch.empty(self.device_shape, dtype=torch.float64, device="cuda")
        L.check(L.lib().vb_store_cons(self._h, C.c_void_p(d.data_ptr()), _stream_ptr(stream)), self._h)
        torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()
        return np.asfortranarray(d.cpu().numpy().transpose(tuple(range(d.dim() - 1, -1, -1))))

    def _check_dev(self, t):
        import torch

        assert t.is_cuda and t.dtype == torch.float64 and t.is_contiguous(), "need a contiguous CUDA float64 tensor"
        assert t.numel() == int(np.prod(self.shape)), (t.shape, self.shape)

    # -- time loop --------------------------------------------------------------------
    def step(self, dt: float, nsteps: int = 1, stream=None):
        L.check(L.lib().vb_step(self._h, float(dt), int(nsteps), _stream_ptr(stream)), self._h)

    @property
    def t(self) -> float:
        v = C.c_double()
        L.check(L.lib().vb_get_time(self._h, C.byref(v)), self._h)
        return v.value

    @t.setter
    def t(self, value: float):
        L.check(L.lib().vb_set_time(self._h, float(value)), self._h)

    def max_signal_speed(self, stream=None) -> float:
        v = C.c_double()
        L.check(L.lib().vb_max_signal_speed(self._h, C.byref(v), _stream_ptr(stream)), self._h)
        return v.value

    def counters(self, stream=None) -> np.ndarray:
        arr = (C.c_uint64 * L.CNT_N)()
        L.check(L.lib().vb_get_counters(self._h, arr, L.CNT_N, _stream_ptr(stream)), self._h)
        return np.array(arr[:], dtype=np.uint64)

    def reset_counters(self, stream=None):
        L.check(L.lib().vb_reset_counters(self._h, _stream_ptr(stream)), self._h)

    def set_tuning(self, split_con2prim: int = -1, force_box: int = 0, learned_fused: int = -1, fp32_pairs: int = -1,
                   tma_tiles: int = -1, fp64_contract: int = 0):
        t = L.VBTuning(split_con2prim, force_box, learned_fused, fp32_pairs, tma_tiles, fp64_contract)
        L.check(L.lib().vb_set_tuning(self._h, C.byref(t)), self._h)

    def get_tuning(self) -> dict:
        t = L.VBTuning()
        L.check(L.lib().vb_get_tuning(self._h, C.byref(t)), self._h)
        return {"split_con2prim": t.split_con2prim, "force_box": t.force_box, "learned_fused": t.learned_fused,
                "fp32_pairs": t.fp32_pairs, "tma_tiles": t.tma_tiles, "fp64_contract": t.fp64_contract}

    def profile(self, enable: bool = True):
        L.check(L.lib().vb_profile_enable(self._h, int(enable)), self._h)

    def profile_read(self):
        """(stage-kernel ms, stage launches, all launches) since the last read."""
        ms, sl, al = C.c_double(), C.c_int64(), C.c_int64()
        L.check(L.lib().vb_profile_read(self._h, C.byref(ms), C.byref(sl), C.byref(al)), self._h)
        return ms.value, sl.value, al.value

    def profile_read2(self):
        """(stage ms, stencil-launcher ms, stage launches, all launches) since the last read."""
        ms, st, sl, al = C.c_double(), C.c_double(), C.c_int64(), C.c_int64()
        L.check(L.lib().vb_profile_read2(self._h, C.byref(ms), C.byref(st), C.byref(sl), C.byref(al)), self._h)
        return ms.value, st.value, sl.value, al.value

    @property
    def tma_tiles_active(self) -> bool:
        """True if the stencil tiles are staged by TMA on this handle."""
        v = C.c_int()
        L.check(L.lib().vb_tma_tiles_active(self._h, C.byref(v)), self._h)
        return bool(v.value)

    @property
    def memory_bytes(self) -> int:
        v = C.c_uint64()
        L.check(L.lib().vb_memory_bytes(self._h, C.byref(v)), self._h)
        return v.value

    def close(self):
        if getattr(self, "_h", None):
            L.lib().vb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
