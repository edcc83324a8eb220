"""Learned con2prim initial guess: training data, training loop and use.

The network (4 -> 64 -> 64 -> 64 -> 1, ReLU, BF16 on the tensor cores with
FP32 accumulation; vb_mlp.cu) maps a conserved state to the pressure guess
as a fraction of the total energy E = tau + D, y ~ p / E; Newton on
W = rho h gamma^2 starts from W0 = E (1 + max(y, 0)). Its training pairs are
conserved/primitive pairs made by the solver itself:
  * synthetic states with log-uniform rho in [1e-4, 10], log-uniform p/rho in
    [1e-6, 1e2], log-uniform Lorentz factor in [1, 100] in a random direction
    and Gamma in {4/3, 5/3};
  * snapshots of the 1D shock tube (Marti & Mueller problem 1) and of a 2D
    relativistic jet run by this library.
Conserved states come from the primitives through the reference's PtoU
(src/3dim/structs.jl:84-96). Training runs the project's forward/backward
tensor-core kernels (vb_mlp_train_step) with Adam.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

from . import _lib as L

N_IN, N_H = 4, 64
HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "data", "mlp_c2p.npz")


def _sig():
    lib = L.lib()
    vp = C.c_void_p
    fp = C.POINTER(C.c_float)
    sigs = {
        "vb_mlp_create": [C.POINTER(vp)],
        "vb_mlp_destroy": [vp],
        "vb_mlp_param_count": [],
        "vb_mlp_set_params": [vp, fp, fp, vp],
        "vb_mlp_get_params": [vp, fp, fp, vp],
        "vb_mlp_features": [vp, vp, vp, C.c_int, C.c_double, vp, vp, vp, vp],
        "vb_mlp_forward": [vp, vp, C.c_int, vp, vp],
        "vb_mlp_train_step": [vp, vp, vp, vp, C.c_int, C.c_float, fp, vp],
        "vb_mlp_get_grad": [vp, fp, vp],
        "vb_attach_mlp": [vp, vp],
        "vb_point_c2p_w": [C.c_double, vp, vp, C.c_double, C.c_int, C.c_int, vp, vp, vp, C.c_int, vp],
        "vb_point_c2p_gated": [C.c_double, vp, vp, C.c_double, C.c_int, C.c_int, vp, vp, vp, C.c_int, vp],
    }
    for k, a in sigs.items():
        f = getattr(lib, k)
        f.argtypes = a
        f.restype = C.c_int
    lib.vb_mlp_last_error.argtypes = [vp]
    lib.vb_mlp_last_error.restype = C.c_char_p
    return lib


def _chk(rc, h=None):
    if rc != 0:
        msg = L.lib().vb_mlp_last_error(h)
        raise L.VBError(rc, (msg or b"").decode())


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def n_params() -> int:
    return _sig().vb_mlp_param_count()


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initialisation of the FP32 parameter vector W1 b1 W2 b2 W3 b3 w4 b4."""
    rng = np.random.default_rng(seed)
    parts = [
        rng.normal(0, math.sqrt(2.0 / N_IN), (N_IN, N_H)), np.zeros(N_H),
        rng.normal(0, math.sqrt(2.0 / N_H), (N_H, N_H)), np.zeros(N_H),
        rng.normal(0, math.sqrt(2.0 / N_H), (N_H, N_H)), np.zeros(N_H),
        rng.normal(0, math.sqrt(1.0 / N_H), N_H), np.zeros(1),
    ]
    return np.concatenate([p.ravel() for p in parts]).astype(np.float32)


def split_params(v):
    v = np.asarray(v, dtype=np.float64)
    o = 0
    out = {}
    for name, shape in (("W1", (N_IN, N_H)), ("b1", (N_H,)), ("W2", (N_H, N_H)), ("b2", (N_H,)),
                        ("W3", (N_H, N_H)), ("b3", (N_H,)), ("w4", (N_H,)), ("b4", (1,))):
        n = int(np.prod(shape))
        out[name] = v[o:o + n].reshape(shape)
        o += n
    return out


# ---- training data ---------------------------------------------------------------------
def prim2con_torch(P, gamma):
    """PtoU (src/3dim/structs.jl:84-96) on a (5, n) FP64 torch tensor; gamma scalar or (n,)."""
    import torch

    gam = torch.sqrt(P[2] ** 2 + P[3] ** 2 + P[4] ** 2 + 1)
    w = gamma * P[1] + P[0]
    U = torch.empty_like(P)
    U[0] = gam * P[0]
    U[1] = (gamma - 1) * P[1] - gam**2 * w
    U[2:] = P[2:] * gam * w
    return U


def synthetic_states(n: int, gamma: float, seed: int = 0, lorentz_max: float = 100.0):
    """Primitive states (5, n) on the device over the training ranges."""
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    u01 = lambda: torch.rand(n, generator=g, dtype=torch.float64, device="cuda")  # noqa: E731
    rho = 10 ** (-4 + 5 * u01())
    p = rho * 10 ** (-6 + 8 * u01())
    lor = 10 ** (math.log10(lorentz_max) * u01())
    d = torch.randn((3, n), generator=g, dtype=torch.float64, device="cuda")
    d = d / d.norm(dim=0, keepdim=True)
    P = torch.empty((5, n), dtype=torch.float64, device="cuda")
    P[0] = rho
    P[1] = p / (gamma - 1)
    P[2:] = torch.sqrt(lor**2 - 1) * d
    return P


def solver_snapshots(gamma: float, max_states: int = 1 << 20):
    """Primitive states (5, n) from runs of this library: the 1D shock tube and a 2D jet."""
    import torch

    from .solver import Solver

    out = []
    # 1D Marti & Mueller problem 1 (gamma 5/3 there; the states are re-used with `gamma`)
    N = 1024
    x = (np.arange(N) + 0.5) / N
    P1 = np.stack([np.where(x < 0.5, 10.0, 1.0), np.where(x < 0.5, 13.33, 1e-6) / (gamma - 1), np.zeros(N)])
    s = Solver(1, (N,), gamma, (1.0 / N,), nghost=0, recon="minmod", n_iter=50, tol=1e-12)
    s.load_prims(np.asfortranarray(P1))
    for _ in range(8):
        s.step(0.4 / N, 128)
        a = s.prims()
        q = np.zeros((5, N))
        q[:3] = a
        out.append(q)
    s.close()
    # 2D jet (nozzle Lorentz factor 10) on 256 x 128
    n2 = (256, 128)
    P2 = np.zeros((4, n2[0] + 6, n2[1] + 6), order="F")
    P2[0] = 1.0
    P2[1] = 1e-3 / (gamma - 1)
    s = Solver(2, n2, gamma, (1.0 / 256, 1.0 / 256), recon="wenoz", riemann="hllc", rk=3, n_iter=50, tol=1e-12,
               floor=1e-8)
    s.set_boundary(0, L.BC_NOZZLE, [8.0, n2[1] / 2, 0.0, 0.01, 1e-3 / (gamma - 1), math.sqrt(99.0), 0.0])
    s.load_prims(P2)
    for _ in range(4):
        s.step(0.4 / (2 * 256), 100)
        a = s.prims()[:, 3:-3, 3:-3].reshape(4, -1)
        q = np.zeros((5, a.shape[1]))
        q[0:2] = a[0:2]
        q[2:4] = a[2:4]
        out.append(q)
    s.close()
    Q = np.concatenate(out, axis=1)
    # keep physical states only (a run may leave NaN cells where its con2prim failed)
    good = np.isfinite(Q).all(0) & (Q[0] > 0) & (Q[1] > 0)
    Q = Q[:, good]
    if Q.shape[1] > max_states:
        Q = Q[:, np.random.default_rng(0).choice(Q.shape[1], max_states, replace=False)]
    return torch.from_numpy(np.ascontiguousarray(Q)).cuda()


class MLP:
    """Owner of one network on the current device (vb_mlp_handle)."""

    def __init__(self, params=None, norm=None, seed=0):
        self.lib = _sig()
        h = C.c_void_p()
        _chk(self.lib.vb_mlp_create(C.byref(h)))
        self._h = h
        self.norm = np.array([0, 0, 0, 0, 1, 1, 1, 1], dtype=np.float32) if norm is None else np.asarray(norm, np.float32)
        self.set_params(init_params(seed) if params is None else params, self.norm)

    def set_params(self, params, norm=None):
        p = np.ascontiguousarray(params, dtype=np.float32)
        if norm is not None:
            self.norm = np.ascontiguousarray(norm, dtype=np.float32)
        fp = C.POINTER(C.c_float)
        _chk(self.lib.vb_mlp_set_params(self._h, p.ctypes.data_as(fp), self.norm.ctypes.data_as(fp), None), self._h)

    def params(self) -> np.ndarray:
        out = np.zeros(n_params(), dtype=np.float32)
        nrm = np.zeros(8, dtype=np.float32)
        fp = C.POINTER(C.c_float)
        _chk(self.lib.vb_mlp_get_params(self._h, out.ctypes.data_as(fp), nrm.ctypes.data_as(fp), None), self._h)
        return out

    def grad(self) -> np.ndarray:
        out = np.zeros(n_params(), dtype=np.float32)
        _chk(self.lib.vb_mlp_get_grad(self._h, out.ctypes.data_as(C.POINTER(C.c_float)), None), self._h)
        return out

    def features(self, U, P=None, gamma=4.0 / 3.0, with_weight=False):
        """U, P: (5, n) FP64 CUDA tensors -> (feat (n, 4), target (n,) or None[, weight (n,)])."""
        import torch

        n = U.shape[1]
        feat = torch.empty((n, 4), dtype=torch.float32, device="cuda")
        tgt = torch.empty(n, dtype=torch.float32, device="cuda") if P is not None else None
        wgt = torch.empty(n, dtype=torch.float32, device="cuda") if (P is not None and with_weight) else None
        _chk(self.lib.vb_mlp_features(self._h, _ptr(U.contiguous()), _ptr(P.contiguous()) if P is not None else None,
                                      n, gamma, _ptr(feat), _ptr(tgt) if tgt is not None else None,
                                      _ptr(wgt) if wgt is not None else None, None), self._h)
        return (feat, tgt, wgt) if with_weight else (feat, tgt)

    def forward(self, feat):
        import torch

        n = feat.shape[0]
        out = torch.empty(n, dtype=torch.float32, device="cuda")
        _chk(self.lib.vb_mlp_forward(self._h, _ptr(feat.contiguous()), n, _ptr(out), None), self._h)
        return out

    def train_step(self, feat, target, lr, weight=None):
        loss = C.c_float()
        _chk(self.lib.vb_mlp_train_step(self._h, _ptr(feat), _ptr(target), _ptr(weight) if weight is not None else None,
                                        feat.shape[0], float(lr), C.byref(loss), None), self._h)
        return loss.value

    def fit_norm(self, U, gamma):
        """Set the feature normalisation to the mean / std of the raw features of U."""
        import torch

        self.norm = np.array([0, 0, 0, 0, 1, 1, 1, 1], dtype=np.float32)
        self.set_params(self.params(), self.norm)
        raw, _ = self.features(U, None, gamma)
        raw = raw[torch.isfinite(raw).all(1)]
        if raw.shape[0] < 16:
            raise ValueError("fit_norm: fewer than 16 states with finite features")
        mu = raw.mean(0).double().cpu().numpy()
        sd = raw.std(0).double().cpu().numpy()
        sd = np.where(sd > 1e-6, sd, 1.0)
        self.norm = np.concatenate([mu, 1.0 / sd]).astype(np.float32)
        self.set_params(self.params(), self.norm)
        del torch

    def train(self, n_samples=1 << 24, gammas=(4.0 / 3.0, 5.0 / 3.0), epochs=4, batch=1 << 12, lr=3e-3, seed=0,
              snapshots=True, log=None):
        """Train on synthetic states (+ solver snapshots); returns the loss history per epoch."""
        import torch

        feats, tgts = [], []
        Ps = []
        for gi, g in enumerate(gammas):
            P = synthetic_states(n_samples // len(gammas), g, seed=seed + gi)
            if snapshots:
                P = torch.cat([P, solver_snapshots(g, max_states=n_samples // (8 * len(gammas)))], dim=1)
            Ps.append((P, g))
        allU = torch.cat([prim2con_torch(P, g) for P, g in Ps], dim=1)
        # normalisation from the first gamma's states, then features of every set
        self.fit_norm(prim2con_torch(Ps[0][0], Ps[0][1]), Ps[0][1])
        del allU
        wgts = []
        for P, g in Ps:
            f, t, w = self.features(prim2con_torch(P, g), P, g, with_weight=True)
            ok = torch.isfinite(t) & torch.isfinite(f).all(1) & torch.isfinite(w)
            feats.append(f[ok])
            tgts.append(t[ok])
            wgts.append(w[ok])
        F = torch.cat(feats)
        T = torch.cat(tgts)
        Wt = torch.cat(wgts)
        n = F.shape[0]
        if n < batch:
            raise ValueError(f"train: only {n} usable samples for batch {batch}")
        # start the output layer at the target's mean and scale
        prm = split_params(self.params())
        tm = float((T * Wt).sum() / Wt.sum())
        ts = float(torch.sqrt(((T - tm) ** 2 * Wt).sum() / Wt.sum()))
        prm["b4"][:] = tm
        prm["w4"][:] = prm["w4"] * ts
        self.set_params(np.concatenate([prm[k].ravel() for k in ("W1", "b1", "W2", "b2", "W3", "b3", "w4", "b4")]))
        gen = torch.Generator(device="cuda")
        gen.manual_seed(seed)
        hist = []
        step = 0
        total_steps = epochs * max(1, n // batch)
        for ep in range(epochs):
            perm = torch.randperm(n, generator=gen, device="cuda")
            tot = 0.0
            nb = 0
            for b0 in range(0, n - batch + 1, batch):
                idx = perm[b0:b0 + batch]
                # cosine learning-rate schedule
                lr_t = lr * 0.5 * (1 + math.cos(math.pi * step / total_steps))
                tot += self.train_step(F[idx].contiguous(), T[idx].contiguous(), lr_t, Wt[idx].contiguous())
                nb += 1
                step += 1
            hist.append(tot / max(nb, 1))
            if log:
                log(f"epoch {ep}: mse {hist[-1]:.3e}")
        return hist

    def evaluate(self, n=1 << 16, gamma=4.0 / 3.0, seed=99, lorentz_max=50.0):
        """Held-out quality of the guess: relative W0 error (median, 99th
        percentile) and the bracketed W Newton's mean iterations and
        fallbacks from it, on n synthetic states that no training set draws
        (seed 99, Lorentz factor up to lorentz_max)."""
        P = synthetic_states(n, gamma, seed=seed, lorentz_max=lorentz_max)
        U = prim2con_torch(P, gamma)
        f, _ = self.features(U, None, gamma)
        y = self.forward(f).double()
        W0 = -U[1] * (1 + y.clamp(min=0))
        Wt = (gamma - 1) * P[1] - U[1]
        err = ((W0 - Wt) / Wt).abs()
        _, it, fb = c2p_w(U, W0, gamma)
        it = it.double()
        return {"w0_rel_err_median": err.median().item(), "w0_rel_err_p99": err.quantile(0.99).item(),
                "newton_iters_mean": it[it > 0].mean().item(), "fallbacks": int(fb.sum().item()),
                "failures": int((it <= 0).sum().item()), "states": n}

    def save(self, path=DEFAULT_WEIGHTS):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez(path, params=self.params(), norm=self.norm)

    @classmethod
    def load(cls, path=DEFAULT_WEIGHTS):
        d = np.load(path)
        return cls(params=d["params"], norm=d["norm"])

    def attach(self, solver):
        _chk(self.lib.vb_attach_mlp(solver._h, self._h))
        solver._mlp = self  # keep the network alive while the solver uses it

    def close(self):
        if getattr(self, "_h", None):
            self.lib.vb_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def c2p_w(U, W0, gamma, rtol=1e-12, max_newton=8, max_bracket=200):
    """vb_point_c2p_w on (5, n) / (n,) FP64 CUDA tensors -> (P, iterations, fallback)."""
    import torch

    lib = _sig()
    n = U.shape[1]
    P = torch.empty_like(U)
    it = torch.empty(n, dtype=torch.int32, device="cuda")
    fb = torch.empty(n, dtype=torch.int32, device="cuda")
    _chk(lib.vb_point_c2p_w(gamma, _ptr(U.contiguous()), _ptr(W0.contiguous()), rtol, max_newton, max_bracket, _ptr(P),
                            _ptr(it), _ptr(fb), n, None))
    return P, it, fb


def c2p_gated(U, W0, gamma, rtol=1e-12, max_newton=8, max_bracket=200):
    """vb_point_c2p_gated on (5, n) FP64 / (n,) FP32 CUDA tensors -> (P, iterations, fp64 flag)."""
    import torch

    lib = _sig()
    n = U.shape[1]
    P = torch.empty_like(U)
    it = torch.empty(n, dtype=torch.int32, device="cuda")
    f64 = torch.empty(n, dtype=torch.int32, device="cuda")
    W0 = W0.to(torch.float32).contiguous()
    _chk(lib.vb_point_c2p_gated(gamma, _ptr(U.contiguous()), _ptr(W0), rtol, max_newton, max_bracket, _ptr(P),
                                _ptr(it), _ptr(f64), n, None))
    return P, it, f64


_cached = {}


def available() -> bool:
    try:
        import torch

        return torch.cuda.is_available() and os.path.exists(L.LIB_PATH)
    except Exception:
        return False


def trained(path=DEFAULT_WEIGHTS, train_if_missing=True, log=None) -> MLP:
    """The network for the current device: loaded from `path`, or trained now."""
    import torch

    dev = torch.cuda.current_device()
    if dev in _cached:
        return _cached[dev]
    if os.path.exists(path):
        m = MLP.load(path)
    elif train_if_missing:
        m = MLP()
        m.train(log=log)
    else:
        raise FileNotFoundError(path)
    _cached[dev] = m
    return m


def attach(solver, log=None):
    trained(log=log).attach(solver)


def main(argv=None):
    """Train the default network on the current GPU and save it."""
    import argparse
    import time

    ap = argparse.ArgumentParser(description="train the learned con2prim guess and save its weights")
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--samples", type=int, default=1 << 24)
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--evaluate", action="store_true", help="print the held-out W0 error and Newton iterations")
    ap.add_argument("--no-save", action="store_true", help="train (and evaluate) without writing the weights")
    a = ap.parse_args(argv)
    t0 = time.time()
    m = MLP(seed=a.seed)
    hist = m.train(n_samples=a.samples, epochs=a.epochs, seed=a.seed, log=print)
    t_train = time.time() - t0
    if not a.no_save:
        m.save(a.out)
        print(f"saved {a.out}")
    print(f"{n_params()} parameters, {a.samples} samples x {a.epochs} epochs, loss per epoch {hist}, "
          f"{t_train:.1f} s")
    if a.evaluate:
        print("held-out:", m.evaluate())


if __name__ == "__main__":
    main()
