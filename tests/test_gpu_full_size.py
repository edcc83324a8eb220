"""The workloads of the benchmark configurations at their full sizes, checked
through properties that hold at any size (the oracle's CPU cost rules out a
cell-by-cell comparison there; that comparison runs at small sizes in
test_gpu_parity.py):

* 2D relativistic jet, 4096^2, FP64, WENOZ + HLLC, SSP-RK3, CFL 0.4, 200
  steps: no con2prim failure, positive density and internal energy, and the
  mirror symmetry about the jet axis of a noise-free ambient with a centred
  nozzle (u^y odd, everything else even). Mirrored faces add their terms in
  different orders, so the symmetry holds to rounding, which the shear layer
  of the jet amplifies over the run: measured 2.2e-10 of each field's
  maximum after 200 steps, bound 1e-8;
* 3D relativistic jet, 512^3, PPM + HLLC, SSP-RK3, 100 steps: the FP32-bulk
  form against the all-FP64 run, L1 density error <= 1e-5 (the precision
  form's bar), L1 pressure and max Lorentz-factor errors reported and bounded
  (the max error sits on the jet's discontinuities, which FP32 rounding
  shifts by a fraction of a cell: 1.3e-2 at Lorentz factor 10, bound 0.1);
* the same jet with WENOZ and the learned con2prim guess on the FP32 bulk:
  L1 density error <= 1e-5 against the FP64 run, no failure;
* 256 uneven 1D/2D Riemann problems in one persistent launch (FP32 bulk):
  no timeout, every state finite, and the FP32 batch within L1 density 1e-5
  of the FP64 batch on all but a few extreme 1D tubes. Some of the seeded
  tubes (|v| up to 0.9 against pressure ratios up to 2e5) make the
  reference's 1D Newton diverge in a few cells; the FP64 batch keeps the
  reference con2prim (parity with the single-grid solver) and solves those
  cells with the bracketed W Newton (counted as fallbacks; the single-grid
  solver keeps the reference's values and counts them as failures). The FP32
  batch runs the W Newton first and the reference Newton as its fallback. On
  four tubes the reference Newton converges, in the cells behind the
  strongest collisions, to a negative-pressure root that the floors then lift,
  where the W Newton finds the physical root: those tubes differ by up to
  3e-3 in L1 density; the others agree to 4.7e-7. Cells with no root at all
  keep their input state and are counted as failures (a handful in 7.9e8
  cell updates)."""
import numpy as np
import pytest

from helpers import nozzle_params

pytestmark = pytest.mark.gpu


def _l1(a, b):
    return float((a - b).abs().mean() / b.abs().mean())


def test_config2_2d_jet_4096_fp64_mirror_symmetry():
    import torch

    from verona_b200 import Solver

    g, N = 4.0 / 3.0, 4096
    s = Solver(2, (N, N), g, (1.0 / N, 1.0 / N), recon="wenoz", riemann="hllc", rk=3, n_iter=50, tol=1e-12,
               floor=1e-8)
    s.init_prims("ambient", rho=1.0, u=1e-3 / (g - 1), noise=0.0)
    s.set_boundary(0, 2, nozzle_params(2, (N, N), 32.0, gamma=g))
    s.step(0.4 / (2.0 * N), 200)
    P = s.store_prims()  # (Ny+6, Nx+6, 4)
    torch.cuda.synchronize()
    cnt = s.counters()
    assert cnt[0] == 0 and torch.isfinite(P).all()
    inner = P[3:-3, 3:-3]
    assert (inner[..., 0] > 0).all() and (inner[..., 1] > 0).all()
    M = P.flip(0)
    sign = torch.tensor([1.0, 1.0, 1.0, -1.0], dtype=P.dtype, device=P.device)
    err = [float(((P[..., v] - sign[v] * M[..., v]).abs().max() / P[..., v].abs().max().clamp(min=1e-300)))
           for v in range(4)]
    jet = float((inner[..., 2] > 1.0).float().mean())
    print("2D 4096^2 after 200 steps: mirror asymmetry per field", err, "jet cell fraction", jet)
    assert max(err) <= 1e-8 and jet > 0


def _jet3d(prec, recon, guess="previous", steps=100, n=512):
    import torch

    from verona_b200 import Solver, mlp

    g = 4.0 / 3.0
    s = Solver(3, (n, n, n), g, (1.0 / n,) * 3, recon=recon, riemann="hllc", rk=3, precision=prec, guess=guess,
               n_iter=50, tol=1e-12, floor=1e-8)
    if guess == "learned":
        mlp.attach(s)
    s.init_prims("ambient", rho=1.0, u=1e-3 / (g - 1), noise=0.03, seed=42)
    s.set_boundary(0, 2, nozzle_params(3, (n, n, n), 16.0, gamma=g))
    s.step(0.4 / (3.0 * n), steps)
    P = s.store_prims()[3:-3, 3:-3, 3:-3]
    torch.cuda.synchronize()
    cnt = s.counters()
    s.close()
    return P, cnt


def _errors(a, b):
    import torch

    la = torch.sqrt(1 + (a[..., 2:] ** 2).sum(-1))
    lb = torch.sqrt(1 + (b[..., 2:] ** 2).sum(-1))
    return _l1(a[..., 0], b[..., 0]), _l1(a[..., 1], b[..., 1]), float((la - lb).abs().max())


def test_config3_3d_jet_512_ppm_fp32_bulk_against_fp64():
    import torch

    P64, c64 = _jet3d("fp64", "ppm")
    P32, c32 = _jet3d("fp32", "ppm")
    assert c64[0] == 0 and c32[0] == 0 and torch.isfinite(P32).all()
    l1r, l1p, dl = _errors(P32, P64)
    print("512^3 PPM+HLLC 100 steps, FP32 bulk vs FP64: L1 rho %.3e L1 p %.3e max |dGamma| %.3e" % (l1r, l1p, dl))
    assert l1r <= 1e-5 and l1p <= 1e-4 and dl <= 0.1


def test_config4_learned_guess_in_the_512_wenoz_jet():
    import torch

    P64, c64 = _jet3d("fp64", "wenoz", steps=20)
    Pl, cl = _jet3d("fp32", "wenoz", guess="learned", steps=20)
    assert c64[0] == 0 and cl[0] == 0 and cl[4] == 0 and torch.isfinite(Pl).all()
    l1r, l1p, dl = _errors(Pl, P64)
    print("512^3 WENOZ+HLLC 20 steps, learned + FP32 vs FP64: L1 rho %.3e L1 p %.3e max |dGamma| %.3e"
          % (l1r, l1p, dl))
    assert l1r <= 1e-5 and l1p <= 1e-4


def test_config5_batch_of_256_uneven_problems_fp32_against_fp64():
    from verona_b200.batch import Batch, riemann_problems

    specs, prims = riemann_problems(42, gamma=5.0 / 3.0)
    assert len(specs) == 256
    out = {}
    for prec in ("fp64", "fp32"):
        b = Batch(specs, 5.0 / 3.0, riemann="hllc", rk=3, precision=prec, n_iter=50, tol=1e-12, floor=1e-8)
        for i, P in enumerate(prims):
            b.load_prims(i, P)
        b.step(10)
        cnt = b.counters()
        cells = b.info()["interior_cells"]
        print(prec, "batch counters", cnt.tolist(), "of", cells * 30, "cell updates")
        assert cnt[4] == 0 and cnt[5] == 0, cnt
        # cells the reference's Newton loses are recovered by the rescue; a few
        # conserved states have no physical root and keep their input state
        assert cnt[0] <= 1e-5 * cells * 30, cnt
        out[prec] = [b.prims(i) for i in range(len(specs))]
        b.close()
    errs = []
    for a, r in zip(out["fp32"], out["fp64"]):
        assert np.all(np.isfinite(a)) and np.all(np.isfinite(r))
        errs.append(float(np.mean(np.abs(a[0] - r[0])) / np.mean(np.abs(r[0]))))
    errs = np.array(errs)
    outliers = np.nonzero(errs > 1e-5)[0]
    print("batch of 256 problems, 10 steps: per-problem L1 rho FP32 vs FP64: median %.3e, 90%% %.3e, worst %.3e "
          "(problem %d), above 1e-5: %s" % (np.median(errs), np.quantile(errs, 0.9), errs.max(), errs.argmax(),
                                             np.nonzero(errs > 1e-5)[0].tolist()))
    assert len(outliers) <= 8 and all(specs[i]["dims"] == 1 for i in outliers), outliers
    assert np.median(errs) <= 1e-7 and np.delete(errs, outliers).max() <= 1e-5


def test_jet_128_fp32_and_learned_against_the_oracle():
    """The 3D jet at 128^3 (WENOZ + HLLC, SSP-RK3, nozzle radius 4 cells,
    Lorentz 10, ambient with 3 % density noise), 5 steps, with the errors
    taken directly against the C FP64 oracle run from the same initial state:
    the plain FP64 path within 1e-10 per field, the FP32-bulk form and the
    learned guess + FP32 bulk within L1 density 1e-5 (the precision form's
    bar) and L1 pressure 1e-4."""
    from helpers import per_field_rel
    from oracle import oracle as O
    from verona_b200 import Solver, mlp

    g, n, steps = 4.0 / 3.0, 128, 5
    dxs = (1.0 / n,) * 3
    dt = 0.4 / (3.0 * n)
    noz = nozzle_params(3, (n, n, n), 4.0, gamma=g)
    got, P0 = {}, None
    for prec, guess in (("fp64", "previous"), ("fp32", "previous"), ("fp32", "learned")):
        s = Solver(3, (n, n, n), g, dxs, recon="wenoz", riemann="hllc", rk=3, precision=prec, guess=guess, n_iter=50,
                   tol=1e-12, floor=1e-8)
        if guess == "learned":
            mlp.attach(s)
        s.init_prims("ambient", rho=1.0, u=1e-3 / (g - 1), noise=0.03, seed=42)
        if P0 is None:
            P0 = s.prims()
        s.set_boundary(0, 2, noz)
        s.step(dt, steps)
        got[(prec, guess)] = s.prims()
        assert s.counters()[0] == 0
        s.close()
    o = O.SolverND(3, (n, n, n), P0, g, 1e-8, 50, 1e-12, O.WENOZ, O.HLLC, 3)
    o.set_grid(*dxs)
    o.set_boundary(0, O.BC_NOZZLE, noz)
    o.step(dt, steps)
    ref = o.prims()
    e64 = per_field_rel(got[("fp64", "previous")], ref)
    print("128^3 FP64 vs oracle: max rel per field", e64, "differing values:",
          int(np.sum(got[("fp64", "previous")] != ref)))
    assert max(e64) <= 1e-10
    r = ref[:, 3:-3, 3:-3, 3:-3]
    lr = np.sqrt(1 + (r[2:] ** 2).sum(0))
    for key in (("fp32", "previous"), ("fp32", "learned")):
        a = got[key][:, 3:-3, 3:-3, 3:-3]
        l1r = float(np.mean(np.abs(a[0] - r[0])) / np.mean(np.abs(r[0])))
        l1p = float(np.mean(np.abs(a[1] - r[1])) / np.mean(np.abs(r[1])))
        dl = float(np.max(np.abs(np.sqrt(1 + (a[2:] ** 2).sum(0)) - lr)))
        print("128^3 %s + %s guess vs oracle: L1 rho %.3e L1 p %.3e max |dGamma| %.3e" % (key + (l1r, l1p, dl)))
        assert np.all(np.isfinite(a)) and l1r <= 1e-5 and l1p <= 1e-4
