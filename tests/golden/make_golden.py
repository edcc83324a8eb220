"""Generate the golden fixtures of tests/golden/ (run from the repo root:
`python tests/golden/make_golden.py`).

  mm1_star.json     exact star state of Marti & Mueller (1994) problem 1
                    (rho_L=10, p_L=13.33, rho_R=1, p_R=1e-6, G=5/3) from
                    oracle/exact_riemann.py, next to the values published in
                    Marti & Mueller, Living Rev. Relativ. 6, 7 (2003), table 2.
  oracle_small.npz  oracle outputs of small runs of every solver mode, the
                    fixed vectors the CPU tests (oracle regressions) and the
                    GPU parity tests (through the C ABI) compare against.

The reference itself (Julia) cannot run here and ships no fixtures; these
vectors pin the restatement, not the reference.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from helpers import jet_ic, nozzle_params, shock_tube_1d  # noqa: E402
from oracle import exact_riemann as ER  # noqa: E402
from oracle import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

# cases: name -> dict(kind, params)
CASES_1D = [(rec, 64, 20) for rec in ("minmod", "ppm", "wenoz")]
CASES_ND = [
    # dims, n, recon, riemann, rk, steps
    (2, (24, 20, 1), O.WENOZ, O.HLL, 2, 6),
    (2, (24, 20, 1), O.PPM, O.HLLC, 3, 4),
    (2, (24, 20, 1), O.MINMOD, O.HLL, 3, 4),
    (3, (12, 10, 8), O.WENOZ, O.HLL, 2, 3),
    (3, (12, 10, 8), O.PPM, O.HLLC, 3, 2),
    (3, (12, 10, 8), O.MINMOD, O.HLLC, 2, 2),
]


def nd_case_name(c):
    dims, n, rec, rs, rk, steps = c
    return f"nd{dims}_{'x'.join(map(str, n[:dims]))}_r{rec}_s{rs}_rk{rk}_n{steps}"


def run_nd_case(c):
    dims, n, rec, rs, rk, steps = c
    g = 4.0 / 3.0
    P = jet_ic(dims, n, gamma=g, noise=0.03, seed=7)
    s = O.SolverND(dims, n[:dims], P, g, 1e-8, 50, 1e-12, rec, rs, rk)
    dxs = [1.0 / n[a] for a in range(dims)] + [1.0] * (3 - dims)
    s.set_grid(*dxs)
    s.set_boundary(0, O.BC_NOZZLE, nozzle_params(dims, n, 3.0, gamma=g))
    dt = 0.4 / sum(1.0 / d for d in dxs[:dims])
    s.step(dt, steps)
    return P, s.prims(), s.cons(), dt, dxs


def run_1d_case(rec, N, steps):
    g = 5.0 / 3.0
    x, rho, u, ux = shock_tube_1d(N, gamma=g)
    s = O.Solver1DRef(rho, u, ux, g, rec, 50, 1e-12)
    dx = 1.0 / N
    dt = 0.4 * dx
    s.step(dt, dx, steps)
    return np.stack([rho, u, ux]), s.prims(), s.cons(), dt, dx


def main():
    O.build()
    ps, vs, rl, rr, sl, sr = ER.star_state(10.0, 13.33, 0.0, 1.0, 1e-6, 0.0, 5.0 / 3.0)
    star = {
        "exact": {"p_star": ps, "v_star": vs, "rho_L_star": rl, "rho_R_star": rr, "shock_R": sr},
        "published": {"p_star": 1.448, "v_star": 0.714, "rho_L_star": 2.639, "rho_R_star": 5.070,
                      "shock_R": 0.828},
        "source": "Marti & Mueller, Living Rev. Relativ. 6, 7 (2003), problem 1 (p_R = 0 there)",
    }
    with open(os.path.join(HERE, "mm1_star.json"), "w") as f:
        json.dump(star, f, indent=1)

    arrays = {}
    for rec, N, steps in CASES_1D:
        P0, P, U, dt, dx = run_1d_case(rec, N, steps)
        arrays[f"r1d_{rec}_P"] = P
        arrays[f"r1d_{rec}_U"] = U
    for c in CASES_ND:
        P0, P, U, dt, dxs = run_nd_case(c)
        name = nd_case_name(c)
        arrays[name + "_P"] = P
        arrays[name + "_U"] = U
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), **arrays)
    print("wrote", len(arrays), "arrays")


if __name__ == "__main__":
    main()
