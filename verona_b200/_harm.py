"""The HARM_HLL time loop shared by the Verona1D/2D/3D mirrors.

It keeps the reference's control flow (src/3dim/algos.jl:274-359): a dump at
t = 0, `while t < Tmax`, t += dt after each step, a dump whenever
t > thres_to_dump. Steps between dumps run on the device in one vb_step
call; the host replays the same t accumulation to know where the dumps fall.
"""
from __future__ import annotations


def steps_until_dump(t: float, dt: float, Tmax: float, thres: float) -> tuple[int, float]:
    n = 0
    while t < Tmax:
        t += dt
        n += 1
        if t > thres:
            break
    return n, t


def run_loop(solver, dt, Tmax, drops, dump, verbose=False):
    """Returns the number of dumps after the initial one (HARM_HLL's return value)."""
    import time

    t = 0.0
    thres = drops
    i = 0
    if dump is not None:
        dump(i, t, solver)
    t0 = time.time()
    while t < Tmax:
        n, t_new = steps_until_dump(t, dt, Tmax, thres)
        solver.step(dt, n)
        t = t_new
        if t > thres:
            i += 1
            thres += drops
            if verbose:
                print(f"{t:.3g} elapsed: {time.time() - t0:.3g} s")
                t0 = time.time()
            if dump is not None:
                dump(i, t, solver)
    return i
