"""CPU tests of the host-side mirror logic (no GPU)."""
from verona_b200 import _lib as L
from verona_b200._harm import steps_until_dump


def _julia_loop(dt, Tmax, drops):
    """The reference's loop (src/3dim/algos.jl:274-359) as plain Python:
    returns the step indices after which a dump happens."""
    t, thres, step, dumps = 0.0, drops, 0, []
    while t < Tmax:
        t += dt
        step += 1
        if t > thres:
            thres += drops
            dumps.append((step, t))
    return step, dumps


def test_dump_schedule_matches_the_reference_loop():
    for dt, Tmax, drops in ((0.4 / 1024, 0.4, 0.4 / 3), (0.1, 1.0, 0.25), (0.37, 480.0, 0.48), (1e-3, 0.0305, 1e-2)):
        ref_steps, ref_dumps = _julia_loop(dt, Tmax, drops)
        t, thres, total, dumps = 0.0, drops, 0, []
        while t < Tmax:
            n, t = steps_until_dump(t, dt, Tmax, thres)
            total += n
            if t > thres:
                thres += drops
                dumps.append((total, t))
        assert total == ref_steps
        assert dumps == ref_dumps


def test_turnoff_boundary_specs():
    from verona_b200 import Verona2D, Verona3D

    b3 = Verona3D.turnoff_boundary(0.01, 48.0, 480.0)
    assert b3[0] == (0, L.BC_FIXED, (2, 160.0, 480.0, 1 - 0.01 / 48.0))
    assert sorted(f for f, k, _ in b3[1:]) == [1, 2, 3, 4, 5]
    b2 = Verona2D.turnoff_boundary(0.01, 80.0, 800.0)
    assert b2[0][2][0] == 3  # the 2D example decays P[4] (u^y)
