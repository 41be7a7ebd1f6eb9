"""The FP64 residual-check schedule of the refinement solve, on the oracle (the engine
follows the same rule; tests/test_parity_gpu.py compares their pair and check counts).

A solve checks after `first_check` pairs (or `check_every` when it is 0), then after the
pairs its decay rate predicts, at least 2 and at most `check_every`."""
from coffee_sim_b200 import scenes
from coffee_sim_b200.sim import MpmSim3D


def _v60(lib, first, ce=10):
    s = scenes.c2_v60(lib, grid=32, max_particles=60000)
    s.raw.rbgs_omega = 1.9
    s.raw.check_every = ce
    s.raw.first_check = first
    s.raw.max_sweeps = 2000
    sim = MpmSim3D(s, lib)
    scenes.populate_c2(sim)
    return sim


def test_first_check_runs_a_full_first_cycle(oracle):
    """The first cycle runs exactly `first_check` pairs even where the target would be
    met earlier; predicted cycles of at most check_every (10) pairs follow when it is not
    (one FP32 correction cycle cannot take the FP64 residual much below ~1e-4 of its
    starting value: the cold first substep needs 330 and 830 pairs)."""
    for first in (300, 800):
        sim = _v60(oracle, first=first)
        for k in range(2):
            sim.step_substep(scenes.C2_DT)
            m = sim.latest_metrics()
            assert m.last_sweeps >= first and m.residual_checks >= 2, (first, m.last_sweeps, m.residual_checks)
            assert m.residual_checks - 2 >= -(-(m.last_sweeps - first) // 10)
            if k == 0:
                assert m.last_sweeps > first  # the cold start does not converge in one cycle
            assert m.last_residual <= 1e-5


def test_first_check_shortens_the_first_cycle(oracle):
    """With a short first interval the solve checks early, then predicts; it reaches the
    target with intervals of at most check_every after the first."""
    ce = 40
    a, b = _v60(oracle, first=0, ce=ce), _v60(oracle, first=6, ce=ce)
    for _ in range(2):
        a.step_substep(scenes.C2_DT)
        b.step_substep(scenes.C2_DT)
        ma, mb = a.latest_metrics(), b.latest_metrics()
        assert ma.last_residual <= 1e-5 and mb.last_residual <= 1e-5
        # b: 6 pairs, then at most ce per cycle
        assert mb.residual_checks >= 3
        assert mb.residual_checks - 2 >= -(-(mb.last_sweeps - 6) // ce)
        assert ma.residual_checks - 1 >= -(-ma.last_sweeps // ce)
