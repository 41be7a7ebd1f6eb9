"""The two large configurations against the CPU oracle, substep by substep:

* 128^3 V60 pour with the spout on the spiral path (1.5 cm, 0.5 Hz), tile-sorted P2G,
  ~2.2M samples;
* 192^3 V60 pour with the two-layer bed (porosity 0.45 / 0.35, 10x lower permeability
  below), the pour 1.2 cm off centre and int64 fixed-point P2G, ~7.8M samples.

Both run the FP32 refinement solve to a relative residual of 1e-5; at these sizes the
engine solves with the grid-wide solve.  The oracle (OpenMP on the host cores) runs the
same substeps; pair counts, the int64 lanes, pressure, grid velocity and every sample
must agree bit for bit."""
import numpy as np
import pytest

from coffee_sim_b200 import scenes
from coffee_sim_b200.sim import MpmSim3D
from helpers import mismatch, relerr

pytestmark = pytest.mark.gpu


def _compare(e, o, what, int64=False):
    me, mo = e.latest_metrics(), o.latest_metrics()
    assert me.last_sweeps == mo.last_sweeps > 0, (what, me.last_sweeps, mo.last_sweeps)
    assert me.residual_checks == mo.residual_checks, what
    assert me.last_residual <= 1e-5 and me.timeout_flag == 0 and me.nan_flag == 0, what
    assert e.particle_count() == o.particle_count(), what
    if int64:
        assert mismatch(e.read_grid_lanes64(), o.read_grid_lanes64()) == 0, what
    for name, a, b in (("pressure", e.read_pressure(), o.read_pressure()),
                       ("grid_vel", e.read_grid_vel(), o.read_grid_vel()),
                       ("particles", e.read_particles(), o.read_particles())):
        assert mismatch(a, b) == 0, (what, name, mismatch(a, b), relerr(a, b))


def test_c3_spiral_pour_matches_oracle(engine, oracle):
    """128^3, spiral spout path, device emission: three substeps bit-exact."""
    sims = []
    for lib in (engine, oracle):
        s = scenes.c3_large(lib)
        s.raw.rbgs_omega = 1.94
        s.raw.max_sweeps = 8000
        s.raw.check_every = 40
        s.raw.device_emission = 1
        sims.append(MpmSim3D(s, lib))
    e, o = sims
    assert scenes.populate_c2(e, seed=2) == scenes.populate_c2(o, seed=2) > 2_000_000
    for k in range(3):
        for sim in sims:
            sim.set_spout_position(*scenes.spiral_spout(k * scenes.C2_DT))
            sim.step_substep(scenes.C2_DT)
        _compare(e, o, f"c3 substep {k}")
    e.close()
    o.close()


def test_c5_two_layer_bed_int64_matches_oracle(engine, oracle):
    """192^3, two-layer bed, off-centre pour, int64 P2G: two substeps bit-exact,
    int64 lanes included."""
    sims = []
    for lib in (engine, oracle):
        s = scenes.c5_scale(lib)
        s.raw.rbgs_omega = 1.95
        s.raw.max_sweeps = 12000
        s.raw.check_every = 40
        s.raw.device_emission = 1
        sims.append(MpmSim3D(s, lib))
    e, o = sims
    assert scenes.populate_c2(e, seed=4) == scenes.populate_c2(o, seed=4) > 7_000_000
    assert e.num_bed == o.num_bed == 81000
    for k in range(2):
        for sim in sims:
            sim.step_substep(scenes.C2_DT)
        _compare(e, o, f"c5 substep {k}", int64=True)
    e.close()
    o.close()
