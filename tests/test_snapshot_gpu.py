"""Snapshots: saving the engine's state and loading it back replays the following
substeps bit for bit, in the same simulation and in a new one with the same settings
(the bench replays its timed window this way)."""
import pytest

from coffee_sim_b200 import scenes
from coffee_sim_b200.sim import MpmSim3D
from helpers import mismatch

pytestmark = pytest.mark.gpu


def _state(sim):
    n = sim.particle_count()
    d = {"particles": sim.read_particles(0, n), "affine": sim.read_affine(0, n), "pressure": sim.read_pressure()}
    if sim.num_bed:
        d["bed_extract"] = sim.read_bed_extract(0, sim.num_bed)
    return d


def _run(sim, k):
    sweeps = []
    for _ in range(k):
        sim.step_substep(scenes.C2_DT)
        sweeps.append(sim.latest_metrics().last_sweeps)
    return sweeps


def _same(a, b):
    assert a.keys() == b.keys()
    for key in a:
        assert a[key].shape == b[key].shape, key
        assert mismatch(a[key], b[key]) == 0, key


def test_snapshot_replays_bit_exact(engine):
    s = scenes.c2_v60(engine, grid=32, max_particles=60000)
    sim = MpmSim3D(s, engine)
    scenes.populate_c2(sim)
    _run(sim, 3)
    blob = sim.snapshot()
    sweeps_a = _run(sim, 3)
    a = _state(sim)
    sim.restore(blob)
    sweeps_b = _run(sim, 3)
    assert sweeps_a == sweeps_b
    _same(a, _state(sim))

    other = MpmSim3D(s, engine)
    other.restore(blob)
    assert _run(other, 3) == sweeps_a
    _same(a, _state(other))


def test_snapshot_rejects_other_sizes(engine):
    s = scenes.c2_v60(engine, grid=32, max_particles=60000)
    sim = MpmSim3D(s, engine)
    blob = sim.snapshot()
    t = scenes.c2_v60(engine, grid=32, max_particles=50000)
    other = MpmSim3D(t, engine)
    with pytest.raises(Exception):
        other.restore(blob)
    with pytest.raises(Exception):
        sim.restore(blob[:64])


def test_snapshot_restores_the_spout_and_kettle(engine):
    """The spout position and target (set_spout_position / set_spout_target, mod.rs:452-458)
    and the kettle angle are part of the saved state: frames after a restore pour from
    where the spout was when the snapshot was taken."""
    from coffee_sim_b200.sim import MpmSettings
    sim = MpmSim3D(MpmSettings.benchmark_free_stream(engine), engine)
    sim.set_kettle_angle(36.0)
    for _ in range(3):
        sim.step_frame(1.0 / 60.0)
    blob = sim.snapshot()
    pos = sim.spout_position()
    for f in range(3):
        sim.set_spout_position(-0.1 * (f + 1), 6.8, 0.0)
        sim.step_frame(1.0 / 60.0)
    moved = _state(sim)
    sim.restore(blob)
    assert sim.spout_position() == pos
    assert sim.kettle_angle() == 36.0
    for f in range(3):
        sim.set_spout_position(-0.1 * (f + 1), 6.8, 0.0)
        sim.step_frame(1.0 / 60.0)
    _same(moved, _state(sim))
    sim.restore(blob)
    for _ in range(3):
        sim.step_frame(1.0 / 60.0)
    still = _state(sim)
    assert mismatch(still["particles"], moved["particles"]) > 0  # the spout did move
