"""Runtime solver parameters and the autotuner (engine extensions without a reference
counterpart)."""
import pytest

from coffee_sim_b200 import _ffi, scenes
from coffee_sim_b200.sim import MpmSim3D
from helpers import mismatch


def _v60(lib, grid=32):
    s = scenes.c2_v60(lib, grid=grid, max_particles=60000)
    sim = MpmSim3D(s, lib)
    scenes.populate_c2(sim)
    return sim


def test_set_solver_changes_settings(oracle):
    sim = _v60(oracle)
    sim.set_solver(omega=1.85, check_every=7, max_sweeps=123)
    st = sim.current_settings()
    assert abs(st.rbgs_omega - 1.85) < 1e-7 and st.check_every == 7 and st.max_sweeps == 123
    sim.set_solver(omega=0.0, check_every=0, max_sweeps=0)  # zeros keep the values
    st = sim.current_settings()
    assert abs(st.rbgs_omega - 1.85) < 1e-7 and st.check_every == 7 and st.max_sweeps == 123
    with pytest.raises(_ffi.CsError):
        sim.set_solver(omega=2.5)
    with pytest.raises(_ffi.CsError):
        sim.set_p2g_mode(_ffi.CS_P2G_INT64)


def test_oracle_has_no_autotuner(oracle):
    sim = _v60(oracle)
    with pytest.raises(_ffi.CsError) as e:
        sim.autotune(scenes.C2_DT, 1)
    assert e.value.code == _ffi.CS_ERR_UNSUPPORTED


@pytest.mark.gpu
def test_autotune_restores_state_and_applies_choice(engine):
    sim = _v60(engine)
    for _ in range(2):
        sim.step_substep(scenes.C2_DT)
    n = sim.particle_count()
    before = (sim.read_particles(0, n), sim.read_pressure())
    r = sim.autotune(scenes.C2_DT, 2)
    assert r.trials >= 20
    assert r.best_ms <= r.initial_ms
    assert 1.79 < r.omega < 1.97 and r.check_every in (10, 20, 40, 60, 80)
    assert r.p2g_mode in (_ffi.CS_P2G_ATOMIC32, _ffi.CS_P2G_SORTED_SHARED)
    assert sim.particle_count() == n
    assert mismatch(sim.read_particles(0, n), before[0]) == 0
    assert mismatch(sim.read_pressure(), before[1]) == 0
    assert r.first_check == 0 or 2 <= r.first_check <= 4000
    assert r.p2g_tile in (4, 8) and r.particle_threads in (128, 256)
    st = sim.current_settings()
    assert st.rbgs_omega == r.omega and st.check_every == r.check_every and st.p2g_mode == r.p2g_mode
    assert st.first_check == r.first_check
    assert st.p2g_tile == r.p2g_tile and st.particle_threads == r.particle_threads
    sim.step_substep(scenes.C2_DT)
    assert sim.latest_metrics().last_residual <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("tile,threads", [(8, 128), (8, 256), (4, 128)])
def test_launch_shapes_give_the_same_state(engine, tile, threads):
    """The launch shapes the autotuner chooses between (P2G tile side, threads per block
    of the particle passes) change no result: the V60 pour at 32^3 with tile-sorted P2G,
    four substeps bit for bit against the default shapes (4^3 tiles, 256 threads)."""
    sims = []
    for t, th in ((0, 0), (tile, threads)):
        s = scenes.c2_v60(engine, grid=32, max_particles=60000)
        s.raw.device_emission = 1
        s.raw.p2g_mode = _ffi.CS_P2G_SORTED_SHARED
        s.raw.p2g_tile = t
        s.raw.particle_threads = th
        sim = MpmSim3D(s, engine)
        scenes.populate_c2(sim)
        sims.append(sim)
    for _ in range(4):
        for sim in sims:
            sim.step_substep(scenes.C2_DT)
    assert mismatch(sims[0].read_particles(), sims[1].read_particles()) == 0
    assert mismatch(sims[0].read_grid_lanes(), sims[1].read_grid_lanes()) == 0
    assert mismatch(sims[0].read_pressure(), sims[1].read_pressure()) == 0
