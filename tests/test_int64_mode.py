"""int64 fixed-point P2G (CS_P2G_INT64: i64 * 2^32 lanes, sorted accumulation).  The
reference's i32 * 2^18 lanes truncate every contribution to 2^-18; the int64 mode keeps
14 more bits and cannot overflow in dense pools."""
import numpy as np
import pytest

from coffee_sim_b200 import _ffi, scenes
from coffee_sim_b200.sim import MpmSettings, MpmSim3D
from helpers import mismatch, relerr

FRAME = 1.0 / 60.0


def _v60(lib, mode, grid=32):
    s = scenes.c2_v60(lib, grid=grid, max_particles=60000)
    s.raw.p2g_mode = mode
    s.raw.rbgs_omega = 1.9
    sim = MpmSim3D(s, lib)
    scenes.populate_c2(sim)
    return sim


def test_oracle_int64_lanes_refine_the_i32_lanes(oracle):
    """The same deposit at two scales: i64 / 2^14 equals the i32 lane up to the
    truncation of the contributions (< 1 quantum each, 27 per sample)."""
    a = _v60(oracle, _ffi.CS_P2G_ATOMIC32)
    b = _v60(oracle, _ffi.CS_P2G_INT64)
    for sim in (a, b):
        sim.step_substep_partial(scenes.C2_DT, 4)  # through P2G
    # lane 0 of the i32 readback carries the encoded FP32 pressure; compare momentum
    # (lanes 1-3) and the rest / current volumes (lanes 4-5)
    l32 = a.read_grid_lanes().astype(np.float64)[1:]
    l64 = b.read_grid_lanes64().astype(np.float64)[1:] / 2.0 ** 14
    assert np.abs(l64).max() > 0
    contributions = 8 * 27  # samples whose stencil covers one node, 8 per cell
    assert np.abs(l64 - l32).max() <= contributions
    # i32 truncation loses up to one 2^-18 quantum per contribution
    assert relerr(l64, l32) < 1e-2


def test_oracle_int64_steps_close_to_i32(oracle):
    a = _v60(oracle, _ffi.CS_P2G_ATOMIC32)
    b = _v60(oracle, _ffi.CS_P2G_INT64)
    for _ in range(3):
        a.step_substep(scenes.C2_DT)
        b.step_substep(scenes.C2_DT)
    n = a.particle_count()
    assert b.particle_count() == n
    assert relerr(b.read_particles(0, n)[:, :3], a.read_particles(0, n)[:, :3]) < 1e-5
    assert b.latest_metrics().last_residual <= 1e-5
    ce = a.current_settings().check_every
    for sim in (a, b):
        m = sim.latest_metrics()
        # the warm start's check plus one per cycle of 2..check_every pairs
        assert -(-m.last_sweeps // ce) <= m.residual_checks - 1 <= -(-m.last_sweeps // 2), (m.last_sweeps, m.residual_checks)


def test_lanes64_only_in_int64_mode(oracle):
    a = _v60(oracle, _ffi.CS_P2G_ATOMIC32)
    with pytest.raises(_ffi.CsError):
        a.read_grid_lanes64()


@pytest.mark.gpu
@pytest.mark.parametrize("passes", [4, 0xFFFFFFFF])
def test_int64_matches_oracle(engine, oracle, passes):
    e = _v60(engine, _ffi.CS_P2G_INT64)
    o = _v60(oracle, _ffi.CS_P2G_INT64)
    for k in range(2):
        if passes == 4 and k == 1:
            for sim in (e, o):
                sim.step_substep_partial(scenes.C2_DT, passes)
        else:
            for sim in (e, o):
                sim.step_substep(scenes.C2_DT)
    assert mismatch(e.read_grid_lanes64(), o.read_grid_lanes64()) == 0
    n = e.particle_count()
    assert mismatch(e.read_particles(0, n), o.read_particles(0, n)) == 0
    assert mismatch(e.read_pressure(), o.read_pressure()) == 0


@pytest.mark.gpu
def test_int64_reference_scene_frames(engine, oracle):
    s = MpmSettings.benchmark_center_pour(engine)
    s.raw.p2g_mode = _ffi.CS_P2G_INT64
    e, o = MpmSim3D(s, engine), MpmSim3D(s, oracle)
    for sim in (e, o):
        sim.set_kettle_angle(36.0)
    for f in range(5):
        e.step_frame(FRAME)
        o.step_frame(FRAME)
    n = e.particle_count()
    assert n == o.particle_count()
    assert mismatch(e.read_particles(0, n), o.read_particles(0, n)) == 0
    assert mismatch(e.read_grid_lanes64(), o.read_grid_lanes64()) == 0
