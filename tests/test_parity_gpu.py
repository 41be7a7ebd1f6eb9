"""CUDA engine vs the CPU oracle, through the C ABI.

The engine is built with -fmad=false and restates every WGSL expression in the same
order as the oracle, so in the reference configuration (fixed-point pressure, fixed
40 red+black pairs, i32 atomics) results are expected to agree bit for bit; each
comparison asserts exact equality and prints the first mismatching pass otherwise.
"""
import numpy as np
import pytest

from coffee_sim_b200 import _ffi, scenes
from coffee_sim_b200.sim import MpmSettings, MpmSim3D
from helpers import copy_state, mismatch, pair, relerr

pytestmark = pytest.mark.gpu

FRAME = 1.0 / 60.0

# Reference dispatch numbering (mod.rs:317-414); a partial substep runs passes [0, n).
AFTER_P2G = 4
AFTER_GRID_UPDATE = 6
AFTER_CLASSIFY = 7
AFTER_RBGS = 8
AFTER_PROJECT = 11
AFTER_PACKING = 13
AFTER_VISCOSITY = 16
AFTER_G2P = 17
AFTER_COUPLING = 18
AFTER_BED = 20
ALL = 0xFFFFFFFF


def _state(sim, cells=True):
    n = sim.particle_count()
    d = {"particles": sim.read_particles(0, n), "affine": sim.read_affine(0, n)}
    if sim.num_bed:
        d["bed_extract"] = sim.read_bed_extract(0, sim.num_bed)
    if cells:
        d["lanes"] = sim.read_grid_lanes()
        d["grid_vel"] = sim.read_grid_vel()
        d["lookup"] = sim.read_bed_lookup()
        d["kind"] = sim.read_cell_kind()
        d["pressure"] = sim.read_pressure()
    return d


def _assert_same(a, b, what, keys=None):
    bad = {}
    for k in keys or a:
        if k not in b:
            continue
        m = mismatch(a[k], b[k])
        if m:
            bad[k] = (m, relerr(a[k], b[k]))
    assert not bad, f"{what}: mismatching arrays (count, norm-rel err) {bad}"


def _prepared(settings, oracle, frames, angle):
    """Run the oracle to an interesting state and return it."""
    src = MpmSim3D(settings, oracle)
    src.set_kettle_angle(angle)
    for _ in range(frames):
        src.step_frame(FRAME)
    return src


@pytest.fixture(scope="module")
def free_stream_state(oracle):
    s = MpmSettings.benchmark_free_stream(oracle)
    return s, _prepared(s, oracle, 18, 36.0)


@pytest.fixture(scope="module")
def center_pour_state(oracle):
    s = MpmSettings.benchmark_center_pour(oracle)
    return s, _prepared(s, oracle, 20, 36.0)


def test_setup_matches_oracle(engine, oracle):
    """SDF texture, solid mask and the seeded bed (state.rs:206-344, bed.rs:107-314)."""
    s = MpmSettings.benchmark_center_pour(engine)
    e, o = pair(s, engine, oracle)
    assert e.num_bed == o.num_bed == 12000
    assert mismatch(e.read_sdf(), o.read_sdf()) == 0
    assert mismatch(e.read_sdf_class(), o.read_sdf_class()) == 0
    _assert_same(_state(e), _state(o), "initial state", ["particles", "affine", "bed_extract", "lookup"])


@pytest.mark.parametrize("passes", [AFTER_P2G, AFTER_GRID_UPDATE, AFTER_CLASSIFY, AFTER_RBGS, AFTER_PROJECT,
                                    AFTER_PACKING, AFTER_VISCOSITY, AFTER_G2P, ALL])
def test_free_stream_pass_by_pass(engine, oracle, free_stream_state, passes):
    settings, src = free_stream_state
    e, o = pair(settings, engine, oracle)
    copy_state(src, e)
    copy_state(src, o)
    for sim in (e, o):
        sim.set_kettle_angle(36.0)
        sim.step_substep_partial(FRAME / 10, passes)
    a, b = _state(e), _state(o)
    keys = ["particles", "affine", "grid_vel", "lookup"]
    if passes in (AFTER_P2G,):
        keys.append("lanes")
    if passes >= AFTER_CLASSIFY:
        keys += ["kind", "pressure"]
    if passes == ALL:
        keys.append("lanes")
    _assert_same(a, b, f"free stream after {passes} passes", keys)


@pytest.mark.parametrize("passes", [AFTER_P2G, AFTER_CLASSIFY, AFTER_RBGS, AFTER_PROJECT, AFTER_G2P,
                                    AFTER_COUPLING, AFTER_BED, ALL])
def test_center_pour_pass_by_pass(engine, oracle, center_pour_state, passes):
    settings, src = center_pour_state
    e, o = pair(settings, engine, oracle)
    copy_state(src, e)
    copy_state(src, o)
    for sim in (e, o):
        sim.set_kettle_angle(36.0)
        sim.step_substep_partial(FRAME / 10, passes)
    a, b = _state(e), _state(o)
    keys = ["particles", "affine", "bed_extract", "grid_vel", "lookup"]
    if passes >= AFTER_CLASSIFY:
        keys += ["kind", "pressure"]
    if passes in (AFTER_P2G, ALL):
        keys.append("lanes")
    _assert_same(a, b, f"center pour after {passes} passes", keys)
    if passes == ALL:
        assert mismatch(e.read_bed_delta(), o.read_bed_delta()) == 0


def test_center_pour_frames_bit_exact(engine, oracle):
    """Ten frames of pouring onto the bed from the initial state, compared every frame."""
    s = MpmSettings.benchmark_center_pour(engine)
    e, o = pair(s, engine, oracle)
    for sim in (e, o):
        sim.set_kettle_angle(36.0)
    for f in range(10):
        e.step_frame(FRAME)
        o.step_frame(FRAME)
        assert e.particle_count() == o.particle_count()
        _assert_same(_state(e, cells=False), _state(o, cells=False), f"frame {f}")
    me, mo = e.latest_metrics(), o.latest_metrics()
    assert (me.fluid_cells, me.div_clamp_fires, me.pressure_clamp_fires) == (
        mo.fluid_cells, mo.div_clamp_fires, mo.pressure_clamp_fires)
    assert me.max_abs_div == mo.max_abs_div
    assert e.total_emitted_mass() == o.total_emitted_mass()


def test_c1_water_block_200_steps(engine, oracle):
    """The C1 water block (32^3, 16.8k samples, 40 pairs): 200 substeps, compared every 50."""
    se = scenes.c1_water_block(engine)
    e, o = MpmSim3D(se, engine), MpmSim3D(se, oracle)
    assert scenes.populate_c1(e) == scenes.populate_c1(o)
    for k in range(200):
        e.step_substep(scenes.C1_DT)
        o.step_substep(scenes.C1_DT)
        if k % 50 == 49:
            _assert_same(_state(e), _state(o), f"C1 step {k}", ["particles", "affine", "grid_vel", "pressure"])


@pytest.mark.parametrize("grid,omega,first", [(32, 1.0, 0), (64, 1.9, 0), (32, 1.9, 25)])
def test_v60_refinement_solve_matches_oracle(engine, oracle, grid, omega, first):
    """FP32-storage residual mode: mixed-precision refinement with red-black
    (over-relaxed) sweeps to 1e-5; per-cell arithmetic identical to the oracle, FP64
    norms reduced in a different order (the sweep counts still agree).  `first`: pairs
    before the first residual check (0: the check interval)."""
    se = scenes.c2_v60(engine, grid=grid)
    se.raw.rbgs_omega = omega
    se.raw.first_check = first
    se.raw.max_sweeps = 600 if omega == 1.0 else 2000
    e, o = MpmSim3D(se, engine), MpmSim3D(se, oracle)
    assert scenes.populate_c2(e) == scenes.populate_c2(o)
    for k in range(2):
        e.step_substep(scenes.C2_DT)
        o.step_substep(scenes.C2_DT)
        me, mo = e.latest_metrics(), o.latest_metrics()
        assert me.last_sweeps == mo.last_sweeps, (k, me.last_sweeps, mo.last_sweeps)
        assert me.residual_checks == mo.residual_checks >= 2, (k, me.residual_checks, mo.residual_checks)
        assert abs(me.last_residual - mo.last_residual) <= 1e-9 * max(mo.last_residual, 1e-30) + 1e-15
        if omega != 1.0:
            assert me.last_residual <= 1e-5
        a, b = _state(e), _state(o)
        _assert_same(a, b, f"V60 {grid}^3 substep {k}", ["particles", "affine", "bed_extract", "grid_vel", "pressure"])


@pytest.mark.parametrize("cluster_kernel", [2, 3])
def test_cluster_solver_matches_per_colour_launches(engine, cluster_kernel):
    """The one-launch cluster-resident solve (solver_cluster.cuh; 2: point-to-point
    mbarrier waits between the colours, 3: cluster barriers) against the per-colour launch
    path on the same state: identical sweep counts and pressures."""
    sims = []
    for kernel in (1, cluster_kernel):
        s = scenes.c2_v60(engine)
        s.raw.rbgs_omega = 1.9
        s.raw.rbgs_kernel = kernel
        sim = MpmSim3D(s, engine)
        scenes.populate_c2(sim)
        sims.append(sim)
    sims[1].profile_enable(True)
    for k in range(3):
        for sim in sims:
            sim.step_substep(scenes.C2_DT)
        ma, mb = sims[0].latest_metrics(), sims[1].latest_metrics()
        # the cluster path ran: one launch in the sweep phase of each substep
        assert sims[1].profile_read().phase_launches[4] == k + 1
        assert ma.last_sweeps == mb.last_sweeps
        assert ma.residual_checks == mb.residual_checks >= 2
        assert mb.last_residual <= 1e-5
        assert mismatch(sims[0].read_pressure(), sims[1].read_pressure()) == 0
        assert mismatch(sims[0].read_particles(), sims[1].read_particles()) == 0


@pytest.mark.parametrize("passes", [AFTER_P2G, ALL])
def test_sorted_p2g_matches_oracle(engine, oracle, center_pour_state, passes):
    """Tile-sorted P2G with shared-memory accumulation (CS_P2G_SORTED_SHARED): the same
    integer lanes as the oracle's per-particle atomics, bit for bit."""
    settings, src = center_pour_state
    settings.raw.p2g_mode = _ffi.CS_P2G_SORTED_SHARED
    try:
        e, o = pair(settings, engine, oracle)
    finally:
        settings.raw.p2g_mode = _ffi.CS_P2G_ATOMIC32
    copy_state(src, e)
    copy_state(src, o)
    for sim in (e, o):
        sim.set_kettle_angle(36.0)
        sim.step_substep_partial(FRAME / 10, passes)
    _assert_same(_state(e), _state(o), f"sorted P2G after {passes} passes",
                 ["particles", "affine", "bed_extract", "grid_vel", "lanes"])


def test_sorted_p2g_matches_atomic_on_v60(engine):
    """The dense V60 pour (8 samples per cell, a carafe pool): sorted and atomic P2G give
    identical states over three substeps."""
    sims = []
    for mode in (_ffi.CS_P2G_ATOMIC32, _ffi.CS_P2G_SORTED_SHARED):
        s = scenes.c2_v60(engine)
        s.raw.rbgs_omega = 1.9
        s.raw.p2g_mode = mode
        sim = MpmSim3D(s, engine)
        scenes.populate_c2(sim)
        sims.append(sim)
    for k in range(3):
        for sim in sims:
            sim.step_substep(scenes.C2_DT)
        _assert_same(_state(sims[0]), _state(sims[1]), f"V60 substep {k}",
                     ["particles", "affine", "bed_extract", "grid_vel", "pressure"])


def test_device_emission_matches_oracle(engine, oracle):
    """Jet samples built by a kernel (device_emission = 1): ten frames of the centre
    pour, bit-exact against the oracle's matching emission mode."""
    s = MpmSettings.benchmark_center_pour(engine)
    s.raw.device_emission = 1
    e, o = pair(s, engine, oracle)
    for sim in (e, o):
        sim.set_kettle_angle(36.0)
    for f in range(10):
        e.step_frame(FRAME)
        o.step_frame(FRAME)
        assert e.particle_count() == o.particle_count()
        _assert_same(_state(e, cells=False), _state(o, cells=False), f"device emission frame {f}")
    assert e.total_emitted_mass() == o.total_emitted_mass()
    assert e.particle_count() > 12000


def test_graph_replay_matches_direct_launches_v60(engine):
    """use_graph = 1: the substep captured once and replayed gives the same states, sweep
    counts and residuals as launching it directly (V60 pour, cluster solve)."""
    sims = []
    for graph in (0, 1):
        s = scenes.c2_v60(engine)
        s.raw.rbgs_omega = 1.9
        s.raw.device_emission = 1
        s.raw.use_graph = graph
        sim = MpmSim3D(s, engine)
        scenes.populate_c2(sim)
        sim.set_flow_override(4.0, 0.8 * s.sim_units_per_meter)
        sims.append(sim)
    for k in range(4):
        for sim in sims:
            sim.step_substep(scenes.C2_DT)
        ma, mb = sims[0].latest_metrics(), sims[1].latest_metrics()
        assert ma.last_sweeps == mb.last_sweeps and ma.last_residual == mb.last_residual
        assert sims[0].particle_count() == sims[1].particle_count()
        _assert_same(_state(sims[0]), _state(sims[1]), f"graph substep {k}",
                     ["particles", "affine", "bed_extract", "grid_vel", "pressure"])


def test_graph_frames_match_oracle_reference_mode(engine, oracle):
    """Reference configuration (fixed-point pressure, 40 pairs) in graph mode with
    device emission: ten frames bit-exact against the oracle."""
    s = MpmSettings.benchmark_center_pour(engine)
    s.raw.device_emission = 1
    s.raw.use_graph = 1
    e, o = pair(s, engine, oracle)
    for sim in (e, o):
        sim.set_kettle_angle(36.0)
    for f in range(10):
        e.step_frame(FRAME)
        o.step_frame(FRAME)
        _assert_same(_state(e, cells=False), _state(o, cells=False), f"graph frame {f}")


def test_prepare_render_matches_oracle(engine, oracle, center_pour_state):
    """prepare_render (shader.rs:2242-2276) into the headless render buffer: 2 x vec4
    per sample in the layout of state.rs:136-144 (position + colour value, radius),
    compared with the oracle's after a full substep of the centre pour, and checked
    against the properties the shader gives it: live samples carry their position,
    water a speed colour in [0, 2], bed samples -1 - saturation, inactive samples
    the parked position y = -1e6 with colour -999."""
    settings, src = center_pour_state
    e, o = pair(settings, engine, oracle)
    copy_state(src, e)
    copy_state(src, o)
    for sim in (e, o):
        sim.set_kettle_angle(36.0)
        sim.step_substep(FRAME / 10)
    n = e.particle_count()
    assert n == o.particle_count() > 12000
    re, ro = e.read_render(0, n), o.read_render(0, n)
    assert re.shape == (n, 8)
    assert mismatch(re, ro) == 0, relerr(re, ro)
    parts = e.read_particles(0, n)
    live = re[:, 3] != -999.0
    assert live.sum() > 12000
    assert np.array_equal(re[live, 0:3], parts[live, 0:3])
    water = live & (re[:, 3] >= 0.0)
    bed = live & (re[:, 3] < 0.0)
    assert water.sum() > 0 and bed.sum() > 0
    assert re[water, 3].max() <= 2.0
    assert np.all(re[bed, 3] <= -1.0)
    assert np.all(re[live, 4] > 0.0)          # radius
    assert np.all(re[~live, 1] == -1e6)
    assert np.all(re[:, 5:8] == 0.0)
