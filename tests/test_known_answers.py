"""Known answers of the reference's host-side code, checked on the CPU oracle.

The reference's step has no golden vectors (its GPU tests are statistical and need a
wgpu adapter), so these host-side known-answer tests are what pin the oracle's
restatement.  Each test cites the reference test it restates; paths are relative to
crates/sim-wasm/src/mpm_3d/.
"""
import ctypes as C
import math

import numpy as np
import pytest

from coffee_sim_b200 import _ffi
from coffee_sim_b200.sim import MpmSettings, MpmSim3D

F = np.float32


@pytest.fixture(scope="module")
def probe(oracle):
    fn = oracle.lib.oracle_eval
    fn.restype = C.c_int32
    fn.argtypes = [C.c_int32, C.POINTER(_ffi.CsSettings), C.POINTER(C.c_float), C.POINTER(C.c_float)]

    def call(kind, settings, *args):
        a = (C.c_float * 8)(*args)
        out = (C.c_float * 4)()
        assert fn(kind, C.byref(settings.raw) if settings is not None else None, a, out) == 0
        return list(out)
    return call


def test_volume_scale_matches_length_scale(oracle):
    """units.rs:578-581: ML_PER_SIM_UNIT_CUBED within 0.05 of 5.20."""
    s = MpmSettings.default_v60(oracle)
    assert abs(s.spout.volume_to_ml - 5.20) < 0.05


def test_v60_height_and_gentle_speed(oracle):
    """units.rs:572-589: 5.77 scene units are 0.10 m; the gentle pour exits at 0.12 m/s."""
    s = MpmSettings.default_v60(oracle)
    upm = s.sim_units_per_meter
    assert abs((s.filter.top_y - s.filter.bot_y) / upm - 0.10) < 1e-6
    assert abs(s.spout.gentle_exit_speed / upm - 0.12) < 1e-6
    assert s.spout.max_exit_speed > s.spout.gentle_exit_speed


def test_kozeny_carman_tracks_grind_size_squared(probe):
    """brew_config.rs:519-527: permeability ratio of 800 um to 400 um grind is 4.0 +/- 0.01."""
    fine = probe(0, None, 400.0, 0.40)[0]
    coarse = probe(0, None, 800.0, 0.40)[0]
    assert fine > 0 and coarse > fine
    assert abs(coarse / fine - 4.0) < 0.01


def test_default_brew_parameters_are_plausible(oracle, probe):
    """brew_config.rs:501-511."""
    s = MpmSettings.default_v60(oracle)
    assert 0.30 <= s.bed.initial_porosity <= 0.55
    assert s.bed.num_particles > 1000
    assert s.brew.bed_sample_radius_dx > s.brew.water_sample_radius_dx
    assert s.bed.initial_permeability > s.brew.min_bed_permeability_m2
    assert abs(s.bed.initial_permeability - probe(0, None, 450.0, 0.40)[0]) == 0.0


def test_default_v60_shader_constants_in_sync(oracle):
    """mod.rs:695-742: support cone follows the filter slope; carafe cylinder; the WGSL
    constants (cone radius span 4.2634315, wall 0.4) agree with the obstacle list."""
    s = MpmSettings.default_v60(oracle)
    cone, cup = s.obstacles[0], s.obstacles[1]
    assert cone.kind == _ffi.CS_OBSTACLE_TRUNCATED_CONE and cup.kind == _ffi.CS_OBSTACLE_CYLINDER
    f = s.filter
    slope = (f.top_radius - f.bot_radius) / (f.top_y - f.bot_y)
    assert abs(cone.top_radius - (s.brew.dripper_outlet_radius + slope * (cone.top_y - cone.bot_y))) < 0.01
    assert abs(cone.bot_radius - s.brew.dripper_outlet_radius) < 1e-6
    assert (cone.top_y, cone.bot_y) == (3.0, -3.0)
    assert abs((cone.top_radius - cone.bot_radius) / (cone.top_y - cone.bot_y) - slope) < 1e-5
    assert (cup.radius, cup.top_y, cup.bot_y) == (3.0, -3.5, -8.0)
    assert abs((cone.top_radius - cone.bot_radius) - s.geom.cone_radius_span) < 1e-5
    assert abs(s.geom.wall_thickness - 0.4) < 1e-7


def test_default_v60_grid_uses_uniform_dx(oracle):
    """mod.rs:744-752."""
    s = MpmSettings.default_v60(oracle)
    dx = s.bounds_size[0] / s.grid_dims[0]
    dz = s.bounds_size[2] / s.grid_dims[2]
    assert abs(dx - dz) < 1e-5
    assert s.grid_dims[1] * dx >= s.bounds_size[1] - dx
    assert list(s.grid_dims) == [80, 115, 80]


def test_default_v60_uses_slow_gooseneck_angle(oracle, probe):
    """mod.rs:754-764."""
    s = MpmSettings.default_v60(oracle)
    assert s.initial_kettle_angle_deg <= 10.0
    assert s.spout.max_flow_rate_ml_s <= 12.0
    exit_speed = probe(1, s, s.initial_kettle_angle_deg)[2]
    assert exit_speed / s.sim_units_per_meter <= 0.13
    assert s.spout.max_exit_speed / s.sim_units_per_meter <= 0.50


def test_occupancy_threshold_accepts_lone_particle(oracle):
    """mod.rs:786-797: 0.1 * nominal mass stays below a lone sample's peak deposit."""
    s = MpmSettings.default_v60(oracle)
    nominal = s.brew.water_mass_units_per_ml / s.brew.water_particles_per_ml
    assert nominal * 0.1 < nominal * 0.75 ** 3


def test_effective_head_zero_below_activation_and_monotonic(oracle, probe):
    """inflow.rs:299-322."""
    s = MpmSettings.default_v60(oracle)
    sp = s.spout
    assert probe(1, s, 0.0)[0] == 0.0
    assert probe(1, s, sp.activation_angle_deg)[0] == 0.0
    low, mid, high = (probe(1, s, a)[0] for a in (16.0, 30.0, 48.0))
    assert 0.0 < low < mid < high
    assert abs(probe(1, s, sp.full_flow_angle_deg)[0] - sp.head_at_full_angle) < 1e-6


def test_exit_speed_from_head_monotonic_and_capped(oracle, probe):
    """inflow.rs:324-335."""
    s = MpmSettings.default_v60(oracle)
    low, mid, high = (probe(2, s, h, 22.0)[0] for h in (0.25, 2.0, 40.0))
    assert 0.0 < low < mid <= high <= 22.0
    assert probe(2, s, 0.0, 22.0)[0] == 0.0


def test_exit_speed_cap_tracks_pour_angle(oracle, probe):
    """inflow.rs:337-349."""
    s = MpmSettings.default_v60(oracle)
    sp = s.spout
    barely, medium, full = (probe(1, s, a)[1] for a in (9.0, 36.0, sp.full_flow_angle_deg))
    assert sp.gentle_exit_speed <= barely <= sp.gentle_exit_speed * 1.01
    assert barely < medium < full
    assert abs(full - sp.max_exit_speed) < 1e-6


def test_flow_rate_from_speed_monotonic_and_capped(oracle, probe):
    """inflow.rs:351-366."""
    s = MpmSettings.default_v60(oracle)
    r = s.spout.nozzle_radius
    low, mid, high = (probe(3, s, v, r, 0.92, 5.4, 4.0)[0] for v in (4.0, 10.0, 40.0))
    assert 0.0 < low < mid <= high <= 4.0
    assert probe(3, s, 0.0, r, 0.92, 5.4, 4.0)[0] == 0.0


def test_inflow_consistent_at_42_degrees(oracle, probe):
    """inflow.rs:368-378."""
    s = MpmSettings.default_v60(oracle)
    head, cap, speed, flow = probe(1, s, 42.0)
    assert speed > 0 and flow > 0
    assert speed <= s.spout.max_exit_speed and flow <= s.spout.max_flow_rate_ml_s


def test_translating_spout_preserves_jet_direction(oracle):
    """inflow.rs:380-398, through the ABI's settings and sim controls."""
    s = MpmSettings.default_v60(oracle)
    oracle.call("cs_settings_aim_spout", C.byref(s.raw), C.c_float(0.0), C.c_float(0.4), C.c_float(0.0))
    s.raw.grid_dims[:] = (8, 8, 8)
    s.raw.has_bed = 0
    s.raw.max_particles = 16
    sim = MpmSim3D(s, oracle)
    before = np.array(sim.spout_position(), dtype=np.float64)
    d0 = np.array(list(s.spout.direction))
    t0 = np.array(list(s.spout.target))
    sim.set_spout_position(before[0] - 0.3, before[1], before[2])
    cur = MpmSettings()
    oracle.call("cs_get_settings", sim._h, C.byref(cur.raw))
    assert np.allclose(np.array(list(cur.spout.target)) - t0, [-0.3, 0.0, 0.0], atol=1e-5)
    assert np.allclose(np.array(list(cur.spout.direction)), d0, atol=1e-5)


# ---- bed seeding (bed.rs:316-524) ----
def _bed_sim(oracle, grid, num_particles=None, bed=None):
    s = MpmSettings.default_v60(oracle)
    s.raw.grid_dims[:] = grid
    s.raw.bounds_size[:] = (14.0, 20.0, 14.0)
    if bed is not None:
        s.raw.bed = bed
    if num_particles is not None:
        s.raw.bed.num_particles = num_particles
    return s, MpmSim3D(s, oracle)


def _default_bed_config():
    """BedConfig::default (bed.rs:20-38), not seated."""
    b = _ffi.CsBed()
    b.center[:] = (0.0, -0.35, 0.0)
    b.top_y, b.bot_y, b.top_radius, b.bot_radius = 0.45, -2.70, 2.65, 0.18
    b.num_particles = 12000
    b.initial_porosity = 0.40
    b.initial_permeability = 2.0e-10
    b.extractable_mass = 0.15
    b.layer_split_y = -1e30
    b.lower_porosity_scale = b.lower_permeability_scale = 1.0
    return b


def test_empty_bed_when_height_collapses(oracle):
    b = _default_bed_config()
    b.top_y = b.bot_y = 0.0
    b.num_particles = 200
    s, sim = _bed_sim(oracle, (16, 16, 16), bed=b)
    s.raw.bounds_size[:] = (8.0, 8.0, 8.0)
    sim = MpmSim3D(s, oracle)
    assert sim.num_bed == 0
    assert (sim.read_bed_lookup() == -1).all()


def test_produces_at_most_target_particles(oracle):
    b = _default_bed_config()
    b.num_particles = 200
    _, sim = _bed_sim(oracle, (32, 32, 32), bed=b)
    assert 0 < sim.num_bed <= 200


def test_downsampled_bed_spans_configured_height(oracle):
    b = _default_bed_config()
    _, sim = _bed_sim(oracle, (32, 32, 32), bed=b)
    y = sim.read_particles(0, sim.num_bed)[:, 1]
    assert y.min() <= b.center[1] + b.bot_y + 0.2
    assert y.max() >= b.center[1] + b.top_y - 0.2


def test_seated_bed_bottom_is_rounded_not_planar(oracle):
    s, sim = _bed_sim(oracle, (64, 64, 64))
    cfg = s.raw.bed
    p = sim.read_particles(0, sim.num_bed)
    bottom = cfg.center[1] + cfg.bot_y
    low = p[p[:, 1] <= bottom + 0.45]
    r = np.sqrt(low[:, 0] ** 2 + low[:, 2] ** 2)
    centre, edge = low[r < cfg.bot_radius * 0.45], low[r > cfg.bot_radius * 0.80]
    assert len(centre) and len(edge)
    assert edge[:, 1].mean() > centre[:, 1].mean() + 0.03


def test_bed_particles_carry_phase_marker_and_extracts(oracle):
    b = _default_bed_config()
    b.num_particles = 200
    _, sim = _bed_sim(oracle, (32, 32, 32), bed=b)
    a = sim.read_affine(0, sim.num_bed)
    assert (a[:, 3] == 1.0).all()
    e = sim.read_bed_extract()
    assert (e[:, 0] == 0).all() and np.allclose(e[:, 1], b.initial_porosity, atol=1e-6)
    assert np.allclose(e[:, 2], b.initial_permeability, rtol=1e-6)
    assert (e[:, 3] == 0).all() and np.allclose(e[:, 4], b.extractable_mass, atol=1e-6)
    assert (e[:, 5] == 0).all() and (e[:, 7] == 0).all()


def test_cell_lookup_only_indexes_existing_particles(oracle):
    b = _default_bed_config()
    b.num_particles = 200
    _, sim = _bed_sim(oracle, (32, 32, 32), bed=b)
    lk = sim.read_bed_lookup()
    assert lk.min() >= -1 and lk.max() < sim.num_bed
    assert (lk >= 0).any()


def _seat(oracle, f):
    fn = oracle.lib.oracle_bed_seated
    fn.restype = C.c_int32
    fn.argtypes = [C.POINTER(_ffi.CsFilter), C.POINTER(_ffi.CsBed)]
    out = _ffi.CsBed()
    assert fn(C.byref(f), C.byref(out)) == 0
    return out


def _filter(**kw):
    f = _ffi.CsFilter()
    f.center[:] = kw.get("center", (0.0, -0.35, 0.0))
    f.top_y, f.bot_y = kw.get("top_y", 2.75), kw.get("bot_y", -3.02)
    f.top_radius, f.bot_radius = kw.get("top_radius", 4.10), kw.get("bot_radius", 0.0)
    f.thickness, f.hole_radius = kw.get("thickness", 0.08), kw.get("hole_radius", 0.0)
    return f


def _inner_radius(f, y):
    h = max(f.top_y - f.bot_y, 1e-6)
    t = min(max((y - f.bot_y) / h, 0.0), 1.0)
    return max(f.bot_radius + (f.top_radius - f.bot_radius) * t - f.thickness, f.hole_radius)


def test_default_bed_sits_inside_filter_interior(oracle):
    f = _filter()
    b = _seat(oracle, f)
    top, bot = b.center[1] + b.top_y, b.center[1] + b.bot_y
    assert b.top_radius < _inner_radius(f, top - f.center[1])
    assert b.bot_radius < _inner_radius(f, bot - f.center[1])
    assert bot > f.center[1] + f.bot_y
    assert bot - (f.center[1] + f.bot_y) >= b.bot_radius * 0.65
    assert top < f.center[1] + f.top_y


def test_seated_in_filter_does_not_fail_on_narrow_filter(oracle):
    b = _seat(oracle, _filter(top_y=0.1, bot_y=-0.1, top_radius=0.3, bot_radius=0.2, thickness=0.02,
                              hole_radius=0.05))
    assert all(math.isfinite(v) for v in (b.top_y, b.bot_y, b.top_radius, b.bot_radius))


def test_seated_in_filter_uses_filter_center_offset(oracle):
    f = _filter(center=(0.0, 2.0, 0.0))
    b = _seat(oracle, f)
    assert b.center[1] + b.top_y <= f.center[1] + f.top_y - 0.3
    assert b.center[1] + b.bot_y >= f.center[1] + f.bot_y + 0.3


def test_sdf_class_matches_live_cell_center_sampling(oracle):
    """state.rs:441-468: the cached solid mask equals sampling the SDF at each cell
    centre (Rust-side trilinear sample, f32::fract = x - trunc(x))."""
    s = MpmSettings.default_v60(oracle)
    s.raw.has_bed = 0
    sim = MpmSim3D(s, oracle)
    sdf = sim.read_sdf().reshape(128, 128, 128)
    cls = sim.read_sdf_class()
    g = [int(v) for v in s.grid_dims]
    b = [F(v) for v in s.bounds_size]
    dx = b[0] / F(g[0])
    iz, iy, ix = np.meshgrid(np.arange(g[2]), np.arange(g[1]), np.arange(g[0]), indexing="ij")
    pos = [F(-b[a] * F(0.5)) + (np.array(idx, dtype=F) + F(0.5)) * dx for a, idx in ((0, ix), (1, iy), (2, iz))]
    uv = [(pos[a] + b[a] * F(0.5)) / b[a] * F(128.0) - F(0.5) for a in range(3)]
    base = [np.floor(u).astype(np.int64) for u in uv]
    fr = [u - np.trunc(u) for u in uv]

    def tex(x, y, z):
        return sdf[np.clip(z, 0, 127), np.clip(y, 0, 127), np.clip(x, 0, 127)]

    x0, y0, z0 = base
    c00 = tex(x0, y0, z0) + (tex(x0 + 1, y0, z0) - tex(x0, y0, z0)) * fr[0]
    c10 = tex(x0, y0 + 1, z0) + (tex(x0 + 1, y0 + 1, z0) - tex(x0, y0 + 1, z0)) * fr[0]
    c01 = tex(x0, y0, z0 + 1) + (tex(x0 + 1, y0, z0 + 1) - tex(x0, y0, z0 + 1)) * fr[0]
    c11 = tex(x0, y0 + 1, z0 + 1) + (tex(x0 + 1, y0 + 1, z0 + 1) - tex(x0, y0 + 1, z0 + 1)) * fr[0]
    c0 = c00 + (c10 - c00) * fr[1]
    c1 = c01 + (c11 - c01) * fr[1]
    live = (c0 + (c1 - c0) * fr[2]) < 0
    assert (live.reshape(-1).astype(np.uint8) == cls).all()


def _filter_radius_at_y(f, y):
    """FilterConfig::radius_at_y (filter.rs:29-33) in float32."""
    height = max(F(f.top_y) - F(f.bot_y), F(1e-6))
    t = min(max((F(y) - F(f.bot_y)) / height, F(0.0)), F(1.0))
    return F(f.bot_radius) + (F(f.top_radius) - F(f.bot_radius)) * t


def _filter_inner_radius_at_y(f, y):
    """FilterConfig::inner_radius_at_y (filter.rs:35-37)."""
    return max(_filter_radius_at_y(f, y) - F(f.thickness), F(f.hole_radius))


def test_filter_preset_is_the_reference_default(oracle):
    """filter.rs:14-26: the V60 preset's paper filter is FilterConfig::default()."""
    f = MpmSettings.default_v60(oracle).filter
    assert (list(f.center), f.top_y, f.bot_y) == ([0.0, F(-0.35), 0.0], F(2.75), F(-3.02))
    assert (f.top_radius, f.bot_radius, f.thickness, f.hole_radius) == (F(4.10), 0.0, F(0.08), 0.0)


def test_filter_radius_decreases_toward_the_apex(oracle):
    """filter.rs:62-66."""
    f = MpmSettings.default_v60(oracle).filter
    assert _filter_radius_at_y(f, f.top_y) > _filter_radius_at_y(f, f.bot_y)


def test_default_filter_paper_comes_to_a_tip(oracle):
    """filter.rs:68-74."""
    f = MpmSettings.default_v60(oracle).filter
    assert f.hole_radius == 0.0
    assert _filter_radius_at_y(f, f.bot_y) == 0.0
    assert _filter_inner_radius_at_y(f, f.bot_y) == 0.0


def test_filter_contains_shell_points_on_the_cone_band(oracle):
    """filter.rs:76-92: a point midway through the paper at mid height is in the shell,
    one 0.5 outside the outer radius is not."""
    f = MpmSettings.default_v60(oracle).filter

    def in_shell(x, y, z):
        if y < f.bot_y or y > f.top_y:
            return False
        r = math.sqrt((x - f.center[0]) ** 2 + (z - f.center[2]) ** 2)
        return _filter_inner_radius_at_y(f, y) <= r <= _filter_radius_at_y(f, y)

    mid_y = (F(f.top_y) + F(f.bot_y)) * F(0.5)
    outer, inner = _filter_radius_at_y(f, mid_y), _filter_inner_radius_at_y(f, mid_y)
    assert in_shell(f.center[0] + (outer + inner) * F(0.5), mid_y, f.center[2])
    assert not in_shell(f.center[0] + outer + F(0.5), mid_y, f.center[2])
