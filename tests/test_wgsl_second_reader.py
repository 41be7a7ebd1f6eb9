"""The CPU oracle against a second, independent restatement of the WGSL step
(`tests/wgsl_numpy.py`), on the CPU.

Most tests take the oracle's state after the first n dispatches of a substep
(`cs_step_substep_partial`, the dispatch numbering of `mod.rs:317-414`), apply the
numpy restatement of dispatch n, and compare with the oracle's state after n + 1
dispatches; one chains the restated dispatches over three whole substeps.  The engine
is compared with the oracle bit for bit by the GPU tests, so agreement here carries
over to it.
"""
import numpy as np
import pytest

from coffee_sim_b200.sim import MpmSettings, MpmSim3D
from helpers import copy_state
import wgsl_numpy as W

FRAME = 1.0 / 60.0
SUB_DT = FRAME / 10

# dispatch numbers of one substep (mod.rs:317-414; the oracle numbers them alike)
P_P2G, P_GRID_UPDATE, P_BOUNDARY0, P_CLASSIFY, P_RBGS = 3, 4, 5, 6, 7
P_PROJECT, P_BOUNDARY1, P_PACK_PREP, P_PACK_APPLY, P_BOUNDARY2 = 8, 9, 10, 11, 12
P_VISC_PREP, P_VISC_APPLY, P_BOUNDARY3, P_G2P = 13, 14, 15, 16


def _pour(oracle):
    """The reference's centre-pour scene (mod.rs:107-160 preset) after 24 frames of a
    strong pour, so that water reaches the bed."""
    s = MpmSettings.benchmark_center_pour(oracle)
    src = MpmSim3D(s, oracle)
    src.set_kettle_angle(36.0)
    src.set_flow_override(40.0, 0.0)
    for _ in range(24):
        src.step_frame(FRAME)
    return s, src


def _scatter(src, seed=5):
    """Every third water sample of the pour moved to a random point of the domain (the
    carafe below the cone included, where the SDF constrains the flow, and the margin of
    the box) with a random velocity of up to 3 units/s: inputs that reach the SDF
    contact and box branches of boundary_project."""
    rng = np.random.default_rng(seed)
    nb, nw = src.num_bed, src.num_water
    p = src.read_particles(nb, nw)
    k = np.arange(0, nw, 3)
    lo, hi = np.array([-6.9, -9.9, -6.9]), np.array([6.9, 9.9, 6.9])
    p[k, 0:3] = rng.uniform(lo, hi, size=(k.size, 3)).astype(np.float32)
    d = rng.normal(size=(k.size, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    p[k, 4:7] = (d * rng.uniform(0.0, 3.0, size=(k.size, 1))).astype(np.float32)
    src.write_particles(nb, p)
    # bed grains: every 7th suspended (phase 2), every 3rd nearly saturated, so that the
    # suspended-grain, redeposit and detach branches of bed_dynamics are reached
    a = src.read_affine(0, nb)
    a[::7, 3] = 2.0
    src.write_affine(0, a)
    be = src.read_bed_extract(0, nb)
    be[::3, 7] = 0.9
    src.write_bed_extract(0, be)
    return src


@pytest.fixture(scope="module", params=["pour", "scattered"])
def source(request, oracle):
    s, src = _pour(oracle)
    if request.param == "scattered":
        _scatter(src)
    return request.param, s, src


class Stages:
    """Oracle states after the first n dispatches of the next substep, one simulation
    per n, all started from the same copied state."""

    def __init__(self, oracle, settings, src):
        self.oracle, self.settings, self.src = oracle, settings, src
        self.cache = {}
        self.static = None

    def __call__(self, n):
        if n not in self.cache:
            sim = MpmSim3D(self.settings, self.oracle)
            copy_state(self.src, sim)
            sim.set_kettle_angle(36.0)
            sim.step_substep_partial(SUB_DT, n)
            st = {"particles": sim.read_particles(0, sim.particle_count()),
                  "affine": sim.read_affine(0, sim.particle_count()),
                  "lanes": sim.read_grid_lanes(), "grid_vel": sim.read_grid_vel(),
                  "lookup": sim.read_bed_lookup(), "bed_delta": sim.read_bed_delta(),
                  "num_water": sim.num_water, "num_bed": sim.num_bed}
            if sim.num_bed:
                st["bed_extract"] = sim.read_bed_extract(0, sim.num_bed)
            if self.static is None:
                self.static = {"sdf": sim.read_sdf(), "sdf_class": sim.read_sdf_class()}
            self.cache[n] = st
            sim.close()
        return self.cache[n]

    def uniforms(self, n):
        st = self(n)
        return W.Uniforms(self.settings.raw, st["num_water"], st["num_bed"], SUB_DT)


@pytest.fixture(scope="module")
def stages(oracle, source):
    name, s, src = source
    st = Stages(oracle, s, src)
    st.name = name
    return st


def _report(name, got, want):
    got, want = np.asarray(got), np.asarray(want)
    bad = np.flatnonzero(got.reshape(-1) != want.reshape(-1))
    if bad.size:
        i = bad[0]
        return f"{name}: {bad.size} of {got.size} differ, first at {i}: {got.reshape(-1)[i]!r} vs {want.reshape(-1)[i]!r}"
    return None


def test_scene_has_water_in_the_bed(stages):
    """The inputs reach the branches under test: water in bed-coupled and interior
    cells (both states), grid velocities changed by the SDF contact (scattered state)."""
    st = stages(P_CLASSIFY + 1)
    assert st["num_water"] > 2000 and st["num_bed"] == 12000
    kind = st["lanes"][3]
    assert np.count_nonzero(kind == W.CELL_BED_COUPLED) > 100
    assert np.count_nonzero(kind == W.CELL_INTERIOR_FLUID) > 100
    if stages.name == "scattered":
        u = stages.uniforms(P_BOUNDARY0)
        sdf = W.Sdf(u, stages.static["sdf"])
        px, py, pz = W.cell_centres(u)
        live = stages(P_BOUNDARY0)["grid_vel"][:, 3] >= 1e-6
        assert np.count_nonzero(live & (sdf.sample(px, py, pz).reshape(-1) < u.contact_offset)) > 50
        assert np.count_nonzero(stages(P_BOUNDARY0)["grid_vel"] != stages(P_BOUNDARY0 + 1)["grid_vel"]) > 50


def test_p2g(stages):
    u = stages.uniforms(P_P2G)
    before = stages(P_P2G)
    after = stages(P_P2G + 1)
    assert not before["lanes"].any()
    lanes = W.p2g(u, before["particles"], before["affine"])
    msg = _report("lanes", lanes, after["lanes"])
    assert msg is None, msg


def test_grid_update(stages):
    u = stages.uniforms(P_GRID_UPDATE)
    before = stages(P_GRID_UPDATE)
    after = stages(P_GRID_UPDATE + 1)
    gv = W.grid_update(u, before["lanes"])
    msg = _report("grid_vel", gv, after["grid_vel"])
    assert msg is None, msg


@pytest.mark.parametrize("n", [P_BOUNDARY0, P_BOUNDARY1])
def test_boundary_project(stages, n):
    u = stages.uniforms(n)
    before = stages(n)
    after = stages(n + 1)
    sdf = W.Sdf(u, stages.static["sdf"])
    gv = W.boundary_project(u, sdf, before["grid_vel"])
    msg = _report("grid_vel", gv, after["grid_vel"])
    assert msg is None, msg


def _bed(stages, n, u):
    st = stages(n)
    return W.Bed(u, st["lookup"], st["particles"], st["affine"], st.get("bed_extract", np.zeros((0, 8), np.float32)))


def test_classify(stages):
    u = stages.uniforms(P_CLASSIFY)
    before, after = stages(P_CLASSIFY), stages(P_CLASSIFY + 1)
    sdf = W.Sdf(u, stages.static["sdf"])
    solid = stages.static["sdf_class"].reshape(u.grid_shape()) != 0
    lanes = W.classify(u, before["lanes"], before["grid_vel"], _bed(stages, P_CLASSIFY, u), sdf, solid,
                       bool(stages.settings.raw.use_sdf_cache))
    for lane, name in ((3, "kind"), (1, "divergence"), (0, "pressure"), (2, "lane 2"), (4, "rest volume"), (5, "current volume")):
        msg = _report(name, lanes[lane], after["lanes"][lane])
        assert msg is None, msg


def test_rbgs_fixed_pairs(stages):
    """The reference configuration: fixed-point pressure, `pressure_rbgs_pairs` red+black
    pairs from the cold start (mod.rs:352-357)."""
    raw = stages.settings.raw
    assert raw.pressure_storage == 0 and raw.solve_mode == 0 and raw.rbgs_omega in (0.0, 1.0)
    u = stages.uniforms(P_RBGS)
    before, after = stages(P_RBGS), stages(P_RBGS + 1)
    lanes = W.rbgs(u, before["lanes"], int(raw.pressure_rbgs_pairs))
    assert np.count_nonzero(after["lanes"][0]) > 100
    msg = _report("pressure", lanes[0], after["lanes"][0])
    assert msg is None, msg


def test_project_with_darcy_drag(stages):
    u = stages.uniforms(P_PROJECT)
    before, after = stages(P_PROJECT), stages(P_PROJECT + 1)
    gv, imp = W.project(u, before["lanes"], before["grid_vel"], _bed(stages, P_PROJECT, u))
    kind = before["lanes"][3]
    darcy = (kind == W.CELL_BED_COUPLED) & (before["grid_vel"][:, 3] >= 1e-6) & (before["lookup"] >= 0)
    assert np.count_nonzero(darcy) > 50
    msg = _report("grid_vel", gv, after["grid_vel"])
    assert msg is None, msg
    added = after["bed_delta"][1:4, :u.num_bed].astype(np.int64) - before["bed_delta"][1:4, :u.num_bed]
    assert np.count_nonzero(imp) > 0
    msg = _report("bed impulse lanes", W.wrap_i32(imp), W.wrap_i32(added))
    assert msg is None, msg


def test_packing(stages):
    u = stages.uniforms(P_PACK_PREP)
    before, mid, after = stages(P_PACK_PREP), stages(P_PACK_APPLY), stages(P_PACK_APPLY + 1)
    lanes = W.packing_prepare(u, before["lanes"])
    msg = _report("lanes", lanes.reshape(6, -1), mid["lanes"])
    assert msg is None, msg
    gv = W.packing_apply(u, mid["lanes"], mid["grid_vel"])
    msg = _report("grid_vel", gv, after["grid_vel"])
    assert msg is None, msg


def test_viscosity(stages):
    u = stages.uniforms(P_VISC_PREP)
    assert u.viscosity > 0
    before, mid, after = stages(P_VISC_PREP), stages(P_VISC_APPLY), stages(P_VISC_APPLY + 1)
    solid = stages.static["sdf_class"].reshape(u.grid_shape()) != 0
    lanes = W.viscosity_prepare(u, before["lanes"], before["grid_vel"], solid)
    msg = _report("lanes", lanes, mid["lanes"])
    assert msg is None, msg
    scratch = W.lane_f32(u, mid["lanes"][1:4]).T
    blended = np.count_nonzero(np.any(scratch != before["grid_vel"][:, :3], axis=1) & (before["grid_vel"][:, 3] > 2 * u.nominal_mass))
    assert blended > 50
    gv = W.viscosity_apply(u, mid["lanes"], mid["grid_vel"])
    msg = _report("grid_vel", gv, after["grid_vel"])
    assert msg is None, msg


def test_g2p(stages):
    """G2P with APIC, weak-support and airborne ballistic blending, porous drag with its
    bed impulses, the J update and the particle-level contacts.  Every value is compared
    bit for bit except J, whose exponential (shader.rs:1853) WGSL leaves to the backend
    (within 4 ulp here, the restatement using float64 exp rounded to float32)."""
    raw = stages.settings.raw
    g = raw.geom
    assert (g.cone_bot_y, g.cone_top_y, g.cup_top_y, g.cup_radius, g.cup_floor_y, g.wall_thickness) == \
        (-3.0, 3.0, -3.5, 3.0, -8.0, np.float32(0.4))
    assert g.cone_radius_span == np.float32(4.2634315)
    u = stages.uniforms(P_G2P)
    before, after = stages(P_G2P), stages(P_G2P + 1)
    sdf = W.Sdf(u, stages.static["sdf"])
    stats = {}
    P, A, imp = W.g2p(u, sdf, _bed(stages, P_G2P, u), np.float32(raw.brew.dripper_outlet_radius),
                      before["particles"], before["affine"], before["grid_vel"], stats=stats)
    assert min(stats["weak"], stats["airborne"], stats["porous"]) > 50, stats
    want_p, want_a = after["particles"], after["affine"]
    cols = [c for c in range(8) if c != 3]
    msg = _report("particles (J excluded)", P[:, cols], want_p[:, cols])
    assert msg is None, msg
    j_ulp = np.abs(P[:, 3].view(np.int32).astype(np.int64) - want_p[:, 3].view(np.int32).astype(np.int64))
    assert j_ulp.max() <= 4, f"J differs by {j_ulp.max()} ulp"
    msg = _report("affine", A, want_a)
    assert msg is None, msg
    added = after["bed_delta"][1:4, :u.num_bed].astype(np.int64) - before["bed_delta"][1:4, :u.num_bed]
    msg = _report("bed impulse lanes", W.wrap_i32(imp), W.wrap_i32(added))
    assert msg is None, msg
    assert np.count_nonzero(imp) > 0


P_LOOKUP_CLEAR, P_COUPLING, P_EXTRACTION, P_RENDER = 1, 17, 18, 20


def test_bed_lookup(stages):
    u = stages.uniforms(P_LOOKUP_CLEAR)
    before, after = stages(P_LOOKUP_CLEAR), stages(P_LOOKUP_CLEAR + 2)
    look = W.bed_lookup(u, before["particles"], before["affine"])
    assert np.count_nonzero(look >= 0) > 1000
    msg = _report("lookup", look, after["lookup"])
    assert msg is None, msg


def test_bed_coupling(stages):
    u = stages.uniforms(P_COUPLING)
    before, after = stages(P_COUPLING), stages(P_COUPLING + 1)
    P, add = W.bed_coupling(u, _bed(stages, P_COUPLING, u), before["particles"], before["affine"])
    assert np.count_nonzero(add) > 20
    msg = _report("particles", P, after["particles"])
    assert msg is None, msg
    got = after["bed_delta"][0, :u.num_bed].astype(np.int64) - before["bed_delta"][0, :u.num_bed]
    msg = _report("bed water lane", W.wrap_i32(add), W.wrap_i32(got))
    assert msg is None, msg


def test_extraction_advect(stages):
    u = stages.uniforms(P_EXTRACTION)
    before, after = stages(P_EXTRACTION), stages(P_EXTRACTION + 1)
    be = W.extraction_advect(u, before["bed_extract"], before["bed_delta"][0])
    assert np.count_nonzero(before["bed_delta"][0, :u.num_bed]) > 20
    msg = _report("bed_extract", be, after["bed_extract"])
    assert msg is None, msg
    assert not after["bed_delta"][0, :u.num_bed].any()


def test_prepare_render(stages):
    u = stages.uniforms(P_RENDER)
    before = stages(P_RENDER)
    sim = MpmSim3D(stages.settings, stages.oracle)
    copy_state(stages.src, sim)
    sim.set_kettle_angle(36.0)
    sim.step_substep_partial(SUB_DT, P_RENDER + 1)
    want = sim.read_render(0, sim.particle_count())
    got = W.prepare_render(u, before["particles"], before["affine"], before.get("bed_extract"))
    msg = _report("render", got, want)
    assert msg is None, msg


P_BED_DYNAMICS = 19


def test_bed_dynamics(stages):
    """bed_dynamics with the other samples' positions read from before the dispatch (the
    WGSL reads them while they are written; the oracle and the engine read a snapshot)."""
    raw = stages.settings.raw
    g = raw.geom
    assert (g.filter_center_y, g.filter_top_rel, g.filter_bot_rel) == (np.float32(-0.35), np.float32(2.75), np.float32(3.02))
    assert (g.filter_top_radius, g.filter_thickness) == (np.float32(4.10), np.float32(0.08))
    assert (g.bed_surface_ref_y, g.bed_surface_span) == (3.0, 3.5)
    u = stages.uniforms(P_BED_DYNAMICS)
    before, after = stages(P_BED_DYNAMICS), stages(P_BED_DYNAMICS + 1)
    sdf = W.Sdf(u, stages.static["sdf"])
    nb = u.num_bed
    P, A, BE = W.bed_dynamics(u, sdf, np.float32(raw.brew.dripper_outlet_radius), before["lanes"],
                              before["grid_vel"], before["lookup"], before["particles"], before["affine"],
                              before["bed_extract"], before["bed_delta"][1:4])
    moved = np.count_nonzero(np.any(before["particles"][:nb, 0:3] != after["particles"][:nb, 0:3], axis=1))
    assert moved > 1000
    if stages.name == "scattered":
        suspended = before["affine"][:nb, 3] >= 1.5
        assert suspended.sum() > 1000
        assert np.count_nonzero(before["affine"][:nb, 3] != after["affine"][:nb, 3]) > 1000
    for name, got, want in (("bed particles", P, after["particles"][:nb]), ("bed affine", A, after["affine"][:nb]),
                            ("bed_extract", BE, after["bed_extract"])):
        msg = _report(name, got, want)
        assert msg is None, msg
    assert not after["bed_delta"][1:4, :nb].any()


def _scene(name, oracle):
    from coffee_sim_b200 import scenes
    if name == "center_pour":
        return MpmSettings.benchmark_center_pour(oracle)
    return scenes.c2_v60(oracle, grid=64, max_particles=1000)


@pytest.mark.parametrize("name", ["center_pour", "v60_si_64cube"])
def test_sdf_texture_and_solid_class(oracle, name):
    """The static SDF texture and the per-cell solid class the simulation is created with
    (state.rs:206-344), for the reference's scene and for an SI-unit V60 scene (whose wall
    thickness is its own, in its units)."""
    s = _scene(name, oracle)
    sim = MpmSim3D(s, oracle)
    if name == "center_pour":
        assert s.raw.geom.wall_thickness == np.float32(0.4)
    sdf = W.generate_sdf(s.raw, s.raw.geom.wall_thickness)
    assert np.count_nonzero(sdf < 900) > 1000
    msg = _report("sdf", sdf, sim.read_sdf())
    assert msg is None, msg
    cls = W.generate_sdf_class(s.raw, sdf)
    assert cls.any() and not cls.all()
    msg = _report("sdf class", cls, sim.read_sdf_class())
    assert msg is None, msg


def test_inflow_emission(oracle):
    """Jet emission of the reference's centre pour at 36 degrees over 12 substeps (no
    dispatch runs, so the samples stay where they were emitted): counts, velocities,
    masses and J exact; positions within 1 ulp (cos/sin of the golden angle)."""
    s = MpmSettings.benchmark_center_pour(oracle)
    sim = MpmSim3D(s, oracle)
    sim.set_kettle_angle(36.0)
    jet = W.Inflow(s.raw, 36.0)
    nb = sim.num_bed
    rows = []
    for _ in range(12):
        rows.append(jet.emit(SUB_DT, sim.particle_count(), int(s.raw.max_particles)))
        sim.step_substep_partial(SUB_DT, 0)
    want = sim.read_particles(nb, sim.num_water)
    got = np.concatenate(rows)
    assert got.shape == want.shape and got.shape[0] > 50
    msg = _report("emitted samples (positions excluded)", got[:, 3:], want[:, 3:])
    assert msg is None, msg
    ulp = np.abs(got[:, 0:3].view(np.int32).astype(np.int64) - want[:, 0:3].view(np.int32))
    assert ulp.max() <= 1, f"positions differ by up to {ulp.max()} ulp"
    assert np.float32(sim.flow_rate_ml_s()) == jet.flow_rate and np.float32(sim.exit_speed()) == jet.exit_speed


def test_whole_substeps_chained(stages):
    """Three whole substeps of the restatement, each dispatch fed by the previous one
    (the dispatch order and lane aliasing of mod.rs:305-414 included), against three
    whole substeps of the oracle from the same state: every sample, affine column and
    bed_extract value bit for bit, except J (the backend's exp; 2 ulp at most measured)."""
    raw = stages.settings.raw
    stages(P_P2G)                      # loads the static SDF texture and solid class
    sim = MpmSim3D(stages.settings, stages.oracle)
    copy_state(stages.src, sim)
    sim.set_kettle_angle(36.0)
    nw, nb = sim.num_water, sim.num_bed
    P, A = sim.read_particles(0, nw + nb), sim.read_affine(0, nw + nb)
    BE = sim.read_bed_extract(0, nb)
    jet = W.Inflow(raw, 36.0)
    for _ in range(3):
        P, A, BE, nw = W.substep(raw, stages.static["sdf"], stages.static["sdf_class"], jet, P, A, BE, nw, nb, SUB_DT)
        sim.step_substep(SUB_DT)
    assert sim.num_water == nw
    want_p, want_a = sim.read_particles(0, nw + nb), sim.read_affine(0, nw + nb)
    cols = [c for c in range(8) if c != 3]
    msg = _report("particles (J excluded)", P[:, cols], want_p[:, cols])
    assert msg is None, msg
    j_ulp = np.abs(P[:, 3].view(np.int32).astype(np.int64) - want_p[:, 3].view(np.int32))
    assert j_ulp.max() <= 4, j_ulp.max()
    for name, got, want in (("affine", A, want_a), ("bed_extract", BE, sim.read_bed_extract(0, nb))):
        msg = _report(name, got, want)
        assert msg is None, msg
    sim.close()


def test_int64_p2g_and_grid_update(oracle, pour_state_int64):
    """The engine's 64-bit P2G mode (the headline workload's): lanes as i64 * 2^32 with a
    wrapping 64-bit sum, and grid_update reading them back as f32(lane) * 2^-32."""
    s, src = pour_state_int64
    sims = []
    for n in (P_P2G, P_P2G + 1, P_GRID_UPDATE + 1):
        sim = MpmSim3D(s, oracle)
        copy_state(src, sim)
        sim.set_kettle_angle(36.0)
        sim.step_substep_partial(SUB_DT, n)
        sims.append(sim)
    before, after_p2g, after_gu = sims
    u = W.Uniforms(s.raw, before.num_water, before.num_bed, SUB_DT)
    n = before.particle_count()
    lanes64 = W.p2g(u, before.read_particles(0, n), before.read_affine(0, n), int64=True)
    assert np.count_nonzero(lanes64[0]) > 1000
    msg = _report("int64 lanes", lanes64, after_p2g.read_grid_lanes64())
    assert msg is None, msg
    gv = W.grid_update(u, after_p2g.read_grid_lanes64())
    msg = _report("grid_vel", gv, after_gu.read_grid_vel())
    assert msg is None, msg


@pytest.fixture(scope="module")
def pour_state_int64(oracle):
    from coffee_sim_b200 import _ffi
    s, src = _pour(oracle)
    s = s.copy()
    s.raw.p2g_mode = _ffi.CS_P2G_INT64
    return s, src


def test_reorder_permutation(oracle, stages):
    """The engine's sample reorder (`reorder_every`): the oracle's permutation of the water
    slots equals a stable sort by the tile key described in the header.  With no dispatch
    run, the state after the substep is the reordered state plus the new jet samples."""
    s = stages.settings.copy()
    s.raw.reorder_every = 1
    sim = MpmSim3D(s, oracle)
    copy_state(stages.src, sim)
    sim.set_kettle_angle(36.0)
    nw, nb = sim.num_water, sim.num_bed
    P, A = sim.read_particles(0, nw + nb), sim.read_affine(0, nw + nb)
    u = W.Uniforms(s.raw, nw, nb, SUB_DT)
    perm = W.reorder_permutation(u, P, A)
    assert np.count_nonzero(perm != np.arange(nw)) > nw // 2
    sim.step_substep_partial(SUB_DT, 0)
    got_p = sim.read_particles(nb, nw)
    got_a = sim.read_affine(nb, nw)
    msg = _report("reordered samples", P[nb:][perm], got_p)
    assert msg is None, msg
    msg = _report("reordered affine", A[nb:][perm], got_a)
    assert msg is None, msg
    sim.close()


@pytest.mark.parametrize("grid,omega,cap,first", [(32, 1.9, 20, 0), (64, 1.92, 60, 125)])
def test_refinement_solve_cold_start(oracle, grid, omega, cap, first):
    """The engine's residual-mode solve (FP32 pressure words, FP64 residual checks,
    over-relaxed correction sweeps, predicted check intervals) restated in numpy from the
    solver inputs the oracle's classify wrote, on the SI-unit V60 pour from a cold start
    (at 64^3 with the bench's omega, check cap and first check): same pair and check
    counts, the pressure's high word bit for bit, and the residuals within 1e-9 relative
    (the oracle sums its FP64 norms per thread)."""
    from coffee_sim_b200 import _ffi, scenes
    s = scenes.c2_v60(oracle, grid=grid, max_particles=340000)
    r = s.raw
    r.warm_start = _ffi.CS_WARM_NONE
    r.rbgs_omega, r.check_every, r.first_check, r.max_sweeps = omega, cap, first, 3000
    sims = []
    for n in (P_CLASSIFY + 1, P_RBGS + 1):
        sim = MpmSim3D(s, oracle)
        assert scenes.populate_c2(sim) > 10000
        sim.step_substep_partial(scenes.C2_DT, n)
        sims.append(sim)
    a, b = sims
    u = W.Uniforms(r, a.num_water, a.num_bed, scenes.C2_DT)
    fill, div = a.read_solver_inputs()
    hi, lo, pairs, checks, r0, r1 = W.refine_solve(u, a.read_cell_kind(), fill, div, r.rbgs_omega,
                                                   r.residual_tol, r.check_every, r.first_check, r.max_sweeps)
    m = b.latest_metrics()
    assert 20 < pairs < r.max_sweeps and r1 <= 1e-5
    assert (pairs, checks) == (m.last_sweeps, m.residual_checks)
    assert abs(r0 - m.initial_residual) <= 1e-9 * r0 and abs(r1 - m.last_residual) <= 1e-9 * r1
    msg = _report("pressure (high word)", hi, b.read_pressure())
    assert msg is None, msg


def test_bed_seeding(oracle):
    """The seeded bed of the reference's scene: BedConfig::seated_in_filter (bed.rs:41-82),
    the lattice with its rounded bottom and the downsampling to the target count
    (bed.rs:107-226), and the initial cell lookup (bed.rs:228-314), against the
    simulation the oracle creates."""
    s = MpmSettings.benchmark_center_pour(oracle)
    b = s.raw.bed
    assert b.log_perm_sigma == 0.0 and b.lower_porosity_scale in (0.0, 1.0)
    seat = W.seated_in_filter(s.raw.filter)
    assert tuple(np.float32(v) for v in (b.center[1], b.top_y, b.bot_y, b.top_radius, b.bot_radius)) == seat
    sim = MpmSim3D(s, oracle)
    P, A, BE, look = W.init_bed(b, s.raw.grid_dims, s.raw.bounds_size)
    nb = sim.num_bed
    assert nb == P.shape[0] == 12000
    for name, got, want in (("bed samples", P, sim.read_particles(0, nb)), ("bed affine", A, sim.read_affine(0, nb)),
                            ("bed_extract", BE, sim.read_bed_extract(0, nb)), ("lookup", look, sim.read_bed_lookup())):
        msg = _report(name, got, want)
        assert msg is None, msg
    sim.close()


@pytest.mark.parametrize("name", ["default_v60", "benchmark_free_stream", "benchmark_center_pour"])
def test_reference_presets(oracle, name):
    """The reference's scene presets (mod.rs:105-177) with the spout defaults and aim
    (inflow.rs:27-59), units (units.rs:9-33) and brew constants (brew_config.rs:38-96),
    restated as float32 arithmetic, against the settings the oracle's preset fills."""
    want = W.reference_presets()[name]
    s = getattr(MpmSettings, name)(oracle).raw
    f = np.float32
    assert [f(v) for v in s.bounds_size] == want["bounds_size"]
    assert list(s.grid_dims) == want["grid_dims"]
    assert (s.max_particles, s.substeps, s.pressure_rbgs_pairs, s.use_sdf_cache) == \
        (want["max_particles"], want["substeps"], want["pressure_rbgs_pairs"], want["use_sdf_cache"])
    for k in ("gravity", "bulk_modulus", "viscosity", "render_radius", "initial_kettle_angle_deg"):
        assert f(getattr(s, k)) == want[k], k
    u = want["units"]
    assert (f(s.sim_units_per_meter), f(s.max_velocity)) == (u["sim_units_per_meter"], u["max_velocity"])
    cone, cup = s.obstacles[0], s.obstacles[1]
    assert s.num_obstacles == 2 and list(cone.center) == [0.0, 0.0, 0.0] and list(cup.center) == [0.0, 0.0, 0.0]
    for k, v in want["cone"].items():
        assert f(getattr(cone, k)) == v, k
    for k, v in want["cup"].items():
        assert f(getattr(cup, k)) == v, k
    sp = want["spout"]
    for k, v in sp.items():
        got = getattr(s.spout, k)
        got = [f(x) for x in got] if isinstance(v, list) else f(got)
        assert got == v, (k, got, v)
    for k, v in want["brew"].items():
        if hasattr(s.brew, k):
            assert f(getattr(s.brew, k)) == v, k
    assert s.has_bed == want["has_bed"]
    if s.has_bed:
        assert f(s.bed.initial_permeability) == want["bed_permeability"]
        assert f(s.bed.initial_porosity) == want["brew"]["bed_porosity"]
        assert s.bed.num_particles == want["brew"]["bed_particle_samples"]


def test_classify_without_sdf_cache(oracle, stages):
    """classify_cells with `use_sdf_cache` off: the solid tests sample the SDF texture at
    the cell centre and at the six neighbour centres (shader.rs:1203-1207, 1279-1326)."""
    s = stages.settings.copy()
    s.raw.use_sdf_cache = 0
    sims = []
    for n in (P_CLASSIFY, P_CLASSIFY + 1):
        sim = MpmSim3D(s, oracle)
        copy_state(stages.src, sim)
        sim.set_kettle_angle(36.0)
        sim.step_substep_partial(SUB_DT, n)
        sims.append(sim)
    before, after = sims
    u = W.Uniforms(s.raw, before.num_water, before.num_bed, SUB_DT)
    sdf = W.Sdf(u, before.read_sdf())
    n = before.particle_count()
    bed = W.Bed(u, before.read_bed_lookup(), before.read_particles(0, n), before.read_affine(0, n),
                before.read_bed_extract(0, before.num_bed))
    lanes = W.classify(u, before.read_grid_lanes(), before.read_grid_vel(), bed, sdf, None, False)
    want = after.read_grid_lanes()
    assert np.count_nonzero(want[3] == W.CELL_SOLID) > 1000
    for lane in (3, 1, 0):
        msg = _report(f"lane {lane}", lanes[lane], want[lane])
        assert msg is None, msg
