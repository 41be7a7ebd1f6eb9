"""Seeded synthetic scenes for the benchmark configurations.

The reference has no generator for these workloads; they are restated here from the
configuration text.  Two conventions hold everywhere:

* The configurations are stated in SI; each scene runs in a length unit of
  1/U metre (U = `sim_units_per_meter`) with every length, speed, acceleration and
  grid viscosity converted.  The reference's fixed-point grid stores volumes,
  momenta and pressures as i32 * 2^18 clamped to +/-8192 (state.rs:13-19), a window
  sized for its own scene unit (1 su = 1/57.7 m, dx = 0.175 su).  In metres a sample
  volume (~1e-9 m^3) truncates to zero quanta, which zeroes every surface cell's
  fill fraction and leaves the pressure system without Dirichlet faces.  U is
  chosen per scene so the sample volume spans hundreds of quanta and the largest
  hydrostatic/impact pressure stays inside the clamp: C1 runs in decimetres
  (U = 10), the V60 scenes at U = 80 (dx = 0.2 units).  The domain is centred on the
  origin as in the reference (mod.rs:603-604), so a [0,1]^3 box runs as
  [-0.5,0.5]^3.
* Mass is in the reference's mass units: a water sample has nominal mass 0.25
  (brew_config.rs:48-49 gives 80/320).  The fixed-point grid (2^18 per unit,
  state.rs:13) is scaled for that; rho = 1000 kg/m^3 maps one mass unit to
  4 * rho * V_sample kg, so only mass ratios enter the solve.
"""
import math
import random

import numpy as np

from . import _ffi
from .sim import MpmSettings


def _si_base(lib, U, bounds_m, grid, max_particles, particles_per_cell, p_vol_cells):
    """Settings for an SI-specified scene run in units of 1/U metre."""
    s = MpmSettings.default_v60(lib)
    r = s.raw
    r.bounds_size[:] = [b * U for b in bounds_m]
    r.grid_dims[:] = grid
    r.max_particles = max_particles
    r.substeps = 1
    r.gravity = -9.81 * U
    r.sim_units_per_meter = U
    r.standard_gravity_m_s2 = 9.80665
    r.max_velocity = 3.0 * U
    r.max_frame_dt = 1.0
    dx_m = bounds_m[0] / grid[0]
    cell_ml = dx_m ** 3 * 1.0e6
    r.brew.water_particles_per_ml = particles_per_cell / cell_ml
    r.brew.water_mass_units_per_ml = 0.25 * r.brew.water_particles_per_ml
    r.particle_volume_cells = p_vol_cells
    r.render_radius = dx_m * U * 0.7
    r.spout.volume_to_ml = 1.0e6 / U ** 3
    r.spout.max_flow_rate_ml_s = 1.0e6
    r.spout.gentle_exit_speed = 0.12 * U
    r.spout.max_exit_speed = 0.45 * U
    g = r.geom
    g.contact_offset = 0.001 * U
    g.wall_thickness = 0.002 * U
    return s


def c1_water_block(lib=None, pairs=40):
    """Plain MLS-MPM water block: 32^3 grid, dx = 1/32 over [0,1]^3 (run as
    [-0.5,0.5]^3); 2x2x2 samples per cell with +/-0.25 dx uniform jitter (seed 0)
    filling [0.3,0.7]x[0.5,0.9]x[0.3,0.7]; gravity -9.81; substep dt 5e-4;
    viscosity nu = 1e-6; `pairs` red+black RBGS pairs; box walls only; no bed.
    Sample rest volume is dx^3/8 (the reference uses /4 for its sparser jet)."""
    s = _si_base(lib, C1_U, (1.0, 1.0, 1.0), (32, 32, 32), 20000, 8.0, 0.125)
    r = s.raw
    r.num_obstacles = 0
    r.has_bed = 0
    r.has_filter = 0
    r.geom.flags = 0
    r.viscosity = 1.0e-6 * C1_U ** 2
    r.pressure_rbgs_pairs = pairs
    r.initial_kettle_angle_deg = 0.0
    return s


C1_U = 10.0
C1_BLOCK = ((-0.2 * C1_U, 0.0, -0.2 * C1_U), (0.2 * C1_U, 0.4 * C1_U, 0.2 * C1_U))
C1_DT = 5.0e-4


def populate_c1(sim, seed=0):
    lo, hi = C1_BLOCK
    return sim.add_water_block(lo, hi, per_axis=2, jitter=0.25, seed=seed)


# ---------------- V60 pour-over (stated in metres, run at U = 80 units/m) ----------------
V60_U = 80.0
V60_HALF_ANGLE = math.radians(30.0)     # 60 degree full apex angle
V60_OUTLET_R = 0.004                    # 4 mm outlet (radius), metres
V60_BOT_Y, V60_TOP_Y = -0.04, 0.06      # 10 cm tall support cone, metres
V60_DOMAIN = 0.16                       # cube side, metres


def _v60_geometry(s, bed_samples, seed, U, log_sigma=0.5, log_mu=math.log(1e-9)):
    r = s.raw
    tan = math.tan(V60_HALF_ANGLE)
    span = (V60_TOP_Y - V60_BOT_Y) * tan
    r.num_obstacles = 1
    cone = r.obstacles[0]
    cone.kind = _ffi.CS_OBSTACLE_TRUNCATED_CONE
    cone.center[:] = (0.0, 0.0, 0.0)
    cone.bot_radius = V60_OUTLET_R * U
    cone.top_radius = (V60_OUTLET_R + span) * U
    cone.bot_y = V60_BOT_Y * U
    cone.top_y = V60_TOP_Y * U
    g = r.geom
    g.flags = _ffi.CS_GEOM_CONE | _ffi.CS_GEOM_FILTER
    g.cone_bot_y = V60_BOT_Y * U
    g.cone_top_y = V60_TOP_Y * U
    g.cone_radius_span = span * U
    r.brew.dripper_outlet_radius = V60_OUTLET_R * U
    # paper filter: a cone on the support cone's inner face, tip below the outlet
    tip_y = V60_BOT_Y - V60_OUTLET_R / tan
    g.filter_center_y = 0.0
    g.filter_top_rel = V60_TOP_Y * U
    g.filter_bot_rel = -tip_y * U
    g.filter_top_radius = (V60_OUTLET_R + span) * U
    g.filter_thickness = 0.0005 * U
    g.cup_top_y = -1.0e9
    r.has_filter = 1
    r.filter.center[:] = (0.0, 0.0, 0.0)
    r.filter.top_y = V60_TOP_Y * U
    r.filter.bot_y = tip_y * U
    r.filter.top_radius = (V60_OUTLET_R + span) * U
    r.filter.bot_radius = 0.0
    r.filter.thickness = 0.0005 * U
    r.filter.hole_radius = 0.0
    # bed in the lower 30 % of the cone (porosity 0.4, log-normal k in m^2)
    bed_top = V60_BOT_Y + 0.3 * (V60_TOP_Y - V60_BOT_Y)
    margin = 0.002
    r.has_bed = 1
    b = r.bed
    b.center[:] = (0.0, 0.0, 0.0)
    b.bot_y = (V60_BOT_Y + 0.5 * margin) * U
    b.top_y = bed_top * U
    b.bot_radius = max(V60_OUTLET_R - 0.5 * margin, 0.001) * U
    b.top_radius = (V60_OUTLET_R + (bed_top - V60_BOT_Y) * tan - margin) * U
    b.num_particles = bed_samples
    b.initial_porosity = 0.4
    b.initial_permeability = math.exp(log_mu)
    b.extractable_mass = 0.15
    b.log_perm_sigma = log_sigma
    b.perm_seed = seed
    b.layer_split_y = -1.0e30
    b.lower_porosity_scale = 1.0
    b.lower_permeability_scale = 1.0
    g.bed_surface_ref_y = -V60_BOT_Y * U
    g.bed_surface_span = (bed_top - V60_BOT_Y) * 1.15 * U
    # bed water retention scaled from the reference's 42 ml per 12k samples / 15 g dose
    r.brew.target_bed_retention_ml = 6.0 * bed_samples / 3000.0
    # spout: centre pour from 1.5 cm above the rim
    sp = r.spout
    sp.origin[:] = (0.0, (V60_TOP_Y + 0.015) * U, 0.0)
    sp.direction[:] = (0.0, -1.0, 0.0)
    sp.target[:] = (0.0, 0.0, 0.0)
    sp.nozzle_radius = 0.004 * U
    r.initial_kettle_angle_deg = 20.0
    r.flow_override_ml_s = 4.0
    r.exit_speed_override = 0.8 * U


def c2_v60(lib=None, grid=64, max_particles=340000, bed_samples=3000, seed=1, U=V60_U):
    """V60 pour-over, plain method: 64^3 grid over a 16 cm cube; support cone with a
    60 degree full apex angle and 4 mm outlet; Darcy bed in the lower 30 % of the cone
    (porosity 0.4, log-normal permeability mu = ln 1e-9 m^2, sigma = 0.5, seed 1); jet
    4 ml/s at 0.8 m/s with 8 samples per cell volume, kettle angle 20 deg, centre pour;
    RBGS to relative residual 1e-5 with the previous substep's pressure as warm start."""
    L = V60_DOMAIN
    s = _si_base(lib, U, (L, L, L), (grid, grid, grid), max_particles, 8.0, 0.125)
    _v60_geometry(s, bed_samples, seed, U)
    r = s.raw
    r.viscosity = 1.0e-6 * U * U
    r.pressure_storage = _ffi.CS_PRESSURE_FP32
    r.solve_mode = _ffi.CS_SOLVE_RESIDUAL
    r.residual_tol = 1.0e-5
    r.max_sweeps = 2000
    r.check_every = 10
    r.warm_start = _ffi.CS_WARM_PREVIOUS
    return s


C2_DT = 5.0e-4


def populate_c2(sim, fill_top=0.05, pool_depth=0.012, seed=1):
    """Mid-pour state of the V60 scene: water above the bed up to `fill_top` inside
    the cone, and a carafe pool `pool_depth` deep on the domain floor (8 samples per
    cell, +/-0.25 dx jitter).  Lengths in metres.  Returns the samples added."""
    U = float(sim.settings.sim_units_per_meter)
    L = V60_DOMAIN
    dx = L / sim.settings.grid_dims[0]
    bed_top = V60_BOT_Y + 0.3 * (V60_TOP_Y - V60_BOT_Y)
    r_top = V60_OUTLET_R + (fill_top - V60_BOT_Y) * math.tan(V60_HALF_ANGLE)
    n = sim.add_water_block((-r_top * U, (bed_top + dx) * U, -r_top * U), (r_top * U, fill_top * U, r_top * U),
                            per_axis=2, jitter=0.25, seed=seed, require_open_sdf=True)
    lo = -L / 2 + 2.5 * dx
    n += sim.add_water_block((lo * U, lo * U, lo * U), (-lo * U, (lo + pool_depth) * U, -lo * U),
                             per_axis=2, jitter=0.25, seed=seed + 1000, require_open_sdf=True)
    return n


def spiral_spout(t, radius=0.015, hz=0.5, y=V60_TOP_Y + 0.015, U=V60_U):
    """Spout origin on the spiral pour path (radius 1.5 cm, 0.5 Hz), in scene units."""
    a = 2.0 * math.pi * hz * t
    return (radius * math.cos(a) * U, y * U, radius * math.sin(a) * U)


def c3_large(lib=None, grid=128, max_particles=2_700_000, bed_samples=24000, seed=2):
    """Large V60 pour: 128^3 over the same 16 cm cube (dx = 1.25 mm) with the C2 cone,
    bed and jet generators (seed 2); `populate_c2` gives ~2.2M samples at this grid.
    The spout follows the spiral pour path: the caller moves it every substep with
    set_spout_position(*spiral_spout(t)).  Bed samples scale with the cell count so
    the bed keeps its sample density.  P2G runs cell-sorted with shared-memory tiles."""
    s = c2_v60(lib, grid=grid, max_particles=max_particles, bed_samples=bed_samples, seed=seed)
    s.raw.p2g_mode = _ffi.CS_P2G_SORTED_SHARED
    return s


def c5_scale(lib=None, grid=192, max_particles=8_600_000, bed_samples=81000, seed=4):
    """Scale and reproducibility sweep: 192^3 (dx = 0.83 mm, ~7.6M samples from
    `populate_c2`); two-layer bed split at its mid-height, porosity 0.45 above and 0.35
    below with a 10x lower permeability below; the pour 1.2 cm off centre; int64
    fixed-point P2G (bit-reproducible grid)."""
    s = c2_v60(lib, grid=grid, max_particles=max_particles, bed_samples=bed_samples, seed=seed)
    r = s.raw
    U = float(r.sim_units_per_meter)
    b = r.bed
    b.layer_split_y = 0.5 * (b.bot_y + b.top_y)
    b.initial_porosity = 0.45
    b.lower_porosity_scale = 0.35 / 0.45
    b.lower_permeability_scale = 0.1
    r.spout.origin[0] = 0.012 * U
    r.p2g_mode = _ffi.CS_P2G_INT64
    return s


def c4_ensemble(lib=None, n=64, seed=3, grid=64, max_particles=340000):
    """Batched ensemble: n independent V60 pours at 64^3 with seeded per-instance
    parameters — water fill height and carafe pool depth (sample counts spread over
    about 20k-300k), flow rate U[2, 6] ml/s, kettle angle U[10, 35] deg, and bed
    log-permeability mean U[ln 5e-10, ln 2e-9] m^2.  Returns (settings list, per-instance
    populate arguments)."""
    rng = random.Random(seed)
    settings, fills = [], []
    bed_top = V60_BOT_Y + 0.3 * (V60_TOP_Y - V60_BOT_Y)
    for i in range(n):
        s = c2_v60(lib, grid=grid, max_particles=max_particles, seed=seed * 1000 + i)
        r = s.raw
        r.bed.initial_permeability = math.exp(rng.uniform(math.log(5e-10), math.log(2e-9)))
        r.initial_kettle_angle_deg = rng.uniform(10.0, 35.0)
        r.flow_override_ml_s = rng.uniform(2.0, 6.0)
        settings.append(s)
        fills.append({"fill_top": rng.uniform(bed_top + 0.006, 0.05), "pool_depth": rng.uniform(0.0, 0.012),
                      "seed": seed * 1000 + i})
    return settings, fills
