"""Reductions over particle readbacks that the reference's GPU scenario tests assert on,
restated over numpy arrays in the reference byte layouts (particles: 8 f32 per sample,
`pos.xyz, J, vel.xyz, mass`, bed samples first; bed_extract: 8 f32 per bed sample).

Each function follows one readback helper of
crates/sim-wasm/src/mpm_3d/physics_tests.rs and cites it.  Sums are taken in float64
(the reference sums in f32; the tolerances the tests use are far wider than that
difference).
"""
from dataclasses import dataclass

import numpy as np

F = np.float32


def nominal_mass(settings):
    """inflow::MASS_UNITS_PER_ML / inflow::PARTICLES_PER_ML."""
    b = settings.raw.brew
    return F(b.water_mass_units_per_ml) / F(b.water_particles_per_ml)


def dx_of(settings):
    return F(settings.raw.bounds_size[0]) / F(settings.raw.grid_dims[0])


def _finite(*arrays):
    return bool(all(np.isfinite(a).all() for a in arrays))


@dataclass
class Mass:
    active_particle_mass: float
    active_water_particle_mass: float
    bed_held_mass: float
    water_slots: int


def mass_snapshot(sim):
    """readback_mass_snapshot (physics_tests.rs:61-140): mass of every sample, of the
    water samples, and the water held in bed pores (bed_extract lane 0)."""
    nb, nw = sim.num_bed, sim.num_water
    p = sim.read_particles(0, nb + nw)
    m = p[:, 7].astype(np.float64)
    held = sim.read_bed_extract(0, nb)[:, 0].astype(np.float64) if nb else np.zeros(0)
    return Mass(float(m.sum()), float(m[nb:].sum()), float(held.sum()), nw)


@dataclass
class WaterVolume:
    all_finite: bool
    active_count: int
    active_mass: float
    rest_volume: float
    current_volume: float
    mean_j: float
    min_j: float
    max_j: float


def water_volume_snapshot(sim, settings):
    """readback_water_particle_volume_snapshot (physics_tests.rs:181-272): rest and
    current volume of the active water samples (mass > 0.1 m_nom) and their J range."""
    nb, nw = sim.num_bed, sim.num_water
    w = sim.read_particles(nb, nw)
    finite = _finite(w[:, 0], w[:, 1], w[:, 2], w[:, 3], w[:, 7])
    m_nom = nominal_mass(settings)
    dx = dx_of(settings)
    pvol = float(dx * dx * dx * F(0.25))
    act = w[:, 7] > m_nom * F(0.1)
    j = w[act, 3].astype(np.float64)
    scale = w[act, 7].astype(np.float64) / float(m_nom)
    n = int(act.sum())
    return WaterVolume(finite, n, float(w[act, 7].astype(np.float64).sum()), float((scale * pvol).sum()),
                       float((scale * pvol * j).sum()), float(j.sum() / max(n, 1)),
                       float(j.min()) if n else 0.0, float(j.max()) if n else 0.0)


@dataclass
class GridPacking:
    all_finite: bool
    active_count: int
    deposited_rest_volume: float
    deposited_current_volume: float
    max_rest_fraction: float
    max_current_fraction: float
    max_packed_fraction: float
    fractional_cell_count: int
    max_fractional_fraction: float
    overpacked_cell_count: int
    overpacked_volume_fraction: float


def grid_packing_snapshot(sim, settings):
    """readback_water_grid_packing_snapshot (physics_tests.rs:274-442): water rest and
    current volume splatted to the grid with the quadratic B-spline, as fractions of the
    cell volume; counts of fractional (0 < f < 1) and overpacked (f > 1.2) cells."""
    nb, nw = sim.num_bed, sim.num_water
    w = sim.read_particles(nb, nw)
    finite = _finite(w[:, 0], w[:, 1], w[:, 2], w[:, 3], w[:, 7])
    gx, gy, gz = (int(v) for v in settings.raw.grid_dims)
    bounds = np.array(settings.raw.bounds_size[:], dtype=F)
    dx = dx_of(settings)
    cell_vol = dx * dx * dx
    pvol = cell_vol * F(0.25)
    m_nom = nominal_mass(settings)
    act = w[:, 7] > m_nom * F(0.1)
    a = w[act]
    origin = -bounds * F(0.5)
    gp = (a[:, 0:3] - origin) / dx
    base = np.floor(gp - F(0.5))
    fx = gp - base
    wts = np.stack([F(0.5) * (F(1.5) - fx) ** 2, F(0.75) - (fx - F(1.0)) ** 2, F(0.5) * (fx - F(0.5)) ** 2])
    rest_p = pvol * a[:, 7] / max(m_nom, F(1e-6))
    cur_p = rest_p * np.clip(a[:, 3], F(0.40), F(2.00))
    ib = base.astype(np.int64)
    ncell = gx * gy * gz
    rest = np.zeros(ncell)
    cur = np.zeros(ncell)
    for i in range(3):
        for j in range(3):
            for k in range(3):
                cx, cy, cz = ib[:, 0] + i, ib[:, 1] + j, ib[:, 2] + k
                ok = (cx >= 0) & (cy >= 0) & (cz >= 0) & (cx < gx) & (cy < gy) & (cz < gz)
                wt = (wts[i, :, 0] * wts[j, :, 1] * wts[k, :, 2])[ok].astype(np.float64)
                cell = (cz[ok] * gx * gy + cy[ok] * gx + cx[ok])
                rest += np.bincount(cell, weights=wt * rest_p[ok], minlength=ncell)
                cur += np.bincount(cell, weights=wt * cur_p[ok], minlength=ncell)
    cv = max(float(cell_vol), 1e-8)
    rf, cf = rest / cv, cur / cv
    packed = np.maximum(rf, cf)
    frac = (packed > 0) & (packed < 1)
    over = packed > 1.20
    return GridPacking(finite, int(act.sum()), float(rest.sum()), float(cur.sum()), float(rf.max(initial=0.0)),
                       float(cf.max(initial=0.0)), float(packed.max(initial=0.0)), int(frac.sum()),
                       float(packed[frac].max(initial=0.0)), int(over.sum()), float((packed[over] - 1.20).sum()))


@dataclass
class WaterVelocity:
    all_finite: bool
    active_count: int
    active_mass: float
    kinetic_energy: float
    rms_speed: float
    mean_speed: float
    lateral_rms_speed: float
    max_speed: float
    momentum: tuple


def water_velocity_snapshot(sim, settings, y_min=-np.inf, y_max=np.inf):
    """readback_water_velocity_snapshot_in_y_range (physics_tests.rs:458-550): kinetic
    energy, mass-weighted RMS speed (total and lateral), mean and max speed and momentum
    of the active water samples with y in [y_min, y_max]."""
    nb, nw = sim.num_bed, sim.num_water
    w = sim.read_particles(nb, nw)
    finite = _finite(w[:, 1], w[:, 4], w[:, 5], w[:, 6], w[:, 7])
    m_nom = nominal_mass(settings)
    sel = (w[:, 7] > m_nom * F(0.1)) & (w[:, 1] >= y_min) & (w[:, 1] <= y_max)
    a = w[sel].astype(np.float64)
    m = a[:, 7]
    v = a[:, 4:7]
    s2 = (v * v).sum(axis=1)
    lat = v[:, 0] ** 2 + v[:, 2] ** 2
    mass = float(m.sum())
    n = int(sel.sum())
    return WaterVelocity(finite, n, mass, float((0.5 * m * s2).sum()),
                         float(np.sqrt((m * s2).sum() / max(mass, 1e-6))), float(np.sqrt(s2).sum() / max(n, 1)),
                         float(np.sqrt((m * lat).sum() / max(mass, 1e-6))), float(np.sqrt(s2).max(initial=0.0)),
                         tuple(float(x) for x in (m[:, None] * v).sum(axis=0)))


@dataclass
class Diag:
    all_finite: bool
    total_mass: float
    active_count: int
    min_mass: float
    max_mass: float
    x_min: float
    x_max: float
    x_extent: float
    y_min: float
    y_max: float
    y_mean: float
    y_extent: float
    z_min: float
    z_max: float
    z_extent: float
    mean_j: float
    min_j: float
    max_j: float


def diag_snapshot(sim, settings, start=0, count=None):
    """readback_diag_snapshot_range (physics_tests.rs:937-1061): mass, bounding box, mean
    height and J range of the active samples in [start, start + count)."""
    total = sim.num_bed + sim.num_water
    if count is None:
        count = total - start
    end = min(start + count, total)
    p = sim.read_particles(start, max(end - start, 0))
    finite = _finite(p[:, 0], p[:, 1], p[:, 2], p[:, 3], p[:, 7])
    act = p[:, 7] > nominal_mass(settings) * F(0.1)
    a = p[act].astype(np.float64)
    n = int(act.sum())
    if n == 0:
        return Diag(finite, 0.0, 0, *([0.0] * 15))
    lo, hi = a[:, 0:3].min(axis=0), a[:, 0:3].max(axis=0)
    return Diag(finite, float(a[:, 7].sum()), n, float(a[:, 7].min()), float(a[:, 7].max()),
                float(lo[0]), float(hi[0]), float(hi[0] - lo[0]), float(lo[1]), float(hi[1]), float(a[:, 1].mean()),
                float(hi[1] - lo[1]), float(lo[2]), float(hi[2]), float(hi[2] - lo[2]), float(a[:, 3].mean()),
                float(a[:, 3].min()), float(a[:, 3].max()))


def bed_diag_snapshot(sim, settings):
    """readback_bed_diag_snapshot (physics_tests.rs:1077-1083): the bed samples only."""
    return diag_snapshot(sim, settings, 0, sim.num_bed)


def bed_bounds_y(settings):
    """benchmark_bed_bounds_y (physics_tests.rs:1085-1091): bed bottom and top heights."""
    b = settings.raw.bed
    return float(F(b.center[1]) + F(b.bot_y)), float(F(b.center[1]) + F(b.top_y))


@dataclass
class BedContainment:
    all_finite: bool
    active_count: int
    max_radial_excess: float
    min_floor_clearance: float


def bed_filter_containment_snapshot(sim, settings):
    """readback_bed_filter_containment_snapshot (physics_tests.rs:608-693): how far the
    active bed samples (radius 0.62 dx) reach past the paper filter's inner cone
    (FilterConfig::inner_radius_at_y, filter.rs:29-37) and below its apex."""
    nb = sim.num_bed
    p = sim.read_particles(0, nb)
    finite = _finite(p[:, 0], p[:, 1], p[:, 2], p[:, 7])
    f = settings.raw.filter
    cy, top, bot = F(f.center[1]), F(f.top_y), F(f.bot_y)
    bed_r = dx_of(settings) * F(0.62)
    act = p[:, 7] > nominal_mass(settings) * F(0.1)
    a = p[act]
    n = int(act.sum())
    if n == 0:
        return BedContainment(finite, 0, 0.0, 0.0)
    local_y = np.clip(a[:, 1] - cy, bot, top)
    t = np.clip((local_y - bot) / max(top - bot, F(1e-6)), F(0), F(1))
    radius = F(f.bot_radius) + (F(f.top_radius) - F(f.bot_radius)) * t
    inner = np.maximum(radius - F(f.thickness), F(f.hole_radius))
    radial = np.sqrt(a[:, 0] * a[:, 0] + a[:, 2] * a[:, 2])
    excess = radial + bed_r - inner
    clearance = a[:, 1] - (cy + bot + bed_r)
    return BedContainment(finite, n, float(excess.max()), float(clearance.min()))


def bed_states(sim):
    """readback_bed_particle_states (physics_tests.rs:695-775): position, mass and
    saturation (bed_extract lane 7) of every bed sample, as (n, 5) float32."""
    nb = sim.num_bed
    p = sim.read_particles(0, nb)
    e = sim.read_bed_extract(0, nb)
    return np.column_stack([p[:, 0:3], p[:, 7], e[:, 7]])


@dataclass
class BedMotion:
    all_finite: bool
    active_count: int
    saturated_count: int
    tracked_count: int
    mean_displacement: float
    max_displacement: float
    mean_downward_displacement: float


def bed_motion_delta(before, after, active_mass, saturated, center_radius):
    """bed_particle_motion_delta_snapshot (physics_tests.rs:777-836): displacement of the
    saturated bed samples within center_radius of the axis between two readbacks."""
    n = min(len(before), len(after))
    b, a = before[:n].astype(np.float64), after[:n].astype(np.float64)
    finite = _finite(b[:, 0:4], a[:, 0:5])
    act = a[:, 3] > active_mass
    sat = act & (a[:, 4] >= saturated)
    tracked = sat & (np.hypot(a[:, 0], a[:, 2]) <= center_radius)
    d = a[tracked, 0:3] - b[tracked, 0:3]
    disp = np.sqrt((d * d).sum(axis=1))
    down = np.maximum(b[tracked, 1] - a[tracked, 1], 0.0)
    k = int(tracked.sum())
    return BedMotion(finite, int(act.sum()), int(sat.sum()), k, float(disp.sum() / max(k, 1)),
                     float(disp.max(initial=0.0)), float(down.sum() / max(k, 1)))


@dataclass
class SaturatedBed:
    all_finite: bool
    active_count: int
    saturated_count: int
    mean_compression: float
    saturated_mean_compression: float


def saturated_bed_motion_snapshot(sim, settings):
    """readback_saturated_bed_motion_snapshot (physics_tests.rs:838-935): mean
    compression (bed_extract lane 3) of the active bed samples and of the saturated
    ones (saturation >= 0.65)."""
    nb = sim.num_bed
    p = sim.read_particles(0, nb)
    e = sim.read_bed_extract(0, nb)
    finite = _finite(p[:, 7], e[:, 3], e[:, 7])
    act = p[:, 7] > nominal_mass(settings) * F(0.1)
    sat = act & (e[:, 7] >= 0.65)
    comp = e[:, 3].astype(np.float64)
    na, ns = int(act.sum()), int(sat.sum())
    return SaturatedBed(finite, na, ns, float(comp[act].sum() / max(na, 1)), float(comp[sat].sum() / max(ns, 1)))
