"""A second, independent restatement of the reference's WGSL step, in vectorised numpy
float32 — test infrastructure only.

The C++ oracle (`oracle/oracle.cpp`) and the CUDA engine were written from the same
reading of `crates/sim-wasm/src/mpm_3d/shader.rs`, so their bit-exact agreement cannot
expose a misreading they share.  This module is a separate reading of the same WGSL,
written directly from the shader text in a different form (whole-grid and whole-sample
array expressions with masks instead of per-cell loops), and the tests compare it with
the oracle dispatch by dispatch and over whole substeps.  It covers every dispatch of
the step, the uniforms (mod.rs:569-660), the SDF texture and solid class (state.rs),
jet emission (inflow.rs), and three engine extensions: the int64 P2G lanes, the sample
reorder and the residual-mode pressure solve.  Every function cites what it restates.

Floating point: every value is an IEEE float32 array and every WGSL expression is
evaluated in its written, left-to-right order (numpy >= 2 keeps Python scalars weak,
so `f32_array * 0.5` stays float32).  WGSL conversions are restated explicitly:
`i32(f)` truncates toward zero and saturates, `f32(i)` rounds to nearest, `mix(a, b, t)`
is `a * (1 - t) + b * t`, `clamp(x, lo, hi)` is `min(max(x, lo), hi)`, `fract(x)` is
`x - floor(x)`, `length(v)` is `sqrt(x*x + y*y + z*z)`.  Integer atomics are
order-independent sums that wrap at 32 bits.
"""
import numpy as np

F32 = np.float32

# shader.rs:172-177 cell kinds
CELL_AIR, CELL_SURFACE_FLUID, CELL_INTERIOR_FLUID, CELL_BED_COUPLED, CELL_SOLID = 0, 1, 2, 3, 4
# state.rs:13-28
FP_SCALE = F32(262144.0)
FP_VALUE_LIMIT = F32(8192.0)
SDF_RES = 128
METRICS_DIV_FP_SCALE = F32(1024.0)
# shader.rs:75-76
BED_REACTION_ALPHA = F32(0.04)
BED_REACTION_IMPULSE_CAP = F32(0.012)
# neighbour order of every six-face loop in the shader (shader.rs:1114-1121, 1388-1395)
FACES = ((-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1))


def f32(x):
    return np.asarray(x, dtype=np.float32)


def to_i32(x):
    """WGSL `i32(f32)`: truncate toward zero, saturate at the i32 range."""
    t = np.trunc(np.asarray(x, dtype=np.float64))
    t = np.where(np.isnan(t), 0.0, t)
    return np.clip(t, -2147483648.0, 2147483647.0).astype(np.int32)


def wrap_i32(x):
    """Two's-complement wrap of an int64 sum to i32 (WGSL atomicAdd on i32)."""
    return (np.asarray(x, dtype=np.int64) & 0xFFFFFFFF).astype(np.uint32).view(np.int32)


def mix(a, b, t):
    return a * (1 - t) + b * t


def clamp(x, lo, hi):
    return np.minimum(np.maximum(x, lo), hi)


def length3(x, y, z):
    return np.sqrt(x * x + y * y + z * z)


def smoothstep(e0, e1, x):
    t = clamp((x - e0) / (e1 - e0), F32(0.0), F32(1.0))
    return t * t * (3 - 2 * t)


class Uniforms:
    """`MpmUniforms` as `MpmSim3D::write_uniforms` fills it (mod.rs:569-660), from the
    settings the simulation was created with and the counts of the substep."""

    def __init__(self, raw, num_water, num_bed, dt):
        gx, gy, gz = (int(v) for v in raw.grid_dims)
        self.gx, self.gy, self.gz = gx, gy, gz
        self.cells = gx * gy * gz
        self.num_water, self.num_bed = int(num_water), int(num_bed)
        self.max_particles = int(raw.max_particles)
        bs = [F32(v) for v in raw.bounds_size]
        self.dx = bs[0] / F32(gx)                                   # mod.rs:573
        self.inv_dx = F32(1.0) / self.dx                            # mod.rs:574
        brew = raw.brew
        self.nominal_mass = F32(brew.water_mass_units_per_ml) / F32(brew.water_particles_per_ml)  # mod.rs:575
        self.p_vol = self.dx * self.dx * self.dx * F32(raw.particle_volume_cells)                # mod.rs:576
        self.dt = F32(dt)
        self.gravity = F32(raw.gravity)
        self.origin = np.array([-b * F32(0.5) for b in bs], dtype=np.float32)
        self.bounds_max = np.array([b * F32(0.5) for b in bs], dtype=np.float32)
        self.bulk_K = F32(raw.bulk_modulus)
        self.viscosity = F32(raw.viscosity)
        self.fp = FP_SCALE
        self.inv_fp = F32(1.0) / FP_SCALE
        self.vel_cap = F32(raw.max_velocity)
        g = raw.geom
        self.friction = F32(g.sdf_friction)
        self.restitution = F32(g.sdf_restitution)
        self.contact_offset = F32(g.contact_offset)
        self.nu_m2s = F32(brew.water_kinematic_viscosity_m2_s)
        self.min_perm = F32(brew.min_bed_permeability_m2)
        self.div_clamp = np.minimum(F32(4.0) * self.vel_cap * self.inv_dx, FP_VALUE_LIMIT - F32(1.0))  # mod.rs:589-590
        self.p_clamp = FP_VALUE_LIMIT - F32(1.0)                    # mod.rs:593
        self.j_alpha, self.j_expand_alpha, self.max_rest_frac = F32(32.0), F32(2.0), F32(1.20)  # mod.rs:656
        self.surface_void_scale = F32(brew.bed_surface_void_scale)
        self.pore_capacity_scale = F32(brew.bed_pore_capacity_scale)
        self.pore_overfill_alpha = F32(brew.bed_pore_overfill_alpha)
        self.absorption_rate = F32(brew.bed_absorption_rate)
        self.filter_absorption = F32(brew.filter_absorption_rate_s)
        self.water_r_dx, self.bed_r_dx = F32(brew.water_sample_radius_dx), F32(brew.bed_sample_radius_dx)
        self.extraction_rate = F32(0.01)                            # mod.rs:643
        self.compaction_rate = F32(brew.bed_compaction_rate)
        self.bed_impact = F32(brew.bed_impact_rate)
        # bed_capacity_per_particle (mod.rs:578-582)
        self.max_saturation = (F32(brew.target_bed_retention_ml) * F32(brew.water_mass_units_per_ml) / F32(num_bed)
                               if num_bed > 0 else F32(0.7))

    # shader.rs:116, 171-172
    @property
    def occupancy(self):
        return self.nominal_mass * F32(0.1)

    @property
    def inactive(self):
        return self.nominal_mass * F32(0.10)

    def grid_shape(self):
        return (self.gz, self.gy, self.gx)


# ---------------------------------------------------------------- neighbour access

def shifted(a, d, fill):
    """b[z, y, x] = a[z + dz, y + dy, x + dx] (last three axes), `fill` off the grid."""
    dxo, dyo, dzo = d
    out = np.empty_like(a)
    out[...] = fill
    nz, ny, nx = a.shape[:3]

    def rng(o, n):
        return (slice(max(0, -o), n - max(0, o)), slice(max(0, o), n - max(0, -o)))

    (zd, zs), (yd, ys), (xd, xs) = rng(dzo, nz), rng(dyo, ny), rng(dxo, nx)
    out[zd, yd, xd] = a[zs, ys, xs]
    return out


def in_grid(u, d):
    """True where the neighbour at offset d lies on the grid."""
    return shifted(np.ones(u.grid_shape(), dtype=bool), d, False)


def cell_centres(u):
    """origin + (vec3(f32(i)) + 0.5) * dx for every cell (shader.rs:1645-1646)."""
    iz, iy, ix = np.meshgrid(np.arange(u.gz, dtype=np.float32), np.arange(u.gy, dtype=np.float32),
                             np.arange(u.gx, dtype=np.float32), indexing="ij")
    return [u.origin[a] + (c + F32(0.5)) * u.dx for a, c in enumerate((ix, iy, iz))]


# ---------------------------------------------------------------- p2g  (shader.rs:955-1052)

def to_i64(x):
    """Truncate toward zero and saturate at the i64 range (NaN to 0)."""
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros(x.shape, np.int64)
    ok = ~np.isnan(x)
    big, small = x >= 9223372036854775807.0, x <= -9223372036854775808.0
    mid = ok & ~big & ~small
    out[mid] = np.trunc(x[mid]).astype(np.int64)
    out[big] = np.iinfo(np.int64).max
    out[small] = np.iinfo(np.int64).min
    return out


INT64_SCALE = F32(4294967296.0)


def p2g(u, particles, affine, int64=False):
    """Six i32 lanes after P2G into a cleared grid: (6, cells) int32.  With `int64`, the
    engine's 64-bit mode (no reference counterpart): every contribution scaled by 2^32
    instead of 2^18, truncated to i64 and summed with 64-bit wrap; (6, cells) int64."""
    n = u.num_water + u.num_bed
    p = np.asarray(particles, np.float32).reshape(-1, 8)[:n]
    a = np.asarray(affine, np.float32).reshape(-1, 12)[:n]
    xp, J, vp, mass = p[:, 0:3], p[:, 3], p[:, 4:7], p[:, 7]
    phase = a[:, 3]
    live = (phase < F32(0.5)) & ~(mass <= u.inactive)               # shader.rs:966-968
    xp, J, vp, mass, a = xp[live], J[live], vp[live], mass[live], a[live]
    grid_pos = (xp - u.origin) * u.inv_dx                           # shader.rs:971
    base_f = np.floor(grid_pos - F32(0.5))
    base = to_i32(base_f)
    fx = grid_pos - base.astype(np.float32)
    w = [[F32(0.5) * (F32(1.5) - fx[:, c]) * (F32(1.5) - fx[:, c]),  # shader.rs:979-987
          F32(0.75) - (fx[:, c] - F32(1.0)) * (fx[:, c] - F32(1.0)),
          F32(0.5) * (fx[:, c] - F32(0.5)) * (fx[:, c] - F32(0.5))] for c in range(3)]
    cols = [a[:, 0:3], a[:, 4:7], a[:, 8:11]]
    aff = [np.stack([mass * C[:, 0], mass * C[:, 1], mass * C[:, 2]], axis=1) for C in cols]  # shader.rs:993-995
    rest_vol = u.p_vol * mass / np.maximum(u.nominal_mass, F32(1e-6))           # shader.rs:999
    cur_vol = rest_vol * clamp(J, F32(0.40), F32(2.00))                          # shader.rs:1000
    mvp = mass[:, None] * vp
    acc = np.zeros((6, u.cells), dtype=np.int64)
    for i in range(3):
        for j in range(3):
            for k in range(3):
                off = np.array([i, j, k], dtype=np.int32)
                cell = base + off
                ok = ((cell >= 0).all(axis=1) & (cell[:, 0] < u.gx) & (cell[:, 1] < u.gy) & (cell[:, 2] < u.gz))
                wt = w[0][i] * w[1][j] * w[2][k]                                   # shader.rs:1010
                dpos = (off.astype(np.float32) - fx) * u.dx                        # shader.rs:1011
                dots = [c[:, 0] * dpos[:, 0] + c[:, 1] * dpos[:, 1] + c[:, 2] * dpos[:, 2] for c in aff]
                mom = [wt * (mvp[:, q] + dots[q]) for q in range(3)]               # shader.rs:1016-1020
                fp = INT64_SCALE if int64 else u.fp
                vals = [wt * mass * fp, mom[0] * fp, mom[1] * fp, mom[2] * fp,
                        wt * rest_vol * fp, wt * cur_vol * fp]                     # shader.rs:1032-1037
                ci = (cell[:, 2].astype(np.int64) * u.gy + cell[:, 1]) * u.gx + cell[:, 0]
                for lane in range(6):
                    q = to_i64(vals[lane][ok]) if int64 else to_i32(vals[lane][ok]).astype(np.int64)
                    np.add.at(acc[lane], ci[ok], q)
    return acc if int64 else wrap_i32(acc)


# ---------------------------------------------------------------- grid_update  (shader.rs:1056-1082)

def grid_update(u, lanes):
    """`grid_vel` after grid_update on a cleared `grid_vel`: (cells, 4) float32.  Int64
    lanes (the 64-bit mode) are read as f32(lane) * 2^-32."""
    L = np.asarray(lanes).reshape(6, -1)
    inv = F32(1.0) / INT64_SCALE if L.dtype == np.int64 else u.inv_fp
    mass = L[0].astype(np.float32) * inv
    live = ~(mass < F32(1e-6))
    m = np.where(live, mass, F32(1.0))
    v = [L[q].astype(np.float32) * inv / m for q in (1, 2, 3)]
    v[1] = v[1] + u.gravity * u.dt
    speed = length3(*v)
    over = speed > u.vel_cap
    s = np.where(over, u.vel_cap / np.where(over, speed, F32(1.0)), F32(1.0))
    v = [np.where(over, c * s, c) for c in v]
    out = np.zeros((u.cells, 4), dtype=np.float32)
    for q in range(3):
        out[:, q] = np.where(live, v[q], F32(0.0))
    out[:, 3] = np.where(live, mass, F32(0.0))
    return out


# ---------------------------------------------------------------- SDF  (shader.rs:668-715)

class Sdf:
    """The 128^3 SDF texture read with `textureLoad` (R32F texels, x fastest)."""

    def __init__(self, u, texels):
        self.u = u
        self.t = np.asarray(texels, np.float32).reshape(SDF_RES, SDF_RES, SDF_RES)

    def load(self, cx, cy, cz):
        m = SDF_RES - 1
        return self.t[np.clip(cz, 0, m), np.clip(cy, 0, m), np.clip(cx, 0, m)]

    def sample(self, px, py, pz):
        """shader.rs:678-699, trilinear by `mix` in x, then y, then z."""
        u = self.u
        bsz = u.bounds_max * F32(2.0)
        res = F32(SDF_RES)
        uv = [(p + u.bounds_max[a]) / bsz[a] * res - F32(0.5) for a, p in enumerate((px, py, pz))]
        fl = [np.floor(c) for c in uv]
        b = [to_i32(c) for c in fl]
        f = [c - d for c, d in zip(uv, fl)]
        c = {}
        for dz in (0, 1):
            for dy in (0, 1):
                for dx_ in (0, 1):
                    c[(dx_, dy, dz)] = self.load(b[0] + dx_, b[1] + dy, b[2] + dz)
        c00 = mix(c[(0, 0, 0)], c[(1, 0, 0)], f[0])
        c10 = mix(c[(0, 1, 0)], c[(1, 1, 0)], f[0])
        c01 = mix(c[(0, 0, 1)], c[(1, 0, 1)], f[0])
        c11 = mix(c[(0, 1, 1)], c[(1, 1, 1)], f[0])
        c0 = mix(c00, c10, f[1])
        c1 = mix(c01, c11, f[1])
        return mix(c0, c1, f[2])

    def gradient(self, px, py, pz):
        """shader.rs:701-715: central differences at +-dx, normalised."""
        e = self.u.dx
        g = [self.sample(px + e, py, pz) - self.sample(px - e, py, pz),
             self.sample(px, py + e, pz) - self.sample(px, py - e, pz),
             self.sample(px, py, pz + e) - self.sample(px, py, pz - e)]
        ln = length3(*g)
        small = ln < F32(1e-8)
        d = np.where(small, F32(1.0), ln)
        return [np.where(small, F32(0.0), c / d) for c in g]


# ---------------------------------------------------------------- boundary_project  (shader.rs:1630-1679)

def boundary_project(u, sdf, grid_vel):
    """`grid_vel` after one boundary_project pass: (cells, 4) float32.  Cells below the
    mass threshold return at once (shader.rs:1636), so only the others are evaluated."""
    gv = np.array(grid_vel, np.float32).reshape(-1, 4)
    live = np.flatnonzero(~(gv[:, 3] < F32(1e-6)))
    v = [gv[live, q] for q in range(3)]
    px, py, pz = (c.reshape(-1)[live] for c in cell_centres(u))
    sd = sdf.sample(px, py, pz)
    near = sd < u.contact_offset
    n = sdf.gradient(px, py, pz)
    vn = v[0] * n[0] + v[1] * n[1] + v[2] * n[2]
    hit = near & (vn < F32(0.0))
    k = F32(1.0) + u.restitution
    v2 = [v[q] - n[q] * vn * k for q in range(3)]                          # shader.rs:1653
    d2 = v2[0] * n[0] + v2[1] * n[1] + v2[2] * n[2]
    vt = [v2[q] - n[q] * d2 for q in range(3)]                             # shader.rs:1655
    vtl = length3(*vt)
    fr = hit & (vtl > F32(1e-6))
    safe = np.where(fr, vtl, F32(1.0))
    imp = np.minimum(u.friction * np.abs(vn), vtl)
    v3 = [np.where(fr, v2[q] - vt[q] * (imp / safe), v2[q]) for q in range(3)]
    v = [np.where(hit, v3[q], v[q]) for q in range(3)]
    margin = F32(2.0) * u.dx                                               # shader.rs:1665-1667
    for q, p in enumerate((px, py, pz)):
        lo = u.origin[q] + margin
        hi = u.bounds_max[q] - margin
        v[q] = np.where((p < lo) & (v[q] < F32(0.0)), F32(0.0), v[q])
        v[q] = np.where((p > hi) & (v[q] > F32(0.0)), F32(0.0), v[q])
    out = gv.copy()
    for q in range(3):
        out[live, q] = v[q]
    return out


# ---------------------------------------------------------------- shared helpers of the pressure passes

def is_fluid(kind):
    """shader.rs:582-591"""
    return (kind == CELL_INTERIOR_FLUID) | (kind == CELL_SURFACE_FLUID) | (kind == CELL_BED_COUPLED)


def lane_f32(u, lane):
    """`f32(atomicLoad(&grid[...])) * inv_fp_scale()` (shader.rs:198-200, 262-264, 285-291)."""
    return lane.astype(np.float32) * u.inv_fp


def fill_fraction(u, kind, rest, cur):
    """liquid_fill_fraction (shader.rs:293-304)."""
    cell_volume = np.maximum(u.dx * u.dx * u.dx, F32(1e-8))
    dep = clamp(np.maximum(rest, cur) / cell_volume, F32(0.0), F32(1.0))
    out = np.where(kind == CELL_SURFACE_FLUID, dep, F32(0.0))
    return np.where((kind == CELL_INTERIOR_FLUID) | (kind == CELL_BED_COUPLED), F32(1.0), out).astype(np.float32)


def face_weight(self_kind, self_fill, nb_kind, nb_fill):
    """pressure_face_weight (shader.rs:306-323); nb_fill = liquid_fill_fraction(neighbour)."""
    w = np.minimum(self_fill, nb_fill)
    w = np.where(~is_fluid(nb_kind), self_fill, w)
    w = np.where((self_kind == CELL_BED_COUPLED) | (nb_kind == CELL_BED_COUPLED), F32(1.0), w)
    return np.where(nb_kind == CELL_SOLID, F32(0.0), w).astype(np.float32)


def store_clamped(u, value, lo, hi):
    """pressure_store / divergence_store / packing_pressure_store: clamp, then
    `i32(clamped * fp_scale())` (shader.rs:202-221, 352-359)."""
    return to_i32(clamp(value, lo, hi) * u.fp)


class Bed:
    """Bed-sample views the grid passes read: lookup per cell, the sample rows."""

    def __init__(self, u, lookup, particles, affine, bed_extract):
        self.u = u
        self.lookup = np.asarray(lookup, np.int32).reshape(u.grid_shape())
        nb = u.num_bed
        self.vel = np.asarray(particles, np.float32).reshape(-1, 8)[:nb, 4:7]
        self.pos_y = np.asarray(particles, np.float32).reshape(-1, 8)[:nb, 1]
        self.phase = np.asarray(affine, np.float32).reshape(-1, 12)[:nb, 3]
        self.bx = np.asarray(bed_extract, np.float32).reshape(-1, 8)[:nb] if nb else np.zeros((0, 8), np.float32)

    def valid_solid(self, idx):
        """is_valid_bed_solid_idx (shader.rs:365-370)."""
        ok = (idx >= 0) & (idx < self.u.num_bed)
        safe = np.where(ok, idx, 0)
        ph = self.phase[safe] if self.u.num_bed else np.zeros(idx.shape, np.float32)
        return ok & ~(ph < F32(0.5))

    def matrix_velocity(self):
        """bed_matrix_velocity_cell (shader.rs:380-407) of every cell: the mean velocity of
        the valid bed samples looked up in the 3x3x3 block, summed x-offset outermost."""
        u = self.u
        sums = [np.zeros(u.grid_shape(), np.float32) for _ in range(3)]
        wsum = np.zeros(u.grid_shape(), np.float32)
        for di in (-1, 0, 1):
            for dj in (-1, 0, 1):
                for dk in (-1, 0, 1):
                    li = shifted(self.lookup, (di, dj, dk), -1)
                    ok = self.valid_solid(li)
                    safe = np.where(ok, li, 0)
                    for q in range(3):
                        vq = self.vel[safe, q] if u.num_bed else np.zeros(li.shape, np.float32)
                        sums[q] = np.where(ok, sums[q] + vq, sums[q])
                    wsum = np.where(ok, wsum + F32(1.0), wsum)
        has = ~(wsum <= F32(0.0))
        d = np.where(has, wsum, F32(1.0))
        return [np.where(has, s / d, F32(0.0)).astype(np.float32) for s in sums]

    def compacted_porosity(self, b):
        """bed_compacted_porosity (shader.rs:435-440)."""
        be = self.bx[b]
        base = clamp(be[:, 1], F32(0.18), F32(0.70))
        comp = clamp(be[:, 3], F32(0.0), F32(2.25))
        return clamp(base - comp * F32(0.12), F32(0.16), base)

    def compacted_permeability(self, b):
        """bed_compacted_permeability (shader.rs:442-449) with kozeny_porosity_factor
        (shader.rs:429-433)."""
        def kozeny(phi_in):
            phi = clamp(phi_in, F32(0.08), F32(0.82))
            solid = np.maximum(F32(1.0) - phi, F32(1e-4))
            return (phi * phi * phi) / (solid * solid)
        be = self.bx[b]
        base = clamp(be[:, 1], F32(0.18), F32(0.70))
        ratio = kozeny(self.compacted_porosity(b)) / np.maximum(kozeny(base), F32(1e-8))
        return np.maximum(be[:, 2] * ratio, self.u.min_perm)


def solid_at(u, sdf, solid_class, use_cache, d):
    """Whether the neighbour at offset d is solid as classify_cells tests it
    (shader.rs:1279-1326): the class texture when the SDF cache is on, else the SDF at the
    neighbour's centre (cell centre + offset * dx) below zero."""
    if use_cache:
        return shifted(solid_class, d, False)
    px, py, pz = cell_centres(u)
    e = u.dx
    q = [px, py, pz]
    for a in range(3):
        if d[a] > 0:
            q[a] = q[a] + e
        elif d[a] < 0:
            q[a] = q[a] + (-e)
    return ~(sdf.sample(*q) >= F32(0.0))


# ---------------------------------------------------------------- classify_cells  (shader.rs:1181-1367)

def volume_target(u, rest, cur):
    """volume_projection_target_divergence (shader.rs:597-619)."""
    cell_volume = u.dx * u.dx * u.dx
    eps = np.maximum(cell_volume * F32(1e-5), u.p_vol * F32(1e-3))
    small = rest <= eps
    j = cur / np.where(small, F32(1.0), rest)
    ce = clamp(F32(1.0) - j, F32(0.0), F32(0.75))
    ee = clamp(j - F32(1.0), F32(0.0), F32(0.75))
    t = ce * u.j_alpha - ee * u.j_expand_alpha
    packed = np.maximum(rest, cur) / np.maximum(cell_volume, F32(1e-8))
    over = np.maximum(packed - u.max_rest_frac, F32(0.0))
    t = np.maximum(t, over * u.j_alpha)
    return np.where(small, F32(0.0), t).astype(np.float32)


def bed_pore_target(u, bed, b, centre_y, rest, cur):
    """bed_pore_projection_target_divergence (shader.rs:621-666) for bed samples b."""
    t = volume_target(u, rest, cur)
    cell_volume = u.dx * u.dx * u.dx
    be = bed.bx[b]
    base = bed.compacted_porosity(b)
    sat = clamp(be[:, 7], F32(0.0), F32(1.0))
    comp = clamp(be[:, 3], F32(0.0), F32(2.25))
    surface_t = smoothstep(F32(-0.25), F32(0.75), (centre_y - bed.pos_y[b]) * u.inv_dx)
    open_pore = clamp((F32(1.0) - F32(0.65) * sat) * (F32(1.0) - F32(0.12) * comp), F32(0.20), F32(1.0))
    opening = surface_t * clamp(u.surface_void_scale, F32(0.0), F32(1.0)) * open_pore
    surface_por = np.minimum(base + F32(0.35), F32(0.82))
    eff = mix(base, surface_por, opening)
    occ = mix(F32(1.0), F32(0.35), opening)
    sat_cap = mix(F32(1.0), F32(0.32), sat)
    comp_cap = mix(F32(1.0), F32(0.58), clamp(comp / F32(1.5), F32(0.0), F32(1.0)))
    cap = eff * cell_volume * np.maximum(u.pore_capacity_scale, F32(0.0)) * sat_cap * comp_cap
    overfill = np.maximum(cur - cap, F32(0.0)) / np.maximum(cell_volume, F32(1e-8))
    resp = u.pore_overfill_alpha * occ * mix(F32(1.0), F32(1.45), sat)
    return np.maximum(t, overfill * resp)


def classify(u, lanes, grid_vel, bed, sdf, solid_class, use_cache):
    """Lanes after classify_cells: pressure (lane 0) zeroed, kind (lane 3) and the
    divergence minus its target (lane 1) written for every cell; (6, cells) int32."""
    L = np.array(lanes, np.int32).reshape(6, *u.grid_shape())
    gv = np.asarray(grid_vel, np.float32).reshape(*u.grid_shape(), 4)
    mass = gv[..., 3]
    px, py, pz = cell_centres(u)
    self_solid = solid_class if use_cache else (sdf.sample(px, py, pz) < F32(0.0))
    occ = u.occupancy
    air = mass <= occ
    air_nb = np.zeros(u.grid_shape(), bool)
    for d in FACES:
        air_nb |= ~in_grid(u, d) | (shifted(mass, d, F32(0.0)) <= occ)
    kind = np.where(air_nb, CELL_SURFACE_FLUID, CELL_INTERIOR_FLUID)
    kind = np.where(bed.lookup >= 0, CELL_BED_COUPLED, kind)
    kind = np.where(air, CELL_AIR, kind)
    kind = np.where(self_solid, CELL_SOLID, kind).astype(np.int32)
    # ghost-mirrored central differences (shader.rs:1270-1328)
    vel = [gv[..., q] for q in range(3)]
    faces = {}
    for a, d in enumerate(FACES):
        axis = a // 2
        open_ = in_grid(u, d) & ~solid_at(u, sdf, solid_class, use_cache, d)
        faces[a] = np.where(open_, shifted(vel[axis], d, F32(0.0)), -vel[axis])
    div = F32(0.5) * u.inv_dx * (((faces[1] - faces[0]) + (faces[3] - faces[2])) + (faces[5] - faces[4]))
    rest, cur = lane_f32(u, L[4]), lane_f32(u, L[5])
    target = volume_target(u, rest, cur)
    li = bed.lookup
    bedc = (kind == CELL_BED_COUPLED) & (li >= 0) & (li < u.num_bed)
    if bedc.any():
        sel = np.nonzero(bedc)
        b = li[sel]
        pore = bed_pore_target(u, bed, b, py[sel], rest[sel], cur[sel])
        porosity = clamp(bed.compacted_porosity(b), F32(0.08), F32(1.0))
        solid_fraction = F32(1.0) - porosity
        bmv = bed.matrix_velocity()
        nbv = {}
        for a, d in enumerate(FACES):
            nbv[a] = shifted(bmv[a // 2], d, F32(0.0))[sel]
        sdiv = F32(0.5) * u.inv_dx * (((nbv[1] - nbv[0]) + (nbv[3] - nbv[2])) + (nbv[5] - nbv[4]))
        target[sel] = (pore - solid_fraction * sdiv) / porosity
    fluid = is_fluid(kind)
    out = L.copy()
    out[0] = 0                                                          # pressure_store(idx, 0.0)
    out[3] = kind
    out[1] = np.where(fluid, store_clamped(u, div - target, -u.div_clamp, u.div_clamp), 0)
    return out.reshape(6, -1)


# ---------------------------------------------------------------- pressure_rbgs  (shader.rs:1371-1453)

def rbgs(u, lanes, pairs):
    """Lane 0 (pressure) after `pairs` red+black sweeps of pressure_update; (6, cells)."""
    L = np.array(lanes, np.int32).reshape(6, *u.grid_shape())
    kind = L[3]
    fill = fill_fraction(u, kind, lane_f32(u, L[4]), lane_f32(u, L[5]))
    div = lane_f32(u, L[1])
    iz, iy, ix = np.meshgrid(np.arange(u.gz), np.arange(u.gy), np.arange(u.gx), indexing="ij")
    parity = (ix + iy + iz) & 1
    fluid = is_fluid(kind)
    nbk = {d: shifted(kind, d, CELL_SOLID) for d in FACES}     # off-grid faces are skipped like solids
    nbf = {d: shifted(fill, d, F32(0.0)) for d in FACES}
    w = {d: face_weight(kind, fill, nbk[d], nbf[d]) for d in FACES}
    use = {d: in_grid(u, d) & (nbk[d] != CELL_SOLID) & ~(w[d] <= F32(0.0)) for d in FACES}
    rhs = div * fill / np.maximum(u.dt, F32(1e-6))
    dx2rhs = u.dx * u.dx * rhs
    p = L[0].copy()
    for _ in range(pairs):
        for colour in (0, 1):
            pf = lane_f32(u, p)
            cnt = np.zeros(u.grid_shape(), np.float32)
            psum = np.zeros(u.grid_shape(), np.float32)
            for d in FACES:
                cnt = np.where(use[d], cnt + w[d], cnt)
                term = w[d] * shifted(pf, d, F32(0.0))
                psum = np.where(use[d] & is_fluid(nbk[d]), psum + term, psum)
            none = cnt <= F32(0.0)
            pnew = (psum - dx2rhs) / np.where(none, F32(1.0), cnt)
            val = np.where(fluid & ~none, pnew, F32(0.0))
            stored = store_clamped(u, val, -u.p_clamp, u.p_clamp)
            p = np.where(parity == colour, stored, p)
    out = L.copy()
    out[0] = p
    return out.reshape(6, -1)


# ---------------------------------------------------------------- project_pressure  (shader.rs:1457-1543)

def project(u, lanes, grid_vel, bed):
    """`grid_vel` after project_pressure and the bed impulses it adds: ((cells, 4) float32,
    (3, num_bed) int64 sums of the impulse lanes)."""
    L = np.asarray(lanes, np.int32).reshape(6, *u.grid_shape())
    gv = np.array(grid_vel, np.float32).reshape(*u.grid_shape(), 4)
    kind = L[3]
    fill = fill_fraction(u, kind, lane_f32(u, L[4]), lane_f32(u, L[5]))
    p = lane_f32(u, L[0])
    act = ~(gv[..., 3] < F32(1e-6)) & is_fluid(kind)
    pn = {}
    for d in FACES:
        ok = in_grid(u, d)
        nk = shifted(kind, d, CELL_SOLID)
        mirror = ~ok | (nk == CELL_SOLID)
        nbp = np.where(is_fluid(nk), shifted(p, d, F32(0.0)), F32(0.0))
        wgt = face_weight(kind, fill, nk, shifted(fill, d, F32(0.0)))
        pn[d] = np.where(mirror, p, mix(p, nbp, wgt))                    # pressure_weighted_or_mirror
    h = F32(0.5) * u.inv_dx
    grad = [h * (pn[FACES[1]] - pn[FACES[0]]), h * (pn[FACES[3]] - pn[FACES[2]]), h * (pn[FACES[5]] - pn[FACES[4]])]
    v = [gv[..., q] - u.dt * grad[q] for q in range(3)]
    imp = np.zeros((3, max(u.num_bed, 1)), np.int64)
    li = bed.lookup
    darcy = act & (kind == CELL_BED_COUPLED) & (li >= 0) & (li < u.num_bed)
    if darcy.any():
        sel = np.nonzero(darcy)
        b = li[sel]
        perm = bed.compacted_permeability(b)
        rate = u.nu_m2s / perm
        damp = F32(1.0) / (F32(1.0) + np.maximum(rate * u.dt, F32(0.0)))
        bmv = bed.matrix_velocity()
        before = [v[q][sel] for q in range(3)]
        after = [bmv[q][sel] + (before[q] - bmv[q][sel]) * damp for q in range(3)]
        water_imp = [gv[..., 3][sel] * (after[q] - before[q]) for q in range(3)]
        share_in = [(-water_imp[q]) * BED_REACTION_ALPHA for q in range(3)]
        for q in range(3):
            v[q][sel] = after[q]
        # bed_impulse_delta_add_neighborhood (shader.rs:479-515)
        cz, cy, cx = (np.asarray(a) for a in sel)
        count = np.zeros(cz.shape, np.float32)
        nbr = []
        for di in (-1, 0, 1):
            for dj in (-1, 0, 1):
                for dk in (-1, 0, 1):
                    x, y, z = cx + di, cy + dj, cz + dk
                    on = (x >= 0) & (y >= 0) & (z >= 0) & (x < u.gx) & (y < u.gy) & (z < u.gz)
                    bi = np.where(on, li[np.clip(z, 0, u.gz - 1), np.clip(y, 0, u.gy - 1), np.clip(x, 0, u.gx - 1)], -1)
                    ok = bed.valid_solid(bi)
                    count = np.where(ok, count + F32(1.0), count)
                    nbr.append((bi, ok))
        has = ~(count <= F32(0.0))
        cnt = np.where(has, count, F32(1.0))
        share = [s / cnt for s in share_in]
        cap = u.nominal_mass * u.vel_cap * BED_REACTION_IMPULSE_CAP
        q_i = [to_i32(clamp(s, -cap, cap) * u.fp).astype(np.int64) for s in share]
        for bi, ok in nbr:
            m = ok & has
            for q in range(3):
                np.add.at(imp[q], bi[m], q_i[q][m])
    speed = length3(*v)
    over = speed > u.vel_cap
    sc = u.vel_cap / np.where(over, speed, F32(1.0))
    v = [np.where(over, c * sc, c) for c in v]
    out = gv.copy()
    for q in range(3):
        out[..., q] = np.where(act, v[q], gv[..., q])
    return out.reshape(-1, 4), imp[:, :u.num_bed]


# ---------------------------------------------------------------- packing  (shader.rs:1545-1626)

def packing_prepare(u, lanes):
    """Lane 2 after packing_prepare; (6, cells)."""
    L = np.array(lanes, np.int32).reshape(6, -1)
    kind = L[3]
    cell_volume = u.dx * u.dx * u.dx
    packed = np.maximum(lane_f32(u, L[4]), lane_f32(u, L[5])) / np.maximum(cell_volume, F32(1e-8))
    target = np.minimum(u.max_rest_frac, F32(1.0))
    over = np.maximum(packed - target, F32(0.0))
    val = np.where(is_fluid(kind) & (kind != CELL_BED_COUPLED), u.bulk_K * over, F32(0.0))
    L[2] = store_clamped(u, val, F32(0.0), u.p_clamp)
    return L


def packing_apply(u, lanes, grid_vel):
    """`grid_vel` after packing_apply; (cells, 4)."""
    L = np.asarray(lanes, np.int32).reshape(6, *u.grid_shape())
    gv = np.array(grid_vel, np.float32).reshape(*u.grid_shape(), 4)
    kind = L[3]
    pk = lane_f32(u, L[2])
    act = ~(gv[..., 3] <= u.occupancy) & is_fluid(kind)
    pn = {}
    for d in FACES:
        nk = shifted(kind, d, CELL_SOLID)
        mirror = ~in_grid(u, d) | (nk == CELL_SOLID)
        val = np.where(is_fluid(nk), shifted(pk, d, F32(0.0)), F32(0.0))
        pn[d] = np.where(mirror, pk, val)                                  # packing_pressure_or_mirror
    h = F32(0.5) * u.inv_dx
    grad = [h * (pn[FACES[1]] - pn[FACES[0]]), h * (pn[FACES[3]] - pn[FACES[2]]), h * (pn[FACES[5]] - pn[FACES[4]])]
    v = [gv[..., q] - u.dt * grad[q] for q in range(3)]
    speed = length3(*v)
    over = speed > u.vel_cap
    sc = u.vel_cap / np.where(over, speed, F32(1.0))
    v = [np.where(over, c * sc, c) for c in v]
    out = gv.copy()
    for q in range(3):
        out[..., q] = np.where(act, v[q], gv[..., q])
    return out.reshape(-1, 4)


# ---------------------------------------------------------------- viscosity  (shader.rs:1086-1177)

def scratch_store(u, v):
    """velocity_scratch_store (shader.rs:274-283): speed cap, then i32(v * fp)."""
    speed = length3(*v)
    over = speed > u.vel_cap
    sc = u.vel_cap / np.where(over, speed, F32(1.0))
    return [to_i32(np.where(over, c * sc, c) * u.fp) for c in v]


def viscosity_prepare(u, lanes, grid_vel, solid_class):
    """Lanes 1-3 (velocity scratch) after viscosity_prepare; (6, cells)."""
    L = np.array(lanes, np.int32).reshape(6, *u.grid_shape())
    gv = np.asarray(grid_vel, np.float32).reshape(*u.grid_shape(), 4)
    m = gv[..., 3]
    vh = [gv[..., q] for q in range(3)]
    plain = (m <= u.occupancy) | (u.viscosity <= F32(0.0)) | (m <= u.nominal_mass * F32(2.0))
    alpha = clamp(u.viscosity * u.dt / np.maximum(u.dx * u.dx, F32(1e-6)), F32(0.0), F32(0.14))
    vs = [np.zeros(u.grid_shape(), np.float32) for _ in range(3)]
    ws = np.zeros(u.grid_shape(), np.float32)
    cnt = np.zeros(u.grid_shape(), np.int32)
    denom = np.maximum(np.maximum(m, u.nominal_mass), F32(1e-6))
    for d in FACES:
        wall = ~in_grid(u, d) | shifted(solid_class, d, False)
        nm = shifted(m, d, F32(0.0))
        fl = ~wall & ~(nm <= u.occupancy)
        nw = clamp(nm / denom, F32(0.0), F32(1.0))
        for q in range(3):
            vs[q] = np.where(fl, vs[q] + shifted(gv[..., q], d, F32(0.0)) * nw, vs[q])
        ws = np.where(wall, ws + F32(1.0), np.where(fl, ws + nw, ws))
        cnt = cnt + fl
    keep = plain | (cnt < 3) | (ws <= F32(1e-6))
    wsd = np.where(keep, F32(1.0), ws)
    avg = [s / wsd for s in vs]
    blend = clamp(alpha * ws, F32(0.0), F32(0.65))
    out_v = [np.where(keep, vh[q], mix(vh[q], avg[q], blend)) for q in range(3)]
    st = scratch_store(u, out_v)
    for q in range(3):
        L[1 + q] = st[q]
    return L.reshape(6, -1)


def viscosity_apply(u, lanes, grid_vel):
    """`grid_vel` after viscosity_apply; (cells, 4)."""
    L = np.asarray(lanes, np.int32).reshape(6, -1)
    gv = np.array(grid_vel, np.float32).reshape(-1, 4)
    m = gv[:, 3]
    dead = m <= u.occupancy
    out = np.zeros_like(gv)
    for q in range(3):
        out[:, q] = np.where(dead, F32(0.0), lane_f32(u, L[1 + q]))
    out[:, 3] = np.where(dead, F32(0.0), m)
    return out


# ---------------------------------------------------------------- g2p  (shader.rs:1683-1881)

# V60 geometry the shader writes as literals (shader.rs:101, 106-107, 749-750, 800-801)
CONE_TOP_Y, CONE_BOT_Y, CONE_RADIUS_SPAN = F32(3.0), F32(-3.0), F32(4.2634315)
CUP_TOP_Y, CUP_RADIUS, CUP_FLOOR_Y, WALL_THICKNESS = F32(-3.5), F32(3.0), F32(-8.0), F32(0.4)


def radial_barrier(u, pos, vel, max_r, on):
    """resolve_radial_barrier (shader.rs:717-742) about the y axis, where `on`."""
    x, z = pos[0], pos[2]
    r = np.sqrt(x * x + z * z)
    hit = on & (r > max_r) & (r > F32(1e-6))
    rs = np.where(hit, r, F32(1.0))
    ox, oz = x / rs, z / rs
    px = np.where(hit, F32(0.0) + ox * max_r, pos[0])
    pz = np.where(hit, F32(0.0) + oz * max_r, pos[2])
    vn = vel[0] * ox + vel[2] * oz
    slide = hit & (vn > F32(0.0))
    k = F32(1.0) - u.friction * F32(0.35)
    vx = np.where(slide, (vel[0] - ox * vn) * k, vel[0])
    vz = np.where(slide, (vel[2] - oz * vn) * k, vel[2])
    return [px, pos[1], pz], [vx, vel[1], vz]


# paper filter literals (shader.rs:137-141, 765-769)
FILTER_CENTER_Y, FILTER_TOP_REL, FILTER_BOT_REL = F32(-0.35), F32(2.75), F32(3.02)
FILTER_TOP_RADIUS, FILTER_THICKNESS = F32(4.10), F32(0.08)


def coffee_filter_floor_y(u):
    """shader.rs:136-146"""
    top = FILTER_CENTER_Y + FILTER_TOP_REL
    bot = FILTER_CENTER_Y - FILTER_BOT_REL
    bco = np.maximum(u.contact_offset, u.dx * u.bed_r_dx)
    height = np.maximum(top - bot, F32(1e-6))
    slope = FILTER_TOP_RADIUS / height
    return bot + (bco + FILTER_THICKNESS) / np.maximum(slope, F32(1e-6))


def scene_obstacles(u, outlet_r, pos, vel, is_bed):
    """resolve_scene_obstacles (shader.rs:744-823): the cone's radial barrier; for bed
    samples the paper filter's barrier and the apex floor; then the carafe's wall and
    floor."""
    y = pos[1]
    in_cone = (y <= CONE_TOP_Y) & (y >= CONE_BOT_Y)
    t = clamp((y - CONE_BOT_Y) / (CONE_TOP_Y - CONE_BOT_Y), F32(0.0), F32(1.0))
    cone_r = mix(outlet_r, outlet_r + CONE_RADIUS_SPAN, t) - u.contact_offset
    pos, vel = radial_barrier(u, pos, vel, cone_r, in_cone)
    k = F32(1.0) - u.friction * F32(0.55)
    if is_bed:
        top = FILTER_CENTER_Y + FILTER_TOP_REL
        bot = FILTER_CENTER_Y - FILTER_BOT_REL
        bco = np.maximum(u.contact_offset, u.dx * u.bed_r_dx)
        y = pos[1]
        in_f = (y <= top) & (y >= bot)
        ft = clamp((y - bot) / (top - bot), F32(0.0), F32(1.0))
        outer = mix(F32(0.0), FILTER_TOP_RADIUS, ft)
        fr = np.maximum(outer - FILTER_THICKNESS, F32(0.0)) - bco
        pos, vel = radial_barrier(u, pos, vel, np.maximum(fr, F32(0.0)), in_f)
        fl = coffee_filter_floor_y(u)
        at = pos[1] <= fl
        stop = at & (vel[1] < F32(0.0))
        pos = [np.where(at, F32(0.0), pos[0]), np.where(at, fl, pos[1]), np.where(at, F32(0.0), pos[2])]
        vx = np.where(stop, vel[0] * k, vel[0])
        vz = np.where(stop, vel[2] * k, vel[2])
        vel = [np.where(at, vx * k, vel[0]), np.where(stop, F32(0.0), vel[1]), np.where(at, vz * k, vel[2])]
    half = WALL_THICKNESS * F32(0.5)
    in_cup = pos[1] <= CUP_TOP_Y
    pos, vel = radial_barrier(u, pos, vel, CUP_RADIUS - half - u.contact_offset, in_cup)
    floor_y = CUP_FLOOR_Y + half + u.contact_offset
    below = in_cup & (pos[1] < floor_y)
    stop = below & (vel[1] < F32(0.0))
    pos = [pos[0], np.where(below, floor_y, pos[1]), pos[2]]
    vel = [np.where(stop, vel[0] * k, vel[0]), np.where(stop, F32(0.0), vel[1]), np.where(stop, vel[2] * k, vel[2])]
    return pos, vel


def sdf_contact(u, sdf, outlet_r, pos, vel, is_bed=False):
    """resolve_sdf_contact (shader.rs:879-903)."""
    sd = sdf.sample(*pos)
    n = sdf.gradient(*pos)
    near = (sd < u.contact_offset) & (length3(*n) > F32(1e-6))
    push = u.contact_offset - sd
    pos = [np.where(near, pos[q] + n[q] * push, pos[q]) for q in range(3)]
    vn = vel[0] * n[0] + vel[1] * n[1] + vel[2] * n[2]
    hit = near & (vn < F32(0.0))
    k = F32(1.0) + u.restitution
    v2 = [vel[q] - n[q] * vn * k for q in range(3)]
    d2 = v2[0] * n[0] + v2[1] * n[1] + v2[2] * n[2]
    vt = [v2[q] - n[q] * d2 for q in range(3)]
    vtl = length3(*vt)
    fr = hit & (vtl > F32(1e-6))
    imp = np.minimum(u.friction * np.abs(vn), vtl)
    safe = np.where(fr, vtl, F32(1.0))
    v3 = [np.where(fr, v2[q] - vt[q] * (imp / safe), v2[q]) for q in range(3)]
    vel = [np.where(hit, v3[q], vel[q]) for q in range(3)]
    return scene_obstacles(u, outlet_r, pos, vel, is_bed)


def g2p(u, sdf, bed, outlet_r, particles, affine, grid_vel, exp=np.exp, stats=None):
    """Particles, affine columns and bed impulse sums after G2P.  Returns (particles
    (n, 8), affine (n, 12), impulse sums (3, num_bed) int64).  `exp` evaluates the J
    update's exponential (shader.rs:1853), whose precision WGSL leaves to the backend.
    `stats`, if a dict, receives how many samples took each branch."""
    n = u.num_water + u.num_bed
    P = np.array(particles, np.float32).reshape(-1, 8)[:n]
    A = np.array(affine, np.float32).reshape(-1, 12)[:n]
    gv = np.asarray(grid_vel, np.float32).reshape(-1, 4)
    imp = np.zeros((3, max(u.num_bed, 1)), np.int64)
    water = A[:, 3] < F32(0.5)
    idle = water & (P[:, 7] <= u.inactive)
    P[idle, 7] = F32(0.0)                                                    # shader.rs:1695-1698
    act = np.flatnonzero(water & ~idle)
    if act.size == 0:
        return P, A, imp[:, :u.num_bed]
    p, a = P[act], A[act]
    xp, J_old, vp, mass = [p[:, q] for q in range(3)], p[:, 3], [p[:, 4 + q] for q in range(3)], p[:, 7]
    gp = [(xp[q] - u.origin[q]) * u.inv_dx for q in range(3)]
    base = [to_i32(np.floor(c - F32(0.5))) for c in gp]
    fx = [gp[q] - base[q].astype(np.float32) for q in range(3)]
    w = [[F32(0.5) * (F32(1.5) - f) * (F32(1.5) - f), F32(0.75) - (f - F32(1.0)) * (f - F32(1.0)),
          F32(0.5) * (f - F32(0.5)) * (f - F32(0.5))] for f in fx]
    m = act.size
    z = lambda: np.zeros(m, np.float32)  # noqa: E731
    new_v, C = [z(), z(), z()], [[z(), z(), z()] for _ in range(3)]
    supported, local_mass, bow, bps = z(), z(), z(), z()
    bvs = [z(), z(), z()]
    B = F32(4.0) * u.inv_dx * u.inv_dx
    lookup = bed.lookup.reshape(-1)
    for i in range(3):
        for j in range(3):
            for k in range(3):
                cx, cy, cz = base[0] + i, base[1] + j, base[2] + k
                ok = (cx >= 0) & (cy >= 0) & (cz >= 0) & (cx < u.gx) & (cy < u.gy) & (cz < u.gz)
                ci = np.where(ok, (cz.astype(np.int64) * u.gy + cy) * u.gx + cx, 0)
                wt = w[0][i] * w[1][j] * w[2][k]
                g = gv[ci]
                dpos = [(F32(o) - fx[q]) * u.dx for q, o in enumerate((i, j, k))]
                sup = ok & (g[:, 3] > F32(1e-6))
                for q in range(3):
                    new_v[q] = np.where(sup, new_v[q] + wt * g[:, q], new_v[q])
                wB = wt * B
                for col in range(3):
                    for q in range(3):
                        C[col][q] = np.where(sup, C[col][q] + wB * g[:, q] * dpos[col], C[col][q])
                supported = np.where(sup, supported + wt, supported)
                local_mass = np.where(sup, local_mass + wt * g[:, 3], local_mass)
                bi = np.where(ok, lookup[ci], -1)
                vb = ok & (u.num_bed > 0) & bed.valid_solid(bi)
                sb = np.where(vb, bi, 0)
                bow = np.where(vb, bow + wt, bow)
                for q in range(3):
                    bvs[q] = np.where(vb, bvs[q] + wt * bed.vel[sb, q], bvs[q]) if u.num_bed else bvs[q]
                if u.num_bed:
                    bps = np.where(vb, bps + wt * bed.compacted_permeability(sb), bps)
    support_ratio = clamp(supported, F32(0.0), F32(1.0))
    jus = support_ratio
    has = supported > F32(1e-6)
    inv = F32(1.0) / np.where(has, supported, F32(1.0))
    new_v = [np.where(has, c * inv, c) for c in new_v]
    C = [[np.where(has, c * inv, c) for c in col] for col in C]
    co = u.contact_offset
    cupr = F32(3.0) + co
    in_cup = (xp[1] < F32(-3.5)) & ((xp[0] * xp[0] + xp[2] * xp[2]) < cupr * cupr)
    dense = clamp(local_mass / np.maximum(u.nominal_mass * F32(4.0), F32(1e-6)), F32(0.0), F32(1.0))
    porous = clamp(bow, F32(0.0), F32(1.0))
    hb = bow > F32(1e-6)
    invb = F32(1.0) / np.where(hb, bow, F32(1.0))
    pbv = [np.where(hb, c * invb, F32(0.0)) for c in bvs]
    pbp = np.where(hb, np.maximum(bps * invb, u.min_perm), u.min_perm)
    ballistic = [vp[0], vp[1] + u.gravity * u.dt, vp[2]]
    # weak stencil support (shader.rs:1778-1792)
    weak = support_ratio < F32(0.999)
    pg = mix(np.where(in_cup, F32(1.15), F32(1.35)), F32(0.18), porous)
    pc = mix(np.where(in_cup, F32(0.95), F32(0.995)), F32(0.16), porous)
    dpd = mix(F32(1.0), F32(0.12), dense)
    keep = clamp((F32(1.0) - support_ratio) * pg * dpd, F32(0.0), pc)
    new_v = [np.where(weak, mix(new_v[q], ballistic[q], keep), new_v[q]) for q in range(3)]
    ad = F32(1.0) - keep * F32(0.75)
    C = [[np.where(weak, c * ad, c) for c in col] for col in C]
    # airborne (shader.rs:1798-1812)
    airborne = (porous <= F32(0.05)) & (sdf.sample(*xp) > co * F32(2.0))
    dr = clamp(local_mass / np.maximum(u.nominal_mass * F32(4.0), F32(1e-6)), F32(0.0), F32(1.0))
    jus = np.where(airborne, np.minimum(jus, dr), jus)
    pg = np.where(in_cup, F32(0.72), F32(0.98))
    pc = np.where(in_cup, F32(0.88), F32(0.98))
    keep = clamp((F32(1.0) - dr) * pg, F32(0.0), pc)
    new_v = [np.where(airborne, mix(new_v[q], ballistic[q], keep), new_v[q]) for q in range(3)]
    ad = F32(1.0) - keep * F32(0.65)
    C = [[np.where(airborne, c * ad, c) for c in col] for col in C]
    # porous drag (shader.rs:1814-1834)
    por = porous > F32(1e-4)
    rel = [new_v[q] - pbv[q] for q in range(3)]
    rate = u.nu_m2s / pbp
    dd = F32(1.0) / (F32(1.0) + np.maximum(rate * u.dt * porous, F32(0.0)))
    rs = length3(*rel)
    idmp = F32(1.0) / (F32(1.0) + np.maximum(rs * u.dt * u.inv_dx * porous * F32(0.35), F32(0.0)))
    dragged = [pbv[q] + rel[q] * dd * idmp for q in range(3)]
    wimp = [mass * (dragged[q] - new_v[q]) for q in range(3)]
    new_v = [np.where(por, dragged[q], new_v[q]) for q in range(3)]
    ad = mix(F32(1.0), dd * idmp, porous)
    C = [[np.where(por, c * ad, c) for c in col] for col in C]
    jus = np.where(por, np.maximum(jus, porous), jus)
    if stats is not None:
        stats.update(active=int(act.size), weak=int(weak.sum()), airborne=int(airborne.sum()), porous=int(por.sum()))
    if por.any() and u.num_bed:
        sel = np.flatnonzero(por)
        cell = [to_i32(np.floor((xp[q][sel] - u.origin[q]) * u.inv_dx)) for q in range(3)]   # world_to_cell
        share_in = [(-wimp[q][sel]) * BED_REACTION_ALPHA for q in range(3)]
        _impulse_neighbourhood(u, bed, cell, share_in, imp)
    # J update (shader.rs:1836-1840)
    trace = C[0][0] + C[1][1] + C[2][2]
    jc = clamp(np.where(J_old > F32(0.0), J_old, F32(1.0)), F32(0.40), F32(2.00))
    ex = exp(clamp(u.dt * trace, F32(-0.35), F32(0.35)).astype(np.float64)).astype(np.float32)
    j_apic = clamp(jc * ex, F32(0.40), F32(2.00))
    jb = smoothstep(F32(0.35), F32(0.85), clamp(jus, F32(0.0), F32(1.0)))
    j_new = clamp(mix(jc, j_apic, jb), F32(0.40), F32(2.00))
    # advection and particle-level contact (shader.rs:1842-1869)
    new_pos = [xp[q] + new_v[q] * u.dt for q in range(3)]
    mid = [mix(xp[q], new_pos[q], F32(0.5)) for q in range(3)]
    _, new_v = sdf_contact(u, sdf, outlet_r, mid, new_v)
    new_pos, new_v = sdf_contact(u, sdf, outlet_r, new_pos, new_v)
    margin = u.dx * F32(0.5)
    new_pos = [clamp(new_pos[q], u.origin[q] + margin, u.bounds_max[q] - margin) for q in range(3)]
    for q in range(3):
        P[act, q] = new_pos[q]
        P[act, 4 + q] = new_v[q]
        for col in range(3):
            A[act, 4 * col + q] = C[col][q]
    P[act, 3] = j_new
    A[act, 7] = F32(0.0)
    A[act, 11] = F32(0.0)
    return P, A, imp[:, :u.num_bed]


def _impulse_neighbourhood(u, bed, cell, share_in, imp):
    """bed_impulse_delta_add_neighborhood (shader.rs:479-515) for a batch of home cells."""
    cx, cy, cz = cell
    count = np.zeros(cx.shape, np.float32)
    lk = bed.lookup
    nbr = []
    for di in (-1, 0, 1):
        for dj in (-1, 0, 1):
            for dk in (-1, 0, 1):
                x, y, z = cx + di, cy + dj, cz + dk
                on = (x >= 0) & (y >= 0) & (z >= 0) & (x < u.gx) & (y < u.gy) & (z < u.gz)
                bi = np.where(on, lk[np.clip(z, 0, u.gz - 1), np.clip(y, 0, u.gy - 1), np.clip(x, 0, u.gx - 1)], -1)
                ok = bed.valid_solid(bi)
                count = np.where(ok, count + F32(1.0), count)
                nbr.append((bi, ok))
    has = ~(count <= F32(0.0))
    cnt = np.where(has, count, F32(1.0))
    cap = u.nominal_mass * u.vel_cap * BED_REACTION_IMPULSE_CAP
    q_i = [to_i32(clamp(s / cnt, -cap, cap) * u.fp).astype(np.int64) for s in share_in]
    for bi, ok in nbr:
        mk = ok & has
        for q in range(3):
            np.add.at(imp[q], bi[mk], q_i[q][mk])


# ---------------------------------------------------------------- bed lookup  (shader.rs:2289-2335)

def world_to_cell(u, pos):
    """shader.rs:668-671 for rows of positions: (n, 3) int32."""
    return np.stack([to_i32(np.floor((pos[:, q] - u.origin[q]) * u.inv_dx)) for q in range(3)], axis=1)


def bed_lookup(u, particles, affine):
    """bed_lookup_clear then bed_lookup_scatter: every solid-phase bed sample stamps its
    id over the 3x3x3 cells around its cell, the highest id winning (atomicMax)."""
    look = np.full(u.cells, -1, np.int64)
    nb = u.num_bed
    if nb == 0:
        return look.astype(np.int32)
    p = np.asarray(particles, np.float32).reshape(-1, 8)[:nb]
    ph = np.asarray(affine, np.float32).reshape(-1, 12)[:nb, 3]
    ids = np.flatnonzero(~(ph < F32(0.5)))
    cell = world_to_cell(u, p[ids, 0:3])
    for di in (-1, 0, 1):
        for dj in (-1, 0, 1):
            for dk in (-1, 0, 1):
                c = cell + np.array([di, dj, dk])
                ok = (c >= 0).all(axis=1) & (c[:, 0] < u.gx) & (c[:, 1] < u.gy) & (c[:, 2] < u.gz)
                ci = (c[ok, 2].astype(np.int64) * u.gy + c[ok, 1]) * u.gx + c[ok, 0]
                np.maximum.at(look, ci, ids[ok])
    return look.astype(np.int32)


# ---------------------------------------------------------------- bed_coupling  (shader.rs:1885-1957)

def bed_coupling(u, bed, particles, affine):
    """Particles after bed_coupling and the water-lane additions it makes: (particles
    (n, 8), (num_bed,) int64 sums).  The paper-absorption branch (shader.rs:1906-1911)
    runs only with a positive filter absorption rate; the default brew has none."""
    assert not u.filter_absorption > 0, "the restatement leaves out paper absorption"
    n = u.num_water + u.num_bed
    P = np.array(particles, np.float32).reshape(-1, 8)[:n]
    ph = np.asarray(affine, np.float32).reshape(-1, 12)[:n, 3]
    add = np.zeros(max(u.num_bed, 1), np.int64)
    cand = np.flatnonzero(ph < F32(0.5))
    cell = world_to_cell(u, P[cand, 0:3])
    on = (cell >= 0).all(axis=1) & (cell[:, 0] < u.gx) & (cell[:, 1] < u.gy) & (cell[:, 2] < u.gz)
    cand, cell = cand[on], cell[on]
    ci = (cell[:, 2].astype(np.int64) * u.gy + cell[:, 1]) * u.gx + cell[:, 0]
    bi = bed.lookup.reshape(-1)[ci]
    ok = (bi >= 0) & (bi < u.num_bed)
    cand, cell, bi = cand[ok], cell[ok], bi[ok]
    be = bed.bx[bi]
    mass = P[cand, 7]
    sat = be[:, 7]
    capacity = np.maximum(u.max_saturation - be[:, 0], F32(0.0))
    go = ~(capacity <= F32(1e-6))
    abs_rate = u.absorption_rate * (F32(1.0) - sat) * u.dt
    v = P[cand, 4:7]
    speed = length3(v[:, 0], v[:, 1], v[:, 2])
    absorbed = np.minimum(np.minimum(mass * clamp(abs_rate, F32(0.0), F32(0.25)), mass * F32(0.5)), capacity)
    rem = mass - absorbed
    retire = (rem > F32(0.0)) & (rem <= u.nominal_mass * F32(0.22))
    almost = np.minimum(mass, capacity)
    wet = ~retire & (sat > F32(0.55)) & (speed < F32(1.35)) & ((mass - almost) <= u.nominal_mass * F32(0.35))
    absorbed = np.where(retire | wet, almost, absorbed)
    remnant = ((mass - absorbed) <= u.inactive) & (absorbed < mass)
    absorbed = np.where(remnant, np.maximum(mass - u.inactive * F32(1.05), F32(0.0)), absorbed)
    go &= ~(absorbed <= F32(1e-6))
    cand, cell, bi, mass, absorbed = cand[go], cell[go], bi[go], mass[go], absorbed[go]
    remaining = mass - absorbed
    gone = remaining <= u.inactive
    P[cand[gone], 4:8] = F32(0.0)
    P[cand[~gone], 7] = remaining[~gone]
    # deposit_absorbed_bed_water (shader.rs:524-576)
    nshare = absorbed * F32(0.35)
    home = absorbed - nshare

    def water_add(ids, amount):
        pos = ~(amount <= F32(0.0))
        np.add.at(add, ids[pos], to_i32(amount[pos] * u.fp).astype(np.int64))

    water_add(bi, home)
    nbr = np.full((bi.size, 6), -1, np.int64)
    lk = bed.lookup
    for f, d in enumerate(FACES):
        c = cell + np.array(d)
        on = (c >= 0).all(axis=1) & (c[:, 0] < u.gx) & (c[:, 1] < u.gy) & (c[:, 2] < u.gz)
        nid = np.where(on, lk[np.clip(c[:, 2], 0, u.gz - 1), np.clip(c[:, 1], 0, u.gy - 1), np.clip(c[:, 0], 0, u.gx - 1)], -1)
        keep = (nid >= 0) & (nid != bi) & (nid < u.num_bed)
        for g in range(f):
            keep &= nbr[:, g] != nid
        nbr[:, f] = np.where(keep, nid, -1)
    count = (nbr >= 0).sum(axis=1)
    lone = count == 0
    water_add(bi[lone], nshare[lone])
    each = nshare / np.where(lone, 1, count).astype(np.float32)
    for f in range(6):
        has = ~lone & (nbr[:, f] >= 0)
        water_add(nbr[has, f], each[has])
    return P, add[:u.num_bed]


# ---------------------------------------------------------------- extraction_advect  (shader.rs:1961-1987)

def extraction_advect(u, bed_extract, water_lane):
    """bed_extract rows after extraction_advect, given the water lane it exchanges to 0."""
    be = np.array(bed_extract, np.float32).reshape(-1, 8)[:u.num_bed]
    absorbed = np.asarray(water_lane, np.int32)[:u.num_bed].astype(np.float32) * u.inv_fp
    got = absorbed > F32(0.0)
    be[:, 0] = np.where(got, be[:, 0] + absorbed, be[:, 0])
    be[:, 7] = np.where(got, clamp(be[:, 0] / np.maximum(u.max_saturation, F32(1e-6)), F32(0.0), F32(1.0)), be[:, 7])
    sat = be[:, 7]
    ex = sat > F32(0.01)
    flux = u.extraction_rate * be[:, 4] * sat * u.dt
    be[:, 4] = np.where(ex, np.maximum(be[:, 4] - flux, F32(0.0)), be[:, 4])
    be[:, 5] = np.where(ex, be[:, 5] + flux, be[:, 5])
    return be


# ---------------------------------------------------------------- prepare_render  (shader.rs:2242-2276)

def prepare_render(u, particles, affine, bed_extract):
    """Render rows (n, 8): position and colour parameter, then radius."""
    n = u.num_water + u.num_bed
    p = np.asarray(particles, np.float32).reshape(-1, 8)[:n]
    ph = np.asarray(affine, np.float32).reshape(-1, 12)[:n, 3]
    out = np.zeros((n, 8), np.float32)
    dead = p[:, 7] <= u.inactive
    water = ph < F32(0.5)
    speed = length3(p[:, 4], p[:, 5], p[:, 6])
    sat = np.zeros(n, np.float32)
    isbed = np.arange(n) < u.num_bed
    if u.num_bed:
        sat[:u.num_bed] = np.asarray(bed_extract, np.float32).reshape(-1, 8)[:u.num_bed, 7]
    colour = np.where(water, clamp(speed / F32(10.0), F32(0.0), F32(2.0)), F32(-1.0) - np.where(isbed, sat, F32(0.0)))
    radius = np.where(~water & isbed, u.dx * u.bed_r_dx, u.dx * u.water_r_dx)
    out[:, 0:3] = p[:, 0:3]
    out[:, 3] = colour
    out[:, 4] = radius
    out[dead] = np.array([0.0, -1e6, 0.0, -999.0, 0, 0, 0, 0], np.float32)
    return out


# ---------------------------------------------------------------- bed_dynamics  (shader.rs:1991-2238)

def _pressure_gradient_at(u, lanes, cell):
    """pressure_gradient_at_cell (shader.rs:238-260) at rows of cells (n, 3): the pressure
    lane and whatever lane 3 holds when it runs (the kind test is `== CELL_SOLID`)."""
    L = np.asarray(lanes, np.int32).reshape(6, -1)
    p = lane_f32(u, L[0])
    kind = L[3]
    cx, cy, cz = cell[:, 0], cell[:, 1], cell[:, 2]

    def on(x, y, z):
        return (x >= 0) & (y >= 0) & (z >= 0) & (x < u.gx) & (y < u.gy) & (z < u.gz)

    def idx(x, y, z):
        return (np.clip(z, 0, u.gz - 1).astype(np.int64) * u.gy + np.clip(y, 0, u.gy - 1)) * u.gx + np.clip(x, 0, u.gx - 1)

    here_on = on(cx, cy, cz)
    ph = p[idx(cx, cy, cz)]
    nbp = []
    for d in FACES:
        x, y, z = cx + d[0], cy + d[1], cz + d[2]
        i = idx(x, y, z)
        mirror = ~on(x, y, z) | (kind[i] == CELL_SOLID)
        nbp.append(np.where(mirror, ph, p[i]))
    h = F32(0.5) * u.inv_dx
    g = [h * (nbp[1] - nbp[0]), h * (nbp[3] - nbp[2]), h * (nbp[5] - nbp[4])]
    return [np.where(here_on, c, F32(0.0)) for c in g]


def _coffee_packing(u, bed_pos, lookup, pos, vel, bids):
    """resolve_coffee_particle_packing (shader.rs:825-877).  Other samples' positions are
    read from `bed_pos`, the positions before the dispatch."""
    cell = world_to_cell(u, np.stack(pos, axis=1))
    m = bids.size
    best = np.full(m, F32(1e9), np.float32)
    bd = [np.zeros(m, np.float32) for _ in range(3)]
    found = np.zeros(m, bool)
    lk = lookup.reshape(-1)
    for di in (-1, 0, 1):
        for dj in (-1, 0, 1):
            for dk in (-1, 0, 1):
                x, y, z = cell[:, 0] + di, cell[:, 1] + dj, cell[:, 2] + dk
                ok = (x >= 0) & (y >= 0) & (z >= 0) & (x < u.gx) & (y < u.gy) & (z < u.gz)
                ci = (np.clip(z, 0, u.gz - 1).astype(np.int64) * u.gy + np.clip(y, 0, u.gy - 1)) * u.gx + np.clip(x, 0, u.gx - 1)
                o = np.where(ok, lk[ci], -1)
                ok &= (o >= 0) & (o != bids) & (o < u.num_bed)
                so = np.where(ok, o, 0)
                d = [pos[q] - bed_pos[so, q] for q in range(3)]
                dist = length3(*d)
                better = ok & (dist < best)
                best = np.where(better, dist, best)
                bd = [np.where(better, d[q], bd[q]) for q in range(3)]
                found |= better
    min_sep = u.dx * u.bed_r_dx * F32(1.78)
    hit = found & (best < min_sep)
    far = best > F32(1e-5)
    sb = np.where(far, best, F32(1.0))
    n = [np.where(far, bd[0] / sb, F32(0.0)), np.where(far, bd[1] / sb, F32(1.0)), np.where(far, bd[2] / sb, F32(0.0))]
    push = np.minimum((min_sep - best) * F32(0.65), u.dx * F32(0.22))
    pos = [np.where(hit, pos[q] + n[q] * push, pos[q]) for q in range(3)]
    vn = vel[0] * n[0] + vel[1] * n[1] + vel[2] * n[2]
    back = hit & (vn < F32(0.0))
    vel = [np.where(back, vel[q] - n[q] * vn, vel[q]) for q in range(3)]
    return pos, vel


def bed_dynamics(u, sdf, outlet_r, lanes, grid_vel, lookup, particles, affine, bed_extract, impulse_lanes,
                 bed_damping=F32(8.5), surface_ref_y=F32(3.0), surface_span=F32(3.5)):
    """Bed samples after bed_dynamics: (particles (num_bed, 8), affine (num_bed, 12),
    bed_extract (num_bed, 8)).  `impulse_lanes` are the three i32 impulse lanes that
    bed_impulse_delta_exchange (shader.rs:517-522) reads and clears.  Another sample's
    position (the packing contact) is its position before the dispatch."""
    nb = u.num_bed
    P = np.array(particles, np.float32).reshape(-1, 8)[:nb].copy()
    A = np.array(affine, np.float32).reshape(-1, 12)[:nb].copy()
    BE = np.array(bed_extract, np.float32).reshape(-1, 8)[:nb].copy()
    gv = np.asarray(grid_vel, np.float32).reshape(-1, 4)
    lk = np.asarray(lookup, np.int32).reshape(-1)
    bed_pos = P[:, 0:3].copy()
    bids = np.arange(nb)
    pos = [P[:, q] for q in range(3)]
    v0 = [P[:, 4 + q] for q in range(3)]
    mass = P[:, 7]
    phase = A[:, 3].copy()
    rest = [A[:, 4 + q].copy() for q in range(3)]
    imp = [np.asarray(impulse_lanes[q], np.int32)[:nb].astype(np.float32) * u.inv_fp for q in range(3)]
    den = np.maximum(mass, u.nominal_mass * F32(0.25))
    brv = [c / den for c in imp]
    max_rs = np.minimum(u.vel_cap * F32(0.012), u.dx / np.maximum(u.dt, F32(1e-6)) * F32(0.02))
    rs = length3(*brv)
    over = (rs > max_rs) & (rs > F32(1e-6))
    sc = max_rs / np.where(over, rs, F32(1.0))
    brv = [np.where(over, c * sc, c) for c in brv]
    gp = [(pos[q] - u.origin[q]) * u.inv_dx for q in range(3)]
    base = [to_i32(np.floor(c - F32(0.5))) for c in gp]
    fx = [gp[q] - base[q].astype(np.float32) for q in range(3)]
    w = [[F32(0.5) * (F32(1.5) - f) * (F32(1.5) - f), F32(0.75) - (f - F32(1.0)) * (f - F32(1.0)),
          F32(0.5) * (f - F32(0.5)) * (f - F32(0.5))] for f in fx]
    z = lambda: np.zeros(nb, np.float32)  # noqa: E731
    wv, wm, asw, lasw = [z(), z(), z()], z(), z(), z()
    for i in range(3):
        for j in range(3):
            for k in range(3):
                cx, cy, cz = base[0] + i, base[1] + j, base[2] + k
                ok = (cx >= 0) & (cy >= 0) & (cz >= 0) & (cx < u.gx) & (cy < u.gy) & (cz < u.gz)
                ci = np.where(ok, (cz.astype(np.int64) * u.gy + cy) * u.gx + cx, 0)
                wt = w[0][i] * w[1][j] * w[2][k]
                g = gv[ci]
                wv = [np.where(ok, wv[q] + wt * g[:, q], wv[q]) for q in range(3)]
                wm = np.where(ok, wm + wt * g[:, 3], wm)
                sb = np.where(ok, lk[ci], -1)
                sup = ok & (sb >= 0) & (sb != bids)
                asw = np.where(sup, asw + wt, asw)
                ccy = u.origin[1] + (cy.astype(np.float32) + F32(0.5)) * u.dx
                lower = sup & (ccy <= pos[1] + u.dx * F32(0.25))
                lasw = np.where(lower, lasw + wt, lasw)
    floor_y = coffee_filter_floor_y(u)
    out_pos, out_vel = [c.copy() for c in pos], [c.copy() for c in v0]
    # suspended grains (shader.rs:2064-2105)
    sus = phase >= F32(1.5)
    ws = clamp(wm / np.maximum(u.nominal_mass * F32(2.0), F32(1e-6)), F32(0.0), F32(1.0))
    drag = clamp((F32(8.0) + F32(18.0) * ws) * u.dt, F32(0.0), F32(1.0))
    unsup = [v0[0] + brv[0] + F32(0.0), v0[1] + brv[1] + u.gravity * u.dt * F32(0.85), v0[2] + brv[2] + F32(0.0)]
    settle = mix(F32(1.10), F32(0.32), ws)
    carried = [wv[0] + F32(0.0), wv[1] + (-settle), wv[2] + F32(0.0)]
    sv = [mix(unsup[q], carried[q], drag) for q in range(3)]
    sp = length3(*sv)
    o = sp > u.vel_cap
    f = u.vel_cap / np.where(o, sp, F32(1.0))
    sv = [np.where(o, c * f, c) for c in sv]
    spos = [pos[q] + sv[q] * u.dt for q in range(3)]
    spos, sv = sdf_contact(u, sdf, outlet_r, spos, sv, True)
    anchored = (lasw > F32(0.06)) | (asw > F32(0.20))
    dense = asw > F32(0.42)
    redeposit = ((spos[1] <= floor_y + u.dx * F32(0.35)) & (ws < F32(0.35))) | \
        (anchored & (sv[1] <= F32(0.20)) & ((ws < F32(0.55)) | dense))
    # anchored grains (shader.rs:2107-2237)
    sat = BE[:, 7]
    wl = clamp(wm / np.maximum(u.nominal_mass * F32(1.5), F32(1e-6)), F32(0.0), F32(1.0))
    mob = clamp((F32(0.30) + wl * F32(0.62)) * (F32(1.0) + sat * F32(0.40)), F32(0.0), F32(1.0))
    sf = clamp((rest[1] + surface_ref_y) / surface_span, F32(0.12), F32(1.0))
    damping = clamp(F32(1.0) - bed_damping * u.dt, F32(0.0), F32(1.0))
    vel = [v0[q] + brv[q] for q in range(3)]
    sr = clamp(F32(1.0) - asw / F32(0.55), F32(0.0), F32(1.0))
    entr = clamp((F32(2.0) + F32(5.0) * sat) * wl * sr * u.dt, F32(0.0), F32(0.08))
    gs = -mix(F32(0.95), F32(0.35), wl)
    tgt = [wv[0] + F32(0.0), wv[1] + gs, wv[2] + F32(0.0)]
    vel = [mix(vel[q], tgt[q], entr) for q in range(3)]
    lsp = np.sqrt(wv[0] * wv[0] + wv[2] * wv[2])
    lon = lsp > F32(1e-6)
    ls = np.where(lon, lsp, F32(1.0))
    ldx, ldz = np.where(lon, wv[0] / ls, F32(0.0)), np.where(lon, wv[2] / ls, F32(0.0))
    down = np.minimum(wv[1], F32(0.0))
    lss = np.minimum(lsp, np.abs(down) * F32(0.18))
    impact = [ldx * lss * F32(0.08), down * F32(0.62), ldz * lss * F32(0.08)]
    bi_ = u.bed_impact
    vel = [vel[q] + impact[q] * bi_ * mob * sf * u.dt for q in range(3)]
    pg = _pressure_gradient_at(u, lanes, world_to_cell(u, np.stack(pos, axis=1)))
    sx, sz = -pg[0], -pg[2]
    ssp = np.sqrt(sx * sx + sz * sz)
    son = ssp > F32(1e-6)
    sss = np.where(son, ssp, F32(1.0))
    sdx, sdz = np.where(son, sx / sss, F32(0.0)), np.where(son, sz / sss, F32(0.0))
    drive = np.minimum(ssp, u.vel_cap / np.maximum(u.dt, F32(1e-6)))
    pl = clamp(wm * (F32(0.25) + sat), F32(0.0), F32(1.0))
    slx, slz = sdx * drive * pl * F32(0.08), sdz * drive * pl * F32(0.08)
    vel[0] = vel[0] + slx * bi_ * mob * sf * u.dt
    vel[2] = vel[2] + slz * bi_ * mob * sf * u.dt
    vel = [c * damping for c in vel]
    npos = [pos[q] + vel[q] * u.dt for q in range(3)]
    off = [npos[q] - rest[q] for q in range(3)]
    ll = np.sqrt(off[0] * off[0] + off[2] * off[2])
    lpt = u.dx * F32(0.22)
    lat = (ll > lpt) & (ll > F32(1e-6))
    lls = np.where(lat, ll, F32(1.0))
    ldx2, ldz2 = off[0] / lls, off[2] / lls
    lex = ll - lpt
    lplast = clamp((F32(0.04) + sat * F32(0.35) + mob * F32(0.45) + pl * F32(0.25)) * sf * u.compaction_rate * u.dt,
                   F32(0.0), F32(0.18))
    rest = [np.where(lat, rest[0] + ldx2 * lex * lplast, rest[0]), rest[1],
            np.where(lat, rest[2] + ldz2 * lex * lplast, rest[2])]
    off = [np.where(lat, npos[q] - rest[q], off[q]) for q in range(3)]
    cll = np.sqrt(off[0] * off[0] + off[2] * off[2])
    max_lat = u.dx * F32(0.9) * sf
    cap = (cll > max_lat) & (cll > F32(1e-6))
    cls = np.where(cap, cll, F32(1.0))
    off[0] = np.where(cap, off[0] / cls * max_lat, off[0])
    off[2] = np.where(cap, off[2] / cls * max_lat, off[2])
    vel[0] = np.where(cap, vel[0] * F32(0.4), vel[0])
    vel[2] = np.where(cap, vel[2] * F32(0.4), vel[2])
    off[1] = clamp(off[1], (-u.dx) * (F32(1.75) * sf + F32(0.2)), u.dx * F32(0.04))
    npos = [rest[q] + off[q] for q in range(3)]
    npos, vel = _coffee_packing(u, bed_pos, lk, npos, vel, bids)
    comp = np.maximum(rest[1] - npos[1], F32(0.0))
    pt = u.dx * F32(0.18)
    plast = clamp((F32(0.05) + sat * F32(0.35) + mob * F32(0.55)) * sf * u.compaction_rate * u.dt, F32(0.0), F32(0.18))
    rest[1] = np.where(comp > pt, rest[1] - (comp - pt) * plast, rest[1])
    hyd = (sat > F32(0.82)) & (pl > F32(0.65)) & (wl > F32(0.65)) & (sr > F32(0.35)) & \
        ((comp > u.dx * F32(0.65)) | (cll > u.dx * F32(0.65)))
    flow = (sat > F32(0.58)) & (wl > F32(0.74)) & (sr > F32(0.55)) & (length3(*wv) > F32(0.95)) & \
        (npos[1] > floor_y + u.dx * F32(0.70))
    iso = (sat > F32(0.55)) & (wm < u.nominal_mass * F32(0.75)) & (asw < F32(0.04)) & (lasw < F32(0.03)) & \
        (npos[1] > floor_y + u.dx * F32(0.50))
    detach = hyd | flow | iso
    rest = [np.where(detach, npos[q], rest[q]) for q in range(3)]
    anchored_phase = np.where(detach, F32(2.0), phase)
    npos, vel = sdf_contact(u, sdf, outlet_r, npos, vel, True)
    gc = np.maximum((rest[1] - npos[1]) / np.maximum(u.dx, F32(1e-6)), F32(0.0))
    for q in range(3):
        P[:, q] = np.where(sus, spos[q], npos[q])
        P[:, 4 + q] = np.where(sus, sv[q], vel[q])
        A[:, 4 + q] = np.where(sus, spos[q], rest[q])
    A[:, 7] = F32(0.0)
    A[:, 3] = np.where(sus, np.where(redeposit, F32(1.0), phase), anchored_phase)
    BE[:, 3] = np.where(sus, BE[:, 3] * F32(0.985), np.maximum(BE[:, 3] * F32(0.995), gc))
    return P, A, BE


# ---------------------------------------------------------------- SDF texture and solid class  (state.rs:206-344)

SDF_NO_CONSTRAINT = F32(999.0)      # state.rs:30


def generate_sdf(raw, wall_thickness=WALL_THICKNESS):
    """generate_sdf_data (state.rs:250-275) with sdf_interior (state.rs:206-248): the
    max-union of the obstacles' interior distances, inset by half the wall thickness, at
    the centres of a 128^3 lattice over the bounds; (128^3,) float32, x fastest.  The
    reference's wall is OBSTACLE_WALL_THICKNESS = 0.4 scene units; scenes in other units
    pass their own."""
    n = SDF_RES
    b = [F32(v) for v in raw.bounds_size]
    iz, iy, ix = np.meshgrid(np.arange(n, dtype=np.float32), np.arange(n, dtype=np.float32),
                             np.arange(n, dtype=np.float32), indexing="ij")
    p = [(-b[a]) * F32(0.5) + (c + F32(0.5)) * b[a] / F32(n) for a, c in enumerate((ix, iy, iz))]
    data = np.full((n, n, n), SDF_NO_CONSTRAINT, np.float32)
    half = F32(wall_thickness) * F32(0.5)
    for ob in raw.obstacles[:raw.num_obstacles]:
        c = [F32(v) for v in ob.center]
        ly = p[1] - c[1]
        ddx, ddz = p[0] - c[0], p[2] - c[2]
        r = np.sqrt(ddx * ddx + ddz * ddz)
        top, bot = F32(ob.top_y), F32(ob.bot_y)
        if ob.kind == 0:                                            # truncated cone
            height = top - bot
            if height < F32(1e-10):
                sd = np.full_like(ly, SDF_NO_CONSTRAINT)
            else:
                t = (ly - bot) / height
                cone_r = F32(ob.bot_radius) + (F32(ob.top_radius) - F32(ob.bot_radius)) * t
                sd = np.where((ly > top) | (ly < bot), SDF_NO_CONSTRAINT, cone_r - r)
        else:                                                       # cylinder
            sd = np.where(ly > top, SDF_NO_CONSTRAINT, np.minimum(F32(ob.radius) - r, ly - bot))
        sd = sd - half
        fresh = data >= SDF_NO_CONSTRAINT - F32(1.0)
        data = np.where(fresh, sd, np.maximum(data, sd))
    return data.reshape(-1)


def generate_sdf_class(raw, sdf):
    """generate_sdf_class_data (state.rs:323-344): 1 where the host-side trilinear sample
    (state.rs:285-321, lerps written `a + (b - a) * f`) at the cell centre is below 0."""
    gx, gy, gz = (int(v) for v in raw.grid_dims)
    b = [F32(v) for v in raw.bounds_size]
    dx = b[0] / F32(gx)
    iz, iy, ix = np.meshgrid(np.arange(gz, dtype=np.float32), np.arange(gy, dtype=np.float32),
                             np.arange(gx, dtype=np.float32), indexing="ij")
    cc = [(-b[a] * F32(0.5)) + (c + F32(0.5)) * dx for a, c in enumerate((ix, iy, iz))]
    t = np.asarray(sdf, np.float32).reshape(SDF_RES, SDF_RES, SDF_RES)
    res = F32(SDF_RES)
    uv = [(cc[a] + b[a] * F32(0.5)) / b[a] * res - F32(0.5) for a in range(3)]
    fl = [np.floor(c) for c in uv]
    base = [to_i32(c) for c in fl]
    f = [c - d for c, d in zip(uv, fl)]
    m = SDF_RES - 1

    def ld(dx_, dy, dz):
        return t[np.clip(base[2] + dz, 0, m), np.clip(base[1] + dy, 0, m), np.clip(base[0] + dx_, 0, m)]

    def lerp(a, b_, s):
        return a + (b_ - a) * s

    c00 = lerp(ld(0, 0, 0), ld(1, 0, 0), f[0])
    c10 = lerp(ld(0, 1, 0), ld(1, 1, 0), f[0])
    c01 = lerp(ld(0, 0, 1), ld(1, 0, 1), f[0])
    c11 = lerp(ld(0, 1, 1), ld(1, 1, 1), f[0])
    c0 = lerp(c00, c10, f[1])
    c1 = lerp(c01, c11, f[1])
    return (lerp(c0, c1, f[2]) < F32(0.0)).astype(np.uint8).reshape(-1)


# ---------------------------------------------------------------- inflow emission  (inflow.rs:108-293)

def _normalized(v):
    """Vec3::normalized with the ZERO guards of `/` (crates/sim-core/src/math.rs:41-92)."""
    ln = np.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    if ln <= F32(1e-6):
        return [F32(0.0)] * 3
    return [c / ln for c in v]


def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


class Inflow:
    """InflowState (inflow.rs:68-242): kettle angle -> head -> exit speed and flow rate,
    and the golden-angle disk emission with back-dated ages.  cos/sin of the golden
    angle are evaluated in float64 and rounded (Rust's f32 functions leave the last bit to
    the platform's libm)."""

    def __init__(self, raw, angle_deg):
        self.raw = raw
        self.angle = F32(angle_deg)
        self.accumulator = F32(0.0)
        self.sequence = 0

    def update(self):
        sp, raw = self.raw.spout, self.raw
        a, act, full = self.angle, F32(sp.activation_angle_deg), F32(sp.full_flow_angle_deg)
        if a <= act:
            s = F32(0.0)
        elif a >= full:
            s = F32(1.0)
        else:
            t = (a - act) / (full - act)
            s = t * t * (F32(3.0) - F32(2.0) * t)
        if a <= act:
            head = F32(0.0)
        elif a >= full:
            head = F32(sp.head_at_full_angle)
        else:
            head = F32(sp.head_at_activation) + s * (F32(sp.head_at_full_angle) - F32(sp.head_at_activation))
        cap = F32(sp.gentle_exit_speed) + s * (F32(sp.max_exit_speed) - F32(sp.gentle_exit_speed))
        if head < F32(1e-6):
            speed = F32(0.0)
        else:
            speed = np.minimum(np.sqrt(F32(2.0) * F32(raw.standard_gravity_m_s2) * F32(raw.sim_units_per_meter) * head), cap)
        if speed < F32(1e-6):
            flow = F32(0.0)
        else:
            r = F32(sp.nozzle_radius)
            area = F32(np.pi) * r * r
            flow = np.minimum(F32(sp.discharge_coeff) * area * speed * F32(sp.volume_to_ml), F32(sp.max_flow_rate_ml_s))
        self.exit_speed, self.flow_rate = F32(speed), F32(flow)

    def emit(self, dt, current_total, max_particles):
        """New sample rows (count, 8) of one substep."""
        self.update()
        brew = self.raw.brew
        if self.flow_rate < F32(1e-6):
            self.accumulator = F32(0.0)
            return np.zeros((0, 8), np.float32)
        self.accumulator = self.accumulator + self.flow_rate * F32(brew.water_particles_per_ml) * F32(dt)
        count = int(self.accumulator)
        if count == 0:
            return np.zeros((0, 8), np.float32)
        self.accumulator = self.accumulator - F32(count)
        count = min(count, max(max_particles - current_total, 0))
        if count == 0:
            return np.zeros((0, 8), np.float32)
        sp = self.raw.spout
        d = [F32(c) for c in sp.direction]
        up = [F32(0.0), F32(1.0), F32(0.0)] if abs(d[1]) < F32(0.9) else [F32(1.0), F32(0.0), F32(0.0)]
        t1 = _normalized(_cross(d, up))
        t2 = _normalized(_cross(d, t1))
        vel = [c * self.exit_speed for c in d]
        eo = [F32(sp.origin[q]) + d[q] * F32(0.18) for q in range(3)]
        jet_r = F32(sp.nozzle_radius) * F32(0.58)
        i = np.arange(count, dtype=np.int64)
        sf = ((self.sequence + i) & 0xFFFFFFFF).astype(np.float32)
        x = (sf + F32(0.5)) * F32(0.7548777)
        radial_u = x - np.trunc(x)
        r = jet_r * np.sqrt(radial_u)
        theta = sf * F32(2.399963)
        c, s = np.cos(theta.astype(np.float64)).astype(np.float32), np.sin(theta.astype(np.float64)).astype(np.float32)
        age = ((i.astype(np.float32) + F32(0.5)) / F32(count)) * F32(dt)
        rows = np.zeros((count, 8), np.float32)
        for q in range(3):
            off = t1[q] * r * c + t2[q] * r * s
            rows[:, q] = eo[q] + off - vel[q] * age
            rows[:, 4 + q] = vel[q]
        rows[:, 3] = F32(1.0)
        rows[:, 7] = F32(brew.water_mass_units_per_ml) / F32(brew.water_particles_per_ml)
        self.sequence = (self.sequence + count) & 0xFFFFFFFF
        return rows


# ---------------------------------------------------------------- one whole substep  (mod.rs:271-419)

def substep(raw, sdf_texels, sdf_class, inflow, particles, affine, bed_extract, num_water, num_bed, dt):
    """One substep of the reference configuration (fixed-point pressure, fixed pairs):
    emission, then every dispatch in the order of mod.rs:305-414, with the lanes passed
    from dispatch to dispatch as the shader aliases them.  Returns the sample rows,
    affine rows and bed_extract rows after it, and the new water count."""
    outlet_r = F32(raw.brew.dripper_outlet_radius)
    P = np.array(particles, np.float32).reshape(-1, 8)[:num_water + num_bed]
    A = np.array(affine, np.float32).reshape(-1, 12)[:num_water + num_bed]
    BE = np.array(bed_extract, np.float32).reshape(-1, 8)[:num_bed]
    new = inflow.emit(dt, num_water + num_bed, int(raw.max_particles))
    if new.shape[0]:
        P = np.concatenate([P, new])
        A = np.concatenate([A, np.zeros((new.shape[0], 12), np.float32)])
        num_water += new.shape[0]
    u = Uniforms(raw, num_water, num_bed, dt)
    sdf = Sdf(u, sdf_texels)
    solid = np.asarray(sdf_class).reshape(u.grid_shape()) != 0
    lookup = bed_lookup(u, P, A)
    lanes = p2g(u, P, A)
    gv = boundary_project(u, sdf, grid_update(u, lanes))
    bed = Bed(u, lookup, P, A, BE)
    lanes = classify(u, lanes, gv, bed, sdf, solid, bool(raw.use_sdf_cache))
    lanes = rbgs(u, lanes, int(raw.pressure_rbgs_pairs))
    gv, imp = project(u, lanes, gv, bed)
    gv = boundary_project(u, sdf, gv)
    lanes = packing_prepare(u, lanes)
    gv = boundary_project(u, sdf, packing_apply(u, lanes, gv))
    lanes = viscosity_prepare(u, lanes, gv, solid)
    gv = boundary_project(u, sdf, viscosity_apply(u, lanes, gv))
    P, A, imp_g2p = g2p(u, sdf, bed, outlet_r, P, A, gv)
    imp = imp + imp_g2p
    P, water = bed_coupling(u, Bed(u, lookup, P, A, BE), P, A)
    if num_bed:
        BE = extraction_advect(u, BE, wrap_i32(water))
        Pb, Ab, BE = bed_dynamics(u, sdf, outlet_r, lanes, gv, lookup, P, A, BE, wrap_i32(imp))
        P[:num_bed], A[:num_bed] = Pb, Ab
    return P, A, BE, num_water


# ---------------------------------------------------------------- sample reorder (engine extension)

def reorder_permutation(u, particles, affine, tile=4):
    """The engine's `reorder_every` permutation of the water slots (no reference
    counterpart): each water sample keyed by the tile of its P2G base cell (tiles of
    `tile`^3 over the (g + 1)-node lattice, base index + 1 clamped to the tiles), samples
    that deposit nothing keyed after every tile, then a stable sort.  Returns, for each
    new water slot, the old water slot."""
    nb, nw = u.num_bed, u.num_water
    p = np.asarray(particles, np.float32).reshape(-1, 8)[nb:nb + nw]
    ph = np.asarray(affine, np.float32).reshape(-1, 12)[nb:nb + nw, 3]
    nt = [(g + 1 + tile - 1) // tile for g in (u.gx, u.gy, u.gz)]
    live = (ph < F32(0.5)) & ~(p[:, 7] <= u.inactive)
    t = []
    for q in range(3):
        b = to_i32(np.floor((p[:, q] - u.origin[q]) * u.inv_dx - F32(0.5))).astype(np.int64)
        t.append(np.minimum(np.maximum(b + 1, 0) // tile, nt[q] - 1))
    key = np.where(live, (t[2] * nt[1] + t[1]) * nt[0] + t[0], nt[0] * nt[1] * nt[2])
    return np.argsort(key, kind="stable")


# ---------------------------------------------------------------- FP32 refinement solve (engine extension)

def next_check_interval(r_new, r_old, k, tol, ce):
    """Pairs until the next FP64 residual check: the pairs the last cycle's decay predicts,
    ceil(k log(tol / r_new) / log(r_new / r_old)), at least 2 and at most ce; ce when no
    decay was measured."""
    import math
    if not (r_old > 0.0) or not (r_new > tol) or not (r_new < r_old) or k == 0:
        return ce
    n = math.ceil(k * math.log(tol / r_new) / math.log(r_new / r_old))
    if not (n < ce):
        return ce
    return 2 if n < 2 else int(n)


def refine_solve(u, kind, fill, div, omega, tol, check_every, first_check, max_sweeps):
    """The engine's residual-mode pressure solve from a cold start (no reference
    counterpart; its operator is pressure_update's, shader.rs:1371-1439): the pressure
    kept as two float32 words (hi + lo); each cycle evaluates the FP64 residual
    r = (sum_f w_f p_f - dx^2 rhs) - W p, relaxes the float32 correction d of W d = r
    (over-relaxed red-black sweeps), and adds it back in FP64.  Returns (hi, lo, pairs,
    checks, r0, r1) over all cells."""
    shp = u.grid_shape()
    kind = np.asarray(kind, np.int32).reshape(shp)
    fill = np.asarray(fill, np.float32).reshape(shp)
    div = np.asarray(div, np.float32).reshape(shp)
    fl = np.flatnonzero(is_fluid(kind).reshape(-1))
    iz, iy, ix = np.unravel_index(fl, shp)
    par = ((ix + iy + iz) & 1)[:]
    nbi, w, wf = [], [], []
    for d in FACES:
        x, y, z = ix + d[0], iy + d[1], iz + d[2]
        on = (x >= 0) & (y >= 0) & (z >= 0) & (x < u.gx) & (y < u.gy) & (z < u.gz)
        ni = np.where(on, (np.clip(z, 0, u.gz - 1) * u.gy + np.clip(y, 0, u.gy - 1)) * u.gx + np.clip(x, 0, u.gx - 1), 0)
        nk = np.where(on, kind.reshape(-1)[ni], CELL_SOLID)
        wt = face_weight(kind.reshape(-1)[fl], fill.reshape(-1)[fl], nk, fill.reshape(-1)[ni])
        use = on & (nk != CELL_SOLID) & ~(wt <= F32(0.0))
        nbi.append(ni)
        w.append(np.where(use, wt, F32(0.0)))
        wf.append(use & is_fluid(nk))
    sf = fill.reshape(-1)[fl]
    rhs = div.reshape(-1)[fl] * sf / np.maximum(u.dt, F32(1e-6))
    b = (u.dx * u.dx * rhs).astype(np.float64)
    nc = np.zeros(fl.size, np.float32)
    wsum = np.zeros(fl.size)
    for q in range(6):
        nc = nc + w[q]                      # zero weights add exactly nothing
        wsum = wsum + w[q].astype(np.float64)
    solvable = ~(nc <= F32(0.0))
    hi = np.zeros(u.cells, np.float32)
    lo = np.zeros(u.cells, np.float32)
    pd = np.zeros(u.cells, np.float32)
    omega = F32(omega)

    def residual():
        p = hi.astype(np.float64) + lo.astype(np.float64)
        psum = np.zeros(fl.size)
        for q in range(6):
            psum = psum + np.where(wf[q], w[q].astype(np.float64) * p[nbi[q]], 0.0)
        r = (psum - b) - wsum * p[fl]
        r = np.where(wsum > 0.0, r, 0.0)
        bb = np.where(wsum > 0.0, b, 0.0)
        b2 = float(np.sum(bb * bb))
        return r.astype(np.float32), (0.0 if b2 <= 0.0 else float(np.sqrt(np.sum(r * r)) / np.sqrt(b2)))

    def sweep(parity, g):
        sel = solvable & (par == parity)
        ds = np.zeros(fl.size, np.float32)
        for q in range(6):
            ds = np.where(wf[q], ds + w[q] * pd[nbi[q]], ds)
        dn = (ds + g) * (F32(1.0) / np.where(solvable, nc, F32(1.0)))
        if omega != F32(1.0):
            dn = pd[fl] + omega * (dn - pd[fl])
        pd[fl[sel]] = dn[sel]

    ce = check_every if check_every else 10
    g, r1 = residual()
    r0, checks, sweeps = r1, 1, 0
    nxt = first_check if first_check else ce
    while not (r1 <= tol) and sweeps < max_sweeps:
        k = min(nxt, max_sweeps - sweeps)
        pd[:] = F32(0.0)
        for _ in range(k):
            sweep(0, g)
            sweep(1, g)
        sweeps += k
        p = (hi[fl].astype(np.float64) + lo[fl].astype(np.float64)) + pd[fl].astype(np.float64)
        hi[fl] = p.astype(np.float32)
        lo[fl] = (p - hi[fl].astype(np.float64)).astype(np.float32)
        before = r1
        g, r1 = residual()
        checks += 1
        nxt = next_check_interval(r1, before, k, tol, ce)
    return hi, lo, sweeps, checks, r0, r1


# ---------------------------------------------------------------- bed seeding  (bed.rs:41-314)

def _order_bounds(lo, hi):
    """bed.rs:84-91"""
    if lo <= hi:
        return lo, hi
    mid = (lo + hi) * F32(0.5)
    return mid, mid


def seated_in_filter(filt):
    """BedConfig::seated_in_filter (bed.rs:41-82) of the default BedConfig (bed.rs:20-38)
    in a paper filter: (center_y, top_y, bot_y, top_radius, bot_radius), the y values
    relative to the filter's centre."""
    cy = F32(filt.center[1])
    ftop, fbot = F32(filt.top_y), F32(filt.bot_y)
    thick, hole, frad = F32(filt.thickness), F32(filt.hole_radius), F32(filt.top_radius)

    def radius_at(y):
        height = np.maximum(ftop - fbot, F32(1e-6))
        t = clamp((y - fbot) / height, F32(0.0), F32(1.0))
        return F32(filt.bot_radius) + (frad - F32(filt.bot_radius)) * t

    def inner_at(y):
        return np.maximum(radius_at(y) - thick, hole)

    fbot_abs, ftop_abs = cy + fbot, cy + ftop
    tlo, thi = _order_bounds(fbot_abs + F32(0.6), ftop_abs - F32(0.35))
    top_abs = clamp(cy + F32(0.45), tlo, thi)
    blo, bhi = _order_bounds(fbot_abs + F32(0.4), top_abs - F32(1.4))
    bot_abs = clamp(cy + F32(-2.70), blo, bhi)
    top_y, bot_y = top_abs - cy, bot_abs - cy
    rlo, rhi = _order_bounds(hole + F32(0.8), frad - thick - F32(0.1))
    top_r = clamp(inner_at(top_abs - cy) - F32(0.18), rlo, rhi)
    blo2, bhi2 = _order_bounds(hole + F32(0.14), top_r - F32(0.25))
    bot_r = clamp(inner_at(bot_abs - cy) - F32(0.12), blo2, bhi2)
    return cy, top_y, bot_y, top_r, bot_r


def init_bed(bed, grid_dims, bounds_size):
    """init_bed_particles (bed.rs:107-226) and build_cell_lookup (bed.rs:228-314) for a
    bed whose per-sample permeability is uniform.  Returns (particles (n, 8), affine
    (n, 12), bed_extract (n, 8), lookup (cells,))."""
    import math
    c = [F32(v) for v in bed.center]
    top_y, bot_y = F32(bed.top_y), F32(bed.bot_y)
    top_r, bot_r = F32(bed.top_radius), F32(bed.bot_radius)
    gx, gy, gz = (int(v) for v in grid_dims)
    height = top_y - bot_y
    if height < F32(1e-6):
        return (np.zeros((0, 8), np.float32), np.zeros((0, 12), np.float32), np.zeros((0, 8), np.float32),
                np.full(gx * gy * gz, -1, np.int32))
    avg = (top_r + bot_r) * F32(0.5)
    q = bot_r / avg
    volume = F32(np.pi) * avg * avg * height / F32(3.0) * (F32(1.0) + bot_r / avg + q * q)
    # f32::cbrt leaves the last bit to the platform's libm: evaluated in float64 and
    # rounded (numpy's own float32 cbrt is one ulp off the rounded cube root here)
    spacing = F32(np.cbrt(np.float64(volume / F32(max(int(bed.num_particles), 1)))))
    nx = int(math.ceil(float((top_r * F32(2.0)) / spacing)))
    ny = int(math.ceil(float(height / spacing)))
    nz = nx
    rows, keys = [], []
    for iy in range(ny):
        base_y = c[1] + bot_y + (F32(iy) + F32(0.5)) * spacing
        t = (base_y - (c[1] + bot_y)) / height
        max_r = bot_r + (top_r - bot_r) * t
        ix = np.repeat(np.arange(nx), nz)
        iz = np.tile(np.arange(nz), nx)
        x = c[0] - max_r + (ix.astype(np.float32) + F32(0.5)) * spacing
        z = c[2] - max_r + (iz.astype(np.float32) + F32(0.5)) * spacing
        ddx, ddz = x - c[0], z - c[2]
        r = np.sqrt(ddx * ddx + ddz * ddz)
        keep = ~(r > max_r)
        cap_t = clamp(t / F32(0.16), F32(0.0), F32(1.0))
        radial_t = r / max_r if max_r > F32(1e-6) else np.zeros_like(r)
        one = F32(1.0) - cap_t
        lift = spacing * F32(0.75) * (one * one) * (radial_t * radial_t)
        y = base_y + lift
        for k in np.flatnonzero(keep):
            rows.append((x[k], y[k], z[k]))
            keys.append((int(ix[k]), iy, int(iz[k])))
    n_src = len(rows)
    src = list(range(n_src))
    target = int(bed.num_particles)
    if n_src > target:
        src = [int(min(math.floor(float((F32(o) + F32(0.5)) * F32(n_src) / F32(target))), float(n_src - 1)))
               for o in range(target)]
    P = np.zeros((len(src), 8), np.float32)
    A = np.zeros((len(src), 12), np.float32)
    BE = np.zeros((len(src), 8), np.float32)
    lattice = {}
    for o, i in enumerate(src):
        x, y, z = rows[i]
        P[o] = (x, y, z, 1.0, 0.0, 0.0, 0.0, 1.0)
        A[o] = (0.0, 0.0, 0.0, 1.0, x, y, z, 0.0, y, 0.0, 0.0, 0.0)
        BE[o] = (0.0, bed.initial_porosity, bed.initial_permeability, 0.0, bed.extractable_mass, 0.0, 93.0, 0.0)
        lattice[keys[i]] = o
    # build_cell_lookup
    bs = [F32(v) for v in bounds_size]
    org = [-b * F32(0.5) for b in bs]
    dx = bs[0] / F32(gx)
    bottom = c[1] + bot_y
    look = np.full(gx * gy * gz, -1, np.int32)
    iz_, iy_, ix_ = np.meshgrid(np.arange(gz), np.arange(gy), np.arange(gx), indexing="ij")
    px = org[0] + (ix_.astype(np.float32) + F32(0.5)) * dx
    py = org[1] + (iy_.astype(np.float32) + F32(0.5)) * dx
    pz = org[2] + (iz_.astype(np.float32) + F32(0.5)) * dx
    inside = ~((py < bottom) | (py > c[1] + top_y))
    t = clamp((py - bottom) / height, F32(0.0), F32(1.0))
    mr = bot_r + (top_r - bot_r) * t
    ddx, ddz = px - c[0], pz - c[2]
    inside &= ~(np.sqrt(ddx * ddx + ddz * ddz) > mr)
    for flat in np.flatnonzero(inside.reshape(-1)):
        k3 = np.unravel_index(flat, inside.shape)
        x, y, z, m = px[k3], py[k3], pz[k3], mr[k3]
        gy_ = int(np.rint((y - bottom) / spacing - F32(0.5)))
        gx_ = int(np.rint((x - (c[0] - m)) / spacing - F32(0.5)))
        gz_ = int(np.rint((z - (c[2] - m)) / spacing - F32(0.5)))
        best, best_d2 = -1, F32(np.inf)
        for dy in (-1, 0, 1):
            for dxi in (-1, 0, 1):
                for dzi in (-1, 0, 1):
                    key = (min(max(gx_ + dxi, 0), max(nx - 1, 0)), min(max(gy_ + dy, 0), max(ny - 1, 0)),
                           min(max(gz_ + dzi, 0), max(nz - 1, 0)))
                    if key not in lattice:
                        continue
                    ly = bottom + (F32(key[1]) + F32(0.5)) * spacing
                    lt = clamp((ly - bottom) / height, F32(0.0), F32(1.0))
                    lr = bot_r + (top_r - bot_r) * lt
                    lx = c[0] - lr + (F32(key[0]) + F32(0.5)) * spacing
                    lz = c[2] - lr + (F32(key[2]) + F32(0.5)) * spacing
                    a, b_, e = x - lx, y - ly, z - lz
                    d2 = a * a + b_ * b_ + e * e
                    if d2 < best_d2:
                        best_d2, best = d2, lattice[key]
        look[flat] = best
    return P, A, BE, look


# ---------------------------------------------------------------- presets  (mod.rs:105-177, inflow.rs:27-58, units.rs, brew_config.rs)

def reference_presets():
    """MpmSettings::default_v60 / benchmark_free_stream / benchmark_center_pour as plain
    float32 values, with the units, brew constants and spout defaults they use."""
    brew = dict(bed_porosity=F32(0.40), bed_particle_samples=12000, water_particles_per_ml=F32(320.0),
                water_mass_units_per_ml=F32(80.0), water_sample_radius_dx=F32(0.18), bed_sample_radius_dx=F32(0.62),
                max_flow_rate_ml_s=F32(12.0), initial_kettle_angle_deg=F32(9.0), water_viscosity=F32(1.2),
                water_kinematic_viscosity_m2_s=F32(1.0e-6), min_bed_permeability_m2=F32(1.0e-12),
                bed_absorption_rate=F32(1.6), target_bed_retention_ml=F32(42.0), bed_pore_capacity_scale=F32(1.0),
                bed_pore_overfill_alpha=F32(18.0), bed_surface_void_scale=F32(1.0), dripper_outlet_radius=F32(0.42),
                filter_absorption_rate_s=F32(0.0), bed_compaction_rate=F32(5.5), bed_impact_rate=F32(8.0))
    # brew_config.rs:92-96 kozeny_carman_permeability_m2(450 um, 0.40)
    d = F32(450.0) * F32(1.0e-6)
    phi = brew["bed_porosity"]
    solid = F32(1.0) - phi
    perm = d * d * phi * phi * phi / (F32(180.0) * solid * solid)
    # units.rs:9-33
    upm = (F32(2.75) - F32(-3.02)) / F32(0.10)
    mpu = F32(1.0) / upm
    units = dict(sim_units_per_meter=upm, ml_per_unit3=mpu * mpu * mpu * F32(1000000.0),
                 gravity=-F32(9.80665) * upm, max_velocity=F32(1.5) * upm,
                 gentle=F32(0.12) * upm, high=F32(0.45) * upm)
    bounds = [F32(14.0), F32(20.0), F32(14.0)]
    dx = bounds[0] / F32(80)
    gy = int(np.ceil(bounds[1] / dx))
    # filter.rs:14-26 and the support cone (mod.rs:163-177)
    ftop, fbot, frad = F32(2.75), F32(-3.02), F32(4.10)
    slope = (frad - F32(0.0)) / np.maximum(ftop - fbot, F32(1e-6))
    outlet = brew["dripper_outlet_radius"]
    cone = dict(top_radius=outlet + slope * (F32(3.0) - F32(-3.0)), bot_radius=outlet, top_y=F32(3.0), bot_y=F32(-3.0))

    def spout(origin=None, target=None):
        o = [F32(-3.4), F32(7.3), F32(0.9)]
        dvec = _normalized([F32(0.36), F32(-0.92), F32(-0.12)])
        t = [F32(-0.7), F32(0.4), F32(0.0)]
        if origin is not None:
            o = [F32(v) for v in origin]
        if target is not None:                  # SpoutSettings::aim_at (inflow.rs:50-59)
            t = [F32(v) for v in target]
            delta = [t[q] - o[q] for q in range(3)]
            if np.sqrt(delta[0] * delta[0] + delta[1] * delta[1] + delta[2] * delta[2]) > F32(1e-5):
                dvec = _normalized(delta)
        return dict(origin=o, direction=dvec, target=t, nozzle_radius=F32(0.18), stem_radius=F32(0.24),
                    activation_angle_deg=F32(8.0), full_flow_angle_deg=F32(56.0), head_at_activation=F32(0.04),
                    head_at_full_angle=F32(24.0), discharge_coeff=F32(0.92), volume_to_ml=units["ml_per_unit3"],
                    max_flow_rate_ml_s=brew["max_flow_rate_ml_s"], gentle_exit_speed=units["gentle"],
                    max_exit_speed=units["high"], stem_length=F32(1.9))

    base = dict(bounds_size=bounds, grid_dims=[80, gy, 80], max_particles=220000, substeps=10,
                gravity=units["gravity"], bulk_modulus=F32(900.0), viscosity=brew["water_viscosity"],
                render_radius=dx * F32(0.7), pressure_rbgs_pairs=40, use_sdf_cache=1, cone=cone,
                cup=dict(radius=F32(3.0), top_y=F32(-3.5), bot_y=F32(-8.0)),
                initial_kettle_angle_deg=brew["initial_kettle_angle_deg"], brew=brew, units=units,
                bed_permeability=perm, has_bed=1)
    presets = {"default_v60": dict(base, spout=spout()),
               "benchmark_free_stream": dict(base, has_bed=0, spout=spout((0.0, 6.8, 0.0), (0.0, -6.8, 0.0))),
               "benchmark_center_pour": dict(base, spout=spout((0.0, 7.1, 0.0), (0.0, 0.4, 0.0)))}
    return presets
