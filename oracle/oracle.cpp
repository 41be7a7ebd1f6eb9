// oracle.cpp — CPU restatement of the reference 3D MLS-MPM substep.
//
// TEST INFRASTRUCTURE.  This is the CPU oracle that checks the CUDA engine; only
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.  It is
// never linked into, or called by, the engine library.
//
// Restates crates/sim-wasm/src/mpm_3d/shader.rs (every helper and entry point) in
// the dispatch order of mod.rs:305-414, with the uniform values of mod.rs:569-670,
// emission of inflow.rs:122-242 and initialisation of state.rs / bed.rs.  Paths
// below are relative to crates/sim-wasm/src/mpm_3d/.
//
// Deliberate deviation: bed_dynamics (shader.rs:1991-2238) reads other bed samples'
// positions while they are written in the same dispatch (shader.rs:848 vs 2231), a
// data race.  The oracle (and the engine) read them from a pre-dispatch snapshot
// (Jacobi semantics).
//
// Templated on the arithmetic type: float reproduces the engine bit for bit; double
// is the FP64 reference run that errors are reported against.  OpenMP parallelises
// the loops; integer fixed-point atomics keep the result independent of thread count.
//
// Parity unpinned: the reference runs its step only as WGSL through wgpu (a graphics
// API) from a Rust crate, neither of which can run here, and its tests hold no golden
// vectors for the step.  What pins this restatement: the reference's host-side known
// answers (tests/test_known_answers.py), its scenario tests run on the engine
// (tests/test_physics_gpu.py), and a second restatement of every dispatch written
// independently in numpy (tests/wgsl_numpy.py), which agrees with this one bit for
// bit except for the backend-defined exp of the J update.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/coffee_sim.h"
#include "oracle_math.h"
#include "oracle_scene.h"

namespace orc {

static thread_local std::string g_err;
static int g_precision_bits = 32;

// Refinement-loop check schedule (engine extension, no reference counterpart): after a
// residual check, the pairs still needed are predicted from the decay over the last
// interval, ceil(k * log(tol / r_new) / log(r_new / r_old)); the next check comes after
// that many pairs, at least 2 and at most ce; ce when no decay was measured.
static uint32_t next_check_interval(double r_new, double r_old, uint32_t k, double tol, uint32_t ce) {
    if (!(r_old > 0.0) || !(r_new > tol) || !(r_new < r_old) || k == 0) return ce;
    const double n = std::ceil((double)k * std::log(tol / r_new) / std::log(r_new / r_old));
    if (!(n < (double)ce)) return ce;
    return n < 2.0 ? 2u : (uint32_t)n;
}
static int g_threads = 0;

static int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

enum { CELL_AIR = 0, CELL_SURFACE = 1, CELL_INTERIOR = 2, CELL_BED = 3, CELL_SOLID = 4 };
enum { M_MAX_DIV = 0, M_FLUID = 1, M_DIV_CLAMP = 2, M_P_CLAMP = 3, M_OVERFLOW = 4 };
static const float FP_SCALE = 262144.0f;  // state.rs:13
static const float FP_VALUE_LIMIT = 8192.0f;  // state.rs:18
static const float METRICS_DIV_FP_SCALE = 1024.0f;  // state.rs:28
static const float BED_REACTION_ALPHA = 0.04f;  // shader.rs:76
static const float BED_REACTION_IMPULSE_CAP = 0.012f;  // shader.rs:77

inline void atomic_add_i32(int32_t* p, int32_t v) {
    __atomic_fetch_add(p, v, __ATOMIC_RELAXED);
}
inline void atomic_add_u32(uint32_t* p, uint32_t v) {
    __atomic_fetch_add(p, v, __ATOMIC_RELAXED);
}
inline void atomic_max_i32(int32_t* p, int32_t v) {
    int32_t cur = __atomic_load_n(p, __ATOMIC_RELAXED);
    while (cur < v && !__atomic_compare_exchange_n(p, &cur, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
    }
}
inline void atomic_max_u32(uint32_t* p, uint32_t v) {
    uint32_t cur = __atomic_load_n(p, __ATOMIC_RELAXED);
    while (cur < v && !__atomic_compare_exchange_n(p, &cur, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
    }
}
inline int32_t atomic_xchg_i32(int32_t* p, int32_t v) { return __atomic_exchange_n(p, v, __ATOMIC_RELAXED); }

struct SimBase {
    virtual ~SimBase() {}
    CsSettings settings;
    // host-side counters (mod.rs:179-193)
    uint32_t num_water = 0, num_bed = 0;
    float total_time = 0.0f, frame_emitted_mass = 0.0f, total_emitted_mass = 0.0f;
    uint32_t frame_dropped = 0, total_dropped = 0;
    // InflowState (inflow.rs:69-75)
    float kettle_angle = 0.0f, flow_rate = 0.0f, exit_speed = 0.0f, accumulator = 0.0f;
    uint32_t emission_sequence = 0;
    float flow_override = 0.0f, speed_override = 0.0f;
    CsMetrics metrics_out{};
    virtual int substep(float sub_dt, uint32_t passes) = 0;
    virtual void reset_state() = 0;
    virtual void read(int what, uint32_t first, uint32_t count, void* out) = 0;
    virtual void write(int what, uint32_t first, uint32_t count, const void* in) = 0;
    virtual float sample_sdf_pub(float x, float y, float z) = 0;
};

enum { RD_PART, RD_AFF, RD_BEDX, RD_LANES, RD_GVEL, RD_P, RD_KIND, RD_LOOKUP, RD_DELTA, RD_RENDER, RD_SDF, RD_CLASS, RD_LANES64,
       RD_DIV, RD_FILL };

template <class R>
struct Sim : SimBase {
    typedef v3<R> V;
    // ---- uniforms (mod.rs:569-670), names follow shader.rs:81-134 ----
    struct U {
        uint32_t gx, gy, gz, cells;
        uint32_t num_water, num_bed, max_p;
        bool use_sdf_cache;
        R dt, gravity, dx, inv_dx;
        V origin, bmax;
        R bulk_K, viscosity, nominal_mass, p_vol;
        R fp_scale, inv_fp, vel_cap, outlet_r;
        R sdf_res, friction, restitution, contact_offset;
        R nu_m2s, absorption_rate, max_saturation, min_perm;
        R extraction_rate, compaction_rate, bed_damping, bed_impact;
        R pore_capacity_scale, pore_overfill_alpha;
        R div_clamp, p_clamp, mdiv_scale, mdiv_inv;
        R p_limit;  // pressure limit: p_clamp with fixed-point storage, none with FP32
        R j_alpha, j_expand_alpha, max_rest_frac, surface_void_scale;
        R water_r_dx, bed_r_dx, filter_absorption;
        R omega;
        CsGeometry g;
    } u;

    std::vector<R> part, aff, bedx, render;  // reference AoS layouts
    std::vector<int32_t> grid;                // 6 lanes
    std::vector<int64_t> grid64;              // 6 lanes, i64 * 2^32 (int64 P2G mode)
    std::vector<R> gvel;                      // 4 per cell
    std::vector<R> pf, divf;                  // FP32-storage pressure/divergence
    std::vector<R> plo, pd, gres;             // refinement: pressure low part, correction, residual
    std::vector<int32_t> lookup, delta;
    uint32_t metrics[8];
    std::vector<float> sdf;
    std::vector<uint8_t> sdf_class;
    std::vector<int32_t> init_lookup;
    size_t cells = 0;
    bool have_prev_p = false;
    uint64_t substeps_done = 0;  // substeps since creation (the reorder schedule)

    explicit Sim(const CsSettings& s) {
        settings = s;
        cells = (size_t)s.grid_dims[0] * s.grid_dims[1] * s.grid_dims[2];
        size_t mp = s.max_particles;
        part.assign(mp * 8, R(0));
        aff.assign(mp * 12, R(0));
        bedx.assign(mp * 8, R(0));
        render.assign(mp * 8, R(0));
        grid.assign(cells * 6, 0);
        grid64.assign(settings.p2g_mode == CS_P2G_INT64 ? cells * 6 : 0, 0);
        gvel.assign(cells * 4, R(0));
        pf.assign(cells, R(0));
        divf.assign(cells, R(0));
        plo.assign(cells, R(0));
        pd.assign(cells, R(0));
        gres.assign(cells, R(0));
        lookup.assign(cells, -1);
        delta.assign(mp * 4, 0);
        std::memset(metrics, 0, sizeof(metrics));
        sdf = generate_sdf(s);
        sdf_class = generate_sdf_class(s, sdf);
        reset_state();
        write_uniforms(R(0));
    }

    // mod.rs:222-262 (init_bed) and mod.rs:432-446 (reset)
    void reset_state() override {
        num_water = num_bed = 0;
        total_time = frame_emitted_mass = total_emitted_mass = 0.0f;
        frame_dropped = total_dropped = 0;
        kettle_angle = settings.initial_kettle_angle_deg;
        flow_rate = exit_speed = accumulator = 0.0f;
        emission_sequence = 0;
        std::fill(part.begin(), part.end(), R(0));
        std::fill(aff.begin(), aff.end(), R(0));
        std::fill(bedx.begin(), bedx.end(), R(0));
        std::fill(render.begin(), render.end(), R(0));
        std::fill(grid.begin(), grid.end(), 0);
        std::fill(grid64.begin(), grid64.end(), 0);
        std::fill(gvel.begin(), gvel.end(), R(0));
        std::fill(pf.begin(), pf.end(), R(0));
        std::fill(divf.begin(), divf.end(), R(0));
        std::fill(plo.begin(), plo.end(), R(0));
        std::fill(pd.begin(), pd.end(), R(0));
        std::fill(gres.begin(), gres.end(), R(0));
        std::fill(lookup.begin(), lookup.end(), -1);
        std::fill(delta.begin(), delta.end(), 0);
        have_prev_p = false;
        substeps_done = 0;
        if (!settings.has_bed) return;
        BedInit bi = init_bed(settings.bed, settings.grid_dims, settings.bounds_size);
        uint32_t n = (uint32_t)(bi.particles.size() / 8);
        if (n == 0) return;
        if (n > settings.max_particles) n = settings.max_particles;
        num_bed = n;
        for (size_t i = 0; i < (size_t)n * 8; ++i) part[i] = R(bi.particles[i]);
        for (size_t i = 0; i < (size_t)n * 12; ++i) aff[i] = R(bi.affines[i]);
        for (size_t i = 0; i < (size_t)n * 8; ++i) bedx[i] = R(bi.extracts[i]);
        for (size_t c = 0; c < cells; ++c) lookup[c] = bi.lookup[c];
    }

    void write_uniforms(R dt) {
        const CsSettings& s = settings;
        u.gx = s.grid_dims[0]; u.gy = s.grid_dims[1]; u.gz = s.grid_dims[2];
        u.cells = u.gx * u.gy * u.gz;
        u.num_water = num_water; u.num_bed = num_bed; u.max_p = s.max_particles;
        u.use_sdf_cache = s.use_sdf_cache != 0;
        float dxf = s.bounds_size[0] / (float)u.gx;
        float inv_dxf = 1.0f / dxf;
        u.dt = dt; u.gravity = R(s.gravity); u.dx = R(dxf); u.inv_dx = R(inv_dxf);
        u.origin = V3<R>(R(-s.bounds_size[0] * 0.5f), R(-s.bounds_size[1] * 0.5f), R(-s.bounds_size[2] * 0.5f));
        u.bmax = V3<R>(R(s.bounds_size[0] * 0.5f), R(s.bounds_size[1] * 0.5f), R(s.bounds_size[2] * 0.5f));
        float nominal = s.brew.water_mass_units_per_ml / s.brew.water_particles_per_ml;
        float pvol = dxf * dxf * dxf * s.particle_volume_cells;
        float bed_cap = num_bed > 0 ? s.brew.target_bed_retention_ml * s.brew.water_mass_units_per_ml / (float)num_bed
                                    : 0.7f;
        float phys_div = 4.0f * s.max_velocity * inv_dxf;
        float div_clamp = std::fmin(phys_div, FP_VALUE_LIMIT - 1.0f);
        u.bulk_K = R(s.bulk_modulus); u.viscosity = R(s.viscosity); u.nominal_mass = R(nominal); u.p_vol = R(pvol);
        u.fp_scale = R(FP_SCALE); u.inv_fp = R(1.0f / FP_SCALE); u.vel_cap = R(s.max_velocity);
        u.outlet_r = R(s.brew.dripper_outlet_radius);
        u.sdf_res = R(128.0f); u.friction = R(s.geom.sdf_friction); u.restitution = R(s.geom.sdf_restitution);
        u.contact_offset = R(s.geom.contact_offset);
        u.nu_m2s = R(s.brew.water_kinematic_viscosity_m2_s); u.absorption_rate = R(s.brew.bed_absorption_rate);
        u.max_saturation = R(bed_cap); u.min_perm = R(s.brew.min_bed_permeability_m2);
        u.extraction_rate = R(0.01f); u.compaction_rate = R(s.brew.bed_compaction_rate);
        u.bed_damping = R(8.5f); u.bed_impact = R(s.brew.bed_impact_rate);
        u.pore_capacity_scale = R(s.brew.bed_pore_capacity_scale); u.pore_overfill_alpha = R(s.brew.bed_pore_overfill_alpha);
        u.div_clamp = R(div_clamp); u.p_clamp = R(FP_VALUE_LIMIT - 1.0f);
        u.p_limit = s.pressure_storage == CS_PRESSURE_FIXED_POINT ? u.p_clamp : R(3.0e38f);
        u.mdiv_scale = R(METRICS_DIV_FP_SCALE); u.mdiv_inv = R(1.0f / METRICS_DIV_FP_SCALE);
        u.j_alpha = R(32.0f); u.j_expand_alpha = R(2.0f); u.max_rest_frac = R(1.20f);
        u.surface_void_scale = R(s.brew.bed_surface_void_scale);
        u.water_r_dx = R(s.brew.water_sample_radius_dx); u.bed_r_dx = R(s.brew.bed_sample_radius_dx);
        u.filter_absorption = R(s.brew.filter_absorption_rate_s);
        u.g = s.geom;
        u.omega = (s.rbgs_omega > 0.0f) ? R(s.rbgs_omega) : R(1);
    }

    // ---- shader.rs:81-171 helpers ----
    uint32_t num_particles() const { return u.num_water + u.num_bed; }
    R dripper_top_radius() const { return u.outlet_r + R(u.g.cone_radius_span); }
    R wall_half() const { return R(u.g.wall_thickness) * R(0.5); }
    R cup_floor_y() const { return R(u.g.cup_floor_y) + wall_half() + u.contact_offset; }
    R water_particle_radius() const { return u.dx * u.water_r_dx; }
    R bed_particle_radius() const { return u.dx * u.bed_r_dx; }
    R inactive_mass_threshold() const { return u.nominal_mass * R(0.10); }
    R occupancy_threshold() const { return u.nominal_mass * R(0.1); }
    R viscosity_support_threshold() const { return u.nominal_mass * R(2.0); }
    static R clamp_j(R v) { return wclamp(v, R(0.40), R(2.00)); }
    uint32_t cell_index(uint32_t ix, uint32_t iy, uint32_t iz) const { return iz * u.gx * u.gy + iy * u.gx + ix; }
    bool in_grid(int x, int y, int z) const {
        return x >= 0 && y >= 0 && z >= 0 && (uint32_t)x < u.gx && (uint32_t)y < u.gy && (uint32_t)z < u.gz;
    }
    // shader.rs:136-146
    R filter_top_y() const { return R(u.g.filter_center_y) + R(u.g.filter_top_rel); }
    R filter_bot_y() const { return R(u.g.filter_center_y) - R(u.g.filter_bot_rel); }
    R coffee_filter_floor_y() const {
        R ftop = filter_top_y(), fbot = filter_bot_y();
        R bco = wmax(u.contact_offset, bed_particle_radius());
        R fh = wmax(ftop - fbot, R(1e-6));
        R slope = R(u.g.filter_top_radius) / fh;
        return fbot + (bco + R(u.g.filter_thickness)) / wmax(slope, R(1e-6));
    }

    int32_t* lane(int l) { return &grid[(size_t)l * u.cells]; }
    bool fixed_point() const { return settings.pressure_storage == CS_PRESSURE_FIXED_POINT; }
    int32_t kind_load(uint32_t c) { return lane(3)[c]; }
    // shader.rs:198-209
    R pressure_load(uint32_t c) {
        if (fixed_point()) return R(lane(0)[c]) * u.inv_fp;
        return pf[c];
    }
    void pressure_store(uint32_t c, R v) {
        R lim = u.p_limit;
        R cl = wclamp(v, -lim, lim);
        if (cl != v) atomic_add_u32(&metrics[M_P_CLAMP], 1u);
        if (fixed_point()) lane(0)[c] = to_i32(cl * u.fp_scale);
        else pf[c] = cl;
    }
    // shader.rs:211-222
    R packing_load(uint32_t c) { return R(lane(2)[c]) * u.inv_fp; }
    void packing_store(uint32_t c, R v) {
        R lim = u.p_clamp;
        R cl = wclamp(v, R(0), lim);
        if (cl != v) atomic_add_u32(&metrics[M_P_CLAMP], 1u);
        lane(2)[c] = to_i32(cl * u.fp_scale);
    }
    // shader.rs:262-264, 352-359
    R div_load(uint32_t c) {
        if (fixed_point()) return R(lane(1)[c]) * u.inv_fp;
        return divf[c];
    }
    void div_store(uint32_t c, R v) {
        R lim = u.div_clamp;
        R cl = wclamp(v, -lim, lim);
        if (cl != v) atomic_add_u32(&metrics[M_DIV_CLAMP], 1u);
        if (fixed_point()) lane(1)[c] = to_i32(cl * u.fp_scale);
        else divf[c] = cl;
    }
    // shader.rs:266-283
    V vscratch_load(uint32_t c) {
        return V3<R>(R(lane(1)[c]) * u.inv_fp, R(lane(2)[c]) * u.inv_fp, R(lane(3)[c]) * u.inv_fp);
    }
    void vscratch_store(uint32_t c, V v) {
        V cl = v;
        R speed = length(cl);
        if (speed > u.vel_cap) cl = cl * (u.vel_cap / speed);
        lane(1)[c] = to_i32(cl.x * u.fp_scale);
        lane(2)[c] = to_i32(cl.y * u.fp_scale);
        lane(3)[c] = to_i32(cl.z * u.fp_scale);
    }
    // P2G lanes 0-5: i32 * 2^18, or i64 * 2^32 in the int64 mode
    bool int64_grid() const { return settings.p2g_mode == CS_P2G_INT64; }
    R p2g_lane(int l, uint32_t c) {
        if (int64_grid()) return R((float)grid64[(size_t)l * cells + c]) * R(1.0f / 4294967296.0f);
        return R(lane(l)[c]) * u.inv_fp;
    }
    R rest_vol(uint32_t c) { return p2g_lane(4, c); }
    R cur_vol(uint32_t c) { return p2g_lane(5, c); }
    static bool is_fluid(int32_t k) { return k == CELL_INTERIOR || k == CELL_SURFACE || k == CELL_BED; }
    static bool is_solid(int32_t k) { return k == CELL_SOLID; }
    static bool is_water_phase(R ph) { return ph < R(0.5); }
    static bool is_suspended(R ph) { return ph >= R(1.5); }

    // shader.rs:224-236 (pressure_or_mirror): the kind read is lane 3 whatever it holds
    R pressure_or_mirror(int x, int y, int z, R mirror) {
        if (!in_grid(x, y, z)) return mirror;
        uint32_t ci = cell_index(x, y, z);
        if (is_solid(kind_load(ci))) return mirror;
        return pressure_load(ci);
    }
    // shader.rs:238-260
    V pressure_gradient_at_cell(int x, int y, int z) {
        if (!in_grid(x, y, z)) return V3<R>(0, 0, 0);
        uint32_t idx = cell_index(x, y, z);
        R ph = pressure_load(idx);
        R pxm = pressure_or_mirror(x - 1, y, z, ph), pxp = pressure_or_mirror(x + 1, y, z, ph);
        R pym = pressure_or_mirror(x, y - 1, z, ph), pyp = pressure_or_mirror(x, y + 1, z, ph);
        R pzm = pressure_or_mirror(x, y, z - 1, ph), pzp = pressure_or_mirror(x, y, z + 1, ph);
        R h = R(0.5) * u.inv_dx;
        return V3<R>(h * (pxp - pxm), h * (pyp - pym), h * (pzp - pzm));
    }
    // shader.rs:293-304
    R liquid_fill(uint32_t c, int32_t kind) {
        if (kind == CELL_INTERIOR || kind == CELL_BED) return R(1);
        if (kind != CELL_SURFACE) return R(0);
        R cv = wmax(u.dx * u.dx * u.dx, R(1e-8));
        R frac = wmax(rest_vol(c), cur_vol(c)) / cv;
        return wclamp(frac, R(0), R(1));
    }
    // shader.rs:306-323
    R face_weight(int32_t self_kind, R self_fill, uint32_t nc, int32_t nk) {
        if (is_solid(nk)) return R(0);
        if (self_kind == CELL_BED || nk == CELL_BED) return R(1);
        if (!is_fluid(nk)) return self_fill;
        return wmin(self_fill, liquid_fill(nc, nk));
    }
    // shader.rs:325-350
    R pressure_weighted_or_mirror(int x, int y, int z, R mirror, int32_t sk, R sf) {
        if (!in_grid(x, y, z)) return mirror;
        uint32_t ci = cell_index(x, y, z);
        int32_t k = kind_load(ci);
        if (is_solid(k)) return mirror;
        R np = R(0);
        if (is_fluid(k)) np = pressure_load(ci);
        R w = face_weight(sk, sf, ci, k);
        return mix(mirror, np, w);
    }
    // shader.rs:361-378
    int32_t lookup_load(uint32_t c) { return lookup[c]; }
    bool valid_bed_solid(int32_t b) {
        if (b < 0 || (uint32_t)b >= u.num_bed) return false;
        return !is_water_phase(aff[(size_t)b * 12 + 3]);
    }
    V pvel(uint32_t p) { return V3<R>(part[(size_t)p * 8 + 4], part[(size_t)p * 8 + 5], part[(size_t)p * 8 + 6]); }
    V ppos(uint32_t p) { return V3<R>(part[(size_t)p * 8 + 0], part[(size_t)p * 8 + 1], part[(size_t)p * 8 + 2]); }
    // shader.rs:380-407
    V bed_matrix_velocity_cell(int x, int y, int z) {
        V sum = V3<R>(0, 0, 0);
        R ws = R(0);
        for (int di = -1; di <= 1; ++di)
            for (int dj = -1; dj <= 1; ++dj)
                for (int dk = -1; dk <= 1; ++dk) {
                    int cx = x + di, cy = y + dj, cz = z + dk;
                    if (!in_grid(cx, cy, cz)) continue;
                    int32_t b = lookup_load(cell_index(cx, cy, cz));
                    if (!valid_bed_solid(b)) continue;
                    sum += pvel(b);
                    ws += R(1);
                }
        if (ws <= R(0)) return V3<R>(0, 0, 0);
        return sum / ws;
    }
    // shader.rs:409-427
    V bed_velocity_load_cell(int x, int y, int z) {
        if (!in_grid(x, y, z)) return V3<R>(0, 0, 0);
        return bed_matrix_velocity_cell(x, y, z);
    }
    R bed_velocity_divergence(int x, int y, int z) {
        R vxm = bed_velocity_load_cell(x - 1, y, z).x, vxp = bed_velocity_load_cell(x + 1, y, z).x;
        R vym = bed_velocity_load_cell(x, y - 1, z).y, vyp = bed_velocity_load_cell(x, y + 1, z).y;
        R vzm = bed_velocity_load_cell(x, y, z - 1).z, vzp = bed_velocity_load_cell(x, y, z + 1).z;
        return R(0.5) * u.inv_dx * (((vxp - vxm) + (vyp - vym)) + (vzp - vzm));
    }
    // shader.rs:429-449
    static R kozeny_factor(R phi_in) {
        R phi = wclamp(phi_in, R(0.08), R(0.82));
        R solid = wmax(R(1) - phi, R(1e-4));
        return (phi * phi * phi) / (solid * solid);
    }
    R bed_compacted_porosity(uint32_t b) {
        R base = wclamp(bedx[(size_t)b * 8 + 1], R(0.18), R(0.70));
        R comp = wclamp(bedx[(size_t)b * 8 + 3], R(0), R(2.25));
        return wclamp(base - comp * R(0.12), R(0.16), base);
    }
    R bed_compacted_permeability(uint32_t b) {
        R base = wclamp(bedx[(size_t)b * 8 + 1], R(0.18), R(0.70));
        R cp = bed_compacted_porosity(b);
        R ratio = kozeny_factor(cp) / wmax(kozeny_factor(base), R(1e-8));
        return wmax(bedx[(size_t)b * 8 + 2] * ratio, u.min_perm);
    }
    // shader.rs:451-522
    int32_t* delta_lane(int l) { return &delta[(size_t)l * u.max_p]; }
    void bed_water_delta_add(uint32_t b, R amount) {
        if (amount <= R(0)) return;
        atomic_add_i32(&delta_lane(0)[b], to_i32(amount * u.fp_scale));
    }
    void bed_impulse_delta_add(uint32_t b, V imp) {
        R cap = u.nominal_mass * u.vel_cap * R(BED_REACTION_IMPULSE_CAP);
        V cl = V3<R>(wclamp(imp.x, -cap, cap), wclamp(imp.y, -cap, cap), wclamp(imp.z, -cap, cap));
        atomic_add_i32(&delta_lane(1)[b], to_i32(cl.x * u.fp_scale));
        atomic_add_i32(&delta_lane(2)[b], to_i32(cl.y * u.fp_scale));
        atomic_add_i32(&delta_lane(3)[b], to_i32(cl.z * u.fp_scale));
    }
    void bed_impulse_neighborhood(int x, int y, int z, V imp) {
        R count = R(0);
        for (int di = -1; di <= 1; ++di)
            for (int dj = -1; dj <= 1; ++dj)
                for (int dk = -1; dk <= 1; ++dk) {
                    int cx = x + di, cy = y + dj, cz = z + dk;
                    if (!in_grid(cx, cy, cz)) continue;
                    if (valid_bed_solid(lookup_load(cell_index(cx, cy, cz)))) count += R(1);
                }
        if (count <= R(0)) return;
        V share = imp / count;
        for (int di = -1; di <= 1; ++di)
            for (int dj = -1; dj <= 1; ++dj)
                for (int dk = -1; dk <= 1; ++dk) {
                    int cx = x + di, cy = y + dj, cz = z + dk;
                    if (!in_grid(cx, cy, cz)) continue;
                    int32_t b = lookup_load(cell_index(cx, cy, cz));
                    if (valid_bed_solid(b)) bed_impulse_delta_add((uint32_t)b, share);
                }
    }
    V bed_impulse_exchange(uint32_t b) {
        int32_t ix = atomic_xchg_i32(&delta_lane(1)[b], 0);
        int32_t iy = atomic_xchg_i32(&delta_lane(2)[b], 0);
        int32_t iz = atomic_xchg_i32(&delta_lane(3)[b], 0);
        return V3<R>(R(ix), R(iy), R(iz)) * u.inv_fp;
    }
    // shader.rs:524-576
    void deposit_absorbed(int hx, int hy, int hz, int32_t home, R absorbed) {
        R ns = absorbed * R(0.35);
        R hs = absorbed - ns;
        bed_water_delta_add((uint32_t)home, hs);
        static const int off[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
        int32_t ids[6];
        uint32_t n = 0;
        for (int i = 0; i < 6; ++i) {
            int cx = hx + off[i][0], cy = hy + off[i][1], cz = hz + off[i][2];
            if (!in_grid(cx, cy, cz)) continue;
            int32_t nid = lookup_load(cell_index(cx, cy, cz));
            if (nid < 0 || nid == home || (uint32_t)nid >= u.num_bed) continue;
            bool dup = false;
            for (uint32_t j = 0; j < n; ++j)
                if (ids[j] == nid) dup = true;
            if (!dup) ids[n++] = nid;
        }
        if (n == 0) {
            bed_water_delta_add((uint32_t)home, ns);
            return;
        }
        R each = ns / R(n);
        for (uint32_t i = 0; i < n; ++i) bed_water_delta_add((uint32_t)ids[i], each);
    }
    bool class_solid(int x, int y, int z) { return sdf_class[cell_index(x, y, z)] != 0; }
    // shader.rs:597-619
    R volume_target(R rest, R cur) {
        R cv = u.dx * u.dx * u.dx;
        R eps = wmax(cv * R(1e-5), u.p_vol * R(1e-3));
        if (rest <= eps) return R(0);
        R j = cur / rest;
        R ce = wclamp(R(1) - j, R(0), R(0.75));
        R ee = wclamp(j - R(1), R(0), R(0.75));
        R t = ce * u.j_alpha - ee * u.j_expand_alpha;
        R packed = wmax(rest, cur) / wmax(cv, R(1e-8));
        R over = wmax(packed - u.max_rest_frac, R(0));
        return wmax(t, over * u.j_alpha);
    }
    // shader.rs:621-666
    R bed_pore_target(uint32_t b, V cc, R rest, R cur) {
        R t = volume_target(rest, cur);
        R cv = u.dx * u.dx * u.dx;
        R porosity = bed_compacted_porosity(b);
        R sat = wclamp(bedx[(size_t)b * 8 + 7], R(0), R(1));
        R comp = wclamp(bedx[(size_t)b * 8 + 3], R(0), R(2.25));
        R bcy = part[(size_t)b * 8 + 1];
        R st = smoothstep(R(-0.25), R(0.75), (cc.y - bcy) * u.inv_dx);
        R open = wclamp((R(1) - R(0.65) * sat) * (R(1) - R(0.12) * comp), R(0.20), R(1));
        R sopen = st * wclamp(u.surface_void_scale, R(0), R(1)) * open;
        R sporo = wmin(porosity + R(0.35), R(0.82));
        R eff = mix(porosity, sporo, sopen);
        R occ = mix(R(1), R(0.35), sopen);
        R satcap = mix(R(1), R(0.32), sat);
        R compcap = mix(R(1), R(0.58), wclamp(comp / R(1.5), R(0), R(1)));
        R cap = eff * cv * wmax(u.pore_capacity_scale, R(0)) * satcap * compcap;
        R over = wmax(cur - cap, R(0)) / wmax(cv, R(1e-8));
        R resp = u.pore_overfill_alpha * occ * mix(R(1), R(1.45), sat);
        return wmax(t, over * resp);
    }
    // shader.rs:668-671
    void world_to_cell(V p, int& x, int& y, int& z) {
        V gp = (p - u.origin) * u.inv_dx;
        x = (int)std::floor(gp.x);
        y = (int)std::floor(gp.y);
        z = (int)std::floor(gp.z);
    }
    // shader.rs:673-699
    R sdf_texel(int x, int y, int z) {
        int mx = (int)u.sdf_res - 1;
        x = std::min(std::max(x, 0), mx);
        y = std::min(std::max(y, 0), mx);
        z = std::min(std::max(z, 0), mx);
        return R(sdf[(size_t)z * SDF_RES * SDF_RES + (size_t)y * SDF_RES + x]);
    }
    R sample_sdf(V p) {
        V bs = u.bmax * R(2);
        R res = u.sdf_res;
        V uv = V3<R>((p.x + u.bmax.x) / bs.x * res - R(0.5), (p.y + u.bmax.y) / bs.y * res - R(0.5),
                     (p.z + u.bmax.z) / bs.z * res - R(0.5));
        int bx = (int)std::floor(uv.x), by = (int)std::floor(uv.y), bz = (int)std::floor(uv.z);
        R fx = wfract(uv.x), fy = wfract(uv.y), fz = wfract(uv.z);
        R c000 = sdf_texel(bx, by, bz), c100 = sdf_texel(bx + 1, by, bz);
        R c010 = sdf_texel(bx, by + 1, bz), c110 = sdf_texel(bx + 1, by + 1, bz);
        R c001 = sdf_texel(bx, by, bz + 1), c101 = sdf_texel(bx + 1, by, bz + 1);
        R c011 = sdf_texel(bx, by + 1, bz + 1), c111 = sdf_texel(bx + 1, by + 1, bz + 1);
        R c00 = mix(c000, c100, fx), c10 = mix(c010, c110, fx);
        R c01 = mix(c001, c101, fx), c11 = mix(c011, c111, fx);
        R c0 = mix(c00, c10, fy), c1 = mix(c01, c11, fy);
        return mix(c0, c1, fz);
    }
    float sample_sdf_pub(float x, float y, float z) override { return (float)sample_sdf(V3<R>(R(x), R(y), R(z))); }
    // shader.rs:701-715
    V sdf_gradient(V p) {
        R e = u.dx;
        R gx = sample_sdf(p + V3<R>(e, 0, 0)) - sample_sdf(p - V3<R>(e, 0, 0));
        R gy = sample_sdf(p + V3<R>(0, e, 0)) - sample_sdf(p - V3<R>(0, e, 0));
        R gz = sample_sdf(p + V3<R>(0, 0, e)) - sample_sdf(p - V3<R>(0, 0, e));
        V g = V3<R>(gx, gy, gz);
        R len = length(g);
        if (len < R(1e-8)) return V3<R>(0, 0, 0);
        return g / len;
    }
    // shader.rs:717-742
    void radial_barrier(V& pos, V& vel, R cx, R cz, R max_r) {
        v2<R> radial{pos.x - cx, pos.z - cz};
        R r = length2(radial);
        if (r > max_r && r > R(1e-6)) {
            v2<R> out{radial.x / r, radial.y / r};
            pos.x = cx + out.x * max_r;
            pos.z = cz + out.y * max_r;
            R vn = dot2(v2<R>{vel.x, vel.z}, out);
            if (vn > R(0)) {
                v2<R> tan{vel.x - out.x * vn, vel.z - out.y * vn};
                vel.x = tan.x * (R(1) - u.friction * R(0.35));
                vel.z = tan.y * (R(1) - u.friction * R(0.35));
            }
        }
    }
    // shader.rs:744-823
    void scene_obstacles(V& pos, V& vel, bool is_bed) {
        if (u.g.flags & CS_GEOM_CONE) {
            R ctop = R(u.g.cone_top_y), cbot = R(u.g.cone_bot_y);
            if (pos.y <= ctop && pos.y >= cbot) {
                R t = wclamp((pos.y - cbot) / (ctop - cbot), R(0), R(1));
                R cr = mix(u.outlet_r, dripper_top_radius(), t) - u.contact_offset;
                radial_barrier(pos, vel, R(0), R(0), cr);
            }
        }
        if ((u.g.flags & CS_GEOM_FILTER) && is_bed) {
            R ftop = filter_top_y(), fbot = filter_bot_y();
            R ftr = R(u.g.filter_top_radius), fth = R(u.g.filter_thickness);
            R bco = wmax(u.contact_offset, bed_particle_radius());
            R floor_y = coffee_filter_floor_y();
            if (pos.y <= ftop && pos.y >= fbot) {
                R ft = wclamp((pos.y - fbot) / (ftop - fbot), R(0), R(1));
                R outer = mix(R(0), ftr, ft);
                R fr = wmax(outer - fth, R(0)) - bco;
                radial_barrier(pos, vel, R(0), R(0), wmax(fr, R(0)));
            }
            if (pos.y <= floor_y) {
                pos.y = floor_y;
                pos.x = R(0);
                pos.z = R(0);
                if (vel.y < R(0)) {
                    vel.y = R(0);
                    vel.x *= R(1) - u.friction * R(0.55);
                    vel.z *= R(1) - u.friction * R(0.55);
                }
                vel.x *= R(1) - u.friction * R(0.55);
                vel.z *= R(1) - u.friction * R(0.55);
            }
        }
        if (u.g.flags & CS_GEOM_CUP) {
            if (pos.y <= R(u.g.cup_top_y)) {
                R cr = R(u.g.cup_radius) - wall_half() - u.contact_offset;
                radial_barrier(pos, vel, R(0), R(0), cr);
                R fy = cup_floor_y();
                if (pos.y < fy) {
                    pos.y = fy;
                    if (vel.y < R(0)) {
                        vel.y = R(0);
                        vel.x *= R(1) - u.friction * R(0.55);
                        vel.z *= R(1) - u.friction * R(0.55);
                    }
                }
            }
        }
    }
    // shader.rs:825-877 (other bed positions come from the pre-dispatch snapshot)
    void coffee_packing(V& pos, V& vel, uint32_t self_bid, const std::vector<R>& snap) {
        V cd = V3<R>(0, 0, 0);
        R cdist = R(1e9);
        bool found = false;
        int cx, cy, cz;
        world_to_cell(pos, cx, cy, cz);
        for (int di = -1; di <= 1; ++di)
            for (int dj = -1; dj <= 1; ++dj)
                for (int dk = -1; dk <= 1; ++dk) {
                    int x = cx + di, y = cy + dj, z = cz + dk;
                    if (!in_grid(x, y, z)) continue;
                    int32_t o = lookup_load(cell_index(x, y, z));
                    if (o < 0 || (uint32_t)o == self_bid || (uint32_t)o >= u.num_bed) continue;
                    V op = V3<R>(snap[(size_t)o * 3], snap[(size_t)o * 3 + 1], snap[(size_t)o * 3 + 2]);
                    V d = pos - op;
                    R dist = length(d);
                    if (dist < cdist) {
                        cdist = dist;
                        cd = d;
                        found = true;
                    }
                }
        R min_sep = bed_particle_radius() * R(1.78);
        if (found && cdist < min_sep) {
            V n = V3<R>(0, 1, 0);
            if (cdist > R(1e-5)) n = cd / cdist;
            R pen = min_sep - cdist;
            pos += n * wmin(pen * R(0.65), u.dx * R(0.22));
            R vn = dot(vel, n);
            if (vn < R(0)) vel -= n * vn;
        }
    }
    // shader.rs:879-903
    void sdf_contact(V& pos, V& vel, bool is_bed) {
        R sv = sample_sdf(pos);
        if (sv < u.contact_offset) {
            V n = sdf_gradient(pos);
            if (length(n) > R(1e-6)) {
                pos += n * (u.contact_offset - sv);
                R vn = dot(vel, n);
                if (vn < R(0)) {
                    vel = vel - n * vn * (R(1) + u.restitution);
                    V vt = vel - n * dot(vel, n);
                    R vtl = length(vt);
                    if (vtl > R(1e-6)) {
                        R fi = wmin(u.friction * std::fabs(vn), vtl);
                        vel = vel - vt * (fi / vtl);
                    }
                }
            }
        }
        scene_obstacles(pos, vel, is_bed);
    }
    // shader.rs:905-935
    R filter_paper_weight(V p) {
        R ftop = filter_top_y(), fbot = filter_bot_y();
        R ftr = R(u.g.filter_top_radius), fth = R(u.g.filter_thickness);
        R pr = wmax(water_particle_radius(), u.dx * R(0.35));
        if (p.y < fbot - pr || p.y > ftop + pr) return R(0);
        R ft = wclamp((p.y - fbot) / (ftop - fbot), R(0), R(1));
        R outer = mix(R(0), ftr, ft);
        R inner = wmax(outer - fth, R(0));
        R r = length2(v2<R>{p.x, p.z});
        R sd = std::fabs(r - inner);
        R sw = R(1) - smoothstep(pr, pr * R(3), sd);
        R dy = p.y - fbot;
        R lv = R(1) - smoothstep(R(0), pr * R(5), wmax(dy, R(0)));
        R lr = R(1) - smoothstep(inner, inner + pr * R(3), r);
        R lw = lv * lr;
        return wclamp(wmax(sw, lw), R(0), R(1));
    }

    static void weights(R f, R w[3]) {
        w[0] = R(0.5) * (R(1.5) - f) * (R(1.5) - f);
        w[1] = R(0.75) - (f - R(1)) * (f - R(1));
        w[2] = R(0.5) * (f - R(0.5)) * (f - R(0.5));
    }

    // ================= kernels =================
    void k_metrics_clear() { std::memset(metrics, 0, sizeof(metrics)); }
    void k_bed_lookup_clear() {
        for (size_t c = 0; c < cells; ++c) lookup[c] = -1;
    }
    // shader.rs:2305-2335
    void k_bed_lookup_scatter() {
        int nb = (int)u.num_bed;
#pragma omp parallel for schedule(static)
        for (int b = 0; b < nb; ++b) {
            if (is_water_phase(aff[(size_t)b * 12 + 3])) continue;
            int cx, cy, cz;
            world_to_cell(ppos(b), cx, cy, cz);
            for (int di = -1; di <= 1; ++di)
                for (int dj = -1; dj <= 1; ++dj)
                    for (int dk = -1; dk <= 1; ++dk) {
                        int x = cx + di, y = cy + dj, z = cz + dk;
                        if (!in_grid(x, y, z)) continue;
                        atomic_max_i32(&lookup[cell_index(x, y, z)], b);
                    }
        }
    }
    // shader.rs:955-1052
    void k_p2g() {
        int np = (int)num_particles();
#pragma omp parallel for schedule(static)
        for (int pid = 0; pid < np; ++pid) {
            const R* p = &part[(size_t)pid * 8];
            const R* a = &aff[(size_t)pid * 12];
            V xp = V3<R>(p[0], p[1], p[2]);
            V vp = V3<R>(p[4], p[5], p[6]);
            R J = p[3], mp = p[7], phase = a[3];
            if (!is_water_phase(phase) || mp <= inactive_mass_threshold()) continue;
            V gp = (xp - u.origin) * u.inv_dx;
            int bx = (int)std::floor(gp.x - R(0.5)), by = (int)std::floor(gp.y - R(0.5)), bz = (int)std::floor(gp.z - R(0.5));
            V fx = gp - V3<R>(R(bx), R(by), R(bz));
            R wx[3], wy[3], wz[3];
            weights(fx.x, wx);
            weights(fx.y, wy);
            weights(fx.z, wz);
            V c0 = V3<R>(a[0], a[1], a[2]), c1 = V3<R>(a[4], a[5], a[6]), c2 = V3<R>(a[8], a[9], a[10]);
            V a0 = V3<R>(mp * c0.x, mp * c0.y, mp * c0.z);
            V a1 = V3<R>(mp * c1.x, mp * c1.y, mp * c1.z);
            V a2 = V3<R>(mp * c2.x, mp * c2.y, mp * c2.z);
            R fp = u.fp_scale, cdx = u.dx;
            R rpv = u.p_vol * mp / wmax(u.nominal_mass, R(1e-6));
            R cpv = rpv * clamp_j(J);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    for (int k = 0; k < 3; ++k) {
                        int cx = bx + i, cy = by + j, cz = bz + k;
                        if (!in_grid(cx, cy, cz)) continue;
                        R w = wx[i] * wy[j] * wz[k];
                        V dpos = (V3<R>(R(i), R(j), R(k)) - fx) * cdx;
                        R mc = w * mp, rvc = w * rpv, cvc = w * cpv;
                        V inner = mp * vp + V3<R>(dot(a0, dpos), dot(a1, dpos), dot(a2, dpos));
                        V mom = w * inner;
                        uint32_t ci = cell_index(cx, cy, cz);
                        const bool i64 = int64_grid();
                        if (i64) fp = R(4294967296.0f);
                        R lim = i64 ? R(1.0e18f) : R(1.0e9);
                        R mfp = mc * fp, rfp = rvc * fp, cfp = cvc * fp;
                        R mxf = mom.x * fp, myf = mom.y * fp, mzf = mom.z * fp;
                        if (std::fabs(mfp) > lim || std::fabs(mxf) > lim || std::fabs(myf) > lim ||
                            std::fabs(mzf) > lim || std::fabs(rfp) > lim || std::fabs(cfp) > lim)
                            atomic_add_u32(&metrics[M_OVERFLOW], 1u);
                        if (i64) {
                            const R vals[6] = {mfp, mxf, myf, mzf, rfp, cfp};
                            for (int l = 0; l < 6; ++l) {
                                // two's-complement sum, like the device's u64 atomics
                                __atomic_fetch_add(reinterpret_cast<uint64_t*>(&grid64[(size_t)l * cells + ci]),
                                                   (uint64_t)to_i64(vals[l]), __ATOMIC_RELAXED);
                            }
                            continue;
                        }
                        atomic_add_i32(&lane(0)[ci], to_i32(mfp));
                        atomic_add_i32(&lane(1)[ci], to_i32(mxf));
                        atomic_add_i32(&lane(2)[ci], to_i32(myf));
                        atomic_add_i32(&lane(3)[ci], to_i32(mzf));
                        atomic_add_i32(&lane(4)[ci], to_i32(rfp));
                        atomic_add_i32(&lane(5)[ci], to_i32(cfp));
                    }
        }
    }
    // shader.rs:1056-1082
    void k_grid_update() {
        int n = (int)cells;
#pragma omp parallel for schedule(static)
        for (int idx = 0; idx < n; ++idx) {
            R mass = p2g_lane(0, idx);
            if (mass < R(1e-6)) continue;
            V v = V3<R>(p2g_lane(1, idx) / mass, p2g_lane(2, idx) / mass, p2g_lane(3, idx) / mass);
            v.y += u.gravity * u.dt;
            R sp = length(v);
            if (sp > u.vel_cap) v = v * (u.vel_cap / sp);
            R* g = &gvel[(size_t)idx * 4];
            g[0] = v.x; g[1] = v.y; g[2] = v.z; g[3] = mass;
        }
    }
    void decompose(uint32_t idx, uint32_t& ix, uint32_t& iy, uint32_t& iz) {
        iz = idx / (u.gx * u.gy);
        uint32_t rem = idx % (u.gx * u.gy);
        iy = rem / u.gx;
        ix = rem % u.gx;
    }
    V cell_center(uint32_t ix, uint32_t iy, uint32_t iz) {
        return u.origin + (V3<R>(R(ix), R(iy), R(iz)) + V3<R>(R(0.5), R(0.5), R(0.5))) * u.dx;
    }
    // shader.rs:1086-1163
    void k_viscosity_prepare() {
        int n = (int)cells;
        static const int off[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
#pragma omp parallel for schedule(static)
        for (int idx = 0; idx < n; ++idx) {
            const R* gv = &gvel[(size_t)idx * 4];
            V vh = V3<R>(gv[0], gv[1], gv[2]);
            R gw = gv[3];
            if (gw <= occupancy_threshold() || u.viscosity <= R(0)) {
                vscratch_store(idx, vh);
                continue;
            }
            uint32_t ix, iy, iz;
            decompose(idx, ix, iy, iz);
            if (gw <= viscosity_support_threshold()) {
                vscratch_store(idx, vh);
                continue;
            }
            R alpha = wclamp(u.viscosity * u.dt / wmax(u.dx * u.dx, R(1e-6)), R(0), R(0.14));
            V nsum = V3<R>(0, 0, 0);
            R wsum = R(0);
            uint32_t nfluid = 0;
            for (int q = 0; q < 6; ++q) {
                int x = (int)ix + off[q][0], y = (int)iy + off[q][1], z = (int)iz + off[q][2];
                if (!in_grid(x, y, z)) {
                    wsum += R(1);
                    continue;
                }
                if (class_solid(x, y, z)) {
                    wsum += R(1);
                    continue;
                }
                const R* ng = &gvel[(size_t)cell_index(x, y, z) * 4];
                if (ng[3] <= occupancy_threshold()) continue;
                R nw = wclamp(ng[3] / wmax(wmax(gw, u.nominal_mass), R(1e-6)), R(0), R(1));
                nsum += V3<R>(ng[0], ng[1], ng[2]) * nw;
                wsum += nw;
                nfluid += 1;
            }
            if (nfluid < 3 || wsum <= R(1e-6)) {
                vscratch_store(idx, vh);
                continue;
            }
            V avg = nsum / wsum;
            R blend = wclamp(alpha * wsum, R(0), R(0.65));
            vscratch_store(idx, mix(vh, avg, blend));
        }
    }
    // shader.rs:1166-1177
    void k_viscosity_apply() {
        int n = (int)cells;
#pragma omp parallel for schedule(static)
        for (int idx = 0; idx < n; ++idx) {
            R* g = &gvel[(size_t)idx * 4];
            R mass = g[3];
            if (mass <= occupancy_threshold()) {
                g[0] = g[1] = g[2] = g[3] = R(0);
                continue;
            }
            V v = vscratch_load(idx);
            g[0] = v.x; g[1] = v.y; g[2] = v.z;
        }
    }
    // shader.rs:1181-1367
    bool open_neighbor(V cc, int x, int y, int z, R ox, R oy, R oz) {
        if (u.use_sdf_cache) return !class_solid(x, y, z);
        return sample_sdf(cc + V3<R>(ox, oy, oz)) >= R(0);
    }
    void k_classify(bool warm) {
        int n = (int)cells;
        static const int off[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
#pragma omp parallel for schedule(static)
        for (int idx = 0; idx < n; ++idx) {
            R mass = gvel[(size_t)idx * 4 + 3];
            R keep_p = (!fixed_point()) ? pf[idx] : R(0);
            R keep_lo = plo[idx];
            pressure_store(idx, R(0));
            plo[idx] = R(0);
            uint32_t ix, iy, iz;
            decompose(idx, ix, iy, iz);
            V cc = cell_center(ix, iy, iz);
            bool solid = u.use_sdf_cache ? class_solid(ix, iy, iz) : (sample_sdf(cc) < R(0));
            if (solid) {
                lane(3)[idx] = CELL_SOLID;
                div_store(idx, R(0));
                continue;
            }
            if (mass <= occupancy_threshold()) {
                lane(3)[idx] = CELL_AIR;
                div_store(idx, R(0));
                continue;
            }
            if (lookup_load(idx) >= 0) {
                lane(3)[idx] = CELL_BED;
            } else {
                bool air = false;
                for (int q = 0; q < 6; ++q) {
                    int x = (int)ix + off[q][0], y = (int)iy + off[q][1], z = (int)iz + off[q][2];
                    if (!in_grid(x, y, z)) { air = true; break; }
                    if (gvel[(size_t)cell_index(x, y, z) * 4 + 3] <= occupancy_threshold()) { air = true; break; }
                }
                lane(3)[idx] = air ? CELL_SURFACE : CELL_INTERIOR;
            }
            int32_t kind = kind_load(idx);
            if (!is_fluid(kind)) {
                div_store(idx, R(0));
                continue;
            }
            if (warm) {
                pf[idx] = keep_p;
                plo[idx] = keep_lo;
            }
            const R* sv = &gvel[(size_t)idx * 4];
            R dxv = u.dx;
            R vxm = -sv[0], vxp = -sv[0], vym = -sv[1], vyp = -sv[1], vzm = -sv[2], vzp = -sv[2];
            if (ix > 0 && open_neighbor(cc, ix - 1, iy, iz, -dxv, 0, 0)) vxm = gvel[(size_t)cell_index(ix - 1, iy, iz) * 4 + 0];
            if (ix + 1 < u.gx && open_neighbor(cc, ix + 1, iy, iz, dxv, 0, 0)) vxp = gvel[(size_t)cell_index(ix + 1, iy, iz) * 4 + 0];
            if (iy > 0 && open_neighbor(cc, ix, iy - 1, iz, 0, -dxv, 0)) vym = gvel[(size_t)cell_index(ix, iy - 1, iz) * 4 + 1];
            if (iy + 1 < u.gy && open_neighbor(cc, ix, iy + 1, iz, 0, dxv, 0)) vyp = gvel[(size_t)cell_index(ix, iy + 1, iz) * 4 + 1];
            if (iz > 0 && open_neighbor(cc, ix, iy, iz - 1, 0, 0, -dxv)) vzm = gvel[(size_t)cell_index(ix, iy, iz - 1) * 4 + 2];
            if (iz + 1 < u.gz && open_neighbor(cc, ix, iy, iz + 1, 0, 0, dxv)) vzp = gvel[(size_t)cell_index(ix, iy, iz + 1) * 4 + 2];
            R div = R(0.5) * u.inv_dx * (((vxp - vxm) + (vyp - vym)) + (vzp - vzm));
            R rest = rest_vol(idx), cur = cur_vol(idx);
            R target = volume_target(rest, cur);
            if (kind == CELL_BED) {
                int32_t b = lookup_load(idx);
                if (b >= 0 && (uint32_t)b < u.num_bed) {
                    R pt = bed_pore_target((uint32_t)b, cc, rest, cur);
                    R poro = wclamp(bed_compacted_porosity((uint32_t)b), R(0.08), R(1));
                    R sfrac = R(1) - poro;
                    R sdiv = bed_velocity_divergence((int)ix, (int)iy, (int)iz);
                    target = (pt - sfrac * sdiv) / poro;
                }
            }
            div_store(idx, div - target);
            R ad = std::fabs(div);
            uint32_t fd = to_u32(wclamp(ad * u.mdiv_scale, R(0), R(2147483648.0f)));
            atomic_max_u32(&metrics[M_MAX_DIV], fd);
            atomic_add_u32(&metrics[M_FLUID], 1u);
        }
    }
    // shader.rs:1371-1439
    void pressure_update(uint32_t idx) {
        uint32_t ix, iy, iz;
        decompose(idx, ix, iy, iz);
        int32_t kind = kind_load(idx);
        if (!is_fluid(kind)) {
            pressure_store(idx, R(0));
            return;
        }
        static const int off[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
        R nc = R(0), ps = R(0);
        R sf = liquid_fill(idx, kind);
        for (int q = 0; q < 6; ++q) {
            int x = (int)ix + off[q][0], y = (int)iy + off[q][1], z = (int)iz + off[q][2];
            if (!in_grid(x, y, z)) continue;
            uint32_t ni = cell_index(x, y, z);
            int32_t nk = kind_load(ni);
            if (is_solid(nk)) continue;
            R w = face_weight(kind, sf, ni, nk);
            if (w <= R(0)) continue;
            nc += w;
            if (is_fluid(nk)) ps += w * pressure_load(ni);
        }
        if (nc <= R(0)) {
            pressure_store(idx, R(0));
            return;
        }
        R rhs = div_load(idx) * sf / wmax(u.dt, R(1e-6));
        R pn = (ps - u.dx * u.dx * rhs) / nc;
        // Over-relaxed update p + w*(p_gs - p); w == 1 is the reference's plain update.
        if (u.omega != R(1)) pn = pressure_load(idx) + u.omega * (pn - pressure_load(idx));
        pressure_store(idx, pn);
    }
    void k_rbgs(uint32_t parity) {
        int n = (int)cells;
#pragma omp parallel for schedule(static)
        for (int idx = 0; idx < n; ++idx) {
            uint32_t ix, iy, iz;
            decompose(idx, ix, iy, iz);
            if (((ix + iy + iz) & 1u) != parity) continue;
            pressure_update(idx);
        }
    }
    // Relative residual ||(sum w p_nb - dx^2 rhs) - W p|| / ||dx^2 rhs|| in FP64
    // over fluid cells, with the face weights of pressure_update.
    double residual() {
        int n = (int)cells;
        int nt = 1;
#ifdef _OPENMP
        nt = omp_get_max_threads();
#endif
        std::vector<double> rs(nt, 0.0), bs(nt, 0.0);
        static const int off[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
#pragma omp parallel num_threads(nt)
        {
            int t = 0;
#ifdef _OPENMP
            t = omp_get_thread_num();
#endif
            double r2 = 0.0, b2 = 0.0;
#pragma omp for schedule(static)
            for (int idx = 0; idx < n; ++idx) {
                int32_t kind = kind_load(idx);
                if (!is_fluid(kind)) continue;
                uint32_t ix, iy, iz;
                decompose(idx, ix, iy, iz);
                R sf = liquid_fill(idx, kind);
                double wsum = 0.0, psum = 0.0;
                for (int q = 0; q < 6; ++q) {
                    int x = (int)ix + off[q][0], y = (int)iy + off[q][1], z = (int)iz + off[q][2];
                    if (!in_grid(x, y, z)) continue;
                    uint32_t ni = cell_index(x, y, z);
                    int32_t nk = kind_load(ni);
                    if (is_solid(nk)) continue;
                    R w = face_weight(kind, sf, ni, nk);
                    if (w <= R(0)) continue;
                    wsum += (double)w;
                    if (is_fluid(nk)) psum += (double)w * (double)pressure_load(ni);
                }
                if (wsum <= 0.0) continue;
                R rhs = div_load(idx) * sf / wmax(u.dt, R(1e-6));
                double b = (double)(u.dx * u.dx * rhs);
                double r = (psum - b) - wsum * (double)pressure_load(idx);
                r2 += r * r;
                b2 += b * b;
            }
            rs[t] = r2;
            bs[t] = b2;
        }
        double r2 = 0.0, b2 = 0.0;
        for (int t = 0; t < nt; ++t) {
            r2 += rs[t];
            b2 += bs[t];
        }
        if (b2 <= 0.0) return 0.0;
        return std::sqrt(r2) / std::sqrt(b2);
    }
    // ---- mixed-precision iterative refinement (FP32 storage, residual mode) ----
    // Pressure is held as p = hi + lo (two fp32 words).  A cycle computes the FP64
    // residual g = (sum w p_nb - dx^2 rhs) - W p of pressure_update's operator, runs
    // red-black sweeps on the correction d of L d = g in fp32, and adds d to p in
    // FP64.  The sweep count and the stopping test use the FP64 residual norm.
    double refine_residual() {
        int n = (int)cells;
        int nt = 1;
#ifdef _OPENMP
        nt = omp_get_max_threads();
#endif
        std::vector<double> rs(nt, 0.0), bs(nt, 0.0);
        static const int off[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
#pragma omp parallel num_threads(nt)
        {
            int t = 0;
#ifdef _OPENMP
            t = omp_get_thread_num();
#endif
            double r2 = 0.0, b2 = 0.0;
#pragma omp for schedule(static)
            for (int idx = 0; idx < n; ++idx) {
                pd[idx] = R(0);
                gres[idx] = R(0);
                int32_t kind = kind_load(idx);
                if (!is_fluid(kind)) continue;
                uint32_t ix, iy, iz;
                decompose(idx, ix, iy, iz);
                R sf = liquid_fill(idx, kind);
                double wsum = 0.0, psum = 0.0;
                for (int q = 0; q < 6; ++q) {
                    int x = (int)ix + off[q][0], y = (int)iy + off[q][1], z = (int)iz + off[q][2];
                    if (!in_grid(x, y, z)) continue;
                    uint32_t ni = cell_index(x, y, z);
                    int32_t nk = kind_load(ni);
                    if (is_solid(nk)) continue;
                    R w = face_weight(kind, sf, ni, nk);
                    if (w <= R(0)) continue;
                    wsum += (double)w;
                    if (is_fluid(nk)) psum += (double)w * ((double)pf[ni] + (double)plo[ni]);
                }
                if (wsum <= 0.0) continue;
                R rhs = div_load(idx) * sf / wmax(u.dt, R(1e-6));
                double b = (double)(u.dx * u.dx * rhs);
                double r = (psum - b) - wsum * ((double)pf[idx] + (double)plo[idx]);
                gres[idx] = R(r);
                r2 += r * r;
                b2 += b * b;
            }
            rs[t] = r2;
            bs[t] = b2;
        }
        double r2 = 0.0, b2 = 0.0;
        for (int t = 0; t < nt; ++t) {
            r2 += rs[t];
            b2 += bs[t];
        }
        if (b2 <= 0.0) return 0.0;
        return std::sqrt(r2) / std::sqrt(b2);
    }
    void refine_sweep(uint32_t parity) {
        int n = (int)cells;
        static const int off[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
#pragma omp parallel for schedule(static)
        for (int idx = 0; idx < n; ++idx) {
            uint32_t ix, iy, iz;
            decompose(idx, ix, iy, iz);
            if (((ix + iy + iz) & 1u) != parity) continue;
            int32_t kind = kind_load(idx);
            if (!is_fluid(kind)) continue;
            R sf = liquid_fill(idx, kind);
            R nc = R(0), ds = R(0);
            for (int q = 0; q < 6; ++q) {
                int x = (int)ix + off[q][0], y = (int)iy + off[q][1], z = (int)iz + off[q][2];
                if (!in_grid(x, y, z)) continue;
                uint32_t ni = cell_index(x, y, z);
                int32_t nk = kind_load(ni);
                if (is_solid(nk)) continue;
                R w = face_weight(kind, sf, ni, nk);
                if (w <= R(0)) continue;
                nc += w;
                if (is_fluid(nk)) ds += w * pd[ni];
            }
            if (nc <= R(0)) continue;
            R dn = (ds + gres[idx]) * (R(1) / nc);
            if (u.omega != R(1)) dn = pd[idx] + u.omega * (dn - pd[idx]);
            pd[idx] = dn;
        }
    }
    void refine_accumulate() {
        int n = (int)cells;
        R lim = u.p_limit;
#pragma omp parallel for schedule(static)
        for (int idx = 0; idx < n; ++idx) {
            if (!is_fluid(kind_load(idx))) continue;
            double p = ((double)pf[idx] + (double)plo[idx]) + (double)pd[idx];
            if (p > (double)lim || p < -(double)lim) {
                p = p > 0.0 ? (double)lim : -(double)lim;
                atomic_add_u32(&metrics[M_P_CLAMP], 1u);
            }
            R hi = R(p);
            pf[idx] = hi;
            plo[idx] = R(p - (double)hi);
        }
    }

    // shader.rs:1457-1543
    void k_project() {
        int n = (int)cells;
#pragma omp parallel for schedule(static)
        for (int idx = 0; idx < n; ++idx) {
            R* g = &gvel[(size_t)idx * 4];
            if (g[3] < R(1e-6)) continue;
            int32_t kind = kind_load(idx);
            if (!is_fluid(kind)) continue;
            uint32_t ix, iy, iz;
            decompose(idx, ix, iy, iz);
            R ph = pressure_load(idx);
            R sf = liquid_fill(idx, kind);
            int x = ix, y = iy, z = iz;
            R pxm = pressure_weighted_or_mirror(x - 1, y, z, ph, kind, sf);
            R pxp = pressure_weighted_or_mirror(x + 1, y, z, ph, kind, sf);
            R pym = pressure_weighted_or_mirror(x, y - 1, z, ph, kind, sf);
            R pyp = pressure_weighted_or_mirror(x, y + 1, z, ph, kind, sf);
            R pzm = pressure_weighted_or_mirror(x, y, z - 1, ph, kind, sf);
            R pzp = pressure_weighted_or_mirror(x, y, z + 1, ph, kind, sf);
            R h = R(0.5) * u.inv_dx;
            V grad = V3<R>(h * (pxp - pxm), h * (pyp - pym), h * (pzp - pzm));
            V v = V3<R>(g[0], g[1], g[2]) - u.dt * grad;
            if (kind == CELL_BED) {
                int32_t b = lookup_load(idx);
                if (b >= 0 && (uint32_t)b < u.num_bed) {
                    R perm = bed_compacted_permeability((uint32_t)b);
                    R rate = u.nu_m2s / perm;
                    R damp = R(1) / (R(1) + wmax(rate * u.dt, R(0)));
                    V bv = bed_matrix_velocity_cell(x, y, z);
                    V vb = v;
                    v = bv + (v - bv) * damp;
                    V wi = g[3] * (v - vb);
                    bed_impulse_neighborhood(x, y, z, (-wi) * R(BED_REACTION_ALPHA));
                }
            }
            R sp = length(v);
            if (sp > u.vel_cap) v = v * (u.vel_cap / sp);
            g[0] = v.x; g[1] = v.y; g[2] = v.z;
        }
    }
    // shader.rs:1547-1564
    R packing_or_mirror(int x, int y, int z, R mirror) {
        if (!in_grid(x, y, z)) return mirror;
        uint32_t ci = cell_index(x, y, z);
        int32_t k = kind_load(ci);
        if (is_solid(k)) return mirror;
        if (!is_fluid(k)) return R(0);
        return packing_load(ci);
    }
    // shader.rs:1566-1583
    void k_packing_prepare() {
        int n = (int)cells;
#pragma omp parallel for schedule(static)
        for (int idx = 0; idx < n; ++idx) {
            int32_t kind = kind_load(idx);
            if (!is_fluid(kind) || kind == CELL_BED) {
                packing_store(idx, R(0));
                continue;
            }
            R cv = u.dx * u.dx * u.dx;
            R packed = wmax(rest_vol(idx), cur_vol(idx)) / wmax(cv, R(1e-8));
            R tgt = wmin(u.max_rest_frac, R(1));
            R over = wmax(packed - tgt, R(0));
            packing_store(idx, u.bulk_K * over);
        }
    }
    // shader.rs:1586-1626
    void k_packing_apply() {
        int n = (int)cells;
#pragma omp parallel for schedule(static)
        for (int idx = 0; idx < n; ++idx) {
            R* g = &gvel[(size_t)idx * 4];
            if (g[3] <= occupancy_threshold()) continue;
            int32_t kind = kind_load(idx);
            if (!is_fluid(kind)) continue;
            uint32_t ix, iy, iz;
            decompose(idx, ix, iy, iz);
            int x = ix, y = iy, z = iz;
            R ph = packing_load(idx);
            R pxm = packing_or_mirror(x - 1, y, z, ph), pxp = packing_or_mirror(x + 1, y, z, ph);
            R pym = packing_or_mirror(x, y - 1, z, ph), pyp = packing_or_mirror(x, y + 1, z, ph);
            R pzm = packing_or_mirror(x, y, z - 1, ph), pzp = packing_or_mirror(x, y, z + 1, ph);
            R h = R(0.5) * u.inv_dx;
            V grad = V3<R>(h * (pxp - pxm), h * (pyp - pym), h * (pzp - pzm));
            V v = V3<R>(g[0], g[1], g[2]) - u.dt * grad;
            R sp = length(v);
            if (sp > u.vel_cap) v = v * (u.vel_cap / sp);
            g[0] = v.x; g[1] = v.y; g[2] = v.z;
        }
    }
    // shader.rs:1630-1679
    void k_boundary() {
        int n = (int)cells;
#pragma omp parallel for schedule(static)
        for (int idx = 0; idx < n; ++idx) {
            R* g = &gvel[(size_t)idx * 4];
            if (g[3] < R(1e-6)) continue;
            V v = V3<R>(g[0], g[1], g[2]);
            uint32_t ix, iy, iz;
            decompose(idx, ix, iy, iz);
            V cp = cell_center(ix, iy, iz);
            R sv = sample_sdf(cp);
            if (sv < u.contact_offset) {
                V nn = sdf_gradient(cp);
                R vn = dot(v, nn);
                if (vn < R(0)) {
                    v = v - nn * vn * (R(1) + u.restitution);
                    V vt = v - nn * dot(v, nn);
                    R vtl = length(vt);
                    if (vtl > R(1e-6)) {
                        R fi = wmin(u.friction * std::fabs(vn), vtl);
                        v = v - vt * (fi / vtl);
                    }
                }
            }
            R margin = R(2) * u.dx;
            V bmin = u.origin + V3<R>(margin, margin, margin);
            V bmx = u.bmax - V3<R>(margin, margin, margin);
            if (cp.x < bmin.x && v.x < R(0)) v.x = R(0);
            if (cp.x > bmx.x && v.x > R(0)) v.x = R(0);
            if (cp.y < bmin.y && v.y < R(0)) v.y = R(0);
            if (cp.y > bmx.y && v.y > R(0)) v.y = R(0);
            if (cp.z < bmin.z && v.z < R(0)) v.z = R(0);
            if (cp.z > bmx.z && v.z > R(0)) v.z = R(0);
            g[0] = v.x; g[1] = v.y; g[2] = v.z;
        }
    }
    // shader.rs:1683-1881
    void k_g2p() {
        int np = (int)num_particles();
#pragma omp parallel for schedule(static)
        for (int pid = 0; pid < np; ++pid) {
            R* p = &part[(size_t)pid * 8];
            R* a = &aff[(size_t)pid * 12];
            V xp = V3<R>(p[0], p[1], p[2]);
            R J_old = p[3], mp = p[7];
            R phase = a[3];
            if (!is_water_phase(phase)) continue;
            if (mp <= inactive_mass_threshold()) {
                p[7] = R(0);
                continue;
            }
            V gp = (xp - u.origin) * u.inv_dx;
            int bx = (int)std::floor(gp.x - R(0.5)), by = (int)std::floor(gp.y - R(0.5)), bz = (int)std::floor(gp.z - R(0.5));
            V fx = gp - V3<R>(R(bx), R(by), R(bz));
            R wx[3], wy[3], wz[3];
            weights(fx.x, wx);
            weights(fx.y, wy);
            weights(fx.z, wz);
            V nv = V3<R>(0, 0, 0), nc0 = nv, nc1 = nv, nc2 = nv;
            R supp = R(0), lmass = R(0), bow = R(0), bperm = R(0);
            V bvs = V3<R>(0, 0, 0);
            R B = R(4) * u.inv_dx * u.inv_dx;
            R cdx = u.dx;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    for (int k = 0; k < 3; ++k) {
                        int cx = bx + i, cy = by + j, cz = bz + k;
                        if (!in_grid(cx, cy, cz)) continue;
                        R w = wx[i] * wy[j] * wz[k];
                        uint32_t ci = cell_index(cx, cy, cz);
                        const R* g = &gvel[(size_t)ci * 4];
                        V gv = V3<R>(g[0], g[1], g[2]);
                        V dpos = (V3<R>(R(i), R(j), R(k)) - fx) * cdx;
                        R gm = g[3];
                        if (gm > R(1e-6)) {
                            nv += w * gv;
                            R wb = w * B;
                            nc0 += (wb * gv) * dpos.x;
                            nc1 += (wb * gv) * dpos.y;
                            nc2 += (wb * gv) * dpos.z;
                            supp += w;
                            lmass += w * gm;
                        }
                        int32_t b = lookup_load(ci);
                        if (u.num_bed > 0u && valid_bed_solid(b)) {
                            bow += w;
                            bvs += w * pvel(b);
                            bperm += w * bed_compacted_permeability(b);
                        }
                    }
            R sr = wclamp(supp, R(0), R(1));
            R jsup = sr;
            if (supp > R(1e-6)) {
                R inv = R(1) / supp;
                nv *= inv; nc0 *= inv; nc1 *= inv; nc2 *= inv;
            }
            R co = R(u.g.cup_radius) + u.contact_offset;
            bool in_cup = (u.g.flags & CS_GEOM_CUP) && xp.y < R(u.g.cup_top_y) && (xp.x * xp.x + xp.z * xp.z) < co * co;
            R dsr = wclamp(lmass / wmax(u.nominal_mass * R(4), R(1e-6)), R(0), R(1));
            R po = wclamp(bow, R(0), R(1));
            V pbv = V3<R>(0, 0, 0);
            R pbk = u.min_perm;
            if (bow > R(1e-6)) {
                R inv = R(1) / bow;
                pbv = bvs * inv;
                pbk = wmax(bperm * inv, u.min_perm);
            }
            if (sr < R(0.999)) {
                V bal = V3<R>(p[4], p[5] + u.gravity * u.dt, p[6]);
                R fg = in_cup ? R(1.15) : R(1.35);
                R fc = in_cup ? R(0.95) : R(0.995);
                R pg = mix(fg, R(0.18), po);
                R pc = mix(fc, R(0.16), po);
                R dpd = mix(R(1), R(0.12), dsr);
                R pres = wclamp((R(1) - sr) * pg * dpd, R(0), pc);
                nv = mix(nv, bal, pres);
                R ad = R(1) - pres * R(0.75);
                nc0 *= ad; nc1 *= ad; nc2 *= ad;
            }
            bool airborne = po <= R(0.05) && sample_sdf(xp) > u.contact_offset * R(2);
            if (airborne) {
                R dm = u.nominal_mass * R(4);
                R dr = wclamp(lmass / wmax(dm, R(1e-6)), R(0), R(1));
                jsup = wmin(jsup, dr);
                V bal = V3<R>(p[4], p[5] + u.gravity * u.dt, p[6]);
                R pg = in_cup ? R(0.72) : R(0.98);
                R pc = in_cup ? R(0.88) : R(0.98);
                R pres = wclamp((R(1) - dr) * pg, R(0), pc);
                nv = mix(nv, bal, pres);
                R ad = R(1) - pres * R(0.65);
                nc0 *= ad; nc1 *= ad; nc2 *= ad;
            }
            if (po > R(1e-4)) {
                V rel = nv - pbv;
                R rate = u.nu_m2s / pbk;
                R dd = R(1) / (R(1) + wmax(rate * u.dt * po, R(0)));
                R rs = length(rel);
                R id = R(1) / (R(1) + wmax(rs * u.dt * u.inv_dx * po * R(0.35), R(0)));
                V nvb = nv;
                nv = pbv + rel * dd * id;
                V wi = mp * (nv - nvb);
                int wcx, wcy, wcz;
                world_to_cell(xp, wcx, wcy, wcz);
                bed_impulse_neighborhood(wcx, wcy, wcz, (-wi) * R(BED_REACTION_ALPHA));
                R ad = mix(R(1), dd * id, po);
                nc0 *= ad; nc1 *= ad; nc2 *= ad;
                jsup = wmax(jsup, po);
            }
            R tr = nc0.x + nc1.y + nc2.z;
            R jo = clamp_j(J_old > R(0) ? J_old : R(1));
            R ja = clamp_j(jo * exp_small(wclamp(u.dt * tr, R(-0.35), R(0.35))));
            R jb = smoothstep(R(0.35), R(0.85), wclamp(jsup, R(0), R(1)));
            R jn = clamp_j(mix(jo, ja, jb));
            V np_ = xp + nv * u.dt;
            V mid = mix(xp, np_, R(0.5));
            V cpos = mid, cvel = nv;
            sdf_contact(cpos, cvel, false);
            nv = cvel;
            cpos = np_;
            sdf_contact(cpos, cvel, false);
            np_ = cpos;
            nv = cvel;
            R margin = u.dx * R(0.5);
            V lo = u.origin + V3<R>(margin, margin, margin);
            V hi = u.bmax - V3<R>(margin, margin, margin);
            np_ = V3<R>(wclamp(np_.x, lo.x, hi.x), wclamp(np_.y, lo.y, hi.y), wclamp(np_.z, lo.z, hi.z));
            p[0] = np_.x; p[1] = np_.y; p[2] = np_.z; p[3] = jn;
            p[4] = nv.x; p[5] = nv.y; p[6] = nv.z; p[7] = mp;
            a[0] = nc0.x; a[1] = nc0.y; a[2] = nc0.z; a[3] = phase;
            a[4] = nc1.x; a[5] = nc1.y; a[6] = nc1.z; a[7] = R(0);
            a[8] = nc2.x; a[9] = nc2.y; a[10] = nc2.z; a[11] = R(0);
        }
    }
    // shader.rs:1885-1957
    void k_bed_coupling() {
        int np = (int)num_particles();
#pragma omp parallel for schedule(static)
        for (int pid = 0; pid < np; ++pid) {
            R* p = &part[(size_t)pid * 8];
            R phase = aff[(size_t)pid * 12 + 3];
            if (!is_water_phase(phase)) continue;
            V pos = V3<R>(p[0], p[1], p[2]);
            int cx, cy, cz;
            world_to_cell(pos, cx, cy, cz);
            if (!in_grid(cx, cy, cz)) continue;
            R mp = p[7];
            R pw = filter_paper_weight(pos);
            if (pw > R(1e-4) && u.filter_absorption > R(0)) {
                R frac = wclamp(u.filter_absorption * pw * u.dt, R(0), R(0.04));
                R ab = wmin(mp * frac, mp * R(0.12));
                mp = wmax(mp - ab, inactive_mass_threshold() * R(1.25));
                p[7] = mp;
            }
            uint32_t ci = cell_index(cx, cy, cz);
            int32_t b = lookup_load(ci);
            if (b < 0 || (uint32_t)b >= u.num_bed) continue;
            const R* be = &bedx[(size_t)b * 8];
            R sat = be[7];
            R cap = wmax(u.max_saturation - be[0], R(0));
            if (cap <= R(1e-6)) continue;
            R ar = u.absorption_rate * (R(1) - sat) * u.dt;
            R speed = length(V3<R>(p[4], p[5], p[6]));
            R absorbed = wmin(wmin(mp * wclamp(ar, R(0), R(0.25)), mp * R(0.5)), cap);
            R rem_partial = mp - absorbed;
            R retire = u.nominal_mass * R(0.22);
            if (rem_partial > R(0) && rem_partial <= retire) {
                absorbed = wmin(mp, cap);
            } else if (sat > R(0.55) && speed < R(1.35)) {
                R almost = wmin(mp, cap);
                if (mp - almost <= u.nominal_mass * R(0.35)) absorbed = almost;
            }
            if (mp - absorbed <= inactive_mass_threshold() && absorbed < mp)
                absorbed = wmax(mp - inactive_mass_threshold() * R(1.05), R(0));
            if (absorbed <= R(1e-6)) continue;
            R remaining = mp - absorbed;
            if (remaining <= inactive_mass_threshold()) {
                p[4] = p[5] = p[6] = p[7] = R(0);
            } else {
                p[7] = remaining;
            }
            deposit_absorbed(cx, cy, cz, b, absorbed);
        }
    }
    // shader.rs:1961-1987
    void k_extraction_advect() {
        int nb = (int)u.num_bed;
#pragma omp parallel for schedule(static)
        for (int b = 0; b < nb; ++b) {
            R* be = &bedx[(size_t)b * 8];
            R absorbed = R(atomic_xchg_i32(&delta_lane(0)[b], 0)) * u.inv_fp;
            if (absorbed > R(0)) {
                be[0] += absorbed;
                be[7] = wclamp(be[0] / wmax(u.max_saturation, R(1e-6)), R(0), R(1));
            }
            R sat = be[7];
            if (sat > R(0.01)) {
                R flux = u.extraction_rate * be[4] * sat * u.dt;
                be[4] = wmax(be[4] - flux, R(0));
                be[5] += flux;
            }
        }
    }
    // shader.rs:1991-2238
    void k_bed_dynamics() {
        int nb = (int)u.num_bed;
        std::vector<R> snap((size_t)nb * 3);
        for (int b = 0; b < nb; ++b) {
            snap[(size_t)b * 3] = part[(size_t)b * 8];
            snap[(size_t)b * 3 + 1] = part[(size_t)b * 8 + 1];
            snap[(size_t)b * 3 + 2] = part[(size_t)b * 8 + 2];
        }
#pragma omp parallel for schedule(static)
        for (int bid = 0; bid < nb; ++bid) {
            R* p = &part[(size_t)bid * 8];
            R* a = &aff[(size_t)bid * 12];
            R* be = &bedx[(size_t)bid * 8];
            R phase = a[3];
            V rest = V3<R>(a[4], a[5], a[6]);
            V pos = V3<R>(p[0], p[1], p[2]);
            V pv = V3<R>(p[4], p[5], p[6]);
            R mp = p[7];
            V brv = bed_impulse_exchange(bid) / wmax(mp, u.nominal_mass * R(0.25));
            R mrs = wmin(u.vel_cap * R(0.012), u.dx / wmax(u.dt, R(1e-6)) * R(0.02));
            R rsp = length(brv);
            if (rsp > mrs && rsp > R(1e-6)) brv *= mrs / rsp;
            V gp = (pos - u.origin) * u.inv_dx;
            int bx = (int)std::floor(gp.x - R(0.5)), by = (int)std::floor(gp.y - R(0.5)), bz = (int)std::floor(gp.z - R(0.5));
            V fx = gp - V3<R>(R(bx), R(by), R(bz));
            R wx[3], wy[3], wz[3];
            weights(fx.x, wx);
            weights(fx.y, wy);
            weights(fx.z, wz);
            V wv = V3<R>(0, 0, 0);
            R wm = R(0), asw = R(0), lasw = R(0);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    for (int k = 0; k < 3; ++k) {
                        int cx = bx + i, cy = by + j, cz = bz + k;
                        if (!in_grid(cx, cy, cz)) continue;
                        R w = wx[i] * wy[j] * wz[k];
                        uint32_t ci = cell_index(cx, cy, cz);
                        const R* g = &gvel[(size_t)ci * 4];
                        wv += w * V3<R>(g[0], g[1], g[2]);
                        wm += w * g[3];
                        int32_t sb = lookup_load(ci);
                        if (sb >= 0 && (uint32_t)sb != (uint32_t)bid) {
                            asw += w;
                            R ccy = u.origin.y + (R(cy) + R(0.5)) * u.dx;
                            if (ccy <= pos.y + u.dx * R(0.25)) lasw += w;
                        }
                    }
            if (is_suspended(phase)) {
                R ws = wclamp(wm / wmax(u.nominal_mass * R(2), R(1e-6)), R(0), R(1));
                R drag = wclamp((R(8) + R(18) * ws) * u.dt, R(0), R(1));
                V unsup = pv + brv + V3<R>(R(0), u.gravity * u.dt * R(0.85), R(0));
                R settle = mix(R(1.10), R(0.32), ws);
                V carried = wv + V3<R>(R(0), -settle, R(0));
                V sv = mix(unsup, carried, drag);
                R sp = length(sv);
                if (sp > u.vel_cap) sv = sv * (u.vel_cap / sp);
                V sp_pos = pos + sv * u.dt;
                sdf_contact(sp_pos, sv, true);
                p[0] = sp_pos.x; p[1] = sp_pos.y; p[2] = sp_pos.z;
                p[4] = sv.x; p[5] = sv.y; p[6] = sv.z; p[7] = mp;
                bool anch = lasw > R(0.06) || asw > R(0.20);
                bool dense = asw > R(0.42);
                bool redep = (sp_pos.y <= coffee_filter_floor_y() + u.dx * R(0.35) && ws < R(0.35)) ||
                             (anch && sv.y <= R(0.20) && (ws < R(0.55) || dense));
                if (redep) phase = R(1);
                a[3] = phase;
                a[4] = sp_pos.x; a[5] = sp_pos.y; a[6] = sp_pos.z; a[7] = R(0);
                be[3] *= R(0.985);
                continue;
            }
            R sat = be[7];
            R wl = wclamp(wm / wmax(u.nominal_mass * R(1.5), R(1e-6)), R(0), R(1));
            R wmob = R(1) + sat * R(0.40);
            R mob = wclamp((R(0.30) + wl * R(0.62)) * wmob, R(0), R(1));
            R sfac = wclamp((rest.y + R(u.g.bed_surface_ref_y)) / R(u.g.bed_surface_span), R(0.12), R(1));
            R damping = wclamp(R(1) - u.bed_damping * u.dt, R(0), R(1));
            V vel = pv + brv;
            R srel = wclamp(R(1) - asw / R(0.55), R(0), R(1));
            R ed = wclamp((R(2) + R(5) * sat) * wl * srel * u.dt, R(0), R(0.08));
            V gsv = V3<R>(R(0), -mix(R(0.95), R(0.35), wl), R(0));
            vel = mix(vel, wv + gsv, ed);
            v2<R> lw{wv.x, wv.z};
            R ls = length2(lw);
            v2<R> ldir = ls > R(1e-6) ? v2<R>{lw.x / ls, lw.y / ls} : v2<R>{R(0), R(0)};
            R lss = wmin(ls, std::fabs(wmin(wv.y, R(0))) * R(0.18));
            V iv = V3<R>(ldir.x * lss * R(0.08), wmin(wv.y, R(0)) * R(0.62), ldir.y * lss * R(0.08));
            vel += iv * u.bed_impact * mob * sfac * u.dt;
            int pcx, pcy, pcz;
            world_to_cell(pos, pcx, pcy, pcz);
            V pg = pressure_gradient_at_cell(pcx, pcy, pcz);
            v2<R> sfxz{-pg.x, -pg.z};
            R ssp = length2(sfxz);
            v2<R> sdir = ssp > R(1e-6) ? v2<R>{sfxz.x / ssp, sfxz.y / ssp} : v2<R>{R(0), R(0)};
            R pdrive = wmin(ssp, u.vel_cap / wmax(u.dt, R(1e-6)));
            R pload = wclamp(wm * (R(0.25) + sat), R(0), R(1));
            v2<R> slv{sdir.x * pdrive * pload * R(0.08), sdir.y * pdrive * pload * R(0.08)};
            vel.x += slv.x * u.bed_impact * mob * sfac * u.dt;
            vel.z += slv.y * u.bed_impact * mob * sfac * u.dt;
            vel *= damping;
            V npos = pos + vel * u.dt;
            V off = npos - rest;
            R ll = length2(v2<R>{off.x, off.z});
            R lpt = u.dx * R(0.22);
            if (ll > lpt && ll > R(1e-6)) {
                v2<R> ld{off.x / ll, off.z / ll};
                R lex = ll - lpt;
                R lpl = wclamp((R(0.04) + sat * R(0.35) + mob * R(0.45) + pload * R(0.25)) * sfac *
                                   u.compaction_rate * u.dt,
                               R(0), R(0.18));
                rest.x += ld.x * lex * lpl;
                rest.z += ld.y * lex * lpl;
                off = npos - rest;
            }
            R cll = length2(v2<R>{off.x, off.z});
            R mlat = u.dx * R(0.9) * sfac;
            if (cll > mlat && cll > R(1e-6)) {
                v2<R> ld{off.x / cll, off.z / cll};
                off.x = ld.x * mlat;
                off.z = ld.y * mlat;
                vel.x *= R(0.4);
                vel.z *= R(0.4);
            }
            off.y = wclamp(off.y, -u.dx * (R(1.75) * sfac + R(0.2)), u.dx * R(0.04));
            npos = rest + off;
            coffee_packing(npos, vel, (uint32_t)bid, snap);
            R comp = wmax(rest.y - npos.y, R(0));
            R pth = u.dx * R(0.18);
            if (comp > pth) {
                R ex = comp - pth;
                R pl = wclamp((R(0.05) + sat * R(0.35) + mob * R(0.55)) * sfac * u.compaction_rate * u.dt, R(0), R(0.18));
                rest.y -= ex * pl;
            }
            R floor_y = coffee_filter_floor_y();
            bool hd = sat > R(0.82) && pload > R(0.65) && wl > R(0.65) && srel > R(0.35) &&
                      (comp > u.dx * R(0.65) || cll > u.dx * R(0.65));
            bool fe = sat > R(0.58) && wl > R(0.74) && srel > R(0.55) && length(wv) > R(0.95) &&
                      npos.y > floor_y + u.dx * R(0.70);
            bool iso = sat > R(0.55) && wm < u.nominal_mass * R(0.75) && asw < R(0.04) && lasw < R(0.03) &&
                       npos.y > floor_y + u.dx * R(0.50);
            if (hd || fe || iso) {
                phase = R(2.0);
                rest = npos;
            }
            sdf_contact(npos, vel, true);
            p[0] = npos.x; p[1] = npos.y; p[2] = npos.z;
            p[4] = vel.x; p[5] = vel.y; p[6] = vel.z; p[7] = mp;
            a[3] = phase;
            a[4] = rest.x; a[5] = rest.y; a[6] = rest.z; a[7] = R(0);
            R gc = wmax((rest.y - npos.y) / wmax(u.dx, R(1e-6)), R(0));
            be[3] = wmax(be[3] * R(0.995), gc);
        }
    }
    // shader.rs:2242-2276
    void k_prepare_render() {
        int np = (int)num_particles();
#pragma omp parallel for schedule(static)
        for (int pid = 0; pid < np; ++pid) {
            const R* p = &part[(size_t)pid * 8];
            R phase = aff[(size_t)pid * 12 + 3];
            R* r = &render[(size_t)pid * 8];
            if (p[7] <= inactive_mass_threshold()) {
                r[0] = R(0); r[1] = R(-1e6); r[2] = R(0); r[3] = R(-999.0);
                r[4] = r[5] = r[6] = r[7] = R(0);
                continue;
            }
            R ct = R(0);
            R rad = water_particle_radius();
            if (is_water_phase(phase)) {
                R speed = length(V3<R>(p[4], p[5], p[6]));
                ct = wclamp(speed / R(10), R(0), R(2));
            } else {
                R sat = R(0);
                if ((uint32_t)pid < u.num_bed) {
                    sat = bedx[(size_t)pid * 8 + 7];
                    rad = bed_particle_radius();
                }
                ct = R(-1) - sat;
            }
            r[0] = p[0]; r[1] = p[1]; r[2] = p[2]; r[3] = ct;
            r[4] = rad; r[5] = r[6] = r[7] = R(0);
        }
    }

    // inflow.rs:109-120 (InflowState::update) + flow override extension
    void inflow_update() {
        const CsSpout& sp = settings.spout;
        if (flow_override > 0.0f) {
            flow_rate = flow_override;
            exit_speed = speed_override;
            return;
        }
        float head = effective_head(kettle_angle, sp);
        float cap = exit_speed_cap(kettle_angle, sp);
        exit_speed = exit_speed_from_head(head, cap, settings.standard_gravity_m_s2, settings.sim_units_per_meter);
        flow_rate = flow_rate_from_speed(exit_speed, sp.nozzle_radius, sp.discharge_coeff, sp.volume_to_ml,
                                         sp.max_flow_rate_ml_s);
    }
    // inflow.rs:122-242 (emit_particles)
    void emit(float dt, float particle_mass, uint32_t& emitted, uint32_t& dropped) {
        emitted = dropped = 0;
        inflow_update();
        if (flow_rate < 1e-6f) {
            accumulator = 0.0f;
            return;
        }
        float pps = flow_rate * settings.brew.water_particles_per_ml;
        accumulator += pps * dt;
        uint32_t requested = to_u32((float)accumulator);
        uint32_t count = requested;
        if (count == 0) return;
        accumulator -= (float)count;
        uint32_t total = num_water + num_bed;
        uint32_t avail = settings.max_particles > total ? settings.max_particles - total : 0;
        if (count > avail) count = avail;
        if (count == 0) {
            dropped = requested;
            return;
        }
        const CsSpout& sp = settings.spout;
        float dir[3] = {sp.direction[0], sp.direction[1], sp.direction[2]};
        float up[3] = {0.0f, 1.0f, 0.0f};
        if (!(std::fabs(dir[1]) < 0.9f)) { up[0] = 1.0f; up[1] = 0.0f; }
        float c1[3] = {dir[1] * up[2] - dir[2] * up[1], dir[2] * up[0] - dir[0] * up[2], dir[0] * up[1] - dir[1] * up[0]};
        float t1[3];
        vnormalize(c1, t1);
        float c2[3] = {dir[1] * t1[2] - dir[2] * t1[1], dir[2] * t1[0] - dir[0] * t1[2], dir[0] * t1[1] - dir[1] * t1[0]};
        float t2[3];
        vnormalize(c2, t2);
        float es = exit_speed;
        float vel[3] = {dir[0] * es, dir[1] * es, dir[2] * es};
        float eo[3] = {sp.origin[0] + dir[0] * 0.18f, sp.origin[1] + dir[1] * 0.18f, sp.origin[2] + dir[2] * 0.18f};
        float jr = sp.nozzle_radius * 0.58f;
        const float golden = 2.399963f;
        const float radial_irr = 0.7548777f;
        for (uint32_t i = 0; i < count; ++i) {
            uint32_t sample = emission_sequence + i;
            float sf = (float)sample;
            float ru_raw = (sf + 0.5f) * radial_irr;
            float ru = ru_raw - std::trunc(ru_raw);
            float r = jr * std::sqrt(ru);
            float theta = sf * golden;
            float age = (((float)i + 0.5f) / (float)count) * dt;
            // inflow.rs:205 uses f32 cos/sin; the device emission mode rounds the double-precision
            // values instead (the same on the GPU and here)
            float ct, st;
            if (settings.device_emission) {
                ct = (float)std::cos((double)theta);
                st = (float)std::sin((double)theta);
            } else {
                ct = std::cos(theta);
                st = std::sin(theta);
            }
            float off[3];
            for (int c = 0; c < 3; ++c) off[c] = t1[c] * r * ct + t2[c] * r * st;
            size_t slot = (size_t)total + i;
            R* p = &part[slot * 8];
            for (int c = 0; c < 3; ++c) p[c] = R(eo[c] + off[c] - vel[c] * age);
            p[3] = R(1);
            p[4] = R(vel[0]); p[5] = R(vel[1]); p[6] = R(vel[2]); p[7] = R(particle_mass);
            R* a = &aff[slot * 12];
            for (int c = 0; c < 12; ++c) a[c] = R(0);
        }
        emission_sequence += count;
        emitted = count;
        dropped = requested - count;
    }

    // mod.rs:271-419, one iteration; passes limits how many dispatches run.
    // reorder_every (an engine extension, no reference counterpart): the water samples'
    // slots reordered stably by the 4^3-cell tile of their P2G base cell, samples that
    // deposit nothing last — the same permutation as the engine's radix sort of the keys.
    void reorder_water() {
        const uint32_t n = num_water;
        if (n < 2) return;
        const uint32_t nt[3] = {(u.gx + 1 + 3) / 4, (u.gy + 1 + 3) / 4, (u.gz + 1 + 3) / 4};
        const uint32_t tiles = nt[0] * nt[1] * nt[2];
        auto axis = [](int b, uint32_t ntile) {
            int q = b + 1;
            q = q < 0 ? 0 : q;
            const uint32_t t = (uint32_t)q / 4u;
            return t < ntile ? t : ntile - 1;
        };
        std::vector<uint32_t> key(n), perm(n);
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t pid = num_bed + i;
            const R* p = &part[(size_t)pid * 8];
            const R phase = aff[(size_t)pid * 12 + 3];
            key[i] = tiles;
            if (is_water_phase(phase) && !(p[7] <= inactive_mass_threshold())) {
                const V gp = (V3<R>(p[0], p[1], p[2]) - u.origin) * u.inv_dx;
                const int bx = (int)std::floor(gp.x - R(0.5)), by = (int)std::floor(gp.y - R(0.5)),
                          bz = (int)std::floor(gp.z - R(0.5));
                key[i] = (axis(bz, nt[2]) * nt[1] + axis(by, nt[1])) * nt[0] + axis(bx, nt[0]);
            }
            perm[i] = i;
        }
        std::stable_sort(perm.begin(), perm.end(), [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
        auto permute = [&](std::vector<R>& v, size_t width) {
            std::vector<R> tmp((size_t)n * width);
            for (uint32_t i = 0; i < n; ++i)
                for (size_t k = 0; k < width; ++k) tmp[(size_t)i * width + k] = v[((size_t)num_bed + perm[i]) * width + k];
            std::copy(tmp.begin(), tmp.end(), v.begin() + (size_t)num_bed * width);
        };
        permute(part, 8);
        permute(aff, 12);
        permute(bedx, 8);
    }

    int substep(float sub_dt, uint32_t passes) override {
        const CsSettings& s = settings;
        if (s.reorder_every && substeps_done % s.reorder_every == 0) {
            write_uniforms(R(sub_dt));
            reorder_water();
        }
        ++substeps_done;
        float pm = s.brew.water_mass_units_per_ml / s.brew.water_particles_per_ml;
        uint32_t em = 0, dr = 0;
        emit(sub_dt, pm, em, dr);
        frame_emitted_mass += (float)em * pm;
        frame_dropped += dr;
        total_emitted_mass += (float)em * pm;
        total_dropped += dr;
        num_water += em;
        write_uniforms(R(sub_dt));
        bool warm = s.warm_start != CS_WARM_NONE && !fixed_point() && have_prev_p;
        // clear_buffer(grid), clear_buffer(grid_vel) (mod.rs:308-309)
        std::fill(grid.begin(), grid.end(), 0);
        std::fill(grid64.begin(), grid64.end(), 0);
        std::fill(gvel.begin(), gvel.end(), R(0));
        uint32_t np = num_particles();
        uint32_t pass = 0;
        // Pass numbers are fixed (a pass skipped for an empty bed still takes its number).
        auto run = [&](bool cond) {
            bool go = pass < passes;
            ++pass;
            return go && cond;
        };
        double r0 = -1.0, r1 = -1.0;
        uint32_t sweeps = 0, checks = 0;
        if (run(true)) k_metrics_clear();
        if (run(true)) k_bed_lookup_clear();
        if (run(u.num_bed > 0)) k_bed_lookup_scatter();
        if (run(np > 0)) k_p2g();
        if (run(true)) k_grid_update();
        if (run(true)) k_boundary();
        if (run(true)) k_classify(warm);
        if (run(true)) {
            if (s.solve_mode == CS_SOLVE_RESIDUAL && !fixed_point()) {
                uint32_t ce = s.check_every ? s.check_every : 10;
                r0 = refine_residual();
                r1 = r0;
                checks = 1;
                uint32_t next = s.first_check ? s.first_check : ce;
                while (!(r1 <= (double)s.residual_tol) && sweeps < s.max_sweeps) {
                    uint32_t k = std::min(next, s.max_sweeps - sweeps);
                    for (uint32_t j = 0; j < k; ++j) {
                        refine_sweep(0);
                        refine_sweep(1);
                    }
                    sweeps += k;
                    refine_accumulate();
                    const double r_before = r1;
                    r1 = refine_residual();
                    ++checks;
                    next = next_check_interval(r1, r_before, k, (double)s.residual_tol, ce);
                }
            } else if (s.solve_mode == CS_SOLVE_RESIDUAL) {
                uint32_t ce = s.check_every ? s.check_every : 1;
                r0 = residual();
                r1 = r0;
                checks = 1;
                if (!(r0 <= (double)s.residual_tol)) {
                    while (sweeps < s.max_sweeps) {
                        k_rbgs(0);
                        k_rbgs(1);
                        ++sweeps;
                        if (sweeps % ce == 0 || sweeps == s.max_sweeps) {
                            r1 = residual();
                            ++checks;
                            if (r1 <= (double)s.residual_tol) break;
                        }
                    }
                }
            } else {
                for (uint32_t i = 0; i < s.pressure_rbgs_pairs; ++i) {
                    k_rbgs(0);
                    k_rbgs(1);
                }
                sweeps = s.pressure_rbgs_pairs;
                if (s.check_every) {
                    r1 = residual();
                    checks = 1;
                }
            }
            have_prev_p = true;
        }
        if (run(true)) k_project();
        if (run(true)) k_boundary();
        if (run(true)) k_packing_prepare();
        if (run(true)) k_packing_apply();
        if (run(true)) k_boundary();
        if (run(true)) k_viscosity_prepare();
        if (run(true)) k_viscosity_apply();
        if (run(true)) k_boundary();
        if (run(np > 0)) k_g2p();
        if (run(np > 0)) k_bed_coupling();
        if (run(u.num_bed > 0)) k_extraction_advect();
        if (run(u.num_bed > 0)) k_bed_dynamics();
        if (run(np > 0)) k_prepare_render();
        total_time += sub_dt;
        metrics_out.max_abs_div = (float)metrics[M_MAX_DIV] * (1.0f / METRICS_DIV_FP_SCALE);
        metrics_out.fluid_cells = metrics[M_FLUID];
        metrics_out.div_clamp_fires = metrics[M_DIV_CLAMP];
        metrics_out.pressure_clamp_fires = metrics[M_P_CLAMP];
        metrics_out.mass_overflow_fires = metrics[M_OVERFLOW];
        metrics_out.last_sweeps = sweeps;
        metrics_out.residual_checks = checks;
        metrics_out.last_residual = r1;
        metrics_out.initial_residual = r0;
        return CS_OK;
    }

    void read(int what, uint32_t first, uint32_t count, void* out) override {
        float* f = (float*)out;
        int32_t* i = (int32_t*)out;
        switch (what) {
            case RD_PART: for (size_t k = 0; k < (size_t)count * 8; ++k) f[k] = (float)part[(size_t)first * 8 + k]; break;
            case RD_AFF: for (size_t k = 0; k < (size_t)count * 12; ++k) f[k] = (float)aff[(size_t)first * 12 + k]; break;
            case RD_BEDX: for (size_t k = 0; k < (size_t)count * 8; ++k) f[k] = (float)bedx[(size_t)first * 8 + k]; break;
            case RD_RENDER: for (size_t k = 0; k < (size_t)count * 8; ++k) f[k] = (float)render[(size_t)first * 8 + k]; break;
            case RD_LANES:
                for (size_t k = 0; k < cells * 6; ++k) i[k] = grid[k];
                if (!fixed_point())
                    for (size_t c = 0; c < cells; ++c) i[c] = to_i32((float)pf[c] * FP_SCALE);
                break;
            case RD_GVEL: for (size_t k = 0; k < cells * 4; ++k) f[k] = (float)gvel[k]; break;
            case RD_LANES64:
                for (size_t k = 0; k < grid64.size(); ++k) reinterpret_cast<int64_t*>(out)[k] = grid64[k];
                break;
            case RD_P:
                for (size_t c = 0; c < cells; ++c)
                    f[c] = fixed_point() ? (float)(R(grid[c]) * R(1.0f / FP_SCALE)) : (float)pf[c];
                break;
            case RD_KIND: for (size_t c = 0; c < cells; ++c) i[c] = grid[3 * cells + c]; break;
            case RD_DIV: for (size_t c = 0; c < cells; ++c) f[c] = (float)div_load((uint32_t)c); break;
            case RD_FILL:
                for (size_t c = 0; c < cells; ++c) f[c] = (float)liquid_fill((uint32_t)c, grid[3 * cells + c]);
                break;
            case RD_LOOKUP: for (size_t c = 0; c < cells; ++c) i[c] = lookup[c]; break;
            case RD_DELTA: for (size_t k = 0; k < delta.size(); ++k) i[k] = delta[k]; break;
            case RD_SDF: std::memcpy(out, sdf.data(), sdf.size() * 4); break;
            case RD_CLASS: std::memcpy(out, sdf_class.data(), sdf_class.size()); break;
        }
    }
    void write(int what, uint32_t first, uint32_t count, const void* in) override {
        const float* f = (const float*)in;
        switch (what) {
            case RD_PART: for (size_t k = 0; k < (size_t)count * 8; ++k) part[(size_t)first * 8 + k] = R(f[k]); break;
            case RD_AFF: for (size_t k = 0; k < (size_t)count * 12; ++k) aff[(size_t)first * 12 + k] = R(f[k]); break;
            case RD_BEDX: for (size_t k = 0; k < (size_t)count * 8; ++k) bedx[(size_t)first * 8 + k] = R(f[k]); break;
        }
    }
};

}  // namespace orc

using namespace orc;

struct CsSim {
    std::unique_ptr<SimBase> impl;
    bool metrics_pending = false;
    CsMetrics metrics_req{};
};

static int check_settings(const CsSettings* s) {
    if (!s) return fail(CS_ERR_INVALID_ARG, "settings is null");
    if (s->abi_version != CS_ABI_VERSION) return fail(CS_ERR_INVALID_ARG, "settings.abi_version mismatch");
    for (int a = 0; a < 3; ++a)
        if (s->grid_dims[a] < 1 || s->grid_dims[a] > 1024) return fail(CS_ERR_INVALID_ARG, "grid_dims out of range");
    if (s->max_particles == 0) return fail(CS_ERR_INVALID_ARG, "max_particles must be > 0");
    if (s->num_obstacles > CS_MAX_OBSTACLES) return fail(CS_ERR_INVALID_ARG, "too many obstacles");
    if (s->warm_start != CS_WARM_NONE && s->pressure_storage == CS_PRESSURE_FIXED_POINT)
        return fail(CS_ERR_INVALID_ARG, "warm start needs CS_PRESSURE_FP32 storage");
    return CS_OK;
}

extern "C" {

const char* cs_last_error_string(void) { return g_err.c_str(); }
uint32_t cs_abi_version(void) { return CS_ABI_VERSION; }
int32_t cs_is_gpu_engine(void) { return 0; }

// Oracle-only knobs: arithmetic precision of subsequent cs_create calls and thread count.
int32_t oracle_set_precision(int32_t bits) {
    if (bits != 32 && bits != 64) return fail(CS_ERR_INVALID_ARG, "precision must be 32 or 64");
    g_precision_bits = bits;
    return CS_OK;
}
int32_t oracle_set_threads(int32_t n) {
    g_threads = n;
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#endif
    return CS_OK;
}
int32_t oracle_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int32_t cs_settings_default_v60(CsSettings* out) {
    if (!out) return fail(CS_ERR_INVALID_ARG, "null");
    preset_default_v60(out);
    return CS_OK;
}
int32_t cs_settings_benchmark_free_stream(CsSettings* out) {
    if (!out) return fail(CS_ERR_INVALID_ARG, "null");
    preset_free_stream(out);
    return CS_OK;
}
int32_t cs_settings_benchmark_center_pour(CsSettings* out) {
    if (!out) return fail(CS_ERR_INVALID_ARG, "null");
    preset_center_pour(out);
    return CS_OK;
}
int32_t cs_settings_aim_spout(CsSettings* s, float x, float y, float z) {
    if (!s) return fail(CS_ERR_INVALID_ARG, "null");
    spout_aim_at(s->spout, x, y, z);
    return CS_OK;
}
float cs_kozeny_carman_permeability_m2(float grind_um, float porosity) {
    return kozeny_carman(grind_um, porosity);
}

int32_t cs_create(const CsSettings* settings, CsSim** out) {
    int rc = check_settings(settings);
    if (rc) return rc;
    if (!out) return fail(CS_ERR_INVALID_ARG, "out is null");
    CsSim* s = new CsSim();
    if (g_precision_bits == 64) s->impl.reset(new Sim<double>(*settings));
    else s->impl.reset(new Sim<float>(*settings));
    s->impl->kettle_angle = settings->initial_kettle_angle_deg;
    s->impl->flow_override = settings->flow_override_ml_s;
    s->impl->speed_override = settings->exit_speed_override;
    *out = s;
    return CS_OK;
}
int32_t cs_destroy(CsSim* sim) {
    delete sim;
    return CS_OK;
}
int32_t cs_reset(CsSim* sim) {
    if (!sim) return fail(CS_ERR_INVALID_ARG, "null sim");
    sim->impl->reset_state();
    return CS_OK;
}
int32_t cs_step_frame(CsSim* sim, float dt) {
    if (!sim) return fail(CS_ERR_INVALID_ARG, "null sim");
    SimBase* b = sim->impl.get();
    float fdt = std::fmin(dt, b->settings.max_frame_dt);
    uint32_t sub = b->settings.substeps > 1 ? b->settings.substeps : 1;
    float sdt = fdt / (float)sub;
    b->frame_emitted_mass = 0.0f;
    b->frame_dropped = 0;
    for (uint32_t i = 0; i < sub; ++i) b->substep(sdt, 0xffffffffu);
    return CS_OK;
}
int32_t cs_step_substep(CsSim* sim, float sub_dt) {
    if (!sim) return fail(CS_ERR_INVALID_ARG, "null sim");
    sim->impl->frame_emitted_mass = 0.0f;
    sim->impl->frame_dropped = 0;
    return sim->impl->substep(sub_dt, 0xffffffffu);
}
int32_t cs_step_substep_partial(CsSim* sim, float sub_dt, uint32_t passes) {
    if (!sim) return fail(CS_ERR_INVALID_ARG, "null sim");
    sim->impl->frame_emitted_mass = 0.0f;
    sim->impl->frame_dropped = 0;
    return sim->impl->substep(sub_dt, passes);
}
int32_t cs_set_kettle_angle(CsSim* sim, float a) {
    if (!sim) return fail(CS_ERR_INVALID_ARG, "null sim");
    sim->impl->kettle_angle = a;
    return CS_OK;
}
int32_t cs_set_spout_position(CsSim* sim, float x, float y, float z) {
    if (!sim) return fail(CS_ERR_INVALID_ARG, "null sim");
    spout_translate_origin_to(sim->impl->settings.spout, x, y, z);
    return CS_OK;
}
int32_t cs_set_spout_target(CsSim* sim, float x, float y, float z) {
    if (!sim) return fail(CS_ERR_INVALID_ARG, "null sim");
    spout_aim_at(sim->impl->settings.spout, x, y, z);
    return CS_OK;
}
int32_t cs_set_flow_override(CsSim* sim, float flow, float speed) {
    if (!sim) return fail(CS_ERR_INVALID_ARG, "null sim");
    sim->impl->flow_override = flow > 0.0f ? flow : 0.0f;
    sim->impl->speed_override = flow > 0.0f ? speed : 0.0f;
    return CS_OK;
}
int32_t cs_set_solver(CsSim* sim, float omega, uint32_t check_every, uint32_t max_sweeps) {
    if (!sim) return fail(CS_ERR_INVALID_ARG, "null sim");
    if (omega != 0.0f && !(omega > 0.0f && omega < 2.0f)) return fail(CS_ERR_INVALID_ARG, "omega must lie in (0, 2)");
    CsSettings& s = sim->impl->settings;
    if (omega != 0.0f) s.rbgs_omega = omega;
    if (check_every) s.check_every = check_every;
    if (max_sweeps) s.max_sweeps = max_sweeps;
    return CS_OK;
}
int32_t cs_set_p2g_mode(CsSim* sim, uint32_t mode) {
    if (!sim) return fail(CS_ERR_INVALID_ARG, "null sim");
    if (mode != CS_P2G_ATOMIC32 && mode != CS_P2G_SORTED_SHARED) return fail(CS_ERR_INVALID_ARG, "bad P2G mode");
    sim->impl->settings.p2g_mode = mode;  // the oracle's deposit is order-independent either way
    return CS_OK;
}
int32_t cs_set_graph_mode(CsSim* sim, uint32_t use_graph) {
    if (!sim) return fail(CS_ERR_INVALID_ARG, "null sim");
    sim->impl->settings.use_graph = use_graph ? 1u : 0u;  // nothing to capture on the CPU
    return CS_OK;
}
int32_t cs_set_learned_weights(CsSim*, const float*, uint64_t) {
    return fail(CS_ERR_UNSUPPORTED, "the oracle has no learned warm start (it runs the previous-substep start)");
}
int32_t cs_learned_capture(CsSim*, uint32_t) { return fail(CS_ERR_UNSUPPORTED, "the oracle captures no samples"); }
int32_t cs_learned_read_sample(CsSim*, void*, float*, float*, float*) {
    return fail(CS_ERR_UNSUPPORTED, "the oracle captures no samples");
}
int32_t cs_autotune(CsSim*, float, uint32_t, CsTuneResult*) {
    return fail(CS_ERR_UNSUPPORTED, "the oracle has no autotuner (it times nothing)");
}
int32_t cs_get_counts(const CsSim* sim, uint32_t* nw, uint32_t* nb, uint32_t* mp) {
    if (!sim) return fail(CS_ERR_INVALID_ARG, "null sim");
    if (nw) *nw = sim->impl->num_water;
    if (nb) *nb = sim->impl->num_bed;
    if (mp) *mp = sim->impl->settings.max_particles;
    return CS_OK;
}
int32_t cs_get_kettle_angle(const CsSim* sim, float* out) {
    if (!sim || !out) return fail(CS_ERR_INVALID_ARG, "null");
    *out = sim->impl->kettle_angle;
    return CS_OK;
}
int32_t cs_get_spout_position(const CsSim* sim, float out[3]) {
    if (!sim || !out) return fail(CS_ERR_INVALID_ARG, "null");
    for (int c = 0; c < 3; ++c) out[c] = sim->impl->settings.spout.origin[c];
    return CS_OK;
}
int32_t cs_get_flow(const CsSim* sim, float* fr, float* es, float* esm) {
    if (!sim) return fail(CS_ERR_INVALID_ARG, "null");
    if (fr) *fr = sim->impl->flow_rate;
    if (es) *es = sim->impl->exit_speed;
    if (esm) *esm = sim->impl->exit_speed * (1.0f / sim->impl->settings.sim_units_per_meter);
    return CS_OK;
}
int32_t cs_get_time(const CsSim* sim, float* t) {
    if (!sim || !t) return fail(CS_ERR_INVALID_ARG, "null");
    *t = sim->impl->total_time;
    return CS_OK;
}
int32_t cs_get_emission(const CsSim* sim, float* fem, float* tem, uint32_t* fd, uint32_t* td) {
    if (!sim) return fail(CS_ERR_INVALID_ARG, "null");
    if (fem) *fem = sim->impl->frame_emitted_mass;
    if (tem) *tem = sim->impl->total_emitted_mass;
    if (fd) *fd = sim->impl->frame_dropped;
    if (td) *td = sim->impl->total_dropped;
    return CS_OK;
}
int32_t cs_get_mass_units_per_ml(const CsSim* sim, float* out) {
    if (!sim || !out) return fail(CS_ERR_INVALID_ARG, "null");
    *out = sim->impl->settings.brew.water_mass_units_per_ml;
    return CS_OK;
}
int32_t cs_get_metrics(CsSim* sim, CsMetrics* out) {
    if (!sim || !out) return fail(CS_ERR_INVALID_ARG, "null");
    *out = sim->impl->metrics_out;
    return CS_OK;
}
// the oracle steps synchronously: a request records the metrics, the wait returns them
int32_t cs_metrics_request(CsSim* sim) {
    if (!sim) return fail(CS_ERR_INVALID_ARG, "null");
    if (sim->metrics_pending) return fail(CS_ERR_INVALID_ARG, "a metrics request is already pending");
    sim->metrics_pending = true;
    sim->metrics_req = sim->impl->metrics_out;
    return CS_OK;
}
int32_t cs_metrics_wait(CsSim* sim, CsMetrics* out) {
    if (!sim || !out) return fail(CS_ERR_INVALID_ARG, "null");
    if (!sim->metrics_pending) return fail(CS_ERR_INVALID_ARG, "no metrics request is pending");
    sim->metrics_pending = false;
    *out = sim->metrics_req;
    return CS_OK;
}
int32_t cs_get_settings(const CsSim* sim, CsSettings* out) {
    if (!sim || !out) return fail(CS_ERR_INVALID_ARG, "null");
    *out = sim->impl->settings;
    return CS_OK;
}

static int rd(CsSim* sim, int what, uint32_t first, uint32_t count, void* out) {
    if (!sim || !out) return fail(CS_ERR_INVALID_ARG, "null");
    if ((what == RD_PART || what == RD_AFF || what == RD_BEDX || what == RD_RENDER) &&
        (uint64_t)first + count > sim->impl->settings.max_particles)
        return fail(CS_ERR_INVALID_ARG, "range beyond max_particles");
    sim->impl->read(what, first, count, out);
    return CS_OK;
}
int32_t cs_read_particles(CsSim* s, uint32_t f, uint32_t c, float* o) { return rd(s, RD_PART, f, c, o); }
int32_t cs_read_affine(CsSim* s, uint32_t f, uint32_t c, float* o) { return rd(s, RD_AFF, f, c, o); }
int32_t cs_read_bed_extract(CsSim* s, uint32_t f, uint32_t c, float* o) { return rd(s, RD_BEDX, f, c, o); }
int32_t cs_read_grid_lanes(CsSim* s, int32_t* o) { return rd(s, RD_LANES, 0, 0, o); }
int32_t cs_read_grid_lanes64(CsSim* s, int64_t* o) {
    if (!s) return fail(CS_ERR_INVALID_ARG, "null sim");
    if (s->impl->settings.p2g_mode != CS_P2G_INT64) return fail(CS_ERR_INVALID_ARG, "not an int64 P2G simulation");
    return rd(s, RD_LANES64, 0, 0, o);
}
int32_t cs_read_grid_vel(CsSim* s, float* o) { return rd(s, RD_GVEL, 0, 0, o); }
int32_t cs_read_pressure(CsSim* s, float* o) { return rd(s, RD_P, 0, 0, o); }
int32_t cs_read_cell_kind(CsSim* s, int32_t* o) { return rd(s, RD_KIND, 0, 0, o); }
int32_t cs_read_bed_lookup(CsSim* s, int32_t* o) { return rd(s, RD_LOOKUP, 0, 0, o); }
int32_t cs_read_bed_delta(CsSim* s, int32_t* o) { return rd(s, RD_DELTA, 0, 0, o); }
int32_t cs_read_render(CsSim* s, uint32_t f, uint32_t c, float* o) { return rd(s, RD_RENDER, f, c, o); }
int32_t cs_read_sdf(CsSim* s, float* o) { return rd(s, RD_SDF, 0, 0, o); }
int32_t cs_read_sdf_class(CsSim* s, uint8_t* o) { return rd(s, RD_CLASS, 0, 0, o); }
int32_t cs_read_solver_inputs(CsSim* s, float* fill, float* div) {
    if (!s || !fill || !div) return fail(CS_ERR_INVALID_ARG, "null");
    if (s->impl->settings.pressure_storage == CS_PRESSURE_FIXED_POINT)
        return fail(CS_ERR_UNSUPPORTED, "the solver's divergence array exists in FP32 pressure storage only");
    s->impl->read(RD_FILL, 0, 0, fill);
    s->impl->read(RD_DIV, 0, 0, div);
    return CS_OK;
}

static int wr(CsSim* sim, int what, uint32_t first, uint32_t count, const void* in) {
    if (!sim || !in) return fail(CS_ERR_INVALID_ARG, "null");
    if ((uint64_t)first + count > sim->impl->settings.max_particles)
        return fail(CS_ERR_INVALID_ARG, "range beyond max_particles");
    sim->impl->write(what, first, count, in);
    return CS_OK;
}
int32_t cs_write_particles(CsSim* s, uint32_t f, uint32_t c, const float* i) { return wr(s, RD_PART, f, c, i); }
int32_t cs_write_affine(CsSim* s, uint32_t f, uint32_t c, const float* i) { return wr(s, RD_AFF, f, c, i); }
int32_t cs_write_bed_extract(CsSim* s, uint32_t f, uint32_t c, const float* i) { return wr(s, RD_BEDX, f, c, i); }
int32_t cs_set_counts(CsSim* sim, uint32_t nw, uint32_t nb) {
    if (!sim) return fail(CS_ERR_INVALID_ARG, "null sim");
    if ((uint64_t)nw + nb > sim->impl->settings.max_particles) return fail(CS_ERR_CAPACITY, "counts exceed max_particles");
    sim->impl->num_water = nw;
    sim->impl->num_bed = nb;
    return CS_OK;
}

// Scene generator (no reference counterpart): water block, per_axis^3 samples per cell.
int32_t cs_add_water_block(CsSim* sim, const float lo[3], const float hi[3], uint32_t per_axis, float jitter,
                           uint32_t seed, uint32_t require_open_sdf, uint32_t* added) {
    if (!sim || !lo || !hi || per_axis == 0) return fail(CS_ERR_INVALID_ARG, "bad water block arguments");
    SimBase* b = sim->impl.get();
    const CsSettings& s = b->settings;
    float dx = s.bounds_size[0] / (float)s.grid_dims[0];
    float org[3] = {-s.bounds_size[0] * 0.5f, -s.bounds_size[1] * 0.5f, -s.bounds_size[2] * 0.5f};
    int c0[3], c1[3];
    for (int a = 0; a < 3; ++a) {
        c0[a] = std::max(0, (int)std::floor((lo[a] - org[a]) / dx));
        c1[a] = std::min((int)s.grid_dims[a], (int)std::ceil((hi[a] - org[a]) / dx));
    }
    SplitMix64 rng(seed);
    std::vector<float> pts;
    float n = (float)per_axis;
    for (int iz = c0[2]; iz < c1[2]; ++iz)
        for (int iy = c0[1]; iy < c1[1]; ++iy)
            for (int ix = c0[0]; ix < c1[0]; ++ix)
                for (uint32_t sz = 0; sz < per_axis; ++sz)
                    for (uint32_t sy = 0; sy < per_axis; ++sy)
                        for (uint32_t sx = 0; sx < per_axis; ++sx) {
                            float px = org[0] + ((float)ix + ((float)sx + 0.5f) / n) * dx;
                            float py = org[1] + ((float)iy + ((float)sy + 0.5f) / n) * dx;
                            float pz = org[2] + ((float)iz + ((float)sz + 0.5f) / n) * dx;
                            if (px < lo[0] || px > hi[0] || py < lo[1] || py > hi[1] || pz < lo[2] || pz > hi[2]) continue;
                            float jx = rng.uniform() * 2.0f - 1.0f;
                            float jy = rng.uniform() * 2.0f - 1.0f;
                            float jz = rng.uniform() * 2.0f - 1.0f;
                            px = px + (jx * jitter) * dx;
                            py = py + (jy * jitter) * dx;
                            pz = pz + (jz * jitter) * dx;
                            if (require_open_sdf) {
                                if (!(b->sample_sdf_pub(px, py, pz) > s.geom.contact_offset)) continue;
                            }
                            pts.push_back(px);
                            pts.push_back(py);
                            pts.push_back(pz);
                        }
    uint32_t cnt = (uint32_t)(pts.size() / 3);
    uint32_t total = b->num_water + b->num_bed;
    if ((uint64_t)total + cnt > s.max_particles) return fail(CS_ERR_CAPACITY, "water block exceeds max_particles");
    float pm = s.brew.water_mass_units_per_ml / s.brew.water_particles_per_ml;
    std::vector<float> pbuf((size_t)cnt * 8), abuf((size_t)cnt * 12, 0.0f);
    for (uint32_t i = 0; i < cnt; ++i) {
        float* p = &pbuf[(size_t)i * 8];
        p[0] = pts[(size_t)i * 3];
        p[1] = pts[(size_t)i * 3 + 1];
        p[2] = pts[(size_t)i * 3 + 2];
        p[3] = 1.0f;
        p[4] = p[5] = p[6] = 0.0f;
        p[7] = pm;
    }
    if (cnt) {
        b->write(RD_PART, total, cnt, pbuf.data());
        b->write(RD_AFF, total, cnt, abuf.data());
    }
    b->num_water += cnt;
    if (added) *added = cnt;
    return CS_OK;
}

int32_t cs_snapshot_size(CsSim*, uint64_t*) { return fail(CS_ERR_UNSUPPORTED, "oracle has no snapshots"); }
int32_t cs_snapshot_save(CsSim*, void*, uint64_t) { return fail(CS_ERR_UNSUPPORTED, "oracle has no snapshots"); }
int32_t cs_snapshot_load(CsSim*, const void*, uint64_t) { return fail(CS_ERR_UNSUPPORTED, "oracle has no snapshots"); }

}  // extern "C"

// Timing/profiling entry points: the oracle runs on the host, so the timer is a
// wall clock and the profile only counts substeps.
#include <chrono>
static std::chrono::steady_clock::time_point g_t0;
extern "C" {
int32_t cs_profile_enable(CsSim* s, int32_t) { return s ? CS_OK : fail(CS_ERR_INVALID_ARG, "null sim"); }
int32_t cs_profile_read(CsSim* s, CsProfile* out) {
    if (!s || !out) return fail(CS_ERR_INVALID_ARG, "null");
    std::memset(out, 0, sizeof(*out));
    return CS_OK;
}
int32_t cs_timer_start(CsSim* s) {
    if (!s) return fail(CS_ERR_INVALID_ARG, "null sim");
    g_t0 = std::chrono::steady_clock::now();
    return CS_OK;
}
int32_t cs_timer_stop(CsSim* s, float* ms) {
    if (!s || !ms) return fail(CS_ERR_INVALID_ARG, "null");
    *ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - g_t0).count();
    return CS_OK;
}
int32_t cs_flush_l2(CsSim* s) { return s ? CS_OK : fail(CS_ERR_INVALID_ARG, "null sim"); }
int32_t cs_sync(CsSim* s) { return s ? CS_OK : fail(CS_ERR_INVALID_ARG, "null sim"); }
}

// Host-function probes for the known-answer tests (inflow.rs:244-293, bed.rs:41-82,
// brew_config.rs:92-96).  fn: 0 kozeny_carman(a0 grind um, a1 porosity);
// 1 effective head, speed cap, exit speed, flow rate at angle a0 for settings s;
// 2 exit_speed_from_head(a0 head, a1 cap, s gravity/units);
// 3 flow_rate_from_speed(a0 speed, a1 nozzle, a2 cd, a3 vol_to_ml, a4 max).
// Test-only: the solver's right-hand side input (classify's divergence minus its volume
// target, per cell, as the pressure sweep reads it), valid after a partial substep that
// ran classify.
extern "C" int32_t oracle_read_divergence(CsSim* s, float* out) {
    if (!s || !s->impl || !out) return fail(CS_ERR_INVALID_ARG, "null");
    s->impl->read(RD_DIV, 0, 0, out);
    return CS_OK;
}

extern "C" int32_t oracle_eval(int32_t fn, const CsSettings* s, const float* a, float* out) {
    if (!a || !out) return fail(CS_ERR_INVALID_ARG, "null");
    switch (fn) {
        case 0: out[0] = kozeny_carman(a[0], a[1]); return CS_OK;
        case 1:
            if (!s) return fail(CS_ERR_INVALID_ARG, "null settings");
            out[0] = effective_head(a[0], s->spout);
            out[1] = exit_speed_cap(a[0], s->spout);
            out[2] = exit_speed_from_head(out[0], out[1], s->standard_gravity_m_s2, s->sim_units_per_meter);
            out[3] = flow_rate_from_speed(out[2], s->spout.nozzle_radius, s->spout.discharge_coeff,
                                          s->spout.volume_to_ml, s->spout.max_flow_rate_ml_s);
            return CS_OK;
        case 2:
            out[0] = exit_speed_from_head(a[0], a[1], s ? s->standard_gravity_m_s2 : 9.80665f,
                                          s ? s->sim_units_per_meter : Units::sim_units_per_meter());
            return CS_OK;
        case 3: out[0] = flow_rate_from_speed(a[0], a[1], a[2], a[3], a[4]); return CS_OK;
    }
    return fail(CS_ERR_INVALID_ARG, "unknown probe");
}

// BedConfig::seated_in_filter (bed.rs:41-82) for an arbitrary filter.
extern "C" int32_t oracle_bed_seated(const CsFilter* f, CsBed* out) {
    if (!f || !out) return fail(CS_ERR_INVALID_ARG, "null");
    *out = bed_seated_in_filter(*f);
    return CS_OK;
}
