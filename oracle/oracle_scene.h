// oracle_scene.h — host-side scene restatement for the CPU oracle: settings presets,
// SDF / class texture generation, bed initialisation, spout inflow model.
//
// TEST INFRASTRUCTURE (CPU oracle).  Every function cites the reference code it
// restates; paths are relative to crates/sim-wasm/src/mpm_3d/ unless noted.
// All arithmetic is f32 in the order the Rust source writes it (-ffp-contract=off).
#pragma once
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#include "../include/coffee_sim.h"
#include "oracle_math.h"

namespace orc {

// units.rs:9-37 (const f32 arithmetic)
struct Units {
    static float model_filter_height() { return 2.75f - (-3.02f); }
    static float sim_units_per_meter() { return model_filter_height() / 0.10f; }
    static float meters_per_sim_unit() { return 1.0f / sim_units_per_meter(); }
    static float ml_per_sim_unit_cubed() {
        float m = meters_per_sim_unit();
        return m * m * m * 1000000.0f;
    }
    static float std_gravity() { return 9.80665f; }
    static float earth_gravity_sim() { return -std_gravity() * sim_units_per_meter(); }
    static float max_water_speed_sim() { return 1.5f * sim_units_per_meter(); }
    static float gentle_exit_sim() { return 0.12f * sim_units_per_meter(); }
    static float high_exit_sim() { return 0.45f * sim_units_per_meter(); }
};

// brew_config.rs:92-96 (kozeny_carman_permeability_m2)
inline float kozeny_carman(float grind_um, float porosity) {
    float d_m = grind_um * 1.0e-6f;
    float solid = 1.0f - porosity;
    return d_m * d_m * porosity * porosity * porosity / (180.0f * solid * solid);
}

// crates/sim-core/src/math.rs:41-48, 83-92 (Vec3::normalized, Div with EPSILON guard)
inline void vnormalize(const float in[3], float out[3]) {
    float len = std::sqrt(in[0] * in[0] + in[1] * in[1] + in[2] * in[2]);
    if (len <= 1.0e-6f) {
        out[0] = out[1] = out[2] = 0.0f;
    } else if (std::fabs(len) <= 1.0e-6f) {
        out[0] = out[1] = out[2] = 0.0f;
    } else {
        out[0] = in[0] / len;
        out[1] = in[1] / len;
        out[2] = in[2] / len;
    }
}

// filter.rs:14-42
inline float filter_radius_at_y(const CsFilter& f, float y) {
    float height = std::fmax(f.top_y - f.bot_y, 1e-6f);
    float t = std::fmin(std::fmax((y - f.bot_y) / height, 0.0f), 1.0f);
    return f.bot_radius + (f.top_radius - f.bot_radius) * t;
}
inline float filter_inner_radius_at_y(const CsFilter& f, float y) {
    return std::fmax(filter_radius_at_y(f, y) - f.thickness, f.hole_radius);
}

// bed.rs:84-91
inline void order_bounds(float mn, float mx, float& lo, float& hi) {
    if (mn <= mx) { lo = mn; hi = mx; }
    else { float mid = (mn + mx) * 0.5f; lo = mid; hi = mid; }
}
inline float fclampf(float x, float lo, float hi) { return std::fmin(std::fmax(x, lo), hi); }

// bed.rs:20-82 (BedConfig::default + seated_in_filter)
inline CsBed bed_seated_in_filter(const CsFilter& filter) {
    CsBed bed;
    std::memset(&bed, 0, sizeof(bed));
    bed.center[0] = filter.center[0];
    bed.center[1] = filter.center[1];
    bed.center[2] = filter.center[2];
    bed.top_y = 0.45f;
    bed.bot_y = -2.70f;
    bed.top_radius = 2.65f;
    bed.bot_radius = 0.18f;
    bed.num_particles = 12000;
    bed.initial_porosity = 0.40f;
    bed.initial_permeability = kozeny_carman(450.0f, 0.40f);
    bed.extractable_mass = 0.15f;
    bed.log_perm_sigma = 0.0f;
    bed.perm_seed = 0;
    bed.layer_split_y = -1.0e30f;
    bed.lower_porosity_scale = 1.0f;
    bed.lower_permeability_scale = 1.0f;
    // BedConfig::default center is (0,-0.35,0); seated_in_filter copies filter.center.
    float default_center_y = -0.35f;
    float filter_bot_abs = filter.center[1] + filter.bot_y;
    float filter_top_abs = filter.center[1] + filter.top_y;
    float top_min, top_max;
    order_bounds(filter_bot_abs + 0.6f, filter_top_abs - 0.35f, top_min, top_max);
    (void)default_center_y;
    float top_abs = fclampf(bed.center[1] + 0.45f, top_min, top_max);
    float bot_min, bot_max;
    order_bounds(filter_bot_abs + 0.4f, top_abs - 1.4f, bot_min, bot_max);
    float bot_abs = fclampf(bed.center[1] + (-2.70f), bot_min, bot_max);
    bed.top_y = top_abs - bed.center[1];
    bed.bot_y = bot_abs - bed.center[1];
    float top_local = top_abs - filter.center[1];
    float bot_local = bot_abs - filter.center[1];
    float tr_min, tr_max;
    order_bounds(filter.hole_radius + 0.8f, filter.top_radius - filter.thickness - 0.1f, tr_min, tr_max);
    bed.top_radius = fclampf(filter_inner_radius_at_y(filter, top_local) - 0.18f, tr_min, tr_max);
    float br_min, br_max;
    order_bounds(filter.hole_radius + 0.14f, bed.top_radius - 0.25f, br_min, br_max);
    bed.bot_radius = fclampf(filter_inner_radius_at_y(filter, bot_local) - 0.12f, br_min, br_max);
    return bed;
}

// mod.rs:106-143 (MpmSettings::default_v60) with inflow.rs:27-47, filter.rs:14-26,
// brew_config.rs:38-71 and the shader constants of shader.rs:101-146.
inline void preset_default_v60(CsSettings* s) {
    std::memset(s, 0, sizeof(*s));
    s->abi_version = CS_ABI_VERSION;
    s->bounds_size[0] = 14.0f;
    s->bounds_size[1] = 20.0f;
    s->bounds_size[2] = 14.0f;
    uint32_t gx = 80;
    float dx = s->bounds_size[0] / (float)gx;
    uint32_t gy = (uint32_t)std::ceil(s->bounds_size[1] / dx);
    s->grid_dims[0] = gx;
    s->grid_dims[1] = gy;
    s->grid_dims[2] = 80;
    s->max_particles = 220000;
    s->substeps = 10;
    s->gravity = Units::earth_gravity_sim();
    s->bulk_modulus = 900.0f;
    s->viscosity = 1.2f;
    s->render_radius = dx * 0.7f;
    s->pressure_rbgs_pairs = 40;
    s->use_sdf_cache = 1;

    CsFilter f;
    f.center[0] = 0.0f; f.center[1] = -0.35f; f.center[2] = 0.0f;
    f.top_y = 2.75f; f.bot_y = -3.02f; f.top_radius = 4.10f; f.bot_radius = 0.0f;
    f.thickness = 0.08f; f.hole_radius = 0.0f;
    s->has_filter = 1;
    s->filter = f;

    // mod.rs:163-177 (v60_support_cone)
    float top_y = 3.0f, bot_y = -3.0f;
    float filter_height = std::fmax(f.top_y - f.bot_y, 1e-6f);
    float slope = (f.top_radius - f.bot_radius) / filter_height;
    float bot_radius = 0.42f;
    s->num_obstacles = 2;
    s->obstacles[0].kind = CS_OBSTACLE_TRUNCATED_CONE;
    s->obstacles[0].top_radius = bot_radius + slope * (top_y - bot_y);
    s->obstacles[0].bot_radius = bot_radius;
    s->obstacles[0].top_y = top_y;
    s->obstacles[0].bot_y = bot_y;
    s->obstacles[1].kind = CS_OBSTACLE_CYLINDER;
    s->obstacles[1].radius = 3.0f;
    s->obstacles[1].top_y = -3.5f;
    s->obstacles[1].bot_y = -8.0f;

    // inflow.rs:27-47 (SpoutSettings::default)
    CsSpout& sp = s->spout;
    sp.origin[0] = -3.4f; sp.origin[1] = 7.3f; sp.origin[2] = 0.9f;
    float d[3] = {0.36f, -0.92f, -0.12f};
    vnormalize(d, sp.direction);
    sp.target[0] = -0.7f; sp.target[1] = 0.4f; sp.target[2] = 0.0f;
    sp.nozzle_radius = 0.18f;
    sp.stem_radius = 0.24f;
    sp.activation_angle_deg = 8.0f;
    sp.full_flow_angle_deg = 56.0f;
    sp.head_at_activation = 0.04f;
    sp.head_at_full_angle = 24.0f;
    sp.discharge_coeff = 0.92f;
    sp.volume_to_ml = Units::ml_per_sim_unit_cubed();
    sp.max_flow_rate_ml_s = 12.0f;
    sp.gentle_exit_speed = Units::gentle_exit_sim();
    sp.max_exit_speed = Units::high_exit_sim();
    sp.stem_length = 1.9f;
    s->initial_kettle_angle_deg = 9.0f;

    s->has_bed = 1;
    s->bed = bed_seated_in_filter(f);

    CsBrew& b = s->brew;
    b.water_particles_per_ml = 320.0f;
    b.water_mass_units_per_ml = 80.0f;
    b.water_sample_radius_dx = 0.18f;
    b.bed_sample_radius_dx = 0.62f;
    b.water_kinematic_viscosity_m2_s = 1.0e-6f;
    b.min_bed_permeability_m2 = 1.0e-12f;
    b.bed_absorption_rate = 1.6f;
    b.target_bed_retention_ml = 42.0f;
    b.bed_pore_capacity_scale = 1.0f;
    b.bed_pore_overfill_alpha = 18.0f;
    b.bed_surface_void_scale = 1.0f;
    b.dripper_outlet_radius = 0.42f;
    b.filter_absorption_rate_s = 0.0f;
    b.bed_compaction_rate = 5.5f;
    b.bed_impact_rate = 8.0f;

    CsGeometry& g = s->geom;
    g.flags = CS_GEOM_CONE | CS_GEOM_FILTER | CS_GEOM_CUP;
    g.cone_bot_y = -3.0f;
    g.cone_top_y = 3.0f;
    g.cone_radius_span = 4.2634315f;
    g.filter_center_y = -0.35f;
    g.filter_top_rel = 2.75f;
    g.filter_bot_rel = 3.02f;
    g.filter_top_radius = 4.10f;
    g.filter_thickness = 0.08f;
    g.cup_top_y = -3.5f;
    g.cup_radius = 3.0f;
    g.cup_floor_y = -8.0f;
    g.wall_thickness = 0.4f;
    g.bed_surface_ref_y = 3.0f;
    g.bed_surface_span = 3.5f;
    g.sdf_friction = 0.3f;
    g.sdf_restitution = 0.0f;
    g.contact_offset = 0.05f;

    s->sim_units_per_meter = Units::sim_units_per_meter();
    s->standard_gravity_m_s2 = Units::std_gravity();
    s->max_velocity = Units::max_water_speed_sim();
    s->particle_volume_cells = 0.25f;
    s->max_frame_dt = 1.0f / 30.0f;

    s->pressure_storage = CS_PRESSURE_FIXED_POINT;
    s->solve_mode = CS_SOLVE_FIXED_PAIRS;
    s->residual_tol = 1.0e-5f;
    s->max_sweeps = 4000;
    s->check_every = 0;
    s->warm_start = CS_WARM_NONE;
    s->p2g_mode = CS_P2G_ATOMIC32;
    s->sort_every = 1;
    s->device_emission = 0;
    s->use_graph = 0;
    s->device = 0;
    s->rbgs_kernel = 0;
    s->flow_override_ml_s = 0.0f;
    s->exit_speed_override = 0.0f;
}

// inflow.rs:50-60 (SpoutSettings::aim_at)
inline void spout_aim_at(CsSpout& sp, float x, float y, float z) {
    sp.target[0] = x; sp.target[1] = y; sp.target[2] = z;
    float d[3] = {x - sp.origin[0], y - sp.origin[1], z - sp.origin[2]};
    float len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (len > 1e-5f) vnormalize(d, sp.direction);
}
// inflow.rs:62-66 (SpoutSettings::translate_origin_to)
inline void spout_translate_origin_to(CsSpout& sp, float x, float y, float z) {
    float d[3] = {x - sp.origin[0], y - sp.origin[1], z - sp.origin[2]};
    sp.origin[0] = x; sp.origin[1] = y; sp.origin[2] = z;
    sp.target[0] = sp.target[0] + d[0];
    sp.target[1] = sp.target[1] + d[1];
    sp.target[2] = sp.target[2] + d[2];
}

// mod.rs:145-160
inline void preset_free_stream(CsSettings* s) {
    preset_default_v60(s);
    s->has_bed = 0;
    s->spout.origin[0] = 0.0f; s->spout.origin[1] = 6.8f; s->spout.origin[2] = 0.0f;
    spout_aim_at(s->spout, 0.0f, -6.8f, 0.0f);
    s->initial_kettle_angle_deg = 9.0f;
}
inline void preset_center_pour(CsSettings* s) {
    preset_default_v60(s);
    s->spout.origin[0] = 0.0f; s->spout.origin[1] = 7.1f; s->spout.origin[2] = 0.0f;
    spout_aim_at(s->spout, 0.0f, 0.4f, 0.0f);
    s->initial_kettle_angle_deg = 9.0f;
}

// ---- SDF (state.rs:204-344) ----
constexpr int SDF_RES = 128;
constexpr float SDF_NO_CONSTRAINT = 999.0f;

inline float sdf_interior(const CsObstacle& o, float px, float py, float pz) {
    if (o.kind == CS_OBSTACLE_TRUNCATED_CONE) {
        float local_y = py - o.center[1];
        if (local_y > o.top_y || local_y < o.bot_y) return SDF_NO_CONSTRAINT;
        float height = o.top_y - o.bot_y;
        if (height < 1e-10f) return SDF_NO_CONSTRAINT;
        float t = (local_y - o.bot_y) / height;
        float cone_r = o.bot_radius + (o.top_radius - o.bot_radius) * t;
        float dx = px - o.center[0];
        float dz = pz - o.center[2];
        float r = std::sqrt(dx * dx + dz * dz);
        return cone_r - r;
    }
    float local_y = py - o.center[1];
    if (local_y > o.top_y) return SDF_NO_CONSTRAINT;
    float dx = px - o.center[0];
    float dz = pz - o.center[2];
    float r = std::sqrt(dx * dx + dz * dz);
    float radial = o.radius - r;
    float floor_d = local_y - o.bot_y;
    return std::fmin(radial, floor_d);
}

inline std::vector<float> generate_sdf(const CsSettings& s) {
    const int n = SDF_RES;
    std::vector<float> data((size_t)n * n * n, SDF_NO_CONSTRAINT);
    const float* b = s.bounds_size;
    for (uint32_t oi = 0; oi < s.num_obstacles; ++oi) {
        const CsObstacle& o = s.obstacles[oi];
        for (int iz = 0; iz < n; ++iz)
            for (int iy = 0; iy < n; ++iy)
                for (int ix = 0; ix < n; ++ix) {
                    float px = -b[0] * 0.5f + ((float)ix + 0.5f) * b[0] / (float)n;
                    float py = -b[1] * 0.5f + ((float)iy + 0.5f) * b[1] / (float)n;
                    float pz = -b[2] * 0.5f + ((float)iz + 0.5f) * b[2] / (float)n;
                    float sd = sdf_interior(o, px, py, pz) - s.geom.wall_thickness * 0.5f;
                    size_t idx = (size_t)iz * n * n + (size_t)iy * n + ix;
                    if (data[idx] >= SDF_NO_CONSTRAINT - 1.0f) data[idx] = sd;
                    else data[idx] = std::fmax(data[idx], sd);
                }
    }
    return data;
}

// state.rs:287-320: Rust-side trilinear sample (f32::fract = x - trunc(x)).
inline float sample_sdf_rust(const CsSettings& s, const std::vector<float>& d, float px, float py, float pz) {
    const float* b = s.bounds_size;
    float res = (float)SDF_RES;
    float u[3] = {(px + b[0] * 0.5f) / b[0] * res - 0.5f, (py + b[1] * 0.5f) / b[1] * res - 0.5f,
                  (pz + b[2] * 0.5f) / b[2] * res - 0.5f};
    int base[3] = {(int)std::floor(u[0]), (int)std::floor(u[1]), (int)std::floor(u[2])};
    float f[3] = {u[0] - std::trunc(u[0]), u[1] - std::trunc(u[1]), u[2] - std::trunc(u[2])};
    auto tex = [&](int x, int y, int z) {
        int mx = SDF_RES - 1;
        x = std::min(std::max(x, 0), mx);
        y = std::min(std::max(y, 0), mx);
        z = std::min(std::max(z, 0), mx);
        return d[(size_t)z * SDF_RES * SDF_RES + (size_t)y * SDF_RES + x];
    };
    float c000 = tex(base[0], base[1], base[2]);
    float c100 = tex(base[0] + 1, base[1], base[2]);
    float c010 = tex(base[0], base[1] + 1, base[2]);
    float c110 = tex(base[0] + 1, base[1] + 1, base[2]);
    float c001 = tex(base[0], base[1], base[2] + 1);
    float c101 = tex(base[0] + 1, base[1], base[2] + 1);
    float c011 = tex(base[0], base[1] + 1, base[2] + 1);
    float c111 = tex(base[0] + 1, base[1] + 1, base[2] + 1);
    float c00 = c000 + (c100 - c000) * f[0];
    float c10 = c010 + (c110 - c010) * f[0];
    float c01 = c001 + (c101 - c001) * f[0];
    float c11 = c011 + (c111 - c011) * f[0];
    float c0 = c00 + (c10 - c00) * f[1];
    float c1 = c01 + (c11 - c01) * f[1];
    return c0 + (c1 - c0) * f[2];
}

inline std::vector<uint8_t> generate_sdf_class(const CsSettings& s, const std::vector<float>& sdf) {
    uint32_t gx = s.grid_dims[0], gy = s.grid_dims[1], gz = s.grid_dims[2];
    std::vector<uint8_t> out((size_t)gx * gy * gz, 0);
    float dx = s.bounds_size[0] / (float)gx;
    float ox = -s.bounds_size[0] * 0.5f, oy = -s.bounds_size[1] * 0.5f, oz = -s.bounds_size[2] * 0.5f;
    for (uint32_t iz = 0; iz < gz; ++iz)
        for (uint32_t iy = 0; iy < gy; ++iy)
            for (uint32_t ix = 0; ix < gx; ++ix) {
                float cx = ox + ((float)ix + 0.5f) * dx;
                float cy = oy + ((float)iy + 0.5f) * dx;
                float cz = oz + ((float)iz + 0.5f) * dx;
                size_t idx = (size_t)iz * gx * gy + (size_t)iy * gx + ix;
                out[idx] = sample_sdf_rust(s, sdf, cx, cy, cz) < 0.0f ? 1 : 0;
            }
    return out;
}

// ---- bed initialisation (bed.rs:107-314) ----
struct BedInit {
    std::vector<float> particles;  // 8 per sample
    std::vector<float> affines;    // 12 per sample
    std::vector<float> extracts;   // 8 per sample
    std::vector<int32_t> lookup;   // cells
};

inline BedInit init_bed(const CsBed& cfg, const uint32_t gd[3], const float bounds[3]) {
    BedInit out;
    size_t cells = (size_t)gd[0] * gd[1] * gd[2];
    float height = cfg.top_y - cfg.bot_y;
    if (height < 1e-6f) {
        out.lookup.assign(cells, -1);
        return out;
    }
    const float PI = 3.14159265358979323846f;
    float avg_radius = (cfg.top_radius + cfg.bot_radius) * 0.5f;
    float ratio = cfg.bot_radius / avg_radius;
    float volume = PI * avg_radius * avg_radius * height / 3.0f * (1.0f + cfg.bot_radius / avg_radius + ratio * ratio);
    uint32_t nmax = cfg.num_particles > 0 ? cfg.num_particles : 1;
    float spacing = std::cbrt(volume / (float)nmax);
    int nx = (int)std::ceil((cfg.top_radius * 2.0f) / spacing);
    int ny = (int)std::ceil(height / spacing);
    int nz = nx;

    std::vector<std::array<float, 8>> parts;
    std::vector<std::array<float, 12>> affs;
    std::vector<std::array<float, 8>> exts;
    std::vector<std::tuple<int, int, int>> keys;
    std::map<std::tuple<int, int, int>, int> lattice;
    for (int iy = 0; iy < ny; ++iy) {
        float base_y = cfg.center[1] + cfg.bot_y + ((float)iy + 0.5f) * spacing;
        float t = (base_y - (cfg.center[1] + cfg.bot_y)) / height;
        float max_r = cfg.bot_radius + (cfg.top_radius - cfg.bot_radius) * t;
        for (int ix = 0; ix < nx; ++ix) {
            float x = cfg.center[0] - max_r + ((float)ix + 0.5f) * spacing;
            for (int iz = 0; iz < nz; ++iz) {
                float z = cfg.center[2] - max_r + ((float)iz + 0.5f) * spacing;
                float ddx = x - cfg.center[0];
                float ddz = z - cfg.center[2];
                float r = std::sqrt(ddx * ddx + ddz * ddz);
                if (r > max_r) continue;
                float cap_t = fclampf(t / 0.16f, 0.0f, 1.0f);
                float radial_t = max_r > 1e-6f ? r / max_r : 0.0f;
                float omc = 1.0f - cap_t;
                float edge_lift = spacing * 0.75f * (omc * omc) * (radial_t * radial_t);
                float y = base_y + edge_lift;
                int pidx = (int)parts.size();
                lattice[std::make_tuple(ix, iy, iz)] = pidx;
                keys.push_back(std::make_tuple(ix, iy, iz));
                parts.push_back({x, y, z, 1.0f, 0.0f, 0.0f, 0.0f, 1.0f});
                affs.push_back({0.0f, 0.0f, 0.0f, 1.0f, x, y, z, 0.0f, y, 0.0f, 0.0f, 0.0f});
                exts.push_back({0.0f, cfg.initial_porosity, cfg.initial_permeability, 0.0f,
                                cfg.extractable_mass, 0.0f, 93.0f, 0.0f});
            }
        }
    }
    size_t target_n = cfg.num_particles;
    if (parts.size() > target_n) {
        size_t src_len = parts.size();
        std::vector<std::array<float, 8>> sp;
        std::vector<std::array<float, 12>> sa;
        std::vector<std::array<float, 8>> se;
        std::map<std::tuple<int, int, int>, int> sl;
        for (size_t o = 0; o < target_n; ++o) {
            float v = std::floor((((float)o + 0.5f) * (float)src_len) / (float)target_n);
            v = std::fmin(v, (float)(src_len - 1));
            size_t si = (size_t)v;
            sp.push_back(parts[si]);
            sa.push_back(affs[si]);
            se.push_back(exts[si]);
            sl[keys[si]] = (int)o;
        }
        parts.swap(sp);
        affs.swap(sa);
        exts.swap(se);
        lattice.swap(sl);
    }
    // Extension: log-normal permeability and two-layer beds (no reference counterpart).
    if (cfg.log_perm_sigma > 0.0f || cfg.layer_split_y > -1.0e29f) {
        SplitMix64 rng(cfg.perm_seed);
        double mu = std::log((double)cfg.initial_permeability);
        for (size_t i = 0; i < parts.size(); ++i) {
            float k = cfg.initial_permeability;
            float phi = cfg.initial_porosity;
            if (cfg.log_perm_sigma > 0.0f) {
                double u1 = rng.uniform_open();
                double u2 = rng.uniform_open();
                double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
                k = (float)std::exp(mu + (double)cfg.log_perm_sigma * z);
            }
            if (parts[i][1] < cfg.layer_split_y) {
                phi = phi * cfg.lower_porosity_scale;
                k = k * cfg.lower_permeability_scale;
            }
            exts[i][1] = phi;
            exts[i][2] = k;
        }
    }
    // bed.rs:228-314 build_cell_lookup
    out.lookup.assign(cells, -1);
    uint32_t gx = gd[0], gy = gd[1], gz = gd[2];
    float ox = -bounds[0] * 0.5f, oy = -bounds[1] * 0.5f, oz = -bounds[2] * 0.5f;
    float dx = bounds[0] / (float)gx;
    float bed_bottom = cfg.center[1] + cfg.bot_y;
    for (uint32_t iz = 0; iz < gz; ++iz)
        for (uint32_t iy = 0; iy < gy; ++iy)
            for (uint32_t ix = 0; ix < gx; ++ix) {
                float px = ox + ((float)ix + 0.5f) * dx;
                float py = oy + ((float)iy + 0.5f) * dx;
                float pz = oz + ((float)iz + 0.5f) * dx;
                if (py < bed_bottom || py > cfg.center[1] + cfg.top_y) continue;
                float t = fclampf((py - bed_bottom) / height, 0.0f, 1.0f);
                float max_r = cfg.bot_radius + (cfg.top_radius - cfg.bot_radius) * t;
                float dxr = px - cfg.center[0];
                float dzr = pz - cfg.center[2];
                if (std::sqrt(dxr * dxr + dzr * dzr) > max_r) continue;
                int iy_g = (int)std::round(((py - bed_bottom) / spacing) - 0.5f);
                int ix_g = (int)std::round(((px - (cfg.center[0] - max_r)) / spacing) - 0.5f);
                int iz_g = (int)std::round(((pz - (cfg.center[2] - max_r)) / spacing) - 0.5f);
                int best = -1;
                float best_d2 = INFINITY;
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dxi = -1; dxi <= 1; ++dxi)
                        for (int dzi = -1; dzi <= 1; ++dzi) {
                            int kx = std::min(std::max(ix_g + dxi, 0), std::max(nx - 1, 0));
                            int ky = std::min(std::max(iy_g + dy, 0), std::max(ny - 1, 0));
                            int kz = std::min(std::max(iz_g + dzi, 0), std::max(nz - 1, 0));
                            auto it = lattice.find(std::make_tuple(kx, ky, kz));
                            if (it == lattice.end()) continue;
                            float qy = bed_bottom + ((float)ky + 0.5f) * spacing;
                            float qt = fclampf((qy - bed_bottom) / height, 0.0f, 1.0f);
                            float qr = cfg.bot_radius + (cfg.top_radius - cfg.bot_radius) * qt;
                            float qx = cfg.center[0] - qr + ((float)kx + 0.5f) * spacing;
                            float qz = cfg.center[2] - qr + ((float)kz + 0.5f) * spacing;
                            float ex = px - qx, ey = py - qy, ez = pz - qz;
                            float d2 = ex * ex + ey * ey + ez * ez;
                            if (d2 < best_d2) {
                                best_d2 = d2;
                                best = it->second;
                            }
                        }
                out.lookup[(size_t)iz * gx * gy + (size_t)iy * gx + ix] = best;
            }
    for (auto& p : parts) out.particles.insert(out.particles.end(), p.begin(), p.end());
    for (auto& a : affs) out.affines.insert(out.affines.end(), a.begin(), a.end());
    for (auto& e : exts) out.extracts.insert(out.extracts.end(), e.begin(), e.end());
    return out;
}

// ---- inflow (inflow.rs:244-293) ----
inline float pour_fraction(float angle, const CsSpout& sp) {
    if (angle <= sp.activation_angle_deg) return 0.0f;
    if (angle >= sp.full_flow_angle_deg) return 1.0f;
    float t = (angle - sp.activation_angle_deg) / (sp.full_flow_angle_deg - sp.activation_angle_deg);
    return t * t * (3.0f - 2.0f * t);
}
inline float effective_head(float angle, const CsSpout& sp) {
    if (angle <= sp.activation_angle_deg) return 0.0f;
    if (angle >= sp.full_flow_angle_deg) return sp.head_at_full_angle;
    float s = pour_fraction(angle, sp);
    return sp.head_at_activation + s * (sp.head_at_full_angle - sp.head_at_activation);
}
inline float exit_speed_cap(float angle, const CsSpout& sp) {
    float s = pour_fraction(angle, sp);
    return sp.gentle_exit_speed + s * (sp.max_exit_speed - sp.gentle_exit_speed);
}
inline float exit_speed_from_head(float head, float max_exit, float std_g, float upm) {
    if (head < 1e-6f) return 0.0f;
    float speed = std::sqrt(2.0f * std_g * upm * head);
    return std::fmin(speed, max_exit);
}
inline float flow_rate_from_speed(float speed, float nozzle_r, float cd, float vol_to_ml, float max_flow) {
    if (speed < 1e-6f) return 0.0f;
    float area = 3.14159265358979323846f * nozzle_r * nozzle_r;
    float q = cd * area * speed;
    return std::fmin(q * vol_to_ml, max_flow);
}

}  // namespace orc
