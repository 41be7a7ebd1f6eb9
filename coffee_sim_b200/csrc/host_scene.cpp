// host_scene.cpp — see host_scene.h.  Reference paths are relative to
// crates/sim-wasm/src/mpm_3d/.
#include "host_scene.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>

namespace cs {
namespace host {

namespace {

// crates/sim-core/src/math.rs:41-48 and 83-92: normalising divides unless |len| <= 1e-6.
void normalized(const float v[3], float out[3]) {
    float len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (len <= 1.0e-6f) {
        out[0] = out[1] = out[2] = 0.0f;
        return;
    }
    out[0] = v[0] / len;
    out[1] = v[1] / len;
    out[2] = v[2] / len;
}
void cross(const float a[3], const float b[3], float out[3]) {
    out[0] = a[1] * b[2] - a[2] * b[1];
    out[1] = a[2] * b[0] - a[0] * b[2];
    out[2] = a[0] * b[1] - a[1] * b[0];
}
float clampf(float x, float lo, float hi) { return std::fmin(std::fmax(x, lo), hi); }

// bed.rs:84-91
void ordered(float a, float b, float& lo, float& hi) {
    if (a <= b) {
        lo = a;
        hi = b;
    } else {
        lo = hi = (a + b) * 0.5f;
    }
}
// filter.rs:28-38
float filter_radius(const CsFilter& f, float y) {
    float h = std::fmax(f.top_y - f.bot_y, 1e-6f);
    float t = clampf((y - f.bot_y) / h, 0.0f, 1.0f);
    return f.bot_radius + (f.top_radius - f.bot_radius) * t;
}
float filter_inner_radius(const CsFilter& f, float y) {
    return std::fmax(filter_radius(f, y) - f.thickness, f.hole_radius);
}

struct SplitMix {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    float unit24() { return (float)(next() >> 40) * (1.0f / 16777216.0f); }
    double unit53_open() { return ((double)(next() >> 11) + 1.0) * (1.0 / 9007199254740992.0); }
};

}  // namespace

float units_per_meter_v60() {
    float filter_height_units = 2.75f - (-3.02f);  // units.rs:11
    return filter_height_units / 0.10f;            // units.rs:17-18
}

float kozeny_carman_m2(float grind_um, float porosity) {
    float d = grind_um * 1.0e-6f;
    float s = 1.0f - porosity;
    return d * d * porosity * porosity * porosity / (180.0f * s * s);
}

void spout_aim_at(CsSpout& sp, float x, float y, float z) {
    sp.target[0] = x;
    sp.target[1] = y;
    sp.target[2] = z;
    float d[3] = {x - sp.origin[0], y - sp.origin[1], z - sp.origin[2]};
    if (std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) > 1e-5f) normalized(d, sp.direction);
}

void spout_translate_origin_to(CsSpout& sp, float x, float y, float z) {
    float d[3] = {x - sp.origin[0], y - sp.origin[1], z - sp.origin[2]};
    sp.origin[0] = x;
    sp.origin[1] = y;
    sp.origin[2] = z;
    for (int c = 0; c < 3; ++c) sp.target[c] = sp.target[c] + d[c];
}

static CsBed seated_bed(const CsFilter& fil) {
    // BedConfig::default (bed.rs:20-38) then seated_in_filter (bed.rs:41-82).
    CsBed b;
    std::memset(&b, 0, sizeof(b));
    for (int c = 0; c < 3; ++c) b.center[c] = fil.center[c];
    b.num_particles = 12000;
    b.initial_porosity = 0.40f;
    b.initial_permeability = kozeny_carman_m2(450.0f, 0.40f);
    b.extractable_mass = 0.15f;
    b.layer_split_y = -1.0e30f;
    b.lower_porosity_scale = 1.0f;
    b.lower_permeability_scale = 1.0f;
    float f_bot = fil.center[1] + fil.bot_y;
    float f_top = fil.center[1] + fil.top_y;
    float lo, hi;
    ordered(f_bot + 0.6f, f_top - 0.35f, lo, hi);
    float top_abs = clampf(b.center[1] + 0.45f, lo, hi);
    ordered(f_bot + 0.4f, top_abs - 1.4f, lo, hi);
    float bot_abs = clampf(b.center[1] + -2.70f, lo, hi);
    b.top_y = top_abs - b.center[1];
    b.bot_y = bot_abs - b.center[1];
    ordered(fil.hole_radius + 0.8f, fil.top_radius - fil.thickness - 0.1f, lo, hi);
    b.top_radius = clampf(filter_inner_radius(fil, top_abs - fil.center[1]) - 0.18f, lo, hi);
    ordered(fil.hole_radius + 0.14f, b.top_radius - 0.25f, lo, hi);
    b.bot_radius = clampf(filter_inner_radius(fil, bot_abs - fil.center[1]) - 0.12f, lo, hi);
    return b;
}

void preset_default_v60(CsSettings* s) {
    std::memset(s, 0, sizeof(*s));
    s->abi_version = CS_ABI_VERSION;
    const float upm = units_per_meter_v60();
    // mod.rs:107-143
    s->bounds_size[0] = 14.0f;
    s->bounds_size[1] = 20.0f;
    s->bounds_size[2] = 14.0f;
    const uint32_t gx = 80;
    const float dx = s->bounds_size[0] / (float)gx;
    s->grid_dims[0] = gx;
    s->grid_dims[1] = (uint32_t)std::ceil(s->bounds_size[1] / dx);
    s->grid_dims[2] = 80;
    s->max_particles = 220000;
    s->substeps = 10;
    s->gravity = -9.80665f * upm;          // units.rs:24
    s->bulk_modulus = 900.0f;
    s->viscosity = 1.2f;                   // brew_config.rs:55
    s->render_radius = dx * 0.7f;
    s->pressure_rbgs_pairs = 40;
    s->use_sdf_cache = 1;
    // filter.rs:14-26
    CsFilter& f = s->filter;
    f.center[0] = 0.0f;
    f.center[1] = -0.35f;
    f.center[2] = 0.0f;
    f.top_y = 2.75f;
    f.bot_y = -3.02f;
    f.top_radius = 4.10f;
    f.bot_radius = 0.0f;
    f.thickness = 0.08f;
    f.hole_radius = 0.0f;
    s->has_filter = 1;
    // mod.rs:163-177 support cone + carafe cylinder
    const float outlet = 0.42f;  // brew_config.rs:64
    float slope = (f.top_radius - f.bot_radius) / std::fmax(f.top_y - f.bot_y, 1e-6f);
    s->num_obstacles = 2;
    CsObstacle& cone = s->obstacles[0];
    cone.kind = CS_OBSTACLE_TRUNCATED_CONE;
    cone.top_y = 3.0f;
    cone.bot_y = -3.0f;
    cone.bot_radius = outlet;
    cone.top_radius = outlet + slope * (cone.top_y - cone.bot_y);
    CsObstacle& cup = s->obstacles[1];
    cup.kind = CS_OBSTACLE_CYLINDER;
    cup.radius = 3.0f;
    cup.top_y = -3.5f;
    cup.bot_y = -8.0f;
    // inflow.rs:27-47
    CsSpout& sp = s->spout;
    sp.origin[0] = -3.4f;
    sp.origin[1] = 7.3f;
    sp.origin[2] = 0.9f;
    const float dir0[3] = {0.36f, -0.92f, -0.12f};
    normalized(dir0, sp.direction);
    sp.target[0] = -0.7f;
    sp.target[1] = 0.4f;
    sp.target[2] = 0.0f;
    sp.nozzle_radius = 0.18f;
    sp.stem_radius = 0.24f;
    sp.activation_angle_deg = 8.0f;
    sp.full_flow_angle_deg = 56.0f;
    sp.head_at_activation = 0.04f;
    sp.head_at_full_angle = 24.0f;
    sp.discharge_coeff = 0.92f;
    float mpu = 1.0f / upm;
    sp.volume_to_ml = mpu * mpu * mpu * 1000000.0f;  // units.rs:19-20
    sp.max_flow_rate_ml_s = 12.0f;
    sp.gentle_exit_speed = 0.12f * upm;               // units.rs:30-32
    sp.max_exit_speed = 0.45f * upm;
    sp.stem_length = 1.9f;
    s->initial_kettle_angle_deg = 9.0f;
    s->has_bed = 1;
    s->bed = seated_bed(f);
    // brew_config.rs:38-71
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
    b.dripper_outlet_radius = outlet;
    b.filter_absorption_rate_s = 0.0f;
    b.bed_compaction_rate = 5.5f;
    b.bed_impact_rate = 8.0f;
    // shader.rs:66, 101, 107, 136-146, 751-819, 1778-1779, 2109; mod.rs:635
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
    s->sim_units_per_meter = upm;
    s->standard_gravity_m_s2 = 9.80665f;
    s->max_velocity = 1.5f * upm;  // units.rs:26-27
    s->particle_volume_cells = 0.25f;
    s->max_frame_dt = 1.0f / 30.0f;
    // engine extensions: reference behaviour by default
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
}

void preset_free_stream(CsSettings* s) {
    preset_default_v60(s);
    s->has_bed = 0;
    s->spout.origin[0] = 0.0f;
    s->spout.origin[1] = 6.8f;
    s->spout.origin[2] = 0.0f;
    spout_aim_at(s->spout, 0.0f, -6.8f, 0.0f);
    s->initial_kettle_angle_deg = 9.0f;
}

void preset_center_pour(CsSettings* s) {
    preset_default_v60(s);
    s->spout.origin[0] = 0.0f;
    s->spout.origin[1] = 7.1f;
    s->spout.origin[2] = 0.0f;
    spout_aim_at(s->spout, 0.0f, 0.4f, 0.0f);
    s->initial_kettle_angle_deg = 9.0f;
}

BedSamples init_bed(const CsBed& cfg, const uint32_t gd[3], const float bounds[3]) {
    BedSamples out;
    const size_t cells = (size_t)gd[0] * gd[1] * gd[2];
    out.lookup.assign(cells, -1);
    const float height = cfg.top_y - cfg.bot_y;
    if (height < 1e-6f) return out;
    // bed.rs:122-129: lattice spacing from the frustum volume
    const float pi = 3.14159265358979323846f;
    float avg = (cfg.top_radius + cfg.bot_radius) * 0.5f;
    float q = cfg.bot_radius / avg;
    float volume = pi * avg * avg * height / 3.0f * (1.0f + cfg.bot_radius / avg + q * q);
    float spacing = std::cbrt(volume / (float)std::max(cfg.num_particles, 1u));
    const int nx = (int)std::ceil((cfg.top_radius * 2.0f) / spacing);
    const int ny = (int)std::ceil(height / spacing);
    const int nz = nx;
    auto key_of = [&](int ix, int iy, int iz) { return ((int64_t)iy * nx + ix) * (int64_t)nz + iz; };

    struct Sample {
        float p[8];
        float a[12];
        float e[8];
        int64_t key;
    };
    std::vector<Sample> all;
    const float y0 = cfg.center[1] + cfg.bot_y;
    for (int iy = 0; iy < ny; ++iy) {
        float base_y = y0 + ((float)iy + 0.5f) * spacing;
        float t = (base_y - y0) / height;
        float max_r = cfg.bot_radius + (cfg.top_radius - cfg.bot_radius) * t;
        for (int ix = 0; ix < nx; ++ix) {
            float x = cfg.center[0] - max_r + ((float)ix + 0.5f) * spacing;
            for (int iz = 0; iz < nz; ++iz) {
                float z = cfg.center[2] - max_r + ((float)iz + 0.5f) * spacing;
                float ex = x - cfg.center[0], ez = z - cfg.center[2];
                float r = std::sqrt(ex * ex + ez * ez);
                if (r > max_r) continue;
                // bed.rs:154-159: lift the rim of the bottom plug
                float cap_t = clampf(t / 0.16f, 0.0f, 1.0f);
                float rt = max_r > 1e-6f ? r / max_r : 0.0f;
                float one_minus = 1.0f - cap_t;
                float lift = spacing * 0.75f * (one_minus * one_minus) * (rt * rt);
                float y = base_y + lift;
                Sample smp = {{x, y, z, 1.0f, 0.0f, 0.0f, 0.0f, 1.0f},
                              {0.0f, 0.0f, 0.0f, 1.0f, x, y, z, 0.0f, y, 0.0f, 0.0f, 0.0f},
                              {0.0f, cfg.initial_porosity, cfg.initial_permeability, 0.0f, cfg.extractable_mass, 0.0f,
                               93.0f, 0.0f},
                              key_of(ix, iy, iz)};
                all.push_back(smp);
            }
        }
    }
    // bed.rs:186-208: even index downsampling to the sample budget
    std::vector<Sample> kept;
    const size_t target = cfg.num_particles;
    if (all.size() > target) {
        const size_t n = all.size();
        kept.reserve(target);
        for (size_t o = 0; o < target; ++o) {
            float v = std::floor((((float)o + 0.5f) * (float)n) / (float)target);
            v = std::fmin(v, (float)(n - 1));
            kept.push_back(all[(size_t)v]);
        }
    } else {
        kept.swap(all);
    }
    std::unordered_map<int64_t, int32_t> slot_of;
    for (size_t i = 0; i < kept.size(); ++i) slot_of[kept[i].key] = (int32_t)i;

    // Log-normal permeability / two-layer bed (extension, no reference counterpart).
    if (cfg.log_perm_sigma > 0.0f || cfg.layer_split_y > -1.0e29f) {
        SplitMix rng{cfg.perm_seed};
        const double ln_k0 = std::log((double)cfg.initial_permeability);
        for (auto& smp : kept) {
            float k = cfg.initial_permeability;
            float phi = cfg.initial_porosity;
            if (cfg.log_perm_sigma > 0.0f) {
                double u1 = rng.unit53_open();
                double u2 = rng.unit53_open();
                double g = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);  // Box-Muller
                k = (float)std::exp(ln_k0 + (double)cfg.log_perm_sigma * g);
            }
            if (smp.p[1] < cfg.layer_split_y) {
                phi = phi * cfg.lower_porosity_scale;
                k = k * cfg.lower_permeability_scale;
            }
            smp.e[1] = phi;
            smp.e[2] = k;
        }
    }

    // bed.rs:228-314: every cell inside the bed frustum points at its nearest lattice sample
    const float ox = -bounds[0] * 0.5f, oy = -bounds[1] * 0.5f, oz = -bounds[2] * 0.5f;
    const float dx = bounds[0] / (float)gd[0];
    for (uint32_t iz = 0; iz < gd[2]; ++iz)
        for (uint32_t iy = 0; iy < gd[1]; ++iy)
            for (uint32_t ix = 0; ix < gd[0]; ++ix) {
                float px = ox + ((float)ix + 0.5f) * dx;
                float py = oy + ((float)iy + 0.5f) * dx;
                float pz = oz + ((float)iz + 0.5f) * dx;
                if (py < y0 || py > cfg.center[1] + cfg.top_y) continue;
                float t = clampf((py - y0) / height, 0.0f, 1.0f);
                float max_r = cfg.bot_radius + (cfg.top_radius - cfg.bot_radius) * t;
                float ex = px - cfg.center[0], ez = pz - cfg.center[2];
                if (std::sqrt(ex * ex + ez * ez) > max_r) continue;
                int gy_ = (int)std::round(((py - y0) / spacing) - 0.5f);
                int gx_ = (int)std::round(((px - (cfg.center[0] - max_r)) / spacing) - 0.5f);
                int gz_ = (int)std::round(((pz - (cfg.center[2] - max_r)) / spacing) - 0.5f);
                int32_t best = -1;
                float best_d2 = INFINITY;
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dxi = -1; dxi <= 1; ++dxi)
                        for (int dzi = -1; dzi <= 1; ++dzi) {
                            int kx = std::clamp(gx_ + dxi, 0, std::max(nx - 1, 0));
                            int ky = std::clamp(gy_ + dy, 0, std::max(ny - 1, 0));
                            int kz = std::clamp(gz_ + dzi, 0, std::max(nz - 1, 0));
                            auto it = slot_of.find(key_of(kx, ky, kz));
                            if (it == slot_of.end()) continue;
                            float sy = y0 + ((float)ky + 0.5f) * spacing;
                            float st = clampf((sy - y0) / height, 0.0f, 1.0f);
                            float sr = cfg.bot_radius + (cfg.top_radius - cfg.bot_radius) * st;
                            float sx = cfg.center[0] - sr + ((float)kx + 0.5f) * spacing;
                            float sz = cfg.center[2] - sr + ((float)kz + 0.5f) * spacing;
                            float ddx = px - sx, ddy = py - sy, ddz = pz - sz;
                            float d2 = ddx * ddx + ddy * ddy + ddz * ddz;
                            if (d2 < best_d2) {
                                best_d2 = d2;
                                best = it->second;
                            }
                        }
                out.lookup[(size_t)iz * gd[0] * gd[1] + (size_t)iy * gd[0] + ix] = best;
            }
    out.count = (uint32_t)kept.size();
    out.particles.reserve(kept.size() * 8);
    out.affines.reserve(kept.size() * 12);
    out.extracts.reserve(kept.size() * 8);
    for (auto& smp : kept) {
        out.particles.insert(out.particles.end(), smp.p, smp.p + 8);
        out.affines.insert(out.affines.end(), smp.a, smp.a + 12);
        out.extracts.insert(out.extracts.end(), smp.e, smp.e + 8);
    }
    return out;
}

// inflow.rs:244-293
static float pour_fraction(float a, const CsSpout& sp) {
    if (a <= sp.activation_angle_deg) return 0.0f;
    if (a >= sp.full_flow_angle_deg) return 1.0f;
    float t = (a - sp.activation_angle_deg) / (sp.full_flow_angle_deg - sp.activation_angle_deg);
    return t * t * (3.0f - 2.0f * t);
}

void Inflow::update(const CsSettings& s) {
    if (flow_override > 0.0f) {
        flow_rate = flow_override;
        exit_speed = speed_override;
        return;
    }
    const CsSpout& sp = s.spout;
    float head;
    if (angle <= sp.activation_angle_deg) head = 0.0f;
    else if (angle >= sp.full_flow_angle_deg) head = sp.head_at_full_angle;
    else head = sp.head_at_activation + pour_fraction(angle, sp) * (sp.head_at_full_angle - sp.head_at_activation);
    float cap = sp.gentle_exit_speed + pour_fraction(angle, sp) * (sp.max_exit_speed - sp.gentle_exit_speed);
    exit_speed = head < 1e-6f ? 0.0f
                              : std::fmin(std::sqrt(2.0f * s.standard_gravity_m_s2 * s.sim_units_per_meter * head), cap);
    if (exit_speed < 1e-6f) {
        flow_rate = 0.0f;
    } else {
        float area = 3.14159265358979323846f * sp.nozzle_radius * sp.nozzle_radius;
        float q = sp.discharge_coeff * area * exit_speed;
        flow_rate = std::fmin(q * sp.volume_to_ml, sp.max_flow_rate_ml_s);
    }
}

uint32_t Inflow::plan(const CsSettings& s, float dt, uint32_t live, uint32_t* dropped) {
    *dropped = 0;
    update(s);
    if (flow_rate < 1e-6f) {
        accumulator = 0.0f;
        return 0;
    }
    accumulator += flow_rate * s.brew.water_particles_per_ml * dt;
    // Rust `f32 as u32` saturates and maps NaN to 0
    uint32_t requested = (accumulator != accumulator || accumulator <= 0.0f) ? 0u
                         : accumulator >= 4294967295.0f                        ? 0xffffffffu
                                                                                : (uint32_t)accumulator;
    if (requested == 0) return 0;
    accumulator -= (float)requested;
    uint32_t avail = s.max_particles > live ? s.max_particles - live : 0u;
    uint32_t count = std::min(requested, avail);
    *dropped = requested - count;
    return count;
}

JetFrame jet_frame(const CsSettings& s, const Inflow& in, float dt, uint32_t count, uint32_t first_slot) {
    JetFrame jf;
    const CsSpout& sp = s.spout;
    const float* d = sp.direction;
    float up[3] = {0.0f, 1.0f, 0.0f};
    if (!(std::fabs(d[1]) < 0.9f)) {
        up[0] = 1.0f;
        up[1] = 0.0f;
    }
    float c[3];
    cross(d, up, c);
    normalized(c, jf.t1);
    cross(d, jf.t1, c);
    normalized(c, jf.t2);
    for (int k = 0; k < 3; ++k) {
        jf.vel[k] = d[k] * in.exit_speed;
        jf.origin[k] = sp.origin[k] + d[k] * 0.18f;  // vena-contracta offset (inflow.rs:185-189)
    }
    jf.jet_radius = sp.nozzle_radius * 0.58f;
    jf.dt = dt;
    jf.particle_mass = s.brew.water_mass_units_per_ml / s.brew.water_particles_per_ml;
    jf.first_sequence = in.sequence;
    jf.count = count;
    jf.first_slot = first_slot;
    return jf;
}

void emit_host(const JetFrame& jf, float* particles, float* affines) {
    const float golden = 2.399963f, radial = 0.7548777f;
    for (uint32_t i = 0; i < jf.count; ++i) {
        float sf = (float)(uint32_t)(jf.first_sequence + i);
        float ru = (sf + 0.5f) * radial;
        ru = ru - std::trunc(ru);  // Rust f32::fract
        float r = jf.jet_radius * std::sqrt(ru);
        float theta = sf * golden;
        float age = (((float)i + 0.5f) / (float)jf.count) * jf.dt;
        float ct = std::cos(theta), st = std::sin(theta);
        float* p = particles + (size_t)i * 8;
        for (int k = 0; k < 3; ++k) {
            float off = jf.t1[k] * r * ct + jf.t2[k] * r * st;
            p[k] = jf.origin[k] + off - jf.vel[k] * age;
        }
        p[3] = 1.0f;
        p[4] = jf.vel[0];
        p[5] = jf.vel[1];
        p[6] = jf.vel[2];
        p[7] = jf.particle_mass;
        std::memset(affines + (size_t)i * 12, 0, 12 * sizeof(float));
    }
}

WaterBlock water_block(const CsSettings& s, const float lo[3], const float hi[3], uint32_t per_axis, float jitter,
                       uint32_t seed) {
    WaterBlock wb;
    const float dx = s.bounds_size[0] / (float)s.grid_dims[0];
    const float org[3] = {-s.bounds_size[0] * 0.5f, -s.bounds_size[1] * 0.5f, -s.bounds_size[2] * 0.5f};
    int a0[3], a1[3];
    for (int a = 0; a < 3; ++a) {
        a0[a] = std::max(0, (int)std::floor((lo[a] - org[a]) / dx));
        a1[a] = std::min((int)s.grid_dims[a], (int)std::ceil((hi[a] - org[a]) / dx));
    }
    SplitMix rng{seed};
    const float n = (float)per_axis;
    for (int iz = a0[2]; iz < a1[2]; ++iz)
        for (int iy = a0[1]; iy < a1[1]; ++iy)
            for (int ix = a0[0]; ix < a1[0]; ++ix)
                for (uint32_t kz = 0; kz < per_axis; ++kz)
                    for (uint32_t ky = 0; ky < per_axis; ++ky)
                        for (uint32_t kx = 0; kx < per_axis; ++kx) {
                            float p[3] = {org[0] + ((float)ix + ((float)kx + 0.5f) / n) * dx,
                                          org[1] + ((float)iy + ((float)ky + 0.5f) / n) * dx,
                                          org[2] + ((float)iz + ((float)kz + 0.5f) / n) * dx};
                            bool inside = true;
                            for (int a = 0; a < 3; ++a) inside = inside && p[a] >= lo[a] && p[a] <= hi[a];
                            if (!inside) continue;
                            for (int a = 0; a < 3; ++a) {
                                float j = rng.unit24() * 2.0f - 1.0f;
                                p[a] = p[a] + (j * jitter) * dx;
                            }
                            wb.xyz.insert(wb.xyz.end(), p, p + 3);
                        }
    return wb;
}

}  // namespace host
}  // namespace cs
