// kernels.cuh — device functions of the MLS-MPM substep: grid-lane access with the
// reference's aliasing, SDF sampling, contact, bed helpers.  Each function cites the
// WGSL it reproduces (crates/sim-wasm/src/mpm_3d/shader.rs).
#pragma once
#include "cs_device.cuh"

namespace cs {

// ---- grid lanes (shader.rs:152-164, 194-291) ----
__device__ __forceinline__ int32_t* lane(const Ctx& c, int l) { return c.lanes + (size_t)l * c.u.cells; }
__device__ __forceinline__ int32_t kind_load(const Ctx& c, uint32_t i) { return lane(c, 3)[i]; }

__device__ __forceinline__ float pressure_load(const Ctx& c, uint32_t i) {
    return c.u.fixed_point ? (float)lane(c, 0)[i] * INV_FP_SCALE : c.pf[i];
}
__device__ __forceinline__ void pressure_store(const Ctx& c, uint32_t i, float v) {
    float lim = c.u.p_limit;
    float cl = wclamp(v, -lim, lim);
    if (cl != v) atomicAdd(&c.metrics[M_P_CLAMP], 1u);
    if (c.u.fixed_point) lane(c, 0)[i] = to_i32(cl * FP_SCALE);
    else c.pf[i] = cl;
}
__device__ __forceinline__ float div_load(const Ctx& c, uint32_t i) {
    return c.u.fixed_point ? (float)lane(c, 1)[i] * INV_FP_SCALE : c.divf[i];
}
__device__ __forceinline__ void div_store(const Ctx& c, uint32_t i, float v) {
    float lim = c.u.div_clamp;
    float cl = wclamp(v, -lim, lim);
    if (cl != v) atomicAdd(&c.metrics[M_DIV_CLAMP], 1u);
    if (c.u.fixed_point) lane(c, 1)[i] = to_i32(cl * FP_SCALE);
    else c.divf[i] = cl;
}
__device__ __forceinline__ float packing_load(const Ctx& c, uint32_t i) { return (float)lane(c, 2)[i] * INV_FP_SCALE; }
__device__ __forceinline__ void packing_store(const Ctx& c, uint32_t i, float v) {
    float lim = c.u.p_clamp;
    float cl = wclamp(v, 0.0f, lim);
    if (cl != v) atomicAdd(&c.metrics[M_P_CLAMP], 1u);
    lane(c, 2)[i] = to_i32(cl * FP_SCALE);
}
__device__ __forceinline__ f3 vscratch_load(const Ctx& c, uint32_t i) {
    return mk((float)lane(c, 1)[i] * INV_FP_SCALE, (float)lane(c, 2)[i] * INV_FP_SCALE, (float)lane(c, 3)[i] * INV_FP_SCALE);
}
__device__ __forceinline__ void vscratch_store(const Ctx& c, uint32_t i, f3 v) {
    float sp = len3(v);
    if (sp > c.u.vel_cap) v = v * (c.u.vel_cap / sp);
    lane(c, 1)[i] = to_i32(v.x * FP_SCALE);
    lane(c, 2)[i] = to_i32(v.y * FP_SCALE);
    lane(c, 3)[i] = to_i32(v.z * FP_SCALE);
}
// P2G lanes 0-5: i32 * 2^18 (the reference), or i64 * 2^32 in the int64 mode
__device__ __forceinline__ float p2g_lane(const Ctx& c, int l, uint32_t i) {
    if (c.u.int64_grid) return (float)c.lanes64[(size_t)l * c.u.cells + i] * INV_FP_SCALE64;
    return (float)lane(c, l)[i] * INV_FP_SCALE;
}
__device__ __forceinline__ float rest_vol(const Ctx& c, uint32_t i) { return p2g_lane(c, 4, i); }
__device__ __forceinline__ float cur_vol(const Ctx& c, uint32_t i) { return p2g_lane(c, 5, i); }

// shader.rs:293-304; evaluated once per cell by classify and stored in c.fill
__device__ __forceinline__ float liquid_fill_of(const Params& u, int32_t kind, float rest, float cur) {
    if (kind == CELL_INTERIOR || kind == CELL_BED) return 1.0f;
    if (kind != CELL_SURFACE) return 0.0f;
    float cv = wmax(u.dx * u.dx * u.dx, 1e-8f);
    return wclamp(wmax(rest, cur) / cv, 0.0f, 1.0f);
}
__device__ __forceinline__ float liquid_fill(const Ctx& c, uint32_t i, int32_t kind) {
    if (kind != CELL_SURFACE) return liquid_fill_of(c.u, kind, 0.0f, 0.0f);
    return liquid_fill_of(c.u, kind, rest_vol(c, i), cur_vol(c, i));
}
// shader.rs:306-323 with the neighbour's fill read from c.fill
__device__ __forceinline__ float face_weight(int32_t sk, float sf, int32_t nk, float nfill) {
    if (is_solid(nk)) return 0.0f;
    if (sk == CELL_BED || nk == CELL_BED) return 1.0f;
    if (!is_fluid(nk)) return sf;
    return wmin(sf, nfill);
}

// ---- derived uniforms (shader.rs:101-146) ----
__device__ __forceinline__ float wall_half(const Params& u) { return u.wall_thickness * 0.5f; }
__device__ __forceinline__ float bed_particle_radius(const Params& u) { return u.dx * u.bed_r_dx; }
__device__ __forceinline__ float water_particle_radius(const Params& u) { return u.dx * u.water_r_dx; }
__device__ __forceinline__ float inactive_mass(const Params& u) { return u.nominal_mass * 0.10f; }
__device__ __forceinline__ float occupancy_mass(const Params& u) { return u.nominal_mass * 0.1f; }
__device__ __forceinline__ float clamp_j(float v) { return wclamp(v, 0.40f, 2.00f); }
__device__ __forceinline__ float filter_top_y(const Params& u) { return u.filter_center_y + u.filter_top_rel; }
__device__ __forceinline__ float filter_bot_y(const Params& u) { return u.filter_center_y - u.filter_bot_rel; }
__device__ __forceinline__ float coffee_floor_y(const Params& u) {
    float ftop = filter_top_y(u), fbot = filter_bot_y(u);
    float bco = wmax(u.contact_offset, bed_particle_radius(u));
    float slope = u.filter_top_radius / wmax(ftop - fbot, 1e-6f);
    return fbot + (bco + u.filter_thickness) / wmax(slope, 1e-6f);
}

// ---- SDF (shader.rs:673-715); texels read through the read-only path ----
__device__ __forceinline__ float sdf_texel(const Ctx& c, int x, int y, int z) {
    x = min(max(x, 0), SDF_RES - 1);
    y = min(max(y, 0), SDF_RES - 1);
    z = min(max(z, 0), SDF_RES - 1);
    return __ldg(c.sdf + ((size_t)z * SDF_RES + y) * SDF_RES + x);
}
__device__ __forceinline__ float sample_sdf(const Ctx& c, f3 p) {
    const Params& u = c.u;
    float bsx = u.bx * 2.0f, bsy = u.by * 2.0f, bsz = u.bz * 2.0f;
    const float res = (float)SDF_RES;
    float ux = (p.x + u.bx) / bsx * res - 0.5f;
    float uy = (p.y + u.by) / bsy * res - 0.5f;
    float uz = (p.z + u.bz) / bsz * res - 0.5f;
    float flx = floorf(ux), fly = floorf(uy), flz = floorf(uz);
    int x = (int)flx, y = (int)fly, z = (int)flz;
    float fx = ux - flx, fy = uy - fly, fz = uz - flz;
    float c000 = sdf_texel(c, x, y, z), c100 = sdf_texel(c, x + 1, y, z);
    float c010 = sdf_texel(c, x, y + 1, z), c110 = sdf_texel(c, x + 1, y + 1, z);
    float c001 = sdf_texel(c, x, y, z + 1), c101 = sdf_texel(c, x + 1, y, z + 1);
    float c011 = sdf_texel(c, x, y + 1, z + 1), c111 = sdf_texel(c, x + 1, y + 1, z + 1);
    float c00 = mixf(c000, c100, fx), c10 = mixf(c010, c110, fx);
    float c01 = mixf(c001, c101, fx), c11 = mixf(c011, c111, fx);
    float c0 = mixf(c00, c10, fy), c1 = mixf(c01, c11, fy);
    return mixf(c0, c1, fz);
}
__device__ __forceinline__ f3 sdf_gradient(const Ctx& c, f3 p) {
    float e = c.u.dx;
    float gx = sample_sdf(c, p + mk(e, 0.0f, 0.0f)) - sample_sdf(c, p - mk(e, 0.0f, 0.0f));
    float gy = sample_sdf(c, p + mk(0.0f, e, 0.0f)) - sample_sdf(c, p - mk(0.0f, e, 0.0f));
    float gz = sample_sdf(c, p + mk(0.0f, 0.0f, e)) - sample_sdf(c, p - mk(0.0f, 0.0f, e));
    f3 g = mk(gx, gy, gz);
    float l = len3(g);
    if (l < 1e-8f) return mk(0.0f, 0.0f, 0.0f);
    return g / l;
}

// ---- contact (shader.rs:717-903) ----
__device__ __forceinline__ void radial_barrier(const Params& u, f3& pos, f3& vel, float max_r) {
    float rx = pos.x, rz = pos.z;  // centre (0,0)
    float r = len2(rx, rz);
    if (r > max_r && r > 1e-6f) {
        float ox = rx / r, oz = rz / r;
        pos.x = 0.0f + ox * max_r;
        pos.z = 0.0f + oz * max_r;
        float vn = vel.x * ox + vel.z * oz;
        if (vn > 0.0f) {
            float tx = vel.x - ox * vn, tz = vel.z - oz * vn;
            vel.x = tx * (1.0f - u.friction * 0.35f);
            vel.z = tz * (1.0f - u.friction * 0.35f);
        }
    }
}
__device__ __forceinline__ void scene_obstacles(const Params& u, f3& pos, f3& vel, bool is_bed) {
    if (u.geom_flags & CS_GEOM_CONE) {
        if (pos.y <= u.cone_top_y && pos.y >= u.cone_bot_y) {
            float t = wclamp((pos.y - u.cone_bot_y) / (u.cone_top_y - u.cone_bot_y), 0.0f, 1.0f);
            radial_barrier(u, pos, vel, mixf(u.outlet_r, u.top_r, t) - u.contact_offset);
        }
    }
    if ((u.geom_flags & CS_GEOM_FILTER) && is_bed) {
        float ftop = filter_top_y(u), fbot = filter_bot_y(u);
        float bco = wmax(u.contact_offset, bed_particle_radius(u));
        float floor_y = coffee_floor_y(u);
        if (pos.y <= ftop && pos.y >= fbot) {
            float ft = wclamp((pos.y - fbot) / (ftop - fbot), 0.0f, 1.0f);
            float outer = mixf(0.0f, u.filter_top_radius, ft);
            float fr = wmax(outer - u.filter_thickness, 0.0f) - bco;
            radial_barrier(u, pos, vel, wmax(fr, 0.0f));
        }
        if (pos.y <= floor_y) {
            pos.y = floor_y;
            pos.x = 0.0f;
            pos.z = 0.0f;
            const float k = 1.0f - u.friction * 0.55f;
            if (vel.y < 0.0f) {
                vel.y = 0.0f;
                vel.x *= k;
                vel.z *= k;
            }
            vel.x *= k;
            vel.z *= k;
        }
    }
    if (u.geom_flags & CS_GEOM_CUP) {
        if (pos.y <= u.cup_top_y) {
            radial_barrier(u, pos, vel, u.cup_radius - wall_half(u) - u.contact_offset);
            float fy = u.cup_floor_y + wall_half(u) + u.contact_offset;
            if (pos.y < fy) {
                pos.y = fy;
                if (vel.y < 0.0f) {
                    const float k = 1.0f - u.friction * 0.55f;
                    vel.y = 0.0f;
                    vel.x *= k;
                    vel.z *= k;
                }
            }
        }
    }
}
__device__ __forceinline__ void sdf_contact(const Ctx& c, f3& pos, f3& vel, bool is_bed) {
    const Params& u = c.u;
    float sv = sample_sdf(c, pos);
    if (sv < u.contact_offset) {
        f3 n = sdf_gradient(c, pos);
        if (len3(n) > 1e-6f) {
            pos += n * (u.contact_offset - sv);
            float vn = dot3(vel, n);
            if (vn < 0.0f) {
                vel = vel - n * vn * (1.0f + u.restitution);
                f3 vt = vel - n * dot3(vel, n);
                float vtl = len3(vt);
                if (vtl > 1e-6f) {
                    float fi = wmin(u.friction * fabsf(vn), vtl);
                    vel = vel - vt * (fi / vtl);
                }
            }
        }
    }
    scene_obstacles(u, pos, vel, is_bed);
}
// shader.rs:1630-1679, applied to a cell velocity already in registers
__device__ __forceinline__ f3 boundary_velocity(const Ctx& c, uint32_t ix, uint32_t iy, uint32_t iz, f3 v) {
    const Params& u = c.u;
    f3 cp = cell_center(u, ix, iy, iz);
    float sv = sample_sdf(c, cp);
    if (sv < u.contact_offset) {
        f3 n = sdf_gradient(c, cp);
        float vn = dot3(v, n);
        if (vn < 0.0f) {
            v = v - n * vn * (1.0f + u.restitution);
            f3 vt = v - n * dot3(v, n);
            float vtl = len3(vt);
            if (vtl > 1e-6f) {
                float fi = wmin(u.friction * fabsf(vn), vtl);
                v = v - vt * (fi / vtl);
            }
        }
    }
    float m = 2.0f * u.dx;
    float lox = u.ox + m, loy = u.oy + m, loz = u.oz + m;
    float hix = u.bx - m, hiy = u.by - m, hiz = u.bz - m;
    if (cp.x < lox && v.x < 0.0f) v.x = 0.0f;
    if (cp.x > hix && v.x > 0.0f) v.x = 0.0f;
    if (cp.y < loy && v.y < 0.0f) v.y = 0.0f;
    if (cp.y > hiy && v.y > 0.0f) v.y = 0.0f;
    if (cp.z < loz && v.z < 0.0f) v.z = 0.0f;
    if (cp.z > hiz && v.z > 0.0f) v.z = 0.0f;
    return v;
}

// ---- bed helpers (shader.rs:361-576) ----
__device__ __forceinline__ bool valid_bed_solid(const Ctx& c, int32_t b) {
    if (b < 0 || (uint32_t)b >= c.u.num_bed) return false;
    return !is_water_phase(c.c0[b].w);
}
__device__ __forceinline__ f3 bed_matrix_velocity(const Ctx& c, int x, int y, int z) {
    f3 sum = mk(0.0f, 0.0f, 0.0f);
    float ws = 0.0f;
    // unrolled so the 27 lookups (and then the sample reads) are in flight together
#pragma unroll
    for (int di = -1; di <= 1; ++di)
#pragma unroll
        for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
            for (int dk = -1; dk <= 1; ++dk) {
                int cx = x + di, cy = y + dj, cz = z + dk;
                if (!in_grid(c.u, cx, cy, cz)) continue;
                int32_t b = c.lookup[cidx(c.u, cx, cy, cz)];
                if (!valid_bed_solid(c, b)) continue;
                sum += xyz(c.vel[b]);
                ws += 1.0f;
            }
    if (ws <= 0.0f) return mk(0.0f, 0.0f, 0.0f);
    return sum / ws;
}
__device__ __forceinline__ f3 bed_velocity_cell(const Ctx& c, int x, int y, int z) {
    if (!in_grid(c.u, x, y, z)) return mk(0.0f, 0.0f, 0.0f);
    return bed_matrix_velocity(c, x, y, z);
}
__device__ __forceinline__ float kozeny_factor(float phi_in) {
    float phi = wclamp(phi_in, 0.08f, 0.82f);
    float solid = wmax(1.0f - phi, 1e-4f);
    return (phi * phi * phi) / (solid * solid);
}
__device__ __forceinline__ float compacted_porosity(const Ctx& c, uint32_t b) {
    float4 a = c.bedA[b];
    float base = wclamp(a.y, 0.18f, 0.70f);
    float comp = wclamp(a.w, 0.0f, 2.25f);
    return wclamp(base - comp * 0.12f, 0.16f, base);
}
__device__ __forceinline__ float compacted_permeability(const Ctx& c, uint32_t b) {
    float4 a = c.bedA[b];
    float base = wclamp(a.y, 0.18f, 0.70f);
    float cp = compacted_porosity(c, b);
    float ratio = kozeny_factor(cp) / wmax(kozeny_factor(base), 1e-8f);
    return wmax(a.z * ratio, c.u.min_perm);
}
__device__ __forceinline__ int32_t* delta_lane(const Ctx& c, int l) { return c.delta + (size_t)l * c.u.max_p; }
__device__ __forceinline__ void bed_water_add(const Ctx& c, uint32_t b, float amount) {
    if (amount <= 0.0f) return;
    atomicAdd(&delta_lane(c, 0)[b], to_i32(amount * FP_SCALE));
}
__device__ __forceinline__ void bed_impulse_add(const Ctx& c, uint32_t b, f3 imp) {
    float cap = c.u.nominal_mass * c.u.vel_cap * BED_REACTION_IMPULSE_CAP;
    atomicAdd(&delta_lane(c, 1)[b], to_i32(wclamp(imp.x, -cap, cap) * FP_SCALE));
    atomicAdd(&delta_lane(c, 2)[b], to_i32(wclamp(imp.y, -cap, cap) * FP_SCALE));
    atomicAdd(&delta_lane(c, 3)[b], to_i32(wclamp(imp.z, -cap, cap) * FP_SCALE));
}
__device__ __forceinline__ void bed_impulse_neighborhood(const Ctx& c, int x, int y, int z, f3 imp) {
    // the 27 lookups and validity reads are issued together and kept for the second
    // pass (nothing this pass writes changes them)
    int32_t ids[27];
    float n = 0.0f;
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const int cx = x + q / 9 - 1, cy = y + (q / 3) % 3 - 1, cz = z + q % 3 - 1;
        ids[q] = in_grid(c.u, cx, cy, cz) ? c.lookup[cidx(c.u, cx, cy, cz)] : -1;
    }
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        if (!valid_bed_solid(c, ids[q])) ids[q] = -1;
        if (ids[q] >= 0) n += 1.0f;
    }
    if (n <= 0.0f) return;
    f3 share = imp / n;
#pragma unroll
    for (int q = 0; q < 27; ++q)
        if (ids[q] >= 0) bed_impulse_add(c, (uint32_t)ids[q], share);
}
__device__ __forceinline__ void world_to_cell(const Params& u, f3 p, int& x, int& y, int& z) {
    x = (int)floorf((p.x - u.ox) * u.inv_dx);
    y = (int)floorf((p.y - u.oy) * u.inv_dx);
    z = (int)floorf((p.z - u.oz) * u.inv_dx);
}

// quadratic B-spline weights (shader.rs:980-988)
__device__ __forceinline__ void bspline(float f, float w[3]) {
    w[0] = 0.5f * (1.5f - f) * (1.5f - f);
    w[1] = 0.75f - (f - 1.0f) * (f - 1.0f);
    w[2] = 0.5f * (f - 0.5f) * (f - 0.5f);
}

}  // namespace cs
