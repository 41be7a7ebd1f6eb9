// kernels.cu — sm_100a kernels of one MLS-MPM substep.
//
// One kernel (or one fused kernel) per reference compute entry point of
// crates/sim-wasm/src/mpm_3d/shader.rs, in the dispatch order of mod.rs:317-414.
// Kernels take an array of Ctx (one per simulation) and use blockIdx.y as the
// instance, so a batched ensemble runs every member in the same launch.  Element
// loops are grid-stride so launch shapes do not depend on the particle count (a
// captured CUDA graph stays valid while particles are emitted).
#include <cuda_bf16.h>

#include "kernels.cuh"
#include "kernels_api.h"

namespace cs {

#define CS_FOR(i, n) for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

// ---------------- set-up: SDF and solid mask (state.rs:206-344) ----------------
__device__ float sdf_interior(const CsObstacle& o, float px, float py, float pz) {
    const float NO = 999.0f;
    if (o.kind == CS_OBSTACLE_TRUNCATED_CONE) {
        float ly = py - o.center[1];
        if (ly > o.top_y || ly < o.bot_y) return NO;
        float h = o.top_y - o.bot_y;
        if (h < 1e-10f) return NO;
        float t = (ly - o.bot_y) / h;
        float cr = o.bot_radius + (o.top_radius - o.bot_radius) * t;
        float ddx = px - o.center[0], ddz = pz - o.center[2];
        return cr - sqrtf(ddx * ddx + ddz * ddz);
    }
    float ly = py - o.center[1];
    if (ly > o.top_y) return NO;
    float ddx = px - o.center[0], ddz = pz - o.center[2];
    float radial = o.radius - sqrtf(ddx * ddx + ddz * ddz);
    return fminf(radial, ly - o.bot_y);
}

__global__ void k_gen_sdf(float* sdf, SdfSpec spec) {
    const uint32_t n = SDF_RES;
    CS_FOR(i, n * n * n) {
        uint32_t ix = i % n, iy = (i / n) % n, iz = i / (n * n);
        float px = -spec.bounds[0] * 0.5f + ((float)ix + 0.5f) * spec.bounds[0] / (float)n;
        float py = -spec.bounds[1] * 0.5f + ((float)iy + 0.5f) * spec.bounds[1] / (float)n;
        float pz = -spec.bounds[2] * 0.5f + ((float)iz + 0.5f) * spec.bounds[2] / (float)n;
        float v = 999.0f;
        for (uint32_t k = 0; k < spec.count; ++k) {
            float sd = sdf_interior(spec.obs[k], px, py, pz) - spec.wall_thickness * 0.5f;
            if (v >= 999.0f - 1.0f) v = sd;
            else v = fmaxf(v, sd);
        }
        sdf[i] = v;
    }
}

// Solid mask from the host-side trilinear sample (state.rs:287-344): f32::fract is
// x - trunc(x) and the lerp is a + (b - a) * t.
__global__ void k_gen_class(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    CS_FOR(i, u.cells) {
        uint32_t ix, iy, iz;
        decompose(u, i, ix, iy, iz);
        float px = u.ox + ((float)ix + 0.5f) * u.dx;
        float py = u.oy + ((float)iy + 0.5f) * u.dx;
        float pz = u.oz + ((float)iz + 0.5f) * u.dx;
        float bsx = u.bx * 2.0f, bsy = u.by * 2.0f, bsz = u.bz * 2.0f;
        const float res = (float)SDF_RES;
        float ux = (px + bsx * 0.5f) / bsx * res - 0.5f;
        float uy = (py + bsy * 0.5f) / bsy * res - 0.5f;
        float uz = (pz + bsz * 0.5f) / bsz * res - 0.5f;
        int x = (int)floorf(ux), y = (int)floorf(uy), z = (int)floorf(uz);
        float fx = ux - truncf(ux), fy = uy - truncf(uy), fz = uz - truncf(uz);
        float c000 = sdf_texel(c, x, y, z), c100 = sdf_texel(c, x + 1, y, z);
        float c010 = sdf_texel(c, x, y + 1, z), c110 = sdf_texel(c, x + 1, y + 1, z);
        float c001 = sdf_texel(c, x, y, z + 1), c101 = sdf_texel(c, x + 1, y, z + 1);
        float c011 = sdf_texel(c, x, y + 1, z + 1), c111 = sdf_texel(c, x + 1, y + 1, z + 1);
        float c00 = c000 + (c100 - c000) * fx, c10 = c010 + (c110 - c010) * fx;
        float c01 = c001 + (c101 - c001) * fx, c11 = c011 + (c111 - c011) * fx;
        float c0 = c00 + (c10 - c00) * fy, c1 = c01 + (c11 - c01) * fy;
        float v = c0 + (c1 - c0) * fz;
        ((uint8_t*)c.cls)[i] = v < 0.0f ? 1 : 0;
    }
}

// ---------------- bed_lookup_scatter (shader.rs:2305-2335) ----------------
__global__ void k_bed_lookup_scatter(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    CS_FOR(b, u.num_bed) {
        if (is_water_phase(c.c0[b].w)) continue;
        int cx, cy, cz;
        world_to_cell(u, xyz(c.pos[b]), cx, cy, cz);
        for (int di = -1; di <= 1; ++di)
            for (int dj = -1; dj <= 1; ++dj)
                for (int dk = -1; dk <= 1; ++dk) {
                    int x = cx + di, y = cy + dj, z = cz + dk;
                    if (!in_grid(u, x, y, z)) continue;
                    atomicMax(&c.lookup[cidx(u, x, y, z)], (int32_t)b);
                }
    }
}

// ---------------- p2g (shader.rs:955-1052) ----------------
// The deposit of one particle: B-spline weights, APIC momentum, rest and current volume,
// each contribution rounded to i32 * 2^18 and handed to `add(node x, y, z, lane, value)`.
// Integer sums do not depend on order, so every accumulation strategy below produces
// the same lanes bit for bit.
struct P2GSample {
    int bx, by, bz;
    float fx, fy, fz, mp, rpv, cpv;
    float wx[3], wy[3], wz[3];
    f3 a0, a1, a2, mv;
};
__device__ __forceinline__ bool p2g_prepare(const Ctx& c, uint32_t pid, P2GSample& q) {
    const Params& u = c.u;
    float4 P = c.pos[pid], Vv = c.vel[pid], A0 = c.c0[pid];
    q.mp = Vv.w;
    if (!is_water_phase(A0.w) || q.mp <= inactive_mass(u)) return false;
    float4 A1 = c.c1[pid], A2 = c.c2[pid];
    float gx = (P.x - u.ox) * u.inv_dx, gy = (P.y - u.oy) * u.inv_dx, gz = (P.z - u.oz) * u.inv_dx;
    q.bx = (int)floorf(gx - 0.5f);
    q.by = (int)floorf(gy - 0.5f);
    q.bz = (int)floorf(gz - 0.5f);
    q.fx = gx - (float)q.bx;
    q.fy = gy - (float)q.by;
    q.fz = gz - (float)q.bz;
    bspline(q.fx, q.wx);
    bspline(q.fy, q.wy);
    bspline(q.fz, q.wz);
    const float mp = q.mp;
    q.a0 = mk(mp * A0.x, mp * A0.y, mp * A0.z);
    q.a1 = mk(mp * A1.x, mp * A1.y, mp * A1.z);
    q.a2 = mk(mp * A2.x, mp * A2.y, mp * A2.z);
    q.mv = mk(mp * Vv.x, mp * Vv.y, mp * Vv.z);
    q.rpv = u.p_vol * mp / wmax(u.nominal_mass, 1e-6f);
    q.cpv = q.rpv * clamp_j(P.w);
    return true;
}
template <bool I64, class Add>
__device__ __forceinline__ void p2g_deposit(const Ctx& c, const P2GSample& q, Add add) {
    const Params& u = c.u;
    const float scale = I64 ? FP_SCALE64 : FP_SCALE;
    const float lim = I64 ? 1.0e18f : 1.0e9f;
    bool overflow = false;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                int cx = q.bx + i, cy = q.by + j, cz = q.bz + k;
                if (!in_grid(u, cx, cy, cz)) continue;
                float w = q.wx[i] * q.wy[j] * q.wz[k];
                f3 dpos = mk(((float)i - q.fx) * u.dx, ((float)j - q.fy) * u.dx, ((float)k - q.fz) * u.dx);
                float mfp = (w * q.mp) * scale;
                float rfp = (w * q.rpv) * scale;
                float cfp = (w * q.cpv) * scale;
                float mx = (w * (q.mv.x + dot3(q.a0, dpos))) * scale;
                float my = (w * (q.mv.y + dot3(q.a1, dpos))) * scale;
                float mz = (w * (q.mv.z + dot3(q.a2, dpos))) * scale;
                overflow |= fabsf(mfp) > lim || fabsf(mx) > lim || fabsf(my) > lim || fabsf(mz) > lim ||
                            fabsf(rfp) > lim || fabsf(cfp) > lim;
                if (I64) {
                    add(cx, cy, cz, 0, to_i64(mfp));
                    add(cx, cy, cz, 1, to_i64(mx));
                    add(cx, cy, cz, 2, to_i64(my));
                    add(cx, cy, cz, 3, to_i64(mz));
                    add(cx, cy, cz, 4, to_i64(rfp));
                    add(cx, cy, cz, 5, to_i64(cfp));
                } else {
                    add(cx, cy, cz, 0, to_i32(mfp));
                    add(cx, cy, cz, 1, to_i32(mx));
                    add(cx, cy, cz, 2, to_i32(my));
                    add(cx, cy, cz, 3, to_i32(mz));
                    add(cx, cy, cz, 4, to_i32(rfp));
                    add(cx, cy, cz, 5, to_i32(cfp));
                }
                if (overflow) {
                    atomicAdd(&c.metrics[M_OVERFLOW], 1u);
                    overflow = false;
                }
            }
}

// One global atomic per node and lane (the reference's scheme).
__global__ void k_p2g_atomic(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    uint32_t n = u.num_water + u.num_bed;
    CS_FOR(pid, n) {
        P2GSample q;
        if (!p2g_prepare(c, pid, q)) continue;
        p2g_deposit<false>(c, q, [&](int x, int y, int z, int l, int32_t v) {
            atomicAdd(&c.lanes[(size_t)l * u.cells + cidx(u, x, y, z)], v);
        });
    }
}

// ---- sorted P2G: counting sort by tile, shared-memory accumulation per tile ----
// A particle whose base cell is b (its stencil covers b..b+2, b >= -1 inside the
// domain) belongs to tile t = (b + 1) / P2G_TILE per axis; the tile's shared-memory
// block covers nodes t*P2G_TILE - 1 .. t*P2G_TILE + P2G_TILE, so every node of its
// particles lands in it.  A particle outside the domain (clamped key) falls back to
// global atomics.
// The tile side is 4 or 8 cells (Params::p2g_tile; a template parameter of the tile
// kernel, which sizes its shared memory by it).
constexpr int P2G_TILE = 4;  // default tile side, and the tiles the sample reorder sorts by
constexpr uint32_t P2G_NO_TILE = 0xffffffffu;
constexpr int P2G_THREADS = 256;

__device__ __forceinline__ uint32_t p2g_tile_axis(int b, uint32_t nt, uint32_t tile) {
    int q = b + 1;
    q = q < 0 ? 0 : q;
    uint32_t t = (uint32_t)q / tile;
    return t < nt ? t : nt - 1;
}

__global__ void k_p2g_keys(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    const uint32_t n = u.num_water + u.num_bed;
    const uint32_t lane = threadIdx.x & 31u;
    // warp-uniform loop (blockDim.x is a multiple of 32) so the warp votes below see
    // every lane
    for (uint32_t w0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; w0 < n; w0 += gridDim.x * blockDim.x) {
        const uint32_t pid = w0 + lane;
        uint32_t key = P2G_NO_TILE, rank = 0;
        if (pid < n) {
            const float4 P = c.pos[pid], Vv = c.vel[pid];
            const float ph = c.c0[pid].w;
            if (is_water_phase(ph) && !(Vv.w <= inactive_mass(u))) {
                const int bx = (int)floorf((P.x - u.ox) * u.inv_dx - 0.5f);
                const int by = (int)floorf((P.y - u.oy) * u.inv_dx - 0.5f);
                const int bz = (int)floorf((P.z - u.oz) * u.inv_dx - 0.5f);
                key = (p2g_tile_axis(bz, u.ntz, u.p2g_tile) * u.nty + p2g_tile_axis(by, u.nty, u.p2g_tile)) * u.ntx +
                      p2g_tile_axis(bx, u.ntx, u.p2g_tile);
            }
        }
        // one counter atomic per distinct tile in the warp (neighbouring particles
        // usually share a tile); ranks inside the warp follow lane order
        const uint32_t same = __match_any_sync(0xffffffffu, key);
        const uint32_t leader = __ffs(same) - 1;
        uint32_t base = 0;
        if (key != P2G_NO_TILE && lane == leader) base = atomicAdd(&c.tile_count[key], (uint32_t)__popc(same));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (key != P2G_NO_TILE) rank = base + __popc(same & ((1u << lane) - 1u));
        if (pid < n) {
            c.p2g_key[pid] = key;
            c.p2g_rank[pid] = rank;
        }
    }
}

// ---- reorder of the water samples by tile (reorder_every) ----
// Key of water slot num_bed + i: the 4^3-cell tile of its P2G base cell (whatever the
// P2G tile size), the tile count for a sample that deposits nothing; the value is its
// own index, for a stable sort.
__global__ void k_reorder_keys(const Ctx* __restrict__ cp, uint32_t* __restrict__ keys, uint32_t* __restrict__ idx) {
    const Ctx& c = cp[0];
    const Params& u = c.u;
    const uint32_t ntx = (u.gx + P2G_TILE) / P2G_TILE, nty = (u.gy + P2G_TILE) / P2G_TILE,
                   ntz = (u.gz + P2G_TILE) / P2G_TILE;
    CS_FOR(i, u.num_water) {
        const uint32_t pid = u.num_bed + i;
        const float4 P = c.pos[pid], Vv = c.vel[pid];
        uint32_t key = ntx * nty * ntz;
        if (is_water_phase(c.c0[pid].w) && !(Vv.w <= inactive_mass(u))) {
            const int bx = (int)floorf((P.x - u.ox) * u.inv_dx - 0.5f);
            const int by = (int)floorf((P.y - u.oy) * u.inv_dx - 0.5f);
            const int bz = (int)floorf((P.z - u.oz) * u.inv_dx - 0.5f);
            key = (p2g_tile_axis(bz, ntz, P2G_TILE) * nty + p2g_tile_axis(by, nty, P2G_TILE)) * ntx +
                  p2g_tile_axis(bx, ntx, P2G_TILE);
        }
        keys[i] = key;
        idx[i] = i;
    }
}

// out[i] = in[num_bed + perm[i]] for the water slots of one particle stream
__global__ void k_reorder_gather(const float4* __restrict__ in, float4* __restrict__ out,
                                 const uint32_t* __restrict__ perm, uint32_t num_bed, uint32_t n) {
    CS_FOR(i, n) out[i] = in[num_bed + perm[i]];
}

__global__ void k_p2g_scatter(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    uint32_t n = c.u.num_water + c.u.num_bed;
    CS_FOR(pid, n) {
        const uint32_t key = c.p2g_key[pid];
        if (key != P2G_NO_TILE) c.p2g_sorted[c.tile_start[key] + c.p2g_rank[pid]] = pid;
    }
}

// T = int32_t (reference lanes) or unsigned long long (int64 mode; two's-complement
// sums are the same as signed ones).  In int64 mode the tile accumulates each lane in
// two 32-bit words: a value v = H * 2^32 + L (L its low 32 bits) adds L to the low word
// with an atomic that returns the old word, so a wrap past 2^32 is seen as a carry,
// and H + carry to the high word only when that is nonzero (almost never for the
// magnitudes of one sample's deposit).  High * 2^32 + low is then the sum of the
// values modulo 2^64, exactly what 64-bit atomics give, at the cost of 32-bit ones.
template <class T, int TILE>
__global__ void __launch_bounds__(P2G_THREADS) k_p2g_tiles(const Ctx* __restrict__ cp) {
    constexpr bool I64 = sizeof(T) == 8;
    constexpr int P2G_SPAN = TILE + 2;
    constexpr int P2G_NODES = P2G_SPAN * P2G_SPAN * P2G_SPAN;
    __shared__ uint32_t acc[I64 ? 12 : 6][P2G_NODES];
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    T* glanes = I64 ? reinterpret_cast<T*>(c.lanes64) : reinterpret_cast<T*>(c.lanes);
    const uint32_t ntiles = u.ntx * u.nty * u.ntz;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint32_t first = c.tile_start[t], last = c.tile_start[t + 1];
        if (first == last) continue;  // uniform across the block
        const uint32_t tx = t % u.ntx, ty = (t / u.ntx) % u.nty, tz = t / (u.ntx * u.nty);
        const int ox = (int)(tx * TILE) - 1, oy = (int)(ty * TILE) - 1, oz = (int)(tz * TILE) - 1;
        for (int i = threadIdx.x; i < (I64 ? 12 : 6) * P2G_NODES; i += blockDim.x) (&acc[0][0])[i] = 0;
        __syncthreads();
        // Particles of one cell are mostly adjacent in the tile list; visiting each block
        // of P2G_THREADS entries in an odd-stride order gives a warp particles of
        // different cells, so its shared-memory atomics rarely hit one address.
        for (uint32_t blk = first; blk < last; blk += P2G_THREADS) {
            const uint32_t k = blk + ((threadIdx.x * 41u) & (P2G_THREADS - 1));
            if (k >= last) continue;
            P2GSample q;
            if (!p2g_prepare(c, c.p2g_sorted[k], q)) continue;
            const bool inside = q.bx >= ox && q.by >= oy && q.bz >= oz && q.bx + 2 < ox + P2G_SPAN &&
                                q.by + 2 < oy + P2G_SPAN && q.bz + 2 < oz + P2G_SPAN;
            if (inside) {
                p2g_deposit<I64>(c, q, [&](int x, int y, int z, int l, auto v) {
                    const int n = ((z - oz) * P2G_SPAN + (y - oy)) * P2G_SPAN + (x - ox);
                    if constexpr (I64) {
                        const unsigned long long w = (unsigned long long)v;
                        const uint32_t lo = (uint32_t)w, hi = (uint32_t)(w >> 32);
                        const uint32_t old = atomicAdd(&acc[l][n], lo);
                        const uint32_t h = hi + ((uint32_t)(old + lo) < old ? 1u : 0u);
                        if (h) atomicAdd(&acc[6 + l][n], h);
                    } else {
                        atomicAdd(reinterpret_cast<int32_t*>(&acc[l][n]), (int32_t)v);
                    }
                });
            } else {
                p2g_deposit<I64>(c, q, [&](int x, int y, int z, int l, auto v) {
                    atomicAdd(&glanes[(size_t)l * u.cells + cidx(u, x, y, z)], (T)v);
                });
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < P2G_NODES; i += blockDim.x) {
            const int x = ox + i % P2G_SPAN, y = oy + (i / P2G_SPAN) % P2G_SPAN, z = oz + i / (P2G_SPAN * P2G_SPAN);
            if (!in_grid(u, x, y, z)) continue;
            const uint32_t ci = cidx(u, x, y, z);
#pragma unroll
            for (int l = 0; l < 6; ++l) {
                T v;
                if constexpr (I64)
                    v = ((unsigned long long)acc[6 + l][i] << 32) | acc[l][i];
                else
                    v = (T)(int32_t)acc[l][i];
                if (v != 0) atomicAdd(&glanes[(size_t)l * u.cells + ci], v);
            }
        }
        __syncthreads();
    }
}

// ---------------- grid_update (shader.rs:1056-1082) [+ boundary_project] ----------------
__global__ void k_grid_update(const Ctx* __restrict__ cp, int with_boundary) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    CS_FOR(i, u.cells) {
        float mass = p2g_lane(c, 0, i);
        if (mass < 1e-6f) continue;
        f3 v = mk(p2g_lane(c, 1, i) / mass, p2g_lane(c, 2, i) / mass, p2g_lane(c, 3, i) / mass);
        v.y += u.gravity * u.dt;
        float sp = len3(v);
        if (sp > u.vel_cap) v = v * (u.vel_cap / sp);
        if (with_boundary) {
            uint32_t ix, iy, iz;
            decompose(u, i, ix, iy, iz);
            v = boundary_velocity(c, ix, iy, iz, v);
        }
        c.gvel[i] = make_float4(v.x, v.y, v.z, mass);
    }
}

// ---------------- boundary_project alone (shader.rs:1630-1679) ----------------
__global__ void k_boundary(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    CS_FOR(i, u.cells) {
        float4 g = c.gvel[i];
        if (g.w < 1e-6f) continue;
        uint32_t ix, iy, iz;
        decompose(u, i, ix, iy, iz);
        f3 v = boundary_velocity(c, ix, iy, iz, xyz(g));
        c.gvel[i] = make_float4(v.x, v.y, v.z, g.w);
    }
}

// bed_matrix_velocity_cell (shader.rs:380-407) of every cell next to the bed, once per substep: the bed
// samples' velocities and the cell lookup do not change between bed_lookup_scatter and
// bed_dynamics, so classify (six neighbours of each bed-coupled cell) and project (each
// bed-coupled cell) read these instead of rescanning 27 cells per call.
__global__ void k_bed_velocity(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    if (!c.bedv) return;
    CS_FOR(i, u.cells) {
        uint32_t ix, iy, iz;
        decompose(u, i, ix, iy, iz);
        // read only at bed-coupled cells (lookup >= 0, by project) and their six
        // neighbours (by classify), so only those cells are written; the seven lookups are
        // loaded together (no short-circuit chain of dependent loads)
        const uint32_t sy = u.gx, sz = u.gx * u.gy;
        const bool in[6] = {ix > 0, ix + 1 < u.gx, iy > 0, iy + 1 < u.gy, iz > 0, iz + 1 < u.gz};
        const uint32_t off[6] = {(uint32_t)-1, 1u, (uint32_t)0 - sy, sy, (uint32_t)0 - sz, sz};
        bool near = c.lookup[i] >= 0;
#pragma unroll
        for (int f = 0; f < 6; ++f) near |= in[f] && c.lookup[i + off[f]] >= 0;
        if (!near) continue;
        const f3 v = bed_matrix_velocity(c, (int)ix, (int)iy, (int)iz);
        c.bedv[i] = make_float4(v.x, v.y, v.z, 0.0f);
    }
}
__device__ __forceinline__ f3 bed_velocity_at(const Ctx& c, int x, int y, int z) {
    if (!in_grid(c.u, x, y, z)) return mk(0.0f, 0.0f, 0.0f);
    return xyz(c.bedv[cidx(c.u, (uint32_t)x, (uint32_t)y, (uint32_t)z)]);
}

// ---------------- classify_cells (shader.rs:1181-1367) ----------------
__device__ float volume_target(const Params& u, float rest, float cur) {
    float cv = u.dx * u.dx * u.dx;
    float eps = wmax(cv * 1e-5f, u.p_vol * 1e-3f);
    if (rest <= eps) return 0.0f;
    float j = cur / rest;
    float ce = wclamp(1.0f - j, 0.0f, 0.75f);
    float ee = wclamp(j - 1.0f, 0.0f, 0.75f);
    float t = ce * u.j_alpha - ee * u.j_expand_alpha;
    float packed = wmax(rest, cur) / wmax(cv, 1e-8f);
    float over = wmax(packed - u.max_rest_frac, 0.0f);
    return wmax(t, over * u.j_alpha);
}
__device__ float bed_pore_target(const Ctx& c, uint32_t b, f3 cc, float rest, float cur) {
    const Params& u = c.u;
    float t = volume_target(u, rest, cur);
    float cv = u.dx * u.dx * u.dx;
    float poro = compacted_porosity(c, b);
    float sat = wclamp(c.bedB[b].w, 0.0f, 1.0f);
    float comp = wclamp(c.bedA[b].w, 0.0f, 2.25f);
    float bcy = c.pos[b].y;
    float st = smoothstepf(-0.25f, 0.75f, (cc.y - bcy) * u.inv_dx);
    float open = wclamp((1.0f - 0.65f * sat) * (1.0f - 0.12f * comp), 0.20f, 1.0f);
    float sopen = st * wclamp(u.surface_void_scale, 0.0f, 1.0f) * open;
    float sporo = wmin(poro + 0.35f, 0.82f);
    float eff = mixf(poro, sporo, sopen);
    float occ = mixf(1.0f, 0.35f, sopen);
    float satcap = mixf(1.0f, 0.32f, sat);
    float compcap = mixf(1.0f, 0.58f, wclamp(comp / 1.5f, 0.0f, 1.0f));
    float cap = eff * cv * wmax(u.pore_capacity_scale, 0.0f) * satcap * compcap;
    float over = wmax(cur - cap, 0.0f) / wmax(cv, 1e-8f);
    float resp = u.pore_overfill_alpha * occ * mixf(1.0f, 1.45f, sat);
    return wmax(t, over * resp);
}
__device__ __forceinline__ bool open_nb(const Ctx& c, f3 cc, uint32_t x, uint32_t y, uint32_t z, float ox, float oy,
                                        float oz) {
    if (c.u.use_sdf_cache) return c.cls[cidx(c.u, x, y, z)] == 0;
    return sample_sdf(c, cc + mk(ox, oy, oz)) >= 0.0f;
}

// One cell of classify_cells, given the loads the caller made ahead for it: its grid
// velocity and mass, its solid class (when the SDF class cache is on), its bed lookup
// and the pressure kept from the last substep.  In the fluid path the six neighbours'
// velocities and both volumes are loaded before the open-face tests and the kind that
// pick from them, so the loads are in flight together.
__device__ __forceinline__ void classify_cell(const Ctx& c, uint32_t i, float4 sv, uint8_t cls, int32_t lk,
                                              float keep, float keep_lo, uint32_t& max_fd, uint32_t& n_fluid) {
    const Params& u = c.u;
    const float mass = sv.w;
    pressure_store(c, i, 0.0f);
    c.plo[i] = 0.0f;
    uint32_t ix, iy, iz;
    decompose(u, i, ix, iy, iz);
    f3 cc = cell_center(u, ix, iy, iz);
    bool solid = u.use_sdf_cache ? (cls != 0) : (sample_sdf(c, cc) < 0.0f);
    int32_t* kl = lane(c, 3);
    if (solid) {
        kl[i] = CELL_SOLID;
        div_store(c, i, 0.0f);
        c.fill[i] = 0.0f;
        c.fcode[i] = -2.0f;
        return;
    }
    if (mass <= occupancy_mass(u)) {
        kl[i] = CELL_AIR;
        div_store(c, i, 0.0f);
        c.fill[i] = 0.0f;
        c.fcode[i] = -1.0f;
        return;
    }
    const uint32_t sy = u.gx, sz = u.gx * u.gy;
    const bool in[6] = {ix > 0, ix + 1 < u.gx, iy > 0, iy + 1 < u.gy, iz > 0, iz + 1 < u.gz};
    const uint32_t off[6] = {(uint32_t)-1, 1u, (uint32_t)0 - sy, sy, (uint32_t)0 - sz, sz};
    float4 nv[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) nv[f] = in[f] ? c.gvel[i + off[f]] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float rest = rest_vol(c, i), cur = cur_vol(c, i);
    int32_t kind;
    if (lk >= 0) {
        kind = CELL_BED;
    } else {
        bool air = !(in[0] && in[1] && in[2] && in[3] && in[4] && in[5]);
        if (!air) {
            const float occ = occupancy_mass(u);
            air = nv[0].w <= occ || nv[1].w <= occ || nv[2].w <= occ || nv[3].w <= occ || nv[4].w <= occ ||
                  nv[5].w <= occ;
        }
        kind = air ? CELL_SURFACE : CELL_INTERIOR;
    }
    kl[i] = kind;
    const float fill = liquid_fill_of(u, kind, rest, cur);
    c.fill[i] = fill;
    c.fcode[i] = kind == CELL_BED ? 2.0f : fill;
    if (u.warm && !u.fixed_point) {
        c.pf[i] = keep;
        c.plo[i] = keep_lo;
    }
    const float d = u.dx;
    float vxm = -sv.x, vxp = -sv.x, vym = -sv.y, vyp = -sv.y, vzm = -sv.z, vzp = -sv.z;
    if (in[0] && open_nb(c, cc, ix - 1, iy, iz, -d, 0.0f, 0.0f)) vxm = nv[0].x;
    if (in[1] && open_nb(c, cc, ix + 1, iy, iz, d, 0.0f, 0.0f)) vxp = nv[1].x;
    if (in[2] && open_nb(c, cc, ix, iy - 1, iz, 0.0f, -d, 0.0f)) vym = nv[2].y;
    if (in[3] && open_nb(c, cc, ix, iy + 1, iz, 0.0f, d, 0.0f)) vyp = nv[3].y;
    if (in[4] && open_nb(c, cc, ix, iy, iz - 1, 0.0f, 0.0f, -d)) vzm = nv[4].z;
    if (in[5] && open_nb(c, cc, ix, iy, iz + 1, 0.0f, 0.0f, d)) vzp = nv[5].z;
    float div = 0.5f * u.inv_dx * (((vxp - vxm) + (vyp - vym)) + (vzp - vzm));
    float target = volume_target(u, rest, cur);
    if (kind == CELL_BED) {
        int32_t b = lk;
        if (b >= 0 && (uint32_t)b < u.num_bed) {
            float pt = bed_pore_target(c, (uint32_t)b, cc, rest, cur);
            float poro = wclamp(compacted_porosity(c, (uint32_t)b), 0.08f, 1.0f);
            float sfrac = 1.0f - poro;
            int x = ix, y = iy, z = iz;
            float bxm = bed_velocity_at(c, x - 1, y, z).x, bxp = bed_velocity_at(c, x + 1, y, z).x;
            float bym = bed_velocity_at(c, x, y - 1, z).y, byp = bed_velocity_at(c, x, y + 1, z).y;
            float bzm = bed_velocity_at(c, x, y, z - 1).z, bzp = bed_velocity_at(c, x, y, z + 1).z;
            float sdiv = 0.5f * u.inv_dx * (((bxp - bxm) + (byp - bym)) + (bzp - bzm));
            target = (pt - sfrac * sdiv) / poro;
        }
    }
    div_store(c, i, div - target);
    uint32_t fd = to_u32(wclamp(fabsf(div) * METRICS_DIV_FP_SCALE, 0.0f, 2147483648.0f));
    max_fd = max_fd > fd ? max_fd : fd;
    n_fluid += 1u;
}

// classify_cells over the whole grid.  The kernel is latency bound (a chain of
// dependent loads per fluid cell), so each thread takes CLS_CELLS cells a grid stride
// apart and issues the first loads of all of them before working on any.  No cell
// reads what another writes here, so the order of the loads changes nothing.  64
// registers (4 blocks of 256 per SM).
constexpr uint32_t CLS_CELLS = 4;
__global__ void __launch_bounds__(256, 4) k_classify(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    // the metrics' max |div| and fluid-cell count, per thread, then one atomic per warp
    uint32_t max_fd = 0u, n_fluid = 0u;
    const uint32_t stride = gridDim.x * blockDim.x;
    const bool kept = !u.fixed_point && u.warm;
    for (uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < u.cells; i0 += CLS_CELLS * stride) {
        float4 sv[CLS_CELLS];
        uint8_t cls[CLS_CELLS];
        int32_t lk[CLS_CELLS];
        float keep[CLS_CELLS], keep_lo[CLS_CELLS];
#pragma unroll
        for (uint32_t j = 0; j < CLS_CELLS; ++j) {
            const uint32_t i = i0 + j * stride;
            if (i >= u.cells) continue;
            sv[j] = c.gvel[i];
            cls[j] = u.use_sdf_cache ? c.cls[i] : (uint8_t)0;
            lk[j] = c.lookup[i];
            keep[j] = kept ? c.pf[i] : 0.0f;
            keep_lo[j] = kept ? c.plo[i] : 0.0f;
        }
#pragma unroll
        for (uint32_t j = 0; j < CLS_CELLS; ++j) {
            const uint32_t i = i0 + j * stride;
            if (i >= u.cells) continue;
            classify_cell(c, i, sv[j], cls[j], lk[j], keep[j], keep_lo[j], max_fd, n_fluid);
        }
    }
    // every lane leaves the loop (blocks are whole warps and nothing returns early)
    max_fd = __reduce_max_sync(0xffffffffu, max_fd);
    n_fluid = __reduce_add_sync(0xffffffffu, n_fluid);
    if ((threadIdx.x & 31u) == 0u && n_fluid) {
        atomicMax(&c.metrics[M_MAX_DIV], max_fd);
        atomicAdd(&c.metrics[M_FLUID], n_fluid);
    }
}

// ---------------- pressure_rbgs_red / _black (shader.rs:1371-1453) ----------------
// Thread t of a colour handles the t-th cell of that colour: rows of (y,z) hold
// ceil(gx/2) slots, x = 2*slot + ((y+z+parity)&1).
__device__ __forceinline__ void pressure_update(const Ctx& c, uint32_t i, uint32_t ix, uint32_t iy, uint32_t iz) {
    const Params& u = c.u;
    const int32_t* kl = lane(c, 3);
    int32_t kind = kl[i];
    if (!is_fluid(kind)) {
        pressure_store(c, i, 0.0f);
        return;
    }
    float sf = c.fill[i];
    float nc = 0.0f, ps = 0.0f;
    const uint32_t sy = u.gx, sz = u.gx * u.gy;
#define CS_FACE(cond, off)                                               \
    if (cond) {                                                          \
        uint32_t ni = i + (off);                                         \
        int32_t nk = kl[ni];                                             \
        if (!is_solid(nk)) {                                             \
            float w = face_weight(kind, sf, nk, c.fill[ni]);             \
            if (w > 0.0f) {                                              \
                nc += w;                                                 \
                if (is_fluid(nk)) ps += w * pressure_load(c, ni);        \
            }                                                            \
        }                                                                \
    }
    CS_FACE(ix > 0, (uint32_t)-1)
    CS_FACE(ix + 1 < u.gx, 1u)
    CS_FACE(iy > 0, (uint32_t)0 - sy)
    CS_FACE(iy + 1 < u.gy, sy)
    CS_FACE(iz > 0, (uint32_t)0 - sz)
    CS_FACE(iz + 1 < u.gz, sz)
#undef CS_FACE
    if (nc <= 0.0f) {
        pressure_store(c, i, 0.0f);
        return;
    }
    float rhs = div_load(c, i) * sf / wmax(u.dt, 1e-6f);
    float pn = (ps - u.dx * u.dx * rhs) / nc;
    // over-relaxed update p + w*(p_gs - p); w == 1 is the reference's plain update
    if (u.omega != 1.0f) pn = pressure_load(c, i) + u.omega * (pn - pressure_load(c, i));
    pressure_store(c, i, pn);
}

__global__ void k_rbgs_colour(const Ctx* __restrict__ cp, uint32_t parity) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    const uint32_t half = (u.gx + 1) / 2;
    const uint32_t n = half * u.gy * u.gz;
    CS_FOR(t, n) {
        uint32_t row = t / half, slot = t - row * half;
        uint32_t iy = row % u.gy, iz = row / u.gy;
        uint32_t ix = 2 * slot + ((iy + iz + parity) & 1u);
        if (ix >= u.gx) continue;
        pressure_update(c, cidx(u, ix, iy, iz), ix, iy, iz);
    }
}

// Residual of the pressure system in FP64 (definition: for each fluid cell
// r = (sum_f w_f p_f - dx^2 rhs) - W p with the face weights of pressure_update).
__global__ void k_residual(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    const int32_t* kl = lane(c, 3);
    double r2 = 0.0, b2 = 0.0;
    CS_FOR(i, u.cells) {
        int32_t kind = kl[i];
        if (!is_fluid(kind)) continue;
        uint32_t ix, iy, iz;
        decompose(u, i, ix, iy, iz);
        float sf = c.fill[i];
        double wsum = 0.0, psum = 0.0;
        const uint32_t sy = u.gx, sz = u.gx * u.gy;
#define CS_RFACE(cond, off)                                                        \
    if (cond) {                                                                    \
        uint32_t ni = i + (off);                                                   \
        int32_t nk = kl[ni];                                                       \
        if (!is_solid(nk)) {                                                       \
            float w = face_weight(kind, sf, nk, c.fill[ni]);                       \
            if (w > 0.0f) {                                                        \
                wsum += (double)w;                                                 \
                if (is_fluid(nk)) psum += (double)w * (double)pressure_load(c, ni); \
            }                                                                      \
        }                                                                          \
    }
        CS_RFACE(ix > 0, (uint32_t)-1)
        CS_RFACE(ix + 1 < u.gx, 1u)
        CS_RFACE(iy > 0, (uint32_t)0 - sy)
        CS_RFACE(iy + 1 < u.gy, sy)
        CS_RFACE(iz > 0, (uint32_t)0 - sz)
        CS_RFACE(iz + 1 < u.gz, sz)
#undef CS_RFACE
        if (wsum <= 0.0) continue;
        float rhs = div_load(c, i) * sf / wmax(u.dt, 1e-6f);
        double b = (double)(u.dx * u.dx * rhs);
        double r = (psum - b) - wsum * (double)pressure_load(c, i);
        r2 += r * r;
        b2 += b * b;
    }
    // warp then block reduction, one double atomic pair per block
    for (int o = 16; o > 0; o >>= 1) {
        r2 += __shfl_down_sync(0xffffffffu, r2, o);
        b2 += __shfl_down_sync(0xffffffffu, b2, o);
    }
    __shared__ double sr[32], sb[32];
    int lane_id = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane_id == 0) {
        sr[warp] = r2;
        sb[warp] = b2;
    }
    __syncthreads();
    if (warp == 0) {
        int nw = (blockDim.x + 31) >> 5;
        r2 = lane_id < nw ? sr[lane_id] : 0.0;
        b2 = lane_id < nw ? sb[lane_id] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            r2 += __shfl_down_sync(0xffffffffu, r2, o);
            b2 += __shfl_down_sync(0xffffffffu, b2, o);
        }
        if (lane_id == 0) {
            atomicAdd(&c.resid[0], r2);
            atomicAdd(&c.resid[1], b2);
        }
    }
}

// ---------------- mixed-precision iterative refinement ----------------
// FP32-storage residual mode: p = pf + plo (two fp32 words).  A cycle computes the
// FP64 residual g = (sum w p_nb - dx^2 rhs) - W p of pressure_update's operator,
// sweeps the correction d of L d = g in fp32 (red-black, over-relaxed), then adds d
// to p in FP64.  Per-cell arithmetic matches the CPU oracle operation for operation.
__device__ __forceinline__ void block_reduce_add2(double a, double b, double* out) {
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    __shared__ double sa[32], sb[32];
    int lane_id = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane_id == 0) {
        sa[warp] = a;
        sb[warp] = b;
    }
    __syncthreads();
    if (warp == 0) {
        int nw = (blockDim.x + 31) >> 5;
        a = lane_id < nw ? sa[lane_id] : 0.0;
        b = lane_id < nw ? sb[lane_id] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
        if (lane_id == 0) {
            atomicAdd(&out[0], a);
            atomicAdd(&out[1], b);
        }
    }
}

__global__ void k_refine_residual(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    const int32_t* kl = lane(c, 3);
    double r2 = 0.0, b2 = 0.0;
    CS_FOR(i, u.cells) {
        c.pd[i] = 0.0f;
        c.gres[i] = 0.0f;
        int32_t kind = kl[i];
        if (!is_fluid(kind)) continue;
        uint32_t ix, iy, iz;
        decompose(u, i, ix, iy, iz);
        float sf = c.fill[i];
        double wsum = 0.0, psum = 0.0;
        const uint32_t sy = u.gx, sz = u.gx * u.gy;
#define CS_GFACE(cond, off)                                                                     \
    if (cond) {                                                                                 \
        uint32_t ni = i + (off);                                                                \
        int32_t nk = kl[ni];                                                                    \
        if (!is_solid(nk)) {                                                                    \
            float w = face_weight(kind, sf, nk, c.fill[ni]);                                    \
            if (w > 0.0f) {                                                                     \
                wsum += (double)w;                                                              \
                if (is_fluid(nk)) psum += (double)w * ((double)c.pf[ni] + (double)c.plo[ni]);   \
            }                                                                                   \
        }                                                                                       \
    }
        CS_GFACE(ix > 0, (uint32_t)-1)
        CS_GFACE(ix + 1 < u.gx, 1u)
        CS_GFACE(iy > 0, (uint32_t)0 - sy)
        CS_GFACE(iy + 1 < u.gy, sy)
        CS_GFACE(iz > 0, (uint32_t)0 - sz)
        CS_GFACE(iz + 1 < u.gz, sz)
#undef CS_GFACE
        if (wsum <= 0.0) continue;
        float rhs = div_load(c, i) * sf / wmax(u.dt, 1e-6f);
        double b = (double)(u.dx * u.dx * rhs);
        double r = (psum - b) - wsum * ((double)c.pf[i] + (double)c.plo[i]);
        c.gres[i] = (float)r;
        r2 += r * r;
        b2 += b * b;
    }
    block_reduce_add2(r2, b2, c.resid);
}

__global__ void k_refine_sweep(const Ctx* __restrict__ cp, uint32_t parity) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    const float* fc = c.fcode;
    const uint32_t half = (u.gx + 1) / 2;
    const uint32_t n = half * u.gy * u.gz;
    CS_FOR(t, n) {
        uint32_t row = t / half, slot = t - row * half;
        uint32_t iy = row % u.gy, iz = row / u.gy;
        uint32_t ix = 2 * slot + ((iy + iz + parity) & 1u);
        if (ix >= u.gx) continue;
        uint32_t i = cidx(u, ix, iy, iz);
        // one fill code per cell carries what face_weight needs (kind and fill): the
        // same weights in the same face order as the kind/fill form
        const float fi = fc[i];
        if (fi < 0.0f) continue;  // not fluid
        const bool bed = fi > 1.5f;
        const float sf = bed ? 1.0f : fi;
        float nc = 0.0f, ds = 0.0f;
        const uint32_t sy = u.gx, sz = u.gx * u.gy;
#define CS_DFACE(cond, off)                                                   \
    if (cond) {                                                               \
        uint32_t ni = i + (off);                                              \
        const float fj = fc[ni];                                              \
        if (fj != -2.0f) {                                                    \
            const float w = (bed || fj > 1.5f) ? 1.0f : (fj < 0.0f ? sf : wmin(sf, fj)); \
            if (w > 0.0f) {                                                   \
                nc += w;                                                      \
                if (fj >= 0.0f) ds += w * c.pd[ni];                           \
            }                                                                 \
        }                                                                     \
    }
        CS_DFACE(ix > 0, (uint32_t)-1)
        CS_DFACE(ix + 1 < u.gx, 1u)
        CS_DFACE(iy > 0, (uint32_t)0 - sy)
        CS_DFACE(iy + 1 < u.gy, sy)
        CS_DFACE(iz > 0, (uint32_t)0 - sz)
        CS_DFACE(iz + 1 < u.gz, sz)
#undef CS_DFACE
        if (nc <= 0.0f) continue;
        float dn = (ds + c.gres[i]) * (1.0f / nc);
        if (u.omega != 1.0f) dn = c.pd[i] + u.omega * (dn - c.pd[i]);
        c.pd[i] = dn;
    }
}

__global__ void k_refine_accumulate(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    const int32_t* kl = lane(c, 3);
    const double lim = (double)u.p_limit;
    CS_FOR(i, u.cells) {
        if (!is_fluid(kl[i])) continue;
        double p = ((double)c.pf[i] + (double)c.plo[i]) + (double)c.pd[i];
        if (p > lim || p < -lim) {
            p = p > 0.0 ? lim : -lim;
            atomicAdd(&c.metrics[M_P_CLAMP], 1u);
        }
        float hi = (float)p;
        c.pf[i] = hi;
        c.plo[i] = (float)(p - (double)hi);
    }
}

// ---------------- project_pressure (shader.rs:1457-1543) [+ boundary + packing_prepare] ----
__device__ __forceinline__ float weighted_or_mirror(const Ctx& c, bool in, uint32_t ni, float mirror, int32_t sk,
                                                    float sf) {
    if (!in) return mirror;
    int32_t k = lane(c, 3)[ni];
    if (is_solid(k)) return mirror;
    float np = 0.0f;
    if (is_fluid(k)) np = pressure_load(c, ni);
    return mixf(mirror, np, face_weight(sk, sf, k, c.fill[ni]));
}

// stages: bit0 project, bit1 boundary, bit2 packing_prepare
__global__ void k_project(const Ctx* __restrict__ cp, int stages) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    CS_FOR(i, u.cells) {
        int32_t kind = lane(c, 3)[i];
        if (stages & 4) {
            // packing_prepare (shader.rs:1566-1583): reads kind and volumes only
            if (!is_fluid(kind) || kind == CELL_BED) {
                packing_store(c, i, 0.0f);
            } else {
                float cv = u.dx * u.dx * u.dx;
                float packed = wmax(rest_vol(c, i), cur_vol(c, i)) / wmax(cv, 1e-8f);
                float over = wmax(packed - wmin(u.max_rest_frac, 1.0f), 0.0f);
                packing_store(c, i, u.bulk_K * over);
            }
        }
        float4 g = c.gvel[i];
        if (g.w < 1e-6f) continue;
        uint32_t ix, iy, iz;
        decompose(u, i, ix, iy, iz);
        f3 v = xyz(g);
        bool changed = false;
        if ((stages & 1) && is_fluid(kind)) {
            float ph = pressure_load(c, i);
            float sf = c.fill[i];
            const uint32_t sy = u.gx, sz = u.gx * u.gy;
            float pxm = weighted_or_mirror(c, ix > 0, i - 1, ph, kind, sf);
            float pxp = weighted_or_mirror(c, ix + 1 < u.gx, i + 1, ph, kind, sf);
            float pym = weighted_or_mirror(c, iy > 0, i - sy, ph, kind, sf);
            float pyp = weighted_or_mirror(c, iy + 1 < u.gy, i + sy, ph, kind, sf);
            float pzm = weighted_or_mirror(c, iz > 0, i - sz, ph, kind, sf);
            float pzp = weighted_or_mirror(c, iz + 1 < u.gz, i + sz, ph, kind, sf);
            float h = 0.5f * u.inv_dx;
            f3 grad = mk(h * (pxp - pxm), h * (pyp - pym), h * (pzp - pzm));
            v = v - u.dt * grad;
            if (kind == CELL_BED) {
                int32_t b = c.lookup[i];
                if (b >= 0 && (uint32_t)b < u.num_bed) {
                    float perm = compacted_permeability(c, (uint32_t)b);
                    float rate = u.nu_m2s / perm;
                    float damp = 1.0f / (1.0f + wmax(rate * u.dt, 0.0f));
                    f3 bv = xyz(c.bedv[i]);
                    f3 before = v;
                    v = bv + (v - bv) * damp;
                    f3 wi = g.w * (v - before);
                    bed_impulse_neighborhood(c, ix, iy, iz, (-wi) * BED_REACTION_ALPHA);
                }
            }
            float sp = len3(v);
            if (sp > u.vel_cap) v = v * (u.vel_cap / sp);
            changed = true;
        }
        if (stages & 2) {
            v = boundary_velocity(c, ix, iy, iz, v);
            changed = true;
        }
        if (changed) c.gvel[i] = make_float4(v.x, v.y, v.z, g.w);
    }
}

// ---------------- packing_apply (shader.rs:1586-1626) [+ boundary] ----------------
__device__ __forceinline__ float packing_or_mirror(const Ctx& c, bool in, uint32_t ni, float mirror) {
    if (!in) return mirror;
    int32_t k = lane(c, 3)[ni];
    if (is_solid(k)) return mirror;
    if (!is_fluid(k)) return 0.0f;
    return packing_load(c, ni);
}

__global__ void k_packing_apply(const Ctx* __restrict__ cp, int with_boundary) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    CS_FOR(i, u.cells) {
        float4 g = c.gvel[i];
        if (g.w < 1e-6f) continue;
        uint32_t ix, iy, iz;
        decompose(u, i, ix, iy, iz);
        f3 v = xyz(g);
        int32_t kind = lane(c, 3)[i];
        if (g.w > occupancy_mass(u) && is_fluid(kind)) {
            const uint32_t sy = u.gx, sz = u.gx * u.gy;
            float ph = packing_load(c, i);
            float pxm = packing_or_mirror(c, ix > 0, i - 1, ph), pxp = packing_or_mirror(c, ix + 1 < u.gx, i + 1, ph);
            float pym = packing_or_mirror(c, iy > 0, i - sy, ph), pyp = packing_or_mirror(c, iy + 1 < u.gy, i + sy, ph);
            float pzm = packing_or_mirror(c, iz > 0, i - sz, ph), pzp = packing_or_mirror(c, iz + 1 < u.gz, i + sz, ph);
            float h = 0.5f * u.inv_dx;
            f3 grad = mk(h * (pxp - pxm), h * (pyp - pym), h * (pzp - pzm));
            v = v - u.dt * grad;
            float sp = len3(v);
            if (sp > u.vel_cap) v = v * (u.vel_cap / sp);
        }
        if (with_boundary) v = boundary_velocity(c, ix, iy, iz, v);
        c.gvel[i] = make_float4(v.x, v.y, v.z, g.w);
    }
}

// ---------------- viscosity_prepare (shader.rs:1086-1163) ----------------
__global__ void k_viscosity_prepare(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    CS_FOR(i, u.cells) {
        float4 g = c.gvel[i];
        f3 vh = xyz(g);
        if (g.w <= occupancy_mass(u) || u.viscosity <= 0.0f || g.w <= u.nominal_mass * 2.0f) {
            vscratch_store(c, i, vh);
            continue;
        }
        uint32_t ix, iy, iz;
        decompose(u, i, ix, iy, iz);
        float alpha = wclamp(u.viscosity * u.dt / wmax(u.dx * u.dx, 1e-6f), 0.0f, 0.14f);
        f3 sum = mk(0.0f, 0.0f, 0.0f);
        float ws = 0.0f;
        uint32_t nf = 0;
        const float denom = wmax(wmax(g.w, u.nominal_mass), 1e-6f);
        const uint32_t sy = u.gx, sz = u.gx * u.gy;
#define CS_VFACE(cond, off)                                          \
    if (!(cond) || c.cls[i + (off)] != 0) {                          \
        ws += 1.0f;                                                  \
    } else {                                                         \
        float4 ng = c.gvel[i + (off)];                               \
        if (ng.w > occupancy_mass(u)) {                              \
            float nw = wclamp(ng.w / denom, 0.0f, 1.0f);             \
            sum += xyz(ng) * nw;                                     \
            ws += nw;                                                \
            nf += 1;                                                 \
        }                                                            \
    }
        CS_VFACE(ix > 0, (uint32_t)-1)
        CS_VFACE(ix + 1 < u.gx, 1u)
        CS_VFACE(iy > 0, (uint32_t)0 - sy)
        CS_VFACE(iy + 1 < u.gy, sy)
        CS_VFACE(iz > 0, (uint32_t)0 - sz)
        CS_VFACE(iz + 1 < u.gz, sz)
#undef CS_VFACE
        if (nf < 3 || ws <= 1e-6f) {
            vscratch_store(c, i, vh);
            continue;
        }
        f3 avg = sum / ws;
        float blend = wclamp(alpha * ws, 0.0f, 0.65f);
        vscratch_store(c, i, mix3(vh, avg, blend));
    }
}

// ---------------- viscosity_apply (shader.rs:1166-1177) [+ boundary] ----------------
__global__ void k_viscosity_apply(const Ctx* __restrict__ cp, int with_boundary) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    CS_FOR(i, u.cells) {
        float mass = c.gvel[i].w;
        if (mass <= occupancy_mass(u)) {
            c.gvel[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            continue;
        }
        f3 v = vscratch_load(c, i);
        if (with_boundary && mass >= 1e-6f) {
            uint32_t ix, iy, iz;
            decompose(u, i, ix, iy, iz);
            v = boundary_velocity(c, ix, iy, iz, v);
        }
        c.gvel[i] = make_float4(v.x, v.y, v.z, mass);
    }
}

// ---------------- g2p (shader.rs:1683-1881) ----------------
__device__ __forceinline__ void g2p_particle(const Ctx& c, uint32_t pid) {
    const Params& u = c.u;
    float4 A0 = c.c0[pid];
    float phase = A0.w;
    if (!is_water_phase(phase)) return;
    float4 P = c.pos[pid], Vv = c.vel[pid];
    float mp = Vv.w;
    if (mp <= inactive_mass(u)) {
        c.vel[pid].w = 0.0f;
        return;
    }
    f3 xp = xyz(P);
    float gx = (xp.x - u.ox) * u.inv_dx, gy = (xp.y - u.oy) * u.inv_dx, gz = (xp.z - u.oz) * u.inv_dx;
    int bx = (int)floorf(gx - 0.5f), by = (int)floorf(gy - 0.5f), bz = (int)floorf(gz - 0.5f);
    float fx = gx - (float)bx, fy = gy - (float)by, fz = gz - (float)bz;
    float wx[3], wy[3], wz[3];
    bspline(fx, wx);
    bspline(fy, wy);
    bspline(fz, wz);
    f3 nv = mk(0.0f, 0.0f, 0.0f), n0 = nv, n1 = nv, n2 = nv, bvs = nv;
    float supp = 0.0f, lmass = 0.0f, bow = 0.0f, bperm = 0.0f;
    const float B = 4.0f * u.inv_dx * u.inv_dx;
    const bool has_bed = u.num_bed > 0u;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                int cx = bx + i, cy = by + j, cz = bz + k;
                if (!in_grid(u, cx, cy, cz)) continue;
                float w = wx[i] * wy[j] * wz[k];
                uint32_t ci = cidx(u, cx, cy, cz);
                float4 g = c.gvel[ci];
                if (g.w > 1e-6f) {
                    f3 gv = xyz(g);
                    f3 dpos = mk(((float)i - fx) * u.dx, ((float)j - fy) * u.dx, ((float)k - fz) * u.dx);
                    nv += w * gv;
                    float wb = w * B;
                    n0 += (wb * gv) * dpos.x;
                    n1 += (wb * gv) * dpos.y;
                    n2 += (wb * gv) * dpos.z;
                    supp += w;
                    lmass += w * g.w;
                }
                if (has_bed) {
                    int32_t b = c.lookup[ci];
                    if (valid_bed_solid(c, b)) {
                        bow += w;
                        bvs += w * xyz(c.vel[b]);
                        bperm += w * compacted_permeability(c, (uint32_t)b);
                    }
                }
            }
    float sr = wclamp(supp, 0.0f, 1.0f);
    float jsup = sr;
    if (supp > 1e-6f) {
        float inv = 1.0f / supp;
        nv *= inv;
        n0 *= inv;
        n1 *= inv;
        n2 *= inv;
    }
    float cr = u.cup_radius + u.contact_offset;
    bool in_cup = (u.geom_flags & CS_GEOM_CUP) && xp.y < u.cup_top_y && (xp.x * xp.x + xp.z * xp.z) < cr * cr;
    float dsr = wclamp(lmass / wmax(u.nominal_mass * 4.0f, 1e-6f), 0.0f, 1.0f);
    float po = wclamp(bow, 0.0f, 1.0f);
    f3 pbv = mk(0.0f, 0.0f, 0.0f);
    float pbk = u.min_perm;
    if (bow > 1e-6f) {
        float inv = 1.0f / bow;
        pbv = bvs * inv;
        pbk = wmax(bperm * inv, u.min_perm);
    }
    if (sr < 0.999f) {
        f3 bal = mk(Vv.x, Vv.y + u.gravity * u.dt, Vv.z);
        float pg = mixf(in_cup ? 1.15f : 1.35f, 0.18f, po);
        float pc = mixf(in_cup ? 0.95f : 0.995f, 0.16f, po);
        float dpd = mixf(1.0f, 0.12f, dsr);
        float pres = wclamp((1.0f - sr) * pg * dpd, 0.0f, pc);
        nv = mix3(nv, bal, pres);
        float ad = 1.0f - pres * 0.75f;
        n0 *= ad;
        n1 *= ad;
        n2 *= ad;
    }
    bool airborne = po <= 0.05f && sample_sdf(c, xp) > u.contact_offset * 2.0f;
    if (airborne) {
        float dr = wclamp(lmass / wmax(u.nominal_mass * 4.0f, 1e-6f), 0.0f, 1.0f);
        jsup = wmin(jsup, dr);
        f3 bal = mk(Vv.x, Vv.y + u.gravity * u.dt, Vv.z);
        float pg = in_cup ? 0.72f : 0.98f;
        float pc = in_cup ? 0.88f : 0.98f;
        float pres = wclamp((1.0f - dr) * pg, 0.0f, pc);
        nv = mix3(nv, bal, pres);
        float ad = 1.0f - pres * 0.65f;
        n0 *= ad;
        n1 *= ad;
        n2 *= ad;
    }
    if (po > 1e-4f) {
        f3 rel = nv - pbv;
        float rate = u.nu_m2s / pbk;
        float dd = 1.0f / (1.0f + wmax(rate * u.dt * po, 0.0f));
        float rs = len3(rel);
        float idmp = 1.0f / (1.0f + wmax(rs * u.dt * u.inv_dx * po * 0.35f, 0.0f));
        f3 before = nv;
        nv = pbv + rel * dd * idmp;
        f3 wi = mp * (nv - before);
        int wx_, wy_, wz_;
        world_to_cell(u, xp, wx_, wy_, wz_);
        bed_impulse_neighborhood(c, wx_, wy_, wz_, (-wi) * BED_REACTION_ALPHA);
        float ad = mixf(1.0f, dd * idmp, po);
        n0 *= ad;
        n1 *= ad;
        n2 *= ad;
        jsup = wmax(jsup, po);
    }
    float tr = n0.x + n1.y + n2.z;
    float jo = clamp_j(P.w > 0.0f ? P.w : 1.0f);
    float ja = clamp_j(jo * exp_small(wclamp(u.dt * tr, -0.35f, 0.35f)));
    float jb = smoothstepf(0.35f, 0.85f, wclamp(jsup, 0.0f, 1.0f));
    float jn = clamp_j(mixf(jo, ja, jb));
    f3 np = xp + nv * u.dt;
    f3 cpos = mix3(xp, np, 0.5f);
    f3 cvel = nv;
    sdf_contact(c, cpos, cvel, false);
    cpos = np;
    sdf_contact(c, cpos, cvel, false);
    np = cpos;
    nv = cvel;
    float m = u.dx * 0.5f;
    np.x = wclamp(np.x, u.ox + m, u.bx - m);
    np.y = wclamp(np.y, u.oy + m, u.by - m);
    np.z = wclamp(np.z, u.oz + m, u.bz - m);
    c.pos[pid] = make_float4(np.x, np.y, np.z, jn);
    c.vel[pid] = make_float4(nv.x, nv.y, nv.z, mp);
    c.c0[pid] = make_float4(n0.x, n0.y, n0.z, phase);
    c.c1[pid] = make_float4(n1.x, n1.y, n1.z, 0.0f);
    c.c2[pid] = make_float4(n2.x, n2.y, n2.z, 0.0f);
}

// 64 registers (four 256-thread blocks per SM) instead of 80: the kernel is bound by the
// latency of its grid, lookup and SDF gathers, and more resident warps hide more of it
__global__ void __launch_bounds__(256, 4) k_g2p(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    uint32_t n = c.u.num_water + c.u.num_bed;
    CS_FOR(pid, n) g2p_particle(c, pid);
}

// ---------------- bed_coupling (shader.rs:1885-1957) ----------------
__device__ float filter_paper_weight(const Params& u, f3 p) {
    float ftop = filter_top_y(u), fbot = filter_bot_y(u);
    float pr = wmax(water_particle_radius(u), u.dx * 0.35f);
    if (p.y < fbot - pr || p.y > ftop + pr) return 0.0f;
    float ft = wclamp((p.y - fbot) / (ftop - fbot), 0.0f, 1.0f);
    float outer = mixf(0.0f, u.filter_top_radius, ft);
    float inner = wmax(outer - u.filter_thickness, 0.0f);
    float r = len2(p.x, p.z);
    float side = 1.0f - smoothstepf(pr, pr * 3.0f, fabsf(r - inner));
    float lv = 1.0f - smoothstepf(0.0f, pr * 5.0f, wmax(p.y - fbot, 0.0f));
    float lr = 1.0f - smoothstepf(inner, inner + pr * 3.0f, r);
    return wclamp(wmax(side, lv * lr), 0.0f, 1.0f);
}

__global__ void k_bed_coupling(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    uint32_t n = u.num_water + u.num_bed;
    CS_FOR(pid, n) {
        if (!is_water_phase(c.c0[pid].w)) continue;
        float4 P = c.pos[pid];
        f3 pos = xyz(P);
        int cx, cy, cz;
        world_to_cell(u, pos, cx, cy, cz);
        if (!in_grid(u, cx, cy, cz)) continue;
        float4 Vv = c.vel[pid];
        float mp = Vv.w;
        float pw = filter_paper_weight(u, pos);
        if (pw > 1e-4f && u.filter_absorption > 0.0f) {
            float frac = wclamp(u.filter_absorption * pw * u.dt, 0.0f, 0.04f);
            float ab = wmin(mp * frac, mp * 0.12f);
            mp = wmax(mp - ab, inactive_mass(u) * 1.25f);
            Vv.w = mp;
            c.vel[pid] = Vv;
        }
        int32_t b = c.lookup[cidx(u, cx, cy, cz)];
        if (b < 0 || (uint32_t)b >= u.num_bed) continue;
        float4 BA = c.bedA[b];
        float sat = c.bedB[b].w;
        float cap = wmax(u.max_saturation - BA.x, 0.0f);
        if (cap <= 1e-6f) continue;
        float ar = u.absorption_rate * (1.0f - sat) * u.dt;
        float speed = len3(xyz(Vv));
        float absorbed = wmin(wmin(mp * wclamp(ar, 0.0f, 0.25f), mp * 0.5f), cap);
        float rem_partial = mp - absorbed;
        if (rem_partial > 0.0f && rem_partial <= u.nominal_mass * 0.22f) {
            absorbed = wmin(mp, cap);
        } else if (sat > 0.55f && speed < 1.35f) {
            float almost = wmin(mp, cap);
            if (mp - almost <= u.nominal_mass * 0.35f) absorbed = almost;
        }
        if (mp - absorbed <= inactive_mass(u) && absorbed < mp) absorbed = wmax(mp - inactive_mass(u) * 1.05f, 0.0f);
        if (absorbed <= 1e-6f) continue;
        float remaining = mp - absorbed;
        if (remaining <= inactive_mass(u)) c.vel[pid] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        else c.vel[pid] = make_float4(Vv.x, Vv.y, Vv.z, remaining);
        // deposit_absorbed_bed_water (shader.rs:524-576)
        float ns = absorbed * 0.35f;
        float hs = absorbed - ns;
        bed_water_add(c, (uint32_t)b, hs);
        int32_t ids[6];
        uint32_t cnt = 0;
        const int off[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            int x = cx + off[q][0], y = cy + off[q][1], z = cz + off[q][2];
            if (!in_grid(u, x, y, z)) continue;
            int32_t nid = c.lookup[cidx(u, x, y, z)];
            if (nid < 0 || nid == b || (uint32_t)nid >= u.num_bed) continue;
            bool dup = false;
            for (uint32_t k = 0; k < cnt; ++k) dup |= ids[k] == nid;
            if (!dup) ids[cnt++] = nid;
        }
        if (cnt == 0) {
            bed_water_add(c, (uint32_t)b, ns);
        } else {
            float each = ns / (float)cnt;
            for (uint32_t k = 0; k < cnt; ++k) bed_water_add(c, (uint32_t)ids[k], each);
        }
    }
}

// ---------------- extraction_advect (shader.rs:1961-1987) + Jacobi snapshot ----------------
__global__ void k_extraction_advect(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    CS_FOR(b, u.num_bed) {
        float4 A = c.bedA[b], Bb = c.bedB[b];
        int32_t raw = atomicExch(&delta_lane(c, 0)[b], 0);
        float absorbed = (float)raw * INV_FP_SCALE;
        if (absorbed > 0.0f) {
            A.x += absorbed;
            Bb.w = wclamp(A.x / wmax(u.max_saturation, 1e-6f), 0.0f, 1.0f);
        }
        if (Bb.w > 0.01f) {
            float flux = u.extraction_rate * Bb.x * Bb.w * u.dt;
            Bb.x = wmax(Bb.x - flux, 0.0f);
            Bb.y += flux;
        }
        c.bedA[b] = A;
        c.bedB[b] = Bb;
        c.snap[b] = c.pos[b];
    }
}

// ---------------- bed_dynamics (shader.rs:1991-2238) ----------------
__device__ __forceinline__ float pressure_or_mirror_aliased(const Ctx& c, int x, int y, int z, float mirror) {
    // shader.rs:224-236: the "kind" read here is lane 3, which viscosity_prepare has
    // overwritten with FP velocity z by the time bed_dynamics runs; kept as is.
    if (!in_grid(c.u, x, y, z)) return mirror;
    uint32_t ci = cidx(c.u, x, y, z);
    if (is_solid(lane(c, 3)[ci])) return mirror;
    return pressure_load(c, ci);
}

__global__ void k_bed_dynamics(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    CS_FOR(bid, u.num_bed) {
        float4 P = c.pos[bid], Vv = c.vel[bid], A0 = c.c0[bid], A1 = c.c1[bid];
        float4 BA = c.bedA[bid], BB = c.bedB[bid];
        float phase = A0.w;
        f3 rest = xyz(A1);
        f3 pos = xyz(P);
        float mp = Vv.w;
        int32_t ex = atomicExch(&delta_lane(c, 1)[bid], 0);
        int32_t ey = atomicExch(&delta_lane(c, 2)[bid], 0);
        int32_t ez = atomicExch(&delta_lane(c, 3)[bid], 0);
        f3 brv = mk((float)ex, (float)ey, (float)ez) * INV_FP_SCALE;
        brv = brv / wmax(mp, u.nominal_mass * 0.25f);
        float mrs = wmin(u.vel_cap * 0.012f, u.dx / wmax(u.dt, 1e-6f) * 0.02f);
        float rsp = len3(brv);
        if (rsp > mrs && rsp > 1e-6f) brv *= mrs / rsp;
        float gx = (pos.x - u.ox) * u.inv_dx, gy = (pos.y - u.oy) * u.inv_dx, gz = (pos.z - u.oz) * u.inv_dx;
        int bx = (int)floorf(gx - 0.5f), by = (int)floorf(gy - 0.5f), bz = (int)floorf(gz - 0.5f);
        float fx = gx - (float)bx, fy = gy - (float)by, fz = gz - (float)bz;
        float wx[3], wy[3], wz[3];
        bspline(fx, wx);
        bspline(fy, wy);
        bspline(fz, wz);
        f3 wv = mk(0.0f, 0.0f, 0.0f);
        float wm = 0.0f, asw = 0.0f, lasw = 0.0f;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) {
                    int cx = bx + i, cy = by + j, cz = bz + k;
                    if (!in_grid(u, cx, cy, cz)) continue;
                    float w = wx[i] * wy[j] * wz[k];
                    uint32_t ci = cidx(u, cx, cy, cz);
                    float4 g = c.gvel[ci];
                    wv += w * xyz(g);
                    wm += w * g.w;
                    int32_t sb = c.lookup[ci];
                    if (sb >= 0 && (uint32_t)sb != bid) {
                        asw += w;
                        float ccy = u.oy + ((float)cy + 0.5f) * u.dx;
                        if (ccy <= pos.y + u.dx * 0.25f) lasw += w;
                    }
                }
        const float floor_y = coffee_floor_y(u);
        if (is_suspended(phase)) {
            float ws = wclamp(wm / wmax(u.nominal_mass * 2.0f, 1e-6f), 0.0f, 1.0f);
            float drag = wclamp((8.0f + 18.0f * ws) * u.dt, 0.0f, 1.0f);
            f3 unsup = xyz(Vv) + brv + mk(0.0f, u.gravity * u.dt * 0.85f, 0.0f);
            float settle = mixf(1.10f, 0.32f, ws);
            f3 carried = wv + mk(0.0f, -settle, 0.0f);
            f3 sv = mix3(unsup, carried, drag);
            float sp = len3(sv);
            if (sp > u.vel_cap) sv = sv * (u.vel_cap / sp);
            f3 sp_pos = pos + sv * u.dt;
            sdf_contact(c, sp_pos, sv, true);
            c.pos[bid] = make_float4(sp_pos.x, sp_pos.y, sp_pos.z, P.w);
            c.vel[bid] = make_float4(sv.x, sv.y, sv.z, mp);
            bool anch = lasw > 0.06f || asw > 0.20f;
            bool dense = asw > 0.42f;
            bool redep = (sp_pos.y <= floor_y + u.dx * 0.35f && ws < 0.35f) ||
                         (anch && sv.y <= 0.20f && (ws < 0.55f || dense));
            if (redep) phase = 1.0f;
            c.c0[bid] = make_float4(A0.x, A0.y, A0.z, phase);
            c.c1[bid] = make_float4(sp_pos.x, sp_pos.y, sp_pos.z, 0.0f);
            BA.w *= 0.985f;
            c.bedA[bid] = BA;
            continue;
        }
        float sat = BB.w;
        float wl = wclamp(wm / wmax(u.nominal_mass * 1.5f, 1e-6f), 0.0f, 1.0f);
        float mob = wclamp((0.30f + wl * 0.62f) * (1.0f + sat * 0.40f), 0.0f, 1.0f);
        float sfac = wclamp((rest.y + u.bed_surface_ref_y) / u.bed_surface_span, 0.12f, 1.0f);
        float damping = wclamp(1.0f - u.bed_damping * u.dt, 0.0f, 1.0f);
        f3 vel = xyz(Vv) + brv;
        float srel = wclamp(1.0f - asw / 0.55f, 0.0f, 1.0f);
        float ed = wclamp((2.0f + 5.0f * sat) * wl * srel * u.dt, 0.0f, 0.08f);
        f3 gsv = mk(0.0f, -mixf(0.95f, 0.35f, wl), 0.0f);
        vel = mix3(vel, wv + gsv, ed);
        float ls = len2(wv.x, wv.z);
        float ldx = 0.0f, ldz = 0.0f;
        if (ls > 1e-6f) {
            ldx = wv.x / ls;
            ldz = wv.z / ls;
        }
        float lss = wmin(ls, fabsf(wmin(wv.y, 0.0f)) * 0.18f);
        f3 iv = mk(ldx * lss * 0.08f, wmin(wv.y, 0.0f) * 0.62f, ldz * lss * 0.08f);
        vel += iv * u.bed_impact * mob * sfac * u.dt;
        int pcx, pcy, pcz;
        world_to_cell(u, pos, pcx, pcy, pcz);
        float pgx = 0.0f, pgz = 0.0f;
        if (in_grid(u, pcx, pcy, pcz)) {
            float ph = pressure_load(c, cidx(u, pcx, pcy, pcz));
            float pxm = pressure_or_mirror_aliased(c, pcx - 1, pcy, pcz, ph);
            float pxp = pressure_or_mirror_aliased(c, pcx + 1, pcy, pcz, ph);
            float pzm = pressure_or_mirror_aliased(c, pcx, pcy, pcz - 1, ph);
            float pzp = pressure_or_mirror_aliased(c, pcx, pcy, pcz + 1, ph);
            float h = 0.5f * u.inv_dx;
            pgx = h * (pxp - pxm);
            pgz = h * (pzp - pzm);
        }
        float sfx = -pgx, sfz = -pgz;
        float ssp = len2(sfx, sfz);
        float sdx = 0.0f, sdz = 0.0f;
        if (ssp > 1e-6f) {
            sdx = sfx / ssp;
            sdz = sfz / ssp;
        }
        float pdrive = wmin(ssp, u.vel_cap / wmax(u.dt, 1e-6f));
        float pload = wclamp(wm * (0.25f + sat), 0.0f, 1.0f);
        float slx = sdx * pdrive * pload * 0.08f, slz = sdz * pdrive * pload * 0.08f;
        vel.x += slx * u.bed_impact * mob * sfac * u.dt;
        vel.z += slz * u.bed_impact * mob * sfac * u.dt;
        vel *= damping;
        f3 npos = pos + vel * u.dt;
        f3 off = npos - rest;
        float ll = len2(off.x, off.z);
        float lpt = u.dx * 0.22f;
        if (ll > lpt && ll > 1e-6f) {
            float lx = off.x / ll, lz = off.z / ll;
            float lex = ll - lpt;
            float lpl = wclamp((0.04f + sat * 0.35f + mob * 0.45f + pload * 0.25f) * sfac * u.compaction_rate * u.dt,
                               0.0f, 0.18f);
            rest.x += lx * lex * lpl;
            rest.z += lz * lex * lpl;
            off = npos - rest;
        }
        float cll = len2(off.x, off.z);
        float mlat = u.dx * 0.9f * sfac;
        if (cll > mlat && cll > 1e-6f) {
            float lx = off.x / cll, lz = off.z / cll;
            off.x = lx * mlat;
            off.z = lz * mlat;
            vel.x *= 0.4f;
            vel.z *= 0.4f;
        }
        off.y = wclamp(off.y, -u.dx * (1.75f * sfac + 0.2f), u.dx * 0.04f);
        npos = rest + off;
        // resolve_coffee_particle_packing (shader.rs:825-877) against the snapshot
        {
            f3 cd = mk(0.0f, 0.0f, 0.0f);
            float cdist = 1e9f;
            bool found = false;
            int qx, qy, qz;
            world_to_cell(u, npos, qx, qy, qz);
            for (int di = -1; di <= 1; ++di)
                for (int dj = -1; dj <= 1; ++dj)
                    for (int dk = -1; dk <= 1; ++dk) {
                        int x = qx + di, y = qy + dj, z = qz + dk;
                        if (!in_grid(u, x, y, z)) continue;
                        int32_t o = c.lookup[cidx(u, x, y, z)];
                        if (o < 0 || (uint32_t)o == bid || (uint32_t)o >= u.num_bed) continue;
                        f3 d = npos - xyz(c.snap[o]);
                        float dist = len3(d);
                        if (dist < cdist) {
                            cdist = dist;
                            cd = d;
                            found = true;
                        }
                    }
            float min_sep = bed_particle_radius(u) * 1.78f;
            if (found && cdist < min_sep) {
                f3 n = mk(0.0f, 1.0f, 0.0f);
                if (cdist > 1e-5f) n = cd / cdist;
                npos += n * wmin((min_sep - cdist) * 0.65f, u.dx * 0.22f);
                float vn = dot3(vel, n);
                if (vn < 0.0f) vel -= n * vn;
            }
        }
        float comp = wmax(rest.y - npos.y, 0.0f);
        float pth = u.dx * 0.18f;
        if (comp > pth) {
            float pl = wclamp((0.05f + sat * 0.35f + mob * 0.55f) * sfac * u.compaction_rate * u.dt, 0.0f, 0.18f);
            rest.y -= (comp - pth) * pl;
        }
        bool hd = sat > 0.82f && pload > 0.65f && wl > 0.65f && srel > 0.35f &&
                  (comp > u.dx * 0.65f || cll > u.dx * 0.65f);
        bool fe = sat > 0.58f && wl > 0.74f && srel > 0.55f && len3(wv) > 0.95f && npos.y > floor_y + u.dx * 0.70f;
        bool iso = sat > 0.55f && wm < u.nominal_mass * 0.75f && asw < 0.04f && lasw < 0.03f &&
                   npos.y > floor_y + u.dx * 0.50f;
        if (hd || fe || iso) {
            phase = 2.0f;
            rest = npos;
        }
        sdf_contact(c, npos, vel, true);
        c.pos[bid] = make_float4(npos.x, npos.y, npos.z, P.w);
        c.vel[bid] = make_float4(vel.x, vel.y, vel.z, mp);
        c.c0[bid] = make_float4(A0.x, A0.y, A0.z, phase);
        c.c1[bid] = make_float4(rest.x, rest.y, rest.z, 0.0f);
        float gc = wmax((rest.y - npos.y) / wmax(u.dx, 1e-6f), 0.0f);
        BA.w = wmax(BA.w * 0.995f, gc);
        c.bedA[bid] = BA;
    }
}

// ---------------- prepare_render (shader.rs:2242-2276) ----------------
__global__ void k_prepare_render(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    uint32_t n = u.num_water + u.num_bed;
    CS_FOR(pid, n) {
        float4 P = c.pos[pid], Vv = c.vel[pid];
        float phase = c.c0[pid].w;
        if (Vv.w <= inactive_mass(u)) {
            c.render[2 * (size_t)pid] = make_float4(0.0f, -1e6f, 0.0f, -999.0f);
            c.render[2 * (size_t)pid + 1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            continue;
        }
        float ct;
        float rad = water_particle_radius(u);
        if (is_water_phase(phase)) {
            ct = wclamp(len3(xyz(Vv)) / 10.0f, 0.0f, 2.0f);
        } else {
            float sat = 0.0f;
            if (pid < u.num_bed) {
                sat = c.bedB[pid].w;
                rad = bed_particle_radius(u);
            }
            ct = -1.0f - sat;
        }
        c.render[2 * (size_t)pid] = make_float4(P.x, P.y, P.z, ct);
        c.render[2 * (size_t)pid + 1] = make_float4(rad, 0.0f, 0.0f, 0.0f);
    }
}

// ---------------- readback helpers ----------------
// Reference AoS layouts from the SoA streams.
__global__ void k_pack_particles(const Ctx* __restrict__ cp, uint32_t first, uint32_t count, float* out, int what) {
    const Ctx& c = cp[blockIdx.y];
    CS_FOR(k, count) {
        uint32_t p = first + k;
        if (what == 0) {
            float4 a = c.pos[p], b = c.vel[p];
            float* o = out + (size_t)k * 8;
            o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
            o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
        } else if (what == 1) {
            float4 a = c.c0[p], b = c.c1[p], d = c.c2[p];
            float* o = out + (size_t)k * 12;
            o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
            o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
            o[8] = d.x; o[9] = d.y; o[10] = d.z; o[11] = d.w;
        } else if (what == 2) {
            float4 a = c.bedA[p], b = c.bedB[p];
            float* o = out + (size_t)k * 8;
            o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
            o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
        } else {
            float4 a = c.render[2 * (size_t)p], b = c.render[2 * (size_t)p + 1];
            float* o = out + (size_t)k * 8;
            o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
            o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
        }
    }
}
// Device jet emission (inflow.rs:196-218): sample i of the substep at golden-angle
// position first_sequence + i on the nozzle disk, back-dated by its age.  cos/sin are
// the double-precision values rounded to float (the oracle's device-emission mode does
// the same; inflow.rs evaluates them in f32).
__global__ void k_emit_jet(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    const JetPlan& j = c.u.jet;
    const float golden = 2.399963f, radial = 0.7548777f;
    CS_FOR(i, j.count) {
        const float sf = (float)(uint32_t)(j.first_sequence + i);
        float ru = (sf + 0.5f) * radial;
        ru = ru - truncf(ru);
        const float r = j.jet_radius * sqrtf(ru);
        const float theta = sf * golden;
        const float age = (((float)i + 0.5f) / (float)j.count) * j.dt;
        const float ct = (float)cos((double)theta), st = (float)sin((double)theta);
        float p[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float off = j.t1[k] * r * ct + j.t2[k] * r * st;
            p[k] = j.origin[k] + off - j.vel[k] * age;
        }
        const uint32_t s = j.first_slot + i;
        c.pos[s] = make_float4(p[0], p[1], p[2], 1.0f);
        c.vel[s] = make_float4(j.vel[0], j.vel[1], j.vel[2], j.particle_mass);
        const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        c.c0[s] = z;
        c.c1[s] = z;
        c.c2[s] = z;
    }
}

// Per-substep clears of every ensemble instance in one launch (the memsets of the
// single-simulation path): P2G lanes, grid velocity, bed lookup, metrics, tile counts.
__global__ void k_clear_batch(const Ctx* __restrict__ cp, uint32_t tiles) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    CS_FOR(i, u.cells) {
#pragma unroll
        for (int l = 0; l < 6; ++l) c.lanes[(size_t)l * u.cells + i] = 0;
        if (u.int64_grid)
#pragma unroll
            for (int l = 0; l < 6; ++l) c.lanes64[(size_t)l * u.cells + i] = 0;
        c.gvel[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        c.lookup[i] = -1;
    }
    CS_FOR(t, tiles) c.tile_count[t] = 0u;
    if (blockIdx.x == 0 && threadIdx.x < 8) c.metrics[threadIdx.x] = 0u;
}
// Copy each instance's solve result into one array (one readback for the ensemble).
__global__ void k_gather_results(const Ctx* __restrict__ cp, uint32_t n, ScResult* __restrict__ out) {
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) out[i] = *cp[i].sb.result;
}

// ---- learned warm start: network inputs, guess, training targets ----
// The inputs come after an FP64 residual evaluation of the previous-substep pressure
// (k_refine_residual leaves r in gres): the network maps the residual to a pressure
// correction, an approximate inverse of the pressure operator.
// acc[0] += r^2, acc[1] += 1 over fluid cells
// Per-block partial sums (sum r^2, fluid cells) of the residual over the fluid cells in
// acc[2 * block], acc[2 * block + 1]; the last block to finish adds them in block order
// into acc[2 * kLearnedStatBlocks], acc[2 * kLearnedStatBlocks + 1], so the totals do not
// depend on the order blocks finish in.  The finish counter sits after them and is left
// at zero.
constexpr int kLearnedStatBlocks = 296;
__global__ void k_learned_stats(const Ctx* __restrict__ cp, double* __restrict__ acc) {
    const Ctx& c = cp[blockIdx.y];
    const int32_t* kl = lane(c, 3);
    __shared__ double part[2][32];
    double r2 = 0.0, n = 0.0;
    CS_FOR(i, c.u.cells) {
        if (!is_fluid(kl[i])) continue;
        const double r = (double)c.gres[i];
        r2 += r * r;
        n += 1.0;
    }
    for (int o = 16; o > 0; o >>= 1) {
        r2 += __shfl_down_sync(0xffffffffu, r2, o);
        n += __shfl_down_sync(0xffffffffu, n, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        part[0][w] = r2;
        part[1][w] = n;
    }
    __syncthreads();
    __shared__ bool last;
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            a += part[0][k];
            b += part[1][k];
        }
        acc[2 * blockIdx.x] = a;
        acc[2 * blockIdx.x + 1] = b;
        __threadfence();
        unsigned int* done = reinterpret_cast<unsigned int*>(acc + 2 * kLearnedStatBlocks + 2);
        last = atomicAdd(done, 1u) == gridDim.x - 1;
        if (last) *done = 0u;
    }
    __syncthreads();
    if (last && threadIdx.x < 32) {
        // lane l adds partials l, l + 32, ... in order, then a fixed shuffle tree
        __threadfence();
        double ta = 0.0, tb = 0.0;
        for (int k = threadIdx.x; k < (int)gridDim.x; k += 32) {
            ta += __ldcg(acc + 2 * k);
            tb += __ldcg(acc + 2 * k + 1);
        }
        for (int o = 16; o > 0; o >>= 1) {
            ta += __shfl_down_sync(0xffffffffu, ta, o);
            tb += __shfl_down_sync(0xffffffffu, tb, o);
        }
        if (threadIdx.x == 0) {
            acc[2 * kLearnedStatBlocks] = ta;
            acc[2 * kLearnedStatBlocks + 1] = tb;
        }
    }
}
// 8 channels per cell: r / s, fill, fluid, bed, solid, 0, 0, 0 with s the RMS of the
// residual over the fluid cells (written to scale[0])
__global__ void k_learned_features(const Ctx* __restrict__ cp, const double* __restrict__ acc,
                                   __nv_bfloat16* __restrict__ feat, float* __restrict__ scale) {
    const Ctx& c = cp[blockIdx.y];
    const int32_t* kl = lane(c, 3);
    const double* tot = acc + 2 * kLearnedStatBlocks;
    const double ms = tot[1] > 0.0 ? tot[0] / tot[1] : 0.0;
    const float sc = ms > 0.0 ? (float)sqrt(ms) : 1.0f;
    const float inv = 1.0f / sc;
    if (blockIdx.x == 0 && threadIdx.x == 0) scale[0] = sc;
    CS_FOR(i, c.u.cells) {
        const int32_t k = kl[i];
        const bool fl = is_fluid(k);
        float f[8];
        f[0] = fl ? c.gres[i] * inv : 0.0f;
        f[1] = fl ? c.fill[i] : 0.0f;
        f[2] = fl ? 1.0f : 0.0f;
        f[3] = k == CELL_BED ? 1.0f : 0.0f;
        f[4] = is_solid(k) ? 1.0f : 0.0f;
        f[5] = 0.0f;
        f[6] = 0.0f;
        f[7] = 0.0f;
        __align__(16) __nv_bfloat16 h[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) h[q] = __float2bfloat16(f[q]);
        *reinterpret_cast<uint4*>(feat + (size_t)i * 8) = *reinterpret_cast<const uint4*>(h);
    }
}
// the previous-substep pressure (the plain warm start) kept for the correction
// target and for the rule that keeps whichever start has the smaller residual
__global__ void k_learned_save(const Ctx* __restrict__ cp, float* __restrict__ bak_hi, float* __restrict__ bak_lo) {
    const Ctx& c = cp[blockIdx.y];
    CS_FOR(i, c.u.cells) {
        bak_hi[i] = c.pf[i];
        bak_lo[i] = c.plo[i];
    }
}
// guess = previous pressure + out * s on fluid cells (the network predicts the change
// of the pressure over the substep in units of s), split into hi/lo words
__global__ void k_learned_apply(const Ctx* __restrict__ cp, const float* __restrict__ out,
                                const float* __restrict__ scale, const float* __restrict__ bak_hi,
                                const float* __restrict__ bak_lo) {
    const Ctx& c = cp[blockIdx.y];
    const int32_t* kl = lane(c, 3);
    const double sc = (double)scale[0];
    CS_FOR(i, c.u.cells) {
        if (!is_fluid(kl[i])) continue;
        const double p = ((double)bak_hi[i] + (double)bak_lo[i]) + (double)out[i] * sc;
        const float hi = (float)p;
        c.pf[i] = hi;
        c.plo[i] = (float)(p - (double)hi);
    }
}
// The acceptance test of the learned guess, on the device: prev and guess hold the FP64
// sums (r^2, b^2) of the residual before and after the guess; the guess is kept when its
// relative residual is below 0.999x the previous one (the FP64 sums are reduced with
// atomics, so equal pressures can differ in their last bits).
__global__ void k_learned_decide(const double* __restrict__ prev, const double* __restrict__ guess,
                                 uint32_t* __restrict__ keep) {
    const double rp = prev[1] > 0.0 ? sqrt(prev[0]) / sqrt(prev[1]) : 0.0;
    const double rg = guess[1] > 0.0 ? sqrt(guess[0]) / sqrt(guess[1]) : 0.0;
    keep[0] = rg < 0.999 * rp ? 1u : 0u;
}
// previous-substep pressure back in place, unless the guess was kept (keep may be null:
// always restore)
__global__ void k_learned_restore(const Ctx* __restrict__ cp, const float* __restrict__ bak_hi,
                                  const float* __restrict__ bak_lo, const uint32_t* __restrict__ keep) {
    const Ctx& c = cp[blockIdx.y];
    if (keep && keep[0]) return;
    CS_FOR(i, c.u.cells) {
        c.pf[i] = bak_hi[i];
        c.plo[i] = bak_lo[i];
    }
}
// training pair of this substep: target = (solved - previous pressure) / s, mask = fluid
__global__ void k_learned_target(const Ctx* __restrict__ cp, const float* __restrict__ scale,
                                 const float* __restrict__ bak_hi, const float* __restrict__ bak_lo,
                                 float* __restrict__ target, float* __restrict__ mask) {
    const Ctx& c = cp[blockIdx.y];
    const int32_t* kl = lane(c, 3);
    const double inv = 1.0 / (double)scale[0];
    CS_FOR(i, c.u.cells) {
        const bool fl = is_fluid(kl[i]);
        const double d = ((double)c.pf[i] + (double)c.plo[i]) - ((double)bak_hi[i] + (double)bak_lo[i]);
        target[i] = fl ? (float)(d * inv) : 0.0f;
        mask[i] = fl ? 1.0f : 0.0f;
    }
}

__global__ void k_unpack_particles(const Ctx* __restrict__ cp, uint32_t first, uint32_t count, const float* in, int what) {
    const Ctx& c = cp[blockIdx.y];
    CS_FOR(k, count) {
        uint32_t p = first + k;
        if (what == 0) {
            const float* s = in + (size_t)k * 8;
            c.pos[p] = make_float4(s[0], s[1], s[2], s[3]);
            c.vel[p] = make_float4(s[4], s[5], s[6], s[7]);
        } else if (what == 1) {
            const float* s = in + (size_t)k * 12;
            c.c0[p] = make_float4(s[0], s[1], s[2], s[3]);
            c.c1[p] = make_float4(s[4], s[5], s[6], s[7]);
            c.c2[p] = make_float4(s[8], s[9], s[10], s[11]);
        } else {
            const float* s = in + (size_t)k * 8;
            c.bedA[p] = make_float4(s[0], s[1], s[2], s[3]);
            c.bedB[p] = make_float4(s[4], s[5], s[6], s[7]);
        }
    }
}
// Pressure as float; lanes with lane 0 re-encoded in FP32 mode.
__global__ void k_pressure_out(const Ctx* __restrict__ cp, float* out) {
    const Ctx& c = cp[blockIdx.y];
    CS_FOR(i, c.u.cells) out[i] = pressure_load(c, i);
}
__global__ void k_lane0_encode(const Ctx* __restrict__ cp, int32_t* out) {
    const Ctx& c = cp[blockIdx.y];
    CS_FOR(i, c.u.cells) out[i] = c.u.fixed_point ? c.lanes[i] : to_i32(c.pf[i] * FP_SCALE);
}

}  // namespace cs
