// cs_device.cuh — per-simulation device context and WGSL-semantics math for the
// sm_100a kernels.
//
// Arithmetic contract (what makes results reproducible against the CPU oracle):
//  * the library is compiled with -fmad=false: every multiply and add rounds on its
//    own, in the order the reference WGSL writes it (crates/sim-wasm/src/mpm_3d/
//    shader.rs); division and sqrt are IEEE round-to-nearest (nvcc defaults);
//  * WGSL mix(a,b,t) = a*(1-t) + b*t, clamp = min(max()), smoothstep, fract(x) =
//    x - floor(x); i32(f) truncates and saturates (cvt.rzi.sat);
//  * exp() in the J update is a degree-10 Taylor polynomial (Horner) on |x| <= 0.35.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/coffee_sim.h"
#include "solver_types.cuh"

namespace cs {

enum : int32_t { CELL_AIR = 0, CELL_SURFACE = 1, CELL_INTERIOR = 2, CELL_BED = 3, CELL_SOLID = 4 };
enum : int { M_MAX_DIV = 0, M_FLUID = 1, M_DIV_CLAMP = 2, M_P_CLAMP = 3, M_OVERFLOW = 4, M_NAN = 5, M_TIMEOUT = 6 };
constexpr float FP_SCALE = 262144.0f;            // state.rs:13, 2^18
constexpr float INV_FP_SCALE = 1.0f / 262144.0f;
constexpr float FP_SCALE64 = 4294967296.0f;      // int64 P2G mode, 2^32
constexpr float INV_FP_SCALE64 = 1.0f / 4294967296.0f;
constexpr float FP_VALUE_LIMIT = 8192.0f;        // state.rs:18
constexpr float METRICS_DIV_FP_SCALE = 1024.0f;  // state.rs:28
constexpr double FP64_SCALE = 4294967296.0;      // 2^32, int64 P2G mode
constexpr float BED_REACTION_ALPHA = 0.04f;      // shader.rs:76
constexpr float BED_REACTION_IMPULSE_CAP = 0.012f;
constexpr int SDF_RES = 128;                     // state.rs:20

// One substep's jet emission, planned on the host (inflow.rs:133-189) and built on
// the device (inflow.rs:196-218).
struct JetPlan {
    float t1[3], t2[3], vel[3], origin[3];
    float jet_radius, dt, particle_mass;
    uint32_t first_sequence, count, first_slot;
};

// Uniform block of one substep (the values of mod.rs:569-670; names follow
// shader.rs:81-134).  Constants the reference hard-codes in the WGSL come from
// CsGeometry so other cones can be simulated.
struct Params {
    uint32_t gx, gy, gz, cells;
    uint32_t num_water, num_bed, max_p, use_sdf_cache;
    float dt, gravity, dx, inv_dx;
    float ox, oy, oz;          // grid origin
    float bx, by, bz;          // bounds max
    float bulk_K, viscosity, nominal_mass, p_vol;
    float vel_cap, outlet_r, top_r;
    float friction, restitution, contact_offset;
    float nu_m2s, absorption_rate, max_saturation, min_perm;
    float extraction_rate, compaction_rate, bed_damping, bed_impact;
    float pore_capacity_scale, pore_overfill_alpha;
    float div_clamp, p_clamp;  // fixed-point lane limits (state.rs:18)
    float p_limit;             // pressure limit: p_clamp with fixed-point storage, none with FP32
    float j_alpha, j_expand_alpha, max_rest_frac, surface_void_scale;
    float water_r_dx, bed_r_dx, filter_absorption;
    // geometry
    uint32_t geom_flags;
    float cone_bot_y, cone_top_y;
    float filter_center_y, filter_top_rel, filter_bot_rel, filter_top_radius, filter_thickness;
    float cup_top_y, cup_radius, cup_floor_y, wall_thickness;
    float bed_surface_ref_y, bed_surface_span;
    // modes
    uint32_t fixed_point;      // pressure/divergence stored as i32*2^18
    uint32_t int64_grid;       // P2G accumulators are i64*2^32
    uint32_t ntx, nty, ntz;    // P2G tile grid (tiles of p2g_tile^3 cells over base cells -1..g-1)
    uint32_t p2g_tile;         // cells per side of a P2G tile (4 or 8)
    JetPlan jet;               // device emission of this substep (count 0: none)
    uint32_t warm;             // keep last substep's pressure in fluid cells
    float omega;               // red-black over-relaxation (1 = plain Gauss-Seidel)
    uint32_t first_check;      // pairs before a solve's first residual check (0: check_every)
};

// Device pointers of one simulation (or one ensemble member).
struct Ctx {
    Params u;
    // particles: SoA of float4 streams, slots [0,num_bed) bed, then water
    float4* pos;      // x, y, z, J
    float4* vel;      // vx, vy, vz, mass
    float4* c0;       // C col0 xyz, phase
    float4* c1;       // C col1 xyz (rest position for bed), w
    float4* c2;       // C col2 xyz, w
    float4* bedA;     // pore_water, porosity, permeability, compaction
    float4* bedB;     // extractable, dissolved, temperature, saturation
    float4* render;   // 2 x float4 per particle
    float4* snap;     // bed positions before bed_dynamics (Jacobi snapshot)
    int32_t* delta;   // 4 lanes x max_p: water, impulse x/y/z
    // grid
    int32_t* lanes;   // 6 x cells, reference aliasing (shader.rs:152-164)
    // cell kind of each cell: lane 3 of `lanes` in a simulation; the pressure solves
    // read the kind only through this pointer, so they can run on a caller's array
    const int32_t* kind;
    long long* lanes64;  // 6 x cells in int64 mode
    // sorted P2G (CS_P2G_SORTED_SHARED): particles counting-sorted by 4^3-cell tile
    uint32_t* p2g_key;     // max_p: tile of each particle (P2G_NO_TILE if it deposits nothing)
    uint32_t* p2g_rank;    // max_p: position inside its tile
    uint32_t* p2g_sorted;  // max_p: particle ids in tile order
    uint32_t* tile_count;  // tiles + 1
    uint32_t* tile_start;  // tiles + 1 (exclusive scan of tile_count)
    float4* gvel;     // v.xyz, mass
    float* pf;        // FP32 pressure (persistent across substeps for warm start)
    float* divf;      // FP32 divergence
    float* fill;      // liquid fill fraction of each cell (written by classify)
    // face-weight code of each cell (classify): -2 solid, -1 not fluid, 2 bed-coupled,
    // else the liquid fill fraction; the per-colour sweep reads only this per face
    float* fcode;
    // bed-matrix velocity of each cell (mean velocity of the solid bed samples looked up in
    // its 3x3x3 neighbourhood, shader.rs:380-407), computed once per substep for classify
    // and project
    float4* bedv;
    float* plo;       // low word of the pressure (refinement mode: p = pf + plo)
    float* pd;        // pressure correction of the current refinement cycle
    float* gres;      // FP64 residual of the cycle, rounded to fp32
    int32_t* lookup;  // cell -> bed id
    const float* sdf;       // 128^3
    const uint8_t* cls;     // cells, 1 = solid
    uint32_t* metrics;      // 8 counters
    double* resid;          // [0] sum r^2, [1] sum b^2
    ScBuffers sb;           // cluster-resident pressure solve scratch of this instance
    ScTotals* totals;       // running solve totals of replayed substeps (graph mode)
    GsBuffers gs;           // grid-wide pressure solve scratch (large grids)
};

// ---------------- math with WGSL semantics ----------------
struct f3 { float x, y, z; };
__host__ __device__ __forceinline__ f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ f3 operator*(float s, f3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ void operator+=(f3& a, f3 b) { a = a + b; }
__device__ __forceinline__ void operator-=(f3& a, f3 b) { a = a - b; }
__device__ __forceinline__ void operator*=(f3& a, float s) { a = a * s; }
__device__ __forceinline__ float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len3(f3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ float len2(float x, float y) { return sqrtf(x * x + y * y); }
__device__ __forceinline__ float wmin(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ float wmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ float wclamp(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ f3 mix3(f3 a, f3 b, float t) { return {mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t)}; }
__device__ __forceinline__ float smoothstepf(float lo, float hi, float x) {
    float t = wclamp((x - lo) / (hi - lo), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
__device__ __forceinline__ float wfract(float x) { return x - floorf(x); }
__device__ __forceinline__ int32_t to_i32(float x) { return __float2int_rz(x); }  // saturating, NaN -> 0
__device__ __forceinline__ long long to_i64(float x) { return __float2ll_rz(x); }  // saturating, NaN -> 0
__device__ __forceinline__ uint32_t to_u32(float x) { return __float2uint_rz(x); }
__device__ __forceinline__ f3 xyz(float4 v) { return {v.x, v.y, v.z}; }

// exp(x), |x| <= 0.35: Taylor series to x^10 in Horner form (same constants and
// order as the CPU oracle, so both round identically).
__device__ __forceinline__ float exp_small(float x) {
    float p = 2.7557319e-07f;
    p = p * x + 2.7557319e-06f;
    p = p * x + 2.4801587e-05f;
    p = p * x + 1.9841270e-04f;
    p = p * x + 1.3888889e-03f;
    p = p * x + 8.3333333e-03f;
    p = p * x + 4.1666667e-02f;
    p = p * x + 1.6666667e-01f;
    p = p * x + 0.5f;
    p = p * x + 1.0f;
    p = p * x + 1.0f;
    return p;
}

__device__ __forceinline__ bool is_fluid(int32_t k) { return k == CELL_INTERIOR || k == CELL_SURFACE || k == CELL_BED; }
__device__ __forceinline__ bool is_solid(int32_t k) { return k == CELL_SOLID; }
__device__ __forceinline__ bool is_water_phase(float ph) { return ph < 0.5f; }
__device__ __forceinline__ bool is_suspended(float ph) { return ph >= 1.5f; }

__device__ __forceinline__ bool in_grid(const Params& u, int x, int y, int z) {
    return x >= 0 && y >= 0 && z >= 0 && (uint32_t)x < u.gx && (uint32_t)y < u.gy && (uint32_t)z < u.gz;
}
__device__ __forceinline__ uint32_t cidx(const Params& u, uint32_t x, uint32_t y, uint32_t z) {
    return z * u.gx * u.gy + y * u.gx + x;
}
__device__ __forceinline__ void decompose(const Params& u, uint32_t idx, uint32_t& ix, uint32_t& iy, uint32_t& iz) {
    uint32_t plane = u.gx * u.gy;
    iz = idx / plane;
    uint32_t rem = idx - iz * plane;
    iy = rem / u.gx;
    ix = rem - iy * u.gx;
}
__device__ __forceinline__ f3 cell_center(const Params& u, uint32_t ix, uint32_t iy, uint32_t iz) {
    return mk(u.ox + ((float)ix + 0.5f) * u.dx, u.oy + ((float)iy + 0.5f) * u.dx, u.oz + ((float)iz + 0.5f) * u.dx);
}

}  // namespace cs
