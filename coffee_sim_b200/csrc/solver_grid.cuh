// solver_grid.cuh — the pressure solve of one substep in one cooperative launch over
// the whole GPU, for grids whose fluid does not fit a thread-block cluster.
//
// It runs the mixed-precision red-black SOR refinement of k_refine_residual /
// k_refine_sweep / k_refine_accumulate (pressure_update, shader.rs:1371-1453, swept
// to an FP64 residual target) with the same per-cell arithmetic in the same face
// order (-x,+x,-y,+y,-z,+z), so it gives the per-colour launches' pressures bit for
// bit; only the FP64 norm sums are added in another order.  What changes is where
// the work happens and how it is synchronised:
//
// Layout.  Every grid row (fixed y, z) that holds fluid keeps its cells in a row
// segment [xlo, xlo + 64 n) with xlo a multiple of 64, n units of 64 cells.  A
// segment stores its red cells first, then its black cells, so the 32 cells of one
// colour of a unit are 32 consecutive slots: a warp's loads of its own cells and of
// each neighbour row are single 128-byte rows, and a sweep touches only the rows that
// hold fluid (the dense grid of a large pour is mostly air and solid).  Per slot:
// (1/W, flags), (correction, fill code) and the pressure (hi, lo) as float2, the
// residual g and dx^2 rhs.  The flags give, per face, whether it is a fluid face with
// weight > 0 (bits 0-5) or an air face with weight > 0 (bits 8-13), and whether all
// fluid faces have weight 1, so no pass recomputes a cell kind.
//
// Prep (k_gs_rows, a CUB scan, k_gs_desc) finds each row's fluid extent, numbers the
// units and writes for every unit its own row's and its four neighbour rows' first
// slot, colour-half length and first x (a neighbour cell's slot follows from its x).
//
// Solve (k_gs_solve).  One CTA of 1024 threads per SM, launched cooperatively so all
// are resident.  CTA b owns whole rows, about 1/148 of the units.  At set-up it turns
// each unit's descriptor into eight index words per colour, kept in shared memory: the
// slot of the unit's first cell and of that cell's six neighbours (cell `lane` then
// sits at slot + lane), and whether the unit is bulk (all 32 cells fluid with six
// unit-weight fluid faces, updated by a plain six-term sum).  A warp sweeps its units
// two at a time with all nine loads of both in flight (own coefficients, residual and
// correction, six neighbours' correction and fill code in one 8-byte load each).  A
// neighbour in a row of another CTA is read from L2 with ld.cg; one in a row this CTA
// owns goes through L1: CTA ranges start at unit boundaries and the slot arrays at
// 128-byte lines, so no other CTA writes those lines, and within the CTA its barriers
// make its own writes visible.  The colours of a red-black pair are separated by a grid-wide
// barrier (a monotonic arrival counter: a release add per CTA, acquire polling).  The
// last pair of a refinement cycle adds the correction to the pressure as it goes (a
// cell's correction is final after its own colour's sweep), so a residual check is one
// pass and one barrier: each CTA writes its FP64 partial sums, and after the barrier
// every CTA adds all partials in CTA order, so all take the same stop decision.  The
// check schedule is sc_next_interval, the same as the oracle's.  Every barrier wait is
// bounded; a CTA whose wait runs out raises an abort word that ends the other CTAs'
// waits too, and the solve reports status 3 (the host then re-solves with per-colour
// launches).
#pragma once
#include <climits>

#include "kernels.cuh"
#include "solver_types.cuh"

namespace cs {

constexpr int GS_THREADS = 1024;
constexpr int GS_UNIT = 64;                 // cells per unit (32 slots of each colour)
// per-slot flags (16 bits)
constexpr uint32_t GS_FLUID_FACES = 0x3fu;  // bits 0-5: fluid face with weight > 0
constexpr uint32_t GS_UNITW = 1u << 6;      // every fluid face has weight 1
constexpr uint32_t GS_EMPTY = 1u << 7;      // no face with weight > 0, not fluid, or outside the grid
constexpr uint32_t GS_AIR_SHIFT = 8;        // bits 8-13: air face with weight > 0
constexpr uint32_t GS_ISFLUID = 1u << 14;   // fluid cell (its pressure is accumulated)
constexpr long long kGsWaitCycles = 1ll << 31;  // ~1 s at 2 GHz
constexpr int GS_SMEM = 24 * 1024;          // dynamic shared memory of a solve CTA: its units' index words
                                            // (384 units; small, so that the rest of the SM's 256 KB is L1)

// Per unit: x of its first cell, y, z, and for its own row and the four neighbour rows
// (y-1, y+1, z-1, z+1) the row's first slot (INT_MIN: no fluid in it), the slots per
// colour half and the segment's first x.  Cell x of a row holds slot
// base + colour * half + (x - xlo) / 2.  `nonunit` bit c: a cell of colour c has a
// fluid face of weight below 1 (written by the solve's set-up).
struct GsRow {
    int base, half, xlo;
};
struct GsDesc {
    int x0, y, z, nonunit;
    GsRow row[5];
};
static_assert(sizeof(GsDesc) == 76, "unit descriptor layout");

// Grid barrier words: [0] arrivals (monotonic: after the g-th barrier it is g times the
// CTA count), [2] abort.  Thread 0 of each CTA adds its arrival with a release add after
// the CTA barrier and polls with acquire loads, so every write a CTA made before the
// barrier is visible to every CTA after it.
__device__ __forceinline__ uint32_t gs_ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void gs_red_release(uint32_t* p, uint32_t v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Returns false (on every thread of the CTA) once any CTA gave up waiting.  The abort
// word is read on every 16th poll only: each read is another L2 round trip in the loop.
__device__ __forceinline__ bool gs_grid_sync(uint32_t* sync, uint32_t nblocks, uint32_t& gen) {
    __shared__ uint32_t s_ok;
    __syncthreads();
    ++gen;
    if (threadIdx.x == 0) {
        uint32_t ok = 1u, polls = 0;
        gs_red_release(&sync[0], 1u);
        const uint32_t target = nblocks * gen;
        const long long t0 = clock64();
        while ((int)(gs_ld_acquire(&sync[0]) - target) < 0) {
            if ((++polls & 15u) != 0u) continue;
            if (gs_ld_acquire(&sync[2]) != 0u) {
                ok = 0u;
                break;
            }
            if (clock64() - t0 > kGsWaitCycles) {
                atomicExch(&sync[2], 1u);
                ok = 0u;
                break;
            }
        }
        if (ok && gs_ld_acquire(&sync[2]) != 0u) ok = 0u;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0u;
}

// ---------------- prep ----------------
// Fluid extent of every row: one warp per row; units = ceil((x1 - xlo) / 64) with
// xlo = x0 rounded down to a multiple of 64.
__global__ void k_gs_rows(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    const GsBuffers& gb = c.gs;
    const uint32_t rows = u.gy * u.gz;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += warps) {
        const int32_t* kr = c.kind + (size_t)r * u.gx;
        int lo = INT_MAX, hi = -1;
        for (uint32_t x0 = 0; x0 < u.gx; x0 += 32) {
            const uint32_t x = x0 + lane;
            const bool f = x < u.gx && is_fluid(kr[x]);
            const uint32_t m = __ballot_sync(0xffffffffu, f);
            if (m) {
                lo = min(lo, (int)(x0 + __ffs(m) - 1));
                hi = (int)(x0 + 31 - __clz(m));
            }
        }
        if (lane == 0) {
            uint32_t n = 0, xlo = 0;
            if (hi >= 0) {
                xlo = (uint32_t)lo & ~63u;
                n = ((uint32_t)hi + 1u - xlo + 63u) / 64u;
            }
            gb.row_units[r] = n;
            gb.row_xlo[r] = xlo;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) gb.row_units[rows] = 0u;
}

__device__ __forceinline__ GsRow gs_row_info(const GsBuffers& gb, uint32_t q) {
    GsRow r;
    const uint32_t n = gb.row_units[q];
    r.base = n ? (int)(gb.row_start[q] * (uint32_t)GS_UNIT) : INT_MIN;
    r.half = (int)(32u * n);
    r.xlo = (int)gb.row_xlo[q];
    return r;
}

// One descriptor per unit (threads over rows).
__global__ void k_gs_desc(const Ctx* __restrict__ cp) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    const GsBuffers& gb = c.gs;
    const uint32_t rows = u.gy * u.gz;
    CS_FOR(r, rows) {
        const uint32_t n = gb.row_units[r];
        if (n == 0) continue;
        const uint32_t y = r % u.gy, z = r / u.gy;
        GsDesc d;
        d.y = (int)y;
        d.z = (int)z;
        d.nonunit = 0;
        d.row[0] = gs_row_info(gb, r);
        const bool in[4] = {y > 0, y + 1 < u.gy, z > 0, z + 1 < u.gz};
        const uint32_t q[4] = {r - 1u, r + 1u, r - u.gy, r + u.gy};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (in[k]) {
                d.row[k + 1] = gs_row_info(gb, q[k]);
            } else {
                d.row[k + 1].base = INT_MIN;
                d.row[k + 1].half = 0;
                d.row[k + 1].xlo = 0;
            }
        }
        const uint32_t u0 = gb.row_start[r];
        for (uint32_t k = 0; k < n; ++k) {
            d.x0 = (int)(gb.row_xlo[r] + 64u * k);
            gb.desc[u0 + k] = d;
        }
    }
}

// ---------------- solve ----------------
__device__ __forceinline__ float gs_weight(float fc_i, float fc_j) {
    return (fc_i > 1.5f || fc_j > 1.5f) ? 1.0f : fminf(fc_i, fc_j);
}

// Cell x (colour col) of row r sits in slot base + col * half + (x - xlo) / 2.
__device__ __forceinline__ int gs_slot(const GsRow& r, int col, int x) {
    return r.base + col * r.half + ((x - r.xlo) >> 1);
}

// The fields of the simulation context the solve reads, staged once per CTA in
// shared memory so that the loops do not reload them from global memory.
struct GsCtx {
    const int32_t* kind;
    const float* fill;
    const float* divf;
    float* pf;
    float* plo;
    uint32_t* metrics;
    uint32_t gx, gy, gz, first_check;
    float dx, dt, omega, p_limit;
    __device__ __forceinline__ uint32_t cell(uint32_t x, uint32_t y, uint32_t z) const {
        return z * gx * gy + y * gx + x;  // cidx
    }
};

// First unit of CTA b: its share of the units rounded to a whole row, so that every
// CTA owns whole rows and its slots are one contiguous range.
__device__ __forceinline__ uint32_t gs_cta_first_unit(const GsBuffers& gb, uint32_t rows, uint32_t n_units,
                                                      uint32_t b, uint32_t nb) {
    const uint32_t target = (uint32_t)(((unsigned long long)n_units * b) / nb);
    uint32_t lo = 0, hi = rows;  // first row r with row_start[r] >= target
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (gb.row_start[mid] >= target)
            hi = mid;
        else
            lo = mid + 1;
    }
    return gb.row_start[lo];
}

// Set-up of one slot from the dense arrays classify wrote: flags, 1/W, fill code,
// dx^2 rhs and the starting pressure (the face weights of face_weight,
// shader.rs:306-323).  Returns the cell's flags.
__device__ __forceinline__ uint32_t gs_setup_cell(const GsCtx& c, const GsBuffers& gb, const GsDesc& d, int col,
                                                  uint32_t lane) {
    const GsCtx& u = c;
    const int x = d.x0 + 2 * (int)lane + ((col + d.y + d.z) & 1);
    const int s = gs_slot(d.row[0], col, x);
    uint32_t fl = GS_EMPTY;
    float invW = 0.0f, fci = -1.0f, b = 0.0f;
    float2 p = make_float2(0.0f, 0.0f);
    if (x < (int)u.gx) {
        const uint32_t ix = (uint32_t)x, iy = (uint32_t)d.y, iz = (uint32_t)d.z;
        const uint32_t ci = c.cell(ix, iy, iz);
        const int32_t kind = c.kind[ci];
        if (is_fluid(kind)) {
            fl = GS_ISFLUID;
            const float sf = c.fill[ci];
            fci = kind == CELL_BED ? 2.0f : sf;
            const uint32_t sy = u.gx, sz = u.gx * u.gy;
            const bool in[6] = {ix > 0, ix + 1 < u.gx, iy > 0, iy + 1 < u.gy, iz > 0, iz + 1 < u.gz};
            const uint32_t off[6] = {(uint32_t)-1, 1u, (uint32_t)0 - sy, sy, (uint32_t)0 - sz, sz};
            float W = 0.0f;
            bool unit = true;
#pragma unroll
            for (int f = 0; f < 6; ++f) {
                if (!in[f]) continue;
                const uint32_t ni = ci + off[f];
                const int32_t nk = c.kind[ni];
                if (is_solid(nk)) continue;
                const float w = face_weight(kind, sf, nk, c.fill[ni]);
                if (!(w > 0.0f)) continue;
                W += w;
                if (is_fluid(nk)) {
                    fl |= 1u << f;
                    unit = unit && (w == 1.0f);
                } else {
                    fl |= 1u << (GS_AIR_SHIFT + f);
                }
            }
            if (unit) fl |= GS_UNITW;
            if (W > 0.0f) {
                invW = 1.0f / W;
            } else {
                fl |= GS_EMPTY;
            }
            // the refinement solves run in FP32 pressure storage only, where the
            // divergence is divf
            const float rhs = c.divf[ci] * sf / wmax(u.dt, 1e-6f);
            b = u.dx * u.dx * rhs;
            p = make_float2(c.pf[ci], c.plo[ci]);
        }
    }
    gb.cf[s] = make_float2(invW, __uint_as_float(fl));
    gb.dfc[s] = make_float2(0.0f, fci);
    gb.g[s] = 0.0f;
    gb.b[s] = b;
    gb.p[s] = p;
    return fl;
}

// Per unit and colour, 8 words the sweeps read instead of the row descriptors: [0] the
// slot of the unit's first cell of this colour; [1 + f] for face f the slot of the
// neighbour of that first cell (cell `lane` of the unit has its neighbour at that slot
// + lane, because every segment starts at an even x; 0 where the neighbour row holds
// no fluid, and such faces are never fluid faces); [7] bit 8 some cell of this colour
// has a fluid face of weight below 1, bit 9 every cell of this colour is a fluid cell
// whose six faces are fluid faces of weight 1 (the bulk of a pool, whose update is a
// plain six-term sum).
constexpr int GS_REC = 8;
constexpr uint32_t GS_REC_NONUNIT = 1u << 8;
constexpr uint32_t GS_REC_BULK = 1u << 9;
// bits 10-15: the neighbour across face f lies in a row of another CTA (or in no fluid
// row), so it is read from L2 (ld.cg); the other neighbours lie in rows this CTA owns,
// whose cache lines no other CTA writes, and are read through L1
constexpr uint32_t GS_REC_FOREIGN_SHIFT = 10;

// Load of a neighbour slot: through L1 when its row belongs to this CTA, else from L2.
template <class T>
__device__ __forceinline__ T gs_ld_nb(const T* p, bool foreign) {
    return foreign ? __ldcg(p) : *p;
}

__device__ __forceinline__ void gs_make_rec(const GsDesc& d, int col, uint32_t flags, int* rec, uint32_t lane) {
    const int t = (col + d.y + d.z) & 1;
    const int oc = col ^ 1;
    const int k = (d.x0 - d.row[0].xlo) >> 6;
    int v = (int)flags;
    if (lane == 0) v = d.row[0].base + col * d.row[0].half + 32 * k;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        if (lane != (uint32_t)(1 + f)) continue;
        const GsRow r = d.row[f < 2 ? 0 : f - 1];
        const int dx = f == 0 ? -1 : (f == 1 ? 1 : 0);
        v = r.base == INT_MIN ? 0 : r.base + oc * r.half + ((d.x0 + t + dx - r.xlo) >> 1);
    }
    if (lane < (uint32_t)GS_REC) rec[lane] = v;
}

// Slot of the neighbour across face f of cell `lane`.  All six are loaded before the
// flags say which are fluid faces; the correction and pressure arrays are padded by
// gx / 2 + 64 slots on both sides, which covers every slot a non-fluid face can give.
__device__ __forceinline__ int gs_nb(const int* rec, int f, uint32_t lane, int n_slots) {
    (void)n_slots;
    return rec[1 + f] + (int)lane;
}

// FP64 residual of one cell; g <- r, d <- 0.  Adds its (r^2, b^2) contributions.
__device__ __forceinline__ void gs_residual_cell(const GsBuffers& gb, const int* rec, uint32_t lane, int n_slots,
                                                 double& r2, double& b2) {
    const int s = rec[0] + (int)lane;
    const float2 cf = gb.cf[s];
    const uint32_t fl = __float_as_uint(cf.y);
    gb.dfc[s].x = 0.0f;
    if (fl & GS_EMPTY) {
        gb.g[s] = 0.0f;
        return;
    }
    float2 pj[6];
    float fj[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int j = gs_nb(rec, f, lane, n_slots);
        const bool foreign = ((uint32_t)rec[7] >> (GS_REC_FOREIGN_SHIFT + f)) & 1u;
        pj[f] = gs_ld_nb(gb.p + j, foreign);
        fj[f] = gs_ld_nb(&gb.dfc[j].y, foreign);
    }
    const float fci = gb.dfc[s].y;
    const float sfi = fci > 1.5f ? 1.0f : fci;
    const bool unit = (fl & GS_UNITW) != 0u;
    double wsum = 0.0, psum = 0.0;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        if (fl & (1u << f)) {
            const float w = unit ? 1.0f : gs_weight(fci, fj[f]);
            wsum += (double)w;
            psum += (double)w * ((double)pj[f].x + (double)pj[f].y);
        } else if (fl & (1u << (GS_AIR_SHIFT + f))) {
            wsum += (double)sfi;
        }
    }
    const float2 pi = gb.p[s];
    const double bb = (double)gb.b[s];
    const double r = (psum - bb) - wsum * ((double)pi.x + (double)pi.y);
    gb.g[s] = (float)r;
    r2 += r * r;
    b2 += bb * bb;
}

// One colour of one unit: the loaded inputs of a cell, then its update.
struct GsLoad {
    float2 cf, me;
    float g;
    float2 nb[6];
    int s;
    uint32_t rf;  // the unit's flag word
};

__device__ __forceinline__ void gs_load(const GsBuffers& gb, const int* rec, uint32_t lane, int n_slots,
                                        GsLoad& L) {
    L.s = rec[0] + (int)lane;
    L.rf = (uint32_t)rec[7];
    L.cf = gb.cf[L.s];
    L.g = gb.g[L.s];
    L.me = gb.dfc[L.s];
#pragma unroll
    for (int f = 0; f < 6; ++f)
        L.nb[f] = gs_ld_nb(gb.dfc + gs_nb(rec, f, lane, n_slots), ((L.rf >> (GS_REC_FOREIGN_SHIFT + f)) & 1u) != 0u);
}

// p <- p + d in FP64 (split back into hi/lo, clamped at the pressure limit).
__device__ __forceinline__ void gs_accumulate(const GsCtx& c, const GsBuffers& gb, int s, float dn) {
    const float2 pi = gb.p[s];
    double p = ((double)pi.x + (double)pi.y) + (double)dn;
    const double lim = (double)c.p_limit;
    if (p > lim || p < -lim) {
        p = p > 0.0 ? lim : -lim;
        atomicAdd(&c.metrics[M_P_CLAMP], 1u);
    }
    const float hi = (float)p;
    gb.p[s] = make_float2(hi, (float)(p - (double)hi));
}

__device__ __forceinline__ void gs_update(const GsCtx& c, const GsBuffers& gb, const GsLoad& L, float omega,
                                          bool last) {
    const float me = L.me.x;
    float ds = 0.0f;
    if (L.rf & GS_REC_BULK) {
        // six fluid faces of weight 1 on every lane: the same sum in face order
#pragma unroll
        for (int f = 0; f < 6; ++f) ds += L.nb[f].x;
    } else {
        const uint32_t fl = __float_as_uint(L.cf.y);
        if (fl & GS_EMPTY) {
            if (last && (fl & GS_ISFLUID)) gs_accumulate(c, gb, L.s, me);
            return;
        }
        if (fl & GS_UNITW) {
#pragma unroll
            for (int f = 0; f < 6; ++f)
                if (fl & (1u << f)) ds += L.nb[f].x;
        } else {
            const float fi = L.me.y;
#pragma unroll
            for (int f = 0; f < 6; ++f)
                if (fl & (1u << f)) ds += gs_weight(fi, L.nb[f].y) * L.nb[f].x;
        }
    }
    float dn = (ds + L.g) * L.cf.x;
    if (omega != 1.0f) dn = me + omega * (dn - me);
    gb.dfc[L.s].x = dn;
    if (last) gs_accumulate(c, gb, L.s, dn);
}

__global__ void __launch_bounds__(GS_THREADS, 1)
    k_gs_solve(const Ctx* __restrict__ cp, float tol, uint32_t max_pairs, uint32_t check_every) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ GsBuffers s_gb;
    __shared__ GsCtx s_c;
    if (threadIdx.x == 0) {
        const Ctx& cg = cp[0];
        s_gb = cg.gs;
        s_c.kind = cg.kind;
        s_c.fill = cg.fill;
        s_c.divf = cg.divf;
        s_c.pf = cg.pf;
        s_c.plo = cg.plo;
        s_c.metrics = cg.metrics;
        s_c.gx = cg.u.gx;
        s_c.gy = cg.u.gy;
        s_c.gz = cg.u.gz;
        s_c.first_check = cg.u.first_check;
        s_c.dx = cg.u.dx;
        s_c.dt = cg.u.dt;
        s_c.omega = cg.u.omega;
        s_c.p_limit = cg.u.p_limit;
    }
    __syncthreads();
    const GsBuffers& gb = s_gb;
    const GsCtx& c = s_c;
    __shared__ double s_red[2][32];
    __shared__ double s_norm;
    uint32_t* sync = gb.sync;
    const uint32_t nb = gridDim.x;
    uint32_t gen = 0;
    const uint32_t rows = c.gy * c.gz;
    const uint32_t n_units = gb.row_start[rows];
    const int n_slots = n_units ? (int)(n_units * (uint32_t)GS_UNIT) : 1;
    const uint32_t ua = gs_cta_first_unit(gb, rows, n_units, blockIdx.x, nb);
    const uint32_t ue = gs_cta_first_unit(gb, rows, n_units, blockIdx.x + 1, nb);
    const uint32_t nu = ue - ua;
    const bool cached = (size_t)nu * 2 * GS_REC * sizeof(int) <= (size_t)GS_SMEM;
    int* const recb = cached ? reinterpret_cast<int*>(smem) : gb.rec + (size_t)ua * 2 * GS_REC;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;

    // set-up of every slot of this CTA's units, and their index words
    for (uint32_t k = warp; k < nu; k += nwarps) {
        const GsDesc d = gb.desc[ua + k];
        const uint32_t f0 = gs_setup_cell(c, gb, d, 0, lane);
        const uint32_t f1 = gs_setup_cell(c, gb, d, 1, lane);
        auto nonunit = [](uint32_t fl) { return (fl & (GS_ISFLUID | GS_EMPTY | GS_UNITW)) == GS_ISFLUID; };
        auto bulk = [](uint32_t fl) {
            return (fl & (GS_ISFLUID | GS_EMPTY | GS_UNITW | GS_FLUID_FACES)) == (GS_ISFLUID | GS_UNITW | GS_FLUID_FACES);
        };
        const uint32_t n0 = __ballot_sync(0xffffffffu, nonunit(f0)), n1 = __ballot_sync(0xffffffffu, nonunit(f1));
        const uint32_t b0 = __ballot_sync(0xffffffffu, bulk(f0)), b1 = __ballot_sync(0xffffffffu, bulk(f1));
        int* r = recb + (size_t)k * 2 * GS_REC;
        // faces whose neighbour row is another CTA's (x faces: the unit's own row)
        uint32_t foreign = 0;
#pragma unroll
        for (int f = 2; f < 6; ++f) {
            const int base = d.row[f - 1].base;
            const bool own = base != INT_MIN && (uint32_t)base / (uint32_t)GS_UNIT >= ua &&
                             (uint32_t)base / (uint32_t)GS_UNIT < ue;
            if (!own) foreign |= 1u << f;
        }
        foreign <<= GS_REC_FOREIGN_SHIFT;
        gs_make_rec(d, 0, foreign | (n0 ? GS_REC_NONUNIT : 0u) | (b0 == 0xffffffffu ? GS_REC_BULK : 0u), r, lane);
        gs_make_rec(d, 1, foreign | (n1 ? GS_REC_NONUNIT : 0u) | (b1 == 0xffffffffu ? GS_REC_BULK : 0u), r + GS_REC, lane);
    }
    bool ok = gs_grid_sync(sync, nb, gen);

    // FP64 residual and the relative norm every CTA agrees on
    auto residual = [&]() -> double {
        double r2 = 0.0, b2 = 0.0;
        for (uint32_t k = warp; k < nu; k += nwarps) {
            const int* r = recb + (size_t)k * 2 * GS_REC;
            gs_residual_cell(gb, r, lane, n_slots, r2, b2);
            gs_residual_cell(gb, r + GS_REC, lane, n_slots, r2, b2);
        }
        for (int o = 16; o > 0; o >>= 1) {
            r2 += __shfl_down_sync(0xffffffffu, r2, o);
            b2 += __shfl_down_sync(0xffffffffu, b2, o);
        }
        if (lane == 0) {
            s_red[0][warp] = r2;
            s_red[1][warp] = b2;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = 0.0, bs = 0.0;
            for (uint32_t w = 0; w < nwarps; ++w) {
                a += s_red[0][w];
                bs += s_red[1][w];
            }
            gb.part[2 * blockIdx.x] = a;
            gb.part[2 * blockIdx.x + 1] = bs;
        }
        ok = ok && gs_grid_sync(sync, nb, gen);
        if (threadIdx.x == 0) {
            double a = 0.0, bs = 0.0;
            for (uint32_t q = 0; q < nb; ++q) {
                a += __ldcg(gb.part + 2 * q);
                bs += __ldcg(gb.part + 2 * q + 1);
            }
            s_norm = bs <= 0.0 ? 0.0 : sqrt(a) / sqrt(bs);
        }
        __syncthreads();
        return s_norm;
    };

    const float omega = c.omega;
    // one colour over this CTA's units, two units per step with all loads in flight
    auto sweep = [&](int col, bool last) {
        uint32_t k = warp;
        for (; k + nwarps < nu; k += 2 * nwarps) {
            GsLoad a, b;
            gs_load(gb, recb + ((size_t)k * 2 + col) * GS_REC, lane, n_slots, a);
            gs_load(gb, recb + ((size_t)(k + nwarps) * 2 + col) * GS_REC, lane, n_slots, b);
            gs_update(c, gb, a, omega, last);
            gs_update(c, gb, b, omega, last);
        }
        if (k < nu) {
            GsLoad a;
            gs_load(gb, recb + ((size_t)k * 2 + col) * GS_REC, lane, n_slots, a);
            gs_update(c, gb, a, omega, last);
        }
    };

    double r0 = -1.0, r1 = -1.0;
    uint32_t pairs = 0, evals = 0;
    if (ok) {
        r0 = residual();
        r1 = r0;
        evals = 1;
    }
    const uint32_t ce = check_every ? check_every : 10u;
    uint32_t next = c.first_check ? c.first_check : ce;
    while (ok && !(r1 <= (double)tol) && pairs < max_pairs) {
        const uint32_t k = min(next, max_pairs - pairs);
        for (uint32_t j = 0; j < k && ok; ++j) {
            const bool last = j + 1 == k;
            sweep(0, last);
            ok = gs_grid_sync(sync, nb, gen);
            if (!ok) break;
            sweep(1, last);
            ok = gs_grid_sync(sync, nb, gen);
        }
        if (!ok) break;
        pairs += k;
        const double r_before = r1;
        r1 = residual();
        ++evals;
        next = sc_next_interval(r1, r_before, k, (double)tol, ce);
    }
    // the solved pressure back to the dense arrays
    for (uint32_t k = warp; k < nu; k += nwarps) {
        const GsDesc d = gb.desc[ua + k];
#pragma unroll
        for (int col = 0; col < 2; ++col) {
            const int x = d.x0 + 2 * (int)lane + ((col + d.y + d.z) & 1);
            if (x >= (int)c.gx) continue;
            const int s = gs_slot(d.row[0], col, x);
            if (!(__float_as_uint(gb.cf[s].y) & GS_ISFLUID)) continue;
            const uint32_t ci = c.cell((uint32_t)x, (uint32_t)d.y, (uint32_t)d.z);
            const float2 p = gb.p[s];
            c.pf[ci] = p.x;
            c.plo[ci] = p.y;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        gb.result->sweeps = pairs;
        gb.result->evals = evals;
        gb.result->r0 = r0;
        gb.result->r1 = r1;
        gb.result->status = ok ? 1u : 3u;
        if (!ok) atomicOr(&c.metrics[M_TIMEOUT], 1u);
    }
}

}  // namespace cs
