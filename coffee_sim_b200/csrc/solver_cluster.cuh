// solver_cluster.cuh — the pressure solve of one substep in a single launch: a
// thread-block cluster keeps every fluid cell's solver state in shared memory and
// runs the mixed-precision red-black SOR refinement of k_refine_* without leaving
// the chip.
//
// Layout.  Fluid cells are numbered by an exclusive scan in Morton order and cut into
// R contiguous chunks (R = cluster size, chunk <= SC_CAP cells); inside a chunk the
// red cells (ix+iy+iz even) come first.  Every cell carries, in the shared memory of
// the CTA that owns it: the correction d and its fill code (float2; fill code 2.0
// marks a bed-coupled cell), the residual g, the fp32 face-weight sum W, the pressure
// hi/lo words, dx^2*rhs, six 16-bit neighbour references (rank << 12 | local index,
// 0xFFFF = no fluid neighbour) and the number of air faces.  Neighbours owned by
// another CTA are read through distributed shared memory.
//
// Arithmetic is that of k_refine_residual / k_refine_sweep / k_refine_accumulate,
// operation for operation (face order -x,+x,-y,+y,-z,+z; weights of fluid faces
// recomputed from fill codes; the FP64 weight sum is exact because it adds at most
// six floats in (0,1]), so the result equals the per-colour-launch solve bit for bit
// except for the order of the FP64 norm reductions.
#pragma once
#include <cooperative_groups.h>

#include "kernels.cuh"

#include "solver_types.cuh"

namespace cs {
namespace cg = cooperative_groups;

// Distributed shared memory through 32-bit cluster addresses.  The loads are volatile
// so they stay between the cluster barriers that order them.
__device__ __forceinline__ uint32_t sc_mapa(uint32_t addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}
__device__ __forceinline__ float2 sc_ld2(uint32_t addr) {
    float2 v;
    asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr) : "memory");
    return v;
}
__device__ __forceinline__ float sc_ld(uint32_t addr) {
    float v;
    asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(addr) : "memory");
    return v;
}

// Cells are numbered along a Morton (Z-order) curve over the grid padded to a power
// of two per side, so each CTA's contiguous chunk is a compact 3-D block and few of
// its neighbours live in other CTAs.
__device__ __forceinline__ uint32_t sc_compact3(uint32_t m) {
    m &= 0x09249249u;
    m = (m ^ (m >> 2)) & 0x030C30C3u;
    m = (m ^ (m >> 4)) & 0x0300F00Fu;
    m = (m ^ (m >> 8)) & 0xFF0000FFu;
    m = (m ^ (m >> 16)) & 0x000003FFu;
    return m;
}
__device__ __forceinline__ bool sc_cell_of_code(const Params& u, uint32_t m, uint32_t& ci, uint32_t& parity) {
    uint32_t x = sc_compact3(m), y = sc_compact3(m >> 1), z = sc_compact3(m >> 2);
    if (x >= u.gx || y >= u.gy || z >= u.gz) return false;
    ci = cidx(u, x, y, z);
    parity = (x + y + z) & 1u;
    return true;
}

__global__ void k_sc_flags(const Ctx* __restrict__ cp, ScBuffers sb, uint32_t codes) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    const int32_t* kl = c.lanes + 3 * (size_t)u.cells;
    CS_FOR(m, codes) {
        unsigned long long f = 0;
        uint32_t ci, par;
        if (sc_cell_of_code(u, m, ci, par) && is_fluid(kl[ci])) f = 1ull | (par == 0u ? (1ull << 32) : 0ull);
        sb.flags[m] = f;
    }
}

// Totals and chunking (one thread), then the red count before each chunk's first cell.
__global__ void k_sc_totals(const Ctx* __restrict__ cp, ScBuffers sb, uint32_t ranks, uint32_t codes) {
    unsigned long long last = sb.scan[codes - 1] + sb.flags[codes - 1];
    uint32_t nf = (uint32_t)(last & 0xffffffffull), nr = (uint32_t)(last >> 32);
    uint32_t chunk = (nf + ranks - 1) / ranks;
    sb.info->n_fluid = nf;
    sb.info->n_red = nr;
    sb.info->chunk = chunk;
    sb.info->overflow = chunk > (uint32_t)SC_CAP ? 1u : 0u;
    for (uint32_t r = 0; r <= SC_MAX_RANKS; ++r) sb.info->red_before[r] = nr;
}

__global__ void k_sc_starts(const Ctx* __restrict__ cp, ScBuffers sb, uint32_t codes) {
    const uint32_t chunk = sb.info->chunk;
    if (chunk == 0) return;
    CS_FOR(m, codes) {
        if (!(sb.flags[m] & 1ull)) continue;
        uint32_t fid = (uint32_t)(sb.scan[m] & 0xffffffffull);
        if (fid % chunk == 0) sb.info->red_before[fid / chunk] = (uint32_t)(sb.scan[m] >> 32);
    }
}

__global__ void k_sc_map(const Ctx* __restrict__ cp, ScBuffers sb, uint32_t codes) {
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    const ScInfo& inf = *sb.info;
    const uint32_t chunk = inf.chunk;
    CS_FOR(m, codes) {
        uint32_t ci, par;
        if (!sc_cell_of_code(u, m, ci, par)) continue;
        unsigned long long f = sb.flags[m];
        if (!(f & 1ull) || chunk == 0 || inf.overflow) {
            sb.ref_of_cell[ci] = SC_NONE;
            continue;
        }
        uint32_t fid = (uint32_t)(sb.scan[m] & 0xffffffffull);
        uint32_t rid = (uint32_t)(sb.scan[m] >> 32);
        uint32_t rank = fid / chunk, start = rank * chunk;
        uint32_t rb = inf.red_before[rank];
        uint32_t nred = inf.red_before[rank + 1] - rb;
        uint32_t red_in = rid - rb;
        uint32_t local = (f >> 32) ? red_in : nred + (fid - start) - red_in;
        sb.ref_of_cell[ci] = (uint16_t)((rank << 12) | local);
        sb.cell_of[rank * 4096u + local] = ci;
    }
}

template <class T>
__device__ __forceinline__ T* sc_arr(unsigned char* base, size_t off) {
    return reinterpret_cast<T*>(base + off);
}

__device__ __forceinline__ float sc_weight(float fc_i, float fc_j) {
    // face_weight for two fluid cells: 1 when either is bed-coupled, else the smaller fill
    return (fc_i > 1.5f || fc_j > 1.5f) ? 1.0f : fminf(fc_i, fc_j);
}

// One cluster per instance (blockIdx.y); R = cluster size along x.
__global__ void __launch_bounds__(SC_THREADS, 1)
    k_sc_solve(const Ctx* __restrict__ cp, ScBuffers sb, float tol, uint32_t max_pairs, uint32_t check_every) {
    extern __shared__ __align__(16) unsigned char smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    const uint32_t R = cluster.num_blocks();
    const uint32_t rank = cluster.block_rank();
    const ScInfo& inf = *sb.info;
    if (inf.overflow) {
        if (rank == 0 && threadIdx.x == 0) sb.result->status = 2;
        return;  // uniform across the cluster: every rank reads the same flag
    }
    const uint32_t chunk = inf.chunk;
    const uint32_t start = rank * chunk;
    const uint32_t n_loc = (chunk == 0 || start >= inf.n_fluid) ? 0u : min(chunk, inf.n_fluid - start);
    const uint32_t n_red = inf.red_before[rank + 1] - inf.red_before[rank];

    float2* dfill = sc_arr<float2>(smem, ScLayout::dfill);
    float* gg = sc_arr<float>(smem, ScLayout::g);
    float* invW = sc_arr<float>(smem, ScLayout::invW);
    float* ph = sc_arr<float>(smem, ScLayout::ph);
    float* pl = sc_arr<float>(smem, ScLayout::pl);
    float* bb = sc_arr<float>(smem, ScLayout::b);
    uint16_t* ref = sc_arr<uint16_t>(smem, ScLayout::ref);
    uint8_t* flg = sc_arr<uint8_t>(smem, ScLayout::flags);
    double* part = sc_arr<double>(smem, ScLayout::part);
    double* red = sc_arr<double>(smem, ScLayout::red);
    const uint32_t a_dfill = (uint32_t)__cvta_generic_to_shared(dfill);
    const uint32_t a_ph = (uint32_t)__cvta_generic_to_shared(ph);
    const uint32_t a_pl = (uint32_t)__cvta_generic_to_shared(pl);

    const int32_t* kl = c.lanes + 3 * (size_t)u.cells;
    const uint32_t sy = u.gx, sz = u.gx * u.gy;

    // ---- set-up: coefficients of the cells this CTA owns ----
    for (uint32_t i = threadIdx.x; i < n_loc; i += blockDim.x) {
        uint32_t ci = sb.cell_of[rank * 4096u + i];
        uint32_t ix, iy, iz;
        decompose(u, ci, ix, iy, iz);
        int32_t kind = kl[ci];
        float sf = c.fill[ci];
        float fci = kind == CELL_BED ? 2.0f : sf;
        float W = 0.0f;
        uint32_t na = 0;
        bool unit = true;
        bool in[6] = {ix > 0, ix + 1 < u.gx, iy > 0, iy + 1 < u.gy, iz > 0, iz + 1 < u.gz};
        uint32_t off[6] = {(uint32_t)-1, 1u, (uint32_t)0 - sy, sy, (uint32_t)0 - sz, sz};
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            uint16_t r = SC_NONE;
            if (in[f]) {
                uint32_t ni = ci + off[f];
                int32_t nk = kl[ni];
                if (!is_solid(nk)) {
                    float w = face_weight(kind, sf, nk, c.fill[ni]);
                    if (w > 0.0f) {
                        W += w;
                        if (is_fluid(nk)) {
                            r = sb.ref_of_cell[ni];
                            unit = unit && (w == 1.0f);
                        } else {
                            ++na;
                        }
                    }
                }
            }
            ref[i * 6 + f] = r;
        }
        invW[i] = W > 0.0f ? 1.0f / W : 0.0f;
        flg[i] = (uint8_t)(na | (unit ? SC_UNIT : 0) | (W > 0.0f ? 0 : SC_EMPTY));
        dfill[i] = make_float2(0.0f, fci);
        ph[i] = c.pf[ci];
        pl[i] = c.plo[ci];
        float rhs = div_load(c, ci) * sf / wmax(u.dt, 1e-6f);
        bb[i] = u.dx * u.dx * rhs;
    }
    cluster.sync();

    // FP64 residual of the current pressure; g <- residual, d <- 0.  Returns the
    // relative norm, identical in every rank (partials summed in rank order).
    auto residual = [&](int slot) -> double {
        double r2 = 0.0, b2 = 0.0;
        for (uint32_t i = threadIdx.x; i < n_loc; i += blockDim.x) {
            dfill[i].x = 0.0f;
            uint8_t fl = flg[i];
            if (fl & SC_EMPTY) {
                gg[i] = 0.0f;
                continue;
            }
            float fci = dfill[i].y;
            float sfi = fci > 1.5f ? 1.0f : fci;
            double wsum = (double)(fl & 7u) * (double)sfi;
            double psum = 0.0;
            const uint32_t* rp = reinterpret_cast<const uint32_t*>(ref + i * 6);
            uint32_t rw[3] = {rp[0], rp[1], rp[2]};
#pragma unroll
            for (int f = 0; f < 6; ++f) {
                uint32_t r = (rw[f >> 1] >> ((f & 1) * 16)) & 0xffffu;
                if (r == SC_NONE) continue;
                uint32_t rr = r >> 12, j = r & 4095u;
                float fcj = sc_ld2(sc_mapa(a_dfill + j * 8u, rr)).y;
                float w = sc_weight(fci, fcj);
                double pj = (double)sc_ld(sc_mapa(a_ph + j * 4u, rr)) + (double)sc_ld(sc_mapa(a_pl + j * 4u, rr));
                wsum += (double)w;
                psum += (double)w * pj;
            }
            double b = (double)bb[i];
            double r = (psum - b) - wsum * ((double)ph[i] + (double)pl[i]);
            gg[i] = (float)r;
            r2 += r * r;
            b2 += b * b;
        }
        for (int o = 16; o > 0; o >>= 1) {
            r2 += __shfl_down_sync(0xffffffffu, r2, o);
            b2 += __shfl_down_sync(0xffffffffu, b2, o);
        }
        int lane_id = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (lane_id == 0) {
            red[warp] = r2;
            red[32 + warp] = b2;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = 0.0, bsum = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
                a += red[w];
                bsum += red[32 + w];
            }
            double* dst = cluster.map_shared_rank(part, 0);
            dst[slot * 2 * SC_MAX_RANKS + rank] = a;
            dst[slot * 2 * SC_MAX_RANKS + SC_MAX_RANKS + rank] = bsum;
        }
        cluster.sync();
        const double* src = cluster.map_shared_rank(part, 0);
        double a = 0.0, bsum = 0.0;
        for (uint32_t q = 0; q < R; ++q) {
            a += src[slot * 2 * SC_MAX_RANKS + q];
            bsum += src[slot * 2 * SC_MAX_RANKS + SC_MAX_RANKS + q];
        }
        if (bsum <= 0.0) return 0.0;
        return sqrt(a) / sqrt(bsum);
    };

    const float omega = u.omega;
    // Neighbour corrections of cell i, fetched before any arithmetic so a thread's
    // loads for its two cells are in flight together.
    struct Face6 {
        float2 v[6];
        uint32_t mask;
    };
    auto gather = [&](uint32_t i, Face6& fc) {
        const uint32_t* rp = reinterpret_cast<const uint32_t*>(ref + i * 6);
        uint32_t rw[3] = {rp[0], rp[1], rp[2]};
        fc.mask = 0;
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            uint32_t r = (rw[f >> 1] >> ((f & 1) * 16)) & 0xffffu;
            if (r != SC_NONE) {
                fc.v[f] = sc_ld2(sc_mapa(a_dfill + (r & 4095u) * 8u, r >> 12));
                fc.mask |= 1u << f;
            } else {
                fc.v[f] = make_float2(0.0f, 0.0f);
            }
        }
    };
    auto relax = [&](uint32_t i, const Face6& fc) {
        uint8_t fl = flg[i];
        if (fl & SC_EMPTY) return;
        float2 me = dfill[i];
        float ds = 0.0f;
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            if (!(fc.mask & (1u << f))) continue;
            ds += (fl & SC_UNIT) ? fc.v[f].x : sc_weight(me.y, fc.v[f].y) * fc.v[f].x;
        }
        float dn = (ds + gg[i]) * invW[i];
        if (omega != 1.0f) dn = me.x + omega * (dn - me.x);
        dfill[i].x = dn;
    };
    auto sweep = [&](uint32_t lo, uint32_t hi) {
        const uint32_t step = 2 * blockDim.x;
        for (uint32_t i0 = lo + threadIdx.x; i0 < hi; i0 += step) {
            const uint32_t i1 = i0 + blockDim.x;
            Face6 a, b;
            gather(i0, a);
            if (i1 < hi) gather(i1, b);
            relax(i0, a);
            if (i1 < hi) relax(i1, b);
        }
    };

    auto accumulate = [&]() {
        const double lim = (double)u.p_clamp;
        for (uint32_t i = threadIdx.x; i < n_loc; i += blockDim.x) {
            double p = ((double)ph[i] + (double)pl[i]) + (double)dfill[i].x;
            if (p > lim || p < -lim) {
                p = p > 0.0 ? lim : -lim;
                atomicAdd(&c.metrics[M_P_CLAMP], 1u);
            }
            float hi = (float)p;
            ph[i] = hi;
            pl[i] = (float)(p - (double)hi);
        }
    };

    const uint32_t ce = check_every ? check_every : 10u;
    int slot = 0;
    double r0 = residual(slot);
    double r1 = r0;
    uint32_t pairs = 0, evals = 1;
    while (!(r1 <= (double)tol) && pairs < max_pairs) {
        uint32_t k = min(ce, max_pairs - pairs);
        for (uint32_t j = 0; j < k; ++j) {
            cluster.sync();
            sweep(0, n_red);
            cluster.sync();
            sweep(n_red, n_loc);
        }
        pairs += k;
        // the black sweep and accumulate map cells to threads differently
        __syncthreads();
        accumulate();
        cluster.sync();
        slot ^= 1;
        r1 = residual(slot);
        ++evals;
    }
    // write the pressure back (non-fluid cells were zeroed by classify)
    for (uint32_t i = threadIdx.x; i < n_loc; i += blockDim.x) {
        uint32_t ci = sb.cell_of[rank * 4096u + i];
        c.pf[ci] = ph[i];
        c.plo[ci] = pl[i];
    }
    if (rank == 0 && threadIdx.x == 0) {
        sb.result->sweeps = pairs;
        sb.result->evals = evals;
        sb.result->status = 1;
        sb.result->r0 = r0;
        sb.result->r1 = r1;
    }
    cluster.sync();  // keep every CTA's shared memory alive until remote reads end
}

}  // namespace cs
