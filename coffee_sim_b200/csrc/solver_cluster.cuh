// solver_cluster.cuh — the pressure solve of one substep in a single launch: a
// thread-block cluster keeps every fluid cell's solver state in shared memory and
// runs the mixed-precision red-black SOR refinement of k_refine_* without leaving
// the chip.
//
// Layout.  Fluid cells are numbered by an exclusive scan in Morton order and cut into
// R contiguous chunks (R = cluster size, chunk <= SC_CAP cells); inside a chunk the
// red cells (ix+iy+iz even) come first.  Each CTA keeps, for the cells it owns: the
// correction d and the fill code (fill code 2.0 marks a bed-coupled cell), the
// residual g, 1/W, the pressure hi/lo words, dx^2*rhs, the flags byte and the six
// neighbour slots (13-bit slot indices packed two per word).  A neighbour owned by
// another CTA is read from a halo slot of the same correction array; after sweeping a
// colour, each CTA pushes the new values of its cells that other CTAs hold as halo
// with posted DSMEM stores, and the cluster barrier that separates the colours
// publishes them.  A face without a fluid
// neighbour points at a slot that always holds zero, so the sweep has no per-face
// branches and every load in it is a local shared-memory load.
//
// The prep kernels (k_sc_flags .. k_sc_halo) run on the whole GPU: Morton scan and
// chunking, neighbour slots, halo and send lists, and the per-cell coefficients.
//
// Arithmetic is that of k_refine_residual / k_refine_sweep / k_refine_accumulate,
// operation for operation (face order -x,+x,-y,+y,-z,+z; weights of fluid faces
// recomputed from fill codes; a missing face adds an exact zero; the FP64 weight sum
// is exact because it adds at most six floats in (0,1]), so the result equals the
// per-colour-launch solve except for the order of the FP64 norm reductions.
#pragma once
#include <cooperative_groups.h>

#include "kernels.cuh"

#include "solver_types.cuh"

namespace cs {
namespace cg = cooperative_groups;

// Distributed shared memory through 32-bit cluster addresses.  The accesses are
// volatile so they stay between the cluster barriers that order them.
__device__ __forceinline__ uint32_t sc_mapa(uint32_t addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}
__device__ __forceinline__ void sc_st(uint32_t addr, float v) {
    asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(addr), "f"(v) : "memory");
}

// Point-to-point halo exchange.  The value goes out as an asynchronous remote store
// whose completion counts 4 bytes on an mbarrier of the receiving CTA; the receiver
// arms that mbarrier with the byte count it expects for the colour and waits for the
// phase to complete.  A store may land before the receiver arms the phase (the
// transaction count goes negative until the expect-tx arrives).
__device__ __forceinline__ void sc_st_async(uint32_t addr, float v, uint32_t mbar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b32 [%0], %1, [%2];" ::"r"(addr),
                 "r"(__float_as_uint(v)), "r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void sc_mbar_init(uint32_t a) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
}
__device__ __forceinline__ void sc_mbar_expect(uint32_t a, uint32_t bytes) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(a),
        "r"(bytes)
        : "memory");
}
// Waits for the phase of parity `parity`; gives up (false) once `cycles` SM clock
// cycles have passed since the first poll.
__device__ __forceinline__ bool sc_mbar_wait(uint32_t a, uint32_t parity, long long cycles) {
    const long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > cycles) return false;
    }
}
constexpr long long kScWaitCycles = 1ll << 30;  // ~0.5 s at 2 GHz

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

__global__ void k_sc_flags(const Ctx* __restrict__ cp, uint32_t codes) {
    const ScBuffers& sb = cp[blockIdx.y].sb;
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    const int32_t* kl = c.kind;
    CS_FOR(m, codes) {
        unsigned long long f = 0;
        uint32_t ci, par;
        if (sc_cell_of_code(u, m, ci, par) && is_fluid(kl[ci])) f = 1ull | (par == 0u ? (1ull << 32) : 0ull);
        sb.flags[m] = f;
    }
}

// Totals and chunking (one thread), then the red count before each chunk's first cell.
__global__ void k_sc_totals(const Ctx* __restrict__ cp, uint32_t ranks, uint32_t codes) {
    const ScBuffers& sb = cp[blockIdx.y].sb;
    unsigned long long last = sb.scan[codes - 1] + sb.flags[codes - 1];
    uint32_t nf = (uint32_t)(last & 0xffffffffull), nr = (uint32_t)(last >> 32);
    uint32_t chunk = (nf + ranks - 1) / ranks;
    sb.info->n_fluid = nf;
    sb.info->n_red = nr;
    sb.info->chunk = chunk;
    sb.info->overflow = chunk > (uint32_t)SC_CAP ? 1u : 0u;
    for (uint32_t r = 0; r <= SC_MAX_RANKS; ++r) sb.info->red_before[r] = nr;
    for (int k = 0; k < SC_COUNTS; ++k) sb.counts[k] = 0u;
}

__global__ void k_sc_starts(const Ctx* __restrict__ cp, uint32_t codes) {
    const ScBuffers& sb = cp[blockIdx.y].sb;
    const uint32_t chunk = sb.info->chunk;
    if (chunk == 0) return;
    CS_FOR(m, codes) {
        if (!(sb.flags[m] & 1ull)) continue;
        uint32_t fid = (uint32_t)(sb.scan[m] & 0xffffffffull);
        if (fid % chunk == 0) sb.info->red_before[fid / chunk] = (uint32_t)(sb.scan[m] >> 32);
    }
}

__global__ void k_sc_map(const Ctx* __restrict__ cp, uint32_t codes) {
    const ScBuffers& sb = cp[blockIdx.y].sb;
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

// Neighbour slots, halo and send lists, and coefficients of every fluid cell.  A face
// toward a cell of the same CTA gets that cell's local slot, a face without a fluid
// neighbour gets SC_DUMMY, and a face toward another CTA's cell gets the halo slot the
// neighbour allocated for it: each cell takes one halo slot in every other CTA that
// owns one of its neighbours, writes that slot into those neighbours' face entries
// (face f of this cell is face f^1 of the neighbour) and adds itself to its own CTA's
// send list for its colour.  Validity of a fluid face is symmetric (face_weight of
// two fluid cells is 1 or min of the fills), so both sides agree on which faces exist.
// Halo slot order comes from atomics and differs between runs; it only places copies.
__global__ void k_sc_halo(const Ctx* __restrict__ cp) {
    const ScBuffers& sb = cp[blockIdx.y].sb;
    const Ctx& c = cp[blockIdx.y];
    const Params& u = c.u;
    const ScInfo& inf = *sb.info;
    if (inf.overflow || inf.chunk == 0) return;
    const int32_t* kl = c.kind;
    const uint32_t sy = u.gx, sz = u.gx * u.gy;
    CS_FOR(ci, u.cells) {
        const uint16_t rc = sb.ref_of_cell[ci];
        if (rc == SC_NONE) continue;
        const uint32_t r = rc >> 12, i = rc & 4095u;
        uint32_t ix, iy, iz;
        decompose(u, ci, ix, iy, iz);
        const uint32_t par = (ix + iy + iz) & 1u;
        const int32_t kind = kl[ci];
        const float sf = c.fill[ci];
        const float fci = kind == CELL_BED ? 2.0f : sf;
        float W = 0.0f;
        uint32_t na = 0;
        bool unit = true;
        const bool in[6] = {ix > 0, ix + 1 < u.gx, iy > 0, iy + 1 < u.gy, iz > 0, iz + 1 < u.gz};
        const uint32_t off[6] = {(uint32_t)-1, 1u, (uint32_t)0 - sy, sy, (uint32_t)0 - sz, sz};
        uint32_t fq[6], fj[6];
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            uint32_t e = SC_DUMMY;
            fq[f] = 0xffu;
            fj[f] = 0u;
            if (in[f]) {
                const uint32_t ni = ci + off[f];
                const int32_t nk = kl[ni];
                if (!is_solid(nk)) {
                    const float w = face_weight(kind, sf, nk, c.fill[ni]);
                    if (w > 0.0f) {
                        W += w;
                        if (is_fluid(nk)) {
                            const uint16_t rn = sb.ref_of_cell[ni];
                            unit = unit && (w == 1.0f);
                            if ((uint32_t)(rn >> 12) == r) {
                                e = rn & 4095u;
                            } else {
                                fq[f] = rn >> 12;
                                fj[f] = rn & 4095u;
                                e = 0xffffffffu;  // written by the neighbour
                            }
                        } else {
                            ++na;
                        }
                    }
                }
            }
            if (e != 0xffffffffu) sb.slot_ref[(((size_t)r * 3 + (f >> 1)) * 4096 + i) * 2 + (f & 1)] = (uint16_t)e;
        }
        // one halo slot per distinct foreign owner
        uint32_t hs[6];
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            hs[f] = 0xffffffffu;
            if (fq[f] == 0xffu) continue;
            for (int g = 0; g < f; ++g)
                if (fq[g] == fq[f]) hs[f] = hs[g];
            if (hs[f] == 0xffffffffu) {
                const uint32_t q = fq[f];
                const uint32_t h = atomicAdd(&sb.counts[q], 1u);
                hs[f] = h;
                if (h < (uint32_t)SC_HALO) {
                    sb.halo_fill[(size_t)q * SC_HALO + h] = fci;
                    atomicAdd(&sb.counts[SC_RECV0 + q * 2 + par], 1u);
                    const uint32_t e = atomicAdd(&sb.counts[SC_MAX_RANKS + r * 2 + par], 1u);
                    if (e < (uint32_t)SC_SEND) sb.send[((size_t)r * 2 + par) * SC_SEND + e] = i | (q << 12) | (h << 16);
                }
            }
            const uint32_t g = f ^ 1;  // the neighbour's face toward this cell
            sb.slot_ref[(((size_t)fq[f] * 3 + (g >> 1)) * 4096 + fj[f]) * 2 + (g & 1)] =
                (uint16_t)(hs[f] < (uint32_t)SC_HALO ? SC_HALO0 + hs[f] : SC_DUMMY);
        }
        // the cluster solve runs in FP32 pressure storage only, where the divergence is divf
        const float rhs = c.divf[ci] * sf / wmax(u.dt, 1e-6f);
        bool sent = false;
#pragma unroll
        for (int f = 0; f < 6; ++f) sent = sent || fq[f] != 0xffu;
        const uint32_t fl = na | (sent ? SC_SENT : 0u) | (unit ? SC_UNIT : 0u) | (W > 0.0f ? 0u : SC_EMPTY);
        sb.slot_coef[(size_t)r * 4096 + i] =
            make_float4(W > 0.0f ? 1.0f / W : 0.0f, fci, u.dx * u.dx * rhs, __uint_as_float(fl));
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

// One cluster per instance (blockIdx.y); R = cluster size along x.  With `p2p` the
// two colours of a red-black pair are separated by point-to-point waits (each CTA waits
// only for the halo values it receives, counted on its mbarriers) instead of cluster
// barriers.  Either way a CTA starts a colour only after every neighbour finished the
// other colour, so the values are the same.  The neighbour relation is symmetric with
// opposite colours (a black cell of CTA i next to a cell of CTA j makes that cell red and
// held by i), so a CTA can only send a colour after receiving the other colour from each
// receiver, which that receiver sent after it finished reading its old halo values:
// no store overwrites a halo value before it was read.
__global__ void __launch_bounds__(SC_THREADS, 1)
    k_sc_solve(const Ctx* __restrict__ cp, float tol, uint32_t max_pairs, uint32_t check_every, uint32_t p2p) {
    extern __shared__ __align__(16) unsigned char smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const Ctx& c = cp[blockIdx.y];
    const ScBuffers& sb = c.sb;
    const Params& u = c.u;
    const uint32_t R = cluster.num_blocks();
    const uint32_t rank = cluster.block_rank();
    const ScInfo& inf = *sb.info;
    // capacity: every rank reads the same counters, so the exit is uniform
    bool over = inf.overflow != 0u;
    for (uint32_t q = 0; q < R; ++q)
        over = over || sb.counts[q] > (uint32_t)SC_HALO || sb.counts[SC_MAX_RANKS + 2 * q] > (uint32_t)SC_SEND ||
               sb.counts[SC_MAX_RANKS + 2 * q + 1] > (uint32_t)SC_SEND;
    if (over) {
        if (rank == 0 && threadIdx.x == 0) sb.result->status = 2;
        return;
    }
    const uint32_t chunk = inf.chunk;
    const uint32_t start = rank * chunk;
    const uint32_t n_loc = (chunk == 0 || start >= inf.n_fluid) ? 0u : min(chunk, inf.n_fluid - start);
    const uint32_t n_red = inf.red_before[rank + 1] - inf.red_before[rank];
    const uint32_t n_halo = sb.counts[rank];
    const uint32_t n_send[2] = {sb.counts[SC_MAX_RANKS + 2 * rank], sb.counts[SC_MAX_RANKS + 2 * rank + 1]};
    const uint32_t n_recv[2] = {sb.counts[SC_RECV0 + 2 * rank], sb.counts[SC_RECV0 + 2 * rank + 1]};

    float* dval = sc_arr<float>(smem, ScLayout::dval);
    float* fcode = sc_arr<float>(smem, ScLayout::fcode);
    float* gg = sc_arr<float>(smem, ScLayout::g);
    float* invW = sc_arr<float>(smem, ScLayout::invW);
    float* ph = sc_arr<float>(smem, ScLayout::ph);
    float* pl = sc_arr<float>(smem, ScLayout::pl);
    float* bb = sc_arr<float>(smem, ScLayout::b);
    uint32_t* ref = sc_arr<uint32_t>(smem, ScLayout::ref);
    uint32_t* snd = sc_arr<uint32_t>(smem, ScLayout::snd);
    uint8_t* flg = sc_arr<uint8_t>(smem, ScLayout::flags);
    double* part = sc_arr<double>(smem, ScLayout::part);
    double* red = sc_arr<double>(smem, ScLayout::red);
    uint32_t* abortf = sc_arr<uint32_t>(smem, ScLayout::abortf);
    const uint32_t a_dval = (uint32_t)__cvta_generic_to_shared(dval);
    const uint32_t a_mbar = (uint32_t)__cvta_generic_to_shared(smem + ScLayout::mbar);  // 8 bytes per colour
    if (p2p && threadIdx.x == 0) {
        sc_mbar_init(a_mbar);
        sc_mbar_init(a_mbar + 8u);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    const uint32_t* cell_of = sb.cell_of + rank * 4096u;
    const uint32_t sy = u.gx, sz = u.gx * u.gy;

    // ---- set-up: copy this CTA's slice of the prep tables into shared memory ----
    {
        const float4* coef = sb.slot_coef + rank * 4096u;
        const uint32_t* sref = reinterpret_cast<const uint32_t*>(sb.slot_ref) + rank * 3u * 4096u;
        for (uint32_t i = threadIdx.x; i < n_loc; i += blockDim.x) {
            const float4 k = coef[i];
            const uint32_t fl = __float_as_uint(k.w);
            invW[i] = k.x;
            dval[i] = 0.0f;
            fcode[i] = k.y;
            bb[i] = k.z;
            flg[i] = (uint8_t)fl;
            ref[i] = sref[i] | ((fl & SC_UNIT) ? SC_REF_UNIT : 0u);
            ref[4096 + i] = sref[4096 + i];
            ref[8192 + i] = sref[8192 + i];
            const uint32_t ci = cell_of[i];
            ph[i] = c.pf[ci];
            pl[i] = c.plo[ci];
        }
        const float* hf = sb.halo_fill + (size_t)rank * SC_HALO;
        for (uint32_t h = threadIdx.x; h < n_halo; h += blockDim.x) {
            dval[SC_HALO0 + h] = 0.0f;
            fcode[SC_HALO0 + h] = hf[h];
        }
        if (threadIdx.x == 0) {
            dval[SC_DUMMY] = 0.0f;
            fcode[SC_DUMMY] = 0.0f;
        }
        for (uint32_t col = 0; col < 2; ++col) {
            const uint32_t* src = sb.send + ((size_t)rank * 2 + col) * SC_SEND;
            for (uint32_t e = threadIdx.x; e < n_send[col]; e += blockDim.x) snd[col * SC_SEND + e] = src[e];
        }
    }
    cluster.sync();

    bool timed_out = false;  // a point-to-point wait of this thread ran out
    bool abort_all = false;  // some CTA timed out (uniform: read from the reduction)

    // FP64 residual of the current pressure; g <- residual, d <- 0 (halo copies too).
    // Neighbour pressures come from this CTA's shared memory or, for halo cells, from
    // the global pressure arrays that accumulate() keeps current for every cell held
    // as halo.  Each CTA pushes its partial sums into every rank's shared memory, so
    // after the barrier all ranks add the same values in the same order and take the
    // same stop decision.
    auto residual = [&](int slot) -> double {
        double r2 = 0.0, b2 = 0.0;
        for (uint32_t i = threadIdx.x; i < n_loc; i += blockDim.x) {
            dval[i] = 0.0f;
            const uint8_t fl = flg[i];
            if (fl & SC_EMPTY) {
                gg[i] = 0.0f;
                continue;
            }
            const float fci = fcode[i];
            const float sfi = fci > 1.5f ? 1.0f : fci;
            double wsum = (double)(fl & 7u) * (double)sfi;
            double psum = 0.0;
            const uint32_t ci = cell_of[i];
            const uint32_t rw[3] = {ref[i], ref[4096 + i], ref[8192 + i]};
            const uint32_t off[6] = {(uint32_t)-1, 1u, (uint32_t)0 - sy, sy, (uint32_t)0 - sz, sz};
#pragma unroll
            for (int f = 0; f < 6; ++f) {
                const uint32_t r = (rw[f >> 1] >> ((f & 1) * 16)) & SC_SLOT_MASK;
                if (r == SC_DUMMY) continue;
                const float w = sc_weight(fci, fcode[r]);
                double pj;
                if (r < (uint32_t)SC_HALO0) {
                    pj = (double)ph[r] + (double)pl[r];
                } else {
                    const uint32_t nj = ci + off[f];
                    pj = (double)__ldcg(c.pf + nj) + (double)__ldcg(c.plo + nj);
                }
                wsum += (double)w;
                psum += (double)w * pj;
            }
            const double b = (double)bb[i];
            const double r = (psum - b) - wsum * ((double)ph[i] + (double)pl[i]);
            gg[i] = (float)r;
            r2 += r * r;
            b2 += b * b;
        }
        for (uint32_t h = threadIdx.x; h < n_halo; h += blockDim.x) dval[SC_HALO0 + h] = 0.0f;
        for (int o = 16; o > 0; o >>= 1) {
            r2 += __shfl_down_sync(0xffffffffu, r2, o);
            b2 += __shfl_down_sync(0xffffffffu, b2, o);
        }
        const int lane_id = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (lane_id == 0) {
            red[warp] = r2;
            red[32 + warp] = b2;
        }
        const uint32_t cta_timed_out = __syncthreads_or(timed_out ? 1 : 0) ? 1u : 0u;
        if (threadIdx.x < R) {
            double a = 0.0, bsum = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
                a += red[w];
                bsum += red[32 + w];
            }
            double* dst = cluster.map_shared_rank(part, threadIdx.x);
            dst[slot * 2 * SC_MAX_RANKS + rank] = a;
            dst[slot * 2 * SC_MAX_RANKS + SC_MAX_RANKS + rank] = bsum;
            uint32_t* fdst = cluster.map_shared_rank(abortf, threadIdx.x);
            fdst[slot * SC_MAX_RANKS + rank] = cta_timed_out;
        }
        cluster.sync();
        double a = 0.0, bsum = 0.0;
        for (uint32_t q = 0; q < R; ++q) {
            a += part[slot * 2 * SC_MAX_RANKS + q];
            bsum += part[slot * 2 * SC_MAX_RANKS + SC_MAX_RANKS + q];
            abort_all = abort_all || abortf[slot * SC_MAX_RANKS + q] != 0u;
        }
        if (bsum <= 0.0) return 0.0;
        return sqrt(a) / sqrt(bsum);
    };

    const float omega = u.omega;
    // New correction of one cell from its six neighbour slots (local loads only).  A
    // cell without faces has 1/W = 0, g = 0 and only zero neighbours, so its
    // correction stays exactly zero without a branch.
    auto relax = [&](uint32_t i) {
        const uint32_t r0 = ref[i], r1 = ref[4096 + i], r2 = ref[8192 + i];
        const uint32_t j0 = r0 & SC_SLOT_MASK, j1 = r0 >> 16, j2 = r1 & 0xffffu, j3 = r1 >> 16, j4 = r2 & 0xffffu,
                       j5 = r2 >> 16;
        const float v0 = dval[j0], v1 = dval[j1], v2 = dval[j2], v3 = dval[j3], v4 = dval[j4], v5 = dval[j5];
        const float me = dval[i];
        float ds = 0.0f;
        if (r0 & SC_REF_UNIT) {
            ds += v0;
            ds += v1;
            ds += v2;
            ds += v3;
            ds += v4;
            ds += v5;
        } else {
            const float fi = fcode[i];
            ds += sc_weight(fi, fcode[j0]) * v0;
            ds += sc_weight(fi, fcode[j1]) * v1;
            ds += sc_weight(fi, fcode[j2]) * v2;
            ds += sc_weight(fi, fcode[j3]) * v3;
            ds += sc_weight(fi, fcode[j4]) * v4;
            ds += sc_weight(fi, fcode[j5]) * v5;
        }
        float dn = (ds + gg[i]) * invW[i];
        if (omega != 1.0f) dn = me + omega * (dn - me);
        dval[i] = dn;
    };
    // push the new values of colour `col` to the CTAs that hold them as halo
    auto push = [&](uint32_t col) {
        const uint32_t* list = snd + col * SC_SEND;
        for (uint32_t e = threadIdx.x; e < n_send[col]; e += blockDim.x) {
            const uint32_t s = list[e];
            const uint32_t src = s & 4095u, q = (s >> 12) & 15u, h = s >> 16;
            const uint32_t dst = sc_mapa(a_dval + (uint32_t)(SC_HALO0 + h) * 4u, q);
            if (p2p)
                sc_st_async(dst, dval[src], sc_mapa(a_mbar + col * 8u, q));
            else
                sc_st(dst, dval[src]);
        }
    };
    auto sweep = [&](uint32_t lo, uint32_t hi, uint32_t col) {
        for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) relax(i);
        __syncthreads();
        push(col);
    };
    // p2p: arm this CTA's mbarrier of colour `col` with the bytes it receives and wait
    uint32_t phase_bits = 0;  // bit col: parity of the next phase of mbarrier col
    auto wait_colour = [&](uint32_t col) {
        const uint32_t a = a_mbar + col * 8u;
        if (threadIdx.x == 0) sc_mbar_expect(a, 4u * n_recv[col]);
        // after one timeout the remaining waits of the solve only poll once
        if (!sc_mbar_wait(a, (phase_bits >> col) & 1u, timed_out ? 0ll : kScWaitCycles)) timed_out = true;
        phase_bits ^= 1u << col;
    };

    // p <- p + d in FP64, split back into hi/lo.  Cells other CTAs hold as halo are
    // published to the global arrays for the next residual (all cells at the end).
    auto accumulate = [&]() {
        const double lim = (double)u.p_limit;
        for (uint32_t i = threadIdx.x; i < n_loc; i += blockDim.x) {
            double p = ((double)ph[i] + (double)pl[i]) + (double)dval[i];
            if (p > lim || p < -lim) {
                p = p > 0.0 ? lim : -lim;
                atomicAdd(&c.metrics[M_P_CLAMP], 1u);
            }
            const float hi = (float)p;
            const float lo = (float)(p - (double)hi);
            ph[i] = hi;
            pl[i] = lo;
            if (flg[i] & SC_SENT) {
                const uint32_t ci = cell_of[i];
                c.pf[ci] = hi;
                c.plo[ci] = lo;
            }
        }
    };

    const uint32_t ce = check_every ? check_every : 10u;
    int slot = 0;
    double r0 = residual(slot);
    double r1 = r0;
    uint32_t pairs = 0, evals = 1;
    uint32_t next = u.first_check ? u.first_check : ce;  // pairs before the next check (same on every CTA)
    while (!(r1 <= (double)tol) && pairs < max_pairs && !abort_all) {
        uint32_t k = min(next, max_pairs - pairs);
        for (uint32_t j = 0; j < k; ++j) {
            if (!p2p)
                cluster.sync();
            else if (j > 0)
                wait_colour(1);  // black values of the previous pair
            sweep(0, n_red, 0);
            if (!p2p)
                cluster.sync();
            else
                wait_colour(0);  // red values of this pair
            sweep(n_red, n_loc, 1);
        }
        if (p2p) wait_colour(1);
        pairs += k;
        __syncthreads();
        accumulate();
        cluster.sync();
        slot ^= 1;
        const double r_before = r1;
        r1 = residual(slot);
        ++evals;
        next = sc_next_interval(r1, r_before, k, (double)tol, ce);
    }
    // publish every owned cell (the loop above published only halo-held ones)
    if (pairs > 0)
        for (uint32_t i = threadIdx.x; i < n_loc; i += blockDim.x)
            if (!(flg[i] & SC_SENT)) {
                const uint32_t ci = cell_of[i];
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
    const bool gave_up = __syncthreads_or(timed_out ? 1 : 0) != 0;
    if (abort_all) {
        // stores that were still travelling when a wait gave up land within microseconds;
        // give them ~10 ms before the CTAs leave
        const long long t0 = clock64();
        while (clock64() - t0 < (1ll << 24)) {
        }
    }
    cluster.sync();  // keep every CTA's shared memory alive until remote accesses end
    if (gave_up && threadIdx.x == 0) {
        // a point-to-point wait ran out: the values are not trusted (the host falls
        // back to per-colour launches) and the timeout is reported
        atomicExch(&sb.result->status, 3u);
        atomicOr(&c.metrics[M_TIMEOUT], 1u);
    }
}

// The same for every instance of a batched launch (thread i: instance i).
__global__ void k_sc_account_batch(const Ctx* __restrict__ cp, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const ScResult r = *cp[i].sb.result;
    ScTotals* tot = cp[i].totals;
    tot->runs += 1;
    if (r.status == 3) {
        tot->timeouts += 1;
    } else if (r.status != 1) {
        tot->failed += 1;
    } else {
        tot->sweeps += r.sweeps;
        tot->evals += r.evals;
    }
    tot->last = r;
}

// Adds one solve's result to the running totals (one thread; graph mode, where the
// host does not read each substep's result).
__global__ void k_sc_account(const ScResult* __restrict__ res, ScTotals* __restrict__ tot) {
    const ScResult r = *res;
    tot->runs += 1;
    if (r.status == 3) {
        tot->timeouts += 1;
    } else if (r.status != 1) {
        tot->failed += 1;
    } else {
        tot->sweeps += r.sweeps;
        tot->evals += r.evals;
    }
    tot->last = r;
}

}  // namespace cs
