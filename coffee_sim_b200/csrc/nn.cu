// nn.cu — BF16 3-D convolution on the tcgen05 tensor cores, and the elementwise pieces
// of the pressure-guess U-Net (learned warm start; no counterpart in the reference).
//
// Activations are channels-last bf16, [voxel][C] with C a multiple of 8, voxel =
// (z * gy + y) * gx + x.  A 3x3x3 "same" convolution is one GEMM per 128-voxel tile:
//   Y[v][co] = b[co] + sum_{t, ci} W[co][t * Cin + ci] * X[v + off_t][ci]
// with M = 128 voxels, N = Cout, K = 27 * Cin taken 64 at a time.  The A operand is
// gathered straight from X into shared memory (implicit im2col: one 16-byte load per
// tap and 8 channels, zero outside the grid), B is the weight matrix, the accumulator
// lives in TMEM, and the epilogue adds the bias, applies ReLU and stores bf16 (and
// optionally f32).  The gradient w.r.t. the input is the same convolution with flipped,
// transposed weights.  The weight gradient is a second GEMM,
//   dW^T[t * Cin + ci][co] = sum_v X[v + off_t][ci] * dY[v][co],
// with M = 27 * Cin, N = Cout and K = voxels split over CTAs; both operands are loaded
// 8 voxels x 8 channels at a time and transposed in registers into K-major form.
//
// Every mbarrier wait is bounded; on a timeout the kernel raises a flag in `err`,
// waits (bounded) for its own MMAs, frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>

#include "../../include/coffee_sim.h"
#include "umma.cuh"

namespace cs {
void set_error(const std::string& msg);

namespace nn {

constexpr int BM = 128;       // voxels (rows) per tile
constexpr int BKC = 8;        // 16-byte K chunks per stage (64 bf16)
constexpr int THREADS = 128;  // 4 warps: warp w owns TMEM lanes 32w..32w+31
constexpr uint32_t WAIT_LIMIT = 1u << 22;
static_assert(BM == 128 && BKC == 8 && THREADS == 128, "loader thread mapping assumes 128 x 8 chunks, 128 threads");

struct Grid3 {
    int gx, gy, gz;
    __host__ __device__ int voxels() const { return gx * gy * gz; }
};

__device__ __forceinline__ int tap_dx(int t) { return t % 3 - 1; }
__device__ __forceinline__ int tap_dy(int t) { return (t / 3) % 3 - 1; }
__device__ __forceinline__ int tap_dz(int t) { return t / 9 - 1; }

// byte offset of (row, k chunk) in a K-major no-swizzle operand of `rows` rows and
// BKC chunks: core matrix (group = row / 8, chunk) at (chunk * rows / 8 + group) * 128
__device__ __forceinline__ uint32_t core_off(int row, int chunk, int rows) {
    return (uint32_t)((chunk * (rows >> 3) + (row >> 3)) * 128 + (row & 7) * 16);
}

// 8x8 transpose of bf16: in[j] holds 8 values of row j; out[r] gets column r.
__device__ __forceinline__ void transpose8(const uint4 (&in)[8], uint4 (&out)[8]) {
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t a = (&in[2 * q].x)[r >> 1], b = (&in[2 * q + 1].x)[r >> 1];
            w[q] = __byte_perm(a, b, (r & 1) ? 0x7632 : 0x5410);
        }
        out[r] = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

struct ConvArgs {
    Grid3 g;
    const __nv_bfloat16* x;  // [vox][cin]
    const __nv_bfloat16* w;  // [cout_pad][kpad], K = t * cin + ci, zero padded
    const float* bias;       // [cout] or null
    __nv_bfloat16* y;        // [vox][cout_store] or null
    float* y32;              // [vox][cout] or null
    int cin, cout_pad, cout_store, kpad, relu;
    const __nv_bfloat16* dy;  // weight gradient: [vox][cout_pad]
    float* dwt;               // weight gradient: [27 * cin][cout_pad], accumulated
    int m_rows;               // weight gradient: 27 * cin
    int k_per_split;          // weight gradient: voxels per CTA (multiple of 64)
    uint32_t* err;
};

// MODE 0: convolution (forward / input gradient); MODE 1: weight gradient.
template <int MODE>
__global__ void __launch_bounds__(THREADS) k_conv_umma(ConvArgs a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t bars[2];
    __shared__ uint32_t tmem_base;
    const int N = a.cout_pad;
    const int a_bytes = BM * BKC * 16, b_bytes = N * BKC * 16;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t ncols = N <= 32 ? 32u : N <= 64 ? 64u : N <= 128 ? 128u : 256u;

    if (warp == 0) {
        umma::tmem_alloc(&tmem_base, ncols);
        umma::tmem_relinquish();
    }
    if (tid == 0) {
        umma::mbar_init(&bars[0], 1);
        umma::mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = tmem_base;

    const int nvox = a.g.voxels();
    const int m0 = blockIdx.x * BM;
    int nstages, k0 = 0;
    if (MODE == 0) {
        nstages = a.kpad / (BKC * 8);
    } else {
        k0 = blockIdx.y * a.k_per_split;
        const int kend = min(k0 + a.k_per_split, nvox);
        nstages = kend > k0 ? (kend - k0 + BKC * 8 - 1) / (BKC * 8) : 0;
    }
    const uint32_t idesc = umma::idesc_bf16_f32((uint32_t)N);
    uint32_t phase0 = 0u, phase1 = 0u;  // completed-phase parity of each buffer's barrier
    bool ok = true;

    // MODE 0 loader: thread tid always fills K chunk (tid & 7) of rows (tid >> 3) + 16 k,
    // k = 0..7; their voxel coordinates are decoded once (x < 0 marks a row past the end)
    int rx[8], ry[8], rz[8];
    if (MODE == 0) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int v = m0 + (tid >> 3) + 16 * k;
            rx[k] = v < nvox ? v % a.g.gx : -1;
            ry[k] = (v / a.g.gx) % a.g.gy;
            rz[k] = v / (a.g.gx * a.g.gy);
        }
    }

    for (int s = 0; s < nstages && ok; ++s) {
        const int buf = s & 1;
        if (s >= 2) {  // the MMAs of stage s-2 read this buffer
            const bool w = umma::mbar_wait(&bars[buf], buf ? phase1 : phase0, WAIT_LIMIT);
            if (buf) phase1 ^= 1u; else phase0 ^= 1u;
            ok = __syncthreads_and(w ? 1 : 0) != 0;  // one decision for the whole CTA
            if (!ok) break;
        }
        unsigned char* A = buf ? sm + a_bytes + b_bytes : sm;
        unsigned char* B = A + a_bytes;
        if (MODE == 0) {
            const int cgroups = a.cin >> 3;
            const int kchunks = 27 * cgroups;
            // A: 128 rows x 8 chunks; this thread's chunk is one (tap, 8-channel group)
            const int c = tid & (BKC - 1);
            const int kc = s * BKC + c;
            const int t = kc / cgroups, cg = kc - t * cgroups;
            const int dx = tap_dx(t), dy = tap_dy(t), dz = tap_dz(t);
            const bool live = kc < kchunks;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int row = (tid >> 3) + 16 * k;
                const int xs = rx[k] + dx, ys = ry[k] + dy, zs = rz[k] + dz;
                uint4 val = make_uint4(0u, 0u, 0u, 0u);
                if (live && rx[k] >= 0 && xs >= 0 && ys >= 0 && zs >= 0 && xs < a.g.gx && ys < a.g.gy &&
                    zs < a.g.gz) {
                    const int src = (zs * a.g.gy + ys) * a.g.gx + xs;
                    val = *reinterpret_cast<const uint4*>(a.x + (size_t)src * a.cin + cg * 8);
                }
                *reinterpret_cast<uint4*>(A + core_off(row, c, BM)) = val;
            }
            for (int i = tid; i < N * BKC; i += THREADS) {
                const int row = i / BKC, c = i % BKC;
                const uint4 val =
                    *reinterpret_cast<const uint4*>(a.w + (size_t)row * a.kpad + (size_t)(s * BKC + c) * 8);
                *reinterpret_cast<uint4*>(B + core_off(row, c, N)) = val;
            }
        } else {
            const int vbase = k0 + s * BKC * 8;
            // A: rows (t, ci) x 8 voxel chunks; one 8x8 block per task
            for (int task = tid; task < (BM >> 3) * BKC; task += THREADS) {
                const int rg = task / BKC, c = task % BKC;
                const int m = m0 + rg * 8;  // first row of the group: (t, ci0)
                uint4 in[8];
                const int t = m / a.cin, ci0 = m % a.cin;
                const int dx = tap_dx(t), dy = tap_dy(t), dz = tap_dz(t);
                // the 8 voxels are consecutive: decode the first, then step along x
                const int v0 = vbase + c * 8;
                int x = v0 % a.g.gx, y = (v0 / a.g.gx) % a.g.gy, z = v0 / (a.g.gx * a.g.gy);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    in[j] = make_uint4(0u, 0u, 0u, 0u);
                    const int v = v0 + j;
                    if (m < a.m_rows && v < nvox && v < k0 + a.k_per_split) {
                        const int xs = x + dx, ys = y + dy, zs = z + dz;
                        if (xs >= 0 && ys >= 0 && zs >= 0 && xs < a.g.gx && ys < a.g.gy && zs < a.g.gz)
                            in[j] = *reinterpret_cast<const uint4*>(
                                a.x + (size_t)((zs * a.g.gy + ys) * a.g.gx + xs) * a.cin + ci0);
                    }
                    if (++x == a.g.gx) {
                        x = 0;
                        if (++y == a.g.gy) {
                            y = 0;
                            ++z;
                        }
                    }
                }
                uint4 out[8];
                transpose8(in, out);
#pragma unroll
                for (int r = 0; r < 8; ++r) *reinterpret_cast<uint4*>(A + core_off(rg * 8 + r, c, BM)) = out[r];
            }
            for (int task = tid; task < (N >> 3) * BKC; task += THREADS) {
                const int rg = task / BKC, c = task % BKC;
                uint4 in[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int v = vbase + c * 8 + j;
                    in[j] = (v < nvox && v < k0 + a.k_per_split)
                                ? *reinterpret_cast<const uint4*>(a.dy + (size_t)v * N + rg * 8)
                                : make_uint4(0u, 0u, 0u, 0u);
                }
                uint4 out[8];
                transpose8(in, out);
#pragma unroll
                for (int r = 0; r < 8; ++r) *reinterpret_cast<uint4*>(B + core_off(rg * 8 + r, c, N)) = out[r];
            }
        }
        umma::fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            umma::fence_after_sync();
            const uint32_t a_addr = umma::smem_addr(A), b_addr = umma::smem_addr(B);
#pragma unroll
            for (int j = 0; j < BKC / 2; ++j) {
                const uint64_t da = umma::smem_desc(a_addr + j * 2 * (BM / 8) * 128, (BM / 8) * 128, 128);
                const uint64_t db = umma::smem_desc(b_addr + j * 2 * (N / 8) * 128, (N / 8) * 128, 128);
                umma::mma_bf16(tmem, da, db, idesc, (s > 0 || j > 0) ? 1u : 0u);
            }
            umma::commit(&bars[buf]);
        }
        __syncthreads();
    }
    // the last commit covers every MMA of this CTA
    if (nstages > 0) {
        const int lb = (nstages - 1) & 1;
        const bool done = umma::mbar_wait(&bars[lb], lb ? phase1 : phase0, WAIT_LIMIT);
        ok = __syncthreads_and((done && ok) ? 1 : 0) != 0;
        if (!ok && tid == 0) atomicOr(a.err, 1u);
    }
    umma::fence_after_sync();
    if (ok && nstages > 0) {
        const int row = warp * 32 + (tid & 31);
        const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
        for (int c0 = 0; c0 < N; c0 += 8) {
            float v[8];
            umma::tmem_ld8(lane_addr + (uint32_t)c0, v);
            umma::tmem_wait_ld();
            if (MODE == 0) {
                const int vox = m0 + row;
                if (vox >= nvox) continue;
                for (int q = 0; q < 8; ++q) {
                    const int co = c0 + q;
                    float r = v[q] + ((a.bias && co < a.cout_store) ? a.bias[co] : 0.0f);
                    if (a.relu) r = fmaxf(r, 0.0f);
                    v[q] = co < a.cout_store ? r : 0.0f;
                }
                if (a.y && c0 < a.cout_store) {
                    __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) h[q] = __float2bfloat16(v[q]);
                    *reinterpret_cast<uint4*>(a.y + (size_t)vox * a.cout_store + c0) =
                        *reinterpret_cast<const uint4*>(h);
                }
                if (a.y32)
                    for (int q = 0; q < 8 && c0 + q < a.cout_store; ++q) a.y32[(size_t)vox * a.cout_store + c0 + q] = v[q];
            } else {
                const int m = m0 + row;
                if (m >= a.m_rows) continue;
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if (v[q] != 0.0f) atomicAdd(&a.dwt[(size_t)m * N + c0 + q], v[q]);
            }
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem, ncols);
}

// ---- forward convolution with an asynchronous copy pipeline ----
// Same GEMM as k_conv_umma<0>, with NBUF stage buffers: the 16-byte operand chunks of
// stage s + LOOKAHEAD are copied with cp.async (zero-filled outside the grid) while the
// tensor cores work on stage s, so the gathers' latency overlaps the MMAs.  A buffer is
// refilled only after the MMAs of the stage that last used it have completed (mbarrier).
constexpr int NBUF = 4, LOOKAHEAD = 2;

__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(umma::smem_addr(dst)), "l"(src),
                 "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__global__ void __launch_bounds__(THREADS) k_conv_fwd(ConvArgs a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t bars[NBUF];
    __shared__ uint32_t tmem_base;
    const int N = a.cout_pad;
    const int a_bytes = BM * BKC * 16, b_bytes = N * BKC * 16, stage_bytes = a_bytes + b_bytes;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t ncols = N <= 32 ? 32u : N <= 64 ? 64u : N <= 128 ? 128u : 256u;
    if (warp == 0) {
        umma::tmem_alloc(&tmem_base, ncols);
        umma::tmem_relinquish();
    }
    if (tid == 0) {
        for (int b = 0; b < NBUF; ++b) umma::mbar_init(&bars[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = tmem_base;

    const int nvox = a.g.voxels();
    const int m0 = blockIdx.x * BM;
    const int nstages = a.kpad / (BKC * 8);
    const int cgroups = a.cin >> 3;
    const int kchunks = 27 * cgroups;
    const uint32_t idesc = umma::idesc_bf16_f32((uint32_t)N);
    // thread tid fills K chunk (tid & 7) of rows (tid >> 3) + 16 k of every A stage
    const int c = tid & (BKC - 1);
    int rx[8], ry[8], rz[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int v = m0 + (tid >> 3) + 16 * k;
        rx[k] = v < nvox ? v % a.g.gx : -1;
        ry[k] = (v / a.g.gx) % a.g.gy;
        rz[k] = v / (a.g.gx * a.g.gy);
    }
    auto issue = [&](int st) {
        unsigned char* A = sm + (st % NBUF) * stage_bytes;
        unsigned char* B = A + a_bytes;
        const int kc = st * BKC + c;
        const int t = kc / cgroups, cg = kc - t * cgroups;
        const int dx = tap_dx(t), dy = tap_dy(t), dz = tap_dz(t);
        const bool live = kc < kchunks;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int xs = rx[k] + dx, ys = ry[k] + dy, zs = rz[k] + dz;
            const bool ok = live && rx[k] >= 0 && xs >= 0 && ys >= 0 && zs >= 0 && xs < a.g.gx && ys < a.g.gy &&
                            zs < a.g.gz;
            const __nv_bfloat16* src = ok ? a.x + (size_t)((zs * a.g.gy + ys) * a.g.gx + xs) * a.cin + cg * 8 : a.x;
            cp_async16(A + core_off((tid >> 3) + 16 * k, c, BM), src, ok);
        }
        for (int i = tid; i < N * BKC; i += THREADS) {
            const int row = i / BKC, cc = i % BKC;
            cp_async16(B + core_off(row, cc, N), a.w + (size_t)row * a.kpad + (size_t)(st * BKC + cc) * 8, true);
        }
    };

    bool ok = true;
    // one copy group per stage (empty past the end), so that waiting until at most
    // LOOKAHEAD groups are pending means stage s has landed
    for (int st = 0; st < LOOKAHEAD; ++st) {
        if (st < nstages) issue(st);
        cp_async_commit();
    }
    for (int s = 0; s < nstages; ++s) {
        const int next = s + LOOKAHEAD;
        if (next < nstages) {
            const int prev = next - NBUF;  // the stage that last used this buffer
            bool w = true;
            if (prev >= 0) w = umma::mbar_wait(&bars[next % NBUF], (uint32_t)((prev / NBUF) & 1), WAIT_LIMIT);
            if (!__syncthreads_and(w ? 1 : 0)) {
                ok = false;
                break;
            }
            issue(next);
        }
        cp_async_commit();  // (possibly empty) group keeps the group count aligned with stages
        cp_async_wait<LOOKAHEAD>();
        umma::fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            umma::fence_after_sync();
            unsigned char* A = sm + (s % NBUF) * stage_bytes;
            const uint32_t a_addr = umma::smem_addr(A), b_addr = umma::smem_addr(A + a_bytes);
#pragma unroll
            for (int j = 0; j < BKC / 2; ++j) {
                const uint64_t da = umma::smem_desc(a_addr + j * 2 * (BM / 8) * 128, (BM / 8) * 128, 128);
                const uint64_t db = umma::smem_desc(b_addr + j * 2 * (N / 8) * 128, (N / 8) * 128, 128);
                umma::mma_bf16(tmem, da, db, idesc, (s > 0 || j > 0) ? 1u : 0u);
            }
            umma::commit(&bars[s % NBUF]);
        }
    }
    cp_async_wait<0>();
    if (nstages > 0) {
        const int last = nstages - 1;
        const bool done = umma::mbar_wait(&bars[last % NBUF], (uint32_t)((last / NBUF) & 1), WAIT_LIMIT);
        ok = __syncthreads_and((done && ok) ? 1 : 0) != 0;
        if (!ok && tid == 0) atomicOr(a.err, 1u);
    }
    umma::fence_after_sync();
    if (ok && nstages > 0) {
        const int row = warp * 32 + (tid & 31);
        const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
        const int vox = m0 + row;
        for (int c0 = 0; c0 < N; c0 += 8) {
            float v[8];
            umma::tmem_ld8(lane_addr + (uint32_t)c0, v);
            umma::tmem_wait_ld();
            if (vox >= nvox) continue;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                float r = v[q] + (a.bias ? a.bias[c0 + q] : 0.0f);
                v[q] = a.relu ? fmaxf(r, 0.0f) : r;
            }
            if (a.y) {
                __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) h[q] = __float2bfloat16(v[q]);
                *reinterpret_cast<uint4*>(a.y + (size_t)vox * N + c0) = *reinterpret_cast<const uint4*>(h);
            }
            if (a.y32)
#pragma unroll
                for (int q = 0; q < 8; ++q) a.y32[(size_t)vox * N + c0 + q] = v[q];
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem, ncols);
}

// Halo-tiled convolution: a CTA computes an 8 (x) x 16 (y) x 1 (z) block of output voxels
// (M = 128).  Its input block with a one-voxel halo, 10 x 18 x 3 voxels, is loaded once
// by TMA (one tiled box per 8-channel block, zeros outside the grid) into shared memory
// as [channel block][z][y][x][8 channels] (16 bytes per voxel and block; the channel
// count is padded to a multiple of 16 with zero blocks).  In that layout the A operand of tap (dx, dy, dz) is the same block shifted:
// a core matrix is 8 consecutive x voxels (128 contiguous bytes), consecutive 8-row
// groups (y) are 10 * 16 = 160 bytes apart (SBO) and consecutive channel blocks one
// block plane apart (LBO), so every tap's MMAs read the one copy through a descriptor
// with a shifted start address.  The weights of each tap (N x Cpad) stream through a
// ring of HB_SLOTS shared-memory slots with cp.async; a slot is refilled once the MMAs
// that read it have completed (tcgen05.commit to the slot's mbarrier).
constexpr int HX = 10, HY = 18, HZ = 3, HVOX = HX * HY * HZ, HB_PLANE = HVOX * 16, HB_SLOTS = 3;
// channel-block planes start 128-byte aligned (a tiled TMA box lands at a 128-byte
// aligned shared address): 8640 bytes of data in an 8704-byte stride
constexpr int HB_PSTRIDE = (HB_PLANE + 127) / 128 * 128;

// shared memory of the halo kernel: input block plus a ring of HB_SLOTS taps' weights
// (`all_taps` false) or every tap's weights at once
static size_t halo_smem(int cin_pad16, int n, bool all_taps) {
    return (size_t)(cin_pad16 / 8) * HB_PSTRIDE + (size_t)(all_taps ? 27 : HB_SLOTS) * n * cin_pad16 * 2;
}

// all_taps: every tap's weights are resident (one copy group, all MMAs issued back to
// back under one commit); otherwise they stream through the ring.
template <bool ALL>
__global__ void __launch_bounds__(THREADS) k_conv_halo(ConvArgs a, const __grid_constant__ CUtensorMap xmap) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t bars[HB_SLOTS];
    __shared__ uint64_t halo_bar;
    __shared__ uint32_t tmem_base;
    const int N = a.cout_pad;
    const int cpad = (a.cin + 15) & ~15;  // channels as the MMAs see them (K = 16 per MMA)
    const int ncb = cpad >> 3;            // 8-channel blocks, even
    const int b_bytes = N * cpad * 2;     // one tap's weights
    unsigned char* halo = sm;
    unsigned char* bring = sm + (size_t)ncb * HB_PSTRIDE;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t ncols = N <= 32 ? 32u : N <= 64 ? 64u : N <= 128 ? 128u : 256u;
    if (warp == 0) {
        umma::tmem_alloc(&tmem_base, ncols);
        umma::tmem_relinquish();
    }
    if (tid == 0) {
        for (int b = 0; b < HB_SLOTS; ++b) umma::mbar_init(&bars[b], 1);
        umma::mbar_init(&halo_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = tmem_base;

    const int tx = (a.g.gx + 7) >> 3, ty = (a.g.gy + 15) >> 4;
    const int bx = blockIdx.x % tx, by = (blockIdx.x / tx) % ty, bz = blockIdx.x / (tx * ty);
    const int x0 = bx * 8, y0 = by * 16, z0 = bz;
    const uint32_t idesc = umma::idesc_bf16_f32((uint32_t)N);

    // input block with halo: one TMA box (8 channels x 10 x 18 x 3 voxels, zeros outside
    // the grid) per 8-channel block, landing as [z][y][x][8 channels]; channel blocks past
    // cin (padding to a multiple of 16) are zeroed here
    const int ncb_in = a.cin >> 3;
    for (int e = ncb_in * HVOX + tid; e < ncb * HVOX; e += THREADS)
        *reinterpret_cast<uint4*>(halo + (size_t)(e / HVOX) * HB_PSTRIDE + (e % HVOX) * 16) =
            make_uint4(0u, 0u, 0u, 0u);
    if (tid == 0) {
        const uint32_t bar = umma::smem_addr(&halo_bar);
        asm volatile(
            "{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(bar),
            "r"((uint32_t)(ncb_in * HB_PLANE))
            : "memory");
        for (int cb = 0; cb < ncb_in; ++cb)
            asm volatile(
                "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
                "%4, %5}], [%6];" ::"r"(umma::smem_addr(halo + (size_t)cb * HB_PSTRIDE)),
                "l"(reinterpret_cast<uint64_t>(&xmap)), "r"(cb * 8), "r"(x0 - 1), "r"(y0 - 1), "r"(z0 - 1), "r"(bar)
                : "memory");
    }
    // tap t's weights into its slot (ring slot t % HB_SLOTS, or slot t with every tap
    // resident), as N x cpad K-major core matrices
    auto slot_of = [&](int t) { return ALL ? t : t % HB_SLOTS; };
    auto load_b = [&](int t) {
        unsigned char* B = bring + (size_t)slot_of(t) * b_bytes;
        for (int i = tid; i < N * ncb; i += THREADS) {
            const int row = i / ncb, cb = i - row * ncb;
            const bool ok = cb * 8 < a.cin;
            const __nv_bfloat16* src = a.w + (size_t)row * a.kpad + (size_t)t * a.cin + cb * 8;
            cp_async16(B + core_off(row, cb, N), ok ? src : a.w, ok);
        }
    };
    bool ok = true;
    int issued = -1;  // last tap whose MMAs were issued
    // weights in flight first (every tap, or the first HB_SLOTS), then the input block
    if (ALL) {
        // each thread owns fixed (row, channel block) pairs and copies them for every tap:
        // tap t's copy is t * b_bytes further in shared memory and t * cin further in
        // the packed weights
        for (int i = tid; i < N * ncb; i += THREADS) {
            const int row = i / ncb, cb = i - row * ncb;
            const bool ok = cb * 8 < a.cin;
            unsigned char* dst = bring + core_off(row, cb, N);
            const __nv_bfloat16* src = a.w + (size_t)row * a.kpad + cb * 8;
            for (int t = 0; t < 27; ++t, dst += b_bytes, src += a.cin) cp_async16(dst, ok ? src : a.w, ok);
        }
        cp_async_commit();
    } else {
        for (int t = 0; t < HB_SLOTS; ++t) {
            load_b(t);
            cp_async_commit();
        }
    }
    const bool halo_ok = umma::mbar_wait(&halo_bar, 0u, WAIT_LIMIT);
    if (ALL) {
        cp_async_wait<0>();
        umma::fence_proxy_async();
        ok = __syncthreads_and(halo_ok ? 1 : 0) != 0;
    }
    if (ALL && ok) {
        if (tid == 0) {
            umma::fence_after_sync();
            for (int t = 0; t < 27; ++t) {
                const int dx = t % 3, dy = (t / 3) % 3, dz = t / 9;
                const uint32_t a_base = umma::smem_addr(halo) + (uint32_t)(((dz * HY + dy) * HX + dx) * 16);
                const uint32_t b_base = umma::smem_addr(bring + (size_t)t * b_bytes);
                for (int j = 0; j < ncb / 2; ++j) {
                    const uint64_t da = umma::smem_desc(a_base + (uint32_t)(2 * j * HB_PSTRIDE), HB_PSTRIDE, HX * 16);
                    const uint64_t db =
                        umma::smem_desc(b_base + (uint32_t)(2 * j * (N / 8) * 128), (N / 8) * 128, 128);
                    umma::mma_bf16(tmem, da, db, idesc, (t > 0 || j > 0) ? 1u : 0u);
                }
            }
            umma::commit(&bars[0]);
        }
        issued = 26;
    }
    if (!ALL) ok = __syncthreads_and(halo_ok ? 1 : 0) != 0;
    for (int t = 0; t < (ALL || !ok ? 0 : 27); ++t) {
        // groups committed after tap t's weights: HB_SLOTS - 1 at t = 0, then one refill
        // per iteration keeps it at one
        if (t == 0)
            cp_async_wait<HB_SLOTS - 1>();
        else
            cp_async_wait<1>();
        umma::fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            umma::fence_after_sync();
            const int dx = t % 3, dy = (t / 3) % 3, dz = t / 9;
            const uint32_t a_base = umma::smem_addr(halo) + (uint32_t)(((dz * HY + dy) * HX + dx) * 16);
            const uint32_t b_base = umma::smem_addr(bring + (size_t)(t % HB_SLOTS) * b_bytes);
            for (int j = 0; j < ncb / 2; ++j) {
                const uint64_t da = umma::smem_desc(a_base + (uint32_t)(2 * j * HB_PSTRIDE), HB_PSTRIDE, HX * 16);
                const uint64_t db = umma::smem_desc(b_base + (uint32_t)(2 * j * (N / 8) * 128), (N / 8) * 128, 128);
                umma::mma_bf16(tmem, da, db, idesc, (t > 0 || j > 0) ? 1u : 0u);
            }
            umma::commit(&bars[t % HB_SLOTS]);
        }
        issued = t;
        // refill the slot of tap t - 1 (its MMAs were issued one iteration ago) with tap
        // t - 1 + HB_SLOTS; every iteration commits one group, empty past the last tap
        const int prev = t - 1, next = prev + HB_SLOTS;
        if (prev >= 0 && next < 27) {
            const bool w = umma::mbar_wait(&bars[prev % HB_SLOTS], (uint32_t)((prev / HB_SLOTS) & 1), WAIT_LIMIT);
            if (!__syncthreads_and(w ? 1 : 0)) {
                ok = false;
                break;
            }
            load_b(next);
        }
        if (t > 0) cp_async_commit();
    }
    cp_async_wait<0>();
    // the last tap's commit covers every MMA issued before it
    if (issued >= 0) {
        const int sl = ALL ? 0 : issued % HB_SLOTS;
        const uint32_t ph = ALL ? 0u : (uint32_t)((issued / HB_SLOTS) & 1);
        const bool done = umma::mbar_wait(&bars[sl], ph, WAIT_LIMIT);
        ok = __syncthreads_and((done && ok) ? 1 : 0) != 0;
    }
    if (!ok && tid == 0) atomicOr(a.err, 1u);
    umma::fence_after_sync();
    if (ok && issued == 26) {
        const int row = warp * 32 + (tid & 31);  // M row: x = row % 8, y = row / 8
        const int xo = x0 + (row & 7), yo = y0 + (row >> 3);
        const bool inside = xo < a.g.gx && yo < a.g.gy;
        const int vox = (z0 * a.g.gy + yo) * a.g.gx + xo;
        const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
        for (int c0 = 0; c0 < N; c0 += 8) {
            float v[8];
            umma::tmem_ld8(lane_addr + (uint32_t)c0, v);
            umma::tmem_wait_ld();
            if (!inside) continue;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                float r = v[q] + (a.bias ? a.bias[c0 + q] : 0.0f);
                v[q] = a.relu ? fmaxf(r, 0.0f) : r;
            }
            if (a.y) {
                __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) h[q] = __float2bfloat16(v[q]);
                *reinterpret_cast<uint4*>(a.y + (size_t)vox * N + c0) = *reinterpret_cast<const uint4*>(h);
            }
            if (a.y32)
#pragma unroll
                for (int q = 0; q < 8; ++q) a.y32[(size_t)vox * N + c0 + q] = v[q];
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem, ncols);
}

static size_t conv_smem(int n) { return (size_t)2 * (BM + n) * BKC * 16; }

template <int MODE>
static int launch(const ConvArgs& a, dim3 grid, cudaStream_t st) {
    const size_t smem = conv_smem(a.cout_pad);
    static bool attr[2] = {false, false};
    if (!attr[MODE]) {
        cudaFuncSetAttribute(k_conv_umma<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
        attr[MODE] = true;
    }
    k_conv_umma<MODE><<<grid, THREADS, smem, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("conv launch: ") + cudaGetErrorString(e));
        return CS_ERR_CUDA;
    }
    return CS_OK;
}

// ---- elementwise pieces ----
// master weights f32 [cout][27][cin] -> bf16 [cout_pad][kpad] (K = t * cin_pad + ci);
// flip != 0 builds the input-gradient weights W'[ci][t][co] = W[co][26 - t][ci].
__global__ void k_pack_weights(const float* __restrict__ w, __nv_bfloat16* __restrict__ out, int cin, int cin_pad,
                               int cout, int rows_pad, int kpad, int flip) {
    const int total = rows_pad * kpad;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int row = i / kpad, k = i % kpad;
        float val = 0.0f;
        if (!flip) {
            const int t = k / cin_pad, ci = k % cin_pad;
            if (row < cout && t < 27 && ci < cin) val = w[((size_t)row * 27 + t) * cin + ci];
        } else {  // row = ci, K = t * cout_pad(=cin_pad here) + co
            const int t = k / cin_pad, co = k % cin_pad;
            if (row < cin && t < 27 && co < cout) val = w[((size_t)co * 27 + (26 - t)) * cin + row];
        }
        out[i] = __float2bfloat16(val);
    }
}

// ---- U-Net glue (CUDA cores) ----
#define NN_FOR(i, n) for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (n); \
                          i += (long long)gridDim.x * blockDim.x)

// 2x2x2 average pool of a channels-last tensor; fine grid (gx, gy, gz) even.
__global__ void k_pool_fwd(const __nv_bfloat16* __restrict__ x, __nv_bfloat16* __restrict__ y, Grid3 f, int c) {
    const int hx = f.gx / 2, hy = f.gy / 2, hz = f.gz / 2;
    const long long n = (long long)hx * hy * hz * c;
    NN_FOR(i, n) {
        const int ch = (int)(i % c);
        const long long v = i / c;
        const int x0 = (int)(v % hx) * 2, y0 = (int)((v / hx) % hy) * 2, z0 = (int)(v / ((long long)hx * hy)) * 2;
        float acc = 0.0f;
        for (int dz = 0; dz < 2; ++dz)
            for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx)
                    acc += __bfloat162float(x[((size_t)((z0 + dz) * f.gy + y0 + dy) * f.gx + x0 + dx) * c + ch]);
        y[i] = __float2bfloat16(acc * 0.125f);
    }
}
// gradient of the pool: dx[v] += dy[parent(v)] / 8 (f32)
__global__ void k_pool_bwd(const float* __restrict__ dy, float* __restrict__ dx, Grid3 f, int c) {
    const long long n = (long long)f.voxels() * c;
    NN_FOR(i, n) {
        const int ch = (int)(i % c);
        const long long v = i / c;
        const int x = (int)(v % f.gx), y = (int)((v / f.gx) % f.gy), z = (int)(v / ((long long)f.gx * f.gy));
        const long long pv = ((long long)(z / 2) * (f.gy / 2) + y / 2) * (f.gx / 2) + x / 2;
        dx[i] += dy[pv * c + ch] * 0.125f;
    }
}
// out[v] = [low[parent(v)] (c1 channels), skip[v] (c2 channels)] on the fine grid
__global__ void k_upcat_fwd(const __nv_bfloat16* __restrict__ low, const __nv_bfloat16* __restrict__ skip,
                            __nv_bfloat16* __restrict__ out, Grid3 f, int c1, int c2) {
    // one 16-byte chunk (8 channels) per thread; c1, c2 multiples of 8
    const int q1 = c1 >> 3, q = (c1 + c2) >> 3;
    const long long n = (long long)f.voxels() * q;
    const int hx = f.gx / 2, hy = f.gy / 2;
    NN_FOR(i, n) {
        const int ch = (int)(i % q);
        const long long v = i / q;
        uint4 val;
        if (ch < q1) {
            const int x = (int)(v % f.gx), y = (int)((v / f.gx) % f.gy), z = (int)(v / ((long long)f.gx * f.gy));
            const long long pv = ((long long)(z / 2) * hy + y / 2) * hx + x / 2;
            val = reinterpret_cast<const uint4*>(low)[pv * q1 + ch];
        } else {
            val = reinterpret_cast<const uint4*>(skip)[v * (q - q1) + (ch - q1)];
        }
        reinterpret_cast<uint4*>(out)[i] = val;
    }
}
// gradient of upcat: dlow[p] += sum over its 8 children, dskip[v] += its part (f32)
__global__ void k_upcat_bwd(const float* __restrict__ dout, float* __restrict__ dlow, float* __restrict__ dskip,
                            Grid3 f, int c1, int c2) {
    const int c = c1 + c2;
    const int hx = f.gx / 2, hy = f.gy / 2, hz = f.gz / 2;
    const long long nlow = (long long)hx * hy * hz * c1;
    NN_FOR(i, nlow) {
        const int ch = (int)(i % c1);
        const long long pv = i / c1;
        const int x0 = (int)(pv % hx) * 2, y0 = (int)((pv / hx) % hy) * 2, z0 = (int)(pv / ((long long)hx * hy)) * 2;
        float acc = 0.0f;
        for (int dz = 0; dz < 2; ++dz)
            for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx)
                    acc += dout[((size_t)((z0 + dz) * f.gy + y0 + dy) * f.gx + x0 + dx) * c + ch];
        dlow[i] += acc;
    }
    const long long nskip = (long long)f.voxels() * c2;
    NN_FOR(i, nskip) {
        const long long v = i / c2;
        dskip[i] += dout[v * c + c1 + (int)(i % c2)];
    }
}
// gradient g (f32) masked by the ReLU of the layer output y -> bf16 operand of the
// backward convolutions; accumulates the bias gradient.
__global__ void k_relu_grad(const float* __restrict__ g, const __nv_bfloat16* __restrict__ y,
                            __nv_bfloat16* __restrict__ out, float* __restrict__ db, long long n, int c) {
    NN_FOR(i, n) {
        const float v = __bfloat162float(y[i]) > 0.0f ? g[i] : 0.0f;
        out[i] = __float2bfloat16(v);
        if (db && v != 0.0f) atomicAdd(&db[i % c], v);
    }
}
// 1x1x1 output layer: out[v] = w[c] + sum_k w[k] x[v][k]
__global__ void k_head_fwd(const __nv_bfloat16* __restrict__ x, const float* __restrict__ w, float* __restrict__ out,
                           long long nv, int c) {
    NN_FOR(v, nv) {
        float acc = w[c];
        for (int k = 0; k < c; ++k) acc += w[k] * __bfloat162float(x[v * c + k]);
        out[v] = acc;
    }
}
__global__ void k_head_bwd(const __nv_bfloat16* __restrict__ x, const float* __restrict__ w,
                           const float* __restrict__ dout, float* __restrict__ dx, float* __restrict__ dw, long long nv,
                           int c) {
    NN_FOR(v, nv) {
        const float d = dout[v];
        for (int k = 0; k < c; ++k) dx[v * c + k] = w[k] * d;
        if (d == 0.0f) continue;
        for (int k = 0; k < c; ++k) atomicAdd(&dw[k], __bfloat162float(x[v * c + k]) * d);
        atomicAdd(&dw[c], d);
    }
}
// masked mean squared error: loss[0] += sum m (o - t)^2 / count, dout = 2 m (o - t) / count
__global__ void k_mse(const float* __restrict__ o, const float* __restrict__ t, const float* __restrict__ m,
                      float* __restrict__ dout, float* __restrict__ loss, long long nv, float inv_count) {
    NN_FOR(v, nv) {
        const float e = (o[v] - t[v]) * m[v];
        dout[v] = 2.0f * e * inv_count;
        if (e != 0.0f) atomicAdd(loss, e * e * inv_count);
    }
}
// dW^T [(t, ci)][co] (cout_pad columns) -> master layout gW[co][t][ci]
__global__ void k_wgrad_master(const float* __restrict__ dwt, float* __restrict__ gw, int cin, int cout, int cout_pad) {
    const long long n = (long long)cout * 27 * cin;
    NN_FOR(i, n) {
        const int ci = (int)(i % cin), t = (int)((i / cin) % 27), co = (int)(i / (27LL * cin));
        gw[i] = dwt[((long long)t * cin + ci) * cout_pad + co];
    }
}
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       long long n, float lr, float b1, float b2, float eps, float c1, float c2) {
    NN_FOR(i, n) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}
__global__ void k_axpy(float* __restrict__ y, const float* __restrict__ x, float a, long long n) {
    NN_FOR(i, n) y[i] += a * x[i];
}

}  // namespace nn
}  // namespace cs

using namespace cs::nn;

static cudaStream_t as_stream(void* s) { return (cudaStream_t)s; }

// Tensor map of a channels-last bf16 activation [gz][gy][gx][cin] for the halo kernel's
// TMA loads: dims (cin, gx, gy, gz), box 8 channels x 10 x 18 x 3 voxels, no swizzle,
// zeros outside the tensor.  False when the driver entry point or the encoding fails
// (the caller then uses the copy-gather kernel).
static bool input_tensor_map(CUtensorMap* map, const void* x, int gx, int gy, int gz, int cin) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", (void**)&encode, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            encode = nullptr;
        cudaGetLastError();
    }
    if (!encode || ((uintptr_t)x & 15u) || cin % 8) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)cin, (cuuint64_t)gx, (cuuint64_t)gy, (cuuint64_t)gz};
    const cuuint64_t strides[3] = {(cuuint64_t)cin * 2, (cuuint64_t)gx * cin * 2, (cuuint64_t)gx * gy * cin * 2};
    const cuuint32_t box[4] = {8, HX, HY, HZ};
    const cuuint32_t estride[4] = {1, 1, 1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(x), dims, strides, box, estride,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

extern "C" {

// Y = relu?(conv3x3x3(X, W) + b).  x: bf16 [vox][cin_pad]; w: bf16 [cout_pad][kpad] from
// cs_nn_pack_weights; y: bf16 [vox][cout_pad] (channels >= cout zero), y32: f32
// [vox][cout_pad] or null.  err: device flag set on a wait timeout.
int32_t cs_nn_conv3d(const void* x, const void* w, const float* bias, void* y, float* y32, int32_t gx, int32_t gy,
                     int32_t gz, int32_t cin_pad, int32_t cout_pad, int32_t relu, uint32_t* err, void* stream) {
    if (cin_pad % 8 || cout_pad % 16 || cout_pad > 256 || cout_pad < 16 || gx < 1 || gy < 1 || gz < 1 || !x || !w ||
        !err) {
        cs::set_error("cs_nn_conv3d: channels must be multiples of 8 (input) and 16 (output, <= 256)");
        return CS_ERR_INVALID_ARG;
    }
    ConvArgs a{};
    a.g = Grid3{gx, gy, gz};
    a.x = (const __nv_bfloat16*)x;
    a.w = (const __nv_bfloat16*)w;
    a.bias = bias;
    a.y = (__nv_bfloat16*)y;
    a.y32 = y32;
    a.cin = cin_pad;
    a.cout_pad = cout_pad;
    a.cout_store = cout_pad;
    a.kpad = ((27 * cin_pad + 63) / 64) * 64;
    a.relu = relu;
    a.err = err;
    // dynamic shared memory cap of the halo kernel (its static part, ~1 KB, adds to it)
    constexpr size_t kHaloSmemCap = 220 * 1024;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_conv_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        cudaFuncSetAttribute(k_conv_halo<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kHaloSmemCap);
        cudaFuncSetAttribute(k_conv_halo<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kHaloSmemCap);
        cudaGetLastError();  // a refused attribute shows up as a launch error below
        attr = true;
    }
    const int cp16 = (cin_pad + 15) & ~15;
    const int tiles = ((gx + 7) / 8) * ((gy + 15) / 16) * gz;
    CUtensorMap xmap;
    const bool tma = input_tensor_map(&xmap, x, gx, gy, gz, cin_pad);
    if (tma && halo_smem(cp16, cout_pad, true) <= kHaloSmemCap) {
        k_conv_halo<true><<<dim3(tiles, 1), THREADS, halo_smem(cp16, cout_pad, true), as_stream(stream)>>>(a, xmap);
    } else if (tma && halo_smem(cp16, cout_pad, false) <= kHaloSmemCap) {
        k_conv_halo<false><<<dim3(tiles, 1), THREADS, halo_smem(cp16, cout_pad, false), as_stream(stream)>>>(a, xmap);
    } else {
        const int tiles = (a.g.voxels() + BM - 1) / BM;
        const size_t smem = (size_t)NBUF * (BM + cout_pad) * BKC * 16;
        k_conv_fwd<<<dim3(tiles, 1), THREADS, smem, as_stream(stream)>>>(a);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        cs::set_error(std::string("conv launch: ") + cudaGetErrorString(e));
        return CS_ERR_CUDA;
    }
    return CS_OK;
}

// dWt[t * cin_pad + ci][co] += sum_v X[v + off_t][ci] * dY[v][co]  (f32, accumulated).
int32_t cs_nn_conv3d_wgrad(const void* x, const void* dy, float* dwt, int32_t gx, int32_t gy, int32_t gz,
                           int32_t cin_pad, int32_t cout_pad, int32_t splits, uint32_t* err, void* stream) {
    if (cin_pad % 8 || cout_pad % 16 || cout_pad > 256 || cout_pad < 16 || splits < 1 || !x || !dy || !dwt || !err) {
        cs::set_error("cs_nn_conv3d_wgrad: bad arguments");
        return CS_ERR_INVALID_ARG;
    }
    ConvArgs a{};
    a.g = Grid3{gx, gy, gz};
    a.x = (const __nv_bfloat16*)x;
    a.dy = (const __nv_bfloat16*)dy;
    a.dwt = dwt;
    a.cin = cin_pad;
    a.cout_pad = cout_pad;
    a.m_rows = 27 * cin_pad;
    const int nvox = a.g.voxels();
    int per = (nvox + splits - 1) / splits;
    per = ((per + 63) / 64) * 64;
    a.k_per_split = per;
    a.err = err;
    const int tiles = (a.m_rows + BM - 1) / BM;
    const int ns = (nvox + per - 1) / per;
    return launch<1>(a, dim3(tiles, ns), as_stream(stream));
}

// Pack f32 master weights [cout][27][cin] into the bf16 GEMM layout; flip = 1 gives the
// input-gradient operator (rows = cin, K = t * cout_pad + co).
int32_t cs_nn_pack_weights(const float* w, void* out, int32_t cin, int32_t cin_pad, int32_t cout, int32_t cout_pad,
                           int32_t flip, void* stream) {
    if (!w || !out) {
        cs::set_error("cs_nn_pack_weights: null pointer");
        return CS_ERR_INVALID_ARG;
    }
    const int rows = flip ? ((cin + 15) / 16) * 16 : cout_pad;
    const int kin = flip ? cout_pad : cin_pad;
    const int kpad = ((27 * kin + 63) / 64) * 64;
    k_pack_weights<<<256, 256, 0, as_stream(stream)>>>(w, (__nv_bfloat16*)out, cin, kin, cout, rows, kpad, flip);
    return cudaGetLastError() == cudaSuccess ? CS_OK : CS_ERR_CUDA;
}


static int nn_check(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        cs::set_error(std::string(what) + ": " + cudaGetErrorString(e));
        return CS_ERR_CUDA;
    }
    return CS_OK;
}
static int nn_blocks(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 32)); }

int32_t cs_nn_pool(const void* x, void* y, const float* dy, float* dx, int32_t gx, int32_t gy, int32_t gz, int32_t c,
                   int32_t backward, void* stream) {
    const Grid3 f{gx, gy, gz};
    if (gx % 2 || gy % 2 || gz % 2 || c < 1) {
        cs::set_error("cs_nn_pool: grid dims must be even");
        return CS_ERR_INVALID_ARG;
    }
    const long long n = (long long)f.voxels() * c;
    if (!backward)
        k_pool_fwd<<<nn_blocks(n / 8), 256, 0, as_stream(stream)>>>((const __nv_bfloat16*)x, (__nv_bfloat16*)y, f, c);
    else
        k_pool_bwd<<<nn_blocks(n), 256, 0, as_stream(stream)>>>(dy, dx, f, c);
    return nn_check("cs_nn_pool");
}
int32_t cs_nn_upcat(const void* low, const void* skip, void* out, const float* dout, float* dlow, float* dskip,
                    int32_t gx, int32_t gy, int32_t gz, int32_t c1, int32_t c2, int32_t backward, void* stream) {
    const Grid3 f{gx, gy, gz};
    if (gx % 2 || gy % 2 || gz % 2 || c1 % 8 || c2 % 8) {
        cs::set_error("cs_nn_upcat: grid dims must be even and channel counts multiples of 8");
        return CS_ERR_INVALID_ARG;
    }
    const long long n = (long long)f.voxels() * (c1 + c2);
    if (!backward)
        k_upcat_fwd<<<nn_blocks(n / 8), 256, 0, as_stream(stream)>>>(
            (const __nv_bfloat16*)low, (const __nv_bfloat16*)skip, (__nv_bfloat16*)out, f, c1, c2);
    else
        k_upcat_bwd<<<nn_blocks(n), 256, 0, as_stream(stream)>>>(dout, dlow, dskip, f, c1, c2);
    return nn_check("cs_nn_upcat");
}
int32_t cs_nn_relu_grad(const float* g, const void* y, void* out, float* db, int64_t n, int32_t c, void* stream) {
    k_relu_grad<<<nn_blocks(n), 256, 0, as_stream(stream)>>>(g, (const __nv_bfloat16*)y, (__nv_bfloat16*)out, db, n, c);
    return nn_check("cs_nn_relu_grad");
}
int32_t cs_nn_head(const void* x, const float* w, float* out, const float* dout, float* dx, float* dw, int64_t nv,
                   int32_t c, int32_t backward, void* stream) {
    if (!backward)
        k_head_fwd<<<nn_blocks(nv), 256, 0, as_stream(stream)>>>((const __nv_bfloat16*)x, w, out, nv, c);
    else
        k_head_bwd<<<nn_blocks(nv), 256, 0, as_stream(stream)>>>((const __nv_bfloat16*)x, w, dout, dx, dw, nv, c);
    return nn_check("cs_nn_head");
}
int32_t cs_nn_mse(const float* o, const float* t, const float* m, float* dout, float* loss, int64_t nv,
                  float inv_count, void* stream) {
    k_mse<<<nn_blocks(nv), 256, 0, as_stream(stream)>>>(o, t, m, dout, loss, nv, inv_count);
    return nn_check("cs_nn_mse");
}
int32_t cs_nn_wgrad_master(const float* dwt, float* gw, int32_t cin, int32_t cout, int32_t cout_pad, void* stream) {
    k_wgrad_master<<<nn_blocks((long long)cout * 27 * cin), 256, 0, as_stream(stream)>>>(dwt, gw, cin, cout, cout_pad);
    return nn_check("cs_nn_wgrad_master");
}
int32_t cs_nn_adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2, float eps,
                   int32_t step, void* stream) {
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_adam<<<nn_blocks(n), 256, 0, as_stream(stream)>>>(p, g, m, v, n, lr, b1, b2, eps, c1, c2);
    return nn_check("cs_nn_adam");
}
int32_t cs_nn_axpy(float* y, const float* x, float a, int64_t n, void* stream) {
    k_axpy<<<nn_blocks(n), 256, 0, as_stream(stream)>>>(y, x, a, n);
    return nn_check("cs_nn_axpy");
}

}  // extern "C"
