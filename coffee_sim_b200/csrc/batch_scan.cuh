// batch_scan.cuh — exclusive prefix sums of many instances' arrays in three launches.
//
// The batched ensemble scans two arrays per instance each substep: the P2G tile counts
// (into tile starts) and the cluster solve's Morton fluid flags (into fluid numbers).
// One CUB call per instance and array costs two launches each; here every instance's
// array is cut into chunks of BS_CHUNK elements and
//   k_bs_reduce  sums each chunk             (grid: chunks x instances)
//   k_bs_offsets scans the chunk sums        (grid: instances)
//   k_bs_down    scans each chunk and adds its offset (grid: chunks x instances).
// Integer sums do not depend on the order they are taken in, so the results equal a
// sequential scan (and CUB's) exactly.
#pragma once
#include "cs_device.cuh"

namespace cs {

constexpr int BS_THREADS = 256;
constexpr int BS_ITEMS = 16;
constexpr int BS_CHUNK = BS_THREADS * BS_ITEMS;

// which arrays of a context: uint32_t = tile_count -> tile_start (P2G),
// unsigned long long = sb.flags -> sb.scan (cluster solve)
template <class T>
__device__ __forceinline__ const T* bs_src(const Ctx& c);
template <>
__device__ __forceinline__ const uint32_t* bs_src<uint32_t>(const Ctx& c) {
    return c.tile_count;
}
template <>
__device__ __forceinline__ const unsigned long long* bs_src<unsigned long long>(const Ctx& c) {
    return c.sb.flags;
}
template <class T>
__device__ __forceinline__ T* bs_dst(const Ctx& c);
template <>
__device__ __forceinline__ uint32_t* bs_dst<uint32_t>(const Ctx& c) {
    return c.tile_start;
}
template <>
__device__ __forceinline__ unsigned long long* bs_dst<unsigned long long>(const Ctx& c) {
    return c.sb.scan;
}

// Exclusive scan of one value per thread across the block; returns the block total.
template <class T>
__device__ __forceinline__ T bs_block_exclusive(T v, T& excl) {
    __shared__ T warp_sum[BS_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) warp_sum[warp] = inc;
    __syncthreads();
    T before = 0, total = 0;
#pragma unroll
    for (int w = 0; w < BS_THREADS / 32; ++w) {
        const T s = warp_sum[w];
        if (w < warp) before += s;
        total += s;
    }
    excl = before + inc - v;
    __syncthreads();
    return total;
}

template <class T>
__global__ void __launch_bounds__(BS_THREADS) k_bs_reduce(const Ctx* __restrict__ cp, uint32_t len,
                                                          T* __restrict__ partial, uint32_t max_chunks) {
    const Ctx& c = cp[blockIdx.y];
    const T* src = bs_src<T>(c);
    const uint32_t base = blockIdx.x * (uint32_t)BS_CHUNK;
    T s = 0;
    for (uint32_t k = threadIdx.x; k < (uint32_t)BS_CHUNK; k += BS_THREADS) {
        const uint32_t i = base + k;
        if (i < len) s += src[i];
    }
    T excl;
    const T total = bs_block_exclusive<T>(s, excl);
    if (threadIdx.x == 0) partial[(size_t)blockIdx.y * max_chunks + blockIdx.x] = total;
}

template <class T>
__global__ void k_bs_offsets(T* __restrict__ partial, uint32_t chunks, uint32_t max_chunks) {
    if (threadIdx.x != 0) return;
    T* p = partial + (size_t)blockIdx.x * max_chunks;
    T run = 0;
    for (uint32_t k = 0; k < chunks; ++k) {
        const T v = p[k];
        p[k] = run;
        run += v;
    }
}

template <class T>
__global__ void __launch_bounds__(BS_THREADS) k_bs_down(const Ctx* __restrict__ cp, uint32_t len,
                                                        const T* __restrict__ partial, uint32_t max_chunks) {
    __shared__ T tile[BS_CHUNK];
    const Ctx& c = cp[blockIdx.y];
    const T* src = bs_src<T>(c);
    T* dst = bs_dst<T>(c);
    const uint32_t base = blockIdx.x * (uint32_t)BS_CHUNK;
    for (uint32_t k = threadIdx.x; k < (uint32_t)BS_CHUNK; k += BS_THREADS) {
        const uint32_t i = base + k;
        tile[k] = i < len ? src[i] : (T)0;
    }
    __syncthreads();
    T v[BS_ITEMS];
    T s = 0;
#pragma unroll
    for (int j = 0; j < BS_ITEMS; ++j) {
        v[j] = tile[threadIdx.x * BS_ITEMS + j];
        s += v[j];
    }
    T excl;
    bs_block_exclusive<T>(s, excl);
    T run = excl + partial[(size_t)blockIdx.y * max_chunks + blockIdx.x];
#pragma unroll
    for (int j = 0; j < BS_ITEMS; ++j) {
        tile[threadIdx.x * BS_ITEMS + j] = run;
        run += v[j];
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < (uint32_t)BS_CHUNK; k += BS_THREADS) {
        const uint32_t i = base + k;
        if (i < len) dst[i] = tile[k];
    }
}

// The three launches for `n` instances' arrays of `len` elements; partial holds
// n x ceil(len / BS_CHUNK) chunk sums.
template <class T>
inline void bs_launch(const Ctx* d_ctx, uint32_t n, uint32_t len, T* partial, cudaStream_t stream) {
    const uint32_t chunks = (len + BS_CHUNK - 1) / BS_CHUNK;
    k_bs_reduce<T><<<dim3(chunks, n), BS_THREADS, 0, stream>>>(d_ctx, len, partial, chunks);
    k_bs_offsets<T><<<dim3(n), 32, 0, stream>>>(partial, chunks, chunks);
    k_bs_down<T><<<dim3(chunks, n), BS_THREADS, 0, stream>>>(d_ctx, len, partial, chunks);
}

}  // namespace cs
