// solver_launch.h — host entry points of the cluster-resident pressure solve, shared
// by the engine and the allocation-free entry point (definitions in engine.cu).
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "cs_device.cuh"
#include "solver_types.cuh"

namespace cs {

constexpr uint32_t kScPrepLaunches = 5;  // own kernels of sc_launch_prep per call (CUB's not counted)

void set_error(const std::string& msg);
int sc_max_cluster_ranks();
size_t sc_scan_temp_bytes(uint32_t codes);
// d_ctx: device array of `instances` contexts (each carrying its ScBuffers); sb: the
// same ScBuffers on the host, for the CUB scans launched from the host.  With
// bs_partial (instances x bs_max_chunks(codes) 64-bit words of device scratch) the fluid
// flags of all instances are scanned by the batched scan kernels instead.
int sc_launch_prep(const Ctx* d_ctx, const ScBuffers* sb, uint32_t codes, int ranks, uint32_t instances,
                   cudaStream_t stream, int sms, void* bs_partial = nullptr);
// Chunks of the batched scan for arrays of `len` elements.
inline uint32_t bs_max_chunks(size_t len) { return (uint32_t)((len + 4095) / 4096); }
// p2p: 1 separates the colours with point-to-point mbarrier waits, 0 with cluster
// barriers (rbgs_kernel = 3).
int sc_launch_cluster(const Ctx* d_ctx, int ranks, uint32_t instances, float tol, uint32_t max_pairs,
                      uint32_t check_every, cudaStream_t stream, uint32_t p2p);

// Grid-wide solve (solver_grid.cuh) of one system.  Grids of at most kClusterMaxCells
// cells are solved on a thread-block cluster by default, larger ones with this solve.
constexpr size_t kClusterMaxCells = (size_t)1 << 18;
constexpr uint32_t kGsPrepLaunches = 2;  // own kernels of gs_launch_prep per call
// CTAs of the cooperative launch on the current device (0 if it cannot launch).
int gs_blocks(int* ctas);
int gs_launch_prep(const Ctx* d_ctx, const GsBuffers* gb, uint32_t rows, cudaStream_t stream, int sms);
int gs_launch_solve(const Ctx* d_ctx, int ctas, float tol, uint32_t max_pairs, uint32_t check_every,
                    cudaStream_t stream);

}  // namespace cs
