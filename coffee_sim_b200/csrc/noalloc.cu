// noalloc.cu — the pressure solve on caller-owned device arrays, without allocating.
//
// Who needs this: hosts that own every byte of device memory themselves and may not
// call cudaMalloc once they are running — a renderer or game engine that reserves
// its GPU budget at start-up, or a real-time frame loop where cudaMalloc's latency
// and implicit synchronisation are not acceptable.  Such a caller cannot create a
// CsSim (cs_create allocates), but can hand this entry point the fields it already
// keeps on the device and get the solved pressure back in place.
//
// Every scratch buffer of the solve (Morton flags and their scan, neighbour
// references, chunk tables, CUB scan storage, the solver context and result, the
// clamp counters) lives in one file-scope __device__ array sized for grids of at
// most 64 cells per side.  Every GPU that loads this library keeps that array
// (about 7.6 MB) until the process exits.  Calls share it and it keeps the previous
// call's contents: each call rewrites or clears everything it reads, and calls that
// overlap on the GPU race with each other.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "cs_device.cuh"
#include "solver_launch.h"

namespace {

constexpr uint32_t kMaxSide = 64;                       // cells per grid side
constexpr size_t kMaxCodes = (size_t)kMaxSide * kMaxSide * kMaxSide;
constexpr size_t kCubBytes = 256 * 1024;
constexpr size_t kOffCtx = 0;
constexpr size_t kOffMetrics = kOffCtx + cs::sc_align(sizeof(cs::Ctx));
constexpr size_t kOffSolver = kOffMetrics + 256;
constexpr cs::ScScratch kSolver = cs::sc_scratch_layout(kMaxCodes, kMaxCodes, kCubBytes);
constexpr size_t kScratchBytes = kOffSolver + kSolver.total;

static __device__ __align__(256) unsigned char g_solve_scratch[kScratchBytes];

struct DeviceSlot {
    bool ready = false;
    unsigned char* base = nullptr;  // device address of g_solve_scratch on this device
    int ranks = 0;
    int sms = 0;
};
constexpr int kMaxDevices = 64;
DeviceSlot g_slots[kMaxDevices];
std::mutex g_setup;

// Once per device, with that device current: the array's device address (the host
// symbol is only a stand-in), the cluster size and the SM count.
int setup_device(int dev, DeviceSlot** out) {
    if (dev < 0 || dev >= kMaxDevices) {
        cs::set_error("device ordinal out of range for the allocation-free solve");
        return CS_ERR_INVALID_ARG;
    }
    std::lock_guard<std::mutex> lock(g_setup);
    DeviceSlot& s = g_slots[dev];
    if (!s.ready) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_solve_scratch);
        if (e != cudaSuccess) {
            cs::set_error(std::string("cudaGetSymbolAddress(g_solve_scratch): ") + cudaGetErrorString(e));
            return CS_ERR_CUDA;
        }
        if (cudaDeviceGetAttribute(&s.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
            cs::set_error("cudaDeviceGetAttribute(multiProcessorCount) failed");
            return CS_ERR_CUDA;
        }
        s.ranks = cs::sc_max_cluster_ranks();
        if (s.ranks == 0) {
            cs::set_error("this device cannot launch the solver's thread-block cluster");
            return CS_ERR_UNSUPPORTED;
        }
        if (cs::sc_scan_temp_bytes((uint32_t)kMaxCodes) > kCubBytes) {
            cs::set_error("scan storage does not fit the reserved scratch");
            return CS_ERR_CAPACITY;
        }
        s.base = (unsigned char*)ptr;
        s.ready = true;
    }
    *out = &s;
    return CS_OK;
}

}  // namespace

extern "C" int32_t cs_pressure_solve_noalloc(uint32_t gx, uint32_t gy, uint32_t gz, float dx, float dt, float omega,
                                             float residual_tol, uint32_t max_pairs, uint32_t check_every,
                                             const int32_t* kind, const float* fill, const float* div, float* p_hi,
                                             float* p_lo, void* stream, uint32_t* pairs_out, double* residual_out) {
    if (gx == 0 || gy == 0 || gz == 0 || gx > kMaxSide || gy > kMaxSide || gz > kMaxSide) {
        cs::set_error("grid exceeds the allocation-free solve's scratch: at most 64 cells per side");
        return CS_ERR_CAPACITY;
    }
    if (!kind || !fill || !div || !p_hi || !p_lo || !(dx > 0.0f) || !(dt > 0.0f) || !(omega > 0.0f) ||
        !(omega < 2.0f)) {
        cs::set_error("invalid argument to cs_pressure_solve_noalloc");
        return CS_ERR_INVALID_ARG;
    }
    cudaStream_t st = (cudaStream_t)stream;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
        cs::set_error("cs_pressure_solve_noalloc synchronises its stream and cannot run on a capturing stream");
        return CS_ERR_INVALID_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cs::set_error("no CUDA device is current");
        return CS_ERR_NO_DEVICE;
    }
    DeviceSlot* slot = nullptr;
    int rc = setup_device(dev, &slot);
    if (rc) return rc;
    unsigned char* base = slot->base;

    uint32_t side = 1;
    while (side < gx || side < gy || side < gz) side <<= 1;
    const uint32_t codes = side * side * side;
    const uint32_t cells = gx * gy * gz;

    cs::Ctx ctx;
    std::memset(&ctx, 0, sizeof(ctx));
    cs::Params& u = ctx.u;
    u.gx = gx;
    u.gy = gy;
    u.gz = gz;
    u.cells = cells;
    u.dx = dx;
    u.inv_dx = 1.0f / dx;
    u.dt = dt;
    u.omega = omega;
    u.p_clamp = cs::FP_VALUE_LIMIT - 1.0f;
    u.p_limit = 3.0e38f;  // FP32 storage: no fixed-point range to respect
    u.fixed_point = 0;
    // the solver reads the cell kind through ctx.kind and nothing through ctx.lanes
    ctx.lanes = nullptr;
    ctx.kind = kind;
    ctx.fill = const_cast<float*>(fill);
    ctx.divf = const_cast<float*>(div);
    ctx.pf = p_hi;
    ctx.plo = p_lo;
    ctx.metrics = reinterpret_cast<uint32_t*>(base + kOffMetrics);

    const cs::ScBuffers sb = cs::sc_buffers_at(base + kOffSolver, kSolver, kCubBytes);
    ctx.sb = sb;
    const cs::Ctx* dctx = reinterpret_cast<const cs::Ctx*>(base + kOffCtx);

    cudaError_t e = cudaMemcpyAsync(base + kOffCtx, &ctx, sizeof(ctx), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(base + kOffMetrics, 0, 256, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(sb.result, 0, sizeof(cs::ScResult), st);
    if (e != cudaSuccess) {
        cs::set_error(std::string("cs_pressure_solve_noalloc: ") + cudaGetErrorString(e));
        return CS_ERR_CUDA;
    }
    if ((rc = cs::sc_launch_prep(dctx, &sb, codes, slot->ranks, 1, st, slot->sms))) return rc;
    // Colours are first separated by point-to-point waits; if one of those bounded
    // waits runs out (status 3) the solve is run again from the pressure reached so far
    // with cluster barriers, which have no time limit to run out, as the engine does.
    cs::ScResult res;
    for (uint32_t p2p = 1;; p2p = 0) {
        if ((rc = cs::sc_launch_cluster(dctx, slot->ranks, 1, residual_tol, max_pairs, check_every, st, p2p)))
            return rc;
        e = cudaMemcpyAsync(&res, sb.result, sizeof(res), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            cs::set_error(std::string("cs_pressure_solve_noalloc: ") + cudaGetErrorString(e));
            return CS_ERR_CUDA;
        }
        if (res.status != 3 || p2p == 0) break;
        e = cudaMemsetAsync(sb.result, 0, sizeof(cs::ScResult), st);
        if (e != cudaSuccess) {
            cs::set_error(std::string("cs_pressure_solve_noalloc: ") + cudaGetErrorString(e));
            return CS_ERR_CUDA;
        }
    }
    if (res.status == 2) {
        cs::set_error("the fluid cells exceed what the solver's thread-block cluster holds "
                      "(16 x 4095 cells, 4095 halo cells per CTA)");
        return CS_ERR_CAPACITY;
    }
    if (res.status == 3) {
        cs::set_error("the cluster solve gave up waiting for a neighbouring CTA; p_hi/p_lo are not solved");
        return CS_ERR_TIMEOUT;
    }
    if (res.status != 1) {
        cs::set_error("the cluster solve did not complete");
        return CS_ERR_CUDA;
    }
    if (pairs_out) *pairs_out = res.sweeps;
    if (residual_out) *residual_out = res.r1;
    return CS_OK;
}
