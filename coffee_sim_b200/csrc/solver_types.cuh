// solver_types.cuh — plain types shared by the cluster-resident pressure solve
// (solver_cluster.cuh) and the callers that launch it.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector_types.h>

namespace cs {

constexpr int SC_CAP = 4095;           // cells per CTA (12-bit local index, 0xFFFF reserved)
constexpr int SC_MAX_RANKS = 16;
constexpr uint16_t SC_NONE = 0xFFFF;
constexpr int SC_THREADS = 1024;

// per-CTA shared memory: SoA arrays of SC_CAP entries
struct ScLayout {
    static constexpr size_t dfill = 0;                                  // float2 (d, fill code)
    static constexpr size_t g = dfill + sizeof(float2) * SC_CAP;        // float residual
    static constexpr size_t invW = g + sizeof(float) * SC_CAP;          // float 1/W (0: no faces)
    static constexpr size_t ph = invW + sizeof(float) * SC_CAP;         // float
    static constexpr size_t pl = ph + sizeof(float) * SC_CAP;           // float
    static constexpr size_t b = pl + sizeof(float) * SC_CAP;            // float dx^2 rhs
    static constexpr size_t ref = b + sizeof(float) * SC_CAP;           // uint16 x 6, cell-major
    static constexpr size_t flags = ref + sizeof(uint16_t) * 6 * SC_CAP;  // uint8
    static constexpr size_t part = (flags + SC_CAP + 15) & ~size_t(15);   // double[2 slots][2][SC_MAX_RANKS]
    static constexpr size_t red = part + sizeof(double) * 4 * SC_MAX_RANKS;  // double[2][32]
    static constexpr size_t bytes = red + sizeof(double) * 64;
};
// flags byte: bits 0-2 air faces, bit 6 all fluid-face weights are 1, bit 7 no faces
constexpr uint8_t SC_UNIT = 0x40, SC_EMPTY = 0x80;


// Solver bookkeeping written by the prep kernels and read by the cluster kernel.
struct ScInfo {
    uint32_t n_fluid, n_red, chunk, overflow;
    uint32_t red_before[SC_MAX_RANKS + 1];
};
// Result of one solve.
struct ScResult {
    uint32_t sweeps, evals, status, pad;
    double r0, r1;
};

struct ScBuffers {
    unsigned long long* flags;   // Morton codes: fluid | red << 32
    unsigned long long* scan;    // exclusive scan of flags
    uint16_t* ref_of_cell;       // cells
    uint32_t* cell_of;           // SC_MAX_RANKS * 4096
    ScInfo* info;
    ScResult* result;
};


}  // namespace cs
