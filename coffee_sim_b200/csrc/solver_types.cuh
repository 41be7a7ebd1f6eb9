// solver_types.cuh — plain types shared by the cluster-resident pressure solve
// (solver_cluster.cuh) and the callers that launch it.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cmath>
#include <vector_types.h>

namespace cs {

constexpr int SC_CAP = 4095;           // owned cells per CTA (12-bit local index, 0xFFFF reserved)
constexpr int SC_MAX_RANKS = 16;
constexpr uint16_t SC_NONE = 0xFFFF;
constexpr int SC_THREADS = 1024;
// Slots of a CTA's correction array: owned cells [0, SC_CAP), halo copies of other
// CTAs' cells [SC_HALO0, SC_HALO0 + SC_HALO), and one slot that always holds zero.
constexpr int SC_HALO0 = 4096;
constexpr int SC_HALO = 4095;
constexpr uint16_t SC_DUMMY = 8191;
constexpr int SC_SLOTS = 8192;
constexpr int SC_SEND = 2048;          // halo updates a CTA sends after one colour

// per-CTA shared memory
struct ScLayout {
    static constexpr size_t dval = 0;                                    // float correction x SC_SLOTS
    static constexpr size_t fcode = dval + sizeof(float) * SC_SLOTS;     // float fill code x SC_SLOTS
    static constexpr size_t g = fcode + sizeof(float) * SC_SLOTS;        // float residual
    static constexpr size_t invW = g + sizeof(float) * 4096;             // float 1/W (0: no faces)
    static constexpr size_t ph = invW + sizeof(float) * 4096;            // float
    static constexpr size_t pl = ph + sizeof(float) * 4096;              // float
    static constexpr size_t b = pl + sizeof(float) * 4096;               // float dx^2 rhs
    static constexpr size_t ref = b + sizeof(float) * 4096;              // uint32 [3][4096]: face pairs
    static constexpr size_t snd = ref + sizeof(uint32_t) * 3 * 4096;     // uint32 [2][SC_SEND]
    static constexpr size_t flags = snd + sizeof(uint32_t) * 2 * SC_SEND;  // uint8 x 4096
    static constexpr size_t part = flags + 4096;                         // double[2 slots][2][SC_MAX_RANKS]
    static constexpr size_t red = part + sizeof(double) * 4 * SC_MAX_RANKS;  // double[2][32]
    static constexpr size_t mbar = red + sizeof(double) * 64;               // uint64 mbarrier per colour
    static constexpr size_t abortf = mbar + sizeof(unsigned long long) * 2;  // uint32[2 slots][SC_MAX_RANKS]
    static constexpr size_t bytes = abortf + sizeof(uint32_t) * 2 * SC_MAX_RANKS;
};
static_assert(ScLayout::bytes <= 232448, "cluster solve state exceeds the 227 KB shared-memory limit");
// A face reference is a 13-bit slot index; bit 15 of the first word marks a cell
// whose fluid faces all have weight 1.
constexpr uint32_t SC_SLOT_MASK = 0x1fffu, SC_REF_UNIT = 0x8000u;
// flags byte: bits 0-2 air faces, bit 5 held as halo by another CTA, bit 6 all
// fluid-face weights are 1, bit 7 no faces
constexpr uint8_t SC_SENT = 0x20, SC_UNIT = 0x40, SC_EMPTY = 0x80;


// Solver bookkeeping written by the prep kernels and read by the cluster kernel.
struct ScInfo {
    uint32_t n_fluid, n_red, chunk, overflow;
    uint32_t red_before[SC_MAX_RANKS + 1];
};
// Pairs to run before the next residual check of the refinement loop.  The check that
// just gave r_new (after k_last pairs that took the residual from r_old) predicts the
// pairs still needed from the decay over that interval,
// ceil(k_last * log(tol / r_new) / log(r_new / r_old)), and the next check comes then:
// at least 2 pairs, at most ce (the configured check interval).  Without a measured
// decay (first interval, or no decrease) the interval is ce.
__host__ __device__ inline uint32_t sc_next_interval(double r_new, double r_old, uint32_t k_last, double tol,
                                                     uint32_t ce) {
    if (!(r_old > 0.0) || !(r_new > tol) || !(r_new < r_old) || k_last == 0) return ce;
    const double n = ceil((double)k_last * log(tol / r_new) / log(r_new / r_old));
    if (!(n < (double)ce)) return ce;
    return n < 2.0 ? 2u : (uint32_t)n;
}

// Result of one solve.
struct ScResult {
    uint32_t sweeps, evals, status, pad;
    double r0, r1;
};
// Running totals of the solves of replayed substeps (graph mode reads them lazily):
// `failed` counts solves whose fluid did not fit (status 2), `timeouts` solves whose
// bounded waits ran out (status 3).
struct ScTotals {
    unsigned long long sweeps, evals, failed, runs, timeouts;
    ScResult last;
};
// counters: halo size per rank, send-list length per (rank, colour), then the halo
// values each rank receives per colour (one per halo slot of a cell of that colour)
constexpr int SC_COUNTS = SC_MAX_RANKS * 5;
constexpr int SC_RECV0 = SC_MAX_RANKS * 3;

struct ScBuffers {
    unsigned long long* flags;   // Morton codes: fluid | red << 32
    unsigned long long* scan;    // exclusive scan of flags
    uint16_t* ref_of_cell;       // per grid cell: rank << 12 | local, SC_NONE if not fluid
    uint32_t* cell_of;           // [rank][4096] grid cell of each owned slot
    uint16_t* slot_ref;          // [rank][3 face pairs][4096][2] neighbour slot per face
    float4* slot_coef;           // [rank][4096] (1/W, fill code, dx^2 rhs, flags bits)
    float* halo_fill;            // [rank][SC_HALO] fill code of each halo slot
    uint32_t* send;              // [rank][colour][SC_SEND] src | dest rank << 12 | halo slot << 16
    uint32_t* counts;            // SC_COUNTS
    ScInfo* info;
    ScResult* result;
    void* cub_temp;              // CUB scan storage (host-side launches)
    size_t cub_bytes;
};

// Grid-wide solve (solver_grid.cuh): row segments of fluid cells, units of 64 cells.
struct GsDesc;
struct GsBuffers {
    uint32_t* row_units;  // [rows + 1] units of each row (last entry 0)
    uint32_t* row_start;  // [rows + 1] exclusive scan of row_units; row_start[rows] = units
    uint32_t* row_xlo;    // [rows] first x of each row's segment (multiple of 64)
    GsDesc* desc;         // [max_units] slot offsets of each unit and of its neighbour rows
    int* rec;             // [max_units][2][8] per-colour index words of the solve (when they do not
                          // fit in shared memory)
    float2* cf;           // [slots] 1 / (sum of the face weights), face flags
    float2* dfc;          // [slots] correction of the refinement cycle, fill code (2: bed-coupled)
    float* g;             // [slots] FP64 residual of the cycle, rounded to fp32
    float* b;             // [slots] dx^2 rhs
    float2* p;            // [slots] pressure hi, lo
    double* part;         // [2 * CTAs] per-CTA partial norms
    uint32_t* sync;       // grid barrier: arrivals, generation, abort
    ScResult* result;
    void* cub_temp;
    size_t cub_bytes;
};

// Byte offsets of every solver scratch buffer inside one allocation.
struct ScScratch {
    size_t flags, scan, ref_of_cell, cell_of, slot_ref, slot_coef, halo_fill, send, counts, info, result, cub, total;
};
constexpr size_t sc_align(size_t n) { return (n + 255) & ~size_t(255); }
constexpr ScScratch sc_scratch_layout(size_t cells, size_t codes, size_t cub_bytes) {
    ScScratch s{};
    s.flags = 0;
    s.scan = s.flags + sc_align(codes * sizeof(unsigned long long));
    s.ref_of_cell = s.scan + sc_align(codes * sizeof(unsigned long long));
    s.cell_of = s.ref_of_cell + sc_align(cells * sizeof(uint16_t));
    s.slot_ref = s.cell_of + sc_align((size_t)SC_MAX_RANKS * 4096 * sizeof(uint32_t));
    s.slot_coef = s.slot_ref + sc_align((size_t)SC_MAX_RANKS * 3 * 4096 * 2 * sizeof(uint16_t));
    s.halo_fill = s.slot_coef + sc_align((size_t)SC_MAX_RANKS * 4096 * sizeof(float4));
    s.send = s.halo_fill + sc_align((size_t)SC_MAX_RANKS * SC_HALO * sizeof(float));
    s.counts = s.send + sc_align((size_t)SC_MAX_RANKS * 2 * SC_SEND * sizeof(uint32_t));
    s.info = s.counts + sc_align(SC_COUNTS * sizeof(uint32_t));
    s.result = s.info + sc_align(sizeof(ScInfo));
    s.cub = s.result + sc_align(sizeof(ScResult));
    s.total = s.cub + sc_align(cub_bytes);
    return s;
}
inline ScBuffers sc_buffers_at(unsigned char* base, const ScScratch& s, size_t cub_bytes) {
    ScBuffers b;
    b.flags = reinterpret_cast<unsigned long long*>(base + s.flags);
    b.scan = reinterpret_cast<unsigned long long*>(base + s.scan);
    b.ref_of_cell = reinterpret_cast<uint16_t*>(base + s.ref_of_cell);
    b.cell_of = reinterpret_cast<uint32_t*>(base + s.cell_of);
    b.slot_ref = reinterpret_cast<uint16_t*>(base + s.slot_ref);
    b.slot_coef = reinterpret_cast<float4*>(base + s.slot_coef);
    b.halo_fill = reinterpret_cast<float*>(base + s.halo_fill);
    b.send = reinterpret_cast<uint32_t*>(base + s.send);
    b.counts = reinterpret_cast<uint32_t*>(base + s.counts);
    b.info = reinterpret_cast<ScInfo*>(base + s.info);
    b.result = reinterpret_cast<ScResult*>(base + s.result);
    b.cub_temp = base + s.cub;
    b.cub_bytes = cub_bytes;
    return b;
}

}  // namespace cs
