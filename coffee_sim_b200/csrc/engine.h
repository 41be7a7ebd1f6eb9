// engine.h — one simulation on one GPU: device buffers, the substep schedule, and
// host-side state (the fields of MpmSim3D, mod.rs:179-193).
#pragma once
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "cs_device.cuh"
#include "host_scene.h"
#include "solver_launch.h"

namespace cs {

struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
};

class Ensemble;

class Engine {
    friend class Ensemble;

public:
    explicit Engine(const CsSettings& s);
    ~Engine();
    int init();           // allocate, generate SDF/mask, seed the bed
    int reset();          // mod.rs:432-446
    int step_frame(float dt);
    int substep(float sub_dt, uint32_t passes);
    int sync();

    // readback / upload (reference layouts)
    int read_particles(int what, uint32_t first, uint32_t count, float* out);
    int write_particles(int what, uint32_t first, uint32_t count, const float* in);
    int read_lanes(int32_t* out);
    int read_lanes64(int64_t* out);
    int read_gvel(float* out);
    int read_pressure(float* out);
    int read_kind(int32_t* out);
    int read_solver_inputs(float* fill, float* div);
    int read_lookup(int32_t* out);
    int read_delta(int32_t* out);
    int read_sdf(float* out);
    int read_class(uint8_t* out);
    int metrics(CsMetrics* out);
    int metrics_request();
    int metrics_wait(CsMetrics* out);
    int add_water_block(const float lo[3], const float hi[3], uint32_t per_axis, float jitter, uint32_t seed,
                        uint32_t require_open_sdf, uint32_t* added);
    int snapshot_size(uint64_t* bytes);
    int snapshot_save(void* buf, uint64_t bytes);
    int snapshot_load(const void* buf, uint64_t bytes);

    CsSettings settings;
    host::Inflow inflow;
    uint32_t num_water = 0, num_bed = 0;
    float total_time = 0.0f, frame_emitted_mass = 0.0f, total_emitted_mass = 0.0f;
    uint32_t frame_dropped = 0, total_dropped = 0;
    bool have_prev_p = false;
    CsMetrics last{};

private:
    int alloc(DeviceBuffer& b, size_t bytes);
    void free_all();
    void fill_params(Params& u, float dt) const;
    int upload_ctx();
    int emit(float dt);
    int solve_pressure(uint32_t& sweeps, double& r0, double& r1);
    double residual();
    double refine_residual();
    int launch_cells_blocks() const;
    int launch_particle_blocks(uint32_t n) const;
    int launch_particle_blocks_pt(uint32_t n) const;  // for particle_threads() threads per block
    uint32_t particle_threads() const;
    uint32_t p2g_tile() const;
    uint32_t p2g_tile_count() const;
    void launch_p2g_tiles(const Ctx* dc, uint32_t instances, cudaStream_t st) const;
    int check(cudaError_t e, const char* what);

    cudaStream_t stream_ = nullptr;
    size_t cells_ = 0;
    int sms_ = 148;
    std::vector<DeviceBuffer*> owned_;
    DeviceBuffer d_ctx_, pos_, vel_, c0_, c1_, c2_, bedA_, bedB_, render_, snap_, delta_;
    DeviceBuffer lanes_, lanes64_, gvel_, pf_, divf_, fill_, fcode_, bedv_, plo_, pd_, gres_, lookup_, sdf_, cls_,
        metrics_, resid_;
    DeviceBuffer staging_;  // AoS upload/readback staging
    // sorted P2G
    DeviceBuffer p2g_key_, p2g_rank_, p2g_sorted_, tile_count_, tile_start_, tile_temp_;
    uint32_t p2g_tiles_ = 0;
    JetPlan jet_{};         // device emission planned for the current substep
    // learned warm start: flat f32 parameters, packed bf16 layers, activations
    int learned_alloc();
    int learned_features();
    int learned_forward();
    int learned_enqueue(bool marks);  // residual, inputs, guess and its device-side acceptance
    int learned_collect();            // outcome of the last guess, after the solve synchronised
    int learned_after_solve();
    DeviceBuffer l_params_, l_feat_, l_out_, l_stats_, l_scale_, l_bak_hi_, l_bak_lo_, l_target_, l_mask_, l_err_,
        l_rprev_, l_keep_;
    DeviceBuffer l_wf_[9], l_act_[13];
    bool l_weights_ = false, l_capture_ = false, l_have_sample_ = false, l_ready_ = false;
    // graph mode: the substep's device work captured once and replayed
    int enqueue(uint32_t P, bool capture, uint32_t& sweeps, double& r0, double& r1);
    int substep_graph(float sub_dt);
    int collect();          // read the solve totals of replayed substeps
    int totals_error(const ScTotals& t, const ScTotals& before);
    struct GraphKey {
        uint32_t p2g_mode, check_every, max_sweeps, solve_mode, pressure_storage, rbgs_kernel, rbgs_pairs, warm_start;
        float residual_tol;
        uint32_t num_bed, max_particles, p2g_tile, particle_threads;
        bool operator==(const GraphKey& o) const { return std::memcmp(this, &o, sizeof(GraphKey)) == 0; }
    };
    GraphKey graph_key() const;
    cudaGraphExec_t gexec_ = nullptr;
    GraphKey gkey_{};
    uint32_t graph_launches_ = 0;  // own kernels per replay
    bool graph_pending_ = false;   // replays whose solve totals are not yet read
    DeviceBuffer sc_totals_;
    ScTotals seen_{};              // totals at the last collect()
    // pipelined metrics readback: device counters and solve totals staged in pinned memory
    struct MetricsStage {
        uint32_t m[8];
        ScTotals t;
    };
    MetricsStage* mstage_ = nullptr;
    cudaEvent_t mevent_ = nullptr;
    bool mreq_ = false, mreq_totals_ = false;
    CsMetrics mreq_last_{};
    // cluster-resident solver
    DeviceBuffer sc_scratch_;  // every solver scratch buffer, laid out by sc_scratch_layout
    ScBuffers sc_buf_{};
    // reorder of the water samples by tile (settings.reorder_every)
    int reorder();
    DeviceBuffer ro_keys_, ro_idx_, ro_tmp_, ro_cub_;
    uint64_t substeps_done_ = 0;   // substeps since creation (reorder schedule; snapshotted)
    // grid-wide solver (grids above kClusterMaxCells cells)
    int gs_alloc();
    int solve_grid(uint32_t& sweeps, double& r0, double& r1, bool& done);
    bool use_cluster_solve() const;
    DeviceBuffer gs_rows_, gs_desc_, gs_slots_, gs_misc_, gs_cub_;
    GsBuffers gs_buf_{};
    int gs_ctas_ = 0;          // CTAs of the cooperative launch (0: cannot launch)
    int sc_ranks_ = 0;      // cluster size usable for the solve (0 = unavailable)
    size_t sc_codes_ = 0;   // Morton codes covering the grid (power-of-two cube)
    int solve_cluster(uint32_t& sweeps, double& r0, double& r1, bool& done);
    DeviceBuffer flush_;    // > L2 scratch for cs_flush_l2 (allocated on first use)
    Ctx ctx_{};             // host copy of the device context
    // two pinned staging slots for the context upload, so that the copy is asynchronous
    // (a pageable source may make the copy wait for the stream); a slot is rewritten only
    // after the copy that last read it has run
    Ctx* ctx_pinned_ = nullptr;
    cudaEvent_t ctx_ev_[2] = {nullptr, nullptr};
    bool ctx_ev_used_[2] = {false, false};
    int ctx_slot_ = 0;
    std::vector<float> sdf_host_;

public:
    // ---- profiling: per-phase CUDA events on the stream, launch and byte counters ----
    int profile_enable(bool on);
    int profile_read(CsProfile* out);
    int timer_start();
    int timer_stop(float* ms);
    int flush_l2();
    int autotune(float sub_dt, uint32_t substeps, CsTuneResult* out);
    // learned warm start (CS_WARM_LEARNED) and training-sample capture
    int set_learned_weights(const float* params, uint64_t count);
    int learned_capture(bool on);
    int learned_read_sample(void* feat, float* target, float* mask, float* scale);
    void mark(int phase);      // close the open phase and open `phase` (-1 closes only)
    void count_launch(uint32_t n = 1) {
        prof_.launches += n;
        if (cur_phase_ >= 0) prof_.phase_launches[cur_phase_] += n;
    }

private:
    struct PhaseSpan {
        int phase;
        cudaEvent_t a, b;
    };
    cudaEvent_t take_event();
    bool prof_on_ = false;
    CsProfile prof_{};
    int cur_phase_ = -1;
    cudaEvent_t cur_event_ = nullptr;
    std::vector<PhaseSpan> spans_;
    std::vector<cudaEvent_t> free_events_;
    cudaEvent_t t0_ = nullptr, t1_ = nullptr;
};

void set_error(const std::string& msg);
int validate_settings(const CsSettings* s);

// n independent pours with the same grid, stepped together: every pass is one launch
// with gridDim.y = n over a device array of the instances' contexts (no counterpart in
// the reference).  Each instance keeps its own Engine (buffers, host state, readback);
// the ensemble's stream runs the batched substeps.
class Ensemble {
public:
    ~Ensemble();
    int init(const CsSettings* settings, uint32_t n);
    int substep(float sub_dt);
    int step_frame(float dt);
    int sync();
    int timer_start();            // CUDA event on the ensemble's stream
    int timer_stop(float* ms);    // device ms since timer_start; synchronises
    Engine& at(uint32_t i) { return *eng[i]; }
    uint32_t size() const { return (uint32_t)eng.size(); }

private:
    int enqueue(bool capture);
    int substep_graph();
    std::vector<Engine*> eng;
    cudaStream_t stream = nullptr;
    void* d_ctx = nullptr;       // n x Ctx
    void* d_results = nullptr;   // n x ScResult
    void* d_partial = nullptr;   // chunk sums of the batched scans
    std::vector<Ctx> hctx;
    std::vector<ScBuffers> hsb;
    std::vector<ScResult> results;
    int ranks = 0;
    bool graph = false;          // substep captured once and replayed (settings[0].use_graph)
    cudaGraphExec_t gexec = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
};

}  // namespace cs
