/*
 * coffee_sim.h — C ABI of the B200 MLS-MPM pour-over engine.
 *
 * The reference (craigxchen/coffee-sim) has no FFI layer: the step sits behind
 * `pub(crate) struct MpmSim3D` (crates/sim-wasm/src/mpm_3d/mod.rs:179-671) and is
 * driven through wasm-bindgen by `WasmSim3D` (crates/sim-wasm/src/lib.rs:19-261).
 * Every entry point below replaces one of those methods; each declaration cites the
 * reference item it stands in for.  A Rust host binds these with `extern "C"`
 * (see the rust/ crate), Python binds them with ctypes (coffee_sim_b200/__init__.py).
 *
 * Conventions
 *  - Every call returns int32 status (CS_OK == 0).  cs_last_error_string() gives the
 *    text of the last failure on the calling thread.  No call aborts the process.
 *  - Plain C types only: pointers, sizes, fixed-width ints, float.
 *  - The handle owns all device memory and one CUDA stream.  The caller owns host
 *    buffers; readback and upload calls are synchronous and keep no pointer.
 *  - One host thread per handle (the reference takes &mut self); separate handles may
 *    live on separate threads or devices.
 *  - Host-side array layouts are the reference's byte layouts (state.rs:90-153):
 *      particle      8 x f32  pos.xyz, J, vel.xyz, mass          (shader.rs:24-27)
 *      affine       12 x f32  col0.xyz, phase, col1.xyzw, col2.xyzw (shader.rs:29-33)
 *      bed_extract   8 x f32  pore_water, porosity, permeability, compaction,
 *                             extractable, dissolved, temperature, saturation
 *                                                                 (shader.rs:35-38)
 *      grid lanes    6 x cells i32, lane-major: mass, mom x/y/z, rest vol, cur vol
 *                                                                 (shader.rs:152-164)
 *      grid_vel      4 x f32 per cell: v.xyz, mass                (shader.rs:56)
 *      render        8 x f32 per particle: pos.xyz, colour_t, radius, 0, 0, 0
 *                                                                 (shader.rs:40-43)
 */
#ifndef COFFEE_SIM_H
#define COFFEE_SIM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CS_ABI_VERSION 5u

typedef enum CsStatus {
    CS_OK = 0,
    CS_ERR_INVALID_ARG = 1,
    CS_ERR_CAPACITY = 2,
    CS_ERR_CUDA = 3,
    CS_ERR_NAN = 4,
    CS_ERR_OVERFLOW = 5,
    CS_ERR_TIMEOUT = 6,
    CS_ERR_UNSUPPORTED = 7,
    CS_ERR_NO_DEVICE = 8
} CsStatus;

/* Obstacle kinds of the analytic SDF (mod.rs:71-85). */
enum { CS_OBSTACLE_TRUNCATED_CONE = 0, CS_OBSTACLE_CYLINDER = 1 };
#define CS_MAX_OBSTACLES 4

typedef struct CsObstacle {
    int32_t kind;
    float center[3];
    float top_radius; /* cone */
    float bot_radius; /* cone */
    float radius;     /* cylinder */
    float top_y;
    float bot_y;
} CsObstacle;

/* SpoutSettings (inflow.rs:8-25). */
typedef struct CsSpout {
    float origin[3];
    float direction[3];
    float target[3];
    float nozzle_radius;
    float stem_radius;
    float activation_angle_deg;
    float full_flow_angle_deg;
    float head_at_activation;
    float head_at_full_angle;
    float discharge_coeff;
    float volume_to_ml;
    float max_flow_rate_ml_s;
    float gentle_exit_speed;
    float max_exit_speed;
    float stem_length;
} CsSpout;

/* FilterConfig (filter.rs:3-26). */
typedef struct CsFilter {
    float center[3];
    float top_y;
    float bot_y;
    float top_radius;
    float bot_radius;
    float thickness;
    float hole_radius;
} CsFilter;

/* BedConfig (bed.rs:7-38) plus an optional log-normal permeability field. */
typedef struct CsBed {
    float center[3];
    float top_y;
    float bot_y;
    float top_radius;
    float bot_radius;
    uint32_t num_particles;
    float initial_porosity;
    float initial_permeability;
    float extractable_mass;
    /* Extension: per-sample permeability = exp(ln(initial_permeability) + sigma*N(0,1))
     * when log_perm_sigma > 0 (SplitMix64 + Box-Muller, seeded by perm_seed).
     * Two-layer beds: samples with y below layer_split_y use porosity/permeability
     * multiplied by lower_porosity_scale / lower_permeability_scale. */
    float log_perm_sigma;
    uint32_t perm_seed;
    float layer_split_y;
    float lower_porosity_scale;
    float lower_permeability_scale;
} CsBed;

/* Run-time members of DEFAULT_BREW (brew_config.rs:38-71). */
typedef struct CsBrew {
    float water_particles_per_ml;
    float water_mass_units_per_ml;
    float water_sample_radius_dx;
    float bed_sample_radius_dx;
    float water_kinematic_viscosity_m2_s;
    float min_bed_permeability_m2;
    float bed_absorption_rate;
    float target_bed_retention_ml;
    float bed_pore_capacity_scale;
    float bed_pore_overfill_alpha;
    float bed_surface_void_scale;
    float dripper_outlet_radius;
    float filter_absorption_rate_s;
    float bed_compaction_rate;
    float bed_impact_rate;
} CsBrew;

/* Constants the reference hard-codes inside the WGSL (shader.rs:101-146, 744-823,
 * 1778-1779, 2109).  The default-V60 presets reproduce them exactly; other scenes
 * (SI-unit cones) set their own.  flags: bit0 cone radial barrier, bit1 paper-filter
 * barrier for coffee, bit2 carafe barrier + floor. */
enum { CS_GEOM_CONE = 1u, CS_GEOM_FILTER = 2u, CS_GEOM_CUP = 4u };
typedef struct CsGeometry {
    uint32_t flags;
    float cone_bot_y;          /* -3.0 */
    float cone_top_y;          /*  3.0 */
    float cone_radius_span;    /*  4.2634315: top radius - outlet radius */
    float filter_center_y;     /* -0.35 */
    float filter_top_rel;      /*  2.75 */
    float filter_bot_rel;      /*  3.02 (subtracted) */
    float filter_top_radius;   /*  4.10 */
    float filter_thickness;    /*  0.08 */
    float cup_top_y;           /* -3.5 */
    float cup_radius;          /*  3.0 */
    float cup_floor_y;         /* -8.0 */
    float wall_thickness;      /*  0.4 */
    float bed_surface_ref_y;   /*  3.0 (surface_factor offset) */
    float bed_surface_span;    /*  3.5 */
    float sdf_friction;        /*  0.3 */
    float sdf_restitution;     /*  0.0 */
    float contact_offset;      /*  0.05 */
} CsGeometry;

/* Pressure storage / solve modes. */
enum {
    CS_PRESSURE_FIXED_POINT = 0, /* i32 * 2^18, as the reference (shader.rs:198-209) */
    CS_PRESSURE_FP32 = 1
};
enum {
    CS_SOLVE_FIXED_PAIRS = 0,    /* pressure_rbgs_pairs red+black pairs (mod.rs:352-357) */
    CS_SOLVE_RESIDUAL = 1        /* sweep until relative residual <= residual_tol */
};
enum {
    CS_P2G_ATOMIC32 = 0,         /* one global i32 atomic per node and lane (shader.rs:1043-1048) */
    CS_P2G_SORTED_SHARED = 1,    /* cell-sorted particles, shared-memory tile accumulation */
    CS_P2G_INT64 = 2             /* sorted + i64 fixed point (scale 2^32) */
};
enum {
    CS_WARM_NONE = 0,            /* cold start, p = 0 (shader.rs:1187) */
    CS_WARM_PREVIOUS = 1,        /* previous substep's pressure */
    CS_WARM_LEARNED = 2          /* 3D U-Net guess, kept only if its residual is lower */
};

/* MpmSettings (mod.rs:87-104) + engine extensions. */
typedef struct CsSettings {
    uint32_t abi_version;         /* must be CS_ABI_VERSION */
    float bounds_size[3];
    uint32_t grid_dims[3];
    uint32_t max_particles;
    uint32_t substeps;
    float gravity;
    float bulk_modulus;
    float viscosity;
    float render_radius;
    uint32_t pressure_rbgs_pairs;
    uint32_t use_sdf_cache;
    uint32_t num_obstacles;
    CsObstacle obstacles[CS_MAX_OBSTACLES];
    CsSpout spout;
    float initial_kettle_angle_deg;
    uint32_t has_filter;
    CsFilter filter;
    uint32_t has_bed;
    CsBed bed;
    CsBrew brew;
    CsGeometry geom;
    /* Unit map (units.rs:9-37). */
    float sim_units_per_meter;    /* 57.7 for the V60 scene; 1.0 for SI scenes */
    float standard_gravity_m_s2;  /* 9.80665 */
    float max_velocity;           /* velocity cap, MAX_WATER_SPEED_SIM_UNITS */
    float particle_volume_cells;  /* particle rest volume / dx^3; 0.25 (mod.rs:576) */
    float max_frame_dt;           /* 1/30 (mod.rs:265) */
    /* Engine extensions. */
    uint32_t pressure_storage;    /* CS_PRESSURE_* */
    uint32_t solve_mode;          /* CS_SOLVE_* */
    float residual_tol;           /* relative residual target (FP64 norm) */
    uint32_t max_sweeps;          /* cap on red+black pairs in residual mode */
    uint32_t check_every;         /* pairs between residual evaluations; in FP32 residual mode
                                     the longest interval: after each check the pairs still
                                     needed are predicted from the decay rate (at least 2) */
    uint32_t warm_start;          /* CS_WARM_* */
    uint32_t p2g_mode;            /* CS_P2G_* */
    uint32_t sort_every;          /* reserved: the sorted P2G mode sorts every substep */
    uint32_t device_emission;     /* 1: emit jet particles with a kernel (graph-capturable) */
    uint32_t use_graph;           /* 1: capture the substep in a CUDA graph */
    int32_t device;               /* CUDA device ordinal */
    uint32_t rbgs_kernel;         /* 0 auto (cluster-resident for grids of at most 2^18 cells,
                                     grid-wide above), 1 per-colour launches, 2 cluster-resident
                                     solve, 3 cluster-resident with cluster barriers between
                                     colours, 4 grid-wide solve (one cooperative launch over
                                     the rows that hold fluid) */
    float flow_override_ml_s;     /* >0: constant flow instead of the kettle-angle model */
    float exit_speed_override;    /* >0 with flow override: jet speed */
    float rbgs_omega;             /* red-black over-relaxation; 0 or 1 = plain Gauss-Seidel */
    uint32_t first_check;         /* FP32 residual mode: pairs before a solve's first residual
                                     check (0: check_every); later intervals are predicted */
    uint32_t reorder_every;       /* >0: every this many substeps (counted from creation), reorder
                                     the water samples' slots stably by the 4^3-cell tile of their
                                     P2G base cell (samples that deposit nothing last), so that
                                     P2G and G2P touch neighbouring cells from neighbouring
                                     threads; slot numbers of water samples change then.  0: off */
    uint32_t p2g_tile;            /* cells per side of a sorted-P2G tile: 0 or 4, or 8 (fewer tile
                                     borders to flush, 4x the shared memory) */
    uint32_t particle_threads;    /* threads per block of the particle passes (P2G keys and
                                     scatter, G2P, bed coupling, render packing): 0 or 256, or 128
                                     (G2P is compiled for at most 256 threads per block) */
    uint32_t reserved[3];
} CsSettings;

/* Observability counters (mod.rs:50-68 / state.rs:22-28) + solver telemetry. */
typedef struct CsMetrics {
    float max_abs_div;
    uint32_t fluid_cells;
    uint32_t div_clamp_fires;
    uint32_t pressure_clamp_fires;
    uint32_t mass_overflow_fires;
    uint32_t last_sweeps;          /* red+black pairs in the last substep's solve */
    double last_residual;          /* relative residual after the solve (FP64), -1 if unmeasured */
    double initial_residual;       /* relative residual of the warm start (FP64), -1 if unmeasured */
    uint32_t nan_flag;             /* a non-finite particle or grid value was seen */
    uint32_t timeout_flag;         /* a bounded device wait gave up */
    uint32_t learned_used;         /* 1 if the learned guess was kept in the last solve */
    uint32_t residual_checks;      /* FP64 residual evaluations in the last solve, the warm start's included */
    double solve_ms;               /* device time of the last pressure solve, if timed */
} CsMetrics;

typedef struct CsSim CsSim;
typedef struct CsEnsemble CsEnsemble;

/* ---- library ---- */
const char* cs_last_error_string(void);
uint32_t cs_abi_version(void);
/* 1 when the library runs the step on a GPU; 0 for the CPU oracle. */
int32_t cs_is_gpu_engine(void);

/* ---- settings presets (mod.rs:106-161) ---- */
int32_t cs_settings_default_v60(CsSettings* out);           /* MpmSettings::default_v60 */
int32_t cs_settings_benchmark_free_stream(CsSettings* out); /* MpmSettings::benchmark_free_stream */
int32_t cs_settings_benchmark_center_pour(CsSettings* out); /* MpmSettings::benchmark_center_pour */
/* SpoutSettings::aim_at / translate_origin_to on a settings value (inflow.rs:49-67). */
int32_t cs_settings_aim_spout(CsSettings* s, float x, float y, float z);
/* kozeny_carman_permeability_m2 (brew_config.rs:92-96): bed permeability in m^2 of a
 * grind of mean particle diameter grind_um at the given porosity. */
float cs_kozeny_carman_permeability_m2(float grind_um, float porosity);

/* ---- lifetime (mod.rs:196-262, 432-446) ---- */
int32_t cs_create(const CsSettings* settings, CsSim** out);   /* MpmSim3D::new */
int32_t cs_destroy(CsSim* sim);
int32_t cs_reset(CsSim* sim);                                  /* MpmSim3D::reset */

/* ---- stepping (mod.rs:264-430) ---- */
int32_t cs_step_frame(CsSim* sim, float dt);                   /* MpmSim3D::step_frame */
/* One substep of length sub_dt: emission, uniforms, every kernel (mod.rs:271-419). */
int32_t cs_step_substep(CsSim* sim, float sub_dt);
/* Run the first `passes` kernels of one substep (debugging / parity localisation).
 * Pass numbering follows the dispatch order of mod.rs:317-414. */
int32_t cs_step_substep_partial(CsSim* sim, float sub_dt, uint32_t passes);

/* ---- controls (mod.rs:448-458, lib.rs:72-86) ---- */
int32_t cs_set_kettle_angle(CsSim* sim, float angle_deg);
int32_t cs_set_spout_position(CsSim* sim, float x, float y, float z);
int32_t cs_set_spout_target(CsSim* sim, float x, float y, float z);
/* Constant jet (ml/s, scene units/s) instead of the kettle-angle model; flow <= 0 clears it. */
int32_t cs_set_flow_override(CsSim* sim, float flow_ml_s, float exit_speed);

/* ---- getters (mod.rs:460-544, lib.rs:87-252) ---- */
int32_t cs_get_counts(const CsSim* sim, uint32_t* num_water, uint32_t* num_bed, uint32_t* max_particles);
int32_t cs_get_kettle_angle(const CsSim* sim, float* out);
int32_t cs_get_spout_position(const CsSim* sim, float out[3]);
int32_t cs_get_flow(const CsSim* sim, float* flow_rate_ml_s, float* exit_speed, float* exit_speed_m_s);
int32_t cs_get_time(const CsSim* sim, float* total_time);
int32_t cs_get_emission(const CsSim* sim, float* frame_emitted_mass, float* total_emitted_mass,
                        uint32_t* frame_dropped, uint32_t* total_dropped);
int32_t cs_get_mass_units_per_ml(const CsSim* sim, float* out);
/* refresh_metrics + metric getters (mod.rs:546-567, lib.rs:219-252); synchronises. */
int32_t cs_get_metrics(CsSim* sim, CsMetrics* out);
/* Pipelined readback (no reference counterpart): cs_metrics_request queues a copy of the
 * latest substep's metrics behind the work already enqueued and returns at once;
 * cs_metrics_wait waits for that copy only and returns the metrics as cs_get_metrics would
 * have after that substep.  Substeps may be enqueued in between, so a host loop can read
 * step k's result while step k+1 runs.  One request at a time (CS_ERR_INVALID_ARG else). */
int32_t cs_metrics_request(CsSim* sim);
int32_t cs_metrics_wait(CsSim* sim, CsMetrics* out);
int32_t cs_get_settings(const CsSim* sim, CsSettings* out);

/* ---- readback into caller buffers (physics_tests.rs:61-1083 read the same layouts) ---- */
int32_t cs_read_particles(CsSim* sim, uint32_t first, uint32_t count, float* out);     /* 8 f32 each */
int32_t cs_read_affine(CsSim* sim, uint32_t first, uint32_t count, float* out);        /* 12 f32 each */
int32_t cs_read_bed_extract(CsSim* sim, uint32_t first, uint32_t count, float* out);   /* 8 f32 each */
int32_t cs_read_grid_lanes(CsSim* sim, int32_t* out);       /* 6 x cells, reference lane aliasing */
int32_t cs_read_grid_lanes64(CsSim* sim, int64_t* out);     /* 6 x cells, i64 * 2^32 P2G lanes (int64 mode) */
int32_t cs_read_grid_vel(CsSim* sim, float* out);           /* 4 x cells */
int32_t cs_read_pressure(CsSim* sim, float* out);           /* cells, decoded to f32 */
int32_t cs_read_cell_kind(CsSim* sim, int32_t* out);        /* cells, kind after classify */
int32_t cs_read_bed_lookup(CsSim* sim, int32_t* out);       /* cells */
int32_t cs_read_bed_delta(CsSim* sim, int32_t* out);        /* 4 x max_particles, lane-major */
int32_t cs_read_render(CsSim* sim, uint32_t first, uint32_t count, float* out);        /* 8 f32 each */
int32_t cs_read_sdf(CsSim* sim, float* out);                /* 128^3 R32F texels */
int32_t cs_read_sdf_class(CsSim* sim, uint8_t* out);        /* cells */
/* The pressure solve's inputs as classify wrote them (no reference counterpart): the
 * liquid fill fraction of every cell (liquid_fill_fraction, shader.rs:293-304) and the
 * divergence the solve reads in FP32 pressure storage (CS_ERR_UNSUPPORTED with
 * fixed-point storage).  cells f32 each. */
int32_t cs_read_solver_inputs(CsSim* sim, float* fill, float* div);

/* ---- upload from caller buffers ---- */
int32_t cs_write_particles(CsSim* sim, uint32_t first, uint32_t count, const float* in);
int32_t cs_write_affine(CsSim* sim, uint32_t first, uint32_t count, const float* in);
int32_t cs_write_bed_extract(CsSim* sim, uint32_t first, uint32_t count, const float* in);
/* Declare how many slots are live: bed first, then water (mod.rs:241-242). */
int32_t cs_set_counts(CsSim* sim, uint32_t num_water, uint32_t num_bed);
/* Append a block of water: per_axis^3 samples per cell inside [lo, hi], each jittered
 * uniformly by +/- jitter*dx per axis (SplitMix64, seed), nominal mass, J = 1.
 * When require_open_sdf != 0 a sample is kept only where the scene SDF exceeds the
 * contact offset.  Returns the number appended in *added. */
int32_t cs_add_water_block(CsSim* sim, const float lo[3], const float hi[3], uint32_t per_axis,
                           float jitter, uint32_t seed, uint32_t require_open_sdf, uint32_t* added);

/* ---- checkpoint / resume (no counterpart: the reference only has reset, mod.rs:432) ---- */
int32_t cs_snapshot_size(CsSim* sim, uint64_t* bytes);
int32_t cs_snapshot_save(CsSim* sim, void* buffer, uint64_t bytes);
int32_t cs_snapshot_load(CsSim* sim, const void* buffer, uint64_t bytes);

/* ---- batched ensemble of independent pours (no counterpart in the reference) ----
 * n instances with their own settings (same grid dims) stepped together: one launch
 * per pass covers every instance through per-instance offset tables.  With
 * settings[0].use_graph = 1 (residual-mode solve, plain warm start) the batched substep
 * is captured once and replayed with no host synchronisation; an instance whose fluid
 * overflows its solve cluster is then reported as CS_ERR_CAPACITY by the next
 * cs_ensemble_get_metrics instead of being re-solved alone. */
int32_t cs_ensemble_create(const CsSettings* settings, uint32_t n, CsEnsemble** out);
int32_t cs_ensemble_destroy(CsEnsemble* ens);
int32_t cs_ensemble_step_substep(CsEnsemble* ens, float sub_dt);
int32_t cs_ensemble_step_frame(CsEnsemble* ens, float dt);
int32_t cs_ensemble_add_water_block(CsEnsemble* ens, uint32_t i, const float lo[3], const float hi[3],
                                    uint32_t per_axis, float jitter, uint32_t seed,
                                    uint32_t require_open_sdf, uint32_t* added);
int32_t cs_ensemble_set_kettle_angle(CsEnsemble* ens, uint32_t i, float angle_deg);
int32_t cs_ensemble_set_flow_override(CsEnsemble* ens, uint32_t i, float flow_ml_s, float exit_speed);
int32_t cs_ensemble_get_counts(CsEnsemble* ens, uint32_t i, uint32_t* num_water, uint32_t* num_bed);
int32_t cs_ensemble_read_particles(CsEnsemble* ens, uint32_t i, uint32_t first, uint32_t count, float* out);
int32_t cs_ensemble_get_metrics(CsEnsemble* ens, uint32_t i, CsMetrics* out);
/* The learned warm start's weights for every instance (CS_WARM_LEARNED ensembles: each
 * instance's guess runs between the batched classify and the batched solve). */
int32_t cs_ensemble_set_learned_weights(CsEnsemble* ens, const float* params, uint64_t count);
int32_t cs_ensemble_timer_start(CsEnsemble* ens);           /* CUDA event on the ensemble's stream */
int32_t cs_ensemble_timer_stop(CsEnsemble* ens, float* ms); /* device ms since the start; synchronises */

/* ---- device timing and profiling (no counterpart: the reference defers timestamp
 * queries, mod.rs:313 `timestamp_writes: None`) ---- */
enum {
    CS_PHASE_EMIT = 0,      /* inflow emission upload + uniforms */
    CS_PHASE_CLEAR = 1,     /* grid clears, bed lookup rebuild */
    CS_PHASE_P2G = 2,
    CS_PHASE_GRID = 3,      /* grid_update + boundary + classify */
    CS_PHASE_SWEEPS = 4,    /* red-black pressure sweeps */
    CS_PHASE_RESIDUAL = 5,  /* FP64 residual evaluations + refinement bookkeeping */
    CS_PHASE_PROJECT = 6,   /* project, packing, viscosity, boundary passes */
    CS_PHASE_G2P = 7,
    CS_PHASE_BED = 8,       /* bed coupling, extraction, bed dynamics */
    CS_PHASE_RENDER = 9,
    CS_PHASE_LEARNED = 10,  /* learned warm start: inputs, U-Net guess, residual comparison */
    CS_PHASE_COUNT = 16
};
typedef struct CsProfile {
    double phase_ms[CS_PHASE_COUNT];        /* device time per phase (CUDA events) */
    uint32_t phase_launches[CS_PHASE_COUNT];
    uint64_t launches;                      /* kernels launched by the engine */
    uint64_t sweeps;                        /* red+black pairs */
    uint64_t residual_evals;
    uint64_t h2d_bytes, d2h_bytes;          /* host<->device traffic of the step calls */
    uint64_t substeps;
} CsProfile;
int32_t cs_profile_enable(CsSim* sim, int32_t on);   /* resets the counters */
int32_t cs_profile_read(CsSim* sim, CsProfile* out); /* synchronises */

/* ---- BF16 3-D convolution on the tensor cores (tcgen05), the layers of the pressure-guess
 * U-Net (no counterpart in the reference).  Device pointers, channels-last bf16
 * activations [voxel][C]; `err` is a device flag raised if a wait times out. ---- */
/* Y = relu?(conv3x3x3(X) + bias): x bf16 [vox][cin_pad], w packed by cs_nn_pack_weights,
 * bias cout_pad floats or null, y bf16 / y32 f32 [vox][cout_pad] (either may be null). */
int32_t cs_nn_conv3d(const void* x, const void* w, const float* bias, void* y, float* y32, int32_t gx, int32_t gy,
                     int32_t gz, int32_t cin_pad, int32_t cout_pad, int32_t relu, uint32_t* err, void* stream);
int32_t cs_nn_conv3d_wgrad(const void* x, const void* dy, float* dwt, int32_t gx, int32_t gy, int32_t gz,
                           int32_t cin_pad, int32_t cout_pad, int32_t splits, uint32_t* err, void* stream);
int32_t cs_nn_pack_weights(const float* w, void* out, int32_t cin, int32_t cin_pad, int32_t cout, int32_t cout_pad,
                           int32_t flip, void* stream);
/* 2x2x2 average pool (bf16 forward; f32 gradient accumulated into dx). */
int32_t cs_nn_pool(const void* x, void* y, const float* dy, float* dx, int32_t gx, int32_t gy, int32_t gz, int32_t c,
                   int32_t backward, void* stream);
/* Nearest x2 upsample of `low` concatenated with `skip` (bf16); the gradient accumulates
 * into dlow / dskip (f32). */
int32_t cs_nn_upcat(const void* low, const void* skip, void* out, const float* dout, float* dlow, float* dskip,
                    int32_t gx, int32_t gy, int32_t gz, int32_t c1, int32_t c2, int32_t backward, void* stream);
/* ReLU-masked gradient to bf16, accumulating the bias gradient db (may be null). */
int32_t cs_nn_relu_grad(const float* g, const void* y, void* out, float* db, int64_t n, int32_t c, void* stream);
/* 1x1x1 output layer with c inputs: w holds c weights then the bias. */
int32_t cs_nn_head(const void* x, const float* w, float* out, const float* dout, float* dx, float* dw, int64_t nv,
                   int32_t c, int32_t backward, void* stream);
/* Masked mean squared error and its gradient (loss accumulated into loss[0]). */
int32_t cs_nn_mse(const float* o, const float* t, const float* m, float* dout, float* loss, int64_t nv,
                  float inv_count, void* stream);
/* Weight gradient from the GEMM layout [(tap, ci)][co] to the master layout [co][tap][ci]. */
int32_t cs_nn_wgrad_master(const float* dwt, float* gw, int32_t cin, int32_t cout, int32_t cout_pad, void* stream);
int32_t cs_nn_adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2, float eps,
                   int32_t step, void* stream);
int32_t cs_nn_axpy(float* y, const float* x, float a, int64_t n, void* stream);

/* ---- Learned warm start (CS_WARM_LEARNED; no counterpart in the reference) ----
 * Weights of the pressure-guess U-Net (coffee_sim_b200/unet.py layout, f32, host memory).
 * From the FP64 residual of the previous-substep pressure the network predicts a pressure
 * correction; before each solve the previous pressure plus that correction replaces it
 * when its FP64 residual is smaller (CsMetrics.learned_used).  Grid dims must be
 * multiples of 4. */
int32_t cs_set_learned_weights(CsSim* sim, const float* params, uint64_t count);
/* Capture one training pair per substep: network inputs before the solve (bf16
 * [cells][8]) and (solved - previous pressure) / s with its fluid mask (f32 [cells]). */
int32_t cs_learned_capture(CsSim* sim, uint32_t on);
/* Copy the last captured pair into device buffers of the caller (any may be null);
 * scale (host) receives s. */
int32_t cs_learned_read_sample(CsSim* sim, void* feat, float* target, float* mask, float* scale);

/* ---- Solver parameters and autotuner (no counterpart in the reference) ---- */

/* Change the residual-mode solver between substeps: over-relaxation (0 keeps the current
 * value), pairs between residual checks (0 keeps), cap on pairs (0 keeps). */
int32_t cs_set_solver(CsSim* sim, float omega, uint32_t check_every, uint32_t max_sweeps);
/* P2G accumulation (CS_P2G_ATOMIC32 or CS_P2G_SORTED_SHARED) from the next substep on. */
int32_t cs_set_p2g_mode(CsSim* sim, uint32_t mode);
/* Graph mode from the next substep on (same conditions as settings.use_graph). */
int32_t cs_set_graph_mode(CsSim* sim, uint32_t use_graph);

typedef struct CsTuneResult {
    float omega;           /* chosen over-relaxation */
    uint32_t check_every;  /* chosen pairs between residual checks */
    uint32_t p2g_mode;     /* chosen P2G accumulation */
    uint32_t trials;       /* configurations timed */
    float best_ms;         /* device ms per substep with the chosen configuration */
    float initial_ms;      /* device ms per substep with the configuration at entry */
    uint32_t first_check;  /* chosen pairs before each solve's first residual check (0: check_every) */
    uint32_t p2g_tile;     /* chosen P2G tile side (4 or 8) */
    uint32_t particle_threads;  /* chosen threads per block of the particle passes */
} CsTuneResult;

/* Time `substeps` substeps of length sub_dt from the current state for each candidate
 * configuration (P2G mode, then over-relaxation 1.80-1.96 x check interval 10/20/40/60/80,
 * then a first-check interval of 0.85/0.92/0.98 of the fewest pairs a substep took, then
 * the launch shapes: P2G tile side 4/8 x 128/256 threads per particle-pass block),
 * restoring the state after every trial; keep the fastest whose every substep reached
 * the residual target.  The simulation ends in the state it had at entry with the
 * chosen configuration applied.  Residual-mode solves only (CS_ERR_UNSUPPORTED else). */
int32_t cs_autotune(CsSim* sim, float sub_dt, uint32_t substeps, CsTuneResult* out);
int32_t cs_timer_start(CsSim* sim);                  /* CUDA event on the sim's stream */
int32_t cs_timer_stop(CsSim* sim, float* ms);        /* device ms since cs_timer_start; synchronises */
int32_t cs_flush_l2(CsSim* sim);                     /* overwrite a buffer larger than L2 on the sim's stream */
int32_t cs_sync(CsSim* sim);

/* ---- allocation-free pressure solve (no counterpart in the reference) ----
 * For hosts that may not call cudaMalloc while they run (an engine that reserves its
 * whole GPU budget up front, a real-time loop that cannot afford cudaMalloc's latency
 * and implicit synchronisation): the mixed-precision red-black SOR solve of the
 * FP32-storage residual mode, run on the caller's device arrays of gx*gy*gz cells:
 * kind (CELL kinds 0..4 as classify writes them), fill (liquid fill fraction),
 * div (classify's divergence minus target), p_hi/p_lo (pressure words: warm start
 * in, solution out).  Scratch lives in a static device array reserved when the
 * library is loaded (about 7.6 MB per GPU, held until exit), so grids are limited to
 * 64 cells per side and 16 x 4095 fluid cells; larger inputs return CS_ERR_CAPACITY.
 * The first call on a device looks up that array's device address.  Calls share the
 * array: calls that overlap on the GPU race.  `stream` is a cudaStream_t (NULL =
 * default stream); every call synchronises it, so it must never be called on a
 * capturing stream (CS_ERR_INVALID_ARG).  It writes the red+black pair count and the
 * final relative residual to the host.  After a call that returns an error, p_hi and
 * p_lo hold unspecified values (a partly solved pressure); CS_ERR_TIMEOUT means a
 * bounded wait between CTAs ran out twice. */
int32_t cs_pressure_solve_noalloc(uint32_t gx, uint32_t gy, uint32_t gz, float dx, float dt, float omega,
                                  float residual_tol, uint32_t max_pairs, uint32_t check_every,
                                  const int32_t* kind, const float* fill, const float* div, float* p_hi,
                                  float* p_lo, void* stream, uint32_t* pairs_out, double* residual_out);

#ifdef __cplusplus
}
#endif

#endif /* COFFEE_SIM_H */
