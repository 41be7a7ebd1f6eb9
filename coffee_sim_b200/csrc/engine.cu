// engine.cu — Engine implementation: the substep schedule of mod.rs:264-430 on one
// CUDA stream, plus the extern "C" entry points of include/coffee_sim.h.
//
// Unity build: the kernels are included here so the launches see their definitions.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "engine.h"
#include "kernels.cu"
#include "batch_scan.cuh"
#include "solver_cluster.cuh"
#include "solver_grid.cuh"

namespace cs {

static thread_local std::string g_error;
void set_error(const std::string& msg) { g_error = msg; }

static const int kThreads = 256;

int Engine::check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return CS_OK;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return CS_ERR_CUDA;
}

Engine::Engine(const CsSettings& s) : settings(s) {
    cells_ = (size_t)s.grid_dims[0] * s.grid_dims[1] * s.grid_dims[2];
    inflow.angle = s.initial_kettle_angle_deg;
    inflow.flow_override = s.flow_override_ml_s;
    inflow.speed_override = s.exit_speed_override;
}

Engine::~Engine() {
    if (stream_) cudaStreamSynchronize(stream_);
    if (gexec_) cudaGraphExecDestroy(gexec_);
    for (auto& sp : spans_) {
        free_events_.push_back(sp.a);
        free_events_.push_back(sp.b);
    }
    std::sort(free_events_.begin(), free_events_.end());
    free_events_.erase(std::unique(free_events_.begin(), free_events_.end()), free_events_.end());
    for (cudaEvent_t e : free_events_) cudaEventDestroy(e);
    if (cur_event_ && spans_.empty()) cudaEventDestroy(cur_event_);
    if (t0_) cudaEventDestroy(t0_);
    if (t1_) cudaEventDestroy(t1_);
    if (mevent_) cudaEventDestroy(mevent_);
    if (mstage_) cudaFreeHost(mstage_);
    for (cudaEvent_t e : ctx_ev_)
        if (e) cudaEventDestroy(e);
    if (ctx_pinned_) cudaFreeHost(ctx_pinned_);
    free_all();
    if (stream_) cudaStreamDestroy(stream_);
}

int Engine::alloc(DeviceBuffer& b, size_t bytes) {
    b.bytes = bytes;
    if (bytes == 0) bytes = 16;
    int rc = check(cudaMalloc(&b.ptr, bytes), "cudaMalloc");
    if (rc) return rc;
    owned_.push_back(&b);
    return check(cudaMemsetAsync(b.ptr, 0, bytes, stream_), "cudaMemsetAsync");
}

void Engine::free_all() {
    for (DeviceBuffer* b : owned_) {
        if (b->ptr) cudaFree(b->ptr);
        b->ptr = nullptr;
    }
    owned_.clear();
}

int Engine::launch_cells_blocks() const {
    size_t b = (cells_ + kThreads - 1) / kThreads;
    return (int)std::min<size_t>(b, (size_t)sms_ * 16);
}
int Engine::launch_particle_blocks(uint32_t n) const {
    size_t b = ((size_t)n + kThreads - 1) / kThreads;
    return (int)std::max<size_t>(1, std::min<size_t>(b, (size_t)sms_ * 16));
}
// Launch shapes the autotuner can choose: threads per block of the particle passes and
// the P2G tile side.
uint32_t Engine::particle_threads() const { return settings.particle_threads ? settings.particle_threads : kThreads; }
int Engine::launch_particle_blocks_pt(uint32_t n) const {
    const size_t t = particle_threads();
    size_t b = ((size_t)n + t - 1) / t;
    return (int)std::max<size_t>(1, std::min<size_t>(b, (size_t)sms_ * (2048 / t)));
}
uint32_t Engine::p2g_tile() const { return settings.p2g_tile ? settings.p2g_tile : (uint32_t)P2G_TILE; }
uint32_t Engine::p2g_tile_count() const {
    const uint32_t t = p2g_tile();
    return ((settings.grid_dims[0] + t) / t) * ((settings.grid_dims[1] + t) / t) * ((settings.grid_dims[2] + t) / t);
}
// The tile-sorted P2G accumulation for `instances` contexts (template by lane width and
// tile side).
void Engine::launch_p2g_tiles(const Ctx* dc, uint32_t instances, cudaStream_t st) const {
    const int tb = (int)std::min<uint32_t>(p2g_tile_count(), (uint32_t)sms_ * 16);
    const dim3 g(tb, instances);
    const bool i64 = settings.p2g_mode == CS_P2G_INT64;
    if (p2g_tile() == 8) {
        if (i64)
            k_p2g_tiles<unsigned long long, 8><<<g, P2G_THREADS, 0, st>>>(dc);
        else
            k_p2g_tiles<int32_t, 8><<<g, P2G_THREADS, 0, st>>>(dc);
    } else {
        if (i64)
            k_p2g_tiles<unsigned long long, 4><<<g, P2G_THREADS, 0, st>>>(dc);
        else
            k_p2g_tiles<int32_t, 4><<<g, P2G_THREADS, 0, st>>>(dc);
    }
}

int Engine::init() {
    int dev = settings.device;
    int rc = check(cudaSetDevice(dev), "cudaSetDevice");
    if (rc) return rc;
    cudaDeviceProp prop;
    if ((rc = check(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties"))) return rc;
    sms_ = prop.multiProcessorCount;
    if ((rc = check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate"))) return rc;
    const size_t mp = settings.max_particles;
    const size_t f4 = sizeof(float4);
    DeviceBuffer* bufs[] = {&pos_, &vel_, &c0_, &c1_, &c2_, &bedA_, &bedB_, &snap_};
    for (DeviceBuffer* b : bufs)
        if ((rc = alloc(*b, mp * f4))) return rc;
    if ((rc = alloc(render_, mp * 2 * f4))) return rc;
    if ((rc = alloc(delta_, mp * 4 * sizeof(int32_t)))) return rc;
    if ((rc = alloc(lanes_, cells_ * 6 * sizeof(int32_t)))) return rc;
    if ((rc = alloc(lanes64_, settings.p2g_mode == CS_P2G_INT64 ? cells_ * 6 * sizeof(long long) : 0))) return rc;
    {  // sort buffers: also used when the mode is switched at run time
        // sized for the smallest tile side (the most tiles)
        uint32_t nt[3];
        for (int a = 0; a < 3; ++a) nt[a] = (settings.grid_dims[a] + 1 + P2G_TILE - 1) / P2G_TILE;
        p2g_tiles_ = nt[0] * nt[1] * nt[2];
        if ((rc = alloc(p2g_key_, (size_t)mp * sizeof(uint32_t)))) return rc;
        if ((rc = alloc(p2g_rank_, (size_t)mp * sizeof(uint32_t)))) return rc;
        if ((rc = alloc(p2g_sorted_, (size_t)mp * sizeof(uint32_t)))) return rc;
        if ((rc = alloc(tile_count_, ((size_t)p2g_tiles_ + 1) * sizeof(uint32_t)))) return rc;
        if ((rc = alloc(tile_start_, ((size_t)p2g_tiles_ + 1) * sizeof(uint32_t)))) return rc;
        size_t temp = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, temp, (uint32_t*)nullptr, (uint32_t*)nullptr, (int)p2g_tiles_ + 1,
                                      stream_);
        if ((rc = alloc(tile_temp_, temp))) return rc;
    }
    if ((rc = alloc(gvel_, cells_ * f4))) return rc;
    if ((rc = alloc(pf_, cells_ * sizeof(float)))) return rc;
    if ((rc = alloc(divf_, cells_ * sizeof(float)))) return rc;
    if ((rc = alloc(fill_, cells_ * sizeof(float)))) return rc;
    if ((rc = alloc(fcode_, cells_ * sizeof(float)))) return rc;
    if ((rc = alloc(bedv_, cells_ * f4))) return rc;
    if ((rc = alloc(plo_, cells_ * sizeof(float)))) return rc;
    if ((rc = alloc(pd_, cells_ * sizeof(float)))) return rc;
    if ((rc = alloc(gres_, cells_ * sizeof(float)))) return rc;
    if ((rc = alloc(lookup_, cells_ * sizeof(int32_t)))) return rc;
    if ((rc = alloc(sdf_, (size_t)SDF_RES * SDF_RES * SDF_RES * sizeof(float)))) return rc;
    if ((rc = alloc(cls_, cells_))) return rc;
    if ((rc = alloc(metrics_, 8 * sizeof(uint32_t)))) return rc;
    if ((rc = alloc(resid_, 4 * sizeof(double)))) return rc;
    if ((rc = alloc(sc_totals_, sizeof(ScTotals)))) return rc;
    cudaMemsetAsync(sc_totals_.ptr, 0, sizeof(ScTotals), stream_);
    ctx_.totals = (ScTotals*)sc_totals_.ptr;
    if ((rc = alloc(d_ctx_, sizeof(Ctx)))) return rc;
    if ((rc = alloc(staging_, std::max<size_t>(mp * 12 * sizeof(float), cells_ * 6 * sizeof(int32_t))))) return rc;
    // cluster-resident solver: buffers and the largest launchable cluster size
    {
        uint32_t side = 1;
        while (side < settings.grid_dims[0] || side < settings.grid_dims[1] || side < settings.grid_dims[2]) side <<= 1;
        sc_codes_ = (size_t)side * side * side;
    }
    {
        const size_t cub = sc_scan_temp_bytes((uint32_t)sc_codes_);
        const ScScratch lay = sc_scratch_layout(cells_, sc_codes_, cub);
        if ((rc = alloc(sc_scratch_, lay.total))) return rc;
        sc_buf_ = sc_buffers_at((unsigned char*)sc_scratch_.ptr, lay, cub);
        ctx_.sb = sc_buf_;
        sc_ranks_ = sc_max_cluster_ranks();
    }
    if ((rc = gs_alloc())) return rc;
    if (settings.reorder_every) {
        size_t cub = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, cub, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                        (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)mp, 0, 32, stream_);
        if ((rc = alloc(ro_keys_, (size_t)mp * 2 * sizeof(uint32_t)))) return rc;
        if ((rc = alloc(ro_idx_, (size_t)mp * 2 * sizeof(uint32_t)))) return rc;
        if ((rc = alloc(ro_tmp_, (size_t)mp * sizeof(float4)))) return rc;
        if ((rc = alloc(ro_cub_, cub))) return rc;
    }

    ctx_.pos = (float4*)pos_.ptr;
    ctx_.vel = (float4*)vel_.ptr;
    ctx_.c0 = (float4*)c0_.ptr;
    ctx_.c1 = (float4*)c1_.ptr;
    ctx_.c2 = (float4*)c2_.ptr;
    ctx_.bedA = (float4*)bedA_.ptr;
    ctx_.bedB = (float4*)bedB_.ptr;
    ctx_.render = (float4*)render_.ptr;
    ctx_.snap = (float4*)snap_.ptr;
    ctx_.delta = (int32_t*)delta_.ptr;
    ctx_.lanes = (int32_t*)lanes_.ptr;
    ctx_.kind = (const int32_t*)lanes_.ptr + 3 * cells_;
    ctx_.lanes64 = (long long*)lanes64_.ptr;
    ctx_.p2g_key = (uint32_t*)p2g_key_.ptr;
    ctx_.p2g_rank = (uint32_t*)p2g_rank_.ptr;
    ctx_.p2g_sorted = (uint32_t*)p2g_sorted_.ptr;
    ctx_.tile_count = (uint32_t*)tile_count_.ptr;
    ctx_.tile_start = (uint32_t*)tile_start_.ptr;
    ctx_.gvel = (float4*)gvel_.ptr;
    ctx_.pf = (float*)pf_.ptr;
    ctx_.divf = (float*)divf_.ptr;
    ctx_.fill = (float*)fill_.ptr;
    ctx_.fcode = (float*)fcode_.ptr;
    ctx_.bedv = (float4*)bedv_.ptr;
    ctx_.plo = (float*)plo_.ptr;
    ctx_.pd = (float*)pd_.ptr;
    ctx_.gres = (float*)gres_.ptr;
    ctx_.lookup = (int32_t*)lookup_.ptr;
    ctx_.sdf = (const float*)sdf_.ptr;
    ctx_.cls = (const uint8_t*)cls_.ptr;
    ctx_.metrics = (uint32_t*)metrics_.ptr;
    ctx_.resid = (double*)resid_.ptr;

    // state.rs:178-182: SDF texture and cell-solid mask, generated on the device
    SdfSpec spec;
    std::memset(&spec, 0, sizeof(spec));
    for (int a = 0; a < 3; ++a) spec.bounds[a] = settings.bounds_size[a];
    spec.wall_thickness = settings.geom.wall_thickness;
    spec.count = settings.num_obstacles;
    for (uint32_t k = 0; k < settings.num_obstacles; ++k) spec.obs[k] = settings.obstacles[k];
    k_gen_sdf<<<sms_ * 8, kThreads, 0, stream_>>>((float*)sdf_.ptr, spec);
    fill_params(ctx_.u, 0.0f);
    if ((rc = upload_ctx())) return rc;
    k_gen_class<<<dim3(launch_cells_blocks(), 1), kThreads, 0, stream_>>>((const Ctx*)d_ctx_.ptr);
    if ((rc = check(cudaGetLastError(), "set-up kernels"))) return rc;
    sdf_host_.resize((size_t)SDF_RES * SDF_RES * SDF_RES);
    if ((rc = check(cudaMemcpyAsync(sdf_host_.data(), sdf_.ptr, sdf_.bytes, cudaMemcpyDeviceToHost, stream_), "sdf copy")))
        return rc;
    if ((rc = sync())) return rc;
    return reset();
}

// mod.rs:222-262 (init_bed) after clearing all particle state (mod.rs:432-446)
int Engine::reset() {
    num_water = num_bed = 0;
    total_time = frame_emitted_mass = total_emitted_mass = 0.0f;
    frame_dropped = total_dropped = 0;
    float fo = inflow.flow_override, so = inflow.speed_override;
    inflow = host::Inflow();
    inflow.angle = settings.initial_kettle_angle_deg;
    inflow.flow_override = fo;
    inflow.speed_override = so;
    have_prev_p = false;
    substeps_done_ = 0;
    std::memset(&last, 0, sizeof(last));
    last.last_residual = last.initial_residual = -1.0;
    DeviceBuffer* zero[] = {&pos_, &vel_, &c0_, &c1_, &c2_, &bedA_, &bedB_, &render_, &snap_, &delta_, &lanes_,
                            &gvel_, &pf_, &divf_, &fill_, &fcode_, &plo_, &pd_, &gres_};
    int rc;
    for (DeviceBuffer* b : zero)
        if ((rc = check(cudaMemsetAsync(b->ptr, 0, b->bytes, stream_), "memset"))) return rc;
    if ((rc = check(cudaMemsetAsync(lookup_.ptr, 0xff, lookup_.bytes, stream_), "memset"))) return rc;
    if (!settings.has_bed) return sync();
    host::BedSamples bed = host::init_bed(settings.bed, settings.grid_dims, settings.bounds_size);
    uint32_t n = std::min(bed.count, settings.max_particles);
    if (n == 0) return sync();
    num_bed = n;
    if ((rc = write_particles(0, 0, n, bed.particles.data()))) return rc;
    if ((rc = write_particles(1, 0, n, bed.affines.data()))) return rc;
    if ((rc = write_particles(2, 0, n, bed.extracts.data()))) return rc;
    if ((rc = check(cudaMemcpyAsync(lookup_.ptr, bed.lookup.data(), cells_ * sizeof(int32_t), cudaMemcpyHostToDevice,
                                    stream_),
                    "lookup upload")))
        return rc;
    return sync();
}

int Engine::sync() {
    int rc = check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
    if (rc) return rc;
    return collect();
}

// mod.rs:569-670 (write_uniforms), plus the WGSL constants of CsGeometry.
void Engine::fill_params(Params& u, float dt) const {
    const CsSettings& s = settings;
    u.gx = s.grid_dims[0];
    u.gy = s.grid_dims[1];
    u.gz = s.grid_dims[2];
    u.cells = u.gx * u.gy * u.gz;
    u.num_water = num_water;
    u.num_bed = num_bed;
    u.max_p = s.max_particles;
    u.use_sdf_cache = s.use_sdf_cache ? 1u : 0u;
    float dx = s.bounds_size[0] / (float)u.gx;
    float inv_dx = 1.0f / dx;
    u.dt = dt;
    u.gravity = s.gravity;
    u.dx = dx;
    u.inv_dx = inv_dx;
    u.ox = -s.bounds_size[0] * 0.5f;
    u.oy = -s.bounds_size[1] * 0.5f;
    u.oz = -s.bounds_size[2] * 0.5f;
    u.bx = s.bounds_size[0] * 0.5f;
    u.by = s.bounds_size[1] * 0.5f;
    u.bz = s.bounds_size[2] * 0.5f;
    u.bulk_K = s.bulk_modulus;
    u.viscosity = s.viscosity;
    u.nominal_mass = s.brew.water_mass_units_per_ml / s.brew.water_particles_per_ml;
    u.p_vol = dx * dx * dx * s.particle_volume_cells;
    u.vel_cap = s.max_velocity;
    u.outlet_r = s.brew.dripper_outlet_radius;
    u.top_r = s.brew.dripper_outlet_radius + s.geom.cone_radius_span;
    u.friction = s.geom.sdf_friction;
    u.restitution = s.geom.sdf_restitution;
    u.contact_offset = s.geom.contact_offset;
    u.nu_m2s = s.brew.water_kinematic_viscosity_m2_s;
    u.absorption_rate = s.brew.bed_absorption_rate;
    u.max_saturation = num_bed > 0 ? s.brew.target_bed_retention_ml * s.brew.water_mass_units_per_ml / (float)num_bed
                                   : 0.7f;
    u.min_perm = s.brew.min_bed_permeability_m2;
    u.extraction_rate = 0.01f;
    u.compaction_rate = s.brew.bed_compaction_rate;
    u.bed_damping = 8.5f;
    u.bed_impact = s.brew.bed_impact_rate;
    u.pore_capacity_scale = s.brew.bed_pore_capacity_scale;
    u.pore_overfill_alpha = s.brew.bed_pore_overfill_alpha;
    u.div_clamp = std::fmin(4.0f * s.max_velocity * inv_dx, FP_VALUE_LIMIT - 1.0f);
    u.p_clamp = FP_VALUE_LIMIT - 1.0f;
    // i32 lanes hold p * 2^18, so fixed-point storage clamps at the lane limit; FP32
    // storage has no such range and does not clamp
    u.p_limit = s.pressure_storage == CS_PRESSURE_FIXED_POINT ? u.p_clamp : 3.0e38f;
    u.j_alpha = 32.0f;
    u.j_expand_alpha = 2.0f;
    u.max_rest_frac = 1.20f;
    u.surface_void_scale = s.brew.bed_surface_void_scale;
    u.water_r_dx = s.brew.water_sample_radius_dx;
    u.bed_r_dx = s.brew.bed_sample_radius_dx;
    u.filter_absorption = s.brew.filter_absorption_rate_s;
    const CsGeometry& g = s.geom;
    u.geom_flags = g.flags;
    u.cone_bot_y = g.cone_bot_y;
    u.cone_top_y = g.cone_top_y;
    u.filter_center_y = g.filter_center_y;
    u.filter_top_rel = g.filter_top_rel;
    u.filter_bot_rel = g.filter_bot_rel;
    u.filter_top_radius = g.filter_top_radius;
    u.filter_thickness = g.filter_thickness;
    u.cup_top_y = g.cup_top_y;
    u.cup_radius = g.cup_radius;
    u.cup_floor_y = g.cup_floor_y;
    u.wall_thickness = g.wall_thickness;
    u.bed_surface_ref_y = g.bed_surface_ref_y;
    u.bed_surface_span = g.bed_surface_span;
    u.fixed_point = s.pressure_storage == CS_PRESSURE_FIXED_POINT ? 1u : 0u;
    u.int64_grid = s.p2g_mode == CS_P2G_INT64 ? 1u : 0u;
    u.p2g_tile = p2g_tile();
    u.ntx = (u.gx + u.p2g_tile) / u.p2g_tile;
    u.nty = (u.gy + u.p2g_tile) / u.p2g_tile;
    u.ntz = (u.gz + u.p2g_tile) / u.p2g_tile;
    u.warm = (s.warm_start != CS_WARM_NONE && !u.fixed_point && have_prev_p) ? 1u : 0u;
    u.omega = s.rbgs_omega > 0.0f ? s.rbgs_omega : 1.0f;
    u.first_check = s.first_check;
}

int Engine::upload_ctx() {
    prof_.h2d_bytes += sizeof(Ctx);
    int rc;
    if (!ctx_pinned_ &&
        (rc = check(cudaHostAlloc((void**)&ctx_pinned_, 2 * sizeof(Ctx), cudaHostAllocDefault), "pinned context")))
        return rc;
    for (cudaEvent_t& e : ctx_ev_)
        if (!e && (rc = check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "context event"))) return rc;
    ctx_slot_ ^= 1;
    if (ctx_ev_used_[ctx_slot_] && (rc = check(cudaEventSynchronize(ctx_ev_[ctx_slot_]), "context slot"))) return rc;
    std::memcpy(&ctx_pinned_[ctx_slot_], &ctx_, sizeof(Ctx));
    if ((rc = check(cudaMemcpyAsync(d_ctx_.ptr, &ctx_pinned_[ctx_slot_], sizeof(Ctx), cudaMemcpyHostToDevice, stream_),
                    "ctx upload")))
        return rc;
    ctx_ev_used_[ctx_slot_] = true;
    return check(cudaEventRecord(ctx_ev_[ctx_slot_], stream_), "context event");
}

// inflow.rs:122-242: plan on the host, build the samples, append them.
int Engine::emit(float dt) {
    uint32_t dropped = 0;
    uint32_t live = num_water + num_bed;
    uint32_t count = inflow.plan(settings, dt, live, &dropped);
    frame_dropped += dropped;
    total_dropped += dropped;
    jet_.count = 0;
    if (count == 0) return CS_OK;
    host::JetFrame jf = host::jet_frame(settings, inflow, dt, count, live);
    if (settings.device_emission) {
        // built by k_emit_jet after the context upload of this substep
        for (int k = 0; k < 3; ++k) {
            jet_.t1[k] = jf.t1[k];
            jet_.t2[k] = jf.t2[k];
            jet_.vel[k] = jf.vel[k];
            jet_.origin[k] = jf.origin[k];
        }
        jet_.jet_radius = jf.jet_radius;
        jet_.dt = jf.dt;
        jet_.particle_mass = jf.particle_mass;
        jet_.first_sequence = jf.first_sequence;
        jet_.count = jf.count;
        jet_.first_slot = jf.first_slot;
        inflow.sequence += count;
        frame_emitted_mass += (float)count * jf.particle_mass;
        total_emitted_mass += (float)count * jf.particle_mass;
        num_water += count;
        return CS_OK;
    }
    std::vector<float> parts((size_t)count * 8), affs((size_t)count * 12);
    host::emit_host(jf, parts.data(), affs.data());
    inflow.sequence += count;
    int rc;
    if ((rc = write_particles(0, live, count, parts.data()))) return rc;
    if ((rc = write_particles(1, live, count, affs.data()))) return rc;
    float pm = jf.particle_mass;
    frame_emitted_mass += (float)count * pm;
    total_emitted_mass += (float)count * pm;
    num_water += count;
    return CS_OK;
}

double Engine::residual() {
    const Ctx* dc = (const Ctx*)d_ctx_.ptr;
    mark(CS_PHASE_RESIDUAL);
    cudaMemsetAsync(resid_.ptr, 0, 2 * sizeof(double), stream_);
    k_residual<<<dim3(launch_cells_blocks(), 1), kThreads, 0, stream_>>>(dc);
    count_launch();
    double h[2] = {0.0, 0.0};
    cudaMemcpyAsync(h, resid_.ptr, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream_);
    prof_.d2h_bytes += sizeof(h);
    prof_.residual_evals += 1;
    cudaStreamSynchronize(stream_);
    if (h[1] <= 0.0) return 0.0;
    return std::sqrt(h[0]) / std::sqrt(h[1]);
}

double Engine::refine_residual() {
    const Ctx* dc = (const Ctx*)d_ctx_.ptr;
    mark(CS_PHASE_RESIDUAL);
    cudaMemsetAsync(resid_.ptr, 0, 2 * sizeof(double), stream_);
    k_refine_residual<<<dim3(launch_cells_blocks(), 1), kThreads, 0, stream_>>>(dc);
    count_launch();
    double h[2] = {0.0, 0.0};
    cudaMemcpyAsync(h, resid_.ptr, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream_);
    prof_.d2h_bytes += sizeof(h);
    prof_.residual_evals += 1;
    cudaStreamSynchronize(stream_);
    if (h[1] <= 0.0) return 0.0;
    return std::sqrt(h[0]) / std::sqrt(h[1]);
}

// The cluster-resident solve serves grids of at most kClusterMaxCells cells (unless the
// per-colour launches or the grid-wide solve are asked for); larger grids use the
// grid-wide solve, whose row segments cover only the rows that hold fluid.
bool Engine::use_cluster_solve() const {
    return sc_ranks_ > 0 && settings.rbgs_kernel != 1 && settings.rbgs_kernel != 4 && cells_ <= kClusterMaxCells;
}

// Grid-wide solve buffers (solver_grid.cuh), sized for the worst case: every row of
// the grid holding fluid across its whole width.
int Engine::gs_alloc() {
    const uint32_t gx = settings.grid_dims[0];
    const size_t rows = (size_t)settings.grid_dims[1] * settings.grid_dims[2];
    const size_t units = rows * ((gx + GS_UNIT - 1) / GS_UNIT);
    const size_t slots = units * GS_UNIT;
    int rc;
    if ((rc = alloc(gs_rows_, (2 * (rows + 1) + rows) * sizeof(uint32_t)))) return rc;
    if ((rc = alloc(gs_desc_, units * (sizeof(GsDesc) + 16 * sizeof(int))))) return rc;
    // the arrays read at neighbour slots (correction + fill code, pressure) get at least
    // gx / 2 + 64 slots of padding on both sides: a neighbour slot computed for a face that
    // is not a fluid face can fall up to gx / 2 + 33 slots outside the used range, and the
    // solve loads all six before the flags pick the real ones.  The padding is a whole
    // number of 128-byte lines, so every unit's slots start on a line of their own and the
    // lines of a CTA's rows hold no other CTA's slots (the solve reads those through L1).
    const size_t pad = (gx / 2 + 64 + 15) & ~(size_t)15;
    if ((rc = alloc(gs_slots_, (slots + 2 * pad) * 2 * sizeof(float2) + slots * (sizeof(float2) + 2 * sizeof(float)))))
        return rc;
    if ((rc = gs_blocks(&gs_ctas_))) return rc;
    if ((rc = alloc(gs_misc_, sc_align(2 * sizeof(double) * (size_t)std::max(gs_ctas_, 1)) + 256 +
                                  sc_align(sizeof(ScResult))))) return rc;
    size_t cub = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, cub, (uint32_t*)nullptr, (uint32_t*)nullptr, (int)rows + 1, stream_);
    if ((rc = alloc(gs_cub_, cub))) return rc;
    GsBuffers& g = gs_buf_;
    uint32_t* r = (uint32_t*)gs_rows_.ptr;
    g.row_units = r;
    g.row_start = r + rows + 1;
    g.row_xlo = r + 2 * (rows + 1);
    g.desc = (GsDesc*)gs_desc_.ptr;
    g.rec = (int*)((unsigned char*)gs_desc_.ptr + units * sizeof(GsDesc));
    float2* f2 = (float2*)gs_slots_.ptr;
    g.dfc = f2 + pad;
    g.p = f2 + (slots + 2 * pad) + pad;
    g.cf = f2 + 2 * (slots + 2 * pad);
    g.g = (float*)(g.cf + slots);
    g.b = g.g + slots;
    unsigned char* m = (unsigned char*)gs_misc_.ptr;
    g.part = (double*)m;
    g.sync = (uint32_t*)(m + sc_align(2 * sizeof(double) * (size_t)std::max(gs_ctas_, 1)));
    g.result = (ScResult*)(m + sc_align(2 * sizeof(double) * (size_t)std::max(gs_ctas_, 1)) + 256);
    g.cub_temp = gs_cub_.ptr;
    g.cub_bytes = cub;
    ctx_.gs = g;
    return CS_OK;
}

// Whole-GPU solve (solver_grid.cuh): row-segment prep, then one cooperative launch.
// `done` is false when the launch could not run on this device or a bounded wait ran
// out (the caller then solves with per-colour launches).
int Engine::solve_grid(uint32_t& sweeps, double& r0, double& r1, bool& done) {
    done = false;
    if (gs_ctas_ <= 0) return CS_OK;
    const Ctx* dc = (const Ctx*)d_ctx_.ptr;
    const CsSettings& s = settings;
    mark(CS_PHASE_RESIDUAL);
    int rc = gs_launch_prep(dc, &gs_buf_, s.grid_dims[1] * s.grid_dims[2], stream_, sms_);
    if (rc) return rc;
    count_launch(kGsPrepLaunches);
    mark(CS_PHASE_SWEEPS);
    if ((rc = gs_launch_solve(dc, gs_ctas_, s.residual_tol, s.max_sweeps, s.check_every, stream_))) return rc;
    count_launch();
    ScResult res;
    if ((rc = check(cudaMemcpyAsync(&res, gs_buf_.result, sizeof(res), cudaMemcpyDeviceToHost, stream_),
                    "grid solve result")))
        return rc;
    prof_.d2h_bytes += sizeof(res);
    if ((rc = sync())) return rc;
    if (res.status != 1) return CS_OK;
    sweeps = res.sweeps;
    r0 = res.r0;
    r1 = res.r1;
    prof_.residual_evals += res.evals;
    done = true;
    return CS_OK;
}

// One-launch solve on a thread-block cluster (solver_cluster.cuh).  `done` is false
// when the fluid cells exceed the cluster's shared-memory capacity.
int Engine::solve_cluster(uint32_t& sweeps, double& r0, double& r1, bool& done) {
    done = false;
    const Ctx* dc = (const Ctx*)d_ctx_.ptr;
    const uint32_t codes = (uint32_t)sc_codes_;
    mark(CS_PHASE_RESIDUAL);
    int rc = sc_launch_prep(dc, &sc_buf_, codes, sc_ranks_, 1, stream_, sms_);
    if (rc) return rc;
    count_launch(kScPrepLaunches);
    mark(CS_PHASE_SWEEPS);
    const CsSettings& s = settings;
    if ((rc = sc_launch_cluster(dc, sc_ranks_, 1, s.residual_tol, s.max_sweeps, s.check_every, stream_,
                                s.rbgs_kernel == 3 ? 0u : 1u)))
        return rc;
    count_launch();
    ScResult res;
    if ((rc = check(cudaMemcpyAsync(&res, sc_buf_.result, sizeof(res), cudaMemcpyDeviceToHost, stream_),
                    "solve result")))
        return rc;
    prof_.d2h_bytes += sizeof(res);
    if ((rc = sync())) return rc;
    if (res.status != 1) return CS_OK;
    sweeps = res.sweeps;
    r0 = res.r0;
    r1 = res.r1;
    prof_.residual_evals += res.evals;
    done = true;
    return CS_OK;
}

int Engine::solve_pressure(uint32_t& sweeps, double& r0, double& r1) {
    const Ctx* dc = (const Ctx*)d_ctx_.ptr;
    const CsSettings& s = settings;
    const uint32_t half = (s.grid_dims[0] + 1) / 2;
    const size_t ncol = (size_t)half * s.grid_dims[1] * s.grid_dims[2];
    const int blocks = (int)std::min<size_t>((ncol + kThreads - 1) / kThreads, (size_t)sms_ * 16);
    auto pair = [&]() {
        k_rbgs_colour<<<dim3(blocks, 1), kThreads, 0, stream_>>>(dc, 0u);
        k_rbgs_colour<<<dim3(blocks, 1), kThreads, 0, stream_>>>(dc, 1u);
        count_launch(2);
    };
    sweeps = 0;
    r0 = r1 = -1.0;
    const uint64_t evals0 = prof_.residual_evals;
    const bool refine = s.solve_mode == CS_SOLVE_RESIDUAL && s.pressure_storage != CS_PRESSURE_FIXED_POINT;
    if (refine && use_cluster_solve()) {
        bool done = false;
        int rc = solve_cluster(sweeps, r0, r1, done);
        if (rc) return rc;
        if (done) {
            last.residual_checks = (uint32_t)(prof_.residual_evals - evals0);
            return CS_OK;
        }
    }
    if (refine && s.rbgs_kernel != 1) {
        bool done = false;
        int rc = solve_grid(sweeps, r0, r1, done);
        if (rc) return rc;
        if (done) {
            last.residual_checks = (uint32_t)(prof_.residual_evals - evals0);
            return CS_OK;
        }
    }
    if (refine) {
        const uint32_t ce = s.check_every ? s.check_every : 10;
        r0 = refine_residual();
        r1 = r0;
        uint32_t next = s.first_check ? s.first_check : ce;
        while (!(r1 <= (double)s.residual_tol) && sweeps < s.max_sweeps) {
            uint32_t k = std::min(next, s.max_sweeps - sweeps);
            mark(CS_PHASE_SWEEPS);
            for (uint32_t j = 0; j < k; ++j) {
                k_refine_sweep<<<dim3(blocks, 1), kThreads, 0, stream_>>>(dc, 0u);
                k_refine_sweep<<<dim3(blocks, 1), kThreads, 0, stream_>>>(dc, 1u);
                count_launch(2);
            }
            sweeps += k;
            mark(CS_PHASE_RESIDUAL);
            k_refine_accumulate<<<dim3(launch_cells_blocks(), 1), kThreads, 0, stream_>>>(dc);
            count_launch();
            const double r_before = r1;
            r1 = refine_residual();
            next = sc_next_interval(r1, r_before, k, (double)s.residual_tol, ce);
        }
    } else if (s.solve_mode == CS_SOLVE_RESIDUAL) {
        uint32_t ce = s.check_every ? s.check_every : 1;
        r0 = residual();
        r1 = r0;
        if (!(r0 <= (double)s.residual_tol)) {
            while (sweeps < s.max_sweeps) {
                mark(CS_PHASE_SWEEPS);
                pair();
                ++sweeps;
                if (sweeps % ce == 0 || sweeps == s.max_sweeps) {
                    r1 = residual();
                    if (r1 <= (double)s.residual_tol) break;
                }
            }
        }
    } else {
        mark(CS_PHASE_SWEEPS);
        for (uint32_t k = 0; k < s.pressure_rbgs_pairs; ++k) pair();
        sweeps = s.pressure_rbgs_pairs;
        if (s.check_every) r1 = residual();
    }
    last.residual_checks = (uint32_t)(prof_.residual_evals - evals0);
    return check(cudaGetLastError(), "rbgs");
}

// mod.rs:271-419, one substep.  `passes` limits how many reference dispatches run
// (numbered in the order of mod.rs:317-414, each number fixed).  The host part (jet
// plan, uniforms, context upload) runs here; the device work is enqueued directly or,
// in graph mode, replayed from a captured graph.
int Engine::substep(float sub_dt, uint32_t P) {
    int rc;
    const bool graph = settings.use_graph && P == 0xffffffffu;
    if (graph && l_capture_) {
        set_error("training-sample capture runs with use_graph = 0");
        return CS_ERR_UNSUPPORTED;
    }
    if (settings.reorder_every && substeps_done_ % settings.reorder_every == 0 && (rc = reorder())) return rc;
    substeps_done_ += 1;
    if (!graph) mark(CS_PHASE_EMIT);
    if ((rc = emit(sub_dt))) return rc;
    fill_params(ctx_.u, sub_dt);
    ctx_.u.jet = jet_;
    if ((rc = upload_ctx())) return rc;
    if (graph) return substep_graph(sub_dt);
    uint32_t sweeps = 0;
    double r0 = -1.0, r1 = -1.0;
    last.residual_checks = 0;
    if ((rc = enqueue(P, false, sweeps, r0, r1))) return rc;
    total_time += sub_dt;
    last.last_sweeps = sweeps;
    last.last_residual = r1;
    last.initial_residual = r0;
    prof_.sweeps += sweeps;
    prof_.substeps += 1;
    return CS_OK;
}

// Reorder the water samples' slots by the tile of their P2G base cell (a stable radix
// sort of the keys, then a gather of every particle stream): samples of one tile sit in
// consecutive slots, so the sorted P2G reads them in order and G2P's warps gather nodes
// of neighbouring cells.  Bed samples keep their slots (bed ids index the lookup and the
// bed deltas).  The CPU oracle applies the same stable permutation.  Launched directly
// ahead of the substep's work (also in graph mode).
int Engine::reorder() {
    const uint32_t n = num_water;
    if (n < 2) return CS_OK;
    const Ctx* dc = (const Ctx*)d_ctx_.ptr;
    fill_params(ctx_.u, 0.0f);
    int rc = upload_ctx();
    if (rc) return rc;
    uint32_t* keys = (uint32_t*)ro_keys_.ptr;
    uint32_t* idx = (uint32_t*)ro_idx_.ptr;
    const size_t mp = settings.max_particles;
    const int pb = launch_particle_blocks(n);
    k_reorder_keys<<<dim3(pb, 1), kThreads, 0, stream_>>>(dc, keys, idx);
    const uint32_t tiles = p2g_tiles_;
    int end_bit = 1;
    while (end_bit < 32 && (1u << end_bit) <= tiles) ++end_bit;
    size_t temp = ro_cub_.bytes;
    if ((rc = check(cub::DeviceRadixSort::SortPairs(ro_cub_.ptr, temp, keys, keys + mp, idx, idx + mp, (int)n, 0,
                                                    end_bit, stream_),
                    "reorder sort")))
        return rc;
    DeviceBuffer* streams[] = {&pos_, &vel_, &c0_, &c1_, &c2_, &bedA_, &bedB_};
    for (DeviceBuffer* b : streams) {
        float4* base = (float4*)b->ptr;
        k_reorder_gather<<<dim3(pb, 1), kThreads, 0, stream_>>>(base, (float4*)ro_tmp_.ptr, idx + mp, num_bed, n);
        if ((rc = check(cudaMemcpyAsync(base + num_bed, ro_tmp_.ptr, (size_t)n * sizeof(float4),
                                        cudaMemcpyDeviceToDevice, stream_),
                        "reorder copy")))
            return rc;
    }
    count_launch(1 + 7);
    return check(cudaGetLastError(), "reorder");
}

// The device work of one substep.  With `capture`, the stream is being captured into a
// graph that later substeps replay: launch shapes then cover max_particles, every
// kernel launches (particle counts live in the uploaded context), phases are not
// marked, and the solve's result goes to the running totals instead of the host.
int Engine::enqueue(uint32_t P, bool capture, uint32_t& sweeps, double& r0, double& r1) {
    int rc;
    const Ctx* dc = (const Ctx*)d_ctx_.ptr;
    const uint32_t np = capture ? settings.max_particles : num_water + num_bed;
    const bool any_p = capture || np > 0, any_bed = capture || num_bed > 0;
    const int cb = launch_cells_blocks();
    const int pb = launch_particle_blocks_pt(np);
    const dim3 TP(particle_threads());
    const int bb = launch_particle_blocks(capture ? settings.max_particles : num_bed);
    // the bed-lookup scatter (27 atomicMax per bed sample, a few thousand samples) runs in
    // warp-sized blocks so that it spreads over the SMs (clear phase 27.7 -> 23.5 us)
    const int bb32 = (int)std::max<size_t>(
        1, std::min<size_t>(((size_t)(capture ? settings.max_particles : num_bed) + 31) / 32, (size_t)sms_ * 16));
    const dim3 T(kThreads);
    auto ph = [&](int phase) {
        if (!capture) mark(phase);
    };
#define CS_LAUNCH(...)  \
    do {                \
        __VA_ARGS__;    \
        count_launch(); \
    } while (0)
    if (capture) {
        CS_LAUNCH(k_emit_jet<<<dim3(16, 1), T, 0, stream_>>>(dc));
    } else if (jet_.count) {
        CS_LAUNCH(k_emit_jet<<<dim3(launch_particle_blocks(jet_.count), 1), T, 0, stream_>>>(dc));
    }
    ph(CS_PHASE_CLEAR);
    // clear_buffer(grid), clear_buffer(grid_vel) (mod.rs:308-309).  In int64 mode (fixed at
    // creation) P2G accumulates in lanes64, and a full substep writes every int32 lane it
    // reads for every cell before reading it: the kind (lane 3) and, with fixed-point
    // storage, pressure and divergence (lanes 0, 1) in classify, the packing pressure
    // (lane 2) in project, the viscosity scratch (lanes 1-3) in viscosity_prepare; lanes
    // 4 and 5 are written only by the int32 P2G modes.  So only a partial substep, whose
    // lanes are compared pass by pass, clears them.
    if (settings.p2g_mode != CS_P2G_INT64 || P <= 20) cudaMemsetAsync(lanes_.ptr, 0, lanes_.bytes, stream_);
    cudaMemsetAsync(gvel_.ptr, 0, gvel_.bytes, stream_);
    if (settings.p2g_mode == CS_P2G_INT64) cudaMemsetAsync(lanes64_.ptr, 0, lanes64_.bytes, stream_);
    if (P > 0) cudaMemsetAsync(metrics_.ptr, 0, metrics_.bytes, stream_);
    if (P > 1) cudaMemsetAsync(lookup_.ptr, 0xff, lookup_.bytes, stream_);
    if (P > 2 && any_bed) CS_LAUNCH(k_bed_lookup_scatter<<<dim3(bb32, 1), 32, 0, stream_>>>(dc));
    ph(CS_PHASE_P2G);
    if (P > 3 && any_p) {
        if (settings.p2g_mode != CS_P2G_ATOMIC32) {
            cudaMemsetAsync(tile_count_.ptr, 0, tile_count_.bytes, stream_);
            CS_LAUNCH(k_p2g_keys<<<dim3(pb, 1), TP, 0, stream_>>>(dc));
            size_t temp = tile_temp_.bytes;
            cub::DeviceScan::ExclusiveSum(tile_temp_.ptr, temp, (const uint32_t*)tile_count_.ptr,
                                          (uint32_t*)tile_start_.ptr, (int)p2g_tile_count() + 1, stream_);
            CS_LAUNCH(k_p2g_scatter<<<dim3(pb, 1), TP, 0, stream_>>>(dc));
            CS_LAUNCH(launch_p2g_tiles(dc, 1, stream_));
        } else {
            CS_LAUNCH(k_p2g_atomic<<<dim3(pb, 1), TP, 0, stream_>>>(dc));
        }
    }
    ph(CS_PHASE_GRID);
    if (P > 4) CS_LAUNCH(k_grid_update<<<dim3(cb, 1), T, 0, stream_>>>(dc, P > 5 ? 1 : 0));
    if (P > 6) {
        if (any_bed) CS_LAUNCH(k_bed_velocity<<<dim3(cb, 1), T, 0, stream_>>>(dc));
        CS_LAUNCH(k_classify<<<dim3(cb, 1), T, 0, stream_>>>(dc));
    }
    if (P > 7) {
        if (capture) {
            const CsSettings& s = settings;
            if (s.solve_mode == CS_SOLVE_RESIDUAL) {
                if (s.warm_start == CS_WARM_LEARNED && (rc = learned_enqueue(false))) return rc;
                if (use_cluster_solve()) {
                    if ((rc = sc_launch_prep(dc, &sc_buf_, (uint32_t)sc_codes_, sc_ranks_, 1, stream_, sms_)))
                        return rc;
                    count_launch(kScPrepLaunches);
                    if ((rc = sc_launch_cluster(dc, sc_ranks_, 1, s.residual_tol, s.max_sweeps, s.check_every,
                                                stream_, s.rbgs_kernel == 3 ? 0u : 1u)))
                        return rc;
                    count_launch();
                    CS_LAUNCH(k_sc_account<<<1, 1, 0, stream_>>>(sc_buf_.result, (ScTotals*)sc_totals_.ptr));
                } else {
                    if ((rc = gs_launch_prep(dc, &gs_buf_, s.grid_dims[1] * s.grid_dims[2], stream_, sms_)))
                        return rc;
                    count_launch(kGsPrepLaunches);
                    if ((rc = gs_launch_solve(dc, gs_ctas_, s.residual_tol, s.max_sweeps, s.check_every, stream_)))
                        return rc;
                    count_launch();
                    CS_LAUNCH(k_sc_account<<<1, 1, 0, stream_>>>(gs_buf_.result, (ScTotals*)sc_totals_.ptr));
                }
            } else {
                const uint32_t half = (s.grid_dims[0] + 1) / 2;
                const size_t ncol = (size_t)half * s.grid_dims[1] * s.grid_dims[2];
                const int blocks = (int)std::min<size_t>((ncol + kThreads - 1) / kThreads, (size_t)sms_ * 16);
                for (uint32_t k = 0; k < s.pressure_rbgs_pairs; ++k) {
                    CS_LAUNCH(k_rbgs_colour<<<dim3(blocks, 1), T, 0, stream_>>>(dc, 0u));
                    CS_LAUNCH(k_rbgs_colour<<<dim3(blocks, 1), T, 0, stream_>>>(dc, 1u));
                }
            }
        } else {
            if ((rc = learned_enqueue(true))) return rc;
            if ((rc = solve_pressure(sweeps, r0, r1))) return rc;
            if ((rc = learned_collect())) return rc;
            if ((rc = learned_after_solve())) return rc;
        }
        have_prev_p = true;
    }
    ph(CS_PHASE_PROJECT);
    if (P > 8) CS_LAUNCH(k_project<<<dim3(cb, 1), T, 0, stream_>>>(dc, 1 | (P > 9 ? 2 : 0) | (P > 10 ? 4 : 0)));
    if (P > 11) CS_LAUNCH(k_packing_apply<<<dim3(cb, 1), T, 0, stream_>>>(dc, P > 12 ? 1 : 0));
    if (P > 13) CS_LAUNCH(k_viscosity_prepare<<<dim3(cb, 1), T, 0, stream_>>>(dc));
    if (P > 14) CS_LAUNCH(k_viscosity_apply<<<dim3(cb, 1), T, 0, stream_>>>(dc, P > 15 ? 1 : 0));
    ph(CS_PHASE_G2P);
    if (P > 16 && any_p) CS_LAUNCH(k_g2p<<<dim3(pb, 1), TP, 0, stream_>>>(dc));
    ph(CS_PHASE_BED);
    if (P > 17 && any_p) CS_LAUNCH(k_bed_coupling<<<dim3(pb, 1), TP, 0, stream_>>>(dc));
    if (P > 18 && any_bed) CS_LAUNCH(k_extraction_advect<<<dim3(bb, 1), T, 0, stream_>>>(dc));
    if (P > 19 && any_bed) CS_LAUNCH(k_bed_dynamics<<<dim3(bb, 1), T, 0, stream_>>>(dc));
    ph(CS_PHASE_RENDER);
    if (P > 20 && any_p) CS_LAUNCH(k_prepare_render<<<dim3(pb, 1), TP, 0, stream_>>>(dc));
#undef CS_LAUNCH
    ph(-1);
    return check(cudaGetLastError(), "substep launch");
}

Engine::GraphKey Engine::graph_key() const {
    GraphKey k;
    std::memset(&k, 0, sizeof(k));
    const CsSettings& s = settings;
    k.p2g_mode = s.p2g_mode;
    k.check_every = s.check_every;
    k.max_sweeps = s.max_sweeps;
    k.solve_mode = s.solve_mode;
    k.pressure_storage = s.pressure_storage;
    k.rbgs_kernel = s.rbgs_kernel;
    k.warm_start = s.warm_start;
    k.rbgs_pairs = s.pressure_rbgs_pairs;
    k.residual_tol = s.residual_tol;
    k.num_bed = num_bed;
    k.max_particles = s.max_particles;
    k.p2g_tile = p2g_tile();
    k.particle_threads = particle_threads();
    return k;
}

// Graph mode: capture the device work once (again when a captured setting changes)
// and replay it; the host does not wait for the substep.
int Engine::substep_graph(float sub_dt) {
    int rc;
    const GraphKey key = graph_key();
    if (!gexec_ || !(key == gkey_)) {
        if (gexec_) {
            cudaGraphExecDestroy(gexec_);
            gexec_ = nullptr;
        }
        if (settings.solve_mode == CS_SOLVE_RESIDUAL && !use_cluster_solve() && gs_ctas_ <= 0) {
            set_error("graph mode needs the cluster-resident or the grid-wide solve, neither of which this "
                      "device can launch");
            return CS_ERR_UNSUPPORTED;
        }
        const uint64_t before = prof_.launches;
        if ((rc = check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture")))
            return rc;
        uint32_t sweeps = 0;
        double r0 = -1.0, r1 = -1.0;
        const int erc = enqueue(0xffffffffu, true, sweeps, r0, r1);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(stream_, &g);
        graph_launches_ = (uint32_t)(prof_.launches - before);
        prof_.launches = before;
        if (erc) {
            if (g) cudaGraphDestroy(g);
            return erc;
        }
        if ((rc = check(ce, "end capture"))) return rc;
        rc = check(cudaGraphInstantiate(&gexec_, g, 0), "graph instantiate");
        cudaGraphDestroy(g);
        if (rc) return rc;
        gkey_ = key;
    }
    if ((rc = check(cudaGraphLaunch(gexec_, stream_), "graph launch"))) return rc;
    prof_.launches += graph_launches_;
    prof_.substeps += 1;
    total_time += sub_dt;
    have_prev_p = true;
    graph_pending_ = true;
    return CS_OK;
}

// The error of the replayed solves counted between two readings of the totals: a solve
// whose fluid did not fit the cluster (capacity) or one whose bounded waits ran out.
int Engine::totals_error(const ScTotals& t, const ScTotals& before) {
    if (t.failed != before.failed) {
        set_error("a replayed substep's pressure solve did not fit the thread-block cluster "
                  "(16 x 4095 fluid cells); run this scene with use_graph = 0");
        return CS_ERR_CAPACITY;
    }
    if (t.timeouts != before.timeouts) {
        set_error("a replayed substep's pressure solve gave up waiting for a neighbouring CTA "
                  "(bounded wait ran out); the pressure of that substep is not solved");
        return CS_ERR_TIMEOUT;
    }
    return CS_OK;
}

// Solve totals of the replayed substeps since the last call: sweep and residual
// counters, the latest substep's metrics, and an error if a solve did not complete.
int Engine::collect() {
    if (!graph_pending_) return CS_OK;
    graph_pending_ = false;
    ScTotals t;
    int rc = check(cudaMemcpyAsync(&t, sc_totals_.ptr, sizeof(t), cudaMemcpyDeviceToHost, stream_), "totals");
    if (rc) return rc;
    prof_.d2h_bytes += sizeof(t);
    if ((rc = check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize"))) return rc;
    prof_.sweeps += t.sweeps - seen_.sweeps;
    prof_.residual_evals += t.evals - seen_.evals;
    const int err = totals_error(t, seen_);
    seen_ = t;
    if (t.runs) {
        last.last_sweeps = t.last.sweeps;
        last.residual_checks = t.last.evals;
        last.last_residual = t.last.r1;
        last.initial_residual = t.last.r0;
    }
    if (err) return err;
    return learned_collect();
}

// mod.rs:264-270
int Engine::step_frame(float dt) {
    float fdt = std::fmin(dt, settings.max_frame_dt);
    uint32_t n = settings.substeps > 1 ? settings.substeps : 1;
    float sdt = fdt / (float)n;
    frame_emitted_mass = 0.0f;
    frame_dropped = 0;
    for (uint32_t k = 0; k < n; ++k) {
        int rc = substep(sdt, 0xffffffffu);
        if (rc) return rc;
    }
    return CS_OK;
}

int Engine::metrics(CsMetrics* out) {
    uint32_t m[8];
    prof_.d2h_bytes += sizeof(m);
    int rc = check(cudaMemcpyAsync(m, metrics_.ptr, sizeof(m), cudaMemcpyDeviceToHost, stream_), "metrics");
    if (rc) return rc;
    if ((rc = sync())) return rc;
    *out = last;
    out->max_abs_div = (float)m[M_MAX_DIV] * (1.0f / METRICS_DIV_FP_SCALE);
    out->fluid_cells = m[M_FLUID];
    out->div_clamp_fires = m[M_DIV_CLAMP];
    out->pressure_clamp_fires = m[M_P_CLAMP];
    out->mass_overflow_fires = m[M_OVERFLOW];
    out->nan_flag = m[M_NAN];
    out->timeout_flag = m[M_TIMEOUT];
    return CS_OK;
}

int Engine::metrics_request() {
    if (mreq_) {
        set_error("a metrics request is already pending");
        return CS_ERR_INVALID_ARG;
    }
    mreq_totals_ = false;
    if (settings.warm_start == CS_WARM_LEARNED) {  // the wait reads synchronously
        mreq_ = true;
        return CS_OK;
    }
    int rc;
    if (!mstage_ &&
        (rc = check(cudaHostAlloc((void**)&mstage_, sizeof(MetricsStage), cudaHostAllocDefault), "pinned stage")))
        return rc;
    if (!mevent_ && (rc = check(cudaEventCreateWithFlags(&mevent_, cudaEventDisableTiming), "event"))) return rc;
    if ((rc = check(cudaMemcpyAsync(mstage_->m, metrics_.ptr, sizeof(mstage_->m), cudaMemcpyDeviceToHost, stream_),
                    "metrics request")))
        return rc;
    prof_.d2h_bytes += sizeof(mstage_->m);
    mreq_totals_ = graph_pending_;
    if (mreq_totals_) {
        if ((rc = check(cudaMemcpyAsync(&mstage_->t, sc_totals_.ptr, sizeof(ScTotals), cudaMemcpyDeviceToHost, stream_),
                        "totals request")))
            return rc;
        prof_.d2h_bytes += sizeof(ScTotals);
    }
    mreq_last_ = last;
    if ((rc = check(cudaEventRecord(mevent_, stream_), "metrics event"))) return rc;
    mreq_ = true;
    return CS_OK;
}

int Engine::metrics_wait(CsMetrics* out) {
    if (!mreq_) {
        set_error("no metrics request is pending");
        return CS_ERR_INVALID_ARG;
    }
    mreq_ = false;
    if (settings.warm_start == CS_WARM_LEARNED) return metrics(out);
    int rc = check(cudaEventSynchronize(mevent_), "metrics wait");
    if (rc) return rc;
    CsMetrics r = mreq_last_;
    if (mreq_totals_) {
        const ScTotals t = mstage_->t;
        int err = 0;
        if (t.runs >= seen_.runs) {  // not already accounted by a later synchronising call
            prof_.sweeps += t.sweeps - seen_.sweeps;
            prof_.residual_evals += t.evals - seen_.evals;
            err = totals_error(t, seen_);
            seen_ = t;
        }
        if (t.runs) {
            r.last_sweeps = t.last.sweeps;
            r.residual_checks = t.last.evals;
            r.last_residual = t.last.r1;
            r.initial_residual = t.last.r0;
        }
        if (err) return err;
    }
    const uint32_t* m = mstage_->m;
    r.max_abs_div = (float)m[M_MAX_DIV] * (1.0f / METRICS_DIV_FP_SCALE);
    r.fluid_cells = m[M_FLUID];
    r.div_clamp_fires = m[M_DIV_CLAMP];
    r.pressure_clamp_fires = m[M_P_CLAMP];
    r.mass_overflow_fires = m[M_OVERFLOW];
    r.nan_flag = m[M_NAN];
    r.timeout_flag = m[M_TIMEOUT];
    *out = r;
    return CS_OK;
}

// what: 0 particles (8 f32), 1 affine (12 f32), 2 bed_extract (8 f32), 3 render (8 f32)
int Engine::read_particles(int what, uint32_t first, uint32_t count, float* out) {
    if ((uint64_t)first + count > settings.max_particles) {
        set_error("readback range beyond max_particles");
        return CS_ERR_INVALID_ARG;
    }
    if (count == 0) return CS_OK;
    size_t width = what == 1 ? 12 : 8;
    k_pack_particles<<<dim3(launch_particle_blocks(count), 1), kThreads, 0, stream_>>>(
        (const Ctx*)d_ctx_.ptr, first, count, (float*)staging_.ptr, what);
    int rc = check(cudaMemcpyAsync(out, staging_.ptr, (size_t)count * width * sizeof(float), cudaMemcpyDeviceToHost,
                                   stream_),
                   "readback");
    if (rc) return rc;
    return sync();
}

int Engine::write_particles(int what, uint32_t first, uint32_t count, const float* in) {
    if ((uint64_t)first + count > settings.max_particles) {
        set_error("upload range beyond max_particles");
        return CS_ERR_INVALID_ARG;
    }
    if (count == 0) return CS_OK;
    size_t width = what == 1 ? 12 : 8;
    int rc = upload_ctx();
    if (rc) return rc;
    prof_.h2d_bytes += (uint64_t)count * width * sizeof(float);
    if ((rc = check(cudaMemcpyAsync(staging_.ptr, in, (size_t)count * width * sizeof(float), cudaMemcpyHostToDevice,
                                    stream_),
                    "upload")))
        return rc;
    k_unpack_particles<<<dim3(launch_particle_blocks(count), 1), kThreads, 0, stream_>>>(
        (const Ctx*)d_ctx_.ptr, first, count, (const float*)staging_.ptr, what);
    // the staging buffer is reused by the next upload: wait for this one
    return sync();
}

int Engine::read_lanes64(int64_t* out) {
    int rc = check(cudaMemcpyAsync(out, lanes64_.ptr, lanes64_.bytes, cudaMemcpyDeviceToHost, stream_), "lanes64");
    if (rc) return rc;
    return sync();
}

int Engine::read_lanes(int32_t* out) {
    int rc = check(cudaMemcpyAsync(out, lanes_.ptr, cells_ * 6 * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_),
                   "lanes");
    if (rc) return rc;
    if (settings.pressure_storage != CS_PRESSURE_FIXED_POINT) {
        k_lane0_encode<<<dim3(launch_cells_blocks(), 1), kThreads, 0, stream_>>>((const Ctx*)d_ctx_.ptr,
                                                                                (int32_t*)staging_.ptr);
        if ((rc = check(cudaMemcpyAsync(out, staging_.ptr, cells_ * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_),
                        "lane0")))
            return rc;
    }
    return sync();
}
int Engine::read_gvel(float* out) {
    int rc = check(cudaMemcpyAsync(out, gvel_.ptr, cells_ * 16, cudaMemcpyDeviceToHost, stream_), "grid_vel");
    return rc ? rc : sync();
}
int Engine::read_pressure(float* out) {
    k_pressure_out<<<dim3(launch_cells_blocks(), 1), kThreads, 0, stream_>>>((const Ctx*)d_ctx_.ptr,
                                                                           (float*)staging_.ptr);
    int rc = check(cudaMemcpyAsync(out, staging_.ptr, cells_ * 4, cudaMemcpyDeviceToHost, stream_), "pressure");
    return rc ? rc : sync();
}
int Engine::read_kind(int32_t* out) {
    int rc = check(cudaMemcpyAsync(out, (int32_t*)lanes_.ptr + 3 * cells_, cells_ * 4, cudaMemcpyDeviceToHost, stream_),
                   "kind");
    return rc ? rc : sync();
}
int Engine::read_solver_inputs(float* fill, float* div) {
    if (settings.pressure_storage == CS_PRESSURE_FIXED_POINT) {
        set_error("the solver's divergence array exists in FP32 pressure storage only");
        return CS_ERR_UNSUPPORTED;
    }
    int rc = check(cudaMemcpyAsync(fill, fill_.ptr, cells_ * 4, cudaMemcpyDeviceToHost, stream_), "fill");
    if (!rc) rc = check(cudaMemcpyAsync(div, divf_.ptr, cells_ * 4, cudaMemcpyDeviceToHost, stream_), "divergence");
    return rc ? rc : sync();
}
int Engine::read_lookup(int32_t* out) {
    int rc = check(cudaMemcpyAsync(out, lookup_.ptr, cells_ * 4, cudaMemcpyDeviceToHost, stream_), "lookup");
    return rc ? rc : sync();
}
int Engine::read_delta(int32_t* out) {
    int rc = check(cudaMemcpyAsync(out, delta_.ptr, delta_.bytes, cudaMemcpyDeviceToHost, stream_), "delta");
    return rc ? rc : sync();
}
int Engine::read_sdf(float* out) {
    int rc = check(cudaMemcpyAsync(out, sdf_.ptr, sdf_.bytes, cudaMemcpyDeviceToHost, stream_), "sdf");
    return rc ? rc : sync();
}
int Engine::read_class(uint8_t* out) {
    int rc = check(cudaMemcpyAsync(out, cls_.ptr, cells_, cudaMemcpyDeviceToHost, stream_), "class");
    return rc ? rc : sync();
}

// Shader-style trilinear SDF sample on the host copy (shader.rs:678-699), used by
// the water-block generator's open-space filter.
static float host_sample_sdf(const std::vector<float>& sdf, const CsSettings& s, float px, float py, float pz) {
    float b[3] = {s.bounds_size[0] * 0.5f, s.bounds_size[1] * 0.5f, s.bounds_size[2] * 0.5f};
    float p[3] = {px, py, pz};
    int base[3];
    float f[3];
    for (int a = 0; a < 3; ++a) {
        float bs = b[a] * 2.0f;
        float uv = (p[a] + b[a]) / bs * (float)SDF_RES - 0.5f;
        float fl = std::floor(uv);
        base[a] = (int)fl;
        f[a] = uv - fl;
    }
    auto tex = [&](int x, int y, int z) {
        x = std::min(std::max(x, 0), SDF_RES - 1);
        y = std::min(std::max(y, 0), SDF_RES - 1);
        z = std::min(std::max(z, 0), SDF_RES - 1);
        return sdf[((size_t)z * SDF_RES + y) * SDF_RES + x];
    };
    auto mixh = [](float a, float bb, float t) { return a * (1.0f - t) + bb * t; };
    float c00 = mixh(tex(base[0], base[1], base[2]), tex(base[0] + 1, base[1], base[2]), f[0]);
    float c10 = mixh(tex(base[0], base[1] + 1, base[2]), tex(base[0] + 1, base[1] + 1, base[2]), f[0]);
    float c01 = mixh(tex(base[0], base[1], base[2] + 1), tex(base[0] + 1, base[1], base[2] + 1), f[0]);
    float c11 = mixh(tex(base[0], base[1] + 1, base[2] + 1), tex(base[0] + 1, base[1] + 1, base[2] + 1), f[0]);
    return mixh(mixh(c00, c10, f[1]), mixh(c01, c11, f[1]), f[2]);
}

int Engine::add_water_block(const float lo[3], const float hi[3], uint32_t per_axis, float jitter, uint32_t seed,
                            uint32_t require_open_sdf, uint32_t* added) {
    host::WaterBlock wb = host::water_block(settings, lo, hi, per_axis, jitter, seed);
    std::vector<float> parts;
    size_t n_all = wb.xyz.size() / 3;
    const float pm = settings.brew.water_mass_units_per_ml / settings.brew.water_particles_per_ml;
    for (size_t k = 0; k < n_all; ++k) {
        float x = wb.xyz[3 * k], y = wb.xyz[3 * k + 1], z = wb.xyz[3 * k + 2];
        if (require_open_sdf && !(host_sample_sdf(sdf_host_, settings, x, y, z) > settings.geom.contact_offset)) continue;
        float row[8] = {x, y, z, 1.0f, 0.0f, 0.0f, 0.0f, pm};
        parts.insert(parts.end(), row, row + 8);
    }
    uint32_t cnt = (uint32_t)(parts.size() / 8);
    uint32_t live = num_water + num_bed;
    if ((uint64_t)live + cnt > settings.max_particles) {
        set_error("water block exceeds max_particles");
        return CS_ERR_CAPACITY;
    }
    std::vector<float> affs((size_t)cnt * 12, 0.0f);
    int rc;
    if ((rc = write_particles(0, live, cnt, parts.data()))) return rc;
    if ((rc = write_particles(1, live, cnt, affs.data()))) return rc;
    num_water += cnt;
    if (added) *added = cnt;
    return CS_OK;
}

// ---- profiling ----
cudaEvent_t Engine::take_event() {
    if (!free_events_.empty()) {
        cudaEvent_t e = free_events_.back();
        free_events_.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void Engine::mark(int phase) {
    if (!prof_on_) {
        cur_phase_ = phase;
        return;
    }
    if (phase == cur_phase_) return;
    if (cur_phase_ < 0 && phase < 0) return;
    cudaEvent_t e = take_event();
    cudaEventRecord(e, stream_);
    if (cur_phase_ >= 0) spans_.push_back(PhaseSpan{cur_phase_, cur_event_, e});
    cur_phase_ = phase;
    cur_event_ = phase >= 0 ? e : nullptr;
}

int Engine::profile_enable(bool on) {
    int rc = sync();
    if (rc) return rc;
    for (auto& sp : spans_) {
        free_events_.push_back(sp.a);
        free_events_.push_back(sp.b);
    }
    spans_.clear();
    std::memset(&prof_, 0, sizeof(prof_));
    prof_on_ = on;
    cur_phase_ = -1;
    cur_event_ = nullptr;
    return CS_OK;
}

int Engine::profile_read(CsProfile* out) {
    int rc = sync();
    if (rc) return rc;
    std::vector<cudaEvent_t> seen;
    for (auto& sp : spans_) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, sp.a, sp.b) == cudaSuccess) prof_.phase_ms[sp.phase] += ms;
        seen.push_back(sp.a);
        seen.push_back(sp.b);
    }
    spans_.clear();
    std::sort(seen.begin(), seen.end());
    seen.erase(std::unique(seen.begin(), seen.end()), seen.end());
    for (cudaEvent_t e : seen) free_events_.push_back(e);
    *out = prof_;
    return CS_OK;
}

int Engine::timer_start() {
    if (!t0_) cudaEventCreate(&t0_);
    if (!t1_) cudaEventCreate(&t1_);
    return check(cudaEventRecord(t0_, stream_), "timer start");
}

int Engine::timer_stop(float* ms) {
    if (!t0_) {
        set_error("timer not started");
        return CS_ERR_INVALID_ARG;
    }
    int rc = check(cudaEventRecord(t1_, stream_), "timer stop");
    if (rc) return rc;
    if ((rc = check(cudaEventSynchronize(t1_), "timer sync"))) return rc;
    return check(cudaEventElapsedTime(ms, t0_, t1_), "timer elapsed");
}

int Engine::flush_l2() {
    if (!flush_.ptr) {
        int rc = alloc(flush_, (size_t)512 << 20);
        if (rc) return rc;
    }
    return check(cudaMemsetAsync(flush_.ptr, (int)(prof_.substeps & 0xff), flush_.bytes, stream_), "flush");
}

// ---- checkpoint: host state + particle streams + warm-start pressure ----
struct SnapHeader {
    uint64_t magic;
    uint32_t version, max_p;
    uint64_t cells;
    uint32_t num_water, num_bed;
    float total_time, total_emitted_mass;
    uint32_t total_dropped, have_prev_p;
    host::Inflow inflow;
    CsSpout spout;  // set_spout_position / set_spout_target move it (mod.rs:452-458)
    uint64_t substeps_done;
};
static const uint64_t kSnapMagic = 0x43534e4150423230ull;  // "CSNAPB20"

int Engine::snapshot_size(uint64_t* bytes) {
    const uint64_t mp = settings.max_particles;
    *bytes = sizeof(SnapHeader) + mp * sizeof(float4) * 7 + mp * 4 * sizeof(int32_t) + cells_ * 2 * sizeof(float);
    return CS_OK;
}

int Engine::snapshot_save(void* buf, uint64_t bytes) {
    uint64_t need;
    snapshot_size(&need);
    if (bytes < need) {
        set_error("snapshot buffer too small");
        return CS_ERR_INVALID_ARG;
    }
    SnapHeader h;
    std::memset(&h, 0, sizeof(h));
    h.magic = kSnapMagic;
    h.version = 4;
    h.substeps_done = substeps_done_;
    h.max_p = settings.max_particles;
    h.cells = cells_;
    h.num_water = num_water;
    h.num_bed = num_bed;
    h.total_time = total_time;
    h.total_emitted_mass = total_emitted_mass;
    h.total_dropped = total_dropped;
    h.have_prev_p = have_prev_p ? 1 : 0;
    h.inflow = inflow;
    h.spout = settings.spout;
    char* p = (char*)buf;
    std::memcpy(p, &h, sizeof(h));
    p += sizeof(h);
    const size_t mpb = (size_t)settings.max_particles * sizeof(float4);
    DeviceBuffer* streams[] = {&pos_, &vel_, &c0_, &c1_, &c2_, &bedA_, &bedB_};
    int rc;
    for (DeviceBuffer* b : streams) {
        if ((rc = check(cudaMemcpyAsync(p, b->ptr, mpb, cudaMemcpyDeviceToHost, stream_), "snapshot"))) return rc;
        p += mpb;
    }
    if ((rc = check(cudaMemcpyAsync(p, delta_.ptr, delta_.bytes, cudaMemcpyDeviceToHost, stream_), "snapshot")))
        return rc;
    p += delta_.bytes;
    if ((rc = check(cudaMemcpyAsync(p, pf_.ptr, cells_ * 4, cudaMemcpyDeviceToHost, stream_), "snapshot"))) return rc;
    p += cells_ * 4;
    // low word of the FP32-storage pressure (the warm start of the next solve)
    if ((rc = check(cudaMemcpyAsync(p, plo_.ptr, cells_ * 4, cudaMemcpyDeviceToHost, stream_), "snapshot"))) return rc;
    return sync();
}

int Engine::snapshot_load(const void* buf, uint64_t bytes) {
    uint64_t need;
    snapshot_size(&need);
    SnapHeader h;
    if (bytes < sizeof(h)) {
        set_error("snapshot too small");
        return CS_ERR_INVALID_ARG;
    }
    std::memcpy(&h, buf, sizeof(h));
    if (h.magic != kSnapMagic || h.version != 4 || h.max_p != settings.max_particles || h.cells != cells_ ||
        bytes < need) {
        set_error("snapshot does not match this simulation's sizes");
        return CS_ERR_INVALID_ARG;
    }
    const char* p = (const char*)buf + sizeof(h);
    const size_t mpb = (size_t)settings.max_particles * sizeof(float4);
    DeviceBuffer* streams[] = {&pos_, &vel_, &c0_, &c1_, &c2_, &bedA_, &bedB_};
    int rc;
    for (DeviceBuffer* b : streams) {
        if ((rc = check(cudaMemcpyAsync(b->ptr, p, mpb, cudaMemcpyHostToDevice, stream_), "restore"))) return rc;
        p += mpb;
    }
    if ((rc = check(cudaMemcpyAsync(delta_.ptr, p, delta_.bytes, cudaMemcpyHostToDevice, stream_), "restore")))
        return rc;
    p += delta_.bytes;
    if ((rc = check(cudaMemcpyAsync(pf_.ptr, p, cells_ * 4, cudaMemcpyHostToDevice, stream_), "restore"))) return rc;
    p += cells_ * 4;
    if ((rc = check(cudaMemcpyAsync(plo_.ptr, p, cells_ * 4, cudaMemcpyHostToDevice, stream_), "restore"))) return rc;
    num_water = h.num_water;
    num_bed = h.num_bed;
    total_time = h.total_time;
    total_emitted_mass = h.total_emitted_mass;
    total_dropped = h.total_dropped;
    have_prev_p = h.have_prev_p != 0;
    substeps_done_ = h.substeps_done;
    inflow = h.inflow;
    settings.spout = h.spout;
    return sync();
}

// ---- batched ensemble ----
Ensemble::~Ensemble() {
    if (stream) cudaStreamSynchronize(stream);
    for (Engine* e : eng) delete e;
    if (gexec) cudaGraphExecDestroy(gexec);
    if (d_ctx) cudaFree(d_ctx);
    if (d_results) cudaFree(d_results);
    if (d_partial) cudaFree(d_partial);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    if (stream) cudaStreamDestroy(stream);
}

static int ens_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return CS_OK;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return CS_ERR_CUDA;
}

int Ensemble::timer_start() {
    int rc;
    if (!t0 && (rc = ens_check(cudaEventCreate(&t0), "ensemble timer"))) return rc;
    if (!t1 && (rc = ens_check(cudaEventCreate(&t1), "ensemble timer"))) return rc;
    return ens_check(cudaEventRecord(t0, stream), "ensemble timer start");
}

int Ensemble::timer_stop(float* ms) {
    if (!t0) {
        set_error("timer not started");
        return CS_ERR_INVALID_ARG;
    }
    int rc = ens_check(cudaEventRecord(t1, stream), "ensemble timer stop");
    if (rc) return rc;
    if ((rc = ens_check(cudaEventSynchronize(t1), "ensemble timer sync"))) return rc;
    return ens_check(cudaEventElapsedTime(ms, t0, t1), "ensemble timer elapsed");
}

int Ensemble::init(const CsSettings* s, uint32_t n) {
    if (n == 0) {
        set_error("an ensemble needs at least one instance");
        return CS_ERR_INVALID_ARG;
    }
    for (uint32_t i = 0; i < n; ++i) {
        CsSettings t = s[i];
        t.device_emission = 1;  // jet samples are built by the batched emission kernel
        t.use_graph = 0;
        int rc = validate_settings(&t);
        if (rc) return rc;
        const CsSettings& a = s[0];
        if (t.grid_dims[0] != a.grid_dims[0] || t.grid_dims[1] != a.grid_dims[1] || t.grid_dims[2] != a.grid_dims[2] ||
            t.p2g_mode != a.p2g_mode || t.solve_mode != a.solve_mode || t.pressure_storage != a.pressure_storage ||
            t.device != a.device || t.pressure_rbgs_pairs != a.pressure_rbgs_pairs || t.max_sweeps != a.max_sweeps ||
            t.check_every != a.check_every || t.first_check != a.first_check || t.residual_tol != a.residual_tol ||
            t.warm_start != a.warm_start || t.p2g_tile != a.p2g_tile || t.particle_threads != a.particle_threads) {
            set_error("ensemble instances must share grid dims, device, P2G mode, warm start and solver settings");
            return CS_ERR_INVALID_ARG;
        }
        Engine* e = new Engine(t);
        eng.push_back(e);
        if ((rc = e->init())) return rc;
    }
    Engine& e0 = *eng[0];
    if (e0.settings.solve_mode == CS_SOLVE_RESIDUAL &&
        (e0.settings.pressure_storage != CS_PRESSURE_FP32 || e0.sc_ranks_ == 0)) {
        set_error("ensembles in residual mode need FP32 storage and the cluster-resident solve");
        return CS_ERR_UNSUPPORTED;
    }
    for (uint32_t i = 0; i < n; ++i)
        if (s[i].reorder_every) {
            set_error("ensemble instances do not reorder their samples (reorder_every must be 0)");
            return CS_ERR_UNSUPPORTED;
        }
    graph = s[0].use_graph != 0;
    if (graph && e0.settings.solve_mode != CS_SOLVE_RESIDUAL) {
        set_error("ensemble graph replay needs the residual-mode solve");
        return CS_ERR_UNSUPPORTED;
    }
    if (graph && e0.settings.warm_start == CS_WARM_LEARNED) {
        set_error("the learned warm start of an ensemble runs without graph replay (use_graph = 0)");
        return CS_ERR_UNSUPPORTED;
    }
    ranks = e0.sc_ranks_;
    const size_t chunks = std::max<size_t>(bs_max_chunks(e0.sc_codes_), bs_max_chunks((size_t)e0.p2g_tiles_ + 1));  // the largest tile count
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&d_ctx, sizeof(Ctx) * n) != cudaSuccess || cudaMalloc(&d_results, sizeof(ScResult) * n) != cudaSuccess ||
        cudaMalloc(&d_partial, sizeof(unsigned long long) * n * chunks) != cudaSuccess) {
        set_error("ensemble allocation failed");
        return CS_ERR_CUDA;
    }
    hctx.resize(n);
    hsb.resize(n);
    results.resize(n);
    for (uint32_t i = 0; i < n; ++i) hsb[i] = eng[i]->sc_buf_;
    return CS_OK;
}

int Ensemble::sync() {
    if (cudaStreamSynchronize(stream) != cudaSuccess) {
        set_error(std::string("ensemble stream: ") + cudaGetErrorString(cudaGetLastError()));
        return CS_ERR_CUDA;
    }
    return CS_OK;
}

// One substep of every instance: host prologues (jet plans, uniforms), one context
// upload, then each pass as a single launch over all instances — enqueued directly, or
// in graph mode replayed from a graph captured at the first substep.
int Ensemble::substep(float sub_dt) {
    int rc;
    const uint32_t n = size();
    for (uint32_t i = 0; i < n; ++i) {
        Engine& e = *eng[i];
        // no work of an instance's own may be in flight (in graph mode an instance has
        // none: its results are read after the ensemble stream synchronised)
        if (!graph && (rc = e.sync())) return rc;
        if ((rc = e.emit(sub_dt))) return rc;
        e.fill_params(e.ctx_.u, sub_dt);
        e.ctx_.u.jet = e.jet_;
        hctx[i] = e.ctx_;
    }
    if (cudaMemcpyAsync(d_ctx, hctx.data(), sizeof(Ctx) * n, cudaMemcpyHostToDevice, stream) != cudaSuccess) {
        set_error("ensemble context upload failed");
        return CS_ERR_CUDA;
    }
    if ((rc = graph ? substep_graph() : enqueue(false))) return rc;
    for (uint32_t i = 0; i < n; ++i) {
        Engine& e = *eng[i];
        e.total_time += sub_dt;
        e.have_prev_p = true;
        e.prof_.substeps += 1;
        if (graph) e.graph_pending_ = true;  // solve totals read at the next synchronising call
    }
    return CS_OK;
}

// Graph mode: the batched substep captured once (launch shapes cover every instance's
// max_particles) and replayed; each instance's solve result goes to its running totals.
// An instance whose fluid overflows its cluster is reported (CS_ERR_CAPACITY) at the
// next metrics read instead of being re-solved alone.
int Ensemble::substep_graph() {
    int rc;
    if (!gexec) {
        if ((rc = ens_check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture")))
            return rc;
        const int erc = enqueue(true);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(stream, &g);
        if (erc) {
            if (g) cudaGraphDestroy(g);
            return erc;
        }
        if ((rc = ens_check(ce, "end capture"))) return rc;
        rc = ens_check(cudaGraphInstantiate(&gexec, g, 0), "graph instantiate");
        cudaGraphDestroy(g);
        if (rc) return rc;
    }
    return ens_check(cudaGraphLaunch(gexec, stream), "graph launch");
}

int Ensemble::enqueue(bool capture) {
    int rc;
    const uint32_t n = size();
    Engine& e0 = *eng[0];
    const CsSettings& s = e0.settings;
    const Ctx* dc = (const Ctx*)d_ctx;
    uint32_t max_np = 0, max_bed = 0, max_jet = 0;
    for (Engine* e : eng) {
        max_np = std::max(max_np, capture ? e->settings.max_particles : e->num_water + e->num_bed);
        max_bed = std::max(max_bed, e->num_bed);
        max_jet = std::max(max_jet, e->jet_.count);
    }
    const int cb = e0.launch_cells_blocks();
    const int pb = e0.launch_particle_blocks_pt(max_np);
    const dim3 TP(e0.particle_threads());
    const int bb = e0.launch_particle_blocks(max_bed);
    const dim3 T(kThreads);
    cudaStream_t st = stream;
    if (capture)
        k_emit_jet<<<dim3(16, n), T, 0, st>>>(dc);
    else if (max_jet)
        k_emit_jet<<<dim3(e0.launch_particle_blocks(max_jet), n), T, 0, st>>>(dc);
    k_clear_batch<<<dim3(cb, n), T, 0, st>>>(dc, e0.p2g_tile_count() + 1);
    if (max_bed) k_bed_lookup_scatter<<<dim3(bb, n), T, 0, st>>>(dc);
    if (max_np) {
        if (s.p2g_mode != CS_P2G_ATOMIC32) {
            k_p2g_keys<<<dim3(pb, n), TP, 0, st>>>(dc);
            bs_launch<uint32_t>(dc, n, e0.p2g_tile_count() + 1, (uint32_t*)d_partial, st);
            k_p2g_scatter<<<dim3(pb, n), TP, 0, st>>>(dc);
            e0.launch_p2g_tiles(dc, n, st);
        } else {
            k_p2g_atomic<<<dim3(pb, n), TP, 0, st>>>(dc);
        }
    }
    k_grid_update<<<dim3(cb, n), T, 0, st>>>(dc, 1);
    if (max_bed) k_bed_velocity<<<dim3(cb, n), T, 0, st>>>(dc);
    k_classify<<<dim3(cb, n), T, 0, st>>>(dc);
    if (s.warm_start == CS_WARM_LEARNED) {
        // each instance's network guess (inputs from its residual, U-Net forward, FP64
        // acceptance test on the device), enqueued on the ensemble stream ahead of the
        // batched solve
        for (Engine* e : eng) {
            cudaStream_t own = e->stream_;
            e->stream_ = st;
            rc = e->upload_ctx();
            if (!rc) rc = e->learned_enqueue(false);
            e->stream_ = own;
            if (rc) return rc;
        }
    }
    if (s.solve_mode == CS_SOLVE_RESIDUAL) {
        if ((rc = sc_launch_prep(dc, hsb.data(), (uint32_t)e0.sc_codes_, ranks, n, st, e0.sms_, d_partial)))
            return rc;
        if ((rc = sc_launch_cluster(dc, ranks, n, s.residual_tol, s.max_sweeps, s.check_every, st,
                                    s.rbgs_kernel == 3 ? 0u : 1u)))
            return rc;
        if (capture) {
            k_sc_account_batch<<<(n + 127) / 128, 128, 0, st>>>(dc, n);
            goto after_solve;
        }
        k_gather_results<<<1, 256, 0, st>>>(dc, n, (ScResult*)d_results);
        if (cudaMemcpyAsync(results.data(), d_results, sizeof(ScResult) * n, cudaMemcpyDeviceToHost, st) !=
                cudaSuccess ||
            (rc = sync()))
            return rc ? rc : CS_ERR_CUDA;
        for (uint32_t i = 0; i < n; ++i) {
            Engine& e = *eng[i];
            const ScResult& r = results[i];
            if ((rc = e.learned_collect())) return rc;
            if (r.status != 1) {
                // this instance's fluid does not fit the cluster: solve it alone with
                // per-colour launches on its own stream
                if ((rc = e.upload_ctx())) return rc;
                const int keep = e.sc_ranks_;
                e.sc_ranks_ = 0;
                uint32_t sw = 0;
                double r0 = -1.0, r1 = -1.0;
                rc = e.solve_pressure(sw, r0, r1);
                e.sc_ranks_ = keep;
                if (rc) return rc;
                if ((rc = e.sync())) return rc;
                e.last.last_sweeps = sw;
                e.last.initial_residual = r0;
                e.last.last_residual = r1;
                e.prof_.sweeps += sw;
                continue;
            }
            e.last.last_sweeps = r.sweeps;
            e.last.residual_checks = r.evals;
            e.last.initial_residual = r.r0;
            e.last.last_residual = r.r1;
            e.prof_.sweeps += r.sweeps;
            e.prof_.residual_evals += r.evals;
        }
    } else {
        const uint32_t half = (s.grid_dims[0] + 1) / 2;
        const size_t ncol = (size_t)half * s.grid_dims[1] * s.grid_dims[2];
        const int blocks = (int)std::min<size_t>((ncol + kThreads - 1) / kThreads, (size_t)e0.sms_ * 16);
        for (uint32_t k = 0; k < s.pressure_rbgs_pairs; ++k) {
            k_rbgs_colour<<<dim3(blocks, n), T, 0, st>>>(dc, 0u);
            k_rbgs_colour<<<dim3(blocks, n), T, 0, st>>>(dc, 1u);
        }
        for (Engine* e : eng) {
            e->last.last_sweeps = s.pressure_rbgs_pairs;
            e->last.residual_checks = 0;
            e->prof_.sweeps += s.pressure_rbgs_pairs;
        }
    }
after_solve:
    k_project<<<dim3(cb, n), T, 0, st>>>(dc, 1 | 2 | 4);
    k_packing_apply<<<dim3(cb, n), T, 0, st>>>(dc, 1);
    k_viscosity_prepare<<<dim3(cb, n), T, 0, st>>>(dc);
    k_viscosity_apply<<<dim3(cb, n), T, 0, st>>>(dc, 1);
    if (max_np) {
        k_g2p<<<dim3(pb, n), TP, 0, st>>>(dc);
        k_bed_coupling<<<dim3(pb, n), TP, 0, st>>>(dc);
    }
    if (max_bed) {
        k_extraction_advect<<<dim3(bb, n), T, 0, st>>>(dc);
        k_bed_dynamics<<<dim3(bb, n), T, 0, st>>>(dc);
    }
    if (max_np) k_prepare_render<<<dim3(pb, n), TP, 0, st>>>(dc);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        set_error(std::string("ensemble substep launch: ") + cudaGetErrorString(err));
        return CS_ERR_CUDA;
    }
    return CS_OK;
}

int Ensemble::step_frame(float dt) {
    const CsSettings& s = eng[0]->settings;
    const float fdt = std::fmin(dt, s.max_frame_dt);
    const uint32_t k = s.substeps > 1 ? s.substeps : 1;
    const float sdt = fdt / (float)k;
    for (Engine* e : eng) {
        e->frame_emitted_mass = 0.0f;
        e->frame_dropped = 0;
    }
    for (uint32_t j = 0; j < k; ++j) {
        int rc = substep(sdt);
        if (rc) return rc;
    }
    return CS_OK;
}

// ---- learned warm start ----
// The network of coffee_sim_b200/unet.py: per layer (level, input, output channels);
// parameters in order, each layer's weights [cout][27][cin] then its bias, then the
// 1x1x1 output layer's 16 weights and bias.
namespace {
struct UnetLayer {
    int level, cin, cout;
};
constexpr UnetLayer kUnet[9] = {{0, 8, 16}, {0, 16, 16}, {1, 16, 32}, {1, 32, 32}, {2, 32, 64},
                                {1, 96, 32}, {1, 32, 32}, {0, 48, 16}, {0, 16, 16}};
constexpr int kHeadC = 16;
uint64_t unet_param_count() {
    uint64_t n = 0;
    for (const UnetLayer& l : kUnet) n += (uint64_t)l.cout * 27 * l.cin + l.cout;
    return n + kHeadC + 1;
}
uint64_t unet_layer_offset(int k) {
    uint64_t n = 0;
    for (int i = 0; i < k; ++i) n += (uint64_t)kUnet[i].cout * 27 * kUnet[i].cin + kUnet[i].cout;
    return n;
}
int r16(int c) { return (c + 15) / 16 * 16; }
}  // namespace

int Engine::learned_alloc() {
    if (l_ready_) return CS_OK;
    const CsSettings& s = settings;
    for (int a = 0; a < 3; ++a)
        if (s.grid_dims[a] % 4) {
            set_error("the learned warm start needs grid dims that are multiples of 4");
            return CS_ERR_INVALID_ARG;
        }
    const size_t v0 = cells_, v1 = v0 / 8, v2 = v1 / 8;
    int rc;
    if ((rc = alloc(l_params_, unet_param_count() * sizeof(float)))) return rc;
    for (int k = 0; k < 9; ++k) {
        const size_t kpad = (size_t)((27 * kUnet[k].cin + 63) / 64 * 64);
        if ((rc = alloc(l_wf_[k], (size_t)r16(kUnet[k].cout) * kpad * 2))) return rc;
    }
    // activations (bf16): e1a e1b p1 e2a e2b p2 e3a u2 d2a d2b u1 d1a d1b
    const size_t sizes[13] = {v0 * 16, v0 * 16, v1 * 16, v1 * 32, v1 * 32, v2 * 32, v2 * 64,
                              v1 * 96, v1 * 32, v1 * 32, v0 * 48, v0 * 16, v0 * 16};
    for (int k = 0; k < 13; ++k)
        if ((rc = alloc(l_act_[k], sizes[k] * 2))) return rc;
    if ((rc = alloc(l_feat_, v0 * 8 * 2))) return rc;
    if ((rc = alloc(l_out_, v0 * sizeof(float)))) return rc;
    if ((rc = alloc(l_stats_, (2 * kLearnedStatBlocks + 3) * sizeof(double)))) return rc;  // zeroed
    if ((rc = alloc(l_scale_, sizeof(float)))) return rc;
    if ((rc = alloc(l_bak_hi_, v0 * sizeof(float)))) return rc;
    if ((rc = alloc(l_bak_lo_, v0 * sizeof(float)))) return rc;
    if ((rc = alloc(l_target_, v0 * sizeof(float)))) return rc;
    if ((rc = alloc(l_mask_, v0 * sizeof(float)))) return rc;
    if ((rc = alloc(l_err_, sizeof(uint32_t)))) return rc;
    if ((rc = alloc(l_rprev_, 2 * sizeof(double)))) return rc;
    if ((rc = alloc(l_keep_, sizeof(uint32_t)))) return rc;
    cudaMemsetAsync(l_err_.ptr, 0, sizeof(uint32_t), stream_);
    l_ready_ = true;
    return CS_OK;
}

int Engine::set_learned_weights(const float* params, uint64_t count) {
    if (count != unet_param_count()) {
        set_error("learned weights: expected " + std::to_string(unet_param_count()) + " parameters");
        return CS_ERR_INVALID_ARG;
    }
    int rc = learned_alloc();
    if (rc) return rc;
    if ((rc = check(cudaMemcpyAsync(l_params_.ptr, params, count * sizeof(float), cudaMemcpyHostToDevice, stream_),
                    "weights upload")))
        return rc;
    const float* dp = (const float*)l_params_.ptr;
    for (int k = 0; k < 9; ++k) {
        const UnetLayer& l = kUnet[k];
        if ((rc = cs_nn_pack_weights(dp + unet_layer_offset(k), l_wf_[k].ptr, l.cin, l.cin, l.cout, r16(l.cout), 0,
                                     stream_)))
            return rc;
    }
    l_weights_ = true;
    return sync();
}

int Engine::learned_features() {
    const Ctx* dc = (const Ctx*)d_ctx_.ptr;
    k_learned_stats<<<dim3(kLearnedStatBlocks, 1), kThreads, 0, stream_>>>(dc, (double*)l_stats_.ptr);
    k_learned_features<<<dim3(launch_cells_blocks(), 1), kThreads, 0, stream_>>>(
        dc, (const double*)l_stats_.ptr, (__nv_bfloat16*)l_feat_.ptr, (float*)l_scale_.ptr);
    count_launch(2);
    return check(cudaGetLastError(), "learned features");
}

int Engine::learned_forward() {
    const CsSettings& s = settings;
    const int d[3][3] = {{(int)s.grid_dims[0], (int)s.grid_dims[1], (int)s.grid_dims[2]},
                         {(int)s.grid_dims[0] / 2, (int)s.grid_dims[1] / 2, (int)s.grid_dims[2] / 2},
                         {(int)s.grid_dims[0] / 4, (int)s.grid_dims[1] / 4, (int)s.grid_dims[2] / 4}};
    const float* dp = (const float*)l_params_.ptr;
    uint32_t* err = (uint32_t*)l_err_.ptr;
    void* a[13];
    for (int k = 0; k < 13; ++k) a[k] = l_act_[k].ptr;
    enum { E1A, E1B, P1, E2A, E2B, P2, E3A, U2, D2A, D2B, U1, D1A, D1B };
    int rc;
    auto conv = [&](int k, const void* x, void* y) {
        const UnetLayer& l = kUnet[k];
        const int* g = d[l.level];
        const float* bias = dp + unet_layer_offset(k) + (uint64_t)l.cout * 27 * l.cin;
        count_launch();
        return cs_nn_conv3d(x, l_wf_[k].ptr, bias, y, nullptr, g[0], g[1], g[2], l.cin, r16(l.cout), 1, err, stream_);
    };
    if ((rc = conv(0, l_feat_.ptr, a[E1A])) || (rc = conv(1, a[E1A], a[E1B]))) return rc;
    if ((rc = cs_nn_pool(a[E1B], a[P1], nullptr, nullptr, d[0][0], d[0][1], d[0][2], 16, 0, stream_))) return rc;
    if ((rc = conv(2, a[P1], a[E2A])) || (rc = conv(3, a[E2A], a[E2B]))) return rc;
    if ((rc = cs_nn_pool(a[E2B], a[P2], nullptr, nullptr, d[1][0], d[1][1], d[1][2], 32, 0, stream_))) return rc;
    if ((rc = conv(4, a[P2], a[E3A]))) return rc;
    if ((rc = cs_nn_upcat(a[E3A], a[E2B], a[U2], nullptr, nullptr, nullptr, d[1][0], d[1][1], d[1][2], 64, 32, 0,
                          stream_)))
        return rc;
    if ((rc = conv(5, a[U2], a[D2A])) || (rc = conv(6, a[D2A], a[D2B]))) return rc;
    if ((rc = cs_nn_upcat(a[D2B], a[E1B], a[U1], nullptr, nullptr, nullptr, d[0][0], d[0][1], d[0][2], 32, 16, 0,
                          stream_)))
        return rc;
    if ((rc = conv(7, a[U1], a[D1A])) || (rc = conv(8, a[D1A], a[D1B]))) return rc;
    const float* head = dp + unet_layer_offset(9);
    count_launch(5);
    return cs_nn_head(a[D1B], head, (float*)l_out_.ptr, nullptr, nullptr, nullptr, (int64_t)cells_, kHeadC, 0,
                      stream_);
}

// Before the solve: the FP64 residual r of the previous-substep pressure p and the
// network inputs built from it; with the learned warm start, p + (network output) * s
// replaces p when that has the smaller FP64 residual (below 0.999x).  Every step is
// enqueued on the stream and the acceptance test runs on the device, so the sequence can
// be captured in a graph; learned_collect reads the outcome once the solve has
// synchronised.  `marks`: record the profiling phase.
int Engine::learned_enqueue(bool marks) {
    const bool learned = settings.warm_start == CS_WARM_LEARNED;
    if (!learned && !l_capture_) return CS_OK;
    if (learned && !l_weights_) {
        set_error("CS_WARM_LEARNED needs weights (cs_set_learned_weights)");
        return CS_ERR_INVALID_ARG;
    }
    int rc;
    if ((rc = learned_alloc())) return rc;
    const Ctx* dc = (const Ctx*)d_ctx_.ptr;
    const int cb = launch_cells_blocks();
    if (marks) mark(CS_PHASE_LEARNED);
    // residual of the previous pressure (left in gres for the inputs), its norms kept
    cudaMemsetAsync(resid_.ptr, 0, 2 * sizeof(double), stream_);
    k_refine_residual<<<dim3(cb, 1), kThreads, 0, stream_>>>(dc);
    cudaMemcpyAsync(l_rprev_.ptr, resid_.ptr, 2 * sizeof(double), cudaMemcpyDeviceToDevice, stream_);
    count_launch();
    prof_.residual_evals += 1;
    if ((rc = learned_features())) return rc;
    k_learned_save<<<dim3(cb, 1), kThreads, 0, stream_>>>(dc, (float*)l_bak_hi_.ptr, (float*)l_bak_lo_.ptr);
    count_launch();
    if (!learned) return check(cudaGetLastError(), "learned inputs");
    if ((rc = learned_forward())) return rc;
    k_learned_apply<<<dim3(cb, 1), kThreads, 0, stream_>>>(dc, (const float*)l_out_.ptr, (const float*)l_scale_.ptr,
                                                        (const float*)l_bak_hi_.ptr, (const float*)l_bak_lo_.ptr);
    cudaMemsetAsync(resid_.ptr, 0, 2 * sizeof(double), stream_);
    k_refine_residual<<<dim3(cb, 1), kThreads, 0, stream_>>>(dc);
    k_learned_decide<<<1, 1, 0, stream_>>>((const double*)l_rprev_.ptr, (const double*)resid_.ptr,
                                           (uint32_t*)l_keep_.ptr);
    k_learned_restore<<<dim3(cb, 1), kThreads, 0, stream_>>>(dc, (const float*)l_bak_hi_.ptr,
                                                            (const float*)l_bak_lo_.ptr, (const uint32_t*)l_keep_.ptr);
    count_launch(4);
    prof_.residual_evals += 1;
    return check(cudaGetLastError(), "learned warm start");
}

int Engine::learned_collect() {
    last.learned_used = 0;
    if (settings.warm_start != CS_WARM_LEARNED || !l_ready_) return CS_OK;
    uint32_t keep = 0, err = 0;
    int rc;
    if ((rc = check(cudaMemcpy(&keep, l_keep_.ptr, sizeof(keep), cudaMemcpyDeviceToHost), "learned outcome")) ||
        (rc = check(cudaMemcpy(&err, l_err_.ptr, sizeof(err), cudaMemcpyDeviceToHost), "learned error flag")))
        return rc;
    prof_.d2h_bytes += 2 * sizeof(uint32_t);
    if (err) {
        set_error("a tensor-core convolution of the learned warm start timed out");
        return CS_ERR_TIMEOUT;
    }
    last.learned_used = keep;
    return CS_OK;
}

int Engine::learned_after_solve() {
    if (!l_capture_) return CS_OK;
    const Ctx* dc = (const Ctx*)d_ctx_.ptr;
    k_learned_target<<<dim3(launch_cells_blocks(), 1), kThreads, 0, stream_>>>(
        dc, (const float*)l_scale_.ptr, (const float*)l_bak_hi_.ptr, (const float*)l_bak_lo_.ptr,
        (float*)l_target_.ptr, (float*)l_mask_.ptr);
    count_launch();
    l_have_sample_ = true;
    return check(cudaGetLastError(), "learned target");
}

int Engine::learned_capture(bool on) {
    if (on) {
        int rc = learned_alloc();
        if (rc) return rc;
    }
    l_capture_ = on;
    if (on) l_have_sample_ = false;  // turning capture off keeps the last pair readable
    return CS_OK;
}

int Engine::learned_read_sample(void* feat, float* target, float* mask, float* scale) {
    if (!l_have_sample_) {
        set_error("no captured sample: enable cs_learned_capture and step a substep first");
        return CS_ERR_INVALID_ARG;
    }
    int rc;
    if (feat && (rc = check(cudaMemcpyAsync(feat, l_feat_.ptr, cells_ * 16, cudaMemcpyDeviceToDevice, stream_),
                            "sample features")))
        return rc;
    if (target && (rc = check(cudaMemcpyAsync(target, l_target_.ptr, cells_ * 4, cudaMemcpyDeviceToDevice, stream_),
                              "sample target")))
        return rc;
    if (mask && (rc = check(cudaMemcpyAsync(mask, l_mask_.ptr, cells_ * 4, cudaMemcpyDeviceToDevice, stream_),
                            "sample mask")))
        return rc;
    if (scale && (rc = check(cudaMemcpyAsync(scale, l_scale_.ptr, 4, cudaMemcpyDeviceToHost, stream_), "scale")))
        return rc;
    return sync();
}

// ---- autotuner: time candidate configurations from one saved state ----
int Engine::autotune(float sub_dt, uint32_t substeps, CsTuneResult* out) {
    CsSettings& s = settings;
    if (s.solve_mode != CS_SOLVE_RESIDUAL || s.pressure_storage == CS_PRESSURE_FIXED_POINT) {
        set_error("the autotuner needs the residual-mode FP32 solve");
        return CS_ERR_UNSUPPORTED;
    }
    if (substeps == 0 || !(sub_dt > 0.0f)) {
        set_error("autotune: substeps and sub_dt must be positive");
        return CS_ERR_INVALID_ARG;
    }
    uint64_t bytes = 0;
    snapshot_size(&bytes);
    std::vector<unsigned char> state(bytes);
    int rc = snapshot_save(state.data(), bytes);
    if (rc) return rc;
    const CsSettings entry = s;
    const float fe = frame_emitted_mass;
    const uint32_t fd = frame_dropped;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    uint32_t trial_min_pairs = 0;  // fewest pairs of one substep in the last trial
    uint32_t tile = p2g_tile(), threads = particle_threads();  // launch shapes of the next trial
    auto trial = [&](float omega, uint32_t ce, uint32_t p2g, uint32_t first, float& ms) -> int {
        int r = snapshot_load(state.data(), bytes);
        if (r) return r;
        s.rbgs_omega = omega;
        s.check_every = ce;
        s.p2g_mode = p2g;
        s.first_check = first;
        s.p2g_tile = tile;
        s.particle_threads = threads;
        bool converged = true;
        trial_min_pairs = 0xffffffffu;
        cudaEventRecord(a, stream_);
        for (uint32_t k = 0; k < substeps; ++k) {
            if ((r = substep(sub_dt, 0xffffffffu))) return r;
            converged = converged && last.last_residual >= 0.0 && last.last_residual <= (double)s.residual_tol;
            trial_min_pairs = std::min(trial_min_pairs, last.last_sweeps);
        }
        cudaEventRecord(b, stream_);
        if ((r = sync())) return r;
        cudaEventElapsedTime(&ms, a, b);
        ms /= (float)substeps;
        if (!converged) ms = INFINITY;
        return CS_OK;
    };
    CsTuneResult res{};
    float ms = 0.0f;
    uint32_t best_pairs = 0;
    if ((rc = trial(entry.rbgs_omega, entry.check_every, entry.p2g_mode, entry.first_check, ms))) goto done;
    res.initial_ms = ms;
    res.best_ms = ms;
    res.omega = entry.rbgs_omega;
    res.check_every = entry.check_every;
    res.p2g_mode = entry.p2g_mode;
    res.first_check = entry.first_check;
    res.p2g_tile = tile;
    res.particle_threads = threads;
    res.trials = 1;
    best_pairs = trial_min_pairs;
    // P2G mode at the entry solver settings, then the solver at the chosen mode
    for (uint32_t m : {(uint32_t)CS_P2G_ATOMIC32, (uint32_t)CS_P2G_SORTED_SHARED}) {
        if (m == entry.p2g_mode || entry.p2g_mode == CS_P2G_INT64) continue;  // int64 changes the numerics
        if ((rc = trial(entry.rbgs_omega, entry.check_every, m, entry.first_check, ms))) goto done;
        ++res.trials;
        if (ms < res.best_ms) {
            res.best_ms = ms;
            res.p2g_mode = m;
            best_pairs = trial_min_pairs;
        }
    }
    for (float omega : {1.80f, 1.85f, 1.88f, 1.90f, 1.92f, 1.94f, 1.96f})
        for (uint32_t ce : {10u, 20u, 40u, 60u, 80u}) {
            if (omega == res.omega && ce == res.check_every && res.first_check == 0) continue;
            if ((rc = trial(omega, ce, res.p2g_mode, 0u, ms))) goto done;
            ++res.trials;
            if (ms < res.best_ms) {
                res.best_ms = ms;
                res.omega = omega;
                res.check_every = ce;
                res.first_check = 0;
                best_pairs = trial_min_pairs;
            }
        }
    // the first check just before the fewest pairs a trial substep took (each check skipped
    // saves an FP64 residual pass; a first interval past convergence costs extra pairs)
    if (best_pairs != 0xffffffffu && best_pairs > 4) {
        const uint32_t base = best_pairs;
        for (double f : {0.85, 0.92, 0.98}) {
            const uint32_t first = (uint32_t)(f * (double)base);
            if (first < 2 || first == res.first_check) continue;
            if ((rc = trial(res.omega, res.check_every, res.p2g_mode, first, ms))) goto done;
            ++res.trials;
            if (ms < res.best_ms) {
                res.best_ms = ms;
                res.first_check = first;
            }
        }
    }
    // launch shapes at the chosen solver settings: threads per block of the particle
    // passes, and the P2G tile side when P2G is tile-sorted
    for (uint32_t t : {4u, 8u})
        for (uint32_t th : {128u, 256u}) {
            if (t != 4u && res.p2g_mode == CS_P2G_ATOMIC32) continue;
            if (t == res.p2g_tile && th == res.particle_threads) continue;
            tile = t;
            threads = th;
            if ((rc = trial(res.omega, res.check_every, res.p2g_mode, res.first_check, ms))) goto done;
            ++res.trials;
            if (ms < res.best_ms) {
                res.best_ms = ms;
                res.p2g_tile = t;
                res.particle_threads = th;
            }
        }
done:
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    const int rc2 = snapshot_load(state.data(), bytes);
    s = entry;
    frame_emitted_mass = fe;
    frame_dropped = fd;
    if (rc) return rc;
    if (rc2) return rc2;
    s.rbgs_omega = res.omega;
    s.check_every = res.check_every;
    s.p2g_mode = res.p2g_mode;
    s.first_check = res.first_check;
    s.p2g_tile = res.p2g_tile;
    s.particle_threads = res.particle_threads;
    if (out) *out = res;
    return CS_OK;
}

// ---- launch helpers shared by Engine and noalloc.cu ----
// Largest cluster size the solve kernel can be launched with on the current device
// (16 with the non-portable opt-in, else 8), 0 when neither fits.
int sc_max_cluster_ranks() {
    if (cudaFuncSetAttribute(k_sc_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ScLayout::bytes) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_sc_solve, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    for (int r : {16, 8}) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(r, 1, 1);
        cfg.blockDim = dim3(SC_THREADS, 1, 1);
        cfg.dynamicSmemBytes = ScLayout::bytes;
        cudaLaunchAttribute attr;
        attr.id = cudaLaunchAttributeClusterDimension;
        attr.val.clusterDim.x = r;
        attr.val.clusterDim.y = 1;
        attr.val.clusterDim.z = 1;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, (void*)k_sc_solve, &cfg) == cudaSuccess && n > 0) return r;
    }
    cudaGetLastError();
    return 0;
}

size_t sc_scan_temp_bytes(uint32_t codes) {
    size_t temp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, temp, (unsigned long long*)nullptr, (unsigned long long*)nullptr, (int)codes,
                                  (cudaStream_t)0);
    return temp;
}

// Morton scan, chunking, neighbour slots, halo/send lists and coefficients for
// `instances` solves whose scratch blocks lie back to back (kScPrepLaunches launches
// for one instance).
int sc_launch_prep(const Ctx* d_ctx, const ScBuffers* sb, uint32_t codes, int ranks, uint32_t instances,
                   cudaStream_t stream, int sms, void* bs_partial) {
    const int cb = (int)std::min<size_t>((codes + kThreads - 1) / kThreads, (size_t)sms * 16);
    k_sc_flags<<<dim3(cb, instances), kThreads, 0, stream>>>(d_ctx, codes);
    if (bs_partial) {
        bs_launch<unsigned long long>(d_ctx, instances, codes, (unsigned long long*)bs_partial, stream);
    } else {
        for (uint32_t k = 0; k < instances; ++k) {
            size_t temp = sb[k].cub_bytes;
            if (cub::DeviceScan::ExclusiveSum(sb[k].cub_temp, temp, sb[k].flags, sb[k].scan, (int)codes, stream) !=
                cudaSuccess) {
                set_error("scan launch failed");
                return CS_ERR_CUDA;
            }
        }
    }
    k_sc_totals<<<dim3(1, instances), 1, 0, stream>>>(d_ctx, (uint32_t)ranks, codes);
    k_sc_starts<<<dim3(cb, instances), kThreads, 0, stream>>>(d_ctx, codes);
    k_sc_map<<<dim3(cb, instances), kThreads, 0, stream>>>(d_ctx, codes);
    k_sc_halo<<<dim3(cb, instances), kThreads, 0, stream>>>(d_ctx);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("solver prep launch: ") + cudaGetErrorString(e));
        return CS_ERR_CUDA;
    }
    return CS_OK;
}

int gs_blocks(int* ctas) {
    *ctas = 0;
    int dev = 0, sms = 0, coop = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CS_OK;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return CS_OK;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop) return CS_OK;
    const size_t smem = (size_t)GS_SMEM;
    // the smallest shared-memory carve-out that fits: the solve reads its own rows through L1
    if (cudaFuncSetAttribute(k_gs_solve, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxL1) !=
        cudaSuccess)
        cudaGetLastError();
    if (cudaFuncSetAttribute(k_gs_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return CS_OK;
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gs_solve, GS_THREADS, smem) != cudaSuccess ||
        per_sm < 1) {
        cudaGetLastError();
        return CS_OK;
    }
    *ctas = sms;  // one CTA per SM: fewer barrier arrivals
    return CS_OK;
}

int gs_launch_prep(const Ctx* d_ctx, const GsBuffers* gb, uint32_t rows, cudaStream_t stream, int sms) {
    const int wb = (int)std::max<size_t>(1, std::min<size_t>(((size_t)rows * 32 + 255) / 256, (size_t)sms * 16));
    k_gs_rows<<<dim3(wb, 1), 256, 0, stream>>>(d_ctx);
    size_t bytes = gb->cub_bytes;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(gb->cub_temp, bytes, gb->row_units, gb->row_start, (int)rows + 1,
                                                  stream);
    if (e == cudaSuccess) {
        const int rb = (int)std::max<size_t>(1, std::min<size_t>(((size_t)rows + 255) / 256, (size_t)sms * 16));
        k_gs_desc<<<dim3(rb, 1), 256, 0, stream>>>(d_ctx);
        e = cudaMemsetAsync(gb->sync, 0, 4 * sizeof(uint32_t), stream);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(gb->result, 0, sizeof(ScResult), stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("grid solve prep: ") + cudaGetErrorString(e));
        return CS_ERR_CUDA;
    }
    return CS_OK;
}

int gs_launch_solve(const Ctx* d_ctx, int ctas, float tol, uint32_t max_pairs, uint32_t check_every,
                    cudaStream_t stream) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ctas, 1, 1);
    cfg.blockDim = dim3(GS_THREADS, 1, 1);
    cfg.dynamicSmemBytes = (size_t)GS_SMEM;
    cfg.stream = stream;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeCooperative;
    attr.val.cooperative = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_gs_solve, d_ctx, tol, max_pairs, check_every);
    if (e != cudaSuccess) {
        set_error(std::string("grid solve launch: ") + cudaGetErrorString(e));
        return CS_ERR_CUDA;
    }
    return CS_OK;
}

// The cluster solve of `instances` independent systems: one cluster of `ranks` CTAs each.
int sc_launch_cluster(const Ctx* d_ctx, int ranks, uint32_t instances, float tol, uint32_t max_pairs,
                      uint32_t check_every, cudaStream_t stream, uint32_t p2p) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ranks, instances, 1);
    cfg.blockDim = dim3(SC_THREADS, 1, 1);
    cfg.dynamicSmemBytes = ScLayout::bytes;
    cfg.stream = stream;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = ranks;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_sc_solve, d_ctx, tol, max_pairs, check_every, p2p);
    if (e != cudaSuccess) {
        set_error(std::string("cluster solve launch: ") + cudaGetErrorString(e));
        return CS_ERR_CUDA;
    }
    return CS_OK;
}

}  // namespace cs

// ============================ C ABI ============================
using cs::Engine;
using cs::set_error;

struct CsSim {
    std::unique_ptr<Engine> e;
};

static int validate(const CsSettings* s) {
    if (!s) {
        set_error("settings is null");
        return CS_ERR_INVALID_ARG;
    }
    if (s->abi_version != CS_ABI_VERSION) {
        set_error("settings.abi_version does not match CS_ABI_VERSION");
        return CS_ERR_INVALID_ARG;
    }
    for (int a = 0; a < 3; ++a)
        if (s->grid_dims[a] < 1 || s->grid_dims[a] > 1024 || !(s->bounds_size[a] > 0.0f)) {
            set_error("grid_dims / bounds_size out of range");
            return CS_ERR_INVALID_ARG;
        }
    if ((uint64_t)s->grid_dims[0] * s->grid_dims[1] * s->grid_dims[2] > (1ull << 30)) {
        set_error("grid too large");
        return CS_ERR_INVALID_ARG;
    }
    if (s->max_particles == 0 || s->max_particles > (1u << 28)) {
        set_error("max_particles out of range");
        return CS_ERR_INVALID_ARG;
    }
    if (s->num_obstacles > CS_MAX_OBSTACLES) {
        set_error("too many obstacles");
        return CS_ERR_INVALID_ARG;
    }
    if (!(s->p2g_tile == 0 || s->p2g_tile == 4 || s->p2g_tile == 8) ||
        !(s->particle_threads == 0 || s->particle_threads == 128 || s->particle_threads == 256)) {
        set_error("p2g_tile must be 0, 4 or 8 and particle_threads 0, 128 or 256");
        return CS_ERR_INVALID_ARG;
    }
    if (s->p2g_mode > CS_P2G_INT64 || s->warm_start > CS_WARM_LEARNED || s->pressure_storage > CS_PRESSURE_FP32 ||
        s->solve_mode > CS_SOLVE_RESIDUAL || s->rbgs_kernel > 4) {
        set_error("unknown mode value in settings");
        return CS_ERR_INVALID_ARG;
    }
    // modes declared by the ABI whose engine path is not built yet
    if (s->use_graph && (!s->device_emission || (s->solve_mode == CS_SOLVE_RESIDUAL &&
                                                  (s->pressure_storage != CS_PRESSURE_FP32 || s->rbgs_kernel == 1)))) {
        set_error("use_graph needs device_emission = 1 and, in residual mode, FP32 storage with the "
                  "cluster-resident or the grid-wide solve");
        return CS_ERR_INVALID_ARG;
    }
    if (s->warm_start == CS_WARM_LEARNED &&
        (s->pressure_storage != CS_PRESSURE_FP32 || s->solve_mode != CS_SOLVE_RESIDUAL)) {
        set_error("the learned warm start needs the residual-mode FP32 solve");
        return CS_ERR_INVALID_ARG;
    }
    if (s->warm_start != CS_WARM_NONE && s->pressure_storage == CS_PRESSURE_FIXED_POINT) {
        set_error("warm start needs CS_PRESSURE_FP32 storage");
        return CS_ERR_INVALID_ARG;
    }
    if (!(s->brew.water_particles_per_ml > 0.0f)) {
        set_error("brew.water_particles_per_ml must be > 0");
        return CS_ERR_INVALID_ARG;
    }
    return CS_OK;
}

namespace cs {
int validate_settings(const CsSettings* s) { return ::validate(s); }
}  // namespace cs

#define CS_SIM(sim)                          \
    if (!(sim) || !(sim)->e) {               \
        set_error("null simulation handle"); \
        return CS_ERR_INVALID_ARG;           \
    }
#define CS_PTR(p)                            \
    if (!(p)) {                              \
        set_error("null output pointer");    \
        return CS_ERR_INVALID_ARG;           \
    }

extern "C" {

const char* cs_last_error_string(void) { return cs::g_error.c_str(); }
uint32_t cs_abi_version(void) { return CS_ABI_VERSION; }
int32_t cs_is_gpu_engine(void) { return 1; }

int32_t cs_settings_default_v60(CsSettings* out) {
    CS_PTR(out);
    cs::host::preset_default_v60(out);
    return CS_OK;
}
int32_t cs_settings_benchmark_free_stream(CsSettings* out) {
    CS_PTR(out);
    cs::host::preset_free_stream(out);
    return CS_OK;
}
int32_t cs_settings_benchmark_center_pour(CsSettings* out) {
    CS_PTR(out);
    cs::host::preset_center_pour(out);
    return CS_OK;
}
int32_t cs_settings_aim_spout(CsSettings* s, float x, float y, float z) {
    CS_PTR(s);
    cs::host::spout_aim_at(s->spout, x, y, z);
    return CS_OK;
}
float cs_kozeny_carman_permeability_m2(float grind_um, float porosity) {
    return cs::host::kozeny_carman_m2(grind_um, porosity);
}

int32_t cs_create(const CsSettings* settings, CsSim** out) {
    int rc = validate(settings);
    if (rc) return rc;
    CS_PTR(out);
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        set_error("no CUDA device visible");
        return CS_ERR_NO_DEVICE;
    }
    if (settings->device < 0 || settings->device >= n) {
        set_error("settings.device is not a visible CUDA device");
        return CS_ERR_INVALID_ARG;
    }
    std::unique_ptr<CsSim> sim(new CsSim());
    sim->e.reset(new Engine(*settings));
    if ((rc = sim->e->init())) return rc;
    *out = sim.release();
    return CS_OK;
}
int32_t cs_destroy(CsSim* sim) {
    delete sim;
    return CS_OK;
}
int32_t cs_reset(CsSim* sim) {
    CS_SIM(sim);
    return sim->e->reset();
}
int32_t cs_step_frame(CsSim* sim, float dt) {
    CS_SIM(sim);
    return sim->e->step_frame(dt);
}
int32_t cs_step_substep(CsSim* sim, float sub_dt) {
    CS_SIM(sim);
    sim->e->frame_emitted_mass = 0.0f;
    sim->e->frame_dropped = 0;
    return sim->e->substep(sub_dt, 0xffffffffu);
}
int32_t cs_step_substep_partial(CsSim* sim, float sub_dt, uint32_t passes) {
    CS_SIM(sim);
    sim->e->frame_emitted_mass = 0.0f;
    sim->e->frame_dropped = 0;
    return sim->e->substep(sub_dt, passes);
}
int32_t cs_set_kettle_angle(CsSim* sim, float a) {
    CS_SIM(sim);
    sim->e->inflow.angle = a;
    return CS_OK;
}
int32_t cs_set_spout_position(CsSim* sim, float x, float y, float z) {
    CS_SIM(sim);
    cs::host::spout_translate_origin_to(sim->e->settings.spout, x, y, z);
    return CS_OK;
}
int32_t cs_set_spout_target(CsSim* sim, float x, float y, float z) {
    CS_SIM(sim);
    cs::host::spout_aim_at(sim->e->settings.spout, x, y, z);
    return CS_OK;
}
int32_t cs_set_flow_override(CsSim* sim, float flow, float speed) {
    CS_SIM(sim);
    sim->e->inflow.flow_override = flow > 0.0f ? flow : 0.0f;
    sim->e->inflow.speed_override = flow > 0.0f ? speed : 0.0f;
    return CS_OK;
}
int32_t cs_set_solver(CsSim* sim, float omega, uint32_t check_every, uint32_t max_sweeps) {
    CS_SIM(sim);
    if (omega != 0.0f && !(omega > 0.0f && omega < 2.0f)) {
        set_error("omega must lie in (0, 2)");
        return CS_ERR_INVALID_ARG;
    }
    CsSettings& s = sim->e->settings;
    if (omega != 0.0f) s.rbgs_omega = omega;
    if (check_every) s.check_every = check_every;
    if (max_sweeps) s.max_sweeps = max_sweeps;
    return CS_OK;
}
int32_t cs_set_p2g_mode(CsSim* sim, uint32_t mode) {
    CS_SIM(sim);
    if (mode != CS_P2G_ATOMIC32 && mode != CS_P2G_SORTED_SHARED &&
        !(mode == CS_P2G_INT64 && sim->e->settings.p2g_mode == CS_P2G_INT64)) {
        set_error("P2G mode must be CS_P2G_ATOMIC32 or CS_P2G_SORTED_SHARED (int64 is chosen at creation)");
        return CS_ERR_INVALID_ARG;
    }
    if (sim->e->settings.p2g_mode == CS_P2G_INT64 && mode != CS_P2G_INT64) {
        set_error("a simulation created with int64 P2G keeps it");
        return CS_ERR_INVALID_ARG;
    }
    sim->e->settings.p2g_mode = mode;
    return CS_OK;
}
int32_t cs_set_graph_mode(CsSim* sim, uint32_t use_graph) {
    CS_SIM(sim);
    CsSettings t = sim->e->settings;
    t.use_graph = use_graph ? 1u : 0u;
    int rc = validate(&t);
    if (rc) return rc;
    if ((rc = sim->e->sync())) return rc;
    sim->e->settings.use_graph = t.use_graph;
    return CS_OK;
}
int32_t cs_set_learned_weights(CsSim* sim, const float* params, uint64_t count) {
    CS_SIM(sim);
    CS_PTR(params);
    return sim->e->set_learned_weights(params, count);
}
int32_t cs_learned_capture(CsSim* sim, uint32_t on) {
    CS_SIM(sim);
    return sim->e->learned_capture(on != 0);
}
int32_t cs_learned_read_sample(CsSim* sim, void* feat, float* target, float* mask, float* scale) {
    CS_SIM(sim);
    return sim->e->learned_read_sample(feat, target, mask, scale);
}
int32_t cs_autotune(CsSim* sim, float sub_dt, uint32_t substeps, CsTuneResult* out) {
    CS_SIM(sim);
    return sim->e->autotune(sub_dt, substeps, out);
}
int32_t cs_get_counts(const CsSim* sim, uint32_t* nw, uint32_t* nb, uint32_t* mp) {
    CS_SIM(sim);
    if (nw) *nw = sim->e->num_water;
    if (nb) *nb = sim->e->num_bed;
    if (mp) *mp = sim->e->settings.max_particles;
    return CS_OK;
}
int32_t cs_get_kettle_angle(const CsSim* sim, float* out) {
    CS_SIM(sim);
    CS_PTR(out);
    *out = sim->e->inflow.angle;
    return CS_OK;
}
int32_t cs_get_spout_position(const CsSim* sim, float out[3]) {
    CS_SIM(sim);
    CS_PTR(out);
    for (int k = 0; k < 3; ++k) out[k] = sim->e->settings.spout.origin[k];
    return CS_OK;
}
int32_t cs_get_flow(const CsSim* sim, float* fr, float* es, float* esm) {
    CS_SIM(sim);
    if (fr) *fr = sim->e->inflow.flow_rate;
    if (es) *es = sim->e->inflow.exit_speed;
    if (esm) *esm = sim->e->inflow.exit_speed * (1.0f / sim->e->settings.sim_units_per_meter);
    return CS_OK;
}
int32_t cs_get_time(const CsSim* sim, float* t) {
    CS_SIM(sim);
    CS_PTR(t);
    *t = sim->e->total_time;
    return CS_OK;
}
int32_t cs_get_emission(const CsSim* sim, float* fem, float* tem, uint32_t* fd, uint32_t* td) {
    CS_SIM(sim);
    if (fem) *fem = sim->e->frame_emitted_mass;
    if (tem) *tem = sim->e->total_emitted_mass;
    if (fd) *fd = sim->e->frame_dropped;
    if (td) *td = sim->e->total_dropped;
    return CS_OK;
}
int32_t cs_get_mass_units_per_ml(const CsSim* sim, float* out) {
    CS_SIM(sim);
    CS_PTR(out);
    *out = sim->e->settings.brew.water_mass_units_per_ml;
    return CS_OK;
}
int32_t cs_get_metrics(CsSim* sim, CsMetrics* out) {
    CS_SIM(sim);
    CS_PTR(out);
    return sim->e->metrics(out);
}
int32_t cs_metrics_request(CsSim* sim) {
    CS_SIM(sim);
    return sim->e->metrics_request();
}
int32_t cs_metrics_wait(CsSim* sim, CsMetrics* out) {
    CS_SIM(sim);
    CS_PTR(out);
    return sim->e->metrics_wait(out);
}
int32_t cs_get_settings(const CsSim* sim, CsSettings* out) {
    CS_SIM(sim);
    CS_PTR(out);
    *out = sim->e->settings;
    return CS_OK;
}
int32_t cs_read_particles(CsSim* s, uint32_t f, uint32_t c, float* o) {
    CS_SIM(s);
    CS_PTR(o);
    return s->e->read_particles(0, f, c, o);
}
int32_t cs_read_affine(CsSim* s, uint32_t f, uint32_t c, float* o) {
    CS_SIM(s);
    CS_PTR(o);
    return s->e->read_particles(1, f, c, o);
}
int32_t cs_read_bed_extract(CsSim* s, uint32_t f, uint32_t c, float* o) {
    CS_SIM(s);
    CS_PTR(o);
    return s->e->read_particles(2, f, c, o);
}
int32_t cs_read_render(CsSim* s, uint32_t f, uint32_t c, float* o) {
    CS_SIM(s);
    CS_PTR(o);
    return s->e->read_particles(3, f, c, o);
}
int32_t cs_read_grid_lanes(CsSim* s, int32_t* o) {
    CS_SIM(s);
    CS_PTR(o);
    return s->e->read_lanes(o);
}
int32_t cs_read_grid_lanes64(CsSim* s, int64_t* o) {
    CS_SIM(s);
    CS_PTR(o);
    if (s->e->settings.p2g_mode != CS_P2G_INT64) {
        set_error("not an int64 P2G simulation");
        return CS_ERR_INVALID_ARG;
    }
    return s->e->read_lanes64(o);
}
int32_t cs_read_grid_vel(CsSim* s, float* o) {
    CS_SIM(s);
    CS_PTR(o);
    return s->e->read_gvel(o);
}
int32_t cs_read_pressure(CsSim* s, float* o) {
    CS_SIM(s);
    CS_PTR(o);
    return s->e->read_pressure(o);
}
int32_t cs_read_cell_kind(CsSim* s, int32_t* o) {
    CS_SIM(s);
    CS_PTR(o);
    return s->e->read_kind(o);
}
int32_t cs_read_solver_inputs(CsSim* s, float* fill, float* div) {
    CS_SIM(s);
    CS_PTR(fill);
    CS_PTR(div);
    return s->e->read_solver_inputs(fill, div);
}
int32_t cs_read_bed_lookup(CsSim* s, int32_t* o) {
    CS_SIM(s);
    CS_PTR(o);
    return s->e->read_lookup(o);
}
int32_t cs_read_bed_delta(CsSim* s, int32_t* o) {
    CS_SIM(s);
    CS_PTR(o);
    return s->e->read_delta(o);
}
int32_t cs_read_sdf(CsSim* s, float* o) {
    CS_SIM(s);
    CS_PTR(o);
    return s->e->read_sdf(o);
}
int32_t cs_read_sdf_class(CsSim* s, uint8_t* o) {
    CS_SIM(s);
    CS_PTR(o);
    return s->e->read_class(o);
}
int32_t cs_write_particles(CsSim* s, uint32_t f, uint32_t c, const float* i) {
    CS_SIM(s);
    CS_PTR(i);
    return s->e->write_particles(0, f, c, i);
}
int32_t cs_write_affine(CsSim* s, uint32_t f, uint32_t c, const float* i) {
    CS_SIM(s);
    CS_PTR(i);
    return s->e->write_particles(1, f, c, i);
}
int32_t cs_write_bed_extract(CsSim* s, uint32_t f, uint32_t c, const float* i) {
    CS_SIM(s);
    CS_PTR(i);
    return s->e->write_particles(2, f, c, i);
}
int32_t cs_set_counts(CsSim* s, uint32_t nw, uint32_t nb) {
    CS_SIM(s);
    if ((uint64_t)nw + nb > s->e->settings.max_particles) {
        set_error("counts exceed max_particles");
        return CS_ERR_CAPACITY;
    }
    s->e->num_water = nw;
    s->e->num_bed = nb;
    return CS_OK;
}
int32_t cs_add_water_block(CsSim* s, const float lo[3], const float hi[3], uint32_t per_axis, float jitter,
                           uint32_t seed, uint32_t require_open_sdf, uint32_t* added) {
    CS_SIM(s);
    if (!lo || !hi || per_axis == 0) {
        set_error("bad water block arguments");
        return CS_ERR_INVALID_ARG;
    }
    return s->e->add_water_block(lo, hi, per_axis, jitter, seed, require_open_sdf, added);
}
int32_t cs_profile_enable(CsSim* s, int32_t on) {
    CS_SIM(s);
    return s->e->profile_enable(on != 0);
}
int32_t cs_profile_read(CsSim* s, CsProfile* out) {
    CS_SIM(s);
    CS_PTR(out);
    return s->e->profile_read(out);
}
int32_t cs_timer_start(CsSim* s) {
    CS_SIM(s);
    return s->e->timer_start();
}
int32_t cs_timer_stop(CsSim* s, float* ms) {
    CS_SIM(s);
    CS_PTR(ms);
    return s->e->timer_stop(ms);
}
int32_t cs_flush_l2(CsSim* s) {
    CS_SIM(s);
    return s->e->flush_l2();
}
int32_t cs_sync(CsSim* s) {
    CS_SIM(s);
    return s->e->sync();
}
int32_t cs_snapshot_size(CsSim* s, uint64_t* b) {
    CS_SIM(s);
    CS_PTR(b);
    return s->e->snapshot_size(b);
}
int32_t cs_snapshot_save(CsSim* s, void* buf, uint64_t b) {
    CS_SIM(s);
    CS_PTR(buf);
    return s->e->snapshot_save(buf, b);
}
int32_t cs_snapshot_load(CsSim* s, const void* buf, uint64_t b) {
    CS_SIM(s);
    CS_PTR(buf);
    return s->e->snapshot_load(buf, b);
}

}  // extern "C"
