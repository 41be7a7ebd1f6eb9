// host_scene.h — host-side scene set-up of the engine: settings presets, the coffee
// bed lattice, and the spout inflow model.  These run on the host in the reference
// as well (mod.rs:106-177, bed.rs:41-314, inflow.rs:49-293; paths relative to
// crates/sim-wasm/src/mpm_3d/).  All arithmetic is f32 in source order.
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/coffee_sim.h"

namespace cs {
namespace host {

// units.rs:17-27
float units_per_meter_v60();
// brew_config.rs:92-96
float kozeny_carman_m2(float grind_um, float porosity);

void preset_default_v60(CsSettings* s);      // mod.rs:107-143
void preset_free_stream(CsSettings* s);      // mod.rs:145-152
void preset_center_pour(CsSettings* s);      // mod.rs:154-160
void spout_aim_at(CsSpout& sp, float x, float y, float z);                // inflow.rs:50-60
void spout_translate_origin_to(CsSpout& sp, float x, float y, float z);   // inflow.rs:62-66

struct BedSamples {
    std::vector<float> particles;  // 8 f32 per sample
    std::vector<float> affines;    // 12 f32 per sample
    std::vector<float> extracts;   // 8 f32 per sample
    std::vector<int32_t> lookup;   // cells
    uint32_t count = 0;
};
// bed.rs:107-314 (init_bed_particles + build_cell_lookup)
BedSamples init_bed(const CsBed& cfg, const uint32_t grid_dims[3], const float bounds[3]);

// InflowState (inflow.rs:69-120) with the constant-flow extension.
struct Inflow {
    float angle = 0.0f, flow_rate = 0.0f, exit_speed = 0.0f, accumulator = 0.0f;
    uint32_t sequence = 0;
    float flow_override = 0.0f, speed_override = 0.0f;
    void update(const CsSettings& s);
    // inflow.rs:133-163: how many samples to emit this substep.  Returns the count
    // actually emitted and sets *dropped.
    uint32_t plan(const CsSettings& s, float dt, uint32_t live, uint32_t* dropped);
};

// Jet emission geometry of one substep (inflow.rs:165-219), shared by the host
// emitter and the device emission kernel.
struct JetFrame {
    float t1[3], t2[3], vel[3], origin[3];
    float jet_radius, dt, particle_mass;
    uint32_t first_sequence, count, first_slot;
};
JetFrame jet_frame(const CsSettings& s, const Inflow& in, float dt, uint32_t count, uint32_t first_slot);
// Host emitter: fills 8+12 floats per sample (inflow.rs:196-218).
void emit_host(const JetFrame& jf, float* particles, float* affines);

// Seeded water-block generator shared by cs_add_water_block (no reference counterpart).
struct WaterBlock {
    std::vector<float> xyz;
};
WaterBlock water_block(const CsSettings& s, const float lo[3], const float hi[3], uint32_t per_axis, float jitter,
                       uint32_t seed);

}  // namespace host
}  // namespace cs
