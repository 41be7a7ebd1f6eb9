// kernels_api.h — small POD types passed by value to set-up kernels.
#pragma once
#include "../../include/coffee_sim.h"

namespace cs {
// Obstacles of the analytic SDF (mod.rs:71-85) for the SDF generation kernel.
struct SdfSpec {
    float bounds[3];
    float wall_thickness;
    uint32_t count;
    CsObstacle obs[CS_MAX_OBSTACLES];
};
}  // namespace cs
