// ensemble.cu — batched ensemble of independent pours (placeholder entry points
// until the batched engine lands).
#include "engine.h"

extern "C" {
int32_t cs_ensemble_create(const CsSettings*, uint32_t, CsEnsemble**) {
    cs::set_error("ensemble not built");
    return CS_ERR_UNSUPPORTED;
}
int32_t cs_ensemble_destroy(CsEnsemble*) { return CS_OK; }
int32_t cs_ensemble_step_substep(CsEnsemble*, float) { return CS_ERR_UNSUPPORTED; }
int32_t cs_ensemble_step_frame(CsEnsemble*, float) { return CS_ERR_UNSUPPORTED; }
int32_t cs_ensemble_add_water_block(CsEnsemble*, uint32_t, const float*, const float*, uint32_t, float, uint32_t,
                                    uint32_t, uint32_t*) {
    return CS_ERR_UNSUPPORTED;
}
int32_t cs_ensemble_set_kettle_angle(CsEnsemble*, uint32_t, float) { return CS_ERR_UNSUPPORTED; }
int32_t cs_ensemble_set_flow_override(CsEnsemble*, uint32_t, float, float) { return CS_ERR_UNSUPPORTED; }
int32_t cs_ensemble_get_counts(CsEnsemble*, uint32_t, uint32_t*, uint32_t*) { return CS_ERR_UNSUPPORTED; }
int32_t cs_ensemble_read_particles(CsEnsemble*, uint32_t, uint32_t, uint32_t, float*) { return CS_ERR_UNSUPPORTED; }
int32_t cs_ensemble_get_metrics(CsEnsemble*, uint32_t, CsMetrics*) { return CS_ERR_UNSUPPORTED; }
}
