// ensemble.cu — C ABI of the batched ensemble (cs::Ensemble in engine.cu): n
// independent pours with the same grid stepped together, each pass one launch over all
// instances.  No counterpart in the reference, which simulates one pour.
#include <memory>

#include "engine.h"

struct CsEnsemble {
    std::unique_ptr<cs::Ensemble> ens;
};

#define CS_ENS(e, i)                                       \
    if (!(e) || !(e)->ens) {                               \
        cs::set_error("null ensemble handle");             \
        return CS_ERR_INVALID_ARG;                         \
    }                                                      \
    if ((i) >= (e)->ens->size()) {                         \
        cs::set_error("ensemble instance index out of range"); \
        return CS_ERR_INVALID_ARG;                         \
    }

extern "C" {

int32_t cs_ensemble_create(const CsSettings* settings, uint32_t n, CsEnsemble** out) {
    if (!settings || !out) {
        cs::set_error("null argument to cs_ensemble_create");
        return CS_ERR_INVALID_ARG;
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cs::set_error("no CUDA device visible");
        return CS_ERR_NO_DEVICE;
    }
    std::unique_ptr<CsEnsemble> e(new CsEnsemble());
    e->ens.reset(new cs::Ensemble());
    int rc = e->ens->init(settings, n);
    if (rc) return rc;
    *out = e.release();
    return CS_OK;
}

int32_t cs_ensemble_destroy(CsEnsemble* ens) {
    delete ens;
    return CS_OK;
}

int32_t cs_ensemble_step_substep(CsEnsemble* e, float sub_dt) {
    CS_ENS(e, 0u);
    for (uint32_t i = 0; i < e->ens->size(); ++i) {
        e->ens->at(i).frame_emitted_mass = 0.0f;
        e->ens->at(i).frame_dropped = 0;
    }
    return e->ens->substep(sub_dt);
}

int32_t cs_ensemble_step_frame(CsEnsemble* e, float dt) {
    CS_ENS(e, 0u);
    return e->ens->step_frame(dt);
}

int32_t cs_ensemble_set_learned_weights(CsEnsemble* e, const float* params, uint64_t count) {
    CS_ENS(e, 0u);
    if (!params) {
        cs::set_error("null weights");
        return CS_ERR_INVALID_ARG;
    }
    int rc = e->ens->sync();
    if (rc) return rc;
    for (uint32_t i = 0; i < e->ens->size(); ++i)
        if ((rc = e->ens->at(i).set_learned_weights(params, count))) return rc;
    return CS_OK;
}

int32_t cs_ensemble_timer_start(CsEnsemble* e) {
    CS_ENS(e, 0u);
    return e->ens->timer_start();
}

int32_t cs_ensemble_timer_stop(CsEnsemble* e, float* ms) {
    CS_ENS(e, 0u);
    if (!ms) {
        cs::set_error("null output pointer");
        return CS_ERR_INVALID_ARG;
    }
    return e->ens->timer_stop(ms);
}

int32_t cs_ensemble_add_water_block(CsEnsemble* e, uint32_t i, const float lo[3], const float hi[3],
                                    uint32_t per_axis, float jitter, uint32_t seed, uint32_t require_open_sdf,
                                    uint32_t* added) {
    CS_ENS(e, i);
    if (!lo || !hi) {
        cs::set_error("null block bounds");
        return CS_ERR_INVALID_ARG;
    }
    int rc = e->ens->sync();
    if (rc) return rc;
    return e->ens->at(i).add_water_block(lo, hi, per_axis, jitter, seed, require_open_sdf, added);
}

int32_t cs_ensemble_set_kettle_angle(CsEnsemble* e, uint32_t i, float angle_deg) {
    CS_ENS(e, i);
    e->ens->at(i).inflow.angle = angle_deg;  // as cs_set_kettle_angle
    return CS_OK;
}

int32_t cs_ensemble_set_flow_override(CsEnsemble* e, uint32_t i, float flow_ml_s, float exit_speed) {
    CS_ENS(e, i);
    cs::Engine& g = e->ens->at(i);
    g.inflow.flow_override = flow_ml_s > 0.0f ? flow_ml_s : 0.0f;
    g.inflow.speed_override = flow_ml_s > 0.0f ? exit_speed : 0.0f;
    return CS_OK;
}

int32_t cs_ensemble_get_counts(CsEnsemble* e, uint32_t i, uint32_t* num_water, uint32_t* num_bed) {
    CS_ENS(e, i);
    if (num_water) *num_water = e->ens->at(i).num_water;
    if (num_bed) *num_bed = e->ens->at(i).num_bed;
    return CS_OK;
}

int32_t cs_ensemble_read_particles(CsEnsemble* e, uint32_t i, uint32_t first, uint32_t count, float* out) {
    CS_ENS(e, i);
    if (!out) {
        cs::set_error("null output pointer");
        return CS_ERR_INVALID_ARG;
    }
    int rc = e->ens->sync();
    if (rc) return rc;
    return e->ens->at(i).read_particles(0, first, count, out);
}

int32_t cs_ensemble_get_metrics(CsEnsemble* e, uint32_t i, CsMetrics* out) {
    CS_ENS(e, i);
    if (!out) {
        cs::set_error("null output pointer");
        return CS_ERR_INVALID_ARG;
    }
    int rc = e->ens->sync();
    if (rc) return rc;
    return e->ens->at(i).metrics(out);
}

}  // extern "C"
