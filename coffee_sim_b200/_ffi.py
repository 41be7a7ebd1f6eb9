"""ctypes mirror of include/coffee_sim.h.

Struct layouts follow the header field by field; `bind(lib)` attaches argument and
return types to every exported function of a library that implements the C ABI.
"""
import ctypes as C

CS_ABI_VERSION = 5
CS_MAX_OBSTACLES = 4

STATUS = {
    0: "CS_OK",
    1: "CS_ERR_INVALID_ARG",
    2: "CS_ERR_CAPACITY",
    3: "CS_ERR_CUDA",
    4: "CS_ERR_NAN",
    5: "CS_ERR_OVERFLOW",
    6: "CS_ERR_TIMEOUT",
    7: "CS_ERR_UNSUPPORTED",
    8: "CS_ERR_NO_DEVICE",
}
CS_OK, CS_ERR_INVALID_ARG, CS_ERR_CAPACITY, CS_ERR_CUDA, CS_ERR_NAN = 0, 1, 2, 3, 4
CS_ERR_OVERFLOW, CS_ERR_TIMEOUT, CS_ERR_UNSUPPORTED, CS_ERR_NO_DEVICE = 5, 6, 7, 8

CS_OBSTACLE_TRUNCATED_CONE = 0
CS_OBSTACLE_CYLINDER = 1
CS_GEOM_CONE, CS_GEOM_FILTER, CS_GEOM_CUP = 1, 2, 4
CS_PRESSURE_FIXED_POINT, CS_PRESSURE_FP32 = 0, 1
CS_SOLVE_FIXED_PAIRS, CS_SOLVE_RESIDUAL = 0, 1
CS_P2G_ATOMIC32, CS_P2G_SORTED_SHARED, CS_P2G_INT64 = 0, 1, 2
CS_WARM_NONE, CS_WARM_PREVIOUS, CS_WARM_LEARNED = 0, 1, 2

F3 = C.c_float * 3


class CsObstacle(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("center", F3),
        ("top_radius", C.c_float),
        ("bot_radius", C.c_float),
        ("radius", C.c_float),
        ("top_y", C.c_float),
        ("bot_y", C.c_float),
    ]


class CsSpout(C.Structure):
    _fields_ = [
        ("origin", F3),
        ("direction", F3),
        ("target", F3),
        ("nozzle_radius", C.c_float),
        ("stem_radius", C.c_float),
        ("activation_angle_deg", C.c_float),
        ("full_flow_angle_deg", C.c_float),
        ("head_at_activation", C.c_float),
        ("head_at_full_angle", C.c_float),
        ("discharge_coeff", C.c_float),
        ("volume_to_ml", C.c_float),
        ("max_flow_rate_ml_s", C.c_float),
        ("gentle_exit_speed", C.c_float),
        ("max_exit_speed", C.c_float),
        ("stem_length", C.c_float),
    ]


class CsFilter(C.Structure):
    _fields_ = [
        ("center", F3),
        ("top_y", C.c_float),
        ("bot_y", C.c_float),
        ("top_radius", C.c_float),
        ("bot_radius", C.c_float),
        ("thickness", C.c_float),
        ("hole_radius", C.c_float),
    ]


class CsBed(C.Structure):
    _fields_ = [
        ("center", F3),
        ("top_y", C.c_float),
        ("bot_y", C.c_float),
        ("top_radius", C.c_float),
        ("bot_radius", C.c_float),
        ("num_particles", C.c_uint32),
        ("initial_porosity", C.c_float),
        ("initial_permeability", C.c_float),
        ("extractable_mass", C.c_float),
        ("log_perm_sigma", C.c_float),
        ("perm_seed", C.c_uint32),
        ("layer_split_y", C.c_float),
        ("lower_porosity_scale", C.c_float),
        ("lower_permeability_scale", C.c_float),
    ]


class CsBrew(C.Structure):
    _fields_ = [
        (n, C.c_float)
        for n in (
            "water_particles_per_ml",
            "water_mass_units_per_ml",
            "water_sample_radius_dx",
            "bed_sample_radius_dx",
            "water_kinematic_viscosity_m2_s",
            "min_bed_permeability_m2",
            "bed_absorption_rate",
            "target_bed_retention_ml",
            "bed_pore_capacity_scale",
            "bed_pore_overfill_alpha",
            "bed_surface_void_scale",
            "dripper_outlet_radius",
            "filter_absorption_rate_s",
            "bed_compaction_rate",
            "bed_impact_rate",
        )
    ]


class CsGeometry(C.Structure):
    _fields_ = [("flags", C.c_uint32)] + [
        (n, C.c_float)
        for n in (
            "cone_bot_y",
            "cone_top_y",
            "cone_radius_span",
            "filter_center_y",
            "filter_top_rel",
            "filter_bot_rel",
            "filter_top_radius",
            "filter_thickness",
            "cup_top_y",
            "cup_radius",
            "cup_floor_y",
            "wall_thickness",
            "bed_surface_ref_y",
            "bed_surface_span",
            "sdf_friction",
            "sdf_restitution",
            "contact_offset",
        )
    ]


class CsSettings(C.Structure):
    _fields_ = [
        ("abi_version", C.c_uint32),
        ("bounds_size", F3),
        ("grid_dims", C.c_uint32 * 3),
        ("max_particles", C.c_uint32),
        ("substeps", C.c_uint32),
        ("gravity", C.c_float),
        ("bulk_modulus", C.c_float),
        ("viscosity", C.c_float),
        ("render_radius", C.c_float),
        ("pressure_rbgs_pairs", C.c_uint32),
        ("use_sdf_cache", C.c_uint32),
        ("num_obstacles", C.c_uint32),
        ("obstacles", CsObstacle * CS_MAX_OBSTACLES),
        ("spout", CsSpout),
        ("initial_kettle_angle_deg", C.c_float),
        ("has_filter", C.c_uint32),
        ("filter", CsFilter),
        ("has_bed", C.c_uint32),
        ("bed", CsBed),
        ("brew", CsBrew),
        ("geom", CsGeometry),
        ("sim_units_per_meter", C.c_float),
        ("standard_gravity_m_s2", C.c_float),
        ("max_velocity", C.c_float),
        ("particle_volume_cells", C.c_float),
        ("max_frame_dt", C.c_float),
        ("pressure_storage", C.c_uint32),
        ("solve_mode", C.c_uint32),
        ("residual_tol", C.c_float),
        ("max_sweeps", C.c_uint32),
        ("check_every", C.c_uint32),
        ("warm_start", C.c_uint32),
        ("p2g_mode", C.c_uint32),
        ("sort_every", C.c_uint32),
        ("device_emission", C.c_uint32),
        ("use_graph", C.c_uint32),
        ("device", C.c_int32),
        ("rbgs_kernel", C.c_uint32),
        ("flow_override_ml_s", C.c_float),
        ("exit_speed_override", C.c_float),
        ("rbgs_omega", C.c_float),
        ("first_check", C.c_uint32),
        ("reorder_every", C.c_uint32),
        ("p2g_tile", C.c_uint32),
        ("particle_threads", C.c_uint32),
        ("reserved", C.c_uint32 * 3),
    ]


class CsMetrics(C.Structure):
    _fields_ = [
        ("max_abs_div", C.c_float),
        ("fluid_cells", C.c_uint32),
        ("div_clamp_fires", C.c_uint32),
        ("pressure_clamp_fires", C.c_uint32),
        ("mass_overflow_fires", C.c_uint32),
        ("last_sweeps", C.c_uint32),
        ("last_residual", C.c_double),
        ("initial_residual", C.c_double),
        ("nan_flag", C.c_uint32),
        ("timeout_flag", C.c_uint32),
        ("learned_used", C.c_uint32),
        ("residual_checks", C.c_uint32),
        ("solve_ms", C.c_double),
    ]


CS_PHASE_COUNT = 16
PHASE_NAMES = ["emit", "clear", "p2g", "grid", "sweeps", "residual", "project", "g2p", "bed", "render", "learned"]


class CsProfile(C.Structure):
    _fields_ = [
        ("phase_ms", C.c_double * CS_PHASE_COUNT),
        ("phase_launches", C.c_uint32 * CS_PHASE_COUNT),
        ("launches", C.c_uint64),
        ("sweeps", C.c_uint64),
        ("residual_evals", C.c_uint64),
        ("h2d_bytes", C.c_uint64),
        ("d2h_bytes", C.c_uint64),
        ("substeps", C.c_uint64),
    ]



class CsTuneResult(C.Structure):
    _fields_ = [
        ("omega", C.c_float),
        ("check_every", C.c_uint32),
        ("p2g_mode", C.c_uint32),
        ("trials", C.c_uint32),
        ("best_ms", C.c_float),
        ("initial_ms", C.c_float),
        ("first_check", C.c_uint32),
        ("p2g_tile", C.c_uint32),
        ("particle_threads", C.c_uint32),
    ]


P = C.c_void_p
I32, U32, U64, F32 = C.c_int32, C.c_uint32, C.c_uint64, C.c_float
PF = C.POINTER(C.c_float)
PI32 = C.POINTER(C.c_int32)
PU32 = C.POINTER(C.c_uint32)
PU8 = C.POINTER(C.c_uint8)
PU64 = C.POINTER(C.c_uint64)
PS = C.POINTER(CsSettings)
PM = C.POINTER(CsMetrics)

# name -> (restype, argtypes); every function declared by include/coffee_sim.h.
PROTOTYPES = {
    "cs_last_error_string": (C.c_char_p, []),
    "cs_abi_version": (U32, []),
    "cs_is_gpu_engine": (I32, []),
    "cs_settings_default_v60": (I32, [PS]),
    "cs_kozeny_carman_permeability_m2": (F32, [F32, F32]),
    "cs_settings_benchmark_free_stream": (I32, [PS]),
    "cs_settings_benchmark_center_pour": (I32, [PS]),
    "cs_settings_aim_spout": (I32, [PS, F32, F32, F32]),
    "cs_create": (I32, [PS, C.POINTER(P)]),
    "cs_destroy": (I32, [P]),
    "cs_reset": (I32, [P]),
    "cs_step_frame": (I32, [P, F32]),
    "cs_step_substep": (I32, [P, F32]),
    "cs_step_substep_partial": (I32, [P, F32, U32]),
    "cs_set_kettle_angle": (I32, [P, F32]),
    "cs_set_spout_position": (I32, [P, F32, F32, F32]),
    "cs_set_spout_target": (I32, [P, F32, F32, F32]),
    "cs_set_flow_override": (I32, [P, F32, F32]),
    "cs_get_counts": (I32, [P, PU32, PU32, PU32]),
    "cs_get_kettle_angle": (I32, [P, PF]),
    "cs_get_spout_position": (I32, [P, PF]),
    "cs_get_flow": (I32, [P, PF, PF, PF]),
    "cs_get_time": (I32, [P, PF]),
    "cs_get_emission": (I32, [P, PF, PF, PU32, PU32]),
    "cs_get_mass_units_per_ml": (I32, [P, PF]),
    "cs_get_metrics": (I32, [P, PM]),
    "cs_metrics_request": (I32, [P]),
    "cs_metrics_wait": (I32, [P, PM]),
    "cs_get_settings": (I32, [P, PS]),
    "cs_read_particles": (I32, [P, U32, U32, PF]),
    "cs_read_affine": (I32, [P, U32, U32, PF]),
    "cs_read_bed_extract": (I32, [P, U32, U32, PF]),
    "cs_read_grid_lanes": (I32, [P, PI32]),
    "cs_read_grid_lanes64": (I32, [P, C.POINTER(C.c_int64)]),
    "cs_read_grid_vel": (I32, [P, PF]),
    "cs_read_pressure": (I32, [P, PF]),
    "cs_read_cell_kind": (I32, [P, PI32]),
    "cs_read_solver_inputs": (I32, [P, PF, PF]),
    "cs_read_bed_lookup": (I32, [P, PI32]),
    "cs_read_bed_delta": (I32, [P, PI32]),
    "cs_read_render": (I32, [P, U32, U32, PF]),
    "cs_read_sdf": (I32, [P, PF]),
    "cs_read_sdf_class": (I32, [P, PU8]),
    "cs_write_particles": (I32, [P, U32, U32, PF]),
    "cs_write_affine": (I32, [P, U32, U32, PF]),
    "cs_write_bed_extract": (I32, [P, U32, U32, PF]),
    "cs_set_counts": (I32, [P, U32, U32]),
    "cs_add_water_block": (I32, [P, PF, PF, U32, F32, U32, U32, PU32]),
    "cs_snapshot_size": (I32, [P, PU64]),
    "cs_snapshot_save": (I32, [P, P, U64]),
    "cs_snapshot_load": (I32, [P, P, U64]),
    "cs_ensemble_create": (I32, [PS, U32, C.POINTER(P)]),
    "cs_ensemble_destroy": (I32, [P]),
    "cs_ensemble_step_substep": (I32, [P, F32]),
    "cs_ensemble_step_frame": (I32, [P, F32]),
    "cs_ensemble_add_water_block": (I32, [P, U32, PF, PF, U32, F32, U32, U32, PU32]),
    "cs_ensemble_set_kettle_angle": (I32, [P, U32, F32]),
    "cs_ensemble_set_flow_override": (I32, [P, U32, F32, F32]),
    "cs_ensemble_get_counts": (I32, [P, U32, PU32, PU32]),
    "cs_ensemble_read_particles": (I32, [P, U32, U32, U32, PF]),
    "cs_ensemble_get_metrics": (I32, [P, U32, PM]),
    "cs_ensemble_set_learned_weights": (I32, [P, PF, U64]),
    "cs_ensemble_timer_start": (I32, [P]),
    "cs_ensemble_timer_stop": (I32, [P, C.POINTER(C.c_float)]),
    "cs_profile_enable": (I32, [P, I32]),
    "cs_profile_read": (I32, [P, C.POINTER(CsProfile)]),
    "cs_timer_start": (I32, [P]),
    "cs_timer_stop": (I32, [P, PF]),
    "cs_flush_l2": (I32, [P]),
    "cs_sync": (I32, [P]),
    "cs_set_learned_weights": (I32, [P, PF, U64]),
    "cs_learned_capture": (I32, [P, U32]),
    "cs_learned_read_sample": (I32, [P, P, P, P, PF]),
    "cs_set_solver": (I32, [P, F32, U32, U32]),
    "cs_set_p2g_mode": (I32, [P, U32]),
    "cs_set_graph_mode": (I32, [P, U32]),
    "cs_autotune": (I32, [P, F32, U32, C.POINTER(CsTuneResult)]),
    "cs_nn_conv3d": (I32, [P, P, P, P, P, I32, I32, I32, I32, I32, I32, P, P]),
    "cs_nn_conv3d_wgrad": (I32, [P, P, P, I32, I32, I32, I32, I32, I32, P, P]),
    "cs_nn_pack_weights": (I32, [P, P, I32, I32, I32, I32, I32, P]),
    "cs_nn_pool": (I32, [P, P, P, P, I32, I32, I32, I32, I32, P]),
    "cs_nn_upcat": (I32, [P, P, P, P, P, P, I32, I32, I32, I32, I32, I32, P]),
    "cs_nn_relu_grad": (I32, [P, P, P, P, C.c_int64, I32, P]),
    "cs_nn_head": (I32, [P, P, P, P, P, P, C.c_int64, I32, I32, P]),
    "cs_nn_mse": (I32, [P, P, P, P, P, C.c_int64, F32, P]),
    "cs_nn_wgrad_master": (I32, [P, P, I32, I32, I32, P]),
    "cs_nn_adam": (I32, [P, P, P, P, C.c_int64, F32, F32, F32, F32, I32, P]),
    "cs_nn_axpy": (I32, [P, P, F32, C.c_int64, P]),
    "cs_pressure_solve_noalloc": (I32, [U32, U32, U32, F32, F32, F32, F32, U32, U32, P, P, P, P, P, P, PU32,
                                       C.POINTER(C.c_double)]),
}


class CsError(RuntimeError):
    """Raised when a C-ABI call returns a non-zero status."""

    def __init__(self, code, func, msg):
        self.code = code
        super().__init__(f"{func} failed with {STATUS.get(code, code)}: {msg}")


class Library:
    """A loaded shared library implementing the coffee_sim C ABI."""

    def __init__(self, path, required=True):
        self.path = str(path)
        self.lib = C.CDLL(self.path)
        self.missing = []
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(self.lib, name, None)
            if fn is None:
                self.missing.append(name)
                continue
            fn.restype = res
            fn.argtypes = args
        if required and "cs_create" in self.missing:
            raise OSError(f"{self.path} does not export the coffee_sim C ABI")

    def has(self, name):
        return name not in self.missing

    def call(self, name, *args):
        fn = getattr(self.lib, name)
        rc = fn(*args)
        if rc != 0:
            msg = self.lib.cs_last_error_string()
            raise CsError(rc, name, msg.decode() if msg else "")
        return rc

    def is_gpu(self):
        return bool(self.lib.cs_is_gpu_engine())
