"""Python mirror of the reference's `MpmSim3D` / `MpmSettings` (crates/sim-wasm/src/
mpm_3d/mod.rs:87-671) over the coffee_sim C ABI.

Method names and argument meanings follow the Rust methods so that tests read like
the reference's own (physics_tests.rs).  Every call goes through the shared library;
errors raise `CsError` with the library's message.
"""
import ctypes as C
import os
from pathlib import Path

import numpy as np

from . import _ffi
from ._ffi import CsMetrics, CsSettings, Library

_PKG = Path(__file__).resolve().parent
ENGINE_SO = _PKG / "libcoffee_sim_b200.so"
_engine = None


def engine_library():
    """Load the CUDA engine (libcoffee_sim_b200.so).  There is no CPU fallback: a
    missing or unloadable library raises."""
    global _engine
    if _engine is None:
        if not ENGINE_SO.exists():
            raise ImportError(
                f"{ENGINE_SO} is missing: build it with `python -m coffee_sim_b200.build` "
                "(nvcc, sm_100a); the engine has no CPU fallback"
            )
        _engine = Library(ENGINE_SO)
        if not _engine.is_gpu():
            raise ImportError(f"{ENGINE_SO} is not the GPU engine")
    return _engine


class MpmSettings:
    """Owns one CsSettings value (mod.rs:87-104 + engine extensions)."""

    def __init__(self, raw=None):
        self.raw = raw if raw is not None else CsSettings()

    @classmethod
    def _preset(cls, fn, lib=None):
        lib = lib or engine_library()
        s = cls()
        lib.call(fn, C.byref(s.raw))
        return s

    @classmethod
    def default_v60(cls, lib=None):
        return cls._preset("cs_settings_default_v60", lib)

    @classmethod
    def benchmark_free_stream(cls, lib=None):
        return cls._preset("cs_settings_benchmark_free_stream", lib)

    @classmethod
    def benchmark_center_pour(cls, lib=None):
        return cls._preset("cs_settings_benchmark_center_pour", lib)

    def copy(self):
        s = MpmSettings()
        C.memmove(C.byref(s.raw), C.byref(self.raw), C.sizeof(CsSettings))
        return s

    def __getattr__(self, name):
        raw = self.__dict__.get("raw")
        if raw is not None and hasattr(raw, name):
            return getattr(raw, name)
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name != "raw" and hasattr(self.raw, name):
            setattr(self.raw, name, value)
        else:
            object.__setattr__(self, name, value)

    @property
    def cells(self):
        g = self.raw.grid_dims
        return int(g[0]) * int(g[1]) * int(g[2])

    @property
    def dx(self):
        return np.float32(self.raw.bounds_size[0]) / np.float32(self.raw.grid_dims[0])

    @property
    def nominal_mass(self):
        b = self.raw.brew
        return np.float32(b.water_mass_units_per_ml) / np.float32(b.water_particles_per_ml)


class MpmSim3D:
    """One simulation handle (mod.rs:179-671).  `lib` defaults to the CUDA engine."""

    def __init__(self, settings, lib=None):
        self.lib = lib or engine_library()
        self.settings = settings.copy() if isinstance(settings, MpmSettings) else MpmSettings(settings)
        self._h = C.c_void_p()
        self.lib.call("cs_create", C.byref(self.settings.raw), C.byref(self._h))

    # -- lifetime --
    def close(self):
        if self._h:
            self.lib.lib.cs_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def reset(self):
        self.lib.call("cs_reset", self._h)

    # -- stepping --
    def step_frame(self, dt):
        self.lib.call("cs_step_frame", self._h, C.c_float(dt))

    def step_substep(self, sub_dt):
        self.lib.call("cs_step_substep", self._h, C.c_float(sub_dt))

    def step_substep_partial(self, sub_dt, passes):
        self.lib.call("cs_step_substep_partial", self._h, C.c_float(sub_dt), passes)

    # -- controls --
    def set_kettle_angle(self, deg):
        self.lib.call("cs_set_kettle_angle", self._h, C.c_float(deg))

    def set_spout_position(self, x, y, z):
        self.lib.call("cs_set_spout_position", self._h, C.c_float(x), C.c_float(y), C.c_float(z))

    def set_spout_target(self, x, y, z):
        self.lib.call("cs_set_spout_target", self._h, C.c_float(x), C.c_float(y), C.c_float(z))

    def set_flow_override(self, flow_ml_s, exit_speed):
        self.lib.call("cs_set_flow_override", self._h, C.c_float(flow_ml_s), C.c_float(exit_speed))

    # -- getters --
    def _counts(self):
        nw, nb, mp = C.c_uint32(), C.c_uint32(), C.c_uint32()
        self.lib.call("cs_get_counts", self._h, C.byref(nw), C.byref(nb), C.byref(mp))
        return nw.value, nb.value, mp.value

    @property
    def num_water(self):
        return self._counts()[0]

    @property
    def num_bed(self):
        return self._counts()[1]

    def particle_count(self):
        nw, nb, _ = self._counts()
        return nw + nb

    def water_slots_used(self):
        return self._counts()[0]

    def bed_particle_count(self):
        return self._counts()[1]

    def max_particles(self):
        return self._counts()[2]

    def kettle_angle(self):
        v = C.c_float()
        self.lib.call("cs_get_kettle_angle", self._h, C.byref(v))
        return v.value

    def spout_position(self):
        v = (C.c_float * 3)()
        self.lib.call("cs_get_spout_position", self._h, v)
        return tuple(v)

    def _flow(self):
        a, b, c = C.c_float(), C.c_float(), C.c_float()
        self.lib.call("cs_get_flow", self._h, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def flow_rate_ml_s(self):
        return self._flow()[0]

    def exit_speed(self):
        return self._flow()[1]

    def exit_speed_m_s(self):
        return self._flow()[2]

    def total_time(self):
        v = C.c_float()
        self.lib.call("cs_get_time", self._h, C.byref(v))
        return v.value

    def _emission(self):
        a, b = C.c_float(), C.c_float()
        c, d = C.c_uint32(), C.c_uint32()
        self.lib.call("cs_get_emission", self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(d))
        return a.value, b.value, c.value, d.value

    def frame_emitted_mass(self):
        return self._emission()[0]

    def total_emitted_mass(self):
        return self._emission()[1]

    def frame_dropped_particles(self):
        return self._emission()[2]

    def total_dropped_particles(self):
        return self._emission()[3]

    def frame_emitted_ml(self):
        return self.frame_emitted_mass() / float(self.settings.brew.water_mass_units_per_ml)

    def total_emitted_ml(self):
        return self.total_emitted_mass() / float(self.settings.brew.water_mass_units_per_ml)

    def latest_metrics(self):
        m = CsMetrics()
        self.lib.call("cs_get_metrics", self._h, C.byref(m))
        return m

    def metrics_request(self):
        """Queue a copy of the latest substep's metrics without waiting for the GPU."""
        self.lib.call("cs_metrics_request", self._h)

    def metrics_wait(self):
        """The metrics of the substep current at the last metrics_request()."""
        m = CsMetrics()
        self.lib.call("cs_metrics_wait", self._h, C.byref(m))
        return m

    # -- readback (reference byte layouts) --
    def _read_rows(self, fn, width, first, count, dtype=np.float32):
        if count is None:
            count = self.particle_count() - first
        out = np.zeros((max(count, 0), width), dtype=dtype)
        if count > 0:
            ptr = out.ctypes.data_as(C.POINTER(C.c_float))
            self.lib.call(fn, self._h, first, count, ptr)
        return out

    def read_particles(self, first=0, count=None):
        return self._read_rows("cs_read_particles", 8, first, count)

    def read_affine(self, first=0, count=None):
        return self._read_rows("cs_read_affine", 12, first, count)

    def read_bed_extract(self, first=0, count=None):
        if count is None:
            count = self.num_bed - first
        return self._read_rows("cs_read_bed_extract", 8, first, count)

    def read_render(self, first=0, count=None):
        return self._read_rows("cs_read_render", 8, first, count)

    def _read_cells(self, fn, dtype, width=1):
        n = self.settings.cells * width
        out = np.zeros(n, dtype=dtype)
        ctype = {np.float32: C.c_float, np.int32: C.c_int32, np.uint8: C.c_uint8}[dtype]
        self.lib.call(fn, self._h, out.ctypes.data_as(C.POINTER(ctype)))
        return out

    def read_grid_lanes(self):
        return self._read_cells("cs_read_grid_lanes", np.int32, 6).reshape(6, -1)

    def read_grid_lanes64(self):
        """P2G lanes of an int64-mode simulation: (6, cells) int64, value * 2^32."""
        out = np.zeros(6 * self.settings.cells, dtype=np.int64)
        self.lib.call("cs_read_grid_lanes64", self._h, out.ctypes.data_as(C.POINTER(C.c_int64)))
        return out.reshape(6, -1)

    def read_grid_vel(self):
        return self._read_cells("cs_read_grid_vel", np.float32, 4).reshape(-1, 4)

    def read_pressure(self):
        return self._read_cells("cs_read_pressure", np.float32)

    def read_cell_kind(self):
        return self._read_cells("cs_read_cell_kind", np.int32)

    def read_solver_inputs(self):
        """(fill, divergence) of every cell as classify wrote them for the pressure solve
        (FP32 pressure storage)."""
        n = self.settings.cells
        fill, div = np.zeros(n, np.float32), np.zeros(n, np.float32)
        self.lib.call("cs_read_solver_inputs", self._h, fill.ctypes.data_as(C.POINTER(C.c_float)),
                      div.ctypes.data_as(C.POINTER(C.c_float)))
        return fill, div

    def read_bed_lookup(self):
        return self._read_cells("cs_read_bed_lookup", np.int32)

    def read_sdf_class(self):
        return self._read_cells("cs_read_sdf_class", np.uint8)

    def read_sdf(self):
        out = np.zeros(128 ** 3, dtype=np.float32)
        self.lib.call("cs_read_sdf", self._h, out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    def read_bed_delta(self):
        n = 4 * self.max_particles()
        out = np.zeros(n, dtype=np.int32)
        self.lib.call("cs_read_bed_delta", self._h, out.ctypes.data_as(C.POINTER(C.c_int32)))
        return out.reshape(4, -1)

    # -- upload --
    def write_particles(self, first, rows):
        rows = np.ascontiguousarray(rows, dtype=np.float32)
        self.lib.call("cs_write_particles", self._h, first, rows.shape[0], rows.ctypes.data_as(C.POINTER(C.c_float)))

    def write_affine(self, first, rows):
        rows = np.ascontiguousarray(rows, dtype=np.float32)
        self.lib.call("cs_write_affine", self._h, first, rows.shape[0], rows.ctypes.data_as(C.POINTER(C.c_float)))

    def write_bed_extract(self, first, rows):
        rows = np.ascontiguousarray(rows, dtype=np.float32)
        self.lib.call("cs_write_bed_extract", self._h, first, rows.shape[0], rows.ctypes.data_as(C.POINTER(C.c_float)))

    def set_counts(self, num_water, num_bed):
        self.lib.call("cs_set_counts", self._h, num_water, num_bed)

    def add_water_block(self, lo, hi, per_axis=2, jitter=0.25, seed=0, require_open_sdf=False):
        lo_a = (C.c_float * 3)(*lo)
        hi_a = (C.c_float * 3)(*hi)
        added = C.c_uint32()
        self.lib.call(
            "cs_add_water_block", self._h, lo_a, hi_a, per_axis, C.c_float(jitter), seed,
            1 if require_open_sdf else 0, C.byref(added),
        )
        return added.value

    # -- device timing / profiling --
    def current_settings(self):
        """The simulation's settings as they are now (the tuner and setters change them)."""
        st = _ffi.CsSettings()
        self.lib.call("cs_get_settings", self._h, C.byref(st))
        return st

    def set_solver(self, omega=0.0, check_every=0, max_sweeps=0):
        """Residual-mode solver parameters from the next substep on (0 keeps a value)."""
        self.lib.call("cs_set_solver", self._h, C.c_float(omega), check_every, max_sweeps)

    def set_p2g_mode(self, mode):
        self.lib.call("cs_set_p2g_mode", self._h, mode)

    def set_learned_weights(self, params):
        """Weights of the pressure-guess U-Net (flat f32 vector, coffee_sim_b200.unet layout)."""
        a = np.ascontiguousarray(params, dtype=np.float32)
        self.lib.call("cs_set_learned_weights", self._h, a.ctypes.data_as(C.POINTER(C.c_float)), a.size)

    def learned_capture(self, on=True):
        self.lib.call("cs_learned_capture", self._h, 1 if on else 0)

    def learned_read_sample(self, feat, target, mask):
        """Copy the last captured (inputs, target, mask) into torch CUDA tensors; returns s."""
        sc = C.c_float()
        self.lib.call("cs_learned_read_sample", self._h, C.c_void_p(feat.data_ptr()), C.c_void_p(target.data_ptr()),
                      C.c_void_p(mask.data_ptr()), C.byref(sc))
        return sc.value

    def set_graph_mode(self, on):
        """Capture the substep in a CUDA graph and replay it (needs device emission)."""
        self.lib.call("cs_set_graph_mode", self._h, 1 if on else 0)

    def autotune(self, sub_dt, substeps=4):
        """Time candidate solver / P2G configurations from the current state and keep
        the fastest that converges; the state itself is left unchanged."""
        r = _ffi.CsTuneResult()
        self.lib.call("cs_autotune", self._h, C.c_float(sub_dt), substeps, C.byref(r))
        return r

    def profile_enable(self, on=True):
        self.lib.call("cs_profile_enable", self._h, 1 if on else 0)

    def profile_read(self):
        p = _ffi.CsProfile()
        self.lib.call("cs_profile_read", self._h, C.byref(p))
        return p

    def timer_start(self):
        self.lib.call("cs_timer_start", self._h)

    def timer_stop(self):
        ms = C.c_float()
        self.lib.call("cs_timer_stop", self._h, C.byref(ms))
        return ms.value

    def flush_l2(self):
        self.lib.call("cs_flush_l2", self._h)

    def sync(self):
        self.lib.call("cs_sync", self._h)

    # -- checkpoint --
    def snapshot(self):
        n = C.c_uint64()
        self.lib.call("cs_snapshot_size", self._h, C.byref(n))
        buf = (C.c_uint8 * n.value)()
        self.lib.call("cs_snapshot_save", self._h, buf, n.value)
        return bytes(buf)

    def restore(self, blob):
        buf = (C.c_uint8 * len(blob)).from_buffer_copy(blob)
        self.lib.call("cs_snapshot_load", self._h, buf, len(blob))


class MpmEnsemble:
    """n independent pours with one grid size stepped together on one GPU (the batched
    engine: every pass is one launch over all instances).  Engine extension without a
    reference counterpart; each instance reads back like an MpmSim3D."""

    def __init__(self, settings_list, lib=None):
        self.lib = lib if lib is not None else engine_library()
        self.settings = [s.copy() if isinstance(s, MpmSettings) else MpmSettings(s) for s in settings_list]
        arr = (_ffi.CsSettings * len(self.settings))(*[s.raw for s in self.settings])
        self._h = C.c_void_p()
        self.lib.call("cs_ensemble_create", arr, len(self.settings), C.byref(self._h))

    def __len__(self):
        return len(self.settings)

    def close(self):
        if self._h:
            self.lib.lib.cs_ensemble_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step_substep(self, sub_dt):
        self.lib.call("cs_ensemble_step_substep", self._h, C.c_float(sub_dt))

    def step_frame(self, dt):
        self.lib.call("cs_ensemble_step_frame", self._h, C.c_float(dt))

    def member(self, i):
        """A view of instance i with the add_water_block / settings interface that the
        scene builders use."""
        return _EnsembleMember(self, i)

    def add_water_block(self, i, lo, hi, per_axis=2, jitter=0.25, seed=0, require_open_sdf=False):
        lo_a = (C.c_float * 3)(*lo)
        hi_a = (C.c_float * 3)(*hi)
        added = C.c_uint32()
        self.lib.call("cs_ensemble_add_water_block", self._h, i, lo_a, hi_a, per_axis, C.c_float(jitter), seed,
                      1 if require_open_sdf else 0, C.byref(added))
        return added.value

    def set_kettle_angle(self, i, deg):
        self.lib.call("cs_ensemble_set_kettle_angle", self._h, i, C.c_float(deg))

    def set_flow_override(self, i, flow_ml_s, exit_speed):
        self.lib.call("cs_ensemble_set_flow_override", self._h, i, C.c_float(flow_ml_s), C.c_float(exit_speed))

    def counts(self, i):
        nw, nb = C.c_uint32(), C.c_uint32()
        self.lib.call("cs_ensemble_get_counts", self._h, i, C.byref(nw), C.byref(nb))
        return nw.value, nb.value

    def particle_count(self, i):
        return sum(self.counts(i))

    def read_particles(self, i, first=0, count=None):
        if count is None:
            count = self.particle_count(i) - first
        out = np.zeros((count, 8), dtype=np.float32)
        self.lib.call("cs_ensemble_read_particles", self._h, i, first, count,
                      out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    def metrics(self, i):
        m = _ffi.CsMetrics()
        self.lib.call("cs_ensemble_get_metrics", self._h, i, C.byref(m))
        return m

    def set_learned_weights(self, params):
        """One weight vector (coffee_sim_b200/unet.py layout) for every instance."""
        p = np.ascontiguousarray(params, dtype=np.float32)
        self.lib.call("cs_ensemble_set_learned_weights", self._h, p.ctypes.data_as(C.POINTER(C.c_float)), p.size)

    def timer_start(self):
        self.lib.call("cs_ensemble_timer_start", self._h)

    def timer_stop(self):
        """Device milliseconds since timer_start (CUDA events on the ensemble's stream)."""
        ms = C.c_float()
        self.lib.call("cs_ensemble_timer_stop", self._h, C.byref(ms))
        return ms.value


class _EnsembleMember:
    def __init__(self, ens, i):
        self.ens, self.i = ens, i
        self.settings = ens.settings[i]

    def add_water_block(self, lo, hi, per_axis=2, jitter=0.25, seed=0, require_open_sdf=False):
        return self.ens.add_water_block(self.i, lo, hi, per_axis, jitter, seed, require_open_sdf)
