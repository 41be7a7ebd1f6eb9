//! Safe wrapper over the B200 MLS-MPM engine with the method names of the reference's
//! `MpmSim3D` (crates/sim-wasm/src/mpm_3d/mod.rs:179-671), so a Rust host can swap its
//! wgpu simulation for this one.  The handle owns all device memory and its CUDA stream;
//! readbacks copy into caller-owned vectors in the reference byte layouts (8 f32 per
//! particle: pos.xyz, J, vel.xyz, mass).

use coffee_sim_b200_sys as sys;
use std::ffi::CStr;
use std::fmt;

/// Non-zero status of an engine call with the engine's message.
#[derive(Debug, Clone)]
pub struct CsError {
    pub code: i32,
    pub message: String,
}

impl fmt::Display for CsError {
    fn fmt(&self, f: &mut fmt::Formatter<'_>) -> fmt::Result {
        write!(f, "coffee_sim status {}: {}", self.code, self.message)
    }
}

impl std::error::Error for CsError {}

fn check(code: i32) -> Result<(), CsError> {
    if code == 0 {
        return Ok(());
    }
    let message = unsafe {
        let p = sys::cs_last_error_string();
        if p.is_null() { String::new() } else { CStr::from_ptr(p).to_string_lossy().into_owned() }
    };
    Err(CsError { code, message })
}

/// Settings of one simulation (MpmSettings, mod.rs:87-104, plus engine extensions).
pub type MpmSettings = sys::CsSettings;

/// The reference's presets (mod.rs:107-160).
pub fn default_v60() -> Result<MpmSettings, CsError> {
    let mut s = MpmSettings::default();
    check(unsafe { sys::cs_settings_default_v60(&mut s) })?;
    Ok(s)
}
pub fn benchmark_center_pour() -> Result<MpmSettings, CsError> {
    let mut s = MpmSettings::default();
    check(unsafe { sys::cs_settings_benchmark_center_pour(&mut s) })?;
    Ok(s)
}
pub fn benchmark_free_stream() -> Result<MpmSettings, CsError> {
    let mut s = MpmSettings::default();
    check(unsafe { sys::cs_settings_benchmark_free_stream(&mut s) })?;
    Ok(s)
}

/// One pour on one GPU.
pub struct MpmSim3D {
    raw: *mut sys::CsSim,
}

// The handle may move between threads; calls on one handle must not overlap.
unsafe impl Send for MpmSim3D {}

impl MpmSim3D {
    pub fn new(settings: &MpmSettings) -> Result<Self, CsError> {
        let mut raw = std::ptr::null_mut();
        check(unsafe { sys::cs_create(settings, &mut raw) })?;
        Ok(Self { raw })
    }
    pub fn step_frame(&mut self, dt: f32) -> Result<(), CsError> {
        check(unsafe { sys::cs_step_frame(self.raw, dt) })
    }
    pub fn reset(&mut self) -> Result<(), CsError> {
        check(unsafe { sys::cs_reset(self.raw) })
    }
    pub fn set_kettle_angle(&mut self, degrees: f32) -> Result<(), CsError> {
        check(unsafe { sys::cs_set_kettle_angle(self.raw, degrees) })
    }
    pub fn set_spout_position(&mut self, x: f32, y: f32, z: f32) -> Result<(), CsError> {
        check(unsafe { sys::cs_set_spout_position(self.raw, x, y, z) })
    }
    pub fn set_spout_target(&mut self, x: f32, y: f32, z: f32) -> Result<(), CsError> {
        check(unsafe { sys::cs_set_spout_target(self.raw, x, y, z) })
    }
    /// (water samples, bed samples, capacity)
    pub fn counts(&self) -> Result<(u32, u32, u32), CsError> {
        let (mut w, mut b, mut m) = (0u32, 0u32, 0u32);
        check(unsafe { sys::cs_get_counts(self.raw, &mut w, &mut b, &mut m) })?;
        Ok((w, b, m))
    }
    pub fn particle_count(&self) -> Result<u32, CsError> {
        let (w, b, _) = self.counts()?;
        Ok(w + b)
    }
    pub fn sim_time(&self) -> Result<f32, CsError> {
        let mut t = 0.0f32;
        check(unsafe { sys::cs_get_time(self.raw, &mut t) })?;
        Ok(t)
    }
    pub fn kettle_angle(&self) -> Result<f32, CsError> {
        let mut a = 0.0f32;
        check(unsafe { sys::cs_get_kettle_angle(self.raw, &mut a) })?;
        Ok(a)
    }
    /// Particles [first, first + count) as 8 f32 each (state.rs:90-101 layout).
    pub fn read_particles(&self, first: u32, count: u32) -> Result<Vec<f32>, CsError> {
        let mut out = vec![0.0f32; count as usize * 8];
        check(unsafe { sys::cs_read_particles(self.raw, first, count, out.as_mut_ptr()) })?;
        Ok(out)
    }
    /// Bed extract of the bed samples as 8 f32 each (state.rs:119-133 layout).
    pub fn read_bed_extract(&self, first: u32, count: u32) -> Result<Vec<f32>, CsError> {
        let mut out = vec![0.0f32; count as usize * 8];
        check(unsafe { sys::cs_read_bed_extract(self.raw, first, count, out.as_mut_ptr()) })?;
        Ok(out)
    }
    /// Solver and clamp counters of the last substep (synchronises).
    pub fn metrics(&self) -> Result<sys::CsMetrics, CsError> {
        let mut m = sys::CsMetrics::default();
        check(unsafe { sys::cs_get_metrics(self.raw, &mut m) })?;
        Ok(m)
    }
    /// Queue a copy of the latest substep's metrics without waiting for the GPU
    /// (engine extension; pair with `metrics_wait` after queuing the next step).
    pub fn metrics_request(&mut self) -> Result<(), CsError> {
        check(unsafe { sys::cs_metrics_request(self.raw) })
    }
    /// The metrics queued by the last `metrics_request`; waits for that copy only.
    pub fn metrics_wait(&mut self) -> Result<sys::CsMetrics, CsError> {
        let mut m = sys::CsMetrics::default();
        check(unsafe { sys::cs_metrics_wait(self.raw, &mut m) })?;
        Ok(m)
    }
    /// One substep of `sub_dt` seconds (engine extension: the reference steps whole
    /// frames, split into its substeps).
    pub fn step_substep(&mut self, sub_dt: f32) -> Result<(), CsError> {
        check(unsafe { sys::cs_step_substep(self.raw, sub_dt) })
    }
    /// Jet flow in ml/s and exit speed in m/s in place of the kettle-angle flow (engine
    /// extension, for the configurations stated in SI).
    pub fn set_flow_override(&mut self, flow_ml_s: f32, exit_speed: f32) -> Result<(), CsError> {
        check(unsafe { sys::cs_set_flow_override(self.raw, flow_ml_s, exit_speed) })
    }
    /// The settings the simulation runs with (after any `cs_set_*` or autotuner change).
    pub fn settings(&self) -> Result<MpmSettings, CsError> {
        let mut s = MpmSettings::default();
        check(unsafe { sys::cs_get_settings(self.raw, &mut s) })?;
        Ok(s)
    }
    /// The whole simulation state as bytes, for checkpoints (engine extension; the
    /// reference only has `reset`).
    pub fn snapshot(&self) -> Result<Vec<u8>, CsError> {
        let mut n = 0u64;
        check(unsafe { sys::cs_snapshot_size(self.raw, &mut n) })?;
        let mut out = vec![0u8; n as usize];
        check(unsafe { sys::cs_snapshot_save(self.raw, out.as_mut_ptr() as *mut std::ffi::c_void, n) })?;
        Ok(out)
    }
    /// Resumes from the bytes of `snapshot` (taken with the same settings).
    pub fn restore(&mut self, bytes: &[u8]) -> Result<(), CsError> {
        check(unsafe {
            sys::cs_snapshot_load(self.raw, bytes.as_ptr() as *const std::ffi::c_void, bytes.len() as u64)
        })
    }
    /// Times candidate solver settings and launch shapes over `substeps` substeps from
    /// the current state (restored after every trial), applies the fastest that reaches
    /// the residual target and returns it (engine extension).
    pub fn autotune(&mut self, sub_dt: f32, substeps: u32) -> Result<sys::CsTuneResult, CsError> {
        let mut r = sys::CsTuneResult::default();
        check(unsafe { sys::cs_autotune(self.raw, sub_dt, substeps, &mut r) })?;
        Ok(r)
    }
    /// Fill fraction and divergence of every cell as the last classify wrote them (the
    /// right-hand side of the pressure system), one f32 per cell each.
    pub fn read_solver_inputs(&self) -> Result<(Vec<f32>, Vec<f32>), CsError> {
        let s = self.settings()?;
        let cells: usize = s.grid_dims.iter().map(|&d| d as usize).product();
        let mut fill = vec![0.0f32; cells];
        let mut div = vec![0.0f32; cells];
        check(unsafe { sys::cs_read_solver_inputs(self.raw, fill.as_mut_ptr(), div.as_mut_ptr()) })?;
        Ok((fill, div))
    }
}

impl Drop for MpmSim3D {
    fn drop(&mut self) {
        if !self.raw.is_null() {
            unsafe { sys::cs_destroy(self.raw) };
        }
    }
}
