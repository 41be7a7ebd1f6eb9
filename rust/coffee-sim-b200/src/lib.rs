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
}

impl Drop for MpmSim3D {
    fn drop(&mut self) {
        if !self.raw.is_null() {
            unsafe { sys::cs_destroy(self.raw) };
        }
    }
}
