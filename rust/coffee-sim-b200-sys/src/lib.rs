//! Raw `extern "C"` bindings to the B200 MLS-MPM engine, generated from
//! `include/coffee_sim.h`.  Every function returns an `i32` status (0 = `CS_OK`); the
//! text of the last error is `cs_last_error_string()`.  Use the `coffee-sim-b200` crate
//! for a safe wrapper with the method names of the reference's `MpmSim3D`.
#![allow(non_upper_case_globals, non_camel_case_types, non_snake_case, dead_code)]
include!(concat!(env!("OUT_DIR"), "/bindings.rs"));
