// Generates the raw bindings from include/coffee_sim.h and links the engine library built
// by `python -m coffee_sim_b200.build` (coffee_sim_b200/libcoffee_sim_b200.so).
use std::env;
use std::path::PathBuf;

fn main() {
    let root = PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap()).join("../..");
    let header = root.join("include/coffee_sim.h");
    let libdir = env::var("COFFEE_SIM_B200_LIB_DIR")
        .map(PathBuf::from)
        .unwrap_or_else(|_| root.join("coffee_sim_b200"));
    println!("cargo:rerun-if-changed={}", header.display());
    println!("cargo:rerun-if-env-changed=COFFEE_SIM_B200_LIB_DIR");
    println!("cargo:rustc-link-search=native={}", libdir.display());
    println!("cargo:rustc-link-lib=dylib=coffee_sim_b200");
    let bindings = bindgen::Builder::default()
        .header(header.to_string_lossy())
        .allowlist_function("cs_.*")
        .allowlist_type("Cs.*")
        .allowlist_var("CS_.*")
        .derive_default(true)
        .generate()
        .expect("bindgen on include/coffee_sim.h");
    bindings
        .write_to_file(PathBuf::from(env::var("OUT_DIR").unwrap()).join("bindings.rs"))
        .expect("write bindings");
}
