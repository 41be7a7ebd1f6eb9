"""The Rust crates cannot be compiled in this image (no cargo), so this checks on the CPU
that every C function and type the safe wrapper names through the bindgen crate is one
include/coffee_sim.h declares (bindgen generates the raw bindings from that header)."""
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _header():
    return (ROOT / "include" / "coffee_sim.h").read_text()


def _wrapper():
    return (ROOT / "rust" / "coffee-sim-b200" / "src" / "lib.rs").read_text()


def test_wrapper_calls_only_declared_functions():
    header = _header()
    declared = set(re.findall(r"\b(cs_\w+)\s*\(", header))
    used = set(re.findall(r"sys::(cs_\w+)", _wrapper()))
    assert used, "the wrapper names no engine function"
    assert used <= declared, sorted(used - declared)


def test_wrapper_types_are_declared():
    header = _header()
    declared = set(re.findall(r"\b(Cs\w+)\b", header))
    used = set(re.findall(r"sys::(Cs\w+)", _wrapper()))
    assert used <= declared, sorted(used - declared)


def test_bindgen_allowlists_cover_the_wrapper():
    build = (ROOT / "rust" / "coffee-sim-b200-sys" / "build.rs").read_text()
    assert '.allowlist_function("cs_.*")' in build
    assert '.allowlist_type("Cs.*")' in build
    # the wrapper builds its out-structs with Default
    assert ".derive_default(true)" in build
