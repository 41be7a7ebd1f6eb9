"""The C ABI: every declared entry point is exported, struct layouts agree with the
ctypes mirror, presets agree between the engine and the oracle, and the engine
refuses to run without a GPU (no CPU fallback)."""
import ctypes as C
import re
import subprocess
import tempfile
from pathlib import Path

import pytest

from coffee_sim_b200 import _ffi
from coffee_sim_b200.sim import ENGINE_SO, MpmSettings

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "coffee_sim.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(cs_\w+)\s*\(", text, re.M)))


def test_header_declares_the_ffi_surface():
    names = declared_functions()
    assert "cs_create" in names and "cs_step_frame" in names
    assert set(names) == set(_ffi.PROTOTYPES), set(names) ^ set(_ffi.PROTOTYPES)


def test_engine_library_exports_every_declared_symbol():
    assert ENGINE_SO.exists(), "build the engine first (python -m coffee_sim_b200.build)"
    lib = C.CDLL(str(ENGINE_SO))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_oracle_exports_the_step_surface(oracle):
    # GPU-only extensions (ensembles, the allocation-free solve, the tensor-core layers)
    # have no CPU restatement
    needed = [n for n in declared_functions()
              if not n.startswith(("cs_ensemble", "cs_nn_")) and not n.endswith("_noalloc")]
    missing = [n for n in needed if not oracle.has(n)]
    assert not missing, missing


def test_struct_layouts_match_the_header():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "coffee_sim.h"
int main(void) {
    printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(CsSettings), sizeof(CsMetrics),
           sizeof(CsSpout), sizeof(CsBed), sizeof(CsBrew), sizeof(CsGeometry),
           offsetof(CsSettings, pressure_storage), offsetof(CsSettings, exit_speed_override),
           offsetof(CsMetrics, solve_ms));
    return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = Path(d) / "t.c"
        c.write_text(src)
        exe = Path(d) / "t"
        subprocess.run(["gcc", "-I", str(ROOT / "include"), str(c), "-o", str(exe)], check=True)
        got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [C.sizeof(_ffi.CsSettings), C.sizeof(_ffi.CsMetrics), C.sizeof(_ffi.CsSpout), C.sizeof(_ffi.CsBed),
            C.sizeof(_ffi.CsBrew), C.sizeof(_ffi.CsGeometry), _ffi.CsSettings.pressure_storage.offset,
            _ffi.CsSettings.exit_speed_override.offset, _ffi.CsMetrics.solve_ms.offset]
    assert got == want


@pytest.mark.parametrize("preset", ["default_v60", "benchmark_free_stream", "benchmark_center_pour"])
def test_engine_presets_match_oracle_presets(engine, oracle, preset):
    a = getattr(MpmSettings, preset)(engine)
    b = getattr(MpmSettings, preset)(oracle)
    assert bytes(a.raw) == bytes(b.raw)


def test_engine_fails_loudly_without_a_gpu(engine):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    s = MpmSettings.benchmark_free_stream(engine)
    h = C.c_void_p()
    rc = engine.lib.cs_create(C.byref(s.raw), C.byref(h))
    assert rc == 8  # CS_ERR_NO_DEVICE
    assert b"CUDA" in engine.lib.cs_last_error_string()


def test_invalid_settings_are_rejected(engine):
    s = MpmSettings.benchmark_free_stream(engine)
    s.raw.abi_version = 999
    h = C.c_void_p()
    assert engine.lib.cs_create(C.byref(s.raw), C.byref(h)) == 1
    assert b"abi_version" in engine.lib.cs_last_error_string()


def test_null_handles_are_rejected(engine):
    assert engine.lib.cs_step_frame(None, C.c_float(0.016)) == 1
    assert engine.lib.cs_get_counts(None, None, None, None) == 1
