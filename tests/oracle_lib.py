"""Loader for the CPU oracle library (test infrastructure only)."""
import ctypes as C
from pathlib import Path

from coffee_sim_b200._ffi import Library

ORACLE_DIR = Path(__file__).resolve().parent.parent / "oracle"


def _has_avx2():
    try:
        return " avx2 " in (" " + open("/proc/cpuinfo").read().replace("\n", " ") + " ")
    except OSError:
        return False


def oracle_path():
    v3 = ORACLE_DIR / "liboracle_v3.so"
    v2 = ORACLE_DIR / "liboracle_v2.so"
    return v3 if (_has_avx2() and v3.exists()) else v2


_lib = None


def oracle_library():
    global _lib
    if _lib is None:
        p = oracle_path()
        if not p.exists():
            raise FileNotFoundError(f"{p} missing; run `make -C oracle`")
        _lib = Library(p)
        _lib.lib.oracle_set_precision.argtypes = [C.c_int32]
        _lib.lib.oracle_set_threads.argtypes = [C.c_int32]
    return _lib


def set_precision(bits):
    oracle_library().lib.oracle_set_precision(bits)


def set_threads(n):
    oracle_library().lib.oracle_set_threads(n)
