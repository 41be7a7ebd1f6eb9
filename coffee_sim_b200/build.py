"""Build libcoffee_sim_b200.so in-tree with nvcc for sm_100a.

    python -m coffee_sim_b200.build [--verbose]

The library is one nvcc invocation over csrc/engine.cu (unity build of the kernels)
and csrc/host_scene.cpp.  -fmad=false keeps every multiply and add separately
rounded so results reproduce the CPU oracle bit for bit.
"""
import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "libcoffee_sim_b200.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-std=c++17", "-lineinfo", "-fmad=false",
    "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
    "-shared", "-cudart", "static",
    "--expt-relaxed-constexpr",
]


def nvcc_path():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def sources():
    return [CSRC / "engine.cu", CSRC / "ensemble.cu", CSRC / "noalloc.cu", CSRC / "nn.cu", CSRC / "host_scene.cpp"]


def deps():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h"))
                  + list(CSRC.glob("*.cpp")) + [PKG.parent / "include" / "coffee_sim.h"])


def up_to_date():
    if not OUT.exists():
        return False
    t = OUT.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in deps())


def build(force=False, verbose=False, ptxas_v=False):
    if not force and up_to_date():
        return OUT
    cmd = [nvcc_path()] + NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_v else []) + [
        "-o", str(OUT) + ".tmp"] + [str(s) for s in sources()] + ["-lrt", "-ldl", "-lpthread"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, cwd=str(CSRC), capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libcoffee_sim_b200.so")
    if verbose or ptxas_v:
        sys.stderr.write(r.stderr)
    os.replace(str(OUT) + ".tmp", OUT)
    return OUT


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_v=a.ptxas_v))


if __name__ == "__main__":
    main()
