"""Shared helpers for the parity tests: build the same scene in the CUDA engine and
in the CPU oracle and compare their state arrays."""
import numpy as np

from coffee_sim_b200.sim import MpmSettings, MpmSim3D


def pair(settings, engine, oracle):
    """One engine simulation and one oracle simulation from the same settings."""
    return MpmSim3D(settings, engine), MpmSim3D(settings, oracle)


def copy_state(src, dst):
    """Overwrite dst's particle state with src's (reference layouts)."""
    nw, nb = src.num_water, src.num_bed
    n = nw + nb
    dst.set_counts(nw, nb)
    if n:
        dst.write_particles(0, src.read_particles(0, n))
        dst.write_affine(0, src.read_affine(0, n))
    if nb:
        dst.write_bed_extract(0, src.read_bed_extract(0, nb))


def relerr(a, b):
    """Norm-relative error ||a-b|| / max(||b||, tiny) in float64."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = max(np.linalg.norm(b), 1e-30)
    return float(np.linalg.norm(a - b) / den)


def mismatch(a, b):
    """Number of entries that differ (values, so -0 == +0)."""
    a = np.asarray(a)
    b = np.asarray(b)
    if a.dtype.kind == "f":
        both_nan = np.isnan(a) & np.isnan(b)
        return int(np.count_nonzero((a != b) & ~both_nan))
    return int(np.count_nonzero(a != b))
