"""Error of one FP32 substep against the same substep run in FP64, on the CPU.

The engine's FP32 substep equals the oracle's FP32 substep bit for bit (the GPU parity
tests), so the oracle's FP32-vs-FP64 difference after one substep from the same seeded
state is the engine's error against an FP64 run.  Measured here on the bench's three
pours (their settings; residual solve to 1e-5; the sample reorder off, as it only
permutes slots) and on the 32^3 water block (the reference configuration: fixed-point
pressure, 40 pairs):

* Sample count and total mass are equal.
* int64 lanes (i64 * 2^32, the headline workload's mode), 64^3 pour: pressure 5e-8,
  grid momentum 4.4e-6, water-sample velocity 1.7e-6 relative; every water sample's
  position within 4.8e-7 of the FP64 one (one float32 ulp).  Two of the 3000 bed grains
  take the other side of a threshold in bed_dynamics and move by a few hundredths of a
  unit, which alone sets the relative position error of all samples (1.8e-5).
* 128^3 spiral pour (i32 lanes): pressure 8.0e-7, grid momentum 4.3e-6, water velocity
  1.4e-6; 27 of 24000 grains across a bed threshold.
* 192^3 headline pour (int64 lanes): pressure 4.4e-7, grid momentum 3.4e-5, water
  velocity 1.5e-5, water positions within 9.5e-7 (two ulp); 95 of 81000 grains across a
  bed threshold.  Here the velocity error is spread over all samples (the 10000 largest
  carry 1.4 % of its square, none is off by 1e-3 of its speed), not set by a few samples
  on the other side of a branch.
* i32 lanes (i32 * 2^18, the reference's format): grid momentum 1e-4 (64^3) and 2.2e-4
  (water block), velocity 4e-5 and 1e-4.  Each deposit is truncated to a 2^-18 quantum;
  evaluated in float or in double, the same deposit truncates to a different quantum in
  a fraction of nodes, and in low-mass cells one quantum of momentum is a visible
  velocity.  The int64 format removes most of it.
"""
import numpy as np
import pytest

import bench
import oracle_lib
from coffee_sim_b200 import _ffi, scenes
from coffee_sim_b200.sim import MpmSim3D
from helpers import copy_state, relerr


def _pair(oracle, settings, populate, step):
    """An FP32 and an FP64 oracle simulation from one seeded state, each stepped once.
    The state is populated in FP32 and copied into the FP64 simulation, so that both
    start from the same samples: populating tests each candidate position against the
    SDF in the simulation's own precision, and a candidate on the boundary can be kept in
    one and dropped in the other.  The sample reorder is off: it only permutes slots, by
    keys that a sample on a tile boundary can get differently in either precision."""
    settings = settings.copy()
    settings.raw.reorder_every = 0
    a = MpmSim3D(settings, oracle)
    populate(a)
    oracle_lib.set_precision(64)
    try:
        b = MpmSim3D(settings, oracle)
    finally:
        oracle_lib.set_precision(32)
    copy_state(a, b)
    for sim in (a, b):
        step(sim)
    return a, b


def _errors(a, b):
    pa, pb = a.read_particles(), b.read_particles()
    ga, gb = a.read_grid_vel(), b.read_grid_vel()
    nb = a.num_bed
    return {
        "count": (a.particle_count(), b.particle_count()),
        "mass": (pa[:, 7].astype(np.float64).sum(), pb[:, 7].astype(np.float64).sum()),
        "pressure": relerr(a.read_pressure(), b.read_pressure()),
        "grid_momentum": relerr(ga[:, :3] * ga[:, 3:4], gb[:, :3] * gb[:, 3:4]),
        "water_velocity": relerr(pa[nb:, 4:7], pb[nb:, 4:7]),
        "water_position_max": float(np.abs(pa[nb:, 0:3].astype(np.float64) - pb[nb:, 0:3]).max()),
        "bed_moved": int(np.count_nonzero(np.abs(pa[:nb, 0:3].astype(np.float64) - pb[:nb, 0:3]).max(axis=1) > 1e-4)),
        "num_bed": nb,
    }


# bench workload, P2G lanes, and the bounds on (pressure, grid momentum, water velocity)
# that the measured errors sit under
POURS = {
    "c2-int64": ("c2", _ffi.CS_P2G_INT64, (1e-6, 1e-5, 1e-5)),
    "c2-i32": ("c2", _ffi.CS_P2G_SORTED_SHARED, (1e-5, 3e-4, 1e-4)),
    "c3": ("c3", None, (1e-5, 1e-5, 1e-5)),
    "c5": ("c5", None, (1e-5, 1e-4, 5e-5)),
}


@pytest.mark.parametrize("case", list(POURS))
def test_bench_pour_one_substep_vs_fp64(oracle, case):
    """The bench's pours with their own settings (64^3 in both lane formats; the 128^3
    spiral pour, i32 lanes; the 192^3 headline pour, int64 lanes), one substep from the
    populated state."""
    key, mode, (tp, tm, tv) = POURS[case]
    args = bench.default_args()
    s = bench.make_settings(oracle, key, args)
    if mode is not None:
        s.raw.p2g_mode = mode
    a, b = _pair(oracle, s, lambda sim: scenes.populate_c2(sim, seed=bench.WORKLOADS[key]["seed"]),
                 lambda sim: bench.step(sim, key, 0))
    e = _errors(a, b)
    assert e["count"][0] == e["count"][1] > 100000
    assert e["mass"][0] == e["mass"][1]
    ma, mb = a.latest_metrics(), b.latest_metrics()
    assert ma.last_residual <= 1e-5 and mb.last_residual <= 1e-5
    assert e["pressure"] < tp and e["grid_momentum"] < tm and e["water_velocity"] < tv, e
    assert e["water_position_max"] < 1e-5, e
    assert e["bed_moved"] <= 0.002 * e["num_bed"], e


@pytest.mark.parametrize("lanes", ["int64", "i32"])
def test_water_block_one_substep_vs_fp64(oracle, lanes):
    s = scenes.c1_water_block(oracle)
    s.raw.p2g_mode = _ffi.CS_P2G_INT64 if lanes == "int64" else _ffi.CS_P2G_ATOMIC32
    a, b = _pair(oracle, s, scenes.populate_c1, lambda sim: sim.step_substep(scenes.C1_DT))
    e = _errors(a, b)
    assert e["count"][0] == e["count"][1] > 10000 and e["mass"][0] == e["mass"][1]
    assert e["pressure"] < 1e-6 and e["water_position_max"] < 1e-6, e
    if lanes == "int64":
        assert e["grid_momentum"] < 3e-5 and e["water_velocity"] < 1e-5, e
    else:
        assert e["grid_momentum"] < 5e-4 and e["water_velocity"] < 2e-4, e
