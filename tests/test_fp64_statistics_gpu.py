"""Long-horizon statistics of the CUDA engine (FP32) against the oracle run in FP64.

Per-substep results are bit-exact with the oracle's FP32 run (test_parity_gpu.py).  Over
hundreds of substeps FP32 and FP64 trajectories separate sample by sample, so these
tests compare what a user reads off a run: total mass (no emission loss), the momentum
vector and the fill level (DiagSnapshot height extent and mean, physics_tests.rs:551-571
and 937-1061, plus the sample counts in eight height bands).  Tolerance: 1 % (momentum:
of its norm; band counts: of the active sample count)."""
import numpy as np
import pytest

from coffee_sim_b200 import scenes
from coffee_sim_b200.sim import MpmSim3D
import oracle_lib
import physics_snapshots as ps

pytestmark = pytest.mark.gpu
TOL = 0.01


@pytest.fixture
def oracle64(oracle):
    oracle_lib.set_precision(64)
    yield oracle
    oracle_lib.set_precision(32)


def _stats(sim, settings):
    p = sim.read_particles(0, sim.particle_count()).astype(np.float64)
    act = p[:, 7] > float(ps.nominal_mass(settings)) * 0.1
    a = p[act]
    m = a[:, 7]
    half = float(settings.raw.bounds_size[1]) * 0.5
    bands = np.histogram(a[:, 1], bins=8, range=(-half, half))[0]
    d = ps.diag_snapshot(sim, settings)
    return {"count": int(act.sum()), "mass": float(m.sum()), "momentum": (m[:, None] * a[:, 4:7]).sum(axis=0),
            "y_extent": d.y_extent, "y_mean": d.y_mean, "bands": bands, "y_min": d.y_min}


def _compare(e, o, where):
    assert e["count"] == o["count"], where
    assert abs(e["mass"] - o["mass"]) <= 1e-6 * o["mass"], where
    pn = np.linalg.norm(o["momentum"])
    assert np.linalg.norm(e["momentum"] - o["momentum"]) <= TOL * pn, (where, e["momentum"], o["momentum"])
    assert abs(e["y_extent"] - o["y_extent"]) <= TOL * abs(o["y_extent"]), (where, e["y_extent"], o["y_extent"])
    # the mean height relative to the lowest sample, so the tolerance is on a length
    le, lo = e["y_mean"] - o["y_min"], o["y_mean"] - o["y_min"]
    assert abs(le - lo) <= TOL * abs(lo), (where, e["y_mean"], o["y_mean"])
    assert np.abs(e["bands"] - o["bands"]).max() <= TOL * o["count"], (where, e["bands"], o["bands"])


def test_c1_water_block_500_steps_vs_fp64(engine, oracle64):
    """The 32^3 water block (16.8k samples, 40 pairs), 500 substeps of 5e-4 s."""
    s = scenes.c1_water_block(engine)
    e, o = MpmSim3D(s, engine), MpmSim3D(s, oracle64)
    assert scenes.populate_c1(e) == scenes.populate_c1(o)
    for k in range(500):
        e.step_substep(scenes.C1_DT)
        o.step_substep(scenes.C1_DT)
        if k % 100 == 99:
            _compare(_stats(e, s), _stats(o, s), f"C1 substep {k + 1}")


def test_v60_pour_500_steps_vs_fp64(engine, oracle64):
    """The V60 pour at 32^3 (jet, coffee bed, residual solve to 1e-5), 500 substeps.

    Bed samples pack and switch between anchored and suspended at thresholds, so a
    last-bit difference can move one by a tenth of a cell: FP32 and FP64 runs of the same
    algorithm (the oracle against itself as well) separate after ~20 substeps, and from
    there net momentum and kinetic energy differ by 5-25 % while mass and fill level
    agree to 0.3 %.  Momentum is compared over the first 10 substeps (to 1e-3 of the
    momentum scale sum m|v|), mass (to 1e-3: the bed and the filter absorb water along
    each trajectory) and fill level every 100 substeps to 500."""
    s = scenes.c2_v60(engine, grid=32, max_particles=60000)
    s.raw.rbgs_omega = 1.9
    s.raw.device_emission = 1
    e, o = MpmSim3D(s, engine), MpmSim3D(s, oracle64)
    assert scenes.populate_c2(e) == scenes.populate_c2(o)
    for k in range(500):
        e.step_substep(scenes.C2_DT)
        o.step_substep(scenes.C2_DT)
        if k < 10:
            pe = e.read_particles(0, e.particle_count()).astype(np.float64)
            po = o.read_particles(0, o.particle_count()).astype(np.float64)
            me = (pe[:, 7:8] * pe[:, 4:7]).sum(axis=0)
            mo = (po[:, 7:8] * po[:, 4:7]).sum(axis=0)
            scale = (po[:, 7] * np.sqrt((po[:, 4:7] ** 2).sum(axis=1))).sum()
            assert np.linalg.norm(me - mo) <= 1e-3 * scale, (k, me, mo)
        if k % 100 == 99:
            assert e.particle_count() == o.particle_count()
            a, b = _stats(e, s), _stats(o, s)
            where = f"V60 substep {k + 1}"
            assert a["count"] == b["count"], where
            # water mass moves into bed pores and the filter along each trajectory
            assert abs(a["mass"] - b["mass"]) <= 1e-3 * b["mass"], where
            assert abs(a["y_extent"] - b["y_extent"]) <= TOL * abs(b["y_extent"]), (where, a["y_extent"], b["y_extent"])
            assert np.abs(a["bands"] - b["bands"]).max() <= TOL * b["count"], (where, a["bands"], b["bands"])
