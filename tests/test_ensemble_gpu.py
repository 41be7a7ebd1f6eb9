"""Batched ensemble (cs_ensemble_*): n pours stepped together, every pass one launch
over all instances, give the same states as the same pours stepped one at a time."""
import pytest

from coffee_sim_b200 import _ffi, scenes
from coffee_sim_b200.sim import MpmEnsemble, MpmSettings, MpmSim3D
from helpers import mismatch

pytestmark = pytest.mark.gpu
FRAME = 1.0 / 60.0


def _v60(engine, flow):
    s = scenes.c2_v60(engine, grid=32, max_particles=60000)
    s.raw.rbgs_omega = 1.9
    s.raw.device_emission = 1
    s.raw.p2g_mode = _ffi.CS_P2G_SORTED_SHARED
    return s


def test_ensemble_matches_independent_pours(engine):
    flows = [2.0, 4.0, 6.0]
    settings = [_v60(engine, f) for f in flows]
    ens = MpmEnsemble(settings, engine)
    singles = [MpmSim3D(s, engine) for s in settings]
    for i, f in enumerate(flows):
        U = float(settings[i].sim_units_per_meter)
        assert scenes.populate_c2(ens.member(i), seed=i + 1) == scenes.populate_c2(singles[i], seed=i + 1)
        ens.set_flow_override(i, f, 0.8 * U)
        singles[i].set_flow_override(f, 0.8 * U)
    for k in range(3):
        ens.step_substep(scenes.C2_DT)
        for sim in singles:
            sim.step_substep(scenes.C2_DT)
        for i, sim in enumerate(singles):
            assert ens.counts(i) == (sim.num_water, sim.num_bed)
            me, ms = ens.metrics(i), sim.latest_metrics()
            assert me.last_sweeps == ms.last_sweeps, (k, i)
            assert me.residual_checks == ms.residual_checks >= 2, (k, i)
            assert me.last_residual <= 1e-5
            assert mismatch(ens.read_particles(i), sim.read_particles()) == 0, (k, i)
    # the pours differ (different flows emit different amounts)
    assert len({ens.counts(i)[0] for i in range(3)}) == 3


def test_ensemble_reference_mode_frames(engine):
    """Fixed-point pressure, 40 pairs (the reference configuration), two instances
    pouring at different kettle angles."""
    settings = []
    for _ in range(2):
        s = MpmSettings.benchmark_center_pour(engine)
        s.raw.device_emission = 1
        settings.append(s)
    ens = MpmEnsemble(settings, engine)
    singles = [MpmSim3D(s, engine) for s in settings]
    for i, a in enumerate((30.0, 42.0)):
        ens.set_kettle_angle(i, a)
        singles[i].set_kettle_angle(a)
    for f in range(3):
        ens.step_frame(FRAME)
        for sim in singles:
            sim.step_frame(FRAME)
    for i, sim in enumerate(singles):
        assert mismatch(ens.read_particles(i), sim.read_particles()) == 0


def test_ensemble_rejects_mixed_grids(engine):
    a = _v60(engine, 2.0)
    b = scenes.c2_v60(engine, grid=48, max_particles=60000)
    with pytest.raises(_ffi.CsError):
        MpmEnsemble([a, b], engine)


def test_ensemble_device_timer(engine):
    ens = MpmEnsemble([_v60(engine, 4.0)], engine)
    scenes.populate_c2(ens.member(0), seed=2)
    with pytest.raises(_ffi.CsError):
        ens.timer_stop()  # not started
    ens.timer_start()
    ens.step_substep(scenes.C2_DT)
    ms = ens.timer_stop()
    assert 0.0 < ms < 5000.0
    ens.close()


def test_ensemble_learned_warm_start_matches_single_pours(engine):
    """CS_WARM_LEARNED in an ensemble: each instance's network guess and its acceptance
    are those of the same pour stepped alone, bit for bit."""
    from pathlib import Path

    import numpy as np

    params = np.load(Path(__file__).resolve().parent.parent / "coffee_sim_b200" / "weights" / "unet_v60_64.npy")
    flows = [2.0, 5.0]
    settings = []
    for f in flows:
        s = _v60(engine, f)
        s.raw.warm_start = _ffi.CS_WARM_LEARNED
        settings.append(s)
    ens = MpmEnsemble(settings, engine)
    ens.set_learned_weights(params)
    singles = [MpmSim3D(s, engine) for s in settings]
    for i, f in enumerate(flows):
        U = float(settings[i].sim_units_per_meter)
        scenes.populate_c2(ens.member(i), seed=i + 7)
        scenes.populate_c2(singles[i], seed=i + 7)
        ens.set_flow_override(i, f, 0.8 * U)
        singles[i].set_flow_override(f, 0.8 * U)
        singles[i].set_learned_weights(params)
    used = 0
    for k in range(4):
        ens.step_substep(scenes.C2_DT)
        for sim in singles:
            sim.step_substep(scenes.C2_DT)
        for i, sim in enumerate(singles):
            me, ms = ens.metrics(i), sim.latest_metrics()
            assert (me.learned_used, me.last_sweeps) == (ms.learned_used, ms.last_sweeps), (k, i)
            assert me.last_residual <= 1e-5
            assert mismatch(ens.read_particles(i), sim.read_particles()) == 0, (k, i)
            used += me.learned_used
    print(f"\nguess kept on {used} of 8 instance-substeps")


def test_ensemble_graph_replay_matches_direct_and_single_pours(engine):
    """The batched substep captured once and replayed (settings[0].use_graph = 1: batched
    prefix scans, per-instance solve totals read lazily, no host synchronisation per
    substep) gives the same states, pair counts and residual checks as the directly
    launched ensemble and as the pours stepped one at a time."""
    flows = [2.0, 4.0, 6.0]
    base = [_v60(engine, f) for f in flows]
    graph_settings = [s.copy() for s in base]
    graph_settings[0].raw.use_graph = 1
    direct, replay = MpmEnsemble(base, engine), MpmEnsemble(graph_settings, engine)
    singles = [MpmSim3D(s, engine) for s in base]
    for i, f in enumerate(flows):
        U = float(base[i].sim_units_per_meter)
        n = scenes.populate_c2(singles[i], seed=i + 1)
        for ens in (direct, replay):
            assert scenes.populate_c2(ens.member(i), seed=i + 1) == n
            ens.set_flow_override(i, f, 0.8 * U)
        singles[i].set_flow_override(f, 0.8 * U)
    for k in range(4):
        for ens in (direct, replay):
            ens.step_substep(scenes.C2_DT)
        for sim in singles:
            sim.step_substep(scenes.C2_DT)
        for i, sim in enumerate(singles):
            mr, md, ms = replay.metrics(i), direct.metrics(i), sim.latest_metrics()
            assert mr.last_sweeps == md.last_sweeps == ms.last_sweeps > 0, (k, i)
            assert mr.residual_checks == md.residual_checks == ms.residual_checks, (k, i)
            assert mr.last_residual <= 1e-5
            assert replay.counts(i) == direct.counts(i) == (sim.num_water, sim.num_bed)
            pr = replay.read_particles(i)
            assert mismatch(pr, direct.read_particles(i)) == 0, (k, i)
            assert mismatch(pr, sim.read_particles()) == 0, (k, i)
    for ens in (direct, replay):
        ens.close()
