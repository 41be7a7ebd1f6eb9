"""Learned warm start in the engine (CS_WARM_LEARNED) and training-sample capture."""
import numpy as np
import pytest

from coffee_sim_b200 import _ffi, scenes, unet
from coffee_sim_b200.sim import MpmSim3D
from helpers import mismatch

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _pour(engine, warm, grid=32):
    s = scenes.c2_v60(engine, grid=grid, max_particles=60000)
    s.raw.rbgs_omega = 1.9
    s.raw.device_emission = 1
    s.raw.warm_start = warm
    sim = MpmSim3D(s, engine)
    scenes.populate_c2(sim, seed=4)
    return sim


def test_capture_gives_consistent_pairs(engine):
    sim = _pour(engine, _ffi.CS_WARM_PREVIOUS)
    for _ in range(2):
        sim.step_substep(scenes.C2_DT)
    p0 = torch.tensor(sim.read_pressure(), device="cuda")  # the warm start of the next solve
    feat, target, mask = unet.collect_samples(sim, scenes.C2_DT, 1)[0]
    m = sim.latest_metrics()
    assert int(mask.sum().item()) == m.fluid_cells > 0
    assert torch.equal(feat[:, 2].float(), mask)  # fluid channel
    fl = mask > 0
    r = feat[:, 0].float()
    assert abs(r[fl].pow(2).mean().sqrt().item() - 1.0) < 1e-2  # residual in units of its RMS
    assert (target[~fl] == 0).all()
    # target * s is the correction the solve applied to the warm start
    scale = sim.learned_read_sample(feat, target, mask)
    p1 = torch.tensor(sim.read_pressure(), device="cuda")
    err = (p0[fl] + target[fl] * scale - p1[fl]).abs().max().item()
    assert err <= 1e-5 * p1[fl].abs().max().item() + 1e-4


def test_rejected_guess_leaves_the_solve_unchanged(engine):
    """With all weights zero the guess equals the previous pressure, is not taken
    (not strictly better), and the substep is bit-identical to the plain warm start."""
    plain = _pour(engine, _ffi.CS_WARM_PREVIOUS)
    learned = _pour(engine, _ffi.CS_WARM_LEARNED)
    learned.set_learned_weights(np.zeros(unet.param_count(), dtype=np.float32))
    for k in range(3):
        plain.step_substep(scenes.C2_DT)
        learned.step_substep(scenes.C2_DT)
        ml, mp = learned.latest_metrics(), plain.latest_metrics()
        assert ml.learned_used == 0
        assert ml.last_sweeps == mp.last_sweeps
        assert mismatch(learned.read_pressure(), plain.read_pressure()) == 0
        n = plain.particle_count()
        assert mismatch(learned.read_particles(0, n), plain.read_particles(0, n)) == 0


def test_learned_mode_needs_weights(engine):
    sim = _pour(engine, _ffi.CS_WARM_LEARNED)
    with pytest.raises(_ffi.CsError):
        sim.step_substep(scenes.C2_DT)
    with pytest.raises(_ffi.CsError):
        sim.set_learned_weights(np.zeros(10, dtype=np.float32))


def test_trained_network_gain_over_previous_substep_start(engine):
    """What the committed network gains on the V60 64^3 pour (substeps 6-25, replayed from
    one snapshot for both warm starts): the guess is kept whenever its FP64 residual is
    below 0.999x the previous-substep start's, which happens on a share of the substeps,
    and every substep still reaches 1e-5.  The pair counts of both runs are printed (the
    network does not shorten the solve materially at this size)."""
    from pathlib import Path

    wfile = Path(__file__).resolve().parent.parent / "coffee_sim_b200" / "weights" / "unet_v60_64.npy"
    params = np.load(wfile)
    runs = {}
    base = None
    for warm in (_ffi.CS_WARM_PREVIOUS, _ffi.CS_WARM_LEARNED):
        s = scenes.c2_v60(engine, grid=64)
        s.raw.rbgs_omega = 1.92
        s.raw.check_every = 20
        s.raw.max_sweeps = 4000
        s.raw.device_emission = 1
        s.raw.p2g_mode = _ffi.CS_P2G_SORTED_SHARED
        s.raw.warm_start = warm
        sim = MpmSim3D(s, engine)
        if base is None:
            scenes.populate_c2(sim)
            for _ in range(5):
                sim.step_substep(scenes.C2_DT)
            base = sim.snapshot()
        else:
            sim.set_learned_weights(params)
            sim.restore(base)
        pairs, kept, r0 = [], 0, []
        for _ in range(20):
            sim.step_substep(scenes.C2_DT)
            m = sim.latest_metrics()
            assert m.last_residual <= 1e-5
            pairs.append(int(m.last_sweeps))
            kept += int(m.learned_used)
            r0.append(float(m.initial_residual))
        runs[warm] = (pairs, kept, r0)
        sim.close()
    plain, learned = runs[_ffi.CS_WARM_PREVIOUS], runs[_ffi.CS_WARM_LEARNED]
    print(f"\nplain pairs {sum(plain[0]) / 20:.1f}, learned pairs {sum(learned[0]) / 20:.1f}, "
          f"guess kept on {learned[1]}/20 substeps")
    assert learned[1] > 0
    assert plain[1] == 0


def test_learned_graph_replay_matches_direct_launches(engine):
    """The learned substep (residual, inputs, U-Net forward, device-side acceptance test,
    solve) replayed as a CUDA graph gives the direct-launch results bit for bit, with the
    same accepted guesses (V60 64^3 from substep 6, where the guess is kept on some
    substeps and rejected on others)."""
    from pathlib import Path

    params = np.load(Path(__file__).resolve().parent.parent / "coffee_sim_b200" / "weights" / "unet_v60_64.npy")

    def v60(warm):
        s = scenes.c2_v60(engine, grid=64)
        s.raw.rbgs_omega = 1.92
        s.raw.check_every = 40
        s.raw.device_emission = 1
        s.raw.p2g_mode = _ffi.CS_P2G_SORTED_SHARED
        s.raw.warm_start = warm
        return MpmSim3D(s, engine)

    base = v60(_ffi.CS_WARM_PREVIOUS)
    scenes.populate_c2(base)
    for _ in range(5):
        base.step_substep(scenes.C2_DT)
    blob = base.snapshot()
    base.close()
    sims = []
    for graph in (False, True):
        sim = v60(_ffi.CS_WARM_LEARNED)
        sim.set_learned_weights(params)
        sim.restore(blob)
        if graph:
            sim.set_graph_mode(True)
        sims.append(sim)
    kept = []
    for k in range(8):
        for sim in sims:
            sim.step_substep(scenes.C2_DT)
        a, b = sims[0].latest_metrics(), sims[1].latest_metrics()
        assert (a.learned_used, a.last_sweeps) == (b.learned_used, b.last_sweeps), k
        assert b.last_residual <= 1e-5
        kept.append(int(a.learned_used))
        assert mismatch(sims[0].read_pressure(), sims[1].read_pressure()) == 0, k
        n = sims[0].particle_count()
        assert mismatch(sims[0].read_particles(0, n), sims[1].read_particles(0, n)) == 0, k
    print(f"\nguess kept on substeps {kept}")
    assert 0 < sum(kept) < len(kept)
