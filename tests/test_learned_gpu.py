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
