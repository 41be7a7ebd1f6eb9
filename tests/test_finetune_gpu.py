"""On-the-fly fine-tuning of the learned warm start (coffee_sim_b200/finetune.py): the
simulation keeps solving to its tolerance while the network retrains on the pairs its
own solver produced, and the engine runs the updated weights."""
from pathlib import Path

import numpy as np
import pytest

from coffee_sim_b200 import _ffi, scenes, unet
from coffee_sim_b200.finetune import OnlineFineTuner
from coffee_sim_b200.sim import MpmSim3D

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
WEIGHTS = Path(__file__).resolve().parent.parent / "coffee_sim_b200" / "weights" / "unet_v60_64.npy"


def test_fine_tuning_rounds_update_the_engine(engine):
    s = scenes.c2_v60(engine, grid=32, max_particles=60000)
    s.raw.rbgs_omega = 1.9
    s.raw.device_emission = 1
    s.raw.warm_start = _ffi.CS_WARM_LEARNED
    sim = MpmSim3D(s, engine)
    scenes.populate_c2(sim, seed=5)
    params = np.load(WEIGHTS)  # trained at 64^3; the network has no fixed size
    tuner = OnlineFineTuner(sim, params, every=4, capture=2, steps=20, lr=3e-4, buffer=4)
    seen = []
    for _ in range(12):
        tuner.step_substep(scenes.C2_DT)
        m = sim.latest_metrics()
        assert m.last_residual <= 1e-5
        seen.append(int(m.learned_used))
    assert [r[0] for r in tuner.rounds] == [4, 8, 12]
    assert len(tuner.samples) == 4
    for _, first, last, _ in tuner.rounds:
        assert np.isfinite(first) and np.isfinite(last)
    tuned = tuner.net.params_numpy()
    assert tuned.shape == (unet.param_count(),)
    assert np.abs(tuned - params).max() > 0.0  # the rounds trained the network
    # the engine runs the tuned weights: a fresh engine with them gives the same substep
    blob = sim.snapshot()
    sim.step_substep(scenes.C2_DT)
    a = sim.read_pressure()
    twin = MpmSim3D(s, engine)
    twin.set_learned_weights(tuned)
    twin.restore(blob)
    twin.step_substep(scenes.C2_DT)
    assert np.array_equal(a, twin.read_pressure())
    print(f"\nrounds {tuner.rounds}, guess kept {sum(seen)}/12")
