"""On-the-fly fine-tuning of the learned warm start: a simulation that runs with
CS_WARM_LEARNED keeps training its network on pairs its own solver produces.

Every `every` substeps the last `capture` substeps before that point are stepped with
sample capture on (network inputs before the solve, the solved correction after it), the
pairs join a rolling buffer of at most `buffer` pairs, the network takes `steps` Adam
steps on random pairs from the buffer (Adam state carries over between rounds), and the
engine gets the new weights.  No counterpart in the reference, which has no learned part.

    tuner = OnlineFineTuner(sim, params, every=500)
    for _ in range(5000):
        tuner.step_substep(dt)
    tuner.rounds   # (substep, first loss, last loss, seconds) per fine-tuning round
"""
import time

import numpy as np

from . import unet


class OnlineFineTuner:
    def __init__(self, sim, params, every=500, capture=4, steps=100, lr=3e-4, buffer=16, seed=0):
        if capture < 1 or capture > every:
            raise ValueError("capture must lie in [1, every]")
        self.sim = sim
        self.every, self.capture, self.steps, self.lr, self.buffer = every, capture, steps, lr, buffer
        dims = tuple(int(d) for d in sim.settings.raw.grid_dims)
        self.net = unet.UNet(dims, sim.lib, params=np.asarray(params, dtype=np.float32), seed=seed)
        self.rng = np.random.default_rng(seed)
        self.samples = []
        self.count = 0
        self.rounds = []
        sim.set_learned_weights(np.asarray(params, dtype=np.float32))

    def _in_capture_window(self, n):
        # substeps every*j - capture + 1 .. every*j (1-based) capture a pair
        return (n % self.every) == 0 or (n % self.every) > self.every - self.capture

    def step_substep(self, sub_dt):
        n = self.count + 1
        if self._in_capture_window(n):
            self.samples += unet.collect_samples(self.sim, sub_dt, 1)
            self.samples = self.samples[-self.buffer:]
        else:
            self.sim.step_substep(sub_dt)
        self.count = n
        if n % self.every == 0:
            self.fine_tune()

    def fine_tune(self):
        import torch

        t0 = time.perf_counter()
        first = last = None
        for k in range(self.steps):
            f, t, m = self.samples[int(self.rng.integers(len(self.samples)))]
            loss = self.net.train_step(f, t, m, lr=self.lr)
            if k == 0:
                first = float(loss.item())
        torch.cuda.synchronize()
        self.net.check_errors()
        last = float(loss.item())
        self.sim.set_learned_weights(self.net.params_numpy())
        self.rounds.append((self.count, first, last, time.perf_counter() - t0))
