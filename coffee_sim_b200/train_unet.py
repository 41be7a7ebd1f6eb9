"""Train the pressure-guess U-Net on pairs generated by the plain solver and compare the
learned warm start with the previous-substep warm start.

    python -m coffee_sim_b200.train_unet [--out coffee_sim_b200/weights/unet_v60_64.npy]

Pairs come from V60 pours at 64^3 (flows 2, 4 and 6 ml/s, different fill seeds): for
every substep the network inputs before the solve and the solved pressure after it.
Training is Adam on the masked MSE in units of s (the RMS of the right-hand side).  The
evaluation restores one held-out pour state into two simulations, one per warm start,
and reports red-black pairs per substep and solve milliseconds for both.
"""
import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
sys.path.insert(0, str(PKG.parent))

from coffee_sim_b200 import _ffi, scenes, unet  # noqa: E402
from coffee_sim_b200.sim import MpmSim3D, engine_library  # noqa: E402

DEFAULT_OUT = PKG / "weights" / "unet_v60_64.npy"


def v60_settings(lib, grid=64, warm=_ffi.CS_WARM_PREVIOUS):
    s = scenes.c2_v60(lib, grid=grid)
    s.raw.rbgs_omega = 1.9
    s.raw.max_sweeps = 4000
    s.raw.check_every = 10
    s.raw.device_emission = 1
    s.raw.p2g_mode = _ffi.CS_P2G_SORTED_SHARED
    s.raw.warm_start = warm
    return s


def make_pour(lib, seed, flow, grid=64, warm=_ffi.CS_WARM_PREVIOUS):
    s = v60_settings(lib, grid, warm)
    sim = MpmSim3D(s, lib)
    scenes.populate_c2(sim, seed=seed)
    sim.set_flow_override(flow, 0.8 * float(s.sim_units_per_meter))
    return sim


def compare(lib, params, state_sim_seed=99, flow=4.0, warmup=10, substeps=20, grid=64):
    """Pairs and solve time per substep, previous-substep vs learned warm start, from the
    same saved state."""
    base = make_pour(lib, state_sim_seed, flow, grid)
    for _ in range(warmup):
        base.step_substep(scenes.C2_DT)
    blob = base.snapshot()
    out = {}
    for name, warm in (("previous", _ffi.CS_WARM_PREVIOUS), ("learned", _ffi.CS_WARM_LEARNED)):
        sim = make_pour(lib, state_sim_seed, flow, grid, warm) if warm != _ffi.CS_WARM_PREVIOUS else base
        if warm == _ffi.CS_WARM_LEARNED:
            sim.set_learned_weights(params)
        sim.restore(blob)
        sim.profile_enable(True)
        pairs, used, res = [], 0, []
        for _ in range(substeps):
            sim.step_substep(scenes.C2_DT)
            m = sim.latest_metrics()
            pairs.append(int(m.last_sweeps))
            used += int(m.learned_used)
            res.append(float(m.last_residual))
        prof = sim.profile_read()
        solve_ms = (prof.phase_ms[4] + prof.phase_ms[5] + prof.phase_ms[10]) / substeps
        out[name] = {"pairs_per_substep": float(np.mean(pairs)), "solve_ms": solve_ms,
                     "learned_phase_ms": prof.phase_ms[10] / substeps, "sweeps_ms": prof.phase_ms[4] / substeps,
                     "learned_used": used, "max_residual": max(res), "pairs": pairs}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(DEFAULT_OUT))
    ap.add_argument("--substeps", type=int, default=60, help="captured substeps per pour")
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    import torch

    lib = engine_library()
    t0 = time.time()
    samples = []
    for seed, flow in ((1, 2.0), (2, 4.0), (3, 6.0)):
        sim = make_pour(lib, seed, flow)
        samples += unet.collect_samples(sim, scenes.C2_DT, args.substeps)
        sim.close()
    t1 = time.time()
    params, hist = unet.train(samples, (64, 64, 64), lib, steps=args.steps, lr=args.lr, seed=args.seed,
                              log_every=100)
    t2 = time.time()
    del samples
    torch.cuda.empty_cache()
    cmp = compare(lib, params)
    out = Path(args.out)
    out.parent.mkdir(parents=True, exist_ok=True)
    np.save(out, params)
    summary = {"pairs_collected": 3 * args.substeps, "collect_s": t1 - t0, "train_s": t2 - t1,
               "train_steps": args.steps, "loss": hist, "comparison": cmp}
    print(json.dumps(summary))


if __name__ == "__main__":
    main()
