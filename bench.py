"""Benchmark: particle-steps/s and pressure-solve ms of the MLS-MPM substep with the
pressure swept to a relative residual of 1e-5, with the previous-substep warm start
("plain", the headline value) and with the learned warm start ("learned").

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
                    [--workload c5|c3|c2|c4] [--nested c3,c2,c4 | --nested none]

The headline workload (default) is the largest single-GPU configuration: the V60 pour
at 192^3 (dx = 0.83 mm) with ~7.8M samples, a two-layer coffee bed (porosity 0.45 above,
0.35 below with 10x lower permeability), the jet 1.2 cm off centre and int64 fixed-point
P2G.  One "step" is one substep (dt = 5e-4 s).  The same JSON line carries, as nested
keys, the 128^3 spiral pour (the learned-warm-start configuration), the 64^3 V60 pour and
the batched ensemble of 64 pours at 64^3.

Timing uses CUDA events on the engine's stream, with the substep replayed as a captured
CUDA graph and L2 flushed (512 MB write) before each timed step.  Under torchrun each rank
steps an independent replica of the pour on its own GPU (a single pour does not shard;
weak scaling) and rank 0 prints the max-over-ranks time.  `--impl reference` times the
CPU restatement of the reference step (the oracle, all host threads) on a bounded sample
of the headline workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particle-steps/sec & pressure-solve ms at 1e-5 residual: learned vs plain RBGS"
UNIT = "particle-steps/s"
DT = 5.0e-4

# The timed configurations.  omega is the measured optimum of each pour (192^3: pairs per
# substep 367/299/222/272/363 for omega 1.93..1.97; 128^3: 228/201/221/285/378); the check cap is the longest interval between FP64 residual checks
# (after each check the solve predicts the pairs it still needs); first_check is the
# interval before a solve's first check (0: the cap).
WORKLOADS = {
    "c5": {"name": "c5_v60_scale_192cube", "scene": "c5_scale", "seed": 4, "omega": 1.95, "check_every": 60,
           "first_check": 0, "p2g": "int64", "spiral": False, "reorder_every": 10, "p2g_tile": 8,
           "text": "V60 pour at 192^3 (dx 0.83 mm), two-layer bed (porosity 0.45/0.35, 10x lower permeability "
                   "below), jet 4 ml/s at 0.8 m/s 1.2 cm off centre, int64 fixed-point P2G"},
    "c3": {"name": "c3_v60_spiral_128cube", "scene": "c3_large", "seed": 2, "omega": 1.94, "check_every": 60,
           "first_check": 0, "p2g": "sorted", "spiral": True, "reorder_every": 10, "p2g_tile": 8,
           "text": "V60 pour at 128^3 (dx 1.25 mm), spout on the spiral path (r 1.5 cm, 0.5 Hz), tile-sorted P2G"},
    "c2": {"name": "c2_v60_midpour_64cube", "scene": "c2_v60", "seed": 1, "omega": 1.92, "check_every": 60,
           "first_check": 125, "p2g": "sorted", "spiral": False, "reorder_every": 0, "p2g_tile": 4,
           "text": "V60 pour at 64^3 (dx 2.5 mm), centre pour, tile-sorted P2G"},
}
PHASES = ["emit", "clear", "p2g", "grid", "sweeps", "residual", "project", "g2p", "bed", "render", "learned"]


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled while the timed region runs:
    NVML read every 5 ms from a thread (read-only queries), with one sample taken on entry
    and one on exit; `nvidia-smi -lms 200` when NVML is unavailable."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_slowdown", "nvmlClocksEventReasonHwPowerBrakeSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index, period_s=0.005):
        self.index = index
        self.period = period_s
        self.samples = []  # (sm_mhz, max_mhz, [reason names])
        self.source = None
        self.proc = None
        self.stop = threading.Event()
        self.thread = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            p = torch.cuda.get_device_properties(self.index)
            bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _nvml_sample(self):
        nv, h = self.nvml, self.handle
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        names = sorted({name for name, attr in self.REASONS if bits & getattr(nv, attr, 0)})
        self.samples.append((float(sm), float(mx), names))

    def _nvml_loop(self):
        while not self.stop.wait(self.period):
            try:
                self._nvml_sample()
            except Exception:
                return

    def _smi_loop(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.proc.stdout:
            r = [x.strip() for x in line.split(",")]
            if len(r) >= 9 and r[1].replace(".", "").isdigit() and r[2].replace(".", "").isdigit():
                self.samples.append((float(r[1]), float(r[2]),
                                     [names[k] for k in range(4) if r[5 + k].lower() == "active"]))

    def __enter__(self):
        try:
            self.nvml, self.handle = self._nvml_handle()
            self._nvml_sample()
            self.source = "nvml every 5 ms"
            self.thread = threading.Thread(target=self._nvml_loop, daemon=True)
        except Exception:
            try:
                self.proc = subprocess.Popen(
                    ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                     "--format=csv,noheader,nounits", "-lms", "200"],
                    stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.source = "nvidia-smi every 200 ms"
                self.thread = threading.Thread(target=self._smi_loop, daemon=True)
            except Exception:
                self.thread = None
        if self.thread:
            self.thread.start()
        return self

    def __exit__(self, *a):
        if self.proc is None and self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)
            try:
                self._nvml_sample()
            except Exception:
                pass
        elif self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(s[0] for s in self.samples),
                "sm_max_mhz": max(s[1] for s in self.samples),
                "reasons": sorted({n for s in self.samples for n in s[2]}),
                "samples": len(self.samples), "source": self.source}


def make_settings(lib, key, args, device=0, learned=False):
    """The settings of workload `key` exactly as the timed loops run them."""
    from coffee_sim_b200 import _ffi, scenes
    wl = WORKLOADS[key]
    s = getattr(scenes, wl["scene"])(lib, **({"grid": args.grid} if args.grid else {}))
    r = s.raw
    if learned:
        r.warm_start = _ffi.CS_WARM_LEARNED
    r.device = device
    r.rbgs_omega = wl["omega"] if args.omega is None else args.omega
    r.max_sweeps = args.max_sweeps
    r.check_every = wl["check_every"] if args.check_every is None else args.check_every
    r.first_check = wl["first_check"] if args.first_check is None else args.first_check
    r.rbgs_kernel = {"auto": 0, "p2p": 2, "cluster": 3, "grid": 4}[args.solve_sync]
    r.p2g_mode = {"atomic": _ffi.CS_P2G_ATOMIC32, "sorted": _ffi.CS_P2G_SORTED_SHARED,
                  "int64": _ffi.CS_P2G_INT64}[p2g_of(key, args)]
    r.device_emission = 1  # jet samples built on the device (the oracle matches this mode)
    # water samples reordered by P2G tile every N substeps (the oracle applies the same
    # permutation); at 192^3 every 10 substeps: G2P 1.68 -> 1.54 ms, every 5 costs more
    r.reorder_every = wl["reorder_every"]
    # 8^3-cell P2G tiles at 128^3 and 192^3 (cs_autotune's launch-shape trials: 192^3 P2G
    # 1.83 -> 1.66 ms per substep; 128 or 512 threads per particle block did not help)
    r.p2g_tile = wl["p2g_tile"]
    return s


def p2g_of(key, args):
    """The P2G mode a run uses: the workload's unless --p2g overrides it."""
    return WORKLOADS[key]["p2g"] if args.p2g == "default" else args.p2g


def build_scene(lib, key, args, device=0, learned=False, populate=True):
    from coffee_sim_b200 import scenes
    from coffee_sim_b200.sim import MpmSim3D
    sim = MpmSim3D(make_settings(lib, key, args, device, learned), lib)
    if populate:
        scenes.populate_c2(sim, seed=WORKLOADS[key]["seed"])
    return sim


def step(sim, key, k):
    """Substep k (0-based, counted from the populated state) of workload `key`; the
    spiral pour moves its spout first."""
    if WORKLOADS[key]["spiral"]:
        from coffee_sim_b200 import scenes
        sim.set_spout_position(*scenes.spiral_spout(k * DT))
    sim.step_substep(DT)


def ncu_traffic(kernel, tag, pairs=None):
    """DRAM bytes (read + write) per launch of `kernel` from the committed ncu summary
    of this workload (profiles/<kernel>_*<tag>*.md): `dram_bytes_per_pair` times the
    launch's red-black pairs when the summary gives it (the solve), else
    `dram_bytes_per_launch`, else None."""
    for f in sorted((ROOT / "profiles").glob(f"{kernel}_*.md")):
        if tag not in f.name:
            continue
        vals = {}
        for ln in f.read_text().splitlines():
            k, _, v = ln.partition("=")
            if k.strip() in ("dram_bytes_per_pair", "dram_bytes_per_launch"):
                try:
                    vals[k.strip()] = float(v.strip().split()[0])
                except (IndexError, ValueError):
                    pass
        if pairs is not None and "dram_bytes_per_pair" in vals:
            return vals["dram_bytes_per_pair"] * pairs
        if "dram_bytes_per_launch" in vals:
            return vals["dram_bytes_per_launch"]
    return None


def algorithmic_bytes(n_p, n_c, pairs, evals, n_bed, int64=False):
    """Compulsory bytes of one substep on the dense grid: 172 N_p + 134 N_c + 17 K N_c +
    13 E N_c, plus 48 N_c in int64 mode and 4 N_c + 200 N_bed with a bed."""
    b = 172 * n_p + 134 * n_c + 17 * pairs * n_c + 13 * evals * n_c
    if int64:
        b += 48 * n_c
    if n_bed:
        b += 4 * n_c + 200 * n_bed
    return b


def roofline(key, prof, n_p, n_c, n_f, peak, peak_kind, int64):
    """Roofline entry of the dominant kernel of the direct-launch profiling pass.

    The pressure solve is one launch per substep (k_gs_solve on grids above 2^18
    cells, k_sc_solve below); its algorithmic bytes are 17 B per cell per red-black pair
    and 13 B per cell per FP64 residual check, counted on the fluid cells it updates
    (N_f, from classify; the dense-grid count N_c is given beside it).  P2G: 72 B per
    sample plus the lane writes (24 B per cell, 48 in int64 mode); G2P: 100 B per sample
    plus the 16 B per cell grid-velocity read."""
    n = max(prof.substeps, 1)
    phase = {PHASES[i]: prof.phase_ms[i] / n for i in range(len(PHASES))}
    pairs = prof.sweeps / n
    evals = prof.residual_evals / n
    cand = {"sweeps": phase["sweeps"], "p2g": phase["p2g"], "g2p": phase["g2p"]}
    dom = max(cand, key=cand.get)
    launches = max(prof.phase_launches[PHASES.index(dom)], 1)
    ms = prof.phase_ms[PHASES.index(dom)] / launches
    if dom == "sweeps":
        kernel = "k_gs_solve" if n_c > (1 << 18) else "k_sc_solve"
        per = (17.0 * pairs + 13.0 * evals) * n_f
        dense = (17.0 * pairs + 13.0 * evals) * n_c
        model = "17 B per fluid cell per red-black pair + 13 B per fluid cell per FP64 residual check"
    elif dom == "p2g":
        kernel = "p2g phase (k_p2g_keys, scan, k_p2g_scatter, k_p2g_tiles)"
        per = 72.0 * n_p + (48.0 if int64 else 24.0) * n_c
        dense = per
        model = "72 B per sample + the lane writes per cell"
    else:
        kernel = "k_g2p"
        per = 100.0 * n_p + 16.0 * n_c
        dense = per
        model = "100 B per sample + 16 B per cell"
    achieved = per / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
    step_ms = sum(phase.values())
    tag = WORKLOADS[key]["name"].split("_")[-1]
    return {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak,
            "traffic": ncu_traffic(kernel.split()[0], tag, pairs * n / launches if dom == "sweeps" else None),
            "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
            else "fallback 6650 GB/s", "algorithmic_bytes_per_launch": per, "bytes_model": model,
            "dense_grid_bytes_per_launch": dense, "launch_ms": ms, "launches": int(launches),
            "share_of_step": ms * launches / n / step_ms if step_ms > 0 else None,
            "fluid_cells": n_f, "grid_cells": n_c,
            "kernel_timing": "CUDA events around the kernel's phase on the engine stream, direct-launch "
                             "profiling pass over the same K substeps"}


def run_pour(lib, key, args, device, world, dist, barrier, with_learned, with_cpu, steps=None, warmup=None):
    """One workload end to end: the plain arm's profiling pass, device-timed graph
    replay and end-to-end loop, then the learned arm and the CPU baseline."""
    K = steps or args.steps
    W = warmup or args.warmup
    sim = build_scene(lib, key, args, device=device)
    n_p = sim.particle_count()
    n_c = sim.settings.cells
    n_bed = sim.num_bed
    int64 = p2g_of(key, args) == "int64"
    # warm-up substeps bring the pour to its state before the window; every timed loop
    # replays the same K substeps from a snapshot of that state
    for k in range(W):
        step(sim, key, k)
    state = sim.snapshot()

    # ---- profiling pass: direct launches, CUDA events around every phase ----
    sim.restore(state)
    sim.profile_enable(True)
    prof_ms, fluid = 0.0, []
    for j in range(K):
        sim.flush_l2()
        sim.timer_start()
        step(sim, key, W + j)
        prof_ms += sim.timer_stop()
        fluid.append(sim.latest_metrics().fluid_cells)
    prof = sim.profile_read()
    n_f = sum(fluid) / len(fluid)

    # ---- device-timed region: the same K substeps replayed as the captured graph ----
    use_graph = not args.no_graph
    if use_graph:
        sim.set_graph_mode(True)
        sim.restore(state)
        step(sim, key, W)
        sim.sync()
    sim.restore(state)
    sim.profile_enable(True)  # counts launches; graph replays record no phase events
    step_ms, particle_steps = [], 0
    barrier()
    with ClockSampler(device) as clocks:
        for j in range(K):
            particle_steps += sim.particle_count()
            sim.flush_l2()
            sim.timer_start()
            step(sim, key, W + j)
            step_ms.append(sim.timer_stop())
    barrier()
    prof_timed = sim.profile_read()
    timed_metrics = sim.latest_metrics()
    total_ms = sum(step_ms)
    if dist:
        import torch
        t = torch.tensor([total_ms, prof_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms, prof_ms = float(t[0].item()), float(t[1].item())
    value = particle_steps * world / (total_ms * 1e-3)

    # ---- end to end through the public API: the same K substeps, each with its
    # context upload and the readback of its metrics (step k's metrics are read after
    # step k+1 is queued: cs_metrics_request / cs_metrics_wait) ----
    sim.restore(state)
    sim.profile_enable(True)
    barrier()
    sim.sync()
    t0 = time.perf_counter()
    e2e_ok = True
    for j in range(K):
        step(sim, key, W + j)
        if j > 0:
            e2e_ok = e2e_ok and sim.metrics_wait().last_residual <= 1e-5
        sim.metrics_request()
    e2e_ok = e2e_ok and sim.metrics_wait().last_residual <= 1e-5
    e2e_s = time.perf_counter() - t0
    if not e2e_ok:
        print(f"warning: an end-to-end substep of {key} missed the residual target", file=sys.stderr)
    prof_e2e = sim.profile_read()
    if use_graph:
        sim.set_graph_mode(False)
    if dist:
        import torch
        t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = particle_steps * world / e2e_s

    peak, peak_kind = load_peaks()
    n = max(prof.substeps, 1)
    pairs_per_step = prof.sweeps / n
    evals_per_step = prof.residual_evals / n
    step_bytes = algorithmic_bytes(particle_steps / K, n_c, pairs_per_step, evals_per_step, n_bed, int64)
    step_gbs = step_bytes / (total_ms / K * 1e-3) / 1e9
    rl = roofline(key, prof, particle_steps / K, n_c, n_f, peak, peak_kind, int64)
    rl["step_algorithmic_bytes_dense_grid"] = step_bytes
    rl["step_achieved_gbs_dense_grid"] = step_gbs
    wl = WORKLOADS[key]
    out = {
        "value": value, "ms_per_step": total_ms / K,
        "config": {"workload": wl["name"], "scene": wl["text"], "grid": [int(g) for g in sim.settings.grid_dims],
                   "particles": n_p, "particles_mean": particle_steps / K, "bed_particles": n_bed,
                   "fluid_cells_mean": n_f, "timed_substeps": f"{W + 1}..{W + K}", "substep_dt_s": DT,
                   "residual_tol": 1e-5, "omega": float(sim.settings.rbgs_omega), "warm_start": "previous substep",
                   "check_every_pairs": int(sim.settings.check_every),
                   "first_check_pairs": int(sim.settings.first_check or sim.settings.check_every),
                   "p2g": p2g_of(key, args), "reorder_every": wl["reorder_every"], "p2g_tile": wl["p2g_tile"], "pressure_solve": "grid-wide cooperative solve" if n_c > (1 << 18)
                   else "thread-block-cluster solve", "emission": "device kernel",
                   "timed_launch": "CUDA graph replay" if use_graph else "direct launches",
                   "e2e_launch": ("CUDA graph replay" if use_graph else "direct launches")
                   + "; each step's metrics read after the next step is queued",
                   "l2": "flushed (512 MB write) before each timed step", "parallelism": f"replicas x{world}"},
        "pressure_solve_ms": (prof.phase_ms[4] + prof.phase_ms[5]) / n,
        "sweeps_per_step": pairs_per_step, "residual_checks_per_step": evals_per_step,
        "sweeps_per_step_timed": prof_timed.sweeps / max(prof_timed.substeps, 1),
        "final_residual": timed_metrics.last_residual,
        "profile_pass": {"ms_per_step": prof_ms / K, "launch": "direct, CUDA events around every phase",
                         "value": particle_steps * world / (prof_ms * 1e-3)},
        "phase_ms_per_step": {PHASES[i]: prof.phase_ms[i] / n for i in range(len(PHASES))},
        "roofline": rl,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": prof_e2e.h2d_bytes / K,
                "d2h_bytes_per_step": prof_e2e.d2h_bytes / K},
        "gpu_launches": int(prof_timed.launches),
        "clocks": clocks.summary(),
    }
    out["plain"] = {"value": value, "pressure_solve_ms": out["pressure_solve_ms"], "sweeps_per_step": pairs_per_step,
                    "warm_start": "previous substep", "value_direct_launches": out["profile_pass"]["value"]}
    if with_learned:
        out["learned"] = learned_arm(lib, key, args, device, state, K, W, barrier, dist, world)
    sim.close()
    if with_cpu:
        try:
            cb = cpu_baseline(key, args, steps=min(K, args.cpu_steps if key == "c2" else 2), warm=W)
            cb.pop("seconds", None)
            cb.pop("particles", None)
            out["cpu_baseline"] = cb
        except Exception as e:  # the oracle is test infrastructure; report its absence
            out["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "port",
                                   "sample": f"unavailable: {e}"}
    return out


def learned_arm(lib, key, args, device, state, K, W, barrier, dist, world):
    """The same timed substeps with the learned warm start (U-Net guess on the tensor
    cores, kept when its FP64 residual beats the previous-substep pressure)."""
    import numpy as np

    wfile = ROOT / "coffee_sim_b200" / "weights" / "unet_v60_64.npy"
    if not wfile.exists():
        return {"unavailable": "coffee_sim_b200/weights/unet_v60_64.npy missing"}
    sim = build_scene(lib, key, args, device=device, learned=True, populate=False)
    sim.set_learned_weights(np.load(wfile))
    # profiling pass: direct launches, per-phase events, the guess's outcome per substep
    sim.restore(state)
    sim.profile_enable(True)
    prof_ms, used = 0.0, 0
    for j in range(K):
        sim.flush_l2()
        sim.timer_start()
        step(sim, key, W + j)
        prof_ms += sim.timer_stop()
        used += int(sim.latest_metrics().learned_used)
    prof = sim.profile_read()
    final_residual = sim.latest_metrics().last_residual
    use_graph = not args.no_graph
    if use_graph:
        sim.set_graph_mode(True)
        sim.restore(state)
        step(sim, key, W)
        sim.sync()
    sim.restore(state)
    step_ms, particle_steps = [], 0
    barrier()
    for j in range(K):
        particle_steps += sim.particle_count()
        sim.flush_l2()
        sim.timer_start()
        step(sim, key, W + j)
        step_ms.append(sim.timer_stop())
    barrier()
    total_ms = sum(step_ms)
    if dist:
        import torch
        t = torch.tensor([total_ms, prof_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms, prof_ms = float(t[0].item()), float(t[1].item())
    n = max(prof.substeps, 1)
    out = {"value": particle_steps * world / (total_ms * 1e-3), "ms_per_step": total_ms / K,
           "value_direct_launches": particle_steps * world / (prof_ms * 1e-3),
           "pressure_solve_ms": (prof.phase_ms[4] + prof.phase_ms[5] + prof.phase_ms[10]) / n,
           "learned_guess_ms": prof.phase_ms[10] / n, "sweeps_per_step": prof.sweeps / n,
           "guess_kept_fraction": used / K, "final_residual": final_residual,
           "weights": "coffee_sim_b200/weights/unet_v60_64.npy (python -m coffee_sim_b200.train_unet)",
           "launch": ("CUDA graph replay" if use_graph else "direct launches") +
                     "; phase times and kept fraction from a direct-launch profiling pass"}
    sim.close()
    return out


def cpu_baseline(key, args, steps, warm):
    """Time the CPU oracle (all host threads) on the substeps the GPU arm times: the
    same scene, `warm` untimed substeps, then the first `steps` of the timed window."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib
    lib = oracle_lib.oracle_library()
    nthreads = int(lib.lib.oracle_get_threads())
    sim = build_scene(lib, key, args)
    for k in range(warm):
        step(sim, key, k)
    n0 = sim.particle_count()
    particle_steps = 0
    sweeps = 0
    t = time.perf_counter()
    for j in range(steps):
        particle_steps += sim.particle_count()
        step(sim, key, warm + j)
        sweeps += sim.latest_metrics().last_sweeps
    dt = time.perf_counter() - t
    out = {"value": particle_steps / dt, "unit": UNIT, "cores": nthreads, "kind": "port",
           "sample": f"substeps {warm + 1}..{warm + steps} of the {WORKLOADS[key]['name']} pour ({n0} samples at "
                     f"the start; {sweeps / max(steps, 1):.0f} red-black pairs per substep), the first {steps} of "
                     f"the GPU arm's timed substeps; oracle/ C++ restatement, OpenMP on {nthreads} threads, -O3",
           "seconds": dt, "particles": n0}
    if key == "c2":
        # the next two substeps on one thread (integer grid atomics make the result the same)
        lib.lib.oracle_set_threads(1)
        ps1, t1 = 0, time.perf_counter()
        for j in range(2):
            ps1 += sim.particle_count()
            step(sim, key, warm + steps + j)
        dt1 = time.perf_counter() - t1
        lib.lib.oracle_set_threads(nthreads)
        out["single_thread"] = {"value": ps1 / dt1, "unit": UNIT, "cores": 1,
                                "sample": f"substeps {warm + steps + 1}..{warm + steps + 2} of the same pour"}
    sim.close()
    return out


def run_reference(args, rank):
    """The reference arm: the oracle on a bounded sample of the headline workload."""
    if rank != 0:
        return 0
    key = args.workload if args.workload != "c4" else "c2"
    steps = min(args.steps, args.cpu_steps if key == "c2" else 2)
    warm = args.warmup if key == "c2" else min(args.warmup, 5)
    res = cpu_baseline(key, args, steps=steps, warm=warm)
    wl = WORKLOADS[key]
    line = {"metric": METRIC, "value": res["value"], "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": steps, "warmup": warm, "ms_per_step": res["seconds"] * 1e3 / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator)",
            "config": {"workload": wl["name"], "particles": res["particles"], "omega": wl["omega"],
                       "residual_tol": 1e-5},
            "cpu_baseline": {"value": res["value"], "unit": UNIT, "cores": res["cores"], "kind": "port",
                             "sample": res["sample"]},
            "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if "single_thread" in res:
        line["cpu_baseline"]["single_thread"] = res["single_thread"]
    print(json.dumps(line), flush=True)
    return 0


def run_c4(args, rank, world, local, dist, steps=None, warmup=None):
    """Batched ensemble workload: `--instances` V60 pours at 64^3 stepped together (one
    launch per pass over all instances); under torchrun each rank runs its share of the
    instances (particle-count balanced) and the statistics are gathered.  Returns the
    workload's JSON object."""
    K = steps or args.steps
    W = warmup or args.warmup
    from coffee_sim_b200 import scenes, shard
    from coffee_sim_b200.sim import MpmEnsemble, engine_library

    lib = engine_library()
    settings, fills = scenes.c4_ensemble(lib, n=args.instances)
    est = [int(f["fill_top"] * 1e6 + f["pool_depth"] * 1e7) for f in fills]  # placement weights
    mine = shard.local_instances(est, rank, world)
    for i in mine:
        settings[i].raw.device = local
        settings[i].raw.device_emission = 1
        settings[i].raw.p2g_mode = 1
        settings[i].raw.rbgs_omega = 1.92 if args.omega is None else args.omega
        settings[i].raw.max_sweeps = args.max_sweeps
        settings[i].raw.check_every = 60 if args.check_every is None else args.check_every
        settings[i].raw.first_check = 0 if args.first_check is None else args.first_check
        settings[i].raw.rbgs_kernel = {"auto": 0, "p2p": 2, "cluster": 3, "grid": 2}[args.solve_sync]
    # the batched substep is captured once and replayed (no host synchronisation per substep)
    settings[mine[0]].raw.use_graph = 0 if args.no_graph else 1
    ens = MpmEnsemble([settings[i] for i in mine], lib)
    settings[mine[0]].raw.use_graph = 0
    for k, i in enumerate(mine):
        f = fills[i]
        scenes.populate_c2(ens.member(k), fill_top=f["fill_top"], pool_depth=f["pool_depth"], seed=f["seed"])
    dt = scenes.C2_DT
    for _ in range(W):
        ens.step_substep(dt)
    ens.metrics(0)  # synchronises
    if dist:
        dist.barrier()
    particle_steps = 0
    with ClockSampler(local) as clocks:
        ens.timer_start()
        for _ in range(K):
            particle_steps += sum(ens.particle_count(k) for k in range(len(mine)))
            ens.step_substep(dt)
        elapsed = ens.timer_stop() * 1e-3  # CUDA events on the ensemble's stream
    ms = [ens.metrics(k) for k in range(len(mine))]
    stats = shard.gather_statistics({i: [float(ens.particle_count(k)), float(ms[k].last_sweeps),
                                         float(ms[k].residual_checks)] for k, i in enumerate(mine)})
    if dist:
        import torch
        t = torch.tensor([elapsed, float(particle_steps)], dtype=torch.float64, device="cuda")
        dist.all_reduce(t[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        elapsed, particle_steps = float(t[0].item()), float(t[1].item())
    counts = [v[0] for v in stats.values()]
    # step roofline: compulsory bytes of every instance's substep (the bench's formula,
    # dense 64^3 grid per instance) over the step time, against the measured HBM peak
    # (pairs and FP64 residual checks: each instance's last substep, standing in for the
    # window's mean)
    n_c = int(settings[0].cells)
    n_bed = int(settings[0].raw.bed.num_particles)
    step_bytes = sum(algorithmic_bytes(v[0], n_c, v[1], v[2], n_bed) for v in stats.values())
    peak, peak_kind = load_peaks()
    step_gbs = step_bytes / (elapsed / K) / 1e9
    line = {"metric": METRIC, "value": particle_steps / elapsed, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": elapsed * 1e3 / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ensemble generator)",
            "config": {"workload": f"c4_ensemble_{args.instances}x64cube", "instances": args.instances,
                       "particles_min": min(counts), "particles_max": max(counts), "particles_total": sum(counts),
                       "pairs_mean": sum(v[1] for v in stats.values()) / len(stats),
                       "residual_checks_mean": sum(v[2] for v in stats.values()) / len(stats), "residual_tol": 1e-5,
                       "omega": float(settings[mine[0]].raw.rbgs_omega),
                       "check_every_pairs": int(settings[mine[0]].raw.check_every),
                       "first_check_pairs": int(settings[mine[0]].raw.first_check or settings[mine[0]].raw.check_every),
                       "timed_launch": "direct launches" if args.no_graph else "CUDA graph replay of the batched substep",
                       "timing": "CUDA events on the ensemble stream, max over ranks",
                       "l2": "not flushed: 64 resident pours' particle and grid arrays exceed the 126 MB L2 many times over"
                             if args.instances >= 16 else "not flushed",
                       "parallelism": f"instances sharded over {world} GPU(s)"},
            "roofline": {"bound": "hbm", "kernel": "whole batched substep", "achieved": step_gbs, "peak": peak,
                         "unit": "GB/s", "frac": step_gbs / peak, "traffic": None,
                         "algorithmic_bytes_per_step": step_bytes,
                         "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                         else "fallback 6650 GB/s"},
            "clocks": clocks.summary()}
    ens.close()
    if not args.no_learned:
        line["learned"] = c4_learned_arm(args, lib, mine, settings, fills, local, dist, K, W)
    return line


def c4_learned_arm(args, lib, mine, settings, fills, local, dist, K, W):
    """The same ensemble with the learned warm start: each instance's U-Net guess runs
    between the batched classify and the batched solve, kept when its FP64 residual is
    lower than the previous-substep start's."""
    import numpy as np
    from coffee_sim_b200 import _ffi, scenes
    from coffee_sim_b200.sim import MpmEnsemble

    wfile = ROOT / "coffee_sim_b200" / "weights" / "unet_v60_64.npy"
    if not wfile.exists():
        return {"unavailable": "coffee_sim_b200/weights/unet_v60_64.npy missing"}
    for i in mine:
        settings[i].raw.warm_start = _ffi.CS_WARM_LEARNED
    ens = MpmEnsemble([settings[i] for i in mine], lib)
    ens.set_learned_weights(np.load(wfile))
    for k, i in enumerate(mine):
        f = fills[i]
        scenes.populate_c2(ens.member(k), fill_top=f["fill_top"], pool_depth=f["pool_depth"], seed=f["seed"])
    dt = scenes.C2_DT
    for _ in range(W):
        ens.step_substep(dt)
    ens.metrics(0)
    if dist:
        dist.barrier()
    particle_steps, kept = 0, 0
    ens.timer_start()
    for _ in range(K):
        particle_steps += sum(ens.particle_count(k) for k in range(len(mine)))
        ens.step_substep(dt)
        kept += sum(int(ens.metrics(k).learned_used) for k in range(len(mine)))
    elapsed = ens.timer_stop() * 1e-3
    pairs = sum(ens.metrics(k).last_sweeps for k in range(len(mine))) / max(len(mine), 1)
    ens.close()
    if dist:
        import torch
        t = torch.tensor([elapsed, float(particle_steps), float(kept)], dtype=torch.float64, device="cuda")
        dist.all_reduce(t[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        elapsed, particle_steps, kept = float(t[0].item()), float(t[1].item()), float(t[2].item())
    return {"value": particle_steps / elapsed, "ms_per_step": elapsed * 1e3 / K,
            "guess_kept_fraction": kept / (K * args.instances), "pairs_mean_last_substep": pairs,
            "timing": "CUDA events on the ensemble stream"}


def make_parser():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--workload", default="c5", choices=["c5", "c3", "c2", "c4"],
                    help="headline workload: c5 (192^3, default), c3 (128^3 spiral pour), c2 (64^3), "
                         "c4 (batched ensemble of 64 pours at 64^3)")
    ap.add_argument("--nested", default="c3,c2,c4",
                    help="workloads also run and reported as nested keys of the line ('none' for none)")
    ap.add_argument("--nested-steps", type=int, default=10, help="timed substeps of each nested workload")
    ap.add_argument("--grid", type=int, default=None, help="grid side override (small CPU checks of the arms)")
    ap.add_argument("--omega", type=float, default=None, help="over-relaxation (default: the workload's)")
    ap.add_argument("--p2g", default="default", choices=["default", "atomic", "sorted", "int64"],
                    help="P2G accumulation (default: the workload's)")
    ap.add_argument("--max-sweeps", type=int, default=12000)
    ap.add_argument("--solve-sync", default="auto", choices=["auto", "p2p", "cluster", "grid"],
                    help="pressure solve: auto (cluster-resident up to 2^18 cells, grid-wide above), the "
                         "cluster solve with point-to-point waits or cluster barriers, or the grid-wide solve")
    ap.add_argument("--check-every", type=int, default=None, help="cap on pairs between FP64 residual checks")
    ap.add_argument("--first-check", type=int, default=None,
                    help="pairs before each solve's first FP64 residual check (default: the workload's)")
    ap.add_argument("--cpu-steps", type=int, default=40, help="cap on the 64^3 CPU baseline's timed substeps")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="timed loops without CUDA-graph replay")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-warm-start arms")
    ap.add_argument("--instances", type=int, default=64)
    return ap


def default_args(argv=()):
    """The bench's arguments as a run with `argv` would have them (tests build the
    timed scenes with these)."""
    args = make_parser().parse_args(list(argv))
    args.warmup = max(args.warmup, 3)
    return args


def main():
    args = default_args(sys.argv[1:])
    nested = [] if args.nested in ("", "none") else [k for k in args.nested.split(",") if k != args.workload]

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    if args.impl == "reference":
        rc = run_reference(args, rank)
        if dist:
            dist.destroy_process_group()
        return rc

    from coffee_sim_b200.sim import engine_library
    lib = engine_library()

    def barrier():
        if dist:
            import torch
            dist.barrier()
            torch.cuda.synchronize()

    solo = rank == 0 and world == 1 and not args.no_cpu
    if args.workload == "c4":
        res = run_c4(args, rank, world, local, dist)
    else:
        res = run_pour(lib, args.workload, args, local, world, dist, barrier, with_learned=not args.no_learned,
                       with_cpu=solo)
    line = {"metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded V60 scene generator; no dataset)"}
    for k, v in res.items():
        if k not in line:
            line[k] = v
    for key in nested:
        ns = min(args.steps, args.nested_steps)
        if key == "c4":
            line["c4"] = run_c4(args, rank, world, local, dist, steps=ns)
        else:
            line[key] = run_pour(lib, key, args, local, world, dist, barrier, with_learned=not args.no_learned,
                                 with_cpu=solo and key == "c2", steps=ns)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
