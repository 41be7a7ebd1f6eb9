"""bench.py's reference arm on the CPU: one JSON line with the fields the bench contract
names (the GPU arm runs under `pytest -m gpu` only through the library tests)."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_prints_one_json_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "2", "--warmup", "3",
                        "--workload", "c2", "--grid", "32"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "particle-steps/s"
    assert d["steps"] == 2 and d["warmup"] == 3 and d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert cb["single_thread"]["cores"] == 1 and cb["single_thread"]["value"] > 0
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


class _Profile:
    """A profiling pass as the engine's CsProfile reports it: K substeps with per-phase
    device milliseconds and launch counts, red-black pairs and residual evaluations."""

    def __init__(self, substeps, phase_ms, phase_launches, sweeps, evals):
        self.substeps, self.phase_ms, self.phase_launches = substeps, phase_ms, phase_launches
        self.sweeps, self.residual_evals = sweeps, evals


def test_roofline_of_the_headline_solve():
    """The bench's roofline entry for a 192^3 profile whose solve dominates: algorithmic
    bytes (17 B per fluid cell per pair + 13 B per fluid cell per residual check) over the
    solve's event-timed launch, the fraction of the peak, and the DRAM traffic scaled
    from the committed ncu summary's bytes per pair."""
    import bench
    ph = bench.PHASES
    ms = [0.0] * len(ph)
    launches = [0] * len(ph)
    k = 20
    ms[ph.index("sweeps")], launches[ph.index("sweeps")] = 3.32 * k, k
    ms[ph.index("p2g")], launches[ph.index("p2g")] = 1.64 * k, 4 * k
    ms[ph.index("g2p")], launches[ph.index("g2p")] = 1.46 * k, k
    prof = _Profile(k, ms, launches, sweeps=231 * k, evals=6 * k)
    n_p, n_c, n_f = 7_880_000, 192 ** 3, 1_090_000
    r = bench.roofline("c5", prof, n_p, n_c, n_f, 6450.0, "measured", True)
    per = (17.0 * 231 + 13.0 * 6) * n_f
    assert r["kernel"] == "k_gs_solve" and r["bound"] == "hbm" and r["unit"] == "GB/s"
    assert r["algorithmic_bytes_per_launch"] == per
    assert abs(r["achieved"] - per / 3.32e-3 / 1e9) < 1e-6 * r["achieved"]
    assert abs(r["frac"] - r["achieved"] / 6450.0) < 1e-12
    assert r["traffic"] == 119433 * 231              # profiles/k_gs_solve_v60_192cube.md
    assert r["dense_grid_bytes_per_launch"] == (17.0 * 231 + 13.0 * 6) * n_c
    assert abs(r["share_of_step"] - 3.32 / (3.32 + 1.64 + 1.46)) < 1e-9


def test_roofline_picks_the_dominant_particle_pass():
    """When G2P outweighs the solve, the entry is G2P's: 100 B per sample + 16 B per cell."""
    import bench
    ph = bench.PHASES
    ms = [0.0] * len(ph)
    launches = [1] * len(ph)
    ms[ph.index("sweeps")], ms[ph.index("g2p")] = 0.2, 0.9
    prof = _Profile(1, ms, launches, sweeps=10, evals=2)
    r = bench.roofline("c2", prof, 280_000, 64 ** 3, 40_000, 6450.0, "fallback", False)
    assert r["kernel"] == "k_g2p"
    assert r["algorithmic_bytes_per_launch"] == 100.0 * 280_000 + 16.0 * 64 ** 3
    assert r["peak_source"].startswith("fallback")
