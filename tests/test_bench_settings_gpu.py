"""The benchmark's exact settings against the CPU oracle.

bench.py times its workloads with a combination of settings that the other parity
tests cover one by one: over-relaxation, the cap on pairs between FP64 residual
checks and the first-check interval of each workload, tile-sorted (or int64) P2G,
device jet emission, and the substep replayed as a captured CUDA graph.  Here the
scenes come from bench.py's own builder and the engine replays its graph, while the
oracle steps the same substeps; pair counts and state must agree bit for bit over
the bench's warm-up and timed window."""
import pytest

import bench
from helpers import mismatch, relerr

pytestmark = pytest.mark.gpu


def _run(engine, oracle, key, substeps, compare_every):
    args = bench.default_args()
    e = bench.build_scene(engine, key, args)
    o = bench.build_scene(oracle, key, args)
    assert e.particle_count() == o.particle_count() > 0
    e.set_graph_mode(True)
    for k in range(substeps):
        bench.step(e, key, k)
        bench.step(o, key, k)
        if (k + 1) % compare_every and k + 1 != substeps:
            continue
        me, mo = e.latest_metrics(), o.latest_metrics()   # graph mode: totals read lazily here
        assert me.last_sweeps == mo.last_sweeps > 0, (key, k, me.last_sweeps, mo.last_sweeps)
        assert me.residual_checks == mo.residual_checks, (key, k)
        assert me.last_residual <= 1e-5, (key, k)
        for name, a, b in (("pressure", e.read_pressure(), o.read_pressure()),
                           ("particles", e.read_particles(), o.read_particles())):
            assert mismatch(a, b) == 0, (key, k, name, relerr(a, b))
    e.close()
    o.close()


def test_bench_c2_window_matches_oracle(engine, oracle):
    """64^3 pour: the bench's 5 warm-up and 20 timed substeps (omega 1.92, check cap 60,
    first check after 125 pairs, tile-sorted P2G, device emission, graph replay)."""
    _run(engine, oracle, "c2", 25, 5)


def test_bench_c5_settings_match_oracle(engine, oracle):
    """192^3 headline pour with the bench's settings (omega 1.95, check cap 60, int64
    P2G, device emission, graph replay of the grid-wide solve): the first three
    substeps of the warm-up."""
    _run(engine, oracle, "c5", 3, 1)
