"""Reorder of the water samples by P2G tile (CsSettings.reorder_every): every N substeps
the water slots are permuted stably by the 4^3-cell tile of each sample's P2G base cell.

The engine sorts the keys with a radix sort and the oracle with a stable comparison
sort, so the permutation is the same and the states stay equal bit for bit; and since
every per-sample update is independent of the slot and every grid sum is an integer
sum, a reordered pour has the same physics as one that is never reordered."""
import numpy as np
import pytest

from coffee_sim_b200 import _ffi, scenes
from coffee_sim_b200.sim import MpmSim3D
from helpers import mismatch, relerr

pytestmark = pytest.mark.gpu


def _v60(lib, reorder_every, grid=48):
    s = scenes.c2_v60(lib, grid=grid, max_particles=200000)
    r = s.raw
    r.rbgs_omega = 1.92
    r.check_every = 40
    r.device_emission = 1
    r.p2g_mode = _ffi.CS_P2G_SORTED_SHARED
    r.reorder_every = reorder_every
    return s


def _rows_sorted(a):
    return a[np.lexsort(a.T[::-1])]


def test_reorder_matches_oracle(engine, oracle):
    """V60 pour at 48^3, reordered every 4 substeps: 10 substeps (reorders before
    substeps 1, 5 and 9) bit for bit against the oracle."""
    e, o = MpmSim3D(_v60(engine, 4), engine), MpmSim3D(_v60(oracle, 4), oracle)
    assert scenes.populate_c2(e) == scenes.populate_c2(o) > 50000
    for k in range(10):
        e.step_substep(scenes.C2_DT)
        o.step_substep(scenes.C2_DT)
        assert e.latest_metrics().last_sweeps == o.latest_metrics().last_sweeps, k
    for name, a, b in (("particles", e.read_particles(), o.read_particles()),
                       ("affine", e.read_affine(), o.read_affine()),
                       ("pressure", e.read_pressure(), o.read_pressure()),
                       ("grid_vel", e.read_grid_vel(), o.read_grid_vel())):
        assert mismatch(a, b) == 0, (name, relerr(a, b))
    e.close()
    o.close()


def test_reorder_keeps_the_physics(engine):
    """Reordered every 3 substeps against never reordered: the same pair counts and
    pressure field, and the same samples (as a set of rows) after 9 substeps; the
    reordered pour's water samples are in tile order after a reorder."""
    a, b = MpmSim3D(_v60(engine, 0), engine), MpmSim3D(_v60(engine, 3), engine)
    assert scenes.populate_c2(a) == scenes.populate_c2(b)
    for k in range(9):
        a.step_substep(scenes.C2_DT)
        b.step_substep(scenes.C2_DT)
        assert a.latest_metrics().last_sweeps == b.latest_metrics().last_sweeps, k
    assert mismatch(a.read_pressure(), b.read_pressure()) == 0
    pa, pb = a.read_particles(), b.read_particles()
    assert mismatch(pa, pb) > 0  # the slots were permuted
    nb = a.num_bed
    assert mismatch(pa[:nb], pb[:nb]) == 0  # bed samples keep their slots
    rows = lambda p, aff: np.concatenate([p, aff], axis=1)[nb:]
    assert mismatch(_rows_sorted(rows(pa, a.read_affine())), _rows_sorted(rows(pb, b.read_affine()))) == 0
    a.close()
    b.close()


def test_reorder_with_graph_replay_matches_direct(engine):
    """The reorder runs ahead of the replayed substep graph: graph replay and direct
    launches give the same state bit for bit over 8 substeps (reordered every 3)."""
    sims = []
    for graph in (False, True):
        sim = MpmSim3D(_v60(engine, 3), engine)
        scenes.populate_c2(sim)
        sim.set_graph_mode(graph)
        sims.append(sim)
    for k in range(8):
        for sim in sims:
            sim.step_substep(scenes.C2_DT)
    assert sims[0].latest_metrics().last_sweeps == sims[1].latest_metrics().last_sweeps
    assert mismatch(sims[0].read_particles(), sims[1].read_particles()) == 0
    assert mismatch(sims[0].read_pressure(), sims[1].read_pressure()) == 0
    for sim in sims:
        sim.close()
