"""The grid-wide pressure solve (solver_grid.cuh: row segments of fluid cells, one
cooperative launch, grid barriers between the colours, FP64 checks on the device)
against the per-colour launch path, the cluster-resident solve and the CPU oracle.

The solve restates k_refine_* cell for cell in the same face order, so pressures and
pair counts are compared for equality."""
import numpy as np
import pytest

from coffee_sim_b200 import _ffi, scenes
from coffee_sim_b200.sim import MpmSim3D
from helpers import mismatch

pytestmark = pytest.mark.gpu

PER_COLOUR, CLUSTER_P2P, GRID = 1, 2, 4


def _v60(engine, grid, kernel, omega=1.92, check_every=40, first_check=0, max_particles=340000):
    s = scenes.c2_v60(engine, grid=grid, max_particles=max_particles)
    r = s.raw
    r.rbgs_omega = omega
    r.rbgs_kernel = kernel
    r.check_every = check_every
    r.first_check = first_check
    r.max_sweeps = 8000
    r.device_emission = 1
    r.p2g_mode = _ffi.CS_P2G_SORTED_SHARED
    return s


@pytest.mark.parametrize("other", [PER_COLOUR, CLUSTER_P2P])
def test_grid_solve_matches_per_colour_and_cluster_at_64(engine, other):
    """V60 pour at 64^3: the grid-wide solve (rbgs_kernel 4) takes the same pairs and
    residual checks as the per-colour launches and the cluster solve, and gives the same
    pressure and particle state bit for bit, substep after substep."""
    sims = []
    for kernel in (other, GRID):
        sim = MpmSim3D(_v60(engine, 64, kernel), engine)
        scenes.populate_c2(sim)
        sims.append(sim)
    sims[1].profile_enable(True)
    for k in range(4):
        for sim in sims:
            sim.step_substep(scenes.C2_DT)
        ma, mb = sims[0].latest_metrics(), sims[1].latest_metrics()
        assert sims[1].profile_read().phase_launches[4] == k + 1  # one solve launch per substep
        assert ma.last_sweeps == mb.last_sweeps > 0
        assert ma.residual_checks == mb.residual_checks >= 2
        assert mb.last_residual <= 1e-5 and mb.timeout_flag == 0
        assert mismatch(sims[0].read_pressure(), sims[1].read_pressure()) == 0
        assert mismatch(sims[0].read_particles(), sims[1].read_particles()) == 0
    for sim in sims:
        sim.close()


def test_grid_solve_matches_oracle_at_96(engine, oracle):
    """V60 pour at 96^3 (884,736 cells, above the cluster solve's grid limit, so the
    engine picks the grid-wide solve by itself): two substeps against the oracle, pair
    counts, pressure, grid velocity and particles bit for bit."""
    e = MpmSim3D(_v60(engine, 96, 0, max_particles=1_100_000), engine)
    o = MpmSim3D(_v60(oracle, 96, 0, max_particles=1_100_000), oracle)
    assert scenes.populate_c2(e) == scenes.populate_c2(o) > 500_000
    e.profile_enable(True)
    for k in range(2):
        e.step_substep(scenes.C2_DT)
        o.step_substep(scenes.C2_DT)
        me, mo = e.latest_metrics(), o.latest_metrics()
        assert e.profile_read().phase_launches[4] == k + 1
        assert me.last_sweeps == mo.last_sweeps > 0, (me.last_sweeps, mo.last_sweeps)
        assert me.last_residual <= 1e-5
        assert mismatch(e.read_pressure(), o.read_pressure()) == 0
        assert mismatch(e.read_grid_vel(), o.read_grid_vel()) == 0
        assert mismatch(e.read_particles(), o.read_particles()) == 0
    e.close()
    o.close()


def test_grid_solve_graph_replay_matches_direct(engine):
    """The grid-wide solve captured in the substep CUDA graph (prep kernels, CUB scan,
    cooperative launch, result accounting) replays bit-exact with direct launches at
    96^3, and the lazily read totals give the same pair counts."""
    sims = []
    for graph in (False, True):
        sim = MpmSim3D(_v60(engine, 96, 0, max_particles=1_100_000), engine)
        scenes.populate_c2(sim)
        sim.set_graph_mode(graph)
        sims.append(sim)
    for k in range(3):
        for sim in sims:
            sim.step_substep(scenes.C2_DT)
        ma, mb = sims[0].latest_metrics(), sims[1].latest_metrics()
        assert ma.last_sweeps == mb.last_sweeps > 0
        assert ma.residual_checks == mb.residual_checks
        assert mb.last_residual <= 1e-5
    assert mismatch(sims[0].read_pressure(), sims[1].read_pressure()) == 0
    assert mismatch(sims[0].read_particles(), sims[1].read_particles()) == 0
    for sim in sims:
        sim.close()


def test_grid_solve_without_fluid(engine):
    """A grid with no fluid: the solve ends at once (zero pairs) and leaves the
    pressure at zero."""
    s = scenes.c1_water_block(engine)
    r = s.raw
    r.grid_dims[:] = (96, 96, 96)
    r.pressure_storage = _ffi.CS_PRESSURE_FP32
    r.solve_mode = _ffi.CS_SOLVE_RESIDUAL
    r.residual_tol = 1e-5
    r.rbgs_kernel = GRID
    sim = MpmSim3D(s, engine)
    sim.step_substep(scenes.C2_DT)
    m = sim.latest_metrics()
    assert m.last_sweeps == 0 and m.timeout_flag == 0
    assert np.count_nonzero(sim.read_pressure()) == 0
    sim.close()
