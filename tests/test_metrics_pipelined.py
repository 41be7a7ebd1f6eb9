"""Pipelined metrics readback (cs_metrics_request / cs_metrics_wait): a host loop reads
substep k's metrics while substep k+1 runs, and gets what a synchronous read after
substep k returns."""
import pytest

from coffee_sim_b200 import _ffi, scenes
from coffee_sim_b200.sim import MpmSim3D

FIELDS = ("last_sweeps", "residual_checks", "last_residual", "initial_residual", "fluid_cells", "max_abs_div",
          "div_clamp_fires", "pressure_clamp_fires", "mass_overflow_fires", "nan_flag", "timeout_flag")


def _v60(lib, graph, grid=64, max_particles=400000):
    s = scenes.c2_v60(lib, grid=grid, max_particles=max_particles)
    s.raw.rbgs_omega = 1.92
    s.raw.device_emission = 1
    s.raw.use_graph = graph
    s.raw.check_every = 60
    sim = MpmSim3D(s, lib)
    scenes.populate_c2(sim)
    return sim


def _pipelined(sim, n):
    out = []
    for k in range(n):
        sim.step_substep(scenes.C2_DT)
        if k > 0:
            out.append(sim.metrics_wait())
        sim.metrics_request()
    out.append(sim.metrics_wait())
    return out


def _synchronous(sim, n):
    out = []
    for _ in range(n):
        sim.step_substep(scenes.C2_DT)
        out.append(sim.latest_metrics())
    return out


def test_request_and_wait_pair_up(oracle):
    sim = _v60(oracle, graph=0, grid=32, max_particles=60000)
    with pytest.raises(_ffi.CsError) as e:
        sim.metrics_wait()
    assert e.value.code == _ffi.CS_ERR_INVALID_ARG
    sim.step_substep(scenes.C2_DT)
    sim.metrics_request()
    with pytest.raises(_ffi.CsError):
        sim.metrics_request()
    m = sim.metrics_wait()
    ref = sim.latest_metrics()
    assert all(getattr(m, f) == getattr(ref, f) for f in FIELDS)


def test_oracle_pipelined_loop_equals_synchronous_loop(oracle):
    a = _v60(oracle, graph=0, grid=32, max_particles=60000)
    b = _v60(oracle, graph=0, grid=32, max_particles=60000)
    for ma, mb in zip(_synchronous(a, 3), _pipelined(b, 3)):
        assert all(getattr(ma, f) == getattr(mb, f) for f in FIELDS)


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [0, 1])
def test_engine_pipelined_loop_equals_synchronous_loop(engine, graph):
    """V60 64^3: six substeps read one behind (graph replay: step k+1 is queued before
    step k's metrics are read) against reading after every step."""
    a, b = _v60(engine, graph), _v60(engine, graph)
    sync, piped = _synchronous(a, 6), _pipelined(b, 6)
    for k, (ma, mb) in enumerate(zip(sync, piped)):
        for f in FIELDS:
            assert getattr(ma, f) == getattr(mb, f), (k, f, getattr(ma, f), getattr(mb, f))
        assert ma.last_residual <= 1e-5
    # the running totals the profile keeps agree as well
    a.profile_enable(True)
    b.profile_enable(True)
    _synchronous(a, 2)
    _pipelined(b, 2)
    pa, pb = a.profile_read(), b.profile_read()
    assert (pa.sweeps, pa.residual_evals) == (pb.sweeps, pb.residual_evals)
