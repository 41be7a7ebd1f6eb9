"""The allocation-free pressure solve (cs_pressure_solve_noalloc) against the
engine's own solve.

Callers that cannot allocate device memory while they run hand the solve their own
device arrays; its scratch is a static device array of the library.  This test
takes the solver inputs from a real engine state - the cell kinds, grid velocity
and volume lanes right after classify - rebuilds the fill fraction and divergence
exactly as classify computes them (float32, same operation order), runs the
allocation-free solve twice in a row on copies of those inputs, and compares each
result with the pressure the engine's own solve produced from the same state, to
the 1e-5 relative tolerance of the solver's parity tests.  A second case takes a V60
pour at 32^3, whose pressure system has solid faces (the cone wall) and bed-coupled
faces (the coffee bed), with the fill and divergence read back from the engine.  Both
check that the calls allocate nothing: the device's free memory is the same before
and after the second call.  Kept in its own file so pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from coffee_sim_b200 import _ffi, scenes
from coffee_sim_b200.sim import MpmSim3D

pytestmark = pytest.mark.gpu

F = np.float32


def _settings(engine):
    s = scenes.c1_water_block(engine)
    r = s.raw
    r.pressure_storage = _ffi.CS_PRESSURE_FP32
    r.solve_mode = _ffi.CS_SOLVE_RESIDUAL
    r.warm_start = _ffi.CS_WARM_NONE
    r.rbgs_omega = 1.9
    r.residual_tol = 1e-5
    r.max_sweeps = 2000
    r.check_every = 10
    return s


def _pool(sim):
    # a resting block on the floor of the 1 m box (decimetre units), so the solve has
    # hydrostatic pressure to find
    return sim.add_water_block((-2.0, -4.8, -2.0), (2.0, -1.5, 2.0), per_axis=2, jitter=0.25, seed=3)


def _classify_inputs(s, kind, lanes, gvel):
    """fill and divergence of every cell as classify writes them (no bed, no solid
    cells in this scene), float32 throughout."""
    g = [int(v) for v in s.raw.grid_dims]
    dx = F(s.raw.bounds_size[0]) / F(g[0])
    inv_dx = F(1.0) / dx
    cv = dx * dx * dx
    p_vol = dx * dx * dx * F(s.raw.particle_volume_cells)
    inv_fp = F(1.0 / 262144.0)
    rest = lanes[4].astype(F) * inv_fp
    cur = lanes[5].astype(F) * inv_fp
    fluid = (kind == 1) | (kind == 2) | (kind == 3)
    fill = np.where((kind == 2) | (kind == 3), F(1.0),
                    np.where(kind == 1, np.clip(np.maximum(rest, cur) / np.maximum(cv, F(1e-8)), F(0.0), F(1.0)),
                             F(0.0))).astype(F)
    v = gvel.reshape(g[2], g[1], g[0], 4)
    out = {}
    for comp, axis in ((0, 2), (1, 1), (2, 0)):
        c = v[..., comp]
        lo = np.roll(c, 1, axis=axis)
        hi = np.roll(c, -1, axis=axis)
        sl_lo = [slice(None)] * 3
        sl_lo[axis] = 0
        sl_hi = [slice(None)] * 3
        sl_hi[axis] = -1
        lo[tuple(sl_lo)] = -c[tuple(sl_lo)]   # ghost mirror at the grid faces
        hi[tuple(sl_hi)] = -c[tuple(sl_hi)]
        out[comp] = (hi - lo).astype(F)
    div = (F(0.5) * inv_dx) * ((out[0] + out[1]) + out[2])
    div = div.reshape(-1).astype(F)
    # volume_projection_target_divergence (shader.rs:597-619)
    eps = np.maximum(cv * F(1e-5), p_vol * F(1e-3))
    safe = np.where(rest > eps, rest, F(1.0))
    j = (cur / safe).astype(F)
    ce = np.clip(F(1.0) - j, F(0.0), F(0.75))
    ee = np.clip(j - F(1.0), F(0.0), F(0.75))
    t = ce * F(32.0) - ee * F(2.0)
    packed = np.maximum(rest, cur) / np.maximum(cv, F(1e-8))
    over = np.maximum(packed - F(1.2), F(0.0))
    target = np.where(rest > eps, np.maximum(t, over * F(32.0)), F(0.0)).astype(F)
    lim = np.minimum(F(4.0) * F(s.raw.max_velocity) * inv_dx, F(8191.0))
    d = np.clip((div - target).astype(F), -lim, lim).astype(F)
    return fill, np.where(fluid, d, F(0.0)).astype(F)


def test_noalloc_solve_matches_engine_solve(engine):
    pytest.importorskip("torch")
    s = _settings(engine)
    a, b = MpmSim3D(s, engine), MpmSim3D(s, engine)
    assert _pool(a) == _pool(b) > 0
    for _ in range(8):
        a.step_substep(scenes.C1_DT)
        b.step_substep(scenes.C1_DT)
    a.step_substep_partial(scenes.C1_DT, 7)   # through classify: solver inputs
    b.step_substep_partial(scenes.C1_DT, 8)   # through the pressure solve: reference output
    kind = a.read_cell_kind()
    fill, div = _classify_inputs(s, kind, a.read_grid_lanes(), a.read_grid_vel())
    want = b.read_pressure()
    mb = b.latest_metrics()
    assert mb.last_sweeps > 0 and np.abs(want).max() > 0

    _solve_twice_and_compare(engine, s, kind, fill, div, want, mb, scenes.C1_DT, omega=1.9)
    a.close()
    b.close()


def _solve_twice_and_compare(engine, s, kind, fill, div, want, mb, dt, omega):
    """Two allocation-free solves in a row on the same inputs, each from a zero
    pressure, against the engine's solved pressure; the device's free memory is read
    after the first call and must be unchanged after the second."""
    import torch
    g = [int(v) for v in s.raw.grid_dims]
    dev = torch.device("cuda", 0)
    d_kind = torch.from_numpy(kind.astype(np.int32)).to(dev)
    d_fill = torch.from_numpy(fill).to(dev)
    d_div = torch.from_numpy(div).to(dev)
    p_hi = torch.zeros(kind.size, dtype=torch.float32, device=dev)
    p_lo = torch.zeros(kind.size, dtype=torch.float32, device=dev)
    dx = F(s.raw.bounds_size[0]) / F(g[0])
    free_after_first = None
    for call in range(2):
        p_hi.zero_()
        p_lo.zero_()
        torch.cuda.synchronize()
        pairs, res = C.c_uint32(), C.c_double()
        engine.call("cs_pressure_solve_noalloc", g[0], g[1], g[2], C.c_float(dx), C.c_float(dt),
                    C.c_float(omega), C.c_float(1e-5), 2000, int(s.raw.check_every), C.c_void_p(d_kind.data_ptr()),
                    C.c_void_p(d_fill.data_ptr()), C.c_void_p(d_div.data_ptr()), C.c_void_p(p_hi.data_ptr()),
                    C.c_void_p(p_lo.data_ptr()), None, C.byref(pairs), C.byref(res))
        torch.cuda.synchronize()
        if call == 0:
            free_after_first = torch.cuda.mem_get_info(dev)[0]
        else:
            assert torch.cuda.mem_get_info(dev)[0] == free_after_first, "the second call allocated device memory"
        got = p_hi.cpu().numpy()
        err = np.linalg.norm(got.astype(np.float64) - want) / np.linalg.norm(want.astype(np.float64))
        assert err <= 1e-5, (call, err)
        assert res.value <= 1e-5
        assert abs(int(pairs.value) - int(mb.last_sweeps)) <= 10, (pairs.value, mb.last_sweeps)


def test_noalloc_solve_with_solid_and_bed_faces(engine):
    """V60 pour at 32^3 (cone wall: solid faces; coffee bed: bed-coupled faces of
    weight 1): the allocation-free solve on the fill and divergence classify wrote
    matches the engine's solve of the same state."""
    pytest.importorskip("torch")
    s = scenes.c2_v60(engine, grid=32, max_particles=60000)
    r = s.raw
    r.warm_start = _ffi.CS_WARM_NONE
    r.rbgs_omega = 1.9
    a, b = MpmSim3D(s, engine), MpmSim3D(s, engine)
    assert scenes.populate_c2(a) == scenes.populate_c2(b) > 0
    for _ in range(4):
        a.step_substep(scenes.C2_DT)
        b.step_substep(scenes.C2_DT)
    a.step_substep_partial(scenes.C2_DT, 7)   # through classify: solver inputs
    b.step_substep_partial(scenes.C2_DT, 8)   # through the pressure solve: reference output
    kind = a.read_cell_kind()
    assert (kind == 3).sum() > 0 and (kind == 4).sum() > 0  # bed-coupled and solid cells
    fill, div = a.read_solver_inputs()
    want = b.read_pressure()
    mb = b.latest_metrics()
    assert mb.last_sweeps > 0 and np.abs(want).max() > 0
    _solve_twice_and_compare(engine, s, kind, fill, div, want, mb, scenes.C2_DT, omega=1.9)
    a.close()
    b.close()


def test_noalloc_rejects_grids_beyond_its_scratch(engine):
    pairs, res = C.c_uint32(), C.c_double()
    rc = engine.lib.cs_pressure_solve_noalloc(65, 8, 8, C.c_float(0.1), C.c_float(1e-3), C.c_float(1.0),
                                              C.c_float(1e-5), 10, 10, C.c_void_p(16), C.c_void_p(16),
                                              C.c_void_p(16), C.c_void_p(16), C.c_void_p(16), None,
                                              C.byref(pairs), C.byref(res))
    assert rc == 2  # CS_ERR_CAPACITY, before any device work
    assert b"64 cells per side" in engine.lib.cs_last_error_string()
