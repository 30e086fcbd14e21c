"""The benchmark step runs its agar solve on a second stream beside the
step's mechanics and divisions (bcg_sim_run with bcg_sim_set_step_mode(..,
0, v)).  The two touch disjoint data, so the result must be exactly what
the same work gives in sequence:

- the multigrid solution after N steps equals N plain bcg_mg_solve calls
  from the same state on a context without any mechanics;
- the cells and lineage equal a run whose steps solve nothing (mode
  (0, 0)), since the solve never feeds the mechanics in this cadence.
"""
import ctypes

import numpy as np
import pytest

from baccolonygrowth_b200 import _abi, params
from baccolonygrowth_b200.colony import Colony, depleted_wall, workload_colony

pytestmark = pytest.mark.gpu

STEPS = 6


def sim_with(lib, p, cells, seed, vcycles):
    sim = ctypes.c_void_p()
    _abi.check(lib.bcg_sim_create(ctypes.byref(p), _abi.ptr(cells), len(cells), seed, 0, ctypes.byref(sim)), "sim")
    _abi.check(lib.bcg_sim_set_step_mode(sim, 0, vcycles), "mode")
    ctx = lib.bcg_sim_ctx(sim)
    g = np.full(p.box_x * p.box_z, 0.9)
    _abi.check(lib.bcg_set_field(ctx, _abi.FIELDS["ENV_GROWTH1"], 0, _abi.ptr(g, ctypes.c_double), g.size), "g")
    _abi.check(lib.bcg_update_density(ctx), "density")
    deplete(lib, ctx, p)
    return sim, ctx


def deplete(lib, ctx, p):
    """depleted wall rows under the colony: a right-hand side for the solve"""
    rows = depleted_wall(p, read_field(lib, ctx, "INSIDE", 0))
    for name, v in zip(("WALLF_CARBON", "WALLF_OXYGEN", "WALLF_ACETATE"), rows):
        v = np.ascontiguousarray(v, dtype=np.float64)
        _abi.check(lib.bcg_set_field(ctx, _abi.FIELDS[name], 0, _abi.ptr(v, ctypes.c_double), v.size), name)


def read_field(lib, ctx, name, level):
    fid = _abi.FIELDS[name]
    n = ctypes.c_size_t()
    _abi.check(lib.bcg_field_size(ctx, fid, level, ctypes.byref(n)), "size")
    out = np.zeros(n.value, dtype=np.float64)
    _abi.check(lib.bcg_get_field(ctx, fid, level, _abi.ptr(out, ctypes.c_double), n.value), "get")
    return out


def mg_state(lib, ctx, p):
    return [read_field(lib, ctx, "MG_SOL_" + sp, l) for l in range(p.mg_levels)
            for sp in ("CARBON", "OXYGEN", "ACETATE")]


def cells_and_lineage(lib, sim, cap):
    ctx = lib.bcg_sim_ctx(sim)
    out = np.zeros(cap, dtype=_abi.CELL_DTYPE)
    got = ctypes.c_int()
    _abi.check(lib.bcg_download_cells(ctx, _abi.ptr(out), cap, ctypes.byref(got)), "download")
    lin = np.zeros(2 * cap, dtype=np.int32)
    nl = ctypes.c_int()
    _abi.check(lib.bcg_sim_lineage(sim, _abi.ptr(lin, ctypes.c_int), cap, ctypes.byref(nl)), "lineage")
    return out[:got.value].tobytes(), lin[:2 * nl.value].copy()


def test_overlapped_solve_equals_sequential(gpu):
    lib = _abi.load()
    p = params.workload_params("scale_262k")
    cells = np.ascontiguousarray(workload_colony("scale_262k", n=20000, seed=21))
    sim, ctx = sim_with(lib, p, cells, 21, 1)
    _abi.check(lib.bcg_sim_run(sim, STEPS), "run")
    got = mg_state(lib, ctx, p)
    cells_a, lin_a = cells_and_lineage(lib, sim, 2 * len(cells))
    lib.bcg_sim_destroy(sim)

    # the same solves in sequence, no mechanics
    col = Colony(p, cells)
    g = np.full(p.box_x * p.box_z, 0.9)
    col.set_field("ENV_GROWTH1", g)
    col.update_density()
    deplete(lib, col.h, p)
    for _ in range(STEPS):
        col.mg_solve(1)
    want = mg_state(lib, col.h, p)
    col.close()
    assert np.ptp(want[0]) > 0
    for a, b in zip(got, want):
        assert np.array_equal(a, b)

    # the same mechanics with no solve
    sim0, _ = sim_with(lib, p, cells, 21, 0)
    _abi.check(lib.bcg_sim_run(sim0, STEPS), "run")
    cells_b, lin_b = cells_and_lineage(lib, sim0, 2 * len(cells))
    lib.bcg_sim_destroy(sim0)
    assert cells_a == cells_b
    assert np.array_equal(lin_a, lin_b)
    assert len(lin_a) > 0


def test_timeline_marks_steps_without_changing_them(gpu):
    """bcg_timeline_*: every step of the benchmark cadence queues its seven
    marks in order; times rise along each stream, the step ends after its
    solve and before the next step starts; a run with the timeline equals
    one without, and a read empties the timeline."""
    lib = _abi.load()
    p = params.workload_params("scale_262k")
    cells = np.ascontiguousarray(workload_colony("scale_262k", n=20000, seed=21))
    sim, ctx = sim_with(lib, p, cells, 21, 1)
    _abi.check(lib.bcg_timeline_enable(ctx, 256), "timeline")
    _abi.check(lib.bcg_sim_run(sim, STEPS), "run")
    tags = np.zeros(256, dtype=np.int32)
    ms = np.zeros(256, dtype=np.float32)
    n = ctypes.c_int()
    _abi.check(lib.bcg_timeline_read(ctx, _abi.ptr(tags, ctypes.c_int), _abi.ptr(ms, ctypes.c_float), 256,
                                     ctypes.byref(n)), "read")
    assert n.value == 7 * STEPS
    assert list(tags[:n.value]) == [1, 2, 3, 4, 5, 6, 7] * STEPS
    t = ms[:n.value].reshape(STEPS, 7).astype(np.float64)
    main = t[:, [0, 3, 4, 5, 6]].ravel()
    assert np.all(np.diff(main) >= 0)
    assert np.all(np.diff(t[:, [1, 2]].ravel()) >= 0)
    assert np.all(t[:, 6] >= t[:, 2] - 1e-3)
    n2 = ctypes.c_int(-1)
    _abi.check(lib.bcg_timeline_read(ctx, _abi.ptr(tags, ctypes.c_int), _abi.ptr(ms, ctypes.c_float), 256,
                                     ctypes.byref(n2)), "read again")
    assert n2.value == 0
    _abi.check(lib.bcg_timeline_enable(ctx, 0), "stop")
    cells_a, lin_a = cells_and_lineage(lib, sim, 2 * len(cells))
    lib.bcg_sim_destroy(sim)

    sim0, _ = sim_with(lib, p, cells, 21, 1)
    _abi.check(lib.bcg_sim_run(sim0, STEPS), "run")
    cells_b, lin_b = cells_and_lineage(lib, sim0, 2 * len(cells))
    lib.bcg_sim_destroy(sim0)
    assert cells_a == cells_b
    assert np.array_equal(lin_a, lin_b)
