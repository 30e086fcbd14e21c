"""Parity of the CUDA mechanics (binning, neighbour lists, MoveCell +
GrowCell, the division loop) with the C restatement in oracle/.

Bars (as stated for this path): neighbour sets and division events
bit-exact; forces/positions/velocities within 1e-10 relative in FP64.
"""
import numpy as np
import pytest

from baccolonygrowth_b200 import _abi, params
from baccolonygrowth_b200.colony import Colony, Rng, workload_colony

import checkers as ck

F = _abi.FIELDS
REL_TOL = 1e-10

pytestmark = pytest.mark.gpu


def setup_pair(n=4096, seed=12345, spread=1.0, growth=0.9, workload="small_4k", mutate=None, max_cells=None):
    p = params.workload_params(workload, max_cells=max_cells)
    cells = workload_colony(workload, n=n, div_phase_spread=spread)
    if mutate is not None:
        mutate(cells)
    orc = ck.Oracle(p, seed=seed)
    orc.load(cells)
    orc.update_height()
    orc.set_field(F["ENV_GROWTH1"], np.full(p.box_x * p.box_z, growth))
    orc.rebuild()
    col = Colony(p, cells)
    for f in ("HEIGHT", "NORMAL_X", "NORMAL_Z", "WALL", "ENV_GROWTH1"):
        col.set_field(f, orc.field(F[f]))
    # Normal.y is 0 on both sides (GetSurfaceNormal writes 0)
    rng = Rng(seed)
    for _ in range(p.box_x * p.box_y):   # the wall draws
        rng.next()
    return p, orc, col, rng


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(np.abs(a).max(), 1e-300)
    return np.abs(a - b).max() / scale


def assert_cells_close(ca, cb, tol=REL_TOL):
    assert len(ca) == len(cb)
    for name in ("p", "q", "length", "velocity", "angular_velocity"):
        e = rel_err(ca[name], cb[name])
        assert e <= tol, (name, e)
    for name in ("ldiv", "type", "ancestor", "age_p", "age_q", "time_p", "time_q"):
        assert np.array_equal(ca[name], cb[name]), name


def nbr_sets(lists):
    return [tuple(sorted(int(x) for x in l)) for l in lists]


def test_bins_and_neighbour_sets(gpu):
    p, orc, col, _ = setup_pair()
    col.rebuild_neighbours()
    a, b = nbr_sets(orc.neighbours()), nbr_sets(col.neighbours())
    assert a == b


def test_one_step_forces_and_growth(gpu):
    p, orc, col, rng = setup_pair()
    col.rebuild_neighbours()
    ids_o, calls_o, lin_o = orc.step(p.dt, 0.0)
    nd, calls = col.move_grow(p.dt)
    assert calls == calls_o
    assert np.array_equal(np.sort(ids_o), col.dividing(nd))
    rng.skip(calls)
    lin = col.divide(rng.frand(9 * nd), 0.0)
    assert np.array_equal(lin, lin_o)
    assert_cells_close(orc.cells(), col.cells())


def test_multi_step_divisions(gpu):
    p, orc, col, rng = setup_pair(spread=1.0)
    col.rebuild_neighbours()
    t = 0.0
    total = 0
    for s in range(40):
        _, calls_o, lin_o = orc.step(p.dt, t)
        lin = col.step(p.dt, t, rng)
        assert np.array_equal(lin, lin_o), s
        total += len(lin)
        t += p.dt
    assert total > 10
    assert_cells_close(orc.cells(), col.cells())
    assert nbr_sets(orc.neighbours()) == nbr_sets(col.neighbours())


def test_crowded_divisions(gpu):
    """Half of the cells divide in the same step, so most divisions have
    neighbouring divisions whose footprints overlap: the device runs them
    in groups, and the result must equal the reference's one-by-one loop
    (lineage, cells, neighbour sets), also over the following steps."""
    def mutate(cells):
        r = np.random.default_rng(5)
        pick = r.random(len(cells)) < 0.5
        cells["ldiv"][pick] = cells["length"][pick]     # divide after this step's growth
    p, orc, col, rng = setup_pair(mutate=mutate, max_cells=16384)
    col.rebuild_neighbours()
    t = 0.0
    for s in range(3):
        _, calls_o, lin_o = orc.step(p.dt, t)
        lin = col.step(p.dt, t, rng)
        assert np.array_equal(lin, lin_o), s
        if s == 0:
            assert len(lin) > 1000
        t += p.dt
    assert_cells_close(orc.cells(), col.cells())
    assert nbr_sets(orc.neighbours()) == nbr_sets(col.neighbours())


def test_neighbour_refresh_after_steps(gpu):
    p, orc, col, rng = setup_pair()
    col.rebuild_neighbours()
    t = 0.0
    for s in range(10):
        orc.step(p.dt, t)
        col.step(p.dt, t, rng)
        t += p.dt
    orc.rebuild()
    col.rebuild_neighbours()
    assert nbr_sets(orc.neighbours()) == nbr_sets(col.neighbours())


@pytest.mark.parametrize("group", [1, 2, 8])
def test_force_group_variants(gpu, group):
    lib = _abi.load()
    p, orc, col, rng = setup_pair(n=2048)
    col.rebuild_neighbours()
    assert lib.bcg_set_force_group(col.h, group) == 0
    _, calls_o, lin_o = orc.step(p.dt, 0.0)
    lin = col.step(p.dt, 0.0, rng)
    assert np.array_equal(lin, lin_o)
    assert_cells_close(orc.cells(), col.cells())


def test_out_of_grid_is_reported(gpu):
    p = params.workload_params("small_4k")
    cells = workload_colony("small_4k", n=256)
    cells["p"][5, 0] = 1e6   # far outside the box grid
    cells["q"][5, 0] = 1e6 + 2
    col = Colony(p, cells)
    # entries are asynchronous: the error surfaces at the next synchronising call
    with pytest.raises(_abi.BcgError) as e:
        col.rebuild_neighbours()
        col.synchronize()
    assert e.value.code == _abi.E_OUT_OF_GRID
    # the context stays usable after the error
    cells["p"][5, 0] = 0.0
    cells["q"][5, 0] = 2.0
    col.upload(cells)
    col.rebuild_neighbours()


def test_mean_stress(gpu):
    import ctypes
    p, orc, col, rng = setup_pair(n=2048)
    col.rebuild_neighbours()
    orc.step(p.dt, 0.0)
    col.step(p.dt, 0.0, rng)
    st_o, fn_o, calls_o = orc.mean_stress()
    n = col.n_cells()
    st = np.zeros(5 * n); fn = np.zeros(3 * n); calls = ctypes.c_int64()
    lib = _abi.load()
    assert lib.bcg_mean_stress(col.h, _abi.ptr(st, ctypes.c_double), _abi.ptr(fn, ctypes.c_double), ctypes.byref(calls)) == 0
    assert calls.value == calls_o
    assert rel_err(st_o.reshape(-1), st) <= 1e-10
    assert rel_err(fn_o.reshape(-1), fn) <= 1e-10


def test_autotune_keeps_state(gpu):
    """Tuning the lane group times trial launches on the live colony: the
    colony (records and per-cell outputs) is unchanged afterwards and the
    next step still matches the oracle."""
    p, orc, col, rng = setup_pair()
    col.rebuild_neighbours()
    before = col.cells().tobytes()
    g = col.autotune("FORCE_GROUP")
    assert g in (1, 2, 4, 8, 16)
    assert col.cells().tobytes() == before
    _, calls_o, lin_o = orc.step(p.dt, 0.0)
    lin = col.step(p.dt, 0.0, rng)
    assert np.array_equal(lin, lin_o)
    assert_cells_close(orc.cells(), col.cells())


def test_pair_geometry_fp32(gpu):
    """Contact search in FP32 on offsets local to cell i (bcg_set_pair_precision
    32), the branch's closest points, distance and forces in FP64: against
    the oracle (the reference's FP64 min_distance) the first step's
    velocities and angular velocities -- the forces and torques divided by
    the mass and inertia, times dt -- and the positions after 20 steps with
    divisions hold the FP64 bar of 1e-10 relative, with the same F_cw draws
    and lineage."""
    p, orc, col, rng = setup_pair()
    col.set_pair_precision(32)
    col.rebuild_neighbours()
    t = 0.0
    errs = []
    for s in range(20):
        _, calls_o, lin_o = orc.step(p.dt, t)
        lin = col.step(p.dt, t, rng)
        assert np.array_equal(lin, lin_o), s
        if s == 0:
            a, b = orc.cells(), col.cells()
            errs = [rel_err(a[k], b[k]) for k in ("velocity", "angular_velocity")]
        t += p.dt
    a, b = orc.cells(), col.cells()
    print("FP32 contact search: first-step velocity %.2e, angular velocity %.2e; after 20 steps p %.2e v %.2e"
          % (errs[0], errs[1], rel_err(a["p"], b["p"]), rel_err(a["velocity"], b["velocity"])))
    assert max(errs) <= REL_TOL, errs
    assert_cells_close(a, b)
