"""Parity at the sizes the benchmark runs, against the C restatement in
oracle/ (1-thread reference order):

- the whole 262,144-cell colony of the scale workload (2304 x 128 colony
  boxes, 2305 x 513 x 3 composite agar grid), growth and division on, for
  500 steps with the full neighbour rebuild every 100 steps (UpdateTime /
  dt): dividing cells, F_cw draw counts and lineage bit-exact every step;
  neighbour sets at the end bit-exact; positions, velocities and lengths
  within 1e-10 relative;
- the whole 1,048,576-cell colony of the benchmark workload (4608 x 200
  boxes, 4609 x 1025 x 3 composite agar grid) with the kernel shapes the
  autotuner picks for it: two mechanics steps, then the density chain and
  one Multigrid::solve (3 V-cycles) on the full grid, every level within
  the field tolerance (1e-12 relative);
- one complete field update of the small workload at the reference's
  schedule (266 solves of 3 V-cycles, 200 colony/wall sweeps after each:
  53,200 sweeps), where the colony sweeps multiply by reciprocals taken
  once instead of dividing per point: the drift stays within 1e-10.

The oracle takes minutes at these sizes (one CPU thread).
"""
import numpy as np
import pytest

from baccolonygrowth_b200 import _abi, params
from baccolonygrowth_b200.colony import Colony, depleted_wall, workload_colony

import checkers as ck
from test_gpu_mechanics import setup_pair, assert_cells_close, nbr_sets, rel_err

F = _abi.FIELDS
pytestmark = pytest.mark.gpu


def _step_both(p, orc, col, rng, t, s):
    ids_o, calls_o, lin_o = orc.step(p.dt, t)
    nd, calls = col.move_grow(p.dt)
    assert calls == calls_o, ("F_cw draws", s, calls, calls_o)
    assert np.array_equal(np.sort(ids_o), col.dividing(nd)), ("dividing cells", s)
    rng.skip(calls)
    lin = col.divide(rng.frand(9 * nd), t)
    assert np.array_equal(lin, lin_o), ("lineage", s)
    return len(lin)


def test_scale_262k_whole_colony_500_steps(gpu):
    p, orc, col, rng = setup_pair(n=262144, workload="scale_262k")
    assert col.n_cells() == 262144
    col.rebuild_neighbours()
    t = 0.0
    divisions = 0
    every = int(round(p.update_time / p.dt))
    for s in range(500):
        if s > 0 and s % every == 0:
            orc.rebuild()
            col.rebuild_neighbours()
        divisions += _step_both(p, orc, col, rng, t, s)
        t += p.dt
    assert divisions > 10000
    a, b = orc.cells(), col.cells()
    assert_cells_close(a, b)
    print("scale_262k: %d cells after 500 steps, %d divisions, max rel err p %.2e v %.2e"
          % (len(b), divisions, rel_err(a["p"], b["p"]), rel_err(a["velocity"], b["velocity"])))
    assert nbr_sets(orc.neighbours()) == nbr_sets(col.neighbours())


def test_bench_1m_colony_steps_and_solve(gpu):
    p, orc, col, rng = setup_pair(n=1048576, workload="mixed_1m")
    assert col.n_cells() == 1048576
    col.rebuild_neighbours()
    group = col.autotune("FORCE_GROUP")
    t = 0.0
    for s in range(2):
        _step_both(p, orc, col, rng, t, s)
        t += p.dt
    assert_cells_close(orc.cells(), col.cells())
    # the agar solve on the full composite grid, at the tuned smoother shape
    orc.update_density()
    col.update_density()
    assert orc.bbox() == col.bbox()
    rows = depleted_wall(p, orc.field(F["INSIDE"]))
    for name, v in zip(("WALLF_CARBON", "WALLF_OXYGEN", "WALLF_ACETATE"), rows):
        orc.set_field(F[name], v, 0)
        col.set_field(name, v, 0)
    warps = col.autotune("SMOOTHER")
    orc.mg_solve(3, p.mg_dt)
    col.mg_solve(3)
    worst = 0.0
    for l in range(p.mg_levels):
        for sp in ("CARBON", "OXYGEN", "ACETATE"):
            a, b = orc.field(F["MG_SOL_" + sp], l), col.field("MG_SOL_" + sp, l)
            e = rel_err(a, b)
            worst = max(worst, e)
            assert e <= 1e-12, (sp, l, e)
    for l in range(p.max_levels_mg):
        for sp in ("CARBON", "OXYGEN", "ACETATE"):
            assert rel_err(orc.field(F["WALLF_" + sp], l), col.field("WALLF_" + sp, l)) <= 1e-12, (sp, l)
    print("mixed_1m: force group %d, smoother warps %d, solve max rel err %.2e" % (group, warps, worst))


def test_full_nutrient_update_drift(gpu):
    p = params.workload_params("small_4k")
    cells = workload_colony("small_4k")
    orc = ck.Oracle(p, seed=12345)
    orc.load(cells)
    col = Colony(p, cells)
    col.set_field("WALL", orc.field(F["WALL"]))
    orc.update_density()
    col.update_density()
    rows = depleted_wall(p, orc.field(F["INSIDE"]))
    for name, v in zip(("WALLF_CARBON", "WALLF_OXYGEN", "WALLF_ACETATE"), rows):
        orc.set_field(F[name], v, 0)
        col.set_field(name, v, 0)
    orc.nutrient_update(0)          # n = int(3600 UpdateTime 740 / 100) = 266
    col.nutrient_update(0, -1)
    x0, x1, z1 = orc.bbox()
    m = np.zeros((p.box_x, p.box_z), dtype=bool)
    m[max(x0, 0):max(x1, 0), :min(z1, p.box_z)] = True
    m = m.reshape(-1)
    worst = {}
    for f in ("ENV_CARBON", "ENV_OXYGEN", "ENV_ACETATE", "ENV_WASTE", "ENV_GROWTH1", "ENV_GROWTH2",
              "OLDENV_CARBON", "OLDENV_OXYGEN", "OLDENV_ACETATE", "OLDENV_WASTE"):
        a, b = orc.field(F[f]), col.field(f)
        worst[f] = rel_err(a[m], b[m])
    for sp in ("CARBON", "OXYGEN", "ACETATE"):
        for l in range(p.max_levels_mg):
            worst["AGARF_%s_%d" % (sp, l)] = rel_err(orc.field(F["AGARF_" + sp], l), col.field("AGARF_" + sp, l))
    # the buffer solve's outputs (diagnostic: nothing reads them), inside the colony
    inside = (orc.field(F["INSIDE"]) > 0.5) & m
    diag = {f: rel_err(orc.field(F[f])[inside], col.field(f)[inside]) for f in ("ENV_PH", "ENV_HYDROX", "ENV_ACETIC")}
    print("full nutrient update (266 x [solve + 200 sweeps]), max rel err:",
          ", ".join("%s %.2e" % kv for kv in sorted(list(worst.items()) + list(diag.items()))))
    for k, v in worst.items():
        assert v <= 1e-10, (k, v)
    for k, v in diag.items():
        assert v <= 1e-9, (k, v)
