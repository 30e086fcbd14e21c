"""The checker itself: the C restatement (oracle/liboracle.so) reproduces
the reference bit for bit on the committed golden vectors (made from the
reference by tests/golden/make_golden.py), and, where the reference tree is
built here (oracle/_ref), on live runs of the reference."""
import json
import os

import numpy as np
import pytest

from baccolonygrowth_b200 import _abi, params
from baccolonygrowth_b200.colony import workload_colony, depleted_wall

import checkers as ck

F = _abi.FIELDS
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_params(js):
    p = _abi.Params()
    for k, v in json.loads(str(js)).items():
        setattr(p, k, v)
    return p


def unpack(counts, flat):
    out, o = [], 0
    for c in counts:
        out.append(flat[o:o + c])
        o += c
    return out


def test_oracle_matches_golden_mechanics():
    g = np.load(os.path.join(GOLD, "mech_small.npz"))
    p = load_params(g["params"])
    orc = ck.Oracle(p, seed=12345)
    orc.load(g["cells_in"])
    orc.update_height()
    orc.set_field(F["ENV_GROWTH1"], np.full(p.box_x * p.box_z, 0.9))
    orc.rebuild()
    for f, key in (("HEIGHT", "height"), ("NORMAL_X", "normal_x"), ("NORMAL_Z", "normal_z"), ("WALL", "wall")):
        assert np.array_equal(orc.field(F[f]), g[key]), f
    nb = orc.neighbours()
    want = unpack(g["nbr0_counts"], g["nbr0_flat"])
    assert all(np.array_equal(a, b) for a, b in zip(nb, want))
    divs = unpack(g["div_counts"], g["div_flat"])
    lins = unpack(g["lineage_counts"], g["lineage"])
    t = 0.0
    for s in range(len(g["rand_calls"])):
        ids, calls, lin = orc.step(p.dt, t)
        t += p.dt
        assert calls == g["rand_calls"][s]
        assert np.array_equal(ids, divs[s])
        assert np.array_equal(lin.reshape(-1), lins[s])
    assert orc.cells().tobytes() == g["cells_out"].tobytes()
    nb = orc.neighbours()
    want = unpack(g["nbr_counts"], g["nbr_flat"])
    assert all(np.array_equal(a, b) for a, b in zip(nb, want))


def test_oracle_matches_golden_fields():
    g = np.load(os.path.join(GOLD, "fields_small.npz"))
    p = load_params(g["params"])
    orc = ck.Oracle(p, seed=12345)
    orc.load(g["cells_in"])
    orc.update_density()
    assert tuple(orc.bbox()) == tuple(g["bbox"])
    # BoxAverage writes only inside the bounding box; the reference leaves
    # the rest of its scratch array uninitialised
    minx, maxx, maxz = (int(v) for v in g["bbox"])
    box = np.zeros((p.box_x, p.box_z), dtype=bool)
    box[minx:maxx, :maxz] = True
    box = box.reshape(-1)
    for f in ("ROUGH_DENSITY", "INSIDE", "HEIGHT", "NORMAL_X", "NORMAL_Z", "WALL"):
        assert np.array_equal(orc.field(F[f]), g["d_" + f]), f
    for f in ("DENSITY_SHIFT", "DENSITY"):
        assert np.array_equal(orc.field(F[f])[box], g["d_" + f][box]), f
    rows = depleted_wall(p, orc.field(F["INSIDE"]))
    for name, v in zip(("WALLF_CARBON", "WALLF_OXYGEN", "WALLF_ACETATE"), rows):
        orc.set_field(F[name], v, 0)
    orc.mg_solve(3, p.mg_dt)
    assert np.ptp(orc.field(F["MG_SOL_CARBON"], 0)) > 0
    for l in range(p.mg_levels):
        for sp in ("CARBON", "OXYGEN", "ACETATE"):
            assert np.array_equal(orc.field(F["MG_SOL_" + sp], l), g["mg_%d_%s" % (l, sp)]), (l, sp)
    orc.nutrient_update(1)
    for f in ("ENV_CARBON", "ENV_WASTE", "ENV_OXYGEN", "ENV_ACETATE", "ENV_GROWTH1", "ENV_PH",
              "OLDENV_CARBON", "OLDENV_WASTE", "OLDENV_OXYGEN", "OLDENV_ACETATE"):
        assert np.array_equal(orc.field(F[f]), g["n_" + f]), f
    X = p.box_x
    for l in range(p.max_levels_mg):
        keep = np.ones(X, dtype=bool)
        if l > 0:   # the reference reads uninitialised locals for these points
            keep[X // 4:X * 3 // 4] = False
        for f in ("WALLF_CARBON", "WALLF_WASTE", "WALLF_OXYGEN", "WALLF_ACETATE", "OLDWALLF_CARBON"):
            assert np.array_equal(orc.field(F[f], l)[keep], g["n_%s_%d" % (f, l)][keep]), (f, l)
        for sp in ("CARBON", "OXYGEN", "ACETATE"):
            assert np.array_equal(orc.field(F["MG_SOL_" + sp], l), g["n_mg_%d_%s" % (l, sp)]), (l, sp)


needs_ref = pytest.mark.skipif(not ck.have_ref(), reason="reference harness (oracle/_ref) not built here")


@needs_ref
def test_oracle_matches_reference_live_loop():
    """The whole while-loop body (Simulation.cpp:256-430) including the
    UpdateFlag field block, with a short nutrient schedule."""
    p = params.workload_params("small_4k")
    p.solves_per_update = 1
    p.update_time = 0.0004   # field update every 4 steps
    cells = workload_colony("small_4k", n=1024)
    ref = ck.Reference(p, seed=777)
    orc = ck.Oracle(p, seed=777)
    ref.load(cells)
    orc.load(cells)
    # the loop body's field / neighbour / mechanics sequence, one solve per update
    ref.initial_fields(False)
    orc.initial_fields(False)
    for s in range(6):
        ref.update_density(); orc.update_density()
        ref.nutrient_update(1); orc.nutrient_update(1)
        ref.rebuild(); orc.rebuild()
        ref.update_height(); orc.update_height()
        r1, r2 = ref.step(p.dt, 0.0001 * s), orc.step(p.dt, 0.0001 * s)
        assert r1[1] == r2[1] and np.array_equal(r1[2], r2[2])
    assert ref.cells().tobytes() == orc.cells().tobytes()
    # outside the bounding box BoxAverage leaves the reference's scratch
    # array uninitialised; compare inside it
    minx, maxx, maxz = ref.bbox()
    box = np.zeros((p.box_x, p.box_z), dtype=bool)
    box[minx:maxx, :maxz] = True
    box = box.reshape(-1)
    for f in ("ENV_CARBON", "ENV_GROWTH1", "DENSITY_SHIFT", "HEIGHT"):
        a, b = ref.field(F[f]), orc.field(F[f])
        if a.size == box.size:
            a, b = a[box], b[box]
        assert np.array_equal(a, b), f


@needs_ref
def test_oracle_mean_stress_matches_reference():
    p = params.workload_params("small_4k")
    cells = workload_colony("small_4k", n=1024)
    ref, orc = ck.Reference(p, seed=99), ck.Oracle(p, seed=99)
    for m in (ref, orc):
        m.load(cells)
        m.update_height()
        m.rebuild()
        m.step(p.dt, 0.0)     # some contacts and velocities
    a, b = ref.mean_stress(), orc.mean_stress()
    assert a[2] == b[2]
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_restart_roundtrip(tmp_path):
    import ctypes
    lib = _abi.load()
    cells = workload_colony("small_4k", n=300)
    path = str(tmp_path / "8.txt").encode()
    assert lib.bcg_save_restart(path, 9.001, 1e-4, _abi.ptr(cells), len(cells)) == 0
    out = np.zeros(400, dtype=_abi.CELL_DTYPE)
    t, dt, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
    assert lib.bcg_load_restart(path, ctypes.byref(t), ctypes.byref(dt), _abi.ptr(out), 400, ctypes.byref(n)) == 0
    assert (t.value, dt.value, n.value) == (9.001, 1e-4, 300)
    assert out[:300].tobytes() == cells.tobytes()
    # the file is exactly the reference's SaveCells layout: two doubles then 208-byte records
    raw = open(path.decode(), "rb").read()
    assert len(raw) == 16 + 208 * 300
    assert np.frombuffer(raw[:16], dtype=np.float64).tolist() == [9.001, 1e-4]


def test_oracle_inputs_equal_library_inputs():
    """The benchmark's reference arm builds its workload with the oracle's
    restatement of the parameter defaults and of the synthetic colony (so
    that it never loads the CUDA library); both must equal the library's
    byte for byte (host code, no GPU needed)."""
    entries = ck.oracle_param_entries()
    for name in params.WORKLOADS:
        a = params.workload_params(name)
        b = params.workload_params(name, entries=entries)
        assert bytes(a) == bytes(b), name
    for name, n in (("small_4k", 4096), ("scale_262k", 20000), ("mixed_1m", 30000)):
        a = workload_colony(name, n=n)
        b = workload_colony(name, n=n, entry=ck.oracle_synth_entry())
        assert a.tobytes() == b.tobytes(), name
    # a denser dome, and an over-packed one that both reject
    from baccolonygrowth_b200.colony import synth_colony
    w, h = params.dome_size(2000, 0.1, 0.6)
    a = synth_colony(2000, w, h, seed=99, div_phase_spread=0.5)
    b = synth_colony(2000, w, h, seed=99, div_phase_spread=0.5, entry=ck.oracle_synth_entry())
    assert len(a) == 2000 and a.tobytes() == b.tobytes()
    w, h = params.dome_size(2000, 0.1, 0.8)
    for entry in (None, ck.oracle_synth_entry()):
        with pytest.raises(_abi.BcgError):
            synth_colony(2000, w, h, seed=99, entry=entry)


def legacy_masks(p):
    """Points of the legacy explicit agar solver that the reference defines:
    on levels > 0 the agar points with BoxX/4 <= x < 3 BoxX/4, z < BoxZAgar/2
    and the wall points with BoxX/4 <= x < 3 BoxX/4 read second differences
    that are never initialised (Nutrients.cpp:509-803); nothing else reads
    them."""
    X, ZA = p.box_x, p.box_z_agar
    agar, wall = [], []
    for l in range(p.max_levels_mg):
        a = np.ones((X, ZA), dtype=bool)
        w = np.ones(X, dtype=bool)
        if l > 0:
            a[X // 4:3 * X // 4, :ZA // 2] = False
            w[X // 4:3 * X // 4] = False
        agar.append(a.reshape(-1))
        wall.append(w)
    return agar, wall


def legacy_pair(n=4096):
    p = params.workload_params("small_4k")
    cells = workload_colony("small_4k", n=n)
    models = [ck.Oracle(p, seed=12345), ck.Reference(p, seed=12345)]
    for m in models:
        m.load(cells)
        m.update_density()
    rows = depleted_wall(p, models[0].field(F["INSIDE"]))
    for m in models:
        for name, v in zip(("WALLF_CARBON", "WALLF_OXYGEN", "WALLF_ACETATE"), rows):
            m.set_field(F[name], v, 0)
            m.set_field(F["OLD" + name], v, 0)
    return p, models


def legacy_compare(p, a, b):
    agar, wall = legacy_masks(p)
    for f in ("ENV_CARBON", "ENV_WASTE", "ENV_OXYGEN", "ENV_ACETATE", "OLDENV_CARBON", "OLDENV_ACETATE"):
        assert np.array_equal(a.field(F[f]), b.field(F[f])), f
    for l in range(p.max_levels_mg):
        for sp in ("CARBON", "OXYGEN", "ACETATE"):
            f = "AGARF_" + sp
            assert np.array_equal(a.field(F[f], l)[agar[l]], b.field(F[f], l)[agar[l]]), (f, l)
            for f in ("WALLF_" + sp, "OLDWALLF_" + sp):
                assert np.array_equal(a.field(F[f], l)[wall[l]], b.field(F[f], l)[wall[l]]), (f, l)


@needs_ref
@pytest.mark.parametrize("iters", [7, 30])
def test_oracle_legacy_env_update_matches_reference(iters):
    """UpdateEnvArray_OxygenAcetate (the legacy explicit colony + wall + agar
    iterations) for a fixed count: the restatement equals the reference bit
    for bit at every point the reference defines."""
    p, (orc, ref) = legacy_pair()
    assert orc.legacy_env_update(iters) == ref.legacy_env_update(iters) == iters
    legacy_compare(p, orc, ref)
    # the agar moved (the wall under the colony is depleted)
    assert np.abs(orc.field(F["AGARF_CARBON"], 0) - p.max_carbon).max() > 0


@needs_ref
def test_oracle_legacy_depletion_matches_reference():
    """nutrientDepletionAgar_OxygenAcetate after a few legacy iterations:
    restriction to the coarsest level, its explicit steps, interpolation
    back; bit for bit at the defined points."""
    p, (orc, ref) = legacy_pair()
    orc.legacy_env_update(5)
    ref.legacy_env_update(5)
    n = orc.legacy_depletion()
    assert n == ref.legacy_depletion() and n > 100
    legacy_compare(p, orc, ref)
