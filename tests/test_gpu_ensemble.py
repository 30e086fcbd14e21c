"""Ensembles (bcg_ensemble_*): colonies of different sizes and grids stepped
together must each end exactly where bcg_sim_run takes them alone (same
records, same lineage), since the ensemble only reorders when the host
waits."""
import ctypes

import numpy as np
import pytest

from baccolonygrowth_b200 import _abi, params
from baccolonygrowth_b200.colony import workload_colony

pytestmark = pytest.mark.gpu

MEMBERS = [("small_4k", 2048, 11), ("small_4k", 4096, 12), ("scale_262k", 20000, 13)]


def make_sim(lib, name, n, seed):
    p = params.workload_params(name)
    cells = np.ascontiguousarray(workload_colony(name, n=n, seed=seed))
    sim = ctypes.c_void_p()
    _abi.check(lib.bcg_sim_create(ctypes.byref(p), _abi.ptr(cells), len(cells), seed, 0, ctypes.byref(sim)), "sim")
    _abi.check(lib.bcg_sim_set_step_mode(sim, 0, 1), "mode")
    ctx = lib.bcg_sim_ctx(sim)
    g = np.full(p.box_x * p.box_z, 0.9)
    _abi.check(lib.bcg_set_field(ctx, _abi.FIELDS["ENV_GROWTH1"], 0, _abi.ptr(g, ctypes.c_double), g.size), "g")
    _abi.check(lib.bcg_update_density(ctx), "density")
    return sim, len(cells)


def state(lib, sim, cap):
    ctx = lib.bcg_sim_ctx(sim)
    out = np.zeros(cap, dtype=_abi.CELL_DTYPE)
    got = ctypes.c_int()
    _abi.check(lib.bcg_download_cells(ctx, _abi.ptr(out), cap, ctypes.byref(got)), "download")
    lin = np.zeros(2 * cap, dtype=np.int32)
    nl = ctypes.c_int()
    _abi.check(lib.bcg_sim_lineage(sim, _abi.ptr(lin, ctypes.c_int), cap, ctypes.byref(nl)), "lineage")
    return out[:got.value].tobytes(), lin[:2 * nl.value].copy()


def test_ensemble_equals_members_run_alone(gpu):
    lib = _abi.load()
    steps = 8
    alone = []
    for name, n, seed in MEMBERS:
        sim, n0 = make_sim(lib, name, n, seed)
        _abi.check(lib.bcg_sim_run(sim, steps), "run")
        alone.append(state(lib, sim, 2 * n0))
        lib.bcg_sim_destroy(sim)
    sims, caps = [], []
    for name, n, seed in MEMBERS:
        sim, n0 = make_sim(lib, name, n, seed)
        sims.append(sim); caps.append(2 * n0)
    arr = (ctypes.c_void_p * len(sims))(*[s.value for s in sims])
    ens = ctypes.c_void_p()
    _abi.check(lib.bcg_ensemble_create(arr, len(sims), ctypes.byref(ens)), "ensemble")
    _abi.check(lib.bcg_ensemble_run(ens, steps), "ensemble run")
    for sim, cap, (cells, lin) in zip(sims, caps, alone):
        c2, l2 = state(lib, sim, cap)
        assert c2 == cells
        assert np.array_equal(l2, lin)
    total_div = sum(len(l) // 2 for _, l in alone)
    assert total_div > 0
    lib.bcg_ensemble_destroy(ens)
    for s in sims:
        lib.bcg_sim_destroy(s)


def test_ensemble_members_match_oracle(gpu):
    """Each member of an ensemble against its own run of the C restatement
    (oracle/, pinned to the reference): the same seed, the same wall draws,
    the benchmark cadence (full neighbour rebuild at the first step, one
    1-V-cycle agar solve and one mechanics step per step).  Lineage
    bit-exact; cells within 1e-10 relative; agar solution within 1e-12."""
    import checkers as ck
    from test_gpu_mechanics import assert_cells_close, rel_err
    lib = _abi.load()
    steps = 8
    sims, caps, models = [], [], []
    for name, n, seed in MEMBERS:
        sim, n0 = make_sim(lib, name, n, seed)
        sims.append(sim); caps.append(2 * n0)
        p = params.workload_params(name)
        orc = ck.Oracle(p, seed=seed)
        orc.load(np.ascontiguousarray(workload_colony(name, n=n, seed=seed)))
        orc.set_field(_abi.FIELDS["ENV_GROWTH1"], np.full(p.box_x * p.box_z, 0.9))
        orc.update_density()
        models.append((p, orc))
    arr = (ctypes.c_void_p * len(sims))(*[s.value for s in sims])
    ens = ctypes.c_void_p()
    _abi.check(lib.bcg_ensemble_create(arr, len(sims), ctypes.byref(ens)), "ensemble")
    _abi.check(lib.bcg_ensemble_run(ens, steps), "ensemble run")
    total = 0
    for sim, cap, (p, orc) in zip(sims, caps, models):
        orc.rebuild()
        t = p.t0
        lins = []
        for s in range(steps):
            orc.mg_solve(1, p.mg_dt)
            _, _, lin = orc.step(p.dt, t)
            lins.append(lin.reshape(-1))
            t += p.dt
        lin_o = np.concatenate(lins) if lins else np.zeros(0, np.int32)
        cells, lin = state(lib, sim, cap)
        assert np.array_equal(lin, lin_o)
        total += len(lin) // 2
        got = np.frombuffer(cells, dtype=_abi.CELL_DTYPE)
        assert_cells_close(orc.cells(), got)
        ctx = lib.bcg_sim_ctx(sim)
        for sp in ("CARBON", "OXYGEN", "ACETATE"):
            f = "MG_SOL_" + sp
            a = orc.field(_abi.FIELDS[f], 0)
            b = np.zeros(a.size)
            _abi.check(lib.bcg_get_field(ctx, _abi.FIELDS[f], 0, _abi.ptr(b, ctypes.c_double), b.size), f)
            assert rel_err(a, b) <= 1e-12, (f, rel_err(a, b))
    assert total > 0
    lib.bcg_ensemble_destroy(ens)
    for s in sims:
        lib.bcg_sim_destroy(s)
