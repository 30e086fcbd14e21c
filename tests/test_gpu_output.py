"""The asynchronous output writer (bcg_writer) on the GPU.

- Its device snapshots give the same bytes as the synchronous calls
  (bcg_download_cells, bcg_mean_stress, bcg_get_field) handed to
  bcg_write_output, for the two halves of an output step taken around
  bcg_move_grow, over several steps in a row with one and two steps in
  flight.
- The initial block: F_surf_tension's forces, computed by the reference
  from the device's own cells, height and normals, give the same Cells file.
- bcg_sim_run with a writer against the reference's loop with its output
  block (oracle/_ref), from the same colony and seed, with an output every
  few steps: the same files (numbers within one unit of their last printed
  digit, fields within 1e-9 of the reference's, Restart records within 1e-9;
  Density only inside the bounding box, outside which the reference prints
  uninitialised memory), the same lineage file, and so the same rand()
  stream across the output steps' mean_stress draws.
"""
import ctypes
import os

import numpy as np
import pytest

from baccolonygrowth_b200 import _abi, output, params
from baccolonygrowth_b200.colony import Colony, Rng, workload_colony

import checkers as ck
import output_ref as orf

pytestmark = pytest.mark.gpu
F = _abi.FIELDS


def ready_colony(n=4096, seed=None):
    p = params.workload_params("small_4k")
    col = Colony(p, workload_colony("small_4k", n=n, seed=seed))
    col.update_density()
    col.deplete_wall()
    col.nutrient_update(1)
    col.update_height()
    col.rebuild_neighbours()
    return p, col


def sync_fields(col, p):
    env = [col.field(m) for m in output.ENV_MEMBERS]
    agar, wall = [], []
    for l in range(p.max_levels_mg):
        agar += [None if m is None else col.field(m, l) for m in output.AGAR_MEMBERS]
        wall += [col.field(m, l) for m in output.WALL_MEMBERS]
    return dict(density=col.field("DENSITY_SHIFT"), env=env, agar=agar, wall=wall)


def mean_stress(col):
    n = col.n_cells()
    st = np.zeros(5 * max(n, 1))
    fcw = ctypes.c_int64()
    _abi.check(col.lib.bcg_mean_stress(col.h, _abi.ptr(st, ctypes.c_double), None, ctypes.byref(fcw)), "mean_stress")
    return st[:5 * n], fcw.value


@pytest.mark.parametrize("max_pending", [1, 2])
def test_snapshots_match_synchronous_downloads(gpu, tmp_path, max_pending):
    """Every file but Restart against the synchronous calls, byte for byte;
    Restart (the moved, grown, undivided colony, which no synchronous call
    reads) against the colony after the division loop, whose cells that did
    not divide keep those records, and against the colony before the move,
    which it must differ from."""
    p, col = ready_colony()
    w = output.Writer(tmp_path / "async", threads=4, max_pending=max_pending)
    rng = Rng(7)
    t = 0.5
    after, before, mothers, times = [], [], [], []
    for k in range(3):
        times.append(t)
        old = col.cells()
        stress, fcw_sync = mean_stress(col)
        fcw = w.cells(col, k, t)
        assert fcw == fcw_sync
        nd, calls = col.move_grow(p.dt)
        w.fields(col, k, t, p.dt)
        d = output.StepData(p, t, p.dt, cells=old, force=stress, force_stride=5, restart=old[:0],
                            **sync_fields(col, p))
        output.write_output(tmp_path / "sync", k, output.OUT_CELLS, d)
        output.write_output(tmp_path / "sync", k, output.OUT_FIELDS, d)
        mothers.append(col.dividing(nd) if nd else np.zeros(0, np.int32))
        rng.skip(fcw + calls)
        col.divide(rng.frand(9 * nd) if nd else np.zeros(0, np.float32), t)
        before.append(old)
        after.append(col.cells())
        t += p.dt
    assert w.close() == _abi.OK
    for k in range(3):
        got, want = orf.read_tree(tmp_path / "async", k), orf.read_tree(tmp_path / "sync", k)
        for name in orf.TREE:
            if name != "Restart":
                assert got[name] == want[name], (k, name)
        assert len(got["Cells"].splitlines()) > 4000
        r = got["Restart"]
        assert r[:16] == np.array([times[k], p.dt]).tobytes()
        moved = np.frombuffer(r[16:], dtype=_abi.CELL_DTYPE)
        n = len(before[k])
        assert len(moved) == n
        keep = np.ones(n, dtype=bool)
        keep[mothers[k]] = False
        assert moved[keep].tobytes() == after[k][:n][keep].tobytes()
        assert not np.array_equal(moved["p"], before[k]["p"])


@pytest.mark.skipif(not ck.have_ref(), reason="oracle/_ref (the compiled reference) is not built")
def test_initial_block_forces_match_reference(gpu, tmp_path):
    p, col = ready_colony(2048)
    w = output.Writer(tmp_path / "async", threads=2)
    w.initial(col, 0.0)
    assert w.close() == _abi.OK
    got = orf.read_tree(tmp_path / "async", 0)
    assert got["Restart"] == b""
    # F_surf_tension on the device's cells, height and normals, by the reference
    ref = ck.Reference(p, seed=12345)
    cells = col.cells()
    ref.load(cells)
    for f in ("HEIGHT", "NORMAL_X", "NORMAL_Z"):
        ref.set_field(F[f], col.field(f))
    d = output.StepData(p, 0.0, 0.0, cells=cells, force=ref.surface_forces(), force_stride=3, restart=None,
                        **sync_fields(col, p))
    output.write_output(tmp_path / "sync", 0, output.OUT_CELLS | output.OUT_FIELDS, d)
    want = orf.read_tree(tmp_path / "sync", 0)
    for name in orf.TREE:
        assert got[name] == want[name], name


def fast_update_params(n_out):
    """small_4k with one agar solve per nutrient update (UpdateTime below dt,
    so an update every step) and an output every n_out steps."""
    p = params.workload_params("small_4k")
    p.update_time = 1.5 * p.mg_dt / (3600.0 * 740.0)
    p.output_time = n_out * p.dt
    return params.finalize(p)


@pytest.mark.skipif(not ck.have_ref(), reason="oracle/_ref (the compiled reference) is not built")
def test_sim_loop_output_matches_reference_loop(gpu, tmp_path):
    p = fast_update_params(3)
    cells = workload_colony("small_4k", n=1024)
    seed, steps = 4242, 10
    lib = _abi.load()
    sim = ctypes.c_void_p()
    _abi.check(lib.bcg_sim_create(ctypes.byref(p), _abi.ptr(cells), len(cells), seed, 1, ctypes.byref(sim)), "sim")
    w = output.Writer(tmp_path / "b200", threads=4)
    try:
        _abi.check(lib.bcg_sim_set_writer(sim, w.h, 1), "set_writer")
        _abi.check(lib.bcg_sim_run(sim, steps), "run")
        _abi.check(lib.bcg_sim_set_writer(sim, None, 0), "detach")
        assert w.close() == _abi.OK
        nl = ctypes.c_int()
        cap = 4 * len(cells)
        lin = np.zeros(2 * cap, dtype=np.int32)
        _abi.check(lib.bcg_sim_lineage(sim, _abi.ptr(lin, ctypes.c_int), cap, ctypes.byref(nl)), "lineage")
        lineage = lin[:2 * nl.value].reshape(-1, 2)
    finally:
        lib.bcg_sim_destroy(sim)

    ref = ck.Reference(p, seed=seed)
    ref.load(cells)
    ref.initial_fields(True)
    ref.output_initial(tmp_path / "ref", p.t0)
    bboxes = set()
    ref_lineage = []
    for _ in range(steps):
        ref_lineage.append(ref.loop_step_out(tmp_path / "ref"))
        bboxes.add(ref.bbox())
    assert len(bboxes) == 1            # one bounding box over the run
    bbox = bboxes.pop()
    ref_lineage = np.concatenate(ref_lineage) if ref_lineage else np.zeros((0, 2), np.int32)

    assert len(ref_lineage) > 0
    assert np.array_equal(lineage, ref_lineage)
    lines = open(os.path.join(tmp_path, "b200", "lineage", "0.txt"), "rb").read()
    assert lines == b"".join(b"%d %d\n" % (a, b) for a, b in ref_lineage)
    steps_written = sorted(int(f[:-4]) for f in os.listdir(tmp_path / "ref" / "Cells"))
    assert steps_written == sorted(int(f[:-4]) for f in os.listdir(tmp_path / "b200" / "Cells"))
    assert len(steps_written) >= 2
    for k in steps_written:
        got, want = orf.read_tree(tmp_path / "b200", k), orf.read_tree(tmp_path / "ref", k)
        for name in orf.TREE:
            assert (got[name] is None) == (want[name] is None), (k, name)
            if name == "Restart":
                orf.restart_close(got[name], want[name])
            elif name == "Density":
                orf.density_close(got[name], want[name], bbox)
            elif want[name]:
                orf.text_close(got[name], want[name]), (k, name)
            else:
                assert got[name] == b"", (k, name)
