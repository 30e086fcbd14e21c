"""Edge cases of the device path, each against the C restatement or the
reference's error rules: an empty colony, a single cell, the MaxCells cut
of the division loop (Simulation.cpp:382, a silent break in the reference,
BCG_E_MAXCELLS here after the same divisions), and an overfull grid box
(UniformGrid.h:35)."""
import ctypes

import numpy as np
import pytest

from baccolonygrowth_b200 import _abi, params
from baccolonygrowth_b200.colony import Colony, workload_colony

from test_gpu_mechanics import setup_pair, assert_cells_close, nbr_sets

pytestmark = pytest.mark.gpu


def test_empty_colony(gpu):
    p = params.workload_params("small_4k")
    col = Colony(p, workload_colony("small_4k", n=16)[:0])
    assert col.n_cells() == 0
    col.rebuild_neighbours()
    nd, calls = col.move_grow(p.dt)
    assert nd == 0 and calls == 0
    assert len(col.divide(np.zeros(0, np.float32), 0.0)) == 0
    col.update_density()
    assert col.bbox() == (p.box_x - 5, 5, 5)        # the empty-colony box of k_bbox_finish
    col.mg_solve(1)
    stress = np.zeros(1)
    fcw = ctypes.c_int64(-1)
    _abi.check(col.lib.bcg_mean_stress(col.h, _abi.ptr(stress, ctypes.c_double), None, ctypes.byref(fcw)), "stress")
    assert fcw.value == 0
    col.synchronize()


def test_single_cell_matches_oracle(gpu):
    p, orc, col, rng = setup_pair(n=1)
    assert col.n_cells() == 1
    col.rebuild_neighbours()
    t = 0.0
    for s in range(5):
        _, calls_o, lin_o = orc.step(p.dt, t)
        lin = col.step(p.dt, t, rng)
        assert np.array_equal(lin, lin_o)
        t += p.dt
    assert_cells_close(orc.cells(), col.cells())


def test_maxcells_cut_matches_reference_order(gpu):
    """40 cells ready to divide, room for 5 more cells: the first 5 parents
    in ascending id divide, as the reference's loop does before it stops."""
    def mutate(cells):
        cells["ldiv"][:40] = cells["length"][:40]
    p, orc, col, rng = setup_pair(n=256, mutate=mutate, max_cells=261)
    col.rebuild_neighbours()
    _, _, lin_o = orc.step(p.dt, 0.0)
    assert len(lin_o) == 5
    with pytest.raises(_abi.BcgError) as e:
        col.step(p.dt, 0.0, rng)
    assert e.value.code == _abi.E_MAXCELLS
    assert col.n_cells() == 261
    assert_cells_close(orc.cells(), col.cells())
    assert nbr_sets(orc.neighbours()) == nbr_sets(col.neighbours())


def test_overfull_box_is_reported(gpu):
    p = params.workload_params("small_4k")
    cells = workload_colony("small_4k", n=p.max_cells_per_box + 5)
    # every centre into one grid box (the box spans box_length um)
    cells["p"][:, 0] = 0.1; cells["q"][:, 0] = 0.3
    cells["p"][:, 2] = 1.0; cells["q"][:, 2] = 1.2
    col = Colony(p, cells)
    with pytest.raises(_abi.BcgError) as e:
        col.rebuild_neighbours()
        col.synchronize()
    assert e.value.code == _abi.E_BOX_OVERFLOW


def test_upload_download_round_trip_in_chunks(gpu):
    """Records pass between host and device through the context's staging
    buffer, 131,072 at a time: a ragged count, a download into a smaller
    buffer and a second, shorter upload all come back byte for byte."""
    p = params.workload_params("scale_262k")
    cells = np.ascontiguousarray(workload_colony("scale_262k"))[:262144 - 12345]
    col = Colony(p, cells)
    assert col.n_cells() == len(cells)
    assert col.cells().tobytes() == cells.tobytes()
    part = np.zeros(140000, dtype=_abi.CELL_DTYPE)
    got = ctypes.c_int()
    _abi.check(col.lib.bcg_download_cells(col.h, _abi.ptr(part), len(part), ctypes.byref(got)), "download")
    assert got.value == len(cells)
    assert part.tobytes() == cells[:len(part)].tobytes()
    short = cells[1000:1000 + 131073]
    col.upload(short)
    assert col.cells().tobytes() == short.tobytes()
    col.close()
