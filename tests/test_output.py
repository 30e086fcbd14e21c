"""Output-step files in the reference's formats: bcg_write_output, the host
half of the output writer (needs no GPU).

- Golden: the committed output step (tests/golden/output_format.npz, made
  by the reference's own writers from seeded arbitrary values) comes out of
  bcg_write_output with the same bytes in all 17 files.
- Live, where the reference is built (oracle/_ref): fresh random steps, a
  physical step (after deposition, a nutrient update and mean_stress) and
  the initial block, written through the reference's writers and through
  bcg_write_output from the same values, byte for byte.
- The directory tree, append mode, thread count and the BCG_E_IO error.
"""
import ctypes
import json
import os

import numpy as np
import pytest

from baccolonygrowth_b200 import _abi, output, params
from baccolonygrowth_b200.colony import workload_colony, depleted_wall

import checkers as ck
import output_ref as orf

F = _abi.FIELDS
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "output_format.npz")
need_ref = pytest.mark.skipif(not ck.have_ref(), reason="oracle/_ref (the compiled reference) is not built")


def golden_step():
    g = np.load(GOLD)
    p = _abi.Params()
    for k, v in json.loads(str(g["params"])).items():
        setattr(p, k, v)
    L = p.max_levels_mg
    agar = []
    for l in range(L):
        agar += [g["agar"][l, 0], g["agar"][l, 1], None, g["agar"][l, 2]]
    d = output.StepData(p, float(g["t"]), float(g["dt"]), cells=g["cells"], force=g["force"], force_stride=5,
                        restart=g["restart"], density=g["density"], env=list(g["env"]), agar=agar,
                        wall=[g["wall"][l, m] for l in range(L) for m in range(4)])
    files = {name: g["file_" + name].tobytes() for name in orf.TREE}
    return int(g["step"]), d, files


def write_both_phases(directory, step, d, threads=0):
    output.write_output(directory, step, output.OUT_CELLS, d, threads=threads)
    output.write_output(directory, step, output.OUT_FIELDS, d, threads=threads)


def assert_same_tree(got, want):
    for name in orf.TREE:
        assert got[name] is not None, name
        assert got[name] == want[name], name


def test_golden_output_format(tmp_path):
    step, d, files = golden_step()
    write_both_phases(tmp_path, step, d)
    assert_same_tree(orf.read_tree(tmp_path, step), files)
    # six files carry data, the other eleven are created empty
    assert sum(1 for b in files.values() if b) == 6


def test_thread_count_does_not_change_bytes(tmp_path):
    step, d, files = golden_step()
    for th in (1, 3, 16):
        write_both_phases(tmp_path / str(th), step, d, threads=th)
        assert_same_tree(orf.read_tree(tmp_path / str(th), step), files)


def test_tree_and_append(tmp_path):
    step, d, files = golden_step()
    write_both_phases(tmp_path, step, d)
    assert sorted(os.listdir(tmp_path)) == sorted(orf.TREE)
    # append mode: CreateOutputFiles opens Cells for append, the rest anew
    output.write_output(tmp_path, step, output.OUT_CELLS, d, append=True)
    got = orf.read_tree(tmp_path, step)
    assert got["Cells"] == files["Cells"] * 2
    assert got["Density"] == b"" and got["Restart"] == b""
    output.write_output(tmp_path, step, output.OUT_FIELDS, d)
    got = orf.read_tree(tmp_path, step)
    assert got["Density"] == files["Density"] and got["Restart"] == files["Restart"]


def test_empty_colony_and_empty_restart(tmp_path):
    step, d, files = golden_step()
    e = output.StepData(d.p, d.t, d.dt, cells=d.cells[:0], force=d.force[:0], restart=None,
                        density=d.density, env=d.env, agar=d.agar, wall=d.wall)
    write_both_phases(tmp_path, step, e)
    got = orf.read_tree(tmp_path, step)
    assert got["Cells"] == b"" and got["Restart"] == b""
    assert got["Environment"] == files["Environment"]
    z = output.StepData(d.p, d.t, d.dt, cells=d.cells[:0], force=d.force[:0], restart=d.restart[:0],
                        density=d.density, env=d.env, agar=d.agar, wall=d.wall)
    output.write_output(tmp_path, step, output.OUT_FIELDS, z)
    # SaveCells with no cells still writes t and dt
    assert orf.read_tree(tmp_path, step)["Restart"] == np.array([d.t, d.dt]).tobytes()


def test_unwritable_directory_is_an_io_error(tmp_path):
    step, d, _ = golden_step()
    blocker = tmp_path / "file"
    blocker.write_text("x")
    with pytest.raises(_abi.BcgError) as e:
        write_both_phases(blocker / "out", step, d)
    assert e.value.code == _abi.E_IO


@need_ref
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_live_random_steps_match_reference_writers(tmp_path, seed):
    p, d = orf.random_step(seed, n=200 + 50 * seed)
    ref = ck.Reference(p, seed=12345)
    orf.reference_tree(ref, tmp_path / "ref", 9, d)
    write_both_phases(tmp_path / "b200", 9, d)
    assert_same_tree(orf.read_tree(tmp_path / "b200", 9), orf.read_tree(tmp_path / "ref", 9))


def physical_reference(n=512):
    p = params.workload_params("small_4k")
    ref = ck.Reference(p, seed=12345)
    ref.load(workload_colony("small_4k", n=n))
    ref.update_density()
    rows = depleted_wall(p, ref.field(F["INSIDE"]))
    for name, v in zip(("WALLF_CARBON", "WALLF_OXYGEN", "WALLF_ACETATE"), rows):
        ref.set_field(F[name], v, 0)
    ref.nutrient_update(1)
    ref.update_height()
    ref.rebuild()
    return p, ref


def reference_fields(ref, p):
    env = [ref.field(F[m]) for m in output.ENV_MEMBERS]
    agar, wall = [], []
    for l in range(p.max_levels_mg):
        agar += [None if m is None else ref.field(F[m], l) for m in output.AGAR_MEMBERS]
        wall += [ref.field(F[m], l) for m in output.WALL_MEMBERS]
    return dict(density=ref.field(F["DENSITY_SHIFT"]), env=env, agar=agar, wall=wall)


@need_ref
def test_live_output_step_matches_reference(tmp_path):
    """Simulation.cpp:316-372 on a physical state: the reference computes
    mean_stress itself; bcg_write_output gets the same values."""
    p, ref = physical_reference()
    t, dt, step = 1.25, p.dt, 3
    old = ref.cells()
    stress, _, calls = ref.mean_stress()
    assert ref.output_cells(tmp_path / "ref", step, t) == calls
    ids = np.zeros(len(old), dtype=np.int32)
    ref._move_grow(dt, ids, ctypes.c_longlong())
    new = ref.new_cells()
    ref.output_fields(t, dt)
    d = output.StepData(p, t, dt, cells=old, force=stress, force_stride=5, restart=new, **reference_fields(ref, p))
    write_both_phases(tmp_path / "b200", step, d)
    got, want = orf.read_tree(tmp_path / "b200", step), orf.read_tree(tmp_path / "ref", step)
    assert_same_tree(got, want)
    # the 17 Environment members carry the colony's values, not defaults
    nz = [np.count_nonzero(a) for a in d.env]
    assert all(c > 0 for c in nz[:10] + nz[13:]), nz


@need_ref
def test_live_initial_block_matches_reference(tmp_path):
    """Simulation.cpp:185-244: F_surf_tension's force in the stress columns
    and an empty Restart file."""
    p, ref = physical_reference(300)
    t = 0.0
    ref.output_initial(tmp_path / "ref", t)
    d = output.StepData(p, t, 0.0, cells=ref.cells(), force=ref.surface_forces(), force_stride=3, restart=None,
                        **reference_fields(ref, p))
    write_both_phases(tmp_path / "b200", 0, d)
    got, want = orf.read_tree(tmp_path / "b200", 0), orf.read_tree(tmp_path / "ref", 0)
    assert want["Restart"] == b""
    assert_same_tree(got, want)


def test_writer_lineage_and_arguments_without_a_device(tmp_path):
    """The writer's host side: lineage lines in queue order, the lineage
    file truncated at creation (CreateOutputFileLineage opens it "w"), and
    its argument and directory errors.  No CUDA call is made."""
    lib = _abi.load()
    lin = tmp_path / "w" / "lineage" / "0.txt"
    lin.parent.mkdir(parents=True)
    lin.write_bytes(b"stale\n")
    w = output.Writer(tmp_path / "w", threads=2)
    assert lin.read_bytes() == b""
    w.lineage([[3, 10], [5, 11]])
    w.lineage(np.zeros((0, 2), dtype=np.int32))
    w.lineage([[0, 12]])
    assert w.wait() == _abi.OK
    assert lin.read_bytes() == b"3 10\n5 11\n0 12\n"
    assert w.close() == _abi.OK
    h = ctypes.c_void_p()
    blocker = tmp_path / "file"
    blocker.write_text("x")
    assert lib.bcg_writer_create(str(blocker / "out").encode(), 0, 1, 2, ctypes.byref(h)) == _abi.E_IO
    assert lib.bcg_writer_create(str(tmp_path / "v").encode(), 0, 1, 0, ctypes.byref(h)) == _abi.E_ARG
    step, d, _ = golden_step()
    with pytest.raises(_abi.BcgError) as e:
        output.write_output(tmp_path / "bad", step, 4, d)
    assert e.value.code == _abi.E_ARG
