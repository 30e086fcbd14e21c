"""Regenerate the golden vectors in this directory from the reference itself.

Runs the unmodified reference sources (oracle/_ref/libbcgref.so, built by
`make -C oracle ref` where the reference tree is mounted) at 1 thread with
srand(12345) on two seeded synthetic scenarios, and stores inputs and
outputs:

  mech_small.npz   1024 cells, GetHeight + smoothing, GrowthRate1 = 0.9,
                   full neighbour rebuild, 12 MoveCell/GrowCell + division
                   steps: per-step rand() draws, dividing ids and lineage,
                   the final cells and neighbour lists.
  fields_small.npz 2048 cells: the UpdateFlag deposition chain, the
                   level-0 wall rows depleted under the colony
                   (colony.depleted_wall), one Multigrid::solve (3
                   V-cycles), then one nutrient update with one solve +
                   200 sweeps.

  output_format.npz one output step of seeded arbitrary values (300 cells,
                   a 40 x 6 colony grid, 2 agar levels of 40 x 5) and the
                   17 files the reference's own writers (Output, SaveCells,
                   the Array2D/Array3D writers) make of it.

Usage:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from baccolonygrowth_b200 import _abi, params  # noqa: E402
from baccolonygrowth_b200.colony import workload_colony, depleted_wall  # noqa: E402
import checkers  # noqa: E402

F = _abi.FIELDS
SEED = 12345


def pack_lists(lists):
    counts = np.array([len(l) for l in lists], dtype=np.int32)
    flat = np.concatenate([np.asarray(l, dtype=np.int32) for l in lists]) if lists else np.zeros(0, np.int32)
    return counts, flat


def mech():
    p = params.workload_params("small_4k")
    cells = workload_colony("small_4k", n=1024, div_phase_spread=1.0)
    ref = checkers.Reference(p, seed=SEED)
    ref.load(cells)
    ref.update_height()
    ref.set_field(F["ENV_GROWTH1"], np.full(p.box_x * p.box_z, 0.9))
    ref.rebuild()
    c0, f0 = pack_lists(ref.neighbours())
    out = dict(params=json.dumps(p.as_dict()), cells_in=cells, nbr0_counts=c0, nbr0_flat=f0,
               height=ref.field(F["HEIGHT"]), normal_x=ref.field(F["NORMAL_X"]),
               normal_z=ref.field(F["NORMAL_Z"]), wall=ref.field(F["WALL"]))
    calls, divs, lins = [], [], []
    t = 0.0
    for s in range(12):
        ids, c, lin = ref.step(p.dt, t)
        t += p.dt
        calls.append(c)
        divs.append(ids)
        lins.append(lin)
    out["rand_calls"] = np.array(calls, dtype=np.int64)
    out["div_counts"], out["div_flat"] = pack_lists(divs)
    out["lineage"] = np.concatenate([l.reshape(-1) for l in lins]).astype(np.int32)
    out["lineage_counts"] = np.array([l.size for l in lins], dtype=np.int32)
    out["cells_out"] = ref.cells()
    out["nbr_counts"], out["nbr_flat"] = pack_lists(ref.neighbours())
    np.savez_compressed(os.path.join(HERE, "mech_small.npz"), **out)
    print("mech_small.npz: %d cells after %d steps, %d divisions" % (len(out["cells_out"]), len(calls), len(out["lineage"]) // 2))


def fields():
    p = params.workload_params("small_4k")
    cells = workload_colony("small_4k", n=2048)
    ref = checkers.Reference(p, seed=SEED)
    ref.load(cells)
    out = dict(params=json.dumps(p.as_dict()), cells_in=cells)
    ref.update_density()
    out["bbox"] = np.array(ref.bbox(), dtype=np.int32)
    for f in ("ROUGH_DENSITY", "INSIDE", "DENSITY_SHIFT", "DENSITY", "HEIGHT", "NORMAL_X", "NORMAL_Z", "WALL"):
        out["d_" + f] = ref.field(F[f])
    rows = depleted_wall(p, ref.field(F["INSIDE"]))
    for name, v in zip(("WALLF_CARBON", "WALLF_OXYGEN", "WALLF_ACETATE"), rows):
        ref.set_field(F[name], v, 0)
    ref.mg_solve(3, p.mg_dt)
    for l in range(p.mg_levels):
        for sp in ("CARBON", "OXYGEN", "ACETATE"):
            out["mg_%d_%s" % (l, sp)] = ref.field(F["MG_SOL_" + sp], l)
    ref.nutrient_update(1)
    for f in ("ENV_CARBON", "ENV_WASTE", "ENV_OXYGEN", "ENV_ACETATE", "ENV_GROWTH1", "ENV_PH",
              "OLDENV_CARBON", "OLDENV_WASTE", "OLDENV_OXYGEN", "OLDENV_ACETATE"):
        out["n_" + f] = ref.field(F[f])
    for l in range(p.max_levels_mg):
        for f in ("WALLF_CARBON", "WALLF_WASTE", "WALLF_OXYGEN", "WALLF_ACETATE", "OLDWALLF_CARBON"):
            out["n_%s_%d" % (f, l)] = ref.field(F[f], l)
        for sp in ("CARBON", "OXYGEN", "ACETATE"):
            out["n_mg_%d_%s" % (l, sp)] = ref.field(F["MG_SOL_" + sp], l)
    np.savez_compressed(os.path.join(HERE, "fields_small.npz"), **out)
    print("fields_small.npz: bbox", tuple(out["bbox"]))


def output_format():
    import tempfile
    import output_ref
    p, d = output_ref.random_step(20261203)
    ref = checkers.Reference(p, seed=SEED)
    step = 5
    with tempfile.TemporaryDirectory() as tmp:
        output_ref.reference_tree(ref, tmp, step, d)
        files = output_ref.read_tree(tmp, step)
    L = p.max_levels_mg
    out = dict(params=json.dumps(p.as_dict()), step=step, t=d.t, dt=d.dt, cells=d.cells, force=d.force,
               restart=d.restart, density=d.density, env=np.stack(d.env),
               agar=np.stack([a for a in d.agar if a is not None]).reshape(L, 3, -1),
               wall=np.stack(d.wall).reshape(L, 4, -1))
    for name, b in files.items():
        out["file_" + name] = np.frombuffer(b, dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "output_format.npz"), **out)
    print("output_format.npz: %d cells, %d bytes of files" % (len(d.cells), sum(len(b) for b in files.values())))


if __name__ == "__main__":
    if not checkers.have_ref():
        sys.exit("oracle/_ref/libbcgref.so is not built (make -C oracle ref)")
    which = sys.argv[1:] or ["mech", "fields", "output_format"]
    for name in which:
        globals()[name]()
