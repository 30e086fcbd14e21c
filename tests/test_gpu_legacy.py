"""Parity of the legacy explicit agar solver on the GPU
(bcg_legacy_env_update, bcg_legacy_agar_depletion) with the C restatement
in oracle/, which tests/test_oracle.py pins bit for bit to the reference
(UpdateEnvArray_OxygenAcetate, nutrientDepletionAgar_OxygenAcetate,
Nutrients.cpp:45-197, 857-1074).

Tolerance: 1e-11 relative, as for the colony sweeps (they multiply by
1/BoxLength^2 and 1/g_s where the reference divides); the diagnostic
buffer-solve outputs 1e-9.  Points the reference leaves undefined (agar
and wall points of levels > 0 with BoxX/4 <= x < 3 BoxX/4, and agar z <
BoxZAgar/2) are excluded.
"""
import numpy as np
import pytest

from baccolonygrowth_b200 import _abi, params
from baccolonygrowth_b200.colony import Colony, depleted_wall, workload_colony

import checkers as ck
from test_oracle import legacy_masks

F = _abi.FIELDS
TOL = 1e-11
pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a); b = np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(a).max(), 1e-300)


def make(n=4096):
    p = params.workload_params("small_4k")
    cells = workload_colony("small_4k", n=n)
    orc = ck.Oracle(p, seed=12345)
    orc.load(cells)
    col = Colony(p, cells)
    col.set_field("WALL", orc.field(F["WALL"]))
    orc.update_density()
    col.update_density()
    rows = depleted_wall(p, orc.field(F["INSIDE"]))
    for name, v in zip(("WALLF_CARBON", "WALLF_OXYGEN", "WALLF_ACETATE"), rows):
        for pre in ("", "OLD"):
            orc.set_field(F[pre + name], v, 0)
            col.set_field(pre + name, v, 0)
    return p, orc, col


def compare(p, orc, col):
    x0, x1, z1 = orc.bbox()
    box = np.zeros((p.box_x, p.box_z), dtype=bool)
    box[max(x0, 0):x1 + 1, :min(z1 + 1, p.box_z)] = True
    box = box.reshape(-1)
    worst = 0.0
    for f in ("ENV_CARBON", "ENV_WASTE", "ENV_OXYGEN", "ENV_ACETATE", "ENV_GROWTH1", "OLDENV_CARBON",
              "OLDENV_ACETATE", "OLDENV_OXYGEN", "OLDENV_WASTE", "ENV_GR_CAR_AER", "ENV_Q_CAR_MNT"):
        e = rel(orc.field(F[f])[box], col.field(f)[box])
        worst = max(worst, e)
        assert e <= TOL, (f, e)
    inside = (orc.field(F["INSIDE"]) > 0.5) & box
    for f in ("ENV_PH", "ENV_HYDROX", "ENV_ACETIC", "ENV_BUFFER"):
        assert rel(orc.field(F[f])[inside], col.field(f)[inside]) <= 1e-9, f
    agar, wall = legacy_masks(p)
    for l in range(p.max_levels_mg):
        for sp in ("CARBON", "OXYGEN", "ACETATE"):
            f = "AGARF_" + sp
            e = rel(orc.field(F[f], l)[agar[l]], col.field(f, l)[agar[l]])
            worst = max(worst, e)
            assert e <= TOL, (f, l, e)
            for f in ("WALLF_" + sp, "OLDWALLF_" + sp):
                e = rel(orc.field(F[f], l)[wall[l]], col.field(f, l)[wall[l]])
                worst = max(worst, e)
                assert e <= TOL, (f, l, e)
    return worst


@pytest.mark.parametrize("iters", [1, 8, 31])
def test_legacy_env_update_fixed_iterations(gpu, iters):
    p, orc, col = make()
    assert orc.legacy_env_update(iters) == iters
    assert col.legacy_env_update(iters) == iters
    compare(p, orc, col)
    assert np.abs(col.field("AGARF_CARBON", 0) - p.max_carbon).max() > 0


def test_legacy_env_update_until_converged(gpu):
    """The stopping rule (count > min_iter and no point moved by more than
    ConvCrit) ends both at the same iteration."""
    p, orc, col = make(n=2048)
    n_o = orc.legacy_env_update(3000, min_iter=20, conv_crit=1e-2)
    n_g = col.legacy_env_update(3000, min_iter=20, conv_crit=1e-2)
    assert n_o == n_g, (n_o, n_g)
    assert 20 < n_g < 3000
    compare(p, orc, col)


def test_legacy_depletion(gpu):
    p, orc, col = make()
    orc.legacy_env_update(6)
    col.legacy_env_update(6)
    n = orc.legacy_depletion()
    assert col.legacy_depletion() == n > 100
    compare(p, orc, col)
