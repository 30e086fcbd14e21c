"""Output-step scenarios for the writer tests, and the reference side of
them (test infrastructure).

`random_step` builds one output step of seeded arbitrary values: cell
records and stress columns over many magnitudes and signs, and field planes
with zeros, signed zeros, integers and values from 1e-14 to 1e14, so that
every printf conversion of the reference's writers is exercised.
`reference_tree` writes a step through the reference's own writers
(oracle/_ref), `read_tree` reads an output directory back.
"""
import os
import re

import numpy as np

from baccolonygrowth_b200 import _abi, output, params

TREE = ("Cells", "Restart", "RoughDensity", "RoughDensity1", "RoughDensity2", "Density", "Density1", "Density2",
        "WallDensity", "WallDensity1", "WallDensity2", "RoughHeight", "Height", "Normal", "Environment",
        "AgarField", "WallField")


def tiny_params():
    """A 40 x 6 colony grid over 2 agar levels of 40 x 5."""
    p = params.workload_params("small_4k", max_cells=1024)
    p.box_x, p.box_z, p.box_z_agar, p.max_levels_mg, p.mg_levels = 40, 6, 5, 2, 2
    return p


def _values(rng, n):
    v = rng.standard_normal(n) * 10.0 ** rng.uniform(-14, 14, n)
    kind = rng.integers(0, 12, n)
    v[kind == 0] = 0.0
    v[kind == 1] = -0.0
    v[kind == 2] = np.round(v[kind == 2] * 1e-10)
    v[kind == 3] = rng.uniform(0, 10, (kind == 3).sum())
    return v


def random_cells(rng, n, p):
    c = np.zeros(n, dtype=_abi.CELL_DTYPE)
    half = p.box_x / 2 * p.box_length
    for end in ("p", "q"):
        c[end][:, 0] = rng.uniform(-0.9 * half, 0.9 * half, n)
        c[end][:, 2] = rng.uniform(0.2, (p.box_z - 1) * p.box_length, n)
    c["time_p"] = rng.uniform(0, 50, n)
    c["time_q"] = rng.uniform(0, 50, n)
    c["age_p"] = rng.integers(0, 30, n)
    c["age_q"] = rng.integers(0, 30, n)
    c["length"] = rng.uniform(1, 4, n)
    c["ldiv"] = rng.uniform(3, 5, n)
    c["radius"] = 0.5
    c["growth_rate"] = _values(rng, n)
    for f in ("velocity", "angular_velocity", "dyn_fric", "sta_fric"):
        c[f] = _values(rng, 3 * n).reshape(n, 3)
    c["type"] = rng.integers(1, 3, n)
    c["ancestor"] = rng.integers(0, 100000, n)
    return c


def random_step(seed, n=300):
    """(params, t, dt, StepData) of arbitrary values on the tiny grid."""
    rng = np.random.default_rng(seed)
    p = tiny_params()
    X, Z, Za, L = p.box_x, p.box_z, p.box_z_agar, p.max_levels_mg
    cells = random_cells(rng, n, p)
    stress = _values(rng, 5 * n)
    new = random_cells(rng, n, p)
    env = [_values(rng, X * Z) for _ in range(17)]
    agar, wall = [], []
    for _ in range(L):
        agar += [_values(rng, X * Za), _values(rng, X * Za), None, _values(rng, X * Za)]
        wall += [_values(rng, X) for _ in range(4)]
    t, dt = float(rng.uniform(0, 90)), 1e-4
    data = output.StepData(p, t, dt, cells=cells, force=stress, force_stride=5, restart=new,
                           density=_values(rng, X * Z), env=env, agar=agar, wall=wall)
    return p, data


def reference_tree(ref, directory, output_id, data):
    """Write `data` through the reference's writers: Output per cell with the
    given stress, SaveCells of the restart cells, the four field writers."""
    F = _abi.FIELDS
    p = data.p
    ref.load(data.cells)
    for m, a in zip(output.ENV_MEMBERS, data.env):
        ref.set_field(F[m], a)
    ref.set_field(F["DENSITY_SHIFT"], data.density)
    for l in range(p.max_levels_mg):
        for k, m in enumerate(output.AGAR_MEMBERS):
            if m is not None:
                ref.set_field(F[m], data.agar[4 * l + k], l)
        for k, m in enumerate(output.WALL_MEMBERS):
            ref.set_field(F[m], data.wall[4 * l + k], l)
    assert ref.output_cells_given(directory, output_id, data.t, data.force, data.force_stride) == 0
    ref.set_new_cells(data.restart)
    ref.output_fields(data.t, data.dt)


def read_tree(directory, output_id):
    """{Name: bytes} of a step's files, None for a missing one."""
    out = {}
    for name in TREE:
        path = os.path.join(directory, name, "%d.txt" % output_id)
        out[name] = open(path, "rb").read() if os.path.exists(path) else None
    return out


_NUM = re.compile(rb"^-?(?:\d+)\.(\d+)(?:E([+-]\d+))?$")


def text_close(a, b, rel=1e-9):
    """Compare two text files of the writers: the same lines, separators and
    token count; integer tokens equal; a number may differ from the other
    file's by one unit in its last printed digit (a value next to a rounding
    boundary) plus `rel` of the largest magnitude on its line (a line is one
    cell, or one row of one member of a field).  Returns the count of
    unequal numbers."""
    la, lb = a.split(b"\n"), b.split(b"\n")
    assert len(la) == len(lb), (len(la), len(lb))
    diff = 0
    for i, (x, y) in enumerate(zip(la, lb)):
        if x == y:
            continue
        tx, ty = re.split(rb"([ \t])", x), re.split(rb"([ \t])", y)
        assert len(tx) == len(ty), "line %d: %r / %r" % (i, x[:80], y[:80])
        scale = max((abs(float(s)) for s in tx if _NUM.match(s)), default=0.0)
        for s, u in zip(tx, ty):
            if s == u:
                continue
            m = _NUM.match(s)
            assert m is not None and _NUM.match(u) is not None, "line %d: %r / %r" % (i, s, u)
            ulp = 10.0 ** (int(m.group(2) or 0) - len(m.group(1)))
            fs, fu = float(s), float(u)
            assert abs(fs - fu) <= 1.0001 * ulp + rel * scale, "line %d: %r / %r" % (i, s, u)
            diff += 1
    return diff


_CELL_FLOATS = ("p", "q", "time_p", "time_q", "length", "ldiv", "radius", "growth_rate", "velocity",
                "angular_velocity", "dyn_fric", "sta_fric")


def restart_close(a, b, rel=1e-9):
    """Two Restart files: the same t, dt and record count; integer members
    equal, float members within `rel` of each member's largest magnitude."""
    assert len(a) == len(b)
    if not a:
        return
    assert a[:16] == b[:16]
    ca = np.frombuffer(a[16:], dtype=_abi.CELL_DTYPE)
    cb = np.frombuffer(b[16:], dtype=_abi.CELL_DTYPE)
    for f in ("age_p", "age_q", "type", "ancestor"):
        assert np.array_equal(ca[f], cb[f]), f
    for f in _CELL_FLOATS:
        x, y = ca[f].astype(np.float64), cb[f].astype(np.float64)
        scale = max(np.abs(x).max() if x.size else 0.0, 1e-300)
        assert np.abs(x - y).max(initial=0.0) <= rel * scale, f


def field_rows(text):
    """The rows of a field file as a float array (one row per non-empty
    line; each line holds Box_x values, each followed by a tab)."""
    rows = [l for l in text.split(b"\n") if l]
    return np.array([[float(v) for v in l.split(b"\t") if v] for l in rows])


def density_close(a, b, bbox, rel=1e-9):
    """Two Density files (rows z of Box_x values).  BoxAverage writes
    DensityShiftP only inside the bounding box (Compute.cpp:669-738); outside
    it the reference's array holds whatever its scratch memory held, which is
    not compared.  Inside the box the printed values agree within one unit
    of the last printed digit plus `rel` of the largest value; outside it
    `a` must be 0."""
    minx, maxx, maxz = bbox
    assert a.count(b"\n") == b.count(b"\n")
    ra, rb = field_rows(a), field_rows(b)
    assert ra.shape == rb.shape
    inside = np.zeros(ra.shape, dtype=bool)
    inside[:maxz, minx:maxx] = True
    scale = max(np.abs(rb[inside]).max(initial=0.0), 1e-300)
    ulp = 10.0 ** (np.floor(np.log10(np.maximum(np.abs(rb), 1e-300))) - 6)
    assert (np.abs(ra - rb)[inside] <= 1.0001 * ulp[inside] + rel * scale).all()
    assert (ra[~inside] == 0).all()
