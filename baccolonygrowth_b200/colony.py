"""Host-side Python API over the C ABI: synthetic colonies and a Colony
handle that owns one bcg_ctx (one colony resident on one GPU).

The methods mirror the reference calls they replace (Neighbours.cpp
getNeighbours, the MoveCell/GrowCell loop and the division loop of
Simulation.cpp, Compute.cpp's deposition, UpdateEnvArrayMG_OxygenAcetate,
Multigrid::solve).  Every call goes through libbcg.so; there is no CPU
implementation here.
"""
import ctypes

import numpy as np

from . import _abi, params as _params


def synth_colony(n, width, height, seed=20261203, radius=0.5, len_lo=2.0, len_hi=4.0,
                 l_divide=3.0, div_phase_spread=0.0, entry=None):
    """Seeded synthetic colony (bcg_synth_colony): n cells in a half-ellipse
    dome of width x height um on the agar, as bcg_cell records.  `entry`
    replaces the library's bcg_synth_colony by another C function of the
    same signature (the benchmark's reference arm passes the oracle's)."""
    out = np.zeros(n, dtype=_abi.CELL_DTYPE)
    got = ctypes.c_int(0)
    fn = entry if entry is not None else _abi.load().bcg_synth_colony
    rc = fn(ctypes.c_uint64(seed), n, ctypes.c_double(width), ctypes.c_double(height), ctypes.c_double(radius),
            ctypes.c_double(len_lo), ctypes.c_double(len_hi), ctypes.c_double(l_divide),
            ctypes.c_double(div_phase_spread), _abi.ptr(out), n, ctypes.byref(got))
    _abi.check(rc, "bcg_synth_colony")
    return out[:got.value]


def packed_colony(n, width, height, seed=20261207, radius=0.5, len_lo=2.0, len_hi=4.0, l_divide=3.0,
                  gap=0.02, div_phase_spread=1.0):
    """A densely packed colony: horizontal cells laid end to end in layers
    one diameter apart (touching, no overlap), each layer starting at a
    random offset, inside a half-ellipse dome of width x height um on the
    agar, filled bottom up until n cells are placed (the dome is scaled up
    if it cannot hold them).  Every cell touches its neighbours in the
    layers above and below, so the reduced neighbour lists hold about 8
    cells where the random packing of synth_colony holds about 2.  Records
    as synth_colony makes them."""
    rng = np.random.default_rng(seed)
    d = 2 * radius
    scale = 1.0
    while True:
        W, H = width * scale, height * scale
        px, pz, qx, lens = [], [], [], []
        z = radius
        while z <= H and len(lens) < n:
            e = np.sqrt(max(0.0, 1.0 - (z / H) ** 2))
            half = 0.5 * W * e
            x = -half + rng.uniform(0.0, len_hi)
            while len(lens) < n:
                L = rng.uniform(len_lo, len_hi)
                if x + L + d > half:
                    break
                px.append(x + radius); qx.append(x + radius + L); pz.append(z); lens.append(L)
                x += L + d + gap
            z += d
        if len(lens) >= n:
            break
        scale *= 1.05
    out = np.zeros(n, dtype=_abi.CELL_DTYPE)
    out["p"][:, 0] = px[:n]; out["p"][:, 2] = pz[:n]
    out["q"][:, 0] = qx[:n]; out["q"][:, 2] = pz[:n]
    out["length"] = lens[:n]
    out["radius"] = radius
    u = rng.uniform(0.0, 1.0, n)
    out["ldiv"] = out["length"] + (l_divide / 2) * (1.0 - div_phase_spread * u)
    out["type"] = 1
    out["ancestor"] = np.arange(1, n + 1, dtype=np.int32)
    return out


def workload_colony(name, seed=None, phi=0.45, div_phase_spread=1.0, n=None, entry=None):
    """Cells of a named workload (params.WORKLOADS)."""
    cells, aspect, *_ = _params.WORKLOADS[name]
    n = n or cells
    w, h = _params.dome_size(n, aspect, phi)
    s = (20261203 + list(_params.WORKLOADS).index(name)) if seed is None else seed
    return synth_colony(n, w, h, seed=s, div_phase_spread=div_phase_spread, entry=entry)


def depleted_wall(p, inside, depth_c=0.6, depth_o=0.8, acetate=2.0):
    """Level-0 wall rows (carbon, oxygen, acetate; length Box_x) of a colony
    that has consumed nutrients: a parabolic dip under the colony footprint,
    `depth_c` / `depth_o` of maxCarbon / Max_Oxygen at its centre, and
    acetate up to `acetate` mM.  `inside` is the INSIDE field (Box_x x
    Box_z, z fastest).  The agar solve copies these rows under the colony
    into its level-0 bottom row (copyToMG, Multigrid.cpp:891-907), which
    gives Multigrid::solve a non-zero right-hand side; from the uniform
    initial state it has none."""
    X = p.box_x
    col = np.asarray(inside).reshape(X, -1)[:, 0] > 0
    xs = np.nonzero(col)[0]
    x = np.arange(X, dtype=np.float64)
    if xs.size == 0:
        u = np.zeros(X)
    else:
        c = 0.5 * (xs[0] + xs[-1])
        w = max(0.5 * (xs[-1] - xs[0]), 1.0)
        u = np.clip(1.0 - ((x - c) / w) ** 2, 0.0, 1.0)
    return (p.max_carbon * (1.0 - depth_c * u), p.max_o2 * (1.0 - depth_o * u), acetate * u)


class Rng:
    """The host's glibc-compatible rand() stream (bcg_rng_*)."""

    def __init__(self, seed):
        self.state = _abi.Rng()
        _abi.load().bcg_rng_seed(ctypes.byref(self.state), seed)

    def next(self):
        return _abi.load().bcg_rng_next(ctypes.byref(self.state))

    def skip(self, k):
        _abi.load().bcg_rng_skip(ctypes.byref(self.state), int(k))

    def frand(self, k):
        """k values of (float)rand()/RAND_MAX as float32."""
        r = np.array([self.next() for _ in range(k)], dtype=np.int64)
        return (r.astype(np.float32) / np.float32(2147483647.0)).astype(np.float32)


class Colony:
    """One colony on the current CUDA device (a bcg_ctx)."""

    def __init__(self, p, cells=None):
        self.lib = _abi.load()
        self.params = p
        self.h = ctypes.c_void_p()
        _abi.check(self.lib.bcg_create(ctypes.byref(p), ctypes.byref(self.h)), "bcg_create")
        if cells is not None:
            self.upload(cells)

    def close(self):
        if self.h:
            self.lib.bcg_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- cells --------------------------------------------------------------
    def upload(self, cells):
        cells = np.ascontiguousarray(cells, dtype=_abi.CELL_DTYPE)
        _abi.check(self.lib.bcg_upload_cells(self.h, _abi.ptr(cells), len(cells)), "bcg_upload_cells")

    def n_cells(self):
        n = ctypes.c_int()
        _abi.check(self.lib.bcg_num_cells(self.h, ctypes.byref(n)), "bcg_num_cells")
        return n.value

    def cells(self):
        n = self.n_cells()
        out = np.zeros(n, dtype=_abi.CELL_DTYPE)
        got = ctypes.c_int()
        _abi.check(self.lib.bcg_download_cells(self.h, _abi.ptr(out), n, ctypes.byref(got)), "bcg_download_cells")
        return out

    # -- neighbours ---------------------------------------------------------
    def rebuild_neighbours(self):
        _abi.check(self.lib.bcg_rebuild_neighbours(self.h), "bcg_rebuild_neighbours")

    def neighbours(self, stride=None):
        n = self.n_cells()
        stride = stride or self.params.max_neighbours
        counts = np.zeros(n, dtype=np.int32)
        lists = np.zeros((max(n, 1), stride), dtype=np.int32)
        _abi.check(self.lib.bcg_get_neighbours(self.h, _abi.ptr(counts, ctypes.c_int), _abi.ptr(lists, ctypes.c_int), stride),
                   "bcg_get_neighbours")
        return [lists[i, :counts[i]].copy() for i in range(n)]

    def set_neighbours(self, lists):
        n = self.n_cells()
        stride = max(1, max((len(l) for l in lists), default=1))
        counts = np.array([len(l) for l in lists], dtype=np.int32)
        arr = np.zeros((max(n, 1), stride), dtype=np.int32)
        for i, l in enumerate(lists):
            arr[i, :len(l)] = l
        _abi.check(self.lib.bcg_set_neighbours(self.h, _abi.ptr(counts, ctypes.c_int), _abi.ptr(arr, ctypes.c_int), stride),
                   "bcg_set_neighbours")

    # -- mechanics ----------------------------------------------------------
    def move_grow(self, dt):
        nd = ctypes.c_int()
        calls = ctypes.c_int64()
        _abi.check(self.lib.bcg_move_grow(self.h, dt, ctypes.byref(nd), ctypes.byref(calls)), "bcg_move_grow")
        return nd.value, calls.value

    def dividing(self, n):
        ids = np.zeros(max(n, 1), dtype=np.int32)
        _abi.check(self.lib.bcg_get_dividing(self.h, _abi.ptr(ids, ctypes.c_int), n), "bcg_get_dividing")
        return ids[:n]

    def divide(self, draws, t):
        draws = np.ascontiguousarray(draws, dtype=np.float32).reshape(-1)
        nsets = draws.size // 9
        done = ctypes.c_int()
        lineage = np.zeros(2 * max(nsets, 1), dtype=np.int32)
        _abi.check(self.lib.bcg_divide(self.h, _abi.ptr(draws, ctypes.c_float), nsets, t, ctypes.byref(done),
                                       _abi.ptr(lineage, ctypes.c_int)), "bcg_divide")
        return lineage[:2 * done.value].reshape(-1, 2)

    def step(self, dt, t, rng):
        """MoveCell/GrowCell over all cells then the division loop, with the
        host rand() stream advanced exactly as the reference's is."""
        nd, calls = self.move_grow(dt)
        rng.skip(calls)
        draws = rng.frand(9 * nd) if nd else np.zeros(0, np.float32)
        return self.divide(draws, t)

    # -- fields -------------------------------------------------------------
    def field(self, name, level=0):
        fid = _abi.FIELDS[name] if isinstance(name, str) else name
        n = ctypes.c_size_t()
        _abi.check(self.lib.bcg_field_size(self.h, fid, level, ctypes.byref(n)), "bcg_field_size")
        out = np.zeros(n.value, dtype=np.float64)
        _abi.check(self.lib.bcg_get_field(self.h, fid, level, _abi.ptr(out, ctypes.c_double), n.value), "bcg_get_field")
        return out

    def set_field(self, name, values, level=0):
        fid = _abi.FIELDS[name] if isinstance(name, str) else name
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        _abi.check(self.lib.bcg_set_field(self.h, fid, level, _abi.ptr(v, ctypes.c_double), v.size), "bcg_set_field")

    def deplete_wall(self, **kw):
        """Set the level-0 wall rows to depleted_wall() of the current
        INSIDE field (call after update_density); returns the rows."""
        rows = depleted_wall(self.params, self.field("INSIDE"), **kw)
        for name, v in zip(("WALLF_CARBON", "WALLF_OXYGEN", "WALLF_ACETATE"), rows):
            self.set_field(name, v, 0)
        return rows

    def bbox(self):
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _abi.check(self.lib.bcg_get_bbox(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)), "bcg_get_bbox")
        return a.value, b.value, c.value

    def set_bbox(self, minx, maxx, maxz):
        _abi.check(self.lib.bcg_set_bbox(self.h, minx, maxx, maxz), "bcg_set_bbox")

    def update_density(self):
        _abi.check(self.lib.bcg_update_density(self.h), "bcg_update_density")

    def update_height(self):
        _abi.check(self.lib.bcg_update_height(self.h), "bcg_update_height")

    def initial_density(self):
        _abi.check(self.lib.bcg_initial_density(self.h), "bcg_initial_density")

    def nutrient_update(self, n=0, sweeps=-1):
        _abi.check(self.lib.bcg_nutrient_update(self.h, n, sweeps), "bcg_nutrient_update")

    def mg_solve(self, vcycles=0):
        _abi.check(self.lib.bcg_mg_solve(self.h, vcycles), "bcg_mg_solve")

    def legacy_env_update(self, max_iter, min_iter=None, conv_crit=1e-4):
        """bcg_legacy_env_update (UpdateEnvArray_OxygenAcetate): exactly
        max_iter iterations unless min_iter is given; returns the count."""
        n = ctypes.c_int()
        _abi.check(self.lib.bcg_legacy_env_update(self.h, max_iter if min_iter is None else min_iter, max_iter,
                                                  conv_crit, ctypes.byref(n)), "bcg_legacy_env_update")
        return n.value

    def legacy_depletion(self):
        """bcg_legacy_agar_depletion (nutrientDepletionAgar_OxygenAcetate); returns the steps run."""
        n = ctypes.c_int()
        _abi.check(self.lib.bcg_legacy_agar_depletion(self.h, ctypes.byref(n)), "bcg_legacy_agar_depletion")
        return n.value

    def colony_sweeps(self, sweeps, count0=0):
        _abi.check(self.lib.bcg_colony_sweeps(self.h, sweeps, count0), "bcg_colony_sweeps")

    def mg_solve_tol(self, rel_tol=1e-8, precision=64, max_iters=50):
        it = ctypes.c_int()
        rr = ctypes.c_double()
        _abi.check(self.lib.bcg_mg_solve_tol(self.h, rel_tol, precision, max_iters, ctypes.byref(it), ctypes.byref(rr)),
                   "bcg_mg_solve_tol")
        return it.value, rr.value

    # -- timers ---------------------------------------------------------------
    def enable_timers(self, on=True):
        _abi.check(self.lib.bcg_enable_timers(self.h, 1 if on else 0), "bcg_enable_timers")

    def timer(self, name):
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        _abi.check(self.lib.bcg_get_timer(self.h, _abi.TIMERS[name], ctypes.byref(ms), ctypes.byref(n)), "bcg_get_timer")
        return ms.value, n.value

    def set_pair_precision(self, bits):
        """bcg_set_pair_precision: 64 (reference FP64 geometry) or 32."""
        _abi.check(self.lib.bcg_set_pair_precision(self.h, int(bits)), "bcg_set_pair_precision")

    def autotune(self, what):
        """bcg_autotune: 'FORCE_GROUP' or 'SMOOTHER'; returns the choice."""
        ch = ctypes.c_int()
        _abi.check(self.lib.bcg_autotune(self.h, _abi.TUNE[what], ctypes.byref(ch)), "bcg_autotune")
        return ch.value

    def synchronize(self):
        _abi.check(self.lib.bcg_synchronize(self.h), "bcg_synchronize")

    def kernel_launches(self):
        return int(self.lib.bcg_kernel_launches(self.h))
