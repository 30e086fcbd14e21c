"""Test infrastructure: ctypes access to the checkers.

- the C restatement oracle/liboracle.so (always built by build());
- the reference itself, oracle/_ref/libbcgref.so (built only where the
  reference tree is present; tests that need it skip otherwise).

Both expose the same scenario API (create, load cells, rebuild neighbours,
move/grow, divide, field access) so a test can run one scenario through the
reference, the oracle and the CUDA library and compare.
"""
import ctypes
import os

import numpy as np

from baccolonygrowth_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_LIB = os.path.join(ROOT, "oracle", "liboracle.so")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libbcgref.so")

_VP = ctypes.c_void_p
_PP = ctypes.POINTER(_abi.Params)
_PI = ctypes.POINTER(ctypes.c_int)
_PD = ctypes.POINTER(ctypes.c_double)
_PLL = ctypes.POINTER(ctypes.c_longlong)


def _proto(lib, name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args


_oracle = None
_ref = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_LIB):
            raise RuntimeError("oracle/liboracle.so not built")
        lib = ctypes.CDLL(ORACLE_LIB)
        _proto(lib, "orc_create", _VP, [_PP, ctypes.c_uint, ctypes.c_int])
        _proto(lib, "orc_destroy", None, [_VP])
        _proto(lib, "orc_load_cells", ctypes.c_int, [_VP, _VP, ctypes.c_int])
        _proto(lib, "orc_get_cells", ctypes.c_int, [_VP, _VP, ctypes.c_int])
        _proto(lib, "orc_num_cells", ctypes.c_int, [_VP])
        _proto(lib, "orc_rand_calls", ctypes.c_longlong, [_VP])
        _proto(lib, "orc_error", ctypes.c_int, [_VP])
        _proto(lib, "orc_rebuild_neighbours", None, [_VP])
        _proto(lib, "orc_get_neighbours", ctypes.c_int, [_VP, _PI, _PI, ctypes.c_int])
        _proto(lib, "orc_set_neighbours", ctypes.c_int, [_VP, _PI, _PI, ctypes.c_int])
        _proto(lib, "orc_move_grow", ctypes.c_int, [_VP, ctypes.c_double, _PI, _PLL])
        _proto(lib, "orc_divide", ctypes.c_int, [_VP, ctypes.c_double, _PI])
        _proto(lib, "orc_field", ctypes.c_long, [_VP, ctypes.c_int, ctypes.c_int, _PD, ctypes.c_long, ctypes.c_int])
        _proto(lib, "orc_bbox", None, [_VP, _PI, _PI, _PI])
        _proto(lib, "orc_set_bbox", None, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int])
        _proto(lib, "orc_initial_fields", None, [_VP, ctypes.c_int])
        _proto(lib, "orc_update_density", None, [_VP])
        _proto(lib, "orc_update_height", None, [_VP])
        _proto(lib, "orc_nutrient_update", None, [_VP, ctypes.c_int])
        _proto(lib, "orc_mg_solve", None, [_VP, ctypes.c_int, ctypes.c_double])
        _proto(lib, "orc_colony_sweeps", None, [_VP, ctypes.c_int, ctypes.c_int])
        _proto(lib, "orc_loop_step", ctypes.c_int, [_VP, _PI])
        _proto(lib, "orc_time", ctypes.c_double, [_VP])
        _proto(lib, "orc_mean_stress", ctypes.c_longlong, [_VP, _PD, _PD])
        _proto(lib, "orc_legacy_env_update", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_double])
        _proto(lib, "orc_legacy_depletion", ctypes.c_int, [_VP])
        _proto(lib, "orc_params_default", ctypes.c_int, [_PP])
        _proto(lib, "orc_params_finalize", ctypes.c_int, [_PP])
        _proto(lib, "orc_synth_colony", ctypes.c_int,
               [ctypes.c_uint64, ctypes.c_int] + [ctypes.c_double] * 7 + [_VP, ctypes.c_int, _PI])
        _oracle = lib
    return _oracle


def oracle_param_entries():
    """The oracle's restatement of bcg_params_default / bcg_params_finalize
    (for params.workload_params(..., entries=...))."""
    lib = oracle_lib()
    return lib.orc_params_default, lib.orc_params_finalize


def oracle_synth_entry():
    """The oracle's restatement of bcg_synth_colony (for
    colony.workload_colony(..., entry=...))."""
    return oracle_lib().orc_synth_colony


def have_ref():
    return os.path.exists(REF_LIB)


def ref_lib():
    global _ref
    if _ref is None:
        if not have_ref():
            raise RuntimeError("oracle/_ref/libbcgref.so not built")
        lib = ctypes.CDLL(REF_LIB)
        _proto(lib, "ref_init", ctypes.c_int, [_PP, ctypes.c_uint, ctypes.c_int, ctypes.c_int])
        _proto(lib, "ref_load_cells", ctypes.c_int, [_VP, ctypes.c_int])
        _proto(lib, "ref_get_cells", ctypes.c_int, [_VP, ctypes.c_int])
        _proto(lib, "ref_num_cells", ctypes.c_int, [])
        _proto(lib, "ref_rand_calls", ctypes.c_longlong, [])
        _proto(lib, "ref_set_threads", None, [ctypes.c_int])
        _proto(lib, "ref_rebuild_neighbours", None, [])
        _proto(lib, "ref_get_neighbours", ctypes.c_int, [_PI, _PI, ctypes.c_int])
        _proto(lib, "ref_set_neighbours", ctypes.c_int, [_PI, _PI, ctypes.c_int])
        _proto(lib, "ref_move_grow", ctypes.c_int, [ctypes.c_double, _PI, _PLL])
        _proto(lib, "ref_divide", ctypes.c_int, [ctypes.c_double, _PI])
        _proto(lib, "ref_field", ctypes.c_long, [ctypes.c_int, ctypes.c_int, _PD, ctypes.c_long, ctypes.c_int])
        _proto(lib, "ref_bbox", None, [_PI, _PI, _PI])
        _proto(lib, "ref_set_bbox", None, [ctypes.c_int, ctypes.c_int, ctypes.c_int])
        _proto(lib, "ref_initial_fields", None, [ctypes.c_int])
        _proto(lib, "ref_update_density", None, [])
        _proto(lib, "ref_update_height", None, [])
        _proto(lib, "ref_nutrient_update", None, [ctypes.c_int])
        _proto(lib, "ref_mg_solve", None, [ctypes.c_int, ctypes.c_double])
        _proto(lib, "ref_loop_step", ctypes.c_int, [_PI])
        _proto(lib, "ref_time", ctypes.c_double, [])
        _proto(lib, "ref_mean_stress", ctypes.c_longlong, [_PD, _PD])
        _proto(lib, "ref_output_cells", ctypes.c_longlong, [ctypes.c_char_p, ctypes.c_int, ctypes.c_double, ctypes.c_int])
        _proto(lib, "ref_output_fields", None, [ctypes.c_double, ctypes.c_double])
        _proto(lib, "ref_output_initial", None, [ctypes.c_char_p, ctypes.c_double, ctypes.c_int])
        _proto(lib, "ref_loop_step_out", ctypes.c_int, [ctypes.c_char_p, _PI])
        _proto(lib, "ref_get_new_cells", ctypes.c_int, [_VP, ctypes.c_int])
        _proto(lib, "ref_surface_forces", None, [_PD])
        _proto(lib, "ref_output_cells_given", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, _PD, ctypes.c_int])
        _proto(lib, "ref_set_new_cells", ctypes.c_int, [_VP, ctypes.c_int])
        _proto(lib, "ref_legacy_env_update", ctypes.c_int, [ctypes.c_int])
        _proto(lib, "ref_legacy_depletion", ctypes.c_int, [])
        _ref = lib
    return _ref


class _Model:
    """Common scenario interface over the oracle / the reference harness."""

    def cells(self):
        out = np.zeros(self.n_cells(), dtype=_abi.CELL_DTYPE)
        self._get_cells(out)
        return out

    def neighbours(self, stride=2674):
        n = self.n_cells()
        counts = np.zeros(n, dtype=np.int32)
        lists = np.zeros((n, stride), dtype=np.int32)
        self._get_nbr(counts, lists, stride)
        return [lists[i, :counts[i]].copy() for i in range(n)]

    def set_neighbours(self, lists):
        n = self.n_cells()
        stride = max(1, max((len(l) for l in lists), default=1))
        counts = np.array([len(l) for l in lists], dtype=np.int32)
        arr = np.zeros((n, stride), dtype=np.int32)
        for i, l in enumerate(lists):
            arr[i, :len(l)] = l
        self._set_nbr(counts, arr, stride)

    def step(self, dt, t):
        """move/grow + divide; returns (dividing ids, rand calls in move, lineage)."""
        ids = np.zeros(max(1, self.n_cells()), dtype=np.int32)
        calls = ctypes.c_longlong(0)
        nd = self._move_grow(dt, ids, calls)
        lineage = np.zeros(2 * max(1, nd), dtype=np.int32)
        done = self._divide(t, lineage)
        return ids[:nd].copy(), calls.value, lineage[:2 * done].reshape(-1, 2).copy()

    def field(self, fid, level=0):
        n = self._field(fid, level, None, 0, 0)
        if n < 0:
            raise ValueError("bad field %d" % fid)
        buf = np.zeros(n, dtype=np.float64)
        self._field(fid, level, buf, n, 0)
        return buf

    def set_field(self, fid, arr, level=0):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        r = self._field(fid, level, arr, arr.size, 1)
        if r != arr.size:
            raise ValueError("field size mismatch")


class Oracle(_Model):
    def __init__(self, params, seed=12345, make_wall=True):
        self.lib = oracle_lib()
        self.h = self.lib.orc_create(ctypes.byref(params), seed, 1 if make_wall else 0)

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    __del__ = close

    def load(self, cells):
        cells = np.ascontiguousarray(cells)
        return self.lib.orc_load_cells(self.h, _abi.ptr(cells), len(cells))

    def n_cells(self):
        return self.lib.orc_num_cells(self.h)

    def error(self):
        return self.lib.orc_error(self.h)

    def rand_calls(self):
        return self.lib.orc_rand_calls(self.h)

    def _get_cells(self, out):
        self.lib.orc_get_cells(self.h, _abi.ptr(out), len(out))

    def rebuild(self):
        self.lib.orc_rebuild_neighbours(self.h)

    def _get_nbr(self, counts, lists, stride):
        self.lib.orc_get_neighbours(self.h, _abi.ptr(counts, ctypes.c_int), _abi.ptr(lists, ctypes.c_int), stride)

    def _set_nbr(self, counts, lists, stride):
        self.lib.orc_set_neighbours(self.h, _abi.ptr(counts, ctypes.c_int), _abi.ptr(lists, ctypes.c_int), stride)

    def _move_grow(self, dt, ids, calls):
        return self.lib.orc_move_grow(self.h, dt, _abi.ptr(ids, ctypes.c_int), ctypes.byref(calls))

    def _divide(self, t, lineage):
        return self.lib.orc_divide(self.h, t, _abi.ptr(lineage, ctypes.c_int))

    def _field(self, fid, level, buf, n, write):
        p = _abi.ptr(buf, ctypes.c_double) if buf is not None else None
        return self.lib.orc_field(self.h, fid, level, p, n, write)

    def bbox(self):
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self.lib.orc_bbox(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return a.value, b.value, c.value

    def set_bbox(self, minx, maxx, maxz):
        self.lib.orc_set_bbox(self.h, minx, maxx, maxz)

    def initial_fields(self, run_nutrients=True):
        self.lib.orc_initial_fields(self.h, 1 if run_nutrients else 0)

    def update_density(self):
        self.lib.orc_update_density(self.h)

    def update_height(self):
        self.lib.orc_update_height(self.h)

    def nutrient_update(self, n=0):
        self.lib.orc_nutrient_update(self.h, n)

    def legacy_env_update(self, iters, min_iter=None, conv_crit=1e-4):
        """UpdateEnvArray_OxygenAcetate: exactly `iters` iterations unless
        min_iter is given (then the convergence test may end it earlier)."""
        return self.lib.orc_legacy_env_update(self.h, iters if min_iter is None else min_iter, iters, conv_crit)

    def legacy_depletion(self):
        return self.lib.orc_legacy_depletion(self.h)

    def mg_solve(self, vcycles=3, dt=100.0):
        self.lib.orc_mg_solve(self.h, vcycles, dt)

    def colony_sweeps(self, sweeps, count0=0):
        self.lib.orc_colony_sweeps(self.h, sweeps, count0)

    def loop_step(self):
        lineage = np.zeros(2 * max(1, self.n_cells()), dtype=np.int32)
        done = self.lib.orc_loop_step(self.h, _abi.ptr(lineage, ctypes.c_int))
        return lineage[:2 * done].reshape(-1, 2).copy()

    def time(self):
        return self.lib.orc_time(self.h)

    def mean_stress(self):
        st = np.zeros(5 * self.n_cells()); fn = np.zeros(3 * self.n_cells())
        calls = self.lib.orc_mean_stress(self.h, _abi.ptr(st, ctypes.c_double), _abi.ptr(fn, ctypes.c_double))
        return st.reshape(-1, 5), fn.reshape(-1, 3), calls


class Reference(_Model):
    """The reference compiled from its sources (one process-wide instance)."""

    def __init__(self, params, seed=12345, make_wall=True, threads=1):
        self.lib = ref_lib()
        self.lib.ref_init(ctypes.byref(params), seed, 1 if make_wall else 0, threads)

    def close(self):
        pass

    def load(self, cells):
        cells = np.ascontiguousarray(cells)
        return self.lib.ref_load_cells(_abi.ptr(cells), len(cells))

    def n_cells(self):
        return self.lib.ref_num_cells()

    def error(self):
        return 0

    def rand_calls(self):
        return self.lib.ref_rand_calls()

    def _get_cells(self, out):
        self.lib.ref_get_cells(_abi.ptr(out), len(out))

    def rebuild(self):
        self.lib.ref_rebuild_neighbours()

    def _get_nbr(self, counts, lists, stride):
        self.lib.ref_get_neighbours(_abi.ptr(counts, ctypes.c_int), _abi.ptr(lists, ctypes.c_int), stride)

    def _set_nbr(self, counts, lists, stride):
        self.lib.ref_set_neighbours(_abi.ptr(counts, ctypes.c_int), _abi.ptr(lists, ctypes.c_int), stride)

    def _move_grow(self, dt, ids, calls):
        return self.lib.ref_move_grow(dt, _abi.ptr(ids, ctypes.c_int), ctypes.byref(calls))

    def _divide(self, t, lineage):
        return self.lib.ref_divide(t, _abi.ptr(lineage, ctypes.c_int))

    def _field(self, fid, level, buf, n, write):
        p = _abi.ptr(buf, ctypes.c_double) if buf is not None else None
        return self.lib.ref_field(fid, level, p, n, write)

    def bbox(self):
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self.lib.ref_bbox(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return a.value, b.value, c.value

    def set_bbox(self, minx, maxx, maxz):
        self.lib.ref_set_bbox(minx, maxx, maxz)

    def initial_fields(self, run_nutrients=True):
        self.lib.ref_initial_fields(1 if run_nutrients else 0)

    def update_density(self):
        self.lib.ref_update_density()

    def update_height(self):
        self.lib.ref_update_height()

    def nutrient_update(self, n=0):
        self.lib.ref_nutrient_update(n)

    def legacy_env_update(self, iters):
        return self.lib.ref_legacy_env_update(iters)

    def legacy_depletion(self):
        return self.lib.ref_legacy_depletion()

    def mg_solve(self, vcycles=3, dt=100.0):
        self.lib.ref_mg_solve(vcycles, dt)

    def loop_step(self):
        lineage = np.zeros(2 * max(1, self.n_cells()), dtype=np.int32)
        done = self.lib.ref_loop_step(_abi.ptr(lineage, ctypes.c_int))
        return lineage[:2 * done].reshape(-1, 2).copy()

    def time(self):
        return self.lib.ref_time()

    def mean_stress(self):
        st = np.zeros(5 * self.n_cells()); fn = np.zeros(3 * self.n_cells())
        calls = self.lib.ref_mean_stress(_abi.ptr(st, ctypes.c_double), _abi.ptr(fn, ctypes.c_double))
        return st.reshape(-1, 5), fn.reshape(-1, 3), calls

    # ---- output steps through the reference's own writers ----------------
    def output_cells(self, directory, output_id, t, append=False):
        """CreateOutputFiles + mean_stress/Output per cell; returns rand() draws."""
        return self.lib.ref_output_cells(str(directory).encode(), output_id, t, 1 if append else 0)

    def output_fields(self, t, dt):
        self.lib.ref_output_fields(t, dt)

    def output_initial(self, directory, t, append=False):
        self.lib.ref_output_initial(str(directory).encode(), t, 1 if append else 0)

    def loop_step_out(self, directory):
        lineage = np.zeros(2 * max(1, self.n_cells()), dtype=np.int32)
        done = self.lib.ref_loop_step_out(str(directory).encode(), _abi.ptr(lineage, ctypes.c_int))
        return lineage[:2 * done].reshape(-1, 2).copy()

    def new_cells(self):
        out = np.zeros(self.n_cells(), dtype=_abi.CELL_DTYPE)
        self.lib.ref_get_new_cells(_abi.ptr(out), len(out))
        return out

    def surface_forces(self):
        f = np.zeros(3 * max(1, self.n_cells()))
        self.lib.ref_surface_forces(_abi.ptr(f, ctypes.c_double))
        return f[:3 * self.n_cells()].reshape(-1, 3)

    def output_cells_given(self, directory, output_id, t, stress, stride=5, append=False):
        st = np.ascontiguousarray(stress, dtype=np.float64).reshape(-1)
        return self.lib.ref_output_cells_given(str(directory).encode(), output_id, t, 1 if append else 0,
                                               _abi.ptr(st, ctypes.c_double), stride)

    def set_new_cells(self, cells):
        cells = np.ascontiguousarray(cells)
        return self.lib.ref_set_new_cells(_abi.ptr(cells), len(cells))
