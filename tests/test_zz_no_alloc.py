"""bcg_mean_stress_noalloc, the allocation-free form of bcg_mean_stress.

Some hosts cannot allocate device memory when they write an output step:
their device memory is reserved up front by another framework's caching
allocator, or their output thread must not call into the CUDA allocator.
For them the stress diagnostics stage their per-cell results in a fixed
device array built into the library instead of per-call buffers.  The
results must be those of bcg_mean_stress.  The array is shared by every
call and keeps the previous call's contents, so the check runs two calls
in a row on two different colonies, the second one smaller, and compares
each with bcg_mean_stress.  It also checks the size limit.

This file is collected last on purpose: it runs after every other test in
a run that stops at the first failure, and it also passes on its own in a
fresh process.
"""
import ctypes

import numpy as np
import pytest

from baccolonygrowth_b200 import _abi, params
from baccolonygrowth_b200.colony import Colony, workload_colony

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12


def _stress(fn, col):
    n = col.n_cells()
    stress = np.full(5 * n, np.nan)
    fnet = np.full(3 * n, np.nan)
    fcw = ctypes.c_int64(-1)
    rc = fn(col.h, _abi.ptr(stress, ctypes.c_double), _abi.ptr(fnet, ctypes.c_double), ctypes.byref(fcw))
    _abi.check(rc, fn.__name__)
    return stress, fnet, fcw.value


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(a).max(), 1e-300)


def _colony(n, seed):
    p = params.workload_params("small_4k")
    col = Colony(p, workload_colony("small_4k", n=n, seed=seed))
    col.update_height()
    col.rebuild_neighbours()
    return col


def test_noalloc_matches_mean_stress_on_two_calls(gpu):
    lib = _abi.load()
    cols = [_colony(4096, 101), _colony(1500, 202)]
    want = [_stress(lib.bcg_mean_stress, c) for c in cols]
    # two calls in a row on the shared staging array
    got = [_stress(lib.bcg_mean_stress_noalloc, c) for c in cols]
    for (ws, wf, wc), (gs, gf, gc), c in zip(want, got, cols):
        assert np.isfinite(gs).all() and np.isfinite(gf).all()
        assert _rel(ws, gs) <= REL_TOL and _rel(wf, gf) <= REL_TOL
        assert wc == gc and gc >= 0            # F_cw draws, counted from zero each call
        c.close()


def test_noalloc_rejects_colonies_above_its_limit(gpu):
    lib = _abi.load()
    p = params.workload_params("scale_262k")
    col = Colony(p, workload_colony("scale_262k", n=_abi.NOALLOC_MAX_CELLS + 1000))
    assert col.n_cells() > _abi.NOALLOC_MAX_CELLS
    col.rebuild_neighbours()
    with pytest.raises(_abi.BcgError) as e:
        _stress(lib.bcg_mean_stress_noalloc, col)
    assert e.value.code == _abi.E_UNSUPPORTED
    col.close()
