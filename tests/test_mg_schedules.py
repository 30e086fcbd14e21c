"""The index schedules of the multigrid kernels, emulated on the CPU.

These restate, in Python, the orders in which csrc/mg.cu visits points and
check them against the reference's order (Multigrid.cpp) with a stand-in
point update: every point's new value is a hash of the values it reads, so
any read that sees another value than the sequential order gives changes
the result.

- The coarsest level's wavefront (k_mg_coarse_wave, k_mg_coarse_cluster):
  at step t sweep s relaxes the even columns of row t - 2s and the odd
  columns of row t - 2s - 1; no item of a step reads what another writes.
- The cluster form: block r owns columns [rW/C, (r+1)W/C), relaxes them and
  H halo columns on each side from its own copy, and takes its halos from
  its neighbours' published edge columns every H steps.
- NestSolAga folded into updateSolAga: the inverse of the nesting map
  (Multigrid.cpp:724-737) as k_mg_update_sol evaluates it.
- The rows restrictionAgaElementwise writes on a composite level, which
  bound the restriction's launch.
"""
import random

import pytest


def reads(i, k, W, nz):
    r = [(i, k)]
    if k > 0:
        r.append((i, k - 1))
    if k < nz:
        r.append((i, k + 1))
    if i > 0:
        r.append((i - 1, k))
    if i < W - 1:
        r.append((i + 1, k))
    return r


def update(vals, i, k):
    return hash(tuple(vals) + (i, k)) & 0xffffffffffff


def sequential(W, nz, sweeps, g0):
    """Multigrid.cpp's relaxation order: per sweep, all even columns, then
    all odd columns, each column bottom to top, in place."""
    g = dict(g0)
    for _ in range(sweeps):
        for par in (0, 1):
            for i in range(par, W, 2):
                for k in range(nz + 1):
                    g[(i, k)] = update([g[p] for p in reads(i, k, W, nz)], i, k)
    return g


def step_items(t, nz, sweeps, par, cols):
    tp = t - par
    if tp < 0:
        return []
    s_lo = (tp - nz + 1) // 2 if tp > nz else 0
    s_hi = min(sweeps - 1, tp // 2)
    return [(i, tp - 2 * s) for s in range(s_lo, s_hi + 1) for i in cols if i % 2 == par]


def wavefront(W, nz, sweeps, g0):
    g = dict(g0)
    steps = nz + 1 + 2 * (sweeps - 1) + 1
    for t in range(steps):
        items = step_items(t, nz, sweeps, 0, range(W)) + step_items(t, nz, sweeps, 1, range(W))
        writes = set(items)
        assert len(writes) == len(items)
        for (i, k) in items:
            assert 0 <= k <= nz
            for p in reads(i, k, W, nz):
                assert p == (i, k) or p not in writes, ("a step reads what it writes", t, (i, k), p)
        g.update({(i, k): update([g[p] for p in reads(i, k, W, nz)], i, k) for (i, k) in items})
    return g


def cluster(W, nz, sweeps, g0, C):
    H = min(8, W // C)
    own = [(r * W // C, (r + 1) * W // C) for r in range(C)]
    ext = [(max(0, c0 - H), min(W, c1 + H)) for c0, c1 in own]
    copies = [dict(g0) for _ in range(C)]
    steps = nz + 1 + 2 * (sweeps - 1) + 1
    t0 = 0
    while t0 < steps:
        t_end = min(steps, t0 + H)
        for t in range(t0, t_end):
            for r in range(C):
                cols = range(*ext[r])
                items = step_items(t, nz, sweeps, 0, cols) + step_items(t, nz, sweeps, 1, cols)
                g = copies[r]
                g.update({(i, k): update([g[p] for p in reads(i, k, W, nz)], i, k) for (i, k) in items})
        if t_end < steps:
            pub = [({(h, k): copies[r][(own[r][0] + h, k)] for h in range(H) for k in range(nz + 1)},
                    {(h, k): copies[r][(own[r][1] - H + h, k)] for h in range(H) for k in range(nz + 1)})
                   for r in range(C)]
            for r in range(C):
                (c0, c1), (e0, e1) = own[r], ext[r]
                for h in range(H):
                    for k in range(nz + 1):
                        if c0 - H + h >= e0:
                            copies[r][(c0 - H + h, k)] = pub[r - 1][1][(h, k)]
                        if c1 + h < e1:
                            copies[r][(c1 + h, k)] = pub[r + 1][0][(h, k)]
        t0 = t_end
    return {(i, k): v for r in range(C) for (i, k), v in copies[r].items() if own[r][0] <= i < own[r][1]}


@pytest.mark.parametrize("W,nz,sweeps", [(5, 3, 4), (9, 6, 7), (12, 10, 100), (145, 32, 100)])
def test_wavefront_is_the_sequential_order(W, nz, sweeps):
    rnd = random.Random(W * 1000 + nz)
    g0 = {(i, k): rnd.getrandbits(40) for i in range(W) for k in range(nz + 1)}
    assert wavefront(W, nz, sweeps, g0) == sequential(W, nz, sweeps, g0)


@pytest.mark.parametrize("W,nz,sweeps,C", [(16, 3, 5, 8), (17, 6, 9, 8), (33, 4, 100, 8), (73, 16, 100, 8),
                                           (145, 32, 100, 8)])
def test_cluster_halo_schedule_is_the_sequential_order(W, nz, sweeps, C):
    rnd = random.Random(W * 7 + nz)
    g0 = {(i, k): rnd.getrandbits(40) for i in range(W) for k in range(nz + 1)}
    assert cluster(W, nz, sweeps, g0, C) == sequential(W, nz, sweeps, g0)


def mg_dims(X, ZA, A, l):
    d, d0 = 1 << l, 1 << A
    return min(X, X * d0 // d // 2), min(ZA, ZA * d0 // d // 2)


GRIDS = [(256, 32, 2, 8), (2304, 512, 3, 8), (4608, 1024, 3, 8), (128, 64, 2, 8), (40, 5, 2, 2)]


@pytest.mark.parametrize("X,ZA,A,levels", GRIDS)
def test_nest_inverse_map(X, ZA, A, levels):
    """k_mg_update_sol on level l-1 writes exactly the points NestSolAga
    copies into level l, from the same sources."""
    for l in range(1, A):
        nx, nz = mg_dims(X, ZA, A, l)
        nxf, nzf = mg_dims(X, ZA, A, l - 1)
        d0 = 1 << A
        nxp, nzp = min((X * d0) >> l, X), min((ZA * d0) >> l, ZA)
        forward = {(i, k): (2 * i - nx + nxp // 2, 2 * k) for i in range(nx + 1) for k in range(nz + 1)
                   if 0 < 2 * i - nx + nxp // 2 < nxp and 2 * k < nzp}
        inverse = {}
        for i in range(nxf + 1):
            for k in range(nzf + 1):
                t = i + nx - nxp // 2
                if k % 2 == 0 and t % 2 == 0 and 0 < i < nxp and k < nzp and 0 <= t // 2 <= nx and k // 2 <= nz:
                    inverse[(t // 2, k // 2)] = (i, k)
        assert forward == inverse
        assert all(0 <= a <= nxf and 0 <= b <= nzf for a, b in forward.values())


@pytest.mark.parametrize("X,ZA,A,levels", GRIDS)
def test_restriction_rows_cover_every_write(X, ZA, A, levels):
    """The rows k_mg_restrict launches on a composite level hold every point
    restrictionAgaElementwise writes there."""
    d0 = 1 << A
    for l in range(1, levels):
        nx, nz = mg_dims(X, ZA, A, l)
        if nx < 2:
            break
        nxp, nzp = min((X * d0) >> l, X), min((ZA * d0) >> l, ZA)
        rows = nz + 1 if l >= A else max(0, min(nzp // 2, nz - 1)) + 1
        for k in range(nz + 1):
            for i in range(nx + 1):
                ip, kp = 2 * i - nx + nxp // 2, 2 * k
                if i == 0 or i == nx or k == nz:
                    written = l >= A
                elif k == 0:
                    written = True
                else:
                    written = (l < A and 0 <= ip <= nxp and kp <= nzp) or l >= A
                if written:
                    assert k < rows, (l, i, k)
                    if l < A and k > 0:
                        assert 0 <= ip <= nxp and kp <= nzp
