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
- The fused smoother of csrc/mg_smooth.cu (k_mg_smooth_tma): a warp owns a
  strip of 128 columns (4 per lane), runs the 2S half-sweeps as a
  pipeline (half-sweep h on row r - h at step r) with its neighbours from
  the adjacent lanes, and stores the middle columns of the strip; with one
  row segment it is the sequential order exactly, and with warm-started
  segments it agrees with it to rounding.
"""
import math
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


def tma_smoother(W, nz, sweeps, g0, upd, WV=116, HL=6, nseg=1, warm=0):
    """The schedule of k_mg_smooth_tma / ts_step for one species: returns
    the stored (E2) values.  `upd(vals, i, k)` takes the values of
    reads(i, k) in that order."""
    H = 2 * sweeps
    nstrip = (W + WV - 1) // WV
    rows = nz + 1
    seg_len = (rows + nseg - 1) // nseg
    nseg = (rows + seg_len - 1) // seg_len
    out = {}

    def E(q, col):
        return g0[(col, q)] if 0 <= q <= nz and 0 <= col < W else 0

    for strip in range(nstrip):
        c0 = strip * WV - HL
        cols = [[c0 + 4 * t + j for j in range(4)] for t in range(32)]
        for seg in range(nseg):
            ks = seg * seg_len
            ke = min(ks + seg_len, nz + 1)
            kw = max(0, ks - warm)
            r_end = ke - 1 + (H - 1)
            init = [[[E(kw - 1, cols[t][(h & 1) + 2 * j]) for j in range(2)] for t in range(32)] for h in range(H)]
            h1 = [[list(x) for x in hh] for hh in init]
            h2 = [[list(x) for x in hh] for hh in init]
            for r in range(kw, r_end + 1):
                # neighbour values from the adjacent lanes (a lane at the
                # warp's edge gets its own value, as a shuffle does)
                nb = []
                for h in range(H):
                    if h & 1:
                        nb.append([h1[h - 1][min(t + 1, 31)][0] for t in range(32)])
                    else:
                        src = [E(r, cols[t][3]) for t in range(32)] if h == 0 else [h1[h - 1][t][1] for t in range(32)]
                        nb.append([src[max(t - 1, 0)] for t in range(32)])
                for h in range(H - 1, -1, -1):
                    k = r - h
                    top = min(nz, ke - 1 + (H - 1 - h) // 2)
                    if k < kw or k > top:
                        h2[h] = [list(x) for x in h1[h]]
                        continue
                    for t in range(32):
                        e0 = [E(r, c) for c in cols[t]]
                        ep = [E(r + 1, c) for c in cols[t]]
                        em = [E(r - 1, c) for c in cols[t]]
                        if h & 1:
                            xm = [h1[h - 1][t][0], h1[h - 1][t][1]]
                            xp = [h1[h - 1][t][1], nb[h][t]]
                            up = [e0[1], e0[3]] if h == 1 else [h1[h - 2][t][0], h1[h - 2][t][1]]
                            old = [em[1], em[3]] if h == 1 else [h2[h - 2][t][0], h2[h - 2][t][1]]
                        else:
                            o = [e0[1], e0[3]] if h == 0 else [h1[h - 1][t][0], h1[h - 1][t][1]]
                            xm = [nb[h][t], o[0]]
                            xp = [o[0], o[1]]
                            up = [ep[0], ep[2]] if h == 0 else [h1[h - 2][t][0], h1[h - 2][t][1]]
                            old = [e0[0], e0[2]] if h == 0 else [h2[h - 2][t][0], h2[h - 2][t][1]]
                        for j in range(2):
                            i = cols[t][(h & 1) + 2 * j]
                            v = {(i, k): old[j], (i, k - 1): h1[h][t][j], (i, k + 1): up[j],
                                 (i - 1, k): xm[j], (i + 1, k): xp[j]}
                            h2[h][t][j] = upd([v[p] for p in reads(i, k, W, nz)], i, k)
                kS = r - (H - 1)
                if ks <= kS < ke:
                    for t in range(32):
                        vals = [h1[H - 2][t][0], h2[H - 1][t][0], h1[H - 2][t][1], h2[H - 1][t][1]]
                        for j in range(4):
                            i = cols[t][j]
                            if c0 + HL <= i < c0 + HL + WV and 0 <= i < W:
                                assert (i, kS) not in out
                                out[(i, kS)] = vals[j]
                h1, h2 = h2, h1
    return out


@pytest.mark.parametrize("W,nz,sweeps,geom", [(5, 3, 3, 64), (50, 7, 3, 64), (128, 4, 3, 64), (129, 9, 2, 64),
                                              (233, 5, 3, 64), (240, 6, 1, 32), (461, 4, 3, 32)])
def test_tma_smoother_is_the_sequential_order(W, nz, sweeps, geom):
    """One row segment: every stored point equals the sequential sweeps'
    value (hash updates: any read out of order changes it), every point is
    stored once; FP64 strips (116 of 128 columns) and FP32 strips (112)."""
    rnd = random.Random(W * 31 + nz)
    g0 = {(i, k): rnd.getrandbits(40) for i in range(W) for k in range(nz + 1)}
    WV, HL = (116, 6) if geom == 64 else (112, 8)
    out = tma_smoother(W, nz, sweeps, g0, update, WV=WV, HL=HL)
    assert out == sequential(W, nz, sweeps, g0)


def sequential_values(W, nz, sweeps, g0, upd):
    g = dict(g0)
    for _ in range(sweeps):
        for par in (0, 1):
            for i in range(par, W, 2):
                for k in range(nz + 1):
                    g[(i, k)] = upd([g[p] for p in reads(i, k, W, nz)], i, k)
    return g


def test_tma_smoother_warm_segments_agree_to_rounding():
    """Row segments that start `warm` rows early from the pre-smoothing
    values: with the reference's contraction (cf = 0.2, so a row carries at
    most 1/4.4 of the error below it) and the warm-up of mg.cu's warm_rows,
    the result is the sequential one to rounding."""
    cf = 0.2
    inv = 1.0 / (cf + 2.0)
    rnd = random.Random(7)
    W, nz = 150, 95
    R = {(i, k): rnd.uniform(-1, 1) for i in range(W) for k in range(nz + 1)}

    def lin(vals, i, k):
        # E = (R cf + 1/2 sum of the neighbours read) / (cf + 2), the interior form
        return (R.get((i, k), 0.0) * cf + 0.5 * sum(vals[1:])) * inv

    a = 0.5 / (cf + 2.0)
    warm = next(w for w in range(1, 64) if a ** w * w * w < 1e-18)
    g0 = {(i, k): rnd.uniform(-1, 1) for i in range(W) for k in range(nz + 1)}
    ref = sequential_values(W, nz, 3, g0, lin)
    for nseg in (2, 3, 4):
        out = tma_smoother(W, nz, 3, g0, lin, nseg=nseg, warm=warm)
        assert set(out) == set(ref)
        err = max(abs(out[p] - ref[p]) for p in ref)
        assert err < 1e-14, (nseg, err)


def test_tma_smoother_r_window_slots():
    """The R window of k_mg_smooth_tma (ts_trip, ts_step): 6 slots, row
    2t + P of the walk written to slot b + P at trip t (b = 2 (t mod 3)),
    and row r - h read at offset m = P + 6 - h from b, wrapped when
    m >= 6 - b.  Every read must find the row it wants, in a slot no later
    row has taken."""
    slots = [None] * 6
    for t in range(30):
        q = t % 3
        b, wrap = 2 * q, 6 - 2 * q
        for P in (0, 1):
            r = 2 * t + P
            assert b + P < 6
            slots[b + P] = r
            for h in range(1, 6):
                m = P + 6 - h
                if m == 6:
                    idx = b
                elif m == 1:
                    idx = b + 1
                else:
                    idx = b + m - 6 if m >= wrap else b + m
                assert 0 <= idx < 6
                if r - h >= 0:
                    assert slots[idx] == r - h, (t, P, h)


def native_level_int(x, X, lv):
    """csrc/nutrients.cu leg_native_level: the finest composite level whose
    extent holds column x of a level-lv row, in integers."""
    if x < X // 2:
        k = 0
        while (X - 2 * x) << (k + 1) <= X:
            k += 1
        return lv - k
    if x > X // 2:
        k = 0
        while ((2 * x - X) << k) < X:
            k += 1
        return lv - k + 1
    return 0


def native_level_ref(x, X, lv):
    """The reference's form (Nutrients.cpp:917-921, 947-951, 1027-1031)."""
    if x < X // 2:
        return math.ceil(math.log(1 - x * 2.0 / X) / math.log(2) + lv)
    if x > X // 2:
        return math.floor(math.log(x * 2.0 / X - 1) / math.log(2) + lv) + 1
    return 0


def row_level_int(z, ZA, A):
    v = (1 + z) << (A - 1)
    if v <= ZA:
        return 0
    k = 0
    while (ZA << k) < v:
        k += 1
    return k


def row_level_ref(z, ZA, A):
    return max(math.ceil(math.log((1 + z) * (2 ** (A - 1)) * 1.0 / ZA) / math.log(2)), 0)


@pytest.mark.parametrize("X,ZA,A", [(256, 32, 2), (2304, 512, 3), (4608, 1024, 3), (1520, 512, 3), (99, 17, 4),
                                    (128, 64, 2)])
def test_depletion_level_maps_in_integers(X, ZA, A):
    """The GPU's integer forms of the legacy solver's level maps give the
    reference's floating-point ceil/floor of log2 at every column and row."""
    for lv in range(A):
        for x in range(X):
            assert native_level_int(x, X, lv) == native_level_ref(x, X, lv), (x, lv)
    for z in range(ZA):
        assert row_level_int(z, ZA, A) == row_level_ref(z, ZA, A), z
