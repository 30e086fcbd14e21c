"""Steady glucose field of a colony and its gradients (bcg_steady_* in the C
ABI; no counterpart in the reference).

    s = Steady(nx=129, nz=65, nz_agar=33, h=2.0, c0=20.0, max_cells=50000)
    s.set_cells(xzlr)                       # (n, 4): x, z, L, R per cell
    C = s.solve(theta, w)                   # theta = (d_agar, d_colony, vmax, km)
    g_theta, g_w = s.vjp(dL_dC)             # gradients of a loss L(C)

`SteadyField` wraps solve/vjp as a torch.autograd.Function (torch is only
imported when it is used), so a loss written in torch, such as
`radial_profile_loss`, back-propagates through the solve.
"""
import ctypes

import numpy as np

from . import _abi


class SteadyParams(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("nz", ctypes.c_int), ("nz_agar", ctypes.c_int), ("max_cells", ctypes.c_int),
                ("h", ctypes.c_double), ("c0", ctypes.c_double)]


class Steady:
    def __init__(self, nx, nz, nz_agar, h, c0, max_cells):
        self.lib = _abi.load()
        self.p = SteadyParams(nx, nz, nz_agar, max_cells, h, c0)
        self.h = ctypes.c_void_p()
        _abi.check(self.lib.bcg_steady_create(ctypes.byref(self.p), ctypes.byref(self.h)), "bcg_steady_create")
        self.ncell = 0
        self.newton_iters = self.cg_iters = 0

    def close(self):
        if self.h:
            self.lib.bcg_steady_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        return (self.p.nz, self.p.nx)

    def set_cells(self, xzlr):
        a = np.ascontiguousarray(xzlr, dtype=np.float64).reshape(-1, 4)
        _abi.check(self.lib.bcg_steady_set_cells(self.h, _abi.ptr(a, ctypes.c_double), len(a)), "bcg_steady_set_cells")
        self.ncell = len(a)

    def solve(self, theta, w, tol=1e-13):
        th = np.ascontiguousarray(theta, dtype=np.float64).reshape(4)
        w = np.ascontiguousarray(w, dtype=np.float64).reshape(-1)
        assert w.size == self.ncell
        C = np.zeros(self.p.nx * self.p.nz)
        ni, ci = ctypes.c_int(), ctypes.c_int()
        _abi.check(self.lib.bcg_steady_solve(self.h, _abi.ptr(th, ctypes.c_double), _abi.ptr(w, ctypes.c_double),
                                             tol, _abi.ptr(C, ctypes.c_double), ctypes.byref(ni), ctypes.byref(ci)),
                   "bcg_steady_solve")
        self.newton_iters, self.cg_iters = ni.value, ci.value
        return C.reshape(self.shape)

    def vjp(self, dL_dC, tol=1e-13):
        g = np.ascontiguousarray(dL_dC, dtype=np.float64).reshape(-1)
        gt = np.zeros(4)
        gw = np.zeros(max(self.ncell, 1))
        _abi.check(self.lib.bcg_steady_vjp(self.h, _abi.ptr(g, ctypes.c_double), _abi.ptr(gt, ctypes.c_double),
                                           _abi.ptr(gw, ctypes.c_double), tol), "bcg_steady_vjp")
        return gt, gw[:self.ncell]


def radial_bins(nx, h, x0, nbins, row):
    """Bin index (distance |x - x0| along the agar surface row) of every
    vertex of `row`, and the bin counts; -1 beyond the last bin."""
    x = np.arange(nx) * h
    r = np.abs(x - x0)
    rmax = r.max() * (1 + 1e-12)
    b = np.minimum((r / rmax * nbins).astype(int), nbins - 1)
    return b, np.bincount(b, minlength=nbins)


def radial_profile(C, h, x0, nbins, row):
    """Mean concentration of `row` of C (nz, nx) per radial bin."""
    b, cnt = radial_bins(C.shape[1], h, x0, nbins, row)
    return np.bincount(b, weights=C[row], minlength=nbins) / cnt


def make_steady_field(torch):
    """The torch.autograd.Function over a Steady solver (built on first
    use so that importing this module does not import torch)."""

    class SteadyField(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta, w, solver, tol):
            C = solver.solve(theta.detach().cpu().double().numpy(), w.detach().cpu().double().numpy(), tol)
            ctx.solver, ctx.tol = solver, tol
            return torch.from_numpy(C.copy()).to(theta.device)

        @staticmethod
        def backward(ctx, grad_C):
            gt, gw = ctx.solver.vjp(grad_C.detach().cpu().double().numpy(), ctx.tol)
            return torch.from_numpy(gt), torch.from_numpy(gw), None, None

    return SteadyField


def radial_profile_loss(torch, C, h, x0, nbins, row, target):
    """L2 distance (sum of squares) of C's radial profile on `row` to a
    target profile, written in torch so that it back-propagates."""
    b, cnt = radial_bins(C.shape[1], h, x0, nbins, row)
    bt = torch.as_tensor(b, device=C.device)
    prof = torch.zeros(nbins, dtype=C.dtype, device=C.device).index_add_(0, bt, C[row]) / torch.as_tensor(cnt, dtype=C.dtype, device=C.device)
    return ((prof - torch.as_tensor(target, dtype=C.dtype, device=C.device)) ** 2).sum()


def synthetic_problem(nx=129, nz=65, nz_agar=33, h=2.0, n_cells=50000, seed=20261207):
    """Seeded synthetic case: cells (x, z, L, R) uniformly in a dome over the
    middle of the colony rows, per-cell growth weights ~ U(0.5, 1.5), and a
    target profile."""
    rng = np.random.default_rng(seed)
    W = (nx - 1) * h
    x0 = W / 2
    ztop = (nz - 1) * h
    zbase = nz_agar * h
    half = 0.35 * W
    xs = rng.uniform(x0 - half, x0 + half, n_cells)
    hgt = (ztop - zbase) * np.sqrt(np.clip(1 - ((xs - x0) / half) ** 2, 0, 1))
    zs = zbase + rng.uniform(0, 1, n_cells) * hgt
    L = rng.uniform(2.0, 4.0, n_cells)
    R = np.full(n_cells, 0.5)
    cells = np.stack([xs, zs, L, R], 1)
    w = rng.uniform(0.5, 1.5, n_cells)
    return cells, w, x0
