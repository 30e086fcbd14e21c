"""FP64 CPU reference of the steady glucose problem (bcg_steady_*) and its
adjoint gradients, with scipy sparse direct solves.  Test infrastructure:
the checker of the CUDA solver in tests/test_steady.py.

Discretisation (the same as the library's): vertices (i, k) of an nx x nz
grid at spacing h, row 0 held at c0; at every other vertex
    F = sum_faces Df (C_nb - C) / h^2 - q vmax C / (km + C) = 0,
Df the harmonic mean of the two vertices' diffusivities (d_agar on rows
k < nz_agar, d_colony above), no flux through the other sides, q the
deposited w L R / h^2 of the cells whose centre rounds to the vertex.
"""
import numpy as np
import scipy.sparse as sps
import scipy.sparse.linalg as spla


def _face(a, b):
    return np.where(a == b, a, 2 * a * b / (a + b))


def deposit(nx, nz, nz_agar, h, cells, w):
    q = np.zeros((nz, nx))
    i = np.rint(cells[:, 0] / h).astype(int)
    k = np.rint(cells[:, 1] / h).astype(int)
    ok = (i >= 0) & (i < nx) & (k >= nz_agar) & (k < nz)
    np.add.at(q, (k[ok], i[ok]), w[ok] * cells[ok, 2] * cells[ok, 3])
    return q / (h * h), np.where(ok, k * nx + i, -1)


def laplacian(nx, nz, nz_agar, h, d_agar, d_col):
    """Sparse operator Lap (n x n): Lap C = sum_faces Df (C_nb - C)/h^2 at
    rows >= 1; rows of row 0 are empty (Dirichlet handled by the caller)."""
    dpt = np.where(np.arange(nz)[:, None] < nz_agar, d_agar, d_col) * np.ones((nz, nx))
    n = nx * nz
    rows, cols, vals = [], [], []
    for k in range(1, nz):
        for i in range(nx):
            p = k * nx + i
            for (kk, ii) in ((k - 1, i), (k + 1, i), (k, i - 1), (k, i + 1)):
                if 0 <= kk < nz and 0 <= ii < nx:
                    df = _face(dpt[k, i], dpt[kk, ii]) / (h * h)
                    rows += [p, p]; cols += [kk * nx + ii, p]; vals += [df, -df]
    return sps.csr_matrix((vals, (rows, cols)), shape=(n, n))


class SteadyRef:
    def __init__(self, nx, nz, nz_agar, h, c0, cells):
        self.nx, self.nz, self.nz_agar, self.h, self.c0 = nx, nz, nz_agar, h, c0
        self.cells = np.asarray(cells, dtype=np.float64).reshape(-1, 4)

    def _F(self, C, q, Lap, vmax, km):
        F = Lap @ C - q * vmax * C / (km + C)
        F[:self.nx] = 0.0
        return F

    def solve(self, theta, w, tol=1e-14):
        d_agar, d_col, vmax, km = theta
        nx, nz = self.nx, self.nz
        q, self.pt = deposit(nx, nz, self.nz_agar, self.h, self.cells, np.asarray(w, dtype=np.float64))
        q = q.reshape(-1)
        Lap = laplacian(nx, nz, self.nz_agar, self.h, d_agar, d_col)
        C = np.full(nx * nz, float(self.c0))
        free = np.arange(nx, nx * nz)
        f0 = None
        for it in range(60):
            F = self._F(C, q, Lap, vmax, km)
            fn = np.abs(F).max()
            f0 = f0 or (fn if fn > 0 else 1.0)
            if fn <= tol * f0:
                break
            J = Lap - sps.diags(q * vmax * km / (km + C) ** 2)
            Jf = J[free][:, free].tocsc()
            C[free] -= spla.spsolve(Jf, F[free])
        self.C, self.q, self.Lap, self.theta = C, q, Lap, np.asarray(theta, dtype=np.float64)
        return C.reshape(nz, nx)

    def gradients(self, dL_dC):
        """dL/dtheta (4) and dL/dw via the adjoint of the converged state."""
        d_agar, d_col, vmax, km = self.theta
        nx, nz, h = self.nx, self.nz, self.h
        C, q = self.C, self.q
        free = np.arange(nx, nx * nz)
        J = self.Lap - sps.diags(q * vmax * km / (km + C) ** 2)
        lam = np.zeros(nx * nz)
        lam[free] = spla.spsolve(J[free][:, free].T.tocsc(), np.asarray(dL_dC, dtype=np.float64).reshape(-1)[free])
        # dL/dtheta = -lam . dF/dtheta, with the analytic face derivatives
        dLap_da, dLap_dc = self._dlap(d_agar, d_col)
        g = np.zeros(4)
        g[0] = -lam @ (dLap_da @ C)
        g[1] = -lam @ (dLap_dc @ C)
        g[2] = lam @ (q * C / (km + C))
        g[3] = -lam @ (q * vmax * C / (km + C) ** 2)
        gw = np.zeros(len(self.cells))
        ok = self.pt >= 0
        p = self.pt[ok]
        gw[ok] = lam[p] * self.cells[ok, 2] * self.cells[ok, 3] / (h * h) * vmax * C[p] / (km + C[p])
        return g, gw

    def _dlap(self, da, dc):
        nx, nz, h, na = self.nx, self.nz, self.h, self.nz_agar
        n = nx * nz
        out = []
        for wrt in (0, 1):
            rows, cols, vals = [], [], []
            for k in range(1, nz):
                for i in range(nx):
                    p = k * nx + i
                    for (kk, ii) in ((k - 1, i), (k + 1, i), (k, i - 1), (k, i + 1)):
                        if not (0 <= kk < nz and 0 <= ii < nx):
                            continue
                        pa, nb = k < na, kk < na
                        if pa and nb:
                            dd = 1.0 if wrt == 0 else 0.0
                        elif not pa and not nb:
                            dd = 1.0 if wrt == 1 else 0.0
                        else:
                            s = da + dc
                            dd = 2 * dc * dc / s ** 2 if wrt == 0 else 2 * da * da / s ** 2
                        if dd:
                            rows += [p, p]; cols += [kk * nx + ii, p]; vals += [dd / (h * h), -dd / (h * h)]
            out.append(sps.csr_matrix((vals, (rows, cols)), shape=(n, n)))
        return out
