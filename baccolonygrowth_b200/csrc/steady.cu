/*
 * steady.cu -- steady glucose field of a colony and its adjoint (VJP).
 * No counterpart in the reference: an extension for gradients of a
 * nutrient-profile loss with respect to the diffusivities, the Monod
 * constants and per-cell uptake weights.
 *
 * Problem (2-D x-z grid, nx x nz vertices, spacing h; rows k < nz_agar
 * are agar, the rest the colony region):
 *   F_p(C) = sum_faces Df (C_nb - C_p) / h^2 - q_p vmax C_p / (km + C_p) = 0
 * for k >= 1, C = c0 on row 0 (the agar reservoir), no flux through the
 * other sides.  A point's diffusivity is d_agar or d_colony by its row,
 * a face takes the harmonic mean of its two points.  The uptake density
 * q_p = sum over cells whose centre rounds to p of w_c L_c R_c / h^2 (the
 * deposition GetDensity makes, Compute.cpp:120-253, with a weight per
 * cell: its growth rate).
 *
 * Solve: Newton, each step A delta = F with A = -dF/dC (symmetric positive
 * definite: the diffusion operator plus diag(q vmax km / (km + C)^2)),
 * by conjugate gradients preconditioned with one symmetric V-cycle
 * (red-black Gauss-Seidel, bilinear prolongation, its transpose / 4 as
 * restriction, coarse operators rediscretised at 2h).
 * Adjoint: for a loss L(C), A lambda = -dL/dC at the converged C (A is
 * symmetric), then dL/dtheta = -lambda . dF/dtheta.  This is the exact
 * gradient of the converged solution (implicit function theorem): the
 * V-cycles and Newton steps are not replayed, only the converged state is
 * kept, so memory does not grow with the iteration count.
 * All arithmetic FP64; every reduction runs in a fixed order.
 */
#include "ctx.cuh"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <vector>

#define ST_MAX_LEVELS 12
#define ST_RED_BLOCKS 256

struct StLevel {
    int nx, nz;
    double h;
    double* x;     /* correction / solution of this level's system */
    double* b;     /* right-hand side */
    double* r;     /* residual */
    double* sig;   /* diagonal term */
    double* dpt;   /* point diffusivity */
};

struct bcg_steady {
    bcg_steady_params P;
    cudaStream_t stream;
    int nlev;
    StLevel L[ST_MAX_LEVELS];
    int n;                       /* nx * nz */
    double *C, *q, *F, *lam, *g;
    double *cg_r, *cg_z, *cg_p, *cg_ap;
    double *part, *scal;         /* reduction partials, scalars */
    int ncell;
    double* cell;                /* x, z, L, R per cell */
    int* cell_pt;                /* grid point of each cell, -1 outside the colony rows */
    double* w;
    double* gw;
    double* gpart;               /* per-block partial sums of the 4 parameter gradients */
    double theta[4];             /* parameters of the last solve */
    bool solved;
};

static int st_err(cudaError_t e) { if (e != cudaSuccess) { bcg_set_cuda_error(e); return BCG_E_CUDA; } return BCG_OK; }
#define ST_TRY(x) do { int r_ = st_err(x); if (r_) return r_; } while (0)

__device__ __forceinline__ double face_d(double a, double b) { return a == b ? a : 2.0 * a * b / (a + b); }

/* ---- operator pieces on one level --------------------------------------- */
/* (A x)_p = sum_f Df (x_p - x_nb) / h^2 + sig_p x_p for rows k >= 1; row 0
 * is the Dirichlet row (x = 0 there) */
__device__ __forceinline__ void st_coeffs(const StLevel& L, int i, int k, double& diag, double& off_sum,
                                          const double* x)
{
    const double ih2 = 1.0 / (L.h * L.h);
    const double dp = L.dpt[k * L.nx + i];
    diag = L.sig[k * L.nx + i];
    off_sum = 0.0;
    /* below (row k-1, Dirichlet when k-1 == 0: x = 0 there) */
    {
        double df = face_d(dp, L.dpt[(k - 1) * L.nx + i]) * ih2;
        diag += df;
        if (k - 1 > 0) off_sum += df * x[(k - 1) * L.nx + i];
    }
    if (k + 1 < L.nz) { double df = face_d(dp, L.dpt[(k + 1) * L.nx + i]) * ih2; diag += df; off_sum += df * x[(k + 1) * L.nx + i]; }
    if (i > 0) { double df = face_d(dp, L.dpt[k * L.nx + i - 1]) * ih2; diag += df; off_sum += df * x[k * L.nx + i - 1]; }
    if (i + 1 < L.nx) { double df = face_d(dp, L.dpt[k * L.nx + i + 1]) * ih2; diag += df; off_sum += df * x[k * L.nx + i + 1]; }
}

__global__ void k_st_apply(StLevel L, const double* __restrict__ x, double* __restrict__ y)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= L.nx * L.nz) return;
    int i = p % L.nx, k = p / L.nx;
    if (k == 0) { y[p] = 0.0; return; }
    double diag, off;
    st_coeffs(L, i, k, diag, off, x);
    y[p] = diag * x[p] - off;
}

/* r = b - A x */
__global__ void k_st_resid(StLevel L)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= L.nx * L.nz) return;
    int i = p % L.nx, k = p / L.nx;
    if (k == 0) { L.r[p] = 0.0; return; }
    double diag, off;
    st_coeffs(L, i, k, diag, off, L.x);
    L.r[p] = L.b[p] - (diag * L.x[p] - off);
}

/* one colour of red-black Gauss-Seidel; nx is odd, so a point's colour
 * (i + k) & 1 is the parity of its index p = k*nx + i */
__global__ void k_st_rbgs(StLevel L, int colour)
{
    int p = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + colour;
    if (p >= L.nx * L.nz) return;
    int i = p % L.nx, k = p / L.nx;
    if (k == 0) return;
    double diag, off;
    st_coeffs(L, i, k, diag, off, L.x);
    L.x[p] = (L.b[p] + off) / diag;
}

/* coarse b = restriction (transpose of bilinear prolongation, / 4) of fine r */
__global__ void k_st_restrict(StLevel Lc, StLevel Lf)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= Lc.nx * Lc.nz) return;
    int I = p % Lc.nx, K = p / Lc.nx;
    Lc.x[p] = 0.0;
    if (K == 0) { Lc.b[p] = 0.0; return; }
    double s = 0.0;
    for (int dk = -1; dk <= 1; dk++) {
        int k = 2 * K + dk;
        if (k <= 0 || k >= Lf.nz) continue;
        double wk = dk == 0 ? 1.0 : 0.5;
        for (int di = -1; di <= 1; di++) {
            int i = 2 * I + di;
            if (i < 0 || i >= Lf.nx) continue;
            double wi = di == 0 ? 1.0 : 0.5;
            s += wi * wk * Lf.r[k * Lf.nx + i];
        }
    }
    Lc.b[p] = 0.25 * s;
}

/* fine x += bilinear prolongation of coarse x */
__global__ void k_st_prolong(StLevel Lf, StLevel Lc)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= Lf.nx * Lf.nz) return;
    int i = p % Lf.nx, k = p / Lf.nx;
    if (k == 0) return;
    int I0 = i / 2, K0 = k / 2;
    int I1 = (i & 1) ? I0 + 1 : I0, K1 = (k & 1) ? K0 + 1 : K0;
    double v = 0.25 * (Lc.x[K0 * Lc.nx + I0] + Lc.x[K0 * Lc.nx + I1] + Lc.x[K1 * Lc.nx + I0] + Lc.x[K1 * Lc.nx + I1]);
    Lf.x[p] += v;
}

/* coarse point diffusivity (injection) and diagonal term (weighted
 * average of the fine one over the restriction stencil) */
__global__ void k_st_coarse_coeffs(StLevel Lc, StLevel Lf)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= Lc.nx * Lc.nz) return;
    int I = p % Lc.nx, K = p / Lc.nx;
    Lc.dpt[p] = Lf.dpt[(2 * K) * Lf.nx + 2 * I];
    double s = 0.0, ws = 0.0;
    for (int dk = -1; dk <= 1; dk++) {
        int k = 2 * K + dk;
        if (k < 0 || k >= Lf.nz) continue;
        double wk = dk == 0 ? 1.0 : 0.5;
        for (int di = -1; di <= 1; di++) {
            int i = 2 * I + di;
            if (i < 0 || i >= Lf.nx) continue;
            double wi = di == 0 ? 1.0 : 0.5;
            s += wi * wk * Lf.sig[k * Lf.nx + i];
            ws += wi * wk;
        }
    }
    Lc.sig[p] = s / ws;
}

/* ---- problem-specific kernels ------------------------------------------ */
__global__ void k_st_init(int n, int nx, int nz_agar, double d_agar, double d_col, double c0,
                          double* dpt, double* C, double* q)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int k = p / nx;
    dpt[p] = k < nz_agar ? d_agar : d_col;
    C[p] = c0;
    q[p] = 0.0;
}

/* deposition of the cells' weighted L*R (one thread per grid point,
 * cells pre-sorted by point on the host, so the sum order is fixed) */
__global__ void k_st_deposit(int n, double h, const int* __restrict__ start, const int* __restrict__ order,
                             const double* __restrict__ cell, const double* __restrict__ w, double* __restrict__ q)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    double s = 0.0;
    for (int j = start[p]; j < start[p + 1]; j++) {
        int c = order[j];
        s += w[c] * cell[4 * c + 2] * cell[4 * c + 3];
    }
    q[p] = s / (h * h);
}

/* F(C) (the Newton right-hand side b = F) and the linearised diagonal */
__global__ void k_st_newton_rhs(StLevel L, const double* __restrict__ C, const double* __restrict__ q,
                                double vmax, double km, double* __restrict__ F)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= L.nx * L.nz) return;
    int i = p % L.nx, k = p / L.nx;
    if (k == 0) { F[p] = 0.0; L.sig[p] = 0.0; L.b[p] = 0.0; return; }
    const double ih2 = 1.0 / (L.h * L.h);
    const double dp = L.dpt[p];
    double flux = 0.0;
    flux += face_d(dp, L.dpt[p - L.nx]) * ih2 * (C[p - L.nx] - C[p]);
    if (k + 1 < L.nz) flux += face_d(dp, L.dpt[p + L.nx]) * ih2 * (C[p + L.nx] - C[p]);
    if (i > 0) flux += face_d(dp, L.dpt[p - 1]) * ih2 * (C[p - 1] - C[p]);
    if (i + 1 < L.nx) flux += face_d(dp, L.dpt[p + 1]) * ih2 * (C[p + 1] - C[p]);
    const double c = C[p];
    const double f = flux - q[p] * vmax * c / (km + c);
    F[p] = f;
    L.b[p] = f;
    L.sig[p] = q[p] * vmax * km / ((km + c) * (km + c));
}

/* deterministic dot product / max-norm: per-block partials, then one block */
__global__ void k_st_dot_part(int n, const double* __restrict__ a, const double* __restrict__ b, double* part, int mode)
{
    __shared__ double sh[256];
    double s = 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        s = mode == 0 ? s + a[p] * b[p] : fmax(s, fabs(a[p]));
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] = mode == 0 ? sh[threadIdx.x] + sh[threadIdx.x + o] : fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}
__global__ void k_st_dot_final(int nb, const double* part, double* out, int mode)
{
    __shared__ double sh[256];
    double s = 0.0;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) s = mode == 0 ? s + part[j] : fmax(s, part[j]);
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] = mode == 0 ? sh[threadIdx.x] + sh[threadIdx.x + o] : fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

/* y = a*x + y, or y = x + a*y (mode 1) */
__global__ void k_st_axpy(int n, const double* __restrict__ a, int neg, const double* __restrict__ x, double* __restrict__ y, int mode)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    double s = neg ? -*a : *a;
    y[p] = mode == 0 ? y[p] + s * x[p] : x[p] + s * y[p];
}
__global__ void k_st_ratio(const double* num, const double* den, double* out) { *out = *den != 0.0 ? *num / *den : 0.0; }
__global__ void k_st_add(int n, const double* __restrict__ x, double* __restrict__ y) { int p = blockIdx.x * blockDim.x + threadIdx.x; if (p < n) y[p] += x[p]; }
/* dst = -src, zero on the Dirichlet row */
__global__ void k_st_neg(int n, int nx, const double* __restrict__ src, double* __restrict__ dst)
{ int p = blockIdx.x * blockDim.x + threadIdx.x; if (p < n) dst[p] = p < nx ? 0.0 : -src[p]; }
__global__ void k_st_copy(int n, const double* __restrict__ a, double* __restrict__ b) { int p = blockIdx.x * blockDim.x + threadIdx.x; if (p < n) b[p] = a[p]; }

/* gradients: per point contributions to dL/d(d_agar, d_colony, vmax, km),
 * reduced per block in fixed order; and dL/dw per cell */
__global__ void k_st_grad_part(StLevel L, int nz_agar, double d_agar, double d_col, const double* __restrict__ C,
                               const double* __restrict__ q, const double* __restrict__ lam, double vmax, double km,
                               double* gpart)
{
    __shared__ double sh[4][256];
    double g[4] = {0, 0, 0, 0};
    const double ih2 = 1.0 / (L.h * L.h);
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < L.nx * L.nz; p += gridDim.x * blockDim.x) {
        int i = p % L.nx, k = p / L.nx;
        if (k == 0) continue;
        const double lp = lam[p], c = C[p];
        /* dF_p/d(d) summed over p's faces */
        double dfa = 0.0, dfc = 0.0;
        auto face = [&](int pn, int kn) {
            const bool pa = k < nz_agar, na = kn < nz_agar;
            const double dc = C[pn] - c;
            if (pa && na) dfa += dc * ih2;
            else if (!pa && !na) dfc += dc * ih2;
            else {
                /* harmonic mean 2 a b / (a + b): d/da = 2 b^2 / (a + b)^2 */
                const double s = d_agar + d_col;
                dfa += 2.0 * d_col * d_col / (s * s) * dc * ih2;
                dfc += 2.0 * d_agar * d_agar / (s * s) * dc * ih2;
            }
        };
        face(p - L.nx, k - 1);
        if (k + 1 < L.nz) face(p + L.nx, k + 1);
        if (i > 0) face(p - 1, k);
        if (i + 1 < L.nx) face(p + 1, k);
        /* dL/dtheta = -lambda . dF/dtheta */
        g[0] -= lp * dfa;
        g[1] -= lp * dfc;
        g[2] += lp * q[p] * c / (km + c);
        g[3] -= lp * q[p] * vmax * c / ((km + c) * (km + c));
    }
    for (int j = 0; j < 4; j++) sh[j][threadIdx.x] = g[j];
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) for (int j = 0; j < 4; j++) sh[j][threadIdx.x] += sh[j][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) for (int j = 0; j < 4; j++) gpart[4 * blockIdx.x + j] = sh[j][0];
}

__global__ void k_st_grad_w(int ncell, double h, const double* __restrict__ cell, const int* __restrict__ cell_pt,
                            const double* __restrict__ C, const double* __restrict__ lam, double vmax, double km,
                            double* __restrict__ gw)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    int p = cell_pt[c];
    if (p < 0) { gw[c] = 0.0; return; }
    const double cc = C[p];
    /* dF_p/dw_c = -(L R / h^2) vmax C / (km + C) */
    gw[c] = lam[p] * cell[4 * c + 2] * cell[4 * c + 3] / (h * h) * vmax * cc / (km + cc);
}

/* ---- host side ---------------------------------------------------------- */
static unsigned nblk(int n) { return (unsigned)((n + 255) / 256); }

static void st_vcycle(bcg_steady* s, int l)
{
    StLevel& L = s->L[l];
    const int n = L.nx * L.nz;
    if (l == s->nlev - 1) {
        for (int j = 0; j < 40; j++) { k_st_rbgs<<<nblk((n + 1) / 2), 256, 0, s->stream>>>(L, 0); k_st_rbgs<<<nblk((n + 1) / 2), 256, 0, s->stream>>>(L, 1); }
        for (int j = 0; j < 40; j++) { k_st_rbgs<<<nblk((n + 1) / 2), 256, 0, s->stream>>>(L, 1); k_st_rbgs<<<nblk((n + 1) / 2), 256, 0, s->stream>>>(L, 0); }
        return;
    }
    for (int j = 0; j < 2; j++) { k_st_rbgs<<<nblk((n + 1) / 2), 256, 0, s->stream>>>(L, 0); k_st_rbgs<<<nblk((n + 1) / 2), 256, 0, s->stream>>>(L, 1); }
    k_st_resid<<<nblk(n), 256, 0, s->stream>>>(L);
    StLevel& Lc = s->L[l + 1];
    k_st_restrict<<<nblk(Lc.nx * Lc.nz), 256, 0, s->stream>>>(Lc, L);
    st_vcycle(s, l + 1);
    k_st_prolong<<<nblk(n), 256, 0, s->stream>>>(L, Lc);
    for (int j = 0; j < 2; j++) { k_st_rbgs<<<nblk((n + 1) / 2), 256, 0, s->stream>>>(L, 1); k_st_rbgs<<<nblk((n + 1) / 2), 256, 0, s->stream>>>(L, 0); }
}

/* z = M^-1 r with M one symmetric V-cycle from zero */
static void st_precond(bcg_steady* s, const double* r, double* z)
{
    StLevel& L = s->L[0];
    const int n = L.nx * L.nz;
    k_st_copy<<<nblk(n), 256, 0, s->stream>>>(n, r, L.b);
    cudaMemsetAsync(L.x, 0, sizeof(double) * n, s->stream);
    st_vcycle(s, 0);
    k_st_copy<<<nblk(n), 256, 0, s->stream>>>(n, L.x, z);
}

static int st_reduce(bcg_steady* s, const double* a, const double* b, int n, int mode, int slot)
{
    k_st_dot_part<<<ST_RED_BLOCKS, 256, 0, s->stream>>>(n, a, b, s->part, mode);
    k_st_dot_final<<<1, 256, 0, s->stream>>>(ST_RED_BLOCKS, s->part, s->scal + slot, mode);
    return st_err(cudaGetLastError());
}

static int st_read(bcg_steady* s, int slot, double* v)
{
    ST_TRY(cudaMemcpyAsync(v, s->scal + slot, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    ST_TRY(cudaStreamSynchronize(s->stream));
    return BCG_OK;
}

/* solve A x = rhs (A from the current level-0 sig/dpt) by PCG to
 * ||r||_inf <= tol * ||rhs||_inf; x in L[0]-sized buffer `x` */
static int st_pcg(bcg_steady* s, const double* rhs, double* x, double tol, int max_it, int* iters)
{
    StLevel& L = s->L[0];
    const int n = L.nx * L.nz;
    /* coarse diagonals for this linearisation */
    for (int l = 1; l < s->nlev; l++)
        k_st_coarse_coeffs<<<nblk(s->L[l].nx * s->L[l].nz), 256, 0, s->stream>>>(s->L[l], s->L[l - 1]);
    cudaMemsetAsync(x, 0, sizeof(double) * n, s->stream);
    k_st_copy<<<nblk(n), 256, 0, s->stream>>>(n, rhs, s->cg_r);
    int rc;
    double bnorm;
    if ((rc = st_reduce(s, rhs, rhs, n, 1, 0)) || (rc = st_read(s, 0, &bnorm))) return rc;
    *iters = 0;
    if (bnorm == 0.0) return BCG_OK;
    st_precond(s, s->cg_r, s->cg_z);
    k_st_copy<<<nblk(n), 256, 0, s->stream>>>(n, s->cg_z, s->cg_p);
    if ((rc = st_reduce(s, s->cg_r, s->cg_z, n, 0, 1))) return rc;        /* rz */
    for (int it = 1; it <= max_it; it++) {
        k_st_apply<<<nblk(n), 256, 0, s->stream>>>(L, s->cg_p, s->cg_ap);
        if ((rc = st_reduce(s, s->cg_p, s->cg_ap, n, 0, 2))) return rc;   /* pAp */
        k_st_ratio<<<1, 1, 0, s->stream>>>(s->scal + 1, s->scal + 2, s->scal + 3);   /* alpha */
        k_st_axpy<<<nblk(n), 256, 0, s->stream>>>(n, s->scal + 3, 0, s->cg_p, x, 0);
        k_st_axpy<<<nblk(n), 256, 0, s->stream>>>(n, s->scal + 3, 1, s->cg_ap, s->cg_r, 0);
        double rn;
        if ((rc = st_reduce(s, s->cg_r, s->cg_r, n, 1, 4)) || (rc = st_read(s, 4, &rn))) return rc;
        *iters = it;
        if (rn <= tol * bnorm) break;
        st_precond(s, s->cg_r, s->cg_z);
        if ((rc = st_reduce(s, s->cg_r, s->cg_z, n, 0, 5))) return rc;   /* rz new */
        k_st_ratio<<<1, 1, 0, s->stream>>>(s->scal + 5, s->scal + 1, s->scal + 6);   /* beta */
        k_st_copy<<<1, 1, 0, s->stream>>>(1, s->scal + 5, s->scal + 1);
        k_st_axpy<<<nblk(n), 256, 0, s->stream>>>(n, s->scal + 6, 0, s->cg_z, s->cg_p, 1);   /* p = z + beta p */
    }
    return st_err(cudaGetLastError());
}

extern "C" int bcg_steady_create(const bcg_steady_params* p, bcg_steady** out)
{
    if (!p || !out) return BCG_E_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return BCG_E_NO_DEVICE;
    auto pow2p1 = [](int v) { return v >= 3 && (((v - 1) & (v - 2)) == 0); };
    if (!pow2p1(p->nx) || !pow2p1(p->nz) || p->nz_agar < 1 || p->nz_agar > p->nz || !(p->h > 0) || p->max_cells < 0)
        return BCG_E_ARG;
    bcg_steady* s = (bcg_steady*)calloc(1, sizeof(bcg_steady));
    if (!s) return BCG_E_ARG;
    s->P = *p;
    int rc = BCG_OK;
#define ST_ALLOC(ptr, bytes) do { if (!rc) rc = st_err(cudaMalloc((void**)&(ptr), (bytes))); } while (0)
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) { free(s); return BCG_E_CUDA; }
    int nx = p->nx, nz = p->nz;
    double h = p->h;
    s->nlev = 0;
    while (s->nlev < ST_MAX_LEVELS) {
        StLevel& L = s->L[s->nlev];
        L.nx = nx; L.nz = nz; L.h = h;
        size_t b = sizeof(double) * (size_t)nx * nz;
        ST_ALLOC(L.x, b); ST_ALLOC(L.b, b); ST_ALLOC(L.r, b); ST_ALLOC(L.sig, b); ST_ALLOC(L.dpt, b);
        s->nlev++;
        if (nx <= 3 || nz <= 3) break;
        nx = (nx + 1) / 2; nz = (nz + 1) / 2; h *= 2;
    }
    s->n = p->nx * p->nz;
    size_t b = sizeof(double) * (size_t)s->n;
    ST_ALLOC(s->C, b); ST_ALLOC(s->q, b); ST_ALLOC(s->F, b); ST_ALLOC(s->lam, b); ST_ALLOC(s->g, b);
    ST_ALLOC(s->cg_r, b); ST_ALLOC(s->cg_z, b); ST_ALLOC(s->cg_p, b); ST_ALLOC(s->cg_ap, b);
    ST_ALLOC(s->part, sizeof(double) * ST_RED_BLOCKS);
    ST_ALLOC(s->scal, sizeof(double) * 16);
    ST_ALLOC(s->gpart, sizeof(double) * 4 * ST_RED_BLOCKS);
    int mc = p->max_cells > 0 ? p->max_cells : 1;
    ST_ALLOC(s->cell, sizeof(double) * 4 * mc);
    ST_ALLOC(s->cell_pt, sizeof(int) * mc);
    ST_ALLOC(s->w, sizeof(double) * mc);
    ST_ALLOC(s->gw, sizeof(double) * mc);
#undef ST_ALLOC
    if (rc) { bcg_steady_destroy(s); return rc; }
    *out = s;
    return BCG_OK;
}

extern "C" int bcg_steady_destroy(bcg_steady* s)
{
    if (!s) return BCG_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (int l = 0; l < s->nlev; l++) { cudaFree(s->L[l].x); cudaFree(s->L[l].b); cudaFree(s->L[l].r); cudaFree(s->L[l].sig); cudaFree(s->L[l].dpt); }
    void* ptrs[] = {s->C, s->q, s->F, s->lam, s->g, s->cg_r, s->cg_z, s->cg_p, s->cg_ap, s->part, s->scal, s->gpart,
                    s->cell, s->cell_pt, s->w, s->gw};
    for (void* q : ptrs) if (q) cudaFree(q);
    if (s->stream) cudaStreamDestroy(s->stream);
    free(s);
    return BCG_OK;
}

/* cell centres (x from the grid's left edge, z from the agar bottom),
 * lengths and radii: 4 doubles per cell */
extern "C" int bcg_steady_set_cells(bcg_steady* s, const double* xzlr, int ncell)
{
    if (!s || ncell < 0 || ncell > s->P.max_cells || (ncell > 0 && !xzlr)) return BCG_E_ARG;
    s->ncell = ncell;
    s->solved = false;
    if (ncell == 0) return BCG_OK;
    ST_TRY(cudaMemcpy(s->cell, xzlr, sizeof(double) * 4 * (size_t)ncell, cudaMemcpyHostToDevice));
    std::vector<int> pt(ncell);
    const int nx = s->P.nx, nz = s->P.nz;
    for (int c = 0; c < ncell; c++) {
        long i = lround(xzlr[4 * c] / s->P.h), k = lround(xzlr[4 * c + 1] / s->P.h);
        pt[c] = (i >= 0 && i < nx && k >= s->P.nz_agar && k < nz) ? (int)(k * nx + i) : -1;
    }
    ST_TRY(cudaMemcpy(s->cell_pt, pt.data(), sizeof(int) * ncell, cudaMemcpyHostToDevice));
    return BCG_OK;
}

static int st_deposit(bcg_steady* s, const double* w_host)
{
    const int n = s->n, nc = s->ncell;
    std::vector<int> pt(nc), start(n + 1, 0), order(nc);
    if (nc) ST_TRY(cudaMemcpy(pt.data(), s->cell_pt, sizeof(int) * nc, cudaMemcpyDeviceToHost));
    for (int c = 0; c < nc; c++) if (pt[c] >= 0) start[pt[c] + 1]++;
    for (int p = 0; p < n; p++) start[p + 1] += start[p];
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (int c = 0; c < nc; c++) if (pt[c] >= 0) order[fill[pt[c]]++] = c;
    int *d_start = nullptr, *d_order = nullptr;
    ST_TRY(cudaMallocAsync((void**)&d_start, sizeof(int) * (n + 1), s->stream));
    ST_TRY(cudaMallocAsync((void**)&d_order, sizeof(int) * (nc > 0 ? nc : 1), s->stream));
    ST_TRY(cudaMemcpyAsync(d_start, start.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s->stream));
    if (nc) ST_TRY(cudaMemcpyAsync(d_order, order.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, s->stream));
    if (nc) ST_TRY(cudaMemcpyAsync(s->w, w_host, sizeof(double) * nc, cudaMemcpyHostToDevice, s->stream));
    k_st_deposit<<<nblk(n), 256, 0, s->stream>>>(n, s->P.h, d_start, d_order, s->cell, s->w, s->q);
    cudaFreeAsync(d_start, s->stream);
    cudaFreeAsync(d_order, s->stream);
    ST_TRY(cudaStreamSynchronize(s->stream));
    return BCG_OK;
}

extern "C" int bcg_steady_solve(bcg_steady* s, const double* theta, const double* w, double tol,
                                double* C_out, int* newton_iters, int* cg_iters)
{
    if (!s || !theta || (s->ncell > 0 && !w)) return BCG_E_ARG;
    const double d_agar = theta[0], d_col = theta[1], vmax = theta[2], km = theta[3];
    if (!(d_agar > 0) || !(d_col > 0) || !(km > 0) || !(tol > 0)) return BCG_E_ARG;
    const int n = s->n;
    StLevel& L = s->L[0];
    k_st_init<<<nblk(n), 256, 0, s->stream>>>(n, s->P.nx, s->P.nz_agar, d_agar, d_col, s->P.c0, L.dpt, s->C, s->q);
    for (int l = 1; l < s->nlev; l++)
        k_st_coarse_coeffs<<<nblk(s->L[l].nx * s->L[l].nz), 256, 0, s->stream>>>(s->L[l], s->L[l - 1]);
    int rc = st_deposit(s, w);
    if (rc) return rc;
    int it = 0, cgt = 0;
    double f0 = 0.0;
    for (; it < 50; it++) {
        k_st_newton_rhs<<<nblk(n), 256, 0, s->stream>>>(L, s->C, s->q, vmax, km, s->F);
        double fn;
        if ((rc = st_reduce(s, s->F, s->F, n, 1, 7)) || (rc = st_read(s, 7, &fn))) return rc;
        if (it == 0) f0 = fn > 0 ? fn : 1.0;
        if (fn <= tol * f0 || fn == 0.0) break;
        int ci = 0;
        const double cg_tol = tol < 1e-8 ? (tol > 1e-14 ? tol : 1e-14) : 1e-8;
        if ((rc = st_pcg(s, s->F, s->g, cg_tol, 200, &ci))) return rc;
        cgt += ci;
        k_st_add<<<nblk(n), 256, 0, s->stream>>>(n, s->g, s->C);   /* C += delta */
    }
    /* keep the converged linearisation (sig, coarse diagonals) for the adjoint */
    k_st_newton_rhs<<<nblk(n), 256, 0, s->stream>>>(L, s->C, s->q, vmax, km, s->F);
    s->solved = true;
    memcpy(s->theta, theta, sizeof(s->theta));
    if (C_out) ST_TRY(cudaMemcpyAsync(C_out, s->C, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
    ST_TRY(cudaStreamSynchronize(s->stream));
    if (newton_iters) *newton_iters = it;
    if (cg_iters) *cg_iters = cgt;
    return BCG_OK;
}

extern "C" int bcg_steady_vjp(bcg_steady* s, const double* dL_dC, double* grad_theta, double* grad_w, double tol)
{
    if (!s || !dL_dC || !grad_theta || !s->solved || !(tol > 0)) return BCG_E_ARG;
    const int n = s->n;
    StLevel& L = s->L[0];
    /* A lambda = -dL/dC (row 0 is fixed: no adjoint there) */
    ST_TRY(cudaMemcpyAsync(s->cg_ap, dL_dC, sizeof(double) * n, cudaMemcpyHostToDevice, s->stream));
    k_st_neg<<<nblk(n), 256, 0, s->stream>>>(n, s->P.nx, s->cg_ap, s->g);   /* g = -dL/dC, 0 on row 0 */
    int ci = 0;
    int rc = st_pcg(s, s->g, s->lam, tol, 500, &ci);
    if (rc) return rc;
    const double* th = s->theta;
    k_st_grad_part<<<ST_RED_BLOCKS, 256, 0, s->stream>>>(L, s->P.nz_agar, th[0], th[1], s->C, s->q, s->lam, th[2], th[3], s->gpart);
    std::vector<double> gp(4 * ST_RED_BLOCKS);
    ST_TRY(cudaMemcpyAsync(gp.data(), s->gpart, sizeof(double) * gp.size(), cudaMemcpyDeviceToHost, s->stream));
    if (grad_w && s->ncell > 0) {
        k_st_grad_w<<<nblk(s->ncell), 256, 0, s->stream>>>(s->ncell, s->P.h, s->cell, s->cell_pt, s->C, s->lam, th[2], th[3], s->gw);
        ST_TRY(cudaMemcpyAsync(grad_w, s->gw, sizeof(double) * s->ncell, cudaMemcpyDeviceToHost, s->stream));
    }
    ST_TRY(cudaStreamSynchronize(s->stream));
    for (int j = 0; j < 4; j++) {
        double t = 0.0;
        for (int b = 0; b < ST_RED_BLOCKS; b++) t += gp[4 * b + j];
        grad_theta[j] = t;
    }
    return BCG_OK;
}
