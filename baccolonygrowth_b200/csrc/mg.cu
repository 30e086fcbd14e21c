/*
 * mg.cu -- the composite-grid agar multigrid (class Multigrid,
 * AgentBasedModel-BacColonyGrowth/Multigrid.cpp:5-981) on the device.
 *
 * Each level holds Sol/Res/Err for carbon (0), oxygen (1), acetate (2),
 * (nx+1) x (nz+1) points, row k contiguous in i with a padded pitch.
 * Composite levels l < agarLevels are full size and each covers twice the
 * extent of the previous one at half the resolution; levels >= agarLevels
 * are plain coarsenings.  The smoother is the reference's zebra-column
 * Gauss-Seidel: all even columns, then all odd columns, each column swept
 * bottom to top in place (one thread per column and species).
 */
#include "ctx.cuh"
#include "mg.cuh"
#include "internal.h"
#include <string.h>
#include <cooperative_groups.h>

namespace cg = cooperative_groups;

__device__ __forceinline__ double dmaxd(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double dmind(double a, double b) { return a < b ? a : b; }

#define AT(arr, L, i, k) (arr)[(size_t)(k) * (L).pitch + (i)]

/* Read (i, k) with the reference's flat index i*(nz+1)+k: on levels with
 * nz <= 1 the stencils reach k = -1 or k = nz+1, which the reference's
 * Array3D maps onto the neighbouring column; an index past either end of
 * the array (undefined in the reference) reads as 0.  In range it is AT. */
template <class P, class LV>
__device__ __forceinline__ P at_ref(const P* a, const LV& L, int i, int k)
{
    if (k >= 0 && k <= L.nz) return AT(a, L, i, k);
    long f = (long)i * (L.nz + 1) + k;
    long n = (long)(L.nx + 1) * (L.nz + 1);
    if (f < 0 || f >= n) return P(0);
    int i2 = (int)(f / (L.nz + 1)), k2 = (int)(f % (L.nz + 1));
    return AT(a, L, i2, k2);
}

MgConst mg_const(const bcg_ctx* c, double dt)
{
    MgConst m;
    const bcg_params& P = c->P;
    m.A = P.max_levels_mg; m.levels = c->mg_levels; m.box_x = P.box_x; m.box_z_agar = P.box_z_agar;
    m.bl2 = P.box_length * P.box_length;
    m.dt = dt;
    m.D[0] = P.diff_agar_carbon; m.D[1] = P.diff_agar_o2; m.D[2] = P.diff_agar_ace;
    m.max_carbon = P.max_carbon; m.max_o2_agar = P.max_o2_agar;
    m.box_z = P.box_z;
    return m;
}

MgLvl mg_lvl(const bcg_ctx* c, int l)
{
    MgLvl v;
    const MgLevel& L = c->mg[l];
    v.nx = L.nx; v.nz = L.nz; v.pitch = L.pitch;
    for (int s = 0; s < 3; s++) { v.s[s] = L.sol[s]; v.r[s] = L.res[s]; v.e[s] = L.err[s]; v.e2[s] = L.err2[s]; }
    return v;
}

MgLvlF mg_lvl_f(const bcg_ctx* c, int l)
{
    MgLvlF v;
    const MgLevel& L = c->mg[l];
    v.nx = L.nx; v.nz = L.nz; v.pitch = L.pitch;
    for (int s = 0; s < 3; s++) { v.s[s] = L.sol[s]; v.r[s] = L.resf[s]; v.e[s] = L.errf[s]; v.e2[s] = L.errf2[s]; }
    return v;
}

/* ------------------------------------------------------------------------ */
/* relaxationAgarElementwise, Multigrid.cpp:160-249, for one species        */
/* ------------------------------------------------------------------------ */
template <class T>
__device__ __forceinline__ void relax_point(const MgConst& m, const MgLvlT<T>& L, int l, int sp, int i, int k,
                                            const double* __restrict__ inside0, T& e_below, bool have_below)
{
    const int nx = L.nx, nz = L.nz;
    const RelaxK<T> K = relax_k<T>(m, l, sp);
    T* E = SP(L.e);
    const T* R = SP(L.r);
    const bool oxy = (sp == 1);
    const bool top_levels = l >= m.A - 1;
    T r = AT(R, L, i, k);
    T e_dn = have_below ? e_below : (k > 0 ? AT(E, L, i, k - 1) : T(0));
    T out;
    bool write = true;
    if (k == 0) {
        int d = 1 << l;
        int i0 = (i - nx / 2) * d + m.box_x / 2;
        i0 = i0 < 0 ? 0 : (i0 > m.box_x - 1 ? m.box_x - 1 : i0);
        if (inside0[(size_t)i0 * m.box_z] > 0) out = r;
        else if (i == 0 || i == nx) {
            if (top_levels) {
                if (oxy) out = r;
                else out = rx_corner(r, (i == 0) ? AT(E, L, i + 1, 0) : AT(E, L, i - 1, 0), at_ref(E, L, i, 1), K);
            } else write = false;
        } else {
            if (oxy) out = r;
            else out = rx_k0(r, at_ref(E, L, i, 1), AT(E, L, i - 1, 0), AT(E, L, i + 1, 0), K);
        }
    } else if (k == nz) {
        if (top_levels) {
            if (i == 0 || i == nx) {
                if (oxy) out = r;
                else out = rx_corner(r, (i == 0) ? AT(E, L, i + 1, k) : AT(E, L, i - 1, k), e_dn, K);
            } else out = rx_top(r, e_dn, AT(E, L, i - 1, k), AT(E, L, i + 1, k), K);
        } else write = false;
    } else if (i == 0 || i == nx) {
        if (top_levels) {
            if (oxy) out = r;
            else out = rx_side(r, e_dn, AT(E, L, i, k + 1), (i == 0) ? AT(E, L, i + 1, k) : AT(E, L, i - 1, k), K);
        } else write = false;
    } else {
        out = rx_in(r, e_dn, AT(E, L, i, k + 1), AT(E, L, i - 1, k), AT(E, L, i + 1, k), K);
    }
    if (write) AT(E, L, i, k) = out;
    e_below = write ? out : AT(E, L, i, k);
}

/* Value the smoother would give point (i, k) of species sp (no write), and
 * whether the point is relaxed and how its update is scaled:
 * kind 0 = not relaxed, 1 = Dirichlet (E = R), 2 = E = (R c + N(E)) / (c + 2). */
template <class T>
__device__ __forceinline__ double relax_eval(const MgConst& m, const MgLvlT<T>& L, const double* __restrict__ R64,
                                             int l, int sp, int i, int k,
                                             const double* __restrict__ inside0, int& kind, double& cfac)
{
    const int nx = L.nx, nz = L.nz;
    const RelaxK<double> K = relax_k<double>(m, l, sp);
    const T* E = SP(L.e);
    const double r = AT(R64, L, i, k);
    const bool oxy = (sp == 1);
    const bool top_levels = l >= m.A - 1;
    cfac = K.cf;
    kind = 2;
    if (k == 0) {
        int d = 1 << l;
        int i0 = (i - nx / 2) * d + m.box_x / 2;
        i0 = i0 < 0 ? 0 : (i0 > m.box_x - 1 ? m.box_x - 1 : i0);
        if (inside0[(size_t)i0 * m.box_z] > 0) { kind = 1; return r; }
        if (i == 0 || i == nx) {
            if (!top_levels) { kind = 0; return 0.0; }
            if (oxy) { kind = 1; return r; }
            double s1 = (i == 0) ? (double)AT(E, L, i + 1, 0) : (double)AT(E, L, i - 1, 0);
            return rx_corner(r, s1, (double)at_ref(E, L, i, 1), K);
        }
        if (oxy) { kind = 1; return r; }
        return rx_k0(r, (double)at_ref(E, L, i, 1), (double)AT(E, L, i - 1, 0), (double)AT(E, L, i + 1, 0), K);
    }
    const double e_dn = (double)AT(E, L, i, k - 1);
    if (k == nz) {
        if (!top_levels) { kind = 0; return 0.0; }
        if (i == 0 || i == nx) {
            if (oxy) { kind = 1; return r; }
            double s1 = (i == 0) ? (double)AT(E, L, i + 1, k) : (double)AT(E, L, i - 1, k);
            return rx_corner(r, s1, e_dn, K);
        }
        return rx_top(r, e_dn, (double)AT(E, L, i - 1, k), (double)AT(E, L, i + 1, k), K);
    }
    if (i == 0 || i == nx) {
        if (!top_levels) { kind = 0; return 0.0; }
        if (oxy) { kind = 1; return r; }
        double s1 = (i == 0) ? (double)AT(E, L, i + 1, k) : (double)AT(E, L, i - 1, k);
        return rx_side(r, e_dn, (double)AT(E, L, i, k + 1), s1, K);
    }
    return rx_in(r, e_dn, (double)AT(E, L, i, k + 1), (double)AT(E, L, i - 1, k), (double)AT(E, L, i + 1, k), K);
}

/* one thread per (column of the given parity, species), bottom to top */
template <class T>
__global__ void k_mg_relax(MgConst m, MgLvlT<T> L, int l, int parity, const double* __restrict__ inside0)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int ncol = (L.nx + 1 - parity + 1) / 2;
    int sp = blockIdx.y;
    if (t >= ncol) return;
    int i = 2 * t + parity;
    T below = T(0);
    for (int k = 0; k <= L.nz; k++) relax_point(m, L, l, sp, i, k, inside0, below, k > 0);
}

/* Segmented form of the same sweep, for tall columns.  Along a column the
 * update is a first-order recurrence E_k = (b_k + w E_{k-1}) / (c + 2) with
 * w/(c + 2) <= 1/4 (c = h^2/(dt D) >= 0, w <= 1), so the influence of the
 * value carried in from below shrinks by 4x per row.  Each thread owns SEG
 * rows of one column and first re-runs the WARM rows below them from the
 * pre-sweep values; after WARM = 32 rows the carried-in difference is
 * below 4^-32 ~ 5e-20 of itself, i.e. the rows are those of the sequential
 * bottom-to-top sweep.  The pre-sweep values a thread reads from rows that
 * another thread of its column writes (its warm-up rows' upper neighbours
 * and the row just above its segment) are loaded before a block barrier, so
 * every thread reads them before any thread writes.  All segments of a
 * column live in one block: blockDim = (32 columns, nseg segments). */
#define RELAX_WARM 32
template <class T>
__global__ void __launch_bounds__(512) k_mg_relax_seg(MgConst m, MgLvlT<T> L, int l, int parity, int seg_len,
                                                      const double* __restrict__ inside0)
{
    const int ncol = (L.nx + 1 - parity + 1) / 2;
    const int t = blockIdx.x * 32 + threadIdx.x;
    const int seg = threadIdx.y;
    const int sp = blockIdx.y;
    const bool active = t < ncol;
    const int i = 2 * t + parity;
    const int nz = L.nz;
    const int k_begin = seg * seg_len;
    const int k_end = min(k_begin + seg_len, nz + 1);
    const int k_start = max(0, k_begin - RELAX_WARM);
    T* E = SP(L.e);
    /* pre-sweep values this thread needs from rows other threads write */
    T up_w[RELAX_WARM + 1];
    T below = T(0), above_end = T(0);
    if (active && k_begin <= nz) {
        for (int k = k_start; k < k_begin; k++) up_w[k - k_start] = AT(E, L, i, k + 1);
        if (k_start > 0) below = AT(E, L, i, k_start - 1);
        if (k_end <= nz) above_end = AT(E, L, i, k_end);
    }
    __syncthreads();
    if (!active || k_begin > nz) return;
    const T* R = SP(L.r);
    const bool oxy = (sp == 1);
    const bool top_levels = l >= m.A - 1;
    const int nx = L.nx;
    const bool side = (i == 0 || i == nx);
    const RelaxK<T> K = relax_k<T>(m, l, sp);
    for (int k = k_start; k < k_end; k++) {
        const bool warm = k < k_begin;
        T r = AT(R, L, i, k);
        T up = (k < nz) ? (warm ? up_w[k - k_start] : (k + 1 == k_end ? above_end : AT(E, L, i, k + 1))) : T(0);
        T e_dn = below;
        T out = T(0);
        bool write = true;
        if (k == 0) {
            int d = 1 << l;
            int i0 = (i - nx / 2) * d + m.box_x / 2;
            i0 = i0 < 0 ? 0 : (i0 > m.box_x - 1 ? m.box_x - 1 : i0);
            if (inside0[(size_t)i0 * m.box_z] > 0) out = r;
            else if (side) {
                if (top_levels) {
                    if (oxy) out = r;
                    else out = rx_corner(r, (i == 0) ? AT(E, L, i + 1, 0) : AT(E, L, i - 1, 0), up, K);
                } else write = false;
            } else {
                if (oxy) out = r;
                else out = rx_k0(r, up, AT(E, L, i - 1, 0), AT(E, L, i + 1, 0), K);
            }
        } else if (k == nz) {
            if (top_levels) {
                if (side) {
                    if (oxy) out = r;
                    else out = rx_corner(r, (i == 0) ? AT(E, L, i + 1, k) : AT(E, L, i - 1, k), e_dn, K);
                } else out = rx_top(r, e_dn, AT(E, L, i - 1, k), AT(E, L, i + 1, k), K);
            } else write = false;
        } else if (side) {
            if (top_levels) {
                if (oxy) out = r;
                else out = rx_side(r, e_dn, up, (i == 0) ? AT(E, L, i + 1, k) : AT(E, L, i - 1, k), K);
            } else write = false;
        } else {
            out = rx_in(r, e_dn, up, AT(E, L, i - 1, k), AT(E, L, i + 1, k), K);
        }
        /* points that are not relaxed keep their value; those columns and
         * rows (composite edges) are written by no thread in this sweep */
        if (!write) out = AT(E, L, i, k);
        if (write && !warm) AT(E, L, i, k) = out;
        below = out;
    }
}

/* All mu2 relaxations of a small (coarsest) level in one block: the sweep
 * order (even columns, then odd, each bottom to top) is kept with a block
 * barrier between half-sweeps. */
template <class T>
__global__ void __launch_bounds__(1024) k_mg_relax_coarse(MgConst m, MgLvlT<T> L, int l, int sweeps,
                                                          const double* __restrict__ inside0)
{
    const int nx = L.nx;
    const int ncols = nx + 1;
    for (int s = 0; s < sweeps; s++)
        for (int parity = 0; parity < 2; parity++) {
            int ncol = (ncols - parity + 1) / 2;
            for (int w = threadIdx.x; w < 3 * ncol; w += blockDim.x) {
                int sp = w / ncol, t = w % ncol;
                int i = 2 * t + parity;
                T below = T(0);
                for (int k = 0; k <= L.nz; k++) relax_point(m, L, l, sp, i, k, inside0, below, k > 0);
            }
            __syncthreads();
        }
}

/* All mu2 relaxations of the coarsest level with the level held in shared
 * memory: one block per species, E and R of that species copied in (row k
 * at offset k*(nx+1)), even then odd columns per sweep with a block barrier
 * between half-sweeps, E copied back.  Reads outside 0..nz follow the
 * reference's flat index i*(nz+1)+k like at_ref. */
template <class T>
__device__ __forceinline__ T at_s(const T* a, int nx, int nz, int i, int k)
{
    if (k >= 0 && k <= nz) return a[k * (nx + 1) + i];
    long f = (long)i * (nz + 1) + k;
    long n = (long)(nx + 1) * (nz + 1);
    if (f < 0 || f >= n) return T(0);
    return a[(int)(f % (nz + 1)) * (nx + 1) + (int)(f / (nz + 1))];
}
template <class T>
__global__ void __launch_bounds__(1024) k_mg_coarse_smem(MgConst m, MgLvlT<T> L, int l, int sweeps,
                                                         const double* __restrict__ inside0)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int sp = blockIdx.x;
    const int nx = L.nx, nz = L.nz, W = nx + 1;
    const int np = W * (nz + 1);
    T* Es = reinterpret_cast<T*>(smem_raw);
    T* Rs = Es + np;
    T* E = SP(L.e);
    const T* R = SP(L.r);
    for (int q = threadIdx.x; q < np; q += blockDim.x) {
        int i = q % W, k = q / W;
        Es[q] = AT(E, L, i, k);
        Rs[q] = AT(R, L, i, k);
    }
    __syncthreads();
    const RelaxK<T> K = relax_k<T>(m, l, sp);
    const bool oxy = (sp == 1);
    const bool top_levels = l >= m.A - 1;
    for (int s = 0; s < sweeps; s++)
        for (int parity = 0; parity < 2; parity++) {
            const int ncol = (W - parity + 1) / 2;
            for (int t = threadIdx.x; t < ncol; t += blockDim.x) {
                const int i = 2 * t + parity;
                const bool side = (i == 0 || i == nx);
                T below = T(0);
                for (int k = 0; k <= nz; k++) {
                    const T r = Rs[k * W + i];
                    const T old = Es[k * W + i];
                    T out = old;
                    if (k == 0) {
                        int d = 1 << l;
                        int i0 = (i - nx / 2) * d + m.box_x / 2;
                        i0 = i0 < 0 ? 0 : (i0 > m.box_x - 1 ? m.box_x - 1 : i0);
                        if (inside0[(size_t)i0 * m.box_z] > 0) out = r;
                        else if (side) {
                            if (top_levels) out = oxy ? r : rx_corner(r, (i == 0) ? Es[i + 1] : Es[i - 1], at_s(Es, nx, nz, i, 1), K);
                        } else out = oxy ? r : rx_k0(r, at_s(Es, nx, nz, i, 1), Es[i - 1], Es[i + 1], K);
                    } else if (k == nz) {
                        if (top_levels) {
                            if (side) out = oxy ? r : rx_corner(r, (i == 0) ? Es[k * W + i + 1] : Es[k * W + i - 1], below, K);
                            else out = rx_top(r, below, Es[k * W + i - 1], Es[k * W + i + 1], K);
                        }
                    } else if (side) {
                        if (top_levels) out = oxy ? r : rx_side(r, below, Es[(k + 1) * W + i], (i == 0) ? Es[k * W + i + 1] : Es[k * W + i - 1], K);
                    } else {
                        out = rx_in(r, below, Es[(k + 1) * W + i], Es[k * W + i - 1], Es[k * W + i + 1], K);
                    }
                    Es[k * W + i] = out;
                    below = out;
                }
            }
            __syncthreads();
        }
    for (int q = threadIdx.x; q < np; q += blockDim.x) {
        int i = q % W, k = q / W;
        AT(E, L, i, k) = Es[q];
    }
}

/* Relaxation of point (i, k) of a level held in shared memory (row k at
 * offset k*(nx+1)), in place; the point code of k_mg_coarse_smem. */
template <class T>
__device__ __forceinline__ void relax_smem(const RelaxK<T>& K, bool oxy, bool top_levels,
                                           int nx, int nz, int i, int k, T* Es, const T* Rs,
                                           const unsigned char* ins_row0)
{
    const int W = nx + 1;
    const bool side = (i == 0 || i == nx);
    const T r = Rs[k * W + i];
    T out = Es[k * W + i];
    if (k == 0) {
        if (ins_row0[i]) out = r;
        else if (side) {
            if (top_levels) out = oxy ? r : rx_corner(r, (i == 0) ? Es[i + 1] : Es[i - 1], at_s(Es, nx, nz, i, 1), K);
        } else out = oxy ? r : rx_k0(r, at_s(Es, nx, nz, i, 1), Es[i - 1], Es[i + 1], K);
    } else {
        const T below = Es[(k - 1) * W + i];
        if (k == nz) {
            if (top_levels) {
                if (side) out = oxy ? r : rx_corner(r, (i == 0) ? Es[k * W + i + 1] : Es[k * W + i - 1], below, K);
                else out = rx_top(r, below, Es[k * W + i - 1], Es[k * W + i + 1], K);
            }
        } else if (side) {
            if (top_levels) out = oxy ? r : rx_side(r, below, Es[(k + 1) * W + i], (i == 0) ? Es[k * W + i + 1] : Es[k * W + i - 1], K);
        } else {
            out = rx_in(r, below, Es[(k + 1) * W + i], Es[k * W + i - 1], Es[k * W + i + 1], K);
        }
    }
    Es[k * W + i] = out;
}

/* All mu2 relaxations of a level of nz >= 1 held in shared memory, as a
 * wavefront over the sweeps: at step t sweep s relaxes the even columns of
 * row t - 2s and the odd columns of row t - 2s - 1, one barrier per step.
 * The lags keep every read on the value the sequential order gives it:
 *   even (k, s) reads its column at k-1 (sweep s, step t-1) and k+1 (sweep
 *   s-1, not rewritten before step t+1) and the odd columns of row k
 *   (sweep s-1's, written at step t-1, rewritten at step t+1);
 *   odd (k, s) reads its column at k-1 (sweep s, step t-1) and k+1 (sweep
 *   s-1) and the even columns of row k (sweep s's, written at step t-1;
 *   sweep s+1 rewrites them at step t+1);
 * and in one step the even writes (rows t - 2s) and odd writes (rows
 * t - 2s - 1) never meet a location another item of the step reads.
 * About (nz+1)/2 sweeps progress per step instead of one. */
template <class T>
__global__ void __launch_bounds__(1024) k_mg_coarse_wave(MgConst m, MgLvlT<T> L, int l, int sweeps,
                                                         const double* __restrict__ inside0)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int sp = blockIdx.x;
    const int nx = L.nx, nz = L.nz, W = nx + 1;
    const int np = W * (nz + 1);
    T* Es = reinterpret_cast<T*>(smem_raw);
    T* Rs = Es + np;
    unsigned char* ins = reinterpret_cast<unsigned char*>(Rs + np);   /* row-0 colony flags per column */
    T* E = SP(L.e);
    const T* R = SP(L.r);
    const int nth = blockDim.x, th = threadIdx.x;
    for (int q = th; q < np; q += nth) {
        int i = q % W, k = q / W;
        Es[q] = AT(E, L, i, k);
        Rs[q] = AT(R, L, i, k);
    }
    for (int i = th; i < W; i += nth) {
        int d = 1 << l;
        int i0 = (i - nx / 2) * d + m.box_x / 2;
        i0 = i0 < 0 ? 0 : (i0 > m.box_x - 1 ? m.box_x - 1 : i0);
        ins[i] = inside0[(size_t)i0 * m.box_z] > 0;
    }
    __syncthreads();
    const RelaxK<T> K = relax_k<T>(m, l, sp);
    const bool oxy = (sp == 1);
    const bool top_levels = l >= m.A - 1;
    /* work item q of a phase = (active sweep q / ncol, column q % ncol); a
     * thread's items q = th and th + nth, split once per parity */
    int a_[2][2], c_[2][2];
    for (int par = 0; par < 2; par++) {
        const int ncol = (W - par + 1) / 2;
        for (int j = 0; j < 2; j++) { int q = th + j * nth; a_[par][j] = q / ncol; c_[par][j] = q % ncol; }
    }
    const int steps = nz + 1 + 2 * (sweeps - 1) + 1;
    for (int t = 0; t < steps; t++) {
#pragma unroll
        for (int par = 0; par < 2; par++) {
            /* parity par relaxes row tp - 2s for the sweeps s with that row in 0..nz */
            const int tp = t - par;
            if (tp < 0) continue;
            const int s_lo = tp > nz ? (tp - nz + 1) / 2 : 0;
            const int s_hi = min(sweeps - 1, tp / 2);
            const int na = s_hi - s_lo + 1;
#pragma unroll
            for (int j = 0; j < 2; j++)
                if (a_[par][j] < na)
                    relax_smem<T>(K, oxy, top_levels, nx, nz, 2 * c_[par][j] + par, tp - 2 * (s_lo + a_[par][j]), Es, Rs, ins);
            /* more active sweeps than two items per thread cover (large levels) */
            const int ncol = (W - par + 1) / 2;
            for (int q = th + 2 * nth; q < na * ncol; q += nth) {
                const int sw = s_lo + q / ncol;
                relax_smem<T>(K, oxy, top_levels, nx, nz, 2 * (q % ncol) + par, tp - 2 * sw, Es, Rs, ins);
            }
        }
        __syncthreads();
    }
    for (int q = th; q < np; q += nth) {
        int i = q % W, k = q / W;
        AT(E, L, i, k) = Es[q];
    }
}

/* k_mg_coarse_wave spread over a thread-block cluster per species.  Block
 * `rank` owns the columns [c0, c1) = [rank W / C, (rank+1) W / C) and keeps
 * the whole level in its shared memory.  The wavefront steps run in
 * blocks of H steps: in a block, a cluster block relaxes its own columns
 * and H columns on each side (a halo), all from its own shared memory, with
 * a block barrier between steps.  A value can only move one column per
 * step (no item of a step reads what another writes), so the stale values
 * beyond the halo reach at most H columns in, and the owned columns stay
 * exact.  Between blocks every cluster block publishes its first and last H
 * owned columns to a publish buffer (two, alternating, so a slow reader of
 * the previous ones is never overwritten), one cluster barrier, and each
 * block copies its halos from its neighbours' buffers.  Every block runs
 * the same barriers; the last one comes after every read of another
 * block's shared memory, so no block leaves while read.  H <= W / C keeps
 * a halo inside the neighbouring block's columns. */
template <class T>
__global__ void __launch_bounds__(768) k_mg_coarse_cluster(MgConst m, MgLvlT<T> L, int l, int sweeps, int H,
                                                            const double* __restrict__ inside0)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cg::cluster_group cluster = cg::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    const int sp = blockIdx.x / C;
    const int nx = L.nx, nz = L.nz, W = nx + 1, NZ = nz + 1;
    const int np = W * NZ;
    T* Es = reinterpret_cast<T*>(smem_raw);
    T* Rs = Es + np;
    T* pub = Rs + np;                      /* [2 buffers][left, right][H][NZ] */
    unsigned char* ins = reinterpret_cast<unsigned char*>(pub + 4 * H * NZ);
    T* E = SP(L.e);
    const T* R = SP(L.r);
    const int nth = blockDim.x, th = threadIdx.x;
    for (int q = th; q < np; q += nth) {
        int i = q % W, k = q / W;
        Es[q] = AT(E, L, i, k);
        Rs[q] = AT(R, L, i, k);
    }
    for (int i = th; i < W; i += nth) {
        int d = 1 << l;
        int i0 = (i - nx / 2) * d + m.box_x / 2;
        i0 = i0 < 0 ? 0 : (i0 > m.box_x - 1 ? m.box_x - 1 : i0);
        ins[i] = inside0[(size_t)i0 * m.box_z] > 0;
    }
    __syncthreads();
    const int c0 = rank * W / C, c1 = (rank + 1) * W / C;
    const int e0 = max(0, c0 - H), e1 = min(W, c1 + H);
    const T* pubL_left = rank > 0 ? cluster.map_shared_rank(pub, rank - 1) : pub;   /* left neighbour's buffers */
    const T* pubR_right = rank < C - 1 ? cluster.map_shared_rank(pub, rank + 1) : pub;
    const RelaxK<T> K = relax_k<T>(m, l, sp);
    const bool oxy = (sp == 1);
    const bool top_levels = l >= m.A - 1;
    /* the first half of the threads relaxes the even columns, the second
     * half the odd ones: the two halves of a step run side by side */
    const int nhalf = nth / 2;
    const int par = th < nhalf ? 0 : 1, tl = th - par * nhalf;
    const int first = e0 + ((e0 & 1) != par ? 1 : 0);
    const int ncol = first < e1 ? (e1 - first + 1) / 2 : 0;
    const int a0 = ncol ? tl / ncol : 0x7fffffff, cc0 = ncol ? tl % ncol : 0;
    const int steps = nz + 1 + 2 * (sweeps - 1) + 1;
    for (int b = 0, t0 = 0; t0 < steps; b++, t0 += H) {
        const int t_end = min(steps, t0 + H);
        for (int t = t0; t < t_end; t++) {
            const int tp = t - par;
            if (tp >= 0 && ncol) {
                const int s_lo = tp > nz ? (tp - nz + 1) / 2 : 0;
                const int s_hi = min(sweeps - 1, tp / 2);
                const int na = s_hi - s_lo + 1;
                if (a0 < na)
                    relax_smem<T>(K, oxy, top_levels, nx, nz, first + 2 * cc0, tp - 2 * (s_lo + a0), Es, Rs, ins);
                for (int q = tl + nhalf; q < na * ncol; q += nhalf)
                    relax_smem<T>(K, oxy, top_levels, nx, nz, first + 2 * (q % ncol), tp - 2 * (s_lo + q / ncol), Es, Rs, ins);
            }
            __syncthreads();
        }
        if (t_end < steps) {
            /* publish the first and last H owned columns, then take the halos */
            T* mine = pub + (b & 1) * 2 * H * NZ;
            for (int q = th; q < H * NZ; q += nth) {
                const int h = q / NZ, k = q % NZ;
                mine[q] = Es[k * W + c0 + h];
                mine[H * NZ + q] = Es[k * W + c1 - H + h];
            }
            cluster.sync();
            const T* lsrc = pubL_left + (b & 1) * 2 * H * NZ + H * NZ;   /* left neighbour's last H columns */
            const T* rsrc = pubR_right + (b & 1) * 2 * H * NZ;           /* right neighbour's first H columns */
            for (int q = th; q < H * NZ; q += nth) {
                const int h = q / NZ, k = q % NZ;
                const int xl = c0 - H + h, xr = c1 + h;
                if (xl >= e0) Es[k * W + xl] = lsrc[q];
                if (xr < e1) Es[k * W + xr] = rsrc[q];
            }
            __syncthreads();
        }
    }
    cluster.sync();              /* no block leaves while another may read its buffers */
    for (int q = th; q < (c1 - c0) * NZ; q += nth) {
        const int i = c0 + q % (c1 - c0), k = q / (c1 - c0);
        AT(E, L, i, k) = Es[k * W + i];
    }
}

/* ------------------------------------------------------------------------ */
/* Fused zebra smoother: S full sweeps (even columns, then odd columns, each */
/* bottom to top) in one pass over the rows, out of place (E -> E2).        */
/* ------------------------------------------------------------------------ */
template <class T> struct Pair2;
template <> struct Pair2<double> { typedef double2 type; };
template <> struct Pair2<float> { typedef float2 type; };

/* Each warp owns a strip of column pairs (lane t: columns c0+2t, c0+2t+1)
 * and one segment of rows.  The S sweeps are 2S half-sweeps (even columns,
 * then odd columns, per sweep) run as a pipeline: half-sweep h relaxes row
 * k = r - h at row step r.  Every input it needs was produced at step r-1
 * or r-2:
 *   even half of sweep s: value above and the point itself from sweep
 *   s-1's even half (steps r-1, r-2), odd neighbours from sweep s-1's odd
 *   half (step r-1; shuffle from lane t-1 and the lane's own odd column);
 *   odd half of sweep s: likewise from sweep s-1's odd half, even
 *   neighbours from sweep s's even half (step r-1; own even column and
 *   shuffle from lane t+1);
 *   value below from the half-sweep itself (step r-1);
 * so the 2S updates of a step are independent.  A half-sweep's result is
 * exact where all of its inputs were, which loses one lane at one strip
 * edge per half-sweep: lanes S .. 31-S are written.  Segments other than
 * the first start `warm` rows early from the pre-smoothing values;
 * the row recurrence contracts by at least 1/4 per row, so the start
 * error is below rounding when the segment's own rows begin.  Rows above
 * the segment are relaxed by the early half-sweeps as far as the later
 * ones need them, and only the segment's rows are stored.
 *
 * Register use: a half-sweep's last two results live in two arrays that
 * swap roles every step (the loop runs two steps per trip), and R and the
 * input rows are re-read through L1, prefetched SMOOTH_PF rows ahead. */
#define SMOOTH_PF 4         /* rows staged ahead of the row step */
#define SMOOTH_RING 11      /* ring slots per array; > SMOOTH_PF + 2S for every S used */
/* slot of a row: (k - kw + 1) mod SMOOTH_RING, all rows read are >= kw - 1 */
__device__ __forceinline__ int ring_wrap(int x) { return x < 0 ? x + SMOOTH_RING : (x >= SMOOTH_RING ? x - SMOOTH_RING : x); }
#define SMOOTH_WARPS 4      /* warps per block */
struct SmoothArgs {
    int nx, nz, pitch, l, sp, ce, co, kind_e, kind_o, kw, ks, ke;
    bool ld_ok, st_e, st_o, plain_cols;
};

/* Row staging: each lane copies its own column pair of E and R row k into
 * a per-warp ring in shared memory (cp.async, zero-filled off the grid)
 * and later reads back only what it copied itself, so the lane's own
 * cp.async.wait_group is the only ordering needed. */
template <class T>
__device__ __forceinline__ void ring_issue(typename Pair2<T>::type* ring, const T* E, const T* R,
                                           const SmoothArgs& g, int k, int slot)
{
    typedef typename Pair2<T>::type T2;
    const bool ok = g.ld_ok && k >= 0 && k <= g.nz;
    const size_t off = ok ? (size_t)k * g.pitch + g.ce : 0;
    T2* se = ring + slot * 32 + (threadIdx.x & 31);
    T2* sr = se + SMOOTH_RING * 32;
    const unsigned de = (unsigned)__cvta_generic_to_shared(se), dr = (unsigned)__cvta_generic_to_shared(sr);
    const int n = ok ? (int)sizeof(T2) : 0;
    if (sizeof(T2) == 16) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" :: "r"(de), "l"(E + off), "r"(n));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" :: "r"(dr), "l"(R + off), "r"(n));
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" :: "r"(de), "l"(E + off), "r"(n));
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" :: "r"(dr), "l"(R + off), "r"(n));
    }
    asm volatile("cp.async.commit_group;");
}
template <class T>
__device__ __forceinline__ typename Pair2<T>::type ring_e(const typename Pair2<T>::type* ring, const SmoothArgs& g, int k)
{
    typename Pair2<T>::type v; v.x = T(0); v.y = T(0);
    if (k >= 0 && k <= g.nz) v = ring[((k - g.kw + 1) % SMOOTH_RING) * 32 + (threadIdx.x & 31)];
    return v;
}
template <class T>
__device__ __forceinline__ typename Pair2<T>::type ring_r(const typename Pair2<T>::type* ring, const SmoothArgs& g, int k)
{
    typename Pair2<T>::type v; v.x = T(0); v.y = T(0);
    if (k >= 0 && k <= g.nz) v = ring[SMOOTH_RING * 32 + ((k - g.kw + 1) % SMOOTH_RING) * 32 + (threadIdx.x & 31)];
    return v;
}

template <class T>
__device__ __forceinline__ typename Pair2<T>::type ld_pair(const T* a, const SmoothArgs& g, int k)
{
    typename Pair2<T>::type v; v.x = T(0); v.y = T(0);
    if (g.ld_ok && k >= 0 && k <= g.nz) v = *reinterpret_cast<const typename Pair2<T>::type*>(a + (size_t)k * g.pitch + g.ce);
    return v;
}

/* one row step: h1 = results of step r-1 (read only), h2 = results of step
 * r-2 on entry and of step r on exit */
template <class T, int S>
__device__ __forceinline__ void smooth_step(const int r, const int sr, const T (&h1)[2 * S], T (&h2)[2 * S],
                                            const T* __restrict__ E, const T* __restrict__ R, T* __restrict__ EO,
                                            typename Pair2<T>::type* ring,
                                            const MgConst& m, const RelaxK<T>& K, const SmoothArgs& g,
                                            const double* __restrict__ inside0)
{
    typedef typename Pair2<T>::type T2;
    constexpr int H = 2 * S;
    static_assert(SMOOTH_RING > SMOOTH_PF + H, "ring slot reused before its last read");
    /* stage row r+1+PF; rows up to r+1 are then complete */
    ring_issue<T>(ring, E, R, g, r + 1 + SMOOTH_PF, ring_wrap(sr + 1 + SMOOTH_PF));
    asm volatile("cp.async.wait_group %0;" :: "n"(SMOOTH_PF));
    /* all half-sweeps on interior rows of this segment, no side column in the warp */
    const bool plain = g.plain_cols && (r - (H - 1) >= g.kw) && (r - (H - 1) >= 1) && (r <= g.nz - 1) && (r <= g.ke - 1);
    if (plain) {
        /* every row read here lies inside the grid: no range checks */
        const T2* rl = ring + (threadIdx.x & 31);
        const T2 inm = rl[ring_wrap(sr - 1) * 32], in0 = rl[sr * 32];
        const T2 inp = rl[ring_wrap(sr + 1) * 32];
        T nb[H];
#pragma unroll
        for (int h = 0; h < H; h++) {
            const T src = (h == 0) ? in0.y : h1[h - 1];
            nb[h] = (h & 1) ? __shfl_down_sync(0xffffffffu, src, 1) : __shfl_up_sync(0xffffffffu, src, 1);
        }
#pragma unroll
        for (int h = H - 1; h >= 0; h--) {
            const bool odd = h & 1;
            const T up = (h == 0) ? inp.x : (h == 1) ? in0.y : h1[h - 2];
            const T own_other = (h == 0) ? in0.y : h1[h - 1];
            const T2 rk = rl[(SMOOTH_RING + ring_wrap(sr - h)) * 32];
            h2[h] = odd ? rx_in(rk.y, h1[h], up, own_other, nb[h], K) : rx_in(rk.x, h1[h], up, nb[h], own_other, K);
        }
        (void)inm;
    } else {
        const T2 inm = ring_e<T>(ring, g, r - 1), in0 = ring_e<T>(ring, g, r), inp = ring_e<T>(ring, g, r + 1);
        T nb[H];
#pragma unroll
        for (int h = 0; h < H; h++) {
            const T src = (h == 0) ? in0.y : h1[h - 1];
            nb[h] = (h & 1) ? __shfl_down_sync(0xffffffffu, src, 1) : __shfl_up_sync(0xffffffffu, src, 1);
        }
#pragma unroll
        for (int h = H - 1; h >= 0; h--) {
            const int k = r - h;
            const bool odd = h & 1;
            const int top = min(g.nz, g.ke - 1 + (H - 1 - h) / 2);
            if (k < g.kw || k > top) { h2[h] = h1[h]; continue; }
            const T old = (h == 0) ? in0.x : (h == 1) ? inm.y : h2[h - 2];
            const T up = (h == 0) ? inp.x : (h == 1) ? in0.y : h1[h - 2];
            const T own_other = (h == 0) ? in0.y : h1[h - 1];
            const T xm = odd ? own_other : nb[h];
            const T xp = odd ? nb[h] : own_other;
            const T2 rk = ring_r<T>(ring, g, k);
            const T rv = odd ? rk.y : rk.x;
            if (k > 0 && k < g.nz)
                h2[h] = rx_row<T>(odd ? g.kind_o : g.kind_e, rv, h1[h], up, xm, xp, old, K);
            else
                h2[h] = relax_val<T>(m, K, g.nx, g.nz, g.l, g.sp, odd ? g.co : g.ce, k, rv, h1[h], up, xm, xp, old, inside0);
        }
    }
    const int kS = r - (H - 1);
    if (kS >= g.ks && kS < g.ke) {
        T* dst = EO + (size_t)kS * g.pitch;
        T2 v; v.x = h1[H - 2]; v.y = h2[H - 1];       /* the even half finished this row one step ago */
        if (g.st_e && g.st_o) *reinterpret_cast<T2*>(dst + g.ce) = v;
        else if (g.st_e) dst[g.ce] = v.x;
    }
}

template <class T, int S>
__global__ void __launch_bounds__(32 * SMOOTH_WARPS) k_mg_smooth(MgConst m, MgLvlT<T> L, int l, int seg_len,
                                                   int warm, const double* __restrict__ inside0)
{
    constexpr int H = 2 * S;
    const int lane = threadIdx.x;
    const int warp = blockIdx.x * blockDim.y + threadIdx.y;
    const int sp = blockIdx.z;
    SmoothArgs g;
    g.nx = L.nx; g.nz = L.nz; g.pitch = L.pitch; g.l = l; g.sp = sp;
    const int OUTP = 32 - 2 * S;
    const int c0 = warp * 2 * OUTP - 2 * S;
    g.ce = c0 + 2 * lane; g.co = g.ce + 1;
    if (warp * 2 * OUTP > g.nx) return;            /* whole warp: strip starts past the last column */
    g.ld_ok = g.ce >= 0 && g.co < g.pitch;
    g.st_e = lane >= S && lane <= 31 - S && g.ce >= 0 && g.ce <= g.nx;
    g.st_o = lane >= S && lane <= 31 - S && g.co >= 0 && g.co <= g.nx;
    g.ks = blockIdx.y * seg_len;
    if (g.ks > g.nz) return;
    g.ke = min(g.ks + seg_len, g.nz + 1);
    g.kw = max(0, g.ks - warm);
    const T* __restrict__ E = SP(L.e);
    const T* __restrict__ R = SP(L.r);
    T* __restrict__ EO = SP(L.e2);
    const RelaxK<T> K = relax_k<T>(m, l, sp);
    const bool oxy = (sp == 1);
    const bool top_levels = l >= m.A - 1;
    g.kind_e = col_kind(g.ce, g.nx, oxy, top_levels);
    g.kind_o = col_kind(g.co, g.nx, oxy, top_levels);
    /* lanes whose columns are outside 0..nx compute garbage that no written
     * lane reads; only real side columns need the per-lane path */
    const bool side_e = (g.ce == 0 || g.ce == g.nx), side_o = (g.co == 0 || g.co == g.nx);
    g.plain_cols = !__any_sync(0xffffffffu, side_e || side_o);
    extern __shared__ __align__(16) unsigned char smooth_smem[];
    typename Pair2<T>::type* ring = reinterpret_cast<typename Pair2<T>::type*>(smooth_smem) + threadIdx.y * (2 * SMOOTH_RING * 32);
    T a[H], b[H];
    {
        const typename Pair2<T>::type e0 = ld_pair(E, g, g.kw - 1);
#pragma unroll
        for (int h = 0; h < H; h++) { a[h] = (h & 1) ? e0.y : e0.x; b[h] = a[h]; }
    }
    for (int k = g.kw - 1; k <= g.kw + SMOOTH_PF; k++) ring_issue<T>(ring, E, R, g, k, k - g.kw + 1);
    const int r_end = g.ke - 1 + (H - 1);
    int sr = 1;                                 /* slot of row r = kw */
    for (int r = g.kw; r <= r_end; r += 2) {
        smooth_step<T, S>(r, sr, a, b, E, R, EO, ring, m, K, g, inside0);
        sr = ring_wrap(sr + 1);
        if (r + 1 <= r_end) smooth_step<T, S>(r + 1, sr, b, a, E, R, EO, ring, m, K, g, inside0);
        sr = ring_wrap(sr + 1);
    }
    asm volatile("cp.async.wait_group 0;");
}

/* ------------------------------------------------------------------------ */
/* restrictionAgaElementwise, Multigrid.cpp:269-405 (level l from l-1)       */
/* ------------------------------------------------------------------------ */
template <class T>
__global__ void k_mg_restrict(MgConst m, MgLvlT<T> Lc, MgLvlT<T> Lf, int l, const double* __restrict__ inside0)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y, sp = blockIdx.z;
    const int nx = Lc.nx, nz = Lc.nz;
    if (i > nx) return;
    const int X = m.box_x, ZA = m.box_z_agar;
    int d = 1 << l, d0 = 1 << m.A;
    /* X d0 / d with d = 2^l, as a shift */
    int nxp = (X * d0) >> l < X ? (X * d0) >> l : X;
    int nzp = (ZA * d0) >> l < ZA ? (ZA * d0) >> l : ZA;
    int ip = 2 * i - nx + nxp / 2, kp = 2 * k;
    /* on a composite level only row 0 and the points over the finer level
     * (0 <= ip <= nxp, kp <= nzp) are written; the launch already stops at
     * row nzp/2 */
    if (l < m.A && k > 0 && !(ip >= 0 && ip <= nxp && kp <= nzp)) return;
    const T h2 = (T)(m.bl2 * d * d);
    const T dt = (T)m.dt, D = (T)SP(m.D);
    const T half = (T)0.5;
    const bool oxy = sp == 1;
    int i0 = (i - nx / 2) * d + X / 2;
    i0 = i0 < 0 ? 0 : (i0 > X ? X : i0);   /* clamped to BoxX as in the reference */
    const T* EP = SP(Lf.e);
    const T* RP = SP(Lf.r);
    const double* AP = SP(Lf.s);
    const double* AL = SP(Lc.s);
    T* R = &AT(SP(Lc.r), Lc, i, k);
#define EPv(a, b) at_ref(EP, Lf, a, b)
#define RPv(a, b) at_ref(RP, Lf, a, b)
#define APv(a, b) ((T)at_ref(AP, Lf, a, b))
#define ALv(a, b) ((T)at_ref(AL, Lc, a, b))
    if (i == 0 || i == nx || k == nz) {
        if (l >= m.A) {
            if (k == nz && (i > 0) && (i < nx)) {
                /* carbon uses (ip,kp), oxygen/acetate (2i,2k): equal for l >= A */
                *R = (RPv(ip, kp) + half * (EPv(ip + 1, kp) + EPv(ip - 1, kp) + 2 * EPv(ip, kp - 1) - 4 * EPv(ip, kp)) * D * dt * 4 / h2 - EPv(ip, kp)) / 2;
            } else {
                int sx = (i == 0) ? 1 : -1;
                if (oxy) *R = RPv(ip, kp) - EPv(ip, kp);
                else if (k == 0)
                    *R = (RPv(ip, kp) + half * (2 * EPv(ip + sx, kp) + 2 * EPv(ip, kp + 1) - 4 * EPv(ip, kp)) * D * dt * 4 / h2 - EPv(ip, kp)) / 2;
                else if (k == nz)
                    *R = (RPv(ip, kp) + half * (2 * EPv(ip + sx, kp) + 2 * EPv(ip, kp - 1) - 4 * EPv(ip, kp)) * D * dt * 4 / h2 - EPv(ip, kp)) / 2;
                else
                    *R = (RPv(ip, kp) + half * (2 * EPv(ip + sx, kp) + EPv(ip, kp + 1) + EPv(ip, kp - 1) - 4 * EPv(ip, kp)) * D * dt * 4 / h2 - EPv(ip, kp)) / 2;
            }
        }
    } else if (k == 0) {
        /* i0 == BoxX lies one row past insideColonyDen (Multigrid.cpp:279);
         * it counts as outside the colony */
        if (i0 < X && inside0[(size_t)i0 * m.box_z] > 0) *R = 0;
        else if (ip > 0 && ip < nxp) {
            if (oxy) *R = (RPv(ip, 0) - EPv(ip, 0)) * half;
            else *R = (RPv(ip, 0) + half * (EPv(ip + 1, 0) + EPv(ip - 1, 0) + 2 * EPv(ip, 1) - 4 * EPv(ip, 0)) * D * dt * 4 / h2 - EPv(ip, 0)) * half;
        } else if ((l < m.A) && (ip >= 0 && ip <= nxp) && ((ip == 0) || (ip == nxp))) {
            if (oxy) *R = (T)m.max_o2_agar - ALv(i, 0);
            else if (ip == 0) *R = (APv(ip + 2, 0) + half * EPv(ip + 2, 0) + ALv(i - 1, 0) + 2 * ALv(i, 1) - 4 * ALv(i, 0)) * D * dt / h2;
            else *R = (ALv(i + 1, 0) + half * EPv(ip - 2, 0) + APv(ip - 2, 0) + 2 * ALv(i, 1) - 4 * ALv(i, 0)) * dt * D / h2;
        }
    } else if (l < m.A && ip >= 0 && ip <= nxp && kp <= nzp) {
        if (kp == nzp) {
            if (ip == 0 || ip == nxp)
                *R = (ALv(i + 1, k) + ALv(i - 1, k) + ALv(i, k + 1) + ALv(i, k - 1) - 4 * ALv(i, k)) * D * dt / h2;
            else
                *R = (ALv(i + 1, k) + ALv(i - 1, k) + ALv(i, k + 1) + APv(ip, kp - 2) + half * EPv(ip, kp - 2) - 4 * ALv(i, k)) * D * dt / h2;
        } else if (ip == 0) {
            *R = (APv(ip + 2, kp) + half * EPv(ip + 2, kp) + ALv(i - 1, k) + ALv(i, k + 1) + ALv(i, k - 1) - 4 * ALv(i, k)) * D * dt / h2;
        } else if (ip == nxp) {
            *R = (ALv(i + 1, k) + half * EPv(ip - 2, kp) + APv(ip - 2, kp) + ALv(i, k + 1) + ALv(i, k - 1) - 4 * ALv(i, k)) * D * dt / h2;
        } else {
            *R = (RPv(ip, kp) + half * (EPv(ip + 1, kp) + EPv(ip - 1, kp) + EPv(ip, kp + 1) + EPv(ip, kp - 1) - 4 * EPv(ip, kp)) * D * dt / h2 * 4 - EPv(ip, kp)) * half;
        }
    } else if (l >= m.A) {
        *R = (RPv(ip, kp) + half * (EPv(ip + 1, kp) + EPv(ip - 1, kp) + EPv(ip, kp + 1) + EPv(ip, kp - 1) - 4 * EPv(ip, kp)) * D * dt / h2 * 4 - EPv(ip, kp)) * half;
    }
#undef EPv
#undef RPv
#undef APv
#undef ALv
}

/* interpolationAga, Multigrid.cpp:407-467 (Err of level l += from l+1).
 * A thread takes the fine columns 2j and 2j+1 of one row: both read the
 * coarse column ip = nxp/2 - nx/4 + j (the odd one also ip + 1), so the
 * coarse values are loaded once and the pair is read and written as one
 * 16-byte (FP32: 8-byte) access. */
template <class T>
__global__ void k_mg_interp(MgConst m, MgLvlT<T> Lf, MgLvlT<T> Lc, int l)
{
    typedef typename Pair2<T>::type T2;
    const int j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y, sp = blockIdx.z;
    const int nx = Lf.nx, i = 2 * j;
    if (i > nx) return;
    const bool has_odd = i + 1 <= nx;
    const int X = m.box_x;
    int d0 = 1 << m.A;
    /* X d0 / 2^l / 4, as a shift */
    int nxp = (X * d0) >> (l + 2) < X ? (X * d0) >> (l + 2) : X;
    const T* C = SP(Lc.e);
    T* e = SP(Lf.e) + (size_t)k * Lf.pitch + i;
    const T half = (T)0.5, quarter = (T)0.25;
    const int ip = nxp / 2 - nx / 4 + j;
#define CV(a, b) at_ref(C, Lc, a, b)
    T inc_e, inc_o = T(0);
    if (k % 2 == 0) {
        const int kp = k / 2;
        const T c0 = CV(ip, kp);
        inc_e = c0;
        if (has_odd) inc_o = half * (c0 + CV(ip + 1, kp));
    } else {
        const int kp = (k - 1) / 2;
        const T c00 = CV(ip, kp), c01 = CV(ip, kp + 1);
        inc_e = half * (c00 + c01);
        if (has_odd) inc_o = quarter * (c00 + c01 + CV(ip + 1, kp) + CV(ip + 1, kp + 1));
    }
#undef CV
    if (has_odd) {
        T2 v = *reinterpret_cast<T2*>(e);
        v.x += inc_e; v.y += inc_o;
        *reinterpret_cast<T2*>(e) = v;
    } else {
        e[0] += inc_e;
    }
}

/* resetZero, Multigrid.cpp:47-82 */
template <class T>
__global__ void k_mg_reset_zero(MgLvlT<T> L, int zero_res)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y, sp = blockIdx.z;
    if (i > L.nx) return;
    AT(SP(L.e), L, i, k) = 0;
    if (zero_res) AT(SP(L.r), L, i, k) = 0;
}

/* updateSolAgaElementwise, Multigrid.cpp:544-568 */
/* With `nest` set it also does NestSolAgaElementwise
 * (Multigrid.cpp:724-737) for level l+1 (Ln): a point (i, k) of this level
 * that level l+1 nests, Sol_{l+1}(i', k') = Sol_l(2i' - nx' + nxp'/2, 2k'),
 * writes its updated value there.  That is the value the separate pass
 * would copy: between the two only the boundary rewrite and Res change,
 * and neither touches a nested point. */
__global__ void k_mg_update_sol(MgConst m, MgLvl L, int l, MgLvl Ln, int nest)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y, sp = blockIdx.z;
    const int nx = L.nx;
    if (i > nx) return;
    const int X = m.box_x, ZA = m.box_z_agar;
    int d0 = 1 << m.A;
    /* X d0 / 2^l, as a shift */
    int nxp = (X * d0) >> l < X ? (X * d0) >> l : X;
    int nzp = (ZA * d0) >> l < ZA ? (ZA * d0) >> l : ZA;
    AT(SP(L.r), L, i, k) = 0;
    int ip = 2 * i - nx + nxp / 2, kp = 2 * k;
    double& e = AT(SP(L.e), L, i, k);
    double& a = AT(SP(L.s), L, i, k);
    if (l < m.A && (l == 0 || ip <= 0 || ip >= nxp || kp >= nzp)) {
        a += e;
        if (sp == 0) a = dmaxd(dmind(a, m.max_carbon), 0.0);
        else if (sp == 1) a = dmaxd(dmind(a, m.max_o2_agar), 0.0);
        else a = dmaxd(a, 0.0);
    }
    e = 0;
    if (nest) {
        const int nxpn = (X * d0) >> (l + 1) < X ? (X * d0) >> (l + 1) : X;
        const int nzpn = (ZA * d0) >> (l + 1) < ZA ? (ZA * d0) >> (l + 1) : ZA;
        const int t = i + Ln.nx - nxpn / 2;
        if ((k & 1) == 0 && (t & 1) == 0 && i > 0 && i < nxpn && k < nzpn) {
            const int in = t >> 1, kn = k >> 1;
            if (in >= 0 && in <= Ln.nx && kn <= Ln.nz) AT(SP(Ln.s), Ln, in, kn) = a;
        }
    }
}

/* per-level constants of the residual pass, worked out on the host with
 * the same operations the point code used: the finer level's extent nxp,
 * nzp and, per species, D/h^2 and dt*D/h^2 (h^2 = BoxLength^2 4^l) */
struct ResConst { int nxp, nzp; double cD[3], cdt[3]; };
static ResConst res_const(const MgConst& m, int l)
{
    ResConst r;
    const int X = m.box_x, ZA = m.box_z_agar;
    const int d = 1 << l, d0 = 1 << m.A;
    r.nxp = X * d0 / d < X ? X * d0 / d : X;
    r.nzp = ZA * d0 / d < ZA ? ZA * d0 / d : ZA;
    const double h2 = m.bl2 * d * d;
    for (int sp = 0; sp < 3; sp++) {
        r.cD[sp] = m.D[sp] / h2;
        r.cdt[sp] = m.dt * m.D[sp] / h2;
    }
    return r;
}

/* updateResAgaElementwise, Multigrid.cpp:570-701.  SETUP: the setup()
 * form after a reset() (Err zero everywhere, Res zero on levels > 0):
 * updateSolAga then only clamps the solution at the uncovered points and
 * zeroes Res, so one pass clamps the stencil values as it reads them,
 * stores the point's clamped value where the clamp changed it, and
 * writes Res (0 where updateResAga leaves it). */
template <bool SETUP, bool LEVEL0>
__global__ void k_mg_update_res(MgConst m, MgLvl L, MgLvl Lp, int l, ResConst rc, const double* __restrict__ inside0)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    const int sp = blockIdx.z;
    const int nx = L.nx, nz = L.nz;
    if (i > nx || l >= m.A) return;
    const int nxp = rc.nxp, nzp = rc.nzp;
    /* the reference scales each residual by dt*D/h^2 (D/h^2 for oxygen's
     * top row) per point; here once per level and species, on the host */
    const double cD = SP(rc.cD), cdt = SP(rc.cdt);
    const bool oxy = sp == 1;
    int ip = 2 * i - nx + nxp / 2, kp = 2 * k;
    const double* A = SP(L.s);
    const double* ctr = A + (size_t)k * L.pitch + i;
    const ptrdiff_t P = L.pitch;
    double* R = &AT(SP(L.r), L, i, k);
    const double hi = sp == 0 ? m.max_carbon : (sp == 1 ? m.max_o2_agar : 1e300);
    /* the solution value updateSolAga leaves at (i + di, k + dk), |di|,
     * |dk| <= 1: clamped where uncovered (everywhere on level 0); the
     * coverage of the three columns and rows is worked out once */
    const bool cu_m = ip - 2 <= 0 || ip - 2 >= nxp, cu_0 = ip <= 0 || ip >= nxp, cu_p = ip + 2 <= 0 || ip + 2 >= nxp;
    const bool ru_m = kp - 2 >= nzp, ru_0 = kp >= nzp, ru_p = kp + 2 >= nzp;
    auto sol = [&](int di, int dk) -> double {
        double v = ctr[di + dk * P];
        if (SETUP) {
            const bool cu = di < 0 ? cu_m : (di > 0 ? cu_p : cu_0);
            const bool ru = dk < 0 ? ru_m : (dk > 0 ? ru_p : ru_0);
            const bool clamp = LEVEL0 || cu || ru;
            if (clamp) v = dmaxd(dmind(v, hi), 0.0);
        }
        return v;
    };
    double res = 0.0;
    bool set = SETUP;
#define AL(a, b) sol((a) - i, (b) - k)
#define APv(a, b) AT(SP(Lp.s), Lp, a, b)
    if (i == 0 || i == nx) {
        if (l == m.A - 1) {
            int sx = (i == 0) ? 1 : -1;
            if (oxy) set = true, res = 0;
            else if (k == 0) set = true, res = (2 * AL(i + sx, k) + 2 * AL(i, k + 1) - 4 * AL(i, k)) * cdt;
            else if (k == nz) set = true, res = (2 * AL(i + sx, k) + 2 * AL(i, k - 1) - 4 * AL(i, k)) * cdt;
            else set = true, res = (2 * AL(i + sx, k) + AL(i, k - 1) + AL(i, k + 1) - 4 * AL(i, k)) * cdt;
        }
    } else if (k == nz) {
        if (l == m.A - 1) {
            /* oxygen omits dt here, as the reference does (Multigrid.cpp:634) */
            if (oxy) set = true, res = (AL(i + 1, k) + AL(i - 1, k) + 2 * AL(i, k - 1) - 4 * AL(i, k)) * cD;
            else set = true, res = (AL(i + 1, k) + AL(i - 1, k) + 2 * AL(i, k - 1) - 4 * AL(i, k)) * cdt;
        }
    } else if (k == 0) {
        if (LEVEL0) {
            if (inside0[(size_t)i * m.box_z] > 0) set = true, res = 0;
            else if (oxy) set = true, res = m.max_o2_agar - AL(i, k);
            else set = true, res = (AL(i + 1, k) + AL(i - 1, k) + 2 * AL(i, k + 1) - 4 * AL(i, k)) * cdt;
        } else if ((ip > 0 && ip < nxp) != 1) {
            if (oxy) set = true, res = m.max_o2_agar - AL(i, k);
            else if (ip == 0) set = true, res = (APv(ip + 2, kp) + AL(i - 1, k) + 2 * AL(i, k + 1) - 4 * AL(i, k)) * cdt;
            else if (ip == nxp) set = true, res = (APv(ip - 2, kp) + AL(i + 1, k) + 2 * AL(i, k + 1) - 4 * AL(i, k)) * cdt;
            else set = true, res = (AL(i + 1, k) + AL(i - 1, k) + 2 * AL(i, k + 1) - 4 * AL(i, k)) * cdt;
        }
    } else {
        if (!LEVEL0) {
            if (kp == nzp && ip > 0 && ip < nxp)
                set = true, res = (AL(i + 1, k) + AL(i - 1, k) + APv(ip, kp - 2) + AL(i, k + 1) - 4 * AL(i, k)) * cdt;
            else if (ip == 0 && kp < nzp)
                set = true, res = (APv(ip + 2, kp) + AL(i - 1, k) + AL(i, k - 1) + AL(i, k + 1) - 4 * AL(i, k)) * cdt;
            else if (ip == nxp && kp < nzp)
                set = true, res = (AL(i + 1, k) + APv(ip - 2, kp) + AL(i, k - 1) + AL(i, k + 1) - 4 * AL(i, k)) * cdt;
            else if (ip <= 0 || ip >= nxp || kp >= nzp)
                set = true, res = (AL(i + 1, k) + AL(i - 1, k) + AL(i, k - 1) + AL(i, k + 1) - 4 * AL(i, k)) * cdt;
        } else {
            set = true, res = (AL(i + 1, k) + AL(i - 1, k) + AL(i, k - 1) + AL(i, k + 1) - 4 * AL(i, k)) * cdt;
        }
    }
#undef AL
#undef APv
    if (set) *R = res;
    if (SETUP) {
        double v = ctr[0], w = sol(0, 0);
        if (w != v) AT(SP(L.s), L, i, k) = w;
    }
}

/* rewriteSolBdryAga, Multigrid.cpp:469-503 (top row, then the side columns) */
__global__ void k_mg_rewrite_bdry(MgConst m, MgLvl L, MgLvl Lc, int l)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int sp = blockIdx.y;
    const int X = m.box_x;
    int d = 1 << l, d0 = 1 << m.A;
    const int nx = L.nx, nz = L.nz;
    int nx2 = X * d0 / d / 4 < X ? X * d0 / d / 4 : X;
    const double* C = SP(Lc.s);
    if (t < nx + 1) {
        int i = t, k2 = nz / 2;
        int i2 = nx2 / 2 + i / 2 - nx / 4, i2p1 = nx2 / 2 + (i + 1) / 2 - nx / 4;
        AT(SP(L.s), L, i, nz) = (AT(C, Lc, i2, k2) + AT(C, Lc, i2p1, k2)) / 2;
    } else if (t < nx + 1 + 2 * nz) {
        int u = t - (nx + 1);
        int k = u >> 1, side = u & 1;
        int i = side ? nx : 0;
        int i2 = nx2 / 2 + i / 2 - nx / 4;
        AT(SP(L.s), L, i, k) = (AT(C, Lc, i2, k / 2) + AT(C, Lc, i2, (k + 1) / 2)) / 2;
    }
}

/* copyToMG, Multigrid.cpp:891-907: wall-under-colony values into level 0,
 * then the periodic copy of column 0 into column BoxX on the last
 * composite level */
__global__ void k_mg_copy_to(MgConst m, MgLvl L0, const double* __restrict__ wC, const double* __restrict__ wO,
                             const double* __restrict__ wA, const double* __restrict__ inside0)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 1 && i <= m.box_x - 1 && inside0[(size_t)i * m.box_z] > 0) {
        AT(L0.s[0], L0, i, 0) = wC[i];
        AT(L0.s[1], L0, i, 0) = wO[i];
        AT(L0.s[2], L0, i, 0) = wA[i];
    }
}
__global__ void k_mg_copy_edge(MgLvl L)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    int sp = blockIdx.y;
    if (k > L.nz) return;
    AT(SP(L.s), L, L.nx, k) = AT(SP(L.s), L, 0, k);
}
/* copyFromMG, Multigrid.cpp:958-981: wall rows of both buffers (the agar
 * field is read straight from the solution rows 1..BoxZAgar) */
__global__ void k_mg_copy_from(MgLvl L, int X, double* cC, double* cO, double* cA, double* pC, double* pO, double* pA)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= X) return;
    double c = AT(L.s[0], L, i, 0), o = AT(L.s[1], L, i, 0), a = AT(L.s[2], L, i, 0);
    cC[i] = c; cO[i] = o; cA[i] = a;
    pC[i] = c; pO[i] = o; pA[i] = a;
}

/* ------------------------------------------------------------------------ */
static inline dim3 grid2(int n, int threads) { return dim3((unsigned)((n + threads - 1) / threads), 3); }
/* 2-D launch over a level: x = columns, y = rows, z = species */
static inline dim3 grid_rows(int ncols, int nrows, int threads)
{ return dim3((unsigned)((ncols + threads - 1) / threads), (unsigned)nrows, 3); }

/* The context's smoother form: 0 = one thread per column and half-sweep,
 * 1 = segmented half-sweeps, 2 = fused sweeps with per-lane row staging
 * (k_mg_smooth), 3 = fused sweeps with TMA-staged rows (k_mg_smooth_tma,
 * the default, set by bcg_create); 2 and 3 on levels of 3 rows or more */
extern "C" int bcg_set_relax_mode(bcg_ctx* c, int mode)
{
    if (!c || mode < 0 || mode > 3) return BCG_E_ARG;
    if (mode != c->relax_mode) nutrient_graphs_drop(c);
    c->relax_mode = mode;
    return BCG_OK;
}

template <class T> static MgLvlT<T> lvl(const bcg_ctx* c, int l);
template <> MgLvlT<double> lvl<double>(const bcg_ctx* c, int l) { return mg_lvl(c, l); }
template <> MgLvlT<float> lvl<float>(const bcg_ctx* c, int l) { return mg_lvl_f(c, l); }

template <class T>
static void relax_level(bcg_ctx* c, const MgConst& m, int l)
{
    MgLvlT<T> L = lvl<T>(c, l);
    const int rows = L.nz + 1;
    if (c->relax_mode == 0 || rows <= 96) {
        for (int par = 0; par < 2; par++) {
            int ncol = (L.nx + 1 - par + 1) / 2;
            k_mg_relax<T><<<grid2(ncol, 64), 64, 0, c->stream>>>(m, L, l, par, c->inside);
        }
    } else {
        int nseg = (rows + 63) / 64;
        if (nseg > 16) nseg = 16;
        int seg_len = (rows + nseg - 1) / nseg;
        for (int par = 0; par < 2; par++) {
            int ncol = (L.nx + 1 - par + 1) / 2;
            dim3 grid((unsigned)((ncol + 31) / 32), 3);
            k_mg_relax_seg<T><<<grid, dim3(32, nseg), 0, c->stream>>>(m, L, l, par, seg_len, c->inside);
        }
    }
    c->launches += 2;
}

#define SMOOTH_WARPS_DEFAULT 1400    /* resident-warp target of k_mg_smooth before tuning */
#define SMOOTH_TMA_WARPS_DEFAULT 0   /* warps of k_mg_smooth_tma before tuning: 0 = one per resident slot */

template <class T> static void swap_err(bcg_ctx* c, int l);
template <> void swap_err<double>(bcg_ctx* c, int l)
{
    for (int sp = 0; sp < 3; sp++) { double* t = c->mg[l].err[sp]; c->mg[l].err[sp] = c->mg[l].err2[sp]; c->mg[l].err2[sp] = t; }
}
template <> void swap_err<float>(bcg_ctx* c, int l)
{
    for (int sp = 0; sp < 3; sp++) { float* t = c->mg[l].errf[sp]; c->mg[l].errf[sp] = c->mg[l].errf2[sp]; c->mg[l].errf2[sp] = t; }
}

/* `sweeps` zebra sweeps of level l.  In mode 2 levels of 3 or more rows
 * take the fused kernel, up to 3 sweeps per launch; each launch swaps the level's two
 * correction buffers.  Pre- and post-smoothing use the same number of
 * launches, so a V-cycle always swaps an even number of times and leaves
 * the buffers where it found them (captured graphs rely on this). */
/* Rows a segment of level l starts early: the row recurrence of a sweep
 * contracts by a = max over species of (1/2)/(cf + 2), cf = h^2/(dt D),
 * and the start error of a segment shrinks by a^w (times a polynomial
 * factor w^2 from the three pipelined sweeps) over w rows; w is taken so
 * that this is below 1e-18.  About 38 rows on the finest level of the
 * shipped input, a handful on the coarse levels, where h is larger. */
static int warm_rows(const MgConst& m, int l)
{
    double a = 0.0;
    for (int sp = 0; sp < 3; sp++) {
        const double cf = m.bl2 * (double)(1 << (2 * l)) / m.dt / m.D[sp];
        const double v = 0.5 / (cf + 2.0);
        a = v > a ? v : a;
    }
    for (int w = 1; w < 64; w++) {
        double e = (double)w * w;
        for (int j = 0; j < w; j++) e *= a;
        if (e < 1e-18) return w;
    }
    return 64;
}

template <class T>
static void smooth_level(bcg_ctx* c, const MgConst& m, int l, int sweeps)
{
    const int rows = c->mg[l].nz + 1;
    /* levels of 0-1 interior rows read across columns through the flat
     * index (at_ref); they keep the in-place kernels */
    if (c->relax_mode < 2 || rows < 3) {
        for (int j = 0; j < sweeps; j++) relax_level<T>(c, m, l);
        return;
    }
    if (c->relax_mode == 3 && mg_smooth_tma_fits(c->mg[l].nx)) {
        const int warm = warm_rows(m, l);
        const int target = c->smooth_warps > 0 ? c->smooth_warps : SMOOTH_TMA_WARPS_DEFAULT;
        while (sweeps > 0) {
            const int S = sweeps >= 3 ? 3 : sweeps;
            MgLvlT<T> L = lvl<T>(c, l);
            /* the launch clamps the warp count to what the level's rows allow */
            const int rc = mg_smooth_tma(c, m, L, l, S, target, warm);
            if (rc) { c->pending_error = rc; return; }
            swap_err<T>(c, l);
            sweeps -= S;
        }
        return;
    }
    while (sweeps > 0) {
        const int S = sweeps >= 3 ? 3 : sweeps;
        MgLvlT<T> L = lvl<T>(c, l);
        const int outp = 32 - 2 * S;
        const int nwx = (L.nx + 1 + 2 * outp - 1) / (2 * outp);
        const int target = c->smooth_warps > 0 ? c->smooth_warps : SMOOTH_WARPS_DEFAULT;
        const int warm = warm_rows(m, l);
        int nseg = (target + 3 * nwx - 1) / (3 * nwx);
        /* segments of at least 16 rows and no shorter than half the warm-up */
        const int min_len = warm / 2 > 16 ? warm / 2 : 16;
        const int max_seg = rows / min_len > 1 ? rows / min_len : 1;
        if (nseg > max_seg) nseg = max_seg;
        if (nseg < 1) nseg = 1;
        const int seg_len = (rows + nseg - 1) / nseg;
        dim3 block(32, SMOOTH_WARPS), grid((unsigned)((nwx + SMOOTH_WARPS - 1) / SMOOTH_WARPS), (unsigned)nseg, 3);
        const size_t smem = (size_t)SMOOTH_WARPS * 2 * SMOOTH_RING * 32 * 2 * sizeof(T);
        if (S == 3) k_mg_smooth<T, 3><<<grid, block, smem, c->stream>>>(m, L, l, seg_len, warm, c->inside);
        else if (S == 2) k_mg_smooth<T, 2><<<grid, block, smem, c->stream>>>(m, L, l, seg_len, warm, c->inside);
        else k_mg_smooth<T, 1><<<grid, block, smem, c->stream>>>(m, L, l, seg_len, warm, c->inside);
        c->launches++;
        swap_err<T>(c, l);
        sweeps -= S;
    }
}

/* device time (ms) of one level-0 launch of the fused 3-sweep smoother at
 * the shape bcg_autotune chose (0 before tuning) */
extern "C" int bcg_smoother_launch_ms(bcg_ctx* c, double* ms)
{
    if (!c || !ms) return BCG_E_ARG;
    *ms = c->smooth_tune_ms;
    return BCG_OK;
}

/* pin the smoother's resident-warp target for a context (0 = the default
 * or the tuned value); used to profile a fixed kernel shape */
extern "C" int bcg_set_smoother_warps(bcg_ctx* c, int warps)
{
    if (!c || warps < 0) return BCG_E_ARG;
    c->smooth_warps = warps;
    nutrient_graphs_drop(c);
    return BCG_OK;
}

int mg_kernel_attributes()
{
    /* set on every context creation: attributes belong to the current
     * device, and the calls are cheap and thread-safe */
    if (cudaFuncSetAttribute(k_mg_coarse_smem<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_coarse_smem<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_coarse_wave<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_coarse_wave<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess)
        return BCG_E_CUDA;
    const int sm_d = SMOOTH_WARPS * 2 * SMOOTH_RING * 32 * 16, sm_f = sm_d / 2;
    if (cudaFuncSetAttribute(k_mg_smooth<double, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm_d) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_smooth<double, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm_d) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_smooth<double, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm_d) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_smooth<float, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm_f) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_smooth<float, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm_f) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_smooth<float, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm_f) != cudaSuccess)
        return BCG_E_CUDA;
    return mg_smooth_tma_attributes();
}

/* bcg_autotune(BCG_TUNE_SMOOTHER): time the fused smoother on the finest
 * level for several warp targets (two launches each, so the correction
 * buffers end where they started) and keep the fastest.  TMA form: 1 to
 * 16 row segments; per-lane staging form: its resident-warp targets. */
int mg_tune_smoother(bcg_ctx* c, int* choice)
{
    const int rows = c->mg[0].nz + 1;
    if (c->relax_mode < 2 || rows <= 96) { if (choice) *choice = 0; return BCG_OK; }
    MgConst m = mg_const(c, c->P.mg_dt);
    int targets[20];
    int nt = 0;
    if (c->relax_mode == 3) {
        /* fractions and multiples of the resident warp slots: one warp per
         * slot balances the SMs; fewer, longer segments save warm-up rows */
        const int slots = mg_smooth_tma_slots();
        const int num[9] = {1, 2, 3, 5, 1, 5, 3, 2, 3}, den[9] = {2, 3, 4, 6, 1, 4, 2, 1, 1};
        for (int i = 0; i < 9; i++) targets[nt++] = slots > 0 ? slots * num[i] / den[i] : 0;
    } else {
        const int t6[6] = {700, 1400, 2800, 5600, 8400, 11200};
        for (int i = 0; i < 6; i++) targets[nt++] = t6[i];
    }
    const int saved = c->smooth_warps;
    cudaEvent_t a, b;
    BCG_CUDA_TRY(cudaEventCreate(&a));
    BCG_CUDA_TRY(cudaEventCreate(&b));
    float best = 3.4e38f;
    int best_t = saved > 0 ? saved : (c->relax_mode == 3 ? SMOOTH_TMA_WARPS_DEFAULT : SMOOTH_WARPS_DEFAULT);
    for (int ti = 0; ti < nt; ti++) {
        c->smooth_warps = targets[ti];
        smooth_level<double>(c, m, 0, 3);                  /* warm-up */
        smooth_level<double>(c, m, 0, 3);
        cudaEventRecord(a, c->stream);
        smooth_level<double>(c, m, 0, 3);
        smooth_level<double>(c, m, 0, 3);
        cudaEventRecord(b, c->stream);
        if (cudaEventSynchronize(b) != cudaSuccess || c->pending_error) {
            cudaEventDestroy(a); cudaEventDestroy(b); c->smooth_warps = saved;
            const int rc = ctx_check_status(c);
            return rc ? rc : BCG_E_CUDA;
        }
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        if (ms < best) { best = ms; best_t = targets[ti]; c->smooth_tune_ms = ms / 2.0; }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    c->smooth_warps = best_t;
    c->mg_clean = 0;                 /* the trial sweeps wrote Err */
    nutrient_graphs_drop(c);
    if (choice) *choice = best_t;
    return ctx_check_status(c);
}

/* blocks per cluster of the coarsest-level solve, threads per block */
#define COARSE_CLUSTER 8
#define COARSE_THREADS 768
/* wavefront steps between cluster barriers (the halo width): at most 8,
 * and no wider than the narrowest block's columns */
static int coarse_halo(int W)
{
    int h = W / COARSE_CLUSTER;
    return h < 8 ? h : 8;
}
/* whether clusters of COARSE_CLUSTER blocks with `smem` bytes each can be
 * resident on the context's device; the answer is kept on the context per
 * precision and shared-memory size */
template <class T>
static bool coarse_cluster_ok(bcg_ctx* c, size_t smem)
{
    const int ti = sizeof(T) == 8 ? 0 : 1;
    if (c->cluster_smem[ti] == smem) return c->cluster_ok[ti] != 0;
    c->cluster_smem[ti] = smem;
    c->cluster_ok[ti] = 0;
    if (cudaFuncSetAttribute(k_mg_coarse_cluster<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(3 * COARSE_CLUSTER, 1, 1);
    cfg.blockDim = dim3(COARSE_THREADS, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = COARSE_CLUSTER;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_mg_coarse_cluster<T>, &cfg) == cudaSuccess && n >= 3) c->cluster_ok[ti] = 1;
    cudaGetLastError();
    return c->cluster_ok[ti] != 0;
}

/* mu2 sweeps on the coarsest level: fused when it fits one block */
template <class T>
static void relax_coarsest(bcg_ctx* c, const MgConst& m, int l, int sweeps)
{
    MgLvlT<T> L = lvl<T>(c, l);
    const size_t smem = 2 * sizeof(T) * (size_t)(L.nx + 1) * (L.nz + 1);
    const int H = coarse_halo(L.nx + 1);
    const size_t csmem = smem + 4 * (size_t)H * (L.nz + 1) * sizeof(T) + L.nx + 1;
    bool done = false;
    if (c->relax_mode >= 1 && csmem <= 200 * 1024 && L.nz >= 1 &&
        L.nx + 1 >= 2 * COARSE_CLUSTER && coarse_cluster_ok<T>(c, csmem)) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(3 * COARSE_CLUSTER, 1, 1);
        cfg.blockDim = dim3(COARSE_THREADS, 1, 1);
        cfg.dynamicSmemBytes = csmem;
        cfg.stream = c->stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = COARSE_CLUSTER;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        if (cudaLaunchKernelEx(&cfg, k_mg_coarse_cluster<T>, m, L, l, sweeps, H, (const double*)c->inside) == cudaSuccess) {
            c->launches++;
            done = true;
        } else {
            /* not launchable after all: use the one-block form from now on */
            cudaGetLastError();
            c->cluster_ok[sizeof(T) == 8 ? 0 : 1] = 0;
        }
    }
    if (done) return;
    if (c->relax_mode >= 1 && smem + L.nx + 1 <= 200 * 1024 && L.nz >= 1) {
        k_mg_coarse_wave<T><<<3, 1024, smem + (L.nx + 1), c->stream>>>(m, L, l, sweeps, c->inside);
        c->launches++;
    } else if (c->relax_mode >= 1 && smem <= 200 * 1024) {
        int ncol = (L.nx + 2) / 2;
        int threads = ((ncol + 31) / 32) * 32;
        if (threads > 1024) threads = 1024;
        k_mg_coarse_smem<T><<<3, threads, smem, c->stream>>>(m, L, l, sweeps, c->inside);
        c->launches++;
    } else if (c->relax_mode >= 1 && 3 * ((L.nx + 2) / 2) <= 4096 && L.nz + 1 <= 96) {
        k_mg_relax_coarse<T><<<1, 1024, 0, c->stream>>>(m, L, l, sweeps, c->inside);
        c->launches++;
    } else {
        for (int j = 0; j < sweeps; j++) relax_level<T>(c, m, l);
    }
}

/* rows of coarse level l that restrictionAgaElementwise writes: on a
 * composite level row 0 and the rows over the finer level (2k <= nzp),
 * on a plain coarsening all of them */
template <class T>
static int restrict_rows(const MgConst& m, const MgLvlT<T>& Lc, int l)
{
    if (l >= m.A) return Lc.nz + 1;
    const int d = 1 << l, d0 = 1 << m.A;
    const int nzp = m.box_z_agar * d0 / d < m.box_z_agar ? m.box_z_agar * d0 / d : m.box_z_agar;
    int last = nzp / 2;
    if (last > Lc.nz - 1) last = Lc.nz - 1;
    if (last < 0) last = 0;
    return last + 1;
}

/* Vcycle, Multigrid.cpp:843-862 */
template <class T>
void mg_vcycle_t(bcg_ctx* c, const MgConst& m, int mu1, int mu2)
{
    const int Lv = c->mg_levels;
    for (int l = 0; l < Lv - 1; l++) {
        smooth_level<T>(c, m, l, mu1);
        MgLvlT<T> Lc = lvl<T>(c, l + 1), Lf = lvl<T>(c, l);
        k_mg_restrict<T><<<grid_rows(Lc.nx + 1, restrict_rows(m, Lc, l + 1), 128), 128, 0, c->stream>>>(m, Lc, Lf, l + 1, c->inside);
        c->launches++;
    }
    relax_coarsest<T>(c, m, Lv - 1, mu2);
    for (int l = Lv - 2; l >= 0; l--) {
        MgLvlT<T> Lf = lvl<T>(c, l), Lc = lvl<T>(c, l + 1);
        k_mg_interp<T><<<grid_rows(Lf.nx / 2 + 1, Lf.nz + 1, 128), 128, 0, c->stream>>>(m, Lf, Lc, l);
        c->launches++;
        smooth_level<T>(c, m, l, mu1);
    }
}
template void mg_vcycle_t<double>(bcg_ctx*, const MgConst&, int, int);
template void mg_vcycle_t<float>(bcg_ctx*, const MgConst&, int, int);

void mg_vcycle(bcg_ctx* c, const MgConst& m, int mu1, int mu2) { mg_vcycle_t<double>(c, m, mu1, mu2); }

static void reset_zero(bcg_ctx* c, int from_level = 0)
{
    for (int l = from_level; l < c->mg_levels; l++) {
        MgLvl L = mg_lvl(c, l);
        k_mg_reset_zero<double><<<grid_rows(L.nx + 1, L.nz + 1, 256), 256, 0, c->stream>>>(L, l > 0);
        c->launches++;
    }
}
static void update_sol(bcg_ctx* c, const MgConst& m, int l, bool nest = false)
{
    MgLvl L = mg_lvl(c, l);
    const bool n = nest && l + 1 < m.A;
    MgLvl Ln = n ? mg_lvl(c, l + 1) : L;
    k_mg_update_sol<<<grid_rows(L.nx + 1, L.nz + 1, 256), 256, 0, c->stream>>>(m, L, l, Ln, n ? 1 : 0);
    c->launches++;
}
static void update_res(bcg_ctx* c, const MgConst& m, int l, bool setup_clean = false)
{
    MgLvl L = mg_lvl(c, l), Lp = mg_lvl(c, l > 0 ? l - 1 : 0);
    dim3 grid((unsigned)((L.nx + 1 + 127) / 128), (unsigned)(L.nz + 1), 3);
    const ResConst rc = res_const(m, l);
    if (l == 0) {
        if (setup_clean) k_mg_update_res<true, true><<<grid, 128, 0, c->stream>>>(m, L, Lp, l, rc, c->inside);
        else k_mg_update_res<false, true><<<grid, 128, 0, c->stream>>>(m, L, Lp, l, rc, c->inside);
    } else {
        if (setup_clean) k_mg_update_res<true, false><<<grid, 128, 0, c->stream>>>(m, L, Lp, l, rc, c->inside);
        else k_mg_update_res<false, false><<<grid, 128, 0, c->stream>>>(m, L, Lp, l, rc, c->inside);
    }
    c->launches++;
}

/* setup(), Multigrid.cpp:818-825 (both forms recompute level 0's Res) */
void mg_setup(bcg_ctx* c, const MgConst& m)
{
    c->mg_res0_stale = 0;
    if (c->mg_clean) {
        /* resetZero and updateSolAga have nothing to do but the clamp */
        c->mg_clean = 0;
        for (int l = 0; l <= m.A - 1; l++) update_res(c, m, l, true);
        return;
    }
    reset_zero(c);
    for (int l = 0; l <= m.A - 1; l++) update_sol(c, m, l);
    for (int l = 0; l <= m.A - 1; l++) update_res(c, m, l);
}

/* reset(), Multigrid.cpp:827-841 (evalUpdateRes's result is discarded there).
 * updateSolAga and NestSolAga run as one pass per level (update_sol with
 * nest).  Level 0's Res, which reset() recomputes last, is read by nothing
 * before the next setup() recomputes it: it is computed only when a caller
 * reads a multigrid array or changes its inputs (mg_res0_materialise). */
void mg_reset(bcg_ctx* c, const MgConst& m)
{
    for (int l = 0; l <= m.A - 1; l++) update_sol(c, m, l, true);
    for (int l = 0; l < m.A - 1; l++) {
        MgLvl L = mg_lvl(c, l), Lc = mg_lvl(c, l + 1);
        int n = L.nx + 1 + 2 * L.nz;
        k_mg_rewrite_bdry<<<grid2(n, 256), 256, 0, c->stream>>>(m, L, Lc, l);
        c->launches++;
    }
    /* the reference recomputes Res on every composite level here, and the
     * resetZero below clears it again on levels > 0: only level 0's stays,
     * computed on demand */
    c->mg_res0_stale = 1;
    /* updateSolAga already zeroed Err and Res on the composite levels */
    reset_zero(c, m.A);
    c->mg_clean = 1;
}

/* level 0's Res as reset() leaves it, before a caller reads or writes a
 * multigrid array or rewrites insideColonyDen */
void mg_res0_materialise(bcg_ctx* c)
{
    if (!c->mg_res0_stale) return;
    c->mg_res0_stale = 0;
    update_res(c, mg_const(c, c->P.mg_dt), 0);
}

void mg_copy_to(bcg_ctx* c, const MgConst& m, int wall_buf)
{
    MgLvl L0 = mg_lvl(c, 0);
    const WallBuf& w = c->wal[wall_buf];
    k_mg_copy_to<<<(m.box_x + 255) / 256, 256, 0, c->stream>>>(m, L0, w.C[0], w.O[0], w.A[0], c->inside);
    MgLvl La = mg_lvl(c, m.A - 1);
    k_mg_copy_edge<<<grid2(La.nz + 1, 256), 256, 0, c->stream>>>(La);
    c->launches += 2;
}

void mg_copy_from(bcg_ctx* c, const MgConst& m, int cur_wall)
{
    c->leg_old_stale = 1;        /* copyFromMG writes FieldAgar and oldFieldAgar alike */
    for (int l = 0; l < m.A; l++) {
        MgLvl L = mg_lvl(c, l);
        const WallBuf& cw = c->wal[cur_wall];
        const WallBuf& pw = c->wal[cur_wall ^ 1];
        k_mg_copy_from<<<(m.box_x + 255) / 256, 256, 0, c->stream>>>(L, m.box_x, cw.C[l], cw.O[l], cw.A[l], pw.C[l], pw.O[l], pw.A[l]);
        c->launches++;
    }
}

/* Multigrid::solve (Multigrid.cpp:864-889) with the given V-cycle count;
 * `wall_buf` is the wall buffer the caller's loop currently calls current */
int mg_solve_impl(bcg_ctx* c, int vcycles, int wall_buf)
{
    MgConst m = mg_const(c, c->P.mg_dt);
    mg_copy_to(c, m, wall_buf);
    mg_setup(c, m);
    for (int v = 0; v < vcycles; v++) mg_vcycle(c, m, c->P.mg_mu1, c->P.mg_mu2);
    mg_reset(c, m);
    mg_copy_from(c, m, wall_buf);
    if (c->pending_error) { const int rc = c->pending_error; c->pending_error = BCG_OK; return rc; }
    return cudaGetLastError() == cudaSuccess ? BCG_OK : BCG_E_CUDA;
}

/* Multigrid::solve as one graph launch.  A solve issues the same kernels
 * with the same arguments every time it starts from the same state: the
 * V-cycle count, the wall buffer and whether Err and Res are clean (the
 * first solve of a context runs the full setup(), later ones the clean
 * form).  The first solve from a state runs as plain launches, the second
 * is captured and later ones replay it; the graph is dropped with the
 * nutrient graphs, whenever a kernel shape of the context changes or a
 * caller writes a multigrid array. */
static int mg_solve_graphed(bcg_ctx* c, int vcycles, int wall_buf, cudaStream_t launch)
{
    const int key = (vcycles << 2) | (wall_buf << 1) | (c->mg_clean ? 1 : 0);
    if (c->solve_graph_off) return mg_solve_impl(c, vcycles, wall_buf);
    if (!c->solve_graph || c->solve_graph_key != key) {
        if (c->solve_graph) { cudaGraphExecDestroy(c->solve_graph); c->solve_graph = nullptr; }
        if (c->solve_graph_seen != key) {
            /* the first solve from a state runs as plain launches on the
             * context's stream: it makes the one-time queries (occupancy,
             * kernel attributes) a capture may not contain */
            c->solve_graph_seen = key;
            const long long l0 = c->launches;
            const int rc = mg_solve_impl(c, vcycles, wall_buf);
            c->solve_graph_launches = (int)(c->launches - l0);
            return rc;
        }
        /* the host state the captured pass changes, restored if the
         * capture fails (it ran nothing on the device) */
        const int s_clean = c->mg_clean, s_res0 = c->mg_res0_stale, s_leg = c->leg_old_stale;
        cudaGraph_t g = nullptr;
        BCG_CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        const long long l0 = c->launches;
        const int rc = mg_solve_impl(c, vcycles, wall_buf);
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        c->solve_graph_launches = (int)(c->launches - l0);
        c->launches = l0;
        if (!rc && e == cudaSuccess) {
            e = cudaGraphInstantiate(&c->solve_graph, g, 0);
            if (e != cudaSuccess) c->solve_graph = nullptr;
        }
        if (g) cudaGraphDestroy(g);
        if (rc || e != cudaSuccess) {
            /* a solve this context cannot capture: plain launches from now
             * on (a real error shows again there) */
            cudaGetLastError();
            c->mg_clean = s_clean; c->mg_res0_stale = s_res0; c->leg_old_stale = s_leg;
            c->pending_error = BCG_OK;
            c->solve_graph_off = 1;
            return mg_solve_impl(c, vcycles, wall_buf);
        }
        c->solve_graph_key = key;
    } else {
        /* the host state a solve leaves (mg_setup, mg_reset, mg_copy_from) */
        c->mg_res0_stale = 1;
        c->mg_clean = 1;
        c->leg_old_stale = 1;
    }
    BCG_CUDA_TRY(cudaGraphLaunch(c->solve_graph, launch));
    c->launches += c->solve_graph_launches;
    return BCG_OK;
}

extern "C" int bcg_mg_solve(bcg_ctx* c, int vcycles)
{
    if (!c) return BCG_E_ARG;
    if (vcycles <= 0) vcycles = c->P.mg_vcycles;
    timer_begin(c, BCG_T_MG_SOLVE);
    long long l0 = c->launches;
    int rc = mg_solve_graphed(c, vcycles, 0, c->stream);
    if (rc) return rc;
    timer_end(c, BCG_T_MG_SOLVE, (int)(c->launches - l0));
    return ctx_check_status(c);
}


/* ======================================================================== */
/* Tolerance-driven solve, FP64 and mixed precision (no reference           */
/* counterpart: the reference runs a fixed 3 V-cycles and discards its      */
/* residual, Multigrid.cpp:835, 869).                                       */
/* ======================================================================== */
/* Defect of the relaxation equations at the relaxed, uncovered points of a
 * composite level (the points updateSolAga updates, Multigrid.cpp:553-561):
 * for E = (R c + N(E)) / (c + 2) points it is R - ((c+2) E - N(E)) / c, for
 * Dirichlet points R - E.  Computed in FP64 from the FP64 right-hand side
 * and the current correction (FP64 or FP32 storage).  Max-norms of the
 * defect and of R go to out[0], out[1] as ordered bit patterns. */
template <class T>
__global__ void k_mg_defect(MgConst m, MgLvlT<T> L, MgLvl L64, int l, const double* __restrict__ inside0,
                            unsigned long long* out)
{
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    int sp = blockIdx.y;
    double dmax = 0.0, rmax = 0.0;
    if (idx < (L.nx + 1) * (L.nz + 1)) {
        int i = idx % (L.nx + 1), k = idx / (L.nx + 1);
        const int X = m.box_x, ZA = m.box_z_agar;
        int d = 1 << l, d0 = 1 << m.A;
        int nxp = X * d0 / d < X ? X * d0 / d : X;
        int nzp = ZA * d0 / d < ZA ? ZA * d0 / d : ZA;
        int ip = 2 * i - L.nx + nxp / 2, kp = 2 * k;
        bool uncovered = (l == 0 || ip <= 0 || ip >= nxp || kp >= nzp);
        if (uncovered) {
            int kind; double cfac;
            double v = relax_eval<T>(m, L, SP(L64.r), l, sp, i, k, inside0, kind, cfac);
            if (kind != 0) {
                double e = (double)AT(SP(L.e), L, i, k);
                double def = (kind == 1) ? (v - e) : (v - e) * (cfac + 2) / cfac;
                dmax = fabs(def);
                rmax = fabs(AT(SP(L64.r), L64, i, k));
            }
        }
    }
    for (int o = 16; o >= 1; o >>= 1) {
        dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
        rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
    }
    if ((threadIdx.x & 31) == 0) {
        /* non-negative doubles order like their bit patterns */
        if (dmax > 0) atomicMax(&out[0], (unsigned long long)__double_as_longlong(dmax));
        if (rmax > 0) atomicMax(&out[1], (unsigned long long)__double_as_longlong(rmax));
    }
}

template <class A, class B>
__global__ void k_mg_convert(const A* __restrict__ in, B* __restrict__ out, size_t n)
{
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (B)in[i];
}

/* relative defect over the composite levels; syncs the stream */
template <class T>
static int mg_rel_defect(bcg_ctx* c, const MgConst& m, double* rel, double* rhs_norm)
{
    unsigned long long* d = (unsigned long long*)c->mg_scratch;
    BCG_CUDA_TRY(cudaMemsetAsync(d, 0, 2 * sizeof(unsigned long long), c->stream));
    for (int l = 0; l < m.A; l++) {
        MgLvlT<T> L = lvl<T>(c, l);
        k_mg_defect<T><<<grid2((L.nx + 1) * (L.nz + 1), 256), 256, 0, c->stream>>>(m, L, mg_lvl(c, l), l, c->inside, d);
        c->launches++;
    }
    unsigned long long h[2];
    BCG_CUDA_TRY(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    BCG_CUDA_TRY(cudaStreamSynchronize(c->stream));
    double dm, rm;
    memcpy(&dm, &h[0], 8);
    memcpy(&rm, &h[1], 8);
    if (rhs_norm) *rhs_norm = rm;
    *rel = rm > 0 ? dm / rm : 0.0;
    return BCG_OK;
}

static void mg_convert_levels(bcg_ctx* c, bool to_float, bool res)
{
    for (int l = 0; l < c->mg_levels; l++) {
        MgLevel& L = c->mg[l];
        size_t n = (size_t)L.pitch * (L.nz + 1);
        for (int sp = 0; sp < 3; sp++) {
            if (to_float) {
                const double* src = res ? L.res[sp] : L.err[sp];
                float* dst = res ? L.resf[sp] : L.errf[sp];
                k_mg_convert<double, float><<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(src, dst, n);
            } else {
                const float* src = res ? L.resf[sp] : L.errf[sp];
                double* dst = res ? L.res[sp] : L.err[sp];
                k_mg_convert<float, double><<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(src, dst, n);
            }
            c->launches++;
        }
    }
}

extern "C" int bcg_mg_solve_tol(bcg_ctx* c, double rel_tol, int precision, int max_iters, int* iters, double* rel_res)
{
    if (!c || rel_tol <= 0 || max_iters < 1 || (precision != 32 && precision != 64)) return BCG_E_ARG;
    timer_begin(c, BCG_T_MG_SOLVE);
    long long l0 = c->launches;
    MgConst m = mg_const(c, c->P.mg_dt);
    mg_copy_to(c, m, 0);
    mg_setup(c, m);
    const int mu1 = c->P.mg_mu1, mu2 = c->P.mg_mu2;
    double rel = 1.0, r0 = 0.0;
    int rc = mg_rel_defect<double>(c, m, &rel, &r0);
    if (rc) return rc;
    int it = 0;
    if (r0 > 0) {
        rel = 1.0;
        if (precision == 32) {
            /* FP32 V-cycles on FP32 copies of Res/Err until the FP64 defect
             * stops falling by at least 2x per cycle (the FP32 floor) */
            mg_convert_levels(c, true, true);
            for (int l = 0; l < c->mg_levels; l++) {
                MgLvlF L = mg_lvl_f(c, l);
                k_mg_reset_zero<float><<<grid_rows(L.nx + 1, L.nz + 1, 256), 256, 0, c->stream>>>(L, 0);
                c->launches++;
            }
            double best = 1.0;
            while (it < max_iters) {
                mg_vcycle_t<float>(c, m, mu1, mu2);
                it++;
                if ((rc = mg_rel_defect<float>(c, m, &rel, nullptr))) return rc;
                if (rel < rel_tol || rel > 0.5 * best) break;
                best = rel;
            }
            /* FP64 refinement continues from the FP32 correction */
            mg_convert_levels(c, false, false);
        }
        while (rel >= rel_tol && it < max_iters) {
            mg_vcycle_t<double>(c, m, mu1, mu2);
            it++;
            if ((rc = mg_rel_defect<double>(c, m, &rel, nullptr))) return rc;
        }
    } else rel = 0.0;
    mg_reset(c, m);
    mg_copy_from(c, m, 0);
    BCG_CUDA_TRY(cudaGetLastError());
    timer_end(c, BCG_T_MG_SOLVE, (int)(c->launches - l0));
    if (iters) *iters = it;
    if (rel_res) *rel_res = rel;
    return ctx_check_status(c);
}

extern "C" int bcg_int_mg_solve_launch(bcg_ctx* c, int vcycles)
{
    if (!c) return BCG_E_ARG;
    if (vcycles <= 0) vcycles = c->P.mg_vcycles;
    return mg_solve_impl(c, vcycles, 0);
}

/* Multigrid::solve on the context's second stream, after the work queued
 * before it, beside the work queued after it until bcg_int_join.  The
 * caller queues nothing that reads or writes the multigrid arrays, the
 * agar and wall fields or the colony's density before the join.  With the
 * timers on, the solve is timed on its own stream (and waited for). */
extern "C" int bcg_int_mg_solve_aside(bcg_ctx* c, int vcycles)
{
    if (!c) return BCG_E_ARG;
    if (vcycles <= 0) vcycles = c->P.mg_vcycles;
    BCG_CUDA_TRY(cudaEventRecord(c->ev_fork, c->stream));
    BCG_CUDA_TRY(cudaStreamWaitEvent(c->aux_stream, c->ev_fork, 0));
    if (c->timers_on) cudaEventRecord(c->ev[BCG_T_MG_SOLVE][0], c->aux_stream);
    long long l0 = c->launches;
    bcg_int_tl_mark(c, 1, BCG_TL_SOLVE_BEGIN);
    int rc = mg_solve_graphed(c, vcycles, 0, c->aux_stream);
    if (rc) return rc;
    bcg_int_tl_mark(c, 1, BCG_TL_SOLVE_END);
    c->timer_launches[BCG_T_MG_SOLVE] += (int)(c->launches - l0);
    if (c->timers_on) {
        cudaEventRecord(c->ev[BCG_T_MG_SOLVE][1], c->aux_stream);
        cudaEventSynchronize(c->ev[BCG_T_MG_SOLVE][1]);
        float ms = 0;
        cudaEventElapsedTime(&ms, c->ev[BCG_T_MG_SOLVE][0], c->ev[BCG_T_MG_SOLVE][1]);
        c->timer_ms[BCG_T_MG_SOLVE] += ms;
    }
    return BCG_OK;
}
/* the context's stream waits for the second stream's work */
extern "C" int bcg_int_join(bcg_ctx* c)
{
    if (!c) return BCG_E_ARG;
    BCG_CUDA_TRY(cudaEventRecord(c->ev_join, c->aux_stream));
    BCG_CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
    return BCG_OK;
}

