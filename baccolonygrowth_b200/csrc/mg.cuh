/* mg.cuh -- shared declarations of the multigrid and sweep translation units */
#pragma once
#include "ctx.cuh"

struct MgConst {
    int A;            /* composite (agar) levels, maxLevelsMG */
    int levels;       /* multigrid levels (8 in the reference) */
    int box_x, box_z_agar, box_z;
    double bl2;       /* BoxLength^2 */
    double dt;        /* the solve's time step (100 in the reference) */
    double D[3];      /* agar diffusivities: carbon, oxygen, acetate */
    double max_carbon, max_o2_agar;
};

/* one level as the kernels see it: the solution is always FP64; the
 * correction (Err) and right-hand side (Res) are T = double or float */
template <class T>
struct MgLvlT {
    int nx, nz, pitch;
    double* s[3];
    T* r[3];
    T* e[3];
    T* e2[3];         /* the other correction buffer (fused smoother output) */
};
typedef MgLvlT<double> MgLvl;
typedef MgLvlT<float> MgLvlF;

MgConst mg_const(const bcg_ctx* c, double dt);
MgLvl mg_lvl(const bcg_ctx* c, int l);
MgLvlF mg_lvl_f(const bcg_ctx* c, int l);
template <class T> void mg_vcycle_t(bcg_ctx* c, const MgConst& m, int mu1, int mu2);
void mg_vcycle(bcg_ctx* c, const MgConst& m, int mu1, int mu2);
void mg_setup(bcg_ctx* c, const MgConst& m);
void mg_reset(bcg_ctx* c, const MgConst& m);
void mg_copy_to(bcg_ctx* c, const MgConst& m, int wall_buf);
void mg_copy_from(bcg_ctx* c, const MgConst& m, int cur_wall);
int mg_solve_impl(bcg_ctx* c, int vcycles, int wall_buf);
/* the TMA-staged fused smoother (mg_smooth.cu): S sweeps of level L from
 * E into E2 with about `target_warps` warps (one row segment of one strip
 * of one species each; 0 = one per resident slot) */
int mg_smooth_tma(bcg_ctx* c, const MgConst& m, const MgLvl& L, int l, int S, int target_warps, int warm);
int mg_smooth_tma(bcg_ctx* c, const MgConst& m, const MgLvlF& L, int l, int S, int target_warps, int warm);
/* resident warps of mg_smooth_tma on the current device */
int mg_smooth_tma_slots();
/* kernel attributes of mg_smooth_tma (on context creation) */
int mg_smooth_tma_attributes();
/* whether mg_smooth_tma takes a level with nx + 1 columns */
int mg_smooth_tma_fits(int nx);

/* One of three kernel-parameter array entries by a runtime index without
 * indexing the parameter array itself (a runtime index into a parameter
 * array makes the compiler copy the whole parameter block to per-thread
 * local memory). */
template <class P>
__device__ __forceinline__ P pick3(const P& a0, const P& a1, const P& a2, int i) { return i == 0 ? a0 : (i == 1 ? a1 : a2); }
#define SP(arr) pick3((arr)[0], (arr)[1], (arr)[2], sp)


/* The relaxation update of relaxationAgarElementwise (Multigrid.cpp:160-249)
 *   E = (R h^2/(dt D) + sum of weighted neighbours) / (h^2/(dt D) + 2)
 * with cf = h^2/(dt D), inv = 1/(cf + 2), c = cf inv and w = inv/2 taken
 * once per level and species, as E = c R + inv (neighbours weighted 1) +
 * w (neighbours weighted 1/2), the value below added last so that the
 * column recurrence is one fused multiply-add deep (the reference divides
 * per point; the results differ by rounding). */
template <class T> struct RelaxK { T cf, inv, c, w; };
template <class T>
__device__ __forceinline__ RelaxK<T> relax_k(const MgConst& m, int l, int sp)
{
    const double cf = m.bl2 * (double)(1 << (2 * l)) / m.dt / SP(m.D);
    const double inv = 1.0 / (cf + 2.0);
    RelaxK<T> k; k.cf = (T)cf; k.inv = (T)inv; k.c = (T)(cf * inv); k.w = (T)(0.5 * inv);
    return k;
}
/* interior: neighbours below, above, left, right with weight 1/2 */
template <class T> __device__ __forceinline__ T rx_in(T r, T b, T u, T xm, T xp, const RelaxK<T>& K)
{ return fma(K.w, b, fma(K.w, (xm + xp) + u, K.c * r)); }
/* bottom row (k = 0): above weight 1, sides 1/2 */
template <class T> __device__ __forceinline__ T rx_k0(T r, T u, T xm, T xp, const RelaxK<T>& K)
{ return fma(K.inv, u, fma(K.w, xm + xp, K.c * r)); }
/* top row (k = nz): below weight 1, sides 1/2 */
template <class T> __device__ __forceinline__ T rx_top(T r, T b, T xm, T xp, const RelaxK<T>& K)
{ return fma(K.inv, b, fma(K.w, xm + xp, K.c * r)); }
/* side column (i = 0 or nx), interior row: inner neighbour weight 1 */
template <class T> __device__ __forceinline__ T rx_side(T r, T b, T u, T s1, const RelaxK<T>& K)
{ return fma(K.w, b, fma(K.w, u, fma(K.inv, s1, K.c * r))); }
/* corners: inner neighbour and the one vertical neighbour, weight 1 each */
template <class T> __device__ __forceinline__ T rx_corner(T r, T s1, T v, const RelaxK<T>& K)
{ return fma(K.inv, v, fma(K.inv, s1, K.c * r)); }

/* The relaxation of relax_point with the stencil values passed in:
 * below = new value at (i, k-1), up = value at (i, k+1) before this sweep,
 * xm/xp = values at (i-1, k)/(i+1, k) as the sweep order sees them, old =
 * the point's value before this sweep (kept where the point is not relaxed).
 * Same operations as relax_point. */
template <class T>
__device__ __forceinline__ T relax_val(const MgConst& m, const RelaxK<T>& K, int nx, int nz, int l, int sp, int i, int k,
                                       T r, T below, T up, T xm, T xp, T old, const double* __restrict__ inside0)
{
    const bool oxy = (sp == 1);
    const bool top_levels = l >= m.A - 1;
    const bool side = (i == 0 || i == nx);
    const T s1 = (i == 0) ? xp : xm;
    if (k == 0) {
        int d = 1 << l;
        int i0 = (i - nx / 2) * d + m.box_x / 2;
        i0 = i0 < 0 ? 0 : (i0 > m.box_x - 1 ? m.box_x - 1 : i0);
        if (inside0[(size_t)i0 * m.box_z] > 0) return r;
        if (side) {
            if (!top_levels) return old;
            if (oxy) return r;
            return rx_corner(r, s1, up, K);
        }
        if (oxy) return r;
        return rx_k0(r, up, xm, xp, K);
    }
    if (k == nz) {
        if (!top_levels) return old;
        if (side) {
            if (oxy) return r;
            return rx_corner(r, s1, below, K);
        }
        return rx_top(r, below, xm, xp, K);
    }
    if (side) {
        if (!top_levels) return old;
        if (oxy) return r;
        return rx_side(r, below, up, s1, K);
    }
    return rx_in(r, below, up, xm, xp, K);
}

/* Interior rows (0 < k < nz) need only the column's kind, fixed per lane:
 * 0 interior column, 1 left side (i = 0), 2 right side (i = nx), 3 side
 * held at R (oxygen on the top levels), 4 side not relaxed (keeps old). */
__device__ __forceinline__ int col_kind(int i, int nx, bool oxy, bool top_levels)
{
    if (i != 0 && i != nx) return 0;
    if (!top_levels) return 4;
    if (oxy) return 3;
    return i == 0 ? 1 : 2;
}
template <class T>
__device__ __forceinline__ T rx_row(int kind, T r, T below, T up, T xm, T xp, T old, const RelaxK<T>& K)
{
    if (kind == 0) return rx_in(r, below, up, xm, xp, K);
    if (kind == 1) return rx_side(r, below, up, xp, K);
    if (kind == 2) return rx_side(r, below, up, xm, K);
    return kind == 3 ? r : old;
}

