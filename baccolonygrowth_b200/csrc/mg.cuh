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

/* One of three kernel-parameter array entries by a runtime index without
 * indexing the parameter array itself (a runtime index into a parameter
 * array makes the compiler copy the whole parameter block to per-thread
 * local memory). */
template <class P>
__device__ __forceinline__ P pick3(const P& a0, const P& a1, const P& a2, int i) { return i == 0 ? a0 : (i == 1 ? a1 : a2); }
#define SP(arr) pick3((arr)[0], (arr)[1], (arr)[2], sp)

