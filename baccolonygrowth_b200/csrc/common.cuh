/*
 * common.cuh -- device-side data layout of a bcg_ctx and shared helpers.
 *
 * Layout in HBM (one context = one colony on one GPU):
 *  - cell gather records, two buffers (old/new, swapped every step):
 *      CellRec { double4 pL; double4 qR; double4 v; double4 w; }  (128 B)
 *    one record is one 128-byte line, so a neighbour fetch in the force
 *    loop is a single line; the rest of the Cell fields are
 *    structure-of-arrays (single buffer: they are written only by the step
 *    that owns them).
 *  - reduced neighbour lists: nbr[i*kmax + j], ncount[i].
 *  - bins (counting sort): box_cnt[nbox], box_start[nbox+1], box_ids[N],
 *    cell_box[N].
 *  - fields: x-major, z fastest (Array2D/Array3D index x*Z+z with Y=1),
 *    one array per quantity (SoA), FP64.
 */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/bcg.h"

#define BCG_PI 3.141592653589793238462643383279502884197

struct __align__(32) CellRec {
    double4 pL;   /* p.x p.y p.z Length */
    double4 qR;   /* q.x q.y q.z Radius */
    double4 v;    /* Velocity, .w unused */
    double4 w;    /* AngularVelocity, .w unused */
};

/* error word bits written by kernels (first error wins via atomicCAS) */
struct DevStatus {
    int code;         /* bcg_status of the first device-side error */
    int info;         /* index of the offending cell / box */
};

/* Parameters the kernels read, copied by value into each launch. */
/* divisions per step handled by bcg_divide, and the footprint-overlap
 * pairs its planner records before falling back to one sequential group */
#define DIV_SORT_MAX 8192
#define DIV_PAIR_CAP 65536
#define DIV_PLAN_SMEM (3 * DIV_SORT_MAX * 4)   /* k_div_plan's dynamic shared memory */

struct MechParams {
    int box_x, box_y, box_z, rgh;
    int xh;             /* Height/Normal length, box_x*rgh */
    int kmax, box_cap;
    double box_length, rc, cell_radius, l_divide;
    double k_cc, k_wc, var_l, var_angle, var_pos, viscosity, gamma_t, cell_mu, wall_mu;
    double tension, delta_h;
    int cross_feeding;
};

struct FieldPtrs {
    const double* height;   /* box_x*rgh */
    const double* nx;       /* Normal.x */
    const double* ny;       /* Normal.y */
    const double* nz;       /* Normal.z */
    const double* wall;     /* box_x*box_y */
    const double* gr1;      /* Environment.GrowthRate1, box_x*box_z */
    const double* gr2;      /* Environment.GrowthRate2 */
};

struct CellSoA {
    double* ldiv; double* gr; double* tp; double* tq; int* ap; int* aq;
    double* dfx; double* dfy; double* dfz; double* sfx; double* sfy; double* sfz;
    int* type; int* anc;
};

/* forward declarations of the context (defined in ctx.cu) */
struct bcg_ctx;

#define BCG_CUDA_TRY(expr) do { cudaError_t e_ = (expr); if (e_ != cudaSuccess) { bcg_set_cuda_error(e_); return BCG_E_CUDA; } } while (0)
void bcg_set_cuda_error(cudaError_t e);

/* device helpers ------------------------------------------------------------ */
__device__ __forceinline__ void dev_error(DevStatus* st, int code, int info)
{
    if (atomicCAS(&st->code, 0, code) == 0) st->info = info;
}
