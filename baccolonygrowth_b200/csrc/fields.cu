/*
 * fields.cu -- cell-to-grid deposition and the surface fields
 * (AgentBasedModel-BacColonyGrowth/Compute.cpp:120-738).
 *
 * GetDensity / GetHeight walk the bins of the current record buffer (one
 * thread per x column, boxes bottom to top); ShiftDensity, BoxAverage,
 * Height_Average, Smooth and GetSurfaceNormal are stencil kernels bounded by
 * the device-resident bounding box, so the chain runs without host syncs.
 */
#include "ctx.cuh"
#include "cellmath.cuh"

int bin_cells(bcg_ctx* c, int buf);

#define IX(x, z) ((size_t)(x) * Z + (z))

__global__ void k_bbox_reset(int* bbox, int X)
{
    if (threadIdx.x == 0) { bbox[0] = X; bbox[1] = 0; bbox[2] = 0; }
}

/* GetDensity (Compute.cpp:120-227): per box sum of Length*Radius, the
 * inside flag, and per column the max top of the cells (starting from the
 * cell radius).  One thread per column. */
__global__ void k_get_density(int X, int Z, int rgh, double box_length, double cell_radius,
                              const CellRec* __restrict__ rec, const int* __restrict__ box_start,
                              const int* __restrict__ box_ids, double* __restrict__ rd,
                              double* __restrict__ inside, double* __restrict__ height, int* bbox)
{
    int bx = blockIdx.x * blockDim.x + threadIdx.x;
    if (bx >= X) return;
    double h[8];
    for (int i = 0; i < rgh && i < 8; i++) h[i] = cell_radius;
    const double Vbox = box_length * box_length;
    int any = 0, top_z = 0;
    for (int bz = 0; bz < Z; bz++) {
        int b = bx * Z + bz;
        int s = box_start[b], e = box_start[b + 1];
        double den = 0;
        for (int t = s; t < e; t++) {
            const CellRec& r = rec[box_ids[t]];
            double4 pl = r.pL, qr = r.qR;
            double cmx = (pl.x + qr.x) * 0.5;
            int i_ht = (int)((cmx / box_length - (bx - X / 2)) * rgh);
            if (i_ht < 0) i_ht = 0;
            if (i_ht > rgh - 1) i_ht = rgh - 1;
            double top = pl.z > qr.z ? pl.z : qr.z;
            if (i_ht < 8) h[i_ht] = h[i_ht] > top ? h[i_ht] : top;
            den += pl.w * qr.w;
        }
        if (e > s) { any = 1; top_z = bz; }
        if (den == 0) { rd[IX(bx, bz)] = 0; inside[IX(bx, bz)] = 0; }
        else { rd[IX(bx, bz)] = den / Vbox; inside[IX(bx, bz)] = 1.0; }
    }
    for (int i = 0; i < rgh && i < 8; i++) height[bx * rgh + i] = h[i];
    if (any) { atomicMin(&bbox[0], bx); atomicMax(&bbox[1], bx); atomicMax(&bbox[2], top_z); }
}

/* the boundary ring of insideColonyDen, Compute.cpp:228-249 (reads only
 * values > 0.5, so the in-place order does not matter) */
__global__ void k_inside_ring(int X, int Z, double* inside)
{
    int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= X * Z) return;
    int bx = id / Z, bz = id % Z;
    if (inside[id] < 0.5) {
        if (bz > 0 && bx > 0 && bx < X - 1 && bz < Z - 1) {
            if ((inside[IX(bx + 1, bz)] > 0.5) || (inside[IX(bx - 1, bz)] > 0.5) || (inside[IX(bx, bz + 1)] > 0.5) || (inside[IX(bx, bz - 1)] > 0.5))
                inside[id] = 0.4;
        } else if (bz == 0 && bx > 0 && bx < X - 1) {
            if ((inside[IX(bx + 1, bz)] > 0.5) || (inside[IX(bx - 1, bz)] > 0.5) || (inside[IX(bx, bz + 1)] > 0.5))
                inside[id] = 0.4;
        }
    }
}

/* GetHeight (Compute.cpp:256-340): top four occupied boxes per column */
__global__ void k_get_height(int X, int Z, int rgh, double box_length, double cell_radius,
                             const CellRec* __restrict__ rec, const int* __restrict__ box_start,
                             const int* __restrict__ box_ids, double* __restrict__ height, int* bbox)
{
    int bx = blockIdx.x * blockDim.x + threadIdx.x;
    if (bx >= X) return;
    double h[8];
    for (int i = 0; i < rgh && i < 8; i++) h[i] = cell_radius;
    int pos_ct = 0, top_z = -1;
    for (int bz = Z - 1; bz >= 0; bz--) {
        int b = bx * Z + bz;
        int s = box_start[b], e = box_start[b + 1];
        if (e > s) { pos_ct++; if (top_z < 0) top_z = bz; }
        for (int t = s; t < e; t++) {
            const CellRec& r = rec[box_ids[t]];
            double4 pl = r.pL, qr = r.qR;
            double cmx = (pl.x + qr.x) * 0.5;
            int i_ht = (int)((cmx - (bx - X / 2) * box_length) / (box_length / rgh));
            if (i_ht < 0) i_ht = 0;
            if (i_ht > rgh - 1) i_ht = rgh - 1;
            double top = pl.z > qr.z ? pl.z : qr.z;
            if (i_ht < 8) h[i_ht] = h[i_ht] > top ? h[i_ht] : top;
        }
        if (pos_ct > 3) break;
    }
    for (int i = 0; i < rgh && i < 8; i++) height[bx * rgh + i] = h[i];
    if (top_z >= 0) { atomicMin(&bbox[0], bx); atomicMax(&bbox[1], bx); atomicMax(&bbox[2], top_z); }
}

/* minx-5, maxx+5, maxz+5 (Compute.cpp:250-252) and the range the stencils
 * below need (the reference reads outside its arrays otherwise) */
__global__ void k_bbox_finish(int* bbox, int X, int Z, int FD, DevStatus* st)
{
    if (threadIdx.x != 0) return;
    if (bbox[0] > bbox[1]) { bbox[0] = X - 5; bbox[1] = 5; bbox[2] = 5; return; }   /* no cells */
    bbox[0] -= 5; bbox[1] += 5; bbox[2] += 5;
    if (bbox[0] - FD < 1 || bbox[1] + FD > X - 2 || bbox[2] + FD > Z) dev_error(st, BCG_E_NEED_MORE_BOXES, bbox[1]);
}

/* ShiftDensity (Compute.cpp:344-463) with Box_y = 1: the y = BoxY-1 passes
 * overwrite the 8-point averages, leaving these values. */
__global__ void k_shift(int X, int Z, const double* __restrict__ D, double* __restrict__ DS, double* __restrict__ WS)
{
    int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= X * Z) return;
    int x = id / Z, z = id % Z;
    double v;
    if (x < X - 1 && z < Z - 1) v = (D[IX(x, z)] + D[IX(x, z + 1)] + D[IX(x + 1, z)] + D[IX(x + 1, z + 1)]) / 4.0;
    else if (x < X - 1) v = (D[IX(x, Z - 1)] + D[IX(x + 1, Z - 1)]) / 2.0;
    else if (z < Z - 1) v = (D[IX(X - 1, z)] + D[IX(X - 1, z)]) / 2.0;
    else v = D[IX(X - 1, Z - 1)];
    DS[id] = v;
    if (z == 0 && WS) WS[x] = (x < X - 1) ? (D[IX(x, 0)] + D[IX(x + 1, 0)]) / 2.0 : D[IX(X - 1, 0)];
}

struct Filter5 { double w[8][8]; };

/* BoxAverage (Compute.cpp:495-605): filter over x-z of the array with the
 * wall row prepended, min(1, avg / density_threshold), inside the bbox. */
__global__ void k_box_average(int X, int Z, int FL, Filter5 f, double thr, const int* __restrict__ bbox,
                              const double* __restrict__ rough, const double* __restrict__ rough_wall,
                              double* __restrict__ out, double* __restrict__ out_wall)
{
    int minx = bbox[0], maxx = bbox[1], maxz = bbox[2];
    int ia = minx + blockIdx.x * blockDim.x + threadIdx.x;
    int ka = blockIdx.y;
    const int FD = FL / 2;
    if (minx - FD < 0 || maxx + FD > X || maxz + FD > Z) return;   /* reported by k_bbox_finish */
    if (ia >= maxx || ka > maxz) return;
    double a = 0.0;
    for (int fi = -FD; fi <= FD; fi++)
        for (int fk = -FD; fk <= FD; fk++) {
            int i = ia + fi, k = ka + fk;
            double w = f.w[fi + FD][fk + FD];
            if (k < 0) {
                double in0 = rough_wall[i];
                if (in0 > 0.00001) a += w * 1.0;
                else a += w * in0;
            } else {
                double in = (k == 0) ? rough_wall[i] : rough[IX(i, k - 1)];
                a += w * in;
            }
        }
    double v = dmin_(1.0, a / thr);
    if (ka == 0) out_wall[ia] = v;
    else if (ka - 1 < Z) out[IX(ia, ka - 1)] = v;
}

/* Height_Average (Compute.cpp:669-705) */
__global__ void k_height_average(int rgh, int xh, const int* __restrict__ bbox, const double* __restrict__ in, double* __restrict__ out)
{
    int i = bbox[0] * rgh + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (bbox[1] + 1) * rgh || i < 1 || i > xh - 2) return;
    double H0 = in[i], Ht = H0;
    int count = 1;
    double H = in[i - 1];
    if (H < H0) { Ht += H; count++; }
    H = in[i + 1];
    if (H < H0) { Ht += H; count++; }
    out[i] = Ht / count;
}
/* Smooth (Compute.cpp:708-738) with the 1/FilterLen box filter */
__global__ void k_smooth(int rgh, int xh, int FL, double w, const int* __restrict__ bbox, const double* __restrict__ in, double* __restrict__ out)
{
    int i = bbox[0] * rgh + blockIdx.x * blockDim.x + threadIdx.x;
    int FD = FL / 2;
    if (i >= (bbox[1] + 1) * rgh || i - FD < 0 || i + FD > xh - 1) return;
    double a = 0.0;
    for (int f = -FD; f <= FD; f++) a += w * in[i + f];
    out[i] = a;
}
/* GetSurfaceNormal (Compute.cpp:466-491) */
__global__ void k_normal(int rgh, int xh, double box_length, const int* __restrict__ bbox, const double* __restrict__ h,
                         double* __restrict__ nx, double* __restrict__ ny, double* __restrict__ nz)
{
    int i = bbox[0] * rgh + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (bbox[1] + 1) * rgh || i < 1 || i > xh - 2) return;
    double d_x = (h[i + 1] - h[i - 1]) / (2.0 * box_length / rgh);
    double d_z = -1.0;
    double l_n = sqrt(d_x * d_x + d_z * d_z);
    nx[i] = d_x / l_n; ny[i] = 0; nz[i] = d_z / l_n;
}

static Filter5 make_filter(int FL)
{
    /* Filter3D of Simulation.cpp:87-110 */
    Filter5 f;
    double norm = 0;
    for (int ii = 0; ii < FL; ii++)
        for (int kk = 0; kk < FL; kk++)
            norm = norm + exp(-(ii - FL / 2) * (ii - FL / 2) - (kk - FL / 2) * (kk - FL / 2));
    for (int ii = 0; ii < FL; ii++)
        for (int kk = 0; kk < FL; kk++)
            f.w[ii][kk] = exp(-(ii - FL / 2) * (ii - FL / 2) - (kk - FL / 2) * (kk - FL / 2)) / norm;
    return f;
}

static int launch_surface(bcg_ctx* c, bool smooth)
{
    const bcg_params& P = c->P;
    const int rgh = P.refinement_grid_height;
    const int XH = P.box_x * rgh;
    unsigned g = (unsigned)((XH + 255) / 256);
    if (smooth) {
        k_height_average<<<g, 256, 0, c->stream>>>(rgh, XH, c->bbox, c->height, c->rough_height);
        k_smooth<<<g, 256, 0, c->stream>>>(rgh, XH, P.filter_len, 1.0 / (double)(P.filter_len), c->bbox, c->rough_height, c->height);
        c->launches += 2;
    }
    k_normal<<<g, 256, 0, c->stream>>>(rgh, XH, P.box_length, c->bbox, c->height, c->nrm_x, c->nrm_y, c->nrm_z);
    c->launches++;
    return cudaGetLastError() == cudaSuccess ? BCG_OK : BCG_E_CUDA;
}

static int deposit(bcg_ctx* c, bool smooth)
{
    const bcg_params& P = c->P;
    if (P.filter_len > 8 || P.refinement_grid_height > 8) return BCG_E_UNSUPPORTED;
    mg_res0_materialise(c);            /* it reads insideColonyDen, rewritten here */
    timer_begin(c, BCG_T_DENSITY);
    int rc = bin_cells(c, c->cur);
    if (rc) return rc;
    const int X = P.box_x, Z = P.box_z;
    k_bbox_reset<<<1, 32, 0, c->stream>>>(c->bbox, X);
    k_get_density<<<(X + 127) / 128, 128, 0, c->stream>>>(X, Z, P.refinement_grid_height, P.box_length, P.cell_radius,
        c->rec[c->cur], c->box_start, c->box_ids, c->rd, c->inside, c->height, c->bbox);
    k_inside_ring<<<(X * Z + 255) / 256, 256, 0, c->stream>>>(X, Z, c->inside);
    k_bbox_finish<<<1, 32, 0, c->stream>>>(c->bbox, X, Z, P.filter_len / 2, c->status);
    k_shift<<<(X * Z + 255) / 256, 256, 0, c->stream>>>(X, Z, c->rd, c->rds, c->rws);
    Filter5 f = make_filter(P.filter_len);
    dim3 grid((X + 127) / 128, Z + 1);
    /* Density from RoughDensity (RoughWallDensity stays zero, ShiftDensity
     * never writes it) and DensityShiftP from RoughDensityShiftP */
    k_box_average<<<grid, 128, 0, c->stream>>>(X, Z, P.filter_len, f, P.density_threshold, c->bbox, c->rd, c->rw, c->dens, c->wd);
    k_box_average<<<grid, 128, 0, c->stream>>>(X, Z, P.filter_len, f, P.density_threshold, c->bbox, c->rds, c->rws, c->ds, c->wds);
    c->launches += 7;
    rc = launch_surface(c, smooth);
    if (rc) return rc;
    timer_end(c, BCG_T_DENSITY, 0);
    return ctx_check_status(c);
}

extern "C" int bcg_update_density(bcg_ctx* c) { return c ? deposit(c, true) : BCG_E_ARG; }
extern "C" int bcg_initial_density(bcg_ctx* c) { return c ? deposit(c, false) : BCG_E_ARG; }

extern "C" int bcg_update_height(bcg_ctx* c)
{
    if (!c) return BCG_E_ARG;
    const bcg_params& P = c->P;
    if (P.refinement_grid_height > 8) return BCG_E_UNSUPPORTED;
    timer_begin(c, BCG_T_DENSITY);
    int rc = bin_cells(c, c->cur);
    if (rc) return rc;
    const int X = P.box_x, Z = P.box_z;
    k_bbox_reset<<<1, 32, 0, c->stream>>>(c->bbox, X);
    k_get_height<<<(X + 127) / 128, 128, 0, c->stream>>>(X, Z, P.refinement_grid_height, P.box_length, P.cell_radius,
        c->rec[c->cur], c->box_start, c->box_ids, c->height, c->bbox);
    k_bbox_finish<<<1, 32, 0, c->stream>>>(c->bbox, X, Z, P.filter_len / 2, c->status);
    c->launches += 3;
    rc = launch_surface(c, true);
    if (rc) return rc;
    timer_end(c, BCG_T_DENSITY, 0);
    return ctx_check_status(c);
}
