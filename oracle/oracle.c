/*
 * oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of the BacColonyGrowth hot path, written from the
 * reference's behaviour (citations are file:line inside
 * AgentBasedModel-BacColonyGrowth/).  It is the checker of the CUDA
 * library: tests compare the library against it, and it is pinned against
 * the reference itself (oracle/_ref) and against committed golden vectors.
 *
 * Every expression keeps the reference's operation order (products left to
 * right, reciprocal-then-multiply where the reference scales by 1/x, float
 * casts where the reference casts) so that, built without FMA contraction,
 * the mechanics are bit-identical to the reference at 1 thread.  The box
 * lists keep the reference's add / swap-remove order (UniformGrid.h:33-55),
 * so neighbour lists come out in the reference's order too.
 *
 * The oracle owns a private glibc-compatible rand() (TYPE_3: r[i] =
 * r[i-31] + r[i-3], output r >> 1), drawn in the same places as the
 * reference's rand().
 */
#include <math.h>
#include <float.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include <stdint.h>
#include "oracle.h"

static const double PI = 3.141592653589793238462643383279502884197;

/* ---------------------------------------------------------------- rand ---- */
typedef struct { uint32_t r[34]; int i; } grand;
static void grand_seed(grand* g, uint32_t seed)
{
    uint32_t r[344];
    int32_t s = (int32_t)seed; if (s == 0) s = 1;
    r[0] = (uint32_t)s;
    for (int i = 1; i < 31; i++) {
        long long w = (16807LL * (long long)(int32_t)r[i - 1]) % 2147483647LL;
        if (w < 0) w += 2147483647LL;
        r[i] = (uint32_t)w;
    }
    for (int i = 31; i < 34; i++) r[i] = r[i - 31];
    for (int i = 34; i < 344; i++) r[i] = r[i - 31] + r[i - 3];
    for (int i = 0; i < 34; i++) g->r[i] = r[310 + i];
    g->i = 0;   /* ring position of the oldest value */
}
static int grand_next(grand* g)
{
    /* ring holds the last 34 values, oldest at g->i */
    uint32_t v = g->r[(g->i + 3) % 34] + g->r[(g->i + 31) % 34];
    g->r[g->i] = v;
    g->i = (g->i + 1) % 34;
    return (int)(v >> 1);
}
#define RAND_MAX_ 2147483647

/* ---------------------------------------------------------------- types --- */
typedef bcg_vec3 V3;
static inline V3 v3(double x, double y, double z) { V3 r = {x, y, z}; return r; }
static inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, -a.x * b.z + a.z * b.x, a.x * b.y - a.y * b.x); }
static inline V3 vdiff(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 vsum(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 vscale(V3 a, double c) { return v3(a.x * c, a.y * c, a.z * c); }
static inline V3 avg(const bcg_cell* c) { return vscale(vsum(c->p, c->q), 0.5); }
static inline double dmax(double a, double b) { return a > b ? a : b; }
static inline double dmin(double a, double b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }
static inline int imin(int a, int b) { return a < b ? a : b; }

/* LocalEnv (Nutrients.h:11-64) and LocalAga (Nutrients.h:66-82) */
typedef struct {
    double Carbon, Waste, GrowthRate1, GrowthRate2, Oxygen, Acetate;
    double pH, Buffer, Acetic, Hydrox;
    double qCarmnt, qAcemnt, pAcemnt, qOxymnt;
    double GrCarAer, GrCarAna, GrAceAer;
} env_t;
typedef struct { double C, W, O, A; } aga_t;

struct orc_state {
    bcg_params P;
    grand rng;
    long long rand_calls;
    int err;
    int N;
    bcg_cell *oldc, *newc;
    /* UniformGrid boxes */
    int nbox, box_cap;
    int* box_count;
    int* box_ids;
    /* neighbour lists: row i = [count, ids...] */
    int nbr_stride;
    int* nbr;
    int* dividing; int ndiv;
    int* idlist;
    /* fields */
    double *height, *rough_height, *normal_x, *normal_y, *normal_z, *wall;
    double t, dt;
    /* colony environment: env = Environment, oenv = oldEnvironment */
    env_t *env, *oenv;
    /* per composite level: FieldAgar / oldFieldAgar (X*ZA), FieldWall / oldFieldWall (X) */
    aga_t **agar, **oagar, **wal, **owal;
    /* Multigrid arrays per MG level, (nx+1)*(nz+1), x-major */
    aga_t **mgA, **mgR, **mgE;
    int mg_levels;
    double mg_dt;
    /* deposition arrays (X*Z) and wall rows (X) */
    double *rd, *rd1, *rd2, *inside, *rds, *rd1s, *rd2s, *dens, *dens1, *dens2, *ds, *d1s, *d2s;
    double *rw, *rw1, *rw2, *rws, *rw1s, *rw2s, *wd, *wd1, *wd2, *wds, *wd1s, *wd2s;
    double filter3d[64 * 64];
    double filter1d[64];
    int minx, maxx, miny, maxy, maxz;
    double next_out, next_update, hd_next_update, hd_update;
    int update_flag, hd_update_flag;
};

static int rnd(orc_state* s) { s->rand_calls++; return grand_next(&s->rng); }
static double frand(orc_state* s) { return (double)((float)rnd(s) / (float)RAND_MAX_); }

/* ------------------------------------------------------- UniformGrid ------ */
/* GetAddress, UniformGrid.h:87-99 */
static int get_address(orc_state* s, V3 pos, int* xi, int* yi, int* zi)
{
    const bcg_params* P = &s->P;
    int x = (int)(pos.x / P->box_length + P->box_x / 2);
    int y = (int)(pos.y / P->box_length + P->box_y / 2 + 0.5);
    int z = (int)(pos.z / P->box_length);
    if (!((x < P->box_x) & (y < P->box_y) & (z < P->box_z) & (x >= 0) & (y >= 0) & (z >= 0))) {
        if (!s->err) s->err = BCG_E_OUT_OF_GRID;
        x = imin(imax(x, 0), P->box_x - 1); y = imin(imax(y, 0), P->box_y - 1); z = imin(imax(z, 0), P->box_z - 1);
    }
    if (xi) { *xi = x; *yi = y; *zi = z; }
    return x * (P->box_y * P->box_z) + y * P->box_z + z;
}
/* Box::Add / Box::Remove, UniformGrid.h:33-55 */
static void box_add(orc_state* s, int id, int a)
{
    if (!(s->box_count[a] + 1 < s->box_cap)) { if (!s->err) s->err = BCG_E_BOX_OVERFLOW; return; }
    s->box_ids[(size_t)a * s->box_cap + s->box_count[a]] = id;
    s->box_count[a]++;
}
static void box_remove(orc_state* s, int id, int a)
{
    int* ids = s->box_ids + (size_t)a * s->box_cap;
    int ii = 0;
    while ((ids[ii] != id) & (ii < s->box_count[a])) ii++;
    if (ii == s->box_count[a]) { if (!s->err) s->err = BCG_E_BOX_OVERFLOW; return; }
    ids[ii] = ids[s->box_count[a] - 1];
    s->box_count[a]--;
}
/* GetNeighbours, UniformGrid.h:141-170: z outer, y, x inner, box order */
static int grid_neighbours(orc_state* s, int id, int a, int* out)
{
    const bcg_params* P = &s->P;
    int YZ = P->box_y * P->box_z;
    int x0 = a / YZ, r = a - x0 * YZ, y0 = r / P->box_z, z0 = r % P->box_z;
    int found = 1;
    for (int za = imax(z0 - 1, 0); za < imin(z0 + 2, P->box_z); za++)
        for (int ya = imax(y0 - 1, 0); ya < imin(y0 + 2, P->box_y); ya++)
            for (int xa = imax(x0 - 1, 0); xa < imin(x0 + 2, P->box_x); xa++) {
                int b = xa * YZ + ya * P->box_z + za;
                const int* ids = s->box_ids + (size_t)b * s->box_cap;
                for (int c = 0; c < s->box_count[b]; c++)
                    if (ids[c] != id) {
                        out[found++] = ids[c];
                        if (!(s->nbr_stride > found)) { if (!s->err) s->err = BCG_E_NEIGH_OVERFLOW; out[0] = found - 1; return found - 1; }
                    }
            }
    out[0] = found - 1;
    return found - 1;
}

/* ------------------------------------------------------- geometry --------- */
static double clampd(double n, double lo, double hi) { return n < lo ? lo : (n > hi ? hi : n); }
/* min_distance, Neighbours.cpp:107-160 */
static void min_distance(const bcg_cell* c1_, const bcg_cell* c2_, double* d, V3* c1, V3* c2)
{
    V3 p1 = c1_->p, q1 = c1_->q, p2 = c2_->p, q2 = c2_->q;
    V3 v1 = vdiff(q1, p1), v2 = vdiff(q2, p2), r = vdiff(p1, p2);
    double l1 = dot(v1, v1), l2 = dot(v2, v2), f = dot(v2, r), c = dot(v1, r), b = dot(v1, v2);
    double denom = l1 * l2 - b * b, s, t, tnom;
    if (denom != 0) s = clampd((b * f - c * l2) / denom, 0, 1);
    else s = 0;
    tnom = b * s + f;
    if (tnom < 0) { t = 0; s = clampd(-c / l1, 0, 1); }
    else if (tnom > l2) { t = 1; s = clampd((b - c) / l1, 0, 1); }
    else t = tnom / l2;
    *c1 = vsum(p1, vscale(v1, s));
    *c2 = vsum(p2, vscale(v2, t));
    V3 cv = vdiff(*c1, *c2);
    *d = sqrt(dot(cv, cv));
}
/* reduceNeighbours, Neighbours.cpp:57-93 */
static int reduce_neighbours(orc_state* s, const bcg_cell* cell, const bcg_cell* arr, int* nb)
{
    double Rc = s->P.rc, d;
    V3 c1, c2, v, cm = avg(cell);
    int kept = 1, n = nb[0];
    for (int k = 1; k < n + 1; k++) {
        int id = nb[k];
        v = vdiff(arr[id].p, cm);
        double dp = sqrt(dot(v, v));
        v = vdiff(arr[id].q, cm);
        double dq = sqrt(dot(v, v));
        if ((dp < (cell->length / 2.0 + Rc * cell->radius)) || (dq < (cell->length / 2.0 + Rc * cell->radius))) {
            min_distance(cell, &arr[id], &d, &c1, &c2);
            if (d < Rc * cell->radius) nb[kept++] = id;
        }
    }
    nb[0] = kept - 1;
    return kept - 1;
}
static int* nbr_row(orc_state* s, int i) { return s->nbr + (size_t)i * s->nbr_stride; }

/* getNeighbours (full), Neighbours.cpp:24-37 */
void orc_rebuild_neighbours(orc_state* s)
{
    for (int i = 0; i < s->N; i++) {
        int a = get_address(s, avg(&s->oldc[i]), 0, 0, 0);
        grid_neighbours(s, i, a, nbr_row(s, i));
        reduce_neighbours(s, &s->oldc[i], s->oldc, nbr_row(s, i));
    }
}
/* getNeighbours (ID list), Neighbours.cpp:39-55 */
static void rebuild_ids(orc_state* s, const bcg_cell* arr, const int* ids, int n)
{
    for (int k = 0; k < n; k++) {
        int i = ids[k];
        int a = get_address(s, avg(&arr[i]), 0, 0, 0);
        grid_neighbours(s, i, a, nbr_row(s, i));
        reduce_neighbours(s, &arr[i], arr, nbr_row(s, i));
    }
}

/* ------------------------------------------------------- forces ----------- */
/* F_cc, Forces.cpp:13-84 */
static void F_cc(orc_state* s, const bcg_cell* a, const bcg_cell* b, V3* F, V3* r, double* d)
{
    const bcg_params* P = &s->P;
    V3 c1, c2;
    double gamma_n = 100.0, sigma = a->radius + b->radius;
    double L1 = a->length + 4.0 / 3 * a->radius, M1 = L1 * a->radius * a->radius * PI;
    double L2 = b->length + 4.0 / 3 * b->radius, M2 = L2 * b->radius * b->radius * PI;
    double Meff = M1 * M2 / (M1 + M2);
    min_distance(a, b, d, &c1, &c2);
    double delta = dmax(sigma - *d, 0.0);
    V3 vn = vscale(vdiff(c2, c1), 1.0 / *d);
    double FE_mag = sqrt(a->radius * b->radius / (a->radius + b->radius)) * P->k_cc * pow(delta, 3.0 / 2.0);
    V3 FE = vscale(vn, -FE_mag);
    *r = vscale(vsum(vscale(c1, b->radius), vscale(c2, a->radius)), 1 / sigma);
    if (FE_mag > DBL_EPSILON) {
        V3 rcm1 = vdiff(*r, avg(a)), rcm2 = vdiff(*r, avg(b));
        V3 va1 = cross(a->angular_velocity, rcm1), va2 = cross(b->angular_velocity, rcm2);
        V3 v1 = vsum(a->velocity, va1), v2 = vsum(b->velocity, va2);
        V3 dv = vdiff(v2, v1);
        double gamma = P->gamma_t, mu = P->cell_mu;
        V3 dvn = vscale(vn, dot(dv, vn));
        V3 FDn = vscale(dvn, gamma_n * Meff * delta);
        V3 dvt = vdiff(dv, dvn);
        double v_mag = sqrt(dot(dvt, dvt));
        V3 FDt = v3(0.0, 0.0, 0.0);
        if (v_mag > 3 * DBL_EPSILON) FDt = vscale(dvt, dmin(gamma * Meff * sqrt(delta), mu * FE_mag / v_mag));
        *F = vsum(vsum(FE, FDt), FDn);
    } else *F = FE;
}

/* F_cw, Forces.cpp:88-204 (one rand() draw per call, :102) */
static void F_cw(orc_state* s, const bcg_cell* c, double Wall_z, V3* F1, V3* F2, V3* r1, V3* r2, V3* sf, V3* df)
{
    const bcg_params* P = &s->P;
    double L = c->length + 4.0 / 3 * c->radius, M = L * c->radius * c->radius * PI, gamma_n = 100.0;
    double sigma = c->radius;
    V3 wall;
    wall.x = c->p.x + ((float)rnd(s) / (float)RAND_MAX_ - 0.5) * P->var_pos;
    wall.y = 0.0; wall.z = Wall_z;
    *r1 = wall;
    double d = c->p.z - wall.z, delta = dmax(sigma - d, 0.0);
    double FE_mag = sqrt(c->radius) * P->k_wc * pow(delta, 3.0 / 2.0);
    V3 FE = v3(0.0, 0.0, 0.0); FE.z = FE_mag;
    V3 rcm, v, va, dv, dvn, dvt, FDt, FDn; double v_mag;
    if (FE_mag > DBL_EPSILON) {
        rcm = vdiff(*r1, avg(c)); va = cross(c->angular_velocity, rcm); v = vsum(c->velocity, va);
        dv = vscale(v, -1.0); dvn = v3(0.0, 0.0, dv.z); dvt = vdiff(dv, dvn); v_mag = sqrt(dot(dvt, dvt));
        if (v_mag > DBL_EPSILON) FDt = vscale(dvt, dmin(P->gamma_t * M * sqrt(delta), P->wall_mu * FE_mag / v_mag));
        else FDt = v3(0, 0, 0);
        FDn = vscale(dvn, gamma_n * M * delta);
        *F1 = vsum(FE, vsum(FDt, FDn));
        *sf = vsum(*sf, vscale(dvt, P->gamma_t * M * sqrt(delta)));
        *df = vsum(*df, vscale(dvt, P->wall_mu * FE_mag / v_mag));
    } else *F1 = v3(0.0, 0.0, 0.0);
    wall.x = c->q.x; wall.y = 0.0; wall.z = Wall_z;
    *r2 = wall;
    d = c->q.z - wall.z; delta = dmax(sigma - d, 0.0);
    FE_mag = sqrt(c->radius) * P->k_wc * pow(delta, 3.0 / 2.0);
    FE.z = FE_mag;
    if (FE_mag > DBL_EPSILON) {
        rcm = vdiff(*r2, avg(c)); va = cross(c->angular_velocity, rcm); v = vsum(c->velocity, va);
        dv = vscale(v, -1.0); dvn = v3(0.0, 0.0, dv.z); dvt = vdiff(dv, dvn); v_mag = sqrt(dot(dvt, dvt));
        if (v_mag > DBL_EPSILON) FDt = vscale(dvt, dmin(P->gamma_t * M * sqrt(delta), P->wall_mu * FE_mag / v_mag));
        else FDt = v3(0, 0, 0);
        FDn = vscale(dvn, gamma_n * M * delta);
        *F2 = vsum(FE, vsum(FDt, FDn));
        *sf = vsum(*sf, vscale(dvt, P->gamma_t * M * sqrt(delta)));
        *df = vsum(*df, vscale(dvt, P->wall_mu * FE_mag / v_mag));
    } else *F2 = v3(0.0, 0.0, 0.0);
}

/* Array2D<double>::linear_interp with float weights, Array.h:282-288 (y = 0) */
static double height_interp(orc_state* s, int x0, double dx)
{
    float x = dx < 0 ? 1 + dx : dx;
    float y = 0.0;
    int H = s->P.box_x * s->P.refinement_grid_height;
    double d0 = s->height[x0], d1 = s->height[x0 + 1];
    /* the reference's y0+1 row aliases x0+1 / x0+2 with weight y = 0 */
    double d2 = s->height[x0 + 1], d3 = (x0 + 2 < H) ? s->height[x0 + 2] : 0.0;
    return d0 * (1 - x) * (1 - y) + d1 * x * (1 - y) + d2 * (1 - x) * y + d3 * x * y;
}

/* F_surf_tension, Forces.cpp:209-317 */
static void F_surf(orc_state* s, const bcg_cell* c, V3* F, V3* T)
{
    const bcg_params* P = &s->P;
    int rgh = P->refinement_grid_height;
    double hb = P->box_length / rgh;
    V3 F1 = v3(0, 0, 0), F2 = v3(0, 0, 0);
    int xa = (int)((avg(c).x + P->box_x / 2 * P->box_length) / (P->box_length / rgh));
    int i_ht;
    double dxp, dxq, dx, distance, dh, F0;
    i_ht = (int)(c->p.x / hb + P->box_x / 2 * rgh);
    dxp = c->p.x / hb - (i_ht - P->box_x / 2 * rgh + 0.5);
    i_ht = (int)ceil(dxp) + i_ht - 1;
    double height_p = height_interp(s, i_ht, dxp);
    i_ht = (int)(c->q.x / hb + P->box_x / 2 * rgh);
    dxq = c->q.x / hb - (i_ht - P->box_x / 2 * rgh + 0.5);
    i_ht = (int)ceil(dxq) + i_ht - 1;
    double height_q = height_interp(s, i_ht, dxq);
    V3 cm = avg(c);
    i_ht = (int)(cm.x / hb + P->box_x / 2 * rgh);
    dx = cm.x / hb - (i_ht - P->box_x / 2 * rgh + 0.5);
    i_ht = (int)ceil(dx) + i_ht - 1;
    double height_cm = height_interp(s, i_ht, dx);
    if (height_cm > (cm.z + P->box_length)) { *F = v3(0, 0, 0); *T = v3(0, 0, 0); return; }
    V3 N = v3(s->normal_x[xa], s->normal_y[xa], s->normal_z[xa]);
    dh = c->p.z - (height_p - P->delta_h / N.z);
    if (dh < 0.0) F1 = v3(0, 0, 0);
    else { distance = -dh * N.z; F0 = 2 * PI * P->tension * dmin(distance / (P->cell_radius / 5.0), 1.0); F1 = vscale(N, F0); }
    dh = c->q.z - (height_q - P->delta_h / N.z);
    if (dh < 0.0) F2 = v3(0, 0, 0);
    else { distance = -dh * N.z; F0 = 2 * PI * P->tension * dmin(distance / (P->cell_radius / 5.0), 1.0); F2 = vscale(N, F0); }
    *F = vsum(F1, F2);
    V3 r = vdiff(c->p, cm);
    *T = cross(r, F1);
    r = vdiff(c->q, cm);
    *T = vsum(*T, cross(r, F2));
}

/* sum_forces, Forces.cpp:332-381 (F_v inlined from :320-329) */
static void sum_forces(orc_state* s, const bcg_cell* c, const bcg_cell* arr, const int* nb, int wall_x,
                       V3* Fnet, V3* Tnet, V3* sf, V3* df)
{
    const bcg_params* P = &s->P;
    *Fnet = v3(0, 0, 0); *Tnet = v3(0, 0, 0);
    V3 F = v3(0, 0, 0), F2 = v3(0, 0, 0), T = v3(0, 0, 0), r, r2, cm = avg(c);
    double d;
    int n = nb[0];
    for (int k = 1; k < n + 1; k++) {
        F_cc(s, c, &arr[nb[k]], &F, &r, &d);
        *Fnet = vsum(*Fnet, F);
        r = vdiff(r, cm);
        *Tnet = vsum(*Tnet, cross(r, F));
    }
    *sf = v3(0, 0, 0); *df = v3(0, 0, 0);
    if (dmin(c->q.z, c->p.z) < 1.2 * c->radius) {
        double wall_y = s->wall[wall_x];
        F_cw(s, c, wall_y, &F, &F2, &r, &r2, sf, df);
        *Fnet = vsum(*Fnet, F); r = vdiff(r, cm); *Tnet = vsum(*Tnet, cross(r, F));
        *Fnet = vsum(*Fnet, F2); r2 = vdiff(r2, cm); *Tnet = vsum(*Tnet, cross(r2, F2));
    }
    F = vscale(c->velocity, -P->viscosity * 6.0 * PI * c->radius);
    T = vscale(c->angular_velocity, -P->viscosity * 6.0 * PI * c->radius);
    *Fnet = vsum(*Fnet, F); *Tnet = vsum(*Tnet, T);
    F_surf(s, c, &F, &T);
    *Fnet = vsum(*Fnet, F); *Tnet = vsum(*Tnet, T);
    Tnet->z = 0; Fnet->y = 0;
}

/* UpdatePositions / UpdateVelocities, Integrate.cpp:34-127 */
static void half_kick(double dt, V3 F, V3 T, const bcg_cell* o, bcg_cell* n)
{
    double R2 = o->radius * o->radius, L2 = o->length * o->length;
    double M = PI * R2 * (o->length + 4.0 / 3.0 * o->radius);
    double Ixy = PI * R2 * (o->length * L2 / 12.0 + o->radius * (8.0 * R2 / 15.0 + L2 / 3.0));
    double Iz = PI * R2 * R2 * (o->length / 2.0 + 8.0 * o->radius / 15.0);
    V3 z = vdiff(o->q, o->p);
    z = vscale(z, 1.0 / o->length);
    V3 vaz = vscale(z, dot(z, o->angular_velocity));
    V3 vaxy = vdiff(o->angular_velocity, vaz);
    V3 Tz = vscale(z, dot(z, T));
    V3 Txy = vdiff(T, Tz);
    n->velocity = vsum(o->velocity, vscale(F, dt / (2.0 * M)));
    n->angular_velocity = vsum(vsum(vaz, vscale(Tz, dt / (2.0 * Iz))), vsum(vaxy, vscale(Txy, dt / (2.0 * Ixy))));
}
static void update_positions(double dt, V3 F, V3 T, const bcg_cell* o, bcg_cell* n)
{
    *n = *o;
    half_kick(dt, F, T, o, n);
    V3 cm = avg(o);
    V3 rcmp = vdiff(o->p, cm), rcmq = vdiff(o->q, cm);
    V3 vap = cross(n->angular_velocity, rcmp), vaq = cross(n->angular_velocity, rcmq);
    V3 vp = vsum(n->velocity, vap), vq = vsum(n->velocity, vaq);
    n->p = vsum(o->p, vscale(vp, dt));
    n->q = vsum(o->q, vscale(vq, dt));
    n->p.y = 0; n->q.y = 0;
}
static void update_velocities(double dt, V3 F, V3 T, const bcg_cell* o, bcg_cell* n)
{
    *n = *o;
    half_kick(dt, F, T, o, n);
    n->velocity.y = 0;
}


/* grow, grow.cpp:17-102 (the live code path; crossFeeding picks GrowthRate2
 * for Type 2 cells, :26-36) */
static void grow(orc_state* s, double dt, bcg_cell* c)
{
    V3 cm = avg(c);
    int a = get_address(s, cm, 0, 0, 0);
    double g;
    if (s->P.cross_feeding) g = (c->type == 1) ? s->env[a].GrowthRate1 : s->env[a].GrowthRate2;
    else g = s->env[a].GrowthRate1;
    g = g * 1.5850;
    V3 v = vdiff(c->q, c->p);
    double dL = c->length * dt * g;
    V3 dv = vscale(v, dL * 0.5 / c->length);
    c->length += dL;
    c->p = vdiff(c->p, dv);
    c->q = vsum(c->q, dv);
    c->growth_rate = g;
}

/* divide, grow.cpp:107-186 */
static void divide(orc_state* s, bcg_cell* m, bcg_cell* d, double t)
{
    const bcg_params* P = &s->P;
    double dl = (frand(s) - 0.5) * P->var_l;
    double dangle = (frand(s) - 0.5) * P->var_angle;
    V3 pq = vdiff(m->p, m->q);
    double a1 = frand(s) - 0.5, a2 = frand(s) - 0.5, a3 = frand(s) - 0.5;
    V3 dd1 = v3(a1, a2, a3);
    dd1 = vdiff(dd1, vscale(pq, dot(dd1, pq) / dot(pq, pq)));
    dd1 = vscale(dd1, 1 / sqrt(dot(dd1, dd1)));
    V3 dO1 = vscale(dd1, dangle);
    double b1 = frand(s) - 0.5, b2 = frand(s) - 0.5, b3 = frand(s) - 0.5;
    V3 dd2 = v3(b1, b2, b3);
    dd2 = vdiff(dd2, vscale(pq, dot(dd2, pq) / dot(pq, pq)));
    dd2 = vscale(dd2, 1 / sqrt(dot(dd2, dd2)));
    V3 dO2 = vscale(dd2, dangle);
    V3 uv = vdiff(m->p, m->q);
    double L = m->length;
    uv = vscale(uv, 1 / L);
    d->q = m->q;
    d->radius = P->cell_radius;
    m->length = L / 2 - m->radius + dl;
    d->length = L / 2 + m->radius - 2 * d->radius - dl;
    d->growth_rate = m->growth_rate;
    d->velocity = m->velocity;
    d->angular_velocity = v3(0, 0, (frand(s) - 0.5) * 0.001);
    m->angular_velocity = v3(0, 0, 0);
    m->q = vdiff(m->p, vscale(uv, m->length));
    d->time_q = m->time_q;
    m->time_q = t;
    d->time_p = t;
    m->age_p++;
    d->age_q = m->age_q + 1;
    d->p = vdiff(m->q, vscale(uv, d->radius + m->radius));
    d->q = vdiff(d->p, vscale(uv, d->length));
    m->p = vsum(m->p, vscale(dO1, m->length));
    m->q = vdiff(m->q, vscale(dO1, m->length));
    d->p = vsum(d->p, vscale(dO2, d->length));
    d->q = vdiff(d->q, vscale(dO2, d->length));
    d->type = m->type;
    d->ancestor = m->ancestor;
    m->ldiv = P->l_divide / 2 + P->cell_radius + m->length;
    d->ldiv = P->l_divide / 2 + P->cell_radius + d->length;
}

/* MoveCell + GrowCell loop, Simulation.cpp:330-336 with Cells.cpp:14-57 and
 * integrate, Integrate.cpp:11-32. */
int orc_move_grow(orc_state* s, double dt, int* div_ids, long long* rand_calls)
{
    long long r0 = s->rand_calls;
    s->ndiv = 0;
    for (int i = 0; i < s->N; i++) {
        const bcg_cell* oc = &s->oldc[i];
        bcg_cell* nc = &s->newc[i];
        int xi, yi, zi;
        int olda = get_address(s, avg(oc), &xi, &yi, &zi);
        const int* nb = nbr_row(s, i);
        V3 F, T, sf, df;
        bcg_cell tmp;
        sum_forces(s, oc, s->oldc, nb, xi * s->P.box_y + yi, &F, &T, &sf, &df);
        update_positions(dt, F, T, oc, &tmp);
        sum_forces(s, &tmp, s->oldc, nb, xi * s->P.box_y + yi, &F, &T, &sf, &df);
        update_velocities(dt, F, T, &tmp, nc);
        nc->dyn_fric = df;
        nc->sta_fric = sf;
        int newa = get_address(s, avg(nc), 0, 0, 0);
        if (newa != olda) { box_remove(s, i, olda); box_add(s, i, newa); }
        grow(s, dt, nc);
        if (nc->length >= nc->ldiv) s->dividing[s->ndiv++] = i;
    }
    if (div_ids) memcpy(div_ids, s->dividing, sizeof(int) * (size_t)s->ndiv);
    if (rand_calls) *rand_calls = s->rand_calls - r0;
    return s->ndiv;
}

/* Division loop and buffer swap, Simulation.cpp:380-413, DivideCell
 * Cells.cpp:60-81. */
int orc_divide(orc_state* s, double t, int* lineage)
{
    int done = 0;
    for (int k = 0; k < s->ndiv; k++) {
        if (s->N > (s->P.max_cells - 1)) { if (!s->err) s->err = BCG_E_MAXCELLS; break; }
        int id = s->dividing[k];
        bcg_cell* m = &s->newc[id];
        bcg_cell* d = &s->newc[s->N];
        int a = get_address(s, avg(m), 0, 0, 0);
        box_remove(s, id, a);
        divide(s, m, d, t);
        box_add(s, id, get_address(s, avg(m), 0, 0, 0));
        box_add(s, s->N, get_address(s, avg(d), 0, 0, 0));
        if (lineage) { lineage[2 * done] = id; lineage[2 * done + 1] = s->N; }
        s->N++;
        done++;
        int* row = nbr_row(s, id);
        int len = row[0];
        memcpy(s->idlist, row, (size_t)(len + 1) * sizeof(int));
        s->idlist[0] = id;
        s->idlist[len + 1] = s->N - 1;
        len += 2;
        rebuild_ids(s, s->newc, s->idlist, len);
    }
    bcg_cell* tmp = s->newc; s->newc = s->oldc; s->oldc = tmp;
    s->ndiv = 0;
    return done;
}

/* ------------------------------------------------------- API -------------- */
static int mg_nx(const orc_state* s, int l)
{
    int d = 1 << l, d0 = 1 << s->P.max_levels_mg;
    return imin(s->P.box_x, s->P.box_x * d0 / d / 2);
}
static int mg_nz(const orc_state* s, int l)
{
    int d = 1 << l, d0 = 1 << s->P.max_levels_mg;
    return imin(s->P.box_z_agar, s->P.box_z_agar * d0 / d / 2);
}
static double* dz(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }

orc_state* orc_create(const bcg_params* p, unsigned seed, int make_wall)
{
    orc_state* s = (orc_state*)calloc(1, sizeof(orc_state));
    s->P = *p;
    grand_seed(&s->rng, seed);
    const int X = p->box_x, Z = p->box_z, ZA = p->box_z_agar, XH = p->box_x * p->refinement_grid_height;
    s->oldc = (bcg_cell*)calloc((size_t)p->max_cells, sizeof(bcg_cell));
    s->newc = (bcg_cell*)calloc((size_t)p->max_cells, sizeof(bcg_cell));
    s->nbox = X * p->box_y * Z;
    s->box_cap = p->max_cells_per_box;
    s->box_count = (int*)calloc((size_t)s->nbox, sizeof(int));
    s->box_ids = (int*)calloc((size_t)s->nbox * s->box_cap, sizeof(int));
    s->nbr_stride = s->box_cap * 27 + 1;
    s->nbr = (int*)calloc((size_t)p->max_cells * s->nbr_stride, sizeof(int));
    s->dividing = (int*)calloc((size_t)p->max_cells, sizeof(int));
    s->idlist = (int*)calloc((size_t)s->nbr_stride + 2, sizeof(int));
    s->height = dz(XH); s->rough_height = dz(XH);
    s->normal_x = dz(XH); s->normal_y = dz(XH); s->normal_z = dz(XH);
    for (int i = 0; i < XH; i++) { s->height[i] = p->cell_radius; s->rough_height[i] = p->cell_radius; s->normal_z[i] = -1.0; }
    s->wall = dz((size_t)X * p->box_y);
    /* LocalEnv / LocalAga defaults, Nutrients.h:13-38, 68-74 */
    s->env = (env_t*)calloc((size_t)X * Z, sizeof(env_t));
    s->oenv = (env_t*)calloc((size_t)X * Z, sizeof(env_t));
    for (long i = 0; i < (long)X * Z; i++) {
        env_t e; memset(&e, 0, sizeof(e)); e.Oxygen = p->max_o2; e.pH = 7.0;
        s->env[i] = e; s->oenv[i] = e;
    }
    aga_t a0 = {p->max_carbon, 0.0, p->max_o2, 0.0};
    int L = p->max_levels_mg;
    s->agar = (aga_t**)calloc(L, sizeof(aga_t*)); s->oagar = (aga_t**)calloc(L, sizeof(aga_t*));
    s->wal = (aga_t**)calloc(L, sizeof(aga_t*)); s->owal = (aga_t**)calloc(L, sizeof(aga_t*));
    for (int l = 0; l < L; l++) {
        s->agar[l] = (aga_t*)malloc(sizeof(aga_t) * (size_t)X * ZA);
        s->oagar[l] = (aga_t*)malloc(sizeof(aga_t) * (size_t)X * ZA);
        s->wal[l] = (aga_t*)malloc(sizeof(aga_t) * (size_t)X);
        s->owal[l] = (aga_t*)malloc(sizeof(aga_t) * (size_t)X);
        for (long i = 0; i < (long)X * ZA; i++) { s->agar[l][i] = a0; s->oagar[l][i] = a0; }
        for (int i = 0; i < X; i++) { s->wal[l][i] = a0; s->owal[l][i] = a0; }
    }
    s->mg_levels = p->mg_levels;
    s->mgA = (aga_t**)calloc(s->mg_levels, sizeof(aga_t*));
    s->mgR = (aga_t**)calloc(s->mg_levels, sizeof(aga_t*));
    s->mgE = (aga_t**)calloc(s->mg_levels, sizeof(aga_t*));
    for (int l = 0; l < s->mg_levels; l++) {
        size_t n = (size_t)(mg_nx(s, l) + 1) * (mg_nz(s, l) + 1);
        s->mgA[l] = (aga_t*)malloc(sizeof(aga_t) * n);
        s->mgR[l] = (aga_t*)malloc(sizeof(aga_t) * n);
        s->mgE[l] = (aga_t*)malloc(sizeof(aga_t) * n);
        for (size_t i = 0; i < n; i++) { s->mgA[l][i] = a0; s->mgR[l][i] = a0; s->mgE[l][i] = a0; }
    }
    size_t n3 = (size_t)X * Z;
    double** a3[] = {&s->rd, &s->rd1, &s->rd2, &s->inside, &s->rds, &s->rd1s, &s->rd2s, &s->dens, &s->dens1, &s->dens2, &s->ds, &s->d1s, &s->d2s};
    for (unsigned i = 0; i < sizeof(a3) / sizeof(a3[0]); i++) *a3[i] = dz(n3);
    double** a2[] = {&s->rw, &s->rw1, &s->rw2, &s->rws, &s->rw1s, &s->rw2s, &s->wd, &s->wd1, &s->wd2, &s->wds, &s->wd1s, &s->wd2s};
    for (unsigned i = 0; i < sizeof(a2) / sizeof(a2[0]); i++) *a2[i] = dz((size_t)X);
    /* filters, Simulation.cpp:61-110 */
    int FL = p->filter_len;
    for (int i = 0; i < FL; i++) s->filter1d[i] = 1.0 / (double)(FL);
    double norm = 0;
    for (int ii = 0; ii < FL; ii++)
        for (int kk = 0; kk < FL; kk++)
            norm = norm + exp(-(ii - FL / 2) * (ii - FL / 2) - (kk - FL / 2) * (kk - FL / 2));
    for (int ii = 0; ii < FL; ii++)
        for (int kk = 0; kk < FL; kk++)
            s->filter3d[ii * FL + kk] = exp(-(ii - FL / 2) * (ii - FL / 2) - (kk - FL / 2) * (kk - FL / 2)) / norm;
    /* rough wall, Simulation.cpp:161-168 */
    for (int ii = 0; ii < X; ii++)
        for (int jj = 0; jj < p->box_y; jj++)
            s->wall[ii * p->box_y + jj] = make_wall ? ((float)rnd(s) / (float)RAND_MAX_ - 0.5) * p->wall_rough : 0.0;
    s->rand_calls = 0;
    s->t = p->t0; s->dt = p->dt;
    s->next_out = p->output_time; s->next_update = p->update_time;
    s->hd_next_update = p->update_time / 10.0; s->hd_update = p->update_time / 10.0;
    s->update_flag = 1; s->hd_update_flag = 1;
    s->mg_dt = p->mg_dt;
    return s;
}

void orc_destroy(orc_state* s)
{
    if (!s) return;
    free(s->oldc); free(s->newc); free(s->box_count); free(s->box_ids); free(s->nbr);
    free(s->dividing); free(s->idlist);
    free(s->height); free(s->rough_height); free(s->normal_x); free(s->normal_y); free(s->normal_z); free(s->wall);
    free(s->env); free(s->oenv);
    for (int l = 0; l < s->P.max_levels_mg; l++) { free(s->agar[l]); free(s->oagar[l]); free(s->wal[l]); free(s->owal[l]); }
    free(s->agar); free(s->oagar); free(s->wal); free(s->owal);
    for (int l = 0; l < s->mg_levels; l++) { free(s->mgA[l]); free(s->mgR[l]); free(s->mgE[l]); }
    free(s->mgA); free(s->mgR); free(s->mgE);
    double* arr[] = {s->rd, s->rd1, s->rd2, s->inside, s->rds, s->rd1s, s->rd2s, s->dens, s->dens1, s->dens2, s->ds, s->d1s, s->d2s,
                     s->rw, s->rw1, s->rw2, s->rws, s->rw1s, s->rw2s, s->wd, s->wd1, s->wd2, s->wds, s->wd1s, s->wd2s};
    for (unsigned i = 0; i < sizeof(arr) / sizeof(arr[0]); i++) free(arr[i]);
    free(s);
}

int orc_load_cells(orc_state* s, const bcg_cell* cells, int n)
{
    if (n > s->P.max_cells) return BCG_E_ARG;
    memcpy(s->oldc, cells, sizeof(bcg_cell) * (size_t)n);
    s->N = n;
    for (int i = 0; i < n; i++) box_add(s, i, get_address(s, avg(&s->oldc[i]), 0, 0, 0));
    return s->err;
}
int orc_get_cells(orc_state* s, bcg_cell* out, int cap)
{
    int n = s->N < cap ? s->N : cap;
    memcpy(out, s->oldc, sizeof(bcg_cell) * (size_t)n);
    return s->N;
}
int orc_num_cells(orc_state* s) { return s->N; }
long long orc_rand_calls(orc_state* s) { return s->rand_calls; }
int orc_error(orc_state* s) { return s->err; }
double orc_time(orc_state* s) { return s->t; }

int orc_get_neighbours(orc_state* s, int* counts, int* lists, int stride)
{
    int mx = 0;
    for (int i = 0; i < s->N; i++) {
        const int* row = nbr_row(s, i);
        counts[i] = row[0];
        if (row[0] > mx) mx = row[0];
        for (int j = 0; j < row[0] && j < stride; j++) lists[(size_t)i * stride + j] = row[j + 1];
    }
    return mx;
}
int orc_set_neighbours(orc_state* s, const int* counts, const int* lists, int stride)
{
    for (int i = 0; i < s->N; i++) {
        int* row = nbr_row(s, i);
        row[0] = counts[i];
        for (int j = 0; j < counts[i]; j++) row[j + 1] = lists[(size_t)i * stride + j];
    }
    return 0;
}
void orc_bbox(orc_state* s, int* mnx, int* mxx, int* mxz) { *mnx = s->minx; *mxx = s->maxx; *mxz = s->maxz; }
void orc_set_bbox(orc_state* s, int mnx, int mxx, int mxz) { s->minx = mnx; s->maxx = mxx; s->maxz = mxz; }

/* ======================================================= deposition ======= */
#define IX3(x, z) ((long)(x) * s->P.box_z + (z))

/* GetDensity, Compute.cpp:120-253 (Box_y = 1).  Sums in box-list order. */
static void get_density(orc_state* s)
{
    const bcg_params* P = &s->P;
    const int X = P->box_x, Z = P->box_z, rgh = P->refinement_grid_height;
    double height[64];
    s->minx = X; s->maxx = 0; s->miny = P->box_y; s->maxy = 0; s->maxz = 0;
    double Vbox = P->box_length * P->box_length;
    for (int bx = 0; bx < X; bx++) {
        for (int i = 0; i < rgh; i++) height[i] = P->cell_radius;
        for (int bz = 0; bz < Z; bz++) {
            int a = bx * P->box_y * Z + bz;
            int count = s->box_count[a];
            const int* ids = s->box_ids + (size_t)a * s->box_cap;
            if (count > 0) {
                s->minx = imin(s->minx, bx); s->maxx = imax(s->maxx, bx);
                s->miny = imin(s->miny, 0); s->maxy = imax(s->maxy, 0); s->maxz = imax(s->maxz, bz);
            }
            double den = 0, den1 = 0, den2 = 0;
            for (int c = 0; c < count; c++) {
                const bcg_cell* cell = &s->oldc[ids[c]];
                V3 cm = avg(cell);
                int i_ht = (int)((cm.x / P->box_length - (bx - X / 2)) * rgh);
                if (i_ht < 0) i_ht = 0;
                if (i_ht > rgh - 1) i_ht = rgh - 1;
                double top = dmax(cell->p.z, cell->q.z);
                height[i_ht] = dmax(height[i_ht], top);
                if (cell->type == 1) den1 += cell->length * cell->radius;
                else if (cell->type == 2) den2 += cell->length * cell->radius;
                den += cell->length * cell->radius;
            }
            if (den == 0) { s->rd1[IX3(bx, bz)] = 0; s->rd2[IX3(bx, bz)] = 0; s->rd[IX3(bx, bz)] = 0; s->inside[IX3(bx, bz)] = 0; }
            else {
                s->rd1[IX3(bx, bz)] = den1 / den; s->rd2[IX3(bx, bz)] = den2 / den;
                s->rd[IX3(bx, bz)] = den / Vbox; s->inside[IX3(bx, bz)] = 1.0;
            }
            for (int i = 0; i < rgh; i++) s->height[bx * rgh + i] = height[i];
        }
    }
    for (int bx = 0; bx < X; bx++)
        for (int bz = 0; bz < Z; bz++) {
            if (s->inside[IX3(bx, bz)] < 0.5) {
                if (bz > 0 && bx > 0 && bx < X - 1 && bz < Z - 1) {
                    if ((s->inside[IX3(bx + 1, bz)] > 0.5) || (s->inside[IX3(bx - 1, bz)] > 0.5) || (s->inside[IX3(bx, bz + 1)] > 0.5) || (s->inside[IX3(bx, bz - 1)] > 0.5))
                        s->inside[IX3(bx, bz)] = 0.4;
                } else if (bz == 0 && bx > 0 && bx < X - 1) {
                    if ((s->inside[IX3(bx + 1, bz)] > 0.5) || (s->inside[IX3(bx - 1, bz)] > 0.5) || (s->inside[IX3(bx, bz + 1)] > 0.5))
                        s->inside[IX3(bx, bz)] = 0.4;
                }
            }
        }
    s->minx -= 5; s->maxx += 5; s->maxz += 5;
}

/* GetHeight, Compute.cpp:256-340: top four occupied boxes of each column. */
static void get_height(orc_state* s)
{
    const bcg_params* P = &s->P;
    const int X = P->box_x, Z = P->box_z, rgh = P->refinement_grid_height;
    double height[64];
    s->minx = X; s->maxx = 0; s->miny = P->box_y; s->maxy = 0; s->maxz = 0;
    for (int bx = 0; bx < X; bx++) {
        for (int i = 0; i < rgh; i++) height[i] = P->cell_radius;
        int pos_ct = 0;
        for (int bz = Z - 1; bz >= 0; bz--) {
            int a = bx * P->box_y * Z + bz;
            int count = s->box_count[a];
            const int* ids = s->box_ids + (size_t)a * s->box_cap;
            if (count > 0) {
                s->minx = imin(s->minx, bx); s->maxx = imax(s->maxx, bx);
                s->miny = imin(s->miny, 0); s->maxy = imax(s->maxy, 0); s->maxz = imax(s->maxz, bz);
                pos_ct++;
            }
            for (int c = 0; c < count; c++) {
                const bcg_cell* cell = &s->oldc[ids[c]];
                V3 cm = avg(cell);
                int i_ht = (int)((cm.x - (bx - X / 2) * P->box_length) / (P->box_length / rgh));
                if (i_ht < 0) i_ht = 0;
                if (i_ht > rgh - 1) i_ht = rgh - 1;
                double top = dmax(cell->p.z, cell->q.z);
                height[i_ht] = dmax(height[i_ht], top);
            }
            for (int i = 0; i < rgh; i++) s->height[bx * rgh + i] = height[i];
            if (pos_ct > 3) break;
        }
    }
    s->minx -= 5; s->maxx += 5; s->maxz += 5;
}

/* ShiftDensity, Compute.cpp:344-463, with Box_y = 1: the y = BoxY-1 passes
 * overwrite the 8-point averages, leaving these final values. */
static void shift_one(orc_state* s, const double* D, double* DS, double* WS)
{
    const int X = s->P.box_x, Z = s->P.box_z;
    for (int x = 0; x < X - 1; x++)
        for (int z = 0; z < Z - 1; z++)
            DS[IX3(x, z)] = (D[IX3(x, z)] + D[IX3(x, z + 1)] + D[IX3(x + 1, z)] + D[IX3(x + 1, z + 1)]) / 4.0;
    for (int x = 0; x < X - 1; x++)
        DS[IX3(x, Z - 1)] = (D[IX3(x, Z - 1)] + D[IX3(x + 1, Z - 1)]) / 2.0;
    for (int z = 0; z < Z - 1; z++)
        DS[IX3(X - 1, z)] = (D[IX3(X - 1, z)] + D[IX3(X - 1, z)]) / 2.0;
    DS[IX3(X - 1, Z - 1)] = D[IX3(X - 1, Z - 1)];
    if (WS) {
        for (int x = 0; x < X - 1; x++) WS[x] = (D[IX3(x, 0)] + D[IX3(x + 1, 0)]) / 2.0;
        WS[X - 1] = D[IX3(X - 1, 0)];
    }
}

/* BoxAverage, Compute.cpp:495-605: 5x5 filter over x-z on the array with
 * the wall row prepended; outputs only inside [minx,maxx) x [0,maxz]
 * (elsewhere the reference leaves its scratch array uninitialised; here
 * those entries are left unchanged). */
static void box_average(orc_state* s, const double* rough, double* out, const double* rough_wall, double* out_wall)
{
    const bcg_params* P = &s->P;
    const int Z = P->box_z, FL = P->filter_len, FD = FL / 2;
    for (int ka = 0; ka < s->maxz + 1; ka++)
        for (int ia = s->minx; ia < s->maxx; ia++) {
            double a = 0.0;
            for (int fi = -FD; fi <= FD; fi++)
                for (int fk = -FD; fk <= FD; fk++) {
                    int i = ia + fi, k = ka + fk;
                    double w = s->filter3d[(fi + FD) * FL + (fk + FD)];
                    if (k < 0) {
                        double in0 = rough_wall[i];
                        if (in0 > 0.00001) a += w * 1.0;
                        else a += w * in0;
                    } else {
                        double in = (k == 0) ? rough_wall[i] : rough[IX3(i, k - 1)];
                        a += w * in;
                    }
                }
            double v = dmin(1.0, a / P->density_threshold);
            if (ka == 0) out_wall[ia] = v;
            else if (ka - 1 < Z) out[IX3(ia, ka - 1)] = v;
        }
}

/* Height_Average, Compute.cpp:669-705 */
static void height_average(orc_state* s, const double* in, double* out)
{
    int rgh = s->P.refinement_grid_height;
    for (int i = s->minx * rgh; i < (s->maxx + 1) * rgh; i++) {
        double H0 = in[i], Ht = H0; int count = 1;
        for (int d = -1; d < 2; d++) {
            if (d == 0) continue;
            double H = in[i + d];
            if (H < H0) { Ht += H; count++; }
        }
        out[i] = Ht / count;
    }
}
/* Smooth, Compute.cpp:708-738 */
static void smooth(orc_state* s, const double* in, double* out)
{
    int rgh = s->P.refinement_grid_height, FD = s->P.filter_len / 2;
    for (int i = s->minx * rgh; i < (s->maxx + 1) * rgh; i++) {
        double a = 0.0;
        for (int f = -FD; f <= FD; f++) a += s->filter1d[f + FD] * in[i + f];
        out[i] = a;
    }
}
/* GetSurfaceNormal, Compute.cpp:466-491 */
static void surface_normal(orc_state* s)
{
    int rgh = s->P.refinement_grid_height;
    for (int i = s->minx * rgh; i < (s->maxx + 1) * rgh; i++) {
        double d_x = (s->height[i + 1] - s->height[i - 1]) / (2.0 * s->P.box_length / rgh);
        double d_z = -1.0;
        double l_n = sqrt(d_x * d_x + d_z * d_z);
        s->normal_x[i] = d_x / l_n; s->normal_y[i] = 0; s->normal_z[i] = d_z / l_n;
    }
}

static void deposit_common(orc_state* s)
{
    get_density(s);
    shift_one(s, s->rd, s->rds, s->rws);
    shift_one(s, s->rd1, s->rd1s, 0);
    shift_one(s, s->rd2, s->rd2s, 0);
    box_average(s, s->rd, s->dens, s->rw, s->wd);
    box_average(s, s->rds, s->ds, s->rws, s->wds);
}
void orc_initial_fields(orc_state* s, int run_nutrients)
{
    deposit_common(s);
    surface_normal(s);
    if (run_nutrients) orc_nutrient_update(s, 0);
}
void orc_update_density(orc_state* s)
{
    deposit_common(s);
    height_average(s, s->height, s->rough_height);
    smooth(s, s->rough_height, s->height);
    surface_normal(s);
}
void orc_update_height(orc_state* s)
{
    get_height(s);
    height_average(s, s->height, s->rough_height);
    smooth(s, s->rough_height, s->height);
    surface_normal(s);
}

/* ======================================================= nutrients ======== */
/* acetateBufferSolve, Nutrients.cpp:806-855: Newton on the 3x3 acid/base
 * system; writes pH/Hydrox/Acetic/Buffer of `e`, returns Cac - y. */
static double buffer_solve(const bcg_params* P, double Cac, env_t* e)
{
    double Kw = P->kw_ph, Ka = P->ka_ph, Kb = P->kb_ph, Cb = P->cb_ph, c1 = P->c1_ph;
    double aH = -(Cb * Kb) / (pow(10, -4) + Kb);
    double x = 1e-7, y = Cac, z = Cb, sv[3];
    for (int it = 0; it < 100; it++) {
        double J[3][4] = {{2 * x + y + z + (Kw / c1) + aH, x, x, -(pow(x, 2) + x * (y + z + (Kw / c1) + aH) - Kw)},
                          {y, 2 * y + x + z + Ka + aH, y, -(pow(y, 2) + y * (x + z + (Ka) + aH) - Ka * Cac)},
                          {z, z, 2 * z + x + y + Kb + aH, -(pow(z, 2) + z * (x + y + (Kb) + aH) - Kb * Cb)}};
        double m1 = J[1][0] / J[0][0], m2 = J[2][0] / J[0][0];
        for (int i = 0; i < 4; i++) { J[1][i] -= m1 * J[0][i]; J[2][i] -= m2 * J[0][i]; }
        double m3 = J[2][1] / J[1][1];
        for (int i = 0; i < 4; i++) J[2][i] -= m3 * J[1][i];
        sv[2] = J[2][3] / J[2][2];
        sv[1] = J[1][3] / J[1][1] - (J[1][2] / J[1][1]) * sv[2];
        sv[0] = J[0][3] / J[0][0] - (J[0][2] / J[0][0]) * sv[2] - (J[0][1] / J[0][0]) * sv[1];
        double mx = 0;
        for (int i = 0; i < 3; i++) if (fabs(sv[i]) > mx) mx = fabs(sv[i]);
        x += sv[0]; y += sv[1]; z += sv[2];
        if (mx < pow(10, -7)) break;
    }
    e->pH = -log((x + y + z + aH) / 1000) / log(10);
    e->Hydrox = x; e->Acetic = y; e->Buffer = z;
    return (Cac - y);
}

/* UpdateEnvironment_OxygenAcetate, Nutrients.cpp:200-506 (crossFeeding = 0) */
static void colony_point(orc_state* s, env_t* Env, env_t* prev, const aga_t* pw, int x, int z)
{
    const bcg_params* P = &s->P;
    const long id = IX3(x, z);
    const double ins = s->inside[id];
    const double BL = P->box_length;
    if (ins > 0.5) {
        double C = prev[id].Carbon, W = prev[id].Waste, A = prev[id].Acetate, O = prev[id].Oxygen;
        buffer_solve(P, A, &prev[id]);
        (void)C; (void)W; (void)O;
        double Cgr = 0, Wgr = 0, Agr = 0, Ogr = 0;
        double mgrCarAers, mgrCarAnas, mgrAceAers, g1s, g2s, g3s;
        if (P->max_gr_car_aer != 0.0) { mgrCarAers = P->q_car_aer_nt / P->q_car_aer; g1s = P->kc_aer * (mgrCarAers / P->max_gr_car_aer); }
        else { mgrCarAers = 0; g1s = 1e6; }
        if (P->max_gr_car_ana != 0.0) { mgrCarAnas = P->q_car_ana_nt / P->q_car_ana; g2s = P->kc_ana * (mgrCarAnas / P->max_gr_car_ana); }
        else { mgrCarAnas = 0; g2s = 1e6; }
        if (P->max_gr_ace_aer != 0.0) { mgrAceAers = P->q_ace_aer_nt / P->q_ace_aer; g3s = P->ka * (mgrAceAers / P->max_gr_ace_aer); }
        else { mgrAceAers = 0; g3s = 1e6; }
        if (x != 0) {
            if (z == 0) {
                Cgr = (pw[x - 1].C + prev[IX3(x - 1, z)].Carbon + pw[x].C + prev[id].Carbon) / 4.0;
                Wgr = (pw[x - 1].W + prev[IX3(x - 1, z)].Waste + pw[x].W + prev[id].Waste) / 4.0;
                Ogr = (pw[x - 1].O + prev[IX3(x - 1, z)].Oxygen + pw[x].O + prev[id].Oxygen) / 4.0;
                Agr = (pw[x - 1].A + prev[IX3(x - 1, z)].Acetate + pw[x].A + prev[id].Acetate) / 4.0;
            } else {
                Cgr = (prev[IX3(x - 1, z - 1)].Carbon + prev[IX3(x - 1, z)].Carbon + prev[IX3(x, z - 1)].Carbon + prev[id].Carbon) / 4.0;
                Wgr = (prev[IX3(x - 1, z - 1)].Waste + prev[IX3(x - 1, z)].Waste + prev[IX3(x, z - 1)].Waste + prev[id].Waste) / 4.0;
                Ogr = (prev[IX3(x - 1, z - 1)].Oxygen + prev[IX3(x - 1, z)].Oxygen + prev[IX3(x, z - 1)].Oxygen + prev[id].Oxygen) / 4.0;
                Agr = (prev[IX3(x - 1, z - 1)].Acetate + prev[IX3(x - 1, z)].Acetate + prev[IX3(x, z - 1)].Acetate + prev[id].Acetate) / 4.0;
            }
        }
        buffer_solve(P, Agr, &prev[id]);
        double fCgr_aer = Cgr / (Cgr + P->kc_aer), fCgr_ana = Cgr / (Cgr + P->kc_ana);
        double fAgr = Agr / (Agr + P->ka), fOgr = Ogr / (Ogr + P->ko), fIgr = 0;
        (void)Wgr;
        double l1 = dmax((P->max_gr_car_aer + mgrCarAers) * fCgr_aer - mgrCarAers, 0.0);
        double l2 = dmax((P->max_gr_car_ana + mgrCarAnas) * fCgr_ana - mgrCarAnas, 0.0);
        double l3 = dmax((P->max_gr_ace_aer + mgrAceAers) * fAgr - mgrAceAers, 0.0);
        double qO = (P->q_o2_car * l1 * fCgr_aer + P->q_o2_ace * l3 * (1 - fCgr_aer)) * fOgr * dmax(1 - fIgr, 0.0) + P->q_o2_car_nt * dmin((Cgr / g1s), 1.0) * fCgr_aer * fOgr + P->q_o2_ace_nt * dmin((Agr / g3s), 1.0) * (1 - fCgr_aer) * fOgr;
        double qC = (P->q_car_aer * l1 * fCgr_aer * fOgr + P->q_car_ana * l2 * (1 - fOgr)) * dmax(1 - fIgr, 0.0) + P->q_car_aer_nt * dmin((Cgr / g1s), 1.0) * fCgr_aer * fOgr + P->q_car_ana_nt * dmin((Cgr / g2s), 1.0) * (1 - fOgr);
        double qA = (P->q_ace_aer * l3 * (1 - fCgr_aer) * fOgr) * dmax(1 - fIgr, 0.0) + P->q_ace_aer_nt * dmin((Agr / g3s), 1.0) * (1 - fCgr_aer) * fOgr;
        double pA = (P->p_ace_aer * l1 * fCgr_aer * fOgr + P->p_ace_ana * l2 * (1 - fOgr)) * dmax(1 - fIgr, 0.0) + P->p_ace_ana_nt * dmin((Cgr / g2s), 1.0) * (1 - fOgr);
        Env[id].qCarmnt = P->q_car_aer_nt * dmin((Cgr / g1s), 1.0) * fCgr_aer * fOgr + P->q_car_ana_nt * dmin((Cgr / g2s), 1.0) * (1 - fOgr);
        Env[id].qAcemnt = P->q_ace_aer_nt * dmin((Agr / g3s), 1.0) * (1 - fCgr_aer) * fOgr;
        Env[id].pAcemnt = P->p_ace_ana_nt * dmin((Cgr / g2s), 1.0) * (1 - fOgr);
        Env[id].qOxymnt = P->q_o2_car_nt * dmin((Cgr / g1s), 1.0) * fCgr_aer * fOgr + P->q_o2_ace_nt * dmin((Agr / g3s), 1.0) * (1 - fCgr_aer) * fOgr;
        double pW = P->carbon_to_waste * qC, qW = 0.0;
        Env[id].GrCarAer = l1 * fCgr_aer * fOgr * dmax(1 - fIgr, 0.0);
        Env[id].GrCarAna = l2 * (1 - fOgr) * dmax(1 - fIgr, 0.0);
        Env[id].GrAceAer = l3 * (1 - fCgr_aer) * fOgr * dmax(1 - fIgr, 0.0);
        Env[id].GrowthRate1 = Env[id].GrCarAer + Env[id].GrCarAna + Env[id].GrAceAer;
        Env[id].GrowthRate2 = Env[id].GrowthRate1;
        if (!(x > 2)) { if (!s->err) s->err = BCG_E_NEED_MORE_BOXES; return; }
        double Czz, Wzz, Azz, Ozz;
        const env_t* c0 = &prev[id];
        const env_t* up = &prev[IX3(x, z + 1)];
        if (z == 0) {
            Wzz = (up->Waste + pw[x].W - 2.0 * c0->Waste) / (BL * BL);
            Czz = (up->Carbon + pw[x].C - 2.0 * c0->Carbon) / (BL * BL);
            Azz = (up->Acetate + pw[x].A - 2.0 * c0->Acetate) / (BL * BL);
            Ozz = (up->Oxygen + pw[x].O - 2.0 * c0->Oxygen) / (BL * BL);
        } else {
            const env_t* dn = &prev[IX3(x, z - 1)];
            Wzz = (up->Waste + dn->Waste - 2.0 * c0->Waste) / (BL * BL);
            Czz = (up->Carbon + dn->Carbon - 2.0 * c0->Carbon) / (BL * BL);
            Azz = (up->Acetate + dn->Acetate - 2.0 * c0->Acetate) / (BL * BL);
            Ozz = (up->Oxygen + dn->Oxygen - 2.0 * c0->Oxygen) / (BL * BL);
        }
        const env_t* xp = &prev[IX3(x + 1, z)];
        const env_t* xm = &prev[IX3(x - 1, z)];
        double Cxx = (xp->Carbon + xm->Carbon - 2.0 * c0->Carbon) / (BL * BL);
        double Wxx = (xp->Waste + xm->Waste - 2.0 * c0->Waste) / (BL * BL);
        double Axx = (xp->Acetate + xm->Acetate - 2.0 * c0->Acetate) / (BL * BL);
        double Oxx = (xp->Oxygen + xm->Oxygen - 2.0 * c0->Oxygen) / (BL * BL);
        double DS = s->ds[id];
        double Cnew = c0->Carbon + (P->diff_colony_carbon * (Cxx + Czz) - qC * 0.25 * DS) * P->cdt;
        double CAcenew = c0->Acetate + (P->diff_colony_ace * (Axx + Azz) + pA * 0.25 * DS - qA * 0.25 * DS) * P->cdt;
        double Onew = c0->Oxygen + (P->diff_colony_o2 * (Oxx + Ozz) - qO * 0.25 * DS) * P->cdt;
        Env[id].Carbon = dmax(0.0, dmin(Cnew, P->max_carbon));
        Env[id].Oxygen = dmax(0.0, dmin(Onew, P->max_o2));
        Env[id].Acetate = dmax(0.0, CAcenew);
        double Wnew = c0->Waste + (P->diff_colony * (Wxx + Wzz) + pW * DS - qW * DS) * P->cdt;
        Env[id].Waste = dmax(0.0, Wnew);
    } else if (ins > 0.3 && z > 0) {
        int bp = s->inside[IX3(x + 1, z)] > 0.5, bm = s->inside[IX3(x - 1, z)] > 0.5;
        int bu = s->inside[IX3(x, z + 1)] > 0.5, bd = s->inside[IX3(x, z - 1)] > 0.5;
        const env_t *ep = &prev[IX3(x + 1, z)], *em = &prev[IX3(x - 1, z)], *eu = &prev[IX3(x, z + 1)], *ed = &prev[IX3(x, z - 1)];
        int den = bp + bm + bu + bd;
        double Cnew = (ep->Carbon * bp + em->Carbon * bm + eu->Carbon * bu + ed->Carbon * bd) / den;
        double Wnew = (ep->Waste * bp + em->Waste * bm + eu->Waste * bu + ed->Waste * bd) / den;
        double CAcenew = (ep->Acetate * bp + em->Acetate * bm + eu->Acetate * bu + ed->Acetate * bd) / den;
        double Onew = P->max_o2;
        Env[id].Carbon = dmax(0.0, dmin(Cnew, P->max_carbon));
        Env[id].Oxygen = dmax(0.0, dmin(Onew, P->max_o2));
        Env[id].Acetate = dmax(0.0, CAcenew);
        Env[id].Waste = dmax(0.0, Wnew);
    } else if (ins > 0.3 && z == 0) {
        int bp = s->inside[IX3(x + 1, z)] > 0.5, bm = s->inside[IX3(x - 1, z)] > 0.5, bu = s->inside[IX3(x, z + 1)] > 0.5;
        const env_t *ep = &prev[IX3(x + 1, z)], *em = &prev[IX3(x - 1, z)], *eu = &prev[IX3(x, z + 1)];
        int den = bp + bm + bu;
        double Cnew = (ep->Carbon * bp + em->Carbon * bm + eu->Carbon * bu) / den;
        double Wnew = (ep->Waste * bp + em->Waste * bm + eu->Waste * bu) / den;
        double CAcenew = (ep->Acetate * bp + em->Acetate * bm + eu->Acetate * bu) / den;
        Env[id].Carbon = dmax(0.0, dmin(Cnew, P->max_carbon));
        double Onew = P->max_o2;
        Env[id].Oxygen = dmax(0.0, dmin(Onew, P->max_o2));
        Env[id].Acetate = dmax(0.0, CAcenew);
        Env[id].Waste = dmax(0.0, Wnew);
    }
}

/* UpdateWallMultigrid_OxygenAcetate, Nutrients.cpp:509-659 (Box_y = 1).
 * For level > 0 and BoxX/4-1 < x < BoxX*3/4 the reference reads
 * uninitialised second differences; those points (never read by any other
 * point before the next copy-out from the multigrid) take Cxx = Wxx = Axx = 0
 * here. */
static void wall_point(orc_state* s, const env_t* Env, aga_t** pagar, aga_t** wal, aga_t** pwal, int level, int x)
{
    const bcg_params* P = &s->P;
    const int X = P->box_x, LM = P->max_levels_mg;
    if (level == 0 && s->inside[IX3(x, 0)] > 0.5) {
        const env_t* e = &Env[IX3(x, 0)];
        const aga_t* g = &pagar[0][(long)x * P->box_z_agar];
        double Cnew = (P->diff_colony_carbon * e->Carbon + P->diff_agar_carbon * g->C) / (P->diff_colony_carbon + P->diff_agar_carbon);
        double Onew = (P->diff_colony_o2 * e->Oxygen + P->diff_agar_o2 * g->O) / (P->diff_colony_o2 + P->diff_agar_o2);
        wal[0][x].C = dmax(0.0, dmin(Cnew, P->max_carbon));
        wal[0][x].O = dmax(0.0, dmin(Onew, P->max_o2));
        double CAcenew = (P->diff_colony_ace * e->Acetate + P->diff_agar_ace * g->A) / (P->diff_colony_ace + P->diff_agar_ace);
        wal[0][x].A = dmax(0.0, CAcenew);
        double Wnew = (P->diff_colony * e->Waste + P->diff_agar * g->W) / (P->diff_colony + P->diff_agar);
        wal[0][x].W = dmax(0.0, Wnew);
        return;
    }
    const aga_t* pw = pwal[level];
    double h2l = P->box_length * P->box_length * pow(4.0, level);
    double Cxx = 0, Wxx = 0, Axx = 0;
    if (level > 0 && (x >= X / 4 - 1) && x <= X * 3 / 4) {
        if (x == X / 4 - 1) {
            const aga_t* q = &pwal[level - 1][0];
            Wxx = (pw[x - 1].W + q->W - 2 * pw[x].W) / h2l;
            Cxx = (pw[x - 1].C + q->C - 2 * pw[x].C) / h2l;
            Axx = (pw[x - 1].A + q->A - 2 * pw[x].A) / h2l;
        } else if (x == X * 3 / 4) {
            const aga_t* q = &pwal[level - 1][X - 2];
            Wxx = (pw[x + 1].W + q->W - 2 * pw[x].W) / h2l;
            Cxx = (pw[x + 1].C + q->C - 2 * pw[x].C) / h2l;
            Axx = (pw[x + 1].A + q->A - 2 * pw[x].A) / h2l;
        }
    } else if (level < LM - 1 && (x == 0 || x == X - 1)) {
        int ly = 0;
        if (x == 0) {
            const aga_t* q = &pwal[level + 1][X / 4 - 1];
            Wxx = (pw[x + 2].W + 1.0 / (ly + 1) * q->W + ly * 1.0 / (ly + 1) * q->W - 2 * pw[x].W) / 4 / h2l;
            Cxx = (pw[x + 2].C + 1.0 / (ly + 1) * q->C + ly * 1.0 / (ly + 1) * q->C - 2 * pw[x].C) / 4 / h2l;
            Axx = (pw[x + 2].A + 1.0 / (ly + 1) * q->A + ly * 1.0 / (ly + 1) * q->A - 2 * pw[x].A) / 4 / h2l;
        } else {
            const aga_t* q = &pwal[level + 1][X * 3 / 4];
            Wxx = (pw[x - 1].W + 1.0 / (ly + 1) * q->W + ly * 1.0 / (ly + 1) * q->W - 2 * pw[x].W) / h2l;
            Cxx = (pw[x - 1].C + 1.0 / (ly + 1) * q->C + ly * 1.0 / (ly + 1) * q->C - 2 * pw[x].C) / h2l;
            Axx = (pw[x - 1].A + 1.0 / (ly + 1) * q->A + ly * 1.0 / (ly + 1) * q->A - 2 * pw[x].A) / h2l;
        }
    } else if (level == LM - 1 && (x == 0 || x == X - 1)) {
        if (x == 0) {
            Wxx = (pw[x + 1].W - 1.0 * pw[x].W) / h2l;
            Cxx = (pw[x + 1].C - 1.0 * pw[x].C) / h2l;
            Axx = (pw[x + 1].A - 1.0 * pw[x].A) / h2l;
        } else {
            Wxx = (pw[x - 1].W - 1.0 * pw[x].W) / h2l;
            Cxx = (pw[x - 1].C - 1.0 * pw[x].C) / h2l;
            Axx = (pw[x - 1].A - 1.0 * pw[x].A) / h2l;
        }
    } else {
        Wxx = (pw[x - 1].W + pw[x + 1].W - 2 * pw[x].W) / h2l;
        Cxx = (pw[x - 1].C + pw[x + 1].C - 2 * pw[x].C) / h2l;
        Axx = (pw[x - 1].A + pw[x + 1].A - 2 * pw[x].A) / h2l;
    }
    const aga_t* g = &pagar[level][(long)x * P->box_z_agar];
    double Wzz = 2.0 * (g->W - pw[x].W) / h2l;
    double Czz = 2.0 * (g->C - pw[x].C) / h2l;
    double Azz = 2.0 * (g->A - pw[x].A) / h2l;
    double Cnew = pw[x].C + P->diff_agar_carbon * (Cxx + Czz) * P->cdt;
    double Onew = P->max_o2;
    wal[level][x].C = dmax(0.0, dmin(Cnew, P->max_carbon));
    wal[level][x].O = dmax(0.0, dmin(Onew, P->max_o2));
    double CAcenew = pw[x].A + P->diff_agar_ace * (Axx + Azz) * P->cdt;
    wal[level][x].A = dmax(0.0, CAcenew);
    double Wnew = pw[x].W + P->diff_agar * (Wxx + Wzz) * P->cdt;
    wal[level][x].W = dmax(0.0, Wnew);
}

/* The sweep loop of UpdateEnvArrayMG_OxygenAcetate, Multigrid.cpp:1017-1120.
 * cur/prev are the locally swapped buffers; *count is the sweep counter. */
static void sweeps(orc_state* s, int nsweeps, env_t** cur, env_t** prev, aga_t*** ca, aga_t*** pa,
                   aga_t*** cw, aga_t*** pw, int* count)
{
    const bcg_params* P = &s->P;
    int maxH = s->maxz;
    for (int j = 0; j < nsweeps; j++) {
        int zmin, zmax, dir;
        if (*count % 2 == 0) { zmin = 0; zmax = maxH + 1; dir = 1; }
        else { zmin = -maxH - 1; zmax = 0; dir = -1; }
        for (int zi = zmin; zi <= zmax; zi++) {
            if (zi * dir > 0) {
                int z = zi * dir - 1;
                for (int xi = s->minx; xi <= s->maxx; xi++)
                    if (s->ds[IX3(xi, z)] > DBL_EPSILON) colony_point(s, *cur, *prev, (*pw)[0], xi, z);
            } else if (zi == 0) {
                for (int level = 0; level < P->max_levels_mg; level++)
                    for (int xi = 0; xi < P->box_x; xi++)
                        wall_point(s, *cur, *pa, *cw, *pw, level, xi);
            }
        }
        if (P->nutrient_gsi == 0) {
            env_t* t1 = *prev; *prev = *cur; *cur = t1;
            aga_t** t2 = *pa; *pa = *ca; *ca = t2;
            aga_t** t3 = *pw; *pw = *cw; *cw = t3;
        }
        (*count)++;
    }
}

/* ======================================================= multigrid ======== */
/* class Multigrid, Multigrid.cpp:5-981.  Arrays are (nx+1) x (nz+1),
 * x-major; the three species are carbon (C), oxygen (O), acetate (A). */
#define MI(l, i, k) ((long)(i) * (mg_nz(s, l) + 1) + (k))
/* Reads go through the reference's flat index i*(nz+1)+k: on levels with
 * nz <= 1 the stencils reach k = -1 or k = nz+1, which Array3D maps onto
 * the neighbouring column (Multigrid.cpp:160-249, 269-467); an index past
 * either end of the array (undefined in the reference) reads as 0. */
static aga_t g_zero_aga;
static aga_t* mg_ref(orc_state* s, aga_t** arr, int l, int i, int k)
{
    long n = (long)(mg_nx(s, l) + 1) * (mg_nz(s, l) + 1);
    long f = MI(l, i, k);
    if (f < 0 || f >= n) { memset(&g_zero_aga, 0, sizeof(g_zero_aga)); return &g_zero_aga; }
    return &arr[l][f];
}
#define AG(l, i, k) (*mg_ref(s, s->mgA, l, i, k))
#define RS(l, i, k) (*mg_ref(s, s->mgR, l, i, k))
#define ER(l, i, k) (*mg_ref(s, s->mgE, l, i, k))
/* insideColonyDen(i, 0, 0).  The restriction clamps i to BoxX, one x-row
 * past the array (Multigrid.cpp:279); that row counts as outside (0). */
static double ins0(orc_state* s, int i) { return i < s->P.box_x ? s->inside[IX3(i, 0)] : 0.0; }

/* relaxationAgarElementwise, Multigrid.cpp:160-249 */
static void relax_point(orc_state* s, int l, int i, int k, int nx, int nz)
{
    const bcg_params* P = &s->P;
    const int A_ = P->max_levels_mg;
    double h2 = P->box_length * P->box_length * (double)(1 << (2 * l));
    double dt = s->mg_dt;
    int d = 1 << l;
    double DC = P->diff_agar_carbon, DA = P->diff_agar_ace, DO = P->diff_agar_o2;
    aga_t* e = &ER(l, i, k);
    const aga_t* r = &RS(l, i, k);
    if (k == 0) {
        int i0 = imin(imax((i - nx / 2) * d + P->box_x / 2, 0), P->box_x - 1);
        if (ins0(s, i0) > 0) { e->C = r->C; e->O = r->O; e->A = r->A; }
        else if (i == 0 || i == nx) {
            if (l >= A_ - 1) {
                const aga_t* s1 = (i == 0) ? &ER(l, i + 1, 0) : &ER(l, i - 1, 0);
                const aga_t* up = &ER(l, i, 1);
                e->C = (r->C * h2 / dt / DC + (s1->C + up->C)) / (h2 / dt / DC + 2);
                e->O = r->O;
                e->A = (r->A * h2 / dt / DA + (s1->A + up->A)) / (h2 / dt / DA + 2);
            }
        } else {
            const aga_t *up = &ER(l, i, 1), *xm = &ER(l, i - 1, 0), *xp = &ER(l, i + 1, 0);
            e->C = (r->C * h2 / dt / DC + up->C + 0.5 * xm->C + 0.5 * xp->C) / (h2 / dt / DC + 2);
            e->O = r->O;
            e->A = (r->A * h2 / dt / DA + up->A + 0.5 * xm->A + 0.5 * xp->A) / (h2 / dt / DA + 2);
        }
    } else if (k == nz) {
        if (l >= A_ - 1) {
            if (i == 0 || i == nx) {
                const aga_t* s1 = (i == 0) ? &ER(l, i + 1, k) : &ER(l, i - 1, k);
                const aga_t* dn = &ER(l, i, k - 1);
                e->C = (r->C * h2 / dt / DC + (s1->C + dn->C)) / (h2 / dt / DC + 2);
                e->O = r->O;
                e->A = (r->A * h2 / dt / DA + (s1->A + dn->A)) / (h2 / dt / DA + 2);
            } else {
                const aga_t *dn = &ER(l, i, k - 1), *xp = &ER(l, i + 1, k), *xm = &ER(l, i - 1, k);
                e->C = (r->C * h2 / dt / DC + dn->C + 0.5 * xp->C + 0.5 * xm->C) / (h2 / dt / DC + 2);
                e->O = (r->O * h2 / dt / DO + dn->O + 0.5 * xp->O + 0.5 * xm->O) / (h2 / dt / DO + 2);
                e->A = (r->A * h2 / dt / DA + dn->A + 0.5 * xp->A + 0.5 * xm->A) / (h2 / dt / DA + 2);
            }
        }
    } else if (i == 0 || i == nx) {
        if (l >= A_ - 1) {
            const aga_t *dn = &ER(l, i, k - 1), *up = &ER(l, i, k + 1);
            const aga_t* s1 = (i == 0) ? &ER(l, i + 1, k) : &ER(l, i - 1, k);
            e->C = (r->C * h2 / dt / DC + 0.5 * dn->C + 0.5 * up->C + s1->C) / (h2 / dt / DC + 2);
            e->O = r->O;
            e->A = (r->A * h2 / dt / DA + 0.5 * dn->A + 0.5 * up->A + s1->A) / (h2 / dt / DA + 2);
        }
    } else {
        const aga_t *dn = &ER(l, i, k - 1), *up = &ER(l, i, k + 1), *xm = &ER(l, i - 1, k), *xp = &ER(l, i + 1, k);
        e->C = (r->C * h2 / dt / DC + 0.5 * dn->C + 0.5 * up->C + 0.5 * xm->C + 0.5 * xp->C) / (h2 / dt / DC + 2);
        e->O = (r->O * h2 / dt / DO + 0.5 * dn->O + 0.5 * up->O + 0.5 * xm->O + 0.5 * xp->O) / (h2 / dt / DO + 2);
        e->A = (r->A * h2 / dt / DA + 0.5 * dn->A + 0.5 * up->A + 0.5 * xm->A + 0.5 * xp->A) / (h2 / dt / DA + 2);
    }
}
/* relaxationAgarAtLevel, Multigrid.cpp:135-158: even columns, then odd,
 * each column bottom to top in place. */
static void relax_level(orc_state* s, int l)
{
    int nx = mg_nx(s, l), nz = mg_nz(s, l);
    for (int i = 0; i < nx + 1; i += 2) for (int k = 0; k < nz + 1; k++) relax_point(s, l, i, k, nx, nz);
    for (int i = 1; i < nx + 1; i += 2) for (int k = 0; k < nz + 1; k++) relax_point(s, l, i, k, nx, nz);
}

/* restrictionAgaElementwise, Multigrid.cpp:269-405 (level l from l-1) */
static void restrict_point(orc_state* s, int l, int i, int k, int nx, int nz, int nxp, int nzp, double h2, int d)
{
    const bcg_params* P = &s->P;
    const int A_ = P->max_levels_mg;
    const double dt = s->mg_dt, DC = P->diff_agar_carbon, DA = P->diff_agar_ace, DO = P->diff_agar_o2;
    int i0 = imin(imax((i - nx / 2) * d + P->box_x / 2, 0), P->box_x);
    int ip = 2 * i - nx + nxp / 2, kp = 2 * k;
    aga_t* R = &RS(l, i, k);
    const int lp = l - 1;
#define EP(a, b) ER(lp, a, b)
#define RP(a, b) RS(lp, a, b)
#define AP(a, b) AG(lp, a, b)
#define AL(a, b) AG(l, a, b)
    if (i == 0 || i == nx || k == nz) {
        if (l >= A_) {
            if (k == nz && (i > 0) && (i < nx)) {
                R->C = (RP(ip, kp).C + 0.5 * (EP(ip + 1, kp).C + EP(ip - 1, kp).C + 2 * EP(ip, kp - 1).C - 4 * EP(ip, kp).C) * DC * dt * 4 / h2 - EP(ip, kp).C) / 2;
                R->O = (RP(ip, kp).O + 0.5 * (EP(2 * i + 1, 2 * k).O + EP(2 * i - 1, 2 * k).O + 2 * EP(2 * i, 2 * k - 1).O - 4 * EP(2 * i, 2 * k).O) * DO * dt * 4 / h2 - EP(2 * i, 2 * k).O) / 2;
                R->A = (RP(ip, kp).A + 0.5 * (EP(2 * i + 1, 2 * k).A + EP(2 * i - 1, 2 * k).A + 2 * EP(2 * i, 2 * k - 1).A - 4 * EP(2 * i, 2 * k).A) * DA * dt * 4 / h2 - EP(2 * i, 2 * k).A) / 2;
            } else {
                int sx = (i == 0) ? 1 : -1;   /* the one x-neighbour inside the domain */
                if (k == 0) {
                    R->C = (RP(ip, kp).C + 0.5 * (2 * EP(ip + sx, kp).C + 2 * EP(ip, kp + 1).C - 4 * EP(ip, kp).C) * DC * dt * 4 / h2 - EP(ip, kp).C) / 2;
                    R->O = RP(ip, kp).O - EP(ip, kp).O;
                    R->A = (RP(ip, kp).A + 0.5 * (2 * EP(2 * i + sx, 2 * k).A + 2 * EP(2 * i, 2 * k + 1).A - 4 * EP(2 * i, 2 * k).A) * DA * dt * 4 / h2 - EP(2 * i, 2 * k).A) / 2;
                } else if (k == nz) {
                    R->C = (RP(ip, kp).C + 0.5 * (2 * EP(ip + sx, kp).C + 2 * EP(ip, kp - 1).C - 4 * EP(ip, kp).C) * DC * dt * 4 / h2 - EP(ip, kp).C) / 2;
                    R->O = RP(ip, kp).O - EP(ip, kp).O;
                    R->A = (RP(ip, kp).A + 0.5 * (2 * EP(2 * i + sx, 2 * k).A + 2 * EP(2 * i, 2 * k - 1).A - 4 * EP(2 * i, 2 * k).A) * DA * dt * 4 / h2 - EP(2 * i, 2 * k).A) / 2;
                } else {
                    R->C = (RP(ip, kp).C + 0.5 * (2 * EP(ip + sx, kp).C + EP(ip, kp + 1).C + EP(ip, kp - 1).C - 4 * EP(ip, kp).C) * DC * dt * 4 / h2 - EP(ip, kp).C) / 2;
                    R->O = RP(ip, kp).O - EP(ip, kp).O;
                    R->A = (RP(ip, kp).A + 0.5 * (2 * EP(2 * i + sx, 2 * k).A + EP(2 * i, 2 * k + 1).A + EP(2 * i, 2 * k - 1).A - 4 * EP(2 * i, 2 * k).A) * DA * dt * 4 / h2 - EP(2 * i, 2 * k).A) / 2;
                }
            }
        }
    } else if (k == 0) {
        if (ins0(s, i0) > 0) { R->C = 0; R->O = 0; R->A = 0; }
        else if (ip > 0 && ip < nxp) {
            R->C = (RP(ip, 0).C + 0.5 * (EP(ip + 1, 0).C + EP(ip - 1, 0).C + 2 * EP(ip, 1).C - 4 * EP(ip, 0).C) * DC * dt * 4 / h2 - EP(ip, 0).C) * 0.5;
            R->A = (RP(ip, 0).A + 0.5 * (EP(ip + 1, 0).A + EP(ip - 1, 0).A + 2 * EP(ip, 1).A - 4 * EP(ip, 0).A) * DA * dt * 4 / h2 - EP(ip, 0).A) * 0.5;
            R->O = (RP(ip, 0).O - EP(ip, 0).O) * 0.5;
        } else if ((l < A_) && (ip >= 0 && ip <= nxp) && ((ip == 0) || (ip == nxp))) {
            if (ip == 0) {
                R->C = (AP(ip + 2, 0).C + 0.5 * EP(ip + 2, 0).C + AL(i - 1, 0).C + 2 * AL(i, 1).C - 4 * AL(i, 0).C) * DC * dt / h2;
                R->A = (AP(ip + 2, 0).A + 0.5 * EP(ip + 2, 0).A + AL(i - 1, 0).A + 2 * AL(i, 1).A - 4 * AL(i, 0).A) * DA * dt / h2;
                R->O = P->max_o2_agar - AL(i, 0).O;
            } else {
                R->C = (AL(i + 1, 0).C + 0.5 * EP(ip - 2, 0).C + AP(ip - 2, 0).C + 2 * AL(i, 1).C - 4 * AL(i, 0).C) * dt * DC / h2;
                R->A = (AL(i + 1, 0).A + 0.5 * EP(ip - 2, 0).A + AP(ip - 2, 0).A + 2 * AL(i, 1).A - 4 * AL(i, 0).A) * dt * DA / h2;
                R->O = P->max_o2_agar - AL(i, 0).O;
            }
        }
    } else if (l < A_ && ip >= 0 && ip <= nxp && kp <= nzp) {
        if (kp == nzp) {
            if (ip == 0 || ip == nxp) {
                R->C = (AL(i + 1, k).C + AL(i - 1, k).C + AL(i, k + 1).C + AL(i, k - 1).C - 4 * AL(i, k).C) * DC * dt / h2;
                R->O = (AL(i + 1, k).O + AL(i - 1, k).O + AL(i, k + 1).O + AL(i, k - 1).O - 4 * AL(i, k).O) * DO * dt / h2;
                R->A = (AL(i + 1, k).A + AL(i - 1, k).A + AL(i, k + 1).A + AL(i, k - 1).A - 4 * AL(i, k).A) * DA * dt / h2;
            } else {
                R->C = (AL(i + 1, k).C + AL(i - 1, k).C + AL(i, k + 1).C + AP(ip, kp - 2).C + 0.5 * EP(ip, kp - 2).C - 4 * AL(i, k).C) * DC * dt / h2;
                R->O = (AL(i + 1, k).O + AL(i - 1, k).O + AL(i, k + 1).O + AP(ip, kp - 2).O + 0.5 * EP(ip, kp - 2).O - 4 * AL(i, k).O) * DO * dt / h2;
                R->A = (AL(i + 1, k).A + AL(i - 1, k).A + AL(i, k + 1).A + AP(ip, kp - 2).A + 0.5 * EP(ip, kp - 2).A - 4 * AL(i, k).A) * DA * dt / h2;
            }
        } else if (ip == 0) {
            R->C = (AP(ip + 2, kp).C + 0.5 * EP(ip + 2, kp).C + AL(i - 1, k).C + AL(i, k + 1).C + AL(i, k - 1).C - 4 * AL(i, k).C) * DC * dt / h2;
            R->O = (AP(ip + 2, kp).O + 0.5 * EP(ip + 2, kp).O + AL(i - 1, k).O + AL(i, k + 1).O + AL(i, k - 1).O - 4 * AL(i, k).O) * DO * dt / h2;
            R->A = (AP(ip + 2, kp).A + 0.5 * EP(ip + 2, kp).A + AL(i - 1, k).A + AL(i, k + 1).A + AL(i, k - 1).A - 4 * AL(i, k).A) * DA * dt / h2;
        } else if (ip == nxp) {
            R->C = (AL(i + 1, k).C + 0.5 * EP(ip - 2, kp).C + AP(ip - 2, kp).C + AL(i, k + 1).C + AL(i, k - 1).C - 4 * AL(i, k).C) * DC * dt / h2;
            R->O = (AL(i + 1, k).O + 0.5 * EP(ip - 2, kp).O + AP(ip - 2, kp).O + AL(i, k + 1).O + AL(i, k - 1).O - 4 * AL(i, k).O) * DO * dt / h2;
            R->A = (AL(i + 1, k).A + 0.5 * EP(ip - 2, kp).A + AP(ip - 2, kp).A + AL(i, k + 1).A + AL(i, k - 1).A - 4 * AL(i, k).A) * DA * dt / h2;
        } else {
            R->C = (RP(ip, kp).C + 0.5 * (EP(ip + 1, kp).C + EP(ip - 1, kp).C + EP(ip, kp + 1).C + EP(ip, kp - 1).C - 4 * EP(ip, kp).C) * DC * dt / h2 * 4 - EP(ip, kp).C) * 0.5;
            R->O = (RP(ip, kp).O + 0.5 * (EP(ip + 1, kp).O + EP(ip - 1, kp).O + EP(ip, kp + 1).O + EP(ip, kp - 1).O - 4 * EP(ip, kp).O) * DO * dt / h2 * 4 - EP(ip, kp).O) * 0.5;
            R->A = (RP(ip, kp).A + 0.5 * (EP(ip + 1, kp).A + EP(ip - 1, kp).A + EP(ip, kp + 1).A + EP(ip, kp - 1).A - 4 * EP(ip, kp).A) * DA * dt / h2 * 4 - EP(ip, kp).A) * 0.5;
        }
    } else if (l >= A_) {
        R->C = (RP(ip, kp).C + 0.5 * (EP(ip + 1, kp).C + EP(ip - 1, kp).C + EP(ip, kp + 1).C + EP(ip, kp - 1).C - 4 * EP(ip, kp).C) * DC * dt / h2 * 4 - EP(ip, kp).C) * 0.5;
        R->O = (RP(ip, kp).O + 0.5 * (EP(ip + 1, kp).O + EP(ip - 1, kp).O + EP(ip, kp + 1).O + EP(ip, kp - 1).O - 4 * EP(ip, kp).O) * DO * dt / h2 * 4 - EP(ip, kp).O) * 0.5;
        R->A = (RP(ip, kp).A + 0.5 * (EP(ip + 1, kp).A + EP(ip - 1, kp).A + EP(ip, kp + 1).A + EP(ip, kp - 1).A - 4 * EP(ip, kp).A) * DA * dt / h2 * 4 - EP(ip, kp).A) * 0.5;
    }
}
/* residueRestrictionAga, Multigrid.cpp:251-267 */
static void restrict_level(orc_state* s, int l)
{
    const int X = s->P.box_x, ZA = s->P.box_z_agar;
    int d = 1 << l, d0 = 1 << s->P.max_levels_mg;
    int nx = mg_nx(s, l), nz = mg_nz(s, l);
    int nxp = imin(X, X * d0 / d), nzp = imin(ZA, ZA * d0 / d);
    double h2 = s->P.box_length * s->P.box_length * d * d;
    for (int i = 0; i < nx + 1; i++) for (int k = 0; k < nz + 1; k++) restrict_point(s, l, i, k, nx, nz, nxp, nzp, h2, d);
}
/* interpolationAga, Multigrid.cpp:407-467 (level l from l+1) */
static void interpolate_level(orc_state* s, int l)
{
    const int X = s->P.box_x;
    int d = 1 << l, d0 = 1 << s->P.max_levels_mg;
    int nx = mg_nx(s, l), nz = mg_nz(s, l);
    int nxp = imin(X, X * d0 / d / 4);
    for (int i = 0; i < nx + 1; i++)
        for (int k = 0; k < nz + 1; k++) {
            aga_t* e = &ER(l, i, k);
            if (i % 2 == 0) {
                int ip = nxp / 2 - nx / 4 + i / 2;
                if (k % 2 == 0) {
                    const aga_t* a = &ER(l + 1, ip, k / 2);
                    e->C += a->C; e->O += a->O; e->A += a->A;
                } else {
                    int kp = (k - 1) / 2;
                    const aga_t *a = &ER(l + 1, ip, kp), *b = &ER(l + 1, ip, kp + 1);
                    e->C += 0.5 * (a->C + b->C); e->O += 0.5 * (a->O + b->O); e->A += 0.5 * (a->A + b->A);
                }
            } else {
                int ip = nxp / 2 - nx / 4 + (i - 1) / 2;
                if (k % 2 == 0) {
                    int kp = k / 2;
                    const aga_t *a = &ER(l + 1, ip, kp), *b = &ER(l + 1, ip + 1, kp);
                    e->C += 0.5 * (a->C + b->C); e->O += 0.5 * (a->O + b->O); e->A += 0.5 * (a->A + b->A);
                } else {
                    int kp = (k - 1) / 2;
                    const aga_t *a = &ER(l + 1, ip, kp), *b = &ER(l + 1, ip, kp + 1), *c = &ER(l + 1, ip + 1, kp), *dd = &ER(l + 1, ip + 1, kp + 1);
                    e->C += 0.25 * (a->C + b->C + c->C + dd->C);
                    e->O += 0.25 * (a->O + b->O + c->O + dd->O);
                    e->A += 0.25 * (a->A + b->A + c->A + dd->A);
                }
            }
        }
}
/* rewriteSolBdryAga, Multigrid.cpp:469-503 */
static void rewrite_bdry(orc_state* s, int l)
{
    const int X = s->P.box_x;
    int d = 1 << l, d0 = 1 << s->P.max_levels_mg;
    int nx = mg_nx(s, l), nz = mg_nz(s, l), nx2 = imin(X, X * d0 / d / 4);
    int k = nz, k2 = nz / 2;
    for (int i = 0; i < nx + 1; i++) {
        int i2 = nx2 / 2 + i / 2 - nx / 4, i2p1 = nx2 / 2 + (i + 1) / 2 - nx / 4;
        const aga_t *a = &AG(l + 1, i2, k2), *b = &AG(l + 1, i2p1, k2);
        aga_t* o = &AG(l, i, k);
        o->C = (a->C + b->C) / 2; o->O = (a->O + b->O) / 2; o->A = (a->A + b->A) / 2;
    }
    for (k = 0; k < nz; k++) {
        int kk2 = k / 2, k2p1 = (k + 1) / 2;
        for (int side = 0; side < 2; side++) {
            int i = side ? nx : 0;
            int i2 = nx2 / 2 + i / 2 - nx / 4;
            const aga_t *a = &AG(l + 1, i2, kk2), *b = &AG(l + 1, i2, k2p1);
            aga_t* o = &AG(l, i, k);
            o->C = (a->C + b->C) / 2; o->O = (a->O + b->O) / 2; o->A = (a->A + b->A) / 2;
        }
    }
}
/* updateSolAgaElementwise, Multigrid.cpp:544-568 */
static void update_sol_level(orc_state* s, int l)
{
    const bcg_params* P = &s->P;
    const int X = P->box_x, ZA = P->box_z_agar;
    int d = 1 << l, d0 = 1 << P->max_levels_mg;
    int nx = mg_nx(s, l), nz = mg_nz(s, l), nxp = imin(X, X * d0 / d), nzp = imin(ZA, ZA * d0 / d);
    for (int i = 0; i < nx + 1; i++)
        for (int k = 0; k < nz + 1; k++) {
            aga_t *R = &RS(l, i, k), *E = &ER(l, i, k), *A = &AG(l, i, k);
            R->C = 0; R->O = 0; R->A = 0;
            int ip = 2 * i - nx + nxp / 2, kp = 2 * k;
            if (l < P->max_levels_mg) {
                if (l == 0 || ip <= 0 || ip >= nxp || kp >= nzp) {
                    A->C += E->C; A->O += E->O; A->A += E->A;
                    A->C = dmax(dmin(A->C, P->max_carbon), 0.0);
                    A->O = dmax(dmin(A->O, P->max_o2_agar), 0.0);
                    A->A = dmax(A->A, 0.0);
                }
            }
            E->C = 0; E->O = 0; E->A = 0;
        }
}
/* updateResAgaElementwise, Multigrid.cpp:570-701 */
static void update_res_level(orc_state* s, int l)
{
    const bcg_params* P = &s->P;
    const int X = P->box_x, ZA = P->box_z_agar, A_ = P->max_levels_mg;
    int d = 1 << l, d0 = 1 << A_;
    int nx = mg_nx(s, l), nz = mg_nz(s, l), nxp = imin(X, X * d0 / d), nzp = imin(ZA, ZA * d0 / d);
    double h2 = P->box_length * P->box_length * d * d, dt = s->mg_dt;
    const double DC = P->diff_agar_carbon, DA = P->diff_agar_ace, DO = P->diff_agar_o2;
    const int lp = l - 1;
    if (l >= A_) return;
    for (int i = 0; i < nx + 1; i++)
        for (int k = 0; k < nz + 1; k++) {
            aga_t* R = &RS(l, i, k);
            int ip = 2 * i - nx + nxp / 2, kp = 2 * k;
            if (i == 0 || i == nx) {
                if (l == A_ - 1) {
                    int sx = (i == 0) ? 1 : -1;
                    if (k == 0) {
                        R->C = (2 * AL(i + sx, k).C + 2 * AL(i, k + 1).C - 4 * AL(i, k).C) * DC * dt / h2;
                        R->O = 0;
                        R->A = (2 * AL(i + sx, k).A + 2 * AL(i, k + 1).A - 4 * AL(i, k).A) * DA * dt / h2;
                    } else if (k == nz) {
                        R->C = (2 * AL(i + sx, k).C + 2 * AL(i, k - 1).C - 4 * AL(i, k).C) * DC * dt / h2;
                        R->O = 0;
                        R->A = (2 * AL(i + sx, k).A + 2 * AL(i, k - 1).A - 4 * AL(i, k).A) * DA * dt / h2;
                    } else {
                        R->C = (2 * AL(i + sx, k).C + AL(i, k - 1).C + AL(i, k + 1).C - 4 * AL(i, k).C) * DC * dt / h2;
                        R->O = 0;
                        R->A = (2 * AL(i + sx, k).A + AL(i, k - 1).A + AL(i, k + 1).A - 4 * AL(i, k).A) * DA * dt / h2;
                    }
                }
            } else if (k == nz) {
                if (l == A_ - 1) {
                    R->C = (AL(i + 1, k).C + AL(i - 1, k).C + 2 * AL(i, k - 1).C - 4 * AL(i, k).C) * dt * DC / h2;
                    R->O = (AL(i + 1, k).O + AL(i - 1, k).O + 2 * AL(i, k - 1).O - 4 * AL(i, k).O) * DO / h2;
                    R->A = (AL(i + 1, k).A + AL(i - 1, k).A + 2 * AL(i, k - 1).A - 4 * AL(i, k).A) * dt * DA / h2;
                }
            } else if (k == 0) {
                if (l == 0) {
                    if (ins0(s, i) > 0) { R->C = 0; R->O = 0; R->A = 0; }
                    else {
                        R->C = (AL(i + 1, k).C + AL(i - 1, k).C + 2 * AL(i, k + 1).C - 4 * AL(i, k).C) * dt * DC / h2;
                        R->O = P->max_o2_agar - AL(i, k).O;
                        R->A = (AL(i + 1, k).A + AL(i - 1, k).A + 2 * AL(i, k + 1).A - 4 * AL(i, k).A) * dt * DA / h2;
                    }
                } else if ((ip > 0 && ip < nxp) != 1) {
                    if (ip == 0) {
                        R->C = (AP(ip + 2, kp).C + AL(i - 1, k).C + 2 * AL(i, k + 1).C - 4 * AL(i, k).C) * dt * DC / h2;
                        R->O = P->max_o2_agar - AL(i, k).O;
                        R->A = (AP(ip + 2, kp).A + AL(i - 1, k).A + 2 * AL(i, k + 1).A - 4 * AL(i, k).A) * dt * DA / h2;
                    } else if (ip == nxp) {
                        R->C = (AP(ip - 2, kp).C + AL(i + 1, k).C + 2 * AL(i, k + 1).C - 4 * AL(i, k).C) * dt * DC / h2;
                        R->O = P->max_o2_agar - AL(i, k).O;
                        R->A = (AP(ip - 2, kp).A + AL(i + 1, k).A + 2 * AL(i, k + 1).A - 4 * AL(i, k).A) * dt * DA / h2;
                    } else {
                        R->C = (AL(i + 1, k).C + AL(i - 1, k).C + 2 * AL(i, k + 1).C - 4 * AL(i, k).C) * dt * DC / h2;
                        R->O = P->max_o2_agar - AL(i, k).O;
                        R->A = (AL(i + 1, k).A + AL(i - 1, k).A + 2 * AL(i, k + 1).A - 4 * AL(i, k).A) * dt * DA / h2;
                    }
                }
            } else {
                if (l > 0) {
                    if (kp == nzp && ip > 0 && ip < nxp) {
                        R->C = (AL(i + 1, k).C + AL(i - 1, k).C + AP(ip, kp - 2).C + AL(i, k + 1).C - 4 * AL(i, k).C) * dt * DC / h2;
                        R->O = (AL(i + 1, k).O + AL(i - 1, k).O + AP(ip, kp - 2).O + AL(i, k + 1).O - 4 * AL(i, k).O) * dt * DO / h2;
                        R->A = (AL(i + 1, k).A + AL(i - 1, k).A + AP(ip, kp - 2).A + AL(i, k + 1).A - 4 * AL(i, k).A) * dt * DA / h2;
                    } else if (ip == 0 && kp < nzp) {
                        R->C = (AP(ip + 2, kp).C + AL(i - 1, k).C + AL(i, k - 1).C + AL(i, k + 1).C - 4 * AL(i, k).C) * dt * DC / h2;
                        R->O = (AP(ip + 2, kp).O + AL(i - 1, k).O + AL(i, k - 1).O + AL(i, k + 1).O - 4 * AL(i, k).O) * dt * DO / h2;
                        R->A = (AP(ip + 2, kp).A + AL(i - 1, k).A + AL(i, k - 1).A + AL(i, k + 1).A - 4 * AL(i, k).A) * dt * DA / h2;
                    } else if (ip == nxp && kp < nzp) {
                        R->C = (AL(i + 1, k).C + AP(ip - 2, kp).C + AL(i, k - 1).C + AL(i, k + 1).C - 4 * AL(i, k).C) * dt * DC / h2;
                        R->O = (AL(i + 1, k).O + AP(ip - 2, kp).O + AL(i, k - 1).O + AL(i, k + 1).O - 4 * AL(i, k).O) * dt * DO / h2;
                        R->A = (AL(i + 1, k).A + AP(ip - 2, kp).A + AL(i, k - 1).A + AL(i, k + 1).A - 4 * AL(i, k).A) * dt * DA / h2;
                    } else if (ip <= 0 || ip >= nxp || kp >= nzp) {
                        R->C = (AL(i + 1, k).C + AL(i - 1, k).C + AL(i, k - 1).C + AL(i, k + 1).C - 4 * AL(i, k).C) * dt * DC / h2;
                        R->O = (AL(i + 1, k).O + AL(i - 1, k).O + AL(i, k - 1).O + AL(i, k + 1).O - 4 * AL(i, k).O) * dt * DO / h2;
                        R->A = (AL(i + 1, k).A + AL(i - 1, k).A + AL(i, k - 1).A + AL(i, k + 1).A - 4 * AL(i, k).A) * dt * DA / h2;
                    }
                } else {
                    R->C = (AL(i + 1, k).C + AL(i - 1, k).C + AL(i, k - 1).C + AL(i, k + 1).C - 4 * AL(i, k).C) * dt * DC / h2;
                    R->O = (AL(i + 1, k).O + AL(i - 1, k).O + AL(i, k - 1).O + AL(i, k + 1).O - 4 * AL(i, k).O) * dt * DO / h2;
                    R->A = (AL(i + 1, k).A + AL(i - 1, k).A + AL(i, k - 1).A + AL(i, k + 1).A - 4 * AL(i, k).A) * dt * DA / h2;
                }
            }
        }
}
/* NestSolAgaElementwise, Multigrid.cpp:724-737 */
static void nest_level(orc_state* s, int l)
{
    const int X = s->P.box_x, ZA = s->P.box_z_agar;
    int d = 1 << l, d0 = 1 << s->P.max_levels_mg;
    const int lp = l - 1;
    if (l >= s->P.max_levels_mg) return;
    int nx = mg_nx(s, l), nz = mg_nz(s, l), nxp = imin(X, X * d0 / d), nzp = imin(ZA, ZA * d0 / d);
    for (int i = 0; i < nx + 1; i++)
        for (int k = 0; k < nz + 1; k++) {
            int ip = 2 * i - nx + nxp / 2, kp = 2 * k;
            if (ip > 0 && ip < nxp && kp < nzp) AG(l, i, k) = (aga_t){AP(ip, kp).C, AG(l, i, k).W, AP(ip, kp).O, AP(ip, kp).A};
        }
}
#undef EP
#undef RP
#undef AP
#undef AL
/* resetZero, Multigrid.cpp:47-82 */
static void reset_zero(orc_state* s)
{
    for (int l = 0; l < s->mg_levels; l++) {
        int nx = mg_nx(s, l), nz = mg_nz(s, l);
        for (int i = 0; i <= nx; i++) for (int k = 0; k <= nz; k++) {
            aga_t* e = &ER(l, i, k); e->C = 0; e->O = 0; e->A = 0;
            if (l > 0) { aga_t* r = &RS(l, i, k); r->C = 0; r->O = 0; r->A = 0; }
        }
    }
}
/* Vcycle, Multigrid.cpp:843-862 */
static void vcycle(orc_state* s, int mu1, int mu2)
{
    int L = s->mg_levels;
    for (int l = 0; l < L - 1; l++) { for (int j = 0; j < mu1; j++) relax_level(s, l); restrict_level(s, l + 1); }
    for (int j = 0; j < mu2; j++) relax_level(s, L - 1);
    for (int l = L - 2; l >= 0; l--) { interpolate_level(s, l); for (int j = 0; j < mu1; j++) relax_level(s, l); }
}
/* copyToMG, Multigrid.cpp:891-907 */
static void copy_to_mg(orc_state* s, aga_t** cw)
{
    const int X = s->P.box_x, ZA = s->P.box_z_agar, A_ = s->P.max_levels_mg;
    for (int i = 1; i <= X - 1; i++)
        if (ins0(s, i) > 0) { AG(0, i, 0).C = cw[0][i].C; AG(0, i, 0).O = cw[0][i].O; AG(0, i, 0).A = cw[0][i].A; }
    for (int k = 0; k <= ZA; k++) {
        AG(A_ - 1, X, k).C = AG(A_ - 1, 0, k).C; AG(A_ - 1, X, k).O = AG(A_ - 1, 0, k).O; AG(A_ - 1, X, k).A = AG(A_ - 1, 0, k).A;
    }
}
/* copyFromMG, Multigrid.cpp:958-981 */
static void copy_from_mg(orc_state* s, aga_t** ca, aga_t** cw, aga_t** pa, aga_t** pw)
{
    const int X = s->P.box_x, ZA = s->P.box_z_agar;
    for (int l = 0; l < s->P.max_levels_mg; l++)
        for (int i = 0; i <= X - 1; i++) {
            const aga_t* a = &AG(l, i, 0);
            cw[l][i].C = a->C; cw[l][i].O = a->O; cw[l][i].A = a->A;
            pw[l][i].C = a->C; pw[l][i].O = a->O; pw[l][i].A = a->A;
            for (int k = 0; k <= ZA - 1; k++) {
                const aga_t* b = &AG(l, i, k + 1);
                aga_t* c = &ca[l][(long)i * ZA + k];
                aga_t* p = &pa[l][(long)i * ZA + k];
                c->C = b->C; c->O = b->O; c->A = b->A;
                p->C = b->C; p->O = b->O; p->A = b->A;
            }
        }
}
/* solve with `vcycles` V-cycles: Multigrid.cpp:864-889, setup :818-825,
 * reset :827-841 */
static void mg_solve(orc_state* s, int vcycles, aga_t** ca, aga_t** cw, aga_t** pa, aga_t** pw)
{
    const int A_ = s->P.max_levels_mg;
    copy_to_mg(s, cw);
    reset_zero(s);
    for (int l = 0; l <= A_ - 1; l++) update_sol_level(s, l);
    for (int l = 0; l <= A_ - 1; l++) update_res_level(s, l);
    for (int i = 0; i < vcycles; i++) vcycle(s, s->P.mg_mu1, s->P.mg_mu2);
    for (int l = 0; l <= A_ - 1; l++) update_sol_level(s, l);
    for (int l = 0; l < A_ - 1; l++) rewrite_bdry(s, l);
    for (int l = 0; l <= A_ - 1; l++) update_res_level(s, l);
    reset_zero(s);
    for (int l = 1; l <= A_; l++) nest_level(s, l);
    copy_from_mg(s, ca, cw, pa, pw);
}
void orc_mg_solve(orc_state* s, int vcycles, double dt)
{
    s->mg_dt = dt;
    mg_solve(s, vcycles, s->agar, s->wal, s->oagar, s->owal);
}

/* UpdateEnvArrayMG_OxygenAcetate, Multigrid.cpp:984-1125 */
void orc_nutrient_update(orc_state* s, int n)
{
    double dtm = s->P.mg_dt;
    if (n <= 0) n = (s->P.solves_per_update > 0) ? s->P.solves_per_update : (int)(3600 * s->P.update_time * 740 / dtm);
    env_t *cur = s->env, *prev = s->oenv;
    aga_t **ca = s->agar, **pa = s->oagar, **cw = s->wal, **pw = s->owal;
    int count = 0;
    s->mg_dt = dtm;
    for (int i = 0; i < n; i++) {
        mg_solve(s, s->P.mg_vcycles, ca, cw, pa, pw);
        sweeps(s, s->P.sweeps_per_solve, &cur, &prev, &ca, &pa, &cw, &pw, &count);
    }
}
void orc_colony_sweeps(orc_state* s, int nsweeps, int count0)
{
    env_t *cur = s->env, *prev = s->oenv;
    aga_t **ca = s->agar, **pa = s->oagar, **cw = s->wal, **pw = s->owal;
    int count = count0;
    sweeps(s, nsweeps, &cur, &prev, &ca, &pa, &cw, &pw, &count);
}

/* mean_stress, Compute.cpp:18-117, for every cell in id order (the output
 * step, Simulation.cpp:320-326); returns the rand() draws made. */
long long orc_mean_stress(orc_state* s, double* stress, double* fnet)
{
    long long r0 = s->rand_calls;
    for (int i = 0; i < s->N; i++) {
        const bcg_cell* c = &s->oldc[i];
        double V = c->length * PI * c->radius * c->radius + 4.0 / 3.0 * PI * c->radius * c->radius * c->radius;
        int xi, yi, zi;
        get_address(s, avg(c), &xi, &yi, &zi);
        const int* nb = nbr_row(s, i);
        double sxx = 0, syy = 0, szz = 0;
        V3 Fn = v3(0, 0, 0), CM = avg(c), F, r, F2, r2, df, sf;
        double d;
        for (int k = 1; k < nb[0] + 1; k++) {
            F_cc(s, c, &s->oldc[nb[k]], &F, &r, &d);
            Fn = vsum(Fn, F);
            r = vdiff(r, CM);
            sxx -= F.x * r.x; syy -= F.y * r.y; szz -= F.z * r.z;
        }
        if (dmin(c->q.z, c->p.z) < 1.2 * c->radius) {
            double wall_y = s->wall[xi * s->P.box_y + yi];
            df = v3(0, 0, 0); sf = v3(0, 0, 0);
            F_cw(s, c, wall_y, &F, &F2, &r, &r2, &df, &sf);
            Fn = vsum(Fn, F); r = vdiff(r, CM);
            sxx -= F.x * r.x; syy -= F.y * r.y; szz -= F.z * r.z;
            Fn = vsum(Fn, F2); r2 = vdiff(r2, CM);
            sxx -= F2.x * r2.x; syy -= F2.y * r2.y; szz -= F2.z * r2.z;
        }
        V3 T;
        F_surf(s, c, &F, &T);
        Fn = vsum(Fn, F);
        r = vdiff(c->p, CM); r.z += c->radius;
        r2 = vdiff(c->q, CM); r2.z += c->radius;
        sxx -= F.x * r.x * 0.5 - F.x * r2.x * 0.5;
        syy -= F.y * r.y * 0.5 - F.y * r2.y * 0.5;
        szz -= F.z * r.z * 0.5 - F.z * r2.z * 0.5;
        sxx /= V; syy /= V; szz /= V;
        double rr, tt, Lcm = sqrt(CM.x * CM.x + CM.y * CM.y);
        if (Lcm > DBL_EPSILON) { V3 uv = vscale(CM, 1.0 / Lcm); rr = sxx * uv.x + syy * uv.y; tt = -sxx * uv.y + syy * uv.x; }
        else { rr = (sxx + syy); tt = 0.0; }
        stress[5 * i] = sxx; stress[5 * i + 1] = syy; stress[5 * i + 2] = szz; stress[5 * i + 3] = rr; stress[5 * i + 4] = tt;
        if (fnet) { fnet[3 * i] = Fn.x; fnet[3 * i + 1] = Fn.y; fnet[3 * i + 2] = Fn.z; }
    }
    return s->rand_calls - r0;
}

/* One iteration of the while loop, Simulation.cpp:256-430, without output. */
int orc_loop_step(orc_state* s, int* lineage)
{
    const bcg_params* P = &s->P;
    if (s->update_flag) {
        s->update_flag = 0;
        orc_update_density(s);
        orc_nutrient_update(s, 0);
        orc_rebuild_neighbours(s);
    }
    if (s->hd_update_flag) {
        s->hd_update_flag = 0;
        orc_update_height(s);
    }
    orc_move_grow(s, s->dt, 0, 0);
    int done = orc_divide(s, s->t, lineage);
    s->t += s->dt;
    int out = (s->next_out <= 0);
    s->next_out = (out ? P->output_time : s->next_out) - s->dt;
    s->update_flag = (s->next_update <= 0);
    s->next_update = (s->update_flag ? P->update_time : s->next_update) - s->dt;
    s->hd_update_flag = (s->hd_next_update <= 0);
    s->hd_next_update = (s->hd_update_flag ? s->hd_update : s->hd_next_update) - s->dt;
    return done;
}

/* field access with the ids of bcg_field_id (x-major, z fastest) */
long orc_field(orc_state* s, int field, int level, double* buf, long n, int write)
{
    const bcg_params* P = &s->P;
    const long X = P->box_x, Z = P->box_z, XH = P->box_x * P->refinement_grid_height, ZA = P->box_z_agar;
    long cnt = 0;
    double* arr = 0;
#define ACC(len, lval) do { cnt = (len); if (buf && n >= cnt) for (long i = 0; i < cnt; i++) { if (write) lval = buf[i]; else buf[i] = lval; } } while (0)
    switch (field) {
    case BCG_F_HEIGHT: arr = s->height; cnt = XH; break;
    case BCG_F_NORMAL_X: arr = s->normal_x; cnt = XH; break;
    case BCG_F_NORMAL_Z: arr = s->normal_z; cnt = XH; break;
    case BCG_F_WALL: arr = s->wall; cnt = X; break;
    case BCG_F_DENSITY_SHIFT: arr = s->ds; cnt = X * Z; break;
    case BCG_F_WALL_DENSITY_SHIFT: arr = s->wds; cnt = X; break;
    case BCG_F_INSIDE: arr = s->inside; cnt = X * Z; break;
    case BCG_F_DENSITY: arr = s->dens; cnt = X * Z; break;
    case BCG_F_ROUGH_DENSITY: arr = s->rd; cnt = X * Z; break;
    case BCG_F_ENV_CARBON: ACC(X * Z, s->env[i].Carbon); return cnt;
    case BCG_F_ENV_WASTE: ACC(X * Z, s->env[i].Waste); return cnt;
    case BCG_F_ENV_OXYGEN: ACC(X * Z, s->env[i].Oxygen); return cnt;
    case BCG_F_ENV_ACETATE: ACC(X * Z, s->env[i].Acetate); return cnt;
    case BCG_F_ENV_GROWTH1: ACC(X * Z, s->env[i].GrowthRate1); return cnt;
    case BCG_F_ENV_GROWTH2: ACC(X * Z, s->env[i].GrowthRate2); return cnt;
    case BCG_F_ENV_PH: ACC(X * Z, s->env[i].pH); return cnt;
    case BCG_F_ENV_HYDROX: ACC(X * Z, s->env[i].Hydrox); return cnt;
    case BCG_F_ENV_ACETIC: ACC(X * Z, s->env[i].Acetic); return cnt;
    case BCG_F_ENV_BUFFER: ACC(X * Z, s->env[i].Buffer); return cnt;
    case BCG_F_ENV_GR_CAR_AER: ACC(X * Z, s->env[i].GrCarAer); return cnt;
    case BCG_F_ENV_GR_CAR_ANA: ACC(X * Z, s->env[i].GrCarAna); return cnt;
    case BCG_F_ENV_GR_ACE_AER: ACC(X * Z, s->env[i].GrAceAer); return cnt;
    case BCG_F_ENV_Q_CAR_MNT: ACC(X * Z, s->env[i].qCarmnt); return cnt;
    case BCG_F_ENV_Q_ACE_MNT: ACC(X * Z, s->env[i].qAcemnt); return cnt;
    case BCG_F_ENV_P_ACE_MNT: ACC(X * Z, s->env[i].pAcemnt); return cnt;
    case BCG_F_ENV_Q_OXY_MNT: ACC(X * Z, s->env[i].qOxymnt); return cnt;
    case BCG_F_OLDENV_CARBON: ACC(X * Z, s->oenv[i].Carbon); return cnt;
    case BCG_F_OLDENV_WASTE: ACC(X * Z, s->oenv[i].Waste); return cnt;
    case BCG_F_OLDENV_OXYGEN: ACC(X * Z, s->oenv[i].Oxygen); return cnt;
    case BCG_F_OLDENV_ACETATE: ACC(X * Z, s->oenv[i].Acetate); return cnt;
    default: break;
    }
    if (arr) { ACC(cnt, arr[i]); return cnt; }
    if (field >= BCG_F_WALLF_CARBON && field <= BCG_F_AGARF_ACETATE) {
        if (level < 0 || level >= P->max_levels_mg) return -1;
        switch (field) {
        case BCG_F_WALLF_CARBON: ACC(X, s->wal[level][i].C); break;
        case BCG_F_WALLF_WASTE: ACC(X, s->wal[level][i].W); break;
        case BCG_F_WALLF_OXYGEN: ACC(X, s->wal[level][i].O); break;
        case BCG_F_WALLF_ACETATE: ACC(X, s->wal[level][i].A); break;
        case BCG_F_OLDWALLF_CARBON: ACC(X, s->owal[level][i].C); break;
        case BCG_F_OLDWALLF_WASTE: ACC(X, s->owal[level][i].W); break;
        case BCG_F_OLDWALLF_OXYGEN: ACC(X, s->owal[level][i].O); break;
        case BCG_F_OLDWALLF_ACETATE: ACC(X, s->owal[level][i].A); break;
        case BCG_F_AGARF_CARBON: ACC(X * ZA, s->agar[level][i].C); break;
        case BCG_F_AGARF_OXYGEN: ACC(X * ZA, s->agar[level][i].O); break;
        case BCG_F_AGARF_ACETATE: ACC(X * ZA, s->agar[level][i].A); break;
        }
        return cnt;
    }
    if (field >= BCG_F_MG_SOL_CARBON && field <= BCG_F_MG_ERR_ACETATE) {
        if (level < 0 || level >= s->mg_levels) return -1;
        long m = (long)(mg_nx(s, level) + 1) * (mg_nz(s, level) + 1);
        aga_t* a = (field <= BCG_F_MG_SOL_ACETATE) ? s->mgA[level] : (field <= BCG_F_MG_RES_ACETATE) ? s->mgR[level] : s->mgE[level];
        int sp = (field - BCG_F_MG_SOL_CARBON) % 3;
        if (sp == 0) ACC(m, a[i].C); else if (sp == 1) ACC(m, a[i].O); else ACC(m, a[i].A);
        return cnt;
    }
    return -1;
#undef ACC
}

/* ================================================ legacy agar solver ===== */
/* The explicit agar solver the reference carries but no longer calls
 * (Simulation.cpp:215-216, 283-284 are commented out):
 * UpdateEnvArray_OxygenAcetate (Nutrients.cpp:45-197) -- pseudo-time Jacobi
 * iterations over the colony, the wall rows and every composite agar level
 * until a convergence count reaches zero -- and
 * nutrientDepletionAgar_OxygenAcetate (Nutrients.cpp:857-1074) -- explicit
 * diffusion with the colony's depletion on the coarsest level, then
 * interpolation back to the finer levels.
 *
 * Points the reference leaves undefined: on levels > 0 the agar points with
 * BoxX/4 <= x < 3 BoxX/4 and z < BoxZAgar/2 (the part a finer level covers)
 * take second differences that are never initialised (Nutrients.cpp:
 * 670-697, 728-747).  No other point reads them.  Here they are not
 * updated (they keep their value, and so add nothing to the convergence
 * count). */
#define AIX(x, z) ((long)(x) * P->box_z_agar + (z))
static int legacy_covered(const bcg_params* P, int level, int x, int z)
{
    return level > 0 && x >= P->box_x / 4 && x < 3 * P->box_x / 4 && z <= P->box_z_agar / 2 - 1;
}

/* UpdateAgarMultigrid_OxygenAcetate (Nutrients.cpp:661-803), NutrientGSI = 0:
 * one agar point of `level` from the previous agar levels `pa` and the
 * current wall row of the level */
static void legacy_agar_point(orc_state* s, aga_t** ca, aga_t** pa, aga_t** cw, int level, int x, int z)
{
    const bcg_params* P = &s->P;
    const int X = P->box_x, ZA = P->box_z_agar, LM = P->max_levels_mg;
    if (legacy_covered(P, level, x, z)) return;
    const aga_t* p = pa[level];
    const aga_t c0 = p[AIX(x, z)];
    const double h2l = P->box_length * P->box_length * pow(4.0, level);
    aga_t up = {0, 0, 0, 0}, dn = {0, 0, 0, 0};
    double Cxx, Czz, Wxx, Wzz, Axx, Azz, Oxx, Ozz;
    /* z direction */
    if (z == 0) {
        up = p[AIX(x, z + 1)]; dn = cw[level][x];
        Wzz = (up.W + dn.W - 2.0 * c0.W) / h2l; Czz = (up.C + dn.C - 2.0 * c0.C) / h2l;
        Azz = (up.A + dn.A - 2.0 * c0.A) / h2l; Ozz = (up.O + dn.O - 2.0 * c0.O) / h2l;
    } else if (level > 0 && x >= X / 4 && x < 3 * X / 4 && z <= ZA / 2) {
        /* z == ZA/2 here (the rows below are covered) */
        up = p[AIX(x, z + 1)]; dn = pa[level - 1][AIX(x * 2 - X / 2, ZA - 1)];
        Wzz = (up.W + dn.W - 2.0 * c0.W) / h2l; Czz = (up.C + dn.C - 2.0 * c0.C) / h2l;
        Azz = (up.A + dn.A - 2.0 * c0.A) / h2l; Ozz = (up.O + dn.O - 2.0 * c0.O) / h2l;
    } else if (level < LM - 1 && z == ZA - 1) {
        const int lx = x % 2;
        const aga_t u2 = p[AIX(x, z - 2)];
        const aga_t q1 = pa[level + 1][AIX(x / 2 + X / 4, ZA / 2)];
        const aga_t q2 = pa[level + 1][AIX((x / 2 + X / 4 + 1) % X, ZA / 2)];
        Wzz = (u2.W + 1.0 / (lx + 1) * q1.W + lx * 1.0 / (lx + 1) * q2.W - 2.0 * c0.W) / 4 / h2l;
        Czz = (u2.C + 1.0 / (lx + 1) * q1.C + lx * 1.0 / (lx + 1) * q2.C - 2.0 * c0.C) / 4 / h2l;
        Azz = (u2.A + 1.0 / (lx + 1) * q1.A + lx * 1.0 / (lx + 1) * q2.A - 2.0 * c0.A) / 4 / h2l;
        Ozz = (u2.O + 1.0 / (lx + 1) * q1.O + lx * 1.0 / (lx + 1) * q2.O - 2.0 * c0.O) / 4 / h2l;
    } else if (level == LM - 1 && z == ZA - 1) {
        const aga_t u1 = p[AIX(x, z - 1)];
        Wzz = 2.0 * (u1.W - c0.W) / h2l; Czz = 2.0 * (u1.C - c0.C) / h2l;
        Azz = 2.0 * (u1.A - c0.A) / h2l; Ozz = 2.0 * (u1.O - c0.O) / h2l;
    } else {
        up = p[AIX(x, z + 1)]; dn = p[AIX(x, z - 1)];
        Wzz = (up.W + dn.W - 2.0 * c0.W) / h2l; Czz = (up.C + dn.C - 2.0 * c0.C) / h2l;
        Azz = (up.A + dn.A - 2.0 * c0.A) / h2l; Ozz = (up.O + dn.O - 2.0 * c0.O) / h2l;
    }
    /* x direction */
    if (level > 0 && x >= X / 4 - 1 && x <= X * 3 / 4 && z <= ZA / 2 - 1) {
        /* x == X/4 - 1 or x == 3X/4 here (the columns between are covered) */
        const int lo = (x == X / 4 - 1);
        const aga_t s1 = p[AIX(lo ? x - 1 : x + 1, z)];
        const aga_t q = pa[level - 1][AIX(lo ? 0 : X - 2, z * 2 + 1)];
        Wxx = (s1.W + q.W - 2 * c0.W) / h2l; Cxx = (s1.C + q.C - 2 * c0.C) / h2l;
        Axx = (s1.A + q.A - 2 * c0.A) / h2l; Oxx = (s1.O + q.O - 2 * c0.O) / h2l;
    } else if (level < LM - 1 && (x == 0 || x == X - 1)) {
        const int lz = (z + 1) % 2;
        const int zq = (z - 1) / 2;
        const int xq = (x == 0) ? X / 4 - 1 : X * 3 / 4;
        const aga_t s1 = p[AIX(x == 0 ? x + 2 : x - 1, z)];
        const aga_t q1 = pa[level + 1][AIX(xq, zq)], q2 = pa[level + 1][AIX(xq, (zq + 1) % ZA)];
        Wxx = s1.W + 1.0 / (lz + 1) * q1.W + lz * 1.0 / (lz + 1) * q2.W - 2 * c0.W;
        Cxx = s1.C + 1.0 / (lz + 1) * q1.C + lz * 1.0 / (lz + 1) * q2.C - 2 * c0.C;
        Axx = s1.A + 1.0 / (lz + 1) * q1.A + lz * 1.0 / (lz + 1) * q2.A - 2 * c0.A;
        Oxx = s1.O + 1.0 / (lz + 1) * q1.O + lz * 1.0 / (lz + 1) * q2.O - 2 * c0.O;
        if (x == 0) { Wxx = Wxx / 4 / h2l; Cxx = Cxx / 4 / h2l; Axx = Axx / 4 / h2l; Oxx = Oxx / 4 / h2l; }
        else { Wxx = Wxx / h2l; Cxx = Cxx / h2l; Axx = Axx / h2l; Oxx = Oxx / h2l; }
    } else if (level == LM - 1 && (x == 0 || x == X - 1)) {
        const aga_t s1 = p[AIX(x == 0 ? x + 1 : x - 1, z)];
        Wxx = (s1.W - 1 * c0.W) / h2l; Cxx = (s1.C - 1.0 * c0.C) / h2l; Axx = (s1.A - 1.0 * c0.A) / h2l;
        Oxx = (x == 0) ? (s1.O + P->max_o2 - 2 * c0.O) / h2l : (P->max_o2 + s1.O - 2 * c0.O) / h2l;
    } else {
        const aga_t xm = p[AIX(x - 1, z)], xp = p[AIX(x + 1, z)];
        Wxx = (xm.W + xp.W - 2 * c0.W) / h2l; Cxx = (xm.C + xp.C - 2 * c0.C) / h2l;
        Axx = (xm.A + xp.A - 2 * c0.A) / h2l; Oxx = (xm.O + xp.O - 2 * c0.O) / h2l;
    }
    aga_t* o = &ca[level][AIX(x, z)];
    double Cnew = c0.C + P->diff_agar_carbon * (Cxx + Czz) * P->cdt;
    double Onew = c0.O + P->diff_agar_o2 * (Oxx + Ozz) * P->cdt;
    o->C = dmax(0.0, dmin(Cnew, P->max_carbon));
    o->O = dmax(0.0, dmin(Onew, P->max_o2));
    double CAcenew = c0.A + P->diff_agar_ace * (Axx + Azz) * P->cdt;
    o->A = dmax(0.0, CAcenew);
    double Wnew = c0.W + P->diff_agar * (Wxx + Wzz) * P->cdt;
    o->W = dmax(0.0, Wnew);
}

/* the per-point test of Nutrients.cpp:98-101 (carbon, acetate, oxygen) */
static int legacy_moved(double cur, double prev, double crit)
{
    return fabs(cur - prev) > crit * dmax(0.1, fabs(cur));
}

/* UpdateEnvArray_OxygenAcetate, Nutrients.cpp:45-197, in the 1-thread
 * order.  Iterations stop after iteration `count` when count > min_iter
 * and no point moved by more than conv_crit, or at max_iter.  Returns the
 * iterations run (NutrientGSI = 0). */
int orc_legacy_env_update(orc_state* s, int min_iter, int max_iter, double conv_crit)
{
    const bcg_params* P = &s->P;
    const int X = P->box_x, ZA = P->box_z_agar, LM = P->max_levels_mg, maxH = s->maxz;
    env_t *cur = s->env, *prev = s->oenv;
    aga_t **ca = s->agar, **pa = s->oagar, **cw = s->wal, **pw = s->owal;
    int count = 0, nbk = 1;
    while (count < max_iter && nbk) {
        long conv = 0;
        int zmin, zmax, dir;
        if (count % 2 == 0) { zmin = -ZA; zmax = maxH + 1; dir = 1; }
        else { zmin = -maxH - 1; zmax = ZA; dir = -1; }
        for (int zi = zmin; zi <= zmax; zi++) {
            if (zi * dir > 0) {
                const int z = zi * dir - 1;
                for (int x = s->minx; x <= s->maxx; x++) {
                    const long id = IX3(x, z);
                    const env_t pv = prev[id];
                    if (s->ds[id] > DBL_EPSILON) colony_point(s, cur, prev, pw[0], x, z);
                    conv += legacy_moved(cur[id].Carbon, pv.Carbon, conv_crit);
                    conv += legacy_moved(cur[id].Acetate, pv.Acetate, conv_crit);
                    conv += legacy_moved(cur[id].Oxygen, pv.Oxygen, conv_crit);
                }
            } else if (zi == 0) {
                for (int level = 0; level < LM; level++)
                    for (int x = 0; x < X; x++) {
                        const aga_t pv = pw[level][x];
                        wall_point(s, cur, pa, cw, pw, level, x);
                        conv += legacy_moved(cw[level][x].C, pv.C, conv_crit);
                        conv += legacy_moved(cw[level][x].O, pv.O, conv_crit);
                        conv += legacy_moved(cw[level][x].A, pv.A, conv_crit);
                    }
            } else {
                const int z = -(zi * dir + 1);
                for (int level = 0; level < LM; level++)
                    for (int x = 0; x < X; x++) {
                        const aga_t pv = pa[level][AIX(x, z)];
                        legacy_agar_point(s, ca, pa, cw, level, x, z);
                        const aga_t* c = &ca[level][AIX(x, z)];
                        conv += legacy_moved(c->C, pv.C, conv_crit);
                        conv += legacy_moved(c->O, pv.O, conv_crit);
                        conv += legacy_moved(c->A, pv.A, conv_crit);
                    }
            }
        }
        env_t* t1 = prev; prev = cur; cur = t1;
        aga_t** t2 = pa; pa = ca; ca = t2;
        aga_t** t3 = pw; pw = cw; cw = t3;
        if (count > min_iter && conv == 0) nbk = 0;
        count++;
    }
    /* the swaps were of local pointers, as in the reference: the arrays
     * keep their roles, and iteration k wrote Environment / FieldAgar /
     * FieldWall when k is even, the old ones when k is odd */
    return count;
}

static int ipow_i(int b, int e) { int r = 1; while (e-- > 0) r *= b; return r; }

/* nutrientDepletionAgar_OxygenAcetate, Nutrients.cpp:857-896, with
 * restrictionAgar (:898-927), UpdateDepletionAgar (:997-1072) and
 * interpolation (:929-995).  Returns the explicit steps run. */
int orc_legacy_depletion(orc_state* s)
{
    const bcg_params* P = &s->P;
    const int X = P->box_x, ZA = P->box_z_agar, LM = P->max_levels_mg;
    aga_t **Aga = s->agar, **prevAga = s->oagar, **Wall = s->wal, **prevWall = s->owal;
    const int level = LM - 1;
    const double h2 = P->box_length * P->box_length * ipow_i(4, level);
    const double dtd = dmin(P->diff_agar_ace, P->diff_agar_carbon) / 10 * h2;
    const int n = (int)(3600 * P->update_time * 740 / dtd);
    /* restrictionAgar: the coarsest level takes each point from the finest
     * level covering it */
    for (int zi = 0; zi < ZA; zi++)
        for (int xi = 0; xi < X; xi++) {
            int l = (int)ceil(log((1 + zi) * ipow_i(2, LM - 1) * 1.0 / ZA) / log(2));
            if (l < 0) l = 0;
            int lx = 0;
            if (xi < X / 2) lx = (int)ceil(log(1 - xi * 2.0 / X) / log(2) + LM - 1);
            else if (xi > X / 2) lx = (int)floor(log(xi * 2.0 / X - 1) / log(2) + LM - 1) + 1;
            if (lx > l) l = lx;
            const int x2 = (xi - X / 2) * ipow_i(2, LM - 1 - l) + X / 2;
            const int z2 = (zi + 1) * ipow_i(2, LM - 1 - l) - 1;
            if (l < LM - 1) {
                Aga[LM - 1][AIX(xi, zi)].C = Aga[l][AIX(x2, z2)].C;
                Aga[LM - 1][AIX(xi, zi)].A = Aga[l][AIX(x2, z2)].A;
                prevAga[LM - 1][AIX(xi, zi)].C = prevAga[l][AIX(x2, z2)].C;
                prevAga[LM - 1][AIX(xi, zi)].A = prevAga[l][AIX(x2, z2)].A;
            }
        }
    aga_t* cur = Aga[level];
    aga_t* prv = prevAga[level];
    const double h2l = P->box_length * P->box_length * pow(4.0, level);
    int count = 0;
    while (count <= n) {
        for (int z = 0; z < ZA; z++)
            for (int x = 0; x < X; x++) {
                const aga_t c0 = prv[AIX(x, z)];
                double Cxx, Axx, Czz, Azz;
                if (x == 0) {
                    Cxx = (2 * prv[AIX(x + 1, z)].C - 2 * c0.C) / h2l;
                    Axx = (2 * prv[AIX(x + 1, z)].A - 2 * c0.A) / h2l;
                } else if (x == X - 1) {
                    Cxx = (prv[AIX(x - 1, z)].C - c0.C) / h2l;
                    Axx = (prv[AIX(x - 1, z)].A - c0.A) / h2l;
                } else {
                    Cxx = (prv[AIX(x + 1, z)].C + prv[AIX(x - 1, z)].C - 2 * c0.C) / h2l;
                    Axx = (prv[AIX(x + 1, z)].A + prv[AIX(x - 1, z)].A - 2 * c0.A) / h2l;
                }
                if (z == 0) {
                    int lx = 0;
                    if (x < X / 2) lx = (int)ceil(log(1 - x * 2.0 / X) / log(2) + LM - 1);
                    else if (x > X / 2) lx = (int)floor(log(x * 2.0 / X - 1) / log(2) + LM - 1) + 1;
                    if (lx < 0) lx = 0;
                    const int xw = (x - X / 2) * ipow_i(2, LM - 1 - lx) + X / 2;
                    if (lx == 0 && s->inside[IX3(xw, 0)] > 0.5) {
                        /* the depletion flux is computed and never used
                         * (Nutrients.cpp:1042-1047): no z flux here */
                        Czz = 0; Azz = 0;
                    } else {
                        Czz = (prv[AIX(x, z + 1)].C + 0.0 * pow(2.0, level) - c0.C) / h2l;
                        Azz = (prv[AIX(x, z + 1)].A + 0.0 * pow(2.0, level) - c0.A) / h2l;
                    }
                } else if (z == ZA - 1) {
                    Czz = (2 * prv[AIX(x, z - 1)].C - 2 * c0.C) / h2l;
                    Azz = (2 * prv[AIX(x, z - 1)].A - 2 * c0.A) / h2l;
                } else {
                    Czz = (prv[AIX(x, z + 1)].C + prv[AIX(x, z - 1)].C - 2 * c0.C) / h2l;
                    Azz = (prv[AIX(x, z + 1)].A + prv[AIX(x, z - 1)].A - 2 * c0.A) / h2l;
                }
                cur[AIX(x, z)].C += dtd * P->diff_agar_carbon * (Cxx + Czz);
                cur[AIX(x, z)].A += dtd * P->diff_agar_ace * (Axx + Azz);
            }
        for (long i = 0; i < (long)X * ZA; i++) { prv[i].C = cur[i].C; prv[i].A = cur[i].A; }
        count++;
    }
    /* interpolation: every finer level from the next coarser one */
    for (int l = LM - 1; l > 0; l--)
        for (int zi = 0; zi < ZA; zi++)
            for (int xi = 0; xi < X; xi++) {
                double a1 = 0, a2 = 0, c1 = 0, c2 = 0;
                if (zi == 0) {
                    for (int i1 = 0; i1 < 2; i1++) {
                        const long q = AIX((xi + i1) / 2 + X / 4, 0);
                        c1 += Aga[l][q].C / 4; c2 += prevAga[l][q].C / 4;
                        a1 += Aga[l][q].A / 4; a2 += prevAga[l][q].A / 4;
                    }
                    int lx = 0;
                    if (xi < X / 2) lx = (int)ceil(log(1 - xi * 2.0 / X) / log(2) + l);
                    else if (xi > X / 2) lx = (int)floor(log(xi * 2.0 / X - 1) / log(2) + l) + 1;
                    if (lx < 0) lx = 0;
                    const int xw = (xi - X / 2) * ipow_i(2, l - lx) + X / 2;
                    c1 += Wall[lx][xw].C / 2; c2 += prevWall[lx][xw].C / 2;
                    a1 += Wall[lx][xw].A / 2; a2 += prevWall[lx][xw].A / 2;
                } else {
                    for (int i1 = 0; i1 < 2; i1++)
                        for (int i2 = 0; i2 < 2; i2++) {
                            const long q = AIX((xi + i1) / 2 + X / 4, (zi - i2) / 2);
                            c1 += Aga[l][q].C / 4; c2 += prevAga[l][q].C / 4;
                            a1 += Aga[l][q].A / 4; a2 += prevAga[l][q].A / 4;
                        }
                }
                Aga[l - 1][AIX(xi, zi)].C = c1; prevAga[l - 1][AIX(xi, zi)].C = c2;
                Aga[l - 1][AIX(xi, zi)].A = a1; prevAga[l - 1][AIX(xi, zi)].A = a2;
            }
    return count;
}
#undef AIX

/* ------------------------------------------------------------------------
 * Inputs for the reference arm of the benchmark, so that it builds its
 * workload without loading the CUDA library: the parameter defaults of
 * Constants.cpp:1-112, main()'s derived sizes (CellMD3D.cpp:52-54), and the
 * seeded synthetic colony.  tests/test_oracle.py checks all three against
 * the library's bcg_params_default, bcg_params_finalize and
 * bcg_synth_colony byte for byte.
 * ---------------------------------------------------------------------- */
int orc_params_default(bcg_params* p)
{
    if (!p) return BCG_E_ARG;
    memset(p, 0, sizeof(*p));
    /* Constants.cpp:1-112 (maxO2_Agar hard-coded 0.26 at :32; C_rate =
     * 3.7e-5 * Tortuosity * 5 with Tortuosity 2, :45-49) */
    p->cell_radius = 0.34; p->l_divide = 5.75; p->k_cc = 100000.0; p->k_wc = 100000.0;
    p->viscosity = 1.0; p->gamma_t = 10000.0; p->wall_mu = 0.15; p->cell_mu = 0.15;
    p->density_threshold = 0.6; p->tension = 10.0; p->rc = 3.0;
    p->t_max = 20.0; p->dt = 0.00001; p->output_time = 100 * 0.00001; p->update_time = 100 * 0.00001;
    p->box_x = 150; p->box_y = 150; p->box_z = 50; p->box_z_agar = 30; p->max_levels_mg = 1;
    p->box_length = 2; p->filter_len = 5; p->max_o2_agar = 0.26; p->max_cells = 100000;
    p->kc_aer = 0.001; p->kc_ana = 0.001; p->kw = 0.001;
    p->c_rate = 3.7e-5 * 2.0 * 5.0; p->w_rate = p->c_rate; p->carbon_to_waste = 1.0;
    p->max_growth_rate1 = 1.0; p->max_growth_rate2 = 1.0;
    p->diff_colony = 1.0; p->diff_agar = 3.0; p->max_carbon = 0.01;
    p->cross_feeding = 1; p->cdt = 0.1; p->interface_condition = 1;
    p->refinement_grid_height = 4;
    p->ko = 1.0; p->ka = 1.0; p->ki = 1.0;
    p->q_car_aer = 1.0; p->q_car_ana = 1.0; p->q_ace_aer = 1.0; p->q_o2_car = 1.0; p->q_o2_ace = 1.0;
    p->p_ace_aer = 1.0; p->p_ace_ana = 1.0;
    p->diff_colony_carbon = 1.0; p->diff_agar_carbon = 1.0; p->diff_colony_o2 = 1.0;
    p->diff_agar_o2 = 1.0; p->diff_colony_ace = 1.0; p->diff_agar_ace = 1.0;
    p->max_o2 = 1.0; p->max_gr_car_aer = 1.0; p->max_gr_car_ana = 1.0; p->max_gr_ace_aer = 1.0;
    p->kw_ph = 1.0; p->ka_ph = 1.0; p->kb_ph = 1.0; p->cb_ph = 1.0; p->c1_ph = 1.0;
    p->q_car_aer_nt = 1.0; p->q_car_ana_nt = 1.0; p->q_ace_aer_nt = 1.0; p->q_o2_car_nt = 1.0;
    p->q_o2_ace_nt = 1.0; p->p_ace_ana_nt = 1.0;
    /* the solve schedule of Multigrid.cpp:995-1017 and Simulation.cpp:157 */
    p->mg_levels = 8; p->mg_vcycles = 3; p->mg_mu1 = 3; p->mg_mu2 = 100;
    p->sweeps_per_solve = 200; p->solves_per_update = 0; p->mg_dt = 100.0;
    return BCG_OK;
}

int orc_params_finalize(bcg_params* p)
{
    if (!p) return BCG_E_ARG;
    /* BoxLength = L_divide + 2R, maxCellsPerBox (CellMD3D.cpp:52-54) */
    p->box_length = p->l_divide + 2 * p->cell_radius;
    double bl = p->box_length;
    p->max_cells_per_box = (int)ceil(bl * bl * bl / (PI * p->cell_radius * p->cell_radius * p->l_divide * p->density_threshold / 2));
    if (p->max_neighbours <= 0) p->max_neighbours = 64;
    if (p->box_x < 8 || p->box_y < 1 || p->box_z < 3 || p->box_z_agar < 2) return BCG_E_ARG;
    if (p->max_levels_mg < 1 || p->mg_levels < p->max_levels_mg || p->mg_levels > 16) return BCG_E_ARG;
    if (p->refinement_grid_height < 1 || p->filter_len < 1 || p->max_cells < 1) return BCG_E_ARG;
    if (p->max_neighbours > 1024) return BCG_E_ARG;
    return BCG_OK;
}

/* 64-bit Mersenne twister (Matsumoto and Nishimura's MT19937-64, the
 * generator std::mt19937_64 names): state of 312 words, seeded by
 * x[i] = 6364136223846793005 (x[i-1] ^ (x[i-1] >> 62)) + i. */
typedef struct { uint64_t x[312]; int i; } mt64;
static void mt64_seed(mt64* g, uint64_t seed)
{
    g->x[0] = seed;
    for (int i = 1; i < 312; i++) g->x[i] = 6364136223846793005ULL * (g->x[i - 1] ^ (g->x[i - 1] >> 62)) + (uint64_t)i;
    g->i = 312;
}
static uint64_t mt64_next(mt64* g)
{
    if (g->i >= 312) {
        for (int k = 0; k < 312; k++) {
            uint64_t y = (g->x[k] & 0xFFFFFFFF80000000ULL) | (g->x[(k + 1) % 312] & 0x7FFFFFFFULL);
            uint64_t v = g->x[(k + 156) % 312] ^ (y >> 1);
            if (y & 1) v ^= 0xB5026F5AA96619E9ULL;
            g->x[k] = v;
        }
        g->i = 0;
    }
    uint64_t z = g->x[g->i++];
    z ^= (z >> 29) & 0x5555555555555555ULL;
    z ^= (z << 17) & 0x71D67FFFEDA60000ULL;
    z ^= (z << 37) & 0xFFF7EEE000000000ULL;
    z ^= z >> 43;
    return z;
}
static double mt64_unit(mt64* g) { return (double)(mt64_next(g) >> 11) * (1.0 / 9007199254740992.0); }

/* squared closest distance of two x-z segments (plain geometry) */
static double syn_dist2(const double* a, const double* b)
{
    double d1x = a[2] - a[0], d1z = a[3] - a[1], d2x = b[2] - b[0], d2z = b[3] - b[1];
    double rx = a[0] - b[0], rz = a[1] - b[1];
    double aa = d1x * d1x + d1z * d1z, ee = d2x * d2x + d2z * d2z, ff = d2x * rx + d2z * rz;
    double cc = d1x * rx + d1z * rz, bb = d1x * d2x + d1z * d2z;
    double den = aa * ee - bb * bb, s = 0, t;
    if (den > 1e-300) { s = (bb * ff - cc * ee) / den; s = s < 0 ? 0 : (s > 1 ? 1 : s); }
    t = (bb * s + ff) / ee;
    if (t < 0) { t = 0; s = -cc / aa; s = s < 0 ? 0 : (s > 1 ? 1 : s); }
    else if (t > 1) { t = 1; s = (bb - cc) / aa; s = s < 0 ? 0 : (s > 1 ? 1 : s); }
    double dx = (a[0] + d1x * s) - (b[0] + d2x * t), dz = (a[1] + d1z * s) - (b[1] + d2z * t);
    return dx * dx + dz * dz;
}

/* The seeded colony of the benchmark workloads: random sequential placement
 * of spherocylinders (length U(len_lo, len_hi), angle U(0, pi), centre
 * uniform in a half-ellipse dome of width x height on the agar, both poles
 * at z >= radius, segment distance >= 2 radius to every earlier cell); the
 * dome widens by 2 % after a bounded run of failed tries.  Records as
 * AddFirstCells fills them (InputOutput.cpp:319-345) with
 * Ldiv = Length + (l_divide/2)(1 - spread u).  Same draws, in the same
 * order, as the library's bcg_synth_colony. */
int orc_synth_colony(uint64_t seed, int n_target, double width, double height,
                     double radius, double len_lo, double len_hi,
                     double l_divide, double div_phase_spread,
                     bcg_cell* out, int capacity, int* n)
{
    if (!out || !n || n_target < 0 || n_target > capacity || width <= 0 || height <= 0 ||
        radius <= 0 || len_lo <= 0 || len_hi < len_lo)
        return BCG_E_ARG;
    mt64* g = (mt64*)malloc(sizeof(mt64));
    if (!g) return BCG_E_ARG;
    mt64_seed(g, seed);
    const double cs = len_hi + 2 * radius;
    double W = width, H = height;
    double gx0 = -W, gz0 = -cs;
    int gnx = (int)ceil(2 * W / cs) + 3, gnz = (int)ceil((2 * H + 2 * cs) / cs) + 3;
    int* head = (int*)malloc(sizeof(int) * (size_t)gnx * gnz);
    int* next = (int*)malloc(sizeof(int) * (size_t)(n_target > 0 ? n_target : 1));
    double* seg = (double*)malloc(sizeof(double) * 4 * (size_t)(n_target > 0 ? n_target : 1));
    double* len = (double*)malloc(sizeof(double) * (size_t)(n_target > 0 ? n_target : 1));
    int rc = BCG_OK;
    if (!head || !next || !seg || !len) { rc = BCG_E_ARG; goto done; }
    for (long q = 0; q < (long)gnx * gnz; q++) head[q] = -1;
    const double min2 = (2 * radius) * (2 * radius);
    long long fails = 0;
    int cnt = 0;
    while (cnt < n_target) {
        double L = len_lo + (len_hi - len_lo) * mt64_unit(g);
        double th = 3.141592653589793 * mt64_unit(g);
        double cx = (mt64_unit(g) - 0.5) * W;
        double cz = mt64_unit(g) * H;
        double e = 2 * cx / W;
        int ok = (e * e < 1.0) && (cz <= H * sqrt(1 - e * e));
        double sg[4];
        sg[0] = cx + 0.5 * L * cos(th); sg[1] = cz + 0.5 * L * sin(th);
        sg[2] = cx - 0.5 * L * cos(th); sg[3] = cz - 0.5 * L * sin(th);
        if (ok && (sg[1] < radius || sg[3] < radius)) ok = 0;
        int ix = (int)floor((cx - gx0) / cs), iz = (int)floor((cz - gz0) / cs);
        if (ok && !(ix >= 0 && iz >= 0 && ix < gnx && iz < gnz)) ok = 0;
        for (int dx = -1; dx <= 1 && ok; dx++)
            for (int dz = -1; dz <= 1 && ok; dz++) {
                int jx = ix + dx, jz = iz + dz;
                if (jx < 0 || jz < 0 || jx >= gnx || jz >= gnz) continue;
                for (int id = head[(long)jx * gnz + jz]; id >= 0; id = next[id])
                    if (syn_dist2(sg, seg + 4 * (size_t)id) < min2) { ok = 0; break; }
            }
        if (!ok) {
            if (++fails > 200000LL + 50LL * (long long)cnt) {
                W *= 1.02; H *= 1.02; fails = 0;
                if (2 * W / cs + 3 > gnx || (2 * H + 2 * cs) / cs + 3 > gnz) { rc = BCG_E_ARG; goto done; }
            }
            continue;
        }
        fails = 0;
        memcpy(seg + 4 * (size_t)cnt, sg, sizeof(sg));
        len[cnt] = L;
        next[cnt] = head[(long)ix * gnz + iz];
        head[(long)ix * gnz + iz] = cnt;
        cnt++;
    }
    for (int i = 0; i < n_target; i++) {
        bcg_cell* c = &out[i];
        memset(c, 0, sizeof(*c));
        c->p.x = seg[4 * i]; c->p.z = seg[4 * i + 1];
        c->q.x = seg[4 * i + 2]; c->q.z = seg[4 * i + 3];
        c->length = len[i];
        c->radius = radius;
        double u = mt64_unit(g);
        c->ldiv = len[i] + (l_divide / 2) * (1.0 - div_phase_spread * u);
        c->type = 1;
        c->ancestor = i + 1;
    }
    *n = n_target;
done:
    free(g); free(head); free(next); free(seg); free(len);
    return rc;
}
