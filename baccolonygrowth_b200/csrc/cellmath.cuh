/*
 * cellmath.cuh -- per-cell and per-pair mechanics as device functions.
 *
 * Each function follows the reference formula and its operation order
 * (citations are AgentBasedModel-BacColonyGrowth/file:line).  The library
 * is compiled with -fmad=false, so products and sums round as in the
 * reference's x86-64 build (which has no FMA); sums over neighbours use a
 * fixed lane tree instead of the reference's sequential order.
 */
#pragma once
#include "common.cuh"
#include <float.h>

struct V3 { double x, y, z; };
__device__ __forceinline__ V3 mk(double x, double y, double z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
__device__ __forceinline__ double dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross3(V3 a, V3 b) { return mk(a.y * b.z - a.z * b.y, -a.x * b.z + a.z * b.x, a.x * b.y - a.y * b.x); }
__device__ __forceinline__ V3 sub3(V3 a, V3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 add3(V3 a, V3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 scl3(V3 a, double c) { return mk(a.x * c, a.y * c, a.z * c); }
__device__ __forceinline__ double dmax_(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double dmin_(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double clamp01(double n) { return n < 0 ? 0 : (n > 1 ? 1 : n); }

/* the state of one cell as the force routines see it */
struct Cst { V3 p, q, v, w; double L, R; };

__device__ __forceinline__ Cst load_cst(const CellRec* __restrict__ r)
{
    /* one 128-byte line as eight 16-byte read-only loads */
    const double2* q = reinterpret_cast<const double2*>(r);
    double2 a0 = __ldg(q + 0), a1 = __ldg(q + 1), b0 = __ldg(q + 2), b1 = __ldg(q + 3);
    double2 c0 = __ldg(q + 4), c1 = __ldg(q + 5), d0 = __ldg(q + 6), d1 = __ldg(q + 7);
    Cst s;
    s.p = mk(a0.x, a0.y, a1.x); s.L = a1.y;
    s.q = mk(b0.x, b0.y, b1.x); s.R = b1.y;
    s.v = mk(c0.x, c0.y, c1.x); s.w = mk(d0.x, d0.y, d1.x);
    return s;
}
/* plain (coherent) load, for records written earlier in the same kernel */
__device__ __forceinline__ Cst load_cst_coh(const CellRec* r)
{
    double4 a = r->pL, b = r->qR, c = r->v, d = r->w;
    Cst s;
    s.p = mk(a.x, a.y, a.z); s.L = a.w;
    s.q = mk(b.x, b.y, b.z); s.R = b.w;
    s.v = mk(c.x, c.y, c.z); s.w = mk(d.x, d.y, d.z);
    return s;
}
__device__ __forceinline__ V3 avg_pq(V3 p, V3 q) { return scl3(add3(p, q), 0.5); }

/* min_distance, Neighbours.cpp:107-160 */
__device__ __forceinline__ double seg_distance(V3 p1, V3 q1, V3 p2, V3 q2, V3& c1, V3& c2)
{
    V3 v1 = sub3(q1, p1), v2 = sub3(q2, p2), r = sub3(p1, p2);
    double l1 = dot3(v1, v1), l2 = dot3(v2, v2), f = dot3(v2, r), c = dot3(v1, r), b = dot3(v1, v2);
    double denom = l1 * l2 - b * b, s, t;
    if (denom != 0) s = clamp01((b * f - c * l2) / denom);
    else s = 0;
    double tnom = b * s + f;
    if (tnom < 0) { t = 0; s = clamp01(-c / l1); }
    else if (tnom > l2) { t = 1; s = clamp01((b - c) / l1); }
    else t = tnom / l2;
    c1 = add3(p1, scl3(v1, s));
    c2 = add3(p2, scl3(v2, t));
    V3 cv = sub3(c1, c2);
    return sqrt(dot3(cv, cv));
}

/* reduceNeighbours test, Neighbours.cpp:74-88: keep j for cell a */
__device__ __forceinline__ bool keep_neighbour(V3 ap, V3 aq, double aL, double aR, V3 acm, V3 bp, V3 bq, double rc)
{
    V3 v = sub3(bp, acm);
    double dp = sqrt(dot3(v, v));
    v = sub3(bq, acm);
    double dq = sqrt(dot3(v, v));
    double lim = aL / 2.0 + rc * aR;
    if ((dp < lim) || (dq < lim)) {
        V3 c1, c2;
        double d = seg_distance(ap, aq, bp, bq, c1, c2);
        return d < rc * aR;
    }
    return false;
}

/* F_cc, Forces.cpp:13-84, from the closest points c1 (on a), c2 (on b)
 * and their distance d.  Returns false (F = 0) when the cells do not
 * overlap, in which case the reference's contribution is a signed zero. */
__device__ __forceinline__ bool pair_force_at(const Cst& a, V3 acm, const Cst& b, const MechParams& mp,
                                              V3 c1, V3 c2, double d, V3& F, V3& r)
{
    double sigma = a.R + b.R;
    double delta = dmax_(sigma - d, 0.0);
    if (!(delta > 0.0)) return false;
    const double gamma_n = 100.0;
    double L1 = a.L + 4.0 / 3 * a.R, M1 = L1 * a.R * a.R * BCG_PI;
    double L2 = b.L + 4.0 / 3 * b.R, M2 = L2 * b.R * b.R * BCG_PI;
    double Meff = M1 * M2 / (M1 + M2);
    V3 vn = scl3(sub3(c2, c1), 1.0 / d);
    /* delta^(3/2) as delta sqrt(delta) (the reference calls pow; the two
     * differ by rounding, and the double pow is a long instruction sequence) */
    double FE_mag = sqrt(a.R * b.R / (a.R + b.R)) * mp.k_cc * (delta * sqrt(delta));
    V3 FE = scl3(vn, -FE_mag);
    r = scl3(add3(scl3(c1, b.R), scl3(c2, a.R)), 1 / sigma);
    if (FE_mag > DBL_EPSILON) {
        V3 rcm1 = sub3(r, acm), rcm2 = sub3(r, avg_pq(b.p, b.q));
        V3 v1 = add3(a.v, cross3(a.w, rcm1)), v2 = add3(b.v, cross3(b.w, rcm2));
        V3 dv = sub3(v2, v1);
        V3 dvn = scl3(vn, dot3(dv, vn));
        V3 FDn = scl3(dvn, gamma_n * Meff * delta);
        V3 dvt = sub3(dv, dvn);
        double v_mag = sqrt(dot3(dvt, dvt));
        V3 FDt = mk(0.0, 0.0, 0.0);
        if (v_mag > 3 * DBL_EPSILON) FDt = scl3(dvt, dmin_(mp.gamma_t * Meff * sqrt(delta), mp.cell_mu * FE_mag / v_mag));
        F = add3(add3(FE, FDt), FDn);
    } else F = FE;
    return true;
}

/* F_cc with the reference's FP64 min_distance */
__device__ __forceinline__ bool pair_force(const Cst& a, V3 acm, const Cst& b, const MechParams& mp, V3& F, V3& r)
{
    V3 c1, c2;
    double d = seg_distance(a.p, a.q, b.p, b.q, c1, c2);
    return pair_force_at(a, acm, b, mp, c1, c2, d, F, r);
}

/* min_distance's search in FP32, on offsets local to a reference point
 * (the centre of cell a): the offsets are a few um, so their FP32 rounding
 * is ~1e-7 um where absolute positions (up to 1e4 um) would lose ~1e-3 um.
 * Same clamping steps as seg_distance; returns which of its branches holds
 * the minimum: 1 = t clamped to 0, 2 = t clamped to 1, 3 = t from the
 * projection with s clamped to an end, 0 = both interior (crossing or
 * nearly parallel segments). */
struct F3 { float x, y, z; };
__device__ __forceinline__ F3 f3_off(V3 a, V3 o) { F3 r; r.x = (float)(a.x - o.x); r.y = (float)(a.y - o.y); r.z = (float)(a.z - o.z); return r; }
__device__ __forceinline__ float f3_dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float clamp01f(float n) { return n < 0.f ? 0.f : (n > 1.f ? 1.f : n); }
__device__ __forceinline__ int seg_branch_f(F3 p1, F3 q1, F3 p2, F3 q2, float& s)
{
    F3 v1 = {q1.x - p1.x, q1.y - p1.y, q1.z - p1.z}, v2 = {q2.x - p2.x, q2.y - p2.y, q2.z - p2.z};
    F3 r = {p1.x - p2.x, p1.y - p2.y, p1.z - p2.z};
    float l1 = f3_dot(v1, v1), l2 = f3_dot(v2, v2), f = f3_dot(v2, r), c = f3_dot(v1, r), b = f3_dot(v1, v2);
    float denom = l1 * l2 - b * b;
    if (denom != 0.f) s = clamp01f((b * f - c * l2) / denom);
    else s = 0.f;
    float tnom = b * s + f;
    if (tnom < 0.f) return 1;
    if (tnom > l2) return 2;
    return (s == 0.f || s == 1.f) ? 3 : 0;
}

/* F_cc with min_distance's branch found in FP32 local to cell a, and the
 * branch's own formula (a projection of a pole, one division) then taken in
 * FP64 from the FP64 poles: the closest points, their distance, the
 * contact normal and the forces are FP64 values, which differ from the
 * all-FP64 search only where FP32 rounding picks another branch at a
 * branch boundary (the distance is continuous there).  Both-interior
 * minima (crossing or nearly parallel segments) take the FP64 search. */
__device__ __forceinline__ bool pair_force_f32geom(const Cst& a, V3 acm, const Cst& b, const MechParams& mp, V3& F, V3& r)
{
    float sf;
    const int br = seg_branch_f(f3_off(a.p, acm), f3_off(a.q, acm), f3_off(b.p, acm), f3_off(b.q, acm), sf);
    V3 c1, c2;
    double d;
    if (br == 0) {
        d = seg_distance(a.p, a.q, b.p, b.q, c1, c2);
    } else {
        const V3 v1 = sub3(a.q, a.p), v2 = sub3(b.q, b.p), rr = sub3(a.p, b.p);
        double s, t;
        if (br == 3) {
            s = (double)sf;
            t = clamp01((dot3(v1, v2) * s + dot3(v2, rr)) / dot3(v2, v2));
        } else {
            const double l1 = dot3(v1, v1), c = dot3(v1, rr);
            t = (br == 1) ? 0.0 : 1.0;
            s = (br == 1) ? clamp01(-c / l1) : clamp01((dot3(v1, v2) - c) / l1);
        }
        c1 = add3(a.p, scl3(v1, s));
        c2 = add3(b.p, scl3(v2, t));
        const V3 cv = sub3(c1, c2);
        d = sqrt(dot3(cv, cv));
    }
    return pair_force_at(a, acm, b, mp, c1, c2, d, F, r);
}

/* one locus of F_cw, Forces.cpp:96-152 (var_pos = 0, so the locus sits at
 * the pole's x) */
__device__ __forceinline__ V3 wall_locus(const Cst& c, V3 cm, V3 pole, double wall_z, const MechParams& mp, V3& rpos, V3& sf, V3& df)
{
    double Lm = c.L + 4.0 / 3 * c.R, M = Lm * c.R * c.R * BCG_PI;
    const double gamma_n = 100.0;
    rpos = mk(pole.x, 0.0, wall_z);
    double d = pole.z - wall_z;
    double delta = dmax_(c.R - d, 0.0);
    double FE_mag = sqrt(c.R) * mp.k_wc * (delta * sqrt(delta));
    if (FE_mag > DBL_EPSILON) {
        V3 FE = mk(0.0, 0.0, FE_mag);
        V3 rcm = sub3(rpos, cm);
        V3 v = add3(c.v, cross3(c.w, rcm));
        V3 dv = scl3(v, -1.0);
        V3 dvn = mk(0.0, 0.0, dv.z);
        V3 dvt = sub3(dv, dvn);
        double v_mag = sqrt(dot3(dvt, dvt));
        V3 FDt;
        if (v_mag > DBL_EPSILON) FDt = scl3(dvt, dmin_(mp.gamma_t * M * sqrt(delta), mp.wall_mu * FE_mag / v_mag));
        else FDt = mk(0, 0, 0);
        V3 FDn = scl3(dvn, gamma_n * M * delta);
        sf = add3(sf, scl3(dvt, mp.gamma_t * M * sqrt(delta)));
        df = add3(df, scl3(dvt, mp.wall_mu * FE_mag / v_mag));
        return add3(FE, add3(FDt, FDn));
    }
    return mk(0.0, 0.0, 0.0);
}

/* Array2D<double>::linear_interp at y = 0 with float weights (Array.h:282-288).
 * The two y+1 terms carry weight exactly 0 and are omitted. */
__device__ __forceinline__ double height_interp(const double* __restrict__ h, int x0, double dx, int xh)
{
    /* a cell outside the grid is reported by the binning; keep reads in bounds */
    x0 = x0 < 0 ? 0 : (x0 > xh - 2 ? xh - 2 : x0);
    float x = dx < 0 ? 1 + dx : dx;
    float y = 0.0f;
    return h[x0] * (1 - x) * (1 - y) + h[x0 + 1] * x * (1 - y);
}

/* F_surf_tension, Forces.cpp:209-317 */
__device__ __forceinline__ void surface_tension(const Cst& c, V3 cm, const FieldPtrs& fp, const MechParams& mp, V3& F, V3& T)
{
    const int rgh = mp.rgh;
    const double hb = mp.box_length / rgh;
    const int half = mp.box_x / 2 * rgh;
    int xa = (int)((cm.x + mp.box_x / 2 * mp.box_length) / (mp.box_length / rgh));
    int i_ht = (int)(c.p.x / hb + half);
    double dxp = c.p.x / hb - (i_ht - half + 0.5);
    i_ht = (int)ceil(dxp) + i_ht - 1;
    double height_p = height_interp(fp.height, i_ht, dxp, mp.xh);
    i_ht = (int)(c.q.x / hb + half);
    double dxq = c.q.x / hb - (i_ht - half + 0.5);
    i_ht = (int)ceil(dxq) + i_ht - 1;
    double height_q = height_interp(fp.height, i_ht, dxq, mp.xh);
    i_ht = (int)(cm.x / hb + half);
    double dxc = cm.x / hb - (i_ht - half + 0.5);
    i_ht = (int)ceil(dxc) + i_ht - 1;
    double height_cm = height_interp(fp.height, i_ht, dxc, mp.xh);
    if (height_cm > (cm.z + mp.box_length)) { F = mk(0, 0, 0); T = mk(0, 0, 0); return; }
    xa = xa < 0 ? 0 : (xa > mp.xh - 1 ? mp.xh - 1 : xa);
    V3 N = mk(fp.nx[xa], fp.ny[xa], fp.nz[xa]);
    V3 F1 = mk(0, 0, 0), F2 = mk(0, 0, 0);
    double dh = c.p.z - (height_p - mp.delta_h / N.z);
    if (!(dh < 0.0)) {
        double distance = -dh * N.z;
        double F0 = 2 * BCG_PI * mp.tension * dmin_(distance / (mp.cell_radius / 5.0), 1.0);
        F1 = scl3(N, F0);
    }
    dh = c.q.z - (height_q - mp.delta_h / N.z);
    if (!(dh < 0.0)) {
        double distance = -dh * N.z;
        double F0 = 2 * BCG_PI * mp.tension * dmin_(distance / (mp.cell_radius / 5.0), 1.0);
        F2 = scl3(N, F0);
    }
    F = add3(F1, F2);
    T = cross3(sub3(c.p, cm), F1);
    T = add3(T, cross3(sub3(c.q, cm), F2));
}

/* half kick of UpdatePositions / UpdateVelocities, Integrate.cpp:55-73,
 * 94-113 */
__device__ __forceinline__ void half_kick(double dt, V3 F, V3 T, const Cst& o, V3& vnew, V3& wnew)
{
    double R2 = o.R * o.R, L2 = o.L * o.L;
    double M = BCG_PI * R2 * (o.L + 4.0 / 3.0 * o.R);
    double Ixy = BCG_PI * R2 * (o.L * L2 / 12.0 + o.R * (8.0 * R2 / 15.0 + L2 / 3.0));
    double Iz = BCG_PI * R2 * R2 * (o.L / 2.0 + 8.0 * o.R / 15.0);
    V3 z = sub3(o.q, o.p);
    z = scl3(z, 1.0 / o.L);
    V3 vaz = scl3(z, dot3(z, o.w));
    V3 vaxy = sub3(o.w, vaz);
    V3 Tz = scl3(z, dot3(z, T));
    V3 Txy = sub3(T, Tz);
    vnew = add3(o.v, scl3(F, dt / (2.0 * M)));
    wnew = add3(add3(vaz, scl3(Tz, dt / (2.0 * Iz))), add3(vaxy, scl3(Txy, dt / (2.0 * Ixy))));
}

/* UniformGrid::GetAddress (UniformGrid.h:87-99); returns -1 outside. */
__device__ __forceinline__ int box_address(V3 pos, const MechParams& mp, int& xi, int& yi, int& zi)
{
    xi = (int)(pos.x / mp.box_length + mp.box_x / 2);
    yi = (int)(pos.y / mp.box_length + mp.box_y / 2 + 0.5);
    zi = (int)(pos.z / mp.box_length);
    if (!((xi < mp.box_x) & (yi < mp.box_y) & (zi < mp.box_z) & (xi >= 0) & (yi >= 0) & (zi >= 0))) return -1;
    return xi * (mp.box_y * mp.box_z) + yi * mp.box_z + zi;
}
