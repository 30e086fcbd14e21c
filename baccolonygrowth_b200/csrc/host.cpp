/*
 * host.cpp -- host-side pieces of the C ABI that need no GPU:
 * parameter defaults/derivation, the glibc-compatible rand() stream with
 * jump-ahead, and the seeded synthetic colony generator.
 */
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <stdint.h>
#include <random>
#include <vector>
#include <algorithm>

#include "../../include/bcg.h"

extern "C" {

/* Defaults of Constants.cpp:1-112 (the values the reference starts from
 * before ReadParameters overrides them).  maxO2_Agar is the hard-coded 0.26
 * of Constants.cpp:32; C_rate = 3.7e-5*Tortuosity*5 with Tortuosity = 2
 * (Constants.cpp:45-49). */
int bcg_params_default(bcg_params* p)
{
    if (!p) return BCG_E_ARG;
    memset(p, 0, sizeof(*p));
    p->cell_radius = 0.34; p->l_divide = 5.75; p->k_cc = 100000.0; p->k_wc = 100000.0;
    p->var_l = 0.0; p->var_angle = 0.0; p->var_pos = 0.0; p->viscosity = 1.0;
    p->wall_rough = 0.0; p->gamma_t = 10000.0; p->wall_mu = 0.15; p->cell_mu = 0.15;
    p->density_threshold = 0.6; p->tension = 10.0; p->delta_h = 0.0; p->rc = 3.0;
    p->t_max = 20.0; p->dt = 0.00001; p->output_time = 100 * 0.00001; p->t0 = 0.0;
    p->update_time = 100 * 0.00001;
    p->box_x = 150; p->box_y = 150; p->box_z = 50; p->box_z_agar = 30; p->max_levels_mg = 1;
    p->box_length = 2; p->filter_len = 5; p->max_o2_agar = 0.26;
    p->max_cells = 100000;
    p->kc_aer = 0.001; p->kc_ana = 0.001; p->kw = 0.001;
    p->c_rate = 3.7e-5 * 2.0 * 5.0; p->w_rate = p->c_rate; p->carbon_to_waste = 1.0;
    p->max_growth_rate1 = 1.0; p->max_growth_rate2 = 1.0; p->maintenance_rate = 0.0;
    p->diff_colony = 1.0; p->diff_agar = 3.0; p->max_carbon = 0.01;
    p->cross_feeding = 1; p->cdt = 0.1; p->interface_condition = 1; p->nutrient_gsi = 0;
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
    p->mg_levels = 8; p->mg_vcycles = 3; p->mg_mu1 = 3; p->mg_mu2 = 100;
    p->sweeps_per_solve = 200; p->solves_per_update = 0; p->mg_dt = 100.0;
    p->max_neighbours = 0;
    return BCG_OK;
}

/* BoxLength and maxCellsPerBox as main() derives them (CellMD3D.cpp:52-54).
 * max_neighbours (device capacity of one reduced list) defaults to 64. */
int bcg_params_finalize(bcg_params* p)
{
    if (!p) return BCG_E_ARG;
    p->box_length = p->l_divide + 2 * p->cell_radius;
    const double PI_ = 3.141592653589793238462643383279502884197;
    double bl = p->box_length;
    p->max_cells_per_box = (int)ceil(bl * bl * bl / (PI_ * p->cell_radius * p->cell_radius * p->l_divide * p->density_threshold / 2));
    if (p->max_neighbours <= 0) p->max_neighbours = 64;
    if (p->box_x < 8 || p->box_y < 1 || p->box_z < 3 || p->box_z_agar < 2) return BCG_E_ARG;
    if (p->max_levels_mg < 1 || p->mg_levels < p->max_levels_mg || p->mg_levels > 16) return BCG_E_ARG;
    if (p->refinement_grid_height < 1 || p->filter_len < 1 || p->max_cells < 1) return BCG_E_ARG;
    if (p->max_neighbours > 1024) return BCG_E_ARG;
    return BCG_OK;
}

/* ---------------------------------------------------------------------------
 * glibc rand() (TYPE_3, degree 31, separation 3).  Published description:
 *   r[0] = seed (1 if seed == 0); r[i] = 16807*r[i-1] mod (2^31-1) for
 *   i = 1..30 (signed, fixed up to be non-negative); r[i] = r[i-31] for
 *   i = 31..33; r[i] = r[i-31] + r[i-3] (mod 2^32) from i = 34 on; the
 *   k-th output is r[k+344] >> 1.
 * The state keeps r[i-34..i-1] in a ring of 34 words; pos = i mod 34.
 * ------------------------------------------------------------------------- */
void bcg_rng_seed(bcg_rng* g, uint32_t seed)
{
    uint32_t r[344];
    int32_t s = (int32_t)seed;
    if (s == 0) s = 1;
    r[0] = (uint32_t)s;
    for (int i = 1; i < 31; i++) {
        long long w = (16807LL * (long long)(int32_t)r[i - 1]) % 2147483647LL;
        if (w < 0) w += 2147483647LL;
        r[i] = (uint32_t)w;
    }
    for (int i = 31; i < 34; i++) r[i] = r[i - 31];
    for (int i = 34; i < 344; i++) r[i] = r[i - 31] + r[i - 3];
    for (int i = 310; i < 344; i++) g->r[i % 34] = r[i];
    g->pos = 344 % 34;
}

int32_t bcg_rng_next(bcg_rng* g)
{
    int i = g->pos;
    uint32_t v = g->r[(i + 34 - 31) % 34] + g->r[(i + 34 - 3) % 34];
    g->r[i] = v;
    g->pos = (i + 1) % 34;
    return (int32_t)(v >> 1);
}

/* Polynomials modulo P(x) = x^31 - x^28 - 1 over Z/2^32 (the recurrence
 * s[n] = s[n-31] + s[n-3]).  x^m mod P gives s[n0+m] as a combination of
 * s[n0..n0+30]. */
namespace {
struct Poly { uint32_t c[31]; };
void poly_mulmod(const Poly& a, const Poly& b, Poly& out)
{
    uint32_t t[61];
    memset(t, 0, sizeof(t));
    for (int i = 0; i < 31; i++) {
        if (!a.c[i]) continue;
        for (int j = 0; j < 31; j++) t[i + j] += a.c[i] * b.c[j];
    }
    for (int d = 60; d >= 31; d--) {   /* x^d = x^(d-31) * (x^28 + 1) */
        uint32_t v = t[d];
        if (!v) continue;
        t[d - 3] += v;
        t[d - 31] += v;
        t[d] = 0;
    }
    memcpy(out.c, t, sizeof(out.c));
}
void poly_mulx(Poly& a)
{
    uint32_t top = a.c[30];
    for (int j = 30; j > 0; j--) a.c[j] = a.c[j - 1];
    a.c[0] = 0;
    a.c[28] += top;
    a.c[0] += top;
}
} // namespace

void bcg_rng_skip(bcg_rng* g, int64_t k)
{
    if (k <= 0) return;
    if (k < 4096) { for (int64_t i = 0; i < k; i++) bcg_rng_next(g); return; }
    /* state s[n0+j] = r[i-31+j], j = 0..30, where i = next index */
    uint32_t s[31];
    for (int j = 0; j < 31; j++) s[j] = g->r[(g->pos + 34 - 31 + j) % 34];
    /* the ring needs the 34 values ending just before the new next index,
     * s[n0+k-3 .. n0+k+30]; start from C = x^(k-3) mod P */
    Poly C; memset(&C, 0, sizeof(C)); C.c[0] = 1;
    int64_t k3 = k - 3;
    int top = 63; while (top >= 0 && !((k3 >> top) & 1)) top--;
    for (int b = top; b >= 0; b--) {
        Poly sq; poly_mulmod(C, C, sq); C = sq;
        if ((k3 >> b) & 1) poly_mulx(C);
    }
    uint32_t vals[34];
    for (int t = 0; t < 34; t++) {
        uint32_t v = 0;
        for (int j = 0; j < 31; j++) v += C.c[j] * s[j];
        vals[t] = v;
        poly_mulx(C);
    }
    /* vals[t] = s[n0 + k - 3 + t]; the next index after the jump is
     * i' = i + k, whose predecessors i'-34..i'-1 = n0+31+k-34 .. n0+30+k */
    int64_t inew = (int64_t)g->pos + k;     /* only the residue mod 34 matters */
    int posn = (int)(inew % 34);
    for (int t = 0; t < 34; t++) {
        /* index n0 + k - 3 + t = (i - 31) + k - 3 + t = inew - 34 + t */
        g->r[(posn + t) % 34] = vals[t];
    }
    g->pos = posn;
}

/* ---------------------------------------------------------------------------
 * Synthetic colony: 2-D x-z half-ellipse dome of the given width/height
 * resting on the agar (z = 0), filled by random sequential placement of
 * spherocylinders with Length ~ U(len_lo, len_hi), in-plane angle
 * theta ~ U(0, pi), centre uniform in the dome, both poles at z >= radius,
 * and no overlap with any earlier cell (segment distance >= 2 radius).
 * Records follow AddFirstCells' field conventions (InputOutput.cpp:319-345):
 * v = w = 0, Type = 1, Ancestor = id + 1, ages and pole times 0, and
 * Ldiv = Length + (l_divide/2) * (1 - div_phase_spread * u), u ~ U(0,1)
 * (div_phase_spread = 0 reproduces Ldiv = Length + L_divide/2).
 * If the dome cannot take n_target cells after a bounded number of tries,
 * it is widened by 2 % in both directions and placement continues.
 * RNG: std::mt19937_64(seed); doubles are (x >> 11) * 2^-53.
 * ------------------------------------------------------------------------- */
namespace {
struct Seg { double px, pz, qx, qz; };
double seg_dist2(const Seg& a, const Seg& b)
{
    /* closest distance between two 2-D segments (plain geometry) */
    double d1x = a.qx - a.px, d1z = a.qz - a.pz, d2x = b.qx - b.px, d2z = b.qz - b.pz;
    double rx = a.px - b.px, rz = a.pz - b.pz;
    double aa = d1x * d1x + d1z * d1z, ee = d2x * d2x + d2z * d2z, ff = d2x * rx + d2z * rz;
    double cc = d1x * rx + d1z * rz, bb = d1x * d2x + d1z * d2z;
    double den = aa * ee - bb * bb, s = 0, t;
    if (den > 1e-300) { s = (bb * ff - cc * ee) / den; s = s < 0 ? 0 : (s > 1 ? 1 : s); }
    t = (bb * s + ff) / ee;
    if (t < 0) { t = 0; s = -cc / aa; s = s < 0 ? 0 : (s > 1 ? 1 : s); }
    else if (t > 1) { t = 1; s = (bb - cc) / aa; s = s < 0 ? 0 : (s > 1 ? 1 : s); }
    double dx = (a.px + d1x * s) - (b.px + d2x * t), dz = (a.pz + d1z * s) - (b.pz + d2z * t);
    return dx * dx + dz * dz;
}
} // namespace

int bcg_synth_colony(uint64_t seed, int n_target, double width, double height,
                     double radius, double len_lo, double len_hi,
                     double l_divide, double div_phase_spread,
                     bcg_cell* out, int capacity, int* n)
{
    if (!out || !n || n_target < 0 || n_target > capacity || width <= 0 || height <= 0 ||
        radius <= 0 || len_lo <= 0 || len_hi < len_lo)
        return BCG_E_ARG;
    std::mt19937_64 gen(seed);
    auto U = [&]() { return (double)(gen() >> 11) * (1.0 / 9007199254740992.0); };
    const double cs = len_hi + 2 * radius;          /* hash cell size */
    double W = width, H = height;
    std::vector<Seg> segs; segs.reserve(n_target);
    std::vector<double> lens; lens.reserve(n_target);
    /* hash grid over a box that can hold the widened dome */
    double gx0 = -W, gz0 = -cs;
    int gnx = (int)ceil(2 * W / cs) + 3, gnz = (int)ceil((2 * H + 2 * cs) / cs) + 3;
    std::vector<std::vector<int>> grid((size_t)gnx * gnz);
    auto gidx = [&](double x, double z, int& ix, int& iz) {
        ix = (int)floor((x - gx0) / cs); iz = (int)floor((z - gz0) / cs);
        return ix >= 0 && iz >= 0 && ix < gnx && iz < gnz;
    };
    const double min2 = (2 * radius) * (2 * radius);
    long long fails = 0;
    while ((int)segs.size() < n_target) {
        double L = len_lo + (len_hi - len_lo) * U();
        double th = 3.141592653589793 * U();
        double cx = (U() - 0.5) * W;
        double cz = U() * H;
        double e = 2 * cx / W;
        bool ok = (e * e < 1.0) && (cz <= H * sqrt(1 - e * e));
        Seg s;
        s.px = cx + 0.5 * L * cos(th); s.pz = cz + 0.5 * L * sin(th);
        s.qx = cx - 0.5 * L * cos(th); s.qz = cz - 0.5 * L * sin(th);
        if (ok && (s.pz < radius || s.qz < radius)) ok = false;
        int ix, iz;
        if (ok && !gidx(cx, cz, ix, iz)) ok = false;
        if (ok) {
            for (int dx = -1; dx <= 1 && ok; dx++)
                for (int dz = -1; dz <= 1 && ok; dz++) {
                    int jx = ix + dx, jz = iz + dz;
                    if (jx < 0 || jz < 0 || jx >= gnx || jz >= gnz) continue;
                    for (int id : grid[(size_t)jx * gnz + jz])
                        if (seg_dist2(s, segs[id]) < min2) { ok = false; break; }
                }
        }
        if (!ok) {
            if (++fails > 200000LL + 50LL * (long long)segs.size()) {
                W *= 1.02; H *= 1.02; fails = 0;
                if (2 * W / cs + 3 > gnx || (2 * H + 2 * cs) / cs + 3 > gnz) return BCG_E_ARG;
            }
            continue;
        }
        fails = 0;
        grid[(size_t)ix * gnz + iz].push_back((int)segs.size());
        segs.push_back(s);
        lens.push_back(L);
    }
    for (int i = 0; i < n_target; i++) {
        bcg_cell& c = out[i];
        memset(&c, 0, sizeof(c));
        c.p.x = segs[i].px; c.p.y = 0; c.p.z = segs[i].pz;
        c.q.x = segs[i].qx; c.q.y = 0; c.q.z = segs[i].qz;
        c.length = lens[i];
        c.radius = radius;
        double u = U();
        c.ldiv = lens[i] + (l_divide / 2) * (1.0 - div_phase_spread * u);
        c.type = 1;
        c.ancestor = i + 1;
    }
    *n = n_target;
    return BCG_OK;
}

/* SaveCells / LoadCells (InputOutput.cpp:394-448): {double t, double dt,
 * Cell[N]} raw; the record count follows from the file size. */
int bcg_save_restart(const char* path, double t, double dt, const bcg_cell* cells, int n)
{
    if (!path || n < 0 || (n > 0 && !cells)) return BCG_E_ARG;
    FILE* f = fopen(path, "wb");
    if (!f) return BCG_E_ARG;
    int ok = fwrite(&t, sizeof(double), 1, f) == 1 && fwrite(&dt, sizeof(double), 1, f) == 1 &&
             (n == 0 || fwrite(cells, sizeof(bcg_cell), (size_t)n, f) == (size_t)n);
    ok = (fclose(f) == 0) && ok;
    return ok ? BCG_OK : BCG_E_ARG;
}

int bcg_load_restart(const char* path, double* t, double* dt, bcg_cell* cells, int capacity, int* n)
{
    if (!path || !t || !dt || !n) return BCG_E_ARG;
    FILE* f = fopen(path, "rb");
    if (!f) return BCG_E_ARG;
    fseek(f, 0, SEEK_END);
    long size = ftell(f);
    rewind(f);
    if (size < (long)(2 * sizeof(double))) { fclose(f); return BCG_E_ARG; }
    long count = (size - 2 * (long)sizeof(double)) / (long)sizeof(bcg_cell);
    if (fread(t, sizeof(double), 1, f) != 1 || fread(dt, sizeof(double), 1, f) != 1) { fclose(f); return BCG_E_ARG; }
    *n = (int)count;
    int m = count < capacity ? (int)count : capacity;
    if (m > 0 && (!cells || fread(cells, sizeof(bcg_cell), (size_t)m, f) != (size_t)m)) { fclose(f); return BCG_E_ARG; }
    fclose(f);
    return count <= capacity ? BCG_OK : BCG_E_ARG;
}

} // extern "C"
