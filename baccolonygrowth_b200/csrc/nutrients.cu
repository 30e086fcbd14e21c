/*
 * nutrients.cu -- the colony/interface Jacobi sweeps and the nutrient
 * update driver (AgentBasedModel-BacColonyGrowth/Multigrid.cpp:984-1125,
 * Nutrients.cpp:200-659, 806-855).
 *
 * One sweep = one launch of k_sweep over the colony grid (the colony
 * points of the bounding box and the wall rows of every level); on even
 * sweep counts the wall reads the colony row z = 0 left in the current
 * buffer, on odd counts the row this sweep wrote (the reference's 1-thread
 * order).
 * Buffers swap after every sweep.  The acetate buffer solve, whose results
 * (pH, Hydrox, Acetic, Buffer) feed nothing else, runs only in the last two
 * sweeps of a call: those are the values that survive in each buffer.  The
 * same holds for the growth-rate components and maintenance rates
 * (GrCarAer .. qOxymnt), which only the Environment writer reads; they are
 * stored for Environment (buffer 0) in the last sweep that writes it.
 */
#include "ctx.cuh"
#include "mg.cuh"
#include <float.h>
#include <vector>

struct NutConst {
    int X, Z, A;
    double BL, cdt;
    double kc_aer, kc_ana, ka, ko;
    double mgrCarAers, mgrCarAnas, mgrAceAers, g1s, g2s, g3s;
    double max_gr_car_aer, max_gr_car_ana, max_gr_ace_aer;
    double q_o2_car, q_o2_ace, q_car_aer, q_car_ana, q_ace_aer, p_ace_aer, p_ace_ana;
    double q_o2_car_nt, q_o2_ace_nt, q_car_aer_nt, q_car_ana_nt, q_ace_aer_nt, p_ace_ana_nt;
    double carbon_to_waste;
    double dcc, dco, dca, dcw;        /* colony diffusivities: carbon, oxygen, acetate, waste */
    double dac, dao, daa, daw;        /* agar diffusivities */
    double max_carbon, max_o2;
    double kw_ph, ka_ph, kb_ph, cb_ph, c1_ph;
    double inv_bl2, inv_g1s, inv_g2s, inv_g3s;   /* 1/BoxLength^2, 1/g1s, 1/g2s, 1/g3s */
};

static NutConst nut_const(const bcg_ctx* c)
{
    const bcg_params& P = c->P;
    NutConst n;
    n.X = P.box_x; n.Z = P.box_z; n.A = P.max_levels_mg;
    n.BL = P.box_length; n.cdt = P.cdt;
    n.kc_aer = P.kc_aer; n.kc_ana = P.kc_ana; n.ka = P.ka; n.ko = P.ko;
    /* maintenance constants, Nutrients.cpp:232-267 */
    if (P.max_gr_car_aer != 0.0) { n.mgrCarAers = P.q_car_aer_nt / P.q_car_aer; n.g1s = P.kc_aer * (n.mgrCarAers / P.max_gr_car_aer); }
    else { n.mgrCarAers = 0; n.g1s = 1e6; }
    if (P.max_gr_car_ana != 0.0) { n.mgrCarAnas = P.q_car_ana_nt / P.q_car_ana; n.g2s = P.kc_ana * (n.mgrCarAnas / P.max_gr_car_ana); }
    else { n.mgrCarAnas = 0; n.g2s = 1e6; }
    if (P.max_gr_ace_aer != 0.0) { n.mgrAceAers = P.q_ace_aer_nt / P.q_ace_aer; n.g3s = P.ka * (n.mgrAceAers / P.max_gr_ace_aer); }
    else { n.mgrAceAers = 0; n.g3s = 1e6; }
    n.max_gr_car_aer = P.max_gr_car_aer; n.max_gr_car_ana = P.max_gr_car_ana; n.max_gr_ace_aer = P.max_gr_ace_aer;
    n.q_o2_car = P.q_o2_car; n.q_o2_ace = P.q_o2_ace; n.q_car_aer = P.q_car_aer; n.q_car_ana = P.q_car_ana;
    n.q_ace_aer = P.q_ace_aer; n.p_ace_aer = P.p_ace_aer; n.p_ace_ana = P.p_ace_ana;
    n.q_o2_car_nt = P.q_o2_car_nt; n.q_o2_ace_nt = P.q_o2_ace_nt; n.q_car_aer_nt = P.q_car_aer_nt;
    n.q_car_ana_nt = P.q_car_ana_nt; n.q_ace_aer_nt = P.q_ace_aer_nt; n.p_ace_ana_nt = P.p_ace_ana_nt;
    n.carbon_to_waste = P.carbon_to_waste;
    n.dcc = P.diff_colony_carbon; n.dco = P.diff_colony_o2; n.dca = P.diff_colony_ace; n.dcw = P.diff_colony;
    n.dac = P.diff_agar_carbon; n.dao = P.diff_agar_o2; n.daa = P.diff_agar_ace; n.daw = P.diff_agar;
    n.max_carbon = P.max_carbon; n.max_o2 = P.max_o2;
    n.kw_ph = P.kw_ph; n.ka_ph = P.ka_ph; n.kb_ph = P.kb_ph; n.cb_ph = P.cb_ph; n.c1_ph = P.c1_ph;
    n.inv_bl2 = 1.0 / (P.box_length * P.box_length);
    n.inv_g1s = 1.0 / n.g1s; n.inv_g2s = 1.0 / n.g2s; n.inv_g3s = 1.0 / n.g3s;
    return n;
}

__device__ __forceinline__ double mx(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double mn(double a, double b) { return a < b ? a : b; }

/* acetateBufferSolve, Nutrients.cpp:806-855 */
__device__ void buffer_solve(const NutConst& n, double Cac, double& pH, double& hyd, double& acetic, double& buf)
{
    const double Kw = n.kw_ph, Ka = n.ka_ph, Kb = n.kb_ph, Cb = n.cb_ph, c1 = n.c1_ph;
    double aH = -(Cb * Kb) / (pow(10.0, -4.0) + Kb);
    double x = 1e-7, y = Cac, z = Cb;
    for (int it = 0; it < 100; it++) {
        double J[3][4] = {{2 * x + y + z + (Kw / c1) + aH, x, x, -(pow(x, 2.0) + x * (y + z + (Kw / c1) + aH) - Kw)},
                          {y, 2 * y + x + z + Ka + aH, y, -(pow(y, 2.0) + y * (x + z + (Ka) + aH) - Ka * Cac)},
                          {z, z, 2 * z + x + y + Kb + aH, -(pow(z, 2.0) + z * (x + y + (Kb) + aH) - Kb * Cb)}};
        double m1 = J[1][0] / J[0][0], m2 = J[2][0] / J[0][0];
#pragma unroll
        for (int i = 0; i < 4; i++) { J[1][i] -= m1 * J[0][i]; J[2][i] -= m2 * J[0][i]; }
        double m3 = J[2][1] / J[1][1];
#pragma unroll
        for (int i = 0; i < 4; i++) J[2][i] -= m3 * J[1][i];
        double s2 = J[2][3] / J[2][2];
        double s1 = J[1][3] / J[1][1] - (J[1][2] / J[1][1]) * s2;
        double s0 = J[0][3] / J[0][0] - (J[0][2] / J[0][0]) * s2 - (J[0][1] / J[0][0]) * s1;
        double m = 0;
        if (fabs(s0) > m) m = fabs(s0);
        if (fabs(s1) > m) m = fabs(s1);
        if (fabs(s2) > m) m = fabs(s2);
        x += s0; y += s1; z += s2;
        if (m < pow(10.0, -7.0)) break;
    }
    pH = -log((x + y + z + aH) / 1000) / log(10.0);
    hyd = x; acetic = y; buf = z;
}

struct EnvP { double *C, *W, *A, *O, *gr1, *gr2, *ph, *hyd, *ace, *buf; };
static EnvP envp(bcg_ctx* c, int b)
{
    EnvBuf& e = c->env[b];
    EnvP p = {e.C, e.W, e.A, e.O, e.gr1, e.gr2, e.ph, e.hydrox, e.acetic, e.buffer};
    return p;
}
struct WallP { const double *C, *W, *O, *A; };
/* Environment's GrCarAer, GrCarAna, GrAceAer, qCarmnt, qAcemnt, pAcemnt,
 * qOxymnt (Nutrients.cpp:328-344); all null when the sweep's current
 * buffer is not Environment or its values do not survive the call */
struct EnvX { double *gca, *gcn, *gaa, *qcm, *qam, *pam, *qom; };

/* UpdateEnvironment_OxygenAcetate (Nutrients.cpp:200-506), crossFeeding = 0,
 * for x in [minx, maxx], z in [0, maxz] where DensityShiftP > DBL_EPSILON
 * (Multigrid.cpp:1037-1047).
 *
 * One point (x, z); the sweep kernel below runs a block of 32 z (the
 * contiguous direction, one warp) x COLONY_COLS columns.  DIAG adds the
 * acetate buffer solve and the Environment-only
 * members; the other sweeps run a variant without them, which needs fewer
 * registers.  The second differences multiply by 1/BoxLength^2 and the
 * maintenance caps min(Cgr/g1s, 1) .. by 1/g1s .., reciprocals taken once on
 * the host, where the reference divides: the results differ from its
 * quotients by rounding only (one unit in the last place per term). */
#define COLONY_COLS 8
template <bool DIAG, bool EXTRA = DIAG>
__device__ __forceinline__ void colony_point(const NutConst& n, int x, int z, const int* __restrict__ bbox,
                                             const EnvP& cur, const EnvP& prev, const WallP& pw0,
                                             const double* __restrict__ inside, const double* __restrict__ ds,
                                             const EnvX& ex, DevStatus* st)
{
    const int Z = n.Z;
    if (z >= Z || x >= n.X) return;
    const size_t id = (size_t)x * Z + z;
    int minx = bbox[0], maxx = bbox[1], maxz = bbox[2];
    if (x < minx || x > maxx || z > maxz) return;
    if (!(ds[id] > DBL_EPSILON)) return;
    /* stencil range guard (the bbox check reports a colony at the edge) */
    if (x < 1 || x > n.X - 2 || z > Z - 2) return;
    const double ins = inside[id];
#define IXZ(a, b) ((size_t)(a) * Z + (b))
    if (ins > 0.5) {
        double Cgr = 0, Agr = 0, Ogr = 0;   /* the waste average Wgr feeds nothing here */
        if (x != 0) {
            if (z == 0) {
                Cgr = (pw0.C[x - 1] + prev.C[IXZ(x - 1, z)] + pw0.C[x] + prev.C[id]) / 4.0;
                Ogr = (pw0.O[x - 1] + prev.O[IXZ(x - 1, z)] + pw0.O[x] + prev.O[id]) / 4.0;
                Agr = (pw0.A[x - 1] + prev.A[IXZ(x - 1, z)] + pw0.A[x] + prev.A[id]) / 4.0;
            } else {
                Cgr = (prev.C[IXZ(x - 1, z - 1)] + prev.C[IXZ(x - 1, z)] + prev.C[IXZ(x, z - 1)] + prev.C[id]) / 4.0;
                Ogr = (prev.O[IXZ(x - 1, z - 1)] + prev.O[IXZ(x - 1, z)] + prev.O[IXZ(x, z - 1)] + prev.O[id]) / 4.0;
                Agr = (prev.A[IXZ(x - 1, z - 1)] + prev.A[IXZ(x - 1, z)] + prev.A[IXZ(x, z - 1)] + prev.A[id]) / 4.0;
            }
        }
        if (DIAG) {
            /* the second solve (for Agr) overwrites the first (for A) */
            double ph, hy, ac, bu;
            buffer_solve(n, Agr, ph, hy, ac, bu);
            prev.ph[id] = ph; prev.hyd[id] = hy; prev.ace[id] = ac; prev.buf[id] = bu;
        }
        /* x / (x + k): for x = 0 and k > 0 the quotient is x itself, taken
         * here without the division, whose zero dividend leaves its fast
         * path (the species start at zero, acetate everywhere) */
        double fCgr_aer = (Cgr == 0.0 && n.kc_aer > 0.0) ? Cgr : Cgr / (Cgr + n.kc_aer);
        double fCgr_ana = (Cgr == 0.0 && n.kc_ana > 0.0) ? Cgr : Cgr / (Cgr + n.kc_ana);
        double fAgr = (Agr == 0.0 && n.ka > 0.0) ? Agr : Agr / (Agr + n.ka);
        double fOgr = (Ogr == 0.0 && n.ko > 0.0) ? Ogr : Ogr / (Ogr + n.ko), fIgr = 0;
        double l1 = mx((n.max_gr_car_aer + n.mgrCarAers) * fCgr_aer - n.mgrCarAers, 0.0);
        double l2 = mx((n.max_gr_car_ana + n.mgrCarAnas) * fCgr_ana - n.mgrCarAnas, 0.0);
        double l3 = mx((n.max_gr_ace_aer + n.mgrAceAers) * fAgr - n.mgrAceAers, 0.0);
        double qO = (n.q_o2_car * l1 * fCgr_aer + n.q_o2_ace * l3 * (1 - fCgr_aer)) * fOgr * mx(1 - fIgr, 0.0) + n.q_o2_car_nt * mn((Cgr * n.inv_g1s), 1.0) * fCgr_aer * fOgr + n.q_o2_ace_nt * mn((Agr * n.inv_g3s), 1.0) * (1 - fCgr_aer) * fOgr;
        double qC = (n.q_car_aer * l1 * fCgr_aer * fOgr + n.q_car_ana * l2 * (1 - fOgr)) * mx(1 - fIgr, 0.0) + n.q_car_aer_nt * mn((Cgr * n.inv_g1s), 1.0) * fCgr_aer * fOgr + n.q_car_ana_nt * mn((Cgr * n.inv_g2s), 1.0) * (1 - fOgr);
        double qA = (n.q_ace_aer * l3 * (1 - fCgr_aer) * fOgr) * mx(1 - fIgr, 0.0) + n.q_ace_aer_nt * mn((Agr * n.inv_g3s), 1.0) * (1 - fCgr_aer) * fOgr;
        double pA = (n.p_ace_aer * l1 * fCgr_aer * fOgr + n.p_ace_ana * l2 * (1 - fOgr)) * mx(1 - fIgr, 0.0) + n.p_ace_ana_nt * mn((Cgr * n.inv_g2s), 1.0) * (1 - fOgr);
        double pW = n.carbon_to_waste * qC, qW = 0.0;
        double GrCarAer = l1 * fCgr_aer * fOgr * mx(1 - fIgr, 0.0);
        double GrCarAna = l2 * (1 - fOgr) * mx(1 - fIgr, 0.0);
        double GrAceAer = l3 * (1 - fCgr_aer) * fOgr * mx(1 - fIgr, 0.0);
        double gr = GrCarAer + GrCarAna + GrAceAer;
        cur.gr1[id] = gr;
        cur.gr2[id] = gr;
        if (EXTRA && ex.gca) {
            ex.qcm[id] = n.q_car_aer_nt * mn((Cgr * n.inv_g1s), 1.0) * fCgr_aer * fOgr + n.q_car_ana_nt * mn((Cgr * n.inv_g2s), 1.0) * (1 - fOgr);
            ex.qam[id] = n.q_ace_aer_nt * mn((Agr * n.inv_g3s), 1.0) * (1 - fCgr_aer) * fOgr;
            ex.pam[id] = n.p_ace_ana_nt * mn((Cgr * n.inv_g2s), 1.0) * (1 - fOgr);
            ex.qom[id] = n.q_o2_car_nt * mn((Cgr * n.inv_g1s), 1.0) * fCgr_aer * fOgr + n.q_o2_ace_nt * mn((Agr * n.inv_g3s), 1.0) * (1 - fCgr_aer) * fOgr;
            ex.gca[id] = GrCarAer; ex.gcn[id] = GrCarAna; ex.gaa[id] = GrAceAer;
        }
        if (!(x > 2)) { dev_error(st, BCG_E_NEED_MORE_BOXES, x); return; }
        const double c0C = prev.C[id], c0W = prev.W[id], c0A = prev.A[id], c0O = prev.O[id];
        const size_t up = IXZ(x, z + 1);
        double Czz, Wzz, Azz, Ozz;
        if (z == 0) {
            Wzz = (prev.W[up] + pw0.W[x] - 2.0 * c0W) * n.inv_bl2;
            Czz = (prev.C[up] + pw0.C[x] - 2.0 * c0C) * n.inv_bl2;
            Azz = (prev.A[up] + pw0.A[x] - 2.0 * c0A) * n.inv_bl2;
            Ozz = (prev.O[up] + pw0.O[x] - 2.0 * c0O) * n.inv_bl2;
        } else {
            const size_t dn = IXZ(x, z - 1);
            Wzz = (prev.W[up] + prev.W[dn] - 2.0 * c0W) * n.inv_bl2;
            Czz = (prev.C[up] + prev.C[dn] - 2.0 * c0C) * n.inv_bl2;
            Azz = (prev.A[up] + prev.A[dn] - 2.0 * c0A) * n.inv_bl2;
            Ozz = (prev.O[up] + prev.O[dn] - 2.0 * c0O) * n.inv_bl2;
        }
        const size_t xp = IXZ(x + 1, z), xm = IXZ(x - 1, z);
        double Cxx = (prev.C[xp] + prev.C[xm] - 2.0 * c0C) * n.inv_bl2;
        double Wxx = (prev.W[xp] + prev.W[xm] - 2.0 * c0W) * n.inv_bl2;
        double Axx = (prev.A[xp] + prev.A[xm] - 2.0 * c0A) * n.inv_bl2;
        double Oxx = (prev.O[xp] + prev.O[xm] - 2.0 * c0O) * n.inv_bl2;
        double DS = ds[id];
        double Cnew = c0C + (n.dcc * (Cxx + Czz) - qC * 0.25 * DS) * n.cdt;
        double CAcenew = c0A + (n.dca * (Axx + Azz) + pA * 0.25 * DS - qA * 0.25 * DS) * n.cdt;
        double Onew = c0O + (n.dco * (Oxx + Ozz) - qO * 0.25 * DS) * n.cdt;
        cur.C[id] = mx(0.0, mn(Cnew, n.max_carbon));
        cur.O[id] = mx(0.0, mn(Onew, n.max_o2));
        cur.A[id] = mx(0.0, CAcenew);
        double Wnew = c0W + (n.dcw * (Wxx + Wzz) + pW * DS - qW * DS) * n.cdt;
        cur.W[id] = mx(0.0, Wnew);
    } else if (ins > 0.3) {
        const size_t ixp = IXZ(x + 1, z), ixm = IXZ(x - 1, z), iu = IXZ(x, z + 1);
        int bp = inside[ixp] > 0.5, bm = inside[ixm] > 0.5, bu = inside[iu] > 0.5;
        double Cnew, Wnew, CAcenew;
        if (z > 0) {
            const size_t id_ = IXZ(x, z - 1);
            int bd = inside[id_] > 0.5;
            int den = bp + bm + bu + bd;
            Cnew = (prev.C[ixp] * bp + prev.C[ixm] * bm + prev.C[iu] * bu + prev.C[id_] * bd) / den;
            Wnew = (prev.W[ixp] * bp + prev.W[ixm] * bm + prev.W[iu] * bu + prev.W[id_] * bd) / den;
            CAcenew = (prev.A[ixp] * bp + prev.A[ixm] * bm + prev.A[iu] * bu + prev.A[id_] * bd) / den;
        } else {
            int den = bp + bm + bu;
            Cnew = (prev.C[ixp] * bp + prev.C[ixm] * bm + prev.C[iu] * bu) / den;
            Wnew = (prev.W[ixp] * bp + prev.W[ixm] * bm + prev.W[iu] * bu) / den;
            CAcenew = (prev.A[ixp] * bp + prev.A[ixm] * bm + prev.A[iu] * bu) / den;
        }
        cur.C[id] = mx(0.0, mn(Cnew, n.max_carbon));
        cur.O[id] = mx(0.0, mn(n.max_o2, n.max_o2));
        cur.A[id] = mx(0.0, CAcenew);
        cur.W[id] = mx(0.0, Wnew);
    }
#undef IXZ
}

struct WallAll { double *C[BCG_MAX_AGAR_LEVELS], *W[BCG_MAX_AGAR_LEVELS], *O[BCG_MAX_AGAR_LEVELS], *A[BCG_MAX_AGAR_LEVELS]; };
static WallAll wall_all(bcg_ctx* c, int b)
{
    WallAll w;
    for (int l = 0; l < BCG_MAX_AGAR_LEVELS; l++) { w.C[l] = c->wal[b].C[l]; w.W[l] = c->wal[b].W[l]; w.O[l] = c->wal[b].O[l]; w.A[l] = c->wal[b].A[l]; }
    return w;
}
/* the agar row z = 0 of each level the wall reads (FieldAgar(x, 0)); the
 * waste row is null where the agar waste is 0 (the multigrid path never
 * writes it) */
struct AgarRow { const double *C[BCG_MAX_AGAR_LEVELS], *O[BCG_MAX_AGAR_LEVELS], *A[BCG_MAX_AGAR_LEVELS], *W[BCG_MAX_AGAR_LEVELS]; };

/* UpdateWallMultigrid_OxygenAcetate (Nutrients.cpp:509-659), Box_y = 1.
 * FieldAgar[l](x, 0) is the multigrid solution row 1 (copyFromMG) or, in the
 * legacy explicit solver, its own agar row; the multigrid path never writes
 * the agar waste, which stays 0 there.  For level > 0 and
 * BoxX/4-1 < x < BoxX*3/4 the reference reads uninitialised second
 * differences; here they are 0 (those points are read by no other point
 * before the next solve overwrites them). */
__device__ __forceinline__ void wall_point(const NutConst& n, int level, int x, const EnvP& curenv, const AgarRow& ag,
                                           const WallAll& cw, const WallAll& pw, const double* __restrict__ inside)
{
    const int X = n.X;
    if (level == 0 && inside[(size_t)x * n.Z] > 0.5) {
        size_t i0 = (size_t)x * n.Z;
        double gC = ag.C[0][x], gO = ag.O[0][x], gA = ag.A[0][x], gW = ag.W[0] ? ag.W[0][x] : 0.0;
        double Cnew = (n.dcc * curenv.C[i0] + n.dac * gC) / (n.dcc + n.dac);
        double Onew = (n.dco * curenv.O[i0] + n.dao * gO) / (n.dco + n.dao);
        cw.C[0][x] = mx(0.0, mn(Cnew, n.max_carbon));
        cw.O[0][x] = mx(0.0, mn(Onew, n.max_o2));
        double CAcenew = (n.dca * curenv.A[i0] + n.daa * gA) / (n.dca + n.daa);
        cw.A[0][x] = mx(0.0, CAcenew);
        double Wnew = (n.dcw * curenv.W[i0] + n.daw * gW) / (n.dcw + n.daw);
        cw.W[0][x] = mx(0.0, Wnew);
        return;
    }
    const double* pC = pw.C[level];
    const double* pW = pw.W[level];
    const double* pA = pw.A[level];
    double h2l = n.BL * n.BL * pow(4.0, (double)level);
    double Cxx = 0, Wxx = 0, Axx = 0;
    if (level > 0 && (x >= X / 4 - 1) && x <= X * 3 / 4) {
        if (x == X / 4 - 1) {
            Wxx = (pW[x - 1] + pw.W[level - 1][0] - 2 * pW[x]) / h2l;
            Cxx = (pC[x - 1] + pw.C[level - 1][0] - 2 * pC[x]) / h2l;
            Axx = (pA[x - 1] + pw.A[level - 1][0] - 2 * pA[x]) / h2l;
        } else if (x == X * 3 / 4) {
            Wxx = (pW[x + 1] + pw.W[level - 1][X - 2] - 2 * pW[x]) / h2l;
            Cxx = (pC[x + 1] + pw.C[level - 1][X - 2] - 2 * pC[x]) / h2l;
            Axx = (pA[x + 1] + pw.A[level - 1][X - 2] - 2 * pA[x]) / h2l;
        }
    } else if (level < n.A - 1 && (x == 0 || x == X - 1)) {
        const int ly = 0;
        if (x == 0) {
            const int q = X / 4 - 1;
            Wxx = (pW[x + 2] + 1.0 / (ly + 1) * pw.W[level + 1][q] + ly * 1.0 / (ly + 1) * pw.W[level + 1][q] - 2 * pW[x]) / 4 / h2l;
            Cxx = (pC[x + 2] + 1.0 / (ly + 1) * pw.C[level + 1][q] + ly * 1.0 / (ly + 1) * pw.C[level + 1][q] - 2 * pC[x]) / 4 / h2l;
            Axx = (pA[x + 2] + 1.0 / (ly + 1) * pw.A[level + 1][q] + ly * 1.0 / (ly + 1) * pw.A[level + 1][q] - 2 * pA[x]) / 4 / h2l;
        } else {
            const int q = X * 3 / 4;
            Wxx = (pW[x - 1] + 1.0 / (ly + 1) * pw.W[level + 1][q] + ly * 1.0 / (ly + 1) * pw.W[level + 1][q] - 2 * pW[x]) / h2l;
            Cxx = (pC[x - 1] + 1.0 / (ly + 1) * pw.C[level + 1][q] + ly * 1.0 / (ly + 1) * pw.C[level + 1][q] - 2 * pC[x]) / h2l;
            Axx = (pA[x - 1] + 1.0 / (ly + 1) * pw.A[level + 1][q] + ly * 1.0 / (ly + 1) * pw.A[level + 1][q] - 2 * pA[x]) / h2l;
        }
    } else if (level == n.A - 1 && (x == 0 || x == X - 1)) {
        int s1 = (x == 0) ? 1 : X - 2;
        Wxx = (pW[s1] - 1.0 * pW[x]) / h2l;
        Cxx = (pC[s1] - 1.0 * pC[x]) / h2l;
        Axx = (pA[s1] - 1.0 * pA[x]) / h2l;
    } else {
        Wxx = (pW[x - 1] + pW[x + 1] - 2 * pW[x]) / h2l;
        Cxx = (pC[x - 1] + pC[x + 1] - 2 * pC[x]) / h2l;
        Axx = (pA[x - 1] + pA[x + 1] - 2 * pA[x]) / h2l;
    }
    double gC = ag.C[level][x], gA = ag.A[level][x], gW = ag.W[level] ? ag.W[level][x] : 0.0;
    double Wzz = 2.0 * (gW - pW[x]) / h2l;
    double Czz = 2.0 * (gC - pC[x]) / h2l;
    double Azz = 2.0 * (gA - pA[x]) / h2l;
    double Cnew = pC[x] + n.dac * (Cxx + Czz) * n.cdt;
    cw.C[level][x] = mx(0.0, mn(Cnew, n.max_carbon));
    cw.O[level][x] = mx(0.0, mn(n.max_o2, n.max_o2));
    double CAcenew = pA[x] + n.daa * (Axx + Azz) * n.cdt;
    cw.A[level][x] = mx(0.0, CAcenew);
    double Wnew = pW[x] + n.daw * (Wxx + Wzz) * n.cdt;
    cw.W[level][x] = mx(0.0, Wnew);
}

static AgarRow agar_rows(bcg_ctx* c)
{
    AgarRow a;
    for (int l = 0; l < BCG_MAX_AGAR_LEVELS; l++) { a.C[l] = nullptr; a.O[l] = nullptr; a.A[l] = nullptr; a.W[l] = nullptr; }
    for (int l = 0; l < c->P.max_levels_mg; l++) {
        const MgLevel& L = c->mg[l];
        a.C[l] = L.sol[0] + L.pitch; a.O[l] = L.sol[1] + L.pitch; a.A[l] = L.sol[2] + L.pitch;
    }
    return a;
}

/* One sweep of Multigrid.cpp:1017-1095 in one launch: the colony points
 * (x, z) of the grid and the wall rows (level, x).  The only dependence
 * between the two within a sweep is the level-0 wall of a colony column
 * reading the column's z = 0 point of the current buffer: before this
 * sweep writes it on even sweep counts (the reference's wall loop runs
 * first), after on odd counts (it runs last).  The thread of (x, 0) does
 * both in that order; threads (x, z) with 1 <= z < A of the first z
 * block take the wall of level z.  Each wall point reads only the
 * previous wall buffer, the agar rows and that one colony value, and no
 * colony point reads the current wall buffer, so nothing else orders
 * them. */
template <bool DIAG, bool WALL_FIRST>
__global__ void __launch_bounds__(32 * COLONY_COLS) k_sweep(NutConst n, const int* __restrict__ bbox, EnvP cur,
                                                            EnvP prev, WallP pw0, const double* __restrict__ inside,
                                                            const double* __restrict__ ds, EnvX ex, AgarRow ag,
                                                            WallAll cw, WallAll pw, DevStatus* st)
{
    const int z = blockIdx.x * 32 + threadIdx.x;
    const int x = blockIdx.y * COLONY_COLS + threadIdx.y;
    if (x >= n.X) return;
    const bool wall = z < n.A;
    if (wall && (WALL_FIRST || z > 0)) wall_point(n, z, x, cur, ag, cw, pw, inside);
    colony_point<DIAG>(n, x, z, bbox, cur, prev, pw0, inside, ds, ex, st);
    if (!WALL_FIRST && z == 0) wall_point(n, 0, x, cur, ag, cw, pw, inside);
}

static void sweep_launch(dim3 grid, dim3 block, bcg_ctx* c, const NutConst& n, EnvP cur, EnvP prev, WallP pw0,
                         int diag, EnvX ex, const AgarRow& ag, const WallAll& cw, const WallAll& pw, bool wall_first)
{
#define SWEEP(D, W) k_sweep<D, W><<<grid, block, 0, c->stream>>>(n, c->bbox, cur, prev, pw0, c->inside, c->ds, ex, ag, cw, pw, c->status)
    if (diag) { if (wall_first) SWEEP(true, true); else SWEEP(true, false); }
    else { if (wall_first) SWEEP(false, true); else SWEEP(false, false); }
#undef SWEEP
}

/* `nsweeps` sweeps with the local buffer indices (ce = current colony
 * buffer, cw = current wall buffer) and sweep counter, as the reference's
 * loop keeps them (Multigrid.cpp:1017-1120); diag_from = first sweep index
 * that runs the acetate buffer solve. */
static void run_sweeps(bcg_ctx* c, int nsweeps, int& ce, int& cwb, int& count, int diag_from)
{
    NutConst n = nut_const(c);
    const int X = c->P.box_x, Z = c->P.box_z;
    AgarRow ag = agar_rows(c);
    /* at least one z block: its first A lanes carry the wall rows */
    const dim3 gcol((unsigned)((Z + 31) / 32), (unsigned)((X + COLONY_COLS - 1) / COLONY_COLS)), bcol(32, COLONY_COLS);
    for (int j = 0; j < nsweeps; j++) {
        EnvP cur = envp(c, ce), prev = envp(c, ce ^ 1);
        WallAll cw = wall_all(c, cwb), pw = wall_all(c, cwb ^ 1);
        WallP pw0 = {pw.C[0], pw.W[0], pw.O[0], pw.A[0]};
        int diag = j >= diag_from;
        EnvX ex = {};
        if (diag && ce == 0) {
            double* const* x = c->env[0].extra;
            ex = EnvX{x[0], x[1], x[2], x[3], x[4], x[5], x[6]};
        }
        sweep_launch(gcol, bcol, c, n, cur, prev, pw0, diag, ex, ag, cw, pw, count % 2 == 0);
        c->launches += 1;
        if (c->P.nutrient_gsi == 0) { ce ^= 1; cwb ^= 1; }
        count++;
    }
}

extern "C" int bcg_colony_sweeps(bcg_ctx* c, int sweeps, int count0)
{
    if (!c || sweeps < 0) return BCG_E_ARG;
    if (c->P.nutrient_gsi != 0) return BCG_E_UNSUPPORTED;
    timer_begin(c, BCG_T_SWEEPS);
    int ce = 0, cw = 0, count = count0;
    long long l0 = c->launches;
    run_sweeps(c, sweeps, ce, cw, count, sweeps - 2);
    BCG_CUDA_TRY(cudaGetLastError());
    timer_end(c, BCG_T_SWEEPS, (int)(c->launches - l0));
    return ctx_check_status(c);
}

/* One unit of the nutrient update -- Multigrid::solve then `sweeps`
 * sweeps -- captured once as a CUDA graph and replayed: with an even sweep
 * count the local buffer indices and the sweep-count parity are back where
 * they started after each unit, so every unit issues the same kernels with
 * the same arguments. */
/* drop the cached graphs, the nutrient units' and the per-step solve's (a
 * kernel shape of this context changed, or Err and Res stopped being clean) */
void nutrient_graphs_drop(bcg_ctx* c)
{
    for (int g = 0; g < 2; g++)
        if (c->nutrient_graph[g]) { cudaGraphExecDestroy(c->nutrient_graph[g]); c->nutrient_graph[g] = nullptr; }
    c->nutrient_graph_sweeps = 0;
    if (c->solve_graph) { cudaGraphExecDestroy(c->solve_graph); c->solve_graph = nullptr; }
    c->solve_graph_seen = 0;
}

static int nutrient_unit_graph(bcg_ctx* c, int sweeps, int last, cudaGraphExec_t* out)
{
    if (c->nutrient_graph_sweeps != sweeps) {
        nutrient_graphs_drop(c);
        c->nutrient_graph_sweeps = sweeps;
    }
    if (!c->nutrient_graph[last]) {
        cudaGraph_t g;
        BCG_CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        long long l0 = c->launches;
        int ce = 0, cw = 0, count = 0;
        int rc = mg_solve_impl(c, c->P.mg_vcycles, cw);
        if (rc == BCG_OK) run_sweeps(c, sweeps, ce, cw, count, last ? sweeps - 2 : sweeps);
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        if (rc) return rc;
        if (e != cudaSuccess) { bcg_set_cuda_error(e); return BCG_E_CUDA; }
        c->nutrient_graph_launches[last] = (int)(c->launches - l0);
        c->launches = l0;
        e = cudaGraphInstantiate(&c->nutrient_graph[last], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) { bcg_set_cuda_error(e); return BCG_E_CUDA; }
    }
    *out = c->nutrient_graph[last];
    return BCG_OK;
}

/* UpdateEnvArrayMG_OxygenAcetate (Multigrid.cpp:984-1125) */
extern "C" int bcg_nutrient_update(bcg_ctx* c, int n, int sweeps)
{
    if (!c) return BCG_E_ARG;
    if (c->P.nutrient_gsi != 0) return BCG_E_UNSUPPORTED;
    const bcg_params& P = c->P;
    if (n <= 0) n = P.solves_per_update > 0 ? P.solves_per_update : (int)(3600 * P.update_time * 740 / P.mg_dt);
    if (sweeps < 0) sweeps = P.sweeps_per_solve;
    timer_begin(c, BCG_T_SWEEPS);
    long long l0 = c->launches;
    if (sweeps % 2 == 0 && sweeps >= 2) {
        for (int i = 0; i < n; i++) {
            int last = (i == n - 1);
            cudaGraphExec_t ge;
            int rc = nutrient_unit_graph(c, sweeps, last, &ge);
            if (rc) return rc;
            BCG_CUDA_TRY(cudaGraphLaunch(ge, c->stream));
            c->launches += c->nutrient_graph_launches[last];
        }
    } else {
        int ce = 0, cw = 0, count = 0;
        for (int i = 0; i < n; i++) {
            int rc = mg_solve_impl(c, P.mg_vcycles, cw);
            if (rc) return rc;
            run_sweeps(c, sweeps, ce, cw, count, (i == n - 1) ? sweeps - 2 : sweeps);
        }
    }
    BCG_CUDA_TRY(cudaGetLastError());
    timer_end(c, BCG_T_SWEEPS, (int)(c->launches - l0));
    return ctx_check_status(c);
}

/* ======================================================================== */
/* The legacy explicit agar solver: UpdateEnvArray_OxygenAcetate            */
/* (Nutrients.cpp:45-197) and nutrientDepletionAgar_OxygenAcetate           */
/* (Nutrients.cpp:857-1074).  The reference keeps them but calls neither    */
/* (Simulation.cpp:215-216, 283-284 are commented out); a host that turns   */
/* them back on calls these two entries in place of bcg_nutrient_update.    */
/*                                                                          */
/* Storage: FieldAgar and oldFieldAgar of every composite level, four       */
/* species (carbon, waste, oxygen, acetate), row z contiguous in x, made on */
/* the first call.  Elsewhere the multigrid solution rows 1..box_z_agar     */
/* stand for FieldAgar: each call loads carbon, oxygen and acetate from     */
/* them (and, after an agar solve, sets oldFieldAgar equal, as copyFromMG   */
/* does) and writes them back at the end.                                   */
/*                                                                          */
/* Points the reference leaves undefined: on levels > 0 the agar points     */
/* with BoxX/4 <= x < 3 BoxX/4, z < BoxZAgar/2 take second differences that */
/* are never initialised; no other point reads them.  They are not updated  */
/* here (and so add nothing to the convergence count).                      */
/* ======================================================================== */
#define LEG_SP 4                 /* species slots: 0 carbon, 1 waste, 2 oxygen, 3 acetate */
#define LEG_CHUNK 64             /* iterations queued between convergence checks */

struct LegArgs {
    NutConst n;
    int ZA;
    const int* bbox;
    EnvP cur, prev;
    WallP pw0;
    const double* inside;
    const double* ds;
    EnvX ex;
    AgarRow pag;                 /* previous agar row z = 0 per level (the wall reads it) */
    WallAll cw, pw;
    double* const* ca;           /* current agar planes, [level * 4 + species] */
    double* const* pa;           /* previous agar planes */
    double* snap_a;              /* colony acetate before this iteration's write (box_x * box_z) */
    double* snap_w;              /* wall level-0 acetate before this iteration's write (box_x) */
    double crit;
    DevStatus* st;
};

__device__ __forceinline__ bool leg_covered(int X, int ZA, int level, int x, int z)
{
    return level > 0 && x >= X / 4 && x < 3 * X / 4 && z <= ZA / 2 - 1;
}
/* the per-point test of Nutrients.cpp:98-101 */
__device__ __forceinline__ int leg_moved(double cur, double prev, double crit)
{
    return fabs(cur - prev) > crit * mx(0.1, fabs(cur));
}

struct Aga4 { double C, W, O, A; };
__device__ __forceinline__ Aga4 leg_get(double* const* t, int X, int level, int x, int z)
{
    const size_t i = (size_t)z * X + x;
    double* const* q = t + level * LEG_SP;
    Aga4 v; v.C = q[0][i]; v.W = q[1][i]; v.O = q[2][i]; v.A = q[3][i];
    return v;
}

/* UpdateAgarMultigrid_OxygenAcetate (Nutrients.cpp:661-803), NutrientGSI = 0;
 * returns the point's convergence count (carbon, oxygen, acetate) */
__device__ int leg_agar_point(const LegArgs& a, int level, int x, int z)
{
    const NutConst& n = a.n;
    const int X = n.X, ZA = a.ZA, LM = n.A;
    if (leg_covered(X, ZA, level, x, z)) return 0;
    const Aga4 c0 = leg_get(a.pa, X, level, x, z);
    const double h2l = n.BL * n.BL * (double)(1LL << (2 * level));
    double Cxx, Czz, Wxx, Wzz, Axx, Azz, Oxx, Ozz;
    if (z == 0) {
        const Aga4 up = leg_get(a.pa, X, level, x, 1);
        const double dW = a.cw.W[level][x], dC = a.cw.C[level][x], dA = a.cw.A[level][x], dO = a.cw.O[level][x];
        Wzz = (up.W + dW - 2.0 * c0.W) / h2l; Czz = (up.C + dC - 2.0 * c0.C) / h2l;
        Azz = (up.A + dA - 2.0 * c0.A) / h2l; Ozz = (up.O + dO - 2.0 * c0.O) / h2l;
    } else if (level > 0 && x >= X / 4 && x < 3 * X / 4 && z <= ZA / 2) {
        const Aga4 up = leg_get(a.pa, X, level, x, z + 1), dn = leg_get(a.pa, X, level - 1, x * 2 - X / 2, ZA - 1);
        Wzz = (up.W + dn.W - 2.0 * c0.W) / h2l; Czz = (up.C + dn.C - 2.0 * c0.C) / h2l;
        Azz = (up.A + dn.A - 2.0 * c0.A) / h2l; Ozz = (up.O + dn.O - 2.0 * c0.O) / h2l;
    } else if (level < LM - 1 && z == ZA - 1) {
        const int lx = x % 2;
        const Aga4 u2 = leg_get(a.pa, X, level, x, z - 2);
        const Aga4 q1 = leg_get(a.pa, X, level + 1, x / 2 + X / 4, ZA / 2);
        const Aga4 q2 = leg_get(a.pa, X, level + 1, (x / 2 + X / 4 + 1) % X, ZA / 2);
        Wzz = (u2.W + 1.0 / (lx + 1) * q1.W + lx * 1.0 / (lx + 1) * q2.W - 2.0 * c0.W) / 4 / h2l;
        Czz = (u2.C + 1.0 / (lx + 1) * q1.C + lx * 1.0 / (lx + 1) * q2.C - 2.0 * c0.C) / 4 / h2l;
        Azz = (u2.A + 1.0 / (lx + 1) * q1.A + lx * 1.0 / (lx + 1) * q2.A - 2.0 * c0.A) / 4 / h2l;
        Ozz = (u2.O + 1.0 / (lx + 1) * q1.O + lx * 1.0 / (lx + 1) * q2.O - 2.0 * c0.O) / 4 / h2l;
    } else if (level == LM - 1 && z == ZA - 1) {
        const Aga4 u1 = leg_get(a.pa, X, level, x, z - 1);
        Wzz = 2.0 * (u1.W - c0.W) / h2l; Czz = 2.0 * (u1.C - c0.C) / h2l;
        Azz = 2.0 * (u1.A - c0.A) / h2l; Ozz = 2.0 * (u1.O - c0.O) / h2l;
    } else {
        const Aga4 up = leg_get(a.pa, X, level, x, z + 1), dn = leg_get(a.pa, X, level, x, z - 1);
        Wzz = (up.W + dn.W - 2.0 * c0.W) / h2l; Czz = (up.C + dn.C - 2.0 * c0.C) / h2l;
        Azz = (up.A + dn.A - 2.0 * c0.A) / h2l; Ozz = (up.O + dn.O - 2.0 * c0.O) / h2l;
    }
    if (level > 0 && x >= X / 4 - 1 && x <= X * 3 / 4 && z <= ZA / 2 - 1) {
        /* x == X/4 - 1 or 3X/4 here (the columns between are covered) */
        const bool lo = (x == X / 4 - 1);
        const Aga4 s1 = leg_get(a.pa, X, level, lo ? x - 1 : x + 1, z);
        const Aga4 q = leg_get(a.pa, X, level - 1, lo ? 0 : X - 2, z * 2 + 1);
        Wxx = (s1.W + q.W - 2 * c0.W) / h2l; Cxx = (s1.C + q.C - 2 * c0.C) / h2l;
        Axx = (s1.A + q.A - 2 * c0.A) / h2l; Oxx = (s1.O + q.O - 2 * c0.O) / h2l;
    } else if (level < LM - 1 && (x == 0 || x == X - 1)) {
        const int lz = (z + 1) % 2;
        const int zq = (z - 1) / 2;
        const int xq = (x == 0) ? X / 4 - 1 : X * 3 / 4;
        const Aga4 s1 = leg_get(a.pa, X, level, x == 0 ? x + 2 : x - 1, z);
        const Aga4 q1 = leg_get(a.pa, X, level + 1, xq, zq), q2 = leg_get(a.pa, X, level + 1, xq, (zq + 1) % ZA);
        Wxx = s1.W + 1.0 / (lz + 1) * q1.W + lz * 1.0 / (lz + 1) * q2.W - 2 * c0.W;
        Cxx = s1.C + 1.0 / (lz + 1) * q1.C + lz * 1.0 / (lz + 1) * q2.C - 2 * c0.C;
        Axx = s1.A + 1.0 / (lz + 1) * q1.A + lz * 1.0 / (lz + 1) * q2.A - 2 * c0.A;
        Oxx = s1.O + 1.0 / (lz + 1) * q1.O + lz * 1.0 / (lz + 1) * q2.O - 2 * c0.O;
        if (x == 0) { Wxx = Wxx / 4 / h2l; Cxx = Cxx / 4 / h2l; Axx = Axx / 4 / h2l; Oxx = Oxx / 4 / h2l; }
        else { Wxx = Wxx / h2l; Cxx = Cxx / h2l; Axx = Axx / h2l; Oxx = Oxx / h2l; }
    } else if (level == LM - 1 && (x == 0 || x == X - 1)) {
        const Aga4 s1 = leg_get(a.pa, X, level, x == 0 ? x + 1 : x - 1, z);
        Wxx = (s1.W - 1 * c0.W) / h2l; Cxx = (s1.C - 1.0 * c0.C) / h2l; Axx = (s1.A - 1.0 * c0.A) / h2l;
        Oxx = (x == 0) ? (s1.O + n.max_o2 - 2 * c0.O) / h2l : (n.max_o2 + s1.O - 2 * c0.O) / h2l;
    } else {
        const Aga4 xm = leg_get(a.pa, X, level, x - 1, z), xp = leg_get(a.pa, X, level, x + 1, z);
        Wxx = (xm.W + xp.W - 2 * c0.W) / h2l; Cxx = (xm.C + xp.C - 2 * c0.C) / h2l;
        Axx = (xm.A + xp.A - 2 * c0.A) / h2l; Oxx = (xm.O + xp.O - 2 * c0.O) / h2l;
    }
    const size_t i = (size_t)z * X + x;
    double* const* o = a.ca + level * LEG_SP;
    const double Cnew = c0.C + n.dac * (Cxx + Czz) * n.cdt;
    const double Onew = c0.O + n.dao * (Oxx + Ozz) * n.cdt;
    const double C = mx(0.0, mn(Cnew, n.max_carbon)), O = mx(0.0, mn(Onew, n.max_o2));
    const double CAcenew = c0.A + n.daa * (Axx + Azz) * n.cdt;
    const double A = mx(0.0, CAcenew);
    const double Wnew = c0.W + n.daw * (Wxx + Wzz) * n.cdt;
    o[0][i] = C; o[1][i] = mx(0.0, Wnew); o[2][i] = O; o[3][i] = A;
    return leg_moved(C, c0.C, a.crit) + leg_moved(O, c0.O, a.crit) + leg_moved(A, c0.A, a.crit);
}

/* a colony point of the bounding box: UpdateEnvironment_OxygenAcetate where
 * DensityShiftP > DBL_EPSILON (no buffer solve; the surviving pH values are
 * computed after the last iteration), and its convergence count */
__device__ int leg_colony_point(const LegArgs& a, int x, int z)
{
    const NutConst& n = a.n;
    if (z >= n.Z || x >= n.X) return 0;
    if (x < a.bbox[0] || x > a.bbox[1] || z > a.bbox[2]) return 0;
    const size_t id = (size_t)x * n.Z + z;
    const double pC = a.prev.C[id], pA = a.prev.A[id], pO = a.prev.O[id];
    a.snap_a[id] = a.cur.A[id];
    colony_point<false, true>(n, x, z, a.bbox, a.cur, a.prev, a.pw0, a.inside, a.ds, a.ex, a.st);
    return leg_moved(a.cur.C[id], pC, a.crit) + leg_moved(a.cur.A[id], pA, a.crit) + leg_moved(a.cur.O[id], pO, a.crit);
}

__device__ int leg_wall(const LegArgs& a, int x)
{
    int cnt = 0;
    a.snap_w[x] = a.cw.A[0][x];
    for (int level = 0; level < a.n.A; level++) {
        const double pC = a.pw.C[level][x], pO = a.pw.O[level][x], pA = a.pw.A[level][x];
        wall_point(a.n, level, x, a.cur, a.pag, a.cw, a.pw, a.inside);
        cnt += leg_moved(a.cw.C[level][x], pC, a.crit) + leg_moved(a.cw.O[level][x], pO, a.crit) +
               leg_moved(a.cw.A[level][x], pA, a.crit);
    }
    return cnt;
}

/* One iteration (count `iter`) of UpdateEnvArray_OxygenAcetate.  Within an
 * iteration only the z = 0 chain depends on the current buffers: the wall
 * reads the colony row z = 0 and the agar row z = 0 reads the wall, before
 * this iteration writes them on even counts (the reference's loop runs the
 * agar first, then the wall, then the colony) and after on odd counts.  One
 * thread per x runs that chain in that order; every other point reads the
 * previous buffers only.  An iteration after the one that met the stopping
 * rule (count > min_iter and a zero convergence count) does nothing. */
template <bool EVEN>
__global__ void __launch_bounds__(256) k_leg_iter(LegArgs a, int iter, int min_iter, unsigned long long* conv)
{
    if (iter > 0 && iter - 1 > min_iter && conv[iter - 1] == 0) return;     /* the same for every thread */
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int X = a.n.X, Z = a.n.Z, ZA = a.ZA;
    const long nI = X, nC = (long)X * (Z - 1), nA = (long)a.n.A * X * (ZA - 1);
    int cnt = 0;
    if (t < nI) {
        const int x = (int)t;
        if (EVEN) {
            for (int level = 0; level < a.n.A; level++) cnt += leg_agar_point(a, level, x, 0);
            cnt += leg_wall(a, x);
            cnt += leg_colony_point(a, x, 0);
        } else {
            cnt += leg_colony_point(a, x, 0);
            cnt += leg_wall(a, x);
            for (int level = 0; level < a.n.A; level++) cnt += leg_agar_point(a, level, x, 0);
        }
    } else if (t < nI + nC) {
        const long u = t - nI;
        cnt = leg_colony_point(a, (int)(u / (Z - 1)), 1 + (int)(u % (Z - 1)));
    } else if (t < nI + nC + nA) {
        const long u = t - nI - nC;
        const long per = (long)X * (ZA - 1);
        const int level = (int)(u / per);
        const long r = u % per;
        cnt = leg_agar_point(a, level, (int)(r % X), 1 + (int)(r / X));
    }
    cnt = __reduce_add_sync(0xffffffffu, cnt);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(conv + iter, (unsigned long long)cnt);
}

/* the surviving acetate buffer solves (Nutrients.cpp:214-222) of one
 * environment buffer: pH, Hydrox, Acetic, Buffer from the 4-point average
 * of acetate around each inside point, as the buffer had it when it was last
 * the previous one; `a_snap`/`w_snap` hold those acetate values where the
 * last iteration overwrote them (null: the buffer's own) */
__global__ void k_leg_diag(NutConst n, const int* __restrict__ bbox, EnvP e, const double* __restrict__ wall_a,
                           const double* __restrict__ a_snap, const double* __restrict__ inside,
                           const double* __restrict__ ds)
{
    const int z = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * COLONY_COLS + threadIdx.y;
    const int Z = n.Z;
    if (z >= Z || x >= n.X) return;
    const int minx = bbox[0], maxx = bbox[1], maxz = bbox[2];
    if (x < minx || x > maxx || z > maxz) return;
    const size_t id = (size_t)x * Z + z;
    if (!(ds[id] > DBL_EPSILON) || x < 1 || x > n.X - 2 || z > Z - 2 || !(inside[id] > 0.5)) return;
    auto A = [&](int xx, int zz) {
        const size_t q = (size_t)xx * Z + zz;
        return (a_snap && xx >= minx && xx <= maxx && zz <= maxz) ? a_snap[q] : e.A[q];
    };
    double Agr;
    if (z == 0) Agr = (wall_a[x - 1] + A(x - 1, z) + wall_a[x] + A(x, z)) / 4.0;
    else Agr = (A(x - 1, z - 1) + A(x - 1, z) + A(x, z - 1) + A(x, z)) / 4.0;
    double ph, hy, ac, bu;
    buffer_solve(n, Agr, ph, hy, ac, bu);
    e.ph[id] = ph; e.hyd[id] = hy; e.ace[id] = ac; e.buf[id] = bu;
}

/* FieldAgar of level l (rows 1..ZA of the agar solution) <-> the legacy planes */
__global__ void k_leg_load(double* const* tab, int X, int ZA, int l, MgLvl L, int refresh_old, int store)
{
    const long r = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= (long)X * ZA) return;
    const int z = (int)(r / X), x = (int)(r % X);
    double* const* cur = tab + l * LEG_SP;
    double* const* old = tab + (BCG_MAX_AGAR_LEVELS + l) * LEG_SP;
    const size_t m = (size_t)(z + 1) * L.pitch + x;
    if (store) {
        L.s[0][m] = cur[0][r]; L.s[1][m] = cur[2][r]; L.s[2][m] = cur[3][r];
        return;
    }
    cur[0][r] = L.s[0][m]; cur[2][r] = L.s[1][m]; cur[3][r] = L.s[2][m];
    if (refresh_old)
        for (int sp = 0; sp < LEG_SP; sp++) old[sp][r] = cur[sp][r];
}

/* ---- nutrientDepletionAgar_OxygenAcetate ---------------------------------- */
/* finest level whose extent holds column x of a level-`lv` row (the
 * reference's ceil/floor of log2 in Nutrients.cpp:917-921, 947-951,
 * 1027-1031, worked out in integers; X/2 in integer division as there):
 * x < X/2: lv + ceil(log2(1 - 2x/X)), x > X/2: lv + floor(log2(2x/X - 1)) + 1,
 * else 0 */
__device__ __forceinline__ int leg_native_level(int x, int X, int lv)
{
    if (x < X / 2) {
        /* ceil(log2(u)), u = (X - 2x)/X in (0, 1]: -(largest k with 2^k (X - 2x) <= X) */
        int k = 0;
        while ((long long)(X - 2 * x) << (k + 1) <= (long long)X) k++;
        return lv - k;
    }
    if (x > X / 2) {
        /* floor(log2(v)), v = (2x - X)/X in (0, 1): -(smallest k with 2^k (2x - X) >= X) */
        int k = 0;
        while (((long long)(2 * x - X) << k) < (long long)X) k++;
        return lv - k + 1;
    }
    return 0;
}
/* level of restrictionAgar's source for row z (Nutrients.cpp:908):
 * max(ceil(log2((1+z) 2^(A-1) / ZA)), 0) */
__device__ __forceinline__ int leg_row_level(int z, int ZA, int A)
{
    const long long v = (long long)(1 + z) << (A - 1);
    if (v <= ZA) return 0;
    int k = 0;
    while (((long long)ZA << k) < v) k++;
    return k;
}

__global__ void k_dep_restrict(double* const* tab, int X, int ZA, int A)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)X * ZA) return;
    const int z = (int)(t / X), x = (int)(t % X);
    int l = leg_row_level(z, ZA, A);
    if (l < 0) l = 0;
    const int lx = leg_native_level(x, X, A - 1);
    if (lx > l) l = lx;
    if (l >= A - 1) return;
    const int x2 = (x - X / 2) * (1 << (A - 1 - l)) + X / 2;
    const int z2 = (z + 1) * (1 << (A - 1 - l)) - 1;
    const size_t src = (size_t)z2 * X + x2;
    double* const* c = tab + (A - 1) * LEG_SP;
    double* const* o = tab + (BCG_MAX_AGAR_LEVELS + A - 1) * LEG_SP;
    double* const* cs = tab + l * LEG_SP;
    double* const* os = tab + (BCG_MAX_AGAR_LEVELS + l) * LEG_SP;
    c[0][t] = cs[0][src]; c[3][t] = cs[3][src];
    o[0][t] = os[0][src]; o[3][t] = os[3][src];
}

/* one explicit step of UpdateDepletionAgar on the coarsest level, carbon and
 * acetate: dst = base + dt D (Cxx + Czz) with the second differences of
 * `lap` (the reference's in-place step reads the previous level and adds to
 * the current one, which the copy after each step makes equal) */
__global__ void k_dep_step(NutConst n, int ZA, int level, double dtd, const double* __restrict__ baseC,
                           const double* __restrict__ baseA, const double* __restrict__ lapC,
                           const double* __restrict__ lapA, double* dstC, double* dstA,
                           const double* __restrict__ inside)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int X = n.X;
    if (t >= (long)X * ZA) return;
    const int z = (int)(t / X), x = (int)(t % X);
    const double h2l = n.BL * n.BL * (double)(1LL << (2 * level));
    const double c0 = lapC[t], a0 = lapA[t];
    double Cxx, Axx, Czz, Azz;
    if (x == 0) {
        Cxx = (2 * lapC[t + 1] - 2 * c0) / h2l;
        Axx = (2 * lapA[t + 1] - 2 * a0) / h2l;
    } else if (x == X - 1) {
        Cxx = (lapC[t - 1] - c0) / h2l;
        Axx = (lapA[t - 1] - a0) / h2l;
    } else {
        Cxx = (lapC[t + 1] + lapC[t - 1] - 2 * c0) / h2l;
        Axx = (lapA[t + 1] + lapA[t - 1] - 2 * a0) / h2l;
    }
    if (z == 0) {
        int lx = leg_native_level(x, X, n.A - 1);
        if (lx < 0) lx = 0;
        const int xw = (x - X / 2) * (1 << (n.A - 1 - lx)) + X / 2;
        if (lx == 0 && inside[(size_t)xw * n.Z] > 0.5) {
            Czz = 0; Azz = 0;        /* the depletion flux is computed and never used */
        } else {
            const double pw2 = (double)(1LL << level);
            Czz = (lapC[t + X] + 0.0 * pw2 - c0) / h2l;
            Azz = (lapA[t + X] + 0.0 * pw2 - a0) / h2l;
        }
    } else if (z == ZA - 1) {
        Czz = (2 * lapC[t - X] - 2 * c0) / h2l;
        Azz = (2 * lapA[t - X] - 2 * a0) / h2l;
    } else {
        Czz = (lapC[t + X] + lapC[t - X] - 2 * c0) / h2l;
        Azz = (lapA[t + X] + lapA[t - X] - 2 * a0) / h2l;
    }
    dstC[t] = baseC[t] + dtd * n.dac * (Cxx + Czz);
    dstA[t] = baseA[t] + dtd * n.daa * (Axx + Azz);
}

/* interpolation (Nutrients.cpp:929-995): level l-1 from level l and the
 * walls, current and previous */
__global__ void k_dep_interp(double* const* tab, int X, int ZA, int l, WallAll cw, WallAll pw)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)X * ZA) return;
    const int z = (int)(t / X), x = (int)(t % X);
    double* const* c = tab + l * LEG_SP;
    double* const* o = tab + (BCG_MAX_AGAR_LEVELS + l) * LEG_SP;
    double a1 = 0, a2 = 0, c1 = 0, c2 = 0;
    if (z == 0) {
        for (int i1 = 0; i1 < 2; i1++) {
            const size_t q = (size_t)((x + i1) / 2 + X / 4);
            c1 += c[0][q] / 4; c2 += o[0][q] / 4;
            a1 += c[3][q] / 4; a2 += o[3][q] / 4;
        }
        int lx = leg_native_level(x, X, l);
        if (lx < 0) lx = 0;
        const int xw = (x - X / 2) * (1 << (l - lx)) + X / 2;
        c1 += cw.C[lx][xw] / 2; c2 += pw.C[lx][xw] / 2;
        a1 += cw.A[lx][xw] / 2; a2 += pw.A[lx][xw] / 2;
    } else {
        for (int i1 = 0; i1 < 2; i1++)
            for (int i2 = 0; i2 < 2; i2++) {
                const size_t q = (size_t)((z - i2) / 2) * X + (x + i1) / 2 + X / 4;
                c1 += c[0][q] / 4; c2 += o[0][q] / 4;
                a1 += c[3][q] / 4; a2 += o[3][q] / 4;
            }
    }
    double* const* cd = tab + (l - 1) * LEG_SP;
    double* const* od = tab + (BCG_MAX_AGAR_LEVELS + l - 1) * LEG_SP;
    cd[0][t] = c1; od[0][t] = c2; cd[3][t] = a1; od[3][t] = a2;
}

/* ---- host side ------------------------------------------------------------ */
static int leg_storage(bcg_ctx* c, int iters)
{
    const bcg_params& P = c->P;
    const size_t plane = (size_t)P.box_x * P.box_z_agar * sizeof(double);
    if (!c->leg[0][0][0]) {
        for (int b = 0; b < 2; b++)
            for (int l = 0; l < P.max_levels_mg; l++)
                for (int sp = 0; sp < LEG_SP; sp++) {
                    BCG_CUDA_TRY(cudaMalloc((void**)&c->leg[b][l][sp], plane));
                    /* LocalAga's waste default 0; the other species come from the agar rows */
                    BCG_CUDA_TRY(cudaMemsetAsync(c->leg[b][l][sp], 0, plane, c->stream));
                }
        BCG_CUDA_TRY(cudaMalloc((void**)&c->leg_snap, ((size_t)P.box_x * P.box_z + P.box_x) * sizeof(double)));
        c->leg_old_stale = 1;
    }
    if (c->leg_conv_cap < iters) {
        if (c->leg_conv) BCG_CUDA_TRY(cudaFree(c->leg_conv));
        c->leg_conv = nullptr;
        c->leg_conv_cap = 0;
        /* the first slots hold the pointer table: [buffer 0 | buffer 1] x levels x species */
        BCG_CUDA_TRY(cudaMalloc((void**)&c->leg_conv, (size_t)(iters + 2 * BCG_MAX_AGAR_LEVELS * LEG_SP) * 8));
        c->leg_conv_cap = iters;
    }
    double* tab[2 * BCG_MAX_AGAR_LEVELS * LEG_SP];
    for (int b = 0; b < 2; b++)
        for (int l = 0; l < BCG_MAX_AGAR_LEVELS; l++)
            for (int sp = 0; sp < LEG_SP; sp++) tab[(b * BCG_MAX_AGAR_LEVELS + l) * LEG_SP + sp] = c->leg[b][l][sp];
    BCG_CUDA_TRY(cudaMemcpyAsync(c->leg_conv, tab, sizeof(tab), cudaMemcpyHostToDevice, c->stream));
    BCG_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return BCG_OK;
}
static double* const* leg_tab(bcg_ctx* c, int b)
{
    return reinterpret_cast<double* const*>(c->leg_conv) + b * BCG_MAX_AGAR_LEVELS * LEG_SP;
}
static unsigned long long* leg_counts(bcg_ctx* c) { return c->leg_conv + 2 * BCG_MAX_AGAR_LEVELS * LEG_SP; }

/* load (store = 0) or write back (store = 1) FieldAgar through the agar rows */
static int leg_transfer(bcg_ctx* c, int store)
{
    const bcg_params& P = c->P;
    const long n = (long)P.box_x * P.box_z_agar;
    const int refresh = (!store && c->leg_old_stale) ? 1 : 0;
    for (int l = 0; l < P.max_levels_mg; l++) {
        k_leg_load<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(leg_tab(c, 0), P.box_x, P.box_z_agar, l,
                                                                       mg_lvl(c, l), refresh, store);
        c->launches++;
    }
    if (refresh) c->leg_old_stale = 0;
    BCG_CUDA_TRY(cudaGetLastError());
    return BCG_OK;
}

static AgarRow leg_agar_rows(bcg_ctx* c, int b)
{
    AgarRow a;
    for (int l = 0; l < BCG_MAX_AGAR_LEVELS; l++) { a.C[l] = a.O[l] = a.A[l] = a.W[l] = nullptr; }
    for (int l = 0; l < c->P.max_levels_mg; l++) {
        a.C[l] = c->leg[b][l][0]; a.W[l] = c->leg[b][l][1]; a.O[l] = c->leg[b][l][2]; a.A[l] = c->leg[b][l][3];
    }
    return a;
}

extern "C" int bcg_legacy_env_update(bcg_ctx* c, int min_iter, int max_iter, double conv_crit, int* iterations)
{
    if (!c || max_iter < 0 || conv_crit < 0) return BCG_E_ARG;
    if (c->P.nutrient_gsi != 0) return BCG_E_UNSUPPORTED;
    if (c->P.box_z_agar < 3) return BCG_E_UNSUPPORTED;
    const bcg_params& P = c->P;
    int rc = leg_storage(c, max_iter > 0 ? max_iter : 1);
    if (rc) return rc;
    mg_res0_materialise(c);
    if ((rc = leg_transfer(c, 0))) return rc;
    BCG_CUDA_TRY(cudaMemsetAsync(leg_counts(c), 0, sizeof(unsigned long long) * (size_t)(max_iter > 0 ? max_iter : 1), c->stream));
    timer_begin(c, BCG_T_SWEEPS);
    long long l0 = c->launches;
    LegArgs a;
    a.n = nut_const(c);
    a.ZA = P.box_z_agar;
    a.bbox = c->bbox;
    a.inside = c->inside;
    a.ds = c->ds;
    a.snap_a = c->leg_snap;
    a.snap_w = c->leg_snap + (size_t)P.box_x * P.box_z;
    a.crit = conv_crit;
    a.st = c->status;
    const long threads = (long)P.box_x + (long)P.box_x * (P.box_z - 1) + (long)P.max_levels_mg * P.box_x * (P.box_z_agar - 1);
    const unsigned blocks = (unsigned)((threads + 255) / 256);
    std::vector<unsigned long long> h((size_t)LEG_CHUNK);
    int count = max_iter;
    for (int i0 = 0; i0 < max_iter && count == max_iter; i0 += LEG_CHUNK) {
        const int i1 = i0 + LEG_CHUNK < max_iter ? i0 + LEG_CHUNK : max_iter;
        for (int it = i0; it < i1; it++) {
            const int b = it & 1;
            a.cur = envp(c, b); a.prev = envp(c, b ^ 1);
            a.cw = wall_all(c, b); a.pw = wall_all(c, b ^ 1);
            a.pw0 = WallP{a.pw.C[0], a.pw.W[0], a.pw.O[0], a.pw.A[0]};
            a.ca = leg_tab(c, b); a.pa = leg_tab(c, b ^ 1);
            a.pag = leg_agar_rows(c, b ^ 1);
            a.ex = EnvX{};
            if (b == 0) {
                double* const* x = c->env[0].extra;
                a.ex = EnvX{x[0], x[1], x[2], x[3], x[4], x[5], x[6]};
            }
            if (b == 0) k_leg_iter<true><<<blocks, 256, 0, c->stream>>>(a, it, min_iter, leg_counts(c));
            else k_leg_iter<false><<<blocks, 256, 0, c->stream>>>(a, it, min_iter, leg_counts(c));
            c->launches++;
        }
        BCG_CUDA_TRY(cudaGetLastError());
        BCG_CUDA_TRY(cudaMemcpyAsync(h.data(), leg_counts(c) + i0, sizeof(unsigned long long) * (size_t)(i1 - i0),
                                     cudaMemcpyDeviceToHost, c->stream));
        if ((rc = ctx_check_status(c))) return rc;
        for (int it = i0; it < i1; it++)
            if (it > min_iter && h[it - i0] == 0) { count = it + 1; break; }
    }
    /* the acetate buffer solves that survive: the last iteration's previous
     * buffer from its own values, the other from the values the last
     * iteration overwrote */
    if (count > 0) {
        const dim3 g((unsigned)((P.box_z + 31) / 32), (unsigned)((P.box_x + COLONY_COLS - 1) / COLONY_COLS)), bl(32, COLONY_COLS);
        const int f = count - 1;
        const int bp = (f + 1) & 1, bc = f & 1;
        NutConst n = nut_const(c);
        k_leg_diag<<<g, bl, 0, c->stream>>>(n, c->bbox, envp(c, bp), c->wal[bp].A[0], nullptr, c->inside, c->ds);
        c->launches++;
        if (f > 0) {
            k_leg_diag<<<g, bl, 0, c->stream>>>(n, c->bbox, envp(c, bc), a.snap_w, a.snap_a, c->inside, c->ds);
            c->launches++;
        }
    }
    if ((rc = leg_transfer(c, 1))) return rc;
    BCG_CUDA_TRY(cudaGetLastError());
    timer_end(c, BCG_T_SWEEPS, (int)(c->launches - l0));
    if (iterations) *iterations = count;
    return ctx_check_status(c);
}

extern "C" int bcg_legacy_agar_depletion(bcg_ctx* c, int* steps)
{
    if (!c) return BCG_E_ARG;
    const bcg_params& P = c->P;
    if (P.box_z_agar < 3 || P.box_x < 8) return BCG_E_UNSUPPORTED;
    int rc = leg_storage(c, 1);
    if (rc) return rc;
    mg_res0_materialise(c);
    if ((rc = leg_transfer(c, 0))) return rc;
    const int A = P.max_levels_mg, X = P.box_x, ZA = P.box_z_agar;
    const int level = A - 1;
    const double h2 = P.box_length * P.box_length * (double)(1LL << (2 * level));
    const double dtd = (P.diff_agar_ace < P.diff_agar_carbon ? P.diff_agar_ace : P.diff_agar_carbon) / 10 * h2;
    const int n = (int)(3600 * P.update_time * 740 / dtd);
    const long pts = (long)X * ZA;
    const unsigned blocks = (unsigned)((pts + 255) / 256);
    NutConst nc = nut_const(c);
    k_dep_restrict<<<blocks, 256, 0, c->stream>>>(leg_tab(c, 0), X, ZA, A);
    c->launches++;
    double *cC = c->leg[0][level][0], *cA = c->leg[0][level][3], *pC = c->leg[1][level][0], *pA = c->leg[1][level][3];
    /* count 0: the current level plus the step from the previous one */
    k_dep_step<<<blocks, 256, 0, c->stream>>>(nc, ZA, level, dtd, cC, cA, pC, pA, cC, cA, c->inside);
    c->launches++;
    /* then the two are equal after every step: alternate them */
    for (int s = 1; s <= n; s++) {
        double *sC = (s & 1) ? cC : pC, *sA = (s & 1) ? cA : pA, *dC = (s & 1) ? pC : cC, *dA = (s & 1) ? pA : cA;
        k_dep_step<<<blocks, 256, 0, c->stream>>>(nc, ZA, level, dtd, sC, sA, sC, sA, dC, dA, c->inside);
        c->launches++;
    }
    /* both hold the last step (the reference copies after every step) */
    double *lC = (n & 1) ? pC : cC, *lA = (n & 1) ? pA : cA, *oC = (n & 1) ? cC : pC, *oA = (n & 1) ? cA : pA;
    BCG_CUDA_TRY(cudaMemcpyAsync(oC, lC, pts * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    BCG_CUDA_TRY(cudaMemcpyAsync(oA, lA, pts * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    WallAll cw = wall_all(c, 0), pw = wall_all(c, 1);
    for (int l = A - 1; l > 0; l--) {
        k_dep_interp<<<blocks, 256, 0, c->stream>>>(leg_tab(c, 0), X, ZA, l, cw, pw);
        c->launches++;
    }
    if ((rc = leg_transfer(c, 1))) return rc;
    BCG_CUDA_TRY(cudaGetLastError());
    if (steps) *steps = n + 1;
    return ctx_check_status(c);
}
