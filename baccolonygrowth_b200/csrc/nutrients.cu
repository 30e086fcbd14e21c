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
template <bool DIAG>
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
        double fCgr_aer = Cgr / (Cgr + n.kc_aer), fCgr_ana = Cgr / (Cgr + n.kc_ana);
        double fAgr = Agr / (Agr + n.ka), fOgr = Ogr / (Ogr + n.ko), fIgr = 0;
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
        if (DIAG && ex.gca) {
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
struct AgarRow { const double *C[BCG_MAX_AGAR_LEVELS], *O[BCG_MAX_AGAR_LEVELS], *A[BCG_MAX_AGAR_LEVELS]; };

/* UpdateWallMultigrid_OxygenAcetate (Nutrients.cpp:509-659), Box_y = 1.
 * FieldAgar[l](x, 0) is the multigrid solution row 1 (copyFromMG); the agar
 * waste is never written by the solve and stays 0.  For level > 0 and
 * BoxX/4-1 < x < BoxX*3/4 the reference reads uninitialised second
 * differences; here they are 0 (those points are read by no other point
 * before the next solve overwrites them). */
__device__ __forceinline__ void wall_point(const NutConst& n, int level, int x, const EnvP& curenv, const AgarRow& ag,
                                           const WallAll& cw, const WallAll& pw, const double* __restrict__ inside)
{
    const int X = n.X;
    if (level == 0 && inside[(size_t)x * n.Z] > 0.5) {
        size_t i0 = (size_t)x * n.Z;
        double gC = ag.C[0][x], gO = ag.O[0][x], gA = ag.A[0][x], gW = 0.0;
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
    double gC = ag.C[level][x], gA = ag.A[level][x], gW = 0.0;
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
    for (int l = 0; l < BCG_MAX_AGAR_LEVELS; l++) { a.C[l] = nullptr; a.O[l] = nullptr; a.A[l] = nullptr; }
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
/* drop the cached graphs (a kernel shape of this context changed) */
void nutrient_graphs_drop(bcg_ctx* c)
{
    for (int g = 0; g < 2; g++)
        if (c->nutrient_graph[g]) { cudaGraphExecDestroy(c->nutrient_graph[g]); c->nutrient_graph[g] = nullptr; }
    c->nutrient_graph_sweeps = 0;
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
