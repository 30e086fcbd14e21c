/*
 * mg_smooth.cu -- the agar smoother on the large levels: S zebra sweeps of
 * relaxationAgarAtLevel (Multigrid.cpp:135-249) fused into one pass over
 * the rows, with the rows staged into shared memory by the tensor memory
 * accelerator (TMA).
 *
 * One warp owns a strip of 128 columns (lane t: columns c0+4t .. c0+4t+3,
 * two even and two odd) and one segment of rows of one species, and walks
 * the rows bottom to top.  The 2S half-sweeps (even columns, then odd
 * columns, per sweep) run as a pipeline: half-sweep h relaxes row k = r - h
 * at row step r.  Every input it needs was produced at step r-1 or r-2:
 *   even half of sweep s: the value above and the point itself from sweep
 *   s-1's even half (steps r-1, r-2), its odd neighbours from sweep s-1's
 *   odd half (step r-1; the left one of column c0+4t from lane t-1 by a
 *   shuffle);
 *   odd half of sweep s: likewise from sweep s-1's odd half, its even
 *   neighbours from sweep s's even half (step r-1; the right one of column
 *   c0+4t+3 from lane t+1);
 *   the value below from the half-sweep itself (step r-1);
 * so the 2S updates of a step are independent, and the recurrence along a
 * column is one fused multiply-add per row.  A half-sweep is exact where
 * its inputs were, so one column at each strip edge goes stale per
 * half-sweep: of the 128 columns a strip loads, the middle 116 (FP64) or
 * 112 (FP32) are written, and neighbouring strips overlap by the rest.
 * (tests/test_mg_schedules.py emulates this schedule against the
 * sequential order.)
 *
 * Segments other than the first start `warm` rows early from the
 * pre-smoothing values: the column recurrence contracts by at least
 * a = 1/2 / (cf + 2) per row, and warm is the smallest count with
 * a^warm warm^2 < 1e-18, so the start error is below rounding when the
 * segment's own rows begin.
 *
 * Staging: the rows of E (the correction before smoothing) and R (the
 * right-hand side) of the strip arrive as 128 x NR boxes through plain
 * (non-multicast) cp.async.bulk.tensor loads into a ring of NS stages per
 * warp, each stage with an mbarrier that its loads complete; the copy
 * engine zero-fills columns and rows outside the level, which is the value
 * the stencil reads there.  A step reads E at row r+1 and R at row r from
 * shared memory; rows r-1, r of E and r-5 .. r of R stay in registers,
 * whose slots the loop fixes by running six steps a trip (a stage is three
 * rows, so a trip covers two stages and the ring positions repeat).
 * Results go straight to global memory (E2, the other correction buffer).
 * Every wait on an mbarrier is bounded: past about a second the warp
 * records BCG_E_TIMEOUT, waits (bounded again) for its loads still in
 * flight, and returns.
 *
 * Boundaries: interior points of interior rows take rx_in.  The side
 * columns (0 and nx), row 0 and row nz take the other cases of relax_val
 * through one branch-free form (ts_point) with per-column flags; a point
 * that keeps its value before smoothing finds it in its R register slot,
 * where the row's load put E instead of R.  Steps whose rows are all
 * interior and inside the segment run without any per-step check; a warp
 * stores at most one side column, whose slot within the lane's four is a
 * template parameter, so only that slot pays for the general form.
 */
#include <cuda.h>
#include <cudaTypedefs.h>
#include <string.h>
#include "ctx.cuh"
#include "mg.cuh"

#define TS_COLS 128          /* columns a warp loads */
#define TS_NR 3              /* rows per stage */
#define TS_NS 3              /* stages per warp */
#define TS_WARPS 2           /* warps per block, each with its own strip and ring */
#define TS_WAIT_CYCLES (2000000000LL)   /* about one second at 2 GHz */

template <class T> struct TsGeom;
template <> struct TsGeom<double> { static constexpr int HL = 6, WV = 116; };
/* FP32: the strip origin must be a multiple of 4 columns (16 B) */
template <> struct TsGeom<float> { static constexpr int HL = 8, WV = 112; };

struct TsMaps { CUtensorMap e[3], r[3]; };

/* one stage: NR rows of E, then NR rows of R, TS_COLS values each */
template <class T> constexpr int ts_stage_elems() { return 2 * TS_NR * TS_COLS; }
template <class T> constexpr int ts_stage_bytes() { return ts_stage_elems<T>() * (int)sizeof(T); }
template <class T> constexpr int ts_ring_elems() { return TS_NS * ts_stage_elems<T>(); }
template <class T> constexpr int ts_smem_bytes() { return TS_WARPS * (TS_NS * ts_stage_bytes<T>() + 8 * TS_NS); }

/* ---- mbarrier and TMA primitives ---------------------------------------- */
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity)
{
    unsigned done;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}" : "=r"(done) : "r"(bar), "r"(parity) : "memory");
    return done != 0;
}
/* bounded wait for the phase of parity `parity` of an mbarrier */
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > TS_WAIT_CYCLES) return false;
    return true;
}
__device__ __forceinline__ void tma_load_2d(unsigned dst, const CUtensorMap* map, int x, int y, unsigned bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                 :: "r"(dst), "l"(map), "r"(x), "r"(y), "r"(bar) : "memory");
}

/* 4 consecutive values of a row in shared memory (this lane's columns) */
__device__ __forceinline__ void lds4(const double* p, double (&v)[4])
{
    double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void lds4(const float* p, float (&v)[4])
{
    float4 a = *reinterpret_cast<const float4*>(p);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}

/* per-warp state that does not change along the rows */
struct TsArgs {
    int nx, nz, pitch, l, sp;
    int c0, col;            /* strip origin; this lane's first column */
    int kw, ks, ke;         /* first row relaxed, first and last+1 row stored */
    int r0;                 /* first row staged (kw - 1) */
    int nstage;             /* stages this warp loads */
    unsigned fl;            /* ts_col_flags of the lane's 4 columns, 8 bits each */
    unsigned sub;           /* keep-old bits of the lane's columns, 3 each (row types) */
    bool st[4];             /* the lane stores that column */
};

/* Row types of the update: interior rows, row 0, row nz. */
#define TS_ROW_IN 0
#define TS_ROW_BOT 1
#define TS_ROW_TOP 2

/* How relax_val (the reference's relaxationAgarElementwise) treats column
 * i on each row type, as 8 flag bits: for row type t, bit 2t = the point
 * keeps a value (R, or its value before smoothing), bit 2t+1 = the side
 * form (the inner neighbour s1 with weight 1 instead of both horizontal
 * neighbours with weight 1/2); bit 6: s1 is the right neighbour (i = 0).
 * *sub gets 3 bits, one per row type: the kept value is the one before
 * smoothing, not R.  Columns off the level (the strip's halo) are plain
 * interior columns: their values feed no column of the level. */
__device__ __forceinline__ unsigned ts_col_flags(const MgConst& m, int i, int nx, int l, int sp,
                                                 const double* __restrict__ inside0, unsigned* sub)
{
    const bool on = i >= 0 && i <= nx;
    const bool side = on && (i == 0 || i == nx);
    const bool oxy = (sp == 1);
    const bool top = l >= m.A - 1;
    bool inside = false;
    if (on) {
        const int d = 1 << l;
        int i0 = (i - nx / 2) * d + m.box_x / 2;
        i0 = i0 < 0 ? 0 : (i0 > m.box_x - 1 ? m.box_x - 1 : i0);
        inside = inside0[(size_t)i0 * m.box_z] > 0;
    }
    /* interior rows: kind 3 (R) and 4 (kept) keep, kinds 1-2 the side form */
    const bool in_keep = side && (!top || oxy), in_side = side && top && !oxy;
    /* row 0: covered by the colony -> R; side: below the top levels kept,
     * oxygen R, else the corner form; others: oxygen R, else rx_k0 */
    const bool bot_keep = inside || (side && !top) || oxy, bot_side = side && !bot_keep;
    /* row nz: below the top levels kept; side: oxygen R, else the corner
     * form; others rx_top */
    const bool top_keep = !top || (side && oxy), top_side = side && !top_keep;
    *sub = (unsigned)(side && !top) | ((unsigned)(side && !top && !inside) << 1) | ((unsigned)(!top) << 2);
    if (!on) *sub = 0;
    return (unsigned)in_keep | ((unsigned)in_side << 1) | ((unsigned)bot_keep << 2) | ((unsigned)bot_side << 3) |
           ((unsigned)top_keep << 4) | ((unsigned)top_side << 5) | ((unsigned)(i == 0) << 6);
}

/* The update of one point in the form shared by every case of relax_val:
 *   fma(W1, V1, fma(w, X + U, fma(A, s1, c slot)))
 * with W1 = w, V1 = below, U = up on interior rows, W1 = inv and U = 0 on
 * rows 0 and nz (V1 = up on row 0, below on row nz), X = xm + xp and A = 0
 * for the plain forms, X = 0 and A = inv for the side and corner forms.
 * Each case gives the same operations as rx_in, rx_side, rx_k0, rx_top and
 * rx_corner (fma(0, s1, y) = y, fma(w, 0, y) = y, x + 0 = x), so the
 * results are the same bits.  `slot` is R, or the point's value before
 * smoothing where the point keeps it; f = the column's 2 flag bits for the
 * row type. */
template <class T>
__device__ __forceinline__ T ts_point(int rt, unsigned f, bool s1p, T slot, T b, T u, T xm, T xp, const RelaxK<T>& K)
{
    const bool side_form = (f & 2u) != 0;
    const T s1 = s1p ? xp : xm;
    const T A = side_form ? K.inv : T(0);
    const T X = side_form ? T(0) : xm + xp;
    const T U = rt == TS_ROW_IN ? u : T(0);
    const T W1 = rt == TS_ROW_IN ? K.w : K.inv;
    const T V1 = rt == TS_ROW_BOT ? u : b;
    const T out = fma(W1, V1, fma(K.w, X + U, fma(A, s1, K.c * slot)));
    return (f & 1u) ? slot : out;
}

/* issue the loads of stage j (rows r0 + j NR ...) into slot j mod NS (lane 0) */
template <class T>
__device__ __forceinline__ void ts_issue(const TsMaps& maps, const TsArgs& g, T* ring, unsigned bar0, int j, int& issued)
{
    issued = j + 1;
    const int slot = j % TS_NS;
    const unsigned bar = bar0 + 8u * slot;
    const unsigned dst = smem_u32(ring + (size_t)slot * ts_stage_elems<T>());
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(bar, (unsigned)ts_stage_bytes<T>());
    const int y = g.r0 + j * TS_NR;
    const CUtensorMap* me = g.sp == 0 ? &maps.e[0] : (g.sp == 1 ? &maps.e[1] : &maps.e[2]);
    const CUtensorMap* mr = g.sp == 0 ? &maps.r[0] : (g.sp == 1 ? &maps.r[1] : &maps.r[2]);
    tma_load_2d(dst, me, g.c0, y, bar);
    tma_load_2d(dst + ts_stage_bytes<T>() / 2, mr, g.c0, y, bar);
}

/* Ring pointers of one trip of six row steps (trip t: rows kw + 6t ..,
 * staged rows 6t .. 6t + 8 counted from r0): the slots of stages 2t,
 * 2t+1 and 2t+2.  The next trip's are those of 2t+2, 2t+3 = 2t (mod 3)
 * and 2t+4 = 2t+1 (mod 3). */
template <class T>
struct TsTrip {
    const T* p[3];
    int t;
};
/* shared-memory row q (0..8 within the trip's stages) of E or R, at this
 * lane's columns */
template <class T>
__device__ __forceinline__ const T* ts_row(const TsTrip<T>& tr, int q, bool is_r)
{
    return tr.p[q / TS_NR] + (is_r ? TS_NR * TS_COLS : 0) + (q % TS_NR) * TS_COLS + 4 * (threadIdx.x & 31);
}

/* One row step at phase P = (r - kw) mod 6 (fixes the register slots and
 * the ring rows).  h1 = results of step r-1 (read only), h2 = results of
 * step r-2 on entry and of step r on exit; Ew[q mod 3] = E row q for q =
 * r-1, r, r+1 (row r+1 loaded here); Rs[(q - kw + 1) mod 6] = R row q for
 * q = r-5 .. r (row r loaded here).  Returns false after a timed-out wait
 * (recorded in the status word). */
template <class T, int S, int SIDE, int P, bool CHECK>
__device__ __forceinline__ bool ts_step(const int r, const TsArgs& g, const TsTrip<T>& tr, T* ring, unsigned bar0,
                                        const TsMaps& maps, int& issued, T (&h1)[2 * S][2], T (&h2)[2 * S][2], T (&Ew)[3][4],
                                        T (&Rs)[6][4], T* __restrict__ EO, const RelaxK<T>& K, DevStatus* st)
{
    constexpr int H = 2 * S;
    const int lane = threadIdx.x & 31;
    /* E row r+1 is ring row 2+P of the trip, R row r ring row 1+P; stage
     * 2t+1 opens at P = 1 (E row 3), stage 2t+2 at P = 4 (E row 6) */
    if (P == 1 || P == 4) {
        const int j = 2 * tr.t + (P == 1 ? 1 : 2);
        if (j < g.nstage) {
            const int slot = j % TS_NS;
            const bool ok = mbar_wait(bar0 + 8u * slot, (unsigned)((j / TS_NS) & 1));
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) dev_error(st, BCG_E_TIMEOUT, 0x5300 + g.sp);
                return false;
            }
        }
    }
    /* stage 2t was last read at P = 1 (R row 2), stage 2t+1 at P = 4 (R
     * row 5): their slots take stages 2t+3 and 2t+4 */
    if (P == 2 || P == 5) {
        const int j = 2 * tr.t + (P == 2 ? 3 : 4);
        __syncwarp();
        if (lane == 0 && j < g.nstage) ts_issue<T>(maps, g, ring, bar0, j, issued);
    }
    lds4(ts_row<T>(tr, 2 + P, false), Ew[(2 + P) % 3]);
    lds4(ts_row<T>(tr, 1 + P, true), Rs[(1 + P) % 6]);
    const T (&e0)[4] = Ew[(1 + P) % 3];     /* row r */
    const T (&ep)[4] = Ew[(2 + P) % 3];     /* row r+1 */
    {
        /* a point that keeps its value before smoothing gets that value in
         * its R slot, which is what ts_point keeps (on interior rows only
         * the side column can keep it) */
        const int rt = !CHECK ? TS_ROW_IN : (r == 0 ? TS_ROW_BOT : (r == g.nz ? TS_ROW_TOP : TS_ROW_IN));
#pragma unroll
        for (int j = 0; j < 4; j++)
            if ((CHECK || j == SIDE) && ((g.sub >> (3 * j + rt)) & 1u)) Rs[(1 + P) % 6][j] = e0[j];
    }
    /* neighbours from other lanes: even half h reads the left lane's last
     * odd column, odd half h the right lane's first even column */
    T nb[H];
#pragma unroll
    for (int h = 0; h < H; h++) {
        if (h & 1) nb[h] = __shfl_down_sync(0xffffffffu, h1[h - 1][0], 1);
        else nb[h] = __shfl_up_sync(0xffffffffu, h == 0 ? e0[3] : h1[h - 1][1], 1);
    }
    const int lo = r - (H - 1);
    /* rows r-H+1 .. r all interior (0 < k < nz) */
    const bool inner = !CHECK || (lo > 0 && r < g.nz);
#pragma unroll
    for (int h = H - 1; h >= 0; h--) {
        const T (&rk)[4] = Rs[(1 + P - h + 6) % 6];
        const int j0 = h & 1;
        T x0m, x0p, x1m, x1p, u0v, u1v;
        if (j0) {
            x0m = h1[h - 1][0]; x0p = h1[h - 1][1]; x1m = h1[h - 1][1]; x1p = nb[h];
            u0v = h == 1 ? e0[1] : h1[h - 2][0]; u1v = h == 1 ? e0[3] : h1[h - 2][1];
        } else {
            const T o0 = h == 0 ? e0[1] : h1[h - 1][0], o1 = h == 0 ? e0[3] : h1[h - 1][1];
            x0m = nb[h]; x0p = o0; x1m = o0; x1p = o1;
            u0v = h == 0 ? ep[0] : h1[h - 2][0]; u1v = h == 0 ? ep[2] : h1[h - 2][1];
        }
        const int c0 = j0, c1 = j0 + 2;     /* the lane's columns of this parity */
        const int k = r - h;
        const int rt = inner ? TS_ROW_IN : (k == 0 ? TS_ROW_BOT : (k == g.nz ? TS_ROW_TOP : TS_ROW_IN));
        if (rt == TS_ROW_IN) {
            /* interior rows: the plain form, except in the column slot that
             * holds the warp's side column (flags 0 give the plain form's
             * operations there too) */
            h2[h][0] = SIDE == c0 ? ts_point<T>(TS_ROW_IN, (g.fl >> (8 * c0)) & 3u, (g.fl >> (8 * c0 + 6)) & 1u, rk[c0],
                                                h1[h][0], u0v, x0m, x0p, K)
                                  : rx_in(rk[c0], h1[h][0], u0v, x0m, x0p, K);
            h2[h][1] = SIDE == c1 ? ts_point<T>(TS_ROW_IN, (g.fl >> (8 * c1)) & 3u, (g.fl >> (8 * c1 + 6)) & 1u, rk[c1],
                                                h1[h][1], u1v, x1m, x1p, K)
                                  : rx_in(rk[c1], h1[h][1], u1v, x1m, x1p, K);
        } else {
            h2[h][0] = ts_point<T>(rt, (g.fl >> (8 * c0 + 2 * rt)) & 3u, (g.fl >> (8 * c0 + 6)) & 1u, rk[c0], h1[h][0],
                                   u0v, x0m, x0p, K);
            h2[h][1] = ts_point<T>(rt, (g.fl >> (8 * c1 + 2 * rt)) & 3u, (g.fl >> (8 * c1 + 6)) & 1u, rk[c1], h1[h][1],
                                   u1v, x1m, x1p, K);
        }
    }
    if (CHECK && (lo < g.kw || r > g.ke - 1 || !inner)) {
        /* ramp steps of the segment: half-sweeps whose row lies below the
         * warm start, above what the later half-sweeps need or above the
         * level keep their last value */
#pragma unroll
        for (int h = 0; h < H; h++) {
            const int k = r - h;
            if (k < g.kw || k > min(g.nz, g.ke - 1 + (H - 1 - h) / 2)) { h2[h][0] = h1[h][0]; h2[h][1] = h1[h][1]; }
        }
    }
    /* row r - (H-1) is final: even columns from the last even half one step
     * ago, odd columns from the last odd half now */
    const int kS = r - (H - 1);
    if (!CHECK || (kS >= g.ks && kS < g.ke)) {
        T* dst = EO + (size_t)kS * g.pitch + g.col;
        const T v[4] = {h1[H - 2][0], h2[H - 1][0], h1[H - 2][1], h2[H - 1][1]};
        if (g.st[0] && g.st[3]) {
            if (sizeof(T) == 8) {
                double2* d2 = reinterpret_cast<double2*>(dst);
                d2[0] = make_double2((double)v[0], (double)v[1]);
                d2[1] = make_double2((double)v[2], (double)v[3]);
            } else {
                *reinterpret_cast<float4*>(dst) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
            }
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (g.st[j]) dst[j] = v[j];
        }
    }
    return true;
}

/* the row loop, six steps a trip (the phases fix every register slot) */
template <class T, int S, int SIDE>
__device__ __forceinline__ bool ts_rows(const TsArgs& g, T* ring, unsigned bar0, const TsMaps& maps, int& issued, T (&Ew)[3][4],
                                        T* __restrict__ EO, const RelaxK<T>& K, DevStatus* st)
{
    constexpr int H = 2 * S;
    const int r_end = g.ke - 1 + (H - 1);
    T Rs[6][4];
#pragma unroll
    for (int q = 0; q < 6; q++)
#pragma unroll
        for (int j = 0; j < 4; j++) Rs[q][j] = T(0);
    T a[H][2], b[H][2];
#pragma unroll
    for (int h = 0; h < H; h++) {
        a[h][0] = b[h][0] = Ew[0][(h & 1)];
        a[h][1] = b[h][1] = Ew[0][(h & 1) + 2];
    }
    TsTrip<T> tr;
    tr.t = 0;
    tr.p[0] = ring;
    tr.p[1] = ring + ts_stage_elems<T>();
    tr.p[2] = ring + 2 * ts_stage_elems<T>();
    /* steps r >= st_lo have rows r-H+1 .. r at or above the warm start, the
     * first stored row and row 1; steps r <= st_hi at or below the last
     * stored row and row nz-1: such steps need no checks */
    const int st_lo = max(max(g.kw, g.ks), 1) + (H - 1);
    const int st_hi = min(g.ke - 1, g.nz - 1);
    for (int r = g.kw; r <= r_end; r += 6) {
        if (r >= st_lo && r + 5 <= st_hi) {
            if (!ts_step<T, S, SIDE, 0, false>(r, g, tr, ring, bar0, maps, issued, a, b, Ew, Rs, EO, K, st)) return false;
            if (!ts_step<T, S, SIDE, 1, false>(r + 1, g, tr, ring, bar0, maps, issued, b, a, Ew, Rs, EO, K, st)) return false;
            if (!ts_step<T, S, SIDE, 2, false>(r + 2, g, tr, ring, bar0, maps, issued, a, b, Ew, Rs, EO, K, st)) return false;
            if (!ts_step<T, S, SIDE, 3, false>(r + 3, g, tr, ring, bar0, maps, issued, b, a, Ew, Rs, EO, K, st)) return false;
            if (!ts_step<T, S, SIDE, 4, false>(r + 4, g, tr, ring, bar0, maps, issued, a, b, Ew, Rs, EO, K, st)) return false;
            if (!ts_step<T, S, SIDE, 5, false>(r + 5, g, tr, ring, bar0, maps, issued, b, a, Ew, Rs, EO, K, st)) return false;
        } else {
            if (!ts_step<T, S, SIDE, 0, true>(r, g, tr, ring, bar0, maps, issued, a, b, Ew, Rs, EO, K, st)) return false;
            if (r + 1 > r_end) break;
            if (!ts_step<T, S, SIDE, 1, true>(r + 1, g, tr, ring, bar0, maps, issued, b, a, Ew, Rs, EO, K, st)) return false;
            if (r + 2 > r_end) break;
            if (!ts_step<T, S, SIDE, 2, true>(r + 2, g, tr, ring, bar0, maps, issued, a, b, Ew, Rs, EO, K, st)) return false;
            if (r + 3 > r_end) break;
            if (!ts_step<T, S, SIDE, 3, true>(r + 3, g, tr, ring, bar0, maps, issued, b, a, Ew, Rs, EO, K, st)) return false;
            if (r + 4 > r_end) break;
            if (!ts_step<T, S, SIDE, 4, true>(r + 4, g, tr, ring, bar0, maps, issued, a, b, Ew, Rs, EO, K, st)) return false;
            if (r + 5 > r_end) break;
            if (!ts_step<T, S, SIDE, 5, true>(r + 5, g, tr, ring, bar0, maps, issued, b, a, Ew, Rs, EO, K, st)) return false;
        }
        const T* q0 = tr.p[0];
        tr.p[0] = tr.p[2];
        tr.p[2] = tr.p[1];
        tr.p[1] = q0;
        tr.t++;
    }
    return true;
}

/* Four blocks (eight warps) an SM: the row step's twelve independent
 * updates need about 220 registers a thread to be scheduled side by side;
 * capping them at 168 for a third warp per scheduler spills and measured
 * slower (0.152-0.166 ms against 0.123 ms per level-0 launch of the
 * 4609 x 1025 grid). */
template <class T, int S>
__global__ void __launch_bounds__(32 * TS_WARPS, 4) k_mg_smooth_tma(const __grid_constant__ TsMaps maps, const __grid_constant__ MgConst m,
                                                      const __grid_constant__ MgLvlT<T> L, int l, int seg_len, int warm,
                                                      const double* __restrict__ inside0, DevStatus* st)
{
    constexpr int H = 2 * S;
    extern __shared__ __align__(128) unsigned char ts_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int strip = (int)blockIdx.x * TS_WARPS + warp;
    TsArgs g;
    g.nx = L.nx; g.nz = L.nz; g.pitch = L.pitch; g.l = l; g.sp = blockIdx.z;
    g.c0 = strip * TsGeom<T>::WV - TsGeom<T>::HL;
    g.col = g.c0 + 4 * lane;
    g.ks = (int)blockIdx.y * seg_len;
    if (g.ks > g.nz || strip * TsGeom<T>::WV > g.nx) return;     /* whole warp (no block-wide barrier follows) */
    g.ke = min(g.ks + seg_len, g.nz + 1);
    g.kw = max(0, g.ks - warm);
    g.r0 = g.kw - 1;
    const int r_end = g.ke - 1 + (H - 1);
    /* rows r0 .. r_end + 1 */
    g.nstage = (r_end + 1 - g.r0) / TS_NR + 1;
    int side_slot = -1;
    g.fl = 0;
    g.sub = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int i = g.col + j;
        unsigned sb;
        g.fl |= ts_col_flags(m, i, g.nx, l, g.sp, inside0, &sb) << (8 * j);
        g.sub |= sb << (3 * j);
        g.st[j] = i >= g.c0 + TsGeom<T>::HL && i < g.c0 + TsGeom<T>::HL + TsGeom<T>::WV && i >= 0 && i <= g.nx;
        /* a side column in the strip's halo is in the columns that go
         * stale anyway: only a stored one needs its own form */
        if (g.st[j] && (i == 0 || i == g.nx)) side_slot = j;
    }
    /* the column slot of the warp's side column, -1 if it stores none (the
     * host gives this kernel only levels whose two sides are in different
     * strips) */
    side_slot = __reduce_max_sync(0xffffffffu, side_slot);
    /* the rings of the block's warps, then their mbarriers */
    T* ring = reinterpret_cast<T*>(ts_smem) + (size_t)warp * ts_ring_elems<T>();
    const unsigned bar0 = smem_u32(ts_smem + TS_WARPS * TS_NS * ts_stage_bytes<T>() + 8 * TS_NS * warp);
    if (lane == 0) {
        for (int s = 0; s < TS_NS; s++) mbar_init(bar0 + 8u * s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    int issued = 0;             /* stages issued so far (kept by lane 0) */
    if (lane == 0)
        for (int j = 0; j < TS_NS && j < g.nstage; j++) ts_issue<T>(maps, g, ring, bar0, j, issued);
    /* rows kw-1 and kw (stage 0) into registers */
    bool ok = __all_sync(0xffffffffu, mbar_wait(bar0, 0));
    if (!ok) {
        if (lane == 0) dev_error(st, BCG_E_TIMEOUT, 0x5300 + g.sp);
    } else {
        const RelaxK<T> K = relax_k<T>(m, l, g.sp);
        T* __restrict__ EO = g.sp == 0 ? L.e2[0] : (g.sp == 1 ? L.e2[1] : L.e2[2]);
        T Ew[3][4];
        lds4(ring + 4 * lane, Ew[0]);
        lds4(ring + TS_COLS + 4 * lane, Ew[1]);
#pragma unroll
        for (int q = 0; q < 4; q++) Ew[2][q] = T(0);
        switch (side_slot) {
        case 0: ok = ts_rows<T, S, 0>(g, ring, bar0, maps, issued, Ew, EO, K, st); break;
        case 1: ok = ts_rows<T, S, 1>(g, ring, bar0, maps, issued, Ew, EO, K, st); break;
        case 2: ok = ts_rows<T, S, 2>(g, ring, bar0, maps, issued, Ew, EO, K, st); break;
        case 3: ok = ts_rows<T, S, 3>(g, ring, bar0, maps, issued, Ew, EO, K, st); break;
        default: ok = ts_rows<T, S, -1>(g, ring, bar0, maps, issued, Ew, EO, K, st); break;
        }
    }
    /* every issued stage must have landed before the block's shared memory
     * goes away.  After a normal run each was waited for before its rows
     * were read; after a timeout, wait (bounded) for the latest stage of
     * each slot, which completes after the earlier ones of that slot. */
    if (lane == 0 && !ok) {
        for (int j = issued - TS_NS; j < issued; j++) {
            if (j < 0) continue;
            if (!mbar_wait(bar0 + 8u * (j % TS_NS), (unsigned)((j / TS_NS) & 1))) {
                dev_error(st, BCG_E_TIMEOUT, 0x5310 + g.sp);
                break;
            }
        }
    }
    __syncwarp();
}

/* ------------------------------------------------------------------------ */
/* host side                                                                 */
/* ------------------------------------------------------------------------ */
/* cuTensorMapEncodeTiled through the runtime's driver entry point (no link
 * against the driver library); looked up once, immutable afterwards */
static PFN_cuTensorMapEncodeTiled_v12000 ts_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        return (PFN_cuTensorMapEncodeTiled_v12000)p;
    }();
    return fn;
}

/* 2-D map of one plane: x = columns 0..nx (row pitch `pitch` elements),
 * y = rows 0..nz, boxes of TS_COLS x TS_NR, zero fill outside */
template <class T>
static int ts_encode(CUtensorMap* map, const T* base, int nx, int nz, int pitch)
{
    PFN_cuTensorMapEncodeTiled_v12000 fn = ts_encoder();
    if (!fn) return BCG_E_CUDA;
    const cuuint64_t dims[2] = {(cuuint64_t)(nx + 1), (cuuint64_t)(nz + 1)};
    const cuuint64_t strides[1] = {(cuuint64_t)pitch * sizeof(T)};
    const cuuint32_t box[2] = {TS_COLS, TS_NR};
    const cuuint32_t estr[2] = {1, 1};
    const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    CUresult r = fn(map, dt, 2, (void*)base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? BCG_OK : BCG_E_CUDA;
}

/* strips of a level (one warp each per segment and species) */
template <class T> static int ts_strips(int nx) { return (nx + 1 + TsGeom<T>::WV - 1) / TsGeom<T>::WV; }
template <class T> static int ts_blocks_x(int nx) { return (ts_strips<T>(nx) + TS_WARPS - 1) / TS_WARPS; }

/* S (1..3) fused sweeps of level L: E -> E2, the level cut into `nseg` row
 * segments that start `warm` rows early */
template <class T>
static int ts_launch(bcg_ctx* c, const MgConst& m, const MgLvlT<T>& L, int l, int S, int nseg, int warm)
{
    TsMaps maps;
    memset(&maps, 0, sizeof(maps));
    for (int sp = 0; sp < 3; sp++) {
        int rc = ts_encode<T>(&maps.e[sp], L.e[sp], L.nx, L.nz, L.pitch);
        if (!rc) rc = ts_encode<T>(&maps.r[sp], L.r[sp], L.nx, L.nz, L.pitch);
        if (rc) return rc;
    }
    const int rows = L.nz + 1;
    if (nseg < 1) nseg = 1;
    if (nseg > rows) nseg = rows;
    const int seg_len = (rows + nseg - 1) / nseg;
    nseg = (rows + seg_len - 1) / seg_len;
    dim3 grid((unsigned)ts_blocks_x<T>(L.nx), (unsigned)nseg, 3);
    const size_t smem = ts_smem_bytes<T>();
    const int block = 32 * TS_WARPS;
    if (S == 3) k_mg_smooth_tma<T, 3><<<grid, block, smem, c->stream>>>(maps, m, L, l, seg_len, warm, c->inside, c->status);
    else if (S == 2) k_mg_smooth_tma<T, 2><<<grid, block, smem, c->stream>>>(maps, m, L, l, seg_len, warm, c->inside, c->status);
    else k_mg_smooth_tma<T, 1><<<grid, block, smem, c->stream>>>(maps, m, L, l, seg_len, warm, c->inside, c->status);
    c->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { bcg_set_cuda_error(e); return BCG_E_CUDA; }
    return BCG_OK;
}

int mg_smooth_tma(bcg_ctx* c, const MgConst& m, const MgLvl& L, int l, int S, int target_warps, int warm)
{
    const int per_seg = 3 * ts_strips<double>(L.nx);
    return ts_launch<double>(c, m, L, l, S, (target_warps + per_seg / 2) / per_seg, warm);
}
int mg_smooth_tma(bcg_ctx* c, const MgConst& m, const MgLvlF& L, int l, int S, int target_warps, int warm)
{
    const int per_seg = 3 * ts_strips<float>(L.nx);
    return ts_launch<float>(c, m, L, l, S, (target_warps + per_seg / 2) / per_seg, warm);
}
int mg_smooth_tma_warps_per_segment(int nx) { return 3 * ts_strips<double>(nx); }
/* the kernel keeps one side-column form per warp: a level whose columns 0
 * and nx fall in one strip goes to the other smoother */
int mg_smooth_tma_fits(int nx) { return ts_strips<double>(nx) >= 2 && ts_strips<float>(nx) >= 2; }
