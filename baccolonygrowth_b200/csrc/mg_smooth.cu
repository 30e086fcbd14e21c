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
 * cp.async.bulk.tensor loads, each into its own CTA, into a ring of NS stages per
 * warp, each stage with an mbarrier that its loads complete; the copy
 * engine zero-fills columns and rows outside the level, which is the value
 * the stencil reads there.  A step reads E at row r+1 and R at row r from
 * shared memory.  E rows r and r+1 live in two register sets that swap
 * roles every step, and R rows r-5 .. r in a lane-private window in shared
 * memory (each row stored twice, six slots apart, so that every read is a
 * fixed offset from the trip's base); the loop runs two steps a trip, a
 * stage is two rows, so a trip opens one stage and frees one.  The small
 * trip keeps the hot loop inside the instruction cache.  Results go
 * straight to global memory (E2, the other correction buffer).  Every wait
 * on an mbarrier is bounded: past about a second the warp records
 * BCG_E_TIMEOUT, waits (bounded again) for its loads still in flight, and
 * returns.
 *
 * Boundaries: interior points of interior rows take rx_in.  The side
 * columns (0 and nx), row 0 and row nz take the other cases of relax_val
 * through one branch-free form (ts_point) with per-column flags; a point
 * that keeps its value before smoothing finds it in its R slot, where the
 * row's load put E instead of R.  Steps whose rows are all interior and
 * inside the segment's relaxed range check only whether their finished row
 * is stored; a warp stores at most one side column, whose slot within the
 * lane's four is a template parameter, so only that slot pays for the
 * general form.
 *
 * Work split: W warps (by default one per resident slot, so that every SM
 * carries the same load) over the 3 x strips columns of the level, each
 * column cut into segments of equal cost (the first segment has no
 * warm-up rows and runs that many more rows of its own).
 */
#include <cuda.h>
#include <cudaTypedefs.h>
#include <string.h>
#include "ctx.cuh"
#include "mg.cuh"

#define TS_COLS 128          /* columns a warp loads */
#define TS_NR 2              /* rows per stage */
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
/* the R window: 6 slots of [parity][lane] pairs (the lane's even
 * columns, then its odd ones); row r of the walk sits in slot
 * (r - kw) mod 6 */
constexpr int ts_wslot_elems() { return 2 * 32; }
template <class T> constexpr int ts_win_bytes() { return 6 * ts_wslot_elems() * 2 * (int)sizeof(T); }
/* per warp: its ring, then its R window; after the warps', their mbarriers */
template <class T> constexpr int ts_warp_bytes() { return TS_NS * ts_stage_bytes<T>() + ts_win_bytes<T>(); }
template <class T> constexpr int ts_smem_bytes() { return TS_WARPS * (ts_warp_bytes<T>() + 8 * TS_NS); }

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

/* this lane's 4 values at byte offset OFF from a shared-space address.
 * Volatile, so that the loads stay after the mbarrier wait that covers
 * them and before the proxy fence that hands their slot back to the copy
 * engine. */
template <int OFF>
__device__ __forceinline__ void ts_lds(unsigned a, double (&v)[4])
{
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%4+%5];\n\tld.shared.v2.f64 {%2, %3}, [%4+%6];"
                 : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3]) : "r"(a), "n"(OFF), "n"(OFF + 16));
}
template <int OFF>
__device__ __forceinline__ void ts_lds(unsigned a, float (&v)[4])
{
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4+%5];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]) : "r"(a), "n"(OFF));
}
template <class T> struct Pair;
template <> struct Pair<double> { typedef double2 t; };
template <> struct Pair<float> { typedef float2 t; };

/* per-warp state that does not change along the rows */
struct TsArgs {
    int nx, nz, pitch, l, sp;
    int c0, col;            /* strip origin; this lane's first column */
    int kw, ks, ke;         /* first row relaxed, first and last+1 row stored */
    int r0;                 /* first row staged (kw - 1) */
    int nstage;             /* stages this warp loads */
    unsigned fl;            /* ts_col_flags of the lane's 4 columns, 8 bits each */
    unsigned sub;           /* keep-old bits of the lane's columns, 3 each (row types) */
    unsigned stm;           /* bit j: the lane stores its column j */
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
__device__ __forceinline__ void ts_issue(const TsMaps& maps, const TsArgs& g, unsigned ring_s, unsigned bar0, int j,
                                         int& issued)
{
    issued = j + 1;
    const int slot = j % TS_NS;
    const unsigned bar = bar0 + 8u * slot;
    const unsigned dst = ring_s + (unsigned)(slot * ts_stage_bytes<T>());
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(bar, (unsigned)ts_stage_bytes<T>());
    const int y = g.r0 + j * TS_NR;
    const CUtensorMap* me = g.sp == 0 ? &maps.e[0] : (g.sp == 1 ? &maps.e[1] : &maps.e[2]);
    const CUtensorMap* mr = g.sp == 0 ? &maps.r[0] : (g.sp == 1 ? &maps.r[1] : &maps.r[2]);
    tma_load_2d(dst, me, g.c0, y, bar);
    tma_load_2d(dst + ts_stage_bytes<T>() / 2, mr, g.c0, y, bar);
}

/* The shared-memory rows a trip reads.  Trip t (steps r = kw + 2t + P, P
 * = 0, 1) reads E rows r+1 and R rows r, staged rows 2t+1 .. 2t+3 counted
 * from r0: stage t (slot t mod NS) and stage t+1.  The R window keeps rows
 * r-5 .. r: row q in slots (q - kw) mod 6 and (q - kw) mod 6 + 6, so that
 * at step r row r-h sits h slots below slot (r - kw) mod 6 + 6, a fixed
 * offset from the trip's window base. */
template <class T>
struct TsTrip {
    unsigned cur, nxt;          /* shared-space address of this lane's columns in the slots of stages t, t+1 */
    typename Pair<T>::t* win;   /* this lane's entry of window slot b = 2 (t mod 3), which takes row 2t of the walk */
    int t;
    int wrap;                   /* 6 - b: the window offsets m >= wrap lie at slot b + m - 6 */
};
template <class T>
__device__ __forceinline__ void ts_trip(TsTrip<T>& tr, unsigned lane_ring, typename Pair<T>::t* lane_win, int t)
{
    static_assert(TS_NS == 3, "the window's slot follows the stage slot");
    const int q = t % TS_NS;
    tr.t = t;
    tr.cur = lane_ring + (unsigned)(q * ts_stage_bytes<T>());
    tr.nxt = lane_ring + (unsigned)((q == TS_NS - 1 ? 0 : q + 1) * ts_stage_bytes<T>());
    tr.win = lane_win + 2 * q * ts_wslot_elems();
    tr.wrap = 6 - 2 * q;
}

/* One row step, P = (r - kw) mod 2.  h1 = results of step r-1 (read only),
 * h2 = results of step r-2 on entry and of step r on exit; e0 = E row r,
 * ep = E row r+1 (loaded here; it held row r-1).  Returns false after a
 * timed-out wait (recorded in the status word). */
template <class T, int S, int SIDE, int P, bool CHECK>
__device__ __forceinline__ bool ts_step(const int r, const TsArgs& g, const TsTrip<T>& tr, unsigned ring_s,
                                        unsigned bar0, const TsMaps& maps, int& issued, T (&h1)[2 * S][2],
                                        T (&h2)[2 * S][2], const T (&e0)[4], T (&ep)[4], T* __restrict__ EO,
                                        long long& orow, const RelaxK<T>& K, DevStatus* st)
{
    constexpr int H = 2 * S;
    typedef typename Pair<T>::t T2;
    constexpr int RB = TS_NR * TS_COLS * (int)sizeof(T);    /* R box offset in a stage */
    constexpr int RW = TS_COLS * (int)sizeof(T);            /* one staged row */
    const int lane = threadIdx.x & 31;
    if (P == 0) {
        /* E row r+1 opens stage t+1 */
        const int j = tr.t + 1;
        if (j < g.nstage) {
            const bool ok = mbar_wait(bar0 + 8u * (j % TS_NS), (unsigned)((j / TS_NS) & 1));
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) dev_error(st, BCG_E_TIMEOUT, 0x5300 + g.sp);
                return false;
            }
        }
    } else {
        /* stage t was last read at P = 0 (R row 2t+1): its slot takes
         * stage t + NS */
        const int j = tr.t + TS_NS;
        __syncwarp();
        if (lane == 0 && j < g.nstage) ts_issue<T>(maps, g, ring_s, bar0, j, issued);
    }
    T rr[4];
    ts_lds<P * RW>(tr.nxt, ep);                              /* E row r+1: stage t+1, row P */
    if (P == 0) ts_lds<RB + RW>(tr.cur, rr);                 /* R row r: stage t, row 1 */
    else ts_lds<RB>(tr.nxt, rr);                             /*          stage t+1, row 0 */
    {
        /* a point that keeps its value before smoothing gets that value in
         * its R slot, which is what ts_point keeps (on interior rows only
         * the side column can keep it) */
        const int rt = !CHECK ? TS_ROW_IN : (r == 0 ? TS_ROW_BOT : (r == g.nz ? TS_ROW_TOP : TS_ROW_IN));
#pragma unroll
        for (int j = 0; j < 4; j++)
            if ((CHECK || j == SIDE) && ((g.sub >> (3 * j + rt)) & 1u)) rr[j] = e0[j];
        T2 ev, od;
        ev.x = rr[0]; ev.y = rr[2]; od.x = rr[1]; od.y = rr[3];
        T2* w = tr.win + P * ts_wslot_elems();
        w[0] = ev; w[32] = od;
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
        const int j0 = h & 1;
        /* R of row r-h at this half's columns */
        T2 rk;
        if (h == 0) { rk.x = rr[0]; rk.y = rr[2]; }
        else {
            /* row r-h sits at offset m = P + 6 - h (1..6) from slot b,
             * wrapped into the 6 slots: m = 6 always wraps (slot b), m = 1
             * never does (b <= 4), the others when m >= 6 - b */
            const int m = P + 6 - h;
            const T2* base = m == 6 ? tr.win - 6 * ts_wslot_elems()
                           : (m == 1 ? tr.win : (m >= tr.wrap ? tr.win - 6 * ts_wslot_elems() : tr.win));
            rk = base[m * ts_wslot_elems() + 32 * j0];
        }
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
            h2[h][0] = SIDE == c0 ? ts_point<T>(TS_ROW_IN, (g.fl >> (8 * c0)) & 3u, (g.fl >> (8 * c0 + 6)) & 1u, rk.x,
                                                h1[h][0], u0v, x0m, x0p, K)
                                  : rx_in(rk.x, h1[h][0], u0v, x0m, x0p, K);
            h2[h][1] = SIDE == c1 ? ts_point<T>(TS_ROW_IN, (g.fl >> (8 * c1)) & 3u, (g.fl >> (8 * c1 + 6)) & 1u, rk.y,
                                                h1[h][1], u1v, x1m, x1p, K)
                                  : rx_in(rk.y, h1[h][1], u1v, x1m, x1p, K);
        } else {
            h2[h][0] = ts_point<T>(rt, (g.fl >> (8 * c0 + 2 * rt)) & 3u, (g.fl >> (8 * c0 + 6)) & 1u, rk.x, h1[h][0],
                                   u0v, x0m, x0p, K);
            h2[h][1] = ts_point<T>(rt, (g.fl >> (8 * c1 + 2 * rt)) & 3u, (g.fl >> (8 * c1 + 6)) & 1u, rk.y, h1[h][1],
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
    if (kS >= g.ks && (!CHECK || kS < g.ke)) {
        T* dst = EO + orow;
        const T v[4] = {h1[H - 2][0], h2[H - 1][0], h1[H - 2][1], h2[H - 1][1]};
        if (SIDE < 0) {
            /* a strip without a side column stores whole pairs (FP64) or a
             * whole group of four (FP32): its stored range starts on a pair
             * (group) boundary and ends inside the level */
            if (sizeof(T) == 8) {
                double2* d2 = reinterpret_cast<double2*>(dst);
                if (g.stm & 1u) d2[0] = make_double2((double)v[0], (double)v[1]);
                if (g.stm & 4u) d2[1] = make_double2((double)v[2], (double)v[3]);
            } else if (g.stm & 1u) {
                *reinterpret_cast<float4*>(dst) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
            }
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++)
                if ((g.stm >> j) & 1u) dst[j] = v[j];
        }
    }
    orow += g.pitch;
    return true;
}

/* the row loop, two steps a trip (E rows and the half-sweep results
 * alternate between two register sets) */
template <class T, int S, int SIDE>
__device__ __forceinline__ bool ts_rows(const TsArgs& g, unsigned ring_s, typename Pair<T>::t* lane_win, unsigned bar0,
                                        const TsMaps& maps, int& issued, T (&EA)[4], T* __restrict__ EO,
                                        const RelaxK<T>& K, DevStatus* st)
{
    constexpr int H = 2 * S;
    const int r_end = g.ke - 1 + (H - 1);
    const unsigned lane_ring = ring_s + 4 * sizeof(T) * (threadIdx.x & 31);
    T EB[4];
    T a[H][2], b[H][2];
    {
        /* the half-sweeps start from row kw-1 (stage 0, row 0) */
        T e[4];
        ts_lds<0>(lane_ring, e);
#pragma unroll
        for (int h = 0; h < H; h++) {
            a[h][0] = b[h][0] = e[(h & 1)];
            a[h][1] = b[h][1] = e[(h & 1) + 2];
        }
#pragma unroll
        for (int q = 0; q < 4; q++) EB[q] = e[q];
    }
    /* offset of the lane's columns in row r - (H-1), the row a step finishes */
    long long orow = (long long)(g.kw - (H - 1)) * g.pitch + g.col;
    TsTrip<T> tr;
    ts_trip<T>(tr, lane_ring, lane_win, 0);
    /* steps r >= st_lo have rows r-H+1 .. r at or above the warm start and
     * row 1; steps r <= st_hi at or below the last stored row and row nz-1:
     * such steps check only whether their finished row is stored (not in
     * the warm-up rows), so that the few checked trips of a segment are
     * all that leave the trip the warp spends its time in */
    const int st_lo = max(g.kw, 1) + (H - 1);
    const int st_hi = min(g.ke - 1, g.nz - 1);
    for (int r = g.kw; r <= r_end; r += 2) {
        if (r >= st_lo && r + 1 <= st_hi) {
            if (!ts_step<T, S, SIDE, 0, false>(r, g, tr, ring_s, bar0, maps, issued, a, b, EA, EB, EO, orow, K, st)) return false;
            if (!ts_step<T, S, SIDE, 1, false>(r + 1, g, tr, ring_s, bar0, maps, issued, b, a, EB, EA, EO, orow, K, st)) return false;
        } else {
            if (!ts_step<T, S, SIDE, 0, true>(r, g, tr, ring_s, bar0, maps, issued, a, b, EA, EB, EO, orow, K, st)) return false;
            if (r + 1 > r_end) break;
            if (!ts_step<T, S, SIDE, 1, true>(r + 1, g, tr, ring_s, bar0, maps, issued, b, a, EB, EA, EO, orow, K, st)) return false;
        }
        ts_trip<T>(tr, lane_ring, lane_win, tr.t + 1);
    }
    return true;
}

/* How a launch cuts the level: W warps over C = 3 x strips columns (a
 * strip of one species), the first `extra` columns in base+1 row segments,
 * the others in base.  The segments of a column cost the same: the first
 * runs `chunk` rows, the others chunk - warm rows after their warm rows. */
struct TsPlan { int W, nstrips, base, extra, warm, rows; };

/* warp gw's strip, species and stored rows ks .. ke-1; false: no rows */
__device__ __forceinline__ bool ts_assign(int gw, const TsPlan& pl, int& strip, int& sp, int& ks, int& ke)
{
    if (gw >= pl.W) return false;
    int c, s, n;
    const int big = pl.extra * (pl.base + 1);
    if (gw < big) {
        n = pl.base + 1; c = gw / n; s = gw - c * n;
    } else {
        n = pl.base;
        const int q = gw - big;
        c = pl.extra + q / n; s = q - (c - pl.extra) * n;
    }
    sp = c / pl.nstrips;
    strip = c - sp * pl.nstrips;
    const int chunk = (pl.rows + (n - 1) * pl.warm + n - 1) / n;
    ks = s == 0 ? 0 : chunk + (s - 1) * (chunk - pl.warm);
    ke = min(ks + (s == 0 ? chunk : chunk - pl.warm), pl.rows);
    return ks < pl.rows;
}

/* Six blocks (twelve warps) an SM; the shared memory of a block (two rings
 * and two R windows, 36.9 KB in FP64) allows no more. */
template <class T, int S>
__global__ void __launch_bounds__(32 * TS_WARPS, 6) k_mg_smooth_tma(const __grid_constant__ TsMaps maps, const __grid_constant__ MgConst m,
                                                      const __grid_constant__ MgLvlT<T> L, int l, TsPlan pl,
                                                      const double* __restrict__ inside0, DevStatus* st)
{
    constexpr int H = 2 * S;
    extern __shared__ __align__(128) unsigned char ts_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    TsArgs g;
    int strip, sp;
    if (!ts_assign((int)blockIdx.x * TS_WARPS + warp, pl, strip, sp, g.ks, g.ke)) return;    /* whole warp (no block-wide barrier follows) */
    g.nx = L.nx; g.nz = L.nz; g.pitch = L.pitch; g.l = l; g.sp = sp;
    g.c0 = strip * TsGeom<T>::WV - TsGeom<T>::HL;
    g.col = g.c0 + 4 * lane;
    g.kw = max(0, g.ks - pl.warm);
    g.r0 = g.kw - 1;
    const int r_end = g.ke - 1 + (H - 1);
    /* rows r0 .. r_end + 1 */
    g.nstage = (r_end + 1 - g.r0) / TS_NR + 1;
    int side_slot = -1;
    g.stm = 0;
    g.fl = 0;
    g.sub = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int i = g.col + j;
        unsigned sb;
        g.fl |= ts_col_flags(m, i, g.nx, l, g.sp, inside0, &sb) << (8 * j);
        g.sub |= sb << (3 * j);
        const bool st = i >= g.c0 + TsGeom<T>::HL && i < g.c0 + TsGeom<T>::HL + TsGeom<T>::WV && i >= 0 && i <= g.nx;
        g.stm |= (unsigned)st << j;
        /* a side column in the strip's halo is in the columns that go
         * stale anyway: only a stored one needs its own form */
        if (st && (i == 0 || i == g.nx)) side_slot = j;
    }
    /* the column slot of the warp's side column, -1 if it stores none (the
     * host gives this kernel only levels whose two sides are in different
     * strips) */
    side_slot = __reduce_max_sync(0xffffffffu, side_slot);
    /* the warps' rings and R windows, then their mbarriers */
    unsigned char* wbase = ts_smem + (size_t)warp * ts_warp_bytes<T>();
    const unsigned ring_s = smem_u32(wbase);
    typename Pair<T>::t* lane_win = reinterpret_cast<typename Pair<T>::t*>(wbase + TS_NS * ts_stage_bytes<T>()) + lane;
    const unsigned bar0 = smem_u32(ts_smem + TS_WARPS * ts_warp_bytes<T>() + 8 * TS_NS * warp);
    if (lane == 0) {
        for (int s = 0; s < TS_NS; s++) mbar_init(bar0 + 8u * s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    int issued = 0;             /* stages issued so far (kept by lane 0) */
    if (lane == 0)
        for (int j = 0; j < TS_NS && j < g.nstage; j++) ts_issue<T>(maps, g, ring_s, bar0, j, issued);
    /* rows kw-1 and kw (stage 0) into registers */
    bool ok = __all_sync(0xffffffffu, mbar_wait(bar0, 0));
    if (!ok) {
        if (lane == 0) dev_error(st, BCG_E_TIMEOUT, 0x5300 + g.sp);
    } else {
        const RelaxK<T> K = relax_k<T>(m, l, g.sp);
        T* __restrict__ EO = g.sp == 0 ? L.e2[0] : (g.sp == 1 ? L.e2[1] : L.e2[2]);
        /* E row kw: stage 0, row 1 */
        T EA[4];
        ts_lds<TS_COLS * (int)sizeof(T)>(ring_s + 4 * sizeof(T) * lane, EA);
        switch (side_slot) {
        case 0: ok = ts_rows<T, S, 0>(g, ring_s, lane_win, bar0, maps, issued, EA, EO, K, st); break;
        case 1: ok = ts_rows<T, S, 1>(g, ring_s, lane_win, bar0, maps, issued, EA, EO, K, st); break;
        case 2: ok = ts_rows<T, S, 2>(g, ring_s, lane_win, bar0, maps, issued, EA, EO, K, st); break;
        case 3: ok = ts_rows<T, S, 3>(g, ring_s, lane_win, bar0, maps, issued, EA, EO, K, st); break;
        default: ok = ts_rows<T, S, -1>(g, ring_s, lane_win, bar0, maps, issued, EA, EO, K, st); break;
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

/* resident warps of the kernel on the current device (blocks an SM x SMs
 * x warps a block); looked up once per device and precision */
template <class T>
static int ts_slots()
{
    static int slots[2][64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) { cudaGetLastError(); return 0; }
    int& v = slots[sizeof(T) == 8][dev];
    if (v == 0) {
        int sms = 0, nb = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_mg_smooth_tma<T, 3>, 32 * TS_WARPS, ts_smem_bytes<T>()) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        v = sms * nb * TS_WARPS;
    }
    return v;
}

/* S (1..3) fused sweeps of level L: E -> E2 with about W warps (0: one per
 * resident slot), segments starting `warm` rows early */
template <class T>
static int ts_launch(bcg_ctx* c, const MgConst& m, const MgLvlT<T>& L, int l, int S, int W, int warm)
{
    TsMaps maps;
    memset(&maps, 0, sizeof(maps));
    for (int sp = 0; sp < 3; sp++) {
        int rc = ts_encode<T>(&maps.e[sp], L.e[sp], L.nx, L.nz, L.pitch);
        if (!rc) rc = ts_encode<T>(&maps.r[sp], L.r[sp], L.nx, L.nz, L.pitch);
        if (rc) return rc;
    }
    TsPlan pl;
    pl.rows = L.nz + 1;
    pl.warm = warm;
    pl.nstrips = ts_strips<T>(L.nx);
    const int C = 3 * pl.nstrips;
    /* segments a column may take: every segment after the first keeps at
     * least 16 rows of its own beyond its warm rows */
    int max_seg = 1;
    while (max_seg < pl.rows) {
        const int n = max_seg + 1;
        const int chunk = (pl.rows + (n - 1) * warm + n - 1) / n;
        if (chunk - warm < 16) break;
        max_seg = n;
    }
    if (W <= 0) W = ts_slots<T>();
    if (W < C) W = C;
    if (W > C * max_seg) W = C * max_seg;
    pl.W = W;
    pl.base = W / C;
    pl.extra = W % C;
    const dim3 grid((unsigned)((W + TS_WARPS - 1) / TS_WARPS));
    const size_t smem = ts_smem_bytes<T>();
    const int block = 32 * TS_WARPS;
    if (S == 3) k_mg_smooth_tma<T, 3><<<grid, block, smem, c->stream>>>(maps, m, L, l, pl, c->inside, c->status);
    else if (S == 2) k_mg_smooth_tma<T, 2><<<grid, block, smem, c->stream>>>(maps, m, L, l, pl, c->inside, c->status);
    else k_mg_smooth_tma<T, 1><<<grid, block, smem, c->stream>>>(maps, m, L, l, pl, c->inside, c->status);
    c->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { bcg_set_cuda_error(e); return BCG_E_CUDA; }
    return BCG_OK;
}

int mg_smooth_tma(bcg_ctx* c, const MgConst& m, const MgLvl& L, int l, int S, int target_warps, int warm)
{
    return ts_launch<double>(c, m, L, l, S, target_warps, warm);
}
int mg_smooth_tma(bcg_ctx* c, const MgConst& m, const MgLvlF& L, int l, int S, int target_warps, int warm)
{
    return ts_launch<float>(c, m, L, l, S, target_warps, warm);
}
int mg_smooth_tma_slots() { return ts_slots<double>(); }
/* each form's dynamic shared memory, and the whole of the SM's shared
 * memory for blocks (six FP64 blocks take 227.6 of its 228 KB with the
 * per-block reserve) */
int mg_smooth_tma_attributes()
{
    const int d = ts_smem_bytes<double>(), f = ts_smem_bytes<float>();
    const int all = cudaSharedmemCarveoutMaxShared;
    if (cudaFuncSetAttribute(k_mg_smooth_tma<double, 1>, cudaFuncAttributePreferredSharedMemoryCarveout, all) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_smooth_tma<double, 2>, cudaFuncAttributePreferredSharedMemoryCarveout, all) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_smooth_tma<double, 3>, cudaFuncAttributePreferredSharedMemoryCarveout, all) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_smooth_tma<float, 1>, cudaFuncAttributePreferredSharedMemoryCarveout, all) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_smooth_tma<float, 2>, cudaFuncAttributePreferredSharedMemoryCarveout, all) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_smooth_tma<float, 3>, cudaFuncAttributePreferredSharedMemoryCarveout, all) != cudaSuccess)
        return BCG_E_CUDA;
    if (cudaFuncSetAttribute(k_mg_smooth_tma<double, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, d) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_smooth_tma<double, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, d) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_smooth_tma<double, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, d) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_smooth_tma<float, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, f) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_smooth_tma<float, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, f) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_smooth_tma<float, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, f) != cudaSuccess)
        return BCG_E_CUDA;
    return BCG_OK;
}
/* the kernel keeps one side-column form per warp: a level whose columns 0
 * and nx fall in one strip goes to the other smoother */
int mg_smooth_tma_fits(int nx) { return ts_strips<double>(nx) >= 2 && ts_strips<float>(nx) >= 2; }
