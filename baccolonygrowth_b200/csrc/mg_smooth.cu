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
 * shared memory; the rows below stay in registers.  Results go straight
 * to global memory (E2, the other correction buffer).  Every wait on an
 * mbarrier is bounded: past about a second the warp records
 * BCG_E_TIMEOUT, waits (bounded again) for its loads still in flight, and
 * returns.
 */
#include <cuda.h>
#include <cudaTypedefs.h>
#include <string.h>
#include "ctx.cuh"
#include "mg.cuh"

#define TS_COLS 128          /* columns a warp loads */
#define TS_NR 4              /* rows per stage */
#define TS_NS 4              /* stages per warp */
#define TS_WAIT_CYCLES (2000000000LL)   /* about one second at 2 GHz */

template <class T> struct TsGeom;
template <> struct TsGeom<double> { static constexpr int HL = 6, WV = 116; };
/* FP32: the strip origin must be a multiple of 4 columns (16 B) */
template <> struct TsGeom<float> { static constexpr int HL = 8, WV = 112; };

struct TsMaps { CUtensorMap e[3], r[3]; };

template <class T> constexpr int ts_stage_bytes() { return 2 * TS_NR * TS_COLS * (int)sizeof(T); }
template <class T> constexpr int ts_smem_bytes() { return TS_NS * ts_stage_bytes<T>() + 64; }

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
    int kind[4];            /* col_kind of the lane's columns (interior rows) */
    bool st[4];             /* the lane stores that column */
    bool plain;             /* no side column in the warp */
};

template <class T>
struct TsRing {
    T* buf;                 /* NS stages, each E box then R box */
    unsigned bar0;          /* shared address of the first mbarrier */
};

/* issue the loads of stage j (rows r0 + j NR ...) into its slot (lane 0) */
template <class T>
__device__ __forceinline__ void ts_issue(const TsMaps& maps, const TsArgs& g, const TsRing<T>& rg, int j, int& issued)
{
    issued = j + 1;
    const int slot = j % TS_NS;
    const unsigned bar = rg.bar0 + 8u * slot;
    const unsigned dst = smem_u32(rg.buf + (size_t)slot * (ts_stage_bytes<T>() / sizeof(T)));
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(bar, (unsigned)ts_stage_bytes<T>());
    const int y = g.r0 + j * TS_NR;
    const CUtensorMap* me = g.sp == 0 ? &maps.e[0] : (g.sp == 1 ? &maps.e[1] : &maps.e[2]);
    const CUtensorMap* mr = g.sp == 0 ? &maps.r[0] : (g.sp == 1 ? &maps.r[1] : &maps.r[2]);
    tma_load_2d(dst, me, g.c0, y, bar);
    tma_load_2d(dst + ts_stage_bytes<T>() / 2, mr, g.c0, y, bar);
}

/* shared-memory row q (E or R) of this lane's columns */
template <class T>
__device__ __forceinline__ const T* ts_row(const TsArgs& g, const TsRing<T>& rg, int q, bool is_r)
{
    const int u = q - g.r0;
    const int slot = (u / TS_NR) % TS_NS;
    const T* st = rg.buf + (size_t)slot * (ts_stage_bytes<T>() / sizeof(T));
    return st + (is_r ? TS_NR * TS_COLS : 0) + (u % TS_NR) * TS_COLS + 4 * (threadIdx.x & 31);
}

/* One row step, phase P = (r - kw) mod 6 (fixes the register slots):
 * h1 = results of step r-1 (read only), h2 = results of step r-2 on entry
 * and of step r on exit; Ew[q mod 3] = E row q for q = r-1, r, r+1; Rs[q
 * mod 6] = R row q for q = r-5 .. r.  Returns false after a timed-out
 * wait (recorded in the status word). */
template <class T, int S, int P>
__device__ __forceinline__ bool ts_step(const int r, const TsArgs& g, const TsRing<T>& rg, const TsMaps& maps, int& issued,
                                        T (&h1)[2 * S][2], T (&h2)[2 * S][2], T (&Ew)[3][4], T (&Rs)[6][4],
                                        T* __restrict__ EO, const MgConst& m, const RelaxK<T>& K,
                                        const double* __restrict__ inside0, DevStatus* st)
{
    constexpr int H = 2 * S;
    const int lane = threadIdx.x & 31;
    const int u1 = r + 1 - g.r0;
    if (u1 % TS_NR == 0) {
        /* E row r+1 opens stage jnext (issued NS-1 stages ago) */
        const int jnext = u1 / TS_NR;
        if (jnext < g.nstage) {
            const unsigned bar = rg.bar0 + 8u * (jnext % TS_NS);
            const bool ok = mbar_wait(bar, (unsigned)((jnext / TS_NS) & 1));
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) dev_error(st, BCG_E_TIMEOUT, 0x5300 + g.sp);
                return false;
            }
        }
    }
    const int u0 = r - g.r0;
    if (u0 % TS_NR == 0 && u0 > 0) {
        /* stage u0/NR - 1 (rows r-NR .. r-1) was last read in the previous
         * step (R row r-1): its slot takes stage u0/NR - 1 + NS */
        const int jfree = u0 / TS_NR - 1;
        __syncwarp();
        if (lane == 0 && jfree + TS_NS < g.nstage) ts_issue<T>(maps, g, rg, jfree + TS_NS, issued);
    }
    lds4(ts_row<T>(g, rg, r + 1, false), Ew[(P + 1) % 3]);
    lds4(ts_row<T>(g, rg, r, true), Rs[P]);
    const T (&em)[4] = Ew[(P + 2) % 3];     /* row r-1 */
    const T (&e0)[4] = Ew[P % 3];           /* row r */
    const T (&ep)[4] = Ew[(P + 1) % 3];     /* row r+1 */
    const bool interior = (r - (H - 1) >= g.kw) && (r - (H - 1) >= 1) && (r <= g.nz - 1) && (r <= g.ke - 1);
    /* neighbours from other lanes: even half h reads the left lane's last
     * odd column, odd half h the right lane's first even column */
    T nb[H];
#pragma unroll
    for (int h = 0; h < H; h++) {
        if (h & 1) nb[h] = __shfl_down_sync(0xffffffffu, h1[h - 1][0], 1);
        else nb[h] = __shfl_up_sync(0xffffffffu, h == 0 ? e0[3] : h1[h - 1][1], 1);
    }
    if (interior && g.plain) {
#pragma unroll
        for (int h = H - 1; h >= 0; h--) {
            const T (&rk)[4] = Rs[(P - h + 6) % 6];
            if (h & 1) {
                const T s0 = h1[h - 1][0], s1 = h1[h - 1][1];
                const T u0v = h == 1 ? e0[1] : h1[h - 2][0], u1v = h == 1 ? e0[3] : h1[h - 2][1];
                h2[h][0] = rx_in(rk[1], h1[h][0], u0v, s0, s1, K);
                h2[h][1] = rx_in(rk[3], h1[h][1], u1v, s1, nb[h], K);
            } else {
                const T o0 = h == 0 ? e0[1] : h1[h - 1][0], o1 = h == 0 ? e0[3] : h1[h - 1][1];
                const T u0v = h == 0 ? ep[0] : h1[h - 2][0], u1v = h == 0 ? ep[2] : h1[h - 2][1];
                h2[h][0] = rx_in(rk[0], h1[h][0], u0v, nb[h], o0, K);
                h2[h][1] = rx_in(rk[2], h1[h][1], u1v, o0, o1, K);
            }
        }
    } else {
#pragma unroll
        for (int h = H - 1; h >= 0; h--) {
            const int k = r - h;
            if (!interior) {
                const int top = min(g.nz, g.ke - 1 + (H - 1 - h) / 2);
                if (k < g.kw || k > top) { h2[h][0] = h1[h][0]; h2[h][1] = h1[h][1]; continue; }
            }
            const T (&rk)[4] = Rs[(P - h + 6) % 6];
            const int j0 = h & 1;
            T xm[2], xp[2], up[2], old[2];
            if (j0) {
                xm[0] = h1[h - 1][0]; xp[0] = h1[h - 1][1];
                xm[1] = h1[h - 1][1]; xp[1] = nb[h];
                up[0] = h == 1 ? e0[1] : h1[h - 2][0]; up[1] = h == 1 ? e0[3] : h1[h - 2][1];
                old[0] = h == 1 ? em[1] : h2[h - 2][0]; old[1] = h == 1 ? em[3] : h2[h - 2][1];
            } else {
                const T o0 = h == 0 ? e0[1] : h1[h - 1][0], o1 = h == 0 ? e0[3] : h1[h - 1][1];
                xm[0] = nb[h]; xp[0] = o0; xm[1] = o0; xp[1] = o1;
                up[0] = h == 0 ? ep[0] : h1[h - 2][0]; up[1] = h == 0 ? ep[2] : h1[h - 2][1];
                old[0] = h == 0 ? e0[0] : h2[h - 2][0]; old[1] = h == 0 ? e0[2] : h2[h - 2][1];
            }
#pragma unroll
            for (int j = 0; j < 2; j++) {
                if (k > 0 && k < g.nz)
                    h2[h][j] = rx_row<T>(g.kind[j0 + 2 * j], rk[j0 + 2 * j], h1[h][j], up[j], xm[j], xp[j], old[j], K);
                else
                    h2[h][j] = relax_val<T>(m, K, g.nx, g.nz, g.l, g.sp, g.col + j0 + 2 * j, k, rk[j0 + 2 * j],
                                            h1[h][j], up[j], xm[j], xp[j], old[j], inside0);
            }
        }
    }
    /* row r - (H-1) is final: even columns from the last even half one step
     * ago, odd columns from the last odd half now */
    const int kS = r - (H - 1);
    if (kS >= g.ks && kS < g.ke) {
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

template <class T, int S>
__global__ void __launch_bounds__(32) k_mg_smooth_tma(const __grid_constant__ TsMaps maps, MgConst m, MgLvlT<T> L,
                                                      int l, int seg_len, int warm, const double* __restrict__ inside0,
                                                      DevStatus* st)
{
    constexpr int H = 2 * S;
    extern __shared__ __align__(128) unsigned char ts_smem[];
    const int lane = threadIdx.x;
    TsArgs g;
    g.nx = L.nx; g.nz = L.nz; g.pitch = L.pitch; g.l = l; g.sp = blockIdx.z;
    g.c0 = (int)blockIdx.x * TsGeom<T>::WV - TsGeom<T>::HL;
    g.col = g.c0 + 4 * lane;
    g.ks = (int)blockIdx.y * seg_len;
    if (g.ks > g.nz || (int)blockIdx.x * TsGeom<T>::WV > g.nx) return;     /* whole warp */
    g.ke = min(g.ks + seg_len, g.nz + 1);
    g.kw = max(0, g.ks - warm);
    g.r0 = g.kw - 1;
    const int r_end = g.ke - 1 + (H - 1);
    /* rows r0 .. r_end + 1 */
    g.nstage = (r_end + 1 - g.r0) / TS_NR + 1;
    const bool oxy = (g.sp == 1);
    const bool top_levels = l >= m.A - 1;
    bool side = false;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int i = g.col + j;
        g.kind[j] = col_kind(i, g.nx, oxy, top_levels);
        side |= (i == 0 || i == g.nx);
        g.st[j] = i >= g.c0 + TsGeom<T>::HL && i < g.c0 + TsGeom<T>::HL + TsGeom<T>::WV && i >= 0 && i <= g.nx;
    }
    g.plain = !__any_sync(0xffffffffu, side);
    TsRing<T> rg;
    rg.buf = reinterpret_cast<T*>(ts_smem);
    rg.bar0 = smem_u32(ts_smem + TS_NS * ts_stage_bytes<T>());
    if (lane == 0) {
        for (int s = 0; s < TS_NS; s++) mbar_init(rg.bar0 + 8u * s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    int issued = 0;             /* stages issued so far (kept by lane 0) */
    if (lane == 0)
        for (int j = 0; j < TS_NS && j < g.nstage; j++) ts_issue<T>(maps, g, rg, j, issued);
    /* rows kw-1 and kw (stage 0) into registers */
    bool ok = __all_sync(0xffffffffu, mbar_wait(rg.bar0, 0));
    if (!ok) {
        if (lane == 0) dev_error(st, BCG_E_TIMEOUT, 0x5300 + g.sp);
    } else {
        const RelaxK<T> K = relax_k<T>(m, l, g.sp);
        T* __restrict__ EO = g.sp == 0 ? L.e2[0] : (g.sp == 1 ? L.e2[1] : L.e2[2]);
        T Ew[3][4], Rs[6][4];
        lds4(ts_row<T>(g, rg, g.kw - 1, false), Ew[2]);
        lds4(ts_row<T>(g, rg, g.kw, false), Ew[0]);
#pragma unroll
        for (int q = 0; q < 6; q++)
#pragma unroll
            for (int j = 0; j < 4; j++) Rs[q][j] = T(0);
        T a[H][2], b[H][2];
#pragma unroll
        for (int h = 0; h < H; h++) {
            a[h][0] = b[h][0] = Ew[2][(h & 1)];
            a[h][1] = b[h][1] = Ew[2][(h & 1) + 2];
        }
        for (int r = g.kw; r <= r_end; r += 6) {
            if (!ts_step<T, S, 0>(r, g, rg, maps, issued, a, b, Ew, Rs, EO, m, K, inside0, st)) { ok = false; break; }
            if (r + 1 > r_end) break;
            if (!ts_step<T, S, 1>(r + 1, g, rg, maps, issued, b, a, Ew, Rs, EO, m, K, inside0, st)) { ok = false; break; }
            if (r + 2 > r_end) break;
            if (!ts_step<T, S, 2>(r + 2, g, rg, maps, issued, a, b, Ew, Rs, EO, m, K, inside0, st)) { ok = false; break; }
            if (r + 3 > r_end) break;
            if (!ts_step<T, S, 3>(r + 3, g, rg, maps, issued, b, a, Ew, Rs, EO, m, K, inside0, st)) { ok = false; break; }
            if (r + 4 > r_end) break;
            if (!ts_step<T, S, 4>(r + 4, g, rg, maps, issued, a, b, Ew, Rs, EO, m, K, inside0, st)) { ok = false; break; }
            if (r + 5 > r_end) break;
            if (!ts_step<T, S, 5>(r + 5, g, rg, maps, issued, b, a, Ew, Rs, EO, m, K, inside0, st)) { ok = false; break; }
        }
    }
    /* every issued stage must have landed before the block's shared memory
     * goes away.  After a normal run each was waited for before its rows
     * were read; after a timeout, wait (bounded) for the latest stage of
     * each slot, which completes after the earlier ones of that slot. */
    if (lane == 0 && !ok) {
        for (int j = issued - TS_NS; j < issued; j++) {
            if (j < 0) continue;
            if (!mbar_wait(rg.bar0 + 8u * (j % TS_NS), (unsigned)((j / TS_NS) & 1))) {
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
    dim3 grid((unsigned)ts_strips<T>(L.nx), (unsigned)nseg, 3);
    const size_t smem = ts_smem_bytes<T>();
    if (S == 3) k_mg_smooth_tma<T, 3><<<grid, 32, smem, c->stream>>>(maps, m, L, l, seg_len, warm, c->inside, c->status);
    else if (S == 2) k_mg_smooth_tma<T, 2><<<grid, 32, smem, c->stream>>>(maps, m, L, l, seg_len, warm, c->inside, c->status);
    else k_mg_smooth_tma<T, 1><<<grid, 32, smem, c->stream>>>(maps, m, L, l, seg_len, warm, c->inside, c->status);
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
