/*
 * mech.cu -- cell binning, neighbour lists, the mechanics step (MoveCell +
 * GrowCell) and the division loop, as sm_100a kernels.
 *
 * Reference: AgentBasedModel-BacColonyGrowth/ UniformGrid.h, Neighbours.cpp,
 * Forces.cpp, Integrate.cpp, grow.cpp, Cells.cpp, Simulation.cpp:330-413.
 */
#include "ctx.cuh"
#include "cellmath.cuh"
#include "internal.h"
#include <string.h>

/* ======================================================================= */
/* binning: counting sort of cell ids by UniformGrid address               */
/* ======================================================================= */
__global__ void k_bin_count(int n, const CellRec* __restrict__ rec, MechParams mp,
                            int* __restrict__ cell_box, int* __restrict__ slot,
                            int* __restrict__ box_cnt, DevStatus* st)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 a = rec[i].pL, b = rec[i].qR;
    V3 cm = avg_pq(mk(a.x, a.y, a.z), mk(b.x, b.y, b.z));
    int xi, yi, zi;
    int box = box_address(cm, mp, xi, yi, zi);
    if (box < 0) { dev_error(st, BCG_E_OUT_OF_GRID, i); box = 0; }
    cell_box[i] = box;
    slot[i] = atomicAdd(&box_cnt[box], 1);
}

/* exclusive scan, 3 phases: per-block sums, scan of block sums, apply */
#define SCAN_BLOCK 1024
#define SCAN_ITEMS 4
__device__ __forceinline__ int block_excl_scan(int v, int* sh, int& total)
{
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int s = (lane < (blockDim.x >> 5)) ? sh[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, s, o); if (lane >= o) s += y; }
        sh[lane] = s;
    }
    __syncthreads();
    int pre = (wid > 0 ? sh[wid - 1] : 0) + x - v;
    total = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    return pre;
}
__global__ void k_scan_partial(int n, const int* __restrict__ in, int* __restrict__ block_sums)
{
    __shared__ int sh[32];
    long base = (long)blockIdx.x * SCAN_BLOCK * SCAN_ITEMS;
    int s = 0;
    for (int j = 0; j < SCAN_ITEMS; j++) {
        long idx = base + (long)threadIdx.x * SCAN_ITEMS + j;
        if (idx < n) s += in[idx];
    }
    int total;
    block_excl_scan(s, sh, total);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}
__global__ void k_scan_blocks(int nb, int* __restrict__ block_sums)
{
    __shared__ int sh[32];
    /* one block; nb <= SCAN_BLOCK * SCAN_ITEMS */
    int v[SCAN_ITEMS]; int s = 0;
    for (int j = 0; j < SCAN_ITEMS; j++) {
        int idx = threadIdx.x * SCAN_ITEMS + j;
        v[j] = idx < nb ? block_sums[idx] : 0;
        s += v[j];
    }
    int total;
    int pre = block_excl_scan(s, sh, total);
    for (int j = 0; j < SCAN_ITEMS; j++) {
        int idx = threadIdx.x * SCAN_ITEMS + j;
        if (idx < nb) block_sums[idx] = pre;
        pre += v[j];
    }
}
__global__ void k_scan_apply(int n, const int* __restrict__ in, const int* __restrict__ block_sums, int* __restrict__ out)
{
    __shared__ int sh[32];
    long base = (long)blockIdx.x * SCAN_BLOCK * SCAN_ITEMS;
    int v[SCAN_ITEMS]; int s = 0;
    for (int j = 0; j < SCAN_ITEMS; j++) {
        long idx = base + (long)threadIdx.x * SCAN_ITEMS + j;
        v[j] = idx < n ? in[idx] : 0;
        s += v[j];
    }
    int total;
    int pre = block_excl_scan(s, sh, total) + block_sums[blockIdx.x];
    for (int j = 0; j < SCAN_ITEMS; j++) {
        long idx = base + (long)threadIdx.x * SCAN_ITEMS + j;
        if (idx < n) out[idx] = pre;
        pre += v[j];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) out[n] = pre;
}

__global__ void k_bin_scatter(int n, const int* __restrict__ cell_box, const int* __restrict__ slot,
                              const int* __restrict__ box_start, int* __restrict__ box_ids)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    box_ids[box_start[cell_box[i]] + slot[i]] = i;
}

/* ascending ids inside each box (boxes hold at most max_cells_per_box - 1) */
__global__ void k_bin_sort(int nbox, const int* __restrict__ box_start, int* __restrict__ box_ids,
                           int box_cap, DevStatus* st)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbox) return;
    int s = box_start[b], e = box_start[b + 1];
    /* an overfull box is an error (UniformGrid.h:35); leave it unsorted so
     * that the work of this thread stays bounded */
    if (e - s > box_cap - 1) { dev_error(st, BCG_E_BOX_OVERFLOW, b); return; }
    for (int i = s + 1; i < e; i++) {
        int v = box_ids[i], j = i - 1;
        while (j >= s && box_ids[j] > v) { box_ids[j + 1] = box_ids[j]; j--; }
        box_ids[j + 1] = v;
    }
}

static int scan_exclusive(bcg_ctx* c, const int* in, int* out, int n)
{
    int nb = (n + SCAN_BLOCK * SCAN_ITEMS - 1) / (SCAN_BLOCK * SCAN_ITEMS);
    if (nb < 1) nb = 1;
    if (nb > SCAN_BLOCK * SCAN_ITEMS) return BCG_E_ARG;
    k_scan_partial<<<nb, SCAN_BLOCK, 0, c->stream>>>(n, in, c->scan_tmp);
    k_scan_blocks<<<1, SCAN_BLOCK, 0, c->stream>>>(nb, c->scan_tmp);
    k_scan_apply<<<nb, SCAN_BLOCK, 0, c->stream>>>(n, in, c->scan_tmp, out);
    c->launches += 3;
    return BCG_OK;
}

/* bin the cells of record buffer `buf` (c->cell_box, box_start, box_ids) */
int bin_cells(bcg_ctx* c, int buf)
{
    MechParams mp = mech_params(c);
    int n = c->n;
    BCG_CUDA_TRY(cudaMemsetAsync(c->box_cnt, 0, sizeof(int) * (size_t)c->nbox, c->stream));
    int* slot = c->delta_ids;   /* scratch: cap ints, unused outside divisions */
    if (n > 0) {
        k_bin_count<<<(n + 255) / 256, 256, 0, c->stream>>>(n, c->rec[buf], mp, c->cell_box, slot, c->box_cnt, c->status);
        c->launches++;
    }
    int rc = scan_exclusive(c, c->box_cnt, c->box_start, c->nbox);
    if (rc) return rc;
    if (n > 0) {
        k_bin_scatter<<<(n + 255) / 256, 256, 0, c->stream>>>(n, c->cell_box, slot, c->box_start, c->box_ids);
        c->launches++;
    }
    k_bin_sort<<<(c->nbox + 255) / 256, 256, 0, c->stream>>>(c->nbox, c->box_start, c->box_ids, c->P.max_cells_per_box, c->status);
    c->launches++;
    c->n_binned = n;
    BCG_CUDA_TRY(cudaGetLastError());
    return BCG_OK;
}

/* ======================================================================= */
/* neighbour lists                                                          */
/* ======================================================================= */
/* Rebuild the reduced list of cell `me` with one warp: gather the 3x3x3
 * box stencil (UniformGrid.h:141-170, z outer, y, x inner), apply the
 * reduceNeighbours filter (Neighbours.cpp:57-93).  Candidates come from the
 * bins; when `moved` is given, binned cells flagged as moved are skipped
 * and the (ids, boxes) of the delta list are gathered instead. */
template <bool COH>
__device__ void warp_rebuild_one(int me, const CellRec* rec, MechParams mp,
                                 const int* __restrict__ box_start, const int* __restrict__ box_ids,
                                 const int* moved, const int* delta_ids,
                                 const int* delta_box, int ndelta,
                                 int* nbr, int* ncount, DevStatus* st)
{
    const int lane = threadIdx.x & 31;
    Cst a = COH ? load_cst_coh(&rec[me]) : load_cst(&rec[me]);
    V3 acm = avg_pq(a.p, a.q);
    int xi, yi, zi;
    int abox = box_address(acm, mp, xi, yi, zi);
    if (abox < 0) { if (lane == 0) dev_error(st, BCG_E_OUT_OF_GRID, me); return; }
    int* out = nbr + (size_t)me * mp.kmax;
    const int YZ = mp.box_y * mp.box_z;
    /* the stencil's boxes in scan order, one a lane: lane i takes
     * (dz, dy, dx) = i / 9, i / 3 % 3, i % 3 around the cell's box, boxes
     * off the grid counting nothing.  Each box contributes its binned cells
     * (in bin order), then the delta cells listed in it. */
    int bs = 0, nbin = 0, ndel = 0, b = -1;
    if (lane < 27) {
        const int za = zi - 1 + lane / 9, ya = yi - 1 + (lane / 3) % 3, xa = xi - 1 + lane % 3;
        if (za >= 0 && za < mp.box_z && ya >= 0 && ya < mp.box_y && xa >= 0 && xa < mp.box_x) {
            b = xa * YZ + ya * mp.box_z + za;
            bs = box_start[b];
            int e = box_start[b + 1];
            if (e - bs > mp.box_cap) e = bs + mp.box_cap;   /* overfull: error already raised by the binning */
            nbin = e - bs;
            for (int t = 0; t < ndelta; t++) ndel += (delta_box[t] == b);
        }
    }
    /* exclusive prefix of the boxes' candidate counts */
    const int tot_i = nbin + ndel;
    int incl = tot_i;
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const int off = incl - tot_i;
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    int cnt = 0;
    for (int t0 = 0; t0 < total; t0 += 32) {
        const int f = t0 + lane;
        /* the box holding candidate f: the last lane whose offset is <= f */
        int box = 0;
        for (int q = 1; q < 27; q++) {
            const int oq = __shfl_sync(0xffffffffu, off, q), tq = __shfl_sync(0xffffffffu, tot_i, q);
            if (tq > 0 && oq <= f) box = q;
        }
        const int ob = __shfl_sync(0xffffffffu, off, box), nb_ = __shfl_sync(0xffffffffu, nbin, box);
        const int sb = __shfl_sync(0xffffffffu, bs, box), bb = __shfl_sync(0xffffffffu, b, box);
        int j = -1;
        bool from_delta = false;
        if (f < total) {
            const int r = f - ob;
            if (r < nb_) {
                j = box_ids[sb + r];
            } else {
                /* the (r - nb_)-th delta cell listed in this box */
                int k = r - nb_;
                for (int t = 0; t < ndelta; t++)
                    if (delta_box[t] == bb) { if (k == 0) { j = delta_ids[t]; break; } k--; }
                from_delta = true;
            }
        }
        bool keep = false;
        if (j >= 0 && j != me && (from_delta || !(moved && moved[j]))) {
            Cst bj = COH ? load_cst_coh(&rec[j]) : load_cst(&rec[j]);
            keep = keep_neighbour(a.p, a.q, a.L, a.R, acm, bj.p, bj.q, mp.rc);
        }
        unsigned m = __ballot_sync(0xffffffffu, keep);
        int pos = cnt + __popc(m & ((1u << lane) - 1));
        if (keep && pos < mp.kmax) out[pos] = j;
        cnt += __popc(m);
    }
    if (cnt > mp.kmax) { if (lane == 0) dev_error(st, BCG_E_NEIGH_OVERFLOW, me); cnt = mp.kmax; }
    if (lane == 0) ncount[me] = cnt;
}

__global__ void k_rebuild_all(int n, const CellRec* __restrict__ rec, MechParams mp,
                              const int* __restrict__ box_start, const int* __restrict__ box_ids,
                              int* __restrict__ nbr, int* __restrict__ ncount, DevStatus* st)
{
    int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= n) return;
    /* walk the cells in bin order so that consecutive warps share boxes */
    int me = box_ids[w];
    warp_rebuild_one<false>(me, rec, mp, box_start, box_ids, nullptr, nullptr, nullptr, 0, nbr, ncount, st);
}

extern "C" int bcg_rebuild_neighbours(bcg_ctx* c)
{
    if (!c) return BCG_E_ARG;
    timer_begin(c, BCG_T_NEIGHBOURS);
    int rc = bin_cells(c, c->cur);
    if (rc) return rc;
    if (c->n > 0) {
        int threads = 256;
        long warps = c->n;
        k_rebuild_all<<<(unsigned)((warps * 32 + threads - 1) / threads), threads, 0, c->stream>>>(
            c->n, c->rec[c->cur], mech_params(c), c->box_start, c->box_ids, c->nbr, c->ncount, c->status);
        c->launches++;
    }
    BCG_CUDA_TRY(cudaGetLastError());
    timer_end(c, BCG_T_NEIGHBOURS, 5);
    return BCG_OK;
}

/* ======================================================================= */
/* MoveCell + GrowCell                                                      */
/* ======================================================================= */
/* Forces on `a` from its neighbour list (lanes of a G-wide group split the
 * list; the group reduces with a fixed butterfly), plus the wall, drag and
 * surface-tension terms (sum_forces, Forces.cpp:332-381). */
template <int G, bool GEOM32>
__device__ __forceinline__ void sum_forces_group(const Cst& a, int me, const CellRec* __restrict__ old,
                                                 const int* __restrict__ list, int cnt, double wall_z,
                                                 const FieldPtrs& fp, const MechParams& mp,
                                                 V3& Fnet, V3& Tnet, V3& sf, V3& df, int& near_wall)
{
    const int gl = threadIdx.x & (G - 1);
    V3 cm = avg_pq(a.p, a.q);
    V3 F = mk(0, 0, 0), T = mk(0, 0, 0);
    for (int j = gl; j < cnt; j += G) {
        int id = __ldg(&list[j]);
        Cst b = load_cst(&old[id]);
        V3 f, r;
        if (GEOM32 ? pair_force_f32geom(a, cm, b, mp, f, r) : pair_force(a, cm, b, mp, f, r)) {
            F = add3(F, f);
            T = add3(T, cross3(sub3(r, cm), f));
        }
    }
#pragma unroll
    for (int o = G / 2; o >= 1; o >>= 1) {
        F.x += __shfl_xor_sync(0xffffffffu, F.x, o); F.y += __shfl_xor_sync(0xffffffffu, F.y, o);
        F.z += __shfl_xor_sync(0xffffffffu, F.z, o); T.x += __shfl_xor_sync(0xffffffffu, T.x, o);
        T.y += __shfl_xor_sync(0xffffffffu, T.y, o); T.z += __shfl_xor_sync(0xffffffffu, T.z, o);
    }
    sf = mk(0, 0, 0); df = mk(0, 0, 0);
    near_wall = dmin_(a.q.z, a.p.z) < 1.2 * a.R;
    if (near_wall) {
        V3 r1, r2;
        V3 F1 = wall_locus(a, cm, a.p, wall_z, mp, r1, sf, df);
        V3 F2 = wall_locus(a, cm, a.q, wall_z, mp, r2, sf, df);
        F = add3(F, F1); T = add3(T, cross3(sub3(r1, cm), F1));
        F = add3(F, F2); T = add3(T, cross3(sub3(r2, cm), F2));
    }
    /* F_v, Forces.cpp:320-329 */
    F = add3(F, scl3(a.v, -mp.viscosity * 6.0 * BCG_PI * a.R));
    T = add3(T, scl3(a.w, -mp.viscosity * 6.0 * BCG_PI * a.R));
    V3 Fs, Ts;
    surface_tension(a, cm, fp, mp, Fs, Ts);
    F = add3(F, Fs); T = add3(T, Ts);
    T.z = 0; F.y = 0;
    Fnet = F; Tnet = T;
}

/* MB = the blocks of 128 threads an SM is to hold: 4 caps the registers at
 * 128 (some spill), 3 at 170 (none spill); the autotuner picks. */
template <int G, bool GEOM32, int MB>
__global__ void __launch_bounds__(128, MB) k_move_grow(int n, int nbinned, const int* __restrict__ order,
        const CellRec* __restrict__ old, CellRec* __restrict__ nw,
        const int* __restrict__ nbr, const int* __restrict__ ncount,
        CellSoA soa, FieldPtrs fp, MechParams mp, double dt,
        int* __restrict__ div_list, int* __restrict__ div_count,
        unsigned long long* __restrict__ fcw_count, DevStatus* st)
{
    int t = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    const int gl = threadIdx.x & (G - 1);
    /* Lanes past the last cell run the body on cell 0 and write nothing:
     * the group reduction is a full-warp shuffle, so every lane of the
     * warp has to reach it (n > 0 at every launch). */
    const bool active = t < n;
    int me = active ? (t < nbinned ? __ldg(&order[t]) : t) : 0;
    int near1 = 0, near2 = 0;
    {
        Cst o = load_cst(&old[me]);
        V3 ocm = avg_pq(o.p, o.q);
        int xi, yi, zi;
        int obox = box_address(ocm, mp, xi, yi, zi);
        if (obox < 0) { if (gl == 0 && active) dev_error(st, BCG_E_OUT_OF_GRID, me); xi = 0; yi = 0; }
        double wall_z = __ldg(&fp.wall[xi * mp.box_y + yi]);
        const int* list = nbr + (size_t)me * mp.kmax;
        int cnt = __ldg(&ncount[me]);
        V3 F, T, sf, df;
        /* integrate, Integrate.cpp:11-32 */
        sum_forces_group<G, GEOM32>(o, me, old, list, cnt, wall_z, fp, mp, F, T, sf, df, near1);
        Cst tmp = o;
        half_kick(dt, F, T, o, tmp.v, tmp.w);
        V3 rcmp = sub3(o.p, ocm), rcmq = sub3(o.q, ocm);
        V3 vp = add3(tmp.v, cross3(tmp.w, rcmp)), vq = add3(tmp.v, cross3(tmp.w, rcmq));
        tmp.p = add3(o.p, scl3(vp, dt));
        tmp.q = add3(o.q, scl3(vq, dt));
        tmp.p.y = 0; tmp.q.y = 0;
        sum_forces_group<G, GEOM32>(tmp, me, old, list, cnt, wall_z, fp, mp, F, T, sf, df, near2);
        Cst nc = tmp;
        half_kick(dt, F, T, tmp, nc.v, nc.w);
        nc.v.y = 0;
        /* grow, grow.cpp:17-102 */
        V3 ncm = avg_pq(nc.p, nc.q);
        int nbox = box_address(ncm, mp, xi, yi, zi);
        if (nbox < 0) { if (gl == 0 && active) dev_error(st, BCG_E_OUT_OF_GRID, me); nbox = 0; }
        double g;
        if (mp.cross_feeding && __ldg(&soa.type[me]) != 1) g = __ldg(&fp.gr2[nbox]);
        else g = __ldg(&fp.gr1[nbox]);
        g = g * 1.5850;
        V3 v = sub3(nc.q, nc.p);
        double dL = nc.L * dt * g;
        V3 dv = scl3(v, dL * 0.5 / nc.L);
        nc.L += dL;
        nc.p = sub3(nc.p, dv);
        nc.q = add3(nc.q, dv);
        if (gl == 0 && active) {
            CellRec r;
            r.pL = make_double4(nc.p.x, nc.p.y, nc.p.z, nc.L);
            r.qR = make_double4(nc.q.x, nc.q.y, nc.q.z, nc.R);
            r.v = make_double4(nc.v.x, nc.v.y, nc.v.z, 0.0);
            r.w = make_double4(nc.w.x, nc.w.y, nc.w.z, 0.0);
            nw[me] = r;
            soa.gr[me] = g;
            soa.dfx[me] = df.x; soa.dfy[me] = df.y; soa.dfz[me] = df.z;
            soa.sfx[me] = sf.x; soa.sfy[me] = sf.y; soa.sfz[me] = sf.z;
            if (nc.L >= __ldg(&soa.ldiv[me])) {
                int k = atomicAdd(div_count, 1);
                div_list[k] = me;
            }
            if (!isfinite(nc.p.x) || !isfinite(nc.p.z) || !isfinite(nc.q.x) || !isfinite(nc.q.z))
                dev_error(st, BCG_E_NAN, me);
        }
    }
    /* F_cw calls (one rand() each, Forces.cpp:102): block-reduce then one atomic */
    unsigned long long calls = (active && gl == 0) ? (unsigned long long)(near1 + near2) : 0ull;
    for (int o = 16; o >= 1; o >>= 1) calls += __shfl_xor_sync(0xffffffffu, calls, o);
    __shared__ unsigned long long wsum[8];
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = calls;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += wsum[w];
        if (s) atomicAdd(fcw_count, s);
    }
}

/* lanes per cell in the force loop: the context's choice (bcg_autotune or
 * bcg_set_force_group), else 4 */
static int force_group_of(const bcg_ctx* c) { return c->force_group ? c->force_group : 4; }
static int force_occ_of(const bcg_ctx* c) { return c->force_occ ? c->force_occ : 4; }
extern "C" int bcg_set_force_group(bcg_ctx* c, int g)
{
    if (!c || (g != 1 && g != 2 && g != 4 && g != 8 && g != 16)) return BCG_E_ARG;
    if (g != force_group_of(c)) nutrient_graphs_drop(c);
    c->force_group = g;
    return BCG_OK;
}

/* Cells are walked in the order of the last binning (spatially coherent,
 * so neighbouring groups share record lines in L1/L2); cells created after
 * that binning follow in id order. */
int launch_move_grow(bcg_ctx* c, double dt, int group, int occ)
{
    int n = c->n;
    BCG_CUDA_TRY(cudaMemsetAsync(c->div_count, 0, sizeof(int), c->stream));
    BCG_CUDA_TRY(cudaMemsetAsync(c->fcw_count, 0, sizeof(unsigned long long), c->stream));
    if (n > 0) {
        MechParams mp = mech_params(c);
        FieldPtrs fp = field_ptrs(c);
        int nb = c->n_binned < n ? c->n_binned : n;
        const int threads = 128;
        long tot = (long)n * group;
        unsigned blocks = (unsigned)((tot + threads - 1) / threads);
        const CellRec* old = c->rec[c->cur];
        CellRec* nw = c->rec[c->cur ^ 1];
#define MG_ARGS(G, M, B) k_move_grow<G, M, B><<<blocks, threads, 0, c->stream>>>(n, nb, c->box_ids, old, nw, c->nbr, c->ncount, \
            c->soa, fp, mp, dt, c->div_list, c->div_count, c->fcw_count, c->status)
#define MG_GROUPS(M, B) switch (group) { \
            case 1: MG_ARGS(1, M, B); break; case 2: MG_ARGS(2, M, B); break; case 4: MG_ARGS(4, M, B); break; \
            case 8: MG_ARGS(8, M, B); break; default: MG_ARGS(16, M, B); break; }
        if (c->pair_f32) { if (occ == 3) { MG_GROUPS(true, 3) } else { MG_GROUPS(true, 4) } }
        else { if (occ == 3) { MG_GROUPS(false, 3) } else { MG_GROUPS(false, 4) } }
#undef MG_GROUPS
#undef MG_ARGS
        c->launches++;
        BCG_CUDA_TRY(cudaGetLastError());
    }
    return BCG_OK;
}

/* split halves of bcg_move_grow (used by the ensemble runner to overlap
 * colonies): the launch queues the kernel and the two counter reads, the
 * finish waits for them */
int move_grow_launch(bcg_ctx* c, double dt)
{
    int rc = launch_move_grow(c, dt, force_group_of(c), force_occ_of(c));
    if (rc) return rc;
    int* hp = (int*)c->pinned;
    BCG_CUDA_TRY(cudaMemcpyAsync(hp, c->div_count, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    BCG_CUDA_TRY(cudaMemcpyAsync(hp + 2, c->fcw_count, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    return BCG_OK;
}
int move_grow_finish(bcg_ctx* c, int* n_div, int64_t* fcw_calls)
{
    int rc = ctx_check_status(c);
    if (rc) return rc;
    c->move_pending = 1;
    int* hp = (int*)c->pinned;
    c->last_ndiv = hp[0];
    if (n_div) *n_div = hp[0];
    if (fcw_calls) *fcw_calls = (int64_t)(*(unsigned long long*)(hp + 2));
    return BCG_OK;
}

extern "C" int bcg_move_grow(bcg_ctx* c, double dt, int* n_div, int64_t* fcw_calls)
{
    if (!c) return BCG_E_ARG;
    timer_begin(c, BCG_T_MOVE_GROW);
    int rc = launch_move_grow(c, dt, force_group_of(c), force_occ_of(c));
    if (rc) return rc;
    timer_end(c, BCG_T_MOVE_GROW, c->n > 0 ? 1 : 0);
    /* the two counters are the only values the host needs this step */
    int* hp = (int*)c->pinned;
    BCG_CUDA_TRY(cudaMemcpyAsync(hp, c->div_count, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    BCG_CUDA_TRY(cudaMemcpyAsync(hp + 2, c->fcw_count, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    return move_grow_finish(c, n_div, fcw_calls);
}

/* time `reps` launches of MoveCell+GrowCell with `group` lanes per cell;
 * the records of the current buffer are read only, so the state is kept */
static int time_move_grow(bcg_ctx* c, int group, int occ, int reps, float* ms)
{
    cudaEvent_t a, b;
    BCG_CUDA_TRY(cudaEventCreate(&a));
    BCG_CUDA_TRY(cudaEventCreate(&b));
    int rc = launch_move_grow(c, c->P.dt, group, occ);      /* warm-up */
    if (!rc) rc = (cudaEventRecord(a, c->stream) == cudaSuccess) ? BCG_OK : BCG_E_CUDA;
    for (int r = 0; r < reps && !rc; r++) rc = launch_move_grow(c, c->P.dt, group, occ);
    if (!rc) rc = (cudaEventRecord(b, c->stream) == cudaSuccess) ? BCG_OK : BCG_E_CUDA;
    if (!rc) rc = (cudaEventSynchronize(b) == cudaSuccess) ? BCG_OK : BCG_E_CUDA;
    if (!rc) cudaEventElapsedTime(ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return rc;
}

extern "C" int bcg_set_pair_precision(bcg_ctx* c, int bits)
{
    if (!c || (bits != 32 && bits != 64)) return BCG_E_ARG;
    int f32 = bits == 32;
    if (f32 != c->pair_f32) { c->pair_f32 = f32; nutrient_graphs_drop(c); }
    return BCG_OK;
}

extern "C" int bcg_autotune(bcg_ctx* c, int what, int* choice)
{
    if (!c) return BCG_E_ARG;
    if (what == BCG_TUNE_SMOOTHER) return mg_tune_smoother(c, choice);
    if (what != BCG_TUNE_FORCE_GROUP) return BCG_E_ARG;
    if (c->n == 0) { if (choice) *choice = force_group_of(c); return BCG_OK; }
    const int saved_ndiv = c->last_ndiv;
    /* the trial launches rewrite the per-cell outputs of a step (growth
     * rate, friction accumulators): keep a copy and put it back */
    double* keep[7] = {c->soa.gr, c->soa.dfx, c->soa.dfy, c->soa.dfz, c->soa.sfx, c->soa.sfy, c->soa.sfz};
    const size_t nb = (size_t)c->n * sizeof(double);
    double* save = nullptr;
    BCG_CUDA_TRY(cudaMallocAsync((void**)&save, 7 * nb, c->stream));
    for (int a = 0; a < 7; a++)
        BCG_CUDA_TRY(cudaMemcpyAsync(save + a * (size_t)c->n, keep[a], nb, cudaMemcpyDeviceToDevice, c->stream));
    const int groups[5] = {1, 2, 4, 8, 16};
    float best = 3.4e38f;
    int best_g = force_group_of(c), best_o = force_occ_of(c);
    int rc = BCG_OK;
    for (int gi = 0; gi < 5 && !rc; gi++)
        for (int occ = 3; occ <= 4 && !rc; occ++) {
            float ms = 0;
            rc = time_move_grow(c, groups[gi], occ, 3, &ms);
            if (!rc && ms < best) { best = ms; best_g = groups[gi]; best_o = occ; }
        }
    for (int a = 0; a < 7; a++)
        cudaMemcpyAsync(keep[a], save + a * (size_t)c->n, nb, cudaMemcpyDeviceToDevice, c->stream);
    cudaFreeAsync(save, c->stream);
    int rc2 = ctx_check_status(c);
    c->last_ndiv = saved_ndiv;
    if (rc) return rc;
    if (rc2) return rc2;
    if (best_g != c->force_group || best_o != c->force_occ) { c->force_group = best_g; c->force_occ = best_o; nutrient_graphs_drop(c); }
    if (choice) *choice = best_g;
    return BCG_OK;
}

/* ======================================================================= */
/* division loop                                                            */
/* ======================================================================= */

/* divide(), grow.cpp:107-186, for mother m into daughter d; u[0..8] are the
 * nine (float)rand()/RAND_MAX draws in call order.  Reads the mother's
 * record, writes the SoA fields of both cells (no other division reads
 * them) and returns the two new records in out_m / out_d; the records are
 * stored in rec[] later, in division order. */
__device__ void divide_compute(int m, int d, const float* u, double t, const CellRec* rec, CellSoA soa,
                               const MechParams& mp, CellRec& out_m, CellRec& out_d)
{
    Cst M = load_cst(&rec[m]);
    double dl = ((double)u[0] - 0.5) * mp.var_l;
    double dangle = ((double)u[1] - 0.5) * mp.var_angle;
    V3 pq = sub3(M.p, M.q);
    V3 dd1 = mk((double)u[2] - 0.5, (double)u[3] - 0.5, (double)u[4] - 0.5);
    dd1 = sub3(dd1, scl3(pq, dot3(dd1, pq) / dot3(pq, pq)));
    dd1 = scl3(dd1, 1 / sqrt(dot3(dd1, dd1)));
    V3 dO1 = scl3(dd1, dangle);
    V3 dd2 = mk((double)u[5] - 0.5, (double)u[6] - 0.5, (double)u[7] - 0.5);
    dd2 = sub3(dd2, scl3(pq, dot3(dd2, pq) / dot3(pq, pq)));
    dd2 = scl3(dd2, 1 / sqrt(dot3(dd2, dd2)));
    V3 dO2 = scl3(dd2, dangle);
    V3 uv = sub3(M.p, M.q);
    double L = M.L;
    uv = scl3(uv, 1 / L);
    double dR = mp.cell_radius;
    double mL = L / 2 - M.R + dl;
    double dLen = L / 2 + M.R - 2 * dR - dl;
    V3 dq = M.q;
    V3 dw = mk(0, 0, ((double)u[8] - 0.5) * 0.001);
    V3 mq = sub3(M.p, scl3(uv, mL));
    double tq_m = soa.tq[m];
    V3 dp = sub3(mq, scl3(uv, dR + M.R));
    dq = sub3(dp, scl3(uv, dLen));
    V3 mp_ = add3(M.p, scl3(dO1, mL));
    mq = sub3(mq, scl3(dO1, mL));
    dp = add3(dp, scl3(dO2, dLen));
    dq = sub3(dq, scl3(dO2, dLen));
    CellRec rm, rd;
    rm.pL = make_double4(mp_.x, mp_.y, mp_.z, mL);
    rm.qR = make_double4(mq.x, mq.y, mq.z, M.R);
    rm.v = make_double4(M.v.x, M.v.y, M.v.z, 0.0);
    rm.w = make_double4(0.0, 0.0, 0.0, 0.0);
    rd.pL = make_double4(dp.x, dp.y, dp.z, dLen);
    rd.qR = make_double4(dq.x, dq.y, dq.z, dR);
    rd.v = make_double4(M.v.x, M.v.y, M.v.z, 0.0);
    rd.w = make_double4(dw.x, dw.y, dw.z, 0.0);
    out_m = rm;
    out_d = rd;
    soa.gr[d] = soa.gr[m];
    soa.tq[d] = tq_m;
    soa.tq[m] = t;
    soa.tp[d] = t;
    soa.ap[m] = soa.ap[m] + 1;
    soa.aq[d] = soa.aq[m] + 1;
    soa.ap[d] = 0;
    soa.dfx[d] = 0; soa.dfy[d] = 0; soa.dfz[d] = 0;
    soa.sfx[d] = 0; soa.sfy[d] = 0; soa.sfz[d] = 0;
    soa.type[d] = soa.type[m];
    soa.anc[d] = soa.anc[m];
    soa.ldiv[m] = mp.l_divide / 2 + mp.cell_radius + mL;
    soa.ldiv[d] = mp.l_divide / 2 + mp.cell_radius + dLen;
}

/* Simulation.cpp:380-404.  The reference divides the parents one after
 * another in ascending id order; each division moves the mother and adds
 * the daughter in the box structure and rebuilds the lists of {mother,
 * mother's neighbours, daughter} (Neighbours.cpp:39-55) against the state
 * left by the divisions before it.
 *
 * Here the divisions run as independent groups.  A division's footprint is
 * the rectangle of boxes, widened by 2, around the boxes of every cell whose
 * list it can rebuild (the mother before and after, her listed neighbours,
 * the daughter).  Every box a rebuild scans, and every box whose content
 * the division changes, lies inside it.  Divisions whose footprints overlap
 * are joined into one group (connected components), and a group runs its
 * divisions in ascending order on one block.  Divisions of different groups
 * neither change a box the other scans nor rebuild a common list, so the
 * lists come out as in the sequential loop.
 *
 * k_div_plan (one CTA): sort the parents, apply the reference's MaxCells
 * cut, compute all divisions' geometry (divide_compute; SoA fields written
 * here), footprints, groups (label propagation over the overlapping pairs,
 * then a sort by (group, division)), and the group-ordered division list.
 * k_div_groups (one block per group): store the records, mark the mother
 * moved, append both cells to the group's delta list, rebuild the lists. */
__global__ void __launch_bounds__(1024) k_div_plan(int n_start, int ndiv, int cap, double t,
        const float* __restrict__ draws, const CellRec* __restrict__ rec, CellSoA soa, MechParams mp,
        const int* __restrict__ div_list, const int* __restrict__ cell_box,
        const int* __restrict__ nbr, const int* __restrict__ ncount,
        CellRec* __restrict__ new_rec, int* __restrict__ new_box, int4* __restrict__ rect,
        int2* __restrict__ pairs, int* __restrict__ par_out, int* __restrict__ order, int* __restrict__ grp,
        int* __restrict__ lineage, int* __restrict__ out, DevStatus* st)
{
    /* dynamic shared memory: the sorted parents (later the group of each
     * root), the union-find parents, the groups' fill counters */
    extern __shared__ int div_smem[];
    int* sd = div_smem;
    int* par = div_smem + DIV_SORT_MAX;
    int* fill = div_smem + 2 * DIV_SORT_MAX;
    __shared__ int s_npairs;
    int P2 = 1;
    while (P2 < ndiv) P2 <<= 1;
    for (int i = threadIdx.x; i < P2; i += blockDim.x) sd[i] = i < ndiv ? div_list[i] : 0x7fffffff;
    if (threadIdx.x == 0) s_npairs = 0;
    __syncthreads();
    for (int k = 2; k <= P2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < P2; i += blockDim.x) {
                int ixj = i ^ j;
                if (ixj > i) {
                    int a = sd[i], b = sd[ixj];
                    bool up = (i & k) == 0;
                    if ((a > b) == up) { sd[i] = b; sd[ixj] = a; }
                }
            }
            __syncthreads();
        }
    /* the loop stops at the first division that would pass MaxCells */
    int nd = cap - n_start;
    if (nd < 0) nd = 0;
    if (nd > ndiv) nd = ndiv;
    if (nd < ndiv && threadIdx.x == 0) dev_error(st, BCG_E_MAXCELLS, nd);
    const int YZ = mp.box_y * mp.box_z;
    for (int d = threadIdx.x; d < nd; d += blockDim.x) {
        const int m = sd[d], N = n_start + d;
        CellRec rm, rd;
        divide_compute(m, N, draws + 9 * (size_t)d, t, rec, soa, mp, rm, rd);
        new_rec[2 * d] = rm; new_rec[2 * d + 1] = rd;
        int xi, yi, zi;
        int bm = box_address(avg_pq(mk(rm.pL.x, rm.pL.y, rm.pL.z), mk(rm.qR.x, rm.qR.y, rm.qR.z)), mp, xi, yi, zi);
        int bd = box_address(avg_pq(mk(rd.pL.x, rd.pL.y, rd.pL.z), mk(rd.qR.x, rd.qR.y, rd.qR.z)), mp, xi, yi, zi);
        if (bm < 0) { dev_error(st, BCG_E_OUT_OF_GRID, m); bm = 0; }
        if (bd < 0) { dev_error(st, BCG_E_OUT_OF_GRID, N); bd = 0; }
        new_box[2 * d] = bm; new_box[2 * d + 1] = bd;
        lineage[2 * d] = m; lineage[2 * d + 1] = N;
        int b0 = cell_box[m];
        int x0 = b0 / YZ, z0 = b0 % mp.box_z;
        int xlo = x0, xhi = x0, zlo = z0, zhi = z0;
        int x = bm / YZ, z = bm % mp.box_z;
        xlo = min(xlo, x); xhi = max(xhi, x); zlo = min(zlo, z); zhi = max(zhi, z);
        x = bd / YZ; z = bd % mp.box_z;
        xlo = min(xlo, x); xhi = max(xhi, x); zlo = min(zlo, z); zhi = max(zhi, z);
        rect[d] = make_int4(xlo, xhi, zlo, zhi);
        par[d] = d;
    }
    __syncthreads();
    /* the boxes of the mother's listed neighbours, one warp per division,
     * then the footprint's margin of 2 boxes */
    {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
        for (int d = wid; d < nd; d += nw) {
            const int m = sd[d];
            const int cnt = ncount[m];
            int xlo = 0x7fffffff, xhi = -0x7fffffff, zlo = 0x7fffffff, zhi = -0x7fffffff;
            for (int j = lane; j < cnt; j += 32) {
                const int bb = cell_box[nbr[(size_t)m * mp.kmax + j]];
                const int x = bb / YZ, z = bb % mp.box_z;
                xlo = min(xlo, x); xhi = max(xhi, x); zlo = min(zlo, z); zhi = max(zhi, z);
            }
            for (int o = 16; o >= 1; o >>= 1) {
                xlo = min(xlo, __shfl_xor_sync(0xffffffffu, xlo, o));
                xhi = max(xhi, __shfl_xor_sync(0xffffffffu, xhi, o));
                zlo = min(zlo, __shfl_xor_sync(0xffffffffu, zlo, o));
                zhi = max(zhi, __shfl_xor_sync(0xffffffffu, zhi, o));
            }
            if (lane == 0) {
                int4 r = rect[d];
                r.x = min(r.x, xlo); r.y = max(r.y, xhi); r.z = min(r.z, zlo); r.w = max(r.w, zhi);
                rect[d] = make_int4(r.x - 2, r.y + 2, r.z - 2, r.w + 2);
            }
        }
    }
    __syncthreads();
    /* overlapping footprints */
    const int np2 = nd * nd;
    for (int q = threadIdx.x; q < np2; q += blockDim.x) {
        int a = q / nd, b = q - a * nd;
        if (a >= b) continue;
        int4 ra = rect[a], rb = rect[b];
        if (ra.x <= rb.y && rb.x <= ra.y && ra.z <= rb.w && rb.z <= ra.w) {
            int k = atomicAdd(&s_npairs, 1);
            if (k < DIV_PAIR_CAP) pairs[k] = make_int2(a, b);
        }
    }
    __syncthreads();
    const int npairs = s_npairs;
    if (npairs > DIV_PAIR_CAP) {
        /* too many overlaps to list: one sequential group */
        for (int d = threadIdx.x; d < nd; d += blockDim.x) par[d] = 0;
        __syncthreads();
    } else {
        /* connected components by label propagation: every division takes
         * the smallest label among the divisions its footprint overlaps,
         * then follows its label's label, until nothing changes; the label
         * ends as the smallest division of its component */
        for (;;) {
            __shared__ int s_changed;
            if (threadIdx.x == 0) s_changed = 0;
            __syncthreads();
            for (int k = threadIdx.x; k < npairs; k += blockDim.x) {
                const int a = pairs[k].x, b = pairs[k].y;
                const int la = par[a], lb = par[b];
                if (la != lb) {
                    const int lo = la < lb ? la : lb;
                    atomicMin(&par[a], lo);
                    atomicMin(&par[b], lo);
                    atomicMin(&par[la], lo);
                    atomicMin(&par[lb], lo);
                    s_changed = 1;
                }
            }
            __syncthreads();
            for (int d = threadIdx.x; d < nd; d += blockDim.x) {
                const int l = par[d], ll = par[l];
                if (ll < l) { atomicMin(&par[d], ll); s_changed = 1; }
            }
            __syncthreads();
            const int ch = s_changed;
            __syncthreads();
            if (!ch) break;
        }
    }
    /* groups in order of their first division, members ascending: sort the
     * keys (label, division) and cut the sorted list where the label
     * changes.  grp[2g] = start in order[], grp[2g+1] = length. */
    int P2n = 1;
    while (P2n < nd) P2n <<= 1;
    for (int i = threadIdx.x; i < P2n; i += blockDim.x) sd[i] = i < nd ? par[i] * DIV_SORT_MAX + i : 0x7fffffff;
    __syncthreads();
    for (int k = 2; k <= P2n; k <<= 1)
        for (int jj = k >> 1; jj > 0; jj >>= 1) {
            for (int i = threadIdx.x; i < P2n; i += blockDim.x) {
                int ixj = i ^ jj;
                if (ixj > i) {
                    int a = sd[i], b = sd[ixj];
                    bool up = (i & k) == 0;
                    if ((a > b) == up) { sd[i] = b; sd[ixj] = a; }
                }
            }
            __syncthreads();
        }
    /* fill[i] = 1 where a group starts, then its inclusive prefix sum */
    for (int i = threadIdx.x; i < P2n; i += blockDim.x)
        fill[i] = (i < nd && (i == 0 || sd[i] / DIV_SORT_MAX != sd[i - 1] / DIV_SORT_MAX)) ? 1 : 0;
    __syncthreads();
    for (int off = 1; off < P2n; off <<= 1) {
        int v[DIV_SORT_MAX / 1024];
        int c = 0;
        for (int i = threadIdx.x; i < P2n; i += blockDim.x) v[c++] = i >= off ? fill[i - off] : 0;
        __syncthreads();
        c = 0;
        for (int i = threadIdx.x; i < P2n; i += blockDim.x) fill[i] += v[c++];
        __syncthreads();
    }
    for (int i = threadIdx.x; i < nd; i += blockDim.x) {
        const int d = sd[i] - (sd[i] / DIV_SORT_MAX) * DIV_SORT_MAX;
        order[i] = d;
        const int g = fill[i] - 1;
        const bool start = i == 0 || sd[i] / DIV_SORT_MAX != sd[i - 1] / DIV_SORT_MAX;
        if (start) grp[2 * g] = i;
    }
    __syncthreads();
    /* the group's length, from its last member and its start */
    for (int i = threadIdx.x; i < nd; i += blockDim.x) {
        const bool last = i == nd - 1 || sd[i] / DIV_SORT_MAX != sd[i + 1] / DIV_SORT_MAX;
        if (last) {
            const int g = fill[i] - 1;
            grp[2 * g + 1] = i + 1 - grp[2 * g];
        }
    }
    if (threadIdx.x == 0) { out[0] = nd; out[1] = n_start + nd; out[2] = nd > 0 ? fill[nd - 1] : 0; }
    (void)par_out;
}

/* One block per group.  The group's divisions run in ascending order; the
 * lists one division rebuilds (the mother's, her listed neighbours', the
 * daughter's) each depend only on the records and the boxes, which the
 * rebuilds do not change, so the block's warps share them out. */
#define DIV_GROUP_WARPS 4
__global__ void __launch_bounds__(32 * DIV_GROUP_WARPS) k_div_groups(int n_start, const int* __restrict__ div_out,
        const int* __restrict__ grp, const int* __restrict__ order, const int* __restrict__ lineage,
        const CellRec* __restrict__ new_rec, const int* __restrict__ new_box,
        CellRec* rec, MechParams mp, int* nbr, int* ncount,
        const int* __restrict__ box_start, const int* __restrict__ box_ids,
        int* moved, int* delta_ids, int* delta_box, DevStatus* st)
{
    __shared__ int idl[1 + 1024 + 1];
    const int w = threadIdx.x >> 5;
    const int g = blockIdx.x;
    if (g >= div_out[2]) return;                       /* whole block */
    const int gs = grp[2 * g], gl = grp[2 * g + 1];
    int* dids = delta_ids + 2 * gs;
    int* dbox = delta_box + 2 * gs;
    for (int j = 0; j < gl; j++) {
        const int d = order[gs + j];
        const int m = lineage[2 * d], N = n_start + d;
        /* the previous division's rebuilds are done (they may have written
         * this mother's list) before her records and list change hands */
        __syncthreads();
        if (threadIdx.x == 0) {
            rec[m] = new_rec[2 * d];
            rec[N] = new_rec[2 * d + 1];
            moved[m] = 1;
            dids[2 * j] = m; dbox[2 * j] = new_box[2 * d];
            dids[2 * j + 1] = N; dbox[2 * j + 1] = new_box[2 * d + 1];
        }
        const int cnt = ncount[m];
        for (int i = threadIdx.x; i < cnt; i += blockDim.x) idl[1 + i] = nbr[(size_t)m * mp.kmax + i];
        if (threadIdx.x == 0) { idl[0] = m; idl[cnt + 1] = N; }
        /* every thread has read the mother's old list before a warp rewrites it */
        __syncthreads();
        for (int k = w; k < cnt + 2; k += DIV_GROUP_WARPS)
            warp_rebuild_one<true>(idl[k], rec, mp, box_start, box_ids, moved, dids, dbox, 2 * (j + 1), nbr, ncount, st);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < gl; j += blockDim.x) moved[lineage[2 * order[gs + j]]] = 0;
}

/* the division planner's shared memory: sorted parents, union-find
 * parents and group fill counters, DIV_SORT_MAX ints each */
int mech_kernel_attributes()
{
    /* set on every context creation: the attribute belongs to the current
     * device, and the call is cheap and thread-safe */
    if (cudaFuncSetAttribute(k_div_plan, cudaFuncAttributeMaxDynamicSharedMemorySize, DIV_PLAN_SMEM) != cudaSuccess)
        return BCG_E_CUDA;
    return BCG_OK;
}

extern "C" int bcg_get_dividing(bcg_ctx* c, int* ids, int capacity)
{
    if (!c || (!ids && capacity > 0)) return BCG_E_ARG;
    int n = c->last_ndiv < capacity ? c->last_ndiv : capacity;
    if (n > 0) {
        BCG_CUDA_TRY(cudaMemcpyAsync(ids, c->div_list, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
        BCG_CUDA_TRY(cudaStreamSynchronize(c->stream));
        /* ascending, as the 1-thread reference collects them */
        for (int i = 1; i < n; i++) { int v = ids[i], j = i - 1; while (j >= 0 && ids[j] > v) { ids[j + 1] = ids[j]; j--; } ids[j + 1] = v; }
    }
    return BCG_OK;
}

/* split halves of bcg_divide: the launch queues the binning, the draw
 * upload, the two division kernels and the read of the counts; the
 * finish waits, copies the lineage and advances the context */
int divide_launch(bcg_ctx* c, const float* draws, int n_draw_sets, double t)
{
    if (n_draw_sets != c->last_ndiv) return BCG_E_ARG;
    const int ndiv = c->last_ndiv;
    if (ndiv > DIV_SORT_MAX) return BCG_E_UNSUPPORTED;
    if (ndiv == 0) return BCG_OK;
    if (!draws) return BCG_E_ARG;
    int nb = c->cur ^ 1;
    int rc = bin_cells(c, nb);
    if (rc) return rc;
    size_t db = sizeof(float) * 9 * (size_t)ndiv;
    rc = ensure_pinned(c, db + 64);
    if (rc) return rc;
    memcpy(c->pinned, draws, db);
    BCG_CUDA_TRY(cudaMemcpyAsync(c->draws_dev, c->pinned, db, cudaMemcpyHostToDevice, c->stream));
    MechParams mp = mech_params(c);
    k_div_plan<<<1, 1024, DIV_PLAN_SMEM, c->stream>>>(c->n, ndiv, c->cap, t, c->draws_dev, c->rec[nb], c->soa, mp,
        c->div_list, c->cell_box, c->nbr, c->ncount, c->div_rec, c->div_box, c->div_rect, c->div_pairs,
        c->div_par, c->div_order, c->div_grp, c->lineage, c->n_done_dev, c->status);
    k_div_groups<<<ndiv, 32 * DIV_GROUP_WARPS, 0, c->stream>>>(c->n, c->n_done_dev, c->div_grp, c->div_order,
        c->lineage, c->div_rec, c->div_box, c->rec[nb], mp, c->nbr, c->ncount, c->box_start, c->box_ids,
        c->moved, c->delta_ids, c->delta_box, c->status);
    c->launches += 2;
    BCG_CUDA_TRY(cudaGetLastError());
    int* hp = (int*)c->pinned;
    BCG_CUDA_TRY(cudaMemcpyAsync(hp, c->n_done_dev, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    return BCG_OK;
}
int divide_finish(bcg_ctx* c, int* n_done, int* lineage)
{
    const int ndiv = c->last_ndiv;
    int done = 0, rc = BCG_OK;
    if (ndiv > 0) {
        rc = ctx_check_status(c);
        done = ((int*)c->pinned)[0];
        if (lineage && done > 0)
            BCG_CUDA_TRY(cudaMemcpy(lineage, c->lineage, sizeof(int) * 2 * (size_t)done, cudaMemcpyDeviceToHost));
        c->n += done;
    }
    c->cur ^= 1;
    c->move_pending = 0;
    c->last_ndiv = 0;
    if (n_done) *n_done = done;
    return rc;
}

extern "C" int bcg_divide(bcg_ctx* c, const float* draws, int n_draw_sets, double t, int* n_done, int* lineage)
{
    if (!c) return BCG_E_ARG;
    timer_begin(c, BCG_T_DIVIDE);
    const int ndiv = c->last_ndiv;
    int rc = divide_launch(c, draws, n_draw_sets, t);
    if (rc) return rc;
    rc = divide_finish(c, n_done, lineage);
    timer_end(c, BCG_T_DIVIDE, ndiv > 0 ? 7 : 0);
    return rc;
}

/* ======================================================================= */
/* mean_stress (Compute.cpp:18-117)                                         */
/* ======================================================================= */
__global__ void k_mean_stress(int n, const CellRec* __restrict__ rec, const int* __restrict__ nbr,
                              const int* __restrict__ ncount, FieldPtrs fp, MechParams mp,
                              double* __restrict__ stress, double* __restrict__ fnet,
                              unsigned long long* fcw_count, DevStatus* st)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int near = 0;
    if (i < n) {
        Cst c = load_cst(&rec[i]);
        double V = c.L * BCG_PI * c.R * c.R + 4.0 / 3.0 * BCG_PI * c.R * c.R * c.R;
        V3 CM = avg_pq(c.p, c.q);
        int xi, yi, zi;
        if (box_address(CM, mp, xi, yi, zi) < 0) { dev_error(st, BCG_E_OUT_OF_GRID, i); xi = 0; yi = 0; }
        double sxx = 0, syy = 0, szz = 0;
        V3 Fn = mk(0, 0, 0);
        const int* list = nbr + (size_t)i * mp.kmax;
        int cnt = ncount[i];
        for (int j = 0; j < cnt; j++) {
            Cst b = load_cst(&rec[list[j]]);
            V3 F, r;
            if (!pair_force(c, CM, b, mp, F, r)) { F = mk(0, 0, 0); continue; }
            Fn = add3(Fn, F);
            r = sub3(r, CM);
            sxx -= F.x * r.x; syy -= F.y * r.y; szz -= F.z * r.z;
        }
        if (dmin_(c.q.z, c.p.z) < 1.2 * c.R) {
            near = 1;
            double wall_z = fp.wall[xi * mp.box_y + yi];
            V3 r1, r2, sf = mk(0, 0, 0), df = mk(0, 0, 0);
            V3 F1 = wall_locus(c, CM, c.p, wall_z, mp, r1, sf, df);
            V3 F2 = wall_locus(c, CM, c.q, wall_z, mp, r2, sf, df);
            Fn = add3(Fn, F1);
            r1 = sub3(r1, CM);
            sxx -= F1.x * r1.x; syy -= F1.y * r1.y; szz -= F1.z * r1.z;
            Fn = add3(Fn, F2);
            r2 = sub3(r2, CM);
            sxx -= F2.x * r2.x; syy -= F2.y * r2.y; szz -= F2.z * r2.z;
        }
        V3 F, T;
        surface_tension(c, CM, fp, mp, F, T);
        Fn = add3(Fn, F);
        V3 r = sub3(c.p, CM); r.z += c.R;
        V3 r2 = sub3(c.q, CM); r2.z += c.R;
        sxx -= F.x * r.x * 0.5 - F.x * r2.x * 0.5;
        syy -= F.y * r.y * 0.5 - F.y * r2.y * 0.5;
        szz -= F.z * r.z * 0.5 - F.z * r2.z * 0.5;
        sxx /= V; syy /= V; szz /= V;
        double rr, tt;
        double Lcm = sqrt(CM.x * CM.x + CM.y * CM.y);
        if (Lcm > DBL_EPSILON) {
            V3 uv = scl3(CM, 1.0 / Lcm);
            rr = sxx * uv.x + syy * uv.y;
            tt = -sxx * uv.y + syy * uv.x;
        } else { rr = (sxx + syy); tt = 0.0; }
        stress[5 * (size_t)i + 0] = sxx; stress[5 * (size_t)i + 1] = syy; stress[5 * (size_t)i + 2] = szz;
        stress[5 * (size_t)i + 3] = rr; stress[5 * (size_t)i + 4] = tt;
        if (fnet) { fnet[3 * (size_t)i] = Fn.x; fnet[3 * (size_t)i + 1] = Fn.y; fnet[3 * (size_t)i + 2] = Fn.z; }
    }
    unsigned long long v = near;
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(fcw_count, v);
}

void launch_mean_stress(bcg_ctx* c, double* stress, unsigned long long* fcw, cudaStream_t s)
{
    if (c->n <= 0) return;
    k_mean_stress<<<(c->n + 127) / 128, 128, 0, s>>>(c->n, c->rec[c->cur], c->nbr, c->ncount, field_ptrs(c),
                                                     mech_params(c), stress, nullptr, fcw, c->status);
    c->launches++;
}

/* F_surf_tension's force on every cell (Forces.cpp:209-317), the cell
 * line's three force columns in the initial output block
 * (Simulation.cpp:229-238) */
__global__ void k_surface_force(int n, const CellRec* __restrict__ rec, FieldPtrs fp, MechParams mp,
                                double* __restrict__ force)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Cst c = load_cst(&rec[i]);
    V3 F, T;
    surface_tension(c, avg_pq(c.p, c.q), fp, mp, F, T);
    force[3 * (size_t)i] = F.x; force[3 * (size_t)i + 1] = F.y; force[3 * (size_t)i + 2] = F.z;
}

void launch_surface_force(bcg_ctx* c, double* force, cudaStream_t s)
{
    if (c->n <= 0) return;
    k_surface_force<<<(c->n + 127) / 128, 128, 0, s>>>(c->n, c->rec[c->cur], field_ptrs(c), mech_params(c), force);
    c->launches++;
}

extern "C" int bcg_mean_stress(bcg_ctx* c, double* stress, double* fnet, int64_t* fcw_calls)
{
    if (!c || !stress) return BCG_E_ARG;
    int n = c->n;
    BCG_CUDA_TRY(cudaMemsetAsync(c->fcw_count, 0, sizeof(unsigned long long), c->stream));
    if (n > 0) {
        double *ds = nullptr, *df = nullptr;
        BCG_CUDA_TRY(cudaMallocAsync((void**)&ds, sizeof(double) * 5 * (size_t)n, c->stream));
        if (fnet) BCG_CUDA_TRY(cudaMallocAsync((void**)&df, sizeof(double) * 3 * (size_t)n, c->stream));
        k_mean_stress<<<(n + 127) / 128, 128, 0, c->stream>>>(n, c->rec[c->cur], c->nbr, c->ncount, field_ptrs(c),
                                                              mech_params(c), ds, df, c->fcw_count, c->status);
        c->launches++;
        BCG_CUDA_TRY(cudaMemcpyAsync(stress, ds, sizeof(double) * 5 * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
        if (fnet) BCG_CUDA_TRY(cudaMemcpyAsync(fnet, df, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
        BCG_CUDA_TRY(cudaFreeAsync(ds, c->stream));
        if (df) BCG_CUDA_TRY(cudaFreeAsync(df, c->stream));
    }
    unsigned long long h = 0;
    BCG_CUDA_TRY(cudaMemcpyAsync(&h, c->fcw_count, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    int rc = ctx_check_status(c);
    if (fcw_calls) *fcw_calls = (int64_t)h;
    return rc;
}

/* ======================================================================= */
/* bcg_mean_stress_noalloc: the same kernel with its staging in a device   */
/* array compiled into the library (no allocation on any call)             */
/* ======================================================================= */
/* 5 stress + 3 force doubles per cell, then the F_cw counter */
static __device__ __align__(256) double g_noalloc_stress[8 * BCG_NOALLOC_MAX_CELLS + 32];

/* The array's device address on the current device.  Looked up on every
 * call rather than kept: the lookup allocates nothing, and an address kept
 * from before a cudaDeviceReset would point into a released context.  In
 * host code the array's name is only a host-side stand-in; kernels must be
 * given this address. */
static int noalloc_staging(double** out)
{
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_stress);
    if (e != cudaSuccess) { bcg_set_cuda_error(e); return BCG_E_CUDA; }
    *out = (double*)p;
    return BCG_OK;
}

extern "C" int bcg_mean_stress_noalloc(bcg_ctx* c, double* stress, double* fnet, int64_t* fcw_calls)
{
    if (!c || !stress) return BCG_E_ARG;
    const int n = c->n;
    if (n > BCG_NOALLOC_MAX_CELLS) return BCG_E_UNSUPPORTED;
    int dev = -1;
    BCG_CUDA_TRY(cudaGetDevice(&dev));
    if (dev != c->device) return BCG_E_ARG;
    double* base = nullptr;
    int rc = noalloc_staging(&base);
    if (rc) return rc;
    double* ds = base;
    double* df = base + 5 * (size_t)BCG_NOALLOC_MAX_CELLS;
    unsigned long long* cnt = reinterpret_cast<unsigned long long*>(base + 8 * (size_t)BCG_NOALLOC_MAX_CELLS);
    /* the counter still holds the previous call's count */
    BCG_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(*cnt), c->stream));
    if (n > 0) {
        k_mean_stress<<<(n + 127) / 128, 128, 0, c->stream>>>(n, c->rec[c->cur], c->nbr, c->ncount, field_ptrs(c),
                                                              mech_params(c), ds, fnet ? df : nullptr, cnt, c->status);
        c->launches++;
        BCG_CUDA_TRY(cudaGetLastError());
        BCG_CUDA_TRY(cudaMemcpyAsync(stress, ds, sizeof(double) * 5 * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
        if (fnet) BCG_CUDA_TRY(cudaMemcpyAsync(fnet, df, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
    }
    unsigned long long h = 0;
    BCG_CUDA_TRY(cudaMemcpyAsync(&h, cnt, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    rc = ctx_check_status(c);
    if (fcw_calls) *fcw_calls = (int64_t)h;
    return rc;
}

extern "C" int bcg_int_move_grow_launch(bcg_ctx* c, double dt) { return c ? move_grow_launch(c, dt) : BCG_E_ARG; }
extern "C" int bcg_int_move_grow_finish(bcg_ctx* c, int* n_div, int64_t* fcw) { return c ? move_grow_finish(c, n_div, fcw) : BCG_E_ARG; }
extern "C" int bcg_int_divide_launch(bcg_ctx* c, const float* draws, int n, double t) { return c ? divide_launch(c, draws, n, t) : BCG_E_ARG; }
extern "C" int bcg_int_divide_finish(bcg_ctx* c, int* done, int* lineage) { return c ? divide_finish(c, done, lineage) : BCG_E_ARG; }

