/*
 * mech.cu -- cell binning, neighbour lists, the mechanics step (MoveCell +
 * GrowCell) and the division loop, as sm_100a kernels.
 *
 * Reference: AgentBasedModel-BacColonyGrowth/ UniformGrid.h, Neighbours.cpp,
 * Forces.cpp, Integrate.cpp, grow.cpp, Cells.cpp, Simulation.cpp:330-413.
 */
#include "ctx.cuh"
#include "cellmath.cuh"
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
    int cnt = 0;
    int* out = nbr + (size_t)me * mp.kmax;
    const int YZ = mp.box_y * mp.box_z;
    for (int za = max(zi - 1, 0); za < min(zi + 2, mp.box_z); za++)
        for (int ya = max(yi - 1, 0); ya < min(yi + 2, mp.box_y); ya++)
            for (int xa = max(xi - 1, 0); xa < min(xi + 2, mp.box_x); xa++) {
                int b = xa * YZ + ya * mp.box_z + za;
                int s = box_start[b], e = box_start[b + 1];
                if (e - s > mp.box_cap) e = s + mp.box_cap;   /* overfull: error already raised by the binning */
                for (int t = s; t < e; t += 32) {
                    int j = (t + lane < e) ? box_ids[t + lane] : -1;
                    bool keep = false;
                    if (j >= 0 && j != me && !(moved && moved[j])) {
                        Cst bj = COH ? load_cst_coh(&rec[j]) : load_cst(&rec[j]);
                        keep = keep_neighbour(a.p, a.q, a.L, a.R, acm, bj.p, bj.q, mp.rc);
                    }
                    unsigned m = __ballot_sync(0xffffffffu, keep);
                    int pos = cnt + __popc(m & ((1u << lane) - 1));
                    if (keep && pos < mp.kmax) out[pos] = j;
                    cnt += __popc(m);
                }
                for (int t = 0; t < ndelta; t += 32) {
                    int j = -1;
                    if (t + lane < ndelta && delta_box[t + lane] == b) j = delta_ids[t + lane];
                    bool keep = false;
                    if (j >= 0 && j != me) {
                        Cst bj = COH ? load_cst_coh(&rec[j]) : load_cst(&rec[j]);
                        keep = keep_neighbour(a.p, a.q, a.L, a.R, acm, bj.p, bj.q, mp.rc);
                    }
                    unsigned m = __ballot_sync(0xffffffffu, keep);
                    int pos = cnt + __popc(m & ((1u << lane) - 1));
                    if (keep && pos < mp.kmax) out[pos] = j;
                    cnt += __popc(m);
                }
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
template <int G>
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
        if (pair_force(a, cm, b, mp, f, r)) {
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

template <int G>
__global__ void __launch_bounds__(256) k_move_grow(int n, int nbinned, const int* __restrict__ order,
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
        sum_forces_group<G>(o, me, old, list, cnt, wall_z, fp, mp, F, T, sf, df, near1);
        Cst tmp = o;
        half_kick(dt, F, T, o, tmp.v, tmp.w);
        V3 rcmp = sub3(o.p, ocm), rcmq = sub3(o.q, ocm);
        V3 vp = add3(tmp.v, cross3(tmp.w, rcmp)), vq = add3(tmp.v, cross3(tmp.w, rcmq));
        tmp.p = add3(o.p, scl3(vp, dt));
        tmp.q = add3(o.q, scl3(vq, dt));
        tmp.p.y = 0; tmp.q.y = 0;
        sum_forces_group<G>(tmp, me, old, list, cnt, wall_z, fp, mp, F, T, sf, df, near2);
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

static int g_group = 4;   /* lanes per cell in the force loop (tunable) */
extern "C" int bcg_set_force_group(int g)
{
    if (g != 1 && g != 2 && g != 4 && g != 8 && g != 16) return BCG_E_ARG;
    g_group = g;
    return BCG_OK;
}

/* Cells are walked in the order of the last binning (spatially coherent,
 * so neighbouring groups share record lines in L1/L2); cells created after
 * that binning follow in id order. */
extern "C" int bcg_move_grow(bcg_ctx* c, double dt, int* n_div, int64_t* fcw_calls)
{
    if (!c) return BCG_E_ARG;
    timer_begin(c, BCG_T_MOVE_GROW);
    int n = c->n;
    BCG_CUDA_TRY(cudaMemsetAsync(c->div_count, 0, sizeof(int), c->stream));
    BCG_CUDA_TRY(cudaMemsetAsync(c->fcw_count, 0, sizeof(unsigned long long), c->stream));
    if (n > 0) {
        MechParams mp = mech_params(c);
        FieldPtrs fp = field_ptrs(c);
        int nb = c->n_binned < n ? c->n_binned : n;
        const int threads = 256;
        long tot = (long)n * g_group;
        unsigned blocks = (unsigned)((tot + threads - 1) / threads);
        const CellRec* old = c->rec[c->cur];
        CellRec* nw = c->rec[c->cur ^ 1];
        switch (g_group) {
        case 1: k_move_grow<1><<<blocks, threads, 0, c->stream>>>(n, nb, c->box_ids, old, nw, c->nbr, c->ncount, c->soa, fp, mp, dt, c->div_list, c->div_count, c->fcw_count, c->status); break;
        case 2: k_move_grow<2><<<blocks, threads, 0, c->stream>>>(n, nb, c->box_ids, old, nw, c->nbr, c->ncount, c->soa, fp, mp, dt, c->div_list, c->div_count, c->fcw_count, c->status); break;
        case 4: k_move_grow<4><<<blocks, threads, 0, c->stream>>>(n, nb, c->box_ids, old, nw, c->nbr, c->ncount, c->soa, fp, mp, dt, c->div_list, c->div_count, c->fcw_count, c->status); break;
        case 8: k_move_grow<8><<<blocks, threads, 0, c->stream>>>(n, nb, c->box_ids, old, nw, c->nbr, c->ncount, c->soa, fp, mp, dt, c->div_list, c->div_count, c->fcw_count, c->status); break;
        default: k_move_grow<16><<<blocks, threads, 0, c->stream>>>(n, nb, c->box_ids, old, nw, c->nbr, c->ncount, c->soa, fp, mp, dt, c->div_list, c->div_count, c->fcw_count, c->status); break;
        }
        c->launches++;
        BCG_CUDA_TRY(cudaGetLastError());
    }
    timer_end(c, BCG_T_MOVE_GROW, n > 0 ? 1 : 0);
    /* the two counters are the only values the host needs this step */
    int* hp = (int*)c->pinned;
    BCG_CUDA_TRY(cudaMemcpyAsync(hp, c->div_count, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    BCG_CUDA_TRY(cudaMemcpyAsync(hp + 2, c->fcw_count, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    int rc = ctx_check_status(c);
    if (rc) return rc;
    c->last_ndiv = hp[0];
    if (n_div) *n_div = hp[0];
    if (fcw_calls) *fcw_calls = (int64_t)(*(unsigned long long*)(hp + 2));
    return BCG_OK;
}

/* ======================================================================= */
/* division loop                                                            */
/* ======================================================================= */
#define DIV_SORT_MAX 8192
#define DIV_THREADS 512

/* divide(), grow.cpp:107-186, for mother m into daughter d; u[0..8] are the
 * nine (float)rand()/RAND_MAX draws in call order. */
__device__ void divide_pair(int m, int d, const float* u, double t, CellRec* rec, CellSoA soa, const MechParams& mp)
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
    rec[m] = rm;
    rec[d] = rd;
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

/* Simulation.cpp:380-404 in one CTA: divisions in ascending parent order;
 * each applies divide(), moves the mother / adds the daughter in the box
 * structure, and rebuilds the lists of {mother, mother's neighbours,
 * daughter} (Neighbours.cpp:39-55) with the warps of the block. */
__global__ void __launch_bounds__(DIV_THREADS) k_divide(int n_start, int ndiv, int cap, double t,
        const float* __restrict__ draws, CellRec* rec, CellSoA soa, MechParams mp,
        const int* __restrict__ div_list, int* nbr, int* ncount,
        const int* __restrict__ box_start, const int* __restrict__ box_ids,
        int* moved, int* delta_ids, int* delta_box, int* lineage, int* out, DevStatus* st)
{
    __shared__ int sd[DIV_SORT_MAX];
    __shared__ int idl[1 + 1024 + 1];
    __shared__ int s_len;
    int P2 = 1;
    while (P2 < ndiv) P2 <<= 1;
    for (int i = threadIdx.x; i < P2; i += blockDim.x) sd[i] = i < ndiv ? div_list[i] : 0x7fffffff;
    __syncthreads();
    /* bitonic sort, ascending */
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
    int N = n_start, done = 0;
    const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int d = 0; d < ndiv; d++) {
        if (N > cap - 1) { if (threadIdx.x == 0) dev_error(st, BCG_E_MAXCELLS, d); break; }
        int m = sd[d];
        if (threadIdx.x == 0) {
            divide_pair(m, N, draws + 9 * (size_t)d, t, rec, soa, mp);
            int xi, yi, zi;
            Cst a = load_cst(&rec[m]), b = load_cst(&rec[N]);
            int bm = box_address(avg_pq(a.p, a.q), mp, xi, yi, zi);
            int bd = box_address(avg_pq(b.p, b.q), mp, xi, yi, zi);
            if (bm < 0) { dev_error(st, BCG_E_OUT_OF_GRID, m); bm = 0; }
            if (bd < 0) { dev_error(st, BCG_E_OUT_OF_GRID, N); bd = 0; }
            moved[m] = 1;
            delta_ids[2 * d] = m; delta_box[2 * d] = bm;
            delta_ids[2 * d + 1] = N; delta_box[2 * d + 1] = bd;
            lineage[2 * d] = m; lineage[2 * d + 1] = N;
            int cnt = ncount[m];
            s_len = cnt + 2;
            idl[0] = m;
            idl[cnt + 1] = N;
        }
        __syncthreads();
        int len = s_len;
        for (int i = threadIdx.x; i < len - 2; i += blockDim.x) idl[1 + i] = nbr[(size_t)m * mp.kmax + i];
        __syncthreads();
        for (int k = warp; k < len; k += nwarps)
            warp_rebuild_one<true>(idl[k], rec, mp, box_start, box_ids, moved, delta_ids, delta_box, 2 * (d + 1), nbr, ncount, st);
        __syncthreads();
        N++; done++;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * done; i += blockDim.x) moved[delta_ids[i]] = 0;
    if (threadIdx.x == 0) { out[0] = done; out[1] = N; }
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

extern "C" int bcg_divide(bcg_ctx* c, const float* draws, int n_draw_sets, double t, int* n_done, int* lineage)
{
    if (!c) return BCG_E_ARG;
    if (n_draw_sets != c->last_ndiv) return BCG_E_ARG;
    timer_begin(c, BCG_T_DIVIDE);
    int done = 0;
    int ndiv = c->last_ndiv;
    if (ndiv > DIV_SORT_MAX) return BCG_E_UNSUPPORTED;
    if (ndiv > 0) {
        if (!draws) return BCG_E_ARG;
        int nb = c->cur ^ 1;
        int rc = bin_cells(c, nb);
        if (rc) return rc;
        size_t db = sizeof(float) * 9 * (size_t)ndiv;
        rc = ensure_pinned(c, db + 64);
        if (rc) return rc;
        memcpy(c->pinned, draws, db);
        BCG_CUDA_TRY(cudaMemcpyAsync(c->draws_dev, c->pinned, db, cudaMemcpyHostToDevice, c->stream));
        k_divide<<<1, DIV_THREADS, 0, c->stream>>>(c->n, ndiv, c->cap, t, c->draws_dev, c->rec[nb], c->soa,
            mech_params(c), c->div_list, c->nbr, c->ncount, c->box_start, c->box_ids,
            c->moved, c->delta_ids, c->delta_box, c->lineage, c->n_done_dev, c->status);
        c->launches++;
        BCG_CUDA_TRY(cudaGetLastError());
        int* hp = (int*)c->pinned;
        BCG_CUDA_TRY(cudaMemcpyAsync(hp, c->n_done_dev, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        rc = ctx_check_status(c);
        done = hp[0];
        if (lineage && done > 0) {
            BCG_CUDA_TRY(cudaMemcpy(lineage, c->lineage, sizeof(int) * 2 * (size_t)done, cudaMemcpyDeviceToHost));
        }
        c->n += done;
        c->cur ^= 1;
        c->last_ndiv = 0;
        timer_end(c, BCG_T_DIVIDE, 6);
        if (n_done) *n_done = done;
        return rc;
    }
    c->cur ^= 1;
    c->last_ndiv = 0;
    timer_end(c, BCG_T_DIVIDE, 0);
    if (n_done) *n_done = 0;
    return BCG_OK;
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
