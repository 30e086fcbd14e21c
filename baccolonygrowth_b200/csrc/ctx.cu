/*
 * ctx.cu -- context lifetime, cell upload/download, field access, status
 * and timers of the C ABI (include/bcg.h).
 */
#include "ctx.cuh"
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

static thread_local cudaError_t g_last_cuda = cudaSuccess;
void bcg_set_cuda_error(cudaError_t e) { g_last_cuda = e; }

extern "C" const char* bcg_status_string(int s)
{
    switch (s) {
    case BCG_OK: return "ok";
    case BCG_E_ARG: return "bad argument";
    case BCG_E_CUDA: return g_last_cuda != cudaSuccess ? cudaGetErrorString(g_last_cuda) : "CUDA error";
    case BCG_E_BOX_OVERFLOW: return "Tried to add too many cells (box overflow)";
    case BCG_E_NEIGH_OVERFLOW: return "Too many neighbours!";
    case BCG_E_OUT_OF_GRID: return "Cells have expanded farther than boxes allows";
    case BCG_E_NAN: return "non-finite cell state";
    case BCG_E_MAXCELLS: return "Too many cells!";
    case BCG_E_TIMEOUT: return "device wait timed out";
    case BCG_E_UNSUPPORTED: return "unsupported parameter combination";
    case BCG_E_NEED_MORE_BOXES: return "Need more boxes";
    case BCG_E_NO_DEVICE: return "no CUDA device";
    case BCG_E_IO: return "Can't open output file.";
    default: return "unknown status";
    }
}

MechParams mech_params(const bcg_ctx* c)
{
    MechParams m;
    const bcg_params& P = c->P;
    m.box_x = P.box_x; m.box_y = P.box_y; m.box_z = P.box_z; m.rgh = P.refinement_grid_height;
    m.xh = P.box_x * P.refinement_grid_height;
    m.kmax = c->kmax; m.box_cap = P.max_cells_per_box;
    m.box_length = P.box_length; m.rc = P.rc; m.cell_radius = P.cell_radius; m.l_divide = P.l_divide;
    m.k_cc = P.k_cc; m.k_wc = P.k_wc; m.var_l = P.var_l; m.var_angle = P.var_angle; m.var_pos = P.var_pos;
    m.viscosity = P.viscosity; m.gamma_t = P.gamma_t; m.cell_mu = P.cell_mu; m.wall_mu = P.wall_mu;
    m.tension = P.tension; m.delta_h = P.delta_h; m.cross_feeding = P.cross_feeding;
    return m;
}

FieldPtrs field_ptrs(const bcg_ctx* c)
{
    FieldPtrs f;
    f.height = c->height; f.nx = c->nrm_x; f.ny = c->nrm_y; f.nz = c->nrm_z; f.wall = c->wall;
    f.gr1 = c->env[0].gr1; f.gr2 = c->env[0].gr2;
    return f;
}

int ctx_check_status(bcg_ctx* c)
{
    if (c->pending_error) {
        /* a launch that could not be set up (the work after it was queued) */
        const int rc = c->pending_error;
        c->pending_error = BCG_OK;
        cudaStreamSynchronize(c->stream);
        return rc;
    }
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { g_last_cuda = e; return BCG_E_CUDA; }
    DevStatus st;
    e = cudaMemcpy(&st, c->status, sizeof(st), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { g_last_cuda = e; return BCG_E_CUDA; }
    if (st.code) {
        DevStatus z = {0, 0};
        cudaMemcpy(c->status, &z, sizeof(z), cudaMemcpyHostToDevice);
        return st.code;
    }
    return BCG_OK;
}

int ensure_pinned(bcg_ctx* c, size_t bytes)
{
    if (bytes <= c->pinned_bytes) return BCG_OK;
    if (c->pinned) { cudaStreamSynchronize(c->stream); cudaFreeHost(c->pinned); c->pinned = nullptr; c->pinned_bytes = 0; }
    size_t b = bytes < 4096 ? 4096 : bytes;
    BCG_CUDA_TRY(cudaMallocHost(&c->pinned, b));
    c->pinned_bytes = b;
    return BCG_OK;
}

void timer_begin(bcg_ctx* c, int t)
{
    if (c->timers_on) cudaEventRecord(c->ev[t][0], c->stream);
}
void timer_end(bcg_ctx* c, int t, int launches)
{
    c->timer_launches[t] += launches;
    if (c->timers_on) {
        cudaEventRecord(c->ev[t][1], c->stream);
        cudaEventSynchronize(c->ev[t][1]);
        float ms = 0;
        cudaEventElapsedTime(&ms, c->ev[t][0], c->ev[t][1]);
        c->timer_ms[t] += ms;
    }
}

extern "C" int bcg_enable_timers(bcg_ctx* c, int on)
{
    if (!c) return BCG_E_ARG;
    c->timers_on = on;
    for (int t = 0; t < BCG_T_COUNT; t++) { c->timer_ms[t] = 0; c->timer_launches[t] = 0; }
    return BCG_OK;
}
extern "C" int bcg_get_timer(bcg_ctx* c, int t, double* ms, int64_t* launches)
{
    if (!c || t < 0 || t >= BCG_T_COUNT) return BCG_E_ARG;
    if (ms) *ms = c->timer_ms[t];
    if (launches) *launches = c->timer_launches[t];
    return BCG_OK;
}

static void timeline_free(bcg_ctx* c)
{
    for (int i = 0; i < c->tl_cap; i++)
        if (c->tl_ev[i]) cudaEventDestroy(c->tl_ev[i]);
    free(c->tl_ev);
    free(c->tl_tag);
    c->tl_ev = nullptr;
    c->tl_tag = nullptr;
    c->tl_cap = c->tl_n = 0;
}

extern "C" int bcg_timeline_enable(bcg_ctx* c, int capacity)
{
    if (!c || capacity < 0) return BCG_E_ARG;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->aux_stream) cudaStreamSynchronize(c->aux_stream);
    timeline_free(c);
    if (capacity == 0) return BCG_OK;
    c->tl_ev = (cudaEvent_t*)calloc((size_t)capacity, sizeof(cudaEvent_t));
    c->tl_tag = (int*)calloc((size_t)capacity, sizeof(int));
    if (!c->tl_ev || !c->tl_tag) { free(c->tl_ev); free(c->tl_tag); c->tl_ev = nullptr; c->tl_tag = nullptr; return BCG_E_ARG; }
    c->tl_cap = capacity;
    for (int i = 0; i < capacity; i++) {
        if (cudaEventCreate(&c->tl_ev[i]) != cudaSuccess) {
            g_last_cuda = cudaGetLastError();
            timeline_free(c);
            return BCG_E_CUDA;
        }
    }
    return BCG_OK;
}

/* one mark on the context's stream (aux = 0) or its second stream */
extern "C" void bcg_int_tl_mark(bcg_ctx* c, int aux, int tag)
{
    if (!c || c->tl_n >= c->tl_cap) return;
    if (cudaEventRecord(c->tl_ev[c->tl_n], aux ? c->aux_stream : c->stream) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    c->tl_tag[c->tl_n++] = tag;
}

extern "C" int bcg_timeline_read(bcg_ctx* c, int* tags, float* ms, int capacity, int* n)
{
    if (!c || capacity < 0 || (capacity > 0 && (!tags || !ms))) return BCG_E_ARG;
    if (c->aux_stream) BCG_CUDA_TRY(cudaStreamSynchronize(c->aux_stream));
    const int rc = ctx_check_status(c);
    const int m = c->tl_n < capacity ? c->tl_n : capacity;
    for (int i = 0; i < m; i++) {
        tags[i] = c->tl_tag[i];
        ms[i] = 0.0f;
        BCG_CUDA_TRY(cudaEventElapsedTime(&ms[i], c->tl_ev[0], c->tl_ev[i]));
    }
    if (n) *n = m;
    c->tl_n = 0;
    return rc;
}

extern "C" void* bcg_stream(bcg_ctx* c) { return c ? (void*)c->stream : nullptr; }
extern "C" int bcg_synchronize(bcg_ctx* c) { return c ? ctx_check_status(c) : BCG_E_ARG; }
extern "C" long long bcg_kernel_launches(bcg_ctx* c) { return c ? c->launches : 0; }

/* ----------------------------------------------------------------------- */
__global__ void k_fill(double* p, double v, size_t n)
{
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}
static int dalloc(void** p, size_t bytes)
{
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e != cudaSuccess) { g_last_cuda = e; return BCG_E_CUDA; }
    return BCG_OK;
}
#define DALLOC(ptr, bytes) do { int r_ = dalloc((void**)&(ptr), (bytes)); if (r_) { bcg_destroy(c); return r_; } } while (0)
static int fill(bcg_ctx* c, double* p, double v, size_t n)
{
    if (n == 0) return BCG_OK;
    k_fill<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(p, v, n);
    c->launches++;
    return cudaGetLastError() == cudaSuccess ? BCG_OK : BCG_E_CUDA;
}

static int mg_nx(const bcg_params& P, int l) { int d = 1 << l, d0 = 1 << P.max_levels_mg; int v = P.box_x * d0 / d / 2; return v < P.box_x ? v : P.box_x; }
static int mg_nz(const bcg_params& P, int l) { int d = 1 << l, d0 = 1 << P.max_levels_mg; int v = P.box_z_agar * d0 / d / 2; return v < P.box_z_agar ? v : P.box_z_agar; }

extern "C" int bcg_create(const bcg_params* p, bcg_ctx** out)
{
    if (!p || !out) return BCG_E_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return BCG_E_NO_DEVICE;
    if (p->box_y != 1) return BCG_E_UNSUPPORTED;            /* the reference is 2-D x-z */
    if (p->cross_feeding != 0 || p->interface_condition != 1) return BCG_E_UNSUPPORTED;
    if (p->var_pos != 0.0) return BCG_E_UNSUPPORTED;        /* wall locus needs the per-call rand value */
    if (p->max_levels_mg > BCG_MAX_AGAR_LEVELS || p->mg_levels > BCG_MAX_MG_LEVELS) return BCG_E_UNSUPPORTED;
    if (p->max_neighbours < 1 || p->max_neighbours > 1024 || p->box_length <= 0) return BCG_E_ARG;
    bcg_ctx* c = (bcg_ctx*)calloc(1, sizeof(bcg_ctx));
    if (!c) return BCG_E_ARG;
    c->P = *p;
    c->relax_mode = 3;
    cudaGetDevice(&c->device);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { free(c); return BCG_E_CUDA; }
    if (cudaStreamCreateWithFlags(&c->aux_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess) {
        bcg_destroy(c);
        return BCG_E_CUDA;
    }
    for (int t = 0; t < BCG_T_COUNT; t++) { cudaEventCreate(&c->ev[t][0]); cudaEventCreate(&c->ev[t][1]); }
    const size_t cap = (size_t)p->max_cells;
    c->cap = p->max_cells;
    c->kmax = p->max_neighbours;
    DALLOC(c->rec[0], cap * sizeof(CellRec));
    DALLOC(c->rec[1], cap * sizeof(CellRec));
    c->stage_cells = c->cap < CTX_STAGE_CELLS ? (c->cap > 0 ? c->cap : 1) : CTX_STAGE_CELLS;
    DALLOC(c->stage, (size_t)c->stage_cells * sizeof(bcg_cell));
    CellSoA& s = c->soa;
    DALLOC(s.ldiv, cap * 8); DALLOC(s.gr, cap * 8); DALLOC(s.tp, cap * 8); DALLOC(s.tq, cap * 8);
    DALLOC(s.ap, cap * 4); DALLOC(s.aq, cap * 4);
    DALLOC(s.dfx, cap * 8); DALLOC(s.dfy, cap * 8); DALLOC(s.dfz, cap * 8);
    DALLOC(s.sfx, cap * 8); DALLOC(s.sfy, cap * 8); DALLOC(s.sfz, cap * 8);
    DALLOC(s.type, cap * 4); DALLOC(s.anc, cap * 4);
    DALLOC(c->nbr, cap * c->kmax * 4);
    DALLOC(c->ncount, cap * 4);
    c->nbox = p->box_x * p->box_y * p->box_z;
    DALLOC(c->box_cnt, (size_t)c->nbox * 4);
    DALLOC(c->box_start, ((size_t)c->nbox + 1) * 4);
    DALLOC(c->box_ids, cap * 4);
    DALLOC(c->cell_box, cap * 4);
    DALLOC(c->scan_tmp, 4096 * 4 + 64);
    DALLOC(c->div_list, cap * 4);
    DALLOC(c->div_count, 64);
    DALLOC(c->fcw_count, 64);
    DALLOC(c->moved, cap * 4);
    DALLOC(c->delta_ids, 2 * cap * 4);
    DALLOC(c->delta_box, 2 * cap * 4);
    DALLOC(c->lineage, 2 * cap * 4);
    DALLOC(c->n_done_dev, 64);
    DALLOC(c->draws_dev, 9 * cap * 4);
    DALLOC(c->div_rec, 2 * (size_t)DIV_SORT_MAX * sizeof(CellRec));
    DALLOC(c->div_box, 2 * (size_t)DIV_SORT_MAX * 4);
    DALLOC(c->div_rect, (size_t)DIV_SORT_MAX * sizeof(int4));
    DALLOC(c->div_pairs, (size_t)DIV_PAIR_CAP * sizeof(int2));
    DALLOC(c->div_par, (size_t)DIV_SORT_MAX * 4);
    DALLOC(c->div_order, (size_t)DIV_SORT_MAX * 4);
    DALLOC(c->div_grp, 2 * (size_t)DIV_SORT_MAX * 4);
    DALLOC(c->status, sizeof(DevStatus));
    BCG_CUDA_TRY(cudaMemsetAsync(c->status, 0, sizeof(DevStatus), c->stream));
    BCG_CUDA_TRY(cudaMemsetAsync(c->moved, 0, cap * 4, c->stream));
    BCG_CUDA_TRY(cudaMemsetAsync(c->ncount, 0, cap * 4, c->stream));
    BCG_CUDA_TRY(cudaMemsetAsync(c->box_start, 0, ((size_t)c->nbox + 1) * 4, c->stream));
    /* fields */
    const size_t X = p->box_x, Z = p->box_z, XH = (size_t)p->box_x * p->refinement_grid_height;
    DALLOC(c->height, XH * 8); DALLOC(c->rough_height, XH * 8);
    DALLOC(c->nrm_x, XH * 8); DALLOC(c->nrm_y, XH * 8); DALLOC(c->nrm_z, XH * 8);
    DALLOC(c->wall, X * p->box_y * 8);
    int rc;
    if ((rc = fill(c, c->height, p->cell_radius, XH)) || (rc = fill(c, c->rough_height, p->cell_radius, XH)) ||
        (rc = fill(c, c->nrm_x, 0.0, XH)) || (rc = fill(c, c->nrm_y, 0.0, XH)) || (rc = fill(c, c->nrm_z, -1.0, XH)) ||
        (rc = fill(c, c->wall, 0.0, X * p->box_y))) { bcg_destroy(c); return rc; }
    for (int b = 0; b < 2; b++) {
        EnvBuf& e = c->env[b];
        double** arrs[] = {&e.C, &e.W, &e.A, &e.O, &e.gr1, &e.gr2, &e.ph, &e.hydrox, &e.acetic, &e.buffer};
        const double init[] = {0.0, 0.0, 0.0, p->max_o2, 0.0, 0.0, 7.0, 0.0, 0.0, 0.0};
        for (int k = 0; k < 10; k++) {
            DALLOC(*arrs[k], X * Z * 8);
            if ((rc = fill(c, *arrs[k], init[k], X * Z))) { bcg_destroy(c); return rc; }
        }
        for (int k = 0; k < 7 && b == 0; k++) {
            DALLOC(e.extra[k], X * Z * 8);
            if ((rc = fill(c, e.extra[k], 0.0, X * Z))) { bcg_destroy(c); return rc; }
        }
        WallBuf& w = c->wal[b];
        for (int l = 0; l < p->max_levels_mg; l++) {
            DALLOC(w.C[l], X * 8); DALLOC(w.W[l], X * 8); DALLOC(w.O[l], X * 8); DALLOC(w.A[l], X * 8);
            if ((rc = fill(c, w.C[l], p->max_carbon, X)) || (rc = fill(c, w.W[l], 0.0, X)) ||
                (rc = fill(c, w.O[l], p->max_o2, X)) || (rc = fill(c, w.A[l], 0.0, X))) { bcg_destroy(c); return rc; }
        }
    }
    double** f3[] = {&c->rd, &c->inside, &c->rds, &c->ds, &c->dens};
    for (auto a : f3) { DALLOC(*a, X * Z * 8); if ((rc = fill(c, *a, 0.0, X * Z))) { bcg_destroy(c); return rc; } }
    double** f2[] = {&c->rws, &c->wds, &c->rw, &c->wd};
    for (auto a : f2) { DALLOC(*a, X * 8); if ((rc = fill(c, *a, 0.0, X))) { bcg_destroy(c); return rc; } }
    DALLOC(c->bbox, 64);
    BCG_CUDA_TRY(cudaMemsetAsync(c->bbox, 0, 64, c->stream));
    /* multigrid levels, Multigrid.cpp:5-33: LocalAga defaults in all arrays */
    c->mg_levels = p->mg_levels;
    for (int l = 0; l < c->mg_levels; l++) {
        MgLevel& L = c->mg[l];
        L.nx = mg_nx(*p, l); L.nz = mg_nz(*p, l);
        /* coarse levels may have nz = 0 (one row; the small input's coarsest
         * level is 4 x 0), never nx < 2 */
        if (L.nx < 2 || L.nz < 0) { bcg_destroy(c); return BCG_E_ARG; }
        L.pitch = ((L.nx + 1) + 31) / 32 * 32;
        size_t np = (size_t)L.pitch * (L.nz + 1);
        const double init[3] = {p->max_carbon, p->max_o2, 0.0};
        for (int sp = 0; sp < 3; sp++) {
            DALLOC(L.sol[sp], np * 8); DALLOC(L.res[sp], np * 8); DALLOC(L.err[sp], np * 8);
            DALLOC(L.errf[sp], np * 4); DALLOC(L.resf[sp], np * 4);
            DALLOC(L.err2[sp], np * 8); DALLOC(L.errf2[sp], np * 4);
            BCG_CUDA_TRY(cudaMemsetAsync(L.err2[sp], 0, np * 8, c->stream));
            BCG_CUDA_TRY(cudaMemsetAsync(L.errf2[sp], 0, np * 4, c->stream));
            BCG_CUDA_TRY(cudaMemsetAsync(L.errf[sp], 0, np * 4, c->stream));
            BCG_CUDA_TRY(cudaMemsetAsync(L.resf[sp], 0, np * 4, c->stream));
            if ((rc = fill(c, L.sol[sp], init[sp], np)) || (rc = fill(c, L.res[sp], init[sp], np)) ||
                (rc = fill(c, L.err[sp], init[sp], np))) { bcg_destroy(c); return rc; }
        }
    }
    DALLOC(c->mg_scratch, 1 << 20);
    if ((rc = mg_kernel_attributes()) || (rc = mech_kernel_attributes())) { bcg_destroy(c); return rc; }
    rc = ensure_pinned(c, 1 << 16);
    if (rc) { bcg_destroy(c); return rc; }
    rc = ctx_check_status(c);
    if (rc) { bcg_destroy(c); return rc; }
    c->cur = 0; c->n = 0; c->n_binned = 0;
    *out = c;
    return BCG_OK;
}

extern "C" int bcg_destroy(bcg_ctx* c)
{
    if (!c) return BCG_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    void* ptrs[] = {c->rec[0], c->rec[1], c->stage, c->soa.ldiv, c->soa.gr, c->soa.tp, c->soa.tq, c->soa.ap, c->soa.aq,
                    c->soa.dfx, c->soa.dfy, c->soa.dfz, c->soa.sfx, c->soa.sfy, c->soa.sfz, c->soa.type, c->soa.anc,
                    c->nbr, c->ncount, c->box_cnt, c->box_start, c->box_ids, c->cell_box, c->scan_tmp,
                    c->div_list, c->div_count, c->fcw_count, c->moved, c->delta_ids, c->delta_box, c->lineage,
                    c->n_done_dev, c->draws_dev, c->div_rec, c->div_box, c->div_rect, c->div_pairs, c->div_par,
                    c->div_order, c->div_grp, c->status, c->height, c->rough_height, c->nrm_x, c->nrm_y, c->nrm_z,
                    c->wall, c->rd, c->inside, c->rds, c->ds, c->dens, c->rws, c->wds, c->rw, c->wd, c->bbox, c->mg_scratch};
    for (void* q : ptrs) if (q) cudaFree(q);
    for (int b = 0; b < 2; b++) {
        EnvBuf& e = c->env[b];
        void* ea[] = {e.C, e.W, e.A, e.O, e.gr1, e.gr2, e.ph, e.hydrox, e.acetic, e.buffer};
        for (void* q : ea) if (q) cudaFree(q);
        for (double* q : e.extra) if (q) cudaFree(q);
        for (int l = 0; l < BCG_MAX_AGAR_LEVELS; l++) {
            void* wa[] = {c->wal[b].C[l], c->wal[b].W[l], c->wal[b].O[l], c->wal[b].A[l]};
            for (void* q : wa) if (q) cudaFree(q);
        }
    }
    for (int l = 0; l < BCG_MAX_MG_LEVELS; l++)
        for (int sp = 0; sp < 3; sp++) {
            void* ma[] = {c->mg[l].sol[sp], c->mg[l].res[sp], c->mg[l].err[sp], c->mg[l].errf[sp], c->mg[l].resf[sp],
                          c->mg[l].err2[sp], c->mg[l].errf2[sp]};
            for (void* q : ma) if (q) cudaFree(q);
        }
    for (int b = 0; b < 2; b++)
        for (int l = 0; l < BCG_MAX_AGAR_LEVELS; l++)
            for (int sp = 0; sp < 4; sp++) if (c->leg[b][l][sp]) cudaFree(c->leg[b][l][sp]);
    if (c->leg_snap) cudaFree(c->leg_snap);
    if (c->leg_conv) cudaFree(c->leg_conv);
    for (int g = 0; g < 2; g++) if (c->nutrient_graph[g]) cudaGraphExecDestroy(c->nutrient_graph[g]);
    if (c->solve_graph) cudaGraphExecDestroy(c->solve_graph);
    if (c->pinned) cudaFreeHost(c->pinned);
    timeline_free(c);
    for (int t = 0; t < BCG_T_COUNT; t++) { if (c->ev[t][0]) cudaEventDestroy(c->ev[t][0]); if (c->ev[t][1]) cudaEventDestroy(c->ev[t][1]); }
    if (c->aux_stream) { cudaStreamSynchronize(c->aux_stream); cudaStreamDestroy(c->aux_stream); }
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->stream) cudaStreamDestroy(c->stream);
    free(c);
    return BCG_OK;
}

/* ----------------------------------------------------------------------- */
/* AoS <-> device layout                                                    */
/* ----------------------------------------------------------------------- */
/* records in[0..n) are cells off..off+n-1 */
__global__ void k_unpack(int n, int off, const bcg_cell* __restrict__ in, CellRec* __restrict__ rec, CellSoA s)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const bcg_cell& c = in[j];
    const int i = off + j;
    CellRec r;
    r.pL = make_double4(c.p.x, c.p.y, c.p.z, c.length);
    r.qR = make_double4(c.q.x, c.q.y, c.q.z, c.radius);
    r.v = make_double4(c.velocity.x, c.velocity.y, c.velocity.z, 0.0);
    r.w = make_double4(c.angular_velocity.x, c.angular_velocity.y, c.angular_velocity.z, 0.0);
    rec[i] = r;
    s.ldiv[i] = c.ldiv; s.gr[i] = c.growth_rate; s.tp[i] = c.time_p; s.tq[i] = c.time_q;
    s.ap[i] = c.age_p; s.aq[i] = c.age_q;
    s.dfx[i] = c.dyn_fric.x; s.dfy[i] = c.dyn_fric.y; s.dfz[i] = c.dyn_fric.z;
    s.sfx[i] = c.sta_fric.x; s.sfy[i] = c.sta_fric.y; s.sfz[i] = c.sta_fric.z;
    s.type[i] = c.type; s.anc[i] = c.ancestor;
}
/* cells off..off+n-1 into out[0..n) */
__global__ void k_pack(int n, int off, bcg_cell* __restrict__ out, const CellRec* __restrict__ rec, CellSoA s)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int i = off + j;
    bcg_cell c;
    CellRec r = rec[i];
    c.p.x = r.pL.x; c.p.y = r.pL.y; c.p.z = r.pL.z; c.length = r.pL.w;
    c.q.x = r.qR.x; c.q.y = r.qR.y; c.q.z = r.qR.z; c.radius = r.qR.w;
    c.velocity.x = r.v.x; c.velocity.y = r.v.y; c.velocity.z = r.v.z;
    c.angular_velocity.x = r.w.x; c.angular_velocity.y = r.w.y; c.angular_velocity.z = r.w.z;
    c.ldiv = s.ldiv[i]; c.growth_rate = s.gr[i]; c.time_p = s.tp[i]; c.time_q = s.tq[i];
    c.age_p = s.ap[i]; c.age_q = s.aq[i];
    c.dyn_fric.x = s.dfx[i]; c.dyn_fric.y = s.dfy[i]; c.dyn_fric.z = s.dfz[i];
    c.sta_fric.x = s.sfx[i]; c.sta_fric.y = s.sfy[i]; c.sta_fric.z = s.sfz[i];
    c.type = s.type[i]; c.ancestor = s.anc[i];
    out[j] = c;
}

void launch_pack_cells(bcg_ctx* c, bcg_cell* dst, cudaStream_t s, int moved)
{
    if (c->n <= 0) return;
    k_pack<<<(c->n + 255) / 256, 256, 0, s>>>(c->n, 0, dst, c->rec[moved ? c->cur ^ 1 : c->cur], c->soa);
    c->launches++;
}

/* The records pass through the context's staging buffer a chunk at a
 * time, copy and unpack in stream order (no allocation per call). */
extern "C" int bcg_upload_cells(bcg_ctx* c, const bcg_cell* cells, int n)
{
    if (!c || n < 0 || n > c->cap || (n > 0 && !cells)) return BCG_E_ARG;
    for (int off = 0; off < n; off += c->stage_cells) {
        const int m = n - off < c->stage_cells ? n - off : c->stage_cells;
        BCG_CUDA_TRY(cudaMemcpyAsync(c->stage, cells + off, sizeof(bcg_cell) * (size_t)m, cudaMemcpyHostToDevice, c->stream));
        k_unpack<<<(m + 255) / 256, 256, 0, c->stream>>>(m, off, c->stage, c->rec[c->cur], c->soa);
        c->launches++;
    }
    BCG_CUDA_TRY(cudaMemsetAsync(c->ncount, 0, sizeof(int) * (size_t)c->cap, c->stream));
    c->n = n;
    c->n_binned = 0;
    c->last_ndiv = 0;
    c->move_pending = 0;
    return ctx_check_status(c);
}

extern "C" int bcg_download_cells(bcg_ctx* c, bcg_cell* cells, int capacity, int* n)
{
    if (!c) return BCG_E_ARG;
    if (n) *n = c->n;
    int m = c->n < capacity ? c->n : capacity;
    if (m > 0 && !cells) return BCG_E_ARG;
    for (int off = 0; off < m; off += c->stage_cells) {
        const int k = m - off < c->stage_cells ? m - off : c->stage_cells;
        k_pack<<<(k + 255) / 256, 256, 0, c->stream>>>(k, off, c->stage, c->rec[c->cur], c->soa);
        c->launches++;
        BCG_CUDA_TRY(cudaMemcpyAsync(cells + off, c->stage, sizeof(bcg_cell) * (size_t)k, cudaMemcpyDeviceToHost, c->stream));
    }
    return ctx_check_status(c);
}

extern "C" int bcg_num_cells(bcg_ctx* c, int* n)
{
    if (!c || !n) return BCG_E_ARG;
    *n = c->n;
    return BCG_OK;
}

extern "C" int bcg_get_neighbours(bcg_ctx* c, int* counts, int* lists, int stride)
{
    if (!c || !counts || !lists || stride < 1) return BCG_E_ARG;
    int n = c->n;
    if (n == 0) return BCG_OK;
    int* tmp = (int*)malloc(sizeof(int) * (size_t)n * c->kmax);
    if (!tmp) return BCG_E_ARG;
    cudaError_t e1 = cudaMemcpyAsync(counts, c->ncount, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, c->stream);
    cudaError_t e2 = cudaMemcpyAsync(tmp, c->nbr, sizeof(int) * (size_t)n * c->kmax, cudaMemcpyDeviceToHost, c->stream);
    cudaError_t e3 = cudaStreamSynchronize(c->stream);
    if (e1 || e2 || e3) { free(tmp); g_last_cuda = e1 ? e1 : (e2 ? e2 : e3); return BCG_E_CUDA; }
    for (int i = 0; i < n; i++)
        for (int j = 0; j < counts[i] && j < stride && j < c->kmax; j++) lists[(size_t)i * stride + j] = tmp[(size_t)i * c->kmax + j];
    free(tmp);
    return BCG_OK;
}

extern "C" int bcg_set_neighbours(bcg_ctx* c, const int* counts, const int* lists, int stride)
{
    if (!c || !counts || !lists || stride < 1) return BCG_E_ARG;
    int n = c->n;
    if (n == 0) return BCG_OK;
    int* tmp = (int*)calloc((size_t)n * c->kmax, sizeof(int));
    if (!tmp) return BCG_E_ARG;
    for (int i = 0; i < n; i++) {
        if (counts[i] > c->kmax) { free(tmp); return BCG_E_NEIGH_OVERFLOW; }
        for (int j = 0; j < counts[i]; j++) tmp[(size_t)i * c->kmax + j] = lists[(size_t)i * stride + j];
    }
    cudaError_t e1 = cudaMemcpy(c->ncount, counts, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice);
    cudaError_t e2 = cudaMemcpy(c->nbr, tmp, sizeof(int) * (size_t)n * c->kmax, cudaMemcpyHostToDevice);
    free(tmp);
    if (e1 || e2) { g_last_cuda = e1 ? e1 : e2; return BCG_E_CUDA; }
    return BCG_OK;
}

/* ----------------------------------------------------------------------- */
/* fields                                                                   */
/* ----------------------------------------------------------------------- */
/* device pointer + element count (+ row layout for MG arrays) of a field */
struct FieldView { double* ptr; size_t n; int mg; int nx, nz, pitch; };

static int field_view(bcg_ctx* c, int f, int level, FieldView* v)
{
    const bcg_params& P = c->P;
    const size_t X = P.box_x, Z = P.box_z, XH = (size_t)P.box_x * P.refinement_grid_height;
    memset(v, 0, sizeof(*v));
    int e = 0;
    switch (f) {
    case BCG_F_HEIGHT: v->ptr = c->height; v->n = XH; return BCG_OK;
    case BCG_F_NORMAL_X: v->ptr = c->nrm_x; v->n = XH; return BCG_OK;
    case BCG_F_NORMAL_Z: v->ptr = c->nrm_z; v->n = XH; return BCG_OK;
    case BCG_F_WALL: v->ptr = c->wall; v->n = X; return BCG_OK;
    case BCG_F_DENSITY_SHIFT: v->ptr = c->ds; v->n = X * Z; return BCG_OK;
    case BCG_F_WALL_DENSITY_SHIFT: v->ptr = c->wds; v->n = X; return BCG_OK;
    case BCG_F_INSIDE: v->ptr = c->inside; v->n = X * Z; return BCG_OK;
    case BCG_F_DENSITY: v->ptr = c->dens; v->n = X * Z; return BCG_OK;
    case BCG_F_ROUGH_DENSITY: v->ptr = c->rd; v->n = X * Z; return BCG_OK;
    case BCG_F_ENV_CARBON: case BCG_F_OLDENV_CARBON: e = f == BCG_F_OLDENV_CARBON; v->ptr = c->env[e].C; v->n = X * Z; return BCG_OK;
    case BCG_F_ENV_WASTE: case BCG_F_OLDENV_WASTE: e = f == BCG_F_OLDENV_WASTE; v->ptr = c->env[e].W; v->n = X * Z; return BCG_OK;
    case BCG_F_ENV_OXYGEN: case BCG_F_OLDENV_OXYGEN: e = f == BCG_F_OLDENV_OXYGEN; v->ptr = c->env[e].O; v->n = X * Z; return BCG_OK;
    case BCG_F_ENV_ACETATE: case BCG_F_OLDENV_ACETATE: e = f == BCG_F_OLDENV_ACETATE; v->ptr = c->env[e].A; v->n = X * Z; return BCG_OK;
    case BCG_F_ENV_GROWTH1: v->ptr = c->env[0].gr1; v->n = X * Z; return BCG_OK;
    case BCG_F_ENV_GROWTH2: v->ptr = c->env[0].gr2; v->n = X * Z; return BCG_OK;
    case BCG_F_ENV_PH: v->ptr = c->env[0].ph; v->n = X * Z; return BCG_OK;
    case BCG_F_ENV_HYDROX: v->ptr = c->env[0].hydrox; v->n = X * Z; return BCG_OK;
    case BCG_F_ENV_ACETIC: v->ptr = c->env[0].acetic; v->n = X * Z; return BCG_OK;
    case BCG_F_ENV_BUFFER: v->ptr = c->env[0].buffer; v->n = X * Z; return BCG_OK;
    case BCG_F_ENV_GR_CAR_AER: case BCG_F_ENV_GR_CAR_ANA: case BCG_F_ENV_GR_ACE_AER:
    case BCG_F_ENV_Q_CAR_MNT: case BCG_F_ENV_Q_ACE_MNT: case BCG_F_ENV_P_ACE_MNT: case BCG_F_ENV_Q_OXY_MNT:
        v->ptr = c->env[0].extra[f - BCG_F_ENV_GR_CAR_AER]; v->n = X * Z; return BCG_OK;
    default: break;
    }
    if (f >= BCG_F_WALLF_CARBON && f <= BCG_F_OLDWALLF_ACETATE) {
        if (level < 0 || level >= P.max_levels_mg) return BCG_E_ARG;
        int b = f >= BCG_F_OLDWALLF_CARBON;
        int sp = (f - BCG_F_WALLF_CARBON) % 4;
        WallBuf& w = c->wal[b];
        v->ptr = sp == 0 ? w.C[level] : sp == 1 ? w.W[level] : sp == 2 ? w.O[level] : w.A[level];
        v->n = X;
        return BCG_OK;
    }
    if (f >= BCG_F_AGARF_CARBON && f <= BCG_F_AGARF_ACETATE) {
        /* FieldAgar[l](i,k) == Aga[l](i,k+1) after every solve (copyFromMG,
         * Multigrid.cpp:958-981); read from the multigrid solution */
        if (level < 0 || level >= P.max_levels_mg) return BCG_E_ARG;
        MgLevel& L = c->mg[level];
        int sp = f - BCG_F_AGARF_CARBON;   /* carbon, oxygen, acetate */
        v->ptr = L.sol[sp]; v->mg = 2; v->nx = (int)X - 1; v->nz = P.box_z_agar - 1; v->pitch = L.pitch;
        v->n = X * (size_t)P.box_z_agar;
        return BCG_OK;
    }
    if (f >= BCG_F_MG_SOL_CARBON && f <= BCG_F_MG_ERR_ACETATE) {
        if (level < 0 || level >= c->mg_levels) return BCG_E_ARG;
        MgLevel& L = c->mg[level];
        int kind = (f - BCG_F_MG_SOL_CARBON) / 3, sp = (f - BCG_F_MG_SOL_CARBON) % 3;
        v->ptr = kind == 0 ? L.sol[sp] : kind == 1 ? L.res[sp] : L.err[sp];
        v->mg = 1; v->nx = L.nx; v->nz = L.nz; v->pitch = L.pitch;
        v->n = (size_t)(L.nx + 1) * (L.nz + 1);
        return BCG_OK;
    }
    return BCG_E_ARG;
}

extern "C" int bcg_field_size(bcg_ctx* c, int f, int level, size_t* n)
{
    if (!c || !n) return BCG_E_ARG;
    FieldView v;
    int rc = field_view(c, f, level, &v);
    if (rc) return rc;
    *n = v.n;
    return BCG_OK;
}

/* MG arrays are stored k-major with a padded pitch on the device; the ABI
 * presents them x-major, z fastest, like Array3D.  The agar view skips the
 * wall row k = 0 and the x = nx column. */
extern "C" int bcg_get_field(bcg_ctx* c, int f, int level, double* out, size_t n)
{
    if (!c || !out) return BCG_E_ARG;
    FieldView v;
    int rc = field_view(c, f, level, &v);
    if (rc) return rc;
    if (n < v.n) return BCG_E_ARG;
    if (!v.mg) {
        BCG_CUDA_TRY(cudaMemcpyAsync(out, v.ptr, v.n * 8, cudaMemcpyDeviceToHost, c->stream));
        return ctx_check_status(c);
    }
    mg_res0_materialise(c);
    int nz1 = v.mg == 1 ? v.nz + 1 : (int)(v.n / (v.nx + 1));   /* rows delivered */
    int k0 = v.mg == 1 ? 0 : 1;
    size_t rows = (size_t)nz1 + k0;
    double* tmp = (double*)malloc(sizeof(double) * rows * v.pitch);
    if (!tmp) return BCG_E_ARG;
    cudaError_t e = cudaMemcpyAsync(tmp, v.ptr, sizeof(double) * rows * v.pitch, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { free(tmp); g_last_cuda = e; return BCG_E_CUDA; }
    for (int i = 0; i <= v.nx; i++)
        for (int k = 0; k < nz1; k++) out[(size_t)i * nz1 + k] = tmp[(size_t)(k + k0) * v.pitch + i];
    free(tmp);
    return ctx_check_status(c);
}

extern "C" int bcg_set_field(bcg_ctx* c, int f, int level, const double* in, size_t n)
{
    if (!c || !in) return BCG_E_ARG;
    FieldView v;
    int rc = field_view(c, f, level, &v);
    if (rc) return rc;
    if (n < v.n) return BCG_E_ARG;
    if (v.mg == 2) return BCG_E_UNSUPPORTED;  /* the agar view is derived */
    mg_res0_materialise(c);                    /* before its inputs change */
    if (v.mg == 1) { c->mg_clean = 0; nutrient_graphs_drop(c); }   /* Err/Res may no longer be zero */
    if (!v.mg) {
        BCG_CUDA_TRY(cudaMemcpy(v.ptr, in, v.n * 8, cudaMemcpyHostToDevice));
        return BCG_OK;
    }
    size_t rows = (size_t)v.nz + 1;
    double* tmp = (double*)malloc(sizeof(double) * rows * v.pitch);
    if (!tmp) return BCG_E_ARG;
    cudaError_t e = cudaMemcpy(tmp, v.ptr, sizeof(double) * rows * v.pitch, cudaMemcpyDeviceToHost);
    for (int i = 0; i <= v.nx; i++)
        for (int k = 0; k <= v.nz; k++) tmp[(size_t)k * v.pitch + i] = in[(size_t)i * (v.nz + 1) + k];
    if (e == cudaSuccess) e = cudaMemcpy(v.ptr, tmp, sizeof(double) * rows * v.pitch, cudaMemcpyHostToDevice);
    free(tmp);
    if (e != cudaSuccess) { g_last_cuda = e; return BCG_E_CUDA; }
    return BCG_OK;
}

extern "C" int bcg_get_bbox(bcg_ctx* c, int* minx, int* maxx, int* maxz)
{
    if (!c) return BCG_E_ARG;
    int h[3];
    BCG_CUDA_TRY(cudaMemcpyAsync(h, c->bbox, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    int rc = ctx_check_status(c);
    if (minx) *minx = h[0];
    if (maxx) *maxx = h[1];
    if (maxz) *maxz = h[2];
    return rc;
}
extern "C" int bcg_set_bbox(bcg_ctx* c, int minx, int maxx, int maxz)
{
    if (!c) return BCG_E_ARG;
    int h[3] = {minx, maxx, maxz};
    BCG_CUDA_TRY(cudaMemcpy(c->bbox, h, sizeof(h), cudaMemcpyHostToDevice));
    return BCG_OK;
}
