/*
 * output.cu -- device snapshots of an output step for the asynchronous
 * writer (writer.cpp).  The output blocks of SimSingleThread
 * (AgentBasedModel-BacColonyGrowth/Simulation.cpp:185-244, 316-372) read
 * the colony, its stress diagnostics and four field arrays at one point of
 * the step; here that point is the context's stream order.
 *
 * Everything one step writes is gathered on the context's stream into one
 * device staging buffer:
 *   - the colony as reference records (k_pack);
 *   - mean_stress's five stress components per cell, or F_surf_tension's
 *     force in the initial block;
 *   - the restart records (the moved, grown, undivided colony: the
 *     second record buffer while a move waits for its division loop);
 *   - the field planes: DensityShiftP and the 17 Environment members by
 *     device-to-device copies; the agar levels as z-major rows straight out
 *     of the multigrid solution (rows 1..Box_z_agar, copyFromMG); the four
 *     wall rows of every level.
 * One device-to-host copy on the writer's copy stream then moves the
 * staging buffer into pinned memory while the context's stream goes on
 * with the next steps.  The staging buffer is freed on the copy stream
 * behind that copy.
 */
#include "ctx.cuh"
#include "internal.h"

#include <string.h>

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

extern "C" int bcg_int_device(bcg_ctx* c) { return c ? c->device : -1; }

extern "C" int bcg_int_out_layout(bcg_ctx* c, int what, int initial, bcg_out_layout* L)
{
    if (!c || !L || (what & ~(BCG_OUT_CELLS | BCG_OUT_FIELDS))) return BCG_E_ARG;
    const bcg_params& P = c->P;
    if (P.box_y != 1) return BCG_E_UNSUPPORTED;
    memset(L, 0, sizeof(*L));
    L->what = what;
    L->initial = initial;
    L->box_x = P.box_x; L->box_z = P.box_z; L->box_z_agar = P.box_z_agar; L->levels = P.max_levels_mg;
    const size_t n = (size_t)c->n;
    size_t o = 0;
    if (what & BCG_OUT_CELLS) {
        L->n_cells = c->n;
        L->force_stride = initial ? 3 : 5;
        L->off_cells = o; o = align256(o + n * sizeof(bcg_cell));
        L->off_force = o; o = align256(o + n * (size_t)L->force_stride * sizeof(double));
    }
    if (what & BCG_OUT_FIELDS) {
        const size_t XZ = (size_t)P.box_x * P.box_z;
        L->n_restart = initial ? -1 : c->n;
        L->off_restart = o; if (!initial) o = align256(o + n * sizeof(bcg_cell));
        L->off_density = o; o = align256(o + XZ * sizeof(double));
        L->off_env = o; o = align256(o + 17 * XZ * sizeof(double));
        L->off_agar = o; o = align256(o + (size_t)L->levels * 3 * P.box_x * P.box_z_agar * sizeof(double));
        L->off_wall = o; o = align256(o + (size_t)L->levels * 4 * P.box_x * sizeof(double));
    }
    L->bytes = o;
    return BCG_OK;
}

/* the field planes, queued on the context's stream into staging `d` */
static int snapshot_fields(bcg_ctx* c, const bcg_out_layout* L, char* d)
{
    cudaStream_t s = c->stream;
    const size_t X = L->box_x, XZ = (size_t)L->box_x * L->box_z, Za = L->box_z_agar;
    BCG_CUDA_TRY(cudaMemcpyAsync(d + L->off_density, c->ds, XZ * 8, cudaMemcpyDeviceToDevice, s));
    /* Array3D<LocalEnv>::Output's member order (Array.h:931-1122) */
    const EnvBuf& e = c->env[0];
    const double* env[17] = {e.C, e.A, e.W, e.O, e.gr1, e.gr2, e.extra[0], e.extra[1], e.extra[2],
                             e.ph, e.hydrox, e.buffer, e.acetic, e.extra[3], e.extra[4], e.extra[5], e.extra[6]};
    for (int k = 0; k < 17; k++)
        BCG_CUDA_TRY(cudaMemcpyAsync(d + L->off_env + k * XZ * 8, env[k], XZ * 8, cudaMemcpyDeviceToDevice, s));
    /* FieldAgar[l](x, z) = Aga[l](x, z + 1) after every solve
     * (copyFromMG, Multigrid.cpp:958-981); sol[] holds carbon, oxygen,
     * acetate; the file order is carbon, acetate, (waste), oxygen */
    const int sp_order[3] = {0, 2, 1};
    for (int l = 0; l < L->levels; l++) {
        const MgLevel& M = c->mg[l];
        for (int j = 0; j < 3; j++) {
            char* dst = d + L->off_agar + ((size_t)(l * 3 + j) * Za * X) * 8;
            BCG_CUDA_TRY(cudaMemcpy2DAsync(dst, X * 8, M.sol[sp_order[j]] + M.pitch, (size_t)M.pitch * 8, X * 8, Za,
                                           cudaMemcpyDeviceToDevice, s));
        }
        const WallBuf& w = c->wal[0];
        const double* wall[4] = {w.C[l], w.A[l], w.W[l], w.O[l]};
        for (int j = 0; j < 4; j++)
            BCG_CUDA_TRY(cudaMemcpyAsync(d + L->off_wall + ((size_t)(l * 4 + j) * X) * 8, wall[j], X * 8,
                                         cudaMemcpyDeviceToDevice, s));
    }
    return BCG_OK;
}

/* queues the snapshot of one output step into the device staging buffer
 * `d` on the context's stream (cells, stress or surface force, restart
 * records, field planes) */
static int snapshot_queue(bcg_ctx* c, const bcg_out_layout* L, char* d, bool stress)
{
    cudaStream_t s = c->stream;
    if (stress) BCG_CUDA_TRY(cudaMemsetAsync(c->fcw_count, 0, sizeof(unsigned long long), s));
    if (L->what & BCG_OUT_CELLS) {
        launch_pack_cells(c, (bcg_cell*)(d + L->off_cells), s, 0);
        if (L->initial) launch_surface_force(c, (double*)(d + L->off_force), s);
        else launch_mean_stress(c, (double*)(d + L->off_force), c->fcw_count, s);
    }
    if (L->what & BCG_OUT_FIELDS) {
        /* SaveCells(new_cells): between MoveCell and the division loop the
         * moved records are the other buffer */
        if (L->n_restart > 0) launch_pack_cells(c, (bcg_cell*)(d + L->off_restart), s, c->move_pending);
        int rc = snapshot_fields(c, L, d);
        if (rc) return rc;
    }
    BCG_CUDA_TRY(cudaGetLastError());
    return BCG_OK;
}

/* hands the staging buffer to the copy stream: device-to-host copy into
 * `host`, then the buffer is released on that stream */
static int snapshot_hand_over(bcg_ctx* c, const bcg_out_layout* L, char* d, void* host, cudaStream_t cs)
{
    cudaEvent_t snap;
    BCG_CUDA_TRY(cudaEventCreateWithFlags(&snap, cudaEventDisableTiming));
    cudaError_t e = cudaEventRecord(snap, c->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, snap, 0);
    cudaEventDestroy(snap);
    if (e != cudaSuccess) { bcg_set_cuda_error(e); return BCG_E_CUDA; }
    if (L->bytes) BCG_CUDA_TRY(cudaMemcpyAsync(host, d, L->bytes, cudaMemcpyDeviceToHost, cs));
    return BCG_OK;
}

extern "C" int bcg_int_out_snapshot(bcg_ctx* c, const bcg_out_layout* L, void* host, void* copy_stream,
                                    void* done_event, int64_t* fcw_calls)
{
    if (!c || !L || !host || !copy_stream || !done_event) return BCG_E_ARG;
    cudaStream_t s = c->stream, cs = (cudaStream_t)copy_stream;
    const bool stress = (L->what & BCG_OUT_CELLS) && !L->initial;
    char* d = nullptr;
    if (L->bytes) BCG_CUDA_TRY(cudaMallocAsync((void**)&d, L->bytes, s));
    int rc = snapshot_queue(c, L, d, stress);
    if (rc == BCG_OK) rc = snapshot_hand_over(c, L, d, host, cs);
    /* the one release of the staging buffer: on the copy stream after its
     * copy, or on the context's stream (after what was queued there) when
     * the hand-over did not happen */
    if (d) {
        cudaError_t e = cudaFreeAsync(d, rc == BCG_OK ? cs : s);
        if (e != cudaSuccess && rc == BCG_OK) { bcg_set_cuda_error(e); rc = BCG_E_CUDA; }
    }
    if (rc) return rc;
    BCG_CUDA_TRY(cudaEventRecord((cudaEvent_t)done_event, cs));
    if (!stress) return BCG_OK;
    unsigned long long h = 0;
    BCG_CUDA_TRY(cudaMemcpyAsync(&h, c->fcw_count, sizeof(h), cudaMemcpyDeviceToHost, s));
    rc = ctx_check_status(c);
    if (fcw_calls) *fcw_calls = (int64_t)h;
    return rc;
}

/* mean_stress's F_cw count alone, for an output step that writes nothing
 * (the reference draws them on every output step, Simulation.cpp:320-326) */
extern "C" int bcg_int_stress_draws(bcg_ctx* c, int64_t* fcw_calls)
{
    if (!c || !fcw_calls) return BCG_E_ARG;
    BCG_CUDA_TRY(cudaMemsetAsync(c->fcw_count, 0, sizeof(unsigned long long), c->stream));
    if (c->n > 0) {
        double* ds = nullptr;
        BCG_CUDA_TRY(cudaMallocAsync((void**)&ds, sizeof(double) * 5 * (size_t)c->n, c->stream));
        launch_mean_stress(c, ds, c->fcw_count, c->stream);
        BCG_CUDA_TRY(cudaFreeAsync(ds, c->stream));
    }
    unsigned long long h = 0;
    BCG_CUDA_TRY(cudaMemcpyAsync(&h, c->fcw_count, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    int rc = ctx_check_status(c);
    *fcw_calls = (int64_t)h;
    return rc;
}
