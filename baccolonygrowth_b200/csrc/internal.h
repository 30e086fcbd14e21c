/* internal.h -- split-phase entries of the library used by the host-side
 * ensemble runner (sim.cpp) and the output writer (writer.cpp).  Not part
 * of the public C ABI. */
#pragma once
#include <stdint.h>
#include "../../include/bcg.h"
#ifdef __cplusplus
extern "C" {
#endif
/* queue MoveCell+GrowCell and the reads of its two counters / wait for them */
int bcg_int_move_grow_launch(bcg_ctx* ctx, double dt);
int bcg_int_move_grow_finish(bcg_ctx* ctx, int* n_div, int64_t* fcw_calls);
/* queue the division loop / wait for it and take the lineage */
int bcg_int_divide_launch(bcg_ctx* ctx, const float* draws, int n_draw_sets, double t);
int bcg_int_divide_finish(bcg_ctx* ctx, int* n_done, int* lineage);
/* queue Multigrid::solve with `vcycles` V-cycles (errors surface at the
 * next synchronising call) */
int bcg_int_mg_solve_launch(bcg_ctx* ctx, int vcycles);
/* queue Multigrid::solve on the context's second stream, beside what is
 * queued after it until bcg_int_join; nothing queued in between may touch
 * the multigrid arrays, the agar and wall fields or the density */
int bcg_int_mg_solve_aside(bcg_ctx* ctx, int vcycles);
/* order the context's stream after its second stream's work */
int bcg_int_join(bcg_ctx* ctx);
/* a step-timeline mark (bcg_timeline_tag) on the context's stream (aux 0)
 * or its second stream; nothing when no timeline is running */
void bcg_int_tl_mark(bcg_ctx* ctx, int aux, int tag);

/* Output-step snapshots (output.cu), used by the writer (writer.cpp).
 * One snapshot is a byte image laid out by bcg_out_layout: cell records,
 * per-cell force columns, restart records, then the field planes. */
typedef struct bcg_out_layout {
    int what;                 /* BCG_OUT_* mask */
    int initial;              /* initial block: F_surf_tension forces, empty Restart */
    int n_cells, force_stride, n_restart;
    int box_x, box_z, box_z_agar, levels;
    size_t off_cells, off_force, off_restart;
    size_t off_density;       /* box_x*box_z, x-major */
    size_t off_env;           /* 17 planes of box_x*box_z, x-major, file order */
    size_t off_agar;          /* 3 per level (carbon, acetate, oxygen) of
                                 box_z_agar rows of box_x, z-major */
    size_t off_wall;          /* 4 per level (carbon, acetate, waste, oxygen), box_x */
    size_t bytes;
} bcg_out_layout;
int bcg_int_out_layout(bcg_ctx* ctx, int what, int initial, bcg_out_layout* L);
/* Queue the snapshot on the context's stream into a device staging buffer,
 * then its copy into `host` (pinned, L->bytes) on `copy_stream`, and record
 * `done_event` there.  For BCG_OUT_CELLS outside the initial block, waits
 * for and returns mean_stress's F_cw count. */
int bcg_int_out_snapshot(bcg_ctx* ctx, const bcg_out_layout* L, void* host, void* copy_stream,
                         void* done_event, int64_t* fcw_calls);
int bcg_int_device(bcg_ctx* ctx);
/* mean_stress's F_cw draw count alone (an output step that writes nothing) */
int bcg_int_stress_draws(bcg_ctx* ctx, int64_t* fcw_calls);
#ifdef __cplusplus
}
#endif
