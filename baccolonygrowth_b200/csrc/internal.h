/* internal.h -- split-phase entries of the library used by the host-side
 * ensemble runner (sim.cpp).  Not part of the public C ABI. */
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
#ifdef __cplusplus
}
#endif
