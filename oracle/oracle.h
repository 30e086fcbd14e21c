/*
 * oracle.h -- TEST INFRASTRUCTURE ONLY.  CPU restatement of the reference
 * hot path (plain C, scalar, sequential, the 1-thread reference order), used
 * as the checker of the CUDA library in tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg.  Nothing in the product links or calls it.
 */
#ifndef BCG_ORACLE_H_
#define BCG_ORACLE_H_
#include "../include/bcg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_state orc_state;

orc_state* orc_create(const bcg_params* p, unsigned seed, int make_wall);
void orc_destroy(orc_state* s);
int  orc_load_cells(orc_state* s, const bcg_cell* cells, int n);
int  orc_get_cells(orc_state* s, bcg_cell* out, int cap);
int  orc_num_cells(orc_state* s);
long long orc_rand_calls(orc_state* s);
int  orc_error(orc_state* s);

void orc_rebuild_neighbours(orc_state* s);
int  orc_get_neighbours(orc_state* s, int* counts, int* lists, int stride);
int  orc_set_neighbours(orc_state* s, const int* counts, const int* lists, int stride);
int  orc_move_grow(orc_state* s, double dt, int* div_ids, long long* rand_calls);
int  orc_divide(orc_state* s, double t, int* lineage);

/* fields (ids of bcg_field_id) */
long orc_field(orc_state* s, int field, int level, double* buf, long n, int write);
void orc_bbox(orc_state* s, int* minx, int* maxx, int* maxz);
void orc_set_bbox(orc_state* s, int minx, int maxx, int maxz);
void orc_initial_fields(orc_state* s, int run_nutrients);
void orc_update_density(orc_state* s);
void orc_update_height(orc_state* s);
void orc_nutrient_update(orc_state* s, int n);
void orc_mg_solve(orc_state* s, int vcycles, double dt);
void orc_colony_sweeps(orc_state* s, int sweeps, int count0);
int  orc_loop_step(orc_state* s, int* lineage);
long long orc_mean_stress(orc_state* s, double* stress, double* fnet);
double orc_time(orc_state* s);

/* the legacy explicit agar solver (UpdateEnvArray_OxygenAcetate,
 * nutrientDepletionAgar_OxygenAcetate) */
int orc_legacy_env_update(orc_state* s, int min_iter, int max_iter, double conv_crit);
int orc_legacy_depletion(orc_state* s);

/* inputs of the benchmark's reference arm (no CUDA library loaded there) */
int orc_params_default(bcg_params* p);
int orc_params_finalize(bcg_params* p);
int orc_synth_colony(uint64_t seed, int n_target, double width, double height,
                     double radius, double len_lo, double len_hi, double l_divide,
                     double div_phase_spread, bcg_cell* out, int capacity, int* n);

#ifdef __cplusplus
}
#endif
#endif
