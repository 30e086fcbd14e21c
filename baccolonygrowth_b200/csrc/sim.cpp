/*
 * sim.cpp -- the C++ host loop: a rewrite of SimSingleThread
 * (AgentBasedModel-BacColonyGrowth/Simulation.cpp:42-434) over the C ABI.
 *
 * The host keeps what the reference keeps on the host: the glibc rand()
 * stream, the time and the three loop flags, and the lineage record.  All
 * cell and field state stays on the device; per step the host reads back
 * two counters (dividing cells, F_cw draws) and uploads 9 draws per
 * division.
 */
#include <stdlib.h>
#include <string.h>
#include <vector>

#include "../../include/bcg.h"
#include "internal.h"

struct bcg_sim {
    bcg_params P;
    bcg_ctx* ctx;
    bcg_rng rng;
    double t, dt;
    double next_out, next_update, hd_next_update, hd_update_time;
    bool update_flag, hd_update_flag;
    bool out_flag;                 /* OutFlag, Simulation.cpp:56, 418 */
    int koutput;                   /* output step id, Simulation.cpp:251 */
    bcg_writer* writer;            /* writes the output steps when set */
    bool reference_cadence;
    int vcycles_per_step;
    bool first_step;
    long long divisions;
    long long rebuilds;            /* full neighbour rebuilds run */
    long long field_updates;       /* field updates (UpdateFlag blocks) run */
    std::vector<int> lineage;
    std::vector<float> draws;
    /* status of a step that failed part-way (the colony may be between
     * MoveCell and the division loop): every later run returns it */
    int failed;
};

static float frand(bcg_rng* g) { return (float)bcg_rng_next(g) / (float)2147483647; }

extern "C" int bcg_sim_create(const bcg_params* p, const bcg_cell* cells, int n, uint32_t seed,
                              int run_initial_fields, bcg_sim** out)
{
    if (!p || !out || (n > 0 && !cells)) return BCG_E_ARG;
    *out = nullptr;
    bcg_sim* s = new bcg_sim();
    s->P = *p;
    int rc = bcg_create(p, &s->ctx);
    if (rc) { delete s; return rc; }
    rc = bcg_upload_cells(s->ctx, cells, n);
    if (rc) { bcg_destroy(s->ctx); delete s; return rc; }
    /* srand(seed) (CellMD3D.cpp:23) then the rough wall (Simulation.cpp:161-168) */
    bcg_rng_seed(&s->rng, seed);
    std::vector<double> wall((size_t)p->box_x * p->box_y);
    for (int ii = 0; ii < p->box_x; ii++)
        for (int jj = 0; jj < p->box_y; jj++)
            wall[(size_t)ii * p->box_y + jj] = ((double)frand(&s->rng) - 0.5) * p->wall_rough;
    rc = bcg_set_field(s->ctx, BCG_F_WALL, 0, wall.data(), wall.size());
    if (rc == BCG_OK && run_initial_fields) {
        /* Simulation.cpp:186-217 */
        rc = bcg_initial_density(s->ctx);
        if (rc == BCG_OK) rc = bcg_nutrient_update(s->ctx, 0, -1);
    }
    if (rc) { bcg_destroy(s->ctx); delete s; return rc; }
    s->t = p->t0;
    s->dt = p->dt;
    s->next_out = p->output_time;
    s->next_update = p->update_time;
    s->hd_next_update = p->update_time / 10.0;
    s->hd_update_time = p->update_time / 10.0;
    s->update_flag = true;
    s->hd_update_flag = true;
    s->out_flag = false;           /* the initial block consumed the first OutFlag */
    s->koutput = 0;
    s->writer = nullptr;
    s->reference_cadence = true;
    s->vcycles_per_step = 0;
    s->first_step = true;
    s->divisions = 0;
    s->rebuilds = 0;
    s->field_updates = 0;
    s->failed = BCG_OK;
    *out = s;
    return BCG_OK;
}

extern "C" int bcg_sim_destroy(bcg_sim* s)
{
    if (!s) return BCG_OK;
    bcg_destroy(s->ctx);
    delete s;
    return BCG_OK;
}

extern "C" bcg_ctx* bcg_sim_ctx(bcg_sim* s) { return s ? s->ctx : nullptr; }

extern "C" int bcg_sim_set_writer(bcg_sim* s, bcg_writer* w, int write_initial)
{
    if (!s) return BCG_E_ARG;
    s->writer = w;
    if (w && write_initial) return bcg_output_initial(w, s->ctx, s->t);
    return BCG_OK;
}

extern "C" int bcg_sim_set_step_mode(bcg_sim* s, int field_cadence_reference, int vcycles_per_step)
{
    if (!s || vcycles_per_step < 0) return BCG_E_ARG;
    s->reference_cadence = field_cadence_reference != 0;
    s->vcycles_per_step = vcycles_per_step;
    return BCG_OK;
}

/* end of a step: lineage, time and the three flags (Simulation.cpp:418-426) */
static int sim_advance(bcg_sim* s, size_t base, int done, int rc)
{
    s->lineage.resize(base + 2 * (size_t)done);
    s->divisions += done;
    if (rc) return rc;
    s->t += s->dt;
    s->out_flag = (s->next_out <= 0);
    s->next_out = (s->out_flag ? s->P.output_time : s->next_out) - s->dt;
    s->update_flag = (s->next_update <= 0);
    s->next_update = (s->update_flag ? s->P.update_time : s->next_update) - s->dt;
    s->hd_update_flag = (s->hd_next_update <= 0);
    s->hd_next_update = (s->hd_update_flag ? s->hd_update_time : s->hd_next_update) - s->dt;
    return BCG_OK;
}

/* the host's share of a step between MoveCell and the division loop:
 * skip the F_cw draws, draw the division floats */
static void sim_draws(bcg_sim* s, int nd, int64_t calls)
{
    bcg_rng_skip(&s->rng, calls);
    s->draws.resize((size_t)9 * (nd > 0 ? nd : 1));
    for (int i = 0; i < 9 * nd; i++) s->draws[i] = frand(&s->rng);
}

/* One iteration of while (t <= t_max), Simulation.cpp:254-431.  In the
 * reference cadence an output step (OutFlag) runs mean_stress on every cell
 * before MoveCell, whose F_cw draws the host skips, and with a writer
 * attached writes the step's files (Simulation.cpp:316-327, 340-372) and
 * the lineage lines (Simulation.cpp:392). */
static int sim_step_body(bcg_sim* s, bool* aside)
{
    int rc;
    const bool out = s->reference_cadence && s->out_flag;
    int64_t stress_calls = 0;
    bcg_int_tl_mark(s->ctx, 0, BCG_TL_STEP);
    if (s->reference_cadence) {
        if (s->update_flag) {
            s->update_flag = false;
            if ((rc = bcg_update_density(s->ctx))) return rc;
            if ((rc = bcg_nutrient_update(s->ctx, 0, -1))) return rc;
            if ((rc = bcg_rebuild_neighbours(s->ctx))) return rc;
            s->field_updates++;
            s->rebuilds++;
        }
        if (s->hd_update_flag) {
            s->hd_update_flag = false;
            if ((rc = bcg_update_height(s->ctx))) return rc;
        }
    } else {
        /* benchmark cadence: neighbour lists follow the reference's
         * UpdateTime period; every step also runs the agar solve */
        if (s->update_flag || s->first_step) {
            s->update_flag = false;
            if ((rc = bcg_rebuild_neighbours(s->ctx))) return rc;
            s->rebuilds++;
        }
        /* the solve touches only the multigrid arrays and the agar and wall
         * fields; the step's mechanics and divisions touch none of them, so
         * the solve runs on the context's second stream beside them */
        if (s->vcycles_per_step > 0) {
            if ((rc = bcg_int_mg_solve_aside(s->ctx, s->vcycles_per_step))) return rc;
            *aside = true;
        }
    }
    s->first_step = false;
    if (out) {
        rc = s->writer ? bcg_output_cells(s->writer, s->ctx, s->koutput, s->t, &stress_calls)
                       : bcg_int_stress_draws(s->ctx, &stress_calls);
        if (rc) return rc;
    }
    int nd = 0;
    int64_t calls = 0;
    bcg_int_tl_mark(s->ctx, 0, BCG_TL_MECH_BEGIN);
    if ((rc = bcg_move_grow(s->ctx, s->dt, &nd, &calls))) return rc;
    bcg_int_tl_mark(s->ctx, 0, BCG_TL_MECH_END);
    if (out) {
        s->out_flag = false;
        if (s->writer && (rc = bcg_output_fields(s->writer, s->ctx, s->koutput, s->t, s->dt))) return rc;
        s->koutput++;
    }
    sim_draws(s, nd, stress_calls + calls);
    size_t base = s->lineage.size();
    s->lineage.resize(base + 2 * (size_t)(nd > 0 ? nd : 0));
    int done = 0;
    rc = bcg_divide(s->ctx, s->draws.data(), nd, s->t, &done, nd > 0 ? s->lineage.data() + base : nullptr);
    bcg_int_tl_mark(s->ctx, 0, BCG_TL_DIVIDE_END);
    if (s->writer && done > 0) {
        int lrc = bcg_writer_lineage(s->writer, s->lineage.data() + base, done);
        if (lrc && !rc) rc = lrc;
    }
    return sim_advance(s, base, done, rc);
}

/* One step; the context's stream waits for the step's agar solve before
 * anything queued after the step */
static int sim_step(bcg_sim* s)
{
    bool aside = false;
    int rc = sim_step_body(s, &aside);
    if (aside) {
        const int jr = bcg_int_join(s->ctx);
        if (!rc) rc = jr;
        bcg_int_tl_mark(s->ctx, 0, BCG_TL_STEP_END);
    }
    return rc;
}

extern "C" int bcg_sim_run(bcg_sim* s, int steps)
{
    if (!s || steps < 0) return BCG_E_ARG;
    if (s->failed) return s->failed;
    for (int i = 0; i < steps; i++) {
        int rc = sim_step(s);
        if (rc) { s->failed = rc; return rc; }
    }
    return BCG_OK;
}

extern "C" int bcg_sim_time(bcg_sim* s, double* t, int* n_cells, int64_t* divisions)
{
    if (!s) return BCG_E_ARG;
    if (t) *t = s->t;
    if (n_cells) bcg_num_cells(s->ctx, n_cells);
    if (divisions) *divisions = s->divisions;
    return BCG_OK;
}

extern "C" int bcg_sim_counters(bcg_sim* s, int64_t* neighbour_rebuilds, int64_t* field_updates)
{
    if (!s) return BCG_E_ARG;
    if (neighbour_rebuilds) *neighbour_rebuilds = s->rebuilds;
    if (field_updates) *field_updates = s->field_updates;
    return BCG_OK;
}

extern "C" int bcg_sim_lineage(bcg_sim* s, int* pairs, int capacity, int* n)
{
    if (!s) return BCG_E_ARG;
    int total = (int)(s->lineage.size() / 2);
    if (n) *n = total;
    int m = total < capacity ? total : capacity;
    if (m > 0 && pairs) memcpy(pairs, s->lineage.data(), sizeof(int) * 2 * (size_t)m);
    return BCG_OK;
}

/* ------------------------------------------------------------------------
 * Ensembles: independent colonies (bcg_sim members in the benchmark
 * cadence) stepped together.  Each phase of the step is queued for every
 * member, on the member's own stream, before any member is waited for:
 *   neighbour rebuild (when due) + agar solve + MoveCell/GrowCell,
 *   wait for the counters; host draws,
 *   division loop, wait.
 * Colonies of uneven size so overlap on the GPU instead of queueing behind
 * each other's host round trips.  Every member follows exactly the steps
 * bcg_sim_run would take for it alone.
 * ------------------------------------------------------------------------ */
struct bcg_ensemble {
    std::vector<bcg_sim*> m;
    std::vector<int> nd;
    std::vector<int64_t> calls;
    std::vector<size_t> base;
    std::vector<char> live;        /* members still stepping in this step */
};

extern "C" int bcg_ensemble_create(bcg_sim* const* members, int n, bcg_ensemble** out)
{
    if (!out || n < 1 || !members) return BCG_E_ARG;
    *out = nullptr;
    for (int i = 0; i < n; i++) {
        if (!members[i]) return BCG_E_ARG;
        if (members[i]->reference_cadence) return BCG_E_UNSUPPORTED;
    }
    bcg_ensemble* e = new bcg_ensemble();
    e->m.assign(members, members + n);
    e->nd.resize(n); e->calls.resize(n); e->base.resize(n);
    *out = e;
    return BCG_OK;
}

extern "C" int bcg_ensemble_destroy(bcg_ensemble* e)
{
    delete e;
    return BCG_OK;
}

/* A member whose step fails is marked failed (its later runs, alone or in
 * an ensemble, return the error); every other member still completes the
 * step, so none is left between MoveCell and its division loop. */
static int ens_step(bcg_ensemble* e)
{
    const int n = (int)e->m.size();
    int first_rc = BCG_OK;
    e->live.assign(n, 1);
    auto fail = [&](int i, int rc) {
        e->m[i]->failed = rc;
        e->live[i] = 0;
        if (!first_rc) first_rc = rc;
    };
    int rc;
    /* each member's agar solve runs on its second stream beside its
     * mechanics (as in bcg_sim_run), joined once the step is done */
    std::vector<char> aside(n, 0);
    for (int i = 0; i < n; i++) {
        bcg_sim* s = e->m[i];
        if (s->update_flag || s->first_step) {
            s->update_flag = false;
            if ((rc = bcg_rebuild_neighbours(s->ctx))) { fail(i, rc); continue; }
            s->rebuilds++;
        }
        if (s->vcycles_per_step > 0) {
            if ((rc = bcg_int_mg_solve_aside(s->ctx, s->vcycles_per_step))) { fail(i, rc); continue; }
            aside[i] = 1;
        }
        s->first_step = false;
        if ((rc = bcg_int_move_grow_launch(s->ctx, s->dt))) fail(i, rc);
    }
    for (int i = 0; i < n; i++) {
        if (!e->live[i]) continue;
        bcg_sim* s = e->m[i];
        if ((rc = bcg_int_move_grow_finish(s->ctx, &e->nd[i], &e->calls[i]))) { fail(i, rc); continue; }
        sim_draws(s, e->nd[i], e->calls[i]);
        e->base[i] = s->lineage.size();
        s->lineage.resize(e->base[i] + 2 * (size_t)(e->nd[i] > 0 ? e->nd[i] : 0));
        if ((rc = bcg_int_divide_launch(s->ctx, s->draws.data(), e->nd[i], s->t))) {
            s->lineage.resize(e->base[i]);
            fail(i, rc);
        }
    }
    for (int i = 0; i < n; i++) {
        if (!e->live[i]) continue;
        bcg_sim* s = e->m[i];
        int done = 0;
        rc = bcg_int_divide_finish(s->ctx, &done, e->nd[i] > 0 ? s->lineage.data() + e->base[i] : nullptr);
        rc = sim_advance(s, e->base[i], done, rc);
        if (rc) fail(i, rc);
    }
    for (int i = 0; i < n; i++) {
        if (!aside[i]) continue;
        if ((rc = bcg_int_join(e->m[i]->ctx))) fail(i, rc);
    }
    return first_rc;
}

extern "C" int bcg_ensemble_run(bcg_ensemble* e, int steps)
{
    if (!e || steps < 0) return BCG_E_ARG;
    for (bcg_sim* s : e->m)
        if (s->failed) return s->failed;
    for (int k = 0; k < steps; k++) {
        int rc = ens_step(e);
        if (rc) return rc;
    }
    return BCG_OK;
}

