/*
 * bcg.h -- C ABI of the B200 (sm_100a) hot path of the BacColonyGrowth
 * agent-based colony simulator.
 *
 * The library replaces the calls that the reference time loop
 * (AgentBasedModel-BacColonyGrowth/Simulation.cpp:42-434, SimSingleThread)
 * makes into Neighbours / Forces / Integrate / grow / Cells / Compute /
 * Nutrients / Multigrid.  All colony and field state lives on one GPU in
 * structure-of-arrays form inside a bcg_ctx; the host keeps the glibc rand()
 * stream and the loop flags, exactly as the reference does; the output
 * files are written from device snapshots by a host thread (bcg_writer).
 * Every entry point returns a bcg_status (0 = OK); no entry point aborts
 * the process, and no kernel traps.
 *
 * Citations are "file:line" inside AgentBasedModel-BacColonyGrowth/.
 */
#ifndef BCG_H_
#define BCG_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* status codes (replace MyAssert, tools.h:13-27, and the silent break   */
/* on maxCells, Simulation.cpp:382-386)                                  */
/* ------------------------------------------------------------------ */
typedef enum bcg_status {
    BCG_OK = 0,
    BCG_E_ARG = 1,              /* bad argument, size or null pointer            */
    BCG_E_CUDA = 2,             /* CUDA runtime / launch error                   */
    BCG_E_BOX_OVERFLOW = 3,     /* "Tried to add too many cells", UniformGrid.h:35 */
    BCG_E_NEIGH_OVERFLOW = 4,   /* neighbour list over capacity, UniformGrid.h:162 */
    BCG_E_OUT_OF_GRID = 5,      /* "Cells have expanded farther than boxes allows", UniformGrid.h:96 */
    BCG_E_NAN = 6,              /* non-finite position / velocity detected        */
    BCG_E_MAXCELLS = 7,         /* division stopped at MaxCells, Simulation.cpp:382 */
    BCG_E_TIMEOUT = 8,          /* a bounded device wait gave up                  */
    BCG_E_UNSUPPORTED = 9,      /* parameter combination the reference leaves undefined */
    BCG_E_NEED_MORE_BOXES = 10, /* colony too close to the grid edge, Nutrients.cpp:360 */
    BCG_E_NO_DEVICE = 11,       /* no CUDA device / kernels not loadable          */
    BCG_E_IO = 12               /* an output file or directory could not be written,
                                   "Can't open output file.", InputOutput.cpp:113-270 */
} bcg_status;

/* ------------------------------------------------------------------ */
/* cell record: byte-identical to `struct Cell` (Cell.h:15-28, with      */
/* Segment from tools.h:71-87), 208 bytes, so the reference's cell arrays */
/* and its binary restart files (InputOutput.cpp:394-448) are passed       */
/* through unchanged.                                                      */
/* ------------------------------------------------------------------ */
typedef struct bcg_vec3 { double x, y, z; } bcg_vec3;

typedef struct bcg_cell {
    bcg_vec3 p;             /* Segment.p */
    bcg_vec3 q;             /* Segment.q */
    double   time_p;        /* Segment.time_p */
    double   time_q;        /* Segment.time_q */
    int32_t  age_p;         /* Segment.age_p */
    int32_t  age_q;         /* Segment.age_q */
    double   length;        /* Cell.Length */
    double   ldiv;          /* Cell.Ldiv */
    double   radius;        /* Cell.Radius */
    double   growth_rate;   /* Cell.GrowthRate */
    bcg_vec3 velocity;      /* Cell.Velocity */
    bcg_vec3 angular_velocity; /* Cell.AngularVelocity */
    bcg_vec3 dyn_fric;      /* Cell.DynFric */
    bcg_vec3 sta_fric;      /* Cell.StaFric */
    int32_t  type;          /* Cell.Type */
    int32_t  ancestor;      /* Cell.Ancestor */
} bcg_cell;

/* ------------------------------------------------------------------ */
/* parameters: one POD mirror of the reference's mutable globals        */
/* (Constants.h, defaults Constants.cpp:1-112, input keys                */
/* InputOutput.cpp:450-677) plus the schedule constants the reference     */
/* hard-codes (Multigrid.cpp:995-1017).                                   */
/* ------------------------------------------------------------------ */
typedef struct bcg_params {
    /* grid (input keys Box_x, Box_y, Box_z, Box_z_agar, maxLevelsMG,
     * FilterLen, refinementGridHeight, MaxCells) */
    int32_t box_x, box_y, box_z, box_z_agar;
    int32_t max_levels_mg;          /* composite agar levels (agarLevels) */
    int32_t filter_len;
    int32_t refinement_grid_height;
    int32_t max_cells;
    /* derived by bcg_params_finalize (CellMD3D.cpp:52-54, 141) */
    int32_t max_cells_per_box;
    int32_t max_neighbours;         /* capacity of one reduced neighbour list (device) */
    double  box_length;

    /* cell mechanics */
    double cell_radius, l_divide, k_cc, k_wc, var_l, var_angle, var_pos;
    double viscosity, wall_rough, gamma_t, cell_mu, wall_mu;
    double density_threshold, tension, delta_h, rc;

    /* time */
    double dt, t0, t_max, output_time, update_time;

    /* nutrients (Nutrients.cpp, Multigrid.cpp) */
    double kc_aer, kc_ana, kw, ko, ka, ki;
    double carbon_to_waste, c_rate, w_rate, maintenance_rate;
    double q_car_aer, q_car_ana, q_ace_aer, q_o2_car, q_o2_ace, p_ace_aer, p_ace_ana;
    double diff_colony, diff_agar;
    double diff_colony_carbon, diff_agar_carbon;
    double diff_colony_o2, diff_agar_o2;
    double diff_colony_ace, diff_agar_ace;
    double max_carbon, max_o2, max_o2_agar;
    double max_growth_rate1, max_growth_rate2;
    double max_gr_car_aer, max_gr_car_ana, max_gr_ace_aer;
    double cdt;
    double q_car_aer_nt, q_car_ana_nt, q_ace_aer_nt, q_o2_car_nt, q_o2_ace_nt, p_ace_ana_nt;
    double kw_ph, ka_ph, kb_ph, cb_ph, c1_ph;     /* Kw, Ka, Kb, Cb, c1 */
    int32_t cross_feeding;          /* only 0 is defined for the oxygen/acetate model */
    int32_t interface_condition;    /* only 1 is implemented by the reference */
    int32_t nutrient_gsi;           /* 0 = Jacobi with buffer swap */

    /* schedule (reference constants as defaults) */
    int32_t mg_levels;              /* 8, Simulation.cpp:157 */
    int32_t mg_vcycles;             /* 3, Multigrid.cpp:869 */
    int32_t mg_mu1;                 /* 3, Multigrid.cpp:1002 */
    int32_t mg_mu2;                 /* 100, Multigrid.cpp:1002 */
    int32_t sweeps_per_solve;       /* 200, Multigrid.cpp:1017 */
    int32_t solves_per_update;      /* <=0: int(3600*UpdateTime*740/mg_dt), Multigrid.cpp:996 */
    double  mg_dt;                  /* 100, Multigrid.cpp:995 */
} bcg_params;

/* Fill *p with the reference defaults (Constants.cpp:1-112). */
int bcg_params_default(bcg_params* p);
/* Derive box_length, max_cells_per_box (CellMD3D.cpp:52-54) and the device
 * neighbour capacity; validate the combination.  Must be called after any
 * change and before bcg_create. */
int bcg_params_finalize(bcg_params* p);

/* ------------------------------------------------------------------ */
/* context                                                              */
/* ------------------------------------------------------------------ */
typedef struct bcg_ctx bcg_ctx;

/* Allocate all device state for p on the current CUDA device.  Replaces
 * the allocations of CellMD3D.cpp:46-142 and the Multigrid constructor
 * (Multigrid.cpp:5-33); fields start at the LocalEnv/LocalAga defaults
 * (Nutrients.h:13-38, 68-74). */
int bcg_create(const bcg_params* p, bcg_ctx** out);
int bcg_destroy(bcg_ctx* ctx);
/* Last device error word (0 if none) and a static message for a status. */
const char* bcg_status_string(int status);
/* The CUDA stream all work of this context is queued on (cudaStream_t).
 * Inside a benchmark-cadence step of bcg_sim_run the agar solve runs on a
 * second stream of the context; the step ends with this stream waiting for
 * it, so work queued here after any call sees every result of that call. */
void* bcg_stream(bcg_ctx* ctx);
/* Block until all queued work of ctx is done; returns the first pending error. */
int bcg_synchronize(bcg_ctx* ctx);

/* ------------------------------------------------------------------ */
/* cells                                                                */
/* ------------------------------------------------------------------ */
/* Replace the colony with n cells (AoS records, host memory); replaces
 * LoadCells' copy + Grid.Add (InputOutput.cpp:394-431).  Records pass
 * through the context's staging buffer (created with it, up to 131,072
 * records) a chunk at a time; nothing is allocated per call.  Pinned host
 * memory gives the full copy rate. */
int bcg_upload_cells(bcg_ctx* ctx, const bcg_cell* cells, int n);
/* Copy the first min(n, capacity) cells back as AoS records through the
 * same staging buffer; *n receives the cell count. */
int bcg_download_cells(bcg_ctx* ctx, bcg_cell* cells, int capacity, int* n);
int bcg_num_cells(bcg_ctx* ctx, int* n);

/* ------------------------------------------------------------------ */
/* neighbours (Neighbours.cpp:24-93, UniformGrid.h:87-170)              */
/* ------------------------------------------------------------------ */
/* Full rebuild: bin every cell by UniformGrid::GetAddress (counting sort),
 * gather the 3x3x3 box stencil and apply reduceNeighbours.  Replaces
 * getNeighbours(cells, N, Grid, NeighbourList, maxNeighbours),
 * Neighbours.cpp:24-37, as called at Simulation.cpp:292. */
int bcg_rebuild_neighbours(bcg_ctx* ctx);
/* Copy the reduced neighbour lists to the host: counts[N] and
 * lists[N*stride] (row i holds counts[i] ids, in device order). */
int bcg_get_neighbours(bcg_ctx* ctx, int* counts, int* lists, int stride);
/* Set the lists from the host (same layout); used to restore a state. */
int bcg_set_neighbours(bcg_ctx* ctx, const int* counts, const int* lists, int stride);

/* ------------------------------------------------------------------ */
/* mechanics step                                                       */
/* ------------------------------------------------------------------ */
/* One pass of MoveCell + GrowCell over every cell (Simulation.cpp:330-336,
 * Cells.cpp:14-57, Integrate.cpp:11-127, Forces.cpp:13-381, grow.cpp:17-102):
 * two-stage inertial integration with forces from the current (stale)
 * neighbour lists, then growth from Environment.GrowthRate1.
 * Outputs: *n_div = cells with Length >= Ldiv (their ids are kept on the
 * device in ascending order, the 1-thread reference order), *fcw_calls =
 * number of F_cw evaluations, i.e. the rand() calls Forces.cpp:102 made. */
int bcg_move_grow(bcg_ctx* ctx, double dt, int* n_div, int64_t* fcw_calls);
/* Ids of the cells flagged by the last bcg_move_grow, ascending. */
int bcg_get_dividing(bcg_ctx* ctx, int* ids, int capacity);
/* The division loop (Simulation.cpp:380-404) followed by the buffer swap
 * (:408-413).  draws holds 9 floats per division, in call order, each equal
 * to (float)rand()/RAND_MAX as drawn by divide() (grow.cpp:109-152).
 * n_draw_sets must equal the n_div of the preceding bcg_move_grow.  Each
 * division applies divide() and the partial neighbour rebuild for
 * {mother, mother's neighbours, daughter} in ascending parent order.
 * lineage (optional, 2 ints per division) receives "parent daughter" pairs
 * as written at Simulation.cpp:392; *n_done receives the divisions done
 * (fewer than requested when MaxCells is reached). */
int bcg_divide(bcg_ctx* ctx, const float* draws, int n_draw_sets, double t,
               int* n_done, int* lineage);

/* ------------------------------------------------------------------ */
/* fields                                                               */
/* ------------------------------------------------------------------ */
typedef enum bcg_field_id {
    BCG_F_HEIGHT = 0,        /* Height (box_x*rGH)                         */
    BCG_F_NORMAL_X = 1,      /* Normal.x (box_x*rGH)                       */
    BCG_F_NORMAL_Z = 2,      /* Normal.z (box_x*rGH)                       */
    BCG_F_WALL = 3,          /* rough wall height (box_x), Simulation.cpp:161-168 */
    BCG_F_DENSITY_SHIFT = 4, /* DensityShiftP (box_x*box_z)                */
    BCG_F_WALL_DENSITY_SHIFT = 5, /* WallDensityShiftP (box_x)             */
    BCG_F_INSIDE = 6,        /* insideColonyDen (box_x*box_z)              */
    BCG_F_ENV_CARBON = 7,    /* Environment (current buffer), box_x*box_z  */
    BCG_F_ENV_WASTE = 8,
    BCG_F_ENV_OXYGEN = 9,
    BCG_F_ENV_ACETATE = 10,
    BCG_F_ENV_GROWTH1 = 11,
    BCG_F_ENV_GROWTH2 = 12,
    BCG_F_ENV_PH = 13,
    BCG_F_OLDENV_CARBON = 14, /* oldEnvironment buffer                     */
    BCG_F_OLDENV_WASTE = 15,
    BCG_F_OLDENV_OXYGEN = 16,
    BCG_F_OLDENV_ACETATE = 17,
    BCG_F_WALLF_CARBON = 18, /* FieldWall[level] (box_x), level in `level` */
    BCG_F_WALLF_WASTE = 19,
    BCG_F_WALLF_OXYGEN = 20,
    BCG_F_WALLF_ACETATE = 21,
    BCG_F_OLDWALLF_CARBON = 22, /* oldFieldWall[level]                     */
    BCG_F_OLDWALLF_WASTE = 23,
    BCG_F_OLDWALLF_OXYGEN = 24,
    BCG_F_OLDWALLF_ACETATE = 25,
    BCG_F_AGARF_CARBON = 26, /* FieldAgar[level] (box_x*box_z_agar)        */
    BCG_F_AGARF_OXYGEN = 27,
    BCG_F_AGARF_ACETATE = 28,
    BCG_F_MG_SOL_CARBON = 29, /* Multigrid::Aga[level] ((nx+1)*(nz+1))     */
    BCG_F_MG_SOL_OXYGEN = 30,
    BCG_F_MG_SOL_ACETATE = 31,
    BCG_F_MG_RES_CARBON = 32, /* Multigrid::AgaRes[level]                  */
    BCG_F_MG_RES_OXYGEN = 33,
    BCG_F_MG_RES_ACETATE = 34,
    BCG_F_MG_ERR_CARBON = 35, /* Multigrid::AgaErr[level]                  */
    BCG_F_MG_ERR_OXYGEN = 36,
    BCG_F_MG_ERR_ACETATE = 37,
    BCG_F_DENSITY = 38,       /* Density (BoxAverage of RoughDensity)      */
    BCG_F_ROUGH_DENSITY = 39, /* RoughDensity (GetDensity)                 */
    BCG_F_ENV_HYDROX = 40,    /* Environment.Hydrox, Acetic, Buffer         */
    BCG_F_ENV_ACETIC = 41,    /*   (acetateBufferSolve, Nutrients.cpp:806-855) */
    BCG_F_ENV_BUFFER = 42,
    BCG_F_ENV_GR_CAR_AER = 43, /* Environment.GrCarAer, GrCarAna, GrAceAer */
    BCG_F_ENV_GR_CAR_ANA = 44, /*   (Nutrients.cpp:342-344)                */
    BCG_F_ENV_GR_ACE_AER = 45,
    BCG_F_ENV_Q_CAR_MNT = 46,  /* Environment.qCarmnt, qAcemnt, pAcemnt,   */
    BCG_F_ENV_Q_ACE_MNT = 47,  /*   qOxymnt (Nutrients.cpp:328-331)        */
    BCG_F_ENV_P_ACE_MNT = 48,
    BCG_F_ENV_Q_OXY_MNT = 49,
    BCG_F_COUNT = 50
} bcg_field_id;

/* Number of doubles of a field at a level (x-major, z fastest, matching
 * Array2D/Array3D indexing x*(Y*Z)+y*Z+z with Y=1). */
int bcg_field_size(bcg_ctx* ctx, int field, int level, size_t* n);
int bcg_get_field(bcg_ctx* ctx, int field, int level, double* out, size_t n);
int bcg_set_field(bcg_ctx* ctx, int field, int level, const double* in, size_t n);
/* Bounding box used by the field chain: minx, maxx, maxz after the +-5
 * widening of Compute.cpp:250-252 (written by the deposition calls). */
int bcg_get_bbox(bcg_ctx* ctx, int* minx, int* maxx, int* maxz);

/* GetDensity + ShiftDensity + 6x BoxAverage + Height_Average + Smooth +
 * GetSurfaceNormal (Simulation.cpp:266-280; Compute.cpp:120-253, 344-605,
 * 669-738, 466-491). */
int bcg_update_density(bcg_ctx* ctx);
/* GetHeight + Height_Average + Smooth + GetSurfaceNormal (Simulation.cpp:
 * 302-306; Compute.cpp:256-340). */
int bcg_update_height(bcg_ctx* ctx);
/* The initial-condition variant of the deposition chain at
 * Simulation.cpp:186-210 (no height smoothing). */
int bcg_initial_density(bcg_ctx* ctx);

/* UpdateEnvArrayMG_OxygenAcetate (Multigrid.cpp:984-1125): n solves, each
 * one Multigrid::solve followed by `sweeps` colony/interface Jacobi sweeps.
 * n <= 0 selects params.solves_per_update; sweeps < 0 selects
 * params.sweeps_per_solve. */
int bcg_nutrient_update(bcg_ctx* ctx, int n, int sweeps);

/* The legacy explicit agar solver, which the reference keeps but no longer
 * calls (its call sites, Simulation.cpp:215-216 and 283-284, are commented
 * out); a host that restores them calls these two in place of
 * bcg_nutrient_update.
 *
 * bcg_legacy_env_update replaces UpdateEnvArray_OxygenAcetate
 * (Nutrients.cpp:45-197): pseudo-time Jacobi iterations over the colony
 * (UpdateEnvironment_OxygenAcetate), the wall rows and every composite agar
 * level (UpdateAgarMultigrid_OxygenAcetate), alternating direction, until
 * after iteration `count` with count > min_iter no point of carbon, oxygen
 * or acetate moved by more than conv_crit * max(0.1, |value|), or max_iter
 * iterations (the reference's ConvCrit, minIter, maxIter: 1e-4, 500, 20000).
 * *iterations receives the count, as the reference returns it.
 *
 * bcg_legacy_agar_depletion replaces nutrientDepletionAgar_OxygenAcetate
 * (Nutrients.cpp:857-1074): the coarsest level takes each point from the
 * finest level that holds it, runs int(3600 UpdateTime 740 / dt) + 1
 * explicit steps of carbon and acetate diffusion (dt = min(D) h^2 / 10),
 * and every finer level is interpolated back from it; *steps receives the
 * steps run.
 *
 * Both keep their own FieldAgar / oldFieldAgar of the four species; the
 * agar solution rows stand for FieldAgar elsewhere, so each call starts
 * from them and writes them back.  On levels > 0 the reference leaves the
 * agar points with BoxX/4 <= x < 3 BoxX/4, z < BoxZAgar/2 undefined
 * (uninitialised second differences) and no other point reads them; they
 * are not updated here. */
int bcg_legacy_env_update(bcg_ctx* ctx, int min_iter, int max_iter, double conv_crit, int* iterations);
int bcg_legacy_agar_depletion(bcg_ctx* ctx, int* steps);
/* One Multigrid::solve (Multigrid.cpp:864-889) with `vcycles` V-cycles
 * (<=0: params.mg_vcycles): copyToMG, setup, V-cycles, reset, copyFromMG.
 * Queued on the context's stream.  The second call from the same starting
 * state captures the launches as a CUDA graph and later calls replay it;
 * a context whose capture fails keeps issuing plain launches. */
int bcg_mg_solve(bcg_ctx* ctx, int vcycles);
/* `sweeps` colony/interface sweeps (the inner loop of Multigrid.cpp:
 * 1017-1120) starting at sweep parity `count0`. */
int bcg_colony_sweeps(bcg_ctx* ctx, int sweeps, int count0);

/* ------------------------------------------------------------------ */
/* mixed precision multigrid (FP32 smoothing/restriction/prolongation in */
/* an FP64 iterative-refinement loop); no reference counterpart.         */
/* ------------------------------------------------------------------ */
/* Solve the backward-Euler agar step (the system Multigrid::solve
 * iterates on) until the FP64 defect max-norm at the relaxed points of the
 * composite levels falls below rel_tol * (its value at the start).
 * precision 64: FP64 V-cycles.  precision 32: V-cycles on FP32 copies of
 * the correction and right-hand side (smoothing, restriction and
 * prolongation in FP32; solution and defect in FP64) while the defect
 * still halves per cycle, then FP64 V-cycles from that correction.
 * *iters receives the V-cycles run and *rel_res the final relative defect
 * (where the V-cycle itself stalls, as on grids whose coarsest levels have
 * 0-1 interior rows, the solve stops at max_iters above rel_tol). */
int bcg_mg_solve_tol(bcg_ctx* ctx, double rel_tol, int precision, int max_iters,
                     int* iters, double* rel_res);

/* ------------------------------------------------------------------ */
/* kernel-shape autotuning (no reference counterpart)                    */
/* ------------------------------------------------------------------ */
/* Precision of the per-pair contact geometry in MoveCell (no reference
 * counterpart).  64 (default): the reference's FP64 min_distance.  32: the
 * closest points and their distance in FP32 on offsets local to cell i
 * (min_distance's steps unchanged), the contact forces, positions and
 * force sums in FP64.  Neighbour lists are built in FP64 either way. */
int bcg_set_pair_precision(bcg_ctx* ctx, int bits);

/* Times the variants of one kernel on the context's current state and
 * keeps the fastest for this context (*choice receives it):
 *   BCG_TUNE_FORCE_GROUP  lanes per cell in MoveCell+GrowCell (1..16);
 *                         needs binned cells and neighbour lists; leaves
 *                         the colony unchanged;
 *   BCG_TUNE_SMOOTHER     resident-warp target of the fused agar smoother
 *                         (how many row segments a level is cut into);
 *                         changes only the multigrid's correction scratch.
 * Every kernel choice belongs to its context: no call changes another
 * context's kernels.  Synchronises the stream; not for use inside a
 * stream capture. */
typedef enum bcg_tune_id { BCG_TUNE_FORCE_GROUP = 1, BCG_TUNE_SMOOTHER = 2 } bcg_tune_id;
int bcg_autotune(bcg_ctx* ctx, int what, int* choice);

/* Fixed kernel shapes for one context, for profiling and for tests of the
 * variants (each drops the context's captured graphs):
 *   bcg_set_force_group    lanes per cell in MoveCell+GrowCell: 1, 2, 4
 *                          (default), 8 or 16; the results do not depend
 *                          on it;
 *   bcg_set_relax_mode     agar smoother form: 0 = one thread per column
 *                          and half-sweep, 1 = half-sweeps with row
 *                          segments, 2 = fused sweeps with rows staged per
 *                          lane, 3 = fused sweeps with rows staged by the
 *                          tensor memory accelerator (default); the forms
 *                          agree to rounding;
 *   bcg_set_smoother_warps resident-warp target of the fused smoother
 *                          (0 = default or tuned);
 *   bcg_smoother_launch_ms device time of one finest-level launch of the
 *                          fused smoother measured by the last
 *                          BCG_TUNE_SMOOTHER (0 before). */
int bcg_set_force_group(bcg_ctx* ctx, int lanes);
int bcg_set_relax_mode(bcg_ctx* ctx, int mode);
int bcg_set_smoother_warps(bcg_ctx* ctx, int warps);
int bcg_smoother_launch_ms(bcg_ctx* ctx, double* ms);

/* ------------------------------------------------------------------ */
/* steady glucose field and its adjoint (no reference counterpart)       */
/* ------------------------------------------------------------------ */
/* A 2-D x-z grid of nx x nz vertices (nx, nz of the form 2^a + 1) at
 * spacing h: rows k < nz_agar are agar, the rest the colony region; row 0
 * is held at c0.  With theta = {d_agar, d_colony, vmax, km} the steady
 * field C solves, at every other vertex,
 *   sum_faces Df (C_nb - C) / h^2 = q vmax C / (km + C),
 * Df the harmonic mean of the two vertices' diffusivities, no flux through
 * the sides and top, q the uptake density: the sum of w_c L_c R_c / h^2
 * over the cells whose centre rounds to the vertex (the deposition of
 * GetDensity, Compute.cpp:120-253, weighted per cell). */
typedef struct bcg_steady_params {
    int nx, nz, nz_agar, max_cells;
    double h, c0;
} bcg_steady_params;
typedef struct bcg_steady bcg_steady;
int bcg_steady_create(const bcg_steady_params* p, bcg_steady** out);
int bcg_steady_destroy(bcg_steady* s);
/* cells as 4 doubles each: centre x (from the grid's left edge), centre z
 * (from the agar bottom), length L, radius R; at most max_cells */
int bcg_steady_set_cells(bcg_steady* s, const double* xzlr, int ncell);
/* Newton to max|F| <= tol * (max|F| at C = c0); C_out (nx*nz, row k at
 * offset k*nx, optional) receives the field.  The converged state is kept
 * for bcg_steady_vjp. */
int bcg_steady_solve(bcg_steady* s, const double* theta, const double* w, double tol,
                     double* C_out, int* newton_iters, int* cg_iters);
/* Vector-Jacobian product at the last solve: given dL/dC (nx*nz), the
 * gradients dL/dtheta (4) and dL/dw (per cell, optional).  Exact for the
 * converged field: one adjoint solve A lambda = -dL/dC with the symmetric
 * Newton operator, to max|residual| <= tol * max|dL/dC|. */
int bcg_steady_vjp(bcg_steady* s, const double* dL_dC, double* grad_theta, double* grad_w, double tol);

/* ------------------------------------------------------------------ */
/* timing: device time of the kernels queued by the last call of each    */
/* kind (CUDA events on the context stream), in milliseconds.            */
/* ------------------------------------------------------------------ */
typedef enum bcg_timer_id {
    BCG_T_MOVE_GROW = 0, BCG_T_DIVIDE = 1, BCG_T_NEIGHBOURS = 2,
    BCG_T_MG_SOLVE = 3, BCG_T_SWEEPS = 4, BCG_T_DENSITY = 5, BCG_T_COUNT = 6
} bcg_timer_id;
int bcg_enable_timers(bcg_ctx* ctx, int on);
int bcg_get_timer(bcg_ctx* ctx, int timer, double* ms, int64_t* launches);

/* Step timeline: CUDA events recorded at the phases of each bcg_sim step,
 * on the stream each phase runs on.  Unlike the timers above it never
 * synchronises, so the benchmark cadence's solve still runs beside the
 * mechanics.  Marks past the capacity are dropped.  The first solve from a
 * starting state runs in order on the context stream (it is captured as a
 * graph from the second one on): that step's two solve marks bracket
 * nothing. */
typedef enum bcg_timeline_tag {
    BCG_TL_STEP = 1,          /* step start (context stream) */
    BCG_TL_SOLVE_BEGIN = 2,   /* agar solve queued on the second stream: its start */
    BCG_TL_SOLVE_END = 3,     /* its end (second stream) */
    BCG_TL_MECH_BEGIN = 4,    /* before MoveCell + GrowCell (context stream) */
    BCG_TL_MECH_END = 5,      /* after their counters were read back */
    BCG_TL_DIVIDE_END = 6,    /* after the division loop */
    BCG_TL_STEP_END = 7       /* context stream after it waited for the solve */
} bcg_timeline_tag;
/* capacity > 0: (re)start a timeline of up to `capacity` marks; 0: stop
 * and release its events. */
int bcg_timeline_enable(bcg_ctx* ctx, int capacity);
/* Wait for the context's streams, then give the marks so far in the order
 * they were queued: tags[i] and ms[i], the time since the first mark
 * (at most `capacity` of them, *n = their count).  The timeline restarts
 * empty. */
int bcg_timeline_read(bcg_ctx* ctx, int* tags, float* ms, int capacity, int* n);

/* ------------------------------------------------------------------ */
/* host helpers                                                         */
/* ------------------------------------------------------------------ */
/* glibc-compatible rand() stream owned by the host (the reference seeds
 * the process-wide rand() with srand, CellMD3D.cpp:23).  Implemented from
 * the published TYPE_3 additive-feedback description; bcg_rng_skip uses a
 * polynomial jump-ahead so skipping the F_cw draws costs O(31^2 log k). */
typedef struct bcg_rng { uint32_t r[34]; int32_t pos; } bcg_rng;
void    bcg_rng_seed(bcg_rng* g, uint32_t seed);
int32_t bcg_rng_next(bcg_rng* g);
void    bcg_rng_skip(bcg_rng* g, int64_t k);

/* Seeded synthetic colony (2-D x-z half-ellipse dome on the agar,
 * random sequential placement, no overlaps); see the generator notes in
 * the design document.  Returns the cell count in *n.  width/height in um. */
int bcg_synth_colony(uint64_t seed, int n_target, double width, double height,
                     double radius, double len_lo, double len_hi,
                     double l_divide, double div_phase_spread,
                     bcg_cell* out, int capacity, int* n);

/* Binary restart files in the reference's format: double t, double dt,
 * then the Cell records (SaveCells / LoadCells, InputOutput.cpp:394-448).
 * bcg_load_restart returns the record count in *n (at most capacity). */
int bcg_save_restart(const char* path, double t, double dt, const bcg_cell* cells, int n);
int bcg_load_restart(const char* path, double* t, double* dt, bcg_cell* cells, int capacity, int* n);

/* mean_stress for every cell (Compute.cpp:18-117, called on output steps at
 * Simulation.cpp:316-327): stress receives 5 doubles per cell (xx, yy, zz,
 * rr, tt of the Tensor), fnet (optional) 3 per cell; *fcw_calls = the
 * rand() draws the reference makes here (one per wall-near cell). */
int bcg_mean_stress(bcg_ctx* ctx, double* stress, double* fnet, int64_t* fcw_calls);

/* bcg_mean_stress without any allocation.  No counterpart in the reference.
 * bcg_mean_stress stages its per-cell results in device buffers it
 * allocates on each call; this variant is for hosts that cannot allocate
 * device memory when they write an output step: a host whose device memory
 * is reserved up front (another framework's caching allocator holding the
 * GPU, so an allocation here can fail), or an output thread that must not
 * call into the CUDA allocator (whose pool operations and frees can wait on
 * other work on the device).  Same arguments and results as
 * bcg_mean_stress.  The results are staged instead in one fixed device array
 * built into the library, room for BCG_NOALLOC_MAX_CELLS cells (2 MiB),
 * which every GPU that loads the library holds until the process exits.
 *   - A colony of more than BCG_NOALLOC_MAX_CELLS cells returns
 *     BCG_E_UNSUPPORTED; a call whose current device is not the context's
 *     returns BCG_E_ARG.
 *   - Every call looks the array's device address up
 *     (cudaGetSymbolAddress), which allocates nothing.  The array itself
 *     comes into being when the library's device code is loaded on a
 *     device, which with lazy loading can be this first call: make the
 *     first call on a device (or create a context there, which loads the
 *     code too) before any stream capture on it and before the host's
 *     allocator reserves that device's memory.
 *   - Every call on a device uses the same array, which keeps the previous
 *     call's contents.  Calls that can overlap on the GPU (other contexts,
 *     other host threads) race on it and must be serialised by the caller. */
#define BCG_NOALLOC_MAX_CELLS 32768
int bcg_mean_stress_noalloc(bcg_ctx* ctx, double* stress, double* fnet, int64_t* fcw_calls);

/* ------------------------------------------------------------------ */
/* Output steps in the reference's on-disk formats.                      */
/* Directory tree of CreateOutputFiles (InputOutput.cpp:42-271):         */
/*   <dir>/<Name>/<id>.txt for Name in Cells, Restart, RoughDensity,     */
/*   RoughDensity1, RoughDensity2, Density, Density1, Density2,          */
/*   WallDensity, WallDensity1, WallDensity2, RoughHeight, Height,       */
/*   Normal, Environment, AgarField, WallField; <dir>/lineage/0.txt      */
/*   (CreateOutputFileLineage, InputOutput.cpp:13-33).  The reference    */
/*   leaves all but Cells, Restart, Density, Environment, AgarField and  */
/*   WallField empty (their writers are commented out in Simulation.cpp), */
/*   and so does this library.                                           */
/* Contents:                                                             */
/*   Cells       one line per cell, Output (InputOutput.cpp:799-817)     */
/*   Restart     {t, dt, Cell[n]} raw, SaveCells (InputOutput.cpp:434-448) */
/*   Density     DensityShiftP, Array3D<double>::Output(f, 1)            */
/*               (Array.h:568-584)                                       */
/*   Environment Array3D<LocalEnv>::Output(f, 1) (Array.h:931-1122):    */
/*               the 17 members of LocalEnv listed in bcg_output_data.env */
/*   AgarField   Array3D<LocalAga>::Append(f, 1) of every level          */
/*               (Array.h:1447-1494): CarbonAgar, AcetateAgar, WasteAgar, */
/*               OxygenAgar                                              */
/*   WallField   Array2D<LocalAga>::Append(f) of every level             */
/*               (Array.h:417-456), the same four members                */
/* Numbers are printed with the reference's printf formats ("%6E\t" for  */
/* fields, the 28-field line of Output for cells), so a file holds the   */
/* same bytes as the reference's for the same values.                    */
/* ------------------------------------------------------------------ */
#define BCG_OUT_CELLS  1   /* create the step's files; write Cells/<id>.txt */
#define BCG_OUT_FIELDS 2   /* write Restart, Density, Environment, AgarField, WallField */

/* One output step's data on the host.  Field arrays are x-major with z
 * fastest, as bcg_get_field returns them (Array3D's own order with
 * box_y = 1).  The reference's MG path never writes FieldAgar's WasteAgar,
 * which keeps its initial 0 (Nutrients.h:66-74); a NULL agar entry prints
 * zeros. */
typedef struct bcg_output_data {
    double t;                     /* time printed on every cell line            */
    double dt;                    /* second double of the restart header        */
    int32_t n_cells;              /* cells printed to Cells/<id>.txt            */
    int32_t force_stride;         /* doubles per cell in cell_force (>= 3)      */
    const bcg_cell* cells;        /* old_cells, before MoveCell                  */
    const double* cell_force;     /* the 3 printed per cell: T.xx, T.yy, T.zz of
                                     mean_stress (bcg_mean_stress's stride 5), or
                                     Fnet of F_surf_tension in the initial block */
    int32_t n_restart;            /* cells saved to Restart/<id>.txt; -1 leaves
                                     the file empty (the initial block)          */
    int32_t levels;               /* maxLevelsMG                                 */
    const bcg_cell* restart_cells;/* new_cells, after MoveCell/GrowCell          */
    int32_t box_x, box_z, box_z_agar, reserved;
    const double* density;        /* DensityShiftP (box_x*box_z)                 */
    const double* env[17];        /* Environment in file order: Carbon, Acetate,
                                     Waste, Oxygen, GrowthRate1, GrowthRate2,
                                     GrCarAer, GrCarAna, GrAceAer, pH, Hydrox,
                                     Buffer, Acetic, qCarmnt, qAcemnt, pAcemnt,
                                     qOxymnt (box_x*box_z each)                  */
    const double* const* agar;    /* 4 per level, level-major: CarbonAgar,
                                     AcetateAgar, WasteAgar, OxygenAgar of
                                     FieldAgar[l] (box_x*box_z_agar each)        */
    const double* const* wall;    /* 4 per level, the same members of
                                     FieldWall[l] (box_x each)                   */
} bcg_output_data;

/* Write one output step's files from host data, synchronously, with
 * `threads` formatting threads (0 = all hardware threads).  `what` is a
 * mask of BCG_OUT_*: BCG_OUT_CELLS creates the step's whole tree the way
 * CreateOutputFiles does (Cells/<id>.txt opened for append when `append`,
 * every other file truncated); BCG_OUT_FIELDS then fills the field files
 * and Restart.  Missing directories are created (mode 0775).  BCG_E_IO
 * when a directory or file cannot be created or written.  Needs no GPU. */
int bcg_write_output(const char* dir, int output_id, int what, int append,
                     const bcg_output_data* d, int threads);

/* Asynchronous output writer.  Each bcg_output_* call snapshots what the
 * step writes on the context's stream (one gather kernel into a device
 * staging buffer), queues one device-to-host copy of it on the writer's
 * own copy stream, and hands the step to the writer's host thread, which
 * waits for the copy, formats with `threads` threads and writes the files
 * while the GPU goes on with the next steps.  At most `max_pending` steps
 * (>= 1) are queued; a further call waits for the oldest.  All contexts
 * given to one writer are on one device.  An error of the host thread
 * (BCG_E_IO) is returned by the next call and by bcg_writer_wait.
 * bcg_writer_create truncates <dir>/lineage/0.txt (CellMD3D.cpp:78). */
typedef struct bcg_writer bcg_writer;
int bcg_writer_create(const char* dir, int append, int threads, int max_pending, bcg_writer** out);
/* Wait until every queued step is on disk; the first error, if any. */
int bcg_writer_wait(bcg_writer* w);
/* Waits, then frees the writer. */
int bcg_writer_destroy(bcg_writer* w);
/* The initial output block, Simulation.cpp:185-244, as output step 0: the
 * fields, then one line per cell with F_surf_tension's force
 * (Forces.cpp:209) in the three stress columns; Restart/0.txt stays empty. */
int bcg_output_initial(bcg_writer* w, bcg_ctx* ctx, double t);
/* First half of an output step, before MoveCell (Simulation.cpp:316-327):
 * CreateOutputFiles(output_id) and one line per cell with mean_stress's
 * T.xx, T.yy, T.zz.  mean_stress calls F_cw, so this reports in fcw_calls
 * the rand() draws the host skips (as after bcg_mean_stress); it waits for
 * that count, not for the copy or the files. */
int bcg_output_cells(bcg_writer* w, bcg_ctx* ctx, int output_id, double t, int64_t* fcw_calls);
/* Second half, after bcg_move_grow and before bcg_divide
 * (Simulation.cpp:340-372): Restart (the moved, grown, undivided cells,
 * t and dt) and the field files.  Does not wait for the GPU. */
int bcg_output_fields(bcg_writer* w, bcg_ctx* ctx, int output_id, double t, double dt);
/* Append lineage pairs (parent, daughter) to <dir>/lineage/0.txt as
 * "%d %d\n" lines (Simulation.cpp:392), in queue order with the steps. */
int bcg_writer_lineage(bcg_writer* w, const int* pairs, int n_pairs);

/* ------------------------------------------------------------------ */
/* C++ host loop (rewrite of SimSingleThread, Simulation.cpp:42-434)     */
/* ------------------------------------------------------------------ */
typedef struct bcg_sim bcg_sim;
/* Build a simulation from params and n cells; seeds the host rand() stream
 * with `seed`, draws the rough wall (Simulation.cpp:161-168) and runs the
 * initial field block (Simulation.cpp:185-217) if run_initial_fields. */
int bcg_sim_create(const bcg_params* p, const bcg_cell* cells, int n, uint32_t seed,
                   int run_initial_fields, bcg_sim** out);
int bcg_sim_destroy(bcg_sim* sim);
/* Advance `steps` iterations of the while loop (Simulation.cpp:254-431),
 * honouring UpdateFlag / HeightDensityUpdateFlag and OutFlag: an output
 * step runs mean_stress on every cell before MoveCell and skips its
 * rand() draws, as the reference does; with a writer attached it also
 * writes the step's files and the lineage lines.  A step that fails
 * returns its status and marks the simulation failed: the colony may be
 * left between MoveCell and the division loop, so every later run returns
 * the same status. */
int bcg_sim_run(bcg_sim* sim, int steps);
/* Attach (or, with NULL, detach) an output writer; the simulation does not
 * own it.  write_initial also writes the initial block's output
 * (Simulation.cpp:185-244) now, as output step 0; call it before the first
 * step.  Later output steps count from 0 again (koutput, Simulation.cpp:251,
 * 319), overwriting step 0 like the reference. */
int bcg_sim_set_writer(bcg_sim* sim, bcg_writer* w, int write_initial);
bcg_ctx* bcg_sim_ctx(bcg_sim* sim);
int bcg_sim_time(bcg_sim* sim, double* t, int* n_cells, int64_t* divisions);
/* Work the simulation has run so far: full neighbour rebuilds
 * (getNeighbours, Simulation.cpp:292, or the benchmark cadence's) and
 * field updates (the UpdateFlag block, Simulation.cpp:261-294). */
int bcg_sim_counters(bcg_sim* sim, int64_t* neighbour_rebuilds, int64_t* field_updates);
/* Lineage pairs recorded so far (parent, daughter), up to capacity pairs. */
int bcg_sim_lineage(bcg_sim* sim, int* pairs, int capacity, int* n);
/* Per-step mode used by benchmarks: each step runs the mechanics step and
 * `vcycles` V-cycles of the agar solve instead of the reference's field
 * cadence (0 = mechanics only).  The solve touches no data of the
 * mechanics in this cadence, so it runs beside them on the context's second
 * stream; results are the same as in sequence. */
int bcg_sim_set_step_mode(bcg_sim* sim, int field_cadence_reference, int vcycles_per_step);

/* Ensembles of independent colonies (no reference counterpart; the
 * reference runs one colony per process).  `members` are simulations in
 * the benchmark cadence (bcg_sim_set_step_mode(.., 0, v)), of any sizes
 * and grids; the ensemble does not own them.  bcg_ensemble_run advances
 * every member by `steps` steps, each exactly as bcg_sim_run would, with
 * every phase queued for all members (one stream each) before any member
 * is waited for.  BCG_E_UNSUPPORTED for a member in the reference cadence.
 * A member whose step fails is marked failed (as by bcg_sim_run) and the
 * run returns the first such status after the other members have finished
 * the step; a run with a failed member returns its status at once. */
typedef struct bcg_ensemble bcg_ensemble;
int bcg_ensemble_create(bcg_sim* const* members, int n, bcg_ensemble** out);
int bcg_ensemble_run(bcg_ensemble* e, int steps);
int bcg_ensemble_destroy(bcg_ensemble* e);

#ifdef __cplusplus
}
#endif
#endif /* BCG_H_ */
