/*
 * ctx.cuh -- the bcg_ctx structure shared by the translation units.
 */
#pragma once
#include "common.cuh"

#define BCG_MAX_MG_LEVELS 16
#define BCG_MAX_AGAR_LEVELS 8
/* records a context's host<->device staging buffer holds (27 MB) */
#define CTX_STAGE_CELLS (1 << 17)

/* one multigrid level: three species, Sol/Res/Err, (nx+1) x (nz+1) points
 * stored k-major (row k holds i = 0..nx contiguously, row pitch `pitch`) */
struct MgLevel {
    int nx, nz, pitch;
    double* sol[3];   /* species 0 = carbon, 1 = oxygen, 2 = acetate */
    double* res[3];
    double* err[3];
    float* errf[3];   /* FP32 shadows used by the mixed-precision solve */
    float* resf[3];
    double* err2[3];  /* second correction buffer: the fused smoother writes */
    float* errf2[3];  /* out of place and the two buffers swap roles */
};

/* one buffer of the colony environment (LocalEnv fields kept on device) */
struct EnvBuf {
    double *C, *W, *A, *O;     /* Carbon, Waste, Acetate, Oxygen */
    double *gr1, *gr2;         /* GrowthRate1/2 */
    double *ph, *hydrox, *acetic, *buffer;
    /* GrCarAer, GrCarAna, GrAceAer, qCarmnt, qAcemnt, pAcemnt, qOxymnt:
     * read by nothing but the Environment writer, so kept for buffer 0
     * (Environment) only; null in buffer 1 */
    double* extra[7];
};

/* one buffer of the wall rows, per composite level, 4 species */
struct WallBuf {
    double *C[BCG_MAX_AGAR_LEVELS], *W[BCG_MAX_AGAR_LEVELS], *O[BCG_MAX_AGAR_LEVELS], *A[BCG_MAX_AGAR_LEVELS];
};

struct bcg_ctx {
    bcg_params P;
    int device;
    cudaStream_t stream;
    int n;                 /* cells */
    int cap;               /* max_cells */
    int cur;               /* index of the "old" record buffer */
    CellRec* rec[2];
    CellSoA soa;
    /* reference-layout records between host and device: uploads and
     * downloads pass through it stage_cells records at a time */
    bcg_cell* stage;
    int stage_cells;
    /* neighbours */
    int kmax;
    int* nbr;
    int* ncount;
    /* bins */
    int nbox;
    int* box_cnt;
    int* box_start;        /* nbox + 1 */
    int* box_ids;          /* cap */
    int* cell_box;         /* cap */
    int n_binned;          /* cells covered by the last binning */
    int* scan_tmp;         /* block sums */
    /* divisions */
    int* div_list;         /* cap */
    int* div_count;        /* device counter */
    unsigned long long* fcw_count;
    int* moved;            /* cap, per-step division bookkeeping */
    int* delta_ids;        /* 2*cap */
    int* delta_box;
    int* lineage;          /* 2*cap */
    int* n_done_dev;
    float* draws_dev;      /* 9*cap */
    /* division planning (DIV_SORT_MAX divisions per step at most) */
    CellRec* div_rec;      /* 2 per division: new mother, daughter */
    int* div_box;          /* 2 per division */
    int4* div_rect;        /* footprint rectangle per division */
    int2* div_pairs;       /* overlapping footprints, DIV_PAIR_CAP */
    int* div_par;          /* union-find parents */
    int* div_order;        /* divisions grouped, ascending inside a group */
    int* div_grp;          /* (start, length) per group */
    int last_ndiv;
    /* set by MoveCell/GrowCell, cleared by the division loop: meanwhile the
     * moved, grown records (the reference's new_cells) are rec[cur ^ 1] */
    int move_pending;
    /* status */
    DevStatus* status;     /* device */
    /* pinned host staging */
    void* pinned;
    size_t pinned_bytes;
    /* fields */
    double *height, *rough_height, *nrm_x, *nrm_y, *nrm_z, *wall;
    EnvBuf env[2];         /* [0] = Environment, [1] = oldEnvironment */
    WallBuf wal[2];        /* [0] = FieldWall, [1] = oldFieldWall */
    double *rd, *inside, *rds, *ds, *dens, *rws, *wds, *rw, *wd;
    int* bbox;             /* device: minx, maxx, maxz (after +-5) */
    int host_bbox[3];
    MgLevel mg[BCG_MAX_MG_LEVELS];
    int mg_levels;
    double* mg_scratch;    /* reductions */
    /* captured [solve + sweeps] units of the nutrient update: [0] plain,
     * [1] with the acetate buffer solve in its last two sweeps */
    cudaGraphExec_t nutrient_graph[2];
    int nutrient_graph_sweeps;           /* 0: none captured (dropped whenever a kernel choice changes) */
    int nutrient_graph_launches[2];
    /* the captured per-step solve (bcg_mg_solve): its key (V-cycles, wall
     * buffer, whether Err and Res were clean on entry; -1: none) */
    cudaGraphExec_t solve_graph;
    int solve_graph_key;
    int solve_graph_seen;         /* key of the last solve run uncaptured (0: none) */
    int solve_graph_off;          /* 1: a capture failed, the context solves with plain launches */
    int solve_graph_launches;
    /* the second stream of the benchmark step's agar solve, which runs beside
     * the step's mechanics; ev_fork orders it after the work before it,
     * ev_join orders the work after the step after it */
    cudaStream_t aux_stream;
    cudaEvent_t ev_fork, ev_join;
    /* timers */
    int timers_on;
    /* step timeline (bcg_timeline_*): tl_cap events, tl_n of them recorded */
    cudaEvent_t* tl_ev;
    int* tl_tag;
    int tl_cap, tl_n;
    cudaEvent_t ev[BCG_T_COUNT][2];
    double timer_ms[BCG_T_COUNT];
    long long timer_launches[BCG_T_COUNT];
    long long launches;    /* kernels queued by this context (all kinds) */
    /* kernel shapes of this context, chosen by bcg_autotune or set by the
     * caller (0 = default); no kernel choice is process-wide */
    int force_group;
    int force_occ;         /* blocks an SM for the force loop's register budget (3 or 4) */
    int smooth_warps;
    int relax_mode;        /* agar smoother form, bcg_set_relax_mode (3 by default) */
    size_t cluster_smem[2];/* coarsest-level cluster kernel: shared-memory size checked */
    int cluster_ok[2];     /* ... and whether its clusters fit (FP64, FP32) */
    /* multigrid Err (all levels) and Res (levels > 0) are zero, as the last
     * reset() left them; setup() then skips its resetZero */
    int mg_clean;
    /* level 0's Res of the last reset() not computed yet (done on demand) */
    int mg_res0_stale;
    int pair_f32;          /* contact geometry in FP32 local to cell i (bcg_set_pair_precision) */
    int pending_error;     /* host-side set-up failure of a queued launch, returned by the next status check */
    /* legacy explicit agar solver (allocated on its first call): FieldAgar
     * [0] and oldFieldAgar [1] per composite level, species carbon, waste,
     * oxygen, acetate, box_z_agar rows of box_x (row z contiguous); the
     * multigrid solution rows 1..box_z_agar stand for FieldAgar elsewhere */
    double* leg[2][BCG_MAX_AGAR_LEVELS][4];
    double* leg_snap;      /* acetate before the last iteration's write (box_x*box_z) + wall row (box_x) */
    unsigned long long* leg_conv;   /* convergence count per iteration */
    int leg_conv_cap;
    int leg_old_stale;     /* an agar solve ran since: oldFieldAgar := FieldAgar (copyFromMG) */
    double smooth_tune_ms; /* device time of one level-0 fused smoother launch at the tuned shape */
};

MechParams mech_params(const bcg_ctx* c);
FieldPtrs field_ptrs(const bcg_ctx* c);
int ctx_check_status(bcg_ctx* c);   /* syncs, reads the device status word */
void timer_begin(bcg_ctx* c, int t);
void timer_end(bcg_ctx* c, int t, int launches);
int ensure_pinned(bcg_ctx* c, size_t bytes);
void nutrient_graphs_drop(bcg_ctx* c);
int launch_move_grow(bcg_ctx* c, double dt, int group, int occ);
/* output-step kernels queued on `s`: the colony as reference records,
 * old_cells or (moved != 0) new_cells (ctx.cu), mean_stress's 5 stress components per cell with the F_cw count
 * added to `fcw` (mech.cu), F_surf_tension's force, 3 per cell (mech.cu) */
void launch_pack_cells(bcg_ctx* c, bcg_cell* dst, cudaStream_t s, int moved);
void launch_mean_stress(bcg_ctx* c, double* stress, unsigned long long* fcw, cudaStream_t s);
void launch_surface_force(bcg_ctx* c, double* force, cudaStream_t s);
int mg_tune_smoother(bcg_ctx* c, int* choice);
/* compute level 0's multigrid Res left pending by the last reset() (mg.cu);
 * called before its inputs (Sol, insideColonyDen) change or it is read */
void mg_res0_materialise(bcg_ctx* c);
int mg_kernel_attributes();
int mech_kernel_attributes();
