/*
 * ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Drives the unmodified reference C++ sources (AgentBasedModel-BacColonyGrowth/
 * *.cpp except CellMD3D.cpp, compiled by oracle/Makefile into oracle/_ref/)
 * through a small C API shaped like include/bcg.h, so that tests can run the
 * same scenario through the reference, through the C restatement in
 * oracle/oracle.c, and through the CUDA library, and compare.
 *
 * The loop bodies below call the reference's own functions in the order
 * SimSingleThread uses them (Simulation.cpp:42-434); no reference arithmetic
 * is re-implemented here.  rand() is wrapped at link time
 * (-Wl,--wrap=rand) so the number of draws the reference makes can be read.
 */
#include <omp.h>
#include <stdio.h>
#include <sys/stat.h>
#include <string.h>
#include <stdlib.h>
#include <math.h>
#include <algorithm>
#include <sstream>
#include <string>
#include <fstream>
#include <iostream>
#include <cmath>

#define private public   /* the harness reads Multigrid's private arrays and dt,
                            and pads Array3D storage (see ref_init) */
#include "tools.h"
#include "Cell.h"
#include "Constants.h"
#include "UniformGrid.h"
#include "Array.h"
#include "Nutrients.h"
#include "Neighbours.h"
#include "Cells.h"
#include "Compute.h"
#include "Forces.h"
#include "Multigrid.h"
#include "InputOutput.h"
#undef private

#include "../include/bcg.h"

static_assert(sizeof(Cell) == sizeof(bcg_cell), "Cell record size");

/* ---- rand() call counter -------------------------------------------------- */
extern "C" int __real_rand(void);
static long long g_rand_calls = 0;
extern "C" int __wrap_rand(void) { ++g_rand_calls; return __real_rand(); }

/* ---- state (mirrors the locals of main() and SimSingleThread) ------------- */
namespace {
struct RefState {
    int N = 0;
    Cell* old_cells = nullptr;
    Cell* new_cells = nullptr;
    UniformGrid* grid = nullptr;
    int maxNeighbours = 0;
    int** nbr = nullptr;
    DoubleArray2D* Height = nullptr;
    DoubleArray3D *Density = nullptr, *Density1 = nullptr, *Density2 = nullptr;
    DoubleArray2D *WallDensity = nullptr, *WallDensity1 = nullptr, *WallDensity2 = nullptr;
    EnvArray3D *Env = nullptr, *oldEnv = nullptr;
    AgaArray3D **FieldAgar = nullptr, **oldFieldAgar = nullptr;
    AgaArray2D **FieldWall = nullptr, **oldFieldWall = nullptr;
    CoordArray2D* Normal = nullptr;
    DoubleArray2D* Wall = nullptr;
    /* SimSingleThread locals */
    DoubleArray2D* Filter = nullptr; int FilterDim = 0;
    DoubleArray3D* Filter3D = nullptr;
    DoubleArray3D *RoughDensity, *RoughDensity1, *RoughDensity2, *insideColonyDen;
    DoubleArray2D *RoughWallDensity, *RoughWallDensity1, *RoughWallDensity2;
    DoubleArray3D *RoughDensityShiftP, *RoughDensity1ShiftP, *RoughDensity2ShiftP;
    DoubleArray2D *RoughWallDensityShiftP, *RoughWallDensity1ShiftP, *RoughWallDensity2ShiftP;
    DoubleArray3D *DensityShiftP, *Density1ShiftP, *Density2ShiftP;
    DoubleArray2D *WallDensityShiftP, *WallDensity1ShiftP, *WallDensity2ShiftP;
    DoubleArray2D* RoughHeight = nullptr;
    Multigrid* mg = nullptr;
    int* dividingCells = nullptr;
    int* IDlist = nullptr;
    int minx = 0, maxx = 0, miny = 0, maxy = 0, maxz = 0;
    double t = 0, dt = 0;
    double NextOutTime, NextUpdateTime, HeightDensityNextUpdateTime, HeightDensityUpdateTime;
    bool UpdateFlag = true, HeightDensityUpdateFlag = true;
    bool OutFlag = false;          /* false once the initial block has run, Simulation.cpp:243 */
    int koutput = 0;
    long long lineage_n = 0;
    int* lineage = nullptr; int lineage_cap = 0;
    int last_numDivide = 0;
};
RefState S;

void set_globals(const bcg_params* p)
{
    BoxX = p->box_x; BoxY = p->box_y; BoxZ = p->box_z; BoxZAgar = p->box_z_agar;
    maxLevelsMG = p->max_levels_mg; FilterLen = p->filter_len;
    refinementGridHeight = p->refinement_grid_height; maxCells = p->max_cells;
    cellRadius = p->cell_radius; L_divide = p->l_divide; k_cc = p->k_cc; k_wc = p->k_wc;
    varL = p->var_l; varAngle = p->var_angle; var_pos = p->var_pos;
    viscosity = p->viscosity; wall_rough = p->wall_rough; gamma_t = p->gamma_t;
    cell_mu = p->cell_mu; wall_mu = p->wall_mu; density_threshold = p->density_threshold;
    tension = p->tension; DH = p->delta_h; Rc = p->rc;
    initial_dt = p->dt; t0 = p->t0; t_max = p->t_max; OutputTime = p->output_time;
    UpdateTime = p->update_time;
    KC_aer = p->kc_aer; KC_ana = p->kc_ana; KW = p->kw; KO = p->ko; KA = p->ka; KI = p->ki;
    Carbon_to_Waste = p->carbon_to_waste; C_rate = p->c_rate; W_rate = p->w_rate;
    Maintenance_rate = p->maintenance_rate;
    qCarAer = p->q_car_aer; qCarAna = p->q_car_ana; qAceAer = p->q_ace_aer;
    qO2Car = p->q_o2_car; qO2Ace = p->q_o2_ace; pAceAer = p->p_ace_aer; pAceAna = p->p_ace_ana;
    DiffColony = p->diff_colony; DiffAgar = p->diff_agar;
    DiffColonyCarbon = p->diff_colony_carbon; DiffAgarCarbon = p->diff_agar_carbon;
    DiffColonyO2 = p->diff_colony_o2; DiffAgarO2 = p->diff_agar_o2;
    DiffColonyAce = p->diff_colony_ace; DiffAgarAce = p->diff_agar_ace;
    maxCarbon = p->max_carbon; maxO2 = p->max_o2; maxO2_Agar = p->max_o2_agar;
    maxGrowthRate1 = p->max_growth_rate1; maxGrowthRate2 = p->max_growth_rate2;
    maxGrowthRateCarAer = p->max_gr_car_aer; maxGrowthRateCarAna = p->max_gr_car_ana;
    maxGrowthRateAceAer = p->max_gr_ace_aer;
    Cdt = p->cdt;
    qCarAernt = p->q_car_aer_nt; qCarAnant = p->q_car_ana_nt; qAceAernt = p->q_ace_aer_nt;
    qO2Carnt = p->q_o2_car_nt; qO2Acent = p->q_o2_ace_nt; pAceAnant = p->p_ace_ana_nt;
    Kw = p->kw_ph; Ka = p->ka_ph; Kb = p->kb_ph; Cb = p->cb_ph; c1 = p->c1_ph;
    crossFeeding = p->cross_feeding != 0; InterfaceCondition = p->interface_condition;
    NutrientGSI = p->nutrient_gsi != 0;
    BoxLength = p->box_length;
}

DoubleArray3D* a3() { return new DoubleArray3D(BoxX, BoxY, BoxZ); }
DoubleArray2D* a2() { return new DoubleArray2D(BoxX, BoxY); }

/* Filters of Simulation.cpp:61-110 */
void make_filters()
{
    S.Filter = new DoubleArray2D(FilterLen, 1);
    double value = 1.0 / (double)(FilterLen);
    for (int ii = 0; ii < FilterLen; ii++) S.Filter->Set(ii, 0, value);
    S.FilterDim = FilterLen / 2;
    S.Filter3D = new DoubleArray3D(FilterLen, FilterLen, FilterLen);
    double norm = 0;
    for (int ii = 0; ii < FilterLen; ii++)
        for (int kk = 0; kk < FilterLen; kk++)
            norm += exp(-(ii - FilterLen / 2) * (ii - FilterLen / 2) - (kk - FilterLen / 2) * (kk - FilterLen / 2));
    for (int ii = 0; ii < FilterLen; ii++)
        for (int kk = 0; kk < FilterLen; kk++)
            S.Filter3D->Set(ii, 0, kk, exp(-(ii - FilterLen / 2) * (ii - FilterLen / 2) - (kk - FilterLen / 2) * (kk - FilterLen / 2)) / norm);
}
} // namespace

extern "C" {

long long ref_rand_calls(void) { return g_rand_calls; }
void ref_set_threads(int n) { omp_set_num_threads(n > 0 ? n : omp_get_max_threads()); }

/* Allocate as main() + the top of SimSingleThread do (CellMD3D.cpp:46-142,
 * Simulation.cpp:44-169).  The rough wall consumes BoxX*BoxY rand() draws
 * right after srand(seed), as in the reference when make_wall != 0. */
/* free the previous scenario (the harness keeps one at a time) */
static void ref_release(void)
{
    if (!S.old_cells) return;
    delete[] S.old_cells; delete[] S.new_cells;
    if (S.nbr) { for (int i = 0; i < maxCells; i++) delete[] S.nbr[i]; delete[] S.nbr; }
    delete S.grid; delete S.Height; delete S.Density; delete S.Density1; delete S.Density2;
    delete S.WallDensity; delete S.WallDensity1; delete S.WallDensity2; delete S.Env; delete S.oldEnv;
    for (int i = 0; i < maxLevelsMG; i++) { delete S.FieldAgar[i]; delete S.oldFieldAgar[i]; delete S.FieldWall[i]; delete S.oldFieldWall[i]; }
    delete[] S.FieldAgar; delete[] S.oldFieldAgar; delete[] S.FieldWall; delete[] S.oldFieldWall;
    delete S.Normal; delete S.Wall; delete S.Filter; delete S.Filter3D;
    DoubleArray3D* a3s[] = {S.RoughDensity, S.RoughDensity1, S.RoughDensity2, S.insideColonyDen, S.RoughDensityShiftP,
        S.RoughDensity1ShiftP, S.RoughDensity2ShiftP, S.DensityShiftP, S.Density1ShiftP, S.Density2ShiftP};
    for (auto* a : a3s) delete a;
    DoubleArray2D* a2s[] = {S.RoughWallDensity, S.RoughWallDensity1, S.RoughWallDensity2, S.RoughWallDensityShiftP,
        S.RoughWallDensity1ShiftP, S.RoughWallDensity2ShiftP, S.WallDensityShiftP, S.WallDensity1ShiftP, S.WallDensity2ShiftP, S.RoughHeight};
    for (auto* a : a2s) delete a;
    /* S.mg holds padded arrays (see ref_init) and is not deleted */
    delete[] S.dividingCells; delete[] S.IDlist;
    S = RefState();
}

int ref_init(const bcg_params* p, unsigned seed, int make_wall, int threads)
{
    ref_release();
    set_globals(p);
    ref_set_threads(threads);
    srand(seed);
    g_rand_calls = 0;
    S = RefState();
    S.old_cells = new Cell[maxCells];
    S.new_cells = new Cell[maxCells];
    memset(S.old_cells, 0, sizeof(Cell) * (size_t)maxCells);
    memset(S.new_cells, 0, sizeof(Cell) * (size_t)maxCells);
    S.grid = new UniformGrid(BoxX, BoxY, BoxZ, p->max_cells_per_box, BoxLength);
    S.maxNeighbours = S.grid->MaxCellsPerBox() * 27 + 1;
    S.nbr = InitializeNeighbourList(maxCells, S.maxNeighbours);
    S.Height = new DoubleArray2D(BoxX * refinementGridHeight, BoxY * refinementGridHeight);
    S.Height->Initialize(cellRadius);
    S.Density = a3(); S.Density1 = a3(); S.Density2 = a3();
    S.WallDensity = a2(); S.WallDensity1 = a2(); S.WallDensity2 = a2();
    S.Env = new EnvArray3D(BoxX, BoxY, BoxZ);
    S.oldEnv = new EnvArray3D(BoxX, BoxY, BoxZ);
    S.FieldAgar = new AgaArray3D*[maxLevelsMG]; S.oldFieldAgar = new AgaArray3D*[maxLevelsMG];
    S.FieldWall = new AgaArray2D*[maxLevelsMG]; S.oldFieldWall = new AgaArray2D*[maxLevelsMG];
    for (int i = 0; i < maxLevelsMG; i++) {
        S.FieldAgar[i] = new AgaArray3D(BoxX, BoxY, BoxZAgar);
        S.oldFieldAgar[i] = new AgaArray3D(BoxX, BoxY, BoxZAgar);
        S.FieldWall[i] = new AgaArray2D(BoxX, BoxY);
        S.oldFieldWall[i] = new AgaArray2D(BoxX, BoxY);
    }
    S.Normal = new CoordArray2D(BoxX * refinementGridHeight, BoxY * refinementGridHeight);
    for (int i = 0; i < BoxX * refinementGridHeight; i++) S.Normal->At(i, 0) = DoubleCoord(0, 0, -1);
    make_filters();
    S.RoughDensity = a3(); S.RoughDensity1 = a3(); S.RoughDensity2 = a3(); S.insideColonyDen = a3();
    S.RoughWallDensity = a2(); S.RoughWallDensity1 = a2(); S.RoughWallDensity2 = a2();
    S.RoughDensityShiftP = a3(); S.RoughDensity1ShiftP = a3(); S.RoughDensity2ShiftP = a3();
    S.RoughWallDensityShiftP = a2(); S.RoughWallDensity1ShiftP = a2(); S.RoughWallDensity2ShiftP = a2();
    S.DensityShiftP = a3(); S.Density1ShiftP = a3(); S.Density2ShiftP = a3();
    S.WallDensityShiftP = a2(); S.WallDensity1ShiftP = a2(); S.WallDensity2ShiftP = a2();
    S.RoughHeight = new DoubleArray2D(BoxX * refinementGridHeight, BoxY * refinementGridHeight);
    S.RoughHeight->Initialize(cellRadius);
    DoubleArray3D* zero3[] = {S.RoughDensity, S.RoughDensity1, S.RoughDensity2, S.insideColonyDen,
        S.RoughDensityShiftP, S.RoughDensity1ShiftP, S.RoughDensity2ShiftP, S.DensityShiftP,
        S.Density1ShiftP, S.Density2ShiftP, S.Density, S.Density1, S.Density2};
    for (auto* a : zero3) a->Initialize(0.0);
    DoubleArray2D* zero2[] = {S.RoughWallDensity, S.RoughWallDensity1, S.RoughWallDensity2,
        S.RoughWallDensityShiftP, S.RoughWallDensity1ShiftP, S.RoughWallDensity2ShiftP,
        S.WallDensityShiftP, S.WallDensity1ShiftP, S.WallDensity2ShiftP, S.WallDensity,
        S.WallDensity1, S.WallDensity2};
    for (auto* a : zero2) a->Initialize(0.0);
    /* Multigrid::restrictionAgaElementwise clamps its column to BoxX and so
     * reads insideColonyDen one x-row past the end (Multigrid.cpp:279, 335);
     * give that row defined storage (0 = outside the colony) so runs are
     * reproducible.  The array's own elements are unchanged. */
    {
        double* padded = new double[(size_t)(BoxX + 1) * BoxY * BoxZ]();
        delete[] S.insideColonyDen->Data;
        S.insideColonyDen->Data = padded;
    }
    S.mg = new Multigrid(maxLevelsMG, p->mg_levels, BoxX, BoxY, BoxZAgar);
    S.mg->setInsideColony(S.insideColonyDen);
    /* On levels with nz <= 1 the smoother and the transfers index k = -1 and
     * k = nz+1, which the flat Array3D index maps onto the neighbouring
     * column, or one element before/after the array at the ends
     * (Multigrid.cpp:160-249, 269-467).  Give those two elements defined
     * storage (0) so runs are reproducible; the array itself is unchanged.
     * The padded arrays are never handed back to Array3D's delete[]
     * (ref_release leaks the Multigrid). */
    for (int l = 0; l < p->mg_levels; l++) {
        AgaArray3D* arrs[3] = {S.mg->Aga[l], S.mg->AgaRes[l], S.mg->AgaErr[l]};
        for (AgaArray3D* a : arrs) {
            size_t n = (size_t)a->m_Size.x * a->m_Size.y * a->m_Size.z;
            LocalAga* base = new LocalAga[n + 2];
            memcpy(base + 1, a->Data, n * sizeof(LocalAga));
            memset(base, 0, sizeof(LocalAga));
            memset(base + n + 1, 0, sizeof(LocalAga));
            delete[] a->Data;
            a->Data = base + 1;
        }
    }
    S.Wall = new DoubleArray2D(BoxX, BoxY);
    for (int ii = 0; ii < BoxX; ii++)
        for (int jj = 0; jj < BoxY; jj++)
            S.Wall->Set(ii, jj, make_wall ? ((float)rand() / RAND_MAX - 0.5) * wall_rough : 0.0);
    S.dividingCells = new int[maxCells];
    S.IDlist = new int[S.maxNeighbours];
    S.t = t0; S.dt = initial_dt;
    S.NextOutTime = OutputTime;
    S.NextUpdateTime = UpdateTime;
    S.HeightDensityNextUpdateTime = UpdateTime / 10.0;
    S.HeightDensityUpdateTime = UpdateTime / 10.0;
    S.UpdateFlag = true; S.HeightDensityUpdateFlag = true;
    return 0;
}

int ref_load_cells(const bcg_cell* cells, int n)
{
    if (n > maxCells) return BCG_E_ARG;
    memcpy(S.old_cells, cells, sizeof(Cell) * (size_t)n);
    S.N = n;
    for (int i = 0; i < n; i++) S.grid->Add(i, S.grid->GetAddress(average(S.old_cells[i].Position)));
    return 0;
}

int ref_get_cells(bcg_cell* out, int cap)
{
    int n = S.N < cap ? S.N : cap;
    memcpy(out, S.old_cells, sizeof(Cell) * (size_t)n);
    return S.N;
}

int ref_num_cells(void) { return S.N; }

/* Full rebuild, Simulation.cpp:292 */
void ref_rebuild_neighbours(void) { getNeighbours(S.old_cells, S.N, *S.grid, S.nbr, S.maxNeighbours); }

int ref_get_neighbours(int* counts, int* lists, int stride)
{
    int mx = 0;
    for (int i = 0; i < S.N; i++) {
        int c = S.nbr[i][0];
        counts[i] = c;
        if (c > mx) mx = c;
        for (int j = 0; j < c && j < stride; j++) lists[(size_t)i * stride + j] = S.nbr[i][j + 1];
    }
    return mx;
}

int ref_set_neighbours(const int* counts, const int* lists, int stride)
{
    for (int i = 0; i < S.N; i++) {
        S.nbr[i][0] = counts[i];
        for (int j = 0; j < counts[i]; j++) S.nbr[i][j + 1] = lists[(size_t)i * stride + j];
    }
    return 0;
}

/* Mechanics: Simulation.cpp:330-336; returns numDivide, fills ids. */
int ref_move_grow(double dt, int* div_ids, long long* rand_calls)
{
    long long r0 = g_rand_calls;
    int numDivide = 0;
    int cellID;
#pragma omp parallel for default(shared) private(cellID) schedule(static)
    for (cellID = 0; cellID < S.N; cellID++) {
        MoveCell(cellID, *S.grid, S.old_cells, S.new_cells, S.nbr[cellID], dt, *S.Height, *S.Normal, *S.Wall);
        GrowCell(S.new_cells[cellID], cellID, dt, S.dividingCells, numDivide, *S.Env, S.FieldWall, *S.grid);
    }
    if (div_ids) memcpy(div_ids, S.dividingCells, sizeof(int) * (size_t)numDivide);
    if (rand_calls) *rand_calls = g_rand_calls - r0;
    S.last_numDivide = numDivide;
    return numDivide;
}

/* Division loop + swap, Simulation.cpp:380-413.  lineage gets pairs. */
int ref_divide(double t, int* lineage)
{
    int done = 0;
    for (int cellCount = 0; cellCount < S.last_numDivide; cellCount++) {
        if (S.N > (maxCells - 1)) break;
        const int cellID = S.dividingCells[cellCount];
        DivideCell(cellID, S.N, S.new_cells, *S.grid, S.nbr[cellID], *S.Wall, *S.Height, *S.Normal, t);
        if (lineage) { lineage[2 * done] = cellID; lineage[2 * done + 1] = S.N; }
        S.N++;
        done++;
        int IDlen = S.nbr[cellID][0];
        memcpy(S.IDlist, S.nbr[cellID], (IDlen + 1) * sizeof(int));
        S.IDlist[0] = cellID;
        S.IDlist[IDlen + 1] = S.N - 1;
        IDlen += 2;
        getNeighbours(S.new_cells, *S.grid, S.nbr, S.maxNeighbours, S.IDlist, IDlen);
    }
    Cell* tmp = S.new_cells; S.new_cells = S.old_cells; S.old_cells = tmp;
    S.last_numDivide = 0;
    return done;
}

/* Initial field block, Simulation.cpp:186-217 */
void ref_initial_fields(int run_nutrients)
{
    GetDensity(*S.RoughDensity, *S.RoughDensity1, *S.RoughDensity2, *S.insideColonyDen, *S.Height, *S.grid, S.old_cells, S.minx, S.maxx, S.miny, S.maxy, S.maxz);
    ShiftDensity(*S.RoughDensity, *S.RoughDensity1, *S.RoughDensity2, *S.RoughWallDensity, *S.RoughWallDensity1, *S.RoughWallDensity2, *S.RoughDensityShiftP, *S.RoughDensity1ShiftP, *S.RoughDensity2ShiftP, *S.RoughWallDensityShiftP, *S.RoughWallDensity1ShiftP, *S.RoughWallDensity2ShiftP, BoxX, BoxY, BoxZ);
    int fd = int((S.Filter3D->m_Size.x) / 2);
    BoxAverage(*S.RoughDensity, *S.Density, *S.RoughWallDensity, *S.WallDensity, *S.Filter3D, fd, S.minx, S.maxx, S.miny, S.maxy, S.maxz, BoxX, BoxY, BoxZ);
    BoxAverage(*S.RoughDensity1, *S.Density1, *S.RoughWallDensity1, *S.WallDensity1, *S.Filter3D, fd, S.minx, S.maxx, S.miny, S.maxy, S.maxz, BoxX, BoxY, BoxZ);
    BoxAverage(*S.RoughDensity2, *S.Density2, *S.RoughWallDensity2, *S.WallDensity2, *S.Filter3D, fd, S.minx, S.maxx, S.miny, S.maxy, S.maxz, BoxX, BoxY, BoxZ);
    BoxAverage(*S.RoughDensityShiftP, *S.DensityShiftP, *S.RoughWallDensityShiftP, *S.WallDensityShiftP, *S.Filter3D, fd, S.minx, S.maxx, S.miny, S.maxy, S.maxz, BoxX, BoxY, BoxZ);
    BoxAverage(*S.RoughDensity1ShiftP, *S.Density1ShiftP, *S.RoughWallDensity1ShiftP, *S.WallDensity1ShiftP, *S.Filter3D, fd, S.minx, S.maxx, S.miny, S.maxy, S.maxz, BoxX, BoxY, BoxZ);
    BoxAverage(*S.RoughDensity2ShiftP, *S.Density2ShiftP, *S.RoughWallDensity2ShiftP, *S.WallDensity2ShiftP, *S.Filter3D, fd, S.minx, S.maxx, S.miny, S.maxy, S.maxz, BoxX, BoxY, BoxZ);
    GetSurfaceNormal(*S.Normal, *S.Height, S.minx, S.maxx, S.miny, S.maxy);
    if (run_nutrients)
        UpdateEnvArrayMG_OxygenAcetate(S.Env, S.oldEnv, S.FieldAgar, S.oldFieldAgar, S.FieldWall, S.oldFieldWall, *S.DensityShiftP, *S.Density1ShiftP, *S.Density2ShiftP, *S.WallDensityShiftP, *S.WallDensity1ShiftP, *S.WallDensity2ShiftP, S.minx, S.maxx, S.miny, S.maxy, S.maxz, *S.Height, *S.insideColonyDen, *S.mg);
}

/* The deposition part of the UpdateFlag block, Simulation.cpp:266-280 */
void ref_update_density(void)
{
    GetDensity(*S.RoughDensity, *S.RoughDensity1, *S.RoughDensity2, *S.insideColonyDen, *S.Height, *S.grid, S.old_cells, S.minx, S.maxx, S.miny, S.maxy, S.maxz);
    ShiftDensity(*S.RoughDensity, *S.RoughDensity1, *S.RoughDensity2, *S.RoughWallDensity, *S.RoughWallDensity1, *S.RoughWallDensity2, *S.RoughDensityShiftP, *S.RoughDensity1ShiftP, *S.RoughDensity2ShiftP, *S.RoughWallDensityShiftP, *S.RoughWallDensity1ShiftP, *S.RoughWallDensity2ShiftP, BoxX, BoxY, BoxZ);
    int fd = int((S.Filter3D->m_Size.x) / 2);
    BoxAverage(*S.RoughDensity, *S.Density, *S.RoughWallDensity, *S.WallDensity, *S.Filter3D, fd, S.minx, S.maxx, S.miny, S.maxy, S.maxz, BoxX, BoxY, BoxZ);
    BoxAverage(*S.RoughDensity1, *S.Density1, *S.RoughWallDensity1, *S.WallDensity1, *S.Filter3D, fd, S.minx, S.maxx, S.miny, S.maxy, S.maxz, BoxX, BoxY, BoxZ);
    BoxAverage(*S.RoughDensity2, *S.Density2, *S.RoughWallDensity2, *S.WallDensity2, *S.Filter3D, fd, S.minx, S.maxx, S.miny, S.maxy, S.maxz, BoxX, BoxY, BoxZ);
    BoxAverage(*S.RoughDensityShiftP, *S.DensityShiftP, *S.RoughWallDensityShiftP, *S.WallDensityShiftP, *S.Filter3D, fd, S.minx, S.maxx, S.miny, S.maxy, S.maxz, BoxX, BoxY, BoxZ);
    BoxAverage(*S.RoughDensity1ShiftP, *S.Density1ShiftP, *S.RoughWallDensity1ShiftP, *S.WallDensity1ShiftP, *S.Filter3D, fd, S.minx, S.maxx, S.miny, S.maxy, S.maxz, BoxX, BoxY, BoxZ);
    BoxAverage(*S.RoughDensity2ShiftP, *S.Density2ShiftP, *S.RoughWallDensity2ShiftP, *S.WallDensity2ShiftP, *S.Filter3D, fd, S.minx, S.maxx, S.miny, S.maxy, S.maxz, BoxX, BoxY, BoxZ);
    Height_Average(*S.Height, *S.RoughHeight, S.minx, S.maxx, S.miny, S.maxy);
    Smooth(*S.RoughHeight, *S.Height, *S.Filter, S.FilterDim, S.minx, S.maxx, S.miny, S.maxy);
    GetSurfaceNormal(*S.Normal, *S.Height, S.minx, S.maxx, S.miny, S.maxy);
}

/* HeightDensityUpdateFlag block, Simulation.cpp:302-306 */
void ref_update_height(void)
{
    GetHeight(*S.RoughDensity, *S.Height, *S.grid, S.old_cells, S.minx, S.maxx, S.miny, S.maxy, S.maxz);
    Height_Average(*S.Height, *S.RoughHeight, S.minx, S.maxx, S.miny, S.maxy);
    Smooth(*S.RoughHeight, *S.Height, *S.Filter, S.FilterDim, S.minx, S.maxx, S.miny, S.maxy);
    GetSurfaceNormal(*S.Normal, *S.Height, S.minx, S.maxx, S.miny, S.maxy);
}

/* UpdateEnvArrayMG_OxygenAcetate with n solves: the reference derives n from
 * UpdateTime (Multigrid.cpp:996), so UpdateTime is set for the call only. */
void ref_nutrient_update(int n)
{
    double save = UpdateTime;
    if (n > 0) UpdateTime = (n + 0.5) * 100.0 / (3600.0 * 740.0);
    UpdateEnvArrayMG_OxygenAcetate(S.Env, S.oldEnv, S.FieldAgar, S.oldFieldAgar, S.FieldWall, S.oldFieldWall, *S.DensityShiftP, *S.Density1ShiftP, *S.Density2ShiftP, *S.WallDensityShiftP, *S.WallDensity1ShiftP, *S.WallDensity2ShiftP, S.minx, S.maxx, S.miny, S.maxy, S.maxz, *S.Height, *S.insideColonyDen, *S.mg);
    UpdateTime = save;
}

/* UpdateEnvArray_OxygenAcetate (Nutrients.cpp:45-197), the legacy explicit
 * solver, for exactly `iters` iterations: minIter = maxIter = iters for the
 * call, so the convergence count (which also counts the points the
 * reference leaves undefined) cannot end it early.  Returns its count. */
int ref_legacy_env_update(int iters)
{
    const int save_min = minIter, save_max = maxIter;
    minIter = iters; maxIter = iters;
    int n = UpdateEnvArray_OxygenAcetate(S.Env, S.oldEnv, S.FieldAgar, S.oldFieldAgar, S.FieldWall, S.oldFieldWall, *S.DensityShiftP, *S.Density1ShiftP, *S.Density2ShiftP, *S.WallDensityShiftP, *S.WallDensity1ShiftP, *S.WallDensity2ShiftP, S.minx, S.maxx, S.miny, S.maxy, S.maxz, *S.Height, *S.insideColonyDen);
    minIter = save_min; maxIter = save_max;
    return n;
}

/* nutrientDepletionAgar_OxygenAcetate (Nutrients.cpp:857-896); returns its count */
int ref_legacy_depletion(void)
{
    return nutrientDepletionAgar_OxygenAcetate(S.FieldAgar, S.oldFieldAgar, S.FieldWall, S.oldFieldWall, *S.insideColonyDen);
}

/* Multigrid::solve with a chosen V-cycle count (solve() fixes 3). */
void ref_mg_solve(int vcycles, double dt)
{
    Multigrid& m = *S.mg;
    m.dt = dt;
    m.copyToMG(S.FieldAgar, S.FieldWall);
    m.setup();
    for (int i = 0; i < vcycles; i++) m.Vcycle(3, 100);
    m.reset();
    m.copyFromMG(S.FieldAgar, S.FieldWall, S.oldFieldAgar, S.oldFieldWall);
}

/* One iteration of the while loop (Simulation.cpp:256-430) minus output.
 * Returns the divisions done. */
int ref_loop_step(int* lineage)
{
    if (S.UpdateFlag) {
        S.UpdateFlag = false;
        ref_update_density();
        UpdateEnvArrayMG_OxygenAcetate(S.Env, S.oldEnv, S.FieldAgar, S.oldFieldAgar, S.FieldWall, S.oldFieldWall, *S.DensityShiftP, *S.Density1ShiftP, *S.Density2ShiftP, *S.WallDensityShiftP, *S.WallDensity1ShiftP, *S.WallDensity2ShiftP, S.minx, S.maxx, S.miny, S.maxy, S.maxz, *S.Height, *S.insideColonyDen, *S.mg);
        getNeighbours(S.old_cells, S.N, *S.grid, S.nbr, S.maxNeighbours);
    }
    if (S.HeightDensityUpdateFlag) {
        S.HeightDensityUpdateFlag = false;
        ref_update_height();
    }
    ref_move_grow(S.dt, nullptr, nullptr);
    int done = ref_divide(S.t, lineage);
    S.t += S.dt;
    S.OutFlag = (S.NextOutTime <= 0);
    S.NextOutTime = (S.OutFlag ? OutputTime : S.NextOutTime) - S.dt;
    S.UpdateFlag = (S.NextUpdateTime <= 0);
    S.NextUpdateTime = (S.UpdateFlag ? UpdateTime : S.NextUpdateTime) - S.dt;
    S.HeightDensityUpdateFlag = (S.HeightDensityNextUpdateTime <= 0);
    S.HeightDensityNextUpdateTime = (S.HeightDensityUpdateFlag ? S.HeightDensityUpdateTime : S.HeightDensityNextUpdateTime) - S.dt;
    return done;
}

/* mean_stress for every cell in id order, as on an output step
 * (Simulation.cpp:320-326); returns the rand() draws made */
long long ref_mean_stress(double* stress, double* fnet)
{
    long long r0 = g_rand_calls;
    Tensor T;
    DoubleCoord F;
    for (int i = 0; i < S.N; i++) {
        mean_stress(S.old_cells[i], S.old_cells, S.nbr[i], *S.grid, *S.Wall, *S.Height, *S.Normal, T, F);
        stress[5 * i] = T.xx; stress[5 * i + 1] = T.yy; stress[5 * i + 2] = T.zz; stress[5 * i + 3] = T.rr; stress[5 * i + 4] = T.tt;
        if (fnet) { fnet[3 * i] = F.x; fnet[3 * i + 1] = F.y; fnet[3 * i + 2] = F.z; }
    }
    return g_rand_calls - r0;
}

/* ---- output steps, through the reference's own writers -------------------- */
static OutputFiles g_files;

/* The files CreateOutputFiles opens (InputOutput.cpp:42-271), opened here.
 * The reference builds each name with sprintf(name, "%s/%d", name, id),
 * whose source and destination overlap; with this machine's glibc that
 * yields "/<id>" and every file of the step lands on "/<id>.txt", so the
 * harness never calls it.  The names below are the intended
 * <dir>/<Name>/<id>.txt; the writers that fill the files are the
 * reference's own. */
static int open_step_files(const char* dir, int id, bool append, OutputFiles& F)
{
    mkdir(dir, S_IRWXU | S_IRWXG | S_IROTH | S_IXOTH);
    const char* names[17] = {"Cells", "Restart", "RoughDensity", "RoughDensity1", "RoughDensity2", "Density",
                             "Density1", "Density2", "WallDensity", "WallDensity1", "WallDensity2", "RoughHeight",
                             "Height", "Normal", "Environment", "AgarField", "WallField"};
    FILE** slots[17] = {&F.cells, &F.restart, &F.roughDensity, &F.roughDensity1, &F.roughDensity2, &F.density,
                        &F.density1, &F.density2, &F.walldensity, &F.walldensity1, &F.walldensity2, &F.roughheight,
                        &F.height, &F.normal, &F.env, &F.aga, &F.wal};
    char path[1024];
    for (int k = 0; k < 17; k++) {
        snprintf(path, sizeof path, "%s/%s", dir, names[k]);
        mkdir(path, S_IRWXU | S_IRWXG | S_IROTH | S_IXOTH);
        snprintf(path, sizeof path, "%s/%s/%d.txt", dir, names[k], id);
        *slots[k] = fopen(path, (k == 0 && append) ? "a" : "w");
        if (!*slots[k]) {
            for (int j = 0; j < k; j++) fclose(*slots[j]);
            return -1;
        }
    }
    return 0;
}

/* First half of an output step, Simulation.cpp:316-327: CreateOutputFiles
 * and one Output line per cell with mean_stress's tensor, at time t.
 * Returns the rand() draws made, or -1 when the files cannot be opened. */
long long ref_output_cells(const char* dir, int id, double t, int append)
{
    if (open_step_files(dir, id, append != 0, g_files)) return -1;
    long long r0 = g_rand_calls;
    Tensor T;
    DoubleCoord F;
    for (int i = 0; i < S.N; i++) {
        mean_stress(S.old_cells[i], S.old_cells, S.nbr[i], *S.grid, *S.Wall, *S.Height, *S.Normal, T, F);
        Output(g_files.cells, i, t, S.old_cells[i], T);
    }
    return g_rand_calls - r0;
}

/* The same first half with given stress columns (T.xx, T.yy, T.zz from
 * `stress`, `stride` doubles per cell) in place of mean_stress: the
 * reference's Output on arbitrary values, for format checks. */
int ref_output_cells_given(const char* dir, int id, double t, int append, const double* stress, int stride)
{
    if (open_step_files(dir, id, append != 0, g_files)) return -1;
    for (int i = 0; i < S.N; i++) {
        Tensor T(stress[(size_t)i * stride], stress[(size_t)i * stride + 1], stress[(size_t)i * stride + 2], 0.0, 0.0);
        Output(g_files.cells, i, t, S.old_cells[i], T);
    }
    return 0;
}

/* overwrite new_cells (the array SaveCells writes on an output step) */
int ref_set_new_cells(const bcg_cell* cells, int n)
{
    if (n > maxCells) return BCG_E_ARG;
    memcpy(S.new_cells, cells, sizeof(Cell) * (size_t)n);
    return 0;
}

/* Second half, Simulation.cpp:342-374 (new_cells as MoveCell/GrowCell left
 * them), then CloseOutputFiles. */
void ref_output_fields(double t, double dt)
{
    SaveCells(g_files.restart, S.new_cells, S.N, t, dt);
    S.DensityShiftP->Output(g_files.density, 1);
    S.Env->Output(g_files.env, 1);
    for (int level = 0; level < maxLevelsMG; level++) {
        S.FieldAgar[level]->Append(g_files.aga, 1);
        S.FieldWall[level]->Append(g_files.wal);
    }
    CloseOutputFiles(g_files);
}

/* The initial block's output, Simulation.cpp:185-244 (step 0). */
void ref_output_initial(const char* dir, double t, int append)
{
    OutputFiles F;
    if (open_step_files(dir, 0, append != 0, F)) return;
    S.DensityShiftP->Output(F.density, 1);
    S.Env->Output(F.env, 1);
    for (int level = 0; level < maxLevelsMG; level++) {
        S.FieldAgar[level]->Append(F.aga, 1);
        S.FieldWall[level]->Append(F.wal);
    }
    DoubleCoord Fnet;
    for (int i = 0; i < S.N; i++) {
        IntCoord XYAddress = S.grid->GetXY(S.grid->GetAddress(average(S.old_cells[i].Position)));
        DoubleCoord T(0, 0, 0);
        F_surf_tension(S.old_cells[i], *S.grid, XYAddress, *S.Height, *S.Normal, Fnet, T);
        Output(F.cells, i, t, S.old_cells[i], Fnet);
    }
    fflush(F.cells);
    CloseOutputFiles(F);
}

/* One iteration of the while loop with its output block
 * (Simulation.cpp:256-431): writes the step's files under `dir` when
 * OutFlag is set.  Returns the divisions done. */
int ref_loop_step_out(const char* dir, int* lineage)
{
    if (S.UpdateFlag) {
        S.UpdateFlag = false;
        ref_update_density();
        UpdateEnvArrayMG_OxygenAcetate(S.Env, S.oldEnv, S.FieldAgar, S.oldFieldAgar, S.FieldWall, S.oldFieldWall, *S.DensityShiftP, *S.Density1ShiftP, *S.Density2ShiftP, *S.WallDensityShiftP, *S.WallDensity1ShiftP, *S.WallDensity2ShiftP, S.minx, S.maxx, S.miny, S.maxy, S.maxz, *S.Height, *S.insideColonyDen, *S.mg);
        getNeighbours(S.old_cells, S.N, *S.grid, S.nbr, S.maxNeighbours);
    }
    if (S.HeightDensityUpdateFlag) {
        S.HeightDensityUpdateFlag = false;
        ref_update_height();
    }
    const bool out = S.OutFlag;
    if (out) ref_output_cells(dir, S.koutput++, S.t, 0);
    ref_move_grow(S.dt, nullptr, nullptr);
    if (out) {
        S.OutFlag = false;
        ref_output_fields(S.t, S.dt);
    }
    int done = ref_divide(S.t, lineage);
    S.t += S.dt;
    S.OutFlag = (S.NextOutTime <= 0);
    S.NextOutTime = (S.OutFlag ? OutputTime : S.NextOutTime) - S.dt;
    S.UpdateFlag = (S.NextUpdateTime <= 0);
    S.NextUpdateTime = (S.UpdateFlag ? UpdateTime : S.NextUpdateTime) - S.dt;
    S.HeightDensityUpdateFlag = (S.HeightDensityNextUpdateTime <= 0);
    S.HeightDensityNextUpdateTime = (S.HeightDensityUpdateFlag ? S.HeightDensityUpdateTime : S.HeightDensityNextUpdateTime) - S.dt;
    return done;
}

/* F_surf_tension's force on every cell, as the initial block computes it
 * (Simulation.cpp:231-236) */
void ref_surface_forces(double* out)
{
    for (int i = 0; i < S.N; i++) {
        IntCoord XYAddress = S.grid->GetXY(S.grid->GetAddress(average(S.old_cells[i].Position)));
        DoubleCoord T(0, 0, 0), F(0, 0, 0);
        F_surf_tension(S.old_cells[i], *S.grid, XYAddress, *S.Height, *S.Normal, F, T);
        out[3 * i] = F.x; out[3 * i + 1] = F.y; out[3 * i + 2] = F.z;
    }
}

/* the moved, grown cells of the last ref_move_grow (new_cells) */
int ref_get_new_cells(bcg_cell* out, int cap)
{
    int n = S.N < cap ? S.N : cap;
    memcpy(out, S.new_cells, sizeof(Cell) * (size_t)n);
    return S.N;
}

double ref_time(void) { return S.t; }
void ref_bbox(int* mnx, int* mxx, int* mxz) { *mnx = S.minx; *mxx = S.maxx; *mxz = S.maxz; }
void ref_set_bbox(int mnx, int mxx, int mxz) { S.minx = mnx; S.maxx = mxx; S.maxz = mxz; }

/* ---- field access (ids from bcg_field_id) --------------------------------- */
static int mg_dims(int level, int* nx, int* nz)
{
    int d = 1 << level, d0 = 1 << maxLevelsMG;
    *nx = std::min(BoxX, BoxX * d0 / d / 2);
    *nz = std::min(BoxZAgar, BoxZAgar * d0 / d / 2);
    return 0;
}

long ref_field(int field, int level, double* buf, long n, int write)
{
    const int X = BoxX, Z = BoxZ, XH = BoxX * refinementGridHeight, ZA = BoxZAgar;
    long cnt = 0;
#define A2(arr, len, expr_get, expr_set) \
    do { cnt = (len); if (buf && n >= cnt) for (long i = 0; i < cnt; i++) { if (write) { expr_set; } else { buf[i] = (expr_get); } } } while (0)
    switch (field) {
    case BCG_F_HEIGHT: A2(0, XH, S.Height->Get(i, 0), S.Height->Set(i, 0, buf[i])); break;
    case BCG_F_NORMAL_X: A2(0, XH, S.Normal->At(i, 0).x, S.Normal->At(i, 0).x = buf[i]); break;
    case BCG_F_NORMAL_Z: A2(0, XH, S.Normal->At(i, 0).z, S.Normal->At(i, 0).z = buf[i]); break;
    case BCG_F_WALL: A2(0, X, S.Wall->Get(i, 0), S.Wall->Set(i, 0, buf[i])); break;
    case BCG_F_DENSITY_SHIFT: A2(0, (long)X * Z, S.DensityShiftP->Get(i / Z, 0, i % Z), S.DensityShiftP->Set(i / Z, 0, i % Z, buf[i])); break;
    case BCG_F_WALL_DENSITY_SHIFT: A2(0, X, S.WallDensityShiftP->Get(i, 0), S.WallDensityShiftP->Set(i, 0, buf[i])); break;
    case BCG_F_INSIDE: A2(0, (long)X * Z, S.insideColonyDen->Get(i / Z, 0, i % Z), S.insideColonyDen->Set(i / Z, 0, i % Z, buf[i])); break;
    case BCG_F_DENSITY: A2(0, (long)X * Z, S.Density->Get(i / Z, 0, i % Z), S.Density->Set(i / Z, 0, i % Z, buf[i])); break;
    case BCG_F_ROUGH_DENSITY: A2(0, (long)X * Z, S.RoughDensity->Get(i / Z, 0, i % Z), S.RoughDensity->Set(i / Z, 0, i % Z, buf[i])); break;
#define ENVF(ID, ARR, M) case ID: A2(0, (long)X * Z, S.ARR->At(i / Z, 0, i % Z).M, S.ARR->At(i / Z, 0, i % Z).M = buf[i]); break;
    ENVF(BCG_F_ENV_CARBON, Env, Carbon)
    ENVF(BCG_F_ENV_WASTE, Env, Waste)
    ENVF(BCG_F_ENV_OXYGEN, Env, Oxygen)
    ENVF(BCG_F_ENV_ACETATE, Env, Acetate)
    ENVF(BCG_F_ENV_GROWTH1, Env, GrowthRate1)
    ENVF(BCG_F_ENV_GROWTH2, Env, GrowthRate2)
    ENVF(BCG_F_ENV_PH, Env, pH)
    ENVF(BCG_F_ENV_HYDROX, Env, Hydrox)
    ENVF(BCG_F_ENV_ACETIC, Env, Acetic)
    ENVF(BCG_F_ENV_BUFFER, Env, Buffer)
    ENVF(BCG_F_ENV_GR_CAR_AER, Env, GrCarAer)
    ENVF(BCG_F_ENV_GR_CAR_ANA, Env, GrCarAna)
    ENVF(BCG_F_ENV_GR_ACE_AER, Env, GrAceAer)
    ENVF(BCG_F_ENV_Q_CAR_MNT, Env, qCarmnt)
    ENVF(BCG_F_ENV_Q_ACE_MNT, Env, qAcemnt)
    ENVF(BCG_F_ENV_P_ACE_MNT, Env, pAcemnt)
    ENVF(BCG_F_ENV_Q_OXY_MNT, Env, qOxymnt)
    ENVF(BCG_F_OLDENV_CARBON, oldEnv, Carbon)
    ENVF(BCG_F_OLDENV_WASTE, oldEnv, Waste)
    ENVF(BCG_F_OLDENV_OXYGEN, oldEnv, Oxygen)
    ENVF(BCG_F_OLDENV_ACETATE, oldEnv, Acetate)
#define WALF(ID, ARR, M) case ID: if (level < 0 || level >= maxLevelsMG) return -1; A2(0, X, S.ARR[level]->At(i, 0).M, S.ARR[level]->At(i, 0).M = buf[i]); break;
    WALF(BCG_F_WALLF_CARBON, FieldWall, CarbonAgar)
    WALF(BCG_F_WALLF_WASTE, FieldWall, WasteAgar)
    WALF(BCG_F_WALLF_OXYGEN, FieldWall, OxygenAgar)
    WALF(BCG_F_WALLF_ACETATE, FieldWall, AcetateAgar)
    WALF(BCG_F_OLDWALLF_CARBON, oldFieldWall, CarbonAgar)
    WALF(BCG_F_OLDWALLF_WASTE, oldFieldWall, WasteAgar)
    WALF(BCG_F_OLDWALLF_OXYGEN, oldFieldWall, OxygenAgar)
    WALF(BCG_F_OLDWALLF_ACETATE, oldFieldWall, AcetateAgar)
#define AGAF(ID, M) case ID: if (level < 0 || level >= maxLevelsMG) return -1; A2(0, (long)X * ZA, S.FieldAgar[level]->At(i / ZA, 0, i % ZA).M, S.FieldAgar[level]->At(i / ZA, 0, i % ZA).M = buf[i]); break;
    AGAF(BCG_F_AGARF_CARBON, CarbonAgar)
    AGAF(BCG_F_AGARF_OXYGEN, OxygenAgar)
    AGAF(BCG_F_AGARF_ACETATE, AcetateAgar)
#define MGF(ID, ARR, M) case ID: { if (level < 0 || level >= S.mg->agarMGLevels) return -1; int nx, nz; mg_dims(level, &nx, &nz); long NZ = nz + 1; \
        A2(0, (long)(nx + 1) * NZ, S.mg->ARR[level]->At(i / NZ, 0, i % NZ).M, S.mg->ARR[level]->At(i / NZ, 0, i % NZ).M = buf[i]); } break;
    MGF(BCG_F_MG_SOL_CARBON, Aga, CarbonAgar)
    MGF(BCG_F_MG_SOL_OXYGEN, Aga, OxygenAgar)
    MGF(BCG_F_MG_SOL_ACETATE, Aga, AcetateAgar)
    MGF(BCG_F_MG_RES_CARBON, AgaRes, CarbonAgar)
    MGF(BCG_F_MG_RES_OXYGEN, AgaRes, OxygenAgar)
    MGF(BCG_F_MG_RES_ACETATE, AgaRes, AcetateAgar)
    MGF(BCG_F_MG_ERR_CARBON, AgaErr, CarbonAgar)
    MGF(BCG_F_MG_ERR_OXYGEN, AgaErr, OxygenAgar)
    MGF(BCG_F_MG_ERR_ACETATE, AgaErr, AcetateAgar)
    default: return -1;
    }
    return cnt;
}

} // extern "C"
