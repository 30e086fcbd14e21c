/* entry points whose kernels live in later translation units */
#include "ctx.cuh"
extern "C" int bcg_update_density(bcg_ctx* c) { return c ? BCG_E_UNSUPPORTED : BCG_E_ARG; }
extern "C" int bcg_update_height(bcg_ctx* c) { return c ? BCG_E_UNSUPPORTED : BCG_E_ARG; }
extern "C" int bcg_initial_density(bcg_ctx* c) { return c ? BCG_E_UNSUPPORTED : BCG_E_ARG; }
extern "C" int bcg_nutrient_update(bcg_ctx* c, int n, int s) { (void)n; (void)s; return c ? BCG_E_UNSUPPORTED : BCG_E_ARG; }
extern "C" int bcg_mg_solve(bcg_ctx* c, int v) { (void)v; return c ? BCG_E_UNSUPPORTED : BCG_E_ARG; }
extern "C" int bcg_colony_sweeps(bcg_ctx* c, int s, int c0) { (void)s; (void)c0; return c ? BCG_E_UNSUPPORTED : BCG_E_ARG; }
extern "C" int bcg_mg_solve_tol(bcg_ctx* c, double t, int p, int m, int* it, double* r) { (void)t; (void)p; (void)m; (void)it; (void)r; return c ? BCG_E_UNSUPPORTED : BCG_E_ARG; }
