/* entry points whose kernels are not built yet */
#include "ctx.cuh"
extern "C" int bcg_mg_solve_tol(bcg_ctx* c, double t, int p, int m, int* it, double* r) { (void)t; (void)p; (void)m; (void)it; (void)r; return c ? BCG_E_UNSUPPORTED : BCG_E_ARG; }
