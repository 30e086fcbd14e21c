/* entry points whose kernels are not built yet */
#include "ctx.cuh"
