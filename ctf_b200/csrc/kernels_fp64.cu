// FP64 step kernels.  This translation unit is compiled with --fmad=false so that every
// multiply and add rounds separately, as in the reference's x86-64 build: the plain FP64
// path then reproduces the reference's arithmetic operation for operation.
// the flux sweep at 3 resident blocks of 128 threads per SM (chosen by a sweep of 1-4)
#ifdef MGPU_FLUX_MINB_OVERRIDE
#define MGPU_FLUX_MINB MGPU_FLUX_MINB_OVERRIDE
#else
#define MGPU_FLUX_MINB 3
#endif
#ifdef MGPU_C2P_MINB_OVERRIDE
#define MGPU_C2P_MINB MGPU_C2P_MINB_OVERRIDE
#endif
#ifdef MGPU_TC_CTAS_OVERRIDE
#define MGPU_TC_CTAS_PER_SM MGPU_TC_CTAS_OVERRIDE
#endif
#include "c2p_mlp.cuh"
#include "rmhd_launch.cuh"
MGPU_DEFINE_PRECISION(fp64, double)
