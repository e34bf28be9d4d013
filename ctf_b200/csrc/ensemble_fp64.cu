// FP64 ensemble kernels, compiled like kernels_fp64.cu (--fmad=false): each box of an
// ensemble advances with the single-box path's arithmetic.
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
#include "rmhd_ensemble.cuh"
MGPU_DEFINE_ENSEMBLE(fp64, double)
