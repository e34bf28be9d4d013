// FP32-bulk ensemble kernels, compiled like kernels_fp32.cu (--use_fast_math).
#ifdef MGPU_FLUX_MINB_OVERRIDE
#define MGPU_FLUX_MINB MGPU_FLUX_MINB_OVERRIDE
#else
#define MGPU_FLUX_MINB 4
#endif
#ifdef MGPU_C2P_MINB_OVERRIDE
#define MGPU_C2P_MINB MGPU_C2P_MINB_OVERRIDE
#endif
#ifdef MGPU_TC_CTAS_OVERRIDE
#define MGPU_TC_CTAS_PER_SM MGPU_TC_CTAS_OVERRIDE
#endif
#include "c2p_mlp.cuh"
#include "rmhd_ensemble.cuh"
MGPU_DEFINE_ENSEMBLE(fp32, float)
