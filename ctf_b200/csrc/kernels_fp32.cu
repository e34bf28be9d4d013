// FP32-bulk step kernels: reconstruction, Riemann fluxes and the RK combine of the five
// hydrodynamic components in FP32; the magnetic field, its constrained-transport update, the
// c2p Newton polish and the dt reduction in FP64.
// the flux sweep at 4 resident blocks of 128 threads per SM (chosen by a sweep of 1-4)
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
#include "rmhd_launch.cuh"
MGPU_DEFINE_PRECISION(fp32, float)
