// FP32-bulk step kernels: reconstruction, Riemann fluxes and the RK combine of the five
// hydrodynamic components in FP32; the magnetic field, its constrained-transport update, the
// c2p Newton polish and the dt reduction in FP64.
#include "c2p_mlp.cuh"
#include "rmhd_launch.cuh"
MGPU_DEFINE_PRECISION(fp32, float)
