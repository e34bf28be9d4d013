// FP64 step kernels.  This translation unit is compiled with --fmad=false so that every
// multiply and add rounds separately, as in the reference's x86-64 build: the plain FP64
// path then reproduces the reference's arithmetic operation for operation.
#include "c2p_mlp.cuh"
#include "rmhd_launch.cuh"
MGPU_DEFINE_PRECISION(fp64, double)
