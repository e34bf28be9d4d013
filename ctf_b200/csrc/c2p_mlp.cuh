// Learned c2p initial guess: device side of the packed network (defined per translation unit
// because the step kernels are compiled without relocatable device code).
#pragma once
#include "rmhd_physics.cuh"
#include "c2p_mlp_net.cuh"
