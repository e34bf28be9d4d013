// The one-pass reduction behind Mara.measure.* (measures.cu) and the layout of its per-block
// partials: MEAS_FIELDS doubles per block, sums first, then the extremes.
#pragma once
#include <cuda_runtime.h>

#include "rmhd_types.cuh"

namespace mgpu {

enum MeasureField {
  MEAS_CONS = 0,        // 8 sums of P->U (mean_cons)
  MEAS_PRIM = 8,        // 8 sums of the primitives (mean_prim)
  MEAS_ENERGY = 16,     // magnetic, kinetic, internal, total (mean_energies)
  MEAS_VEL = 20,        // W, |vx|, |vy|, |vz| (mean_velocity)
  MEAS_T = 24,          // temperature in MeV (mean_max_temperature)
  MEAS_B = 25,          // |B| (mean_max_magnetic_field)
  MEAS_MS = 26,         // sonic Mach number (mean_max_sonic_mach)
  MEAS_MA = 27,         // Alfvenic Mach number (mean_min_alfvenic_mach)
  MEAS_SUMS = 28,
  MEAS_TMAX = 28, MEAS_BMAX = 29, MEAS_MSMAX = 30, MEAS_MAMIN = 31,
  MEAS_FIELDS = 32
};

constexpr int MEAS_BLOCKS = 592;   // 148 SMs x 4

// Unit conversions of the measures (PhysicalUnits, Mara/units.cpp), computed on the host.
struct MeasureUnits {
  double erg_cc;    // ErgPerCubicCentimeter()
  double gcc;       // GramsPerCubicCentimeter()
  double mp_kb;     // ProtonMass() / BoltzmannConstant()
  double gauss;     // Gauss()
};

// Enqueues the reduction over the interior zones of an 8-component primitive array (float
// when fp32, else double) into partial[MEAS_BLOCKS * MEAS_FIELDS].
cudaError_t measures_launch(const Grid &g, const void *PA, bool fp32, double gamma, const MeasureUnits &units,
                            double *partial, cudaStream_t st);

}  // namespace mgpu
