// Device reductions behind Mara.measure.* (Mara/mara.cpp:1954-2230): one pass over the
// interior zones of the measured primitive array computes every per-zone quantity the eight
// measures sum or take the extreme of, with each per-zone value in the reference's
// operation order (this unit is compiled with --fmad=false, like the FP64 step kernels).
// Per-block partial sums are written in a fixed order and summed on the host, so a result
// depends only on the launch shape, not on timing.
#include <cuda_runtime.h>
#include <math.h>

#include "measures.h"
#include "c2p_mlp.cuh"   // rmhd_physics.cuh with the learned-guess function it declares

namespace mgpu {
namespace {

constexpr int MEAS_THREADS = 256;

// Temperature in MeV of AdiabaticEos::TemperatureMeV (Mara/eos.cpp:39-49): the unit
// conversions come from the host (erg_cc = units->ErgPerCubicCentimeter(), gcc =
// units->GramsPerCubicCentimeter(), mp_kb = ProtonMass() / BoltzmannConstant()).
__device__ __forceinline__ double temperature_mev(const MeasureUnits &u, double rho, double P)
{
  P /= u.erg_cc;
  rho /= u.gcc;
  const double T_Kelvin = (P / rho) * u.mp_kb;
  return T_Kelvin * 8.621738e-11;   // Kelvin_to_MeV, Mara/eos.cpp:4
}

template <class T>
__global__ void __launch_bounds__(MEAS_THREADS) k_measures(Grid g, const T *PA, double gamma, MeasureUnits units,
                                                           double *partial)
{
  double acc[MEAS_SUMS];
#pragma unroll
  for (int i = 0; i < MEAS_SUMS; ++i) acc[i] = 0.0;
  double tmax = 0.0, bmax = 0.0, msmax = 0.0, mamin = 1e20;
  for (long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x; t < g.ninterior;
       t += (long long) gridDim.x * blockDim.x) {
    int i, j, k;
    interior_coords(g, t, i, j, k);
    const long long z = ((long long) i * g.G[1] + j) * g.G[2] + k;
    double P0[8], U0[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) P0[q] = double(PA[q * g.cs + z]);
    prim_to_cons(gamma, P0, U0);
    // mean_cons, mean_prim
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      acc[MEAS_CONS + q] += U0[q];
      acc[MEAS_PRIM + q] += P0[q];
    }
    const double v2 = P0[vx] * P0[vx] + P0[vy] * P0[vy] + P0[vz] * P0[vz];
    const double T0 = P0[pre];                  // AdiabaticEos::Temperature_p
    const double u0 = T0 / (gamma - 1);         // AdiabaticEos::Internal
    // mean_energies (relativistic branch)
    {
      const double rhoh = P0[rho] + u0 + P0[pre];
      const double W0 = 1.0 / sqrt(1.0 - v2);
      const double e_f = rhoh * W0 * W0 - P0[pre] - U0[ddd];
      const double e_m = U0[tau] - e_f;
      acc[MEAS_ENERGY + 0] += e_m;
      acc[MEAS_ENERGY + 1] += P0[rho] * W0 * (W0 - 1);
      acc[MEAS_ENERGY + 2] += W0 * u0;
      acc[MEAS_ENERGY + 3] += U0[tau];
    }
    // mean_velocity
    acc[MEAS_VEL + 0] += 1.0 / sqrt(1.0 - v2);
    acc[MEAS_VEL + 1] += fabs(P0[vx]);
    acc[MEAS_VEL + 2] += fabs(P0[vy]);
    acc[MEAS_VEL + 3] += fabs(P0[vz]);
    // mean_max_temperature
    {
      const double Tm = temperature_mev(units, P0[rho], P0[pre]);
      acc[MEAS_T] += Tm;
      if (Tm > tmax) tmax = Tm;
    }
    // mean_max_sonic_mach (relativistic branch; AdiabaticEos::SoundSpeed2Sr)
    {
      const double rhoh = P0[rho] + T0 / (gamma - 1) + T0;
      const double cs2 = gamma * T0 / rhoh;
      const double M0 = sqrt((v2 / (1 - v2)) / (cs2 / (1 - cs2)));
      acc[MEAS_MS] += M0;
      if (M0 > msmax) msmax = M0;
    }
    // mean_min_alfvenic_mach
    {
      const double B2 = P0[Bx] * P0[Bx] + P0[By] * P0[By] + P0[Bz] * P0[Bz];
      const double rhoh = P0[rho] + u0 + P0[pre];
      const double va2 = B2 / (B2 + rhoh);
      const double M0 = sqrt((v2 / (1 - v2)) / (va2 / (1 - va2)));
      acc[MEAS_MA] += M0;
      if (M0 < mamin) mamin = M0;
    }
    // mean_max_magnetic_field
    {
      const double B0 = sqrt(P0[Bx] * P0[Bx] + P0[By] * P0[By] + P0[Bz] * P0[Bz]);
      acc[MEAS_B] += B0;
      if (B0 > bmax) bmax = B0;
    }
  }
  // block reduction in a fixed order: one shared column per quantity
  __shared__ double sh[MEAS_THREADS];
  for (int qi = 0; qi < MEAS_FIELDS; ++qi) {
    double v;
    if (qi < MEAS_SUMS) v = acc[qi];
    else if (qi == MEAS_TMAX) v = tmax;
    else if (qi == MEAS_BMAX) v = bmax;
    else if (qi == MEAS_MSMAX) v = msmax;
    else v = mamin;
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) {
        const double a = sh[threadIdx.x], b = sh[threadIdx.x + o];
        double r;
        if (qi < MEAS_SUMS) r = a + b;
        else if (qi == MEAS_MAMIN) r = b < a ? b : a;
        else r = b > a ? b : a;
        sh[threadIdx.x] = r;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) partial[(long long) blockIdx.x * MEAS_FIELDS + qi] = sh[0];
    __syncthreads();
  }
}

}  // namespace

cudaError_t measures_launch(const Grid &g, const void *PA, bool fp32, double gamma, const MeasureUnits &units,
                            double *partial, cudaStream_t st)
{
  if (fp32)
    k_measures<float><<<MEAS_BLOCKS, MEAS_THREADS, 0, st>>>(g, (const float *) PA, gamma, units, partial);
  else
    k_measures<double><<<MEAS_BLOCKS, MEAS_THREADS, 0, st>>>(g, (const double *) PA, gamma, units, partial);
  return cudaGetLastError();
}

}  // namespace mgpu
