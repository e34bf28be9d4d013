// Function-level entry points: the FP64 device functions of the advance, applied to n
// independent states, so that each can be compared with the reference's function of the same
// name state by state (the parity suite's per-function layer; whole steps are compared
// through mgpu_advance).  Compiled with --fmad=false like the FP64 step kernels, so the
// arithmetic is the one those kernels run.
//
//   mgpu_probe_prim_to_cons   AdiabaticIdealRmhd::PrimToCons        Mara/rmhd.cpp:177-207
//   mgpu_probe_c2p            AdiabaticIdealRmhd::ConsToPrim ladder Mara/rmhd.cpp:103-176, and
//                             rmhd_c2p_solve_anton2dzw / _noble1dw  Mara/rmhd-c2p.c:182-326
//                             from rmhd_c2p_estimate_from_cons or
//                             rmhd_c2p_set_starting_prim            Mara/rmhd-c2p.c:96-119
//   mgpu_probe_flux           FluxAndEigenvalues                    Mara/rmhd.cpp:208-310
//   mgpu_probe_riemann        Hll/Hllc/HlldRmhdRiemannSolver::IntercellFlux at s = 0
//                             (Mara/riemann_hll.cpp:19-64, riemann_hllc-rmhd.cpp:26-178,
//                             riemann_hlld-rmhd.cpp:143-277), with RiemannSolver::MaxLambda
//   mgpu_probe_reconstruct    reconstruct: PLM minmod / WENO5 FV    Mara/weno.c:58-154
#include <cuda_runtime.h>

#include "../../include/mara_gpu.h"
#include "c2p_mlp.cuh"   // rmhd_physics.cuh with the learned-guess function it declares

namespace mgpu {
namespace {

constexpr int PROBE_BLOCK = 128;

inline int blocks_for(long long n) { return (int) ((n + PROBE_BLOCK - 1) / PROBE_BLOCK); }

__global__ void k_probe_p2c(double gamma, const double *P, long long n, double *U, int *err)
{
  const long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double p[8], u[8];
  for (int q = 0; q < 8; ++q) p[q] = P[8 * i + q];
  err[i] = prim_to_cons(gamma, p, u);
  for (int q = 0; q < 8; ++q) U[8 * i + q] = u[q];
}

// mode 0: the ladder, previous primitives = guess; P = guess on failure (written only on
// success, as the reference leaves its output untouched).  mode 1 + 2 * solver + start:
// one solver (0 Anton 2D, 1 Noble 1D) from the estimate (start 0) or from the guess (1).
__global__ void k_probe_c2p(int mode, double gamma, double pfloor, const double *U, const double *G, long long n,
                            double *P, int *err, int *iters)
{
  const long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double u[8], p[8];
  for (int q = 0; q < 8; ++q) {
    u[q] = U[8 * i + q];
    p[q] = G[8 * i + q];
  }
  int e, it = 0;
  if (mode == 0) {
    PhysParams pp{};
    pp.gamma = gamma;
    pp.pfloor = pfloor;
    C2PTally tally{0, 0};
    e = cons_to_prim<false, 2>(pp, u, p, &tally);
    it = tally.iters;
  } else {
    const int solver = (mode - 1) >> 1, start = (mode - 1) & 1;
    C2PState s;
    s.gamma = gamma;
    s.gamf = (gamma - 1.0) / gamma;
    s.pfloor = pfloor;
    c2p_new_state(s, u);
    double Z, W;
    if (start == 0) c2p_estimate(s, Z, W);
    else c2p_from_prim(s, p, Z, W);
    double out[8];
    for (int q = 0; q < 8; ++q) out[q] = 0.0;
    e = solver == 0 ? c2p_anton2dzw(s, Z, W, out, it) : c2p_noble1dw(s, Z, out, it);
    for (int q = 0; q < 8; ++q) p[q] = out[q];
  }
  for (int q = 0; q < 8; ++q) P[8 * i + q] = p[q];
  err[i] = e;
  iters[i] = it;
}

__global__ void k_probe_flux(double gamma, int dim, const double *P, long long n, double *F, double *lam)
{
  const long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double p[8], u[8], f[8], ap, am;
  for (int q = 0; q < 8; ++q) p[q] = P[8 * i + q];
  prim_to_cons(gamma, p, u);
  flux_and_eigenvalues(gamma, u, p, f, ap, am, dim);
  for (int q = 0; q < 8; ++q) F[8 * i + q] = f[q];
  lam[2 * i] = ap;
  lam[2 * i + 1] = am;
}

template <int dim>
__device__ int riemann_dim(int solver, const PhysParams &pp, const double *pl, const double *pr, double *f,
                           double &ml, int &used_hllc)
{
  used_hllc = 0;
  if (solver == RIEMANN_HLL) return riemann_hll<double, dim>(pp.gamma, pl, pr, f, ml);
  if (solver == RIEMANN_HLLC) return riemann_hllc<double, dim>(pp.gamma, pl, pr, f, ml);
  C2PTally t{0, 0};
  return riemann_hlld<double, dim>(pp, pl, pr, f, ml, used_hllc, &t);
}

// dims: per-face direction (1-3) when not null, else `dim` for every face.
__global__ void k_probe_riemann(int solver, int dim, const int *dims, double gamma, double pfloor, const double *Pl,
                                const double *Pr, long long n, double *F, int *err, double *max_lambda,
                                int *used_hllc)
{
  const long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  PhysParams pp{};
  pp.gamma = gamma;
  pp.pfloor = pfloor;
  pp.riemann = solver;
  double pl[8], pr[8], f[8];
  for (int q = 0; q < 8; ++q) {
    pl[q] = Pl[8 * i + q];
    pr[q] = Pr[8 * i + q];
    f[q] = 0.0;
  }
  double ml = 0.0;
  int hllc = 0, e;
  const int d = dims ? dims[i] : dim;
  if (d == 1) e = riemann_dim<1>(solver, pp, pl, pr, f, ml, hllc);
  else if (d == 2) e = riemann_dim<2>(solver, pp, pl, pr, f, ml, hllc);
  else e = riemann_dim<3>(solver, pp, pl, pr, f, ml, hllc);
  for (int q = 0; q < 8; ++q) F[8 * i + q] = f[q];
  err[i] = e;
  max_lambda[i] = ml;
  if (used_hllc) used_hllc[i] = hllc;
}

// op 0 / 1: PLM face value to the left / right of the centre of V[i, 1..3]; op 4 / 5: WENO5
// centre-to-right / centre-to-left on V[i, 0..4] (the reference's reconstruct operations).
__global__ void k_probe_recon(int op, double theta, int is_mode, double sz10A, const double *V, long long n,
                              double *out)
{
  const long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double *v = V + 5 * i;
  double r = 0.0;
  if (op == 0) r = plm(theta, v[1], v[2], v[3], -1.0);
  else if (op == 1) r = plm(theta, v[1], v[2], v[3], +1.0);
  else if (op == 4) r = weno5(is_mode, sz10A, v[0], v[1], v[2], v[3], v[4], true);
  else if (op == 5) r = weno5(is_mode, sz10A, v[0], v[1], v[2], v[3], v[4], false);
  out[i] = r;
}

int finish()
{
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  return e == cudaSuccess ? MGPU_OK : MGPU_ERR_CUDA;
}

}  // namespace
}  // namespace mgpu

using namespace mgpu;

extern "C" {

int mgpu_probe_prim_to_cons(double gamma, const double *dev_P, long long n, double *dev_U, int *dev_err)
{
  if (n < 0 || (n && (!dev_P || !dev_U || !dev_err))) return MGPU_ERR_ARG;
  if (n) k_probe_p2c<<<blocks_for(n), PROBE_BLOCK>>>(gamma, dev_P, n, dev_U, dev_err);
  return finish();
}

int mgpu_probe_c2p(int mode, double gamma, double pfloor, const double *dev_U, const double *dev_guess, long long n,
                   double *dev_P, int *dev_err, int *dev_iters)
{
  if (mode < 0 || mode > 4 || n < 0 || (n && (!dev_U || !dev_guess || !dev_P || !dev_err || !dev_iters)))
    return MGPU_ERR_ARG;
  if (n) k_probe_c2p<<<blocks_for(n), PROBE_BLOCK>>>(mode, gamma, pfloor, dev_U, dev_guess, n, dev_P, dev_err,
                                                     dev_iters);
  return finish();
}

int mgpu_probe_flux(double gamma, int dim, const double *dev_P, long long n, double *dev_F, double *dev_lam)
{
  if (dim < 1 || dim > 3 || n < 0 || (n && (!dev_P || !dev_F || !dev_lam))) return MGPU_ERR_ARG;
  if (n) k_probe_flux<<<blocks_for(n), PROBE_BLOCK>>>(gamma, dim, dev_P, n, dev_F, dev_lam);
  return finish();
}

int mgpu_probe_riemann(int riemann, int dim, const int *dev_dims, double gamma, double pfloor, const double *dev_Pl,
                       const double *dev_Pr, long long n, double *dev_F, int *dev_err, double *dev_max_lambda,
                       int *dev_used_hllc)
{
  if (riemann < MGPU_RIEMANN_HLL || riemann > MGPU_RIEMANN_HLLD || (!dev_dims && (dim < 1 || dim > 3)) || n < 0 ||
      (n && (!dev_Pl || !dev_Pr || !dev_F || !dev_err || !dev_max_lambda)))
    return MGPU_ERR_ARG;
  if (n)
    k_probe_riemann<<<blocks_for(n), PROBE_BLOCK>>>(riemann, dim, dev_dims, gamma, pfloor, dev_Pl, dev_Pr, n,
                                                    dev_F, dev_err, dev_max_lambda, dev_used_hllc);
  return finish();
}

int mgpu_probe_reconstruct(int op, double theta, int is_mode, double sz10A, const double *dev_V, long long n,
                           double *dev_out)
{
  if (!(op == 0 || op == 1 || op == 4 || op == 5) || is_mode < 0 || is_mode > 2 || n < 0 ||
      (n && (!dev_V || !dev_out)))
    return MGPU_ERR_ARG;
  if (n) k_probe_recon<<<blocks_for(n), PROBE_BLOCK>>>(op, theta, is_mode, sz10A, dev_V, n, dev_out);
  return finish();
}

}  // extern "C"
