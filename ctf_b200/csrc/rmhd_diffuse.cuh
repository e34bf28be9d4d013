// Mara.diffuse(P, r) (luaC_Mara_diffuse, Mara/mara.cpp:343-366) on the device: P -> U of the
// committed primitives, U += GodunovOperator::LaxDiffusion(U, r) (Mara/hydro.cpp:205-283),
// then c2p back into the committed buffer with the measured primitive array (PA, the
// reference's PrimitiveArray) as the previous-state guess.  LaxDiffusion puts a Lax-Friedrichs
// flux -c r (U[i+s] - U[i]) dx_d on every face whose zone on either side failed the last c2p
// (the FailureMask, Ctl::fmask), c = 1/2, 1/4, 1/6 in 1, 2, 3 dimensions, runs flux-CT on it
// and adds its divergence.  PA is not changed (the reference's diffuse writes a local copy);
// the mask becomes this c2p's.
#pragma once
#include "rmhd_step.cuh"

namespace mgpu {

// The periodic interior image of guarded coordinate c along an axis of n interior zones.
__device__ __forceinline__ int interior_image(int c, int n, int ng)
{
  int m = (c - ng) % n;
  if (m < 0) m += n;
  return ng + m;
}

// P -> U (FP64) of guarded zone (i, j, k) from the committed primitives of its interior image
// (GodunovOperator::PrimToCons applies the periodic boundaries to P first).
template <class T>
__device__ __forceinline__ void diffuse_cons(const Grid &g, StateCPtr<T> P, double gamma, int i, int j, int k,
                                             double *U)
{
  if (self_periodic(g, 0)) i = interior_image(i, g.n[0], g.ng);
  if (self_periodic(g, 1)) j = interior_image(j, g.n[1], g.ng);
  if (self_periodic(g, 2)) k = interior_image(k, g.n[2], g.ng);
  const long long z = ((long long) i * g.G[1] + j) * g.G[2] + k;
  double p[8];
  load_state(g, P, z, p);
  prim_to_cons(gamma, p, U);
}

// Lax fluxes of direction dim on the faces (z, z + S) for z over the interior zones widened by
// one layer on each side of every used axis -- every face the CT update of an interior zone
// reads -- from the committed primitives (P0 or P1 by Ctl::cur).  coef = -c * r and
// dxd = dx_dim; the flux is zero where neither side failed the last c2p.
template <class T>
__global__ void __launch_bounds__(128) k_diffuse_flux(Grid g, int dim, StateCPtr<T> P0, StateCPtr<T> P1,
                                                      const Ctl *ctl, double gamma, double coef, double dxd, T *F)
{
  int e[3];
  for (int d = 0; d < 3; ++d) e[d] = g.nd > d ? g.n[d] + 2 : 1;
  const long long total = (long long) e[0] * e[1] * e[2];
  const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  const int i = (g.nd > 0 ? g.ng - 1 : 0) + (int) (t / ((long long) e[1] * e[2]));
  const int j = (g.nd > 1 ? g.ng - 1 : 0) + (int) ((t / e[2]) % e[1]);
  const int k = (g.nd > 2 ? g.ng - 1 : 0) + (int) (t % e[2]);
  const long long S = g.s[dim - 1];
  const long long z = ((long long) i * g.G[1] + j) * g.G[2] + k;
  const unsigned char *fm = ctl->fmask;
  double Fo[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (fm[z] || fm[z + S]) {
    const StateCPtr<T> P = ctl->cur ? P1 : P0;
    double Ul[8], Ur[8];
    diffuse_cons<T>(g, P, gamma, i, j, k, Ul);
    diffuse_cons<T>(g, P, gamma, i + (dim == 1), j + (dim == 2), k + (dim == 3), Ur);
#pragma unroll
    for (int q = 0; q < 8; ++q) Fo[q] = coef * (Ur[q] - Ul[q]) * dxd;
  }
#pragma unroll
  for (int q = 0; q < 8; ++q) F[q * g.cs + z] = T(Fo[q]);
}

// U1 = U0 + L (the Euler combine at dt = 1: U += L) with L the CT'd divergence of the Lax
// fluxes -- the advance's update_zone, so the arithmetic is the step's own.
template <class T, int ND>
__global__ void __launch_bounds__(256) k_diffuse_update(Grid g, StateCPtr<T> U0, const T *__restrict__ F,
                                                        const T *__restrict__ G, const T *__restrict__ H,
                                                        StatePtr<T> U1)
{
  const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.ninterior) return;
  const UpdateArgs a{COMB_EULER, 0.0};
  const StateCPtr<T> none{nullptr, nullptr};
  update_zone<T, ND>(g, a, U0, none, F, G, H, U1, StatePtr<T>{nullptr, nullptr}, none, none, none, 1.0,
                     interior_zone(g, t));
}

static __global__ void k_diffuse_begin(Ctl *ctl)
{
  if (threadIdx.x == 0 && blockIdx.x == 0) ctl->diffuse_err = 0;
}

// Enqueues one diffusion of the committed state (standard layout, single domain).
template <class T>
inline cudaError_t launch_diffuse(const AdvanceArgs &A, double r)
{
  const Grid &g = A.g;
  const AdvanceBuffers &b = A.b;
  cudaStream_t st = A.stream;
  const StatePtr<T> P0{(T *) b.Pc_bulk[0], b.Pc_B[0]}, P1{(T *) b.Pc_bulk[1], b.Pc_B[1]};
  const StatePtr<T> U0{(T *) b.U0_bulk, b.U0_B}, U1{(T *) b.U1_bulk, b.U1_B};
  k_diffuse_begin<<<1, 32, 0, st>>>(A.ctl);
  const unsigned zb = 256;
  k_prim_to_cons<T><<<(unsigned) ((g.ninterior + zb - 1) / zb), zb, 0, st>>>(
      g, StateCPtr<T>{P0.bulk, P0.B}, StateCPtr<T>{P1.bulk, P1.B}, U0, A.pp.gamma, A.ctl);
  const double c = g.nd == 1 ? 0.5 : g.nd == 2 ? 0.25 : 1.0 / 6.0;
  const double coef = -c * r;
  const double dxs[3] = {g.dx, g.dy, g.dz};
  long long faces = 1;
  for (int d = 0; d < g.nd; ++d) faces *= g.n[d] + 2;
  for (int d = 1; d <= g.nd; ++d)
    k_diffuse_flux<T><<<(unsigned) ((faces + 127) / 128), 128, 0, st>>>(
        g, d, StateCPtr<T>{P0.bulk, P0.B}, StateCPtr<T>{P1.bulk, P1.B}, A.ctl, A.pp.gamma, coef, dxs[d - 1],
        (T *) b.F[d - 1]);
  const unsigned ug = (unsigned) ((g.ninterior + zb - 1) / zb);
  const T *F = (const T *) b.F[0], *G = (const T *) b.F[1], *H = (const T *) b.F[2];
  const StateCPtr<T> Un{U0.bulk, U0.B};
  if (g.nd == 1) k_diffuse_update<T, 1><<<ug, zb, 0, st>>>(g, Un, F, G, H, U1);
  else if (g.nd == 2) k_diffuse_update<T, 2><<<ug, zb, 0, st>>>(g, Un, F, G, H, U1);
  else k_diffuse_update<T, 3><<<ug, zb, 0, st>>>(g, Un, F, G, H, U1);
  k_cons_to_prim<T, 2><<<(unsigned) ((g.ninterior + 127) / 128), 128, 0, st>>>(
      g, StateCPtr<T>{U1.bulk, U1.B}, (T *) b.PA, (const T *) b.PA, P0, P1, A.pp, A.ctl, 0, 0, C2P_DIFFUSE, A.ereset, A.preset,
      A.dreset);
  return cudaGetLastError();
}

}  // namespace mgpu
