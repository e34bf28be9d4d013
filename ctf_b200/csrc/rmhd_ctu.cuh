// CTU-Hancock operator on the device: one Runge-Kutta stage of PlmCtuHancockOperator
// (set_godunov('plm-muscl'), Mara/ctu-hancock.cpp:53-494) at its default safety level, where
// every failed check aborts the stage.
//
//   stage c2p (launch_phase, final == 2): the zone primitives P, failures not counted
//       (:61-66; the reference ignores that count)
//   k_ctu_flux, pass 1 (step 2, :131-212): every face f in [0, nz - sx) of each direction,
//       states P -+ half the limited slopes; a face whose states fail PrimCheck counts one
//       failure, its flux stays zero
//   k_ctu_predict (steps 3 and 3b, :224-393): every zone z >= sx checks the states on its own
//       two faces of each direction; interior zones form the Hancock predictor of each
//       direction -- the difference of the physical fluxes of those face states plus the
//       transverse Godunov fluxes of pass 1, over half a step -- invert it with the zone's P as
//       guess (a failure counts once per guarded array holding the zone, as the reference's
//       loop over all guarded zones does after its periodic fill) and scatter the predicted
//       primitives to the zone's periodic images
//   k_ctu_flux, pass 2 (step 4, :406-456): faces [sx, nz - sx) from the predicted primitives
//       of the face's direction -+ the same slopes; a face whose solver fails keeps its pass-1
//       flux
//   k_ctu_close: the stage fails with the count of the first check that failed (the four
//       abort points :211, :330, :393, :492; FailureMask is cleared at :102)
// followed by the shared CT + divergence + RK combine (k_update), which is the reference's
// ConstrainedTransport3d/2d and L = -div F on the final fluxes (:458-489).
//
// The slopes dPdx/dPdy/dPdz are recomputed from P where they are used instead of being
// stored: each is one minmod of three values already loaded for the face states.  Index
// ranges are the reference's flattened ones (x slowest, so z - sy and z + sy of a zone in
// [sx, nz - sx) stay inside the array; rows wrap as in the reference).
#pragma once
#include "rmhd_step.cuh"

namespace mgpu {

// plm_minmod of Mara/ctu-hancock.cpp:27-35 (its own copy of the limiter, with the theta of
// SetPlmTheta).
template <class T>
__device__ __forceinline__ T ctu_minmod(T theta, T ul, T u0, T ur)
{
  const T a = theta * (u0 - ul);
  const T b = T(0.5) * (ur - ul);
  const T c = theta * (ur - u0);
  const int sa = sgn(a), sb = sgn(b), sc = sgn(c);
  const T fa = m_abs(a), fb = m_abs(b), fc = m_abs(c);
  const T ab = (fa < fb) ? fa : fb;
  const T m = (ab < fc) ? ab : fc;
  return T(0.25) * T(abs(sa + sb)) * T(sa + sc) * m;
}

// Limited slope of component array a at zone z along stride S: zero outside [sx, nz - sx),
// where the reference's slope arrays keep their initial zeros (:116-120).
template <class T>
__device__ __forceinline__ T ctu_slope(const Grid &g, const T *a, long long z, long long S, T theta)
{
  if (z < g.s[0] || z >= g.nz - g.s[0]) return T(0);
  return ctu_minmod(theta, a[z - S], a[z], a[z + S]);
}

__device__ __forceinline__ void warp_add_int(int *ctr, int v)
{
  const unsigned mask = __activemask();
  const int sum = __reduce_add_sync(mask, v);
  if ((threadIdx.x & 31) == __ffs(mask) - 1 && sum) atomicAdd(ctr, sum);
}

// RiemannSolver::IntercellFlux at s = 0 of the compile-time solver; 0 on success.
template <class T, int dim, int RS>
__device__ __forceinline__ int ctu_riemann(const PhysParams &pp, const T *Pl, const T *Pr, T *Fo, T &ml,
                                           FluxTally &ft)
{
  int err;
  if constexpr (RS == RIEMANN_HLLD) {
    C2PTally t{0, 0};
    int used_hllc = 0;
    err = riemann_hlld<T, dim>(pp, Pl, Pr, Fo, ml, used_hllc, &t);
    ft.hlld_ok += 1 - used_hllc;
    ft.hlld_hllc += used_hllc;
    ft.face_c2p_calls += t.attempts > 0;
    ft.face_c2p_iters += t.iters;
  } else if constexpr (RS == RIEMANN_HLLC) {
    err = riemann_hllc<T, dim>(T(pp.gamma), Pl, Pr, Fo, ml);
  } else {
    err = riemann_hll<T, dim>(T(pp.gamma), Pl, Pr, Fo, ml);
  }
  return err;
}

// Both flux passes of one direction (dim 1..3); pass 1 reads its states from PA, pass 2 from
// the predicted primitives Pd of this direction.  One thread per face.
template <class T, int dim, int RS>
__global__ void __launch_bounds__(128, MGPU_FLUX_MINB) k_ctu_flux(Grid g, const T *__restrict__ PA,
                                                                  const T *__restrict__ Pd, T *__restrict__ F,
                                                                  PhysParams pp, Ctl *ctl, int stage, int pass)
{
  if (stage_failed(ctl, stage)) return;
  if (pass == 2 && (ctl->ctu_err[0] | ctl->ctu_err[1] | ctl->ctu_err[2])) return;
  const long long S = g.s[dim - 1], sx = g.s[0];
  const long long f = (pass == 1 ? 0 : sx) + (long long) blockIdx.x * blockDim.x + threadIdx.x;
  const T *src = pass == 1 ? PA : Pd;
  const T theta = T(pp.theta);
  T ml = T(0);
  FluxTally ft{0, 0, 0, 0, 0};
  int bad = 0;
  if (f < g.nz - sx) {
    T Pl[8], Pr[8], Fo[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const T *a = PA + q * g.cs;
      const T *b = src + q * g.cs;
      Pr[q] = b[f + S] - T(0.5) * ctu_slope(g, a, f + S, S, theta);
      Pl[q] = b[f] + T(0.5) * ctu_slope(g, a, f, S, theta);
    }
    bad = check_prim(Pl) || check_prim(Pr);
    const int err = bad ? 1 : ctu_riemann<T, dim, RS>(pp, Pl, Pr, Fo, ml, ft);
    if (pass == 1 || !err) {
#pragma unroll
      for (int q = 0; q < 8; ++q) F[q * g.cs + f] = err ? T(0) : Fo[q];
    }
  }
  flux_block_finish(double(ml), ft, ctl, RS == RIEMANN_HLLD);
  warp_add_int(&ctl->ctu_err[pass == 1 ? 0 : 3], bad);
}

// Transverse Godunov flux difference of the predictor, in the reference's term order.
template <class T>
__device__ __forceinline__ double ctu_dflux(const T *X, const Grid &g, int q, long long z, long long s, double h)
{
  return double(X[q * g.cs + z] - X[q * g.cs + z - s]) / h;
}

// Hancock predictor of every direction for zone z >= sx (one thread per zone).  U is the
// stage's conserved input (replaced by P->U of the stage primitives when the stage c2p made
// an emergency reset); F, G, H the pass-1 fluxes.
template <class T, int ND>
__global__ void __launch_bounds__(128) k_ctu_predict(Grid g, StateCPtr<T> U, const T *__restrict__ PA,
                                                     const T *__restrict__ F, const T *__restrict__ G,
                                                     const T *__restrict__ H, T *Pd0, T *Pd1, T *Pd2,
                                                     PhysParams pp, Ctl *ctl, int stage)
{
  if (stage_failed(ctl, stage) || ctl->ctu_err[0]) return;
  const long long sx = g.s[0], sy = g.s[1], sz = g.s[2];
  const long long z = sx + (long long) blockIdx.x * blockDim.x + threadIdx.x;
  int bad = 0, c2p_bad = 0;
  unsigned calls = 0, iters = 0;
  if (z < g.nz) {
    const int i = (int) (z / sx);
    const long long r = z - (long long) i * sx;
    const int j = (int) (r / g.G[2]);
    const int k = (int) (r - (long long) j * g.G[2]);
    const bool interior = i >= g.ng && i < g.ng + g.n[0] && (ND < 2 || (j >= g.ng && j < g.ng + g.n[1])) &&
                          (ND < 3 || (k >= g.ng && k < g.ng + g.n[2]));
    const T theta = T(pp.theta), gamma = T(pp.gamma);
    const double hd[3] = {g.dx, g.dy, g.dz};
    const double dt = ctl->dt;
    double u[8];
    if (interior) {
      if (ctl->ctu_reset) {
        double p0[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) p0[q] = double(PA[q * g.cs + z]);
        prim_to_cons(pp.gamma, p0, u);
      } else {
        load_state(g, U, z, u);
      }
    }
#pragma unroll 1
    for (int d = 0; d < ND; ++d) {
      const long long S = d == 0 ? sx : d == 1 ? sy : sz;
      T PL[8], PR[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const T *a = PA + q * g.cs;
        const T s = ctu_slope(g, a, z, S, theta);
        PL[q] = a[z] - T(0.5) * s;
        PR[q] = a[z] + T(0.5) * s;
      }
      const bool ok = !(check_prim(PL) || check_prim(PR));
      bad += !ok;
      if (!interior) continue;
      T FL[8], FR[8];
      if (ok) {
        T UL[8], UR[8], ap, am;
        prim_to_cons(gamma, PL, UL);
        prim_to_cons(gamma, PR, UR);
        flux_and_eigenvalues(gamma, UL, PL, FL, ap, am, d + 1, false);
        flux_and_eigenvalues(gamma, UR, PR, FR, ap, am, d + 1, false);
      } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) FL[q] = FR[q] = T(0);   // the stage aborts at this check
      }
      double ud[8], p[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const double dn = double(FR[q] - FL[q]) / hd[d];
        double sum;
        if (ND == 1) sum = dn;
        else if (ND == 2) sum = d == 0 ? dn + ctu_dflux(G, g, q, z, sy, g.dy) : dn + ctu_dflux(F, g, q, z, sx, g.dx);
        else if (d == 0) sum = dn + ctu_dflux(G, g, q, z, sy, g.dy) + ctu_dflux(H, g, q, z, sz, g.dz);
        else if (d == 1) sum = dn + ctu_dflux(H, g, q, z, sz, g.dz) + ctu_dflux(F, g, q, z, sx, g.dx);
        else sum = dn + ctu_dflux(F, g, q, z, sx, g.dx) + ctu_dflux(G, g, q, z, sy, g.dy);
        ud[q] = u[q] - sum * 0.5 * dt;
        p[q] = double(PA[q * g.cs + z]);
      }
      // Rmhd::ConsToPrim of the predicted state, the zone's primitives as its guess; on
      // failure the guess stays (:347-391)
      C2PTally tally{0, 0};
      const int err = cons_to_prim<(sizeof(T) < sizeof(double)), 2>(pp, ud, p, &tally) != 0;
      calls += 1;
      iters += (unsigned) tally.iters;
      if (err) c2p_bad += multiplicity(g, i, j, k);
      T *Pd = d == 0 ? Pd0 : d == 1 ? Pd1 : Pd2;
      int pi[3], pj[3], pk[3];
      const int ni = images_1d(i, g.n[0], g.ng, self_periodic(g, 0), pi);
      const int nj = images_1d(j, g.n[1], g.ng, self_periodic(g, 1), pj);
      const int nk = images_1d(k, g.n[2], g.ng, self_periodic(g, 2), pk);
      for (int a = 0; a < ni; ++a)
        for (int b = 0; b < nj; ++b)
          for (int c = 0; c < nk; ++c) {
            const long long w = ((long long) pi[a] * g.G[1] + pj[b]) * g.G[2] + pk[c];
#pragma unroll
            for (int q = 0; q < 8; ++q) Pd[q * g.cs + w] = T(p[q]);
          }
    }
  }
  warp_add_int(&ctl->ctu_err[1], bad);
  warp_add_int(&ctl->ctu_err[2], c2p_bad);
  warp_add(&stat_slot(ctl).c2p_calls, calls);
  warp_add(&stat_slot(ctl).c2p_iters, iters);
}

static __global__ void k_ctu_close(Ctl *ctl, int stage)
{
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int e = 0;
    for (int c = 0; c < 4 && !e; ++c) e = ctl->ctu_err[c];
    if (!stage_failed(ctl, stage)) ctl->stage_err[stage] = e;
    for (int c = 0; c < 4; ++c) ctl->ctu_err[c] = 0;
    ctl->ctu_c2p_err = 0;
    ctl->ctu_reset = 0;
  }
}

template <class T>
inline void launch_ctu_flux(const Grid &g, int d, int rs, unsigned grid, unsigned blk, cudaStream_t st, const T *PA,
                            const T *Pd, T *F, const PhysParams &pp, Ctl *ctl, int s, int pass)
{
#define MGPU_CTU_CASE(D, R)                                                             \
  if (d == D && rs == R) {                                                              \
    k_ctu_flux<T, D, R><<<grid, blk, 0, st>>>(g, PA, Pd, F, pp, ctl, s, pass);          \
    return;                                                                             \
  }
  MGPU_CTU_CASE(1, RIEMANN_HLLD) MGPU_CTU_CASE(2, RIEMANN_HLLD) MGPU_CTU_CASE(3, RIEMANN_HLLD)
  MGPU_CTU_CASE(1, RIEMANN_HLLC) MGPU_CTU_CASE(2, RIEMANN_HLLC) MGPU_CTU_CASE(3, RIEMANN_HLLC)
  MGPU_CTU_CASE(1, RIEMANN_HLL) MGPU_CTU_CASE(2, RIEMANN_HLL) MGPU_CTU_CASE(3, RIEMANN_HLL)
#undef MGPU_CTU_CASE
}

// Everything of a CTU stage before the update: pass 1, the predictor, pass 2, the close.
template <class T>
inline void launch_ctu_stage(const AdvanceArgs &A, int s, StateCPtr<T> Uin)
{
  const Grid &g = A.g;
  const AdvanceBuffers &b = A.b;
  cudaStream_t st = A.stream;
  LaunchProfiler *pr = A.prof;
  const T *PA = (const T *) b.PA;
  const long long sx = g.s[0];
  const unsigned fb = 128;
  const long long n1 = g.nz - sx, n2 = g.nz - 2 * sx;
  for (int d = 1; d <= g.nd && n1 > 0; ++d) {
    ProfScope ps(pr, st, KC_FLUX, n1);
    launch_ctu_flux<T>(g, d, A.pp.riemann, (unsigned) ((n1 + fb - 1) / fb), fb, st, PA, PA, (T *) b.F[d - 1], A.pp,
                       A.ctl, s, 1);
  }
  if (n1 > 0) {
    ProfScope ps(pr, st, KC_PREDICT, n1);
    const unsigned grid = (unsigned) ((n1 + 127) / 128);
    const T *F = (const T *) b.F[0], *G = (const T *) b.F[1], *H = (const T *) b.F[2];
    T *P0 = (T *) b.Pd[0], *P1 = (T *) b.Pd[1], *P2 = (T *) b.Pd[2];
    if (g.nd == 1) k_ctu_predict<T, 1><<<grid, 128, 0, st>>>(g, Uin, PA, F, G, H, P0, P1, P2, A.pp, A.ctl, s);
    else if (g.nd == 2) k_ctu_predict<T, 2><<<grid, 128, 0, st>>>(g, Uin, PA, F, G, H, P0, P1, P2, A.pp, A.ctl, s);
    else k_ctu_predict<T, 3><<<grid, 128, 0, st>>>(g, Uin, PA, F, G, H, P0, P1, P2, A.pp, A.ctl, s);
  }
  for (int d = 1; d <= g.nd && n2 > 0; ++d) {
    ProfScope ps(pr, st, KC_FLUX, n2);
    launch_ctu_flux<T>(g, d, A.pp.riemann, (unsigned) ((n2 + fb - 1) / fb), fb, st, PA, (const T *) b.Pd[d - 1],
                       (T *) b.F[d - 1], A.pp, A.ctl, s, 2);
  }
  ProfScope ps(pr, st, KC_BEGIN, 1);
  k_ctu_close<<<1, 32, 0, st>>>(A.ctl, s);
}

}  // namespace mgpu
