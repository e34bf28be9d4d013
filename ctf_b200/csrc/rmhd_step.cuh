// Step kernels of the B200 RMHD advance, templated on the bulk type T.
//
// Data layout in HBM (structure of arrays, one contiguous array per component):
//   zone index z = (i*G1 + j)*G2 + k over the guarded grid (x slowest, as in the reference's
//   AoS layout, Mara/hydro.cpp:80-110), component c at base + c*cs.
//   "state" arrays (committed prims, conserved RK registers): components 0..4 in T,
//                 components 5..7 (the magnetic field) in double, always;
//   "face" arrays (stage prims PA, fluxes F/G/H): all 8 components in T.
// Guard zones of a state are never read: the c2p kernel writes each interior zone's
// primitives to the zone and to every periodic image of it in the guard layers, which gives
// exactly the arrays SimpleCartesianDomain::Synchronize (Mara/simple-cart.cpp:81-174) would.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "rmhd_physics.cuh"

// Minimum resident blocks of 128 threads per SM requested for the flux sweep (caps its
// registers at 65536 / (128 * MGPU_FLUX_MINB)).
#ifndef MGPU_FLUX_MINB
#define MGPU_FLUX_MINB 2
#endif
// The same for the zone c2p kernel (5 blocks: chosen by a sweep of 3-5; its natural register
// count allows 3).
#ifndef MGPU_C2P_MINB
#define MGPU_C2P_MINB 5
#endif

namespace mgpu {

__device__ __forceinline__ bool stage_failed(const Ctl *ctl, int upto)
{
  int e = 0;
  for (int s = 0; s < upto && s < MAX_STAGES; ++s) e |= ctl->stage_err[s];
  return e != 0;
}

// Positions of zone m_d and its periodic guard images along one dimension.
__device__ __forceinline__ int images_1d(int m, int n, int ng, bool active, int *pos)
{
  pos[0] = m;
  if (!active) return 1;
  int c = 1;
  if (m - n >= 0 && m - n < ng) pos[c++] = m - n;
  if (m + n >= n + ng && m + n < n + 2 * ng) pos[c++] = m + n;
  return c;
}

// Whether dimension d (0-based) gets its guard layers from the periodic images of this
// grid's own zones (false for unused dimensions and for dimensions whose guards a halo
// exchange fills).
__device__ __forceinline__ bool self_periodic(const Grid &g, int d) { return g.nd > d && !g.ext[d]; }

// Number of guarded arrays holding zone (i, j, k) -- this grid's, counting the zone's
// periodic images, and on a decomposed domain its neighbours' -- which is how many times
// the reference's ConsToPrim over every guarded zone of every rank counts its failure
// (Mara/hydro.cpp:133-149,201).
__device__ __forceinline__ int multiplicity(const Grid &g, int i, int j, int k)
{
  int p[3];
  const int m[3] = {i, j, k};
  int c = 1;
  for (int d = 0; d < 3; ++d) {
    if (g.ext[d]) c *= g.mult[d][m[d] - g.ng];
    else c *= images_1d(m[d], g.n[d], g.ng, g.nd > d, p);
  }
  return c;
}

template <class T>
__device__ __forceinline__ void load_state(const Grid &g, StateCPtr<T> s, long long z, double *U)
{
#pragma unroll
  for (int c = 0; c < 5; ++c) U[c] = double(s.bulk[c * g.cs + z]);
#pragma unroll
  for (int c = 0; c < 3; ++c) U[5 + c] = s.B[c * g.cs + z];
}

// The statistics slot of the calling block.
__device__ __forceinline__ StatSlot &stat_slot(Ctl *ctl) { return ctl->stat[blockIdx.x % STAT_SLOTS]; }

// Zeroes the statistics slots (all threads of the calling block take part).
__device__ __forceinline__ void stat_reset(Ctl *ctl)
{
  for (int i = threadIdx.x; i < STAT_SLOTS * (int) (sizeof(StatSlot) / 8); i += blockDim.x)
    reinterpret_cast<unsigned long long *>(ctl->stat)[i] = 0ull;
}

// Warp-aggregated counter increment.
__device__ __forceinline__ void warp_add(unsigned long long *ctr, unsigned v)
{
  const unsigned mask = __activemask();
  const unsigned sum = __reduce_add_sync(mask, v);
  if ((threadIdx.x & 31) == __ffs(mask) - 1 && sum) atomicAdd(ctr, (unsigned long long) sum);
}

// ---- begin: dt and counters ----------------------------------------------------------------
// dt_mode 0: dt given by the host; 1: dt = cfl * min_dx / MaxLambda of the previous advance
// (luaC_Mara_get_timestep, Mara/mara.cpp:374-381), computed on the device.
static __global__ void k_begin(Ctl *ctl, int dt_mode, double dt, double cfl, double min_dx)
{
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    if (dt_mode == 1) dt = cfl * min_dx / __longlong_as_double((long long) ctl->max_lambda_bits);
    ctl->dt = dt;
    ctl->max_lambda_bits = 0ull;   // RiemannSolver::ResetMaxLambda
    for (int s = 0; s < MAX_STAGES; ++s) ctl->stage_err[s] = 0;
    ctl->final_err = 0;
    for (int s = 0; s < 4; ++s) ctl->ctu_err[s] = 0;
    ctl->ctu_c2p_err = ctl->ctu_reset = 0;
    ctl->committed = 0;
  }
  if (blockIdx.x == 0) stat_reset(ctl);
}

static __global__ void k_commit(Ctl *ctl, int nstages)
{
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int e = 0, first = 0;
    for (int s = 0; s < nstages; ++s) {
      e |= ctl->stage_err[s];
      if (!first) first = ctl->stage_err[s];
    }
    e |= ctl->final_err;
    if (!first) first = ctl->final_err;
    ctl->n_advances += 1;
    if (e == 0) {
      ctl->cur ^= 1;
      ctl->committed = 1;
    } else {
      ctl->n_failed += 1;
      ctl->n_failed_zones += (unsigned) first;
    }
  }
}

// ---- P -> U on interior zones (GodunovOperator::PrimToCons, Mara/hydro.cpp:112-123) ----------
template <class T>
__device__ __forceinline__ void p2c_zone(const Grid &g, StateCPtr<T> P, StatePtr<T> U, double gamma, long long t)
{
  int i, j, k;
  interior_coords(g, t, i, j, k);
  const long long z = ((long long) i * g.G[1] + j) * g.G[2] + k;
  double p[8], u[8];
  load_state(g, P, z, p);
  prim_to_cons(gamma, p, u);
#pragma unroll
  for (int c = 0; c < 5; ++c) U.bulk[c * g.cs + z] = T(u[c]);
#pragma unroll
  for (int c = 0; c < 3; ++c) U.B[c * g.cs + z] = u[5 + c];
}

template <class T>
__global__ void __launch_bounds__(256) k_prim_to_cons(Grid g, StateCPtr<T> P0, StateCPtr<T> P1, StatePtr<T> U,
                                                      double gamma, const Ctl *ctl)
{
  const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.ninterior) return;
  p2c_zone<T>(g, ctl->cur ? P1 : P0, U, gamma, t);
}

// ---- c2p with guard scatter (GodunovOperator::ConsToPrim, Mara/hydro.cpp:125-202) -----------
// Stage c2p (final == 0): guess from PA (or zeros on the first stage, as the reference's
// PrimitiveArray is zero-filled by every advance, Mara/mara.cpp:321); result into PA.
// Closing c2p (final == 1): guess from PA, result into the next committed state.
// CTU-Hancock stage c2p (final == 2): as a stage c2p, but its failures do not abort the stage
// (PlmCtuHancockOperator::dUdt ignores the count, Mara/ctu-hancock.cpp:61-66; a failed zone
// keeps its guess) and its emergency resets are recorded, because the reset also replaces the
// operator's conserved input by P->U of the repaired primitives (Mara/hydro.cpp:186-195).
// Counts a zone's c2p outcome and scatters its primitives to the zone and its guard images.
template <class T>
__device__ __forceinline__ void c2p_finish(const Grid &g, T *PA, StatePtr<T> Pn, Ctl *ctl, int stage, int final,
                                           int ereset, double preset, double dreset, int i, int j, int k,
                                           const double *u, double *p, int err, const C2PTally &tally)
{
  const bool counted = final != C2P_LEAN_RESTORE;
  if (counted && final != C2P_DIFFUSE) {
    StatSlot &st = stat_slot(ctl);
    warp_add(&st.c2p_calls, 1u);
    warp_add(&st.c2p_iters, (unsigned) tally.iters);
    if (tally.attempts >= 1 && tally.attempts <= 5) warp_add(&st.c2p_attempt[tally.attempts], 1u);
    warp_add(&st.c2p_failed, err ? 1u : 0u);
  }
  if (err) {
    if (ereset) {   // emergency reset of the failed zone
      p[0] = dreset;
      p[1] = preset;
      p[2] = p[3] = p[4] = 0.0;
      p[5] = u[5];
      p[6] = u[6];
      p[7] = u[7];
      if (final == 2) atomicAdd(&ctl->ctu_reset, 1);
    } else if (final == C2P_DIFFUSE) {
      atomicAdd(&ctl->diffuse_err, multiplicity(g, i, j, k));
    } else if (counted) {
      const bool closing = final == C2P_CLOSING || final == C2P_LEAN_CLOSING;
      atomicAdd(closing ? &ctl->final_err : final == C2P_CTU_STAGE ? &ctl->ctu_c2p_err : &ctl->stage_err[stage],
                multiplicity(g, i, j, k));
    }
  }
  // the failure mask of this c2p at the zone and its images (an emergency reset clears it)
  unsigned char *const fm = counted ? ctl->fmask : nullptr;
  const unsigned char failed = (unsigned char) (err && !ereset);
  int pi[3], pj[3], pk[3];
  const int ni = images_1d(i, g.n[0], g.ng, self_periodic(g, 0), pi);
  const int nj = images_1d(j, g.n[1], g.ng, self_periodic(g, 1), pj);
  const int nk = images_1d(k, g.n[2], g.ng, self_periodic(g, 2), pk);
  for (int a = 0; a < ni; ++a)
    for (int b = 0; b < nj; ++b)
      for (int c = 0; c < nk; ++c) {
        const long long w = ((long long) pi[a] * g.G[1] + pj[b]) * g.G[2] + pk[c];
        if (fm) fm[w] = failed;
        if (final == C2P_CLOSING || final == C2P_DIFFUSE) {
#pragma unroll
          for (int q = 0; q < 5; ++q) Pn.bulk[q * g.cs + w] = T(p[q]);
#pragma unroll
          for (int q = 0; q < 3; ++q) Pn.B[q * g.cs + w] = p[5 + q];
        } else {
#pragma unroll
          for (int q = 0; q < 8; ++q) PA[q * g.cs + w] = T(p[q]);
          if (final == C2P_LEAN_CLOSING) {   // the field of the register about to be committed
#pragma unroll
            for (int q = 0; q < 3; ++q) Pn.B[q * g.cs + w] = u[5 + q];
          }
        }
      }
}

// The conserved input of a c2p launch: U, or in the lean layout one of the two conserved
// registers (Pn0 = U[0], Pn1 = U[1]) by the committed role bit ctl->cur -- U[cur] for the
// restore, U[!cur] (the RK register) otherwise.
template <class T>
__device__ __forceinline__ StateCPtr<T> c2p_input(const Ctl *ctl, int final, StateCPtr<T> U, StatePtr<T> Pn0,
                                                  StatePtr<T> Pn1)
{
  if (final < C2P_LEAN_STAGE || final == C2P_DIFFUSE) return U;
  const int r = final == C2P_LEAN_RESTORE ? ctl->cur : ctl->cur ^ 1;
  const StatePtr<T> R = r ? Pn1 : Pn0;
  return StateCPtr<T>{R.bulk, R.B};
}

// Whether a c2p launch has nothing to do: an earlier stage failed, or (restore) the advance
// committed.
__device__ __forceinline__ bool c2p_skip(const Ctl *ctl, int stage, int final)
{
  return final == C2P_LEAN_RESTORE ? ctl->committed != 0 : stage_failed(ctl, stage);
}

// One interior zone's c2p.  Guess: 0 compiles in the per-thread network guess (used when
// pp.learned), 2 leaves it out -- the network's activations would otherwise set the register
// and stack budget of every c2p launch.  PAg holds the previous primitives the ladder may start
// from (PA itself, except in the pipelined host advance, whose stages alternate two arrays).
template <class T, int Guess = 2>
__device__ __forceinline__ void c2p_zone(const Grid &g, StateCPtr<T> U, T *PA, const T *PAg, StatePtr<T> Pn,
                                         const PhysParams &pp,
                                         Ctl *ctl, int stage, int zero_guess, int final, int ereset, double preset,
                                         double dreset, long long t)
{
  int i, j, k;
  interior_coords(g, t, i, j, k);
  const long long z = ((long long) i * g.G[1] + j) * g.G[2] + k;
  double u[8], p[8];
  load_state(g, U, z, u);
  // the previous primitives are read only when the ladder needs them or a failure keeps them
  const auto prev = [&](double *q) {
#pragma unroll
    for (int c = 0; c < 8; ++c) q[c] = zero_guess ? 0.0 : double(PAg[c * g.cs + z]);
  };
  C2PTally tally;
  const int err = cons_to_prim<(sizeof(T) < sizeof(double)), Guess>(pp, u, p, &tally, 0.0, 0.0, true, prev) != 0;
  c2p_finish<T>(g, PA, Pn, ctl, stage, final, ereset, preset, dreset, i, j, k, u, p, err, tally);
}

template <class T, int Guess>
__global__ void __launch_bounds__(128, MGPU_C2P_MINB) k_cons_to_prim(Grid g, StateCPtr<T> U, T *PA, const T *PAg,
                                                      StatePtr<T> Pn0, StatePtr<T> Pn1,
                                                      PhysParams pp, Ctl *ctl, int stage, int zero_guess, int final,
                                                      int ereset, double preset, double dreset)
{
  if (c2p_skip(ctl, stage, final)) return;
  const long long t = win_tbeg(g) + (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= win_tend(g)) return;
  // the uncommitted buffer, or for Mara.diffuse the committed one (rewritten in place)
  const int target = final == C2P_DIFFUSE ? ctl->cur : ctl->cur ^ 1;
  c2p_zone<T, Guess>(g, c2p_input(ctl, final, U, Pn0, Pn1), PA, PAg, target ? Pn1 : Pn0, pp, ctl, stage, zero_guess,
                     final, ereset, preset, dreset, t);
}

// The boundary shell of a decomposed block: interior zones within Ng of a face whose guards a
// halo exchange fills (region 1), and the rest (region 2, the core).  The exchange reads only
// shell zones (and their periodic images along the unsplit dimensions), so the core's c2p can
// run while the slabs travel.
__device__ __forceinline__ bool in_shell(const Grid &g, int i, int j, int k)
{
  const int m[3] = {i, j, k};
  for (int d = 0; d < 3; ++d) {
    if (!g.ext[d]) continue;
    const int r = m[d] - g.ng;
    if (r < g.ng || r >= g.n[d] - g.ng) return true;
  }
  return false;
}

// The stage c2p of one region of the interior (1 shell, 2 core); zones of the other region
// exit at once.
template <class T>
__global__ void __launch_bounds__(128, MGPU_C2P_MINB) k_cons_to_prim_region(Grid g, StateCPtr<T> U, T *PA,
                                                                            StatePtr<T> Pn0, StatePtr<T> Pn1,
                                                                            PhysParams pp, Ctl *ctl, int stage,
                                                                            int zero_guess, int final, int ereset,
                                                                            double preset, double dreset, int region)
{
  if (c2p_skip(ctl, stage, final)) return;
  const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.ninterior) return;
  int i, j, k;
  interior_coords(g, t, i, j, k);
  if (in_shell(g, i, j, k) != (region == 1)) return;
  const int target = ctl->cur ^ 1;
  c2p_zone<T, 2>(g, c2p_input(ctl, final, U, Pn0, Pn1), PA, PA, target ? Pn1 : Pn0, pp, ctl, stage, zero_guess, final,
                 ereset, preset, dreset, t);
}

// ---- flux sweep (MethodOfLinesSplit::intercell_flux_sweep, Mara/plm-split.cpp:43-73) ---------
// One thread per face.  The face set is the reference's: every zone index f with
// 2*S <= f < nz - 3*S in the flattened guarded array (S the zone stride of `dim`), the face
// between zones f and f + S.  Faces that straddle a row end in the flattened array are
// evaluated too, because they enter MaxLambda in the reference.
// Per-thread flux statistics, summed per block.
struct FluxTally {
  int hlld_ok, hlld_hllc, pcm_retry, face_c2p_calls, face_c2p_iters;
};

// One face: reconstruct, Riemann solve (PCM retry on failure), the flux in Fo (zero when both
// attempts fail); the face's |lambda| is folded into ml.
template <class T, int dim, int RS>
__device__ __forceinline__ void face_flux(const Grid &g, const T *__restrict__ PA, const PhysParams &pp, long long f,
                                          T &ml, FluxTally &ft, T *Fo, HlldSlot<T> *slot = nullptr)
{
  const long long S = g.s[dim - 1];
  T Pl[8], Pr[8];
  const T theta = T(pp.theta);
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const T *a = PA + q * g.cs + f;
    if (pp.recon == RECON_PCM) {
      Pl[q] = a[0];
      Pr[q] = a[S];
    } else if (pp.recon == RECON_PLM) {
      const T vm = a[-S], v0 = a[0], vp = a[S], vpp = a[2 * S];
      Pl[q] = plm(theta, vm, v0, vp, T(+1));
      Pr[q] = plm(theta, v0, vp, vpp, T(-1));
    } else {
      const T vm2 = a[-2 * S], vm1 = a[-S], v0 = a[0], vp1 = a[S], vp2 = a[2 * S], vp3 = a[3 * S];
      Pl[q] = weno5(pp.is_mode, T(pp.sz10A), vm2, vm1, v0, vp1, vp2, true);
      Pr[q] = weno5(pp.is_mode, T(pp.sz10A), vm1, v0, vp1, vp2, vp3, false);
    }
  }
  const T gamma = T(pp.gamma);
  int err = 1, used_hllc = 0;
  constexpr bool hlld = RS == RIEMANN_HLLD;
  C2PTally tally{0, 0};
  // attempt 0: reconstructed states; attempt 1: the zone states themselves (PCM retry).
  // One call site per solver keeps a single inlined copy of it.
#pragma unroll 1
  for (int attempt = 0; attempt < 2 && err; ++attempt) {
    if (attempt == 1) {
      ft.pcm_retry += 1;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        Pl[q] = PA[q * g.cs + f];
        Pr[q] = PA[q * g.cs + f + S];
      }
    }
    C2PTally t{0, 0};
    if constexpr (RS == RIEMANN_HLLD) err = riemann_hlld<T, dim>(pp, Pl, Pr, Fo, ml, used_hllc, &t, slot);
    else if constexpr (RS == RIEMANN_HLLC) err = riemann_hllc<T, dim>(gamma, Pl, Pr, Fo, ml);
    else err = riemann_hll<T, dim>(gamma, Pl, Pr, Fo, ml);
    tally.iters += t.iters;
    tally.attempts += t.attempts;
  }
  if (err) {
#pragma unroll
    for (int q = 0; q < 8; ++q) Fo[q] = T(0);
  }
  if constexpr (hlld) {
    ft.hlld_ok += 1 - used_hllc;
    ft.hlld_hllc += used_hllc;
  }
  ft.face_c2p_calls += tally.attempts > 0;
  ft.face_c2p_iters += tally.iters;
}

// One face, its flux stored in F.
template <class T, int dim, int RS>
__device__ __forceinline__ void flux_face(const Grid &g, const T *__restrict__ PA, T *__restrict__ F,
                                          const PhysParams &pp, long long f, T &ml, FluxTally &ft)
{
  T Fo[8];
  face_flux<T, dim, RS>(g, PA, pp, f, ml, ft, Fo);
#pragma unroll
  for (int q = 0; q < 8; ++q) F[q * g.cs + f] = Fo[q];
}

// MaxLambda of a block: warp max -> block max -> one atomicMax (non-negative doubles order
// like their bit patterns); plus the block's flux statistics.  All threads must call.
__device__ __forceinline__ void flux_block_finish(double m, const FluxTally &ft, Ctl *ctl, bool hlld)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double wmax[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();   // wmax may still be read from a previous tile
  if (lane == 0) wmax[warp] = m;
  __syncthreads();
  if (warp == 0) {
    m = lane < (blockDim.x >> 5) ? wmax[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0 && m > 0.0) atomicMax(&ctl->max_lambda_bits, (unsigned long long) __double_as_longlong(m));
  }
  StatSlot &st = stat_slot(ctl);
  if (hlld) {
    warp_add(&st.hlld_ok, (unsigned) ft.hlld_ok);
    warp_add(&st.hlld_hllc, (unsigned) ft.hlld_hllc);
  }
  warp_add(&st.pcm_retry, (unsigned) ft.pcm_retry);
  warp_add(&st.face_c2p_calls, (unsigned) ft.face_c2p_calls);
  warp_add(&st.face_c2p_iters, (unsigned) ft.face_c2p_iters);
}

template <class T, int dim, int RS>
__global__ void __launch_bounds__(128, MGPU_FLUX_MINB) k_flux(Grid g, const T *__restrict__ PA, T *__restrict__ F,
                                                              PhysParams pp, Ctl *ctl, int stage)
{
  if (stage_failed(ctl, stage + 1)) return;
  const long long S = g.s[dim - 1];
  const long long f = 2 * S + (long long) blockIdx.x * blockDim.x + threadIdx.x;
  T ml = T(0);
  FluxTally ft{0, 0, 0, 0, 0};
  if (f < g.nz - 3 * S) flux_face<T, dim, RS>(g, PA, F, pp, f, ml, ft);
  flux_block_finish(double(ml), ft, ctl, RS == RIEMANN_HLLD);
}

// ---- CT + flux divergence + Runge-Kutta combine ---------------------------------------------
// Flux-CT (AdiabaticIdealRmhd::ConstrainedTransport3d/2d, Mara/rmhd.cpp:311-381), the
// divergence L = -(dF/dx + dG/dy + dH/dz) (Mara/plm-split.cpp:75-122) and the stage combine
// of Mara/runge-kutta.hpp:129-177, fused, on interior zones only.
struct UpdateArgs {
  int combine;
  double c;        // COMB_RK4_K coefficient
};

template <class T>
__device__ __forceinline__ double fval(const T *F, const Grid &g, int q, long long z)
{
  return double(F[q * g.cs + z]);
}

// Zone index of interior flat index t.
__device__ __forceinline__ long long interior_zone(const Grid &g, long long t)
{
  int i, j, k;
  interior_coords(g, t, i, j, k);
  return ((long long) i * g.G[1] + j) * g.G[2] + k;
}

// 8-point corner-EMF average for the B-flux component (normal dir a, field component b):
// (2 F0 + F[+b] + F[-b] - G0 - G[+a] - G[-b] - G[+a-b]) / 8 with F the a-flux of B_b and G
// the b-flux of B_a, strides sa (normal dir) and sb (field dir).
template <class T>
__device__ __forceinline__ double ct_emf(const T *Fa, const T *Fb, const Grid &g, int qb, int qa, long long z,
                                         long long sa, long long sb)
{
  const T *F = Fa + qb * g.cs + z;
  const T *G = Fb + qa * g.cs + z;
  return (2 * double(F[0]) + double(F[sb]) + double(F[-sb]) - double(G[0]) - double(G[sa]) - double(G[-sb]) -
          double(G[sa - sb])) * 0.125;
}

template <class T>
__device__ __forceinline__ T combine_bulk(const UpdateArgs &a, T un, T us, T dt, T L, T *K, T k1, T k2, T k3)
{
  switch (a.combine) {
  case COMB_EULER: return un + dt * L;
  case COMB_RK2_2: return T(0.5) * (un + us + dt * L);
  case COMB_RK3_2: return T(3. / 4) * un + T(1. / 4) * us + T(1. / 4) * dt * L;
  case COMB_RK3_3: return T(1. / 3) * un + T(2. / 3) * us + T(2. / 3) * dt * L;
  case COMB_RK4_K: { const T kk = dt * L; *K = kk; return un + T(a.c) * kk; }
  default: return un + (T(1.0) / T(6.0)) * (k1 + T(2.0) * k2 + T(2.0) * k3 + dt * L);
  }
}

template <class T, int ND>
__device__ __forceinline__ void update_zone(const Grid &g, const UpdateArgs &a, StateCPtr<T> Un, StateCPtr<T> Us,
                                            const T *__restrict__ F, const T *__restrict__ G,
                                            const T *__restrict__ H, StatePtr<T> Uout, StatePtr<T> Kout,
                                            StateCPtr<T> K1, StateCPtr<T> K2, StateCPtr<T> K3, double dtd,
                                            long long z)
{
  const long long sx = g.s[0], sy = g.s[1], sz = g.s[2];
  const double dx = g.dx, dy = g.dy, dz = g.dz;
  const T dt = T(dtd);
  const bool rk4 = a.combine >= COMB_RK4_K;
  // bulk components 0..4: plain flux differences in T
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    T L;
    if (ND == 1) {
      L = -(F[q * g.cs + z] - F[q * g.cs + z - sx]) / T(dx);
    } else if (ND == 2) {
      L = -(F[q * g.cs + z] - F[q * g.cs + z - sx]) / T(dx) - (G[q * g.cs + z] - G[q * g.cs + z - sy]) / T(dy);
    } else {
      L = -(F[q * g.cs + z] - F[q * g.cs + z - sx]) / T(dx) - (G[q * g.cs + z] - G[q * g.cs + z - sy]) / T(dy) -
          (H[q * g.cs + z] - H[q * g.cs + z - sz]) / T(dz);
    }
    const T un = Un.bulk[q * g.cs + z];
    const T us = (a.combine == COMB_RK2_2 || a.combine == COMB_RK3_2 || a.combine == COMB_RK3_3) ? Us.bulk[q * g.cs + z] : T(0);
    T k1 = T(0), k2 = T(0), k3 = T(0), kk = T(0);
    if (a.combine == COMB_RK4_4) { k1 = K1.bulk[q * g.cs + z]; k2 = K2.bulk[q * g.cs + z]; k3 = K3.bulk[q * g.cs + z]; }
    Uout.bulk[q * g.cs + z] = combine_bulk<T>(a, un, us, dt, L, &kk, k1, k2, k3);
    if (rk4 && a.combine == COMB_RK4_K) Kout.bulk[q * g.cs + z] = kk;
  }
  // magnetic components 5..7 in double, with the constrained-transport fluxes
  double Lb[3];
  if (ND == 1) {
#pragma unroll
    for (int c = 0; c < 3; ++c) Lb[c] = -(fval(F, g, 5 + c, z) - fval(F, g, 5 + c, z - sx)) / dx;
  } else if (ND == 2) {
    // CT2d: Fx[Bx] = 0, Fx[By] = FxBy, Fy[Bx] = FyBx, Fy[By] = 0; Bz keeps its Godunov fluxes
    const double FxBy0 = ct_emf(F, G, g, By, Bx, z, sx, sy), FxBym = ct_emf(F, G, g, By, Bx, z - sx, sx, sy);
    const double FyBx0 = ct_emf(G, F, g, Bx, By, z, sy, sx), FyBxm = ct_emf(G, F, g, Bx, By, z - sy, sy, sx);
    if constexpr (sizeof(T) < sizeof(double)) {   // FP32 bulk: reciprocals, zeroed fluxes dropped
      const double idx = 1.0 / dx, idy = 1.0 / dy;
      Lb[0] = -(FyBx0 - FyBxm) * idy;
      Lb[1] = -(FxBy0 - FxBym) * idx;
      Lb[2] = -(fval(F, g, Bz, z) - fval(F, g, Bz, z - sx)) * idx - (fval(G, g, Bz, z) - fval(G, g, Bz, z - sy)) * idy;
    } else {   // the reference's expressions, bit for bit
      Lb[0] = -(0.0 - 0.0) / dx - (FyBx0 - FyBxm) / dy;
      Lb[1] = -(FxBy0 - FxBym) / dx - (0.0 - 0.0) / dy;
      Lb[2] = -(fval(F, g, Bz, z) - fval(F, g, Bz, z - sx)) / dx - (fval(G, g, Bz, z) - fval(G, g, Bz, z - sy)) / dy;
    }
  } else {
    const double FxBy0 = ct_emf(F, G, g, By, Bx, z, sx, sy), FxBym = ct_emf(F, G, g, By, Bx, z - sx, sx, sy);
    const double FyBx0 = ct_emf(G, F, g, Bx, By, z, sy, sx), FyBxm = ct_emf(G, F, g, Bx, By, z - sy, sy, sx);
    const double FyBz0 = ct_emf(G, H, g, Bz, By, z, sy, sz), FyBzm = ct_emf(G, H, g, Bz, By, z - sy, sy, sz);
    const double FzBy0 = ct_emf(H, G, g, By, Bz, z, sz, sy), FzBym = ct_emf(H, G, g, By, Bz, z - sz, sz, sy);
    const double FzBx0 = ct_emf(H, F, g, Bx, Bz, z, sz, sx), FzBxm = ct_emf(H, F, g, Bx, Bz, z - sz, sz, sx);
    const double FxBz0 = ct_emf(F, H, g, Bz, Bx, z, sx, sz), FxBzm = ct_emf(F, H, g, Bz, Bx, z - sx, sx, sz);
    if constexpr (sizeof(T) < sizeof(double)) {   // FP32 bulk: reciprocals, zeroed fluxes dropped
      const double idx = 1.0 / dx, idy = 1.0 / dy, idz = 1.0 / dz;
      Lb[0] = -(FyBx0 - FyBxm) * idy - (FzBx0 - FzBxm) * idz;
      Lb[1] = -(FxBy0 - FxBym) * idx - (FzBy0 - FzBym) * idz;
      Lb[2] = -(FxBz0 - FxBzm) * idx - (FyBz0 - FyBzm) * idy;
    } else {   // the reference's expressions, bit for bit
      Lb[0] = -(0.0 - 0.0) / dx - (FyBx0 - FyBxm) / dy - (FzBx0 - FzBxm) / dz;
      Lb[1] = -(FxBy0 - FxBym) / dx - (0.0 - 0.0) / dy - (FzBy0 - FzBym) / dz;
      Lb[2] = -(FxBz0 - FxBzm) / dx - (FyBz0 - FyBzm) / dy - (0.0 - 0.0) / dz;
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double un = Un.B[c * g.cs + z];
    const double L = Lb[c];
    double out;
    switch (a.combine) {
    case COMB_EULER: out = un + dtd * L; break;
    case COMB_RK2_2: out = 0.5 * (un + Us.B[c * g.cs + z] + dtd * L); break;
    case COMB_RK3_2: out = 3. / 4 * un + 1. / 4 * Us.B[c * g.cs + z] + 1. / 4 * dtd * L; break;
    case COMB_RK3_3: out = 1. / 3 * un + 2. / 3 * Us.B[c * g.cs + z] + 2. / 3 * dtd * L; break;
    case COMB_RK4_K: { const double kk = dtd * L; Kout.B[c * g.cs + z] = kk; out = un + a.c * kk; } break;
    default:
      out = un + (1.0 / 6.0) * (K1.B[c * g.cs + z] + 2.0 * K2.B[c * g.cs + z] + 2.0 * K3.B[c * g.cs + z] + dtd * L);
      break;
    }
    Uout.B[c * g.cs + z] = out;
  }
}

#ifndef MGPU_UPDATE_MINB
#define MGPU_UPDATE_MINB 4   // 64 registers: chosen by a sweep of 3-4 (the natural count, 74, allows 3)
#endif

template <class T, int ND>
__global__ void __launch_bounds__(256, MGPU_UPDATE_MINB) k_update(Grid g, UpdateArgs a, StateCPtr<T> Un, StateCPtr<T> Us,
                                                const T *__restrict__ F, const T *__restrict__ G,
                                                const T *__restrict__ H, StatePtr<T> Uout, StatePtr<T> Kout,
                                                StateCPtr<T> K1, StateCPtr<T> K2, StateCPtr<T> K3,
                                                const Ctl *ctl, int stage)
{
  if (stage_failed(ctl, stage + 1)) return;
  const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.ninterior) return;
  update_zone<T, ND>(g, a, Un, Us, F, G, H, Uout, Kout, K1, K2, K3, ctl->dt, interior_zone(g, t));
}

}  // namespace mgpu
