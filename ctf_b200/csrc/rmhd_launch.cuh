// Enqueues one advance (luaC_Mara_advance, Mara/mara.cpp:297-341) on a stream:
//   begin (dt, reset MaxLambda) -> P->U -> per RK stage: c2p | flux x,y,z | CT+div+combine
//   -> closing c2p into the uncommitted prim buffer -> commit if no zone failed.
// With the CTU-Hancock operator a stage is c2p | CTU passes (rmhd_ctu.cuh) | CT+div+combine.
// Nothing is read back: the host learns the outcome from the control block when it asks.
#pragma once
#include <algorithm>
#include "rmhd_step.cuh"
#include "rmhd_step_tc.cuh"
#include "rmhd_ctu.cuh"
#include "rmhd_lean.cuh"
#include "rmhd_diffuse.cuh"

#ifndef MGPU_TC_CTAS_PER_SM
#define MGPU_TC_CTAS_PER_SM 4
#endif
#ifndef MGPU_TC_SPLIT
#define MGPU_TC_SPLIT 1   // learned c2p as network kernel + polish kernel (0: one fused kernel)
#endif

namespace mgpu {
// The learned c2p over the grid's window: the split network + polish kernels with the guesses
// in `scratch` (a face array, idle while a whole-domain c2p runs, or an array of its own, one
// float2 per interior zone), or the fused kernel.
template <class T>
inline void launch_learned_c2p(const Grid &g, cudaStream_t st, StateCPtr<T> U, T *PA, const T *PAg, StatePtr<T> Pn0,
                               StatePtr<T> Pn1, const PhysParams &pp, Ctl *ctl, int s, int zero_guess, int mode,
                               int ereset, double preset, double dreset, void *scratch)
{
  const long long ntiles = (win_tend(g) - win_tbeg(g) + 127) / 128;
  if (MGPU_TC_SPLIT) {
    const long long nmax = 148ll * MGPU_TCNET_CTAS_PER_SM;
    float2 *guess = (float2 *) scratch;
    k_c2p_guess_tc<T><<<(unsigned) (ntiles < nmax ? ntiles : nmax), 128, tc::SMEM_BYTES, st>>>(g, U, Pn0, Pn1, pp,
                                                                                               ctl, s, mode, guess);
    k_cons_to_prim_guessed<T><<<(unsigned) ntiles, 128, 0, st>>>(g, U, PA, PAg, Pn0, Pn1, pp, ctl, s, zero_guess, mode,
                                                               ereset, preset, dreset, guess);
  } else {
    const long long tmax = 148ll * MGPU_TC_CTAS_PER_SM;
    k_cons_to_prim_tc<T><<<(unsigned) (ntiles < tmax ? ntiles : tmax), 128, tc::SMEM_BYTES, st>>>(
        g, U, PA, PAg, Pn0, Pn1, pp, ctl, s, zero_guess, mode, ereset, preset, dreset);
  }
}
}  // namespace mgpu

namespace mgpu {

// One sweep: the flux kernel for (sweep direction, Riemann solver), both compile-time.
template <class T>
inline void launch_flux(const Grid &g, int d, int rs, unsigned grid, unsigned blk, cudaStream_t st, const T *PA,
                        T *F, const PhysParams &pp, Ctl *ctl, int s)
{
#define MGPU_FLUX_CASE(D, R)                                                            \
  if (d == D && rs == R) {                                                              \
    k_flux<T, D, R><<<grid, blk, 0, st>>>(g, PA, F, pp, ctl, s);                        \
    return;                                                                             \
  }
  MGPU_FLUX_CASE(1, RIEMANN_HLLD) MGPU_FLUX_CASE(2, RIEMANN_HLLD) MGPU_FLUX_CASE(3, RIEMANN_HLLD)
  MGPU_FLUX_CASE(1, RIEMANN_HLLC) MGPU_FLUX_CASE(2, RIEMANN_HLLC) MGPU_FLUX_CASE(3, RIEMANN_HLLC)
  MGPU_FLUX_CASE(1, RIEMANN_HLL) MGPU_FLUX_CASE(2, RIEMANN_HLL) MGPU_FLUX_CASE(3, RIEMANN_HLL)
#undef MGPU_FLUX_CASE
}


// The phases of an advance in the lean layout (rmhd_lean.cuh): no P->U (the committed state
// is conserved), no c2p at the first stage, sweeps that accumulate into U[!cur], CT from the
// stored face fields, and after the commit a restore c2p that runs only if nothing committed.
template <class T>
inline cudaError_t launch_lean_phase(const AdvanceArgs &A, int phase, int s)
{
  const Grid &g = A.g;
  const AdvanceBuffers &b = A.b;
  cudaStream_t st = A.stream;
  const StatePtr<T> UA{(T *) b.U0_bulk, b.U0_B}, UB{(T *) b.U1_bulk, b.U1_B};
  T *PA = (T *) b.PA;
  const T *PAg = b.PAg ? (const T *) b.PAg : PA;   // the stage c2p's previous primitives
  T *Bf = (T *) b.Bf;
  const int ns = num_stages(A.rk);
  LaunchProfiler *pr = A.prof;
  // zone launches cover the grid's window of x rows (the whole interior by default)
  const long long nwin = win_tend(g) - win_tbeg(g);
  const unsigned cgrid = (unsigned) ((nwin + 127) / 128);
  const StateCPtr<T> none{nullptr, nullptr};
  auto c2p = [&](int mode, int zero_guess, bool learned) {
    ProfScope ps(pr, st, KC_C2P, nwin);
    if (learned) {
      launch_learned_c2p<T>(g, st, none, PA, PAg, UA, UB, A.pp, A.ctl, s, zero_guess, mode, A.ereset, A.preset,
                            A.dreset, b.guess ? b.guess : b.Bf);
    } else {
      k_cons_to_prim<T, 2><<<cgrid, 128, 0, st>>>(g, none, PA, PAg, UA, UB, A.pp, A.ctl, s, zero_guess, mode,
                                                   A.ereset, A.preset, A.dreset);
    }
  };
  const bool learned = A.pp.learned && A.pp.mlp_tc;
  if (phase == PH_BEGIN) {
    ProfScope ps(pr, st, KC_BEGIN, 1);
    k_begin<<<1, 32, 0, st>>>(A.ctl, A.dt_mode, A.dt, A.cfl, A.min_dx);
  } else if (phase == PH_C2P) {
    if (s > 0) c2p(s == ns ? C2P_LEAN_CLOSING : C2P_LEAN_STAGE, 0, learned);
  } else if (phase == PH_C2P_SHELL || phase == PH_C2P_CORE) {
    // a stage's c2p by region (decomposed blocks); the first stage has none
    if (s == 0) return cudaGetLastError();
    if (learned) {
      if (phase == PH_C2P_SHELL) c2p(C2P_LEAN_STAGE, 0, true);
      return cudaGetLastError();
    }
    ProfScope ps(pr, st, KC_C2P, g.ninterior);
    k_cons_to_prim_region<T><<<cgrid, 128, 0, st>>>(g, none, PA, UA, UB, A.pp, A.ctl, s, 0, C2P_LEAN_STAGE, A.ereset,
                                                     A.preset, A.dreset, phase == PH_C2P_SHELL ? 1 : 2);
  } else if (phase == PH_FLUX_UPDATE) {
    const StageKind kind = stage_kind(A.rk, s);
    const LeanCombine c = lean_combine(kind.combine);
    for (int d = 1; d <= 3; ++d) {
      ProfScope ps(pr, st, KC_FLUX, nwin);
      launch_lean_sweep<T>(g, d, A.pp.riemann, st, PA, UA, UB, Bf, c, A.pp, A.ctl, s);
    }
    ProfScope ps(pr, st, KC_UPDATE, nwin);
    const unsigned zb = 256;
    k_lean_ct<T><<<(unsigned) ((lean_ct_threads(g) + zb - 1) / zb), zb, 0, st>>>(
        g, kind.combine, UA, UB, Bf, A.ctl, s, make_double3(1.0 / g.dx, 1.0 / g.dy, 1.0 / g.dz));
  } else if (phase == PH_COMMIT) {
    {
      ProfScope ps(pr, st, KC_BEGIN, 1);
      k_commit<<<1, 32, 0, st>>>(A.ctl, ns);
    }
    c2p(C2P_LEAN_RESTORE, 1, false);
  }
  return cudaGetLastError();
}

template <class T>
inline cudaError_t launch_phase(const AdvanceArgs &A, int phase, int s)
{
  if (A.lean) return launch_lean_phase<T>(A, phase, s);
  const Grid &g = A.g;
  const AdvanceBuffers &b = A.b;
  cudaStream_t st = A.stream;
  auto state = [&](void *bulk, double *B) { return StatePtr<T>{(T *) bulk, B}; };
  auto cstate = [&](void *bulk, double *B) { return StateCPtr<T>{(const T *) bulk, B}; };
  const StatePtr<T> Pc0 = state(b.Pc_bulk[0], b.Pc_B[0]), Pc1 = state(b.Pc_bulk[1], b.Pc_B[1]);
  const StatePtr<T> U0 = state(b.U0_bulk, b.U0_B), U1 = state(b.U1_bulk, b.U1_B);
  StatePtr<T> K[3];
  for (int i = 0; i < 3; ++i) K[i] = state(b.K_bulk[i], b.K_B[i]);
  T *PA = (T *) b.PA;
  const T *F = (const T *) b.F[0], *G = (const T *) b.F[1], *H = (const T *) b.F[2];
  const int ns = num_stages(A.rk);

  const unsigned zb = 256, fb = 128;
  const unsigned zgrid = (unsigned) ((g.ninterior + zb - 1) / zb);
  LaunchProfiler *pr = A.prof;

  if (phase == PH_BEGIN) {
    {
      ProfScope ps(pr, st, KC_BEGIN, 1);
      k_begin<<<1, 32, 0, st>>>(A.ctl, A.dt_mode, A.dt, A.cfl, A.min_dx);
    }
    ProfScope ps(pr, st, KC_P2C, g.ninterior);
    k_prim_to_cons<T><<<zgrid, zb, 0, st>>>(g, cstate(b.Pc_bulk[0], b.Pc_B[0]), cstate(b.Pc_bulk[1], b.Pc_B[1]),
                                            U0, A.pp.gamma, A.ctl);
  } else if (phase == PH_C2P_SHELL || phase == PH_C2P_CORE) {
    const int final = A.godunov ? 2 : 0;
    const StateCPtr<T> Uin = s == 0 ? StateCPtr<T>{U0.bulk, U0.B} : StateCPtr<T>{U1.bulk, U1.B};
    const bool learned = A.pp.learned && (A.pp.mlp_tc || A.pp.mlp);
    if (learned) {   // the learned guess converts the whole interior in one pass: no split
      if (phase == PH_C2P_SHELL) return launch_phase<T>(A, PH_C2P, s);
      return cudaGetLastError();
    }
    ProfScope ps(pr, st, KC_C2P, g.ninterior);
    k_cons_to_prim_region<T><<<(unsigned) ((g.ninterior + 127) / 128), 128, 0, st>>>(
        g, Uin, PA, Pc0, Pc1, A.pp, A.ctl, s, s == 0, final, A.ereset, A.preset, A.dreset,
        phase == PH_C2P_SHELL ? 1 : 2);
  } else if (phase == PH_C2P) {
    // stage s < ns reads the stage input (U0 first, U1 after) into PA; s == ns is the
    // closing c2p of U0 into the uncommitted primitive buffer
    // final: 1 closing c2p, 2 CTU-Hancock stage c2p (failures do not abort), 0 stage c2p
    const int final = s == ns ? 1 : A.godunov ? 2 : 0;
    const StateCPtr<T> Uin = (s == 0 || final == 1) ? StateCPtr<T>{U0.bulk, U0.B} : StateCPtr<T>{U1.bulk, U1.B};
    const int zero_guess = s == 0;
    // learned guess on the tensor cores (launch_learned_c2p; its guesses go to F[0], idle here)
    const bool tc_c2p = A.pp.learned && A.pp.mlp_tc;
    const bool simt_net = A.pp.learned && A.pp.mlp && !A.pp.mlp_tc;   // per-thread network guess
    ProfScope ps(pr, st, KC_C2P, g.ninterior);
    if (tc_c2p)
      launch_learned_c2p<T>(g, st, Uin, PA, PA, Pc0, Pc1, A.pp, A.ctl, s, zero_guess, final, A.ereset, A.preset,
                            A.dreset, b.F[0]);
    else if (simt_net)
      k_cons_to_prim<T, 0><<<(unsigned) ((g.ninterior + 127) / 128), 128, 0, st>>>(
          g, Uin, PA, PA, Pc0, Pc1, A.pp, A.ctl, s, zero_guess, final, A.ereset, A.preset, A.dreset);
    else
      k_cons_to_prim<T, 2><<<(unsigned) ((g.ninterior + 127) / 128), 128, 0, st>>>(
          g, Uin, PA, PA, Pc0, Pc1, A.pp, A.ctl, s, zero_guess, final, A.ereset, A.preset, A.dreset);
  } else if (phase == PH_FLUX_UPDATE) {
    if (A.godunov)
      launch_ctu_stage<T>(A, s, s == 0 ? StateCPtr<T>{U0.bulk, U0.B} : StateCPtr<T>{U1.bulk, U1.B});
    for (int d = 1; d <= g.nd && !A.godunov; ++d) {
      const long long S = g.s[d - 1];
      const long long nf = g.nz - 5 * S;
      if (nf <= 0) continue;
      const unsigned fgrid = (unsigned) ((nf + fb - 1) / fb);
      ProfScope ps(pr, st, KC_FLUX, nf);
      launch_flux<T>(g, d, A.pp.riemann, fgrid, fb, st, PA, (T *) b.F[d - 1], A.pp, A.ctl, s);
    }
    const StageKind kind = stage_kind(A.rk, s);
    UpdateArgs ua{kind.combine, kind.c};
    StatePtr<T> Uout, Kout{nullptr, nullptr};
    if (A.rk == 4) {
      Uout = s == 3 ? U0 : U1;
      if (s < 3) Kout = K[s];
    } else if (A.rk == 1) {
      Uout = U0;
    } else {
      Uout = (s == ns - 1) ? U0 : U1;
    }
    ProfScope ps(pr, st, KC_UPDATE, g.ninterior);
    const StateCPtr<T> cU0{U0.bulk, U0.B}, cU1{U1.bulk, U1.B}, cK0{K[0].bulk, K[0].B}, cK1{K[1].bulk, K[1].B},
        cK2{K[2].bulk, K[2].B};
    if (g.nd == 1)
      k_update<T, 1><<<zgrid, zb, 0, st>>>(g, ua, cU0, cU1, F, G, H, Uout, Kout, cK0, cK1, cK2, A.ctl, s);
    else if (g.nd == 2)
      k_update<T, 2><<<zgrid, zb, 0, st>>>(g, ua, cU0, cU1, F, G, H, Uout, Kout, cK0, cK1, cK2, A.ctl, s);
    else
      k_update<T, 3><<<zgrid, zb, 0, st>>>(g, ua, cU0, cU1, F, G, H, Uout, Kout, cK0, cK1, cK2, A.ctl, s);
  } else if (phase == PH_COMMIT) {
    ProfScope ps(pr, st, KC_BEGIN, 1);
    k_commit<<<1, 32, 0, st>>>(A.ctl, ns);
  }
  return cudaGetLastError();
}

template <class T>
inline cudaError_t launch_advance(const AdvanceArgs &A)
{
  const int ns = num_stages(A.rk);
  cudaError_t e = launch_phase<T>(A, PH_BEGIN, 0);
  for (int s = 0; s < ns && e == cudaSuccess; ++s) {
    e = launch_phase<T>(A, PH_C2P, s);
    if (e == cudaSuccess) e = launch_phase<T>(A, PH_FLUX_UPDATE, s);
  }
  if (e == cudaSuccess) e = launch_phase<T>(A, PH_C2P, ns);
  if (e == cudaSuccess) e = launch_phase<T>(A, PH_COMMIT, 0);
  return e;
}

// AoS (host reference layout, 8 doubles per zone) <-> state arrays.
template <class T>
__global__ void k_aos_to_state(Grid g, const double *__restrict__ aos, long long z0, long long count,
                               StatePtr<T> P0, StatePtr<T> P1, const Ctl *ctl)
{
  const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const long long z = z0 + t;
  const StatePtr<T> P = ctl->cur ? P1 : P0;
  const double *a = aos + t * 8;
#pragma unroll
  for (int c = 0; c < 5; ++c) P.bulk[c * g.cs + z] = T(a[c]);
#pragma unroll
  for (int c = 0; c < 3; ++c) P.B[c * g.cs + z] = a[5 + c];
}

template <class T>
__global__ void k_state_to_aos(Grid g, double *__restrict__ aos, long long z0, long long count,
                               StateCPtr<T> P0, StateCPtr<T> P1, const Ctl *ctl)
{
  const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const long long z = z0 + t;
  const StateCPtr<T> P = ctl->cur ? P1 : P0;
  double *a = aos + t * 8;
#pragma unroll
  for (int c = 0; c < 5; ++c) a[c] = double(P.bulk[c * g.cs + z]);
#pragma unroll
  for (int c = 0; c < 3; ++c) a[5 + c] = P.B[c * g.cs + z];
}

// Face array (8 x T, e.g. the stage prims PA) -> AoS
template <class T>
__global__ void k_face_to_aos(Grid g, double *__restrict__ aos, long long z0, long long count, const T *PA)
{
  const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const long long z = z0 + t;
#pragma unroll
  for (int c = 0; c < 8; ++c) aos[t * 8 + c] = double(PA[c * g.cs + z]);
}

template <class T>
__global__ void k_aos_to_face(Grid g, const double *__restrict__ aos, long long z0, long long count, T *PA)
{
  const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const long long z = z0 + t;
#pragma unroll
  for (int c = 0; c < 8; ++c) PA[c * g.cs + z] = T(aos[t * 8 + c]);
}

template <class T>
inline cudaError_t launch_upload(const TransferArgs &A, const double *d_aos, long long z0, long long count)
{
  const unsigned blk = 256, grid = (unsigned) ((count + blk - 1) / blk);
  if (A.lean) {
    k_lean_upload<T><<<grid, blk, 0, A.stream>>>(A.g, d_aos, z0, count, (T *) A.b.PA,
                                                 StatePtr<T>{(T *) A.b.U0_bulk, A.b.U0_B},
                                                 StatePtr<T>{(T *) A.b.U1_bulk, A.b.U1_B}, A.gamma, A.ctl);
    return cudaGetLastError();
  }
  k_aos_to_state<T><<<grid, blk, 0, A.stream>>>(A.g, d_aos, z0, count, StatePtr<T>{(T *) A.b.Pc_bulk[0], A.b.Pc_B[0]},
                                                StatePtr<T>{(T *) A.b.Pc_bulk[1], A.b.Pc_B[1]}, A.ctl);
  return cudaGetLastError();
}

template <class T>
inline cudaError_t launch_download(const TransferArgs &A, double *d_aos, long long z0, long long count)
{
  const unsigned blk = 256, grid = (unsigned) ((count + blk - 1) / blk);
  if (A.lean) {
    k_lean_download<T><<<grid, blk, 0, A.stream>>>(A.g, d_aos, z0, count, (const T *) A.b.PA,
                                                   StateCPtr<T>{(const T *) A.b.U0_bulk, A.b.U0_B},
                                                   StateCPtr<T>{(const T *) A.b.U1_bulk, A.b.U1_B}, A.ctl,
                                                   A.pending);
    return cudaGetLastError();
  }
  k_state_to_aos<T><<<grid, blk, 0, A.stream>>>(A.g, d_aos, z0, count,
                                                StateCPtr<T>{(const T *) A.b.Pc_bulk[0], A.b.Pc_B[0]},
                                                StateCPtr<T>{(const T *) A.b.Pc_bulk[1], A.b.Pc_B[1]}, A.ctl);
  return cudaGetLastError();
}

template <class T>
inline cudaError_t launch_face_io(const TransferArgs &A, double *d_aos, long long z0, long long count, int to_aos)
{
  const unsigned blk = 256, grid = (unsigned) ((count + blk - 1) / blk);
  if (to_aos) k_face_to_aos<T><<<grid, blk, 0, A.stream>>>(A.g, d_aos, z0, count, (const T *) A.b.PA);
  else k_aos_to_face<T><<<grid, blk, 0, A.stream>>>(A.g, d_aos, z0, count, (T *) A.b.PA);
  return cudaGetLastError();
}

// ---- halo slabs of a decomposed domain ------------------------------------------------------
// A slab is Ng layers of dimension `dim` over the full guarded cross-section of the other two
// dimensions (so that exchanging dimensions in order x, y, z fills edges and corners as the
// reference's sequential Synchronize does, Mara/subgrids.cpp:12-116).  Buffer layout:
// [component][layer][cross-section index], the cross-section in zone order.
__device__ __forceinline__ long long slab_zone(const Grid &g, int dim, int layer, long long c)
{
  if (dim == 0) return (long long) layer * g.s[0] + c;   // c = j*G2 + k
  if (dim == 1) {                                        // c = i*G2 + k
    const long long i = c / g.G[2], k = c - i * g.G[2];
    return i * g.s[0] + (long long) layer * g.s[1] + k;
  }
  const long long i = c / g.G[1], j = c - i * g.G[1];   // c = i*G1 + j
  return i * g.s[0] + j * g.s[1] + layer;
}

__host__ __device__ inline long long slab_cross(const Grid &g, int dim)
{
  return dim == 0 ? (long long) g.G[1] * g.G[2] : dim == 1 ? (long long) g.G[0] * g.G[2] : (long long) g.G[0] * g.G[1];
}

// to_buf 1: A[q][layers first..first+ng) -> buf; 0: buf -> A.  A has ncomp components of E.
template <class E>
__global__ void k_halo_copy(Grid g, E *A, int ncomp, int dim, int first, E *buf, int to_buf)
{
  const long long cross = slab_cross(g, dim);
  const long long per = cross * g.ng;
  const long long total = per * ncomp;
  for (long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long) gridDim.x * blockDim.x) {
    const int q = (int) (t / per);
    const long long r = t - q * per;
    const int layer = (int) (r / cross);
    const long long c = r - (long long) layer * cross;
    const long long z = slab_zone(g, dim, first + layer, c);
    if (to_buf) buf[t] = A[q * g.cs + z];
    else A[q * g.cs + z] = buf[t];
  }
}

// which 0: the stage primitives PA (8 x T); 1: the committed state (5 x T, then 3 x double).
// side 0: the low slab (pack: interior layers [ng, 2ng) for the low neighbour; unpack: guard
// layers [0, ng)); side 1: the high slab (pack: [n, n + ng); unpack: [n + ng, n + 2ng)).
template <class T>
inline cudaError_t launch_halo(const TransferArgs &A, int which, int dim, int side, void *buf, int pack)
{
  const Grid &g = A.g;
  const int n = g.n[dim], ng = g.ng;
  const int first = pack ? (side == 0 ? ng : n) : (side == 0 ? 0 : n + ng);
  const long long per = slab_cross(g, dim) * ng;
  const unsigned blk = 256;
  const unsigned grid = (unsigned) std::min<long long>((per * 8 + blk - 1) / blk, 148ll * 16);
  if (which == 0) {
    k_halo_copy<T><<<grid, blk, 0, A.stream>>>(g, (T *) A.b.PA, 8, dim, first, (T *) buf, pack);
  } else {
    // the committed buffer is chosen on the host (it read ctl->cur after a synchronize)
    const int cur = A.cur;
    k_halo_copy<T><<<grid, blk, 0, A.stream>>>(g, (T *) A.b.Pc_bulk[cur], 5, dim, first, (T *) buf, pack);
    k_halo_copy<double><<<grid, blk, 0, A.stream>>>(g, A.b.Pc_B[cur], 3, dim, first,
                                                    (double *) ((char *) buf + per * 5 * sizeof(T)), pack);
  }
  return cudaGetLastError();
}

}  // namespace mgpu

#define MGPU_DEFINE_PRECISION(suffix, T)                                                                  \
  namespace mgpu {                                                                                       \
  cudaError_t advance_##suffix(const AdvanceArgs &A) { return launch_advance<T>(A); }                   \
  cudaError_t phase_##suffix(const AdvanceArgs &A, int phase, int s) { return launch_phase<T>(A, phase, s); } \
  cudaError_t upload_##suffix(const TransferArgs &A, const double *d_aos, long long z0, long long count) \
  { return launch_upload<T>(A, d_aos, z0, count); }                                                      \
  cudaError_t download_##suffix(const TransferArgs &A, double *d_aos, long long z0, long long count)     \
  { return launch_download<T>(A, d_aos, z0, count); }                                                    \
  cudaError_t face_io_##suffix(const TransferArgs &A, double *d_aos, long long z0, long long count, int to_aos) \
  { return launch_face_io<T>(A, d_aos, z0, count, to_aos); }                                             \
  cudaError_t halo_##suffix(const TransferArgs &A, int which, int dim, int side, void *buf, int pack)     \
  { return launch_halo<T>(A, which, dim, side, buf, pack); }                                             \
  cudaError_t diffuse_##suffix(const AdvanceArgs &A, double r) { return launch_diffuse<T>(A, r); }       \
  }
