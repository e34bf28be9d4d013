// Enqueues one advance (luaC_Mara_advance, Mara/mara.cpp:297-341) on a stream:
//   begin (dt, reset MaxLambda) -> P->U -> per RK stage: c2p | flux x,y,z | CT+div+combine
//   -> closing c2p into the uncommitted prim buffer -> commit if no zone failed.
// Nothing is read back: the host learns the outcome from the control block when it asks.
#pragma once
#include "rmhd_step.cuh"
#include "rmhd_step_tc.cuh"

#ifndef MGPU_TC_CTAS_PER_SM
#define MGPU_TC_CTAS_PER_SM 4
#endif

namespace mgpu {

template <class T>
inline cudaError_t launch_advance(const AdvanceArgs &A)
{
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

  const unsigned zb = 256, fb = 128;
  // learned guess on the tensor cores: persistent c2p kernel, MGPU_TC_CTAS_PER_SM CTAs per SM
  // (4 x 128 threads x 128 registers fill the register file)
  const bool tc_c2p = A.pp.learned && A.pp.mlp_tc;
  const bool simt_net = A.pp.learned && A.pp.mlp && !A.pp.mlp_tc;   // per-thread network guess
  const long long ntiles = (g.ninterior + 127) / 128;
  const long long tc_max = 148ll * MGPU_TC_CTAS_PER_SM;
  const unsigned tcgrid = (unsigned) (ntiles < tc_max ? ntiles : tc_max);
  auto c2p = [&](StateCPtr<T> Uin, int s, int zero_guess, int final) {
    if (tc_c2p)
      k_cons_to_prim_tc<T><<<tcgrid, 128, tc::SMEM_BYTES, st>>>(g, Uin, PA, Pc0, Pc1, A.pp, A.ctl, s, zero_guess,
                                                                final, A.ereset, A.preset, A.dreset);
    else if (simt_net)
      k_cons_to_prim<T, 0><<<(unsigned) ((g.ninterior + 127) / 128), 128, 0, st>>>(
          g, Uin, PA, Pc0, Pc1, A.pp, A.ctl, s, zero_guess, final, A.ereset, A.preset, A.dreset);
    else
      k_cons_to_prim<T, 2><<<(unsigned) ((g.ninterior + 127) / 128), 128, 0, st>>>(
          g, Uin, PA, Pc0, Pc1, A.pp, A.ctl, s, zero_guess, final, A.ereset, A.preset, A.dreset);
  };
  const unsigned zgrid = (unsigned) ((g.ninterior + zb - 1) / zb);

  LaunchProfiler *pr = A.prof;
  {
    ProfScope ps(pr, st, KC_BEGIN, 1);
    k_begin<<<1, 32, 0, st>>>(A.ctl, A.dt_mode, A.dt, A.cfl, A.min_dx);
  }
  {
    ProfScope ps(pr, st, KC_P2C, g.ninterior);
    k_prim_to_cons<T><<<zgrid, zb, 0, st>>>(g, cstate(b.Pc_bulk[0], b.Pc_B[0]), cstate(b.Pc_bulk[1], b.Pc_B[1]),
                                            U0, A.pp.gamma, A.ctl);
  }
  const int ns = num_stages(A.rk);
  for (int s = 0; s < ns; ++s) {
    const StatePtr<T> Uin = s == 0 ? U0 : U1;
    {
      ProfScope ps(pr, st, KC_C2P, g.ninterior);
      c2p(StateCPtr<T>{Uin.bulk, Uin.B}, s, s == 0, 0);
    }
    for (int d = 1; d <= g.nd; ++d) {
      const long long S = g.s[d - 1];
      const long long nf = g.nz - 5 * S;
      if (nf <= 0) continue;
      const unsigned fgrid = (unsigned) ((nf + fb - 1) / fb);
      ProfScope ps(pr, st, KC_FLUX, nf);
      if (d == 1) k_flux<T, 1><<<fgrid, fb, 0, st>>>(g, PA, (T *) b.F[0], A.pp, A.ctl, s);
      else if (d == 2) k_flux<T, 2><<<fgrid, fb, 0, st>>>(g, PA, (T *) b.F[1], A.pp, A.ctl, s);
      else k_flux<T, 3><<<fgrid, fb, 0, st>>>(g, PA, (T *) b.F[2], A.pp, A.ctl, s);
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
  }
  {
    ProfScope ps(pr, st, KC_C2P, g.ninterior);
    c2p(StateCPtr<T>{U0.bulk, U0.B}, ns, 0, 1);
  }
  {
    ProfScope ps(pr, st, KC_BEGIN, 1);
    k_commit<<<1, 32, 0, st>>>(A.ctl, ns);
  }
  return cudaGetLastError();
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
  k_aos_to_state<T><<<grid, blk, 0, A.stream>>>(A.g, d_aos, z0, count, StatePtr<T>{(T *) A.b.Pc_bulk[0], A.b.Pc_B[0]},
                                                StatePtr<T>{(T *) A.b.Pc_bulk[1], A.b.Pc_B[1]}, A.ctl);
  return cudaGetLastError();
}

template <class T>
inline cudaError_t launch_download(const TransferArgs &A, double *d_aos, long long z0, long long count)
{
  const unsigned blk = 256, grid = (unsigned) ((count + blk - 1) / blk);
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

}  // namespace mgpu

#define MGPU_DEFINE_PRECISION(suffix, T)                                                                  \
  namespace mgpu {                                                                                       \
  cudaError_t advance_##suffix(const AdvanceArgs &A) { return launch_advance<T>(A); }                   \
  cudaError_t upload_##suffix(const TransferArgs &A, const double *d_aos, long long z0, long long count) \
  { return launch_upload<T>(A, d_aos, z0, count); }                                                      \
  cudaError_t download_##suffix(const TransferArgs &A, double *d_aos, long long z0, long long count)     \
  { return launch_download<T>(A, d_aos, z0, count); }                                                    \
  cudaError_t face_io_##suffix(const TransferArgs &A, double *d_aos, long long z0, long long count, int to_aos) \
  { return launch_face_io<T>(A, d_aos, z0, count, to_aos); }                                             \
  }
