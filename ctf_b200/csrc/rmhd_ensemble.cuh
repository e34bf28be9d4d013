// Ensembles of independent boxes of uneven size advanced together (no reference
// counterpart: the reference solver is a process-global singleton, Mara/mara.cpp:135).
//
// Every phase of the step (P->U, c2p, the flux sweeps, the CT + divergence + RK update) is one
// persistent launch over the concatenated work of all boxes: the work of box b is cut into
// tiles (`tile` consecutive interior zones, or faces of a sweep), the tiles of all boxes are
// numbered consecutively, and a map gives each tile its (box, tile-within-box).  Each CTA
// walks tiles w = blockIdx.x, +gridDim.x, ...; per tile it reads its map entry and stages
// the box's descriptor in shared memory (one coalesced copy), then runs the single-box
// kernels' device bodies (rmhd_step.cuh) on the tile.  A tile never spans two boxes, so a
// CTA's block-level reductions (MaxLambda) and its stage-failure early exit stay per box;
// each box keeps its own control block: its own dt, MaxLambda, error counts and commit.
#pragma once
#include "rmhd_step.cuh"

namespace mgpu {

static_assert(sizeof(BoxDev) % 8 == 0, "BoxDev is copied in 8-byte words");

// Stage box `src`'s descriptor in shared memory (all threads of the CTA call this).
__device__ __forceinline__ void load_box(BoxDev &sd, const BoxDev *src)
{
  __syncthreads();   // every thread is done with the previous tile's descriptor
  constexpr int W = (int) (sizeof(BoxDev) / 8);
  for (int i = threadIdx.x; i < W; i += blockDim.x)
    reinterpret_cast<long long *>(&sd)[i] = reinterpret_cast<const long long *>(src)[i];
  __syncthreads();
}

template <class T> __device__ __forceinline__ StatePtr<T> box_state(void *bulk, double *B) { return {(T *) bulk, B}; }
template <class T> __device__ __forceinline__ StateCPtr<T> box_cstate(void *bulk, double *B)
{
  return {(const T *) bulk, B};
}

// dt per box: the host's value (dt_mode 0) or cfl * min_dx / MaxLambda of its last advance.
static __global__ void k_ens_begin(const BoxDev *boxes, int nb, int dt_mode, const double *dt_in, double cfl)
{
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  Ctl *ctl = boxes[b].ctl;
  double dt = dt_in ? dt_in[b] : 0.0;
  if (dt_mode == 1) dt = cfl * boxes[b].min_dx / __longlong_as_double((long long) ctl->max_lambda_bits);
  ctl->dt = dt;
  ctl->max_lambda_bits = 0ull;
  for (int s = 0; s < MAX_STAGES; ++s) ctl->stage_err[s] = 0;
  ctl->final_err = 0;
  ctl->committed = 0;
  for (int i = 0; i < STAT_SLOTS; ++i) ctl->stat[i] = StatSlot{};
}

static __global__ void k_ens_commit(const BoxDev *boxes, int nb, int nstages, int commit)
{
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  Ctl *ctl = boxes[b].ctl;
  int e = 0;
  for (int s = 0; s < nstages; ++s) e |= ctl->stage_err[s];
  e |= ctl->final_err;
  if (e == 0 && commit) {
    ctl->cur ^= 1;
    ctl->committed = 1;
  }
}

template <class T>
__global__ void __launch_bounds__(256) k_ens_p2c(const BoxDev *boxes, const int2 *map, long long ntiles, int tile,
                                                 double gamma)
{
  __shared__ BoxDev d;
  for (long long w = blockIdx.x; w < ntiles; w += gridDim.x) {
    const int2 m = map[w];
    load_box(d, boxes + m.x);
    const long long base = (long long) m.y * tile;
    const int cur = d.ctl->cur;
    const StateCPtr<T> P = box_cstate<T>(d.b.Pc_bulk[cur], d.b.Pc_B[cur]);
    const StatePtr<T> U = box_state<T>(d.b.U0_bulk, d.b.U0_B);
    for (int s = threadIdx.x; s < tile; s += blockDim.x) {
      const long long t = base + s;
      if (t < d.g.ninterior) p2c_zone<T>(d.g, P, U, gamma, t);
    }
  }
}

// uin: 0 reads U0, 1 reads U1
template <class T>
__global__ void __launch_bounds__(128) k_ens_c2p(const BoxDev *boxes, const int2 *map, long long ntiles, int tile,
                                                 PhysParams pp, int stage, int uin, int zero_guess, int final,
                                                 int ereset, double preset, double dreset)
{
  __shared__ BoxDev d;
  for (long long w = blockIdx.x; w < ntiles; w += gridDim.x) {
    const int2 m = map[w];
    load_box(d, boxes + m.x);
    if (stage_failed(d.ctl, stage)) continue;   // uniform over the block
    const long long base = (long long) m.y * tile;
    const StateCPtr<T> U = uin ? box_cstate<T>(d.b.U1_bulk, d.b.U1_B) : box_cstate<T>(d.b.U0_bulk, d.b.U0_B);
    const int nxt = d.ctl->cur ^ 1;
    const StatePtr<T> Pn = box_state<T>(d.b.Pc_bulk[nxt], d.b.Pc_B[nxt]);
    for (int s = threadIdx.x; s < tile; s += blockDim.x) {
      const long long t = base + s;
      if (t < d.g.ninterior)
        c2p_zone<T>(d.g, U, (T *) d.b.PA, (const T *) d.b.PA, Pn, pp, d.ctl, stage, zero_guess, final, ereset, preset, dreset, t);
    }
  }
}

template <class T, int dim, int RS>
__global__ void __launch_bounds__(128, MGPU_FLUX_MINB) k_ens_flux(const BoxDev *boxes, const int2 *map,
                                                                  long long ntiles, int tile, PhysParams pp,
                                                                  int stage)
{
  __shared__ BoxDev d;
  constexpr bool hlld = RS == RIEMANN_HLLD;
  for (long long w = blockIdx.x; w < ntiles; w += gridDim.x) {
    const int2 m = map[w];
    load_box(d, boxes + m.x);
    if (stage_failed(d.ctl, stage + 1)) continue;   // uniform over the block
    const long long S = d.g.s[dim - 1];
    const long long base = 2 * S + (long long) m.y * tile;
    const long long end = d.g.nz - 3 * S;
    T ml = T(0);
    FluxTally ft{0, 0, 0, 0, 0};
    for (int s = threadIdx.x; s < tile; s += blockDim.x) {
      const long long f = base + s;
      if (f < end) flux_face<T, dim, RS>(d.g, (const T *) d.b.PA, (T *) d.b.F[dim - 1], pp, f, ml, ft);
    }
    flux_block_finish(double(ml), ft, d.ctl, hlld);
  }
}

// out: 0 writes U0, 1 writes U1; kout: -1 none, else K[kout] (RK4).  ND: the boxes' common
// dimensionality.  At least MGPU_ENS_UPDATE_MINB resident blocks (an HBM-bound kernel wants
// occupancy more than the loop-invariant box fields the compiler would otherwise hoist).
#ifndef MGPU_ENS_UPDATE_MINB
#define MGPU_ENS_UPDATE_MINB 4   // chosen by a sweep of 2-4
#endif
template <class T, int ND>
__global__ void __launch_bounds__(256, MGPU_ENS_UPDATE_MINB) k_ens_update(const BoxDev *boxes, const int2 *map, long long ntiles,
                                                    int tile, UpdateArgs a, int stage, int out, int kout)
{
  __shared__ BoxDev d;
  for (long long w = blockIdx.x; w < ntiles; w += gridDim.x) {
    const int2 m = map[w];
    load_box(d, boxes + m.x);
    if (stage_failed(d.ctl, stage + 1)) continue;
    const long long base = (long long) m.y * tile;
    const StateCPtr<T> U0 = box_cstate<T>(d.b.U0_bulk, d.b.U0_B), U1 = box_cstate<T>(d.b.U1_bulk, d.b.U1_B);
    const StatePtr<T> Uout = out ? box_state<T>(d.b.U1_bulk, d.b.U1_B) : box_state<T>(d.b.U0_bulk, d.b.U0_B);
    StatePtr<T> Kout{nullptr, nullptr};
    if (kout >= 0) Kout = box_state<T>(d.b.K_bulk[kout], d.b.K_B[kout]);
    const StateCPtr<T> K1 = box_cstate<T>(d.b.K_bulk[0], d.b.K_B[0]), K2 = box_cstate<T>(d.b.K_bulk[1], d.b.K_B[1]),
                       K3 = box_cstate<T>(d.b.K_bulk[2], d.b.K_B[2]);
    const double dt = d.ctl->dt;
    for (int s = threadIdx.x; s < tile; s += blockDim.x) {
      const long long t = base + s;
      if (t < d.g.ninterior)
        update_zone<T, ND>(d.g, a, U0, U1, (const T *) d.b.F[0], (const T *) d.b.F[1], (const T *) d.b.F[2], Uout,
                           Kout, K1, K2, K3, dt, interior_zone(d.g, t));
    }
  }
}

template <class T>
inline void launch_ens_flux(const EnsembleArgs &E, int d, int s)
{
#define MGPU_ENS_FLUX_CASE(D, R)                                                                             \
  if (d == D && E.pp.riemann == R) {                                                                         \
    k_ens_flux<T, D, R><<<E.grid_face, 128, 0, E.stream>>>(E.boxes, E.face_map[D - 1], E.face_tiles[D - 1], \
                                                           E.face_tile, E.pp, s);                            \
    return;                                                                                                  \
  }
  MGPU_ENS_FLUX_CASE(1, RIEMANN_HLLD) MGPU_ENS_FLUX_CASE(2, RIEMANN_HLLD) MGPU_ENS_FLUX_CASE(3, RIEMANN_HLLD)
  MGPU_ENS_FLUX_CASE(1, RIEMANN_HLLC) MGPU_ENS_FLUX_CASE(2, RIEMANN_HLLC) MGPU_ENS_FLUX_CASE(3, RIEMANN_HLLC)
  MGPU_ENS_FLUX_CASE(1, RIEMANN_HLL) MGPU_ENS_FLUX_CASE(2, RIEMANN_HLL) MGPU_ENS_FLUX_CASE(3, RIEMANN_HLL)
#undef MGPU_ENS_FLUX_CASE
}

template <class T>
inline cudaError_t launch_ensemble_advance(const EnsembleArgs &E)
{
  cudaStream_t st = E.stream;
  const int nb = E.nb;
  LaunchProfiler *pr = E.prof;
  {
    ProfScope ps(pr, st, KC_BEGIN, nb);
    k_ens_begin<<<(nb + 127) / 128, 128, 0, st>>>(E.boxes, nb, E.dt_mode, E.dt, E.cfl);
  }
  {
    ProfScope ps(pr, st, KC_P2C, E.total_zones);
    k_ens_p2c<T><<<E.grid_zone, 256, 0, st>>>(E.boxes, E.zone_map, E.zone_tiles, E.zone_tile, E.pp.gamma);
  }
  const int ns = num_stages(E.rk);
  for (int s = 0; s < ns; ++s) {
    {
      ProfScope ps(pr, st, KC_C2P, E.total_zones);
      k_ens_c2p<T><<<E.grid_c2p, 128, 0, st>>>(E.boxes, E.zone_map, E.zone_tiles, E.zone_tile, E.pp, s, s == 0 ? 0 : 1,
                                               s == 0, 0, E.ereset, E.preset, E.dreset);
    }
    for (int d = 1; d <= E.nd; ++d) {
      ProfScope ps(pr, st, KC_FLUX, E.total_faces[d - 1]);
      launch_ens_flux<T>(E, d, s);
    }
    const StageKind kind = stage_kind(E.rk, s);
    const UpdateArgs ua{kind.combine, kind.c};
    int out, kout = -1;
    if (E.rk == 4) {
      out = s == 3 ? 0 : 1;
      if (s < 3) kout = s;
    } else if (E.rk == 1) {
      out = 0;
    } else {
      out = (s == ns - 1) ? 0 : 1;
    }
    ProfScope ps(pr, st, KC_UPDATE, E.total_zones);
    if (E.nd == 1)
      k_ens_update<T, 1><<<E.grid_zone, 256, 0, st>>>(E.boxes, E.zone_map, E.zone_tiles, E.zone_tile, ua, s, out, kout);
    else if (E.nd == 2)
      k_ens_update<T, 2><<<E.grid_zone, 256, 0, st>>>(E.boxes, E.zone_map, E.zone_tiles, E.zone_tile, ua, s, out, kout);
    else
      k_ens_update<T, 3><<<E.grid_zone, 256, 0, st>>>(E.boxes, E.zone_map, E.zone_tiles, E.zone_tile, ua, s, out, kout);
  }
  {
    ProfScope ps(pr, st, KC_C2P, E.total_zones);
    k_ens_c2p<T><<<E.grid_c2p, 128, 0, st>>>(E.boxes, E.zone_map, E.zone_tiles, E.zone_tile, E.pp, ns, 0, 0, 1, E.ereset,
                                             E.preset, E.dreset);
  }
  {
    ProfScope ps(pr, st, KC_BEGIN, nb);
    k_ens_commit<<<(nb + 127) / 128, 128, 0, st>>>(E.boxes, nb, ns, E.commit);
  }
  return cudaGetLastError();
}

}  // namespace mgpu

#define MGPU_DEFINE_ENSEMBLE(suffix, T)                                                                  \
  namespace mgpu {                                                                                       \
  cudaError_t ensemble_advance_##suffix(const EnsembleArgs &E) { return launch_ensemble_advance<T>(E); } \
  }
