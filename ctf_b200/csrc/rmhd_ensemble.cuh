// Ensembles of independent boxes of uneven size advanced together (no reference
// counterpart: the reference solver is a process-global singleton, Mara/mara.cpp:135).
//
// Every phase of the step (P->U, c2p, the flux sweeps, the CT + divergence + RK update) is one
// persistent launch over the concatenated work of all boxes: the work of box b is cut into
// tiles (`tile` zones or faces), the tiles of all boxes are numbered consecutively
// (prefix[b] = first tile of box b), and each CTA walks tiles w = blockIdx.x, +gridDim.x, ...
// finding its box by binary search of the prefix array.  A tile never spans two boxes, so a
// CTA's block-level reductions (MaxLambda) and its stage-failure early exit stay per box.
// Each box keeps its own control block: its own dt, MaxLambda, error counts and commit.
// The per-item work is the single-box kernels' device bodies (rmhd_step.cuh).
#pragma once
#include "rmhd_step.cuh"

namespace mgpu {

__device__ __forceinline__ int find_box(const long long *prefix, int nb, long long w)
{
  int lo = 0, hi = nb;   // invariant: prefix[lo] <= w < prefix[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (prefix[mid] <= w) lo = mid;
    else hi = mid;
  }
  return lo;
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
  ctl->c2p_calls = ctl->c2p_iters = 0;
  for (int a = 0; a < 6; ++a) ctl->c2p_attempt[a] = 0;
  ctl->face_c2p_calls = ctl->face_c2p_iters = 0;
  ctl->hlld_ok = ctl->hlld_hllc = ctl->pcm_retry = 0;
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
__global__ void __launch_bounds__(256) k_ens_p2c(const BoxDev *boxes, const long long *prefix, int nb, int tile,
                                                 double gamma)
{
  const long long total = prefix[nb];
  for (long long w = blockIdx.x; w < total; w += gridDim.x) {
    const int bi = find_box(prefix, nb, w);
    const BoxDev &d = boxes[bi];
    const long long base = (w - prefix[bi]) * tile;
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
__global__ void __launch_bounds__(128) k_ens_c2p(const BoxDev *boxes, const long long *prefix, int nb, int tile,
                                                 PhysParams pp, int stage, int uin, int zero_guess, int final,
                                                 int ereset, double preset, double dreset)
{
  const long long total = prefix[nb];
  for (long long w = blockIdx.x; w < total; w += gridDim.x) {
    const int bi = find_box(prefix, nb, w);
    const BoxDev &d = boxes[bi];
    if (stage_failed(d.ctl, stage)) continue;
    const long long base = (w - prefix[bi]) * tile;
    const StateCPtr<T> U = uin ? box_cstate<T>(d.b.U1_bulk, d.b.U1_B) : box_cstate<T>(d.b.U0_bulk, d.b.U0_B);
    const int nxt = d.ctl->cur ^ 1;
    const StatePtr<T> Pn = box_state<T>(d.b.Pc_bulk[nxt], d.b.Pc_B[nxt]);
    for (int s = threadIdx.x; s < tile; s += blockDim.x) {
      const long long t = base + s;
      if (t < d.g.ninterior)
        c2p_zone<T>(d.g, U, (T *) d.b.PA, Pn, pp, d.ctl, stage, zero_guess, final, ereset, preset, dreset, t);
    }
  }
}

template <class T, int dim>
__global__ void __launch_bounds__(128, MGPU_FLUX_MINB) k_ens_flux(const BoxDev *boxes, const long long *prefix,
                                                                  int nb, int tile, PhysParams pp, int stage)
{
  const long long total = prefix[nb];
  const bool hlld = pp.riemann == RIEMANN_HLLD;
  for (long long w = blockIdx.x; w < total; w += gridDim.x) {
    const int bi = find_box(prefix, nb, w);
    const BoxDev &d = boxes[bi];
    if (stage_failed(d.ctl, stage + 1)) continue;   // uniform over the block: one box per tile
    const long long S = d.g.s[dim - 1];
    const long long base = 2 * S + (w - prefix[bi]) * tile;
    const long long end = d.g.nz - 3 * S;
    T ml = T(0);
    FluxTally ft{0, 0, 0, 0, 0};
    for (int s = threadIdx.x; s < tile; s += blockDim.x) {
      const long long f = base + s;
      if (f < end) flux_face<T, dim>(d.g, (const T *) d.b.PA, (T *) d.b.F[dim - 1], pp, f, ml, ft);
    }
    flux_block_finish(double(ml), ft, d.ctl, hlld);
  }
}

// out: 0 writes U0, 1 writes U1; kout: -1 none, else K[kout] (RK4)
template <class T>
__global__ void __launch_bounds__(256) k_ens_update(const BoxDev *boxes, const long long *prefix, int nb, int tile,
                                                    UpdateArgs a, int stage, int out, int kout)
{
  const long long total = prefix[nb];
  for (long long w = blockIdx.x; w < total; w += gridDim.x) {
    const int bi = find_box(prefix, nb, w);
    const BoxDev &d = boxes[bi];
    if (stage_failed(d.ctl, stage + 1)) continue;
    const long long base = (w - prefix[bi]) * tile;
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
        update_zone<T>(d.g, a, U0, U1, (const T *) d.b.F[0], (const T *) d.b.F[1], (const T *) d.b.F[2], Uout,
                       Kout, K1, K2, K3, dt, t);
    }
  }
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
    k_ens_p2c<T><<<E.grid_zone, 256, 0, st>>>(E.boxes, E.zone_prefix, nb, E.zone_tile, E.pp.gamma);
  }
  const int ns = num_stages(E.rk);
  for (int s = 0; s < ns; ++s) {
    {
      ProfScope ps(pr, st, KC_C2P, E.total_zones);
      k_ens_c2p<T><<<E.grid_c2p, 128, 0, st>>>(E.boxes, E.zone_prefix, nb, E.zone_tile, E.pp, s, s == 0 ? 0 : 1,
                                               s == 0, 0, E.ereset, E.preset, E.dreset);
    }
    for (int d = 1; d <= E.nd; ++d) {
      ProfScope ps(pr, st, KC_FLUX, E.total_faces[d - 1]);
      if (d == 1)
        k_ens_flux<T, 1><<<E.grid_face, 128, 0, st>>>(E.boxes, E.face_prefix[0], nb, E.face_tile, E.pp, s);
      else if (d == 2)
        k_ens_flux<T, 2><<<E.grid_face, 128, 0, st>>>(E.boxes, E.face_prefix[1], nb, E.face_tile, E.pp, s);
      else
        k_ens_flux<T, 3><<<E.grid_face, 128, 0, st>>>(E.boxes, E.face_prefix[2], nb, E.face_tile, E.pp, s);
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
    k_ens_update<T><<<E.grid_zone, 256, 0, st>>>(E.boxes, E.zone_prefix, nb, E.zone_tile, ua, s, out, kout);
  }
  {
    ProfScope ps(pr, st, KC_C2P, E.total_zones);
    k_ens_c2p<T><<<E.grid_c2p, 128, 0, st>>>(E.boxes, E.zone_prefix, nb, E.zone_tile, E.pp, ns, 0, 0, 1, E.ereset,
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
