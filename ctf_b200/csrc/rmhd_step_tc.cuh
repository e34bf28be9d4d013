// The zone c2p kernel with the learned initial guess evaluated on the tensor cores.
//
// Persistent: each CTA sets up the network image, TMEM and its mbarrier once, then walks
// tiles of 128 interior zones.  Per tile the 128 threads stage their zones' features, the
// CTA runs the four MMA layers (c2p_mlp_tc.cuh), and each thread polishes its own zone with
// the FP64 Newton iteration from the network's (Z, W) -- the reference's ladder follows when
// that attempt fails -- then scatters the primitives to the zone's guard images, exactly as
// k_cons_to_prim does.
#pragma once
#include "c2p_mlp_tc.cuh"
#include "rmhd_step.cuh"

namespace mgpu {

#ifndef MGPU_TC_CTAS_PER_SM
#define MGPU_TC_CTAS_PER_SM 4
#endif

template <class T>
__global__ void __launch_bounds__(128, MGPU_TC_CTAS_PER_SM) k_cons_to_prim_tc(Grid g, StateCPtr<T> U, T *PA, const T *PAg, StatePtr<T> Pn0,
                                                         StatePtr<T> Pn1, PhysParams pp, Ctl *ctl, int stage,
                                                         int zero_guess, int final, int ereset, double preset,
                                                         double dreset)
{
  if (c2p_skip(ctl, stage, final)) return;
  extern __shared__ unsigned char tc_smem[];
  tc::TcNet net = tc::tc_setup(tc_smem, (const unsigned char *) pp.mlp_tc);
  U = c2p_input(ctl, final, U, Pn0, Pn1);
  const long long tb = win_tbeg(g), te = win_tend(g);
  const long long ntiles = (te - tb + 127) / 128;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long t = tb + tile * 128 + threadIdx.x;
    const bool valid = t < te;
    int i = 0, j = 0, k = 0;
    long long z = 0;
    double u[8], p[8];
    float xn[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    bool good = false;
    if (valid) {
      interior_coords(g, t, i, j, k);
      z = ((long long) i * g.G[1] + j) * g.G[2] + k;
      load_state(g, U, z, u);
      if (check_cons(u) == C2P_SUCCESS) {
        const double S2 = u[Sx] * u[Sx] + u[Sy] * u[Sy] + u[Sz] * u[Sz];
        const double B2 = u[Bx] * u[Bx] + u[By] * u[By] + u[Bz] * u[Bz];
        const double BS = u[Bx] * u[Sx] + u[By] * u[Sy] + u[Bz] * u[Sz];
        float x[5];
        c2p_features_f32(u[ddd], u[tau], S2, B2, BS * BS, x);
        net.normalise(x, xn);
        good = isfinite(xn[0]) && isfinite(xn[1]) && isfinite(xn[2]) && isfinite(xn[3]) && isfinite(xn[4]);
        if (!good) xn[0] = xn[1] = xn[2] = xn[3] = xn[4] = 0.f;
      }
    }
    float y[2];
    const bool have = net.forward(xn, y);
    if (!valid) continue;
    double Zg = 0.0, Wg = 0.0;
    const bool use = have && good && c2p_guess_from_output_f32(u[ddd], y, Zg, Wg);
    C2PTally tally;
    // the previous primitives are read only when the ladder needs them or a failure keeps them
    const auto prev = [&](double *q) {
#pragma unroll
      for (int c = 0; c < 8; ++c) q[c] = zero_guess ? 0.0 : double(PAg[c * g.cs + z]);
    };
    const int err = cons_to_prim<(sizeof(T) < sizeof(double)), 1>(pp, u, p, &tally, Zg, Wg, use, prev) != 0;
    c2p_finish<T>(g, PA, ctl->cur ? Pn0 : Pn1, ctl, stage, final, ereset, preset, dreset, i, j, k, u, p, err,
                  tally);
  }
  if (!net.ok && threadIdx.x == 0) atomicExch(&ctl->tc_fault, 1);
  tc::tc_teardown(net);
}

// Split form (MGPU_TC_SPLIT): k_c2p_guess_tc runs the tile loop above without the polish --
// features, the four MMA layers, and the two raw network outputs of every interior zone into
// `guess` (-1, -1 where there is no guess) -- and k_cons_to_prim_guessed then polishes one zone
// per thread from them, at the plain c2p kernel's occupancy.  The network kernel holds no
// per-zone state across the layers, so more CTAs fit per SM.
#ifndef MGPU_TCNET_CTAS_PER_SM
#define MGPU_TCNET_CTAS_PER_SM 5
#endif

template <class T>
__global__ void __launch_bounds__(128, MGPU_TCNET_CTAS_PER_SM) k_c2p_guess_tc(Grid g, StateCPtr<T> U, StatePtr<T> Pn0,
                                                                            StatePtr<T> Pn1, PhysParams pp, Ctl *ctl,
                                                                            int stage, int final, float2 *guess)
{
  if (c2p_skip(ctl, stage, final)) return;
  extern __shared__ unsigned char tc_smem[];
  tc::TcNet net = tc::tc_setup(tc_smem, (const unsigned char *) pp.mlp_tc);
  U = c2p_input(ctl, final, U, Pn0, Pn1);
  const long long tb = win_tbeg(g), te = win_tend(g);
  const long long ntiles = (te - tb + 127) / 128;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long t = tb + tile * 128 + threadIdx.x;
    const bool valid = t < te;
    float xn[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    bool good = false;
    if (valid) {
      int i, j, k;
      interior_coords(g, t, i, j, k);
      const long long z = ((long long) i * g.G[1] + j) * g.G[2] + k;
      double u[8];
      load_state(g, U, z, u);
      if (check_cons(u) == C2P_SUCCESS) {
        const double S2 = u[Sx] * u[Sx] + u[Sy] * u[Sy] + u[Sz] * u[Sz];
        const double B2 = u[Bx] * u[Bx] + u[By] * u[By] + u[Bz] * u[Bz];
        const double BS = u[Bx] * u[Sx] + u[By] * u[Sy] + u[Bz] * u[Sz];
        float x[5];
        c2p_features_f32(u[ddd], u[tau], S2, B2, BS * BS, x);
        net.normalise(x, xn);
        good = isfinite(xn[0]) && isfinite(xn[1]) && isfinite(xn[2]) && isfinite(xn[3]) && isfinite(xn[4]);
        if (!good) xn[0] = xn[1] = xn[2] = xn[3] = xn[4] = 0.f;
      }
    }
    float y[2];
    const bool have = net.forward(xn, y);
    if (valid) guess[t] = (have && good) ? make_float2(y[0], y[1]) : make_float2(-1.f, -1.f);
  }
  if (!net.ok && threadIdx.x == 0) atomicExch(&ctl->tc_fault, 1);
  tc::tc_teardown(net);
}

template <class T>
__global__ void __launch_bounds__(128, MGPU_C2P_MINB) k_cons_to_prim_guessed(Grid g, StateCPtr<T> U, T *PA, const T *PAg,
                                                                           StatePtr<T> Pn0, StatePtr<T> Pn1,
                                                                           PhysParams pp, Ctl *ctl, int stage,
                                                                           int zero_guess, int final, int ereset,
                                                                           double preset, double dreset,
                                                                           const float2 *guess)
{
  if (c2p_skip(ctl, stage, final)) return;
  const long long t = win_tbeg(g) + (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= win_tend(g)) return;
  const StateCPtr<T> Uz = c2p_input(ctl, final, U, Pn0, Pn1);
  int i, j, k;
  interior_coords(g, t, i, j, k);
  const long long z = ((long long) i * g.G[1] + j) * g.G[2] + k;
  double u[8], p[8];
  load_state(g, Uz, z, u);
  const float2 gy = guess[t];
  const float y[2] = {gy.x, gy.y};
  double Zg = 0.0, Wg = 0.0;
  const bool use = c2p_guess_from_output_f32(u[ddd], y, Zg, Wg);
  // the previous primitives are read only when the ladder needs them or a failure keeps them
  const auto prev = [&](double *q) {
#pragma unroll
    for (int c = 0; c < 8; ++c) q[c] = zero_guess ? 0.0 : double(PAg[c * g.cs + z]);
  };
  C2PTally tally;
  const int err = cons_to_prim<(sizeof(T) < sizeof(double)), 1>(pp, u, p, &tally, Zg, Wg, use, prev) != 0;
  c2p_finish<T>(g, PA, ctl->cur ? Pn0 : Pn1, ctl, stage, final, ereset, preset, dreset, i, j, k, u, p, err, tally);
}

}  // namespace mgpu
