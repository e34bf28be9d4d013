// Learned c2p initial guess: the network, its features and its per-thread evaluation.
//
// The network maps five scale-free features of the c2p invariants (D, tau, S^2, B^2,
// (S.B)^2) to (log W, log h); the Newton polish then starts at W and Z = D W h.  For a
// gamma-law gas the c2p problem is invariant under D, tau, S, B^2 -> lambda * (...), so the
// features are ratios to powers of D:
//   x0 = log(1 + tau/D), x1 = log(1 + S^2/D^2), x2 = log(1 + B^2/D),
//   x3 = log(1 + (S.B)^2/D^3), x4 = (S.B)^2 / (S^2 B^2)  (cos^2 of the S-B angle)
// Layers 5 -> 64 -> 64 -> 64 -> 2 with tanh; inputs standardised and outputs de-standardised
// with constants stored after the weights.  Packed float32 layout (N_PARAMS floats):
//   W1[64][5] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[2][64] b4[2]
//   xmean[5] xstd[5] ymean[2] ystd[2]
// The reference has no learned component; this is an initial guess only: the reference's
// Newton iteration always polishes it and the reference's ladder runs if that fails.
#pragma once
#include "rmhd_physics.cuh"

namespace mgpu {

namespace mlp {
constexpr int NIN = 5, NH = 64, NOUT = 2;
constexpr int OW1 = 0, OB1 = OW1 + NH * NIN, OW2 = OB1 + NH, OB2 = OW2 + NH * NH, OW3 = OB2 + NH,
              OB3 = OW3 + NH * NH, OW4 = OB3 + NH, OB4 = OW4 + NOUT * NH, N_TRAIN = OB4 + NOUT,
              OXM = N_TRAIN, OXS = OXM + NIN, OYM = OXS + NIN, OYS = OYM + NOUT, N_PARAMS = OYS + NOUT;
}  // namespace mlp

__device__ __forceinline__ void c2p_features(double D, double Tau, double S2, double B2, double BS2, float *x)
{
  const double iD = 1.0 / D;
  x[0] = (float) log1p(Tau * iD);
  x[1] = (float) log1p(S2 * iD * iD);
  x[2] = (float) log1p(B2 * iD);
  x[3] = (float) log1p(BS2 * iD * iD * iD);
  x[4] = (float) (BS2 / (S2 * B2 + 1e-30));
}

// The same features and guess with FP32 transcendentals, for inference: the network reads its
// inputs as BF16 and its guess only seeds the FP64 Newton polish, so FP32 logarithms and
// exponentials (a few instructions each, against software FP64 routines) lose nothing.
__device__ __forceinline__ void c2p_features_f32(double D, double Tau, double S2, double B2, double BS2, float *x)
{
  const double iD = 1.0 / D;
  x[0] = log1pf((float) (Tau * iD));
  x[1] = log1pf((float) (S2 * iD * iD));
  x[2] = log1pf((float) (B2 * iD));
  x[3] = log1pf((float) (BS2 * iD * iD * iD));
  x[4] = (float) (BS2 / (S2 * B2 + 1e-30));
}

__device__ __forceinline__ bool c2p_guess_from_output_f32(double D, const float *y, double &Z, double &W)
{
  const float lw = y[0], lh = y[1];
  if (!(lw >= 0.f && lw < 30.f && lh >= 0.f && lh < 60.f)) return false;
  W = (double) expf(lw);
  Z = D * (double) expf(lw + lh);
  return Z > 0.0 && W >= 1.0;
}

// Per-thread forward pass in FP32 (weights read through the read-only cache).
__device__ __forceinline__ void mlp_forward_thread(const float *__restrict__ p, const float *xin, float *y)
{
  using namespace mlp;
  float x[NIN], a[NH], b[NH];
#pragma unroll
  for (int i = 0; i < NIN; ++i) x[i] = (xin[i] - __ldg(p + OXM + i)) / __ldg(p + OXS + i);
#pragma unroll 4
  for (int j = 0; j < NH; ++j) {
    float s = __ldg(p + OB1 + j);
#pragma unroll
    for (int i = 0; i < NIN; ++i) s = fmaf(__ldg(p + OW1 + j * NIN + i), x[i], s);
    a[j] = tanhf(s);
  }
#pragma unroll 2
  for (int j = 0; j < NH; ++j) {
    float s = __ldg(p + OB2 + j);
#pragma unroll
    for (int i = 0; i < NH; ++i) s = fmaf(__ldg(p + OW2 + j * NH + i), a[i], s);
    b[j] = tanhf(s);
  }
#pragma unroll 2
  for (int j = 0; j < NH; ++j) {
    float s = __ldg(p + OB3 + j);
#pragma unroll
    for (int i = 0; i < NH; ++i) s = fmaf(__ldg(p + OW3 + j * NH + i), b[i], s);
    a[j] = tanhf(s);
  }
#pragma unroll
  for (int k = 0; k < NOUT; ++k) {
    float s = __ldg(p + OB4 + k);
#pragma unroll
    for (int i = 0; i < NH; ++i) s = fmaf(__ldg(p + OW4 + k * NH + i), a[i], s);
    y[k] = s * __ldg(p + OYS + k) + __ldg(p + OYM + k);
  }
}

// (log W, log h) -> (Z, W); rejects guesses that are not a valid starting point.
__device__ __forceinline__ bool c2p_guess_from_output(double D, const float *y, double &Z, double &W)
{
  const double lw = (double) y[0], lh = (double) y[1];
  if (!(lw >= 0.0 && lw < 30.0 && lh >= 0.0 && lh < 60.0)) return false;
  W = exp(lw);
  Z = D * W * exp(lh);
  return Z > 0.0 && W >= 1.0;
}

__device__ __forceinline__ bool c2p_learned_guess(const void *net, const C2PState &s, double &Z, double &W)
{
  float x[mlp::NIN], y[mlp::NOUT];
  c2p_features(s.D, s.Tau, s.S2, s.B2, s.BS2, x);
  mlp_forward_thread((const float *) net, x, y);
  return c2p_guess_from_output(s.D, y, Z, W);
}

}  // namespace mgpu
