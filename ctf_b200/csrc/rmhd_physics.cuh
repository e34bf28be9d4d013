// Per-state RMHD physics for the B200 step kernels: gamma-law EOS, P->U, flux and exact
// fast-magnetosonic speeds (quartic), the c2p Newton ladder, PLM / WENO5 reconstruction and
// the HLL / HLLC / HLLD Riemann solvers.
//
// Everything is templated on the bulk arithmetic type T.  With T = double and the
// translation unit compiled with --fmad=false, every expression is evaluated in the same
// IEEE operation order as the reference's gcc build, so the plain FP64 path reproduces the
// reference bit for bit except where CUDA's pow/acos/cos/sin differ from glibc by an ulp
// (the quartic only).  With T = float the same algorithms run in FP32 with tolerances
// rescaled to FP32 resolution (RmhdTol<float>); the c2p Newton polish stays FP64 always.
//
// Reference sources restated here (paths within the reference project):
//   EOS          Mara/eos.cpp:13-29                    P->U         Mara/rmhd.cpp:177-207
//   flux, speeds Mara/rmhd.cpp:208-310                 quartic      Mara/quartic.cpp:28-148
//   c2p          Mara/rmhd-c2p.c:132-376, Mara/rmhd.cpp:103-176
//   PLM / WENO5  Mara/weno.c:15-154                    HLL          Mara/riemann_hll.cpp:19-64
//   HLLC         Mara/riemann_hllc-rmhd.cpp:26-178
//   HLLD         Mara/riemann_hlld-rmhd.cpp:179-615, Newton Mara/nrsolver.cpp:89-152
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include "rmhd_types.cuh"

namespace mgpu {

// Tolerances of the Riemann solvers.  For double they are the reference's literals; the
// float set is scaled to FP32 resolution (the FP32 bulk path has no reference oracle and is
// compared with the FP64 path).
template <class T> struct RmhdTol;
template <> struct RmhdTol<double> {
  static constexpr double newton_eps = 1e-12;   // NewtonRaphesonSolver(15, 1e-12)
  static constexpr double jac_dp = 1e-8;        // HlldEquation48::Jacobian
  static constexpr double x_small = 1e-8;       // |X| < 1e-8 (eqs 23-25)
  static constexpr double k_small = 1e-10;      // |Kr-Kl|, |delK|, |Bc_x|, |denom|
  static constexpr double tol54 = 1e-14;        // TOL in ReconstructSolution
  static constexpr double contact = 1e-8;       // UnmatchedContactSpeed
  static constexpr double degenerate = 1e-8;    // |am - aL.v| etc.
  static constexpr double bx_small = 1e-8;      // |Bx| < 1e-8 -> eq. (55) guess only
  static constexpr double bjump = 1e-12;        // JumpInNormalBfield
  static constexpr double hllc_bx = 1e-12;      // SMALL_BX
  static constexpr double hllc_a = 1e-10;       // SMALL_A
};
template <> struct RmhdTol<float> {
  static constexpr float newton_eps = 2e-6f;
  static constexpr float jac_dp = 2e-3f;
  static constexpr float x_small = 1e-6f;
  static constexpr float k_small = 1e-6f;
  static constexpr float tol54 = 1e-6f;
  static constexpr float contact = 2e-4f;
  static constexpr float degenerate = 1e-6f;
  static constexpr float bx_small = 1e-6f;
  static constexpr float bjump = 1e-6f;
#ifdef MGPU_HLLC_BX_F32
  static constexpr float hllc_bx = MGPU_HLLC_BX_F32;
#else
  static constexpr float hllc_bx = 1e-7f;
#endif
  static constexpr float hllc_a = 1e-6f;
};

__device__ __forceinline__ double m_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float m_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double m_abs(double x) { return fabs(x); }
__device__ __forceinline__ float m_abs(float x) { return fabsf(x); }
__device__ __forceinline__ double m_cbrt_pow(double x) { return pow(x, 1. / 3.); }
__device__ __forceinline__ float m_cbrt_pow(float x) { return cbrtf(x); }
__device__ __forceinline__ double m_acos(double x) { return acos(x); }
__device__ __forceinline__ float m_acos(float x) { return acosf(x); }
__device__ __forceinline__ double m_cos(double x) { return cos(x); }
__device__ __forceinline__ float m_cos(float x) { return cosf(x); }
__device__ __forceinline__ double m_sin(double x) { return sin(x); }
__device__ __forceinline__ float m_sin(float x) { return sinf(x); }

// ---- EOS (Mara/eos.cpp:13-29) -------------------------------------------------------
template <class T> __device__ __forceinline__ T eos_internal(T gamma, T p) { return p / (gamma - 1); }
template <class T> __device__ __forceinline__ T eos_cs2(T gamma, T r, T p)
{
  const T rhoh = r + eos_internal(gamma, p) + p;
  return gamma * p / rhoh;
}

// ---- P -> U (Mara/rmhd.cpp:177-207) ---------------------------------------------------
template <class T>
__device__ __forceinline__ int check_cons(const T *U)
{
  if (U[ddd] < T(0)) return C2P_CONS_NEG_DENSITY;
  if (U[tau] < T(0)) return C2P_CONS_NEG_ENERGY;
#pragma unroll
  for (int i = 0; i < 8; ++i)
    if (isnan(U[i])) return C2P_CONS_NAN;
  return C2P_SUCCESS;
}

template <class T>
__device__ __forceinline__ int prim_to_cons(T gamma, const T *P, T *U)
{
  const T V2 = P[vx] * P[vx] + P[vy] * P[vy] + P[vz] * P[vz];
  const T B2 = P[Bx] * P[Bx] + P[By] * P[By] + P[Bz] * P[Bz];
  const T Bv = P[Bx] * P[vx] + P[By] * P[vy] + P[Bz] * P[vz];
  const T W2 = T(1) / (T(1) - V2);
  const T W = m_sqrt(W2);
  const T b0 = W * Bv;
  const T b2 = (B2 + b0 * b0) / W2;
  const T bx = (P[Bx] + b0 * W * P[vx]) / W;
  const T by = (P[By] + b0 * W * P[vy]) / W;
  const T bz = (P[Bz] + b0 * W * P[vz]) / W;
  const T e = eos_internal(gamma, P[pre]) / P[rho];
  const T e_ = e + T(0.5) * b2 / P[rho];
  const T p_ = P[pre] + T(0.5) * b2;
  const T h_ = T(1) + e_ + p_ / P[rho];
  U[ddd] = P[rho] * W;
  U[tau] = P[rho] * h_ * W2 - p_ - b0 * b0 - U[ddd];
  U[Sx] = P[rho] * h_ * W2 * P[vx] - b0 * bx;
  U[Sy] = P[rho] * h_ * W2 * P[vy] - b0 * by;
  U[Sz] = P[rho] * h_ * W2 * P[vz] - b0 * bz;
  U[Bx] = P[Bx];
  U[By] = P[By];
  U[Bz] = P[Bz];
  if (V2 >= T(1)) return C2P_PRIM_SUPERLUMINAL;
  return check_cons(U);
}

// ---- quartic (Mara/quartic.cpp:28-148) -------------------------------------------------
template <class T>
__device__ __forceinline__ void cubic(T c2, T c1, T c0, T &x1, T &x2, T &x3, int &nr)
{
  // c3 = 1: the reference divides by it, which is exact.
  const T a2 = c2, a1 = c1, a0 = c0;
  const T q = a1 / T(3) - a2 * a2 / T(9);
  const T r = (a1 * a2 - T(3) * a0) / T(6) - a2 * a2 * a2 / T(27);
  const T delta = q * q * q + r * r;
  if (delta > T(0)) {
    T s1 = r + m_sqrt(delta);
    s1 = (s1 >= T(0)) ? m_cbrt_pow(s1) : -m_cbrt_pow(-s1);
    T s2 = r - m_sqrt(delta);
    s2 = (s2 >= T(0)) ? m_cbrt_pow(s2) : -m_cbrt_pow(-s2);
    x1 = (s1 + s2) - a2 / T(3);
    x2 = x3 = T(-0.5) * (s1 + s2) - a2 / T(3);
    nr = 1;
  } else if (delta < T(0)) {
    const T theta = m_acos(r / m_sqrt(-q * q * q)) / T(3);
    const T costh = m_cos(theta), sinth = m_sin(theta), sq = m_sqrt(-q);
    const T sqrt3 = T(1.7320508075688772);
    x1 = T(2) * sq * costh - a2 / T(3);
    x2 = -sq * costh - a2 / T(3) - sqrt3 * sq * sinth;
    x3 = -sq * costh - a2 / T(3) + sqrt3 * sq * sinth;
    nr = 3;
  } else {
    const T s = (r >= T(0)) ? m_cbrt_pow(r) : -m_cbrt_pow(-r);
    x1 = T(2) * s - a2 / T(3);
    x2 = x3 = -s - a2 / T(3);
    nr = 3;
  }
}

// Returns (max root, min root) over the real roots of d4 x^4 + ... + d0 with the fold used
// by FluxAndEigenvalues: start at (-1, +1), then clamp to (1, -1) if either exceeds 1.
// MGPU_QUARTIC_INLINE: inlined at every call site (the default), or __noinline__ for one
// shared copy (less code in the long HLLD kernels).
#ifndef MGPU_QUARTIC_INLINE
#define MGPU_QUARTIC_INLINE __forceinline__
#endif
template <class T>
__device__ MGPU_QUARTIC_INLINE void quartic_extreme_roots(T d4, T d3, T d2, T d1, T d0, T &ap, T &am)
{
  const T a3 = d3 / d4, a2 = d2 / d4, a1 = d1 / d4, a0 = d0 / d4;
  const T au2 = -a2;
  const T au1 = (a1 * a3 - T(4) * a0);
  const T au0 = T(4) * a0 * a2 - a1 * a1 - a0 * a3 * a3;
  T x1, x2, x3;
  int nr;
  cubic<T>(au2, au1, au0, x1, x2, x3, nr);
  const T u1 = (nr == 1) ? x1 : ((x1 > x3) ? x1 : x3);
  const T R2 = T(0.25) * a3 * a3 + u1 - a2;
  const T R = (R2 > T(0)) ? m_sqrt(R2) : T(0);
  T D2, E2;
  if (R != T(0)) {
    const T foo1 = T(0.75) * a3 * a3 - R2 - T(2) * a2;
    const T foo2 = T(0.25) * (T(4) * a3 * a2 - T(8) * a1 - a3 * a3 * a3) / R;
    D2 = foo1 + foo2;
    E2 = foo1 - foo2;
  } else {
    const T foo1 = T(0.75) * a3 * a3 - T(2) * a2;
    const T foo2 = T(2) * m_sqrt(u1 * u1 - T(4) * a0);
    D2 = foo1 + foo2;
    E2 = foo1 - foo2;
  }
  ap = T(-1);
  am = T(1);
  if (D2 >= T(0)) {
    const T D = m_sqrt(D2);
    const T r1 = T(-0.25) * a3 + T(0.5) * R - T(0.5) * D;
    const T r2 = T(-0.25) * a3 + T(0.5) * R + T(0.5) * D;
    if (r1 > ap) ap = r1;
    if (r1 < am) am = r1;
    if (r2 > ap) ap = r2;
    if (r2 < am) am = r2;
  }
  if (E2 >= T(0)) {
    const T E = m_sqrt(E2);
    const T r3 = T(-0.25) * a3 - T(0.5) * R - T(0.5) * E;
    const T r4 = T(-0.25) * a3 - T(0.5) * R + T(0.5) * E;
    if (r3 > ap) ap = r3;
    if (r3 < am) am = r3;
    if (r4 > ap) ap = r4;
    if (r4 < am) am = r4;
  }
  if (m_abs(ap) > T(1) || m_abs(am) > T(1)) {
    ap = T(1);
    am = T(-1);
  }
}

// ---- flux and fast speeds (Mara/rmhd.cpp:208-310) ---------------------------------------
// dim is 1, 2 or 3.  Computes F (8) and, when want_speeds, (ap, am).
template <class T>
__device__ __forceinline__ void flux_and_eigenvalues(T gamma, const T *U, const T *P, T *F, T &ap,
                                                     T &am, int dim, bool want_speeds = true)
{
  const T V2 = P[vx] * P[vx] + P[vy] * P[vy] + P[vz] * P[vz];
  const T B2 = P[Bx] * P[Bx] + P[By] * P[By] + P[Bz] * P[Bz];
  const T Bv = P[Bx] * P[vx] + P[By] * P[vy] + P[Bz] * P[vz];
  const T W2 = T(1) / (T(1) - V2);
  const T W = m_sqrt(W2);
  const T b0 = W * Bv;
  const T b2 = (B2 + b0 * b0) / W2;
  const T bx = (P[Bx] + b0 * W * P[vx]) / W;
  const T by = (P[By] + b0 * W * P[vy]) / W;
  const T bz = (P[Bz] + b0 * W * P[vz]) / W;
  const T e = eos_internal(gamma, P[pre]) / P[rho];
  const T p_ = P[pre] + T(0.5) * b2;
  const T h = T(1) + e + P[pre] / P[rho];
  T vi, bi;
  if (dim == 1) {
    F[ddd] = U[ddd] * P[vx];
    F[tau] = U[tau] * P[vx] - b0 * P[Bx] / W + p_ * P[vx];
    F[Sx] = U[Sx] * P[vx] - bx * P[Bx] / W + p_;
    F[Sy] = U[Sy] * P[vx] - by * P[Bx] / W;
    F[Sz] = U[Sz] * P[vx] - bz * P[Bx] / W;
    F[Bx] = T(0);
    F[By] = P[vx] * P[By] - P[vy] * P[Bx];
    F[Bz] = P[vx] * P[Bz] - P[vz] * P[Bx];
    vi = P[vx];
    bi = bx;
  } else if (dim == 2) {
    F[ddd] = U[ddd] * P[vy];
    F[tau] = U[tau] * P[vy] - b0 * P[By] / W + p_ * P[vy];
    F[Sx] = U[Sx] * P[vy] - bx * P[By] / W;
    F[Sy] = U[Sy] * P[vy] - by * P[By] / W + p_;
    F[Sz] = U[Sz] * P[vy] - bz * P[By] / W;
    F[Bx] = P[vy] * P[Bx] - P[vx] * P[By];
    F[By] = T(0);
    F[Bz] = P[vy] * P[Bz] - P[vz] * P[By];
    vi = P[vy];
    bi = by;
  } else {
    F[ddd] = U[ddd] * P[vz];
    F[tau] = U[tau] * P[vz] - b0 * P[Bz] / W + p_ * P[vz];
    F[Sx] = U[Sx] * P[vz] - bx * P[Bz] / W;
    F[Sy] = U[Sy] * P[vz] - by * P[Bz] / W;
    F[Sz] = U[Sz] * P[vz] - bz * P[Bz] / W + p_;
    F[Bx] = P[vz] * P[Bx] - P[vx] * P[Bz];
    F[By] = P[vz] * P[By] - P[vy] * P[Bz];
    F[Bz] = T(0);
    vi = P[vz];
    bi = bz;
  }
  if (!want_speeds) return;
  const T cs2 = eos_cs2(gamma, P[rho], P[pre]);
  const T W4 = W2 * W2, v2 = vi * vi, v3 = vi * v2, v4 = vi * v3;
  const T K = P[rho] * h * (T(1) / cs2 - T(1)) * W4;
  const T L = -(P[rho] * h + b2 / cs2) * W2;
  const T A4 = K - L - b0 * b0;
  const T A3 = T(-4) * K * vi + L * vi * T(2) + T(2) * b0 * bi;
  const T A2 = T(6) * K * v2 + L * (T(1) - v2) + b0 * b0 - bi * bi;
  const T A1 = T(-4) * K * v3 - L * vi * T(2) - T(2) * b0 * bi;
  const T A0 = K * v4 + L * v2 + bi * bi;
  quartic_extreme_roots<T>(A4, A3, A2, A1, A0, ap, am);
}

// ---- c2p: Newton solvers and the four-attempt ladder (FP64 always) --------------------------
struct C2PState {
  double D, Tau, S2, B2, BS, BS2, gamma, gamf, pfloor;
  double Sxyz[3], Bxyz[3];
};

__device__ __forceinline__ void c2p_new_state(C2PState &s, const double *U)
{
  s.D = U[ddd];
  s.Tau = U[tau];
  s.S2 = U[Sx] * U[Sx] + U[Sy] * U[Sy] + U[Sz] * U[Sz];
  s.B2 = U[Bx] * U[Bx] + U[By] * U[By] + U[Bz] * U[Bz];
  s.BS = U[Bx] * U[Sx] + U[By] * U[Sy] + U[Bz] * U[Sz];
  s.BS2 = s.BS * s.BS;
  s.Sxyz[0] = U[Sx]; s.Sxyz[1] = U[Sy]; s.Sxyz[2] = U[Sz];
  s.Bxyz[0] = U[Bx]; s.Bxyz[1] = U[By]; s.Bxyz[2] = U[Bz];
}

__device__ __forceinline__ void c2p_estimate(const C2PState &s, double &Z, double &W)
{
  Z = sqrt(s.S2 + s.D * s.D);
  W = Z / s.D;
}

__device__ __forceinline__ void c2p_from_prim(const C2PState &s, const double *P, double &Z, double &W)
{
  const double V2 = P[vx] * P[vx] + P[vy] * P[vy] + P[vz] * P[vz];
  const double W2 = 1.0 / (1.0 - V2);
  const double e = P[pre] / (P[rho] * (s.gamma - 1.0));
  const double h = 1.0 + e + P[pre] / P[rho];
  Z = P[rho] * h * W2;
  W = sqrt(W2);
}

template <class T>
__device__ __forceinline__ int check_prim(const T *P)
{
  const T v2 = P[vx] * P[vx] + P[vy] * P[vy] + P[vz] * P[vz];
  if (v2 >= T(1)) return C2P_PRIM_SUPERLUMINAL;
  if (P[pre] < T(0)) return C2P_PRIM_NEG_PRESSURE;
  if (P[rho] < T(0)) return C2P_PRIM_NEG_RESTMASS;
#pragma unroll
  for (int i = 0; i < 8; ++i)
    if (isnan(P[i])) return C2P_PRIM_NAN;
  return C2P_SUCCESS;
}

__device__ __forceinline__ int c2p_reconstruct(const C2PState &s, double Z, double W, double *Pout)
{
  double P[8];
  const double b0 = s.BS * W / Z;
  P[rho] = s.D / W;
  P[pre] = (s.D / W) * (Z / (s.D * W) - 1.0) * s.gamf;
  P[vx] = (s.Sxyz[0] + b0 * s.Bxyz[0] / W) / (Z + s.B2);
  P[vy] = (s.Sxyz[1] + b0 * s.Bxyz[1] / W) / (Z + s.B2);
  P[vz] = (s.Sxyz[2] + b0 * s.Bxyz[2] / W) / (Z + s.B2);
  P[Bx] = s.Bxyz[0];
  P[By] = s.Bxyz[1];
  P[Bz] = s.Bxyz[2];
  if (P[pre] < s.pfloor && s.pfloor > 0.0) P[pre] = s.pfloor;
  const int e = check_prim(P);
  if (e) return e;
#pragma unroll
  for (int i = 0; i < 8; ++i) Pout[i] = P[i];
  return C2P_SUCCESS;
}

// The same reconstruction for the FP32-bulk path's Newton (c2p_anton2dzw_fast), from the
// reciprocals of W, Z and D it holds already: one FP64 division instead of nine.  Same
// formulas and checks; the primitives differ from c2p_reconstruct's at FP64 round-off.
__device__ __forceinline__ int c2p_reconstruct_fast(const C2PState &s, double Z, double W, double iZ, double iW,
                                                    double iD, double *Pout)
{
  double P[8];
  const double b0 = s.BS * W * iZ;
  const double iZB = 1.0 / (Z + s.B2);
  P[rho] = s.D * iW;
  P[pre] = P[rho] * (Z * iD * iW - 1.0) * s.gamf;
  P[vx] = (s.Sxyz[0] + b0 * s.Bxyz[0] * iW) * iZB;
  P[vy] = (s.Sxyz[1] + b0 * s.Bxyz[1] * iW) * iZB;
  P[vz] = (s.Sxyz[2] + b0 * s.Bxyz[2] * iW) * iZB;
  P[Bx] = s.Bxyz[0];
  P[By] = s.Bxyz[1];
  P[Bz] = s.Bxyz[2];
  if (P[pre] < s.pfloor && s.pfloor > 0.0) P[pre] = s.pfloor;
  const int e = check_prim(P);
  if (e) return e;
#pragma unroll
  for (int i = 0; i < 8; ++i) Pout[i] = P[i];
  return C2P_SUCCESS;
}

// Anton et al. (2006) eqs 84-85, 2-D Newton in (Z, W) (Mara/rmhd-c2p.c:232-303).
__device__ __forceinline__ int c2p_anton2dzw(const C2PState &s, double Z, double W, double *P, int &iters)
{
  const double D = s.D, B2 = s.B2, BS2 = s.BS2, S2 = s.S2, gamf = s.gamf, Tau = s.Tau;
  double error = 1.0;
  iters = 0;
  while (error > 1e-12) {
    const double Z2 = Z * Z, Z3 = Z * Z2, W2 = W * W, W3 = W * W2;
    const double Pre = (D / W) * (Z / (D * W) - 1.0) * gamf;
    const double df0dZ = 2 * (B2 + Z) * (BS2 * W2 + (W2 - 1) * Z3) / (W2 * Z3);
    const double df0dW = 2 * (B2 + Z) * (B2 + Z) / W3;
    const double df1dZ = 1.0 + BS2 / Z3 - gamf / W2;
    const double df1dW = B2 / W3 + (2 * Z - D * W) / W3 * gamf;
    const double f0 = -S2 + (Z + B2) * (Z + B2) * (W2 - 1) / W2 - (2 * Z + B2) * BS2 / Z2;
    const double f1 = -Tau + Z + B2 - Pre - 0.5 * B2 / W2 - 0.5 * BS2 / Z2 - D;
    const double det = df0dZ * df1dW - df0dW * df1dZ;
    const double G0 = df1dW / det, G1 = -df0dW / det, G2 = -df1dZ / det, G3 = df0dZ / det;
    const double dZ = -(G0 * f0 + G1 * f1);
    const double dW = -(G2 * f0 + G3 * f1);
    double Zn = Z + dZ, Wn = W + dW;
    Zn = (Zn > 0.0) ? Zn : -Zn;
    Zn = (Zn < 1e20) ? Zn : Z;
    Wn = (Wn > 1.0) ? Wn : 1.0;
    Wn = (Wn < 1e12) ? Wn : 1e12;
    Z = Zn;
    W = Wn;
    error = fabs(dZ / Z) + fabs(dW / W);
    if (++iters == 250) return C2P_MAXITER;
  }
  return c2p_reconstruct(s, Z, W, P);
}

// The same Anton et al. Newton iteration with the divisions replaced by three reciprocals
// per iteration (1/W, 1/Z, 1/det); algebraically identical, rounded differently.  Used by
// the FP32-bulk path, whose c2p is an FP64 polish compared with the FP64 path rather than
// the reference's bit pattern.
__device__ __forceinline__ int c2p_anton2dzw_fast(const C2PState &s, double Z, double W, double *P, int &iters)
{
  const double D = s.D, B2 = s.B2, BS2 = s.BS2, S2 = s.S2, gamf = s.gamf, Tau = s.Tau;
  const double iD = 1.0 / D;
  double iW = 1.0 / W, iZ = 1.0 / Z;
  double error = 1.0;
  iters = 0;
  while (error > 1e-12) {
    const double W2 = W * W, Z2 = Z * Z, Z3 = Z * Z2;
    const double iW2 = iW * iW, iW3 = iW2 * iW, iZ2 = iZ * iZ, iZ3 = iZ2 * iZ;
    const double Pre = D * iW * (Z * iD * iW - 1.0) * gamf;
    const double BZ = B2 + Z;
    const double df0dZ = 2 * BZ * (BS2 * W2 + (W2 - 1) * Z3) * iW2 * iZ3;
    const double df0dW = 2 * BZ * BZ * iW3;
    const double df1dZ = 1.0 + BS2 * iZ3 - gamf * iW2;
    const double df1dW = (B2 + (2 * Z - D * W) * gamf) * iW3;
    const double f0 = -S2 + BZ * BZ * (W2 - 1) * iW2 - (2 * Z + B2) * BS2 * iZ2;
    const double f1 = -Tau + Z + B2 - Pre - 0.5 * B2 * iW2 - 0.5 * BS2 * iZ2 - D;
    const double idet = 1.0 / (df0dZ * df1dW - df0dW * df1dZ);
    const double dZ = -(df1dW * f0 - df0dW * f1) * idet;
    const double dW = -(df0dZ * f1 - df1dZ * f0) * idet;
    double Zn = Z + dZ, Wn = W + dW;
    Zn = (Zn > 0.0) ? Zn : -Zn;
    Zn = (Zn < 1e20) ? Zn : Z;
    Wn = (Wn > 1.0) ? Wn : 1.0;
    Wn = (Wn < 1e12) ? Wn : 1e12;
    Z = Zn;
    W = Wn;
    iZ = 1.0 / Z;
    iW = 1.0 / W;
    error = fabs(dZ * iZ) + fabs(dW * iW);
    if (++iters == 250) return C2P_MAXITER;
  }
  return c2p_reconstruct_fast(s, Z, W, iZ, iW, iD, P);
}

// Noble et al. (2006) 1-D Newton in Z (Mara/rmhd-c2p.c:311-376).
__device__ __forceinline__ int c2p_noble1dw(const C2PState &s, double Z, double *P, int &iters)
{
  const double D = s.D, B2 = s.B2, BS2 = s.BS2, S2 = s.S2, gamf = s.gamf, Tau = s.Tau;
  double error = 1.0;
  iters = 0;
  while (error > 1e-12) {
    const double Z2 = Z * Z, Z3 = Z * Z2;
    const double a = S2 * Z2 + BS2 * (B2 + 2 * Z);
    const double b = (B2 + Z) * (B2 + Z) * Z2;
    const double ap = 2 * (S2 * Z + BS2);
    const double bp = 2 * Z * (B2 + Z) * (B2 + 2 * Z);
    const double V2 = a / b;
    const double W2 = 1.0 / (1.0 - V2);
    const double W = sqrt(W2);
    const double W3 = W * W2;
    const double Pre = (D / W) * (Z / (D * W) - 1.0) * gamf;
    const double dv2dZ = (ap * b - bp * a) / (b * b);
    const double delPdelZ = gamf / W2;
    const double delPdelW = gamf * (D / W2 - 2 * Z / W3);
    const double dWdv2 = 0.5 * W3;
    const double dPdZ = delPdelW * dWdv2 * dv2dZ + delPdelZ;
    const double f = Tau + D - 0.5 * B2 * (1 + V2) + 0.5 * BS2 / Z2 - Z + Pre;
    const double g = -0.5 * B2 * dv2dZ - BS2 / Z3 - 1.0 + dPdZ;
    const double dZ = -f / g;
    double Zn = Z + dZ;
    Zn = (Zn > 0.0) ? Zn : -Zn;
    Zn = (Zn < 1e20) ? Zn : Z;
    Z = Zn;
    error = fabs(dZ / Z);
    if (++iters == 250) return C2P_MAXITER;
  }
  const double Z2 = Z * Z;
  const double a = S2 * Z2 + BS2 * (B2 + 2 * Z);
  const double b = (B2 + Z) * (B2 + Z) * Z2;
  const double V2 = a / b;
  const double W2 = 1.0 / (1.0 - V2);
  const double W = sqrt(W2);
  return c2p_reconstruct(s, Z, W, P);
}

// Per-call c2p statistics (iterations of the Newton that succeeded, attempts used).
struct C2PTally {
  int iters;      // Newton iterations summed over attempts
  int attempts;   // 1..4 (5 = learned guess rejected and ladder used)
};

// Optional learned initial guess: (Z, W) from the packed network; defined in c2p_mlp.cuh.
__device__ __forceinline__ bool c2p_learned_guess(const void *net, const C2PState &s, double &Z, double &W);

// The ladder's rungs 2-4 (previous prim -> Anton; estimate -> Noble; previous prim ->
// Noble), reached only when the first attempt fails: kept out of line, state by value.
struct C2PRungs {
  double P[8];
  int err, iters, attempt;
};
static __device__ __noinline__ C2PRungs c2p_rungs(const C2PState s, C2PRungs r)
{
  double Z, W;
  int it = 0;
  r.err = 1;
  r.iters = 0;
  c2p_from_prim(s, r.P, Z, W);
  r.err = c2p_anton2dzw(s, Z, W, r.P, it);
  r.iters += it;
  r.attempt = 2;
  if (r.err) {
    c2p_estimate(s, Z, W);
    r.err = c2p_noble1dw(s, Z, r.P, it);
    r.iters += it;
    r.attempt = 3;
  }
  if (r.err) {
    c2p_from_prim(s, r.P, Z, W);
    r.err = c2p_noble1dw(s, Z, r.P, it);
    r.iters += it;
    r.attempt = 4;
  }
  return r;
}

// AdiabaticIdealRmhd::ConsToPrim gamma-law ladder (Mara/rmhd.cpp:103-176).  P holds the
// previous primitive state on entry (second guess) and is written only on success.  With a
// learned network the first attempt starts from its guess instead, and the reference ladder
// follows unchanged if that attempt fails.  The first Anton attempt is inlined (one call
// site serves both the learned and the estimated starting point); the other rungs are not.
// Guess (compile time): 0 = the per-thread network when pp.learned; 1 = the given (Zg, Wg)
// when `have`; 2 = none (no network code is compiled in).  `prev` fills P with the previous
// primitive state when P does not hold it yet: it is called only on the paths that read P
// (the ladder's rungs) or leave it as the result (a failure), so a caller can defer that load.
struct C2PPrevInP {
  __device__ void operator()(double *) const {}
};
template <bool Fast = false, int Guess = 0, class Prev = C2PPrevInP>
__device__ __forceinline__ int cons_to_prim(const PhysParams &pp, const double *U, double *P,
                                            C2PTally *tally = nullptr, double Zg = 0.0, double Wg = 0.0,
                                            bool have = true, const Prev &prev = Prev())
{
  int error = check_cons(U);
  if (error) {
    prev(P);
    if (tally) { tally->iters = 0; tally->attempts = 0; }
    return error;
  }
  C2PState s;
  s.gamma = pp.gamma;
  s.gamf = (pp.gamma - 1.0) / pp.gamma;
  s.pfloor = pp.pfloor;
  c2p_new_state(s, U);
  int total = 0, attempts = 1;
  error = 1;
  const bool use_net = (Guess == 1 && have) || (Guess == 0 && pp.learned && pp.mlp);
  for (int a = use_net ? 0 : 1; a < 2 && error; ++a) {
    double Z, W;
    if (a == 0) {
      if (Guess == 1) {
        Z = Zg;
        W = Wg;
      } else if (Guess == 0) {
        if (!c2p_learned_guess(pp.mlp, s, Z, W)) continue;
      } else {
        continue;
      }
    } else {
      c2p_estimate(s, Z, W);
    }
    int it = 0;
    error = Fast ? c2p_anton2dzw_fast(s, Z, W, P, it) : c2p_anton2dzw(s, Z, W, P, it);
    total += it;
    if (error && a == 0) attempts = 5;
  }
  if (error) {
    prev(P);
    C2PRungs r;
#pragma unroll
    for (int i = 0; i < 8; ++i) r.P[i] = P[i];
    r = c2p_rungs(s, r);
    total += r.iters;
    error = r.err;
    if (attempts != 5) attempts = r.attempt;
    if (!error) {
#pragma unroll
      for (int i = 0; i < 8; ++i) P[i] = r.P[i];
    }
  }
  if (tally) { tally->iters = total; tally->attempts = attempts; }
  return error;
}

// ---- reconstruction (Mara/weno.c:85-154) ---------------------------------------------------
template <class T> __device__ __forceinline__ int sgn(T x) { return (x > T(0)) - (x < T(0)); }

template <class T>
__device__ __forceinline__ T min3(T a, T b, T c)
{
  const T x01 = a < b ? a : b;
  return x01 < c ? x01 : c;
}
template <class T>
__device__ __forceinline__ T max3(T a, T b, T c)
{
  const T x01 = a > b ? a : b;
  return x01 > c ? x01 : c;
}

// PLM minmod(theta): face value v0 + sgn * slope / 2
template <class T>
__device__ __forceinline__ T plm(T theta, T vm, T v0, T vp, T sg)
{
  const T a = theta * (v0 - vm);
  const T b = T(0.5) * (vp - vm);
  const T c = theta * (vp - v0);
  const int sa = sgn(a), sb = sgn(b), sc = sgn(c);
  const T mm = T(0.25) * T(abs(sa + sb)) * T(sa + sc) * min3(m_abs(a), m_abs(b), m_abs(c));
  return v0 + sg * T(0.5) * mm;
}

// WENO5 finite-volume, centre-to-right (c2r = true) or centre-to-left face, on the stencil
// v[-2..2] given as (vm2, vm1, v0, vp1, vp2).
template <class T>
__device__ __forceinline__ T weno5(int is_mode, T sz10A, T vm2, T vm1, T v0, T vp1, T vp2, bool c2r)
{
  // coefficient tables CeesC2R_FV / CeesC2L_FV and DeesC2R_FV / DeesC2L_FV (weno.c:21-28)
  T c00, c01, c02, c10, c11, c12, c20, c21, c22, d0, d1, d2;
  if (c2r) {
    c00 = T(3. / 8.);  c01 = T(3. / 4.);  c02 = T(-1. / 8.);
    c10 = T(-1. / 8.); c11 = T(3. / 4.);  c12 = T(3. / 8.);
    c20 = T(3. / 8.);  c21 = T(-5. / 4.); c22 = T(15. / 8.);
    d0 = T(5. / 16.); d1 = T(5. / 8.); d2 = T(1. / 16.);
  } else {
    c00 = T(15. / 8.); c01 = T(-5. / 4.); c02 = T(3. / 8.);
    c10 = T(3. / 8.);  c11 = T(3. / 4.);  c12 = T(-1. / 8.);
    c20 = T(-1. / 8.); c21 = T(3. / 4.);  c22 = T(3. / 8.);
    d0 = T(1. / 16.); d1 = T(5. / 8.); d2 = T(5. / 16.);
  }
  const T vs0 = c00 * v0 + c01 * vp1 + c02 * vp2;
  const T vs1 = c10 * vm1 + c11 * v0 + c12 * vp1;
  const T vs2 = c20 * vm2 + c21 * vm1 + c22 * v0;
  const T t0a = T(1) * v0 - T(2) * vp1 + T(1) * vp2, t0b = T(3) * v0 - T(4) * vp1 + T(1) * vp2;
  const T t1a = T(1) * vm1 - T(2) * v0 + T(1) * vp1, t1b = T(1) * vm1 - T(0) * v0 - T(1) * vp1;
  const T t2a = T(1) * vm2 - T(2) * vm1 + T(1) * v0, t2b = T(1) * vm2 - T(4) * vm1 + T(3) * v0;
  T B0 = T(13. / 12.) * (t0a * t0a) + T(1. / 4.) * (t0b * t0b);
  T B1 = T(13. / 12.) * (t1a * t1a) + T(1. / 4.) * (t1b * t1b);
  T B2 = T(13. / 12.) * (t2a * t2a) + T(1. / 4.) * (t2b * t2b);
  T w0, w1, w2;
  if (is_mode == IS_B08) {
    const T eps = T(1e-14);
    const T tau5 = m_abs(B0 - B2);
    w0 = d0 * (T(1) + (tau5 / (B0 + eps)));
    w1 = d1 * (T(1) + (tau5 / (B1 + eps)));
    w2 = d2 * (T(1) + (tau5 / (B2 + eps)));
  } else if (is_mode == IS_SZ10) {
    const T epsp = T(1e-10);
    const T minB = min3(B0, B1, B2), maxB = max3(B0, B1, B2);
    const T R0 = minB / (maxB + epsp);
    B0 = R0 * sz10A * minB + B0;
    B1 = R0 * sz10A * minB + B1;
    B2 = R0 * sz10A * minB + B2;
    w0 = d0 / ((epsp + B0) * (epsp + B0));
    w1 = d1 / ((epsp + B1) * (epsp + B1));
    w2 = d2 / ((epsp + B2) * (epsp + B2));
  } else {
    const T epsp = T(1e-6);
    w0 = d0 / ((epsp + B0) * (epsp + B0));
    w1 = d1 / ((epsp + B1) * (epsp + B1));
    w2 = d2 / ((epsp + B2) * (epsp + B2));
  }
  const T wtot = w0 + w1 + w2;
  return (w0 * vs0 + w1 * vs1 + w2 * vs2) / wtot;
}

// ---- Riemann solvers ------------------------------------------------------------------------
template <class T> struct RiemannCount {
  int hlld_ok, hlld_fallback;
};

// Index permutation of a sweep direction (compile time, so that the permuted state arrays
// stay in registers): (B1, B2, B3), (S1, S2, S3), (v1, v2, v3) as in the reference's
// IntercellFlux switch (e.g. Mara/riemann_hlld-rmhd.cpp:199-217).
template <int DIM> struct DimMap;
template <> struct DimMap<1> { enum { B1 = Bx, B2 = By, B3 = Bz, S1 = Sx, S2 = Sy, S3 = Sz, v1 = vx, v2 = vy, v3 = vz }; };
template <> struct DimMap<2> { enum { B1 = By, B2 = Bz, B3 = Bx, S1 = Sy, S2 = Sz, S3 = Sx, v1 = vy, v2 = vz, v3 = vx }; };
template <> struct DimMap<3> { enum { B1 = Bz, B2 = Bx, B3 = By, S1 = Sz, S2 = Sx, S3 = Sy, v1 = vz, v2 = vx, v3 = vy }; };

template <class T>
__device__ __forceinline__ T face_lambda(T ap, T am)
{
  return (m_abs(am) < m_abs(ap)) ? m_abs(ap) : m_abs(am);
}

// HllRiemannSolver::IntercellFlux at s = 0 (Mara/riemann_hll.cpp:19-64)
template <class T, int dim>
__device__ __forceinline__ int riemann_hll(T gamma, const T *Pl, const T *Pr, T *F, T &ml)
{
  T Ul[8], Ur[8], Fl[8], Fr[8], epl, eml, epr, emr;
  if (prim_to_cons(gamma, Pl, Ul)) return 1;
  if (prim_to_cons(gamma, Pr, Ur)) return 1;
  flux_and_eigenvalues(gamma, Ul, Pl, Fl, epl, eml, dim);
  flux_and_eigenvalues(gamma, Ur, Pr, Fr, epr, emr, dim);
  const T ap = (epl > epr) ? epl : epr;
  const T am = (eml < emr) ? eml : emr;
  const T l = face_lambda(ap, am);
  if (ml < l) ml = l;
  const T s = T(0);
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const T Fh = (ap * Fl[i] - am * Fr[i] + ap * am * (Ur[i] - Ul[i])) / (ap - am);
    if (s <= am) F[i] = Fl[i];
    else if (am < s && s <= ap) F[i] = Fh;
    else if (ap < s) F[i] = Fr[i];
  }
  return 0;
}

// Contact speed of HLLC: the root (-b - sqrt(b^2 - 4ac)) / (2a) of a x^2 + b x + c, or -c/b
// when |a| is below SMALL_A (Mara/riemann_hllc-rmhd.cpp:96,134).  In FP64 the reference's
// expression is kept as written.  In FP32 it cancels catastrophically when a is small and
// b < 0 (an error of ~eps * |b| / a), so the FP32 path uses the algebraically identical
// 2c / (-b + sqrt(b^2 - 4ac)) there.
template <class T>
__device__ __forceinline__ T hllc_contact_speed(T a, T b, T c)
{
  using Tol = RmhdTol<T>;
  if (m_abs(a) < T(Tol::hllc_a)) return -c / b;
  if (sizeof(T) == sizeof(double)) return (-b - m_sqrt(b * b - T(4) * a * c)) / (T(2) * a);
  const T sq = m_sqrt(b * b - T(4) * a * c);
  return b <= T(0) ? T(2) * c / (-b + sq) : -(b + sq) / (T(2) * a);
}

// The HLL average, the HLLC star states and the flux at s = 0 from the two sides' states,
// fluxes (total-energy convention) and the outer speeds.  `safeguard` (the FP32 path): a
// non-finite contact speed or star state -- which FP32 overflow or a vanishing FP32
// denominator can produce where FP64 stays finite -- takes the HLL flux instead.  Star
// states that are merely unphysical (negative pressure, superluminal contact) are kept, as
// the reference keeps them, so the two precisions take the same branch.
template <class C, int dim>
__device__ __forceinline__ void hllc_star_flux(const C *Pl, const C *Pr, const C *Ul, const C *Ur, const C *Fl,
                                               const C *Fr, C ap, C am, C *F, bool safeguard)
{
  using T = C;
  using Tol = RmhdTol<T>;
  using M = DimMap<dim>;
  constexpr int B1 = M::B1, B2 = M::B2, B3 = M::B3, S1 = M::S1, S2 = M::S2, S3 = M::S3, v1 = M::v1;
  T Uh[8], Fh[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    Uh[i] = (ap * Ur[i] - am * Ul[i] + (Fl[i] - Fr[i])) / (ap - am);
    Fh[i] = (ap * Fl[i] - am * Fr[i] + ap * am * (Ur[i] - Ul[i])) / (ap - am);
  }
  T Ul_[8], Ur_[8], lc, hllc_star_p;
  if (m_abs(Uh[B1]) > T(Tol::hllc_bx)) {
    const T BdFB = Uh[B2] * Fh[B2] + Uh[B3] * Fh[B3];
    const T a = Fh[tau] - BdFB;
    const T b = -Fh[S1] - Uh[tau] + (Uh[B2] * Uh[B2] + Uh[B3] * Uh[B3]) + (Fh[B2] * Fh[B2] + Fh[B3] * Fh[B3]);
    const T c = Uh[S1] - BdFB;
    const T w1 = lc = hllc_contact_speed(a, b, c);
    const T w2 = (Uh[B2] * w1 - Fh[B2]) / Uh[B1];
    const T w3 = (Uh[B3] * w1 - Fh[B3]) / Uh[B1];
    const T b1 = Uh[B1], b2 = Uh[B2], b3 = Uh[B3];
    const T vdB = w1 * b1 + w2 * b2 + w3 * b3;
    const T vdv = w1 * w1 + w2 * w2 + w3 * w3;
    const T gm2 = T(1) / (T(1) - vdv);
    const T ps = Fh[S1] + b1 * b1 / gm2 - (Fh[tau] - b1 * vdB) * w1;
    hllc_star_p = ps;
    Ul_[ddd] = (am - Pl[v1]) / (am - w1) * Ul[ddd];
    Ur_[ddd] = (ap - Pr[v1]) / (ap - w1) * Ur[ddd];
    Ul_[tau] = (am * Ul[tau] - Ul[S1] + ps * w1 - vdB * b1) / (am - w1);
    Ur_[tau] = (ap * Ur[tau] - Ur[S1] + ps * w1 - vdB * b1) / (ap - w1);
    Ul_[S1] = (Ul_[tau] + ps) * w1 - vdB * b1;
    Ur_[S1] = (Ur_[tau] + ps) * w1 - vdB * b1;
    Ul_[S2] = (-b1 * (b2 / gm2 + vdB * w2) + am * Ul[S2] - Fl[S2]) / (am - w1);
    Ur_[S2] = (-b1 * (b2 / gm2 + vdB * w2) + ap * Ur[S2] - Fr[S2]) / (ap - w1);
    Ul_[S3] = (-b1 * (b3 / gm2 + vdB * w3) + am * Ul[S3] - Fl[S3]) / (am - w1);
    Ur_[S3] = (-b1 * (b3 / gm2 + vdB * w3) + ap * Ur[S3] - Fr[S3]) / (ap - w1);
    Ul_[B1] = Ur_[B1] = b1;
    Ul_[B2] = Ur_[B2] = b2;
    Ul_[B3] = Ur_[B3] = b3;
  } else {
    const T a = Fh[tau];
    const T b = -Fh[S1] - Uh[tau];
    const T c = Uh[S1];
    const T v1_ = lc = hllc_contact_speed(a, b, c);
    const T p_ = -Fh[tau] * v1_ + Fh[S1];
    hllc_star_p = p_;
    Ul_[ddd] = (am - Pl[v1]) / (am - v1_) * Ul[ddd];
    Ur_[ddd] = (ap - Pr[v1]) / (ap - v1_) * Ur[ddd];
    Ul_[tau] = (am * Ul[tau] - Ul[S1] + p_ * v1_) / (am - v1_);
    Ur_[tau] = (ap * Ur[tau] - Ur[S1] + p_ * v1_) / (ap - v1_);
    Ul_[S1] = (Ul_[tau] + p_) * v1_;
    Ur_[S1] = (Ur_[tau] + p_) * v1_;
    Ul_[S2] = (am - Pl[v1]) / (am - v1_) * Ul[S2];
    Ur_[S2] = (ap - Pr[v1]) / (ap - v1_) * Ur[S2];
    Ul_[S3] = (am - Pl[v1]) / (am - v1_) * Ul[S3];
    Ur_[S3] = (ap - Pr[v1]) / (ap - v1_) * Ur[S3];
    Ul_[B1] = Uh[B1];
    Ur_[B1] = Uh[B1];
    Ul_[B2] = (am - Pl[v1]) / (am - v1_) * Ul[B2];
    Ur_[B2] = (ap - Pr[v1]) / (ap - v1_) * Ur[B2];
    Ul_[B3] = (am - Pl[v1]) / (am - v1_) * Ul[B3];
    Ur_[B3] = (ap - Pr[v1]) / (ap - v1_) * Ur[B3];
  }
  const T s = T(0);
  if (safeguard) {
    bool bad = !(isfinite(lc) && isfinite(hllc_star_p));
#pragma unroll
    for (int i = 0; i < 8; ++i) bad = bad || !isfinite(Ul_[i]) || !isfinite(Ur_[i]);
    if (bad) {
#pragma unroll
      for (int i = 0; i < 8; ++i) F[i] = (s <= am) ? Fl[i] : (s <= ap ? Fh[i] : Fr[i]);
      F[tau] -= F[ddd];
      return;
    }
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    if (s <= am) F[i] = Fl[i];
    else if (am < s && s <= lc) F[i] = Fl[i] + am * (Ul_[i] - Ul[i]);
    else if (lc < s && s <= ap) F[i] = Fr[i] + ap * (Ur_[i] - Ur[i]);
    else if (ap < s) F[i] = Fr[i];
  }
  F[tau] -= F[ddd];
}


// HllcRmhdRiemannSolver::IntercellFlux at s = 0 (Mara/riemann_hllc-rmhd.cpp:26-178)
template <class T, int dim>
__device__ __forceinline__ int riemann_hllc(T gamma, const T *pl, const T *pr, T *F, T &ml)
{
  using M = DimMap<dim>;
  constexpr int B1 = M::B1;
  T Pl[8], Pr[8], Ul[8], Ur[8], Fl[8], Fr[8], epl, eml, epr, emr;
#pragma unroll
  for (int i = 0; i < 8; ++i) { Pl[i] = pl[i]; Pr[i] = pr[i]; }
  Pl[B1] = Pr[B1] = T(0.5) * (Pl[B1] + Pr[B1]);
  if (prim_to_cons(gamma, Pl, Ul)) return 1;
  if (prim_to_cons(gamma, Pr, Ur)) return 1;
  flux_and_eigenvalues(gamma, Ul, Pl, Fl, epl, eml, dim);
  flux_and_eigenvalues(gamma, Ur, Pr, Fr, epr, emr, dim);
  Ul[tau] += Ul[ddd]; Fl[tau] += Fl[ddd];
  Ur[tau] += Ur[ddd]; Fr[tau] += Fr[ddd];
  const T ap = (epl > epr) ? epl : epr;
  const T am = (eml < emr) ? eml : emr;
  const T l = face_lambda(ap, am);
  if (ml < l) ml = l;
  hllc_star_flux<T, dim>(Pl, Pr, Ul, Ur, Fl, Fr, ap, am, F, sizeof(T) < sizeof(double));
  return 0;
}

// Out-of-line HLLC for the HLLD fallback (rare): arguments and result by value so that the
// caller's face states stay in registers on its hot path.
template <class T> struct Face8 { T v[8]; };
template <class T> struct HllcOut { T F[8]; T ml; int err; };
template <class T, int dim>
static __device__ __noinline__ HllcOut<T> riemann_hllc_fallback(T gamma, Face8<T> pl, Face8<T> pr, T ml)
{
  HllcOut<T> o;
  o.ml = ml;
  o.err = riemann_hllc<T, dim>(gamma, pl.v, pr.v, o.F, o.ml);
  return o;
}

// ---- HLLD (Mignone, Ugliano & Bodo 2009; Mara/riemann_hlld-rmhd.cpp) -------------------------
template <class T> struct HlldJump { T E, D, B[3], m[3]; };
template <class T> struct HlldInner { T B[3], v[3]; };

template <class T>
struct HlldEqn {
  T Ul[8], Ur[8], Fl[8], Fr[8];   // normal-frame states, total-energy convention (tau + D)
  T ap, am, PlBx, PrBx;
  HlldJump<T> L, R;
};

template <class T> __device__ __forceinline__ T dot3(const T *v, const T *w) { return v[0] * w[0] + v[1] * w[1] + v[2] * w[2]; }
template <class T> __device__ __forceinline__ T dot1(const T *v) { return v[0] * v[0] + v[1] * v[1] + v[2] * v[2]; }

template <class T>
__device__ __forceinline__ void hlld_side(const HlldJump<T> &J, T a, T UBx, T p, HlldInner<T> &s)
{
  using Tol = RmhdTol<T>;
  const T A = J.m[0] - a * J.E + p * (T(1) - a * a);
  const T G = J.B[1] * J.B[1] + J.B[2] * J.B[2];
  const T C = J.B[1] * J.m[1] + J.B[2] * J.m[2];
  const T Q = -A - G + (UBx * UBx) * (T(1) - a * a);
  T X = UBx * (A * a * UBx + C) - (A + G) * (a * p + J.E);
  if (m_abs(X) < T(Tol::x_small)) X = T(Tol::x_small);
  s.v[0] = (UBx * (A * UBx + a * C) - (A + G) * (p + J.m[0])) / X;
  s.v[1] = (Q * J.m[1] + J.B[1] * (C + UBx * (a * J.m[0] - J.E))) / X;
  s.v[2] = (Q * J.m[2] + J.B[2] * (C + UBx * (a * J.m[0] - J.E))) / X;
  s.B[0] = (J.B[0] - UBx * s.v[0]) / (a - s.v[0]);
  s.B[1] = (J.B[1] - UBx * s.v[1]) / (a - s.v[0]);
  s.B[2] = (J.B[2] - UBx * s.v[2]) / (a - s.v[0]);
}

// FillInnerWaveStates (riemann_hlld-rmhd.cpp:357-420)
template <class T>
__device__ __forceinline__ void hlld_fill(const HlldEqn<T> &q, T p, T *Kl, T *Kr, T *Bc, T &etaL, T &etaR,
                                          T &wL, T &wR, HlldInner<T> &aL, HlldInner<T> &aR)
{
  using Tol = RmhdTol<T>;
  hlld_side(q.L, q.am, q.Ul[Bx], p, aL);
  hlld_side(q.R, q.ap, q.Ur[Bx], p, aR);
  wL = p + (q.L.E - dot3(aL.v, q.L.m)) / (q.am - aL.v[0]);
  wR = p + (q.R.E - dot3(aR.v, q.R.m)) / (q.ap - aR.v[0]);
  if (wL < T(0)) wL *= T(-1);
  if (wR < T(0)) wR *= T(-1);
  etaL = T(-sgn(q.Ul[Bx])) * m_sqrt(wL);
  etaR = T(+sgn(q.Ur[Bx])) * m_sqrt(wR);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    Kl[k] = (q.L.m[k] + p * T(k == 0) + q.L.B[k] * etaL) / (q.am * p + q.L.E + q.Ul[Bx] * etaL);
    Kr[k] = (q.R.m[k] + p * T(k == 0) + q.R.B[k] * etaR) / (q.ap * p + q.R.E + q.Ur[Bx] * etaR);
    Bc[k] = ((aR.B[k] * (Kr[0] - aR.v[0]) + aR.B[0] * aR.v[k]) -
             (aL.B[k] * (Kl[0] - aL.v[0]) + aL.B[0] * aL.v[k])) / (Kr[0] - Kl[0]);
    if (m_abs(Kr[0] - Kl[0]) < T(Tol::k_small)) Bc[k] = T(0);
  }
}

// HlldEquation48::Function (riemann_hlld-rmhd.cpp:422-452); returns non-zero on "throw".
template <class T>
__device__ __forceinline__ int hlld_function(const HlldEqn<T> &q, T p, T &y)
{
  using Tol = RmhdTol<T>;
  if (m_abs(q.PlBx - q.PrBx) > T(Tol::bjump)) return 1;
  if (isinf(p)) return 1;
  T Kl[3], Kr[3], Bc[3], etaL, etaR, wL, wR;
  HlldInner<T> aL, aR;
  hlld_fill(q, p, Kl, Kr, Bc, etaL, etaR, wL, wR, aL, aR);
  const T delK = Kr[0] - Kl[0];
  const T Bch[3] = { Bc[0] * delK, Bc[1] * delK, Bc[2] * delK };
  const T Yl = (T(1) - dot1(Kl)) / (etaL * delK - dot3(Kl, Bch));
  const T Yr = (T(1) - dot1(Kr)) / (etaR * delK - dot3(Kr, Bch));
  if (m_abs(delK) < T(Tol::k_small)) y = T(0);
  else if (m_abs(Bc[0]) < T(Tol::k_small)) y = delK;
  else y = delK * (T(1) - Bc[0] * (Yr - Yl));
  return 0;
}

// NewtonRaphesonSolver::Solve, rank 1 (nrsolver.cpp:89-152) with the central-difference
// Jacobian of HlldEquation48::Jacobian.  At most 16 evaluations; bounded.
template <class T>
__device__ __forceinline__ int hlld_newton(const HlldEqn<T> &q, T &x)
{
  using Tol = RmhdTol<T>;
  const int MaxIterations = 15;
  const T dp = T(Tol::jac_dp);
  int worse = 0, it = 0;
  T eps = T(0), eps_last;
  do {
    eps_last = eps;
    // f(x), f(x - dp/2), f(x + dp/2): one evaluation site, three points
    T y = T(0), f0 = T(0), f1 = T(0);
#pragma unroll 1
    for (int e = 0; e < 3; ++e) {
      const T pe = e == 0 ? x : (e == 1 ? x - T(0.5) * dp : x + T(0.5) * dp);
      T r;
      if (hlld_function(q, pe, r)) return 1;
      if (e == 0) y = r;
      else if (e == 1) f0 = r;
      else f1 = r;
    }
    const T J = (f1 - f0) / dp;
    const T G = T(1) / J;
    T dx = T(0);
    dx += G * y;
    x -= dx;
    eps = T(0);
    eps += y > T(0) ? y : -y;
    worse += (eps > eps_last);
    if (worse >= 10 || it == MaxIterations) return 1;
    if (isnan(eps)) return 1;
  } while (eps > T(Tol::newton_eps) && ++it <= MaxIterations);
  return 0;
}

// Secant iteration on equation 48 (the structure of SecantMethodSolver::Solve,
// Mara/secant.cpp:19-60, which the reference constructs for this equation but does not
// call): one evaluation per iteration instead of Newton's three.  Used by the FP32-bulk
// path only; the FP64 path keeps the reference's Newton-Raphson.
template <class T>
__device__ __forceinline__ int hlld_secant(const HlldEqn<T> &q, T &x)
{
  using Tol = RmhdTol<T>;
  const int MaxIterations = 15;
  T x0 = x, x1 = x + T(Tol::jac_dp), y0 = T(0), y1 = T(0);
  int worse = 0;
#pragma unroll 1
  for (int it = -2; it <= MaxIterations; ++it) {
    // it == -2, -1: the two starting points; then one secant step per iteration
    T xe;
    if (it == -2) xe = x0;
    else if (it == -1) xe = x1;
    else xe = x1 - y1 * (x1 - x0) / (y1 - y0);
    T r;
    if (hlld_function(q, xe, r)) return 1;
    if (isnan(r)) return 1;
    if (it == -2) {
      y0 = r;
      if (m_abs(y0) < T(Tol::newton_eps)) return 0;
      continue;
    }
    if (it >= 0) {
      x0 = x1;
      y0 = y1;
      x1 = xe;
    }
    y1 = r;
    if (it >= 0) {
      worse += (m_abs(y1) > m_abs(y0));
      if (worse >= 10) return 1;
    }
    if (m_abs(y1) <= T(Tol::newton_eps)) {
      x = x1;
      return 0;
    }
  }
  return 1;
}

// ReconstructSolution (riemann_hlld-rmhd.cpp:453-575) at s = 0, flux only.
template <class T>
__device__ __forceinline__ int hlld_reconstruct(const HlldEqn<T> &q, T p, T *F)
{
  using Tol = RmhdTol<T>;
  T Kl[3], Kr[3], Bc[3], etaL, etaR, wL, wR;
  HlldInner<T> aL, aR;
  hlld_fill(q, p, Kl, Kr, Bc, etaL, etaR, wL, wR, aL, aR);
  const T am = q.am, ap = q.ap;
  const T denomL = etaL - dot3(Kl, Bc);
  const T denomR = etaR - dot3(Kr, Bc);
  T cLv[3], cRv[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    cLv[k] = Kl[k] - Bc[k] * (T(1) - dot1(Kl)) / denomL;
    cRv[k] = Kr[k] - Bc[k] * (T(1) - dot1(Kr)) / denomR;
    if (m_abs(denomL) < T(Tol::k_small)) cLv[k] = aL.v[k];
    if (m_abs(denomR) < T(Tol::k_small)) cRv[k] = aR.v[k];
  }
  const T lamC = cRv[0], lmaL = Kl[0], lmaR = Kr[0], TOL = T(Tol::tol54);
  if (p < T(0)) return 1;
  if (lmaL < T(-1) || lmaR > T(1) || m_abs(lamC) > T(1)) return 1;
  if (!((wL > p) && (aL.v[0] > am - TOL) && (cLv[0] > lmaL - TOL))) return 1;
  if (!((wR > p) && (aR.v[0] < ap + TOL) && (cRv[0] < lmaR + TOL))) return 1;
  if (m_abs(cRv[0] - cLv[0]) > T(Tol::contact)) return 1;

  const T s = T(0);
  // The flux needs only the states of the region containing s = 0 and those between it and
  // the outer fast wave; the region test below is the reference's, evaluated first.
  int region;
  if (s <= am) region = 0;
  else if (am < s && s <= lmaL) region = 1;
  else if (lmaL < s && s <= lamC) region = 2;
  else if (lamC < s && s <= lmaR) region = 3;
  else if (lmaR < s && s <= ap) region = 4;
  else if (ap < s) region = 5;
  else region = 6;   // unordered (NaN) speeds: the reference leaves F unset
  if (region == 6) {
#pragma unroll
    for (int i = 0; i < 8; ++i) F[i] = T(0);
    return 0;
  }
  const bool left = region <= 2;
  const HlldJump<T> &J = left ? q.L : q.R;
  const HlldInner<T> &a = left ? aL : aR;
  const T *Uo = left ? q.Ul : q.Ur;
  const T wave = left ? am : ap;
  // The outer flux.  FP32 bulk recovers it from the jump across the fast wave, Fo = wave Uo - J,
  // so that Fl and Fr are dead through the pressure iteration (sixteen registers); FP64 keeps
  // the stored flux.
  T Fo[8];
  if constexpr (sizeof(T) < sizeof(double)) {
    Fo[ddd] = wave * Uo[ddd] - J.D;
    Fo[tau] = wave * Uo[tau] - J.E;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      Fo[Sx + k] = wave * Uo[Sx + k] - J.m[k];
      Fo[Bx + k] = wave * Uo[Bx + k] - J.B[k];
    }
  } else {
#pragma unroll
    for (int i = 0; i < 8; ++i) Fo[i] = left ? q.Fl[i] : q.Fr[i];
  }
  if (region == 0 || region == 5) {
#pragma unroll
    for (int i = 0; i < 8; ++i) F[i] = Fo[i];
    F[tau] -= F[ddd];
    return 0;
  }
  // States between the fast and Alfven waves (aL / aR)
  T aU[8];
  T denom;
  if (m_abs(denom = wave - a.v[0]) < T(Tol::degenerate)) {
#pragma unroll
    for (int i = 0; i < 8; ++i) aU[i] = Uo[i];
  } else {
    const T vB = dot3(a.v, a.B);
    aU[ddd] = J.D / denom;
    aU[tau] = (J.E + p * a.v[0] - vB * a.B[0]) / denom;
    aU[Sx] = (aU[tau] + p) * a.v[0] - vB * a.B[0];
    aU[Sy] = (aU[tau] + p) * a.v[1] - vB * a.B[1];
    aU[Sz] = (aU[tau] + p) * a.v[2] - vB * a.B[2];
    aU[Bx] = a.B[0];
    aU[By] = a.B[1];
    aU[Bz] = a.B[2];
  }
  if (region == 1 || region == 4) {
#pragma unroll
    for (int i = 0; i < 8; ++i) F[i] = Fo[i] + wave * (aU[i] - Uo[i]);
    F[tau] -= F[ddd];
    return 0;
  }
  // States between the Alfven and contact waves (cL / cR)
  const T lma = left ? lmaL : lmaR;
  const T *cv = left ? cLv : cRv;
  T cU[8];
  if (m_abs(denom = lma - lamC) < T(Tol::degenerate)) {
#pragma unroll
    for (int i = 0; i < 8; ++i) cU[i] = aU[i];
  } else {
    const T vBc = dot3(cv, Bc);
    cU[ddd] = aU[ddd] * (lma - a.v[0]) / denom;
    cU[tau] = (lma * aU[tau] - aU[Sx] + p * lamC - vBc * Bc[0]) / denom;
    cU[Sx] = (cU[tau] + p) * cv[0] - vBc * Bc[0];
    cU[Sy] = (cU[tau] + p) * cv[1] - vBc * Bc[1];
    cU[Sz] = (cU[tau] + p) * cv[2] - vBc * Bc[2];
    cU[Bx] = Bc[0];
    cU[By] = Bc[1];
    cU[Bz] = Bc[2];
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) F[i] = Fo[i] + wave * (aU[i] - Uo[i]) + lma * (cU[i] - aU[i]);
  F[tau] -= F[ddd];
  return 0;
}

// First attempt of the HLL-state c2p in the FP32-bulk HLLD: the Anton et al. 2-D Newton of
// c2p_anton2dzw_fast in FP32 from the average face state (in P), to a step tolerance of 1e-6,
// with the reference's clamps, reconstruction, pressure floor and checks.  The HLL state's
// primitives only seed the eq. 48 pressure guess and are kept in FP32 anyway, so an FP32
// polish loses nothing; returns nonzero (the caller then runs the FP64 ladder) when the state
// fails check_cons, the guess is unusable, Newton does not converge in 32 iterations or the
// primitives fail check_prim.
__device__ __forceinline__ int c2p_hll_f32(const PhysParams &pp, const float *U, float *P, int &iters)
{
  iters = 0;
  if (check_cons(U)) return 1;
  const float V2g = P[vx] * P[vx] + P[vy] * P[vy] + P[vz] * P[vz];
  if (!(V2g < 1.f && P[rho] > 0.f && P[pre] > 0.f)) return 1;
  const float gamma = float(pp.gamma), gamf = (gamma - 1.f) / gamma;
  const float D = U[ddd], Tau = U[tau];
  const float S2 = U[Sx] * U[Sx] + U[Sy] * U[Sy] + U[Sz] * U[Sz];
  const float B2 = U[Bx] * U[Bx] + U[By] * U[By] + U[Bz] * U[Bz];
  const float BS = U[Bx] * U[Sx] + U[By] * U[Sy] + U[Bz] * U[Sz];
  const float BS2 = BS * BS;
  const float W2g = 1.f / (1.f - V2g);
  float Z = P[rho] * (1.f + P[pre] / P[rho] * (1.f / (gamma - 1.f) + 1.f)) * W2g;
  float W = sqrtf(W2g);
  const float iD = 1.f / D;
  float iW = 1.f / W, iZ = 1.f / Z;
  float error = 1.f;
  while (error > 1e-6f) {
    const float W2 = W * W, Z2 = Z * Z, Z3 = Z * Z2;
    const float iW2 = iW * iW, iW3 = iW2 * iW, iZ2 = iZ * iZ, iZ3 = iZ2 * iZ;
    const float Pre = D * iW * (Z * iD * iW - 1.f) * gamf;
    const float BZ = B2 + Z;
    const float df0dZ = 2.f * BZ * (BS2 * W2 + (W2 - 1.f) * Z3) * iW2 * iZ3;
    const float df0dW = 2.f * BZ * BZ * iW3;
    const float df1dZ = 1.f + BS2 * iZ3 - gamf * iW2;
    const float df1dW = (B2 + (2.f * Z - D * W) * gamf) * iW3;
    const float f0 = -S2 + BZ * BZ * (W2 - 1.f) * iW2 - (2.f * Z + B2) * BS2 * iZ2;
    const float f1 = -Tau + Z + B2 - Pre - 0.5f * B2 * iW2 - 0.5f * BS2 * iZ2 - D;
    const float idet = 1.f / (df0dZ * df1dW - df0dW * df1dZ);
    const float dZ = -(df1dW * f0 - df0dW * f1) * idet;
    const float dW = -(df0dZ * f1 - df1dZ * f0) * idet;
    float Zn = fabsf(Z + dZ), Wn = W + dW;
    Zn = (Zn < 1e20f) ? Zn : Z;
    Wn = fminf(fmaxf(Wn, 1.f), 1e12f);
    Z = Zn;
    W = Wn;
    iZ = 1.f / Z;
    iW = 1.f / W;
    error = fabsf(dZ * iZ) + fabsf(dW * iW);
    if (!(error == error) || ++iters == 32) return 1;
  }
  float Q[8];
  const float b0 = BS * W * iZ;
  Q[rho] = D * iW;
  Q[pre] = D * iW * (Z * iD * iW - 1.f) * gamf;
  const float iZB = 1.f / (Z + B2);
  Q[vx] = (U[Sx] + b0 * U[Bx] * iW) * iZB;
  Q[vy] = (U[Sy] + b0 * U[By] * iW) * iZB;
  Q[vz] = (U[Sz] + b0 * U[Bz] * iW) * iZB;
  Q[Bx] = U[Bx];
  Q[By] = U[By];
  Q[Bz] = U[Bz];
  if (pp.pfloor > 0.0 && Q[pre] < float(pp.pfloor)) Q[pre] = float(pp.pfloor);
  if (check_prim(Q)) return 1;
#pragma unroll
  for (int i = 0; i < 8; ++i) P[i] = Q[i];
  return 0;
}

// Converts a flux-solver state to double for the FP64 c2p and back.  P holds the average of
// the two face states on entry.  The FP64 path runs the reference's ladder as it is (first
// attempt from the estimate of the conserved state).  The FP32-bulk path first tries
// c2p_hll_f32; when that fails it runs the FP64 Newton from the average state -- in smooth
// flow the HLL state's primitives are close to it, so that polish takes 2 iterations instead
// of 6 (measured, 256^3 turbulence) -- and then the estimate and the reference ladder; the
// root it lands on is the same to the Newton tolerance.
template <class T>
__device__ __forceinline__ int cons_to_prim_T(const PhysParams &pp, const T *U, T *P, C2PTally *tally)
{
  if constexpr (sizeof(T) < sizeof(double)) {
    int it = 0;
    if (c2p_hll_f32(pp, U, P, it) == 0) {
      if (tally) { tally->iters = it; tally->attempts = 1; }
      return 0;
    }
  }
  double Ud[8], Pd[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) { Ud[i] = double(U[i]); Pd[i] = double(P[i]); }
  int e;
  if constexpr (sizeof(T) < sizeof(double)) {
    const double V2 = Pd[vx] * Pd[vx] + Pd[vy] * Pd[vy] + Pd[vz] * Pd[vz];
    const double W2 = 1.0 / (1.0 - V2);
    const double h = 1.0 + Pd[pre] / Pd[rho] * (1.0 / (pp.gamma - 1.0) + 1.0);   // 1 + e + p/rho
    const bool usable = V2 < 1.0 && Pd[rho] > 0.0 && Pd[pre] > 0.0;
    e = cons_to_prim<true, 1>(pp, Ud, Pd, tally, Pd[rho] * h * W2, sqrt(W2), usable);
  } else {
    e = cons_to_prim<false, 2>(pp, Ud, Pd, tally);
  }
  if (e == 0) {
#pragma unroll
    for (int i = 0; i < 8; ++i) P[i] = T(Pd[i]);
  }
  return e;
}

// HLL total pressure, EstimateSolution(0) (riemann_hlld-rmhd.cpp:543-553), from the HLL
// state's primitives.
template <class T>
__device__ __forceinline__ T hlld_estimate0(const T *P)
{
  const T V2 = P[vx] * P[vx] + P[vy] * P[vy] + P[vz] * P[vz];
  const T B2 = P[Bx] * P[Bx] + P[By] * P[By] + P[Bz] * P[Bz];
  const T Bv = P[Bx] * P[vx] + P[By] * P[vy] + P[Bz] * P[vz];
  const T W2 = T(1) / (T(1) - V2);
  const T W = m_sqrt(W2);
  const T b0 = W * Bv;
  const T b2 = (B2 + b0 * b0) / W2;
  return P[pre] + T(0.5) * b2;
}

// Eq. (55), EstimateSolution(1) (riemann_hlld-rmhd.cpp:557-574): the smaller root of
// p^2 + (E - Fm) p + (FE m - E Fm) = 0 from the HLL state's total energy E, normal momentum m
// and their fluxes.
template <class T>
__device__ __forceinline__ T hlld_estimate1(T E, T FE, T m, T Fm)
{
  const T a = T(1);
  const T b = E - Fm;
  const T c = FE * m - E * Fm;
  const T p1 = m_abs((-b + m_sqrt(b * b - T(4) * a * c)) / (T(2) * a));
  const T p2 = m_abs((-b - m_sqrt(b * b - T(4) * a * c)) / (T(2) * a));
  return (p1 < p2) ? p1 : p2;
}

// HlldRmhdRiemannSolver::IntercellFlux at s = 0 (riemann_hlld-rmhd.cpp:179-313).
// Returns 1 when a face state is unphysical (the caller retries with PCM states);
// `used_hllc` reports the fallback.
// A thread's slot for the HLLD equation state in shared memory (53 words: an odd stride, so
// the threads of a warp hit different banks).
template <class T>
struct HlldSlot {
  HlldEqn<T> q;
  T pad;
};

// slot: where the equation state lives through the pressure iteration -- nullptr for
// registers (the compiler's choice), or this thread's HlldSlot in shared memory, so that the
// ~50 values are read from there when needed instead of occupying registers throughout.
template <class T, int dim>
__device__ __forceinline__ int riemann_hlld(const PhysParams &pp, const T *pl, const T *pr, T *f, T &ml,
                                         int &used_hllc, C2PTally *tally, HlldSlot<T> *slot = nullptr)
{
  using Tol = RmhdTol<T>;
  const T gamma = T(pp.gamma);
  using M = DimMap<dim>;
  constexpr int B1 = M::B1, B2 = M::B2, B3 = M::B3, S1 = M::S1, S2 = M::S2, S3 = M::S3;
  constexpr int v1 = M::v1, v2 = M::v2, v3 = M::v3;
  HlldEqn<T> q_regs;
  HlldEqn<T> &q = slot ? slot->q : q_regs;
  T Pl[8], Pr[8], epl, eml, epr, emr;
  Pl[pre] = pl[pre]; Pr[pre] = pr[pre];
  Pl[rho] = pl[rho]; Pr[rho] = pr[rho];
  Pl[vx] = pl[v1];   Pr[vx] = pr[v1];
  Pl[vy] = pl[v2];   Pr[vy] = pr[v2];
  Pl[vz] = pl[v3];   Pr[vz] = pr[v3];
  Pl[By] = pl[B2];   Pr[By] = pr[B2];
  Pl[Bz] = pl[B3];   Pr[Bz] = pr[B3];
  Pl[Bx] = Pr[Bx] = T(0.5) * (pl[B1] + pr[B1]);
  used_hllc = 0;
  if (tally) { tally->iters = 0; tally->attempts = 0; }
  if (prim_to_cons(gamma, Pl, q.Ul)) return 1;
  if (prim_to_cons(gamma, Pr, q.Ur)) return 1;
  flux_and_eigenvalues(gamma, q.Ul, Pl, q.Fl, epl, eml, 1);
  flux_and_eigenvalues(gamma, q.Ur, Pr, q.Fr, epr, emr, 1);
  const T am = (eml < emr) ? eml : emr;
  const T ap = (epl > epr) ? epl : epr;
  const T l = face_lambda(ap, am);
  if (ml < l) ml = l;
  T P_hll[8], U_hll[8], F_hll[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    P_hll[i] = T(0.5) * (Pl[i] + Pr[i]);
    U_hll[i] = (ap * q.Ur[i] - am * q.Ul[i] + (q.Fl[i] - q.Fr[i])) / (ap - am);
    F_hll[i] = (ap * q.Fl[i] - am * q.Fr[i] + ap * am * (q.Ur[i] - q.Ul[i])) / (ap - am);
  }
  const int hll_c2p_failed = cons_to_prim_T(pp, U_hll, P_hll, tally);
  // FP32 bulk takes both pressure estimates here, so that P_hll, U_hll and F_hll are dead
  // through the pressure iteration; FP64 keeps the reference's order (and its in-place shift
  // and restore of tau, which the Bx ~ 0 retries repeat).
  T p_est0 = T(0), p_est1 = T(0);
  if constexpr (sizeof(T) < sizeof(double)) {
    p_est0 = hlld_estimate0(P_hll);
    p_est1 = hlld_estimate1(U_hll[tau] + U_hll[ddd], F_hll[tau] + F_hll[ddd], U_hll[Sx], F_hll[Sx]);
  }
  // HlldEquation48 constructor (riemann_hlld-rmhd.cpp:315-345)
  q.ap = ap; q.am = am; q.PlBx = Pl[Bx]; q.PrBx = Pr[Bx];
  q.Ul[tau] += q.Ul[ddd];
  q.Fl[tau] += q.Fl[ddd];
  q.Ur[tau] += q.Ur[ddd];
  q.Fr[tau] += q.Fr[ddd];
  q.L.E = am * q.Ul[tau] - q.Fl[tau];
  q.R.E = ap * q.Ur[tau] - q.Fr[tau];
  q.L.D = am * q.Ul[ddd] - q.Fl[ddd];
  q.R.D = ap * q.Ur[ddd] - q.Fr[ddd];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    q.L.B[k] = am * q.Ul[Bx + k] - q.Fl[Bx + k];
    q.R.B[k] = ap * q.Ur[Bx + k] - q.Fr[Bx + k];
    q.L.m[k] = am * q.Ul[Sx + k] - q.Fl[Sx + k];
    q.R.m[k] = ap * q.Ur[Sx + k] - q.Fr[Sx + k];
  }
  T F[8];
  int attempt = 0, success = 0;
  while (!hll_c2p_failed && attempt < 3 && !success) {
    T p_star;
    int rc;
    const int est = (m_abs(Pl[Bx]) < T(Tol::bx_small) || m_abs(Pr[Bx]) < T(Tol::bx_small)) ? 1 : attempt;
    if constexpr (sizeof(T) < sizeof(double)) {
      p_star = est == 0 ? p_est0 : (est == 1 ? p_est1 : T(0));
    } else if (est == 0) {
      p_star = hlld_estimate0(P_hll);
    } else if (est == 1) {   // EstimateSolution(1) shifts tau and restores it afterwards
      F_hll[tau] += F_hll[ddd];
      U_hll[tau] += U_hll[ddd];
      p_star = hlld_estimate1(U_hll[tau], F_hll[tau], U_hll[Sx], F_hll[Sx]);
      F_hll[tau] -= F_hll[ddd];
      U_hll[tau] -= U_hll[ddd];
    } else {
      p_star = T(0);
    }
    if (m_abs(Pl[Bx]) < T(Tol::bx_small) || m_abs(Pr[Bx]) < T(Tol::bx_small)) {
      rc = hlld_reconstruct(q, p_star, F);
    } else {
      rc = sizeof(T) < sizeof(double) ? hlld_secant(q, p_star) : hlld_newton(q, p_star);
      if (rc == 0) rc = hlld_reconstruct(q, p_star, F);
    }
    success = (rc == 0);
    ++attempt;
  }
  if (success) {
    f[ddd] = F[ddd];
    f[tau] = F[tau];
    f[S1] = F[Sx];
    f[S2] = F[Sy];
    f[S3] = F[Sz];
    f[B1] = F[Bx];
    f[B2] = F[By];
    f[B3] = F[Bz];
    return 0;
  }
  used_hllc = 1;
  Face8<T> a, b;
#pragma unroll
  for (int i = 0; i < 8; ++i) { a.v[i] = pl[i]; b.v[i] = pr[i]; }
  const HllcOut<T> o = riemann_hllc_fallback<T, dim>(gamma, a, b, ml);
  ml = o.ml;
#pragma unroll
  for (int i = 0; i < 8; ++i) f[i] = o.F[i];
  return o.err;
}

}  // namespace mgpu
