/* CPU restatement of Mara's RMHD step -- the oracle for the CUDA path.
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the CPU-baseline
 * leg of bench.py, never by the product library.  Every function names the reference
 * source it restates (paths relative to the reference project).  Arithmetic is written in
 * the reference's operation order and compiled with -ffp-contract=off so that, like the
 * reference's gcc -O3 x86-64 build, no multiply-add is fused.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "mara_port.h"

enum { ddd, tau, Sx, Sy, Sz, Bx, By, Bz };   /* conserved, Mara/rmhd.hpp:19 */
enum { rho, pre, vx, vy, vz };               /* primitive, Mara/rmhd.hpp:20 */

enum { C2P_SUCCESS, C2P_CONS_NAN, C2P_CONS_NEG_DENSITY, C2P_CONS_NEG_ENERGY,
       C2P_PRIM_NAN, C2P_PRIM_NEG_PRESSURE, C2P_PRIM_NEG_RESTMASS,
       C2P_PRIM_SUPERLUMINAL, C2P_MAXITER };                 /* Mara/rmhd-c2p.h:10-20 */

#define SGN(x) (((x) > 0) - ((x) < 0))

/* Conditioning probe (oracle variant built with -DPORT_PERTURB_LIBM only): moves each libm
 * result of the wave-speed quartic by one ulp, to measure how sensitive the reference's own
 * result is to the last bit of pow/acos/cos/sin. */
#ifdef PORT_PERTURB_LIBM
#define LIBM(x) nextafter((x), INFINITY)
#else
#define LIBM(x) (x)
#endif

void port_default_config(port_config *c)
{
  memset(c, 0, sizeof(*c));
  c->nd = 3; c->n[0] = c->n[1] = c->n[2] = 8; c->ng = 3;
  c->x1[0] = c->x1[1] = c->x1[2] = 1.0;
  c->gamma = 4.0 / 3.0;
  c->recon = 1; c->theta = 2.0; c->is_mode = 0; c->sz10A = 50.0;
  c->riemann = 2; c->rk = 2; c->pfloor = -1.0;
  c->ereset = 0; c->preset = 1.0; c->dreset = 1.0;
}

static void shape(const port_config *c, int G[3])
{
  for (int d = 0; d < 3; ++d) G[d] = (d < c->nd) ? c->n[d] + 2 * c->ng : 1;
}

long port_num_zones(const port_config *c)
{
  int G[3];
  shape(c, G);
  return (long) G[0] * G[1] * G[2];
}

/* ---- EOS: AdiabaticEos (Mara/eos.cpp:13-29) ------------------------------------------ */
static double eos_internal(const port_config *c, double p) { return p / (c->gamma - 1); }
static double eos_cs2(const port_config *c, double r, double p)
{
  const double rhoh = r + eos_internal(c, p) + p;
  return c->gamma * p / rhoh;
}

/* ---- c2p: Mara/rmhd-c2p.c ------------------------------------------------------------- */
typedef struct {
  double gamma, gamf, pfloor;
  double D, Tau, S2, B2, BS, BS2, U[8];
  double Zs, Ws;
  int iters;
} c2p_state;

static void c2p_init(c2p_state *s, const port_config *c)
{
  s->gamma = c->gamma;
  s->gamf = (c->gamma - 1.0) / c->gamma;                       /* :110-114 */
  s->pfloor = c->pfloor;
  s->iters = 0;
}

static void c2p_new_state(c2p_state *s, const double *U)     /* :132-142 */
{
  s->D = U[ddd];
  s->Tau = U[tau];
  s->S2 = U[Sx] * U[Sx] + U[Sy] * U[Sy] + U[Sz] * U[Sz];
  s->B2 = U[Bx] * U[Bx] + U[By] * U[By] + U[Bz] * U[Bz];
  s->BS = U[Bx] * U[Sx] + U[By] * U[Sy] + U[Bz] * U[Sz];
  s->BS2 = s->BS * s->BS;
  memcpy(s->U, U, sizeof(s->U));
}

static void c2p_estimate(c2p_state *s)                      /* :146-150 */
{
  s->Zs = sqrt(s->S2 + s->D * s->D);
  s->Ws = s->Zs / s->D;
}

static void c2p_starting_prim(c2p_state *s, const double *P) /* :158-167 */
{
  const double V2 = P[vx] * P[vx] + P[vy] * P[vy] + P[vz] * P[vz];
  const double W2 = 1.0 / (1.0 - V2);
  const double e = P[pre] / (P[rho] * (s->gamma - 1.0));
  const double h = 1.0 + e + P[pre] / P[rho];
  s->Zs = P[rho] * h * W2;
  s->Ws = sqrt(W2);
}

static int check_cons(const double *U)                       /* :203-214 */
{
  if (U[ddd] < 0.0) return C2P_CONS_NEG_DENSITY;
  if (U[tau] < 0.0) return C2P_CONS_NEG_ENERGY;
  for (int i = 0; i < 8; ++i) if (isnan(U[i])) return C2P_CONS_NAN;
  return C2P_SUCCESS;
}

static int check_prim(const double *P)                       /* :215-228 */
{
  const double v2 = P[vx] * P[vx] + P[vy] * P[vy] + P[vz] * P[vz];
  if (v2 >= 1.0) return C2P_PRIM_SUPERLUMINAL;
  if (P[pre] < 0.0) return C2P_PRIM_NEG_PRESSURE;
  if (P[rho] < 0.0) return C2P_PRIM_NEG_RESTMASS;
  for (int i = 0; i < 8; ++i) if (isnan(P[i])) return C2P_PRIM_NAN;
  return C2P_SUCCESS;
}

static int c2p_reconstruct(const c2p_state *s, double Z, double W, double *Pout) /* :171-199 */
{
  double P[8];
  const double b0 = s->BS * W / Z;
  P[rho] = s->D / W;
  P[pre] = (s->D / W) * (Z / (s->D * W) - 1.0) * s->gamf;
  P[vx] = (s->U[Sx] + b0 * s->U[Bx] / W) / (Z + s->B2);
  P[vy] = (s->U[Sy] + b0 * s->U[By] / W) / (Z + s->B2);
  P[vz] = (s->U[Sz] + b0 * s->U[Bz] / W) / (Z + s->B2);
  P[Bx] = s->U[Bx];
  P[By] = s->U[By];
  P[Bz] = s->U[Bz];
  if (P[pre] < s->pfloor && s->pfloor > 0.0) P[pre] = s->pfloor;
  int e = check_prim(P);
  if (e) return e;
  memcpy(Pout, P, sizeof(P));
  return C2P_SUCCESS;
}

static int c2p_anton2dzw(c2p_state *s, double *P)            /* :232-303 */
{
  int bad = check_cons(s->U);
  if (bad) return bad;
  s->iters = 0;
  double error = 1.0, W = s->Ws, Z = s->Zs;
  const double D = s->D, B2 = s->B2, BS2 = s->BS2, S2 = s->S2, gamf = s->gamf;
  while (error > 1e-12) {
    const double Z2 = Z * Z, Z3 = Z * Z2, W2 = W * W, W3 = W * W2;
    const double Pre = (D / W) * (Z / (D * W) - 1.0) * gamf;
    const double df0dZ = 2 * (B2 + Z) * (BS2 * W2 + (W2 - 1) * Z3) / (W2 * Z3);
    const double df0dW = 2 * (B2 + Z) * (B2 + Z) / W3;
    const double df1dZ = 1.0 + BS2 / Z3 - gamf / W2;
    const double df1dW = B2 / W3 + (2 * Z - D * W) / W3 * gamf;
    const double f0 = -S2 + (Z + B2) * (Z + B2) * (W2 - 1) / W2 - (2 * Z + B2) * BS2 / Z2;
    const double f1 = -s->Tau + Z + B2 - Pre - 0.5 * B2 / W2 - 0.5 * BS2 / Z2 - D;
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
    if (++s->iters == 250) return C2P_MAXITER;
  }
  return c2p_reconstruct(s, Z, W, P);
}

static int c2p_noble1dw(c2p_state *s, double *P)             /* :311-376 */
{
  int bad = check_cons(s->U);
  if (bad) return bad;
  s->iters = 0;
  double error = 1.0, Z = s->Zs;
  const double D = s->D, B2 = s->B2, BS2 = s->BS2, S2 = s->S2, gamf = s->gamf;
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
    const double f = s->Tau + D - 0.5 * B2 * (1 + V2) + 0.5 * BS2 / Z2 - Z + Pre;
    const double g = -0.5 * B2 * dv2dZ - BS2 / Z3 - 1.0 + dPdZ;
    const double dZ = -f / g;
    double Zn = Z + dZ;
    Zn = (Zn > 0.0) ? Zn : -Zn;
    Zn = (Zn < 1e20) ? Zn : Z;
    Z = Zn;
    error = fabs(dZ / Z);
    if (++s->iters == 250) return C2P_MAXITER;
  }
  const double Z2 = Z * Z;
  const double a = S2 * Z2 + BS2 * (B2 + 2 * Z);
  const double b = (B2 + Z) * (B2 + Z) * Z2;
  const double V2 = a / b;
  const double W2 = 1.0 / (1.0 - V2);
  const double W = sqrt(W2);
  return c2p_reconstruct(s, Z, W, P);
}

/* AdiabaticIdealRmhd::ConsToPrim, gamma-law branch (Mara/rmhd.cpp:103-176): the
 * four-attempt ladder.  P holds the previous primitive state on entry (used as the
 * second guess) and is written only on success. */
int port_cons_to_prim(const port_config *c, const double *U, double *P)
{
  int error = check_cons(U);
  if (error) return error;
  c2p_state s;
  c2p_init(&s, c);
  c2p_new_state(&s, U);
  c2p_estimate(&s);
  error = c2p_anton2dzw(&s, P);
  if (error) { c2p_starting_prim(&s, P); error = c2p_anton2dzw(&s, P); }
  if (error) { c2p_estimate(&s); error = c2p_noble1dw(&s, P); }
  if (error) { c2p_starting_prim(&s, P); error = c2p_noble1dw(&s, P); }
  return error;
}

int port_c2p_solve(const port_config *c, const double *U, int solver, int guess,
                   const double *Pguess, double *P, int *iters)
{
  c2p_state s;
  c2p_init(&s, c);
  c2p_new_state(&s, U);
  if (guess == 0) c2p_estimate(&s); else c2p_starting_prim(&s, Pguess);
  int e = solver == 0 ? c2p_anton2dzw(&s, P) : c2p_noble1dw(&s, P);
  if (iters) *iters = s.iters;
  return e;
}

/* ---- P -> U: AdiabaticIdealRmhd::PrimToCons (Mara/rmhd.cpp:177-207) -------------------- */
int port_prim_to_cons(const port_config *c, const double *P, double *U)
{
  const double V2 = P[vx] * P[vx] + P[vy] * P[vy] + P[vz] * P[vz];
  const double B2 = P[Bx] * P[Bx] + P[By] * P[By] + P[Bz] * P[Bz];
  const double Bv = P[Bx] * P[vx] + P[By] * P[vy] + P[Bz] * P[vz];
  const double W2 = 1.0 / (1.0 - V2);
  const double W = sqrt(W2);
  const double b0 = W * Bv;
  const double b2 = (B2 + b0 * b0) / W2;
  const double bx = (P[Bx] + b0 * W * P[vx]) / W;
  const double by = (P[By] + b0 * W * P[vy]) / W;
  const double bz = (P[Bz] + b0 * W * P[vz]) / W;
  const double e = eos_internal(c, P[pre]) / P[rho];
  const double e_ = e + 0.5 * b2 / P[rho];
  const double p_ = P[pre] + 0.5 * b2;
  const double h_ = 1 + e_ + p_ / P[rho];
  U[ddd] = P[rho] * W;
  U[tau] = P[rho] * h_ * W2 - p_ - b0 * b0 - U[ddd];
  U[Sx] = P[rho] * h_ * W2 * P[vx] - b0 * bx;
  U[Sy] = P[rho] * h_ * W2 * P[vy] - b0 * by;
  U[Sz] = P[rho] * h_ * W2 * P[vz] - b0 * bz;
  U[Bx] = P[Bx];
  U[By] = P[By];
  U[Bz] = P[Bz];
  if (V2 >= 1.0) return C2P_PRIM_SUPERLUMINAL;
  return check_cons(U);
}

/* ---- quartic: QuarticEquation::SolveOld + solve_cubic_equation (Mara/quartic.cpp:28-148) */
static void cubic(double c3, double c2, double c1, double c0, double *x1, double *x2,
                  double *x3, int *nr)
{
  const double a2 = c2 / c3, a1 = c1 / c3, a0 = c0 / c3;
  const double q = a1 / 3.0 - a2 * a2 / 9.0;
  const double r = (a1 * a2 - 3.0 * a0) / 6.0 - a2 * a2 * a2 / 27.0;
  const double delta = q * q * q + r * r;
  if (delta > 0.0) {
    double s1 = r + sqrt(delta);
    s1 = (s1 >= 0.0) ? LIBM(pow(s1, 1. / 3.)) : -LIBM(pow(-s1, 1. / 3.));
    double s2 = r - sqrt(delta);
    s2 = (s2 >= 0.0) ? LIBM(pow(s2, 1. / 3.)) : -LIBM(pow(-s2, 1. / 3.));
    *x1 = (s1 + s2) - a2 / 3.0;
    *x2 = *x3 = -0.5 * (s1 + s2) - a2 / 3.0;
    *nr = 1;
  } else if (delta < 0.0) {
    const double theta = LIBM(acos(r / sqrt(-q * q * q))) / 3.0;
    const double costh = LIBM(cos(theta)), sinth = LIBM(sin(theta)), sq = sqrt(-q);
    *x1 = 2.0 * sq * costh - a2 / 3.0;
    *x2 = -sq * costh - a2 / 3.0 - sqrt(3.) * sq * sinth;
    *x3 = -sq * costh - a2 / 3.0 + sqrt(3.) * sq * sinth;
    *nr = 3;
  } else {
    const double s = (r >= 0.0) ? LIBM(pow(r, 1. / 3.)) : -LIBM(pow(-r, 1. / 3.));
    *x1 = 2.0 * s - a2 / 3.0;
    *x2 = *x3 = -s - a2 / 3.0;
    *nr = 3;
  }
}

int port_quartic(double d4, double d3, double d2, double d1, double d0, double *roots)
{
  double r1, r2, r3, r4;
  int nr12, nr34;
  const double a3 = d3 / d4, a2 = d2 / d4, a1 = d1 / d4, a0 = d0 / d4;
  const double au2 = -a2;
  const double au1 = (a1 * a3 - 4.0 * a0);
  const double au0 = 4.0 * a0 * a2 - a1 * a1 - a0 * a3 * a3;
  double x1, x2, x3;
  int nr;
  cubic(1.0, au2, au1, au0, &x1, &x2, &x3, &nr);
  const double u1 = (nr == 1) ? x1 : ((x1 > x3) ? x1 : x3);
  const double R2 = 0.25 * a3 * a3 + u1 - a2;
  const double R = (R2 > 0.0) ? sqrt(R2) : 0.0;
  double D2, E2;
  if (R != 0.0) {
    const double foo1 = 0.75 * a3 * a3 - R2 - 2.0 * a2;
    const double foo2 = 0.25 * (4.0 * a3 * a2 - 8.0 * a1 - a3 * a3 * a3) / R;
    D2 = foo1 + foo2;
    E2 = foo1 - foo2;
  } else {
    const double foo1 = 0.75 * a3 * a3 - 2.0 * a2;
    const double foo2 = 2.0 * sqrt(u1 * u1 - 4.0 * a0);
    D2 = foo1 + foo2;
    E2 = foo1 - foo2;
  }
  if (D2 >= 0.0) {
    const double D = sqrt(D2);
    r1 = -0.25 * a3 + 0.5 * R - 0.5 * D;
    r2 = -0.25 * a3 + 0.5 * R + 0.5 * D;
    nr12 = 2;
  } else {
    r1 = r2 = -0.25 * a3 + 0.5 * R;
    nr12 = 0;
  }
  if (E2 >= 0.0) {
    const double E = sqrt(E2);
    r3 = -0.25 * a3 - 0.5 * R - 0.5 * E;
    r4 = -0.25 * a3 - 0.5 * R + 0.5 * E;
    nr34 = 2;
  } else {
    r3 = r4 = -0.25 * a3 - 0.5 * R;
    nr34 = 0;
  }
  int i = 0;
  if (nr12) { roots[i++] = r1; roots[i++] = r2; }
  if (nr34) { roots[i++] = r3; roots[i++] = r4; }
  return nr12 + nr34;
}

/* ---- flux + fast speeds: AdiabaticIdealRmhd::FluxAndEigenvalues (Mara/rmhd.cpp:208-310) */
void port_flux_and_eigenvalues(const port_config *c, const double *U, const double *P,
                               double *F, double *ap, double *am, int dim)
{
  const double V2 = P[vx] * P[vx] + P[vy] * P[vy] + P[vz] * P[vz];
  const double B2 = P[Bx] * P[Bx] + P[By] * P[By] + P[Bz] * P[Bz];
  const double Bv = P[Bx] * P[vx] + P[By] * P[vy] + P[Bz] * P[vz];
  const double W2 = 1.0 / (1.0 - V2);
  const double W = sqrt(W2);
  const double b0 = W * Bv;
  const double b2 = (B2 + b0 * b0) / W2;
  const double bx = (P[Bx] + b0 * W * P[vx]) / W;
  const double by = (P[By] + b0 * W * P[vy]) / W;
  const double bz = (P[Bz] + b0 * W * P[vz]) / W;
  const double e = eos_internal(c, P[pre]) / P[rho];
  const double p_ = P[pre] + 0.5 * b2;
  const double h = 1 + e + P[pre] / P[rho];
  switch (dim) {
  case 1:
    F[ddd] = U[ddd] * P[vx];
    F[tau] = U[tau] * P[vx] - b0 * P[Bx] / W + p_ * P[vx];
    F[Sx] = U[Sx] * P[vx] - bx * P[Bx] / W + p_;
    F[Sy] = U[Sy] * P[vx] - by * P[Bx] / W;
    F[Sz] = U[Sz] * P[vx] - bz * P[Bx] / W;
    F[Bx] = 0.0;
    F[By] = P[vx] * P[By] - P[vy] * P[Bx];
    F[Bz] = P[vx] * P[Bz] - P[vz] * P[Bx];
    break;
  case 2:
    F[ddd] = U[ddd] * P[vy];
    F[tau] = U[tau] * P[vy] - b0 * P[By] / W + p_ * P[vy];
    F[Sx] = U[Sx] * P[vy] - bx * P[By] / W;
    F[Sy] = U[Sy] * P[vy] - by * P[By] / W + p_;
    F[Sz] = U[Sz] * P[vy] - bz * P[By] / W;
    F[Bx] = P[vy] * P[Bx] - P[vx] * P[By];
    F[By] = 0.0;
    F[Bz] = P[vy] * P[Bz] - P[vz] * P[By];
    break;
  case 3:
    F[ddd] = U[ddd] * P[vz];
    F[tau] = U[tau] * P[vz] - b0 * P[Bz] / W + p_ * P[vz];
    F[Sx] = U[Sx] * P[vz] - bx * P[Bz] / W;
    F[Sy] = U[Sy] * P[vz] - by * P[Bz] / W;
    F[Sz] = U[Sz] * P[vz] - bz * P[Bz] / W + p_;
    F[Bx] = P[vz] * P[Bx] - P[vx] * P[Bz];
    F[By] = P[vz] * P[By] - P[vy] * P[Bz];
    F[Bz] = 0.0;
    break;
  }
  if (ap == NULL || am == NULL) return;
  double vi = 0, bi = 0;
  switch (dim) {
  case 1: vi = P[vx]; bi = bx; break;
  case 2: vi = P[vy]; bi = by; break;
  case 3: vi = P[vz]; bi = bz; break;
  }
  const double cs2 = eos_cs2(c, P[rho], P[pre]);
  const double W4 = W2 * W2, v2 = vi * vi, v3 = vi * v2, v4 = vi * v3;
  const double K = P[rho] * h * (1.0 / cs2 - 1) * W4;
  const double L = -(P[rho] * h + b2 / cs2) * W2;
  const double A4 = K - L - b0 * b0;
  const double A3 = -4 * K * vi + L * vi * 2 + 2 * b0 * bi;
  const double A2 = 6 * K * v2 + L * (1.0 - v2) + b0 * b0 - bi * bi;
  const double A1 = -4 * K * v3 - L * vi * 2 - 2 * b0 * bi;
  const double A0 = K * v4 + L * v2 + bi * bi;
  double roots[4];
  const int nr = port_quartic(A4, A3, A2, A1, A0, roots);
  *ap = -1.0;
  *am = 1.0;
  for (int i = 0; i < nr; ++i) {
    if (roots[i] > *ap) *ap = roots[i];
    if (roots[i] < *am) *am = roots[i];
  }
  if (fabs(*ap) > 1.0 || fabs(*am) > 1.0) { *ap = 1.0; *am = -1.0; }
}

/* ---- reconstruction: Mara/weno.c ------------------------------------------------------ */
static const double C2L_FV[3][3] = { {15./8., -5./4., 3./8.}, {3./8., 3./4., -1./8.},
                                     {-1./8., 3./4., 3./8.} };             /* :21-23 */
static const double C2R_FV[3][3] = { {3./8., 3./4., -1./8.}, {-1./8., 3./4., 3./8.},
                                     {3./8., -5./4., 15./8.} };            /* :24-26 */
static const double D_C2L_FV[3] = { 1./16., 5./8., 5./16. };               /* :27 */
static const double D_C2R_FV[3] = { 5./16., 5./8., 1./16. };               /* :28 */

static double min3(const double *x)
{
  const double x01 = x[0] < x[1] ? x[0] : x[1];
  return x01 < x[2] ? x01 : x[2];
}
static double max3(const double *x)
{
  const double x01 = x[0] > x[1] ? x[0] : x[1];
  return x01 > x[2] ? x01 : x[2];
}

static double plm(const port_config *c, const double *v, double sgn) /* :85-96 */
{
  const double a = c->theta * (v[0] - v[-1]);
  const double b = 0.5 * (v[1] - v[-1]);
  const double cc = c->theta * (v[1] - v[0]);
  const double fabc[3] = { fabs(a), fabs(b), fabs(cc) };
  const double mm = 0.25 * abs(SGN(a) + SGN(b)) * (SGN(a) + SGN(cc)) * min3(fabc);
  return v[0] + sgn * 0.5 * mm;
}

#define SQU(x) ((x) * (x))
static double weno5(const port_config *c, const double *v, const double cf[3][3],
                    const double *d)                                     /* :97-154 */
{
  const double vs[3] = {
    cf[0][0] * v[+0] + cf[0][1] * v[+1] + cf[0][2] * v[2],
    cf[1][0] * v[-1] + cf[1][1] * v[+0] + cf[1][2] * v[1],
    cf[2][0] * v[-2] + cf[2][1] * v[-1] + cf[2][2] * v[0],
  };
  double B[3] = {
    (13. / 12.) * SQU(1 * v[+0] - 2 * v[+1] + 1 * v[+2]) +
    (1. / 4.) * SQU(3 * v[+0] - 4 * v[+1] + 1 * v[+2]),
    (13. / 12.) * SQU(1 * v[-1] - 2 * v[+0] + 1 * v[+1]) +
    (1. / 4.) * SQU(1 * v[-1] - 0 * v[+0] - 1 * v[+1]),
    (13. / 12.) * SQU(1 * v[-2] - 2 * v[-1] + 1 * v[+0]) +
    (1. / 4.) * SQU(1 * v[-2] - 4 * v[-1] + 3 * v[+0])
  };
  double w[3];
  if (c->is_mode == 1) {
    const double eps = 1e-14;
    const double tau5 = fabs(B[0] - B[2]);
    for (int k = 0; k < 3; ++k) w[k] = d[k] * (1.0 + (tau5 / (B[k] + eps)));
  } else if (c->is_mode == 2) {
    const double epsp = 1e-10;
    const double A = c->sz10A;
    const double minB = min3(B), maxB = max3(B);
    const double R0 = minB / (maxB + epsp);
    for (int k = 0; k < 3; ++k) B[k] = R0 * A * minB + B[k];
    for (int k = 0; k < 3; ++k) w[k] = d[k] / SQU(epsp + B[k]);
  } else {
    const double epsp = 1e-6;
    for (int k = 0; k < 3; ++k) w[k] = d[k] / SQU(epsp + B[k]);
  }
  const double wtot = w[0] + w[1] + w[2];
  return (w[0] * vs[0] + w[1] * vs[1] + w[2] * vs[2]) / wtot;
}

/* op codes follow enum ReconstructOperation (Mara/weno.h): 0 PLM_C2L, 1 PLM_C2R,
 * 4 WENO5_FV_C2R, 5 WENO5_FV_C2L (the FD and A2C/C2A variants are not on the path). */
double port_reconstruct(const port_config *c, const double *v, int op)
{
  switch (op) {
  case 0: return plm(c, v, -1.0);
  case 1: return plm(c, v, +1.0);
  case 4: return weno5(c, v, C2R_FV, D_C2R_FV);
  case 5: return weno5(c, v, C2L_FV, D_C2L_FV);
  default: return 0.0;
  }
}

/* ---- Riemann solvers ------------------------------------------------------------------ */
static void hll_state(double ap, double am, const double *Ul, const double *Ur,
                      const double *Fl, const double *Fr, double *Uh, double *Fh)
{
  for (int i = 0; i < 8; ++i) {
    Uh[i] = (ap * Ur[i] - am * Ul[i] + (Fl[i] - Fr[i])) / (ap - am);
    Fh[i] = (ap * Fl[i] - am * Fr[i] + ap * am * (Ur[i] - Ul[i])) / (ap - am);
  }
}

static void note_lambda(port_stats *s, double ap, double am)
{
  const double ml = (fabs(am) < fabs(ap)) ? fabs(ap) : fabs(am);
  if (s->max_lambda < ml) s->max_lambda = ml;
}

/* HllRiemannSolver::IntercellFlux (Mara/riemann_hll.cpp:19-64), at s = 0 */
static int riemann_hll(const port_config *c, port_stats *st, const double *pl,
                       const double *pr, double *F, int dim)
{
  double Ul[8], Ur[8], Fl[8], Fr[8], epl, eml, epr, emr, Uh[8], Fh[8];
  if (port_prim_to_cons(c, pl, Ul)) return 1;
  if (port_prim_to_cons(c, pr, Ur)) return 1;
  port_flux_and_eigenvalues(c, Ul, pl, Fl, &epl, &eml, dim);
  port_flux_and_eigenvalues(c, Ur, pr, Fr, &epr, &emr, dim);
  const double ap = (epl > epr) ? epl : epr;
  const double am = (eml < emr) ? eml : emr;
  note_lambda(st, ap, am);
  hll_state(ap, am, Ul, Ur, Fl, Fr, Uh, Fh);
  const double s = 0.0;
  if (s <= am) memcpy(F, Fl, sizeof(Fl));
  else if (am < s && s <= ap) memcpy(F, Fh, sizeof(Fh));
  else if (ap < s) memcpy(F, Fr, sizeof(Fr));
  return 0;
}

static void dim_map(int dim, int *B1, int *B2, int *B3, int *S1, int *S2, int *S3,
                    int *v1, int *v2, int *v3)
{
  switch (dim) {
  case 1: *B1 = Bx; *B2 = By; *B3 = Bz; *S1 = Sx; *S2 = Sy; *S3 = Sz;
          *v1 = vx; *v2 = vy; *v3 = vz; break;
  case 2: *B1 = By; *B2 = Bz; *B3 = Bx; *S1 = Sy; *S2 = Sz; *S3 = Sx;
          *v1 = vy; *v2 = vz; *v3 = vx; break;
  default: *B1 = Bz; *B2 = Bx; *B3 = By; *S1 = Sz; *S2 = Sx; *S3 = Sy;
           *v1 = vz; *v2 = vx; *v3 = vy; break;
  }
}

/* HllcRmhdRiemannSolver::IntercellFlux (Mara/riemann_hllc-rmhd.cpp:26-178), at s = 0 */
static int riemann_hllc(const port_config *c, port_stats *st, const double *pl,
                        const double *pr, double *F, int dim)
{
  int B1, B2, B3, S1, S2, S3, v1, v2, v3;
  dim_map(dim, &B1, &B2, &B3, &S1, &S2, &S3, &v1, &v2, &v3);
  double Pl[8], Pr[8], Ul[8], Ur[8], Fl[8], Fr[8], epl, eml, epr, emr;
  memcpy(Pl, pl, sizeof(Pl));
  memcpy(Pr, pr, sizeof(Pr));
  Pl[B1] = Pr[B1] = 0.5 * (Pl[B1] + Pr[B1]);
  if (port_prim_to_cons(c, Pl, Ul)) return 1;
  if (port_prim_to_cons(c, Pr, Ur)) return 1;
  port_flux_and_eigenvalues(c, Ul, Pl, Fl, &epl, &eml, dim);
  port_flux_and_eigenvalues(c, Ur, Pr, Fr, &epr, &emr, dim);
  Ul[tau] += Ul[ddd]; Fl[tau] += Fl[ddd];
  Ur[tau] += Ur[ddd]; Fr[tau] += Fr[ddd];
  const double ap = (epl > epr) ? epl : epr;
  const double am = (eml < emr) ? eml : emr;
  note_lambda(st, ap, am);
  double Uh[8], Fh[8];
  hll_state(ap, am, Ul, Ur, Fl, Fr, Uh, Fh);
  double Ul_[8], Ur_[8], P_[8], lc;
  if (fabs(Uh[B1]) > 1e-12) {
    const double BdFB = Uh[B2] * Fh[B2] + Uh[B3] * Fh[B3];
    const double a = Fh[tau] - BdFB;
    const double b = -Fh[S1] - Uh[tau] + (Uh[B2] * Uh[B2] + Uh[B3] * Uh[B3]) +
                     (Fh[B2] * Fh[B2] + Fh[B3] * Fh[B3]);
    const double cc = Uh[S1] - BdFB;
    P_[v1] = lc = (fabs(a) < 1e-10) ? -cc / b : (-b - sqrt(b * b - 4 * a * cc)) / (2 * a);
    P_[v2] = (Uh[B2] * P_[v1] - Fh[B2]) / Uh[B1];
    P_[v3] = (Uh[B3] * P_[v1] - Fh[B3]) / Uh[B1];
    P_[B1] = Uh[B1];
    P_[B2] = Uh[B2];
    P_[B3] = Uh[B3];
    const double vdB = P_[v1] * P_[B1] + P_[v2] * P_[B2] + P_[v3] * P_[B3];
    const double vdv = P_[v1] * P_[v1] + P_[v2] * P_[v2] + P_[v3] * P_[v3];
    const double gm2 = 1.0 / (1.0 - vdv);
    P_[pre] = Fh[S1] + P_[B1] * P_[B1] / gm2 - (Fh[tau] - P_[B1] * vdB) * P_[v1];
    Ul_[ddd] = (am - Pl[v1]) / (am - P_[v1]) * Ul[ddd];
    Ur_[ddd] = (ap - Pr[v1]) / (ap - P_[v1]) * Ur[ddd];
    Ul_[tau] = (am * Ul[tau] - Ul[S1] + P_[pre] * P_[v1] - vdB * P_[B1]) / (am - P_[v1]);
    Ur_[tau] = (ap * Ur[tau] - Ur[S1] + P_[pre] * P_[v1] - vdB * P_[B1]) / (ap - P_[v1]);
    Ul_[S1] = (Ul_[tau] + P_[pre]) * P_[v1] - vdB * P_[B1];
    Ur_[S1] = (Ur_[tau] + P_[pre]) * P_[v1] - vdB * P_[B1];
    Ul_[S2] = (-P_[B1] * (P_[B2] / gm2 + vdB * P_[v2]) + am * Ul[S2] - Fl[S2]) / (am - P_[v1]);
    Ur_[S2] = (-P_[B1] * (P_[B2] / gm2 + vdB * P_[v2]) + ap * Ur[S2] - Fr[S2]) / (ap - P_[v1]);
    Ul_[S3] = (-P_[B1] * (P_[B3] / gm2 + vdB * P_[v3]) + am * Ul[S3] - Fl[S3]) / (am - P_[v1]);
    Ur_[S3] = (-P_[B1] * (P_[B3] / gm2 + vdB * P_[v3]) + ap * Ur[S3] - Fr[S3]) / (ap - P_[v1]);
    Ul_[B1] = Ur_[B1] = P_[B1];
    Ul_[B2] = Ur_[B2] = P_[B2];
    Ul_[B3] = Ur_[B3] = P_[B3];
  } else {
    const double a = Fh[tau];
    const double b = -Fh[S1] - Uh[tau];
    const double cc = Uh[S1];
    const double v1_ = lc = (fabs(a) < 1e-10) ? -cc / b : (-b - sqrt(b * b - 4 * a * cc)) / (2 * a);
    const double p_ = -Fh[tau] * v1_ + Fh[S1];
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
  const double s = 0.0;
  int i;
  if (s <= am) for (i = 0; i < 8; ++i) F[i] = Fl[i];
  else if (am < s && s <= lc) for (i = 0; i < 8; ++i) F[i] = Fl[i] + am * (Ul_[i] - Ul[i]);
  else if (lc < s && s <= ap) for (i = 0; i < 8; ++i) F[i] = Fr[i] + ap * (Ur_[i] - Ur[i]);
  else if (ap < s) for (i = 0; i < 8; ++i) F[i] = Fr[i];
  F[tau] -= F[ddd];
  return 0;
}

/* HlldEquation48 (Mara/riemann_hlld-rmhd.cpp:67-175, 315-615): exceptions become
 * non-zero status codes. */
typedef struct { double E, D, B[3], m[3]; } jump_t;
typedef struct { double U[8], B[3], v[3]; } inner_t;
typedef struct {
  const double *Pl, *Pr;
  double *Ul, *Ur, *Fl, *Fr;
  double ap, am;
  jump_t L, R;
  double *P_hll, *U_hll, *F_hll;
} hlld_eqn;

static double dot3(const double *v, const double *w) { return v[0]*w[0] + v[1]*w[1] + v[2]*w[2]; }
static double dot1(const double *v) { return v[0]*v[0] + v[1]*v[1] + v[2]*v[2]; }

static void hlld_init(hlld_eqn *q)                                     /* :315-345 */
{
  q->Ul[tau] += q->Ul[ddd];
  q->Fl[tau] += q->Fl[ddd];
  q->Ur[tau] += q->Ur[ddd];
  q->Fr[tau] += q->Fr[ddd];
  q->L.E = q->am * q->Ul[tau] - q->Fl[tau];
  q->R.E = q->ap * q->Ur[tau] - q->Fr[tau];
  q->L.D = q->am * q->Ul[ddd] - q->Fl[ddd];
  q->R.D = q->ap * q->Ur[ddd] - q->Fr[ddd];
  for (int k = 0; k < 3; ++k) {
    q->L.B[k] = q->am * q->Ul[Bx + k] - q->Fl[Bx + k];
    q->R.B[k] = q->ap * q->Ur[Bx + k] - q->Fr[Bx + k];
    q->L.m[k] = q->am * q->Ul[Sx + k] - q->Fl[Sx + k];
    q->R.m[k] = q->ap * q->Ur[Sx + k] - q->Fr[Sx + k];
  }
}

static void hlld_side(const jump_t *J, double a, double UBx, double p, inner_t *s)
{
  const double A = J->m[0] - a * J->E + p * (1 - a * a);
  const double G = J->B[1] * J->B[1] + J->B[2] * J->B[2];
  const double C = J->B[1] * J->m[1] + J->B[2] * J->m[2];
  const double Q = -A - G + (UBx * UBx) * (1 - a * a);
  double X = UBx * (A * a * UBx + C) - (A + G) * (a * p + J->E);
  if (fabs(X) < 1e-8) X = 1e-8;
  s->v[0] = (UBx * (A * UBx + a * C) - (A + G) * (p + J->m[0])) / X;
  s->v[1] = (Q * J->m[1] + J->B[1] * (C + UBx * (a * J->m[0] - J->E))) / X;
  s->v[2] = (Q * J->m[2] + J->B[2] * (C + UBx * (a * J->m[0] - J->E))) / X;
  s->B[0] = (J->B[0] - UBx * s->v[0]) / (a - s->v[0]);
  s->B[1] = (J->B[1] - UBx * s->v[1]) / (a - s->v[0]);
  s->B[2] = (J->B[2] - UBx * s->v[2]) / (a - s->v[0]);
}

static void hlld_fill(const hlld_eqn *q, double p, double *Kl, double *Kr, double *Bc,
                      double *etaL, double *etaR, double *wL, double *wR,
                      inner_t *aL, inner_t *aR)                          /* :357-420 */
{
  hlld_side(&q->L, q->am, q->Ul[Bx], p, aL);
  hlld_side(&q->R, q->ap, q->Ur[Bx], p, aR);
  *wL = p + (q->L.E - dot3(aL->v, q->L.m)) / (q->am - aL->v[0]);
  *wR = p + (q->R.E - dot3(aR->v, q->R.m)) / (q->ap - aR->v[0]);
  if (*wL < 0) *wL *= -1;
  if (*wR < 0) *wR *= -1;
  *etaL = -((q->Ul[Bx] > 0) - (q->Ul[Bx] < 0)) * sqrt(*wL);
  *etaR = +((q->Ur[Bx] > 0) - (q->Ur[Bx] < 0)) * sqrt(*wR);
  for (int k = 0; k < 3; ++k) {
    Kl[k] = (q->L.m[k] + p * (k == 0) + q->L.B[k] * *etaL) /
            (q->am * p + q->L.E + q->Ul[Bx] * *etaL);
    Kr[k] = (q->R.m[k] + p * (k == 0) + q->R.B[k] * *etaR) /
            (q->ap * p + q->R.E + q->Ur[Bx] * *etaR);
    Bc[k] = ((aR->B[k] * (Kr[0] - aR->v[0]) + aR->B[0] * aR->v[k]) -
             (aL->B[k] * (Kl[0] - aL->v[0]) + aL->B[0] * aL->v[k])) / (Kr[0] - Kl[0]);
    if (fabs(Kr[0] - Kl[0]) < 1e-10) Bc[k] = 0.0;
  }
}

static int hlld_function(const hlld_eqn *q, double p, double *y)      /* :422-452 */
{
  if (fabs(q->Pl[Bx] - q->Pr[Bx]) > 1e-12) return 1;
  if (isinf(p)) return 1;
  double Kl[3], Kr[3], Bc[3], etaL, etaR, wL, wR;
  inner_t aL, aR;
  hlld_fill(q, p, Kl, Kr, Bc, &etaL, &etaR, &wL, &wR, &aL, &aR);
  const double delK = Kr[0] - Kl[0];
  const double Bch[3] = { Bc[0] * delK, Bc[1] * delK, Bc[2] * delK };
  const double Yl = (1 - dot1(Kl)) / (etaL * delK - dot3(Kl, Bch));
  const double Yr = (1 - dot1(Kr)) / (etaR * delK - dot3(Kr, Bch));
  if (fabs(delK) < 1e-10) *y = 0.0;
  else if (fabs(Bc[0]) < 1e-10) *y = delK;
  else *y = delK * (1 - Bc[0] * (Yr - Yl));
  return 0;
}

/* NewtonRaphesonSolver::Solve for rank 1 (Mara/nrsolver.cpp:89-152 with the numerical
 * Jacobian of Mara/riemann_hlld-rmhd.cpp:347-356 and GetErrorUpdateX, eqnbase.hpp:179-187) */
static int hlld_newton(const hlld_eqn *q, double *x)
{
  const int MaxIterations = 15;
  const double MinEpsilon = 1e-12;
  int worse = 0, it = 0;
  double eps = 0.0, eps_last;
  do {
    eps_last = eps;
    double y, f0, f1;
    if (hlld_function(q, *x, &y)) return 1;
    const double dp = 1e-8;
    const double p0 = *x - 0.5 * dp, p1 = *x + 0.5 * dp;
    if (hlld_function(q, p0, &f0)) return 1;
    if (hlld_function(q, p1, &f1)) return 1;
    const double J = (f1 - f0) / dp;
    const double G = 1.0 / J;
    double dx = 0.0;
    dx += G * y;
    *x -= dx;
    eps = 0;
    eps += y > 0 ? y : -y;
    worse += (eps > eps_last);
    if (worse >= 10 || it == MaxIterations) return 1;
    if (isnan(eps)) return 1;
  } while (eps > MinEpsilon && ++it <= MaxIterations);
  return 0;
}

static int hlld_reconstruct(const hlld_eqn *q, double p, double *F)   /* :453-575 */
{
  double Kl[3], Kr[3], Bc[3], etaL, etaR, wL, wR;
  inner_t aL, aR, cL, cR;
  hlld_fill(q, p, Kl, Kr, Bc, &etaL, &etaR, &wL, &wR, &aL, &aR);
  const double *Ul = q->Ul, *Ur = q->Ur, *Fl = q->Fl, *Fr = q->Fr;
  const double am = q->am, ap = q->ap;
  const double denomL = etaL - dot3(Kl, Bc);
  const double denomR = etaR - dot3(Kr, Bc);
  for (int k = 0; k < 3; ++k) {
    cL.v[k] = Kl[k] - Bc[k] * (1 - dot1(Kl)) / denomL;
    cR.v[k] = Kr[k] - Bc[k] * (1 - dot1(Kr)) / denomR;
    if (fabs(denomL) < 1e-10) cL.v[k] = aL.v[k];
    if (fabs(denomR) < 1e-10) cR.v[k] = aR.v[k];
  }
  const double lamC = cR.v[0], lmaL = Kl[0], lmaR = Kr[0], TOL = 1e-14;
  if (p < 0.0) return 1;
  if (lmaL < -1.0 || lmaR > 1.0 || fabs(lamC) > 1.0) return 1;
  if (!((wL > p) && (aL.v[0] > am - TOL) && (cL.v[0] > lmaL - TOL))) return 1;
  if (!((wR > p) && (aR.v[0] < ap + TOL) && (cR.v[0] < lmaR + TOL))) return 1;
  if (fabs(cR.v[0] - cL.v[0]) > 1e-8) return 1;
  double denom;
  int i;
  if (fabs(denom = am - aL.v[0]) < 1e-8) {
    for (i = 0; i < 8; ++i) aL.U[i] = Ul[i];
  } else {
    const double vB = dot3(aL.v, aL.B);
    aL.U[ddd] = q->L.D / denom;
    aL.U[tau] = (q->L.E + p * aL.v[0] - vB * aL.B[0]) / denom;
    aL.U[Sx] = (aL.U[tau] + p) * aL.v[0] - vB * aL.B[0];
    aL.U[Sy] = (aL.U[tau] + p) * aL.v[1] - vB * aL.B[1];
    aL.U[Sz] = (aL.U[tau] + p) * aL.v[2] - vB * aL.B[2];
    aL.U[Bx] = aL.B[0];
    aL.U[By] = aL.B[1];
    aL.U[Bz] = aL.B[2];
  }
  if (fabs(denom = ap - aR.v[0]) < 1e-8) {
    for (i = 0; i < 8; ++i) aR.U[i] = Ur[i];
  } else {
    const double vB = dot3(aR.v, aR.B);
    aR.U[ddd] = q->R.D / denom;
    aR.U[tau] = (q->R.E + p * aR.v[0] - vB * aR.B[0]) / denom;
    aR.U[Sx] = (aR.U[tau] + p) * aR.v[0] - vB * aR.B[0];
    aR.U[Sy] = (aR.U[tau] + p) * aR.v[1] - vB * aR.B[1];
    aR.U[Sz] = (aR.U[tau] + p) * aR.v[2] - vB * aR.B[2];
    aR.U[Bx] = aR.B[0];
    aR.U[By] = aR.B[1];
    aR.U[Bz] = aR.B[2];
  }
  if (fabs(denom = lmaL - lamC) < 1e-8) {
    for (i = 0; i < 8; ++i) cL.U[i] = aL.U[i];
  } else {
    const double vBc = dot3(cL.v, Bc);
    cL.U[ddd] = aL.U[ddd] * (lmaL - aL.v[0]) / denom;
    cL.U[tau] = (lmaL * aL.U[tau] - aL.U[Sx] + p * lamC - vBc * Bc[0]) / denom;
    cL.U[Sx] = (cL.U[tau] + p) * cL.v[0] - vBc * Bc[0];
    cL.U[Sy] = (cL.U[tau] + p) * cL.v[1] - vBc * Bc[1];
    cL.U[Sz] = (cL.U[tau] + p) * cL.v[2] - vBc * Bc[2];
    cL.U[Bx] = Bc[0];
    cL.U[By] = Bc[1];
    cL.U[Bz] = Bc[2];
  }
  if (fabs(denom = lmaR - lamC) < 1e-8) {
    for (i = 0; i < 8; ++i) cR.U[i] = aR.U[i];
  } else {
    const double vBc = dot3(cR.v, Bc);
    cR.U[ddd] = aR.U[ddd] * (lmaR - aR.v[0]) / denom;
    cR.U[tau] = (lmaR * aR.U[tau] - aR.U[Sx] + p * lamC - vBc * Bc[0]) / denom;
    cR.U[Sx] = (cR.U[tau] + p) * cR.v[0] - vBc * Bc[0];
    cR.U[Sy] = (cR.U[tau] + p) * cR.v[1] - vBc * Bc[1];
    cR.U[Sz] = (cR.U[tau] + p) * cR.v[2] - vBc * Bc[2];
    cR.U[Bx] = Bc[0];
    cR.U[By] = Bc[1];
    cR.U[Bz] = Bc[2];
  }
  const double s = 0.0;
  if (s <= am) for (i = 0; i < 8; ++i) F[i] = Fl[i];
  else if (am < s && s <= lmaL) for (i = 0; i < 8; ++i) F[i] = Fl[i] + am * (aL.U[i] - Ul[i]);
  else if (lmaL < s && s <= lamC)
    for (i = 0; i < 8; ++i) F[i] = Fl[i] + am * (aL.U[i] - Ul[i]) + lmaL * (cL.U[i] - aL.U[i]);
  else if (lamC < s && s <= lmaR)
    for (i = 0; i < 8; ++i) F[i] = Fr[i] + ap * (aR.U[i] - Ur[i]) + lmaR * (cR.U[i] - aR.U[i]);
  else if (lmaR < s && s <= ap) for (i = 0; i < 8; ++i) F[i] = Fr[i] + ap * (aR.U[i] - Ur[i]);
  else if (ap < s) for (i = 0; i < 8; ++i) F[i] = Fr[i];
  F[tau] -= F[ddd];
  return 0;
}

static double hlld_estimate(hlld_eqn *q, int attempt)                  /* :576-615 */
{
  if (attempt == 0) {
    const double *P = q->P_hll;
    const double V2 = P[vx] * P[vx] + P[vy] * P[vy] + P[vz] * P[vz];
    const double B2 = P[Bx] * P[Bx] + P[By] * P[By] + P[Bz] * P[Bz];
    const double Bv = P[Bx] * P[vx] + P[By] * P[vy] + P[Bz] * P[vz];
    const double W2 = 1.0 / (1.0 - V2);
    const double W = sqrt(W2);
    const double b0 = W * Bv;
    const double b2 = (B2 + b0 * b0) / W2;
    return P[pre] + 0.5 * b2;
  } else if (attempt == 1) {
    double *Fh = q->F_hll, *Uh = q->U_hll;
    Fh[tau] += Fh[ddd];
    Uh[tau] += Uh[ddd];
    const double a = 1.0;
    const double b = Uh[tau] - Fh[Sx];
    const double cc = Fh[tau] * Uh[Sx] - Uh[tau] * Fh[Sx];
    const double p1 = fabs((-b + sqrt(b * b - 4 * a * cc)) / (2 * a));
    const double p2 = fabs((-b - sqrt(b * b - 4 * a * cc)) / (2 * a));
    Fh[tau] -= Fh[ddd];
    Uh[tau] -= Uh[ddd];
    return (p1 < p2) ? p1 : p2;
  }
  return 0.0;
}

/* HlldRmhdRiemannSolver::IntercellFlux (Mara/riemann_hlld-rmhd.cpp:179-313), at s = 0 */
static int riemann_hlld(const port_config *c, port_stats *st, const double *pl,
                        const double *pr, double *f, int dim)
{
  int B1, B2, B3, S1, S2, S3, v1, v2, v3;
  dim_map(dim, &B1, &B2, &B3, &S1, &S2, &S3, &v1, &v2, &v3);
  double Pl[8], Pr[8], Ul[8], Ur[8], Fl[8], Fr[8], epl, eml, epr, emr;
  Pl[pre] = pl[pre]; Pr[pre] = pr[pre];
  Pl[rho] = pl[rho]; Pr[rho] = pr[rho];
  Pl[vx] = pl[v1];   Pr[vx] = pr[v1];
  Pl[vy] = pl[v2];   Pr[vy] = pr[v2];
  Pl[vz] = pl[v3];   Pr[vz] = pr[v3];
  Pl[Bx] = pl[B1];   Pr[Bx] = pr[B1];
  Pl[By] = pl[B2];   Pr[By] = pr[B2];
  Pl[Bz] = pl[B3];   Pr[Bz] = pr[B3];
  Pl[Bx] = Pr[Bx] = 0.5 * (pl[B1] + pr[B1]);
  if (port_prim_to_cons(c, Pl, Ul)) return 1;
  if (port_prim_to_cons(c, Pr, Ur)) return 1;
  port_flux_and_eigenvalues(c, Ul, Pl, Fl, &epl, &eml, 1);
  port_flux_and_eigenvalues(c, Ur, Pr, Fr, &epr, &emr, 1);
  const double am = (eml < emr) ? eml : emr;
  const double ap = (epl > epr) ? epl : epr;
  note_lambda(st, ap, am);
  double P_hll[8], U_hll[8], F_hll[8];
  for (int i = 0; i < 8; ++i) P_hll[i] = 0.5 * (Pl[i] + Pr[i]);
  hll_state(ap, am, Ul, Ur, Fl, Fr, U_hll, F_hll);
  const int hll_c2p_failed = port_cons_to_prim(c, U_hll, P_hll);
  hlld_eqn q = { Pl, Pr, Ul, Ur, Fl, Fr, ap, am, {0}, {0}, P_hll, U_hll, F_hll };
  hlld_init(&q);
  double F[8];
  int attempt = 0, success = 0;
  while (!hll_c2p_failed && attempt < 3 && !success) {
    double p_star;
    int rc;
    if (fabs(Pl[Bx]) < 1e-8 || fabs(Pr[Bx]) < 1e-8) {
      p_star = hlld_estimate(&q, 1);
      rc = hlld_reconstruct(&q, p_star, F);
    } else {
      p_star = hlld_estimate(&q, attempt);
      rc = hlld_newton(&q, &p_star);
      if (rc == 0) rc = hlld_reconstruct(&q, p_star, F);
    }
    success = (rc == 0);
    ++attempt;
  }
  st->hlld_path = hll_c2p_failed ? 0 : success ? attempt : 4;
  if (success) {
    st->hlld_success++;
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
  st->hlld_failure++;
  return riemann_hllc(c, st, pl, pr, f, dim);
}

int port_riemann(const port_config *c, port_stats *s, const double *pl, const double *pr,
                 double *F, int dim)
{
  switch (c->riemann) {
  case 0: return riemann_hll(c, s, pl, pr, F, dim);
  case 1: return riemann_hllc(c, s, pl, pr, F, dim);
  default: return riemann_hlld(c, s, pl, pr, F, dim);
  }
}

/* ---- constrained transport (Mara/rmhd.cpp:311-381) ------------------------------------ */
void port_ct2d(double *Fx, double *Fy, const int *stride)
{
  const long N = stride[0] / 8;
  double *FxBy = calloc(N, sizeof(double)), *FyBx = calloc(N, sizeof(double));
  const int sx = stride[1], sy = stride[2];
  for (long i = sx; i < stride[0] - sx; i += 8) {
    const double *F = &Fx[By + i], *G = &Fy[Bx + i];
    FxBy[i / 8] = (2 * F[0] + F[sy] + F[-sy] - G[0] - G[sx] - G[-sy] - G[sx - sy]) * 0.125;
    FyBx[i / 8] = (2 * G[0] + G[sx] + G[-sx] - F[0] - F[sy] - F[-sx] - F[-sx + sy]) * 0.125;
  }
  for (long i = 0; i < stride[0]; i += 8) {
    Fx[i + Bx] = 0.0;          Fx[i + By] = FxBy[i / 8];
    Fy[i + Bx] = FyBx[i / 8];  Fy[i + By] = 0.0;
  }
  free(FxBy);
  free(FyBx);
}

void port_ct3d(double *Fx, double *Fy, double *Fz, const int *stride)
{
  const long N = stride[0] / 8;
  double *FxBy = calloc(N, sizeof(double)), *FxBz = calloc(N, sizeof(double));
  double *FyBz = calloc(N, sizeof(double)), *FyBx = calloc(N, sizeof(double));
  double *FzBx = calloc(N, sizeof(double)), *FzBy = calloc(N, sizeof(double));
  const int sx = stride[1], sy = stride[2], sz = stride[3];
  for (long i = sx; i < stride[0] - sx; i += 8) {
    const double *F, *G, *H;
    F = &Fx[By + i];
    G = &Fy[Bx + i];
    FxBy[i / 8] = (2 * F[0] + F[sy] + F[-sy] - G[0] - G[sx] - G[-sy] - G[sx - sy]) * 0.125;
    FyBx[i / 8] = (2 * G[0] + G[sx] + G[-sx] - F[0] - F[sy] - F[-sx] - F[-sx + sy]) * 0.125;
    G = &Fy[Bz + i];
    H = &Fz[By + i];
    FyBz[i / 8] = (2 * G[0] + G[sz] + G[-sz] - H[0] - H[sy] - H[-sz] - H[sy - sz]) * 0.125;
    FzBy[i / 8] = (2 * H[0] + H[sy] + H[-sy] - G[0] - G[sz] - G[-sy] - G[-sy + sz]) * 0.125;
    H = &Fz[Bx + i];
    F = &Fx[Bz + i];
    FzBx[i / 8] = (2 * H[0] + H[sx] + H[-sx] - F[0] - F[sz] - F[-sx] - F[sz - sx]) * 0.125;
    FxBz[i / 8] = (2 * F[0] + F[sz] + F[-sz] - H[0] - H[sx] - H[-sz] - H[-sz + sx]) * 0.125;
  }
  for (long i = 0; i < stride[0]; i += 8) {
    Fx[i + Bx] = 0.0;         Fx[i + By] = FxBy[i / 8]; Fx[i + Bz] = FxBz[i / 8];
    Fy[i + Bx] = FyBx[i / 8]; Fy[i + By] = 0.0;         Fy[i + Bz] = FyBz[i / 8];
    Fz[i + Bx] = FzBx[i / 8]; Fz[i + By] = FzBy[i / 8]; Fz[i + Bz] = 0.0;
  }
  free(FxBy); free(FyBz); free(FzBx);
  free(FxBz); free(FyBx); free(FzBy);
}

/* ---- grid operations ------------------------------------------------------------------ */
typedef struct {
  int G[3];
  long nz;           /* zones incl. guard */
  int stride[4];     /* in doubles, as GodunovOperator::prepare_integration */
  double dx, dy, dz;
} grid_t;

static void grid_init(const port_config *c, grid_t *g)               /* hydro.cpp:80-110 */
{
  shape(c, g->G);
  g->nz = (long) g->G[0] * g->G[1] * g->G[2];
  g->stride[0] = g->G[0] * g->G[1] * g->G[2] * 8;
  g->stride[1] = g->G[1] * g->G[2] * 8;
  g->stride[2] = g->G[2] * 8;
  g->stride[3] = 8;
  double dd[3];
  for (int d = 0; d < 3; ++d) {
    const double x0 = (d < c->nd) ? c->x0[d] : 0.0;
    const double x1 = (d < c->nd) ? c->x1[d] : 1.0;
    const int Gd = (d < c->nd) ? g->G[d] : 1;
    dd[d] = (x1 - x0) / (Gd - 2 * c->ng);
  }
  g->dx = dd[0]; g->dy = dd[1]; g->dz = dd[2];
}

/* SimpleCartesianDomain::Synchronize, periodic (Mara/simple-cart.cpp:81-174) */
static void sync_periodic(const port_config *c, const grid_t *g, double *A)
{
  const int ng = c->ng, Nx = c->n[0], Ny = c->n[1], Nz = c->n[2];
  const int Gx = g->G[0], Gy = g->G[1], Gz = g->G[2];
#define AT(i, j, k) (&A[(((long) (i) * Gy + (j)) * Gz + (k)) * 8])
#define CP(i, j, k, a, b, cc) memcpy(AT(i, j, k), AT(a, b, cc), 8 * sizeof(double))
  if (c->nd >= 1) {
    for (int i = 0; i < ng; ++i)
      for (int j = 0; j < Gy; ++j) for (int k = 0; k < Gz; ++k) CP(i, j, k, i + Nx, j, k);
    for (int i = Nx + ng; i < Nx + 2 * ng; ++i)
      for (int j = 0; j < Gy; ++j) for (int k = 0; k < Gz; ++k) CP(i, j, k, i - Nx, j, k);
  }
  if (c->nd >= 2) {
    for (int i = 0; i < Gx; ++i) {
      for (int j = 0; j < ng; ++j) for (int k = 0; k < Gz; ++k) CP(i, j, k, i, j + Ny, k);
      for (int j = Ny + ng; j < Ny + 2 * ng; ++j)
        for (int k = 0; k < Gz; ++k) CP(i, j, k, i, j - Ny, k);
    }
  }
  if (c->nd >= 3) {
    for (int i = 0; i < Gx; ++i)
      for (int j = 0; j < Gy; ++j) {
        for (int k = 0; k < ng; ++k) CP(i, j, k, i, j, k + Nz);
        for (int k = Nz + ng; k < Nz + 2 * ng; ++k) CP(i, j, k, i, j, k - Nz);
      }
  }
#undef CP
#undef AT
}

/* GodunovOperator::ConsToPrim (Mara/hydro.cpp:125-202), with the emergency reset.
 * U is ghost-filled in place; P holds the previous prims (guess) and is overwritten. */
static int c2p_all_mask(const port_config *c, const grid_t *g, double *U, double *P, int *mask_out);

static int c2p_all(const port_config *c, const grid_t *g, double *U, double *P)
{
  return c2p_all_mask(c, g, U, P, NULL);
}

/* ... and GodunovOperator's FailureMask afterwards (zeroed by an emergency reset) in mask_out
 * when it is not NULL. */
static int c2p_all_mask(const port_config *c, const grid_t *g, double *U, double *P, int *mask_out)
{
  sync_periodic(c, g, U);
  int ttl = 0;
  char *mask = calloc(g->nz, 1);
  for (long z = 0; z < g->nz; ++z) {
    const int e = port_cons_to_prim(c, &U[z * 8], &P[z * 8]) != 0;
    mask[z] = (char) e;
    ttl += e;
  }
  if (ttl && c->ereset) {
    for (long z = 0; z < g->nz; ++z) {
      if (!mask[z]) continue;
      double *Pz = &P[z * 8];
      Pz[0] = c->dreset;
      Pz[1] = c->preset;
      Pz[2] = Pz[3] = Pz[4] = 0.0;
      Pz[5] = U[z * 8 + 5];
      Pz[6] = U[z * 8 + 6];
      Pz[7] = U[z * 8 + 7];
    }
    for (long z = 0; z < g->nz; ++z) port_prim_to_cons(c, &P[z * 8], &U[z * 8]);
    ttl = 0;
    memset(mask, 0, g->nz);
  }
  if (mask_out)
    for (long z = 0; z < g->nz; ++z) mask_out[z] = mask[z];
  free(mask);
  return ttl;
}

/* MethodOfLinesSplit::intercell_flux_sweep (Mara/plm-split.cpp:43-73) */
static void flux_sweep(const port_config *c, port_stats *st, const grid_t *g,
                       const double *P, double *F, int dim)
{
  const int S = g->stride[dim];
  double Pl[8], Pr[8];
  for (long i = 2 * S; i < g->stride[0] - 3 * S; i += 8) {
    for (int q = 0; q < 8; ++q) {
      const long m = i + q;
      const double v[6] = { P[m - 2 * S], P[m - S], P[m], P[m + S], P[m + 2 * S], P[m + 3 * S] };
      switch (c->recon) {
      case 0: Pl[q] = v[2]; Pr[q] = v[3]; break;
      case 1: Pl[q] = port_reconstruct(c, &v[2], 1); Pr[q] = port_reconstruct(c, &v[3], 0); break;
      default: Pl[q] = port_reconstruct(c, &v[2], 4); Pr[q] = port_reconstruct(c, &v[3], 5); break;
      }
    }
    if (port_riemann(c, st, Pl, Pr, &F[i], dim))
      port_riemann(c, st, &P[i], &P[i + S], &F[i], dim);
  }
}

/* MethodOfLinesSplit::dUdt + drive_sweeps_{1,2,3}d (Mara/plm-split.cpp:11-122).
 * Returns the c2p failure count (non-zero aborts the step); L is the time derivative. */
static int dUdt_split(const port_config *c, port_stats *st, const grid_t *g, const double *Uin,
                      double *PA, double *L)
{
  const long n = g->nz * 8;
  double *U = malloc(n * sizeof(double));
  memcpy(U, Uin, n * sizeof(double));
  const int err = c2p_all(c, g, U, PA);
  free(U);
  if (err) return err;
  double *F = calloc(n, sizeof(double)), *G = calloc(n, sizeof(double));
  double *H = calloc(n, sizeof(double));
  const int sx = g->stride[1], sy = g->stride[2], sz = g->stride[3];
  memset(L, 0, n * sizeof(double));
  if (c->nd == 1) {
    flux_sweep(c, st, g, PA, F, 1);
    for (long i = sx; i < g->stride[0]; ++i) L[i] = -(F[i] - F[i - sx]) / g->dx;
  } else if (c->nd == 2) {
    flux_sweep(c, st, g, PA, F, 1);
    flux_sweep(c, st, g, PA, G, 2);
    port_ct2d(F, G, g->stride);
    for (long i = sx; i < g->stride[0]; ++i)
      L[i] = -(F[i] - F[i - sx]) / g->dx - (G[i] - G[i - sy]) / g->dy;
  } else {
    flux_sweep(c, st, g, PA, F, 1);
    flux_sweep(c, st, g, PA, G, 2);
    flux_sweep(c, st, g, PA, H, 3);
    port_ct3d(F, G, H, g->stride);
    for (long i = sx; i < g->stride[0]; ++i)
      L[i] = -(F[i] - F[i - sx]) / g->dx - (G[i] - G[i - sy]) / g->dy - (H[i] - H[i - sz]) / g->dz;
  }
  free(F); free(G); free(H);
  return 0;
}

/* ---- PlmCtuHancockOperator (Mara/ctu-hancock.cpp:53-494), default safety level ---------- */
/* its own minmod, with the static plm_theta that config_solver{theta} sets (:27-35) */
static double ctu_minmod(double theta, double ul, double u0, double ur)
{
  const double a = theta * (u0 - ul);
  const double b = 0.5 * (ur - ul);
  const double cc = theta * (ur - u0);
  const double sa = SGN(a), sb = SGN(b), sc = SGN(cc);
  const double fa = fabs(a), fb = fabs(b), fc = fabs(cc);
  const double ab = (fa < fb) ? fa : fb;
  const double m = (ab < fc) ? ab : fc;
  return 0.25 * fabs(sa + sb) * (sa + sc) * m;
}

/* dUdt of the CTU-Hancock operator: c2p of U into PA, slopes, first (transverse) fluxes,
 * per-direction Hancock predictors with their c2p, final fluxes from the predicted states,
 * CT and the divergence.  Returns the failure count of the first check that fails (each
 * aborts the step, :215, :334, :375, :494); L is the time derivative. */
static int dUdt_ctu(const port_config *c, port_stats *st, const grid_t *g, const double *Uin,
                    double *PA, double *L, double dt)
{
  const long n = g->nz * 8;
  const int nd = c->nd;
  const long S0 = g->stride[0];
  const long sx = g->stride[1], sy = g->stride[2], sz = g->stride[3];
  const long Sd[3] = {sx, sy, sz};
  double *U = malloc(n * sizeof(double));
  memcpy(U, Uin, n * sizeof(double));
  /* the c2p count is not checked here (:61-66): failed zones keep what the inversion left in
   * PA, and ctu_hancock clears FailureMask before its own checks (:102) */
  c2p_all(c, g, U, PA);
  int fail = 0;
  const double *P = PA;
  double *Fd[3] = {NULL, NULL, NULL}, *dP[3] = {NULL, NULL, NULL}, *Ud[3] = {NULL, NULL, NULL};
  double *Pd[3] = {NULL, NULL, NULL};
  for (int d = 0; d < nd; ++d) {
    Fd[d] = calloc(n, sizeof(double));
    dP[d] = calloc(n, sizeof(double));
    Ud[d] = calloc(n, sizeof(double));
    Pd[d] = calloc(n, sizeof(double));
  }
  double Pl[8], Pr[8];
  /* step 1: slopes */
  for (long i = sx; i < S0 - sx; ++i)
    for (int d = 0; d < nd; ++d) dP[d][i] = ctu_minmod(c->theta, P[i - Sd[d]], P[i], P[i + Sd[d]]);
  /* step 2: fluxes of the reconstructed zone-centre states, every direction */
  for (long i = 0; i < S0 - sx; i += 8)
    for (int d = 0; d < nd; ++d) {
      for (int j = 0; j < 8; ++j) {
        Pr[j] = P[i + Sd[d] + j] - 0.5 * dP[d][i + Sd[d] + j];
        Pl[j] = P[i + j] + 0.5 * dP[d][i + j];
      }
      if (check_prim(Pl) || check_prim(Pr)) fail += 1;
      else port_riemann(c, st, Pl, Pr, &Fd[d][i], d + 1);
    }
  if (fail) goto done;
  /* step 3: Hancock predictors, normal flux difference of the zone's own face states plus the
   * transverse Godunov fluxes, half a step */
  for (long i = sx; i < S0; i += 8) {
    double FL[3][8], FR[3][8], UL[8], UR[8], PL[8], PR[8];
    for (int d = 0; d < nd; ++d) {
      for (int j = 0; j < 8; ++j) {
        PL[j] = P[i + j] - 0.5 * dP[d][i + j];
        PR[j] = P[i + j] + 0.5 * dP[d][i + j];
      }
      if (check_prim(PL) || check_prim(PR)) {
        fail += 1;
        memset(FL[d], 0, sizeof(FL[d]));
        memset(FR[d], 0, sizeof(FR[d]));
      } else {
        port_prim_to_cons(c, PL, UL);
        port_prim_to_cons(c, PR, UR);
        port_flux_and_eigenvalues(c, UL, PL, FL[d], NULL, NULL, d + 1);   /* no speeds (:262) */
        port_flux_and_eigenvalues(c, UR, PR, FR[d], NULL, NULL, d + 1);
      }
    }
    for (int j = 0; j < 8; ++j) {
      const long m = i + j;
      if (nd == 1) {
        Ud[0][m] = U[m] - ((FR[0][j] - FL[0][j]) / g->dx) * 0.5 * dt;
      } else if (nd == 2) {
        Ud[0][m] = U[m] - ((FR[0][j] - FL[0][j]) / g->dx + (Fd[1][m] - Fd[1][m - sy]) / g->dy) * 0.5 * dt;
        Ud[1][m] = U[m] - ((FR[1][j] - FL[1][j]) / g->dy + (Fd[0][m] - Fd[0][m - sx]) / g->dx) * 0.5 * dt;
      } else {
        Ud[0][m] = U[m] - ((FR[0][j] - FL[0][j]) / g->dx + (Fd[1][m] - Fd[1][m - sy]) / g->dy +
                           (Fd[2][m] - Fd[2][m - sz]) / g->dz) * 0.5 * dt;
        Ud[1][m] = U[m] - ((FR[1][j] - FL[1][j]) / g->dy + (Fd[2][m] - Fd[2][m - sz]) / g->dz +
                           (Fd[0][m] - Fd[0][m - sx]) / g->dx) * 0.5 * dt;
        Ud[2][m] = U[m] - ((FR[2][j] - FL[2][j]) / g->dz + (Fd[0][m] - Fd[0][m - sx]) / g->dx +
                           (Fd[1][m] - Fd[1][m - sy]) / g->dy) * 0.5 * dt;
      }
    }
  }
  if (fail) goto done;
  /* predicted primitives: guards from the periodic fill, c2p from the zone's primitives */
  for (int d = 0; d < nd; ++d) sync_periodic(c, g, Ud[d]);
  for (long i = 0; i < S0; i += 8)
    for (int d = 0; d < nd; ++d) {
      memcpy(&Pd[d][i], &P[i], 8 * sizeof(double));
      if (port_cons_to_prim(c, &Ud[d][i], &Pd[d][i])) fail += 1;
    }
  if (fail) goto done;
  /* step 4: fluxes of the predicted states (a face keeps its step-2 flux where the solver
   * fails) */
  for (long i = sx; i < S0 - sx; i += 8)
    for (int d = 0; d < nd; ++d) {
      for (int j = 0; j < 8; ++j) {
        Pr[j] = Pd[d][i + Sd[d] + j] - 0.5 * dP[d][i + Sd[d] + j];
        Pl[j] = Pd[d][i + j] + 0.5 * dP[d][i + j];
      }
      if (check_prim(Pl) || check_prim(Pr)) fail += 1;
      else port_riemann(c, st, Pl, Pr, &Fd[d][i], d + 1);
    }
  memset(L, 0, n * sizeof(double));
  if (nd == 1) {
    for (long i = sx; i < S0; ++i) L[i] = -((Fd[0][i] - Fd[0][i - sx]) / g->dx);
  } else if (nd == 2) {
    port_ct2d(Fd[0], Fd[1], g->stride);
    for (long i = sx; i < S0; ++i) L[i] = -((Fd[0][i] - Fd[0][i - sx]) / g->dx + (Fd[1][i] - Fd[1][i - sy]) / g->dy);
  } else {
    port_ct3d(Fd[0], Fd[1], Fd[2], g->stride);
    for (long i = sx; i < S0; ++i)
      L[i] = -((Fd[0][i] - Fd[0][i - sx]) / g->dx + (Fd[1][i] - Fd[1][i - sy]) / g->dy +
               (Fd[2][i] - Fd[2][i - sz]) / g->dz);
  }
done:
  for (int d = 0; d < nd; ++d) { free(Fd[d]); free(dP[d]); free(Ud[d]); free(Pd[d]); }
  free(U);
  return fail;
}

/* GodunovOperator::dUdt of the selected operator (set_godunov, Mara/mara.cpp:960-994) */
static int dUdt(const port_config *c, port_stats *st, const grid_t *g, const double *Uin, double *PA,
                double *L, double dt)
{
  return c->godunov ? dUdt_ctu(c, st, g, Uin, PA, L, dt) : dUdt_split(c, st, g, Uin, PA, L);
}

/* luaC_Mara_advance (Mara/mara.cpp:297-341) with the Runge-Kutta integrators of
 * Mara/runge-kutta.hpp:129-177.  prim is updated only when no zone fails. */
int port_advance(const port_config *c, port_stats *st, double *prim, double dt, int *errors)
{
  grid_t g;
  grid_init(c, &g);
  const long n = g.nz * 8;
  double *P = malloc(n * sizeof(double)), *U = malloc(n * sizeof(double));
  double *U1 = malloc(n * sizeof(double)), *L = malloc(n * sizeof(double));
  double *PA = calloc(n, sizeof(double));     /* PrimitiveArray, zero-filled by resize */
  memcpy(P, prim, n * sizeof(double));
  st->max_lambda = 0.0;
  sync_periodic(c, &g, P);
  for (long z = 0; z < g.nz; ++z) port_prim_to_cons(c, &P[z * 8], &U[z * 8]);

  int err = 0;
  long i;
  switch (c->rk) {
  case 1:
    if ((err = dUdt(c, st, &g, U, PA, L, dt))) break;
    for (i = 0; i < n; ++i) U[i] += dt * L[i];
    break;
  case 2:
    if ((err = dUdt(c, st, &g, U, PA, L, dt))) break;
    for (i = 0; i < n; ++i) U1[i] = U[i] + dt * L[i];
    if ((err = dUdt(c, st, &g, U1, PA, L, dt))) break;
    for (i = 0; i < n; ++i) U[i] = 0.5 * (U[i] + U1[i] + dt * L[i]);
    break;
  case 3:
    if ((err = dUdt(c, st, &g, U, PA, L, dt))) break;
    for (i = 0; i < n; ++i) U1[i] = U[i] + dt * L[i];
    if ((err = dUdt(c, st, &g, U1, PA, L, dt))) break;
    for (i = 0; i < n; ++i) U1[i] = 3. / 4 * U[i] + 1. / 4 * U1[i] + 1. / 4 * dt * L[i];
    if ((err = dUdt(c, st, &g, U1, PA, L, dt))) break;
    for (i = 0; i < n; ++i) U[i] = 1. / 3 * U[i] + 2. / 3 * U1[i] + 2. / 3 * dt * L[i];
    break;
  default: {
    double *L1 = malloc(n * sizeof(double)), *L2 = malloc(n * sizeof(double));
    double *L3 = malloc(n * sizeof(double));
    if (!(err = dUdt(c, st, &g, U, PA, L, dt))) {
      for (i = 0; i < n; ++i) { L1[i] = dt * L[i]; U1[i] = U[i] + 0.5 * L1[i]; }
      if (!(err = dUdt(c, st, &g, U1, PA, L, dt))) {
        for (i = 0; i < n; ++i) { L2[i] = dt * L[i]; U1[i] = U[i] + 0.5 * L2[i]; }
        if (!(err = dUdt(c, st, &g, U1, PA, L, dt))) {
          for (i = 0; i < n; ++i) { L3[i] = dt * L[i]; U1[i] = U[i] + 1.0 * L3[i]; }
          if (!(err = dUdt(c, st, &g, U1, PA, L, dt))) {
            for (i = 0; i < n; ++i)
              U[i] += (1.0 / 6.0) * (L1[i] + 2.0 * L2[i] + 2.0 * L3[i] + dt * L[i]);
          }
        }
      }
    }
    free(L1); free(L2); free(L3);
  } break;
  }
  if (!err) {
    memcpy(P, PA, n * sizeof(double));
    err = c2p_all(c, &g, U, P);
    if (!err) memcpy(prim, P, n * sizeof(double));
  }
  *errors = err;
  free(P); free(U); free(U1); free(L); free(PA);
  return 0;
}

/* luaC_Mara_get_timestep (Mara/mara.cpp:374-381) with SimpleCartesianDomain::min_dx
 * (Mara/simple-cart.cpp:20-24) */
double port_timestep(const port_config *c, double max_lambda, double cfl)
{
  double min_dx = c->x1[0] - c->x0[0];
  for (int d = 0; d < c->nd; ++d) {
    const double dx = (c->x1[d] - c->x0[d]) / c->n[d];
    if (dx < min_dx) min_dx = dx;
  }
  return cfl * min_dx / max_lambda;
}

/* luaC_mean_max_divB (Mara/mara.cpp:2264-2324) */
void port_mean_max_divB(const port_config *c, const double *P, double *mean, double *max)
{
  int G[3];
  shape(c, G);
  const long nz = (long) G[0] * G[1] * G[2];
  double *div = calloc(nz, sizeof(double));
  const int ng = c->ng;
#define B(q, i, j, k) P[(((long) (i) * G[1] + (j)) * G[2] + (k)) * 8 + (q)]
  if (c->nd == 2) {
    for (int i = ng; i < G[0] - ng - 1; ++i)
      for (int j = ng; j < G[1] - ng - 1; ++j)
        div[(long) i * G[1] + j] =
            (B(5, i + 1, j, 0) + B(5, i + 1, j + 1, 0) - B(5, i, j, 0) - B(5, i, j + 1, 0)) / 2.0 +
            (B(6, i, j + 1, 0) + B(6, i + 1, j + 1, 0) - B(6, i, j, 0) - B(6, i + 1, j, 0)) / 2.0;
  } else if (c->nd == 3) {
    for (int i = ng; i < G[0] - ng - 1; ++i)
      for (int j = ng; j < G[1] - ng - 1; ++j)
        for (int k = ng; k < G[2] - ng - 1; ++k)
          div[((long) i * G[1] + j) * G[2] + k] =
              ((B(5, i + 1, j, k) + B(5, i + 1, j + 1, k) + B(5, i + 1, j, k + 1) + B(5, i + 1, j + 1, k + 1)) -
               (B(5, i, j, k) + B(5, i, j + 1, k) + B(5, i, j, k + 1) + B(5, i, j + 1, k + 1))) / 4.0 +
              ((B(6, i, j + 1, k) + B(6, i, j + 1, k + 1) + B(6, i + 1, j + 1, k) + B(6, i + 1, j + 1, k + 1)) -
               (B(6, i, j, k) + B(6, i, j, k + 1) + B(6, i + 1, j, k) + B(6, i + 1, j, k + 1))) / 4.0 +
              ((B(7, i, j, k + 1) + B(7, i + 1, j, k + 1) + B(7, i, j + 1, k + 1) + B(7, i + 1, j + 1, k + 1)) -
               (B(7, i, j, k) + B(7, i + 1, j, k) + B(7, i, j + 1, k) + B(7, i + 1, j + 1, k))) / 4.0;
  }
#undef B
  double sum = 0.0, mx = div[0];
  for (long z = 0; z < nz; ++z) {
    sum += div[z];
    if (div[z] > mx) mx = div[z];
  }
  long glb = 1;
  for (int d = 0; d < c->nd; ++d) glb *= c->n[d];
  *mean = (sum / nz) / glb;
  *max = mx;
  free(div);
}

/* luaC_max_lorentz_factor (Mara/mara.cpp:2232-2260), interior zones only */
double port_max_lorentz_factor(const port_config *c, const double *P)
{
  int G[3];
  shape(c, G);
  double mx = 0.0;
  for (int i = 0; i < G[0]; ++i)
    for (int j = 0; j < G[1]; ++j)
      for (int k = 0; k < G[2]; ++k) {
        if (i < c->ng || i >= G[0] - c->ng) continue;
        if (c->nd >= 2 && (j < c->ng || j >= G[1] - c->ng)) continue;
        if (c->nd >= 3 && (k < c->ng || k >= G[2] - c->ng)) continue;
        const double *p = &P[(((long) i * G[1] + j) * G[2] + k) * 8];
        const double v2 = p[2] * p[2] + p[3] * p[3] + p[4] * p[4];
        const double W0 = 1.0 / sqrt(1.0 - v2);
        if (W0 > mx) mx = W0;
      }
  return mx;
}


#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* luaC_Mara_diffuse (Mara/mara.cpp:343-366) with GodunovOperator::LaxDiffusion
 * (Mara/hydro.cpp:205-283): prim <- c2p(P->U(prim) + L), L the CT'd divergence of the
 * Lax fluxes -c r (U[i+s] - U[i]) dx_d on faces with a failed zone (mask_in, one entry per
 * guarded zone) on either side.  prev = the PrimitiveArray the c2p starts from and keeps in
 * failed zones; mask_out = the FailureMask after (may alias mask_in).  Returns the c2p's
 * failure count, which the reference discards. */
int port_diffuse(const port_config *c, double *prim, double r, const int *mask_in, const double *prev,
                 int *mask_out)
{
  grid_t g;
  grid_init(c, &g);
  const long n = g.nz * 8;
  const int nd = c->nd, NQ = 8;
  double *P = malloc(n * sizeof(double)), *U = malloc(n * sizeof(double));
  double *L = calloc(n, sizeof(double));
  double *Fiph = calloc(n, sizeof(double)), *Giph = calloc(n, sizeof(double));
  double *Hiph = calloc(n, sizeof(double));
  int *FM = malloc(g.nz * sizeof(int));
  for (long z = 0; z < g.nz; ++z) FM[z] = mask_in[z];
  memcpy(P, prim, n * sizeof(double));
  sync_periodic(c, &g, P);                                  /* GodunovOperator::PrimToCons */
  for (long z = 0; z < g.nz; ++z) port_prim_to_cons(c, &P[z * 8], &U[z * 8]);
  sync_periodic(c, &g, U);                                  /* LaxDiffusion: ApplyBoundaries(U) */
  const int Ni = g.stride[0], sx = g.stride[1], sy = g.stride[2], sz = g.stride[3];
  if (nd == 1) {
    for (int i = 0; i < Ni - sx; i += NQ)
      if (FM[i / NQ] || FM[(i + sx) / NQ])
        for (int j = 0; j < NQ; ++j) Fiph[i + j] = -0.5 * r * (U[i + j + sx] - U[i + j]) * g.dx;
    for (int i = sx; i < Ni - sx; ++i) L[i] = -((Fiph[i] - Fiph[i - sx]) / g.dx);
  } else if (nd == 2) {
    for (int i = 0; i < Ni - sx; i += NQ) {
      if (FM[i / NQ] || FM[(i + sx) / NQ])
        for (int j = 0; j < NQ; ++j) Fiph[i + j] = -0.25 * r * (U[i + j + sx] - U[i + j]) * g.dx;
      if (FM[i / NQ] || FM[(i + sy) / NQ])
        for (int j = 0; j < NQ; ++j) Giph[i + j] = -0.25 * r * (U[i + j + sy] - U[i + j]) * g.dy;
    }
    port_ct2d(Fiph, Giph, g.stride);
    for (int i = sx; i < Ni - sx; ++i)
      L[i] = -((Fiph[i] - Fiph[i - sx]) / g.dx + (Giph[i] - Giph[i - sy]) / g.dy);
  } else {
    for (int i = 0; i < Ni - sx; i += NQ) {
      if (FM[i / NQ] || FM[(i + sx) / NQ])
        for (int j = 0; j < NQ; ++j) Fiph[i + j] = -(1.0 / 6.0) * r * (U[i + j + sx] - U[i + j]) * g.dx;
      if (FM[i / NQ] || FM[(i + sy) / NQ])
        for (int j = 0; j < NQ; ++j) Giph[i + j] = -(1.0 / 6.0) * r * (U[i + j + sy] - U[i + j]) * g.dy;
      if (FM[i / NQ] || FM[(i + sz) / NQ])
        for (int j = 0; j < NQ; ++j) Hiph[i + j] = -(1.0 / 6.0) * r * (U[i + j + sz] - U[i + j]) * g.dz;
    }
    port_ct3d(Fiph, Giph, Hiph, g.stride);
    for (int i = sx; i < Ni - sx; ++i)
      L[i] = -((Fiph[i] - Fiph[i - sx]) / g.dx + (Giph[i] - Giph[i - sy]) / g.dy + (Hiph[i] - Hiph[i - sz]) / g.dz);
  }
  for (long i = 0; i < n; ++i) U[i] += L[i];
  memcpy(P, prev, n * sizeof(double));                      /* P = Mara->PrimitiveArray */
  const int err = c2p_all_mask(c, &g, U, P, FM);
  memcpy(prim, P, n * sizeof(double));
  for (long z = 0; z < g.nz; ++z) mask_out[z] = FM[z];
  free(P); free(U); free(L); free(Fiph); free(Giph); free(Hiph); free(FM);
  return err;
}

/* The eight other measures of Mara.measure (Mara/mara.cpp:1954-2230) on the interior zones of
 * P, in the cgs units of a started reference (PhysicalUnits(1, 1, 1), Mara/hydro.cpp:20):
 * out[0..7] mean_cons, [8..15] mean_prim, [16..19] mean_energies (magnetic, kinetic, internal,
 * total), [20..23] mean_velocity, [24, 25] mean_max_temperature, [26, 27]
 * mean_max_magnetic_field, [28, 29] mean_max_sonic_mach, [30, 31] mean_min_alfvenic_mach. */
void port_measures(const port_config *c, const double *P, double *out)
{
  int G[3];
  shape(c, G);
  const double Gamma = c->gamma;
  /* PhysicalUnits (Mara/units.cpp) at Length = Mass = Time = 1 */
  const double gram = 1.0 / 1.0, cm = 1.0 / 1.0, sec = 1.0 / 1.0;
  const double erg = gram * pow(cm / sec, 2.0);
  const double erg_cc = 1.60217648740e-06 * erg / pow(1e-13 * cm, 3) * 1e-33;
  const double g_cc = gram / pow(cm, 3.0);
  const double mp = 1.67262177774e-24 * gram, kb = 1.38064881300e-16 * erg;
  const double gauss = sqrt(erg / pow(cm, 3.0) / (4 * M_PI));
  double U[8], sumU[8] = {0}, sumP[8] = {0}, Vrms[4] = {0};
  double kinetic = 0, internal = 0, magnetic = 0, total = 0;
  double tT = 0, mT = 0, tMs = 0, mMs = 0, tMa = 0, mMa = 1e20, tB = 0, mB = 0;
  for (int i = 0; i < G[0]; ++i)
    for (int j = 0; j < G[1]; ++j)
      for (int k = 0; k < G[2]; ++k) {
        if (i < c->ng || i >= G[0] - c->ng) continue;
        if (c->nd >= 2 && (j < c->ng || j >= G[1] - c->ng)) continue;
        if (c->nd >= 3 && (k < c->ng || k >= G[2] - c->ng)) continue;
        const double *P0 = &P[(((long) i * G[1] + j) * G[2] + k) * 8];
        port_prim_to_cons(c, P0, U);
        for (int q = 0; q < 8; ++q) {
          sumU[q] += U[q];
          sumP[q] += P0[q];
        }
        const double v2 = P0[2] * P0[2] + P0[3] * P0[3] + P0[4] * P0[4];
        const double T0 = P0[1];
        const double u0 = T0 / (Gamma - 1);
        {
          const double rhoh = P0[0] + u0 + P0[1];
          const double W0 = 1.0 / sqrt(1.0 - v2);
          const double e_f = rhoh * W0 * W0 - P0[1] - U[0];
          const double e_m = U[1] - e_f;
          magnetic += e_m;
          kinetic += P0[0] * W0 * (W0 - 1);
          internal += W0 * u0;
          total += U[1];
        }
        Vrms[0] += 1.0 / sqrt(1.0 - v2);
        Vrms[1] += fabs(P0[2]);
        Vrms[2] += fabs(P0[3]);
        Vrms[3] += fabs(P0[4]);
        {
          const double Pc = P0[1] / erg_cc, rc = P0[0] / g_cc;
          const double T_K = (Pc / rc) * (mp / kb);
          const double Tm = T_K * 8.621738e-11;
          tT += Tm;
          if (Tm > mT) mT = Tm;
        }
        {
          const double rhoh = P0[0] + T0 / (Gamma - 1) + T0;
          const double cs2 = Gamma * T0 / rhoh;
          const double M0 = sqrt((v2 / (1 - v2)) / (cs2 / (1 - cs2)));
          tMs += M0;
          if (M0 > mMs) mMs = M0;
        }
        {
          const double B2 = P0[5] * P0[5] + P0[6] * P0[6] + P0[7] * P0[7];
          const double rhoh = P0[0] + u0 + P0[1];
          const double va2 = B2 / (B2 + rhoh);
          const double M0 = sqrt((v2 / (1 - v2)) / (va2 / (1 - va2)));
          tMa += M0;
          if (M0 < mMa) mMa = M0;
        }
        {
          const double B0 = sqrt(P0[5] * P0[5] + P0[6] * P0[6] + P0[7] * P0[7]);
          tB += B0;
          if (B0 > mB) mB = B0;
        }
      }
  long ttl = 1;
  for (int d = 0; d < c->nd; ++d) ttl *= c->n[d];
  for (int q = 0; q < 8; ++q) {
    out[q] = sumU[q] / ttl;
    out[8 + q] = sumP[q] / ttl;
  }
  out[16] = magnetic / ttl;
  out[17] = kinetic / ttl;
  out[18] = internal / ttl;
  out[19] = total / ttl;
  for (int q = 0; q < 4; ++q) out[20 + q] = Vrms[q] / ttl;
  out[24] = tT / ttl;
  out[25] = mT;
  out[26] = (1.0 / gauss) * tB / ttl;
  out[27] = (1.0 / gauss) * mB;
  out[28] = tMs / ttl;
  out[29] = mMs;
  out[30] = tMa / ttl;
  out[31] = mMa;
}
