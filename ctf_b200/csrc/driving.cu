// Stochastic velocity forcing: the reference's Ornstein-Uhlenbeck driving field
// (StochasticVectorField2d/3d, Mara/ou-field.cpp; OrnsteinUhlenbeckProcess, Mara/ornuhl.hpp;
// RandomNumberStream, Mara/random.cpp) and its application to the primitive state after
// each successful advance (DrivingProcedure::Drive_rmhd, Mara/driving.cpp:154-187).
//
// The field is a sum over the (2 k1 + 1)^nd integer wave vectors K = 2 pi (a, b, c) of
// complex amplitudes F_m, each advanced by its own OU process (theta 1, sigma^2 = 2 P0
// P(|K|) / sum P, P the StoneProfile spectrum) and projected to a zeta-weighted mix of
// solenoidal and compressive parts.  The mode amplitudes and their random streams live on
// the host (a few thousand numbers, advanced with the same generator, inverse error
// function and libm as the reference, so a serialized field from the reference continues
// identically here).  Sampling the field at every guarded zone and the per-zone
// 4-velocity kick run on the device:
//   * k_drive_sample: F(x) = Re sum_m F_m exp(i K_m . x), factorised per axis -- the zone's
//     phase e^{i 2 pi a x} comes from a small per-axis table, so a zone costs (2k1+1)^nd
//     complex products instead of as many complex exponentials;
//   * k_drive_kick: u = W0 v + F dt / W0, v' = u / sqrt(1 + u^2), rho' = rho W0 / W1 (rest
//     mass per zone kept), applied to every guarded zone of the newly committed state when
//     (and only when) the advance committed.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <complex>
#include <vector>

#include "solver.h"
#include "c2p_mlp.cuh"
#include "rmhd_physics.cuh"

using namespace mgpu;

namespace {

// RandomNumberStream (Mara/random.cpp:17-49): the generator whose sequence the reference's
// driving fields carry in their serialized state.
struct RngState {
  uint64_t u, v, w;
};

uint64_t rng_next(RngState &s)
{
  s.u = s.u * 2862933555777941757ULL + 7046029254386353087ULL;
  s.v ^= s.v >> 17;
  s.v ^= s.v << 31;
  s.v ^= s.v >> 8;
  s.w = 4294957665ULL * (s.w & 0xffffffffULL) + (s.w >> 32);
  uint64_t x = s.u ^ (s.u << 21);
  x ^= x >> 35;
  x ^= x << 4;
  return (x + s.v) ^ s.w;
}

RngState rng_seeded(int n)
{
  RngState s;
  s.v = 4101842887655102017ULL;
  s.w = 1;
  s.u = (uint64_t) (int64_t) n ^ s.v;
  rng_next(s);
  s.v = s.u;
  rng_next(s);
  s.w = s.v;
  rng_next(s);
  return s;
}

// A uniform double in [a, b): the 64-bit draw scaled in single precision, as the
// reference's float-suffixed constant makes it.
double rng_uniform(RngState &s, double a, double b)
{
  const float scaled = (float) rng_next(s) * 5.42101086242752217E-20f;
  return (double) scaled * (b - a) + a;
}

// Inverse error function by Newton from the series start (Mara/ornuhl.hpp:57-67).
double erf_inverse(double y)
{
  double x = 0.5 * sqrt(M_PI) * (y + M_PI / 12.0 * pow(y, 3));
  double step;
  do {
    const double f = erf(x) - y;
    const double g = 2.0 / sqrt(M_PI) * exp(-x * x);
    step = f / g;
    x -= step;
  } while (fabs(step) > 1e-12);
  return x;
}

// One OU process: its random stream and (theta, sigma); 40 bytes, the serialized layout.
struct OuProcess {
  RngState rng;
  double theta, sigma;
};
static_assert(sizeof(OuProcess) == 40, "serialized OU process is 40 bytes");

double sample_normal(OuProcess &p, double var)
{
  const double c = rng_uniform(p.rng, -1.0, 1.0);
  return sqrt(2 * var) * erf_inverse(c);
}

// OrnsteinUhlenbeckProcess::Deviate of a complex amplitude: -theta z dt + sigma dW, with the
// two normal draws taken imaginary part first, as the reference's build evaluates the
// constructor arguments of its complex dW.
std::complex<double> ou_deviate(OuProcess &p, std::complex<double> z, double dt)
{
  const double im = sample_normal(p, dt);
  const double re = sample_normal(p, dt);
  return -p.theta * z * dt + p.sigma * std::complex<double>(re, im);
}

double stone_profile(double k)
{
  const double peak = 2.0;
  return pow(k, 6) * exp(-8 * k / (2 * M_PI * peak));
}

}  // namespace

struct MgpuDriving {
  int nd = 3, k1 = 3, numk = 0;
  double P0 = 0, zeta = 0;
  std::vector<std::complex<double>> K[3], F[3];
  std::vector<OuProcess> proc;
  void *dev_F = nullptr;            // sampled field, 3 x nz doubles (floats in the lean layout)
  int f32 = 0;                      // dev_F holds floats
  double2 *dev_modes = nullptr;     // F_m per component, 3 x numk (device)
  double2 *dev_phase = nullptr;     // per-axis phases e^{i 2 pi a x_i}: 3 x (2k1+1) x G_max
  int gmax = 0;

  int rank() const { return 2 * k1 + 1; }

  // StochasticVectorField{2d,3d} constructor (Mara/ou-field.cpp:22-95)
  void build(int nd_, double P0_, double zeta_, int k1_, int seed)
  {
    nd = nd_;
    k1 = k1_;
    P0 = P0_;
    zeta = zeta_;
    const int r = rank();
    numk = nd == 3 ? r * r * r : r * r;
    for (int d = 0; d < 3; ++d) {
      K[d].assign(d < nd ? numk : 0, 0.0);
      F[d].assign(d < nd ? numk : 0, 0.0);
    }
    double total = 0.0;
    std::vector<double> kmag(numk);
    for (int m = 0; m < numk; ++m) {
      int idx[3];
      if (nd == 3) {
        idx[0] = m / (r * r) - k1;
        idx[1] = (m / r) % r - k1;
        idx[2] = m % r - k1;
      } else {
        idx[0] = m / r - k1;
        idx[1] = m % r - k1;
        idx[2] = 0;
      }
      double kk = 0.0;
      for (int d = 0; d < nd; ++d) {
        K[d][m] = 2 * M_PI * idx[d];
        kk += K[d][m].real() * K[d][m].real();
      }
      kmag[m] = sqrt(kk);
      total += stone_profile(kmag[m]);
    }
    proc.resize(numk);
    for (int m = 0; m < numk; ++m) {
      proc[m].rng = rng_seeded(seed + m);
      proc[m].theta = 1.0;
      proc[m].sigma = sqrt(2 * P0 * stone_profile(kmag[m]) / total);
    }
  }

  // StochasticVectorField*::AdvanceField (Mara/ou-field.cpp:160-215)
  void advance(double dt)
  {
    const double norm = sqrt(1 - 1.25 * zeta + 3 * zeta * zeta);
    for (int m = 0; m < numk; ++m) {
      double k[3] = {0, 0, 0}, kk = 0;
      for (int d = 0; d < nd; ++d) {
        k[d] = K[d][m].real();
        kk += k[d] * k[d];
      }
      if (kk < 1e-8) continue;   // the zero mode stays
      std::complex<double> dW[3], dV[3];
      for (int q = 0; q < nd; ++q) dW[q] = ou_deviate(proc[m], F[q][m], dt);
      for (int p = 0; p < nd; ++p) {
        dV[p] = 0.0;
        for (int q = 0; q < nd; ++q) {
          const double P = (1 - 2 * zeta) * k[p] * k[q] / kk + zeta * (p == q);
          if (nd == 3) dV[p] += P * dW[q] / norm;
          else dV[p] += P * dW[q];
        }
      }
      for (int p = 0; p < nd; ++p) F[p][m] += dV[p];
    }
  }

  // Serialize / deserialize: int k1, double P0, zeta, then per dimension the wave vectors,
  // then per dimension the amplitudes (complex double, numk each), then the OU processes.
  std::vector<unsigned char> serialize() const
  {
    std::vector<unsigned char> out(4 + 16 + (size_t) nd * 2 * numk * 16 + (size_t) numk * sizeof(OuProcess));
    size_t o = 0;
    auto put = [&](const void *p, size_t n) {
      memcpy(out.data() + o, p, n);
      o += n;
    };
    put(&k1, 4);
    put(&P0, 8);
    put(&zeta, 8);
    for (int d = 0; d < nd; ++d) put(K[d].data(), (size_t) numk * 16);
    for (int d = 0; d < nd; ++d) put(F[d].data(), (size_t) numk * 16);
    put(proc.data(), (size_t) numk * sizeof(OuProcess));
    return out;
  }

  bool deserialize(int nd_, const unsigned char *p, size_t n)
  {
    if (n < 20) return false;
    nd = nd_;
    memcpy(&k1, p, 4);
    memcpy(&P0, p + 4, 8);
    memcpy(&zeta, p + 12, 8);
    if (k1 < 0 || k1 > 64) return false;
    const int r = rank();
    numk = nd == 3 ? r * r * r : r * r;
    if (n != 20 + (size_t) nd * 2 * numk * 16 + (size_t) numk * sizeof(OuProcess)) return false;
    size_t o = 20;
    for (int d = 0; d < 3; ++d) {
      K[d].assign(d < nd ? numk : 0, 0.0);
      F[d].assign(d < nd ? numk : 0, 0.0);
    }
    for (int d = 0; d < nd; ++d, o += (size_t) numk * 16) memcpy(K[d].data(), p + o, (size_t) numk * 16);
    for (int d = 0; d < nd; ++d, o += (size_t) numk * 16) memcpy(F[d].data(), p + o, (size_t) numk * 16);
    proc.resize(numk);
    memcpy(proc.data(), p + o, (size_t) numk * sizeof(OuProcess));
    return true;
  }
};

namespace {

int fail(mgpu_solver *h, int code, const char *msg)
{
  if (h) h->err = msg;
  return code;
}

// F(x) at every guarded zone (DrivingProcedure::ResampleField, Mara/driving.cpp:44-84):
// zone coordinates x_at(i) = x0 + dx (i - Ng + 1/2), guards included.
template <class FT>
__global__ void k_drive_sample(Grid g, int nd, int k1, const double2 *modes, const double2 *phase, int gmax,
                               FT *F)
{
  const int r = 2 * k1 + 1;
  const int numk = nd == 3 ? r * r * r : r * r;
  for (long long z = (long long) blockIdx.x * blockDim.x + threadIdx.x; z < g.nz;
       z += (long long) gridDim.x * blockDim.x) {
    int i, j, k;
    zone_coords(g, z, i, j, k);
    const double2 *px = phase + (size_t) 0 * r * gmax;
    const double2 *py = phase + (size_t) 1 * r * gmax;
    const double2 *pz = phase + (size_t) 2 * r * gmax;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < r; ++a) {
      const double2 ea = px[a * gmax + i];
      for (int b = 0; b < r; ++b) {
        const double2 eb = py[b * gmax + j];
        const double2 eab = make_double2(ea.x * eb.x - ea.y * eb.y, ea.x * eb.y + ea.y * eb.x);
        const int cmax = nd == 3 ? r : 1;
        for (int c = 0; c < cmax; ++c) {
          double2 e = eab;
          if (nd == 3) {
            const double2 ec = pz[c * gmax + k];
            e = make_double2(eab.x * ec.x - eab.y * ec.y, eab.x * ec.y + eab.y * ec.x);
          }
          const int m = nd == 3 ? (a * r + b) * r + c : a * r + b;
          for (int q = 0; q < nd; ++q) {
            const double2 f = modes[q * numk + m];
            acc[q] += f.x * e.x - f.y * e.y;
          }
        }
      }
    }
    for (int q = 0; q < 3; ++q) F[q * g.nz + z] = FT(acc[q]);
  }
}

// The 4-velocity kick of Drive_rmhd on one zone's primitives p (rho, vx, vy, vz updated).
// In 2D the reference kicks vx, vy and carries vz as given (its 4-velocity array holds the
// 3-velocity vz there).
template <class FT>
__device__ __forceinline__ void drive_kick_zone(const Grid &g, int nd, const FT *F, long long z, double dt, double *p)
{
  double uf[4] = {0.0, p[vx], p[vy], p[vz]};
  const double v2 = uf[1] * uf[1] + uf[2] * uf[2] + uf[3] * uf[3];
  const double W0 = 1.0 / sqrt(1.0 - v2);
  uf[1] *= W0;
  uf[1] += double(F[0 * g.nz + z]) * (dt / W0);
  uf[2] *= W0;
  uf[2] += double(F[1 * g.nz + z]) * (dt / W0);
  if (nd == 3) {
    uf[3] *= W0;
    uf[3] += double(F[2 * g.nz + z]) * (dt / W0);
  }
  const double u2 = uf[1] * uf[1] + uf[2] * uf[2] + uf[3] * uf[3];
  const double W1 = sqrt(1.0 + u2);
  p[vx] = uf[1] / W1;
  p[vy] = uf[2] / W1;
  p[vz] = uf[3] / W1;
  p[rho] = p[rho] * (W0 / W1);
}

// The kick on the committed state, every guarded zone, only if the advance committed.
template <class T>
__global__ void k_drive_kick(Grid g, int nd, const double *F, T *bulk0, T *bulk1, const Ctl *ctl)
{
  if (!ctl->committed) return;
  T *P = ctl->cur ? bulk1 : bulk0;
  const double dt = ctl->dt;
  for (long long z = (long long) blockIdx.x * blockDim.x + threadIdx.x; z < g.nz;
       z += (long long) gridDim.x * blockDim.x) {
    double p[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) p[q] = double(P[q * g.cs + z]);
    drive_kick_zone<double>(g, nd, F, z, dt, p);
    P[vx * g.cs + z] = T(p[vx]);
    P[vy * g.cs + z] = T(p[vy]);
    P[vz * g.cs + z] = T(p[vz]);
    P[rho * g.cs + z] = T(p[rho]);
  }
}

// The kick in the lean layout: the committed primitives are PA, every guarded zone; the
// committed conserved state U[cur] is rebuilt from the kicked primitives at interior zones
// (the next advance starts from it).
template <class T, class FT>
__global__ void k_drive_kick_lean(Grid g, int nd, const FT *F, T *PA, StatePtr<T> UA, StatePtr<T> UB, double gamma,
                                  const Ctl *ctl)
{
  if (!ctl->committed) return;
  const StatePtr<T> U = ctl->cur ? UB : UA;
  const double dt = ctl->dt;
  for (long long z = (long long) blockIdx.x * blockDim.x + threadIdx.x; z < g.nz;
       z += (long long) gridDim.x * blockDim.x) {
    double p[8], u[8];
#pragma unroll
    for (int q = 0; q < 5; ++q) p[q] = double(PA[q * g.cs + z]);
    drive_kick_zone<FT>(g, nd, F, z, dt, p);
    PA[vx * g.cs + z] = T(p[vx]);
    PA[vy * g.cs + z] = T(p[vy]);
    PA[vz * g.cs + z] = T(p[vz]);
    PA[rho * g.cs + z] = T(p[rho]);
    int i, j, k;
    zone_coords(g, z, i, j, k);
    if (i < g.ng || i >= g.ng + g.n[0] || j < g.ng || j >= g.ng + g.n[1] || k < g.ng || k >= g.ng + g.n[2]) continue;
#pragma unroll
    for (int q = 0; q < 3; ++q) p[5 + q] = U.B[q * g.cs + z];
    prim_to_cons(gamma, p, u);
#pragma unroll
    for (int q = 0; q < 5; ++q) U.bulk[q * g.cs + z] = T(u[q]);
  }
}

bool fp32(const mgpu_solver *h) { return h->cfg.precision == MGPU_PREC_FP32; }
bool lean(const mgpu_solver *h) { return h->cfg.layout == MGPU_LAYOUT_LEAN; }

int resample(mgpu_solver *h)
{
  MgpuDriving &D = *h->driving;
  const Grid &g = h->g;
  const int r = D.rank();
  // per-axis phases e^{i K x_at(i)} on the host (libm, as the reference's complex exp)
  std::vector<double2> ph((size_t) 3 * r * D.gmax, make_double2(1.0, 0.0));
  const double x0[3] = {h->x0[0], h->x0[1], h->x0[2]};
  const double dx[3] = {g.dx, g.dy, g.dz};
  for (int d = 0; d < D.nd; ++d)
    for (int a = 0; a < r; ++a)
      for (int i = 0; i < g.G[d]; ++i) {
        const double x = x0[d] + dx[d] * (i - g.ng + 0.5);
        const double th = 2 * M_PI * (a - D.k1) * x;
        ph[((size_t) d * r + a) * D.gmax + i] = make_double2(cos(th), sin(th));
      }
  std::vector<double2> modes((size_t) 3 * D.numk, make_double2(0.0, 0.0));
  for (int q = 0; q < D.nd; ++q)
    for (int m = 0; m < D.numk; ++m) modes[(size_t) q * D.numk + m] = make_double2(D.F[q][m].real(), D.F[q][m].imag());
  cudaError_t e = cudaMemcpyAsync(D.dev_phase, ph.data(), ph.size() * sizeof(double2), cudaMemcpyHostToDevice,
                                  h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(D.dev_modes, modes.data(), modes.size() * sizeof(double2), cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) {
    if (D.f32)
      k_drive_sample<float><<<148 * 8, 256, 0, h->stream>>>(g, D.nd, D.k1, D.dev_modes, D.dev_phase, D.gmax,
                                                            (float *) D.dev_F);
    else
      k_drive_sample<double><<<148 * 8, 256, 0, h->stream>>>(g, D.nd, D.k1, D.dev_modes, D.dev_phase, D.gmax,
                                                             (double *) D.dev_F);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);   // host vectors die here
  if (e != cudaSuccess) {
    h->err = std::string("driving resample: ") + cudaGetErrorString(e);
    return MGPU_ERR_CUDA;
  }
  return MGPU_OK;
}

}  // namespace

cudaError_t mgpu_driving_enqueue(mgpu_solver *h)
{
  if (!h->driving) return cudaSuccess;
  const Grid &g = h->g;
  const MgpuDriving &D = *h->driving;
  const AdvanceBuffers &b = h->b;
  if (lean(h)) {
    if (fp32(h))
      k_drive_kick_lean<float, float><<<148 * 8, 256, 0, h->stream>>>(
          g, D.nd, (const float *) D.dev_F, (float *) b.PA, StatePtr<float>{(float *) b.U0_bulk, b.U0_B},
          StatePtr<float>{(float *) b.U1_bulk, b.U1_B}, h->cfg.gamma, h->ctl);
    else
      k_drive_kick_lean<double, float><<<148 * 8, 256, 0, h->stream>>>(
          g, D.nd, (const float *) D.dev_F, (double *) b.PA, StatePtr<double>{(double *) b.U0_bulk, b.U0_B},
          StatePtr<double>{(double *) b.U1_bulk, b.U1_B}, h->cfg.gamma, h->ctl);
    return cudaGetLastError();
  }
  if (fp32(h))
    k_drive_kick<float><<<148 * 8, 256, 0, h->stream>>>(g, h->driving->nd, (const double *) h->driving->dev_F,
                                                        (float *) h->b.Pc_bulk[0], (float *) h->b.Pc_bulk[1], h->ctl);
  else
    k_drive_kick<double><<<148 * 8, 256, 0, h->stream>>>(g, h->driving->nd, (const double *) h->driving->dev_F,
                                                         (double *) h->b.Pc_bulk[0], (double *) h->b.Pc_bulk[1], h->ctl);
  return cudaGetLastError();
}

void mgpu_driving_free(mgpu_solver *h)
{
  if (!h || !h->driving) return;
  if (h->stream) cudaStreamSynchronize(h->stream);
  cudaFree(h->driving->dev_F);
  cudaFree(h->driving->dev_modes);
  cudaFree(h->driving->dev_phase);
  delete h->driving;
  h->driving = nullptr;
}

extern "C" {

int mgpu_new_ou_field(int nd, double P0, double zeta, int k1, int seed, void *out, long long *bytes)
{
  if ((nd != 2 && nd != 3) || k1 < 0 || k1 > 16 || !bytes) return MGPU_ERR_ARG;
  MgpuDriving D;
  D.build(nd, P0, zeta, k1, seed);
  const std::vector<unsigned char> s = D.serialize();
  if (out) {
    if (*bytes < (long long) s.size()) return MGPU_ERR_ARG;
    memcpy(out, s.data(), s.size());
  }
  *bytes = (long long) s.size();
  return MGPU_OK;
}

int mgpu_ou_field_advance(void *field, long long bytes, int nd, double dt)
{
  if (!field || (nd != 2 && nd != 3)) return MGPU_ERR_ARG;
  MgpuDriving D;
  if (!D.deserialize(nd, (const unsigned char *) field, (size_t) bytes)) return MGPU_ERR_ARG;
  D.advance(dt);
  const std::vector<unsigned char> s = D.serialize();
  memcpy(field, s.data(), s.size());
  return MGPU_OK;
}

int mgpu_set_driving(mgpu_solver *h, const void *field, long long bytes)
{
  if (!h) return MGPU_ERR_ARG;
  if (!h->have_domain) return fail(h, MGPU_ERR_STATE, "need a domain to run this, use set_domain");
  if (h->g.nd < 2) return fail(h, MGPU_ERR_ARG, "driving needs a 2d or 3d domain");
  mgpu_driving_free(h);
  if (!field || bytes <= 0) return MGPU_OK;   // clears the driving
  MgpuDriving *D = new MgpuDriving;
  if (!D->deserialize(h->g.nd, (const unsigned char *) field, (size_t) bytes)) {
    delete D;
    return fail(h, MGPU_ERR_ARG, "driving field does not match the domain's dimensionality or is corrupt");
  }
  const Grid &g = h->g;
  D->gmax = g.G[0] > g.G[1] ? (g.G[0] > g.G[2] ? g.G[0] : g.G[2]) : (g.G[1] > g.G[2] ? g.G[1] : g.G[2]);
  D->f32 = lean(h);   // the lean layout's boxes keep the sampled field in FP32 (12 B per zone)
  cudaError_t e = cudaMalloc(&D->dev_F, (D->f32 ? sizeof(float) : sizeof(double)) * 3 * (size_t) g.nz);
  if (e == cudaSuccess) e = cudaMalloc((void **) &D->dev_modes, sizeof(double2) * 3 * (size_t) D->numk);
  if (e == cudaSuccess) e = cudaMalloc((void **) &D->dev_phase, sizeof(double2) * 3 * (size_t) D->rank() * D->gmax);
  if (e != cudaSuccess) {
    cudaFree(D->dev_F);
    cudaFree(D->dev_modes);
    cudaFree(D->dev_phase);
    delete D;
    cudaGetLastError();
    return fail(h, MGPU_ERR_NOMEM, "driving: out of device memory");
  }
  h->driving = D;
  return resample(h);   // DrivingProcedure's constructor samples the field
}

int mgpu_driving_advance(mgpu_solver *h, double dt)
{
  if (!h) return MGPU_ERR_ARG;
  if (h->driving) h->driving->advance(dt);
  return MGPU_OK;
}

int mgpu_driving_resample(mgpu_solver *h)
{
  if (!h) return MGPU_ERR_ARG;
  return h->driving ? resample(h) : MGPU_OK;
}

int mgpu_driving_serialize(mgpu_solver *h, void *out, long long *bytes)
{
  if (!h || !bytes) return MGPU_ERR_ARG;
  if (!h->driving) {
    *bytes = 0;
    return MGPU_OK;
  }
  const std::vector<unsigned char> s = h->driving->serialize();
  if (out) {
    if (*bytes < (long long) s.size()) return fail(h, MGPU_ERR_ARG, "serialize buffer too small");
    memcpy(out, s.data(), s.size());
  }
  *bytes = (long long) s.size();
  return MGPU_OK;
}

// DrivingProcedure::AveragePowerInFields (Mara/driving.cpp:31-39): mean over every guarded
// zone of |F|^2 (computed on the host from a copy of the sampled field).
int mgpu_driving_power(mgpu_solver *h, double *power)
{
  if (!h || !power) return MGPU_ERR_ARG;
  *power = 0.0;
  if (!h->driving) return MGPU_OK;
  const long long nz = h->g.nz;
  const MgpuDriving &D = *h->driving;
  const size_t esz = D.f32 ? sizeof(float) : sizeof(double);
  const long long chunk = 1ll << 22;   // zones per host copy
  std::vector<unsigned char> buf((size_t) 3 * chunk * esz);
  auto at = [&](int q, long long z) {
    return D.f32 ? (double) ((const float *) buf.data())[q * chunk + z] : ((const double *) buf.data())[q * chunk + z];
  };
  cudaError_t e = cudaStreamSynchronize(h->stream);
  double s = 0.0;
  for (long long z0 = 0; z0 < nz && e == cudaSuccess; z0 += chunk) {
    const long long cnt = nz - z0 < chunk ? nz - z0 : chunk;
    for (int q = 0; q < D.nd && e == cudaSuccess; ++q)
      e = cudaMemcpy(buf.data() + (size_t) q * chunk * esz, (const unsigned char *) D.dev_F + ((size_t) q * nz + z0) * esz,
                     (size_t) cnt * esz, cudaMemcpyDeviceToHost);
    for (long long z = 0; z < cnt && e == cudaSuccess; ++z) {
      double v = at(0, z) * at(0, z) + at(1, z) * at(1, z);
      if (D.nd == 3) v += at(2, z) * at(2, z);
      s += v;
    }
  }
  if (e != cudaSuccess) return fail(h, MGPU_ERR_CUDA, cudaGetErrorString(e));
  *power = s / (double) nz;
  return MGPU_OK;
}

}  // extern "C"
