// Training and evaluation of the learned c2p initial guess (no counterpart in the reference).
//
//   mgpu_c2p_harvest   (features, targets) of every interior zone of a solver's committed
//                      state: the (conserved, primitive) pairs the method itself produced
//   mgpu_mlp_loss_grad mean squared error over n samples and its gradient (deterministic:
//                      per-block partial sums reduced in a fixed order)
//   mgpu_mlp_train     minibatch Adam on the device
//   mgpu_mlp_forward   the network on n feature rows (the per-thread evaluation the c2p uses)
//
// Hand-written SIMT kernels: one thread per sample, weights and the block's activations in
// shared memory; weight gradients are block reductions over the block's samples.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "../../include/mara_gpu.h"
#include "c2p_mlp.cuh"
#include "c2p_mlp_tc.cuh"

using namespace mgpu;
using namespace mgpu::mlp;

namespace {

constexpr int TB = 128;          // samples (threads) per block
constexpr int LD = NH + 1;       // padded row of the activation tiles (bank-conflict free)

// ---- harvest -------------------------------------------------------------------------------
template <class T>
__global__ void k_harvest(Grid g, StateCPtr<T> P0, StateCPtr<T> P1, const Ctl *ctl, double gamma, float *X,
                          float *Y)
{
  const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.ninterior) return;
  int i, j, k;
  interior_coords(g, t, i, j, k);
  const long long z = ((long long) i * g.G[1] + j) * g.G[2] + k;
  const StateCPtr<T> P = ctl->cur ? P1 : P0;
  double p[8], u[8];
#pragma unroll
  for (int c = 0; c < 5; ++c) p[c] = double(P.bulk[c * g.cs + z]);
#pragma unroll
  for (int c = 0; c < 3; ++c) p[5 + c] = P.B[c * g.cs + z];
  prim_to_cons(gamma, p, u);
  const double S2 = u[Sx] * u[Sx] + u[Sy] * u[Sy] + u[Sz] * u[Sz];
  const double B2 = u[Bx] * u[Bx] + u[By] * u[By] + u[Bz] * u[Bz];
  const double BS = u[Bx] * u[Sx] + u[By] * u[Sy] + u[Bz] * u[Sz];
  float x[NIN];
  c2p_features(u[ddd], u[tau], S2, B2, BS * BS, x);
#pragma unroll
  for (int c = 0; c < NIN; ++c) X[t * NIN + c] = x[c];
  const double v2 = p[vx] * p[vx] + p[vy] * p[vy] + p[vz] * p[vz];
  const double W = 1.0 / sqrt(1.0 - v2);
  const double h = 1.0 + gamma / (gamma - 1.0) * p[pre] / p[rho];
  Y[t * NOUT + 0] = (float) log(W);
  Y[t * NOUT + 1] = (float) log(h);
}

// ---- forward + backward, per-block partial gradients ------------------------------------------
// Block b handles samples [b*TB, b*TB + TB) of the index list idx (or of 0..n-1 when idx is
// null), writes its summed gradient (N_TRAIN floats) and summed squared error to part.
__global__ void __launch_bounds__(TB) k_grad(const float *__restrict__ P, const float *__restrict__ X,
                                             const float *__restrict__ Y, const int *__restrict__ idx,
                                             long long n, float scale, float *__restrict__ part)
{
  extern __shared__ float sm[];
  float *w = sm;                         // N_PARAMS
  float *A1 = w + N_PARAMS;              // TB x LD
  float *A2 = A1 + TB * LD;
  float *A3 = A2 + TB * LD;
  float *D = A3 + TB * LD;               // TB x LD deltas (reused per layer)
  float *Xs = D + TB * LD;               // TB x NIN
  float *red = Xs + TB * NIN;            // TB
  const int t = threadIdx.x;
  for (int e = t; e < N_PARAMS; e += TB) w[e] = P[e];
  const long long s = (long long) blockIdx.x * TB + t;
  const bool valid = s < n;
  const long long row = valid ? (idx ? (long long) idx[s] : s) : 0;
  __syncthreads();
  float x[NIN], yt[NOUT];
#pragma unroll
  for (int i = 0; i < NIN; ++i) {
    x[i] = valid ? (X[row * NIN + i] - w[OXM + i]) / w[OXS + i] : 0.f;
    Xs[t * NIN + i] = x[i];
  }
#pragma unroll
  for (int k = 0; k < NOUT; ++k) yt[k] = valid ? (Y[row * NOUT + k] - w[OYM + k]) / w[OYS + k] : 0.f;
  // forward
  for (int j = 0; j < NH; ++j) {
    float a = w[OB1 + j];
#pragma unroll
    for (int i = 0; i < NIN; ++i) a = fmaf(w[OW1 + j * NIN + i], x[i], a);
    A1[t * LD + j] = tanhf(a);
  }
  for (int j = 0; j < NH; ++j) {
    float a = w[OB2 + j];
    for (int i = 0; i < NH; ++i) a = fmaf(w[OW2 + j * NH + i], A1[t * LD + i], a);
    A2[t * LD + j] = tanhf(a);
  }
  for (int j = 0; j < NH; ++j) {
    float a = w[OB3 + j];
    for (int i = 0; i < NH; ++i) a = fmaf(w[OW3 + j * NH + i], A2[t * LD + i], a);
    A3[t * LD + j] = tanhf(a);
  }
  float gy[NOUT], se = 0.f;
#pragma unroll
  for (int k = 0; k < NOUT; ++k) {
    float a = w[OB4 + k];
    for (int i = 0; i < NH; ++i) a = fmaf(w[OW4 + k * NH + i], A3[t * LD + i], a);
    const float r = valid ? a - yt[k] : 0.f;
    se += r * r;
    gy[k] = 2.f * r * scale;
  }
  red[t] = se;
  // backward: delta of layer 3
  for (int j = 0; j < NH; ++j) {
    float d = 0.f;
#pragma unroll
    for (int k = 0; k < NOUT; ++k) d = fmaf(w[OW4 + k * NH + j], gy[k], d);
    const float a = A3[t * LD + j];
    D[t * LD + j] = d * (1.f - a * a);
  }
  // per-thread gy into the delta tile's spare column space for the W4 reduction
  __syncthreads();
  float *out = part + (long long) blockIdx.x * (N_TRAIN + 1);
  // W4, b4: thread e reduces entry e over the block's samples
  {
    __shared__ float GY[TB][NOUT];
#pragma unroll
    for (int k = 0; k < NOUT; ++k) GY[t][k] = gy[k];
    __syncthreads();
    for (int e = t; e < NOUT * NH + NOUT; e += TB) {
      float acc = 0.f;
      if (e < NOUT * NH) {
        const int k = e / NH, i = e % NH;
        for (int q = 0; q < TB; ++q) acc = fmaf(GY[q][k], A3[q * LD + i], acc);
        out[OW4 + e] = acc;
      } else {
        const int k = e - NOUT * NH;
        for (int q = 0; q < TB; ++q) acc += GY[q][k];
        out[OB4 + k] = acc;
      }
    }
  }
  // W3, b3 from D (layer-3 delta) and A2
  for (int e = t; e < NH * NH; e += TB) {
    const int j = e / NH, i = e % NH;
    float acc = 0.f;
    for (int q = 0; q < TB; ++q) acc = fmaf(D[q * LD + j], A2[q * LD + i], acc);
    out[OW3 + e] = acc;
  }
  if (t < NH) {
    float acc = 0.f;
    for (int q = 0; q < TB; ++q) acc += D[q * LD + t];
    out[OB3 + t] = acc;
  }
  // delta of layer 2 (into A3, once every thread is done reading it above)
  __syncthreads();
  for (int j = 0; j < NH; ++j) {
    float d = 0.f;
    for (int k = 0; k < NH; ++k) d = fmaf(w[OW3 + k * NH + j], D[t * LD + k], d);
    const float a = A2[t * LD + j];
    A3[t * LD + j] = d * (1.f - a * a);
  }
  __syncthreads();
  for (int e = t; e < NH * NH; e += TB) {
    const int j = e / NH, i = e % NH;
    float acc = 0.f;
    for (int q = 0; q < TB; ++q) acc = fmaf(A3[q * LD + j], A1[q * LD + i], acc);
    out[OW2 + e] = acc;
  }
  if (t < NH) {
    float acc = 0.f;
    for (int q = 0; q < TB; ++q) acc += A3[q * LD + t];
    out[OB2 + t] = acc;
  }
  // delta of layer 1 (into D)
  __syncthreads();
  for (int j = 0; j < NH; ++j) {
    float d = 0.f;
    for (int k = 0; k < NH; ++k) d = fmaf(w[OW2 + k * NH + j], A3[t * LD + k], d);
    const float a = A1[t * LD + j];
    D[t * LD + j] = d * (1.f - a * a);
  }
  __syncthreads();
  for (int e = t; e < NH * NIN; e += TB) {
    const int j = e / NIN, i = e % NIN;
    float acc = 0.f;
    for (int q = 0; q < TB; ++q) acc = fmaf(D[q * LD + j], Xs[q * NIN + i], acc);
    out[OW1 + e] = acc;
  }
  if (t < NH) {
    float acc = 0.f;
    for (int q = 0; q < TB; ++q) acc += D[q * LD + t];
    out[OB1 + t] = acc;
  }
  // summed squared error (fixed-order tree)
  for (int o = TB / 2; o > 0; o >>= 1) {
    __syncthreads();
    if (t < o) red[t] += red[t + o];
  }
  if (t == 0) out[N_TRAIN] = red[0];
}

// Sum the per-block partials in block order (deterministic); optionally apply Adam.
__global__ void k_reduce_adam(const float *__restrict__ part, int nblocks, float *__restrict__ grad,
                              double *loss_out, float *P, float *M, float *V, int step, float lr, int apply,
                              double loss_scale)
{
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e > N_TRAIN) return;
  double acc = 0.0;
  for (int b = 0; b < nblocks; ++b) acc += (double) part[(long long) b * (N_TRAIN + 1) + e];
  if (e == N_TRAIN) {
    if (loss_out) *loss_out = acc * loss_scale;
    return;
  }
  const float gsum = (float) acc;
  if (grad) grad[e] = gsum;
  if (apply) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float m = b1 * M[e] + (1.f - b1) * gsum;
    const float v = b2 * V[e] + (1.f - b2) * gsum * gsum;
    M[e] = m;
    V[e] = v;
    const float mh = m / (1.f - powf(b1, (float) step));
    const float vh = v / (1.f - powf(b2, (float) step));
    P[e] -= lr * mh / (sqrtf(vh) + eps);
  }
}

__global__ void k_forward(const float *__restrict__ P, const float *__restrict__ X, long long n, float *Y)
{
  const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  float x[NIN], y[NOUT];
#pragma unroll
  for (int i = 0; i < NIN; ++i) x[i] = X[t * NIN + i];
  mlp_forward_thread(P, x, y);
#pragma unroll
  for (int k = 0; k < NOUT; ++k) Y[t * NOUT + k] = y[k];
}

// Fisher-Yates-free shuffle: a per-epoch random permutation via sort keys is not needed;
// minibatches take a strided, epoch-rotated sample of the data instead.
__global__ void k_batch_index(int *idx, long long n, int batch, long long offset, long long stride)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= batch) return;
  idx[t] = (int) ((offset + (long long) t * stride) % n);
}

// The network on n rows with the tensor-core path (the same TcNet the c2p kernel uses).
__global__ void __launch_bounds__(128) k_forward_tc(const unsigned char *image, const float *__restrict__ X,
                                                    long long n, float *Y, int *fault)
{
  extern __shared__ unsigned char sm_tc[];
  tc::TcNet net = tc::tc_setup(sm_tc, image);
  const long long ntiles = (n + 127) / 128;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long t = tile * 128 + threadIdx.x;
    const bool valid = t < n;
    float x[NIN] = {0.f, 0.f, 0.f, 0.f, 0.f}, xn[NIN] = {0.f, 0.f, 0.f, 0.f, 0.f}, y[NOUT];
    if (valid) {
#pragma unroll
      for (int i = 0; i < NIN; ++i) x[i] = X[t * NIN + i];
      net.normalise(x, xn);
    }
    const bool ok = net.forward(xn, y);
    if (valid) {
      Y[t * NOUT + 0] = ok ? y[0] : NAN;
      Y[t * NOUT + 1] = ok ? y[1] : NAN;
    }
  }
  if (!net.ok && threadIdx.x == 0) atomicExch(fault, 1);
  tc::tc_teardown(net);
}

uint16_t float_to_bf16(float f)
{
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t) ((u >> 16) | ((u & 0xffffu) ? 0x40u : 0u));
  u += 0x7fffu + ((u >> 16) & 1u);   // round to nearest, ties to even
  return (uint16_t) (u >> 16);
}

// Float offset of the FP64 loss after nb blocks of partials (N_TRAIN + 1 floats each, an odd
// count): rounded up to an even float index so that the double is 8-byte aligned.
inline size_t loss_slot(long long nb) { return ((size_t) nb * (N_TRAIN + 1) + 1) & ~(size_t) 1; }

constexpr size_t grad_smem() { return sizeof(float) * (N_PARAMS + 4 * TB * LD + TB * NIN + TB); }

int cuda_check(cudaError_t e, const char *what)
{
  if (e != cudaSuccess) {
    fprintf(stderr, "[mgpu] %s: %s\n", what, cudaGetErrorString(e));
    return MGPU_ERR_CUDA;
  }
  return MGPU_OK;
}

}  // namespace

// Host access to a solver's grid and state for the harvest (defined in mara_gpu.cu).
extern "C" int mgpu_internal_state(mgpu_solver *h, mgpu::Grid *g, mgpu::AdvanceBuffers *b, mgpu::Ctl **ctl,
                                   void **stream, int *fp32, double *gamma);

extern "C" {

int mgpu_mlp_param_count(void) { return N_PARAMS; }

int mgpu_c2p_harvest(mgpu_solver *h, float *dev_x, float *dev_y, long long capacity, long long *count)
{
  Grid g;
  AdvanceBuffers b;
  Ctl *ctl;
  void *stream;
  int is32;
  double gamma;
  int rc = mgpu_internal_state(h, &g, &b, &ctl, &stream, &is32, &gamma);
  if (rc) return rc;
  if (!dev_x || !dev_y || !count) return MGPU_ERR_ARG;
  *count = g.ninterior;
  if (capacity < g.ninterior) return MGPU_ERR_ARG;
  const unsigned blk = 256, grid = (unsigned) ((g.ninterior + blk - 1) / blk);
  cudaStream_t st = (cudaStream_t) stream;
  if (is32)
    k_harvest<float><<<grid, blk, 0, st>>>(g, StateCPtr<float>{(const float *) b.Pc_bulk[0], b.Pc_B[0]},
                                           StateCPtr<float>{(const float *) b.Pc_bulk[1], b.Pc_B[1]}, ctl, gamma,
                                           dev_x, dev_y);
  else
    k_harvest<double><<<grid, blk, 0, st>>>(g, StateCPtr<double>{(const double *) b.Pc_bulk[0], b.Pc_B[0]},
                                            StateCPtr<double>{(const double *) b.Pc_bulk[1], b.Pc_B[1]}, ctl,
                                            gamma, dev_x, dev_y);
  if ((rc = cuda_check(cudaGetLastError(), "harvest"))) return rc;
  return cuda_check(cudaStreamSynchronize(st), "harvest");
}

int mgpu_mlp_loss_grad(const float *dev_params, const float *dev_x, const float *dev_y, long long n,
                       float *dev_grad, float *dev_work, double *loss)
{
  // dev_work: at least mgpu_mlp_work_floats(n) floats
  if (!dev_params || !dev_x || !dev_y || n <= 0 || !dev_grad || !dev_work || !loss) return MGPU_ERR_ARG;
  const int nb = (int) ((n + TB - 1) / TB);
  const size_t smem = grad_smem();
  int rc = cuda_check(cudaFuncSetAttribute(k_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem), "smem");
  if (rc) return rc;
  const float scale = 1.f / (float) (n * NOUT);
  k_grad<<<nb, TB, smem>>>(dev_params, dev_x, dev_y, nullptr, n, scale, dev_work);
  double *dloss = (double *) (dev_work + loss_slot(nb));
  k_reduce_adam<<<(N_TRAIN + 1 + 255) / 256, 256>>>(dev_work, nb, dev_grad, dloss, nullptr, nullptr, nullptr, 0,
                                                     0.f, 0, 1.0 / (double) (n * NOUT));
  if ((rc = cuda_check(cudaGetLastError(), "loss_grad"))) return rc;
  rc = cuda_check(cudaMemcpy(loss, dloss, sizeof(double), cudaMemcpyDeviceToHost), "loss_grad");
  return rc;
}

long long mgpu_mlp_work_floats(long long batch)
{
  const long long nb = (batch + TB - 1) / TB;
  return loss_slot(nb) + 2 + batch;   // partials, an 8-byte aligned double loss, the batch index list
}

int mgpu_mlp_train(float *dev_params, float *dev_m, float *dev_v, const float *dev_x, const float *dev_y,
                   long long n, int batch, int steps, float lr, int step0, float *dev_work, double *last_loss)
{
  if (!dev_params || !dev_m || !dev_v || !dev_x || !dev_y || n <= 0 || batch <= 0 || steps <= 0 || !dev_work)
    return MGPU_ERR_ARG;
  const int nb = (batch + TB - 1) / TB;
  const size_t smem = grad_smem();
  int rc = cuda_check(cudaFuncSetAttribute(k_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem), "smem");
  if (rc) return rc;
  float *part = dev_work;
  double *dloss = (double *) (dev_work + loss_slot(nb));
  int *idx = (int *) (dev_work + loss_slot(nb) + 2);
  const float scale = 1.f / (float) ((long long) batch * NOUT);
  // a stride coprime with n walks through the data set; each step starts where the last ended
  long long stride = 7919;
  while (n % stride == 0) stride += 2;
  for (int s = 0; s < steps; ++s) {
    const long long offset = ((long long) (step0 + s) * batch) % n;
    k_batch_index<<<(batch + 255) / 256, 256>>>(idx, n, batch, offset, stride);
    k_grad<<<nb, TB, smem>>>(dev_params, dev_x, dev_y, idx, batch, scale, part);
    k_reduce_adam<<<(N_TRAIN + 1 + 255) / 256, 256>>>(part, nb, nullptr, dloss, dev_params, dev_m, dev_v,
                                                       step0 + s + 1, lr, 1, 1.0 / (double) (batch * NOUT));
  }
  if ((rc = cuda_check(cudaGetLastError(), "train"))) return rc;
  if (last_loss) rc = cuda_check(cudaMemcpy(last_loss, dloss, sizeof(double), cudaMemcpyDeviceToHost), "train");
  else rc = cuda_check(cudaDeviceSynchronize(), "train");
  return rc;
}

int mgpu_mlp_build_tc_image(const float *params, void *image)
{
  if (!params || !image) return MGPU_ERR_ARG;
  unsigned char *img = (unsigned char *) image;
  memset(img, 0, tc::IMAGE_BYTES);
  auto put = [&](int off, float v) {
    const uint16_t b = float_to_bf16(v);
    memcpy(img + off, &b, 2);
  };
  for (int j = 0; j < NH; ++j) {
    for (int k = 0; k < NIN; ++k) put(tc::W1_OFF + tc::canon_offset(j, k, 16), params[OW1 + j * NIN + k]);
    for (int k = 0; k < NH; ++k) {
      put(tc::W2_OFF + tc::canon_offset(j, k, 64), params[OW2 + j * NH + k]);
      put(tc::W3_OFF + tc::canon_offset(j, k, 64), params[OW3 + j * NH + k]);
    }
  }
  for (int j = 0; j < NOUT; ++j)
    for (int k = 0; k < NH; ++k) put(tc::W4_OFF + tc::canon_offset(j, k, 64), params[OW4 + j * NH + k]);
  float *f = (float *) (img + tc::F_OFF);
  for (int j = 0; j < NH; ++j) {
    f[tc::F_B1 + j] = params[OB1 + j];
    f[tc::F_B2 + j] = params[OB2 + j];
    f[tc::F_B3 + j] = params[OB3 + j];
  }
  for (int k = 0; k < NOUT; ++k) {
    f[tc::F_B4 + k] = params[OB4 + k];
    f[tc::F_YM + k] = params[OYM + k];
    f[tc::F_YS + k] = params[OYS + k];
  }
  for (int i = 0; i < NIN; ++i) {
    f[tc::F_XM + i] = params[OXM + i];
    f[tc::F_XS + i] = params[OXS + i];
  }
  return MGPU_OK;
}

int mgpu_mlp_tc_image_bytes(void) { return tc::IMAGE_BYTES; }

int mgpu_mlp_forward_tc(const float *params, const float *dev_x, long long n, float *dev_y)
{
  if (!params || !dev_x || !dev_y || n <= 0) return MGPU_ERR_ARG;
  unsigned char host[tc::IMAGE_BYTES];
  mgpu_mlp_build_tc_image(params, host);
  unsigned char *dimg = nullptr;
  int *dfault = nullptr;
  int rc = cuda_check(cudaMalloc((void **) &dimg, tc::IMAGE_BYTES), "forward_tc");
  if (!rc) rc = cuda_check(cudaMalloc((void **) &dfault, sizeof(int)), "forward_tc");
  if (!rc) rc = cuda_check(cudaMemcpy(dimg, host, tc::IMAGE_BYTES, cudaMemcpyHostToDevice), "forward_tc");
  if (!rc) rc = cuda_check(cudaMemset(dfault, 0, sizeof(int)), "forward_tc");
  if (!rc) {
    const long long ntiles = (n + 127) / 128;
    const unsigned grid = (unsigned) (ntiles < 148 * 3 ? ntiles : 148 * 3);
    k_forward_tc<<<grid, 128, tc::SMEM_BYTES>>>(dimg, dev_x, n, dev_y, dfault);
    rc = cuda_check(cudaGetLastError(), "forward_tc");
    if (!rc) rc = cuda_check(cudaDeviceSynchronize(), "forward_tc");
  }
  int fault = 0;
  if (!rc) rc = cuda_check(cudaMemcpy(&fault, dfault, sizeof(int), cudaMemcpyDeviceToHost), "forward_tc");
  if (dimg) cudaFree(dimg);
  if (dfault) cudaFree(dfault);
  if (!rc && fault) {
    fprintf(stderr, "[mgpu] forward_tc: a tensor-core wait timed out\n");
    rc = MGPU_ERR_CUDA;
  }
  return rc;
}

int mgpu_mlp_forward(const float *dev_params, const float *dev_x, long long n, float *dev_y)
{
  if (!dev_params || !dev_x || !dev_y || n <= 0) return MGPU_ERR_ARG;
  k_forward<<<(unsigned) ((n + 127) / 128), 128>>>(dev_params, dev_x, n, dev_y);
  int rc = cuda_check(cudaGetLastError(), "forward");
  if (rc) return rc;
  return cuda_check(cudaDeviceSynchronize(), "forward");
}

}  // extern "C"
