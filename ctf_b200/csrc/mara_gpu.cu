// Host side of libmaragpu.so: the solver handle, device buffers, transfers, measures and the
// C ABI declared in include/mara_gpu.h.  Kernels live in kernels_fp64.cu (compiled with
// --fmad=false) and kernels_fp32.cu.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <chrono>
#include <string>
#include <vector>
#include <utility>

#include "../../include/mara_gpu.h"
#include "rmhd_types.cuh"

MGPU_DECLARE_PRECISION(fp64)
MGPU_DECLARE_PRECISION(fp32)

using namespace mgpu;

#include "solver.h"
#include "host_copy.h"
#include "measures.h"

namespace {

constexpr int RED_BLOCKS = 1184;   // 148 SMs x 8

int fail(mgpu_solver *h, int code, const std::string &msg)
{
  if (h) h->err = msg;
  return code;
}

int cuda_fail(mgpu_solver *h, cudaError_t e, const char *where)
{
  return fail(h, MGPU_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                               \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return cuda_fail(h, e_, #call);     \
  } while (0)

bool fp32(const mgpu_solver *h) { return h->cfg.precision == MGPU_PREC_FP32; }
bool lean(const mgpu_solver *h) { return h->cfg.layout == MGPU_LAYOUT_LEAN; }

PhysParams phys(const mgpu_solver *h)
{
  PhysParams p;
  p.gamma = h->cfg.gamma;
  p.pfloor = h->cfg.pfloor;
  p.theta = h->cfg.theta;
  p.sz10A = h->cfg.sz10A;
  p.is_mode = h->cfg.is_mode;
  p.recon = h->cfg.recon;
  p.riemann = h->cfg.riemann;
  p.learned = h->cfg.learned_c2p && h->mlp != nullptr;
  p.learned_faces = 0;
  p.mlp = h->mlp;
  p.mlp_tc = h->mlp_tc;
  return p;
}

// The pipelined host advance's buffers (allocated on its first use for the current domain).
void pipe_free(mgpu_solver *h, bool streams)
{
  if (h->pipe_in) cudaFree(h->pipe_in);
  if (h->pipe_out) cudaFree(h->pipe_out);
  if (h->pipe_guess) cudaFree(h->pipe_guess);
  if (h->pipe_pa) cudaFree(h->pipe_pa);
  h->pipe_in = h->pipe_out = nullptr;
  h->pipe_guess = h->pipe_pa = nullptr;
  h->pipe_state = 0;
  if (h->pipe_host) cudaFreeHost(h->pipe_host);
  h->pipe_host = nullptr;
  h->pipe_host_state = 0;
  if (h->xfer_host) cudaFreeHost(h->xfer_host);
  h->xfer_host = nullptr;
  h->xfer_host_state = 0;
  if (!streams) return;
  for (cudaEvent_t e : h->pipe_ev) cudaEventDestroy(e);
  h->pipe_ev.clear();
  delete h->pipe_pool;
  h->pipe_pool = nullptr;
  for (cudaEvent_t e : h->xfer_ev) cudaEventDestroy(e);
  h->xfer_ev.clear();
  if (h->pipe_h2d) cudaStreamDestroy(h->pipe_h2d);
  if (h->pipe_d2h) cudaStreamDestroy(h->pipe_d2h);
  h->pipe_h2d = h->pipe_d2h = nullptr;
}

void free_buffers(mgpu_solver *h)
{
  pipe_free(h, false);
  for (void *p : h->allocations) cudaFree(p);
  h->allocations.clear();
  h->b = AdvanceBuffers{};
  h->staging = nullptr;
  h->red = nullptr;
  h->meas = nullptr;
  h->fmask = nullptr;
}

cudaError_t dalloc(mgpu_solver *h, void **p, size_t bytes)
{
  cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaSuccess) {
    h->allocations.push_back(*p);
    e = cudaMemsetAsync(*p, 0, bytes, h->stream);
  }
  return e;
}

TransferArgs transfer_args(mgpu_solver *h)
{
  TransferArgs t;
  t.g = h->g;
  t.b = h->b;
  t.ctl = h->ctl;
  t.stream = h->stream;
  t.cur = 0;
  t.lean = lean(h);
  t.gamma = h->cfg.gamma;
  return t;
}

int ensure_ready(mgpu_solver *h)
{
  if (!h) return MGPU_ERR_ARG;
  if (!h->have_domain) return fail(h, MGPU_ERR_STATE, "need a domain to run this, use set_domain");
  return MGPU_OK;
}

// ---- measures (Mara/mara.cpp:2232-2324) on an 8 x T face array ------------------------------
template <class T>
__device__ __forceinline__ void k_divB_body(Grid g, const T *P, double *partial);

template <class T>
__global__ void k_divB(Grid g, const T *P, double *partial)
{
  k_divB_body<T>(g, P, partial);
}

template <class T>
__device__ __forceinline__ void k_divB_body(Grid g, const T *P, double *partial)
{
  // corner-centred divergence over i in [ng, G0-ng-1) etc. (interior corners but the last)
  const int ng = g.ng;
  const long long ni = g.G[0] - 2 * ng - 1;
  const long long nj = g.nd >= 2 ? g.G[1] - 2 * ng - 1 : 1;
  const long long nk = g.nd >= 3 ? g.G[2] - 2 * ng - 1 : 1;
  const long long total = (ni > 0 && nj > 0 && nk > 0) ? ni * nj * nk : 0;
  double sum = 0.0, mx = -INFINITY;
  for (long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long) gridDim.x * blockDim.x) {
    const int i = ng + (int) (t / (nj * nk));
    const int j = (g.nd >= 2 ? ng : 0) + (int) ((t / nk) % nj);
    const int k = (g.nd >= 3 ? ng : 0) + (int) (t % nk);
    auto B = [&](int q, int a, int b, int c) {
      return double(P[(long long) q * g.cs + ((long long) a * g.G[1] + b) * g.G[2] + c]);
    };
    double d;
    if (g.nd == 2) {
      d = (B(5, i + 1, j, 0) + B(5, i + 1, j + 1, 0) - B(5, i, j, 0) - B(5, i, j + 1, 0)) / 2.0 +
          (B(6, i, j + 1, 0) + B(6, i + 1, j + 1, 0) - B(6, i, j, 0) - B(6, i + 1, j, 0)) / 2.0;
    } else {
      d = ((B(5, i + 1, j, k) + B(5, i + 1, j + 1, k) + B(5, i + 1, j, k + 1) + B(5, i + 1, j + 1, k + 1)) -
           (B(5, i, j, k) + B(5, i, j + 1, k) + B(5, i, j, k + 1) + B(5, i, j + 1, k + 1))) / 4.0 +
          ((B(6, i, j + 1, k) + B(6, i, j + 1, k + 1) + B(6, i + 1, j + 1, k) + B(6, i + 1, j + 1, k + 1)) -
           (B(6, i, j, k) + B(6, i, j, k + 1) + B(6, i + 1, j, k) + B(6, i + 1, j, k + 1))) / 4.0 +
          ((B(7, i, j, k + 1) + B(7, i + 1, j, k + 1) + B(7, i, j + 1, k + 1) + B(7, i + 1, j + 1, k + 1)) -
           (B(7, i, j, k) + B(7, i + 1, j, k) + B(7, i, j + 1, k) + B(7, i + 1, j + 1, k))) / 4.0;
    }
    sum += d;
    mx = fmax(mx, d);
  }
  __shared__ double ss[256], sm[256];
  ss[threadIdx.x] = sum;
  sm[threadIdx.x] = mx;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      ss[threadIdx.x] += ss[threadIdx.x + o];
      sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = ss[0];
    partial[2 * blockIdx.x + 1] = sm[0];
  }
}

// Corner divergence of a state's FP64 magnetic field (components 5..7 at B + (q-5)*cs).
__global__ void k_divB_state(Grid g, const double *B, double *partial)
{
  // k_divB reads P[q*cs + z] for q = 5..7: shift the base so that q = 5 lands on B[0].
  k_divB_body<double>(g, B - 5 * g.cs, partial);
}

template <class T>
__global__ void k_wmax(Grid g, const T *P, double *partial)
{
  double mx = 0.0;
  for (long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x; t < g.ninterior;
       t += (long long) gridDim.x * blockDim.x) {
    int i, j, k;
    interior_coords(g, t, i, j, k);
    const long long z = ((long long) i * g.G[1] + j) * g.G[2] + k;
    const double v0 = double(P[2 * g.cs + z]), v1 = double(P[3 * g.cs + z]), v2 = double(P[4 * g.cs + z]);
    const double W0 = 1.0 / sqrt(1.0 - (v0 * v0 + v1 * v1 + v2 * v2));
    mx = fmax(mx, W0);
  }
  __shared__ double sm[256];
  sm[threadIdx.x] = mx;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sm[0];
}

}  // namespace

static void prof_free(mgpu_solver *h)
{
  for (cudaEvent_t e : h->prof_ev) cudaEventDestroy(e);
  h->prof_ev.clear();
  h->prof_tag.clear();
  h->prof_units.clear();
  h->prof_on = false;
}


extern "C" {

int mgpu_default_config(mgpu_config *c)
{
  if (!c) return MGPU_ERR_ARG;
  memset(c, 0, sizeof(*c));
  c->fluid = MGPU_FLUID_RMHD;
  c->gamma = 4.0 / 3.0;
  c->recon = MGPU_RECON_PLM;
  c->theta = 2.0;
  c->is_mode = MGPU_IS_JS96;
  c->sz10A = 50.0;
  c->riemann = MGPU_RIEMANN_HLLD;
  c->rk = 2;
  c->pfloor = -1.0;
  c->ereset = 0;
  c->preset = 1.0;
  c->dreset = 1.0;
  c->precision = MGPU_PREC_FP64;
  c->learned_c2p = 0;
  c->godunov = MGPU_GODUNOV_PLM_SPLIT;
  c->layout = MGPU_LAYOUT_STANDARD;
  return MGPU_OK;
}

static int check_config(mgpu_solver *h, const mgpu_config *c)
{
  if (c->fluid != MGPU_FLUID_RMHD) return fail(h, MGPU_ERR_UNSUPPORTED, "only the 'rmhd' fluid is provided");
  if (!(c->gamma > 1.0)) return fail(h, MGPU_ERR_ARG, "gamma-law index must exceed 1");
  if (c->recon < 0 || c->recon > 2) return fail(h, MGPU_ERR_ARG, "no such extrap");
  if (c->riemann < 0 || c->riemann > 2) return fail(h, MGPU_ERR_ARG, "no such riemann solver");
  if (c->rk < 1 || c->rk > 4) return fail(h, MGPU_ERR_ARG, "no such advance option");
  if (c->is_mode < 0 || c->is_mode > 2) return fail(h, MGPU_ERR_ARG, "no such IS");
  if (c->precision != MGPU_PREC_FP64 && c->precision != MGPU_PREC_FP32)
    return fail(h, MGPU_ERR_ARG, "no such precision");
  if (c->godunov != MGPU_GODUNOV_PLM_SPLIT && c->godunov != MGPU_GODUNOV_PLM_MUSCL)
    return fail(h, MGPU_ERR_ARG, "no such integration scheme");
  if (c->layout != MGPU_LAYOUT_STANDARD && c->layout != MGPU_LAYOUT_LEAN) return fail(h, MGPU_ERR_ARG, "no such layout");
  if (c->layout == MGPU_LAYOUT_LEAN && (c->godunov != MGPU_GODUNOV_PLM_SPLIT || c->rk > 3))
    return fail(h, MGPU_ERR_UNSUPPORTED, "the lean layout runs 'plm-split' with single, rk2 or rk3");
  return MGPU_OK;
}

int mgpu_create(const mgpu_config *cfg, mgpu_solver **out)
{
  if (!out) return MGPU_ERR_ARG;
  *out = nullptr;
  mgpu_solver *h = new mgpu_solver;
  if (cfg) h->cfg = *cfg;
  else mgpu_default_config(&h->cfg);
  int rc = check_config(h, &h->cfg);
  if (rc) {
    fprintf(stderr, "[mgpu] %s\n", h->err.c_str());
    delete h;
    return rc;
  }
  cudaError_t e = cudaGetDevice(&h->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc((void **) &h->ctl, sizeof(Ctl));
  if (e == cudaSuccess) e = cudaMemset(h->ctl, 0, sizeof(Ctl));
  if (e == cudaSuccess) e = cudaMallocHost((void **) &h->ctl_host, sizeof(Ctl));
  if (e == cudaSuccess) e = cudaMallocHost((void **) &h->red_host, sizeof(double) * 2 * RED_BLOCKS);
  if (e == cudaSuccess) e = cudaMallocHost((void **) &h->meas_host, sizeof(double) * MEAS_BLOCKS * MEAS_FIELDS);
  if (e != cudaSuccess) {
    fprintf(stderr, "[mgpu] CUDA unavailable: %s\n", cudaGetErrorString(e));
    if (h->stream) cudaStreamDestroy(h->stream);
    if (h->ctl) cudaFree(h->ctl);
    if (h->ctl_host) cudaFreeHost(h->ctl_host);
    if (h->red_host) cudaFreeHost(h->red_host);
    delete h;
    return MGPU_ERR_CUDA;
  }
  h->own_stream = true;
  *out = h;
  return MGPU_OK;
}

int mgpu_destroy(mgpu_solver *h)
{
  if (!h) return MGPU_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  mgpu_driving_free(h);
  free_buffers(h);
  pipe_free(h, true);
  prof_free(h);
  if (h->mlp) cudaFree(h->mlp);
  if (h->mlp_tc) cudaFree(h->mlp_tc);
  if (h->mult) cudaFree(h->mult);
  if (h->ctl) cudaFree(h->ctl);
  if (h->ctl_host) cudaFreeHost(h->ctl_host);
  if (h->red_host) cudaFreeHost(h->red_host);
  if (h->meas_host) cudaFreeHost(h->meas_host);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return MGPU_OK;
}

int mgpu_set_stream(mgpu_solver *h, void *stream)
{
  if (!h) return MGPU_ERR_ARG;
  CK(cudaStreamSynchronize(h->stream));
  if (h->own_stream) cudaStreamDestroy(h->stream);
  if (stream) {
    h->stream = (cudaStream_t) stream;
    h->own_stream = false;
  } else {
    CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
  }
  return MGPU_OK;
}

const char *mgpu_last_error(const mgpu_solver *h) { return h ? h->err.c_str() : "null handle"; }

int mgpu_set_domain(mgpu_solver *h, const double *x0, const double *x1, const int *N, int nd, int nq, int ng)
{
  if (!h || !x0 || !x1 || !N) return MGPU_ERR_ARG;
  if (nd < 1 || nd > 3) return fail(h, MGPU_ERR_ARG, "domain must have 1, 2 or 3 dimensions");
  if (nq != 8) return fail(h, MGPU_ERR_ARG, "the rmhd fluid has Nq = 8");
  if (ng < 3) return fail(h, MGPU_ERR_ARG, "the step's stencils need Ng >= 3");
  for (int d = 0; d < nd; ++d)
    if (N[d] < ng) return fail(h, MGPU_ERR_ARG, "periodic guard fill needs N >= Ng on every axis");
  if (lean(h) && nd != 3) return fail(h, MGPU_ERR_UNSUPPORTED, "the lean layout is for 3D boxes");
  CK(cudaStreamSynchronize(h->stream));
  free_buffers(h);
  mgpu_driving_free(h);
  if (h->mult) cudaFree(h->mult);
  h->mult = nullptr;
  h->have_domain = false;
  Grid &g = h->g;
  g = Grid{};
  g.nd = nd;
  g.ng = ng;
  for (int d = 0; d < 3; ++d) {
    h->N[d] = d < nd ? N[d] : 1;
    h->x0[d] = d < nd ? x0[d] : 0.0;
    h->x1[d] = d < nd ? x1[d] : 1.0;
    g.n[d] = h->N[d];
    g.G[d] = d < nd ? N[d] + 2 * ng : 1;
  }
  g.nz = (long long) g.G[0] * g.G[1] * g.G[2];
  g.cs = (g.nz + 31) / 32 * 32;
  g.s[0] = (long long) g.G[1] * g.G[2];
  g.s[1] = g.G[2];
  g.s[2] = 1;
  // GodunovOperator::prepare_integration (Mara/hydro.cpp:80-110)
  double dd[3];
  for (int d = 0; d < 3; ++d) dd[d] = (h->x1[d] - h->x0[d]) / (g.G[d] - 2 * ng);
  g.dx = dd[0];
  g.dy = dd[1];
  g.dz = dd[2];
  g.ninterior = (long long) g.n[0] * g.n[1] * g.n[2];
  // SimpleCartesianDomain min_dx (Mara/simple-cart.cpp:20-24)
  h->min_dx = h->x1[0] - h->x0[0];
  for (int d = 0; d < nd; ++d) {
    const double dx = (h->x1[d] - h->x0[d]) / h->N[d];
    if (dx < h->min_dx) h->min_dx = dx;
  }

  const size_t tsz = fp32(h) ? sizeof(float) : sizeof(double);
  const size_t cs = (size_t) g.cs;
  auto state = [&](void **bulk, double **B) -> cudaError_t {
    cudaError_t e = dalloc(h, bulk, 5 * cs * tsz);
    if (e == cudaSuccess) e = dalloc(h, (void **) B, 3 * cs * sizeof(double));
    return e;
  };
  cudaError_t e = cudaSuccess;
  // lean layout: PA, the two conserved registers and the six transverse face fields only
  for (int i = 0; i < 2 && e == cudaSuccess && !lean(h); ++i) e = state(&h->b.Pc_bulk[i], &h->b.Pc_B[i]);
  if (e == cudaSuccess) e = state(&h->b.U0_bulk, &h->b.U0_B);
  if (e == cudaSuccess) e = state(&h->b.U1_bulk, &h->b.U1_B);
  if (h->cfg.rk == 4)
    for (int i = 0; i < 3 && e == cudaSuccess; ++i) e = state(&h->b.K_bulk[i], &h->b.K_B[i]);
  if (e == cudaSuccess) e = dalloc(h, &h->b.PA, 8 * cs * tsz);
  for (int d = 0; d < 3 && e == cudaSuccess && !lean(h); ++d) {
    if (d < nd) e = dalloc(h, &h->b.F[d], 8 * cs * tsz);
    else h->b.F[d] = h->b.F[0];
  }
  if (e == cudaSuccess && lean(h)) e = dalloc(h, &h->b.Bf, 6 * cs * tsz);
  // CTU-Hancock: predicted primitives of each direction
  for (int d = 0; d < 3 && e == cudaSuccess && h->cfg.godunov == MGPU_GODUNOV_PLM_MUSCL; ++d) {
    if (d < nd) e = dalloc(h, &h->b.Pd[d], 8 * cs * tsz);
    else h->b.Pd[d] = h->b.Pd[0];
  }
  h->staging_zones = g.nz < (1ll << 22) ? g.nz : (1ll << 22);   // up to 256 MB of AoS
  if (e == cudaSuccess) e = dalloc(h, (void **) &h->staging, (size_t) h->staging_zones * 8 * sizeof(double));
  if (e == cudaSuccess) e = dalloc(h, (void **) &h->red, sizeof(double) * 2 * RED_BLOCKS);
  if (e == cudaSuccess) e = dalloc(h, (void **) &h->meas, sizeof(double) * MEAS_BLOCKS * MEAS_FIELDS);
  // the failure mask of the last c2p (one byte per guarded zone; not kept in the lean layout,
  // whose Mara.diffuse is not offered)
  h->fmask = nullptr;
  if (e == cudaSuccess && !lean(h)) e = dalloc(h, (void **) &h->fmask, (size_t) g.nz);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->ctl, 0, sizeof(Ctl), h->stream);
  if (e == cudaSuccess && h->fmask)
    e = cudaMemcpyAsync(&h->ctl->fmask, &h->fmask, sizeof(h->fmask), cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    free_buffers(h);
    cudaGetLastError();
    return fail(h, e == cudaErrorMemoryAllocation ? MGPU_ERR_NOMEM : MGPU_ERR_CUDA,
                std::string("set_domain: ") + cudaGetErrorString(e));
  }
  h->have_domain = true;
  return MGPU_OK;
}

int mgpu_num_zones(const mgpu_solver *h, long long *nz)
{
  if (!h || !nz) return MGPU_ERR_ARG;
  if (!h->have_domain) return MGPU_ERR_STATE;
  *nz = h->g.nz;
  return MGPU_OK;
}

static bool pipe_host_setup(mgpu_solver *h);

// Two pinned slots of the device staging chunk's size and two events, for the chunked host
// transfers of a large pageable buffer, and the copy threads; false when they cannot be had
// (the copies then read and write the pageable buffer directly).
static bool xfer_host_setup(mgpu_solver *h)
{
  if (h->xfer_host_state == 0) {
    cudaError_t e = cudaHostAlloc((void **) &h->xfer_host, (size_t) h->staging_zones * 2 * 8 * sizeof(double),
                                  cudaHostAllocDefault);
    while (h->xfer_ev.size() < 2 && e == cudaSuccess) {   // the events outlive a new domain
      cudaEvent_t ev;
      e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
      if (e == cudaSuccess) h->xfer_ev.push_back(ev);
    }
    if (e != cudaSuccess) {
      cudaGetLastError();
      if (h->xfer_host) cudaFreeHost(h->xfer_host);
      h->xfer_host = nullptr;
      h->xfer_host_state = -1;
      return false;
    }
    h->xfer_host_state = 1;
  }
  if (h->xfer_host_state < 0) return false;
  if (!h->pipe_pool) {
    const unsigned hc = std::thread::hardware_concurrency();
    h->pipe_pool = new HostCopyPool(hc >= 16 ? 8 : (hc >= 2 ? (int) hc / 2 : 1));
  }
  return true;
}

static int transfer(mgpu_solver *h, double *host, const void *dev_in, void *dev_out, int kind, long long zbeg = 0,
                    long long zcount = -1)
{
  // kind 0: upload committed state, 1: download committed state, 2: upload PA, 3: download PA;
  // zones [zbeg, zbeg + zcount) of the guarded array (all of it when zcount < 0), host[0] being
  // zone zbeg
  int rc = ensure_ready(h);
  if (rc) return rc;
  // the lean layout's stage array holds the committed primitives: setting the measured array
  // is an upload of the committed state there (Mara.advance(buf) uploads it again anyway)
  if (lean(h) && kind >= 2) kind -= 2;
  const TransferArgs t = transfer_args(h);
  if (zcount < 0) zcount = h->g.nz - zbeg;
  if (zbeg < 0 || zbeg + zcount > h->g.nz) return fail(h, MGPU_ERR_ARG, "zone range outside the guarded array");
  const long long nz = zbeg + zcount;
  host -= zbeg * 8;
  const bool upload = kind == 0 || kind == 2;
  if (dev_in || dev_out) {
    double *d = (double *) (dev_in ? const_cast<void *>(dev_in) : dev_out);
    cudaError_t e;
    if (kind == 0) e = fp32(h) ? upload_fp32(t, d, 0, nz) : upload_fp64(t, d, 0, nz);
    else if (kind == 1) e = fp32(h) ? download_fp32(t, d, 0, nz) : download_fp64(t, d, 0, nz);
    else e = fp32(h) ? face_io_fp32(t, d, 0, nz, kind == 3) : face_io_fp64(t, d, 0, nz, kind == 3);
    (void) host;
    CK(e);
    CK(cudaStreamSynchronize(h->stream));
    return MGPU_OK;
  }
  // a large pageable buffer goes through two pinned chunk slots (xfer_host), chunk by chunk:
  // the threaded host copy of one chunk overlaps the DMA copy and conversion of the other
  bool staged = false;
  if ((size_t) (nz - zbeg) * 8 * sizeof(double) >= (size_t(64) << 20)) {
    cudaPointerAttributes pa{};
    const bool pinned = cudaPointerGetAttributes(&pa, host + zbeg * 8) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();   // an unregistered pointer may leave an error behind
    staged = !pinned && xfer_host_setup(h);
  }
  const long long slot_doubles = h->staging_zones * 8;
  auto slot = [&](int c) { return h->xfer_host + (c % 2) * slot_doubles; };
  int nchunk = 0;
  for (long long z0 = zbeg; z0 < nz; z0 += h->staging_zones) {
    const long long cnt = (nz - z0) < h->staging_zones ? (nz - z0) : h->staging_zones;
    const size_t bytes = (size_t) cnt * 8 * sizeof(double);
    double *dma = staged ? slot(nchunk) : host + z0 * 8;   // where this chunk's DMA copy reads or writes
    if (upload) {
      if (staged) {
        if (nchunk >= 2) CK(cudaEventSynchronize(h->xfer_ev[nchunk % 2]));   // the slot's previous copy
        h->pipe_pool->copy(dma, host + z0 * 8, bytes);
      }
      CK(cudaMemcpyAsync(h->staging, dma, bytes, cudaMemcpyHostToDevice, h->stream));
      if (staged) CK(cudaEventRecord(h->xfer_ev[nchunk % 2], h->stream));
      cudaError_t e = kind == 0 ? (fp32(h) ? upload_fp32(t, h->staging, z0, cnt) : upload_fp64(t, h->staging, z0, cnt))
                                : (fp32(h) ? face_io_fp32(t, h->staging, z0, cnt, 0)
                                           : face_io_fp64(t, h->staging, z0, cnt, 0));
      CK(e);
    } else {
      cudaError_t e = kind == 1 ? (fp32(h) ? download_fp32(t, h->staging, z0, cnt)
                                           : download_fp64(t, h->staging, z0, cnt))
                                : (fp32(h) ? face_io_fp32(t, h->staging, z0, cnt, 1)
                                           : face_io_fp64(t, h->staging, z0, cnt, 1));
      CK(e);
      CK(cudaMemcpyAsync(dma, h->staging, bytes, cudaMemcpyDeviceToHost, h->stream));
      if (staged) {
        CK(cudaEventRecord(h->xfer_ev[nchunk % 2], h->stream));
        if (nchunk >= 1) {   // the previous chunk, from its slot into the caller's buffer
          const long long zp = z0 - h->staging_zones;
          CK(cudaEventSynchronize(h->xfer_ev[(nchunk - 1) % 2]));
          h->pipe_pool->copy(host + zp * 8, slot(nchunk - 1), (size_t) h->staging_zones * 8 * sizeof(double));
        }
      }
    }
    ++nchunk;
  }
  if (staged && !upload && nchunk >= 1) {   // the last chunk
    const long long zl = zbeg + (long long) (nchunk - 1) * h->staging_zones;
    CK(cudaEventSynchronize(h->xfer_ev[(nchunk - 1) % 2]));
    h->pipe_pool->copy(host + zl * 8, slot(nchunk - 1), (size_t) (nz - zl) * 8 * sizeof(double));
  }
  CK(cudaStreamSynchronize(h->stream));
  return MGPU_OK;
}

int mgpu_upload_prim(mgpu_solver *h, const double *host_aos)
{
  if (!host_aos) return fail(h, MGPU_ERR_ARG, "null primitive buffer");
  return transfer(h, const_cast<double *>(host_aos), nullptr, nullptr, 0);
}
int mgpu_download_prim(mgpu_solver *h, double *host_aos)
{
  if (!host_aos) return fail(h, MGPU_ERR_ARG, "null primitive buffer");
  return transfer(h, host_aos, nullptr, nullptr, 1);
}
int mgpu_upload_prim_device(mgpu_solver *h, const void *dev_aos)
{
  if (!dev_aos) return fail(h, MGPU_ERR_ARG, "null primitive buffer");
  return transfer(h, nullptr, dev_aos, nullptr, 0);
}
int mgpu_download_prim_device(mgpu_solver *h, void *dev_aos)
{
  if (!dev_aos) return fail(h, MGPU_ERR_ARG, "null primitive buffer");
  return transfer(h, nullptr, nullptr, dev_aos, 1);
}
int mgpu_upload_prim_range(mgpu_solver *h, const double *host_aos, long long z0, long long count)
{
  if (!host_aos || count < 0) return fail(h, MGPU_ERR_ARG, "bad primitive range");
  return transfer(h, const_cast<double *>(host_aos), nullptr, nullptr, 0, z0, count);
}
int mgpu_download_prim_range(mgpu_solver *h, double *host_aos, long long z0, long long count)
{
  if (!host_aos || count < 0) return fail(h, MGPU_ERR_ARG, "bad primitive range");
  return transfer(h, host_aos, nullptr, nullptr, 1, z0, count);
}
int mgpu_set_primitive(mgpu_solver *h, const double *host_aos)
{
  if (!host_aos) return fail(h, MGPU_ERR_ARG, "null primitive buffer");
  return transfer(h, const_cast<double *>(host_aos), nullptr, nullptr, 2);
}

static AdvanceArgs advance_args(mgpu_solver *h, int dt_mode, double dt, double cfl)
{
  AdvanceArgs A;
  A.g = h->g;
  A.pp = phys(h);
  A.rk = h->cfg.rk;
  A.godunov = h->cfg.godunov;
  A.lean = lean(h);
  A.ereset = h->cfg.ereset;
  A.preset = h->cfg.preset;
  A.dreset = h->cfg.dreset;
  A.dt_mode = dt_mode;
  A.dt = dt;
  A.cfl = cfl;
  A.min_dx = h->min_dx;
  A.b = h->b;
  A.ctl = h->ctl;
  A.stream = h->stream;
  A.prof = h->prof_on ? &h->prof : nullptr;
  return A;
}

static int enqueue_advance(mgpu_solver *h, int dt_mode, double dt, double cfl)
{
  const AdvanceArgs A = advance_args(h, dt_mode, dt, cfl);
  cudaError_t e = fp32(h) ? advance_fp32(A) : advance_fp64(A);
  CK(e);
  CK(mgpu_driving_enqueue(h));
  return MGPU_OK;
}

static int read_ctl(mgpu_solver *h)
{
  CK(cudaMemcpyAsync(h->ctl_host, h->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return MGPU_OK;
}

static int errors_of(const Ctl &c, int rk)
{
  const int ns = num_stages(rk);
  for (int s = 0; s < ns; ++s)
    if (c.stage_err[s]) return c.stage_err[s];
  return c.final_err;
}

int mgpu_advance(mgpu_solver *h, double dt, int *errors)
{
  int rc = ensure_ready(h);
  if (rc) return rc;
  rc = enqueue_advance(h, 0, dt, 0.0);
  if (rc) return rc;
  rc = read_ctl(h);
  if (rc) return rc;
  if (h->ctl_host->tc_fault) return fail(h, MGPU_ERR_CUDA, "a tensor-core wait of the learned c2p timed out");
  if (errors) *errors = errors_of(*h->ctl_host, h->cfg.rk);
  return MGPU_OK;
}

// ---- the pipelined Mara.advance(buf, dt) of the lean layout -------------------------------------
// The box is cut into S slabs of x rows.  The operations of one advance on a slab are
//   e = 0        upload: the copy in of its rows, then k_lean_upload (P->U into the committed
//                register, the primitives into PA)
//   e = 2k + 1   stage k's sweeps and CT over the slab (k = 0 .. K-1)
//   e = 2k       stage k's c2p over the slab (k = 1 .. K-1), e = 2K the closing c2p
//   e = 2K + 1   download: the result into the device copy-out buffer, then the copy out.
// The stages' primitives alternate between two arrays (the solver's PA and a second one), so
// that a c2p never overwrites primitives a neighbour's sweeps still read.  A slab's sweeps
// (e odd) may run once the operation before them has run on the slab and on both neighbouring
// slabs (periodic in x: slab 0's images lie next to slab S-1), because they read the
// neighbours' stage primitives up to three rows deep; a c2p or a download needs only the
// slab's own previous operation.  CT reads y and z face fields one row beyond the slab: the
// same operation's sweeps compute those halo rows, except the one next to the neighbour
// toward slab 0 (pipe_pred), whose sweeps of the same stage computed it as their own row and
// run first.  Each window launch computes exactly the faces and zones of the
// whole-box launch that fall in it, so the result is the whole-box advance's.
// The slabs are uploaded outward from slab 0 in both directions, so that slab 0's neighbourhood
// arrives first; after each upload the compute stream takes every operation that became ready,
// the latest first.  The copies run on their own streams, so the copy in of later slabs and the
// copy out of earlier ones overlap the advance.  With a pinned caller buffer the copies out
// write it before the advance is known to commit; its original contents stay in the device
// copy-in buffer and go back when the advance does not commit.  A pageable buffer goes through
// a pinned copy of the AoS buffer (pipe_host_setup) with the same schedule, the pool's threads
// copying each slab's rows in before its copy in and its result out as its copy out lands;
// without that pinned copy it is written after the commit only (copies of pageable memory
// would block the host thread).

#ifndef MGPU_PIPE_THIN
#define MGPU_PIPE_THIN 6     // rows of the thin slabs of the automatic layout
#endif
#ifndef MGPU_PIPE_THICK
#define MGPU_PIPE_THICK 16   // rows of the others
#endif

// Slab boundaries of the pipelined host advance over n0 interior x rows: wb[0..S] (slab s is
// rows [wb[s], wb[s+1])), or nothing when n0 is too small (at least 3 slabs of 4 rows, deeper
// than any stencil's reach).  slabs > 0: that many equal slabs.  Automatic (-1): below 96 rows,
// slabs of about 11 rows; from 96 rows, slabs of 16 rows except thin ones of 6 rows around slab
// 0 and around the far side uploaded last.  The thin slabs start the pipeline after fewer rows
// have arrived and shorten the work and the copies out that follow the last copy in; the thick
// ones recompute fewer halo rows of face fields.
static std::vector<int> pipe_bounds(int n0, int slabs)
{
  std::vector<int> wb;
  const int smax = n0 / 4;
  if (smax < 3) return wb;
  if (slabs > 0 || n0 < 96) {
    int S = slabs > 0 ? slabs : n0 / 11;
    S = S < 3 ? 3 : (S > smax ? smax : S);
    for (int s = 0; s <= S; ++s) wb.push_back((int) ((long long) n0 * s / S));
    return wb;
  }
  const int thin_w = MGPU_PIPE_THIN, thick_w = MGPU_PIPE_THICK;
  auto thin = [](int S, int s) {
    const int d = s < S - s ? s : S - s;   // ring distance from slab 0
    return d <= 1 || d >= S / 2 - 3;
  };
  auto total = [&](int S) {
    int t = 0;
    for (int s = 0; s < S; ++s) t += thin(S, s) ? thin_w : thick_w;
    return t;
  };
  int S = 3;
  while (total(S + 1) <= n0) ++S;
  std::vector<int> w(S);
  int nthick = 0;
  for (int s = 0; s < S; ++s) {
    w[s] = thin(S, s) ? thin_w : thick_w;
    nthick += !thin(S, s);
  }
  for (int rem = n0 - total(S), s = 0; rem > 0; s = (s + 1) % S)   // the rows left over
    if (!thin(S, s) || nthick == 0) {
      ++w[s];
      --rem;
    }
  wb.push_back(0);
  for (int s = 0; s < S; ++s) wb.push_back(wb.back() + w[s]);
  return wb;
}

// Slab boundaries for this solver's pipelined host advance (empty: run unpipelined).
static std::vector<int> pipe_slab_bounds(const mgpu_solver *h)
{
  const Grid &g = h->g;
  if (h->pipe_slabs == 0 || !lean(h) || g.nd != 3 || g.ext[0] || g.ext[1] || g.ext[2] || h->driving ||
      h->prof_on)
    return {};
  return pipe_bounds(g.n[0], h->pipe_slabs);
}

// Device buffers, streams and events of the pipeline; 1 when device memory does not allow it.
static int pipe_setup(mgpu_solver *h, int S)
{
  const Grid &g = h->g;
  const bool learned = phys(h).learned && h->mlp_tc;
  if (h->pipe_state == 0) {
    const size_t aos = (size_t) g.nz * 8 * sizeof(double);
    const size_t guess = learned ? (size_t) g.ninterior * sizeof(float2) : 0;
    const size_t pa = (size_t) g.cs * 8 * (fp32(h) ? sizeof(float) : sizeof(double));
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    if (free_b < 2 * aos + pa + guess + (size_t(1) << 30)) {
      h->pipe_state = -1;
      return 1;
    }
    cudaError_t e = cudaMalloc((void **) &h->pipe_in, aos);
    if (e == cudaSuccess) e = cudaMalloc((void **) &h->pipe_out, aos);
    if (e == cudaSuccess) e = cudaMalloc(&h->pipe_pa, pa);
    if (e == cudaSuccess && guess) e = cudaMalloc(&h->pipe_guess, guess);
    if (e != cudaSuccess) {
      cudaGetLastError();
      pipe_free(h, false);
      h->pipe_state = -1;
      return 1;
    }
    h->pipe_state = 1;
  }
  if (h->pipe_state < 0) return 1;
  if (learned && !h->pipe_guess) {   // the learned c2p was switched on after the setup
    if (cudaMalloc(&h->pipe_guess, (size_t) g.ninterior * sizeof(float2)) != cudaSuccess) {
      cudaGetLastError();
      return 1;
    }
  }
  if (!h->pipe_h2d) CK(cudaStreamCreateWithFlags(&h->pipe_h2d, cudaStreamNonBlocking));
  if (!h->pipe_d2h) CK(cudaStreamCreateWithFlags(&h->pipe_d2h, cudaStreamNonBlocking));
  while ((int) h->pipe_ev.size() < 3 * S) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    h->pipe_ev.push_back(e);
  }
  return 0;
}

// The neighbour whose sweeps a slab's sweeps wait for, so as to reuse the y and z face fields
// of the halo row they computed as their own (-1: none, the slab computes both halo rows).  The
// slabs on either side of slab 0, uploaded outward from it, take the one toward slab 0; slab 0
// and slab S-1 compute both (their outer halo rows are guard rows no other slab computes).
static int pipe_pred(int S, int s)
{
  if (s >= 1 && s <= S / 2) return s - 1;
  if (s > S / 2 && s <= S - 2) return s + 1;
  return -1;
}

// Grid::whskip of a slab's sweeps: the halo row its pipe_pred neighbour computes.
static int pipe_whskip(int S, int s)
{
  const int p = pipe_pred(S, s);
  return p < 0 ? 0 : (p == s - 1 ? 1 : 2);
}

// The order in which the pipelined advance issues its operations: (slab, operation) pairs,
// the uploads included, for S slabs and K Runge-Kutta stages.
static std::vector<std::pair<int, int>> pipe_schedule(int S, int K)
{
  const int E = 2 * K + 2;   // operations per slab
  std::vector<std::pair<int, int>> out;
  std::vector<int> order, done(S, 0);
  order.push_back(0);
  for (int d = 1; (int) order.size() < S; ++d) {
    order.push_back(d);
    if ((int) order.size() < S) order.push_back(S - d);
  }
  auto ready = [&](int s, int e) {
    if (done[s] != e) return false;
    if (e % 2 == 0 || e == E - 1) return true;
    const int p = pipe_pred(S, s);
    return done[(s + S - 1) % S] >= e && done[(s + 1) % S] >= e && (p < 0 || done[p] > e);
  };
  for (int u : order) {
    out.emplace_back(u, 0);
    done[u] = 1;
    for (bool any = true; any;) {   // every operation that became ready, the latest first
      any = false;
      for (int e = E - 1; e >= 1; --e)
        for (int s : order)
          if (ready(s, e)) {
            out.emplace_back(s, e);
            done[s] = e + 1;
            any = true;
          }
    }
  }
  return out;
}

// The pinned staging copy of the AoS buffer and the copy threads, for a pageable caller
// buffer; false when pinned host memory of that size cannot be had (the copies then go to the
// pageable buffer directly, the copy out after the commit).
static bool pipe_host_setup(mgpu_solver *h)
{
  if (h->pipe_host_state == 0) {
    if (cudaHostAlloc((void **) &h->pipe_host, (size_t) h->g.nz * 8 * sizeof(double), cudaHostAllocDefault) !=
        cudaSuccess) {
      cudaGetLastError();
      h->pipe_host = nullptr;
      h->pipe_host_state = -1;
      return false;
    }
    h->pipe_host_state = 1;
  }
  if (h->pipe_host_state < 0) return false;
  if (!h->pipe_pool) {
    const unsigned hc = std::thread::hardware_concurrency();
    h->pipe_pool = new HostCopyPool(hc >= 16 ? 8 : (hc >= 2 ? (int) hc / 2 : 1));
  }
  return true;
}

static int pipe_advance_host(mgpu_solver *h, double *host, double dt, const std::vector<int> &wb, int *errors)
{
  const int S = (int) wb.size() - 1;
  const Grid &g = h->g;
  const int K = num_stages(h->cfg.rk);
  const int E = 2 * K + 2;   // operations per slab
  const long long s0 = g.s[0], row_bytes = s0 * 8 * (long long) sizeof(double);
  const int G0 = g.G[0], ng = g.ng;
  cudaPointerAttributes pa{};
  const bool pinned = cudaPointerGetAttributes(&pa, host) == cudaSuccess && pa.type == cudaMemoryTypeHost;
  cudaGetLastError();   // an unregistered pointer may leave an error behind
  // a pageable buffer goes through the pinned staging copy: the DMA copies read and write
  // `dma`, and the pool copies between it and the caller's buffer
  const bool staged = !pinned && pipe_host_setup(h);
  double *dma = staged ? h->pipe_host : host;
  const bool early_out = pinned || staged;   // copies out while later slabs compute
  cudaEvent_t *ev_in = h->pipe_ev.data(), *ev_dl = ev_in + S, *ev_out = ev_in + 2 * S;
  std::vector<int> out_order;   // slabs in the order of their copies out
  const AdvanceArgs A = advance_args(h, 0, dt, 0.0);
  // the primitives of stage v (v = K: the closing c2p's) live in buf(v), the last in the
  // solver's own PA
  auto buf = [&](int v) { return (v + K) % 2 == 0 ? h->b.PA : h->pipe_pa; };
  auto window = [&](int s, int v) {
    AdvanceArgs W = A;
    W.g.w0 = wb[s];
    W.g.w1 = wb[s + 1];
    W.b.guess = h->pipe_guess;
    W.b.PA = buf(v);
    W.b.PAg = v > 0 ? buf(v - 1) : nullptr;
    W.g.whskip = pipe_whskip(S, s);
    return W;
  };
  auto phase = [&](const AdvanceArgs &W, int ph, int k) { return fp32(h) ? phase_fp32(W, ph, k) : phase_fp64(W, ph, k); };
  // the guarded rows [r0, r1) between the host buffer and a device AoS buffer
  auto copy_rows = [&](double *dst, const double *src, long long r0, long long r1, cudaMemcpyKind kind,
                       cudaStream_t st) {
    const size_t off = (size_t) (r0 * s0 * 8);
    return cudaMemcpyAsync(dst + off, src + off, (size_t) ((r1 - r0) * row_bytes), kind, st);
  };
  TransferArgs T = transfer_args(h);
  T.b.PA = buf(0);
  TransferArgs Tp = transfer_args(h);
  Tp.b.PA = buf(K);
  Tp.pending = 1;
  auto download_rows = [&](long long r0, long long r1) {
    return fp32(h) ? download_fp32(Tp, h->pipe_out + r0 * s0 * 8, r0 * s0, (r1 - r0) * s0)
                   : download_fp64(Tp, h->pipe_out + r0 * s0 * 8, r0 * s0, (r1 - r0) * s0);
  };
  // the rows a slab's copy out covers: its own, and for the end slabs the guard rows that
  // hold their images (slab 0: the right guards, slab S-1: the left guards)
  auto out_ranges = [&](int s, long long r[3][2]) {
    int n = 0;
    r[n][0] = ng + wb[s];
    r[n][1] = ng + wb[s + 1];
    ++n;
    if (s == 0) { r[n][0] = ng + g.n[0]; r[n][1] = G0; ++n; }
    if (s == S - 1) { r[n][0] = 0; r[n][1] = ng; ++n; }
    return n;
  };
  CK(phase(A, PH_BEGIN, 0));
  for (const auto &op : pipe_schedule(S, K)) {
    const int s = op.first, e = op.second;
    if (e == 0) {
      // the copy in: the slab's rows, and the end slabs' guard rows (kept for the restore)
      const long long r0 = s == 0 ? 0 : ng + wb[s], r1 = s == S - 1 ? G0 : ng + wb[s + 1];
      if (staged) h->pipe_pool->copy(dma + r0 * s0 * 8, host + r0 * s0 * 8, (size_t) ((r1 - r0) * row_bytes));
      CK(copy_rows(h->pipe_in, dma, r0, r1, cudaMemcpyHostToDevice, h->pipe_h2d));
      CK(cudaEventRecord(ev_in[s], h->pipe_h2d));
      CK(cudaStreamWaitEvent(h->stream, ev_in[s], 0));
      const long long z0 = (ng + wb[s]) * s0, cnt = (long long) (wb[s + 1] - wb[s]) * s0;
      CK(fp32(h) ? upload_fp32(T, h->pipe_in + z0 * 8, z0, cnt) : upload_fp64(T, h->pipe_in + z0 * 8, z0, cnt));
    } else if (e == E - 1) {   // download
      long long r[3][2];
      const int n = out_ranges(s, r);
      for (int i = 0; i < n; ++i) CK(download_rows(r[i][0], r[i][1]));
      if (early_out) {
        CK(cudaEventRecord(ev_dl[s], h->stream));
        CK(cudaStreamWaitEvent(h->pipe_d2h, ev_dl[s], 0));
        for (int i = 0; i < n; ++i)
          CK(copy_rows(dma, h->pipe_out, r[i][0], r[i][1], cudaMemcpyDeviceToHost, h->pipe_d2h));
        CK(cudaEventRecord(ev_out[s], h->pipe_d2h));
        out_order.push_back(s);
      }
    } else if (e % 2 == 1) {
      CK(phase(window(s, (e - 1) / 2), PH_FLUX_UPDATE, (e - 1) / 2));
    } else {
      CK(phase(window(s, e / 2), PH_C2P, e / 2));
    }
  }
  CK(phase(A, PH_COMMIT, 0));
  CK(cudaMemcpyAsync(h->ctl_host, h->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, h->stream));
  if (staged) {   // each slab's result from the staging copy into the caller's buffer as it lands
    for (int s : out_order) {
      CK(cudaEventSynchronize(ev_out[s]));
      long long r[3][2];
      const int n = out_ranges(s, r);
      for (int i = 0; i < n; ++i)
        h->pipe_pool->copy(host + r[i][0] * s0 * 8, dma + r[i][0] * s0 * 8, (size_t) ((r[i][1] - r[i][0]) * row_bytes));
    }
  }
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaStreamSynchronize(h->pipe_d2h));
  CK(cudaStreamSynchronize(h->pipe_h2d));
  if (h->ctl_host->tc_fault) return fail(h, MGPU_ERR_CUDA, "a tensor-core wait of the learned c2p timed out");
  const int err = errors_of(*h->ctl_host, h->cfg.rk);
  const size_t all = (size_t) g.nz * 8 * sizeof(double);
  if (early_out && err) {       // the copies out went ahead: put the caller's buffer back
    CK(cudaMemcpyAsync(dma, h->pipe_in, all, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (staged) h->pipe_pool->copy(host, dma, all);
  } else if (!early_out && !err) {
    CK(cudaMemcpyAsync(host, h->pipe_out, all, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  }
  *errors = err;
  return MGPU_OK;
}

int mgpu_set_pipeline(mgpu_solver *h, int slabs)
{
  if (!h || slabs < -1 || slabs == 1 || slabs == 2) return fail(h, MGPU_ERR_ARG, "pipeline slabs: 0, -1 or >= 3");
  h->pipe_slabs = slabs;
  return MGPU_OK;
}

int mgpu_get_pipeline(const mgpu_solver *h, int *slabs, int *last_slabs)
{
  if (!h) return MGPU_ERR_ARG;
  if (slabs) *slabs = h->pipe_slabs;
  if (last_slabs) *last_slabs = h->pipe_last;
  return MGPU_OK;
}

int mgpu_pipeline_bounds(int n0, int slabs, int *bounds, int capacity)
{
  if (n0 < 0 || slabs < -1 || slabs == 0 || slabs == 1 || slabs == 2 || capacity < 0) return -MGPU_ERR_ARG;
  const std::vector<int> wb = pipe_bounds(n0, slabs);
  if (bounds) {
    if (capacity < (int) wb.size()) return -MGPU_ERR_ARG;
    for (size_t i = 0; i < wb.size(); ++i) bounds[i] = wb[i];
  }
  return wb.empty() ? 0 : (int) wb.size() - 1;
}

int mgpu_pipeline_schedule(int slabs, int stages, int *out, int capacity)
{
  if (slabs < 3 || stages < 1 || stages > 3 || capacity < 0) return -MGPU_ERR_ARG;
  const auto sched = pipe_schedule(slabs, stages);
  if (out) {
    if (capacity < (int) sched.size()) return -MGPU_ERR_ARG;
    for (size_t i = 0; i < sched.size(); ++i) {
      out[2 * i] = sched[i].first;
      out[2 * i + 1] = sched[i].second;
    }
  }
  return (int) sched.size();
}

int mgpu_advance_host(mgpu_solver *h, double *host_aos, double dt, double *kzps, int *errors)
{
  int rc = ensure_ready(h);
  if (rc) return rc;
  if (!host_aos) return fail(h, MGPU_ERR_ARG, "null primitive buffer");
  const auto t0 = std::chrono::steady_clock::now();
  int err = 0;
  const std::vector<int> wb = pipe_slab_bounds(h);
  const int S = wb.empty() ? 0 : (int) wb.size() - 1;
  h->pipe_last = 0;
  if (S && pipe_setup(h, S) == 0) {
    h->pipe_last = S;
    rc = pipe_advance_host(h, host_aos, dt, wb, &err);
    if (rc) return rc;
  } else {
    rc = mgpu_upload_prim(h, host_aos);
    if (rc) return rc;
    rc = mgpu_advance(h, dt, &err);
    if (rc) return rc;
    if (err == 0) {
      rc = mgpu_download_prim(h, host_aos);
      if (rc) return rc;
    }
  }
  const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (kzps) *kzps = 1e-3 * (double) h->g.nz / sec;
  if (errors) *errors = err;
  return MGPU_OK;
}

int mgpu_advance_async(mgpu_solver *h, int n, int dt_mode, double dt, double cfl)
{
  int rc = ensure_ready(h);
  if (rc) return rc;
  if (n < 0 || (dt_mode != 0 && dt_mode != 1)) return fail(h, MGPU_ERR_ARG, "bad advance_async arguments");
  for (int i = 0; i < n; ++i) {
    rc = enqueue_advance(h, dt_mode, dt, cfl);
    if (rc) return rc;
  }
  return MGPU_OK;
}

int mgpu_synchronize(mgpu_solver *h)
{
  if (!h) return MGPU_ERR_ARG;
  CK(cudaStreamSynchronize(h->stream));
  return MGPU_OK;
}

int mgpu_get_timestep(mgpu_solver *h, double cfl, double *dt)
{
  int rc = ensure_ready(h);
  if (rc) return rc;
  rc = read_ctl(h);
  if (rc) return rc;
  double ml;
  memcpy(&ml, &h->ctl_host->max_lambda_bits, sizeof(double));
  *dt = cfl * h->min_dx / ml;
  return MGPU_OK;
}

int mgpu_get_stats(mgpu_solver *h, mgpu_stats *s)
{
  int rc = ensure_ready(h);
  if (rc) return rc;
  rc = read_ctl(h);
  if (rc) return rc;
  const Ctl &c = *h->ctl_host;
  memset(s, 0, sizeof(*s));
  memcpy(&s->max_lambda, &c.max_lambda_bits, sizeof(double));
  s->dt = c.dt;
  s->errors = errors_of(c, h->cfg.rk);
  s->committed = c.committed;
  const StatSlot t = stat_sum(c);
  s->c2p_calls = t.c2p_calls;
  s->c2p_iters = t.c2p_iters;
  for (int a = 0; a < 6; ++a) s->c2p_attempt[a] = t.c2p_attempt[a];
  s->face_c2p_calls = t.face_c2p_calls;
  s->face_c2p_iters = t.face_c2p_iters;
  s->hlld_ok = t.hlld_ok;
  s->hlld_hllc = t.hlld_hllc;
  s->pcm_retry = t.pcm_retry;
  s->c2p_failed = t.c2p_failed;
  s->advances = c.n_advances;
  s->failed_advances = c.n_failed;
  s->failed_zones = c.n_failed_zones;
  return MGPU_OK;
}

int mgpu_measure_divB(mgpu_solver *h, double *mean, double *max)
{
  int rc = ensure_ready(h);
  if (rc) return rc;
  if (h->g.nd < 2) {
    *mean = 0.0;
    *max = 0.0;
    return MGPU_OK;
  }
  if (fp32(h)) k_divB<float><<<RED_BLOCKS, 256, 0, h->stream>>>(h->g, (const float *) h->b.PA, h->red);
  else k_divB<double><<<RED_BLOCKS, 256, 0, h->stream>>>(h->g, (const double *) h->b.PA, h->red);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h->red_host, h->red, sizeof(double) * 2 * RED_BLOCKS, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  double sum = 0.0, mx = 0.0;   // zones outside the stencil's range count as div = 0
  for (int b = 0; b < RED_BLOCKS; ++b) {
    sum += h->red_host[2 * b];
    mx = fmax(mx, h->red_host[2 * b + 1]);
  }
  long long glb = 1;
  for (int d = 0; d < h->g.nd; ++d) glb *= h->N[d];
  *mean = (sum / (double) h->g.nz) / (double) glb;
  *max = mx;
  return MGPU_OK;
}

int mgpu_measure_divB_state(mgpu_solver *h, double *mean, double *max)
{
  int rc = ensure_ready(h);
  if (rc) return rc;
  if (h->g.nd < 2) {
    *mean = 0.0;
    *max = 0.0;
    return MGPU_OK;
  }
  CK(cudaMemcpyAsync(h->ctl_host, h->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  const double *B = lean(h) ? (h->ctl_host->cur ? h->b.U1_B : h->b.U0_B) : h->b.Pc_B[h->ctl_host->cur];
  k_divB_state<<<RED_BLOCKS, 256, 0, h->stream>>>(h->g, B, h->red);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h->red_host, h->red, sizeof(double) * 2 * RED_BLOCKS, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  double sum = 0.0, mx = 0.0;
  for (int b = 0; b < RED_BLOCKS; ++b) {
    sum += h->red_host[2 * b];
    mx = fmax(mx, h->red_host[2 * b + 1]);
  }
  long long glb = 1;
  for (int d = 0; d < h->g.nd; ++d) glb *= h->N[d];
  *mean = (sum / (double) h->g.nz) / (double) glb;
  *max = mx;
  return MGPU_OK;
}

int mgpu_max_lorentz_factor(mgpu_solver *h, double *wmax)
{
  int rc = ensure_ready(h);
  if (rc) return rc;
  if (fp32(h)) k_wmax<float><<<RED_BLOCKS, 256, 0, h->stream>>>(h->g, (const float *) h->b.PA, h->red);
  else k_wmax<double><<<RED_BLOCKS, 256, 0, h->stream>>>(h->g, (const double *) h->b.PA, h->red);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h->red_host, h->red, sizeof(double) * RED_BLOCKS, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  double mx = 0.0;
  for (int b = 0; b < RED_BLOCKS; ++b) mx = fmax(mx, h->red_host[b]);
  *wmax = mx;
  return MGPU_OK;
}

// ---- the other Mara.measure.* (Mara/mara.cpp:1954-2230): one device pass, host sums ----------
namespace {

// PhysicalUnits(1, 1, 1) (cgs), the units a started reference holds (Mara/hydro.cpp:20), as
// Mara/units.cpp computes them.
MeasureUnits default_units()
{
  const double length = 1.0, mass = 1.0, time = 1.0;
  const double gram = 1.0 / mass, centimeter = 1.0 / length, second = 1.0 / time;
  const double erg = gram * pow(centimeter / second, 2.0);
  const double mev = 1.60217648740e-06 * erg;                       // MEV_TO_ERG (Mara/eos.hpp:15)
  const double mev_fm3 = mev / pow(1e-13 * centimeter, 3);
  MeasureUnits u;
  u.erg_cc = mev_fm3 * 1e-33;
  u.gcc = gram / pow(centimeter, 3.0);
  const double mp = 1.67262177774e-24 * gram;                        // PROTON_MASS
  const double kb = 1.38064881300e-16 * erg;                         // BOLTZMANN_CONSTANT
  u.mp_kb = mp / kb;
  u.gauss = sqrt(erg / pow(centimeter, 3.0) / (4 * M_PI));
  return u;
}

// Runs the reduction over the measured primitive array and sums the block partials in block
// order: out[MEAS_FIELDS] (sums, then the extremes).  ttl = the global interior zone count.
int measure_all(mgpu_solver *h, double *out, double *ttl, MeasureUnits *units)
{
  int rc = ensure_ready(h);
  if (rc) return rc;
  const MeasureUnits u = default_units();
  CK(measures_launch(h->g, h->b.PA, fp32(h), h->cfg.gamma, u, h->meas, h->stream));
  CK(cudaMemcpyAsync(h->meas_host, h->meas, sizeof(double) * MEAS_BLOCKS * MEAS_FIELDS, cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int q = 0; q < MEAS_FIELDS; ++q) {
    double v = q < MEAS_SUMS ? 0.0 : h->meas_host[q];
    for (int b = q < MEAS_SUMS ? 0 : 1; b < MEAS_BLOCKS; ++b) {
      const double x = h->meas_host[(size_t) b * MEAS_FIELDS + q];
      if (q < MEAS_SUMS) v += x;
      else if (q == MEAS_MAMIN) v = x < v ? x : v;
      else v = x > v ? x : v;
    }
    out[q] = v;
  }
  long long glb = 1;
  for (int d = 0; d < h->g.nd; ++d) glb *= h->N[d];
  *ttl = (double) glb;
  if (units) *units = u;
  return MGPU_OK;
}

}  // namespace

int mgpu_measure_mean_cons(mgpu_solver *h, double *out)
{
  double m[MEAS_FIELDS], ttl;
  if (!out) return MGPU_ERR_ARG;
  const int rc = measure_all(h, m, &ttl, nullptr);
  if (rc) return rc;
  for (int q = 0; q < 8; ++q) out[q] = m[MEAS_CONS + q] / ttl;
  return MGPU_OK;
}

int mgpu_measure_mean_prim(mgpu_solver *h, double *out)
{
  double m[MEAS_FIELDS], ttl;
  if (!out) return MGPU_ERR_ARG;
  const int rc = measure_all(h, m, &ttl, nullptr);
  if (rc) return rc;
  for (int q = 0; q < 8; ++q) out[q] = m[MEAS_PRIM + q] / ttl;
  return MGPU_OK;
}

int mgpu_measure_mean_energies(mgpu_solver *h, double *out)
{
  double m[MEAS_FIELDS], ttl;
  if (!out) return MGPU_ERR_ARG;
  const int rc = measure_all(h, m, &ttl, nullptr);
  if (rc) return rc;
  for (int q = 0; q < 4; ++q) out[q] = m[MEAS_ENERGY + q] / ttl;
  return MGPU_OK;
}

int mgpu_measure_mean_velocity(mgpu_solver *h, double *out)
{
  double m[MEAS_FIELDS], ttl;
  if (!out) return MGPU_ERR_ARG;
  const int rc = measure_all(h, m, &ttl, nullptr);
  if (rc) return rc;
  for (int q = 0; q < 4; ++q) out[q] = m[MEAS_VEL + q] / ttl;
  return MGPU_OK;
}

int mgpu_measure_mean_max_temperature(mgpu_solver *h, double *mean, double *max)
{
  double m[MEAS_FIELDS], ttl;
  if (!mean || !max) return MGPU_ERR_ARG;
  const int rc = measure_all(h, m, &ttl, nullptr);
  if (rc) return rc;
  *mean = m[MEAS_T] / ttl;
  *max = m[MEAS_TMAX];
  return MGPU_OK;
}

int mgpu_measure_mean_max_magnetic_field(mgpu_solver *h, double *mean, double *max)
{
  double m[MEAS_FIELDS], ttl;
  MeasureUnits u;
  if (!mean || !max) return MGPU_ERR_ARG;
  const int rc = measure_all(h, m, &ttl, &u);
  if (rc) return rc;
  *mean = (1.0 / u.gauss) * m[MEAS_B] / ttl;
  *max = (1.0 / u.gauss) * m[MEAS_BMAX];
  return MGPU_OK;
}

int mgpu_measure_mean_max_sonic_mach(mgpu_solver *h, double *mean, double *max)
{
  double m[MEAS_FIELDS], ttl;
  if (!mean || !max) return MGPU_ERR_ARG;
  const int rc = measure_all(h, m, &ttl, nullptr);
  if (rc) return rc;
  *mean = m[MEAS_MS] / ttl;
  *max = m[MEAS_MSMAX];
  return MGPU_OK;
}

int mgpu_measure_mean_min_alfvenic_mach(mgpu_solver *h, double *mean, double *min)
{
  double m[MEAS_FIELDS], ttl;
  if (!mean || !min) return MGPU_ERR_ARG;
  const int rc = measure_all(h, m, &ttl, nullptr);
  if (rc) return rc;
  *mean = m[MEAS_MA] / ttl;
  *min = m[MEAS_MAMIN];
  return MGPU_OK;
}

// ---- Mara.diffuse / Mara.set_failmask (Mara/mara.cpp:343-373) ----------------------------------
static int diffuse_ready(mgpu_solver *h)
{
  int rc = ensure_ready(h);
  if (rc) return rc;
  if (lean(h)) return fail(h, MGPU_ERR_UNSUPPORTED, "diffuse is not offered in the lean layout");
  for (int d = 0; d < 3; ++d)
    if (h->g.ext[d]) return fail(h, MGPU_ERR_UNSUPPORTED, "diffuse needs a single (undecomposed) domain");
  return MGPU_OK;
}

int mgpu_diffuse(mgpu_solver *h, double r, int *errors)
{
  int rc = diffuse_ready(h);
  if (rc) return rc;
  const AdvanceArgs A = advance_args(h, 0, 0.0, 0.0);
  CK(fp32(h) ? diffuse_fp32(A, r) : diffuse_fp64(A, r));
  rc = read_ctl(h);
  if (rc) return rc;
  if (errors) *errors = h->ctl_host->diffuse_err;
  return MGPU_OK;
}

int mgpu_diffuse_host(mgpu_solver *h, double *host_aos, double r, int *errors)
{
  int rc = diffuse_ready(h);
  if (rc) return rc;
  rc = mgpu_upload_prim(h, host_aos);
  if (rc) return rc;
  rc = mgpu_diffuse(h, r, errors);
  if (rc) return rc;
  return mgpu_download_prim(h, host_aos);
}

int mgpu_set_failmask(mgpu_solver *h, int value)
{
  int rc = diffuse_ready(h);
  if (rc) return rc;
  CK(cudaMemsetAsync(h->fmask, value != 0, (size_t) h->g.nz, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return MGPU_OK;
}

int mgpu_reconfigure(mgpu_solver *h, const mgpu_config *cfg)
{
  if (!h || !cfg) return MGPU_ERR_ARG;
  mgpu_solver probe;
  int rc = check_config(&probe, cfg);
  if (rc) return fail(h, rc, probe.err);
  const mgpu_config &c = h->cfg;
  if (cfg->fluid != c.fluid || cfg->precision != c.precision || cfg->layout != c.layout)
    return fail(h, MGPU_ERR_UNSUPPORTED, "reconfigure keeps the fluid, precision and layout of the solver");
  if (h->have_domain) {
    for (int d = 0; d < 3; ++d)
      if (h->g.ext[d] && cfg->godunov == MGPU_GODUNOV_PLM_MUSCL)
        return fail(h, MGPU_ERR_UNSUPPORTED, "'plm-muscl' needs a single domain");
    CK(cudaStreamSynchronize(h->stream));
    const size_t cs = (size_t) h->g.cs, tsz = fp32(h) ? sizeof(float) : sizeof(double);
    cudaError_t e = cudaSuccess;
    if (cfg->rk == 4 && !h->b.K_bulk[0])
      for (int i = 0; i < 3 && e == cudaSuccess; ++i) {
        e = dalloc(h, &h->b.K_bulk[i], 5 * cs * tsz);
        if (e == cudaSuccess) e = dalloc(h, (void **) &h->b.K_B[i], 3 * cs * sizeof(double));
      }
    if (cfg->godunov == MGPU_GODUNOV_PLM_MUSCL && !h->b.Pd[0])
      for (int d = 0; d < 3 && e == cudaSuccess; ++d) {
        if (d < h->g.nd) e = dalloc(h, &h->b.Pd[d], 8 * cs * tsz);
        else h->b.Pd[d] = h->b.Pd[0];
      }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(h, e == cudaErrorMemoryAllocation ? MGPU_ERR_NOMEM : MGPU_ERR_CUDA,
                  std::string("reconfigure: ") + cudaGetErrorString(e));
    }
  }
  h->cfg = *cfg;
  return MGPU_OK;
}

int mgpu_profile_enable(mgpu_solver *h, int capacity)
{
  if (!h || capacity <= 0) return MGPU_ERR_ARG;
  CK(cudaStreamSynchronize(h->stream));
  prof_free(h);
  h->prof_ev.resize(2 * (size_t) capacity);
  for (auto &e : h->prof_ev) CK(cudaEventCreate(&e));
  h->prof_tag.assign(capacity, 0);
  h->prof_units.assign(capacity, 0);
  h->prof_count = 0;
  h->prof.ev = h->prof_ev.data();
  h->prof.tag = h->prof_tag.data();
  h->prof.units = h->prof_units.data();
  h->prof.capacity = capacity;
  h->prof.count = &h->prof_count;
  h->prof_on = true;
  return MGPU_OK;
}

int mgpu_profile_disable(mgpu_solver *h)
{
  if (!h) return MGPU_ERR_ARG;
  CK(cudaStreamSynchronize(h->stream));
  prof_free(h);
  return MGPU_OK;
}

int mgpu_profile_read(mgpu_solver *h, double *ms, long long *launches, long long *units)
{
  if (!h || !ms || !launches || !units) return MGPU_ERR_ARG;
  if (!h->prof_on) return fail(h, MGPU_ERR_STATE, "profiling is not enabled");
  CK(cudaStreamSynchronize(h->stream));
  for (int c = 0; c < KC_COUNT; ++c) { ms[c] = 0.0; launches[c] = 0; units[c] = 0; }
  for (int i = 0; i < h->prof_count; ++i) {
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, h->prof_ev[2 * i], h->prof_ev[2 * i + 1]));
    const int c = h->prof_tag[i];
    ms[c] += t;
    launches[c] += 1;
    units[c] += h->prof_units[i];
  }
  h->prof_count = 0;
  return MGPU_OK;
}

int mgpu_advance_phase(mgpu_solver *h, int phase, int stage, int dt_mode, double dt, double cfl)
{
  int rc = ensure_ready(h);
  if (rc) return rc;
  const int ns = num_stages(h->cfg.rk);
  if (phase < 0 || phase > 5 || stage < 0 || stage > ns || ((phase == 2 || phase >= 4) && stage >= ns) ||
      (dt_mode != 0 && dt_mode != 1))
    return fail(h, MGPU_ERR_ARG, "bad advance phase arguments");
  AdvanceArgs A;
  A.g = h->g;
  A.pp = phys(h);
  A.rk = h->cfg.rk;
  A.godunov = h->cfg.godunov;
  A.lean = lean(h);
  A.ereset = h->cfg.ereset;
  A.preset = h->cfg.preset;
  A.dreset = h->cfg.dreset;
  A.dt_mode = dt_mode;
  A.dt = dt;
  A.cfl = cfl;
  A.min_dx = h->min_dx;
  A.b = h->b;
  A.ctl = h->ctl;
  A.stream = h->stream;
  A.prof = h->prof_on ? &h->prof : nullptr;
  CK(fp32(h) ? phase_fp32(A, phase, stage) : phase_fp64(A, phase, stage));
  if (phase == 3) CK(mgpu_driving_enqueue(h));
  return MGPU_OK;
}

int mgpu_reduction_targets(mgpu_solver *h, void **err_counts, void **max_lambda_bits)
{
  int rc = ensure_ready(h);
  if (rc) return rc;
  if (err_counts) *err_counts = (void *) &h->ctl->stage_err[0];
  if (max_lambda_bits) *max_lambda_bits = (void *) &h->ctl->max_lambda_bits;
  return MGPU_OK;
}

int mgpu_set_external_guards(mgpu_solver *h, const int *ext, const int *mult)
{
  int rc = ensure_ready(h);
  if (rc) return rc;
  if (!ext) return fail(h, MGPU_ERR_ARG, "null ext");
  CK(cudaStreamSynchronize(h->stream));
  Grid &g = h->g;
  long long total = 0;
  for (int d = 0; d < g.nd; ++d)
    if (ext[d]) total += g.n[d];
  if (total > 0 && !mult) return fail(h, MGPU_ERR_ARG, "external guards need multiplicity tables");
  if (total > 0 && h->cfg.godunov != MGPU_GODUNOV_PLM_SPLIT)
    return fail(h, MGPU_ERR_UNSUPPORTED, "the CTU-Hancock operator runs on single domains only");
  for (long long i = 0; i < total; ++i)
    if (mult[i] < 1) return fail(h, MGPU_ERR_ARG, "multiplicities must be >= 1");
  if (h->mult) cudaFree(h->mult);
  h->mult = nullptr;
  for (int d = 0; d < 3; ++d) {
    g.ext[d] = 0;
    g.mult[d] = nullptr;
  }
  if (total == 0) return MGPU_OK;
  CK(cudaMalloc((void **) &h->mult, sizeof(int) * (size_t) total));
  CK(cudaMemcpy(h->mult, mult, sizeof(int) * (size_t) total, cudaMemcpyHostToDevice));
  long long off = 0;
  for (int d = 0; d < g.nd; ++d)
    if (ext[d]) {
      g.ext[d] = 1;
      g.mult[d] = h->mult + off;
      off += g.n[d];
    }
  return MGPU_OK;
}

int mgpu_halo_bytes(mgpu_solver *h, int which, int dim, long long *bytes)
{
  int rc = ensure_ready(h);
  if (rc) return rc;
  if (!bytes || dim < 0 || dim >= h->g.nd || (which != 0 && which != 1)) return fail(h, MGPU_ERR_ARG, "bad halo arguments");
  const Grid &g = h->g;
  const long long cross = dim == 0 ? (long long) g.G[1] * g.G[2] : dim == 1 ? (long long) g.G[0] * g.G[2]
                                                                          : (long long) g.G[0] * g.G[1];
  const long long per = cross * g.ng;
  const long long tsz = fp32(h) ? 4 : 8;
  *bytes = which == 0 ? per * 8 * tsz : per * (5 * tsz + 3 * 8);
  return MGPU_OK;
}

static int halo(mgpu_solver *h, int which, int dim, int side, void *buf, int pack, cudaStream_t stream = nullptr,
                bool use_stream = false)
{
  int rc = ensure_ready(h);
  if (rc) return rc;
  if (!buf || dim < 0 || dim >= h->g.nd || (which != 0 && which != 1) || (side != 0 && side != 1))
    return fail(h, MGPU_ERR_ARG, "bad halo arguments");
  if (lean(h) && which == 1)   // the lean layout's committed state is PA (which 0) and U[cur]
    return fail(h, MGPU_ERR_UNSUPPORTED, "the lean layout exchanges its stage primitives only (which 0)");
  TransferArgs t = transfer_args(h);
  if (use_stream) t.stream = stream;
  if (which == 1) {
    rc = read_ctl(h);
    if (rc) return rc;
    t.cur = h->ctl_host->cur;
  }
  CK(fp32(h) ? halo_fp32(t, which, dim, side, buf, pack) : halo_fp64(t, which, dim, side, buf, pack));
  return MGPU_OK;
}

int mgpu_halo_pack_on(mgpu_solver *h, int which, int dim, int side, void *dev_buf, void *stream)
{
  return halo(h, which, dim, side, dev_buf, 1, (cudaStream_t) stream, true);
}

int mgpu_halo_unpack_on(mgpu_solver *h, int which, int dim, int side, const void *dev_buf, void *stream)
{
  return halo(h, which, dim, side, const_cast<void *>(dev_buf), 0, (cudaStream_t) stream, true);
}

int mgpu_halo_pack(mgpu_solver *h, int which, int dim, int side, void *dev_buf)
{
  return halo(h, which, dim, side, dev_buf, 1);
}

int mgpu_halo_unpack(mgpu_solver *h, int which, int dim, int side, const void *dev_buf)
{
  return halo(h, which, dim, side, const_cast<void *>(dev_buf), 0);
}

// Grid, buffers and stream of a solver, for the learned-c2p harvest (c2p_mlp.cu).
int mgpu_internal_state(mgpu_solver *h, Grid *g, AdvanceBuffers *b, Ctl **ctl, void **stream, int *is32,
                        double *gamma)
{
  int rc = ensure_ready(h);
  if (rc) return rc;
  if (lean(h)) return fail(h, MGPU_ERR_UNSUPPORTED, "pairs are harvested from standard-layout solvers");
  *g = h->g;
  *b = h->b;
  *ctl = h->ctl;
  *stream = (void *) h->stream;
  *is32 = fp32(h);
  *gamma = h->cfg.gamma;
  return MGPU_OK;
}

int mgpu_set_c2p_network(mgpu_solver *h, const float *params, long long count)
{
  if (!h || !params) return MGPU_ERR_ARG;
  if (count != mgpu_mlp_param_count()) return fail(h, MGPU_ERR_ARG, "network has the wrong number of parameters");
  cudaStreamSynchronize(h->stream);
  if (h->mlp) cudaFree(h->mlp);
  if (h->mlp_tc) cudaFree(h->mlp_tc);
  h->mlp = nullptr;
  h->mlp_tc = nullptr;
  CK(cudaMalloc((void **) &h->mlp, count * sizeof(float)));
  CK(cudaMemcpy(h->mlp, params, count * sizeof(float), cudaMemcpyHostToDevice));
  std::vector<unsigned char> img(mgpu_mlp_tc_image_bytes());
  mgpu_mlp_build_tc_image(params, img.data());
  CK(cudaMalloc(&h->mlp_tc, img.size()));
  CK(cudaMemcpy(h->mlp_tc, img.data(), img.size(), cudaMemcpyHostToDevice));
  h->mlp_count = count;
  return MGPU_OK;
}

}  // extern "C"
