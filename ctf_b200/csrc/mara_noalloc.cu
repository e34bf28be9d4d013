// mgpu_advance_noalloc: one FP64 advance of a small box that allocates no memory.
//
// Who needs this: code that runs where it may not call cudaMalloc -- an allocation-free
// section of a larger application (real-time loops that must not block or fragment the
// device heap, a host library that hands out only pre-owned buffers, or a process whose
// memory pool is fixed at start).  The regular entry points allocate the solver's working
// arrays in mgpu_set_domain; this one instead keeps them in a fixed array in the library's
// own device memory, declared below, so a call needs nothing but the caller's input and
// output buffers.
//
// The price: the array below exists on every GPU that loads the library, for the life of
// the process, so it is kept small (NOALLOC_SCRATCH_BYTES, about 7.8 MiB), which limits the
// box to MGPU_NOALLOC_MAX_ZONES guarded zones.  All calls share it; each call clears the
// control block it reads before use, but two calls whose work overlaps on the GPU (other
// streams, other host threads) overwrite each other's arrays -- serialise them.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include "../../include/mara_gpu.h"
#include "rmhd_types.cuh"

MGPU_DECLARE_PRECISION(fp64)

using namespace mgpu;

namespace {

constexpr long long CS_MAX = MGPU_NOALLOC_MAX_ZONES;   // a multiple of 32
constexpr size_t ALIGN = 256;
constexpr size_t align_up(size_t n) { return (n + ALIGN - 1) / ALIGN * ALIGN; }
// 7 state arrays (two committed prim buffers, U0, U1, K1-K3 for RK4) of 64 B per zone,
// 4 face arrays (stage prims and three flux directions) of 64 B per zone, the control block
constexpr size_t STATE_BYTES = align_up(5 * CS_MAX * sizeof(double)) + align_up(3 * CS_MAX * sizeof(double));
constexpr size_t FACE_BYTES = align_up(8 * CS_MAX * sizeof(double));
constexpr size_t NOALLOC_SCRATCH_BYTES = 7 * STATE_BYTES + 4 * FACE_BYTES + align_up(sizeof(Ctl));
static_assert(CS_MAX % 32 == 0, "component stride must be a multiple of 32");

}  // namespace

// The working memory of mgpu_advance_noalloc (file scope, one copy per device).
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

namespace {

void put_err(char *buf, int len, const char *msg)
{
  if (buf && len > 0) {
    strncpy(buf, msg, (size_t) len - 1);
    buf[len - 1] = '\0';
  }
}

}  // namespace

extern "C" int mgpu_advance_noalloc(const mgpu_config *cfg, const double *x0, const double *x1, const int *N,
                                    int nd, const void *dev_prim_in, void *dev_prim_out, double dt, int *errors,
                                    double *max_lambda, void *stream, char *errbuf, int errbuf_len)
{
  if (!cfg || !x0 || !x1 || !N || !dev_prim_in || !dev_prim_out || !errors) {
    put_err(errbuf, errbuf_len, "mgpu_advance_noalloc: null argument");
    return MGPU_ERR_ARG;
  }
  if (cfg->fluid != MGPU_FLUID_RMHD || cfg->precision != MGPU_PREC_FP64 || cfg->rk < 1 || cfg->rk > 4 ||
      cfg->recon < 0 || cfg->recon > 2 || cfg->riemann < 0 || cfg->riemann > 2 || cfg->is_mode < 0 ||
      cfg->is_mode > 2 || !(cfg->gamma > 1.0) || cfg->learned_c2p || cfg->godunov != MGPU_GODUNOV_PLM_SPLIT ||
      cfg->layout != MGPU_LAYOUT_STANDARD) {
    put_err(errbuf, errbuf_len,
            "mgpu_advance_noalloc: needs an rmhd FP64 plm-split configuration without a learned c2p network");
    return MGPU_ERR_ARG;
  }
  if (nd < 1 || nd > 3) {
    put_err(errbuf, errbuf_len, "mgpu_advance_noalloc: domain must have 1, 2 or 3 dimensions");
    return MGPU_ERR_ARG;
  }
  const int ng = 3;
  Grid g{};
  g.nd = nd;
  g.ng = ng;
  double lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    if (d < nd && N[d] < ng) {
      put_err(errbuf, errbuf_len, "mgpu_advance_noalloc: periodic guard fill needs N >= 3 on every axis");
      return MGPU_ERR_ARG;
    }
    g.n[d] = d < nd ? N[d] : 1;
    g.G[d] = d < nd ? N[d] + 2 * ng : 1;
    lo[d] = d < nd ? x0[d] : 0.0;
    hi[d] = d < nd ? x1[d] : 1.0;
  }
  g.nz = (long long) g.G[0] * g.G[1] * g.G[2];
  if (g.nz > MGPU_NOALLOC_MAX_ZONES) {
    char msg[200];
    snprintf(msg, sizeof(msg),
             "mgpu_advance_noalloc: box has %lld guarded zones, more than the %d this entry point "
             "can hold; use mgpu_create/mgpu_set_domain for larger boxes",
             g.nz, (int) MGPU_NOALLOC_MAX_ZONES);
    put_err(errbuf, errbuf_len, msg);
    return MGPU_ERR_ARG;
  }
  g.cs = (g.nz + 31) / 32 * 32;
  g.s[0] = (long long) g.G[1] * g.G[2];
  g.s[1] = g.G[2];
  g.s[2] = 1;
  g.dx = (hi[0] - lo[0]) / (g.G[0] - 2 * ng);
  g.dy = (hi[1] - lo[1]) / (g.G[1] - 2 * ng);
  g.dz = (hi[2] - lo[2]) / (g.G[2] - 2 * ng);
  g.ninterior = (long long) g.n[0] * g.n[1] * g.n[2];

  // Set-up, on every call, with the caller's device current: the device address of the
  // scratch array (the host-side name g_noalloc_scratch is not a device address).  It is
  // looked up each time rather than cached, because a cudaDeviceReset or another context on
  // the same device between two calls would leave a cached address stale.  The lookup is a
  // table read once the library's device code is loaded; the first call on a device loads it.
  unsigned char *base;
  {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      char msg[200];
      snprintf(msg, sizeof(msg), "mgpu_advance_noalloc: cudaGetSymbolAddress failed: %s",
               cudaGetErrorString(e));
      put_err(errbuf, errbuf_len, msg);
      return MGPU_ERR_CUDA;
    }
    base = (unsigned char *) p;
  }

  // Carve the scratch into the advance's arrays (sized for the largest box, CS_MAX).
  size_t off = 0;
  auto take = [&](size_t bytes) {
    unsigned char *p = base + off;
    off += align_up(bytes);
    return (void *) p;
  };
  AdvanceBuffers b{};
  auto state = [&](void **bulk, double **B) {
    *bulk = take(5 * CS_MAX * sizeof(double));
    *B = (double *) take(3 * CS_MAX * sizeof(double));
  };
  state(&b.Pc_bulk[0], &b.Pc_B[0]);
  state(&b.Pc_bulk[1], &b.Pc_B[1]);
  state(&b.U0_bulk, &b.U0_B);
  state(&b.U1_bulk, &b.U1_B);
  for (int i = 0; i < 3; ++i) state(&b.K_bulk[i], &b.K_B[i]);
  b.PA = take(8 * CS_MAX * sizeof(double));
  for (int d = 0; d < 3; ++d) b.F[d] = take(8 * CS_MAX * sizeof(double));
  Ctl *ctl = (Ctl *) take(sizeof(Ctl));
  // (the carving uses CS_MAX strides for the array bases but g.cs inside each array)

  cudaStream_t st = (cudaStream_t) stream;
  // The control block keeps the previous call's contents: clear it (committed buffer 0,
  // MaxLambda, error counters) before this call reads it.
  cudaError_t e = cudaMemsetAsync(ctl, 0, sizeof(Ctl), st);

  TransferArgs t;
  t.g = g;
  t.b = b;
  t.ctl = ctl;
  t.stream = st;
  t.cur = 0;
  if (e == cudaSuccess) e = upload_fp64(t, (const double *) dev_prim_in, 0, g.nz);

  AdvanceArgs A;
  A.g = g;
  A.pp.gamma = cfg->gamma;
  A.pp.pfloor = cfg->pfloor;
  A.pp.theta = cfg->theta;
  A.pp.sz10A = cfg->sz10A;
  A.pp.is_mode = cfg->is_mode;
  A.pp.recon = cfg->recon;
  A.pp.riemann = cfg->riemann;
  A.pp.learned = 0;
  A.pp.learned_faces = 0;
  A.pp.mlp = nullptr;
  A.pp.mlp_tc = nullptr;
  A.rk = cfg->rk;
  A.godunov = 0;
  A.ereset = cfg->ereset;
  A.preset = cfg->preset;
  A.dreset = cfg->dreset;
  A.dt_mode = 0;
  A.dt = dt;
  A.cfl = 0.0;
  A.min_dx = 0.0;
  A.b = b;
  A.ctl = ctl;
  A.stream = st;
  A.prof = nullptr;
  if (e == cudaSuccess) e = advance_fp64(A);

  Ctl c;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&c, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    char msg[200];
    snprintf(msg, sizeof(msg), "mgpu_advance_noalloc: CUDA error: %s", cudaGetErrorString(e));
    put_err(errbuf, errbuf_len, msg);
    return MGPU_ERR_CUDA;
  }
  int err = 0;
  for (int s = 0; s < num_stages(cfg->rk) && !err; ++s) err = c.stage_err[s];
  if (!err) err = c.final_err;
  *errors = err;
  if (max_lambda) memcpy(max_lambda, &c.max_lambda_bits, sizeof(double));
  if (err == 0) {
    e = download_fp64(t, (double *) dev_prim_out, 0, g.nz);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      char msg[200];
      snprintf(msg, sizeof(msg), "mgpu_advance_noalloc: CUDA error: %s", cudaGetErrorString(e));
      put_err(errbuf, errbuf_len, msg);
      return MGPU_ERR_CUDA;
    }
  }
  put_err(errbuf, errbuf_len, "");
  return MGPU_OK;
}
