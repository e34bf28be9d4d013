// Host side of the ensemble API (include/mara_gpu.h, mgpu_ensemble_*): many independent
// boxes of uneven size, one scheme, advanced together by the persistent tile-walking kernels
// of rmhd_ensemble.cuh, with the sequence of launches of nsteps advances replayed as one
// CUDA graph, and the launch-shape autotuner.
//
// Memory: one arena per ensemble holding, per box, the same arrays an mgpu_solver of that
// box allocates (two committed primitive states, U0, U1, K1-K3 for RK4, the stage
// primitives and one flux array per dimension), each 256-byte aligned; the boxes' control
// blocks are one contiguous device array so that a single copy reads every box's outcome.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <string>
#include <vector>

#include "../../include/mara_gpu.h"
#include "rmhd_types.cuh"

MGPU_DECLARE_PRECISION(fp64)
MGPU_DECLARE_PRECISION(fp32)

using namespace mgpu;

struct mgpu_ensemble {
  mgpu_config cfg;
  std::string err;
  int nb = 0, nd = 0;
  int num_sms = 148;
  std::vector<Grid> grids;
  std::vector<double> min_dx;
  std::vector<AdvanceBuffers> bufs;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  void *arena = nullptr;
  size_t arena_bytes = 0;
  Ctl *ctl = nullptr;            // nb control blocks (device)
  Ctl *ctl_host = nullptr;       // pinned mirror
  BoxDev *boxes = nullptr;       // device descriptors
  int2 *maps = nullptr;          // device tile maps: zone tiles, then the face tiles of each sweep
  size_t maps_cap = 0;           // entries allocated
  size_t face_off[3] = {0, 0, 0};
  double *dt_dev = nullptr;      // per-box dt (device)
  double *staging = nullptr;     // AoS staging for host transfers
  long long staging_zones = 0;
  mgpu_ensemble_launch launch{};
  long long zone_tiles = 0, face_tiles[3] = {0, 0, 0};
  // cached graph of `graph_steps` advances
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0, graph_dt_mode = -1, graph_commit = 1;
  double graph_cfl = 0.0;
  mgpu_ensemble_launch graph_launch{};
  // kernel timing of direct (not graph) advances
  std::vector<cudaEvent_t> prof_ev;
  std::vector<int> prof_tag;
  std::vector<long long> prof_units;
  int prof_count = 0;
  LaunchProfiler prof{};
  bool prof_on = false;
};

namespace {

int fail(mgpu_ensemble *e, int code, const std::string &msg)
{
  if (e) e->err = msg;
  return code;
}

int cuda_fail(mgpu_ensemble *e, cudaError_t c, const char *where)
{
  return fail(e, MGPU_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(c));
}

#define CK(call)                                                \
  do {                                                          \
    cudaError_t c_ = (call);                                    \
    if (c_ != cudaSuccess) return cuda_fail(e, c_, #call);      \
  } while (0)

constexpr size_t ALIGN = 256;
size_t align_up(size_t n) { return (n + ALIGN - 1) / ALIGN * ALIGN; }

bool fp32(const mgpu_ensemble *e) { return e->cfg.precision == MGPU_PREC_FP32; }

PhysParams phys(const mgpu_ensemble *e)
{
  PhysParams p;
  p.gamma = e->cfg.gamma;
  p.pfloor = e->cfg.pfloor;
  p.theta = e->cfg.theta;
  p.sz10A = e->cfg.sz10A;
  p.is_mode = e->cfg.is_mode;
  p.recon = e->cfg.recon;
  p.riemann = e->cfg.riemann;
  p.learned = 0;
  p.learned_faces = 0;
  p.mlp = nullptr;
  p.mlp_tc = nullptr;
  return p;
}

// The grid of one box, as mgpu_set_domain lays it out (Ng = 3).
Grid make_grid(int nd, const int *N, const double *x0, const double *x1, double *min_dx)
{
  const int ng = 3;
  Grid g{};
  g.nd = nd;
  g.ng = ng;
  double lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    g.n[d] = d < nd ? N[d] : 1;
    g.G[d] = d < nd ? N[d] + 2 * ng : 1;
    lo[d] = d < nd ? x0[d] : 0.0;
    hi[d] = d < nd ? x1[d] : 1.0;
  }
  g.nz = (long long) g.G[0] * g.G[1] * g.G[2];
  g.cs = (g.nz + 31) / 32 * 32;
  g.s[0] = (long long) g.G[1] * g.G[2];
  g.s[1] = g.G[2];
  g.s[2] = 1;
  g.dx = (hi[0] - lo[0]) / (g.G[0] - 2 * ng);
  g.dy = (hi[1] - lo[1]) / (g.G[1] - 2 * ng);
  g.dz = (hi[2] - lo[2]) / (g.G[2] - 2 * ng);
  g.ninterior = (long long) g.n[0] * g.n[1] * g.n[2];
  double m = hi[0] - lo[0];
  for (int d = 0; d < nd; ++d) m = std::min(m, (hi[d] - lo[d]) / N[d]);
  *min_dx = m;
  return g;
}

long long faces_of(const Grid &g, int dim) { return std::max(0ll, g.nz - 5 * g.s[dim - 1]); }

// Tile maps for the current launch shape: entry w of a map is (box, tile within the box) of
// the w-th tile of the concatenated work; uploaded to e->maps.
int build_maps(mgpu_ensemble *e)
{
  const int nb = e->nb;
  const long long zt = e->launch.zone_tile, ft = e->launch.face_tile;
  std::vector<int2> h;
  for (int b = 0; b < nb; ++b) {
    const long long n = (e->grids[b].ninterior + zt - 1) / zt;
    for (long long t = 0; t < n; ++t) h.push_back(make_int2(b, (int) t));
  }
  e->zone_tiles = (long long) h.size();
  for (int d = 0; d < 3; ++d) {
    e->face_off[d] = h.size();
    if (d < e->nd)
      for (int b = 0; b < nb; ++b) {
        const long long n = (faces_of(e->grids[b], d + 1) + ft - 1) / ft;
        for (long long t = 0; t < n; ++t) h.push_back(make_int2(b, (int) t));
      }
    e->face_tiles[d] = (long long) (h.size() - e->face_off[d]);
  }
  CK(cudaStreamSynchronize(e->stream));
  if (h.size() > e->maps_cap) {
    if (e->maps) cudaFree(e->maps);
    e->maps = nullptr;
    e->maps_cap = 0;
    CK(cudaMalloc((void **) &e->maps, h.size() * sizeof(int2)));
    e->maps_cap = h.size();
  }
  CK(cudaMemcpyAsync(e->maps, h.data(), h.size() * sizeof(int2), cudaMemcpyHostToDevice, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  return MGPU_OK;
}

int check_launch(mgpu_ensemble *e, const mgpu_ensemble_launch &L)
{
  auto tile_ok = [](int t) { return t >= 32 && t <= (1 << 20) && t % 32 == 0; };
  auto cps_ok = [](int c) { return c >= 1 && c <= 64; };
  if (!tile_ok(L.zone_tile) || !tile_ok(L.face_tile))
    return fail(e, MGPU_ERR_ARG, "ensemble tiles must be multiples of 32 between 32 and 2^20");
  if (!cps_ok(L.zone_ctas_per_sm) || !cps_ok(L.face_ctas_per_sm) || !cps_ok(L.c2p_ctas_per_sm))
    return fail(e, MGPU_ERR_ARG, "ensemble CTAs per SM must be between 1 and 64");
  return MGPU_OK;
}

EnsembleArgs args_of(mgpu_ensemble *e, int dt_mode, double cfl, int commit, bool capture)
{
  EnsembleArgs E;
  const int nb = e->nb;
  E.boxes = e->boxes;
  E.nb = nb;
  E.nd = e->nd;
  E.zone_map = e->maps;
  E.zone_tiles = e->zone_tiles;
  for (int d = 0; d < 3; ++d) {
    E.face_map[d] = e->maps + e->face_off[d];
    E.face_tiles[d] = e->face_tiles[d];
  }
  E.zone_tile = e->launch.zone_tile;
  E.face_tile = e->launch.face_tile;
  auto grid = [&](long long tiles, int cps) {
    const long long g = std::min<long long>(tiles, (long long) e->num_sms * cps);
    return (int) std::max<long long>(g, 1);
  };
  E.grid_zone = grid(e->zone_tiles, e->launch.zone_ctas_per_sm);
  E.grid_face = grid(std::max(e->face_tiles[0], std::max(e->face_tiles[1], e->face_tiles[2])),
                     e->launch.face_ctas_per_sm);
  E.grid_c2p = grid(e->zone_tiles, e->launch.c2p_ctas_per_sm);
  E.pp = phys(e);
  E.rk = e->cfg.rk;
  E.ereset = e->cfg.ereset;
  E.preset = e->cfg.preset;
  E.dreset = e->cfg.dreset;
  E.dt_mode = dt_mode;
  E.dt = e->dt_dev;
  E.cfl = cfl;
  E.commit = commit;
  E.stream = e->stream;
  E.prof = (e->prof_on && !capture) ? &e->prof : nullptr;
  E.total_zones = 0;
  for (int d = 0; d < 3; ++d) E.total_faces[d] = 0;
  for (const Grid &g : e->grids) {
    E.total_zones += g.ninterior;
    for (int d = 0; d < e->nd; ++d) E.total_faces[d] += faces_of(g, d + 1);
  }
  return E;
}

cudaError_t enqueue(mgpu_ensemble *e, int nsteps, int dt_mode, double cfl, int commit, bool capture)
{
  const EnsembleArgs E = args_of(e, dt_mode, cfl, commit, capture);
  for (int s = 0; s < nsteps; ++s) {
    const cudaError_t c = fp32(e) ? ensemble_advance_fp32(E) : ensemble_advance_fp64(E);
    if (c != cudaSuccess) return c;
  }
  return cudaSuccess;
}

bool same_launch(const mgpu_ensemble_launch &a, const mgpu_ensemble_launch &b)
{
  return a.zone_tile == b.zone_tile && a.face_tile == b.face_tile && a.zone_ctas_per_sm == b.zone_ctas_per_sm &&
         a.face_ctas_per_sm == b.face_ctas_per_sm && a.c2p_ctas_per_sm == b.c2p_ctas_per_sm;
}

void drop_graph(mgpu_ensemble *e)
{
  if (e->graph) cudaGraphExecDestroy(e->graph);
  e->graph = nullptr;
  e->graph_steps = 0;
}

// Replay (capturing first if the cached graph is for other arguments) nsteps advances.
int run_graph(mgpu_ensemble *e, int nsteps, int dt_mode, double cfl, int commit)
{
  if (!e->graph || e->graph_steps != nsteps || e->graph_dt_mode != dt_mode || e->graph_cfl != cfl ||
      e->graph_commit != commit || !same_launch(e->graph_launch, e->launch)) {
    drop_graph(e);
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    const cudaError_t c = enqueue(e, nsteps, dt_mode, cfl, commit, true);
    const cudaError_t c2 = cudaStreamEndCapture(e->stream, &g);
    if (c != cudaSuccess || c2 != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return cuda_fail(e, c != cudaSuccess ? c : c2, "ensemble graph capture");
    }
    const cudaError_t c3 = cudaGraphInstantiate(&e->graph, g, 0);
    cudaGraphDestroy(g);
    if (c3 != cudaSuccess) {
      e->graph = nullptr;
      return cuda_fail(e, c3, "cudaGraphInstantiate");
    }
    e->graph_steps = nsteps;
    e->graph_dt_mode = dt_mode;
    e->graph_cfl = cfl;
    e->graph_commit = commit;
    e->graph_launch = e->launch;
  }
  CK(cudaGraphLaunch(e->graph, e->stream));
  return MGPU_OK;
}

int check_box(mgpu_ensemble *e, int box)
{
  if (!e) return MGPU_ERR_ARG;
  if (box < 0 || box >= e->nb) return fail(e, MGPU_ERR_ARG, "no such box");
  return MGPU_OK;
}

TransferArgs transfer_args(const mgpu_ensemble *e, int box)
{
  TransferArgs t;
  t.g = e->grids[box];
  t.b = e->bufs[box];
  t.ctl = e->ctl + box;
  t.stream = e->stream;
  t.cur = 0;
  return t;
}

// kind 0: upload, 1: download of box `box`'s committed primitives.
int transfer(mgpu_ensemble *e, int box, double *host, const void *dev_in, void *dev_out, int kind)
{
  int rc = check_box(e, box);
  if (rc) return rc;
  const TransferArgs t = transfer_args(e, box);
  const long long nz = e->grids[box].nz;
  if (dev_in || dev_out) {
    double *d = (double *) (dev_in ? const_cast<void *>(dev_in) : dev_out);
    const cudaError_t c = kind == 0 ? (fp32(e) ? upload_fp32(t, d, 0, nz) : upload_fp64(t, d, 0, nz))
                                    : (fp32(e) ? download_fp32(t, d, 0, nz) : download_fp64(t, d, 0, nz));
    CK(c);
    CK(cudaStreamSynchronize(e->stream));
    return MGPU_OK;
  }
  for (long long z0 = 0; z0 < nz; z0 += e->staging_zones) {
    const long long cnt = std::min(nz - z0, e->staging_zones);
    const size_t bytes = (size_t) cnt * 8 * sizeof(double);
    if (kind == 0) {
      CK(cudaMemcpyAsync(e->staging, host + z0 * 8, bytes, cudaMemcpyHostToDevice, e->stream));
      CK(fp32(e) ? upload_fp32(t, e->staging, z0, cnt) : upload_fp64(t, e->staging, z0, cnt));
    } else {
      CK(fp32(e) ? download_fp32(t, e->staging, z0, cnt) : download_fp64(t, e->staging, z0, cnt));
      CK(cudaMemcpyAsync(host + z0 * 8, e->staging, bytes, cudaMemcpyDeviceToHost, e->stream));
    }
  }
  CK(cudaStreamSynchronize(e->stream));
  return MGPU_OK;
}

int read_ctl(mgpu_ensemble *e)
{
  CK(cudaMemcpyAsync(e->ctl_host, e->ctl, sizeof(Ctl) * (size_t) e->nb, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  return MGPU_OK;
}

int errors_of(const Ctl &c, int rk)
{
  const int ns = num_stages(rk);
  for (int s = 0; s < ns; ++s)
    if (c.stage_err[s]) return c.stage_err[s];
  return c.final_err;
}

void prof_free(mgpu_ensemble *e)
{
  for (cudaEvent_t ev : e->prof_ev) cudaEventDestroy(ev);
  e->prof_ev.clear();
  e->prof_tag.clear();
  e->prof_units.clear();
  e->prof_on = false;
}

void release(mgpu_ensemble *e)
{
  drop_graph(e);
  prof_free(e);
  if (e->arena) cudaFree(e->arena);
  if (e->ctl) cudaFree(e->ctl);
  if (e->boxes) cudaFree(e->boxes);
  if (e->maps) cudaFree(e->maps);
  if (e->dt_dev) cudaFree(e->dt_dev);
  if (e->staging) cudaFree(e->staging);
  if (e->ctl_host) cudaFreeHost(e->ctl_host);
  if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
  e->arena = nullptr;
  e->ctl = nullptr;
  e->ctl_host = nullptr;
  e->stream = nullptr;
}

}  // namespace

extern "C" {

int mgpu_ensemble_create(const mgpu_config *cfg, int nd, int nboxes, const int *N, const double *x0,
                         const double *x1, mgpu_ensemble **out)
{
  if (!out || !cfg || !N) return MGPU_ERR_ARG;
  *out = nullptr;
  auto reject = [](const char *msg, int code) {
    fprintf(stderr, "[mgpu] ensemble: %s\n", msg);
    return code;
  };
  if (cfg->fluid != MGPU_FLUID_RMHD) return reject("only the 'rmhd' fluid is provided", MGPU_ERR_UNSUPPORTED);
  if (!(cfg->gamma > 1.0) || cfg->recon < 0 || cfg->recon > 2 || cfg->riemann < 0 || cfg->riemann > 2 ||
      cfg->rk < 1 || cfg->rk > 4 || cfg->is_mode < 0 || cfg->is_mode > 2 ||
      (cfg->precision != MGPU_PREC_FP64 && cfg->precision != MGPU_PREC_FP32))
    return reject("bad configuration", MGPU_ERR_ARG);
  if (cfg->learned_c2p) return reject("the learned c2p guess is not offered for ensembles", MGPU_ERR_UNSUPPORTED);
  if (cfg->layout != MGPU_LAYOUT_STANDARD)
    return reject("ensembles use the standard layout", MGPU_ERR_UNSUPPORTED);
  if (cfg->godunov != MGPU_GODUNOV_PLM_SPLIT)
    return reject("ensembles use the method-of-lines operator (plm-split)", MGPU_ERR_UNSUPPORTED);
  if (nd < 1 || nd > 3) return reject("boxes must have 1, 2 or 3 dimensions", MGPU_ERR_ARG);
  if (nboxes < 1) return reject("an ensemble needs at least one box", MGPU_ERR_ARG);
  for (long long i = 0; i < (long long) nboxes * nd; ++i)
    if (N[i] < 3) return reject("periodic guard fill needs N >= 3 on every axis", MGPU_ERR_ARG);

  mgpu_ensemble *e = new mgpu_ensemble;
  e->cfg = *cfg;
  e->nb = nboxes;
  e->nd = nd;
  e->grids.resize(nboxes);
  e->min_dx.resize(nboxes);
  e->bufs.resize(nboxes);
  const double one[3] = {1.0, 1.0, 1.0}, zero[3] = {0.0, 0.0, 0.0};
  long long max_nz = 0;
  for (int b = 0; b < nboxes; ++b) {
    const double *lo = x0 ? x0 + (size_t) b * nd : zero, *hi = x1 ? x1 + (size_t) b * nd : one;
    e->grids[b] = make_grid(nd, N + (size_t) b * nd, lo, hi, &e->min_dx[b]);
    max_nz = std::max(max_nz, e->grids[b].nz);
  }
  // arena layout: per box the arrays of mgpu_set_domain
  const size_t tsz = fp32(e) ? sizeof(float) : sizeof(double);
  const int nstate = cfg->rk == 4 ? 7 : 4;
  std::vector<size_t> base(nboxes);
  size_t total = 0;
  for (int b = 0; b < nboxes; ++b) {
    const size_t cs = (size_t) e->grids[b].cs;
    base[b] = total;
    total += nstate * (align_up(5 * cs * tsz) + align_up(3 * cs * sizeof(double)));
    total += (1 + nd) * align_up(8 * cs * tsz);
  }
  e->arena_bytes = total;
  cudaError_t c = cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, 0);
  int dev = 0;
  if (c == cudaSuccess) c = cudaGetDevice(&dev);
  if (c == cudaSuccess) c = cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, dev);
  if (c == cudaSuccess) c = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
  if (c == cudaSuccess) e->own_stream = true;
  if (c == cudaSuccess) c = cudaMalloc(&e->arena, total);
  if (c == cudaSuccess) c = cudaMemsetAsync(e->arena, 0, total, e->stream);
  if (c == cudaSuccess) c = cudaMalloc((void **) &e->ctl, sizeof(Ctl) * (size_t) nboxes);
  if (c == cudaSuccess) c = cudaMemsetAsync(e->ctl, 0, sizeof(Ctl) * (size_t) nboxes, e->stream);
  if (c == cudaSuccess) c = cudaMallocHost((void **) &e->ctl_host, sizeof(Ctl) * (size_t) nboxes);
  if (c == cudaSuccess) c = cudaMalloc((void **) &e->boxes, sizeof(BoxDev) * (size_t) nboxes);
  if (c == cudaSuccess) c = cudaMalloc((void **) &e->dt_dev, sizeof(double) * (size_t) nboxes);
  if (c == cudaSuccess) c = cudaMemsetAsync(e->dt_dev, 0, sizeof(double) * (size_t) nboxes, e->stream);
  e->staging_zones = std::min<long long>(max_nz, 1ll << 22);
  if (c == cudaSuccess) c = cudaMalloc((void **) &e->staging, (size_t) e->staging_zones * 8 * sizeof(double));
  if (c != cudaSuccess) {
    fprintf(stderr, "[mgpu] ensemble: %s (%zu bytes of box arrays)\n", cudaGetErrorString(c), total);
    cudaGetLastError();
    release(e);
    delete e;
    return c == cudaErrorMemoryAllocation ? MGPU_ERR_NOMEM : MGPU_ERR_CUDA;
  }
  std::vector<BoxDev> hb(nboxes);
  unsigned char *arena = (unsigned char *) e->arena;
  for (int b = 0; b < nboxes; ++b) {
    const size_t cs = (size_t) e->grids[b].cs;
    size_t off = base[b];
    auto take = [&](size_t bytes) {
      void *p = arena + off;
      off += align_up(bytes);
      return p;
    };
    AdvanceBuffers &B = e->bufs[b];
    B = AdvanceBuffers{};
    auto state = [&](void **bulk, double **Bp) {
      *bulk = take(5 * cs * tsz);
      *Bp = (double *) take(3 * cs * sizeof(double));
    };
    state(&B.Pc_bulk[0], &B.Pc_B[0]);
    state(&B.Pc_bulk[1], &B.Pc_B[1]);
    state(&B.U0_bulk, &B.U0_B);
    state(&B.U1_bulk, &B.U1_B);
    if (cfg->rk == 4)
      for (int i = 0; i < 3; ++i) state(&B.K_bulk[i], &B.K_B[i]);
    B.PA = take(8 * cs * tsz);
    for (int d = 0; d < 3; ++d) B.F[d] = d < nd ? take(8 * cs * tsz) : B.F[0];
    hb[b].g = e->grids[b];
    hb[b].b = B;
    hb[b].ctl = e->ctl + b;
    hb[b].min_dx = e->min_dx[b];
  }
  c = cudaMemcpyAsync(e->boxes, hb.data(), sizeof(BoxDev) * (size_t) nboxes, cudaMemcpyHostToDevice, e->stream);
  if (c == cudaSuccess) c = cudaStreamSynchronize(e->stream);
  if (c != cudaSuccess) {
    fprintf(stderr, "[mgpu] ensemble: %s\n", cudaGetErrorString(c));
    release(e);
    delete e;
    return MGPU_ERR_CUDA;
  }
  // default launch shape (the tuner's starting point)
  e->launch.zone_tile = 1024;
  e->launch.face_tile = 512;
  e->launch.zone_ctas_per_sm = 8;
  e->launch.face_ctas_per_sm = fp32(e) ? 4 : 3;
  e->launch.c2p_ctas_per_sm = 8;
  if (build_maps(e)) {
    fprintf(stderr, "[mgpu] ensemble: %s\n", e->err.c_str());
    release(e);
    delete e;
    return MGPU_ERR_CUDA;
  }
  *out = e;
  return MGPU_OK;
}

int mgpu_ensemble_destroy(mgpu_ensemble *e)
{
  if (!e) return MGPU_ERR_ARG;
  if (e->stream) cudaStreamSynchronize(e->stream);
  release(e);
  delete e;
  return MGPU_OK;
}

const char *mgpu_ensemble_last_error(const mgpu_ensemble *e) { return e ? e->err.c_str() : "null handle"; }

int mgpu_ensemble_set_stream(mgpu_ensemble *e, void *stream)
{
  if (!e) return MGPU_ERR_ARG;
  if (!stream) return fail(e, MGPU_ERR_ARG, "an ensemble needs a created stream (graphs cannot capture stream 0)");
  CK(cudaStreamSynchronize(e->stream));
  if (e->own_stream) cudaStreamDestroy(e->stream);
  e->stream = (cudaStream_t) stream;
  e->own_stream = false;
  drop_graph(e);
  return MGPU_OK;
}

int mgpu_ensemble_num_zones(const mgpu_ensemble *e, int box, long long *nz)
{
  if (!e || !nz || box < 0 || box >= e->nb) return MGPU_ERR_ARG;
  *nz = e->grids[box].nz;
  return MGPU_OK;
}

int mgpu_ensemble_total_interior(const mgpu_ensemble *e, long long *n)
{
  if (!e || !n) return MGPU_ERR_ARG;
  long long s = 0;
  for (const Grid &g : e->grids) s += g.ninterior;
  *n = s;
  return MGPU_OK;
}

int mgpu_ensemble_upload_prim(mgpu_ensemble *e, int box, const double *host_aos)
{
  if (!host_aos) return fail(e, MGPU_ERR_ARG, "null primitive buffer");
  return transfer(e, box, const_cast<double *>(host_aos), nullptr, nullptr, 0);
}

int mgpu_ensemble_download_prim(mgpu_ensemble *e, int box, double *host_aos)
{
  if (!host_aos) return fail(e, MGPU_ERR_ARG, "null primitive buffer");
  return transfer(e, box, host_aos, nullptr, nullptr, 1);
}

int mgpu_ensemble_upload_prim_device(mgpu_ensemble *e, int box, const void *dev_aos)
{
  if (!dev_aos) return fail(e, MGPU_ERR_ARG, "null primitive buffer");
  return transfer(e, box, nullptr, dev_aos, nullptr, 0);
}

int mgpu_ensemble_download_prim_device(mgpu_ensemble *e, int box, void *dev_aos)
{
  if (!dev_aos) return fail(e, MGPU_ERR_ARG, "null primitive buffer");
  return transfer(e, box, nullptr, nullptr, dev_aos, 1);
}

int mgpu_ensemble_get_launch(const mgpu_ensemble *e, mgpu_ensemble_launch *L)
{
  if (!e || !L) return MGPU_ERR_ARG;
  *L = e->launch;
  return MGPU_OK;
}

int mgpu_ensemble_set_launch(mgpu_ensemble *e, const mgpu_ensemble_launch *L)
{
  if (!e || !L) return MGPU_ERR_ARG;
  int rc = check_launch(e, *L);
  if (rc) return rc;
  CK(cudaStreamSynchronize(e->stream));
  e->launch = *L;
  return build_maps(e);
}

int mgpu_ensemble_advance(mgpu_ensemble *e, int nsteps, int dt_mode, const double *dt, double cfl, int use_graph)
{
  if (!e) return MGPU_ERR_ARG;
  if (nsteps < 0 || (dt_mode != 0 && dt_mode != 1) || (dt_mode == 0 && !dt))
    return fail(e, MGPU_ERR_ARG, "bad ensemble advance arguments");
  if (nsteps == 0) return MGPU_OK;
  if (dt_mode == 0)
    CK(cudaMemcpyAsync(e->dt_dev, dt, sizeof(double) * (size_t) e->nb, cudaMemcpyHostToDevice, e->stream));
  if (use_graph) return run_graph(e, nsteps, dt_mode, cfl, 1);
  CK(enqueue(e, nsteps, dt_mode, cfl, 1, false));
  return MGPU_OK;
}

int mgpu_ensemble_synchronize(mgpu_ensemble *e)
{
  if (!e) return MGPU_ERR_ARG;
  CK(cudaStreamSynchronize(e->stream));
  return MGPU_OK;
}

int mgpu_ensemble_errors(mgpu_ensemble *e, int *errors)
{
  if (!e || !errors) return MGPU_ERR_ARG;
  int rc = read_ctl(e);
  if (rc) return rc;
  for (int b = 0; b < e->nb; ++b) errors[b] = errors_of(e->ctl_host[b], e->cfg.rk);
  return MGPU_OK;
}

int mgpu_ensemble_get_stats(mgpu_ensemble *e, int box, mgpu_stats *s)
{
  int rc = check_box(e, box);
  if (rc) return rc;
  if (!s) return MGPU_ERR_ARG;
  rc = read_ctl(e);
  if (rc) return rc;
  const Ctl &c = e->ctl_host[box];
  memset(s, 0, sizeof(*s));
  memcpy(&s->max_lambda, &c.max_lambda_bits, sizeof(double));
  s->dt = c.dt;
  s->errors = errors_of(c, e->cfg.rk);
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
  return MGPU_OK;
}

int mgpu_ensemble_get_timesteps(mgpu_ensemble *e, double cfl, double *dt)
{
  if (!e || !dt) return MGPU_ERR_ARG;
  int rc = read_ctl(e);
  if (rc) return rc;
  for (int b = 0; b < e->nb; ++b) {
    double ml;
    memcpy(&ml, &e->ctl_host[b].max_lambda_bits, sizeof(double));
    dt[b] = cfl * e->min_dx[b] / ml;
  }
  return MGPU_OK;
}

int mgpu_ensemble_profile_enable(mgpu_ensemble *e, int capacity)
{
  if (!e || capacity <= 0) return MGPU_ERR_ARG;
  CK(cudaStreamSynchronize(e->stream));
  prof_free(e);
  e->prof_ev.resize(2 * (size_t) capacity);
  for (auto &ev : e->prof_ev) CK(cudaEventCreate(&ev));
  e->prof_tag.assign(capacity, 0);
  e->prof_units.assign(capacity, 0);
  e->prof_count = 0;
  e->prof.ev = e->prof_ev.data();
  e->prof.tag = e->prof_tag.data();
  e->prof.units = e->prof_units.data();
  e->prof.capacity = capacity;
  e->prof.count = &e->prof_count;
  e->prof_on = true;
  return MGPU_OK;
}

int mgpu_ensemble_profile_disable(mgpu_ensemble *e)
{
  if (!e) return MGPU_ERR_ARG;
  CK(cudaStreamSynchronize(e->stream));
  prof_free(e);
  return MGPU_OK;
}

int mgpu_ensemble_profile_read(mgpu_ensemble *e, double *ms, long long *launches, long long *units)
{
  if (!e || !ms || !launches || !units) return MGPU_ERR_ARG;
  if (!e->prof_on) return fail(e, MGPU_ERR_STATE, "profiling is not enabled");
  CK(cudaStreamSynchronize(e->stream));
  for (int c = 0; c < KC_COUNT; ++c) {
    ms[c] = 0.0;
    launches[c] = 0;
    units[c] = 0;
  }
  for (int i = 0; i < e->prof_count; ++i) {
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, e->prof_ev[2 * i], e->prof_ev[2 * i + 1]));
    const int c = e->prof_tag[i];
    ms[c] += t;
    launches[c] += 1;
    units[c] += e->prof_units[i];
  }
  e->prof_count = 0;
  return MGPU_OK;
}

int mgpu_ensemble_time_advance(mgpu_ensemble *e, const mgpu_ensemble_launch *L, const double *dt, int reps, double *ms)
{
  if (!e || !L || !dt || !ms || reps < 1) return MGPU_ERR_ARG;
  int rc = check_launch(e, *L);
  if (rc) return rc;
  const mgpu_ensemble_launch keep = e->launch;
  rc = read_ctl(e);   // every box's control block, put back afterwards
  if (rc) return rc;
  std::vector<Ctl> saved(e->ctl_host, e->ctl_host + e->nb);
  e->launch = *L;
  rc = build_maps(e);
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  if (!rc) {
    CK(cudaMemcpyAsync(e->dt_dev, dt, sizeof(double) * (size_t) e->nb, cudaMemcpyHostToDevice, e->stream));
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    rc = run_graph(e, 1, 0, 0.0, 0);   // capture + warm-up
    if (!rc) CK(cudaEventRecord(t0, e->stream));
    for (int r = 0; r < reps && !rc; ++r) rc = run_graph(e, 1, 0, 0.0, 0);
    if (!rc) CK(cudaEventRecord(t1, e->stream));
    if (!rc) CK(cudaEventSynchronize(t1));
    float t = 0.f;
    if (!rc) CK(cudaEventElapsedTime(&t, t0, t1));
    *ms = (double) t / reps;
  }
  if (t0) cudaEventDestroy(t0);
  if (t1) cudaEventDestroy(t1);
  drop_graph(e);
  e->launch = keep;
  const int rc2 = build_maps(e);
  memcpy(e->ctl_host, saved.data(), sizeof(Ctl) * (size_t) e->nb);
  CK(cudaMemcpyAsync(e->ctl, e->ctl_host, sizeof(Ctl) * (size_t) e->nb, cudaMemcpyHostToDevice, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  return rc ? rc : rc2;
}

int mgpu_ensemble_autotune(mgpu_ensemble *e, const double *dt, int reps, mgpu_ensemble_launch *best, double *best_ms)
{
  if (!e || !dt) return MGPU_ERR_ARG;
  mgpu_ensemble_launch cur = e->launch;
  double cur_ms = 0.0;
  int rc = mgpu_ensemble_time_advance(e, &cur, dt, reps, &cur_ms);
  if (rc) return rc;
  // Coordinate descent: the flux launches dominate, so their shape first; two passes.
  const int face_tiles[] = {128, 256, 512, 1024, 2048, 4096};
  const int zone_tiles[] = {256, 512, 1024, 2048, 4096, 8192};
  const int face_cps[] = {2, 3, 4, 5, 6, 8};
  const int zone_cps[] = {2, 4, 6, 8, 12, 16};
  for (int pass = 0; pass < 2; ++pass) {
    for (int axis = 0; axis < 5; ++axis) {
      const int *vals = axis == 0 ? face_tiles : axis == 1 ? face_cps : axis == 2 ? zone_tiles : zone_cps;
      for (int v = 0; v < 6; ++v) {
        mgpu_ensemble_launch L = cur;
        switch (axis) {
        case 0: L.face_tile = vals[v]; break;
        case 1: L.face_ctas_per_sm = vals[v]; break;
        case 2: L.zone_tile = vals[v]; break;
        case 3: L.zone_ctas_per_sm = vals[v]; break;
        default: L.c2p_ctas_per_sm = zone_cps[v]; break;
        }
        if (same_launch(L, cur)) continue;
        double ms = 0.0;
        rc = mgpu_ensemble_time_advance(e, &L, dt, reps, &ms);
        if (rc) return rc;
        if (ms < cur_ms) {
          cur = L;
          cur_ms = ms;
        }
      }
    }
  }
  rc = mgpu_ensemble_set_launch(e, &cur);
  if (rc) return rc;
  if (best) *best = cur;
  if (best_ms) *best_ms = cur_ms;
  return MGPU_OK;
}

}  // extern "C"
