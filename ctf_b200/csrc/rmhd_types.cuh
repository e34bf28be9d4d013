// Plain data shared by the host library and the kernel translation units: physics
// parameters, the grid description, the device control block and the launch arguments.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mgpu {

enum { ddd = 0, tau = 1, Sx = 2, Sy = 3, Sz = 4, Bx = 5, By = 6, Bz = 7 };   // conserved
enum { rho = 0, pre = 1, vx = 2, vy = 3, vz = 4 };                            // primitive

enum C2PError {
  C2P_SUCCESS = 0, C2P_CONS_NAN, C2P_CONS_NEG_DENSITY, C2P_CONS_NEG_ENERGY, C2P_PRIM_NAN,
  C2P_PRIM_NEG_PRESSURE, C2P_PRIM_NEG_RESTMASS, C2P_PRIM_SUPERLUMINAL, C2P_MAXITER
};

enum Recon { RECON_PCM = 0, RECON_PLM = 1, RECON_WENO5 = 2 };
enum Riemann { RIEMANN_HLL = 0, RIEMANN_HLLC = 1, RIEMANN_HLLD = 2 };
enum ISMode { IS_JS96 = 0, IS_B08 = 1, IS_SZ10 = 2 };

// Solver constants that enter the physics (mirrors of the reference's global statics).
struct PhysParams {
  double gamma;      // AdiabaticEos::Gamma
  double pfloor;     // rmhd_c2p_set_pressure_floor
  double theta;      // reconstruct_set_plm_theta
  double sz10A;      // reconstruct_set_shenzha10_A
  int is_mode;       // reconstruct_set_smoothness_indicator
  int recon;         // GodunovOperator::reconstruct_method
  int riemann;
  int learned;       // learned c2p initial guess on/off (zone c2p)
  int learned_faces; // also for the HLL-state c2p inside HLLD (per-thread evaluation)
  const void *mlp;   // device pointer to the packed FP32 c2p network (nullptr when off)
  const void *mlp_tc;// device pointer to its tensor-core image (nullptr: per-thread path)
};

constexpr int MAX_STAGES = 4;

// Statistics counters of an advance, kept in STAT_SLOTS copies 128 bytes apart: block b adds
// to slot b % STAT_SLOTS and the host sums the slots.  With one copy every warp's atomic went
// to the same cache line and they serialised (2 ms per 256^3 step in the zone c2p alone).
constexpr int STAT_SLOTS = 32;
struct StatSlot {
  unsigned long long c2p_calls, c2p_iters, c2p_attempt[6];
  unsigned long long face_c2p_calls, face_c2p_iters;
  unsigned long long hlld_ok, hlld_hllc, pcm_retry;
  unsigned long long c2p_failed;   // zone c2p calls that failed every rung (reset or not)
  unsigned long long pad[2];       // 128 bytes
};

// What a c2p launch reads, where it writes and which counter its failures go to.
enum C2PMode {
  C2P_STAGE = 0,          // stage input -> PA, failures abort the stage
  C2P_CLOSING = 1,        // final state -> the uncommitted primitive buffer
  C2P_CTU_STAGE = 2,      // CTU-Hancock stage input -> PA, failures do not abort
  // lean layout: the conserved registers are U[cur] (committed) and U[!cur] (RK register)
  C2P_LEAN_STAGE = 3,     // U[!cur] -> PA
  C2P_LEAN_CLOSING = 4,   // U[!cur] -> PA, plus its field to U[!cur]'s guard images
  C2P_LEAN_RESTORE = 5,   // U[cur] -> PA after an advance that did not commit; uncounted
  C2P_DIFFUSE = 6         // Mara.diffuse: U -> the committed buffer in place, guess PA; sets
                          // the failure mask, counted only into Ctl::diffuse_err
};

// Device control block of one solver (one per handle, in device memory).
struct Ctl {
  unsigned long long max_lambda_bits;   // MaxLambda of the current/last advance (double bits)
  double dt;                            // dt used by the current/last advance
  int stage_err[MAX_STAGES];            // c2p failures per stage (guard images included)
  int final_err;                        // failures of the closing c2p
  int cur;                              // committed primitive buffer (0/1)
  int committed;                        // 1 if the last advance was committed
  int tc_fault;                         // a tensor-core wait timed out (sticky)
  // CTU-Hancock stage: failures of its four checks (first-flux face states, predictor face
  // states, predictor c2p, second-flux face states), the uncounted stage c2p failures and the
  // emergency resets of the stage c2p
  int ctu_err[4];
  int ctu_c2p_err;
  int ctu_reset;
  // GodunovOperator's FailureMask (Mara/hydro.cpp:133-149): one byte per guarded zone, set by
  // every counted c2p to whether the zone failed (0 after an emergency reset), read by
  // Mara.diffuse; nullptr where the solver keeps no mask (lean layout, ensembles)
  unsigned char *fmask;
  int diffuse_err;                      // failed zones of the last Mara.diffuse c2p
  // since the solver was created (never reset by an advance): advances run, advances not
  // committed, and the failed zones those reported (as Mara.advance returns them)
  unsigned long long n_advances, n_failed, n_failed_zones;
  // statistics, accumulated over the advance
  StatSlot stat[STAT_SLOTS];
};

// The statistics of an advance: the sum of the slots (host side, after a copy of the block).
inline StatSlot stat_sum(const Ctl &c)
{
  StatSlot t{};
  for (int i = 0; i < STAT_SLOTS; ++i) {
    const StatSlot &s = c.stat[i];
    t.c2p_calls += s.c2p_calls;
    t.c2p_iters += s.c2p_iters;
    for (int a = 0; a < 6; ++a) t.c2p_attempt[a] += s.c2p_attempt[a];
    t.face_c2p_calls += s.face_c2p_calls;
    t.face_c2p_iters += s.face_c2p_iters;
    t.hlld_ok += s.hlld_ok;
    t.hlld_hllc += s.hlld_hllc;
    t.pcm_retry += s.pcm_retry;
    t.c2p_failed += s.c2p_failed;
  }
  return t;
}

struct Grid {
  int nd, ng;
  int n[3];       // interior zones per dim (1 for unused dims)
  int G[3];       // guarded extent per dim (1 for unused dims)
  long long nz;   // guarded zones
  long long cs;   // component stride of the SoA arrays (elements)
  long long s[3]; // zone strides of x, y, z
  double dx, dy, dz;
  long long ninterior;
  // Decomposed domains: ext[d] = 1 when a halo exchange fills the guard layers of dimension
  // d (the c2p then scatters no periodic images along d), and mult[d][m] is the number of
  // guarded arrays, over all ranks, that hold interior index m of d (device, n[d] entries).
  int ext[3];
  const int *mult[3];
  // Window of the lean-layout launches: interior x rows [w0, w1) (w1 == 0: all rows).  A
  // window's launches read the rows within the stencil's reach around it and write only its
  // own rows, plus one halo row each side of the y and z face fields (the values the
  // neighbouring window writes there too).  whskip bit 0 / bit 1 leaves out the lower / upper
  // halo row, when the neighbouring window has already written it.
  int w0, w1, whskip;
};

__host__ __device__ inline int win_lo(const Grid &g) { return g.w1 ? g.w0 : 0; }
__host__ __device__ inline int win_hi(const Grid &g) { return g.w1 ? g.w1 : g.n[0]; }
__host__ __device__ inline int win_rows(const Grid &g) { return win_hi(g) - win_lo(g); }
// The x rows (interior-relative, -1 = the lower guard row) whose y and z face fields the
// window's sweeps compute: [win_flo, win_fhi)
__host__ __device__ inline int win_flo(const Grid &g) { return win_lo(g) - 1 + (g.whskip & 1); }
__host__ __device__ inline int win_fhi(const Grid &g) { return win_hi(g) + 1 - ((g.whskip >> 1) & 1); }
// The window's interior flat indices: [win_tbeg, win_tend)
__host__ __device__ inline long long win_tbeg(const Grid &g) { return (long long) win_lo(g) * g.n[1] * g.n[2]; }
__host__ __device__ inline long long win_tend(const Grid &g) { return (long long) win_hi(g) * g.n[1] * g.n[2]; }

template <class T> struct StatePtr {   // components 0..4 in T, 5..7 in double
  T *bulk;
  double *B;
};
template <class T> struct StateCPtr {
  const T *bulk;
  const double *B;
};

// Interior flat index t -> zone coordinates (guards counted).  Indices that fit in 32 bits
// (every box up to 1024^3: 1.1e9 guarded zones) take 32-bit unsigned division, the emulated
// 64-bit one costing several times as many instructions; the integers are the same.
__device__ __forceinline__ void interior_coords(const Grid &g, long long t, int &i, int &j, int &k)
{
  const long long nyz = (long long) g.n[1] * g.n[2];
  if (t < (1ll << 32) && nyz < (1ll << 32)) {
    const unsigned tt = (unsigned) t, d1 = (unsigned) nyz, d2 = (unsigned) g.n[2];
    const unsigned ii = tt / d1, r = tt - ii * d1, jj = r / d2;
    i = (int) ii;
    j = (int) jj;
    k = (int) (r - jj * d2);
  } else {
    i = (int) (t / nyz);
    const long long r = t - (long long) i * nyz;
    j = (int) (r / g.n[2]);
    k = (int) (r - (long long) j * g.n[2]);
  }
  i += g.ng;
  if (g.nd >= 2) j += g.ng;
  if (g.nd >= 3) k += g.ng;
}

// Guarded flat zone index z -> (i, j, k), with the same 32-bit fast path.
__device__ __forceinline__ void zone_coords(const Grid &g, long long z, int &i, int &j, int &k)
{
  if (z < (1ll << 32) && g.s[0] < (1ll << 32)) {
    const unsigned zz = (unsigned) z, s0 = (unsigned) g.s[0], G2 = (unsigned) g.G[2];
    const unsigned ii = zz / s0, r = zz - ii * s0, jj = r / G2;
    i = (int) ii;
    j = (int) jj;
    k = (int) (r - jj * G2);
  } else {
    i = (int) (z / g.s[0]);
    const long long r = z - (long long) i * g.s[0];
    j = (int) (r / g.G[2]);
    k = (int) (r - (long long) j * g.G[2]);
  }
}

struct AdvanceBuffers {
  void *Pc_bulk[2];
  double *Pc_B[2];
  void *PA;
  void *U0_bulk, *U1_bulk, *K_bulk[3];
  double *U0_B, *U1_B, *K_B[3];
  void *F[3];
  void *Pd[3];   // CTU-Hancock: predicted primitives per direction (8 x T each)
  void *Bf;      // lean layout: the six transverse magnetic face fluxes (6 x T)
  void *guess;   // learned c2p guesses, one float2 per interior zone (nullptr: Bf is the scratch)
  void *PAg;     // lean stage c2p: the previous primitives the ladder may start from (nullptr: PA)
};

// Optional per-launch timing: the launcher records an event pair around every kernel and
// tags it with its class (KC_*); the host sums the elapsed times after a synchronize.
enum KernelClass { KC_BEGIN = 0, KC_P2C = 1, KC_C2P = 2, KC_FLUX = 3, KC_UPDATE = 4, KC_PREDICT = 5, KC_COUNT = 6 };
struct LaunchProfiler {
  cudaEvent_t *ev;    // 2 * capacity events
  int *tag;
  long long *units;   // work units of the launch (faces or zones)
  int capacity;
  int *count;         // host counter
};

// Records an event pair around the launches of its scope when a profiler is attached.
struct ProfScope {
  LaunchProfiler *p;
  cudaStream_t s;
  int slot;
  ProfScope(LaunchProfiler *p_, cudaStream_t s_, int tag, long long units) : p(p_), s(s_), slot(-1)
  {
    if (p && *p->count < p->capacity) {
      slot = (*p->count)++;
      p->tag[slot] = tag;
      p->units[slot] = units;
      cudaEventRecord(p->ev[2 * slot], s);
    }
  }
  ~ProfScope()
  {
    if (slot >= 0) cudaEventRecord(p->ev[2 * slot + 1], s);
  }
};

// Phases of an advance.  The whole advance is PH_BEGIN, then (PH_C2P, PH_FLUX_UPDATE) per RK
// stage, then PH_C2P with stage = number of stages (the closing c2p into the uncommitted
// buffer), then PH_COMMIT.  A decomposed domain exchanges the guard layers of the stage
// primitives between PH_C2P and PH_FLUX_UPDATE, and sums the error counters over ranks
// before PH_COMMIT.
// PH_C2P_SHELL and PH_C2P_CORE together are PH_C2P of a stage (s < number of stages), split
// so that a decomposed domain can exchange the shell's slabs while the core converts.
enum Phase { PH_BEGIN = 0, PH_C2P = 1, PH_FLUX_UPDATE = 2, PH_COMMIT = 3, PH_C2P_SHELL = 4, PH_C2P_CORE = 5 };

struct AdvanceArgs {
  Grid g;
  PhysParams pp;
  int rk;           // 1 single, 2 rk2, 3 rk3, 4 rk4
  int godunov;      // 0 method of lines (plm-split), 1 CTU-Hancock (plm-muscl)
  int lean = 0;     // 1: lean layout (rmhd_lean.cuh)
  int ereset;
  double preset, dreset;
  int dt_mode;      // 0: dt from the host, 1: dt = cfl*min_dx/MaxLambda(previous)
  double dt, cfl, min_dx;
  AdvanceBuffers b;
  Ctl *ctl;
  cudaStream_t stream;
  LaunchProfiler *prof;   // nullptr: no timing
};

enum Combine {
  COMB_EULER = 0,     // Uout = Un + dt L                        (single; RK2/RK3 stage 1)
  COMB_RK2_2 = 1,     // Uout = 0.5 (Un + Us + dt L)
  COMB_RK3_2 = 2,     // Uout = 3/4 Un + 1/4 Us + 1/4 dt L
  COMB_RK3_3 = 3,     // Uout = 1/3 Un + 2/3 Us + 2/3 dt L
  COMB_RK4_K = 4,     // K = dt L; Uout = Un + c K                (c = 1/2, 1/2, 1)
  COMB_RK4_4 = 5      // Uout = Un + 1/6 (K1 + 2 K2 + 2 K3 + dt L)
};

struct StageKind {
  int combine;
  double c;
};

inline int num_stages(int rk) { return rk == 1 ? 1 : rk == 2 ? 2 : rk == 3 ? 3 : 4; }

inline StageKind stage_kind(int rk, int s)
{
  switch (rk) {
  case 1: return {COMB_EULER, 0};
  case 2: return {s == 0 ? COMB_EULER : COMB_RK2_2, 0};
  case 3: return {s == 0 ? COMB_EULER : s == 1 ? COMB_RK3_2 : COMB_RK3_3, 0};
  default: return {s == 3 ? COMB_RK4_4 : COMB_RK4_K, s == 2 ? 1.0 : 0.5};
  }
}

struct TransferArgs {
  Grid g;
  AdvanceBuffers b;
  Ctl *ctl;
  cudaStream_t stream;
  int cur;   // committed buffer, for the halo copies of the committed state
  int lean = 0;        // lean layout: the committed state is (PA, U[cur]); see rmhd_lean.cuh
  double gamma = 0.0;  // for the lean upload's P->U
  int pending = 0;     // lean download of an advance's result before its commit (k_lean_download)
};

// One member of an ensemble of boxes (device-side descriptor).
struct BoxDev {
  Grid g;
  AdvanceBuffers b;
  Ctl *ctl;
  double min_dx;
};

// Launch arguments of an ensemble advance.
struct EnsembleArgs {
  const BoxDev *boxes;
  int nb, nd;
  const int2 *zone_map;              // per tile of interior zones: (box, tile within the box)
  const int2 *face_map[3];           // the same for the faces of each sweep direction
  long long zone_tiles, face_tiles[3];
  int zone_tile, face_tile;
  int grid_zone, grid_face, grid_c2p;
  long long total_zones, total_faces[3];   // work units, for the profiler
  PhysParams pp;
  int rk, ereset;
  double preset, dreset;
  int dt_mode;
  const double *dt;   // per box (device), dt_mode 0
  double cfl;
  int commit;         // 0: leave every box's committed state as it was (launch-shape timing)
  cudaStream_t stream;
  LaunchProfiler *prof;   // nullptr: no timing (never set while capturing a graph)
};

}  // namespace mgpu

// Entry points exported by each precision's translation unit.
#define MGPU_DECLARE_PRECISION(suffix)                                                                   \
  namespace mgpu {                                                                                       \
  cudaError_t advance_##suffix(const AdvanceArgs &A);                                                    \
  cudaError_t phase_##suffix(const AdvanceArgs &A, int phase, int s);                                    \
  cudaError_t upload_##suffix(const TransferArgs &A, const double *d_aos, long long z0, long long count); \
  cudaError_t download_##suffix(const TransferArgs &A, double *d_aos, long long z0, long long count);     \
  cudaError_t face_io_##suffix(const TransferArgs &A, double *d_aos, long long z0, long long count, int to_aos); \
  cudaError_t halo_##suffix(const TransferArgs &A, int which, int dim, int side, void *buf, int pack);   \
  cudaError_t ensemble_advance_##suffix(const EnsembleArgs &E);                                          \
  cudaError_t diffuse_##suffix(const AdvanceArgs &A, double r);                                          \
  }

