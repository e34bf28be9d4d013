// Lean layout of the method-of-lines advance: 3D FP32-bulk boxes too large for the standard
// layout's 304 bytes per zone (a 1024^3 box is 1030^3 guarded zones).
//
// Device arrays (144 bytes per zone in FP32 bulk):
//   PA      8 x T   stage primitives; between advances the committed primitives, exactly the
//                   c2p of U[cur] with every guard image filled
//   U[0..1] 5 x T + 3 x double   two conserved registers: U[cur] is the committed state,
//                   U[!cur] the Runge-Kutta register; a commit flips ctl->cur on the device
//   Bf      6 x T   the transverse magnetic face fluxes flux-CT reads: Fx[By], Fx[Bz], Fy[Bx],
//                   Fy[Bz], Fz[Bx], Fz[By], at the face's lower zone index
// No hydrodynamic face flux is stored: each sweep adds its flux differences to the register,
//   U1 = alpha U0 + beta U1 + gamma dt L,
// the x sweep with the combine, the y and z sweeps with += gamma dt L_d, and the field is
// updated by k_lean_ct from Bf afterwards (Mara/rmhd.cpp:311-381, Mara/runge-kutta.hpp).
//
// One advance: begin | per stage: c2p of U[!cur] -> PA (skipped at stage 1, where PA already
// holds the primitives of U[cur]) | sweeps x, y, z | CT | closing c2p of U[!cur] -> PA, and
// its field to U[!cur]'s guard images | commit (flip cur if nothing failed) | restore (after
// a failure: c2p of the unchanged U[cur] back into PA).
//
// Differences from the standard layout, all at FP32 rounding: the hydrodynamic flux
// differences are added sweep by sweep; an advance starts from the committed conserved state
// instead of P->U of the committed primitives; the first stage's primitives are the committed
// ones instead of their P->U->P round trip; MaxLambda is taken over the faces the interior
// update and CT read (the reference also visits faces of guard rows further out).
#pragma once
#include "rmhd_step.cuh"


namespace mgpu {

struct LeanCombine {   // U1 = alpha U0 + beta U1 + gamma dt L
  double alpha, beta, gamma;
  int first;           // 1: the x sweep applies the combine (0: y/z sweeps add)
  int euler;           // beta == 0: U1's previous contents are not read
};

__host__ __device__ inline LeanCombine lean_combine(int combine)
{
  switch (combine) {
  case COMB_RK2_2: return {0.5, 0.5, 0.5, 1, 0};
  case COMB_RK3_2: return {0.75, 0.25, 0.25, 1, 0};
  case COMB_RK3_3: return {1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0, 1, 0};
  default: return {1.0, 0.0, 1.0, 1, 1};
  }
}

template <class T>
__device__ __forceinline__ void lean_regs(const Ctl *ctl, StatePtr<T> UA, StatePtr<T> UB, StatePtr<T> &U0,
                                          StatePtr<T> &U1)
{
  U0 = ctl->cur ? UB : UA;
  U1 = ctl->cur ? UA : UB;
}

// Bf component written by a sweep of direction dim (1..3) for field component b (Bx..Bz).
__host__ __device__ constexpr int bf_slot(int dim, int b)
{
  return dim == 1 ? (b == By ? 0 : 1) : dim == 2 ? (b == Bx ? 2 : 3) : (b == Bx ? 4 : 5);
}

// Adds one direction's flux difference to interior zone z of the register (bulk components).
template <class T>
__device__ __forceinline__ void lean_accumulate(const Grid &g, StatePtr<T> U0, StatePtr<T> U1, long long z,
                                                const T *Flo, const T *Fhi, T inv_dx, const LeanCombine &c, T dt,
                                                bool first)
{
  const T gdt = T(c.gamma) * dt;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    const T L = -(Fhi[q] - Flo[q]) * inv_dx;
    T *u1 = U1.bulk + q * g.cs + z;
    if (first) {
      const T u0 = U0.bulk[q * g.cs + z];
      const T prev = c.euler ? T(0) : *u1;
      *u1 = T(c.alpha) * u0 + T(c.beta) * prev + gdt * L;
    } else {
      *u1 += gdt * L;
    }
  }
}

// ---- x and y sweeps: one thread per (column, chunk), marching along the sweep direction ---------
// Columns cover the two other dimensions with one zone of halo ([ng-1, ng+n] each: flux-CT
// reads transverse neighbours' face fields); a chunk is `chunk` zones of the sweep direction
// (lean_chunk picks it per launch).  The thread computes the lower face of its first zone, then per zone the upper
// face, and adds the difference to the zone when the column is interior.  Consecutive threads
// take consecutive k, so every load and store is coalesced.
template <class T, int dim, int RS>
__global__ void __launch_bounds__(128, MGPU_FLUX_MINB) k_lean_sweep(Grid g, const T *__restrict__ PA, StatePtr<T> UA,
                                                                    StatePtr<T> UB, T *__restrict__ Bf,
                                                                    LeanCombine c, PhysParams pp, Ctl *ctl, int stage,
                                                                    int chunk_len)
{
  static_assert(dim == 1 || dim == 2, "x or y sweep");
  if (stage_failed(ctl, stage + 1)) return;
  StatePtr<T> U0, U1;
  lean_regs(ctl, UA, UB, U0, U1);
  const int d = dim - 1;
  const int oa = dim == 1 ? 1 : 0;                  // the other two dimensions: a (outer), k (inner)
  // the window of x rows: the x sweep marches over its rows, the y sweep takes its columns
  // (rows a - 1 in [win_flo, win_fhi): its own and the halo rows it computes)
  const int alo = dim == 2 ? win_lo(g) : 0, ahi = dim == 2 ? win_hi(g) : g.n[oa];
  const int a0 = dim == 2 ? win_flo(g) + 1 : 0, na = dim == 2 ? win_fhi(g) - win_flo(g) : g.n[oa] + 2;
  const int mlo = dim == 1 ? win_lo(g) : 0, mhi = dim == 1 ? win_hi(g) : g.n[d];
  const int nk = g.n[2] + 2;
  const long long ncol = (long long) na * nk;
  const int nchunk = (mhi - mlo + chunk_len - 1) / chunk_len;
  const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  T ml = T(0);
  FluxTally ft{0, 0, 0, 0, 0};
  __shared__ T flo[128][5];   // the carried lower-face flux of each thread
  __shared__ HlldSlot<T> hslot[RS == RIEMANN_HLLD && sizeof(T) < sizeof(double) ? 128 : 1];
  if (t < ncol * nchunk) {
    const int chunk = (int) (t / ncol);
    const long long col = t - (long long) chunk * ncol;
    const int ar = (int) (col / nk), b = (int) (col - (long long) ar * nk);
    const int a = a0 + ar;
    const int ca = g.ng - 1 + a, k = g.ng - 1 + b;
    const bool interior = a >= alo + 1 && a <= ahi && b >= 1 && b <= g.n[2];
    const long long S = g.s[d];
    const long long base = (long long) ca * g.s[oa] + k;   // zone (0 along dim, ca, k)
    const int m0 = g.ng + mlo + chunk * chunk_len;
    const int m1 = min(m0 + chunk_len, g.ng + mhi);
    const T inv_dx = T(1.0 / (dim == 1 ? g.dx : g.dy));
    const T dt = T(ctl->dt);
    T *slot0 = Bf + (long long) bf_slot(dim, dim == 1 ? By : Bx) * g.cs;
    T *slot1 = Bf + (long long) bf_slot(dim, Bz) * g.cs;
#pragma unroll 1
    for (int m = m0 - 1; m < m1; ++m) {   // face between zones m and m + 1
      const long long f = base + (long long) m * S;
      if (m >= m0 && interior) {   // the register entries this face updates: into L2 while HLLD runs
#pragma unroll
        for (int q = 0; q < 5; ++q) {
          asm volatile("prefetch.global.L2 [%0];" ::"l"(U1.bulk + q * g.cs + f));
          if (dim == 1) asm volatile("prefetch.global.L2 [%0];" ::"l"(U0.bulk + q * g.cs + f));
        }
      }
      T Fo[8];
      face_flux<T, dim, RS>(g, PA, pp, f, ml, ft, Fo,
                            RS == RIEMANN_HLLD && sizeof(T) < sizeof(double) ? &hslot[threadIdx.x] : nullptr);
      if (m >= m0 || chunk == 0) {            // the chunk's first face is its neighbour's last
        slot0[f] = Fo[dim == 1 ? By : Bx];
        slot1[f] = Fo[Bz];
      }
      if (m >= m0 && interior) lean_accumulate<T>(g, U0, U1, f, flo[threadIdx.x], Fo, inv_dx, c, dt, dim == 1);
#pragma unroll
      for (int q = 0; q < 5; ++q) flo[threadIdx.x][q] = Fo[q];
    }
  }
  flux_block_finish(double(ml), ft, ctl, RS == RIEMANN_HLLD);
}

// ---- z sweep (contiguous direction): 128 consecutive faces per CTA, shared-memory pairing ------
// Rows are (i, j) with one zone of halo; a row holds the n2 + 1 faces [ng-1, ng+n2-1].  The
// faces of all rows are numbered consecutively; CTA c computes faces 127 c - 1 .. 127 c + 126
// and updates the zones whose both faces it holds (its first face is the previous CTA's last).
template <class T, int RS>
__global__ void __launch_bounds__(128, MGPU_FLUX_MINB) k_lean_sweep_z(Grid g, const T *__restrict__ PA, StatePtr<T> UA,
                                                                      StatePtr<T> UB, T *__restrict__ Bf,
                                                                      LeanCombine c, PhysParams pp, Ctl *ctl,
                                                                      int stage)
{
  if (stage_failed(ctl, stage + 1)) return;
  StatePtr<T> U0, U1;
  lean_regs(ctl, UA, UB, U0, U1);
  const int nf = g.n[2] + 1, nj = g.n[1] + 2;
  // the window's x rows and the halo rows it computes: a - 1 in [win_flo, win_fhi)
  const int alo = win_lo(g), ahi = win_hi(g), a0 = win_flo(g) + 1;
  const long long total = (long long) (win_fhi(g) - win_flo(g)) * nj * nf;
  const long long q = (long long) blockIdx.x * 127 - 1 + threadIdx.x;
  T ml = T(0);
  FluxTally ft{0, 0, 0, 0, 0};
  __shared__ T fs[5][128];
  __shared__ HlldSlot<T> hslot[RS == RIEMANN_HLLD && sizeof(T) < sizeof(double) ? 128 : 1];
  const bool active = q >= 0 && q < total;
  long long f = 0;
  bool upd = false;
  if (active) {
    const long long row = q / nf;
    const int fk = (int) (q - row * nf);              // face fk + ng - 1
    const int ar = (int) (row / nj), b = (int) (row - (long long) ar * nj);
    const int a = a0 + ar;
    const int i = g.ng - 1 + a, j = g.ng - 1 + b;
    f = (long long) i * g.s[0] + (long long) j * g.s[1] + (g.ng - 1 + fk);
#pragma unroll
    for (int r = 0; r < 5; ++r) asm volatile("prefetch.global.L2 [%0];" ::"l"(U1.bulk + r * g.cs + f));
    T Fo[8];
    face_flux<T, 3, RS>(g, PA, pp, f, ml, ft, Fo,
                        RS == RIEMANN_HLLD && sizeof(T) < sizeof(double) ? &hslot[threadIdx.x] : nullptr);
    if (threadIdx.x > 0 || blockIdx.x == 0) {
      Bf[(long long) bf_slot(3, Bx) * g.cs + f] = Fo[Bx];
      Bf[(long long) bf_slot(3, By) * g.cs + f] = Fo[By];
    }
#pragma unroll
    for (int r = 0; r < 5; ++r) fs[r][threadIdx.x] = Fo[r];
    upd = threadIdx.x > 0 && fk >= 1 && a >= alo + 1 && a <= ahi && b >= 1 && b <= g.n[1];
  }
  __syncthreads();
  if (upd) {
    T lo[5], hi[5];
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      lo[r] = fs[r][threadIdx.x - 1];
      hi[r] = fs[r][threadIdx.x];
    }
    lean_accumulate<T>(g, U0, U1, f, lo, hi, T(1.0 / g.dz), c, T(ctl->dt), false);
  }
  flux_block_finish(double(ml), ft, ctl, RS == RIEMANN_HLLD);
}

// ---- flux-CT of the field from Bf, FP64 (ConstrainedTransport3d, Mara/rmhd.cpp:311-381) ------
template <class T>
__device__ __forceinline__ double lean_emf(const T *F, const T *G, long long z, long long sa, long long sb)
{
  return (2 * double(F[z]) + double(F[z + sb]) + double(F[z - sb]) - double(G[z]) - double(G[z + sa]) -
          double(G[z - sb]) - double(G[z + sa - sb])) * 0.125;
}

// The field update of one interior zone z: U1.B = combine(U0.B, U1.B, dt L), L the divergence
// of the twelve corner EMFs around it (the zeroed normal fluxes dropped, 1/dx from the host).
template <class T>
__device__ __forceinline__ void lean_ct_zone(const Grid &g, int combine, StatePtr<T> U0, StatePtr<T> U1,
                                             const T *__restrict__ Bf, double dtd, double3 inv, long long z)
{
  const long long sx = g.s[0], sy = g.s[1], sz = g.s[2];
  const T *xBy = Bf + 0 * g.cs, *xBz = Bf + 1 * g.cs, *yBx = Bf + 2 * g.cs, *yBz = Bf + 3 * g.cs,
          *zBx = Bf + 4 * g.cs, *zBy = Bf + 5 * g.cs;
  const double FxBy0 = lean_emf(xBy, yBx, z, sx, sy), FxBym = lean_emf(xBy, yBx, z - sx, sx, sy);
  const double FyBx0 = lean_emf(yBx, xBy, z, sy, sx), FyBxm = lean_emf(yBx, xBy, z - sy, sy, sx);
  const double FyBz0 = lean_emf(yBz, zBy, z, sy, sz), FyBzm = lean_emf(yBz, zBy, z - sy, sy, sz);
  const double FzBy0 = lean_emf(zBy, yBz, z, sz, sy), FzBym = lean_emf(zBy, yBz, z - sz, sz, sy);
  const double FzBx0 = lean_emf(zBx, xBz, z, sz, sx), FzBxm = lean_emf(zBx, xBz, z - sz, sz, sx);
  const double FxBz0 = lean_emf(xBz, zBx, z, sx, sz), FxBzm = lean_emf(xBz, zBx, z - sx, sx, sz);
  double Lb[3];
  Lb[0] = -(FyBx0 - FyBxm) * inv.y - (FzBx0 - FzBxm) * inv.z;
  Lb[1] = -(FxBy0 - FxBym) * inv.x - (FzBy0 - FzBym) * inv.z;
  Lb[2] = -(FxBz0 - FxBzm) * inv.x - (FyBz0 - FyBzm) * inv.y;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const double un = U0.B[q * g.cs + z];
    double out;
    switch (combine) {
    case COMB_RK2_2: out = 0.5 * (un + U1.B[q * g.cs + z] + dtd * Lb[q]); break;
    case COMB_RK3_2: out = 3. / 4 * un + 1. / 4 * U1.B[q * g.cs + z] + 1. / 4 * dtd * Lb[q]; break;
    case COMB_RK3_3: out = 1. / 3 * un + 2. / 3 * U1.B[q * g.cs + z] + 2. / 3 * dtd * Lb[q]; break;
    default: out = un + dtd * Lb[q]; break;
    }
    U1.B[q * g.cs + z] = out;
  }
}

// Two zones per thread, neighbours along the contiguous axis: their EMF stencils share most
// operands (and two EMFs: zone k+1's lower z-EMFs are zone k's upper ones), which the compiler
// loads and widens once.  Each zone's arithmetic is lean_ct_zone's.
template <class T>
__global__ void __launch_bounds__(256, MGPU_UPDATE_MINB) k_lean_ct(Grid g, int combine, StatePtr<T> UA, StatePtr<T> UB,
                                                                   const T *__restrict__ Bf, const Ctl *ctl,
                                                                   int stage, double3 inv)
{
  if (stage_failed(ctl, stage + 1)) return;
  const long long npair = (g.n[2] + 1) / 2;
  const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long) win_rows(g) * g.n[1] * npair) return;
  StatePtr<T> U0, U1;
  lean_regs(ctl, UA, UB, U0, U1);
  const int kp = (int) (t % npair);
  const long long ij = t / npair;
  const int j = (int) (ij % g.n[1]), i = win_lo(g) + (int) (ij / g.n[1]);
  const int k = 2 * kp;
  const long long z = ((long long) (i + g.ng) * g.G[1] + (j + g.ng)) * g.G[2] + (k + g.ng);
  const double dtd = ctl->dt;
  lean_ct_zone<T>(g, combine, U0, U1, Bf, dtd, inv, z);
  if (k + 1 < g.n[2]) lean_ct_zone<T>(g, combine, U0, U1, Bf, dtd, inv, z + 1);
}

// Threads of k_lean_ct for a grid's window (two zones along k each).
inline long long lean_ct_threads(const Grid &g) { return (long long) win_rows(g) * g.n[1] * ((g.n[2] + 1) / 2); }

// ---- commit of the lean layout ------------------------------------------------------------------
// As k_commit, then the restore c2p (C2P_LEAN_RESTORE) runs when nothing was committed.

// ---- host <-> lean committed state ---------------------------------------------------------------
// Upload of a range of zones of the AoS primitives: each interior zone goes to PA and its
// periodic images (along the dimensions this grid fills itself; a decomposed block's split
// dimensions get their guards from the exchange), P->U of its FP64 primitives to U[cur]
// (field to the images too); guard
// zones of the range are skipped (their images come from the interior zones, as the
// reference's PrimToCons fills guards before converting, Mara/hydro.cpp:112-123).
template <class T>
__global__ void k_lean_upload(Grid g, const double *__restrict__ aos, long long z0, long long count, T *PA,
                              StatePtr<T> UA, StatePtr<T> UB, double gamma, const Ctl *ctl)
{
  const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const long long z = z0 + t;
  int i, j, k;
  zone_coords(g, z, i, j, k);
  if (i < g.ng || i >= g.ng + g.n[0] || j < g.ng || j >= g.ng + g.n[1] || k < g.ng || k >= g.ng + g.n[2]) return;
  const StatePtr<T> U = ctl->cur ? UB : UA;
  double p[8], u[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) p[q] = aos[t * 8 + q];
  prim_to_cons(gamma, p, u);
#pragma unroll
  for (int q = 0; q < 5; ++q) U.bulk[q * g.cs + z] = T(u[q]);
  int pi[3], pj[3], pk[3];
  const int ni = images_1d(i, g.n[0], g.ng, self_periodic(g, 0), pi);
  const int nj = images_1d(j, g.n[1], g.ng, self_periodic(g, 1), pj);
  const int nk = images_1d(k, g.n[2], g.ng, self_periodic(g, 2), pk);
  for (int a = 0; a < ni; ++a)
    for (int b = 0; b < nj; ++b)
      for (int c = 0; c < nk; ++c) {
        const long long w = ((long long) pi[a] * g.G[1] + pj[b]) * g.G[2] + pk[c];
#pragma unroll
        for (int q = 0; q < 8; ++q) PA[q * g.cs + w] = T(p[q]);
#pragma unroll
        for (int q = 0; q < 3; ++q) U.B[q * g.cs + w] = u[5 + q];
      }
}

// Download: the committed primitives are PA's bulk components and U[cur]'s field.  pending = 1
// reads an advance's result before its commit: after the closing c2p, PA's bulk components and
// the field of the register U[!cur].
template <class T>
__global__ void k_lean_download(Grid g, double *__restrict__ aos, long long z0, long long count, const T *PA,
                                StateCPtr<T> UA, StateCPtr<T> UB, const Ctl *ctl, int pending)
{
  const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const long long z = z0 + t;
  const StateCPtr<T> U = (ctl->cur ^ pending) ? UB : UA;
#pragma unroll
  for (int q = 0; q < 5; ++q) aos[t * 8 + q] = double(PA[q * g.cs + z]);
#pragma unroll
  for (int q = 0; q < 3; ++q) aos[t * 8 + 5 + q] = U.B[q * g.cs + z];
}

// ---- launch sequence ---------------------------------------------------------------------------
// Chunk length of a marching sweep over ncol columns of n zones: every chunk costs one face
// more than its zones, and the launch takes ceil(threads / resident threads) waves of
// chunk + 1 faces each, so pick the length in [16, 64] that minimises their product.
inline int lean_chunk(long long ncol, int n, long long resident_threads)
{
  int best = 32;
  double best_cost = 1e300;
  for (int L = 16; L <= 64; ++L) {
    const long long nchunk = (n + L - 1) / L;
    const long long Lr = (n + nchunk - 1) / nchunk;   // the longest chunk with this count
    if (Lr != L) continue;
    const long long threads = ncol * nchunk;
    const double cost = (double) ((threads + resident_threads - 1) / resident_threads) * (double) (L + 1);
    if (cost < best_cost) {
      best_cost = cost;
      best = L;
    }
  }
  return best;
}

template <class T>
inline void launch_lean_sweep(const Grid &g, int dim, int rs, cudaStream_t st, const T *PA, StatePtr<T> UA,
                              StatePtr<T> UB, T *Bf, const LeanCombine &c, const PhysParams &pp, Ctl *ctl, int s)
{
  const unsigned blk = 128;
  if (dim == 3) {
    const long long total = (long long) (win_fhi(g) - win_flo(g)) * (g.n[1] + 2) * (g.n[2] + 1);
    const unsigned grid = (unsigned) ((total + 126) / 127);
#define MGPU_LEANZ_CASE(R) \
  if (rs == R) { k_lean_sweep_z<T, R><<<grid, blk, 0, st>>>(g, PA, UA, UB, Bf, c, pp, ctl, s); return; }
    MGPU_LEANZ_CASE(RIEMANN_HLLD) MGPU_LEANZ_CASE(RIEMANN_HLLC) MGPU_LEANZ_CASE(RIEMANN_HLL)
#undef MGPU_LEANZ_CASE
    return;
  }
  // x sweep: columns over (y, z), marching over the window's rows; y sweep: columns over the
  // window's rows (one halo row each side) and z, marching over y
  const long long ncol = dim == 1 ? (long long) (g.n[1] + 2) * (g.n[2] + 2)
                                  : (long long) (win_fhi(g) - win_flo(g)) * (g.n[2] + 2);
  const int nmarch = dim == 1 ? win_rows(g) : g.n[1];
  const int L = lean_chunk(ncol, nmarch, 148ll * MGPU_FLUX_MINB * blk);
  const long long nchunk = (nmarch + L - 1) / L;
  const unsigned grid = (unsigned) ((ncol * nchunk + blk - 1) / blk);
#define MGPU_LEAN_CASE(D, R) \
  if (dim == D && rs == R) { k_lean_sweep<T, D, R><<<grid, blk, 0, st>>>(g, PA, UA, UB, Bf, c, pp, ctl, s, L); return; }
  MGPU_LEAN_CASE(1, RIEMANN_HLLD) MGPU_LEAN_CASE(2, RIEMANN_HLLD)
  MGPU_LEAN_CASE(1, RIEMANN_HLLC) MGPU_LEAN_CASE(2, RIEMANN_HLLC)
  MGPU_LEAN_CASE(1, RIEMANN_HLL) MGPU_LEAN_CASE(2, RIEMANN_HLL)
#undef MGPU_LEAN_CASE
}

}  // namespace mgpu
