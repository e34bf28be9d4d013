// The solver handle behind the C ABI (shared by the host translation units of libmaragpu.so).
#pragma once
#include <cuda_runtime.h>
#include <string>
#include <vector>

#include "../../include/mara_gpu.h"
#include "rmhd_types.cuh"

struct MgpuDriving;   // OU driving field (driving.cu)
class HostCopyPool;   // threaded host copies (host_copy.h)

struct mgpu_solver {
  mgpu_config cfg;
  std::string err;
  bool have_domain = false;
  mgpu::Grid g{};
  double x0[3] = {0, 0, 0}, x1[3] = {1, 1, 1};
  double min_dx = 1.0;
  int N[3] = {1, 1, 1};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int device = 0;
  mgpu::AdvanceBuffers b{};
  std::vector<void *> allocations;
  mgpu::Ctl *ctl = nullptr;           // device
  mgpu::Ctl *ctl_host = nullptr;      // pinned mirror
  double *staging = nullptr;    // device AoS staging for host transfers
  long long staging_zones = 0;
  double *red = nullptr;        // reduction partials (device)
  double *red_host = nullptr;   // pinned
  double *meas = nullptr;       // per-block partials of the measures (device)
  double *meas_host = nullptr;  // pinned
  unsigned char *fmask = nullptr;   // failure mask of the last c2p (device, guarded zones)
  float *mlp = nullptr;         // learned c2p network (device)
  long long mlp_count = 0;
  void *mlp_tc = nullptr;       // its tensor-core image (device)
  int *mult = nullptr;          // multiplicity tables of a decomposed domain (device)
  MgpuDriving *driving = nullptr;   // velocity forcing applied after each committed advance
  // kernel timing
  std::vector<cudaEvent_t> prof_ev;
  std::vector<int> prof_tag;
  std::vector<long long> prof_units;
  int prof_count = 0;
  mgpu::LaunchProfiler prof{};
  bool prof_on = false;
  // pipelined mgpu_advance_host (lean layout): device copies of the AoS buffer in and out, a
  // second stage-primitive array, the learned c2p's guesses, copy streams and per-slab events
  int pipe_slabs = -1;          // 0 off, -1 automatic, else the slab count
  int pipe_last = 0;            // slabs of the last mgpu_advance_host (0: unpipelined)
  int pipe_state = 0;           // 0 not set up, 1 ready, -1 not enough device memory
  double *pipe_in = nullptr, *pipe_out = nullptr;
  void *pipe_guess = nullptr, *pipe_pa = nullptr;
  cudaStream_t pipe_h2d = nullptr, pipe_d2h = nullptr;
  std::vector<cudaEvent_t> pipe_ev;
  // a pageable caller buffer is staged through this pinned copy of the AoS buffer, its host
  // copies spread over the pool's threads (0 / -1: not set up / not available)
  double *pipe_host = nullptr;
  int pipe_host_state = 0;
  HostCopyPool *pipe_pool = nullptr;
  // the plain host transfers of a large pageable buffer: two pinned chunk slots and their events
  double *xfer_host = nullptr;
  int xfer_host_state = 0;
  std::vector<cudaEvent_t> xfer_ev;
};


// Enqueues the driving kick of the just-committed state (no-op without a driving field or
// when the advance did not commit); defined in driving.cu.
cudaError_t mgpu_driving_enqueue(mgpu_solver *h);
void mgpu_driving_free(mgpu_solver *h);
