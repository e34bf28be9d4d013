/* mara_gpu.h -- C ABI of the B200 RMHD step (libmaragpu.so).
 *
 * A drop-in for the CPU advance behind the reference's Lua module `Mara`
 * (Mara/mara.cpp:137-268, registered by ctf-core/ctf.c:139).  Plain C types only: host
 * pointers, device pointers as void*, sizes, int status codes (0 = ok, never an exception
 * or longjmp across the boundary).  One handle = one solver = one CUDA stream; calls on one
 * handle are not thread-safe, separate handles are independent (unlike the reference, whose
 * solver is a process-global singleton, Mara/mara.cpp:135).
 *
 * Layout at the boundary is the reference's: AoS float64 primitives with guard zones,
 * ((i*G1 + j)*G2 + k)*8 + q, q = rho, pre, vx, vy, vz, Bx, By, Bz (Mara/rmhd.hpp:20),
 * G_d = N_d + 2*Ng.
 */
#ifndef MARA_GPU_H
#define MARA_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mgpu_solver mgpu_solver;

enum { MGPU_OK = 0, MGPU_ERR_ARG = 1, MGPU_ERR_STATE = 2, MGPU_ERR_CUDA = 3, MGPU_ERR_NOMEM = 4,
       MGPU_ERR_UNSUPPORTED = 5 };

enum { MGPU_FLUID_RMHD = 0 };
enum { MGPU_RECON_PCM = 0, MGPU_RECON_PLM = 1, MGPU_RECON_WENO5 = 2 };
enum { MGPU_RIEMANN_HLL = 0, MGPU_RIEMANN_HLLC = 1, MGPU_RIEMANN_HLLD = 2 };
enum { MGPU_IS_JS96 = 0, MGPU_IS_B08 = 1, MGPU_IS_SZ10 = 2 };
enum { MGPU_PREC_FP64 = 0, MGPU_PREC_FP32 = 1 };
enum { MGPU_GODUNOV_PLM_SPLIT = 0, MGPU_GODUNOV_PLM_MUSCL = 1 };
enum { MGPU_LAYOUT_STANDARD = 0, MGPU_LAYOUT_LEAN = 1 };
#define MGPU_KERNEL_CLASSES 6

/* Solver selection: the union of Mara.set_fluid/set_eos/set_godunov/set_riemann/set_advance
 * and the keys of Mara.config_solver (Mara/mara.cpp:813-1167). */
typedef struct {
  int    fluid;        /* MGPU_FLUID_RMHD (set_fluid('rmhd')) */
  double gamma;        /* set_eos('gamma-law', gamma) */
  int    recon;        /* config_solver{extrap = 'pcm' | 'plm' | 'weno5'} */
  double theta;        /* config_solver{theta} (PLM minmod) */
  int    is_mode;      /* config_solver{IS = 'js96' | 'b08' | 'sz10'} */
  double sz10A;        /* config_solver{sz10A} */
  int    riemann;      /* set_riemann('hll' | 'hllc' | 'hlld') */
  int    rk;           /* set_advance: 1 'single', 2 'rk2', 3 'rk3', 4 'rk4' */
  double pfloor;       /* config_solver{pfloor}, disabled when <= 0 */
  int    ereset;       /* config_solver{ereset} */
  double preset;       /* config_solver{preset} */
  double dreset;       /* config_solver{dreset} */
  int    precision;    /* MGPU_PREC_FP64: plain path, reference arithmetic;
                          MGPU_PREC_FP32: FP32 bulk, FP64 c2p polish / magnetic field / dt */
  int    learned_c2p;  /* 1: first c2p attempt starts from the network set by
                          mgpu_set_c2p_network (Newton polish, reference ladder as fallback) */
  int    godunov;      /* set_godunov: MGPU_GODUNOV_PLM_SPLIT 'plm-split' (method of lines,
                          reconstruction `recon`, MethodOfLinesSplit, Mara/plm-split.cpp) or
                          MGPU_GODUNOV_PLM_MUSCL 'plm-muscl' (CTU-Hancock with PLM slopes of
                          limiter `theta`, PlmCtuHancockOperator, Mara/ctu-hancock.cpp:53-494;
                          single domains only: not with external guards, ensembles or
                          mgpu_advance_noalloc) */
  int    layout;       /* device memory layout (no counterpart in the reference, whose state
                          is host memory).  MGPU_LAYOUT_STANDARD: stored face fluxes, two
                          committed primitive buffers (304 B per guarded zone in FP32 bulk,
                          512 B in FP64).  MGPU_LAYOUT_LEAN: 3D boxes too large for that
                          (a 1024^3 FP32-bulk box): the sweeps add their flux differences
                          straight into the Runge-Kutta register and only the six transverse
                          face fields are stored (144 B per zone in FP32 bulk, 240 B in FP64).
                          Lean needs nd = 3, 'plm-split' and rk 1-3 (decomposed blocks
                          exchange their stage primitives, which 0, every stage); results
                          agree with the standard layout to the bulk type's rounding, the
                          magnetic field and its divergence stay FP64 as there; after a failed
                          advance the primitives are the c2p of the unchanged conserved state;
                          the stage array holds the committed primitives, so
                          mgpu_set_primitive uploads the committed state. */
} mgpu_config;

typedef struct {
  double max_lambda;          /* RiemannSolver::MaxLambda of the last advance */
  double dt;                  /* dt of the last advance */
  int    errors;              /* failed zones of the last advance (as Mara.advance returns) */
  int    committed;           /* 1 if the last advance replaced the primitive state */
  unsigned long long c2p_calls, c2p_iters;          /* zone c2p calls and Newton iterations */
  unsigned long long c2p_attempt[6];                /* attempts used: [1..4] ladder rung,
                                                       [5] learned guess rejected */
  unsigned long long face_c2p_calls, face_c2p_iters; /* HLL-state c2p inside HLLD */
  unsigned long long hlld_ok, hlld_hllc, pcm_retry;  /* HLLD successes / HLLC fallbacks /
                                                        PCM retries of a face */
  unsigned long long c2p_failed;                     /* zone c2p calls that failed every rung of the
                                                        ladder (emergency resets included) */
  unsigned long long advances, failed_advances,      /* since mgpu_set_domain: advances run, those */
                     failed_zones;                   /* not committed, and the failed zones
                                                        they reported (sum of their `errors`) */
} mgpu_stats;

/* Defaults of a freshly started reference plus set_fluid('rmhd'), gamma 4/3, PLM theta 2,
 * HLLD, RK2, FP64 (Mara/hydro.cpp:18-32,70-78; Mara/weno.c:10-12; Mara/rmhd-c2p.c:104). */
int mgpu_default_config(mgpu_config *cfg);

/* replaces luaC_Mara_start (Mara/mara.cpp:271-287) + the set_* selectors */
int mgpu_create(const mgpu_config *cfg, mgpu_solver **out);
/* replaces luaC_Mara_close (Mara/mara.cpp:288-295) */
int mgpu_destroy(mgpu_solver *h);
/* Use an existing CUDA stream (cudaStream_t passed as void*); NULL = the handle's own. */
int mgpu_set_stream(mgpu_solver *h, void *stream);
const char *mgpu_last_error(const mgpu_solver *h);

/* replaces luaC_set_domain (Mara/mara.cpp:726-755): x0/x1/N have nd entries; nq must be 8;
 * periodic boundaries (set_boundary('periodic')) with N_d >= ng on every axis. */
int mgpu_set_domain(mgpu_solver *h, const double *x0, const double *x1, const int *N, int nd, int nq,
                    int ng);
/* SimpleCartesianDomain::GetNumberOfZones (guard zones included, Mara/simple-cart.hpp:31) */
int mgpu_num_zones(const mgpu_solver *h, long long *nzones);

/* Primitive state (AoS with guard zones, nzones*8 doubles).  Host or device pointers. */
int mgpu_upload_prim(mgpu_solver *h, const double *host_aos);
int mgpu_download_prim(mgpu_solver *h, double *host_aos);
int mgpu_upload_prim_device(mgpu_solver *h, const void *dev_aos);
int mgpu_download_prim_device(mgpu_solver *h, void *dev_aos);
/* The same for zones [z0, z0 + count) of the guarded AoS array (host pointer to count*8
 * doubles), so that a box larger than host memory allows is filled or read slab by slab (no
 * counterpart in the reference, whose Mara.init_prim fills one host buffer).  In the lean
 * layout an upload takes the interior zones of the range and fills their periodic guard
 * images; guard zones of the range are ignored. */
int mgpu_upload_prim_range(mgpu_solver *h, const double *host_aos, long long z0, long long count);
int mgpu_download_prim_range(mgpu_solver *h, double *host_aos, long long z0, long long count);

/* replaces luaC_Mara_advance (Mara/mara.cpp:297-341) on the device-resident state:
 * returns in *errors the number of failed zones (state unchanged when > 0).  Synchronous. */
int mgpu_advance(mgpu_solver *h, double dt, int *errors);
/* Mara.advance(buf, dt) exactly: copies the host buffer in, advances, copies it back when
 * errors == 0; *kzps is 1e-3 * zones (guards included) / wall seconds of the call.
 * In the 3-D lean layout the call is pipelined over slabs of x rows when device memory allows
 * (two device copies of the AoS buffer and a second stage-primitive array): the copy in, the
 * advance's stages and the copy out of different slabs overlap.  The result is the same as
 * the unpipelined call's, bit for bit, and when the advance fails the buffer gets its original
 * contents back.  A pageable buffer is staged through a pinned host copy that the solver
 * allocates on its first such call, with the host copies on a few threads of its own. */
int mgpu_advance_host(mgpu_solver *h, double *host_aos, double dt, double *kzps, int *errors);
/* Slab count of the pipelined mgpu_advance_host: 0 off, -1 automatic (the default; see
 * mgpu_pipeline_bounds), >= 3 that many equal slabs (at least 4 x rows each).  *last_slabs
 * (may be NULL) gets the count the previous mgpu_advance_host used, 0 when it ran
 * unpipelined. */
int mgpu_set_pipeline(mgpu_solver *h, int slabs);
int mgpu_get_pipeline(const mgpu_solver *h, int *slabs, int *last_slabs);
/* The pipelined advance's issue order for `slabs` slabs and `stages` Runge-Kutta stages, as
 * (slab, operation) pairs into out[2*i], out[2*i+1] (operation 0 the upload, 2k+1 stage k's
 * sweeps and CT, 2k stage k's c2p -- 2*stages the closing one -- and 2*stages+1 the download).
 * Returns the number of pairs (out may be NULL), or -MGPU_ERR_ARG.  Needs no GPU. */
int mgpu_pipeline_schedule(int slabs, int stages, int *out, int capacity);
/* The slabs the pipelined advance cuts n0 interior x rows into for a slab setting (-1 or >= 3):
 * bounds[0..S] (slab s is rows [bounds[s], bounds[s+1])).  Automatic: from 96 rows, slabs of 16
 * rows and thin ones of 6 around slab 0 and around the far side; below, about 11 rows each.
 * Returns S (0: too few rows to pipeline; bounds may be NULL), or -MGPU_ERR_ARG.  Needs no GPU. */
int mgpu_pipeline_bounds(int n0, int slabs, int *bounds, int capacity);
/* Enqueue n advances without host synchronisation: dt_mode 0 uses `dt` for every step,
 * dt_mode 1 takes each step's dt = cfl*min_dx/MaxLambda of the step before (the first step
 * uses the MaxLambda left by the previous advance).  A step that fails is not committed;
 * later steps then restart from the last committed state.  Read the outcome with
 * mgpu_get_stats after mgpu_synchronize. */
int mgpu_advance_async(mgpu_solver *h, int n, int dt_mode, double dt, double cfl);
int mgpu_synchronize(mgpu_solver *h);

/* replaces luaC_Mara_get_timestep (Mara/mara.cpp:374-381) */
int mgpu_get_timestep(mgpu_solver *h, double cfl, double *dt);
int mgpu_get_stats(mgpu_solver *h, mgpu_stats *stats);

/* Mara.set_primitive (Mara/mara.cpp:1284-1295): sets the array the measures read. */
int mgpu_set_primitive(mgpu_solver *h, const double *host_aos);
/* Mara.measure.mean_max_divB / max_lorentz_factor (Mara/mara.cpp:2232-2324) on the
 * measured primitive array (the last RK stage's primitives after an advance, as in the
 * reference, or the array given to mgpu_set_primitive). */
int mgpu_measure_divB(mgpu_solver *h, double *mean, double *max);
int mgpu_max_lorentz_factor(mgpu_solver *h, double *wmax);
/* The same corner divergence on the committed state, whose magnetic field is FP64 in both
 * precisions (the FP32-bulk path keeps B, its CT update and ∇·B in FP64). */
int mgpu_measure_divB_state(mgpu_solver *h, double *mean, double *max);

/* The other measures of Mara.measure (Mara/mara.cpp:1954-2230), on the same measured
 * primitive array as mgpu_measure_divB: means over the interior zones (sums divided by the
 * global interior zone count, as the reference's TTL_ZONES), extremes over them.  Units are
 * the reference's default PhysicalUnits(1, 1, 1) (Mara/hydro.cpp:20).  One device pass per
 * call; each per-zone value in the reference's operation order, the sums in another order.
 *   mean_cons       out[8]  mean of P->U                      (luaC_mean_cons)
 *   mean_prim       out[8]  mean of the primitives            (luaC_mean_prim)
 *   mean_energies   out[4]  magnetic, kinetic, internal, total (luaC_mean_energies)
 *   mean_velocity   out[4]  mean W, |vx|, |vy|, |vz|          (luaC_mean_velocity)
 *   mean_max_temperature     mean, max of T in MeV            (luaC_mean_max_temperature)
 *   mean_max_magnetic_field  mean, max of |B| in Gauss        (luaC_mean_max_magnetic_field)
 *   mean_max_sonic_mach      mean, max of the sonic Mach number (luaC_mean_max_sonic_mach)
 *   mean_min_alfvenic_mach   mean, min of the Alfvenic Mach number (luaC_mean_min_alfvenic_mach) */
int mgpu_measure_mean_cons(mgpu_solver *h, double *out);
int mgpu_measure_mean_prim(mgpu_solver *h, double *out);
int mgpu_measure_mean_energies(mgpu_solver *h, double *out);
int mgpu_measure_mean_velocity(mgpu_solver *h, double *out);
int mgpu_measure_mean_max_temperature(mgpu_solver *h, double *mean, double *max);
int mgpu_measure_mean_max_magnetic_field(mgpu_solver *h, double *mean, double *max);
int mgpu_measure_mean_max_sonic_mach(mgpu_solver *h, double *mean, double *max);
int mgpu_measure_mean_min_alfvenic_mach(mgpu_solver *h, double *mean, double *min);

/* replaces luaC_Mara_diffuse (Mara/mara.cpp:343-366): the committed state becomes c2p of
 * P->U(P) + GodunovOperator::LaxDiffusion(U, r) (Mara/hydro.cpp:205-283) -- Lax-Friedrichs
 * fluxes of strength r on the faces next to zones that failed the last c2p (the failure mask
 * of the last advance or diffuse, or of mgpu_set_failmask), with flux-CT -- with the measured
 * primitive array as the c2p's previous state; that array is left unchanged and the mask
 * becomes this c2p's.  *errors = the failed zones of that c2p (the reference discards the
 * count).  Standard layout, single domain.  Synchronous. */
int mgpu_diffuse(mgpu_solver *h, double r, int *errors);
/* Mara.diffuse(buf, r) exactly: the host buffer is copied in, diffused and copied back. */
int mgpu_diffuse_host(mgpu_solver *h, double *host_aos, double r, int *errors);
/* replaces luaC_Mara_set_failmask (Mara/mara.cpp:368-373): every zone's mask entry = value. */
int mgpu_set_failmask(mgpu_solver *h, int value);
/* Changes the scheme of a solver in place (the set_riemann / set_advance / set_godunov /
 * config_solver calls of the reference's crash ladders, e.g. ctf-core/drvtrb.lua:276-352),
 * keeping its state, MaxLambda, failure mask, measured array and driving field, as the
 * reference's process-wide solver keeps them.  The fluid, precision and layout cannot change
 * (MGPU_ERR_UNSUPPORTED: create a new solver); arrays the new scheme needs (RK4 registers,
 * CTU-Hancock predictions) are allocated here. */
int mgpu_reconfigure(mgpu_solver *h, const mgpu_config *cfg);

/* Kernel timing (no counterpart in the reference): while enabled, every kernel launch of an
 * advance is bracketed by CUDA events on the handle's stream.  Classes (MGPU_KERNEL_CLASSES):
 * 0 begin/commit, 1 P->U, 2 c2p, 3 flux sweep, 4 CT+divergence+RK update, 5 CTU-Hancock
 * predictor (half-step states and their c2p).  mgpu_profile_read synchronizes and returns per
 * class, in arrays of MGPU_KERNEL_CLASSES entries, the summed milliseconds, the number of
 * launches and the work units (faces for the flux class, zones otherwise); it then starts a
 * new window. */
int mgpu_profile_enable(mgpu_solver *h, int capacity);
int mgpu_profile_disable(mgpu_solver *h);
int mgpu_profile_read(mgpu_solver *h, double *ms, long long *launches, long long *units);

/* Learned c2p initial guess (no counterpart in the reference).  A 5 -> 64 -> 64 -> 64 -> 2
 * tanh network maps scale-free features of the c2p invariants (D, tau, S^2, B^2, (S.B)^2)
 * to (log W, log h); the FP64 Newton polish starts there and the reference's ladder runs if
 * it fails.  Packed float32 parameters (mgpu_mlp_param_count of them; layout in
 * ctf_b200/csrc/c2p_mlp_net.cuh).  All pointers named dev_* are device pointers. */
int mgpu_set_c2p_network(mgpu_solver *h, const float *params, long long count);
int mgpu_mlp_param_count(void);
/* (features, targets) of every interior zone of the committed state: n = interior zones,
 * dev_x n x 5 floats, dev_y n x 2 floats (log W, log h). */
int mgpu_c2p_harvest(mgpu_solver *h, float *dev_x, float *dev_y, long long capacity, long long *count);
/* Scratch for mgpu_mlp_loss_grad / mgpu_mlp_train over `batch` samples, in floats. */
long long mgpu_mlp_work_floats(long long batch);
/* Mean squared error of the standardised outputs over n samples and its gradient with
 * respect to the trainable parameters (deterministic order). */
int mgpu_mlp_loss_grad(const float *dev_params, const float *dev_x, const float *dev_y, long long n,
                       float *dev_grad, float *dev_work, double *loss);
/* `steps` minibatch Adam steps (batch samples each, learning rate lr; step0 = steps taken
 * before, for the bias corrections and the data walk); *last_loss = last minibatch loss. */
int mgpu_mlp_train(float *dev_params, float *dev_m, float *dev_v, const float *dev_x, const float *dev_y,
                   long long n, int batch, int steps, float lr, int step0, float *dev_work, double *last_loss);
/* The network on n feature rows (dev_x n x 5) -> dev_y n x 2 (log W, log h). */
int mgpu_mlp_forward(const float *dev_params, const float *dev_x, long long n, float *dev_y);
/* The same on the tensor cores (BF16 weights and activations, FP32 accumulation), from the
 * host-side FP32 parameters: the path the zone c2p kernel uses when a network is set. */
int mgpu_mlp_forward_tc(const float *params, const float *dev_x, long long n, float *dev_y);
/* The tensor-core image of a network (mgpu_mlp_tc_image_bytes bytes, host memory). */
int mgpu_mlp_tc_image_bytes(void);
int mgpu_mlp_build_tc_image(const float *params, void *image);

/* ---- stochastic driving (Mara.new_ou_field / set_driving / driving.*, Mara/mara.cpp:1169-1190,
 * 1378-1401, 1771-1808; Mara/ou-field.cpp, Mara/driving.cpp) ---------------------------------
 * A driving field is the reference's serialized StochasticVectorField (the bytes
 * Mara.new_ou_field returns and Mara.driving.Serialize writes to checkpoints): mode
 * amplitudes and their OU random streams.  While a solver holds one, every advance that
 * commits kicks the 4-velocity of every zone by F dt / W (rest mass per zone kept) --
 * DrivingProcedure::Drive_rmhd.  Two-call pattern for sizes: out NULL -> *bytes. */
int mgpu_new_ou_field(int nd, double P0, double zeta, int k1, int seed, void *out, long long *bytes);
/* replaces luaC_set_driving; field NULL clears it.  Samples the field on the grid. */
int mgpu_set_driving(mgpu_solver *h, const void *field, long long bytes);
int mgpu_driving_advance(mgpu_solver *h, double dt);      /* Mara.driving.Advance(dt): OU step */
int mgpu_driving_resample(mgpu_solver *h);                /* Mara.driving.Resample() */
int mgpu_driving_serialize(mgpu_solver *h, void *out, long long *bytes);   /* Mara.driving.Serialize() */
int mgpu_driving_power(mgpu_solver *h, double *power);    /* Mara.driving.Power() */
/* The OU step of a serialized field in place, without a solver (host only). */
int mgpu_ou_field_advance(void *field, long long bytes, int nd, double dt);

/* ---- domain decomposition (the reference's DecomposedCartesianDomain with MPI,
 * Mara/subgrids.cpp:12-147, Mara/mara_mpi.c:96-130; here any transport, e.g. NCCL) --------
 * A rank's solver holds its subdomain (mgpu_set_domain with the local x0, x1, N).  For every
 * dimension split across ranks, mgpu_set_external_guards turns off the periodic guard fill
 * and takes multiplicity tables: mult lists, for each such dimension in order and each
 * local interior index along it, how many guarded arrays over all ranks hold that zone (the
 * reference counts a failed zone once per array holding it, Mara/hydro.cpp:133-149,201).
 * The host then drives each advance phase by phase and fills the guards between them
 * (phases 0 begin, 1 c2p, 2 flux+update, 3 commit; 4 and 5 below):
 *   mgpu_advance_phase(0 begin) ; per stage s: phase(1 c2p, s), exchange the stage
 *   primitives (which 0) for every split dimension in order x, y, z with
 *   mgpu_halo_pack / mgpu_halo_unpack, phase(2 flux+update, s) ; phase(1 c2p, stages) ;
 *   sum the five error counters and max the MaxLambda bits (mgpu_reduction_targets, device
 *   memory: int[5] = stage 1-4 and closing c2p, uint64 = a non-negative double's bits) over
 *   all ranks ; phase(3 commit).
 * Slabs are Ng layers over the full guarded cross-section (edges and corners follow from
 * the x, y, z order); side 0 packs the low interior layers / unpacks the low guards, side 1
 * the high ones.  which 1 exchanges the committed state (before a download with guards).
 * Asynchronous on the handle's stream except where noted. */
int mgpu_advance_phase(mgpu_solver *h, int phase, int stage, int dt_mode, double dt, double cfl);
int mgpu_reduction_targets(mgpu_solver *h, void **err_counts, void **max_lambda_bits);
int mgpu_set_external_guards(mgpu_solver *h, const int *ext, const int *mult);   /* synchronous */
int mgpu_halo_bytes(mgpu_solver *h, int which, int dim, long long *bytes);
int mgpu_halo_pack(mgpu_solver *h, int which, int dim, int side, void *dev_buf);
int mgpu_halo_unpack(mgpu_solver *h, int which, int dim, int side, const void *dev_buf);
/* Overlapped exchange (no counterpart in the reference, whose Synchronize blocks): phase 4
 * converts the stage's boundary shell -- interior zones within Ng of a split face, all the
 * slabs read -- and phase 5 the core; together they are phase 1 of that stage (s < stages;
 * with a learned c2p network phase 4 converts everything and phase 5 nothing).  Between
 * them the caller can pack, exchange and unpack on another stream (the _on variants, stream
 * = cudaStream_t; order it after phase 4 and phase 2 after the unpacks with events) while
 * phase 5 runs on the handle's stream: the core's c2p writes no zone a slab reads or fills. */
int mgpu_halo_pack_on(mgpu_solver *h, int which, int dim, int side, void *dev_buf, void *stream);
int mgpu_halo_unpack_on(mgpu_solver *h, int which, int dim, int side, const void *dev_buf, void *stream);

/* ---- function-level probes (test infrastructure of the parity suite; no counterpart in
 * the reference's Lua API).  Each applies one FP64 device function of the advance to n
 * independent states held in device memory (AoS, 8 doubles per state) and returns after the
 * work is done; each replaces, for per-function comparison, the reference function named:
 *   mgpu_probe_prim_to_cons  AdiabaticIdealRmhd::PrimToCons (Mara/rmhd.cpp:177-207); err =
 *                            its check of the conserved state.
 *   mgpu_probe_c2p           mode 0: AdiabaticIdealRmhd::ConsToPrim, the gamma-law ladder
 *                            (Mara/rmhd.cpp:103-176) with dev_guess as the previous primitives
 *                            (dev_P = dev_guess where it fails); mode 1 + 2*solver + start: one
 *                            solver, rmhd_c2p_solve_anton2dzw (solver 0) or _noble1dw (1)
 *                            (Mara/rmhd-c2p.c:182-326), started from rmhd_c2p_estimate_from_cons
 *                            (start 0) or rmhd_c2p_set_starting_prim(dev_guess) (start 1)
 *                            (Mara/rmhd-c2p.c:96-119); iters = Newton iterations.
 *   mgpu_probe_flux          FluxAndEigenvalues (Mara/rmhd.cpp:208-310) of P->U(P) in
 *                            direction dim: dev_F n x 8, dev_lam n x 2 (lambda+, lambda-).
 *   mgpu_probe_riemann       IntercellFlux at s = 0 of MGPU_RIEMANN_HLL / HLLC / HLLD
 *                            (Mara/riemann_hll.cpp:19-64, riemann_hllc-rmhd.cpp:26-178,
 *                            riemann_hlld-rmhd.cpp:143-277) on face pairs in direction dim, or
 *                            per face dev_dims[i] when dev_dims is not NULL; dev_max_lambda[i]
 *                            = RiemannSolver::MaxLambda after that face alone; dev_used_hllc
 *                            (may be NULL) = 1 where HLLD fell back to HLLC.
 *   mgpu_probe_reconstruct   reconstruct (Mara/weno.c:58-154) on stencils dev_V (n x 5, centre
 *                            at 2): op 0 / 1 PLM minmod(theta) left / right face, op 4 / 5
 *                            WENO5 FV centre-to-right / centre-to-left (is_mode, sz10A). */
int mgpu_probe_prim_to_cons(double gamma, const double *dev_P, long long n, double *dev_U, int *dev_err);
int mgpu_probe_c2p(int mode, double gamma, double pfloor, const double *dev_U, const double *dev_guess, long long n,
                   double *dev_P, int *dev_err, int *dev_iters);
int mgpu_probe_flux(double gamma, int dim, const double *dev_P, long long n, double *dev_F, double *dev_lam);
int mgpu_probe_riemann(int riemann, int dim, const int *dev_dims, double gamma, double pfloor, const double *dev_Pl,
                       const double *dev_Pr, long long n, double *dev_F, int *dev_err, double *dev_max_lambda,
                       int *dev_used_hllc);
int mgpu_probe_reconstruct(int op, double theta, int is_mode, double sz10A, const double *dev_V, long long n,
                           double *dev_out);

/* Allocation-free advance (no counterpart in the reference).  For callers that may not
 * allocate device memory -- allocation-free sections of a larger application, real-time
 * loops, hosts that hand out only pre-owned buffers: one FP64 advance of a box of at most
 * MGPU_NOALLOC_MAX_ZONES guarded zones, using working arrays kept in a fixed ~7.8 MiB region
 * of the library's own device memory (present on every GPU that loads the library, for the
 * life of the process) instead of cudaMalloc.  The caller passes device AoS primitives with
 * guard zones in (dev_prim_in) and out (dev_prim_out, written only when *errors == 0) and a
 * stream (NULL = the default stream); cfg must select MGPU_PREC_FP64 without learned_c2p;
 * Ng is 3.  The call is synchronous (it returns after its work on the stream has finished)
 * and returns the reference's error count and MaxLambda.  Larger boxes are rejected with
 * MGPU_ERR_ARG and a message in errbuf.  Every call looks up the current device's address of
 * the region (cudaGetSymbolAddress, with that device current), so a cudaDeviceReset or
 * another context between calls is harmless; the first call on a device also loads the
 * library's device code there.  All calls share the region: calls whose work overlaps on the
 * GPU (several streams or host threads) race and must be serialised by the caller. */
#define MGPU_NOALLOC_MAX_ZONES 11520
int mgpu_advance_noalloc(const mgpu_config *cfg, const double *x0, const double *x1, const int *N, int nd,
                         const void *dev_prim_in, void *dev_prim_out, double dt, int *errors,
                         double *max_lambda, void *stream, char *errbuf, int errbuf_len);

/* ---- ensembles of independent boxes (no counterpart in the reference, whose solver is a
 * process-global singleton, Mara/mara.cpp:135).  Every box of an ensemble has the same
 * scheme (one mgpu_config) and dimensionality but its own size, extent, primitives, dt,
 * MaxLambda, error counts and commit; box b advances exactly as an mgpu_solver of that box
 * would.  One advance of the whole ensemble is a fixed sequence of persistent launches,
 * each walking the tiles of all boxes, replayed as one CUDA graph.  Ng is 3; learned_c2p
 * is not offered here. */
typedef struct mgpu_ensemble mgpu_ensemble;

/* Launch shape: tile lengths (contiguous flattened zones or faces per tile, multiples of
 * 32) and persistent grid sizes (CTAs per SM) of the zone, face and c2p launches. */
typedef struct {
  int zone_tile, face_tile;
  int zone_ctas_per_sm, face_ctas_per_sm, c2p_ctas_per_sm;
} mgpu_ensemble_launch;

/* N, x0, x1: nboxes * nd entries, box-major (x0/x1 NULL: the unit box for all). */
int mgpu_ensemble_create(const mgpu_config *cfg, int nd, int nboxes, const int *N, const double *x0,
                         const double *x1, mgpu_ensemble **out);
int mgpu_ensemble_destroy(mgpu_ensemble *e);
const char *mgpu_ensemble_last_error(const mgpu_ensemble *e);
int mgpu_ensemble_set_stream(mgpu_ensemble *e, void *stream);
int mgpu_ensemble_num_zones(const mgpu_ensemble *e, int box, long long *nz);   /* guarded zones */
int mgpu_ensemble_total_interior(const mgpu_ensemble *e, long long *n);       /* over all boxes */
int mgpu_ensemble_upload_prim(mgpu_ensemble *e, int box, const double *host_aos);
int mgpu_ensemble_download_prim(mgpu_ensemble *e, int box, double *host_aos);
int mgpu_ensemble_upload_prim_device(mgpu_ensemble *e, int box, const void *dev_aos);
int mgpu_ensemble_download_prim_device(mgpu_ensemble *e, int box, void *dev_aos);
int mgpu_ensemble_get_launch(const mgpu_ensemble *e, mgpu_ensemble_launch *L);
int mgpu_ensemble_set_launch(mgpu_ensemble *e, const mgpu_ensemble_launch *L);
/* Enqueue nsteps advances of every box.  dt_mode 0: box b uses dt[b] (host array, copied
 * before the call returns); dt_mode 1: cfl * min_dx_b / MaxLambda_b of its previous advance.
 * use_graph 1 replays a cached CUDA graph of the nsteps advances (captured on first use of
 * a given nsteps, dt_mode, cfl and launch shape); 0 launches directly.  Asynchronous. */
int mgpu_ensemble_advance(mgpu_ensemble *e, int nsteps, int dt_mode, const double *dt, double cfl,
                          int use_graph);
int mgpu_ensemble_synchronize(mgpu_ensemble *e);
int mgpu_ensemble_errors(mgpu_ensemble *e, int *errors);          /* nboxes entries, last advance */
int mgpu_ensemble_get_stats(mgpu_ensemble *e, int box, mgpu_stats *s);
int mgpu_ensemble_get_timesteps(mgpu_ensemble *e, double cfl, double *dt);   /* nboxes entries */
/* Per-kernel-class timing of direct (use_graph 0) advances, as mgpu_profile_*. */
int mgpu_ensemble_profile_enable(mgpu_ensemble *e, int capacity);
int mgpu_ensemble_profile_disable(mgpu_ensemble *e);
int mgpu_ensemble_profile_read(mgpu_ensemble *e, double *ms, long long *launches, long long *units);
/* Mean device time of one advance (dt_mode 0, dt[] per box) with launch shape L, over reps
 * graph replays after one warm-up; nothing is committed and every box's state and control
 * block are left as they were. */
int mgpu_ensemble_time_advance(mgpu_ensemble *e, const mgpu_ensemble_launch *L, const double *dt, int reps,
                               double *ms);
/* Search the launch shapes (coordinate descent over tile lengths and grid sizes, timed with
 * mgpu_ensemble_time_advance), install the fastest and return it and its time. */
int mgpu_ensemble_autotune(mgpu_ensemble *e, const double *dt, int reps, mgpu_ensemble_launch *best,
                           double *best_ms);

#ifdef __cplusplus
}
#endif
#endif
