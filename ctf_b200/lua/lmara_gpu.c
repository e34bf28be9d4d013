/* lmara_gpu.c -- the Lua module `Mara` on the B200 RMHD step (libmaragpu.so).
 *
 * A link-time drop-in for the reference's luaopen_Mara (Mara/mara.cpp:137-268): a host that
 * registers it with luaL_requiref(L, "Mara", luaopen_Mara, 1), as ctf-core/ctf.c:139 does,
 * runs the reference's driver loops unchanged for the RMHD step:
 *
 *   start, close, set_fluid('rmhd'), set_eos('gamma-law', G), set_boundary('periodic'),
 *   set_godunov('plm-split' | 'plm-muscl'), set_riemann, set_advance, config_solver{...}[, quiet],
 *   set_domain(x0, x1, N, Nq, Ng), init_prim(buf, f), set_primitive(buf),
 *   advance(buf, dt) -> kzps, errors, get_timestep(CFL) -> dt, diffuse(buf, r),
 *   set_failmask(v), cooling_rate(dt) (0: no cooling module), measure.mean_max_divB(),
 *   measure.max_lorentz_factor(), measure.mean_cons/mean_prim/mean_energies/mean_velocity/
 *   mean_max_temperature/mean_max_magnetic_field/mean_max_sonic_mach/mean_min_alfvenic_mach(),
 *   fluid.GetPrimNames()
 *
 * with the reference's argument conventions and error messages (luaL_error for misuse,
 * an error count for numerical failure with the buffer left unchanged).  Entry points of
 * the reference outside the RMHD step (other fluids and EOSs, cooling, driving, sampling,
 * images) exist in the table and raise an error naming themselves.
 *
 * Additions: config_solver accepts precision = 'fp64' | 'fp32' (the FP32-bulk path),
 * learned_c2p = true | false and layout = 'standard' | 'lean' (the device layout of large 3D
 * boxes, include/mara_gpu.h); Mara.set_c2p_network(buf) takes a buffer of float32 network
 * parameters; Mara.gpu_stats() returns the device counters of the last advance;
 * Mara.upload_primitive(buf), Mara.advance_device(dt) and Mara.download_primitive(buf) step a
 * device-resident state without the per-step host copies of Mara.advance(buf, dt).
 *
 * The solver is one module-level object, as the reference's is (mara.cpp:135).  Scheme
 * changes after set_domain are applied to the device solver in place at its next use
 * (mgpu_reconfigure: MaxLambda, the failure mask and the measured array carry over, as in
 * the reference); only a change of precision or layout rebuilds it, and the rebuilt solver
 * starts without those.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "lua.h"
#include "lauxlib.h"

#include "../../include/mara_gpu.h"

typedef struct {
  mgpu_config cfg;
  int started;
  mgpu_solver *h;
  int dirty;                 /* cfg changed since h was built */
  int have_domain;
  int nd, nq, ng, N[3];
  double x0[3], x1[3];
  double *prim;              /* host mirror of the primitive array init_prim fills */
  long long nzones;
  float *net;                /* learned c2p parameters (host copy) */
  long long net_count;
  char *drive;               /* driving field carried across a solver rebuild */
  long long drive_len;
  int have_godunov;          /* set_godunov was called since start */
  int resident;              /* the device solver holds a state from upload_primitive */
} MaraGpu;

static MaraGpu M;
static double ctu_theta = 2.0;   /* the CTU-Hancock operator's plm_theta (a process static) */

static void free_solver(void)
{
  if (M.h) mgpu_destroy(M.h);
  M.h = NULL;
}

static int raise_abi(lua_State *L, int rc, const char *what)
{
  return luaL_error(L, "[Mara] %s: %s (code %d)", what, M.h ? mgpu_last_error(M.h) : "no solver", rc);
}

/* The device solver for the current scheme and domain, built on first use. */
static mgpu_solver *solver(lua_State *L)
{
  if (!M.started) luaL_error(L, "[Mara] call Mara.start() first");
  if (!M.have_domain) luaL_error(L, "[Mara] need a domain to run this, use set_domain");
  if (M.h && !M.dirty) return M.h;
  if (M.h) {   /* a scheme change: in place where the solver allows it (state, MaxLambda,
                  failure mask and measured array carry over, as in the reference) */
    mgpu_config cfg = M.cfg;
    if (cfg.godunov == MGPU_GODUNOV_PLM_MUSCL) cfg.theta = ctu_theta;
    if (mgpu_reconfigure(M.h, &cfg) == 0) {
      M.dirty = 0;
      return M.h;
    }
  }
  if (M.h) {   /* keep the driving field (its OU state) across the rebuild */
    long long n = 0;
    free(M.drive);
    M.drive = NULL;
    M.drive_len = 0;
    if (mgpu_driving_serialize(M.h, NULL, &n) == 0 && n > 0 && (M.drive = (char *) malloc((size_t) n))) {
      mgpu_driving_serialize(M.h, M.drive, &n);
      M.drive_len = n;
    }
  }
  free_solver();
  M.resident = 0;
  mgpu_config cfg = M.cfg;
  if (cfg.godunov == MGPU_GODUNOV_PLM_MUSCL) cfg.theta = ctu_theta;
  int rc = mgpu_create(&cfg, &M.h);
  if (rc) {
    M.h = NULL;
    luaL_error(L, "[Mara] could not create the GPU solver (code %d)", rc);
  }
  rc = mgpu_set_domain(M.h, M.x0, M.x1, M.N, M.nd, M.nq, M.ng);
  if (rc) raise_abi(L, rc, "set_domain");
  if (M.net) {
    rc = mgpu_set_c2p_network(M.h, M.net, M.net_count);
    if (rc) raise_abi(L, rc, "set_c2p_network");
  }
  if (M.drive) {
    rc = mgpu_set_driving(M.h, M.drive, M.drive_len);
    if (rc) raise_abi(L, rc, "set_driving");
  }
  M.dirty = 0;
  return M.h;
}

static double *check_prim_buffer(lua_State *L, int idx)
{
  if (lua_type(L, idx) != LUA_TUSERDATA) luaL_error(L, "[Mara] expected a buffer as argument %d", idx);
  const size_t n = lua_rawlen(L, idx) / sizeof(double);
  if (!M.have_domain) luaL_error(L, "[Mara] need a domain to run this, use set_domain");
  if ((long long) n != M.nzones * M.nq) luaL_error(L, "[Mara] primitive has the wrong size for the domain");
  return (double *) lua_touserdata(L, idx);
}

/* a Lua array of numbers (at most `cap` read) -> out; returns its length */
static int check_numbers(lua_State *L, int idx, double *out, int cap)
{
  idx = lua_absindex(L, idx);
  if (lua_type(L, idx) != LUA_TTABLE) luaL_error(L, "[Mara] expected a table as argument %d", idx);
  const int n = (int) lua_rawlen(L, idx);
  for (int i = 0; i < n && i < cap; ++i) {
    lua_rawgeti(L, idx, i + 1);
    out[i] = lua_tonumber(L, -1);
    lua_pop(L, 1);
  }
  return n;
}

/* ---- Mara.* ------------------------------------------------------------------------------ */

/* luaC_Mara_start (mara.cpp:271-287): a new application object.  As in the reference, the
 * reconstruction settings of config_solver (extrap, theta, IS, sz10A, pfloor: process-wide
 * statics there) survive a restart; everything held by the application object does not. */
static int l_start(lua_State *L)
{
  (void) L;
  mgpu_config keep = M.cfg;
  const int had = M.started;
  free_solver();
  free(M.prim);
  free(M.net);
  free(M.drive);
  memset(&M, 0, sizeof(M));
  mgpu_default_config(&M.cfg);
  if (had) {
    M.cfg.recon = keep.recon;
    M.cfg.theta = keep.theta;
    M.cfg.is_mode = keep.is_mode;
    M.cfg.sz10A = keep.sz10A;
    M.cfg.pfloor = keep.pfloor;
  }
  M.started = 1;
  return 0;
}

static int l_close(lua_State *L)
{
  (void) L;
  free_solver();
  free(M.prim);
  free(M.net);
  free(M.drive);
  memset(&M, 0, sizeof(M));
  return 0;
}

static int l_git_sha(lua_State *L)
{
  lua_pushstring(L, "b200");
  return 1;
}

static void changed(void) { M.dirty = 1; }

static int l_set_fluid(lua_State *L)
{
  const char *key = luaL_checkstring(L, 1);
  if (strcmp(key, "rmhd") == 0) {
    M.cfg.fluid = MGPU_FLUID_RMHD;
    changed();
  } else if (strcmp(key, "euler") == 0 || strcmp(key, "srhd") == 0) {
    luaL_error(L, "[Mara] fluid '%s' is not provided by the GPU module (only 'rmhd')", key);
  } else {
    luaL_error(L, "[Mara] no such fluid '%s'", key);
  }
  return 0;
}

static int l_set_eos(lua_State *L)
{
  const char *key = luaL_checkstring(L, 1);
  if (strcmp(key, "gamma-law") == 0) {
    M.cfg.gamma = luaL_checknumber(L, 2);   /* BuildAdiabaticEos, mara.cpp:435-439 */
    changed();
  } else if (strcmp(key, "gamma-law + polytrope") == 0 || strcmp(key, "shen") == 0 ||
             strcmp(key, "tabulated") == 0) {
    luaL_error(L, "[Mara] eos '%s' is not provided by the GPU module (only 'gamma-law')", key);
  } else {
    luaL_error(L, "[Mara] no such eos '%s'", key);
  }
  return 0;
}

static int l_set_boundary(lua_State *L)
{
  const char *key = luaL_checkstring(L, 1);
  if (strcmp(key, "periodic") == 0) return 0;
  if (strcmp(key, "outflow") == 0 || strcmp(key, "perxouty") == 0 || strcmp(key, "reflect2d") == 0 ||
      strcmp(key, "magnetic-bubble") == 0 || strcmp(key, "wind-inflow") == 0)
    return luaL_error(L, "[Mara] boundary '%s' is not provided by the GPU module (only 'periodic')", key);
  return luaL_error(L, "[Mara] no such boundary conditions '%s'", key);
}

/* A new operator carries the constructor's emergency-reset settings (hydro.cpp:18-32).
 * 'plm-muscl' is the CTU-Hancock operator, whose PLM limiter parameter is its own
 * process-wide static (ctu-hancock.cpp:11, default 2), changed only by config_solver{theta}
 * while it is the current operator (mara.cpp:1068-1074). */
static int l_set_godunov(lua_State *L)
{
  const char *key = luaL_checkstring(L, 1);
  const int muscl = strcmp(key, "plm-muscl") == 0;
  if (strcmp(key, "plm-split") == 0 || muscl) {
    mgpu_config d;
    mgpu_default_config(&d);
    M.cfg.ereset = d.ereset;
    M.cfg.preset = d.preset;
    M.cfg.dreset = d.dreset;
    M.cfg.godunov = muscl ? MGPU_GODUNOV_PLM_MUSCL : MGPU_GODUNOV_PLM_SPLIT;
    M.have_godunov = 1;
    changed();
    return 0;
  }
  if (strcmp(key, "weno-split") == 0)
    return luaL_error(L, "[Mara] integration scheme '%s' is not provided by the GPU module "
                         "(only 'plm-split' and 'plm-muscl')", key);
  return luaL_error(L, "[Mara] no such integration scheme '%s'", key);
}

static int l_set_riemann(lua_State *L)
{
  const char *key = luaL_checkstring(L, 1);
  if (strcmp(key, "hll") == 0) M.cfg.riemann = MGPU_RIEMANN_HLL;
  else if (strcmp(key, "hllc") == 0) M.cfg.riemann = MGPU_RIEMANN_HLLC;
  else if (strcmp(key, "hlld") == 0) M.cfg.riemann = MGPU_RIEMANN_HLLD;
  else return luaL_error(L, "[Mara] no such riemann solver '%s'", key);
  changed();
  return 0;
}

static int l_set_advance(lua_State *L)
{
  const char *key = luaL_checkstring(L, 1);
  if (strcmp(key, "single") == 0) M.cfg.rk = 1;
  else if (strcmp(key, "rk2") == 0) M.cfg.rk = 2;
  else if (strcmp(key, "rk3") == 0) M.cfg.rk = 3;
  else if (strcmp(key, "rk4") == 0) M.cfg.rk = 4;
  else return luaL_error(L, "[Mara] no such advance option '%s'", key);
  changed();
  return 0;
}

/* luaC_config_solver (mara.cpp:996-1138): the keys of the reference, plus precision and
 * learned_c2p. */
static int l_config_solver(lua_State *L)
{
  luaL_checktype(L, 1, LUA_TTABLE);
  const int quiet = lua_gettop(L) == 2 ? lua_toboolean(L, 2) : 0;

  lua_getfield(L, 1, "fsplit");
  if (lua_isstring(L, -1)) {
    const char *key = lua_tostring(L, -1);
    if (strcmp(key, "llf") && strcmp(key, "marq")) luaL_error(L, "[Mara] no such fsplit '%s'", key);
    if (!quiet) printf("[config] setting fsplit=%s\n", key);   /* used only by weno-split */
  }
  lua_pop(L, 1);

  lua_getfield(L, 1, "extrap");
  if (lua_isstring(L, -1)) {
    const char *key = lua_tostring(L, -1);
    if (strcmp(key, "pcm") == 0) M.cfg.recon = MGPU_RECON_PCM;
    else if (strcmp(key, "plm") == 0) M.cfg.recon = MGPU_RECON_PLM;
    else if (strcmp(key, "weno5") == 0) M.cfg.recon = MGPU_RECON_WENO5;
    else luaL_error(L, "[Mara] no such extrap '%s'", key);
    if (!quiet) printf("[config] setting extrap=%s\n", key);
  }
  lua_pop(L, 1);

  lua_getfield(L, 1, "theta");
  if (lua_isnumber(L, -1)) {
    M.cfg.theta = lua_tonumber(L, -1);
    if (!quiet) printf("[Mara] setting theta=%f\n", M.cfg.theta);
    if (M.have_godunov && M.cfg.godunov == MGPU_GODUNOV_PLM_MUSCL) ctu_theta = M.cfg.theta;
  }
  lua_pop(L, 1);

  lua_getfield(L, 1, "IS");
  if (lua_isstring(L, -1)) {
    const char *key = lua_tostring(L, -1);
    if (strcmp(key, "js96") == 0) M.cfg.is_mode = MGPU_IS_JS96;
    else if (strcmp(key, "b08") == 0) M.cfg.is_mode = MGPU_IS_B08;
    else if (strcmp(key, "sz10") == 0) M.cfg.is_mode = MGPU_IS_SZ10;
    else luaL_error(L, "no such IS: %s", key);
    if (!quiet) printf("[Mara] setting IS=%s\n", key);
  }
  lua_pop(L, 1);

  lua_getfield(L, 1, "sz10A");
  if (lua_isnumber(L, -1)) {
    M.cfg.sz10A = lua_tonumber(L, -1);
    if (!quiet) printf("[Mara] setting sz10A=%f\n", M.cfg.sz10A);
  }
  lua_pop(L, 1);

  lua_getfield(L, 1, "pfloor");
  if (lua_isnumber(L, -1)) {
    M.cfg.pfloor = lua_tonumber(L, -1);
    if (!quiet) printf("[Mara] setting pfloor=%f\n", M.cfg.pfloor);
  }
  lua_pop(L, 1);

  lua_getfield(L, 1, "ereset");
  if (lua_isboolean(L, -1)) {
    M.cfg.ereset = lua_toboolean(L, -1);
    if (!quiet) printf("[Mara] setting ereset=%d\n", M.cfg.ereset);
  }
  lua_pop(L, 1);

  lua_getfield(L, 1, "preset");
  if (lua_isnumber(L, -1)) {
    M.cfg.preset = lua_tonumber(L, -1);
    if (!quiet) printf("[Mara] setting preset=%f\n", M.cfg.preset);
  }
  lua_pop(L, 1);

  lua_getfield(L, 1, "dreset");
  if (lua_isnumber(L, -1)) {
    M.cfg.dreset = lua_tonumber(L, -1);
    if (!quiet) printf("[Mara] setting dreset=%f\n", M.cfg.dreset);
  }
  lua_pop(L, 1);

  lua_getfield(L, 1, "precision");
  if (lua_isstring(L, -1)) {
    const char *key = lua_tostring(L, -1);
    if (strcmp(key, "fp64") == 0) M.cfg.precision = MGPU_PREC_FP64;
    else if (strcmp(key, "fp32") == 0) M.cfg.precision = MGPU_PREC_FP32;
    else luaL_error(L, "[Mara] no such precision '%s'", key);
    if (!quiet) printf("[Mara] setting precision=%s\n", key);
  }
  lua_pop(L, 1);

  lua_getfield(L, 1, "learned_c2p");
  if (lua_isboolean(L, -1)) {
    M.cfg.learned_c2p = lua_toboolean(L, -1);
    if (!quiet) printf("[Mara] setting learned_c2p=%d\n", M.cfg.learned_c2p);
  }
  lua_pop(L, 1);

  lua_getfield(L, 1, "layout");
  if (lua_isstring(L, -1)) {
    const char *key = lua_tostring(L, -1);
    if (strcmp(key, "standard") == 0) M.cfg.layout = MGPU_LAYOUT_STANDARD;
    else if (strcmp(key, "lean") == 0) M.cfg.layout = MGPU_LAYOUT_LEAN;
    else luaL_error(L, "[Mara] no such layout '%s'", key);
    if (!quiet) printf("[Mara] setting layout=%s\n", key);
  }
  lua_pop(L, 1);

  changed();
  return 0;
}

/* luaC_set_domain (mara.cpp:726-755): x0, x1, N tables, Nq, Ng (an MPI communicator as a
 * sixth argument is accepted and ignored: one device). */
static int l_set_domain(lua_State *L)
{
  if (!M.started) return luaL_error(L, "[Mara] call Mara.start() first");
  double x0[3] = {0, 0, 0}, x1[3] = {1, 1, 1}, Nd[3] = {1, 1, 1};
  const int n0 = check_numbers(L, 1, x0, 3);
  const int n1 = check_numbers(L, 2, x1, 3);
  const int nd = check_numbers(L, 3, Nd, 3);
  const int nq = (int) luaL_checkinteger(L, 4);
  const int ng = (int) luaL_checkinteger(L, 5);
  if (nd < 1 || nd > 3 || n0 < nd || n1 < nd) return luaL_error(L, "[Mara] set_domain needs 1 to 3 dimensions");
  M.nd = nd;
  M.nq = nq;
  M.ng = ng;
  M.nzones = 1;
  for (int d = 0; d < 3; ++d) {
    M.N[d] = d < nd ? (int) Nd[d] : 1;
    M.x0[d] = x0[d];
    M.x1[d] = x1[d];
    M.nzones *= d < nd ? M.N[d] + 2 * ng : 1;
  }
  free(M.prim);
  free(M.drive);
  M.drive = NULL;
  M.drive_len = 0;
  M.prim = (double *) calloc((size_t) (M.nzones * nq), sizeof(double));
  if (!M.prim) return luaL_error(L, "[Mara] out of host memory");
  M.have_domain = 1;
  changed();
  solver(L);   /* validates the domain now, as the reference's constructor would */
  return 0;
}

/* luaC_Mara_init_prim (mara.cpp:531-629): f(x, y, z) -> primitive table at every interior
 * zone centre x0 + dx (i + 1/2); the whole array (guards as they were) into buf. */
static int l_init_prim(lua_State *L)
{
  if (!M.have_domain) return luaL_error(L, "[Mara] need a domain to run this, use set_domain");
  if (lua_type(L, 2) != LUA_TFUNCTION) return luaL_error(L, "[Mara] argument must be a function");
  double *buf = check_prim_buffer(L, 1);
  const int ng = M.ng, nq = M.nq;
  const int G1 = M.nd >= 2 ? M.N[1] + 2 * ng : 1, G2 = M.nd >= 3 ? M.N[2] + 2 * ng : 1;
  double dx[3];
  for (int d = 0; d < 3; ++d) dx[d] = (M.x1[d] - M.x0[d]) / M.N[d];
  double P[64];
  for (int i = 0; i < M.N[0]; ++i)
    for (int j = 0; j < M.N[1]; ++j)
      for (int k = 0; k < M.N[2]; ++k) {
        const double x = M.x0[0] + dx[0] * (i + 0.5);
        const double y = M.nd >= 2 ? M.x0[1] + dx[1] * (j + 0.5) : 0.0;
        const double z = M.nd >= 3 ? M.x0[2] + dx[2] * (k + 0.5) : 0.0;
        lua_pushvalue(L, 2);
        lua_pushnumber(L, x);
        lua_pushnumber(L, y);
        lua_pushnumber(L, z);
        lua_call(L, 3, 1);
        memset(P, 0, sizeof(P));
        check_numbers(L, -1, P, nq < 64 ? nq : 64);
        lua_pop(L, 1);
        const long long zi = ((long long) (i + ng) * G1 + (M.nd >= 2 ? j + ng : 0)) * G2 + (M.nd >= 3 ? k + ng : 0);
        memcpy(M.prim + zi * nq, P, sizeof(double) * (size_t) nq);
      }
  memcpy(buf, M.prim, sizeof(double) * (size_t) (M.nzones * nq));
  const int rc = mgpu_set_primitive(solver(L), M.prim);
  if (rc) return raise_abi(L, rc, "init_prim");
  return 0;
}

static int l_set_primitive(lua_State *L)
{
  double *buf = check_prim_buffer(L, 1);
  memcpy(M.prim, buf, sizeof(double) * (size_t) (M.nzones * M.nq));
  const int rc = mgpu_set_primitive(solver(L), buf);
  if (rc) return raise_abi(L, rc, "set_primitive");
  return 0;
}

/* luaC_Mara_advance (mara.cpp:297-341) -> kzps, errors; buf unchanged when errors > 0 */
static int l_advance(lua_State *L)
{
  if (!M.have_domain) return luaL_error(L, "[Mara] need a domain to run this, use set_domain");
  double *buf = check_prim_buffer(L, 1);
  const double dt = luaL_checknumber(L, 2);
  double kzps = 0.0;
  int errors = 0;
  const int rc = mgpu_advance_host(solver(L), buf, dt, &kzps, &errors);
  if (rc) return raise_abi(L, rc, "advance");
  lua_pushnumber(L, kzps);
  lua_pushnumber(L, errors);
  return 2;
}

/* Device-resident stepping (no counterpart in the reference, whose state lives in the caller's
 * buffer): upload_primitive(buf) copies a primitive buffer to the device once,
 * advance_device(dt) -> kzps, errors advances it there without host copies (state unchanged
 * when errors > 0, as Mara.advance), download_primitive(buf) copies it back.  A driver loop
 * that only reads get_timestep and the measures between steps then moves no state over PCIe;
 * a scheme change rebuilds the solver and needs a new upload. */
static int l_upload_primitive(lua_State *L)
{
  double *buf = check_prim_buffer(L, 1);
  const int rc = mgpu_upload_prim(solver(L), buf);
  if (rc) return raise_abi(L, rc, "upload_primitive");
  M.resident = 1;
  return 0;
}

static double now_seconds(void)
{
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double) t.tv_sec + 1e-9 * (double) t.tv_nsec;
}

static int l_advance_device(lua_State *L)
{
  const double dt = luaL_checknumber(L, 1);
  mgpu_solver *h = solver(L);
  if (!M.resident) return luaL_error(L, "[Mara] advance_device needs a state: call Mara.upload_primitive(P) first");
  int errors = 0;
  const double t0 = now_seconds();
  const int rc = mgpu_advance(h, dt, &errors);
  if (rc) return raise_abi(L, rc, "advance_device");
  lua_pushnumber(L, 1e-3 * (double) M.nzones / (now_seconds() - t0));
  lua_pushnumber(L, errors);
  return 2;
}

static int l_download_primitive(lua_State *L)
{
  double *buf = check_prim_buffer(L, 1);
  mgpu_solver *h = solver(L);
  if (!M.resident) return luaL_error(L, "[Mara] download_primitive needs a state: call Mara.upload_primitive(P) first");
  const int rc = mgpu_download_prim(h, buf);
  if (rc) return raise_abi(L, rc, "download_primitive");
  return 0;
}

static int l_get_timestep(lua_State *L)
{
  const double cfl = luaL_checknumber(L, 1);
  double dt = 0.0;
  const int rc = mgpu_get_timestep(solver(L), cfl, &dt);
  if (rc) return raise_abi(L, rc, "get_timestep");
  lua_pushnumber(L, dt);
  return 1;
}

static int l_set_c2p_network(lua_State *L)
{
  if (lua_type(L, 1) != LUA_TUSERDATA) return luaL_error(L, "[Mara] expected a buffer of float32 parameters");
  const size_t n = lua_rawlen(L, 1) / sizeof(float);
  if ((long long) n != mgpu_mlp_param_count())
    return luaL_error(L, "[Mara] the network needs %d float32 parameters, got %d", mgpu_mlp_param_count(), (int) n);
  free(M.net);
  M.net = (float *) malloc(n * sizeof(float));
  if (!M.net) return luaL_error(L, "[Mara] out of host memory");
  memcpy(M.net, lua_touserdata(L, 1), n * sizeof(float));
  M.net_count = (long long) n;
  changed();
  return 0;
}

/* ---- driving (Mara.new_ou_field, Mara.set_driving, Mara.driving.*; mara.cpp:1169-1190,
 * 1378-1401, 1771-1808): the reference's serialized fields, as Lua strings ------------------ */
static int l_new_ou_field(lua_State *L)
{
  const int nd = (int) luaL_checkinteger(L, 1);
  const double P0 = luaL_checknumber(L, 2), zeta = luaL_checknumber(L, 3);
  const int k1 = (int) luaL_checkinteger(L, 4), seed = (int) luaL_checkinteger(L, 5);
  long long n = 0;
  if (mgpu_new_ou_field(nd, P0, zeta, k1, seed, NULL, &n)) return luaL_error(L, "[Mara] bad new_ou_field arguments");
  char *buf = (char *) malloc((size_t) n);
  if (!buf) return luaL_error(L, "[Mara] out of host memory");
  mgpu_new_ou_field(nd, P0, zeta, k1, seed, buf, &n);
  lua_pushlstring(L, buf, (size_t) n);
  free(buf);
  return 1;
}

static int l_set_driving(lua_State *L)
{
  size_t len = 0;
  const char *f = luaL_checklstring(L, 1, &len);
  const int rc = mgpu_set_driving(solver(L), f, (long long) len);
  if (rc) return raise_abi(L, rc, "set_driving");
  return 0;
}

static int l_driving_advance(lua_State *L)
{
  const int rc = mgpu_driving_advance(solver(L), luaL_checknumber(L, 1));
  if (rc) return raise_abi(L, rc, "driving.Advance");
  return 0;
}

static int l_driving_resample(lua_State *L)
{
  const int rc = mgpu_driving_resample(solver(L));
  if (rc) return raise_abi(L, rc, "driving.Resample");
  return 0;
}

static int l_driving_serialize(lua_State *L)
{
  long long n = 0;
  mgpu_solver *h = solver(L);
  int rc = mgpu_driving_serialize(h, NULL, &n);
  if (rc) return raise_abi(L, rc, "driving.Serialize");
  if (n == 0) return 0;   /* no driving: nothing, as the reference */
  char *buf = (char *) malloc((size_t) n);
  if (!buf) return luaL_error(L, "[Mara] out of host memory");
  rc = mgpu_driving_serialize(h, buf, &n);
  if (rc) {
    free(buf);
    return raise_abi(L, rc, "driving.Serialize");
  }
  lua_pushlstring(L, buf, (size_t) n);
  free(buf);
  return 1;
}

static int l_driving_power(lua_State *L)
{
  double p = 0.0;
  const int rc = mgpu_driving_power(solver(L), &p);
  if (rc) return raise_abi(L, rc, "driving.Power");
  lua_pushnumber(L, p);
  return 1;
}

static int l_gpu_stats(lua_State *L)
{
  mgpu_stats s;
  const int rc = mgpu_get_stats(solver(L), &s);
  if (rc) return raise_abi(L, rc, "gpu_stats");
  lua_newtable(L);
#define FIELD(name, val) (lua_pushnumber(L, (double) (val)), lua_setfield(L, -2, name))
  FIELD("max_lambda", s.max_lambda);
  FIELD("dt", s.dt);
  FIELD("errors", s.errors);
  FIELD("committed", s.committed);
  FIELD("c2p_calls", s.c2p_calls);
  FIELD("c2p_iters", s.c2p_iters);
  FIELD("face_c2p_calls", s.face_c2p_calls);
  FIELD("face_c2p_iters", s.face_c2p_iters);
  FIELD("hlld_ok", s.hlld_ok);
  FIELD("hlld_hllc", s.hlld_hllc);
  FIELD("pcm_retry", s.pcm_retry);
#undef FIELD
  return 1;
}

/* ---- Mara.measure.* ---------------------------------------------------------------------- */

static int l_mean_max_divB(lua_State *L)
{
  double mean = 0.0, mx = 0.0;
  const int rc = mgpu_measure_divB(solver(L), &mean, &mx);
  if (rc) return raise_abi(L, rc, "mean_max_divB");
  lua_pushnumber(L, mean);
  lua_pushnumber(L, mx);
  return 2;
}

static int l_max_lorentz_factor(lua_State *L)
{
  double w = 0.0;
  const int rc = mgpu_max_lorentz_factor(solver(L), &w);
  if (rc) return raise_abi(L, rc, "max_lorentz_factor");
  lua_pushnumber(L, w);
  return 1;
}

static int push_array(lua_State *L, const double *a, int n)   /* luaU_pusharray, mara.cpp:1882 */
{
  lua_newtable(L);
  for (int i = 0; i < n; ++i) {
    lua_pushnumber(L, a[i]);
    lua_rawseti(L, -2, i + 1);
  }
  return 1;
}

static int l_mean_cons(lua_State *L)
{
  double a[8];
  const int rc = mgpu_measure_mean_cons(solver(L), a);
  if (rc) return raise_abi(L, rc, "mean_cons");
  return push_array(L, a, 8);
}

static int l_mean_prim(lua_State *L)
{
  double a[8];
  const int rc = mgpu_measure_mean_prim(solver(L), a);
  if (rc) return raise_abi(L, rc, "mean_prim");
  return push_array(L, a, 8);
}

static int l_mean_velocity(lua_State *L)
{
  double a[4];
  const int rc = mgpu_measure_mean_velocity(solver(L), a);
  if (rc) return raise_abi(L, rc, "mean_velocity");
  return push_array(L, a, 4);
}

static int l_mean_energies(lua_State *L)   /* a table keyed as luaC_mean_energies' */
{
  double a[4];
  const int rc = mgpu_measure_mean_energies(solver(L), a);
  if (rc) return raise_abi(L, rc, "mean_energies");
  lua_newtable(L);
  lua_pushstring(L, "magnetic"); lua_pushnumber(L, a[0]); lua_settable(L, -3);
  lua_pushstring(L, "kinetic");  lua_pushnumber(L, a[1]); lua_settable(L, -3);
  lua_pushstring(L, "internal"); lua_pushnumber(L, a[2]); lua_settable(L, -3);
  lua_pushstring(L, "total");    lua_pushnumber(L, a[3]); lua_settable(L, -3);
  return 1;
}

#define MEAN_EXTREME(fn, api, name)                    \
  static int fn(lua_State *L)                          \
  {                                                    \
    double a = 0.0, b = 0.0;                           \
    const int rc = api(solver(L), &a, &b);             \
    if (rc) return raise_abi(L, rc, name);             \
    lua_pushnumber(L, a);                              \
    lua_pushnumber(L, b);                              \
    return 2;                                          \
  }
MEAN_EXTREME(l_mean_max_temperature, mgpu_measure_mean_max_temperature, "mean_max_temperature")
MEAN_EXTREME(l_mean_max_magnetic_field, mgpu_measure_mean_max_magnetic_field, "mean_max_magnetic_field")
MEAN_EXTREME(l_mean_max_sonic_mach, mgpu_measure_mean_max_sonic_mach, "mean_max_sonic_mach")
MEAN_EXTREME(l_mean_min_alfvenic_mach, mgpu_measure_mean_min_alfvenic_mach, "mean_min_alfvenic_mach")
#undef MEAN_EXTREME

/* luaC_Mara_diffuse (mara.cpp:343-366): Mara.diffuse(P, r), P changed in place */
static int l_diffuse(lua_State *L)
{
  double *P = check_prim_buffer(L, 1);
  const double r = luaL_checknumber(L, 2);
  int err = 0;
  const int rc = mgpu_diffuse_host(solver(L), P, r, &err);
  if (rc) return raise_abi(L, rc, "diffuse");
  return 0;
}

/* luaC_Mara_set_failmask (mara.cpp:368-373) */
static int l_set_failmask(lua_State *L)
{
  const int value = (int) luaL_checkinteger(L, 1);
  printf("[Mara] set fail mask value everywhere to %d\n", value);
  const int rc = mgpu_set_failmask(solver(L), value);
  if (rc) return raise_abi(L, rc, "set_failmask");
  return 0;
}

/* luaC_cooling_rate (mara.cpp:1296-1308): the GPU module has no cooling (set_cooling is not
 * provided), so the rate is the reference's value without a cooling module, 0. */
static int l_cooling_rate(lua_State *L)
{
  (void) luaL_checknumber(L, 1);
  lua_pushnumber(L, 0.0);
  return 1;
}

/* ---- Mara.fluid.* ------------------------------------------------------------------------ */

static int l_GetPrimNames(lua_State *L)
{
  static const char *names[8] = {"rho", "pre", "vx", "vy", "vz", "Bx", "By", "Bz"};   /* rmhd.cpp:28-34 */
  lua_newtable(L);
  for (int n = 0; n < 8; ++n) {
    lua_pushstring(L, names[n]);
    lua_rawseti(L, -2, n + 1);
  }
  return 1;
}

/* Entry points of the reference that are not part of the RMHD step. */
static int l_not_provided(lua_State *L)
{
  return luaL_error(L, "[Mara] %s is not provided by the GPU module", lua_tostring(L, lua_upvalueindex(1)));
}

static void register_absent(lua_State *L, const char *const *names)
{
  for (; *names; ++names) {
    lua_pushstring(L, *names);
    lua_pushcclosure(L, l_not_provided, 1);
    lua_setfield(L, -2, *names);
  }
}

int luaopen_Mara(lua_State *L)
{
  static const luaL_Reg module[] = {
      {"start", l_start},
      {"close", l_close},
      {"git_sha", l_git_sha},
      {"advance", l_advance},
      {"init_prim", l_init_prim},
      {"get_timestep", l_get_timestep},
      {"set_domain", l_set_domain},
      {"set_boundary", l_set_boundary},
      {"set_fluid", l_set_fluid},
      {"set_eos", l_set_eos},
      {"set_godunov", l_set_godunov},
      {"set_riemann", l_set_riemann},
      {"set_advance", l_set_advance},
      {"set_primitive", l_set_primitive},
      {"config_solver", l_config_solver},
      {"set_c2p_network", l_set_c2p_network},
      {"new_ou_field", l_new_ou_field},
      {"set_driving", l_set_driving},
      {"gpu_stats", l_gpu_stats},
      {"upload_primitive", l_upload_primitive},
      {"advance_device", l_advance_device},
      {"download_primitive", l_download_primitive},
      {"diffuse", l_diffuse},
      {"set_failmask", l_set_failmask},
      {"cooling_rate", l_cooling_rate},
      {NULL, NULL}};
  static const char *const absent[] = {"show", "prim_at_point", "set_units",
                                       "set_cooling", "set_fluxsrc", "set_srcterm",
                                       "load_shen", "test_shen",
                                       "test_rmhd_c2p", "test_sampling", "test_sampling_many", NULL};
  static const luaL_Reg measure[] = {{"mean_max_divB", l_mean_max_divB},
                                     {"max_lorentz_factor", l_max_lorentz_factor},
                                     {"mean_cons", l_mean_cons},
                                     {"mean_prim", l_mean_prim},
                                     {"mean_energies", l_mean_energies},
                                     {"mean_velocity", l_mean_velocity},
                                     {"mean_max_temperature", l_mean_max_temperature},
                                     {"mean_max_magnetic_field", l_mean_max_magnetic_field},
                                     {"mean_max_sonic_mach", l_mean_max_sonic_mach},
                                     {"mean_min_alfvenic_mach", l_mean_min_alfvenic_mach},
                                     {NULL, NULL}};
  static const char *const measure_absent[] = {NULL};
  static const luaL_Reg fluid[] = {{"GetPrimNames", l_GetPrimNames}, {NULL, NULL}};
  static const char *const fluid_absent[] = {"PrimToCons", "ConsToPrim", "Eigensystem", "FluxFunction", NULL};

  lua_newtable(L);
  luaL_setfuncs(L, module, 0);
  register_absent(L, absent);

  lua_newtable(L);
  luaL_setfuncs(L, measure, 0);
  register_absent(L, measure_absent);
  lua_setfield(L, -2, "measure");

  lua_newtable(L);
  luaL_setfuncs(L, fluid, 0);
  register_absent(L, fluid_absent);
  lua_setfield(L, -2, "fluid");

  static const luaL_Reg driving[] = {{"Advance", l_driving_advance},
                                     {"Resample", l_driving_resample},
                                     {"Serialize", l_driving_serialize},
                                     {"Power", l_driving_power},
                                     {NULL, NULL}};
  lua_newtable(L);
  luaL_setfuncs(L, driving, 0);
  lua_setfield(L, -2, "driving");

  static const char *const sub[] = {"eos", "units", "image", "models", NULL};
  for (const char *const *s = sub; *s; ++s) {
    lua_newtable(L);
    lua_setfield(L, -2, *s);
  }
  return 1;
}
