/* Driving shim for the compiled reference (test infrastructure only).
 *
 * Exposes a plain C API over the reference's own public entry points so that Python
 * tests can call them through ctypes:
 *   - the Lua module `Mara` (Mara/mara.cpp:137-268), driven through a private Lua 5.2
 *     state exactly as a ctf-main script would (start, set_*, config_solver, set_domain,
 *     advance, get_timestep, measure.*);
 *   - the per-state C++ objects behind it (Mara/rmhd.cpp, Mara/riemann_hll*.cpp,
 *     Mara/weno.c, Mara/rmhd-c2p.c) for function-level golden vectors.
 * Nothing here re-implements physics: every number comes out of the reference code.
 */
#include <cstdio>
#include <cstring>
#include <string>
#include <valarray>

extern "C" {
#include "lua.h"
#include "lauxlib.h"
#include "lualib.h"
#include "weno.h"
#include "rmhd-c2p.h"
int luaopen_Mara(lua_State *L);
int luaopen_buffer(lua_State *L);
}
#include "hydro.hpp"
#include "rmhd.hpp"

static lua_State *L = NULL;
static std::string last_error;

static int fail(const char *what)
{
  last_error = what;
  return 1;
}

extern "C" {

const char *ref_last_error(void) { return last_error.c_str(); }

int ref_open(void)
{
  if (L) lua_close(L);
  L = luaL_newstate();
  luaL_openlibs(L);
  luaL_requiref(L, "Mara", luaopen_Mara, 1);
  lua_pop(L, 1);
  luaL_requiref(L, "buffer", luaopen_buffer, 1);   /* as ctf-core/ctf.c preloads it */
  lua_pop(L, 1);
  return 0;
}

int ref_close(void)
{
  if (L) {
    luaL_dostring(L, "Mara.close()");
    lua_close(L);
    L = NULL;
  }
  return 0;
}

/* Run a chunk of Lua in the shim's state (used for Mara.start / set_* / set_domain). */
int ref_dostring(const char *code)
{
  if (!L) return fail("ref_open not called");
  if (luaL_dostring(L, code)) {
    last_error = lua_tostring(L, -1);
    lua_pop(L, 1);
    return 1;
  }
  return 0;
}

/* Mara.advance(buf, dt) -> kzps, errors.  `prim` is the AoS primitive array with guard
 * zones (G^d x 8 doubles); it is copied into a Lua userdata, advanced, copied back. */
int ref_advance(double *prim, long n, double dt, double *kzps, int *errors)
{
  if (!L) return fail("ref_open not called");
  lua_getglobal(L, "Mara");
  lua_getfield(L, -1, "advance");
  void *ud = lua_newuserdata(L, n * sizeof(double));
  memcpy(ud, prim, n * sizeof(double));
  lua_pushvalue(L, -1);
  lua_setglobal(L, "__ref_buf");          /* keep alive across the call */
  lua_pushnumber(L, dt);
  if (lua_pcall(L, 2, 2, 0)) {
    last_error = lua_tostring(L, -1);
    lua_pop(L, 2);
    return 1;
  }
  if (kzps) *kzps = lua_tonumber(L, -2);
  if (errors) *errors = (int) lua_tonumber(L, -1);
  lua_pop(L, 3);
  memcpy(prim, ud, n * sizeof(double));
  lua_pushnil(L);
  lua_setglobal(L, "__ref_buf");
  return 0;
}

static int call_numbers(const char *tbl, const char *fn, double arg, int use_arg,
                        int nret, double *out)
{
  if (!L) return fail("ref_open not called");
  lua_getglobal(L, "Mara");
  if (tbl) lua_getfield(L, -1, tbl);
  lua_getfield(L, -1, fn);
  int nargs = 0;
  if (use_arg) { lua_pushnumber(L, arg); nargs = 1; }
  if (lua_pcall(L, nargs, nret, 0)) {
    last_error = lua_tostring(L, -1);
    lua_pop(L, tbl ? 3 : 2);
    return 1;
  }
  for (int i = 0; i < nret; ++i) out[i] = lua_tonumber(L, -nret + i);
  lua_pop(L, nret + (tbl ? 2 : 1));
  return 0;
}

int ref_get_timestep(double cfl, double *dt)
{
  return call_numbers(NULL, "get_timestep", cfl, 1, 1, dt);
}

int ref_set_primitive(const double *prim, long n)
{
  if (!L) return fail("ref_open not called");
  lua_getglobal(L, "Mara");
  lua_getfield(L, -1, "set_primitive");
  void *ud = lua_newuserdata(L, n * sizeof(double));
  memcpy(ud, prim, n * sizeof(double));
  if (lua_pcall(L, 1, 0, 0)) {
    last_error = lua_tostring(L, -1);
    lua_pop(L, 2);
    return 1;
  }
  lua_pop(L, 1);
  return 0;
}

int ref_mean_max_divB(double *mean, double *max)
{
  double r[2];
  int e = call_numbers("measure", "mean_max_divB", 0, 0, 2, r);
  *mean = r[0];
  *max = r[1];
  return e;
}

int ref_max_lorentz_factor(double *w)
{
  return call_numbers("measure", "max_lorentz_factor", 0, 0, 1, w);
}

/* Mara.diffuse(buf, r) (Mara/mara.cpp:343-366) on a copy of `prim`, copied back. */
int ref_diffuse(double *prim, long n, double r)
{
  if (!L) return fail("ref_open not called");
  lua_getglobal(L, "Mara");
  lua_getfield(L, -1, "diffuse");
  void *ud = lua_newuserdata(L, n * sizeof(double));
  memcpy(ud, prim, n * sizeof(double));
  lua_pushvalue(L, -1);
  lua_setglobal(L, "__ref_buf");
  lua_pushnumber(L, r);
  if (lua_pcall(L, 2, 0, 0)) {
    last_error = lua_tostring(L, -1);
    lua_pop(L, 2);
    return 1;
  }
  lua_pop(L, 1);
  memcpy(prim, ud, n * sizeof(double));
  lua_pushnil(L);
  lua_setglobal(L, "__ref_buf");
  return 0;
}

int ref_set_failmask(int value)
{
  char code[64];
  snprintf(code, sizeof(code), "Mara.set_failmask(%d)", value);
  return ref_dostring(code);
}

/* Mara.measure.<name>() -> up to nmax numbers: the returned numbers, or the entries 1..n of
 * a returned array table, or (mean_energies) the keys magnetic, kinetic, internal, total. */
int ref_measure(const char *name, double *out, int nmax, int *nout)
{
  if (!L) return fail("ref_open not called");
  const int top = lua_gettop(L);
  lua_getglobal(L, "Mara");
  lua_getfield(L, -1, "measure");
  lua_getfield(L, -1, name);
  if (lua_pcall(L, 0, LUA_MULTRET, 0)) {
    last_error = lua_tostring(L, -1);
    lua_settop(L, top);
    return 1;
  }
  const int nret = lua_gettop(L) - (top + 2);
  int n = 0;
  if (nret == 1 && lua_istable(L, -1)) {
    if (lua_rawlen(L, -1) > 0) {
      for (int i = 1; i <= (int) lua_rawlen(L, -1) && n < nmax; ++i) {
        lua_rawgeti(L, -1, i);
        out[n++] = lua_tonumber(L, -1);
        lua_pop(L, 1);
      }
    } else {
      static const char *keys[4] = {"magnetic", "kinetic", "internal", "total"};
      for (int i = 0; i < 4 && n < nmax; ++i) {
        lua_getfield(L, -1, keys[i]);
        out[n++] = lua_tonumber(L, -1);
        lua_pop(L, 1);
      }
    }
  } else {
    for (int i = 0; i < nret && n < nmax; ++i) out[n++] = lua_tonumber(L, top + 3 + i);
  }
  *nout = n;
  lua_settop(L, top);
  return 0;
}

/* ---- function-level access to the reference objects ------------------------------- */

static MaraApplication *app(void) { return HydroModule::Mara; }

/* GodunovOperator's FailureMask and the application's PrimitiveArray (the state the next
 * Mara.diffuse reads), copied out: n entries / n doubles at most; returns the count. */
long ref_failure_mask(int *out, long n)
{
  const std::valarray<int> &m = app()->FailureMask;
  long k = 0;
  for (; k < (long) m.size() && k < n; ++k) out[k] = m[k];
  return k;
}

long ref_primitive_array(double *out, long n)
{
  const std::valarray<double> &P = app()->PrimitiveArray;
  long k = 0;
  for (; k < (long) P.size() && k < n; ++k) out[k] = P[k];
  return k;
}

int ref_prim_to_cons(const double *P, double *U)
{
  return app()->fluid->PrimToCons(P, U);
}

/* Rmhd::ConsToPrim (Mara/rmhd.cpp:103-176).  P is the previous-prim guess on entry and
 * the result on success (it is left untouched on failure, as in the reference). */
int ref_cons_to_prim(const double *U, double *P)
{
  return app()->fluid->ConsToPrim(U, P);
}

void ref_flux_and_eigenvalues(const double *P, int dim, double *F, double *ap, double *am)
{
  double U[8];
  app()->fluid->PrimToCons(P, U);
  app()->fluid->FluxAndEigenvalues(U, P, F, ap, am, dim);
}

/* Mara->riemann->IntercellFlux(Pl, Pr, 0, F, 0.0, dim) (the call made by
 * Mara/plm-split.cpp:68). Updates the reference's static MaxLambda. */
int ref_riemann(const double *Pl, const double *Pr, int dim, double *F)
{
  return app()->riemann->IntercellFlux(Pl, Pr, 0, F, 0.0, dim);
}

double ref_get_max_lambda(void) { return RiemannSolver::GetMaxLambda(); }
void ref_reset_max_lambda(void) { RiemannSolver::ResetMaxLambda(); }

/* reconstruct(v, op) from Mara/weno.c:58-71; v points at the central value of a
 * stencil v[-2..2] (op codes as in Mara/weno.h). */
double ref_reconstruct(const double *v, int op)
{
  return reconstruct(v, (enum ReconstructOperation) op);
}

void ref_ct3d(double *Fx, double *Fy, double *Fz, const int *stride)
{
  int s[4] = { stride[0], stride[1], stride[2], stride[3] };
  app()->fluid->ConstrainedTransport3d(Fx, Fy, Fz, s);
}

void ref_ct2d(double *Fx, double *Fy, const int *stride)
{
  int s[4] = { stride[0], stride[1], stride[2], stride[3] };
  app()->fluid->ConstrainedTransport2d(Fx, Fy, s);
}

/* One c2p solver run (Mara/rmhd-c2p.c): solver 0 = anton2dzw, 1 = noble1dw; guess 0 =
 * estimate_from_cons, 1 = set_starting_prim(Pguess).  Returns the error code. */
int ref_c2p_solver(const double *U, int solver, int guess, const double *Pguess,
                   double gamma, double *P, int *iters)
{
  rmhd_c2p_set_gamma(gamma);
  rmhd_c2p_new_state(U);
  if (guess == 0) rmhd_c2p_estimate_from_cons();
  else rmhd_c2p_set_starting_prim(Pguess);
  int e = solver == 0 ? rmhd_c2p_solve_anton2dzw(P) : rmhd_c2p_solve_noble1dw(P);
  if (iters) *iters = rmhd_c2p_get_iterations();
  return e;
}

}
