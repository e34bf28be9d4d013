/* CPU restatement of Mara's RMHD step (test infrastructure, not product code).
 *
 * A single-threaded FP64 restatement of the reference algorithm, written to be read
 * against the reference sources (citations are per function, file:line within the
 * reference project).  It keeps the reference's AoS layout with guard zones:
 * zone index ((i*Gy + j)*Gz + k), 8 doubles per zone, x slowest, component fastest
 * (Mara/hydro.cpp:80-110).  It is pinned against the compiled reference by the tests
 * (tests/test_oracle_port.py) and serves as the checker of the CUDA path.
 */
#ifndef MARA_PORT_H
#define MARA_PORT_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int    nd;          /* 1, 2 or 3 */
  int    n[3];        /* interior zones per dimension (1 for unused dims) */
  int    ng;          /* guard zones per side (the reference always uses 3) */
  double x0[3], x1[3];
  double gamma;       /* adiabatic index of the gamma-law EOS */
  int    recon;       /* 0 pcm, 1 plm, 2 weno5 */
  double theta;       /* PLM minmod theta */
  int    is_mode;     /* WENO smoothness indicator: 0 js96, 1 b08, 2 sz10 */
  double sz10A;
  int    riemann;     /* 0 hll, 1 hllc, 2 hlld */
  int    rk;          /* 1 single, 2 rk2 (TVD), 3 rk3 (Shu-Osher), 4 rk4 (classic) */
  double pfloor;      /* c2p pressure floor, disabled when <= 0 */
  int    ereset;      /* emergency reset of failed zones */
  double preset, dreset;
  int    godunov;     /* 0 plm-split (MethodOfLinesSplit), 1 plm-muscl (PlmCtuHancockOperator) */
} port_config;

typedef struct {
  double max_lambda;      /* RiemannSolver::MaxLambda */
  long   hlld_success;    /* HlldRmhdRiemannSolver::NumberOfSuccess */
  long   hlld_failure;    /* HlldRmhdRiemannSolver::NumberOfFailure */
  int    hlld_path;       /* the last HLLD face (test instrumentation, not in the reference):
                             1-3 = the attempt whose pressure guess succeeded, 0 = the HLL-state
                             c2p failed, 4 = all attempts failed (both: HLLC fallback) */
} port_stats;

void   port_default_config(port_config *c);
long   port_num_zones(const port_config *c);

int    port_prim_to_cons(const port_config *c, const double *P, double *U);
int    port_cons_to_prim(const port_config *c, const double *U, double *P);
int    port_c2p_solve(const port_config *c, const double *U, int solver, int guess,
                      const double *Pguess, double *P, int *iters);
void   port_flux_and_eigenvalues(const port_config *c, const double *U, const double *P,
                                 double *F, double *ap, double *am, int dim);
int    port_quartic(double d4, double d3, double d2, double d1, double d0, double *roots);
double port_reconstruct(const port_config *c, const double *v, int op);
int    port_riemann(const port_config *c, port_stats *s, const double *pl,
                    const double *pr, double *F, int dim);
void   port_ct3d(double *Fx, double *Fy, double *Fz, const int *stride);
void   port_ct2d(double *Fx, double *Fy, const int *stride);

int    port_advance(const port_config *c, port_stats *s, double *prim, double dt,
                    int *errors);
double port_timestep(const port_config *c, double max_lambda, double cfl);
void   port_mean_max_divB(const port_config *c, const double *prim, double *mean,
                          double *max);
double port_max_lorentz_factor(const port_config *c, const double *prim);

int    port_diffuse(const port_config *c, double *prim, double r, const int *mask_in, const double *prev,
                    int *mask_out);
void   port_measures(const port_config *c, const double *P, double *out);

#ifdef __cplusplus
}
#endif
#endif
