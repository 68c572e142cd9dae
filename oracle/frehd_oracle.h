/* CPU restatement oracle of the FrehdC step (test infrastructure only). */
#ifndef FREHD_ORACLE_H
#define FREHD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Same fields, order and meaning as frehd_config in include/frehd_b200.h. */
typedef struct oracle_cfg {
  int nx, ny;
  double dx, dy, dt;
  double g, NUx, NUy, Kx, Ky;
  double CDx, CDy, manningN, CDmax, hD, CwT;
  int CDnotN, useThinLayer;
  int useSubgrid, useSubDrag, staggeredV, useminA, useminV;
  double dxf, dyf, subR;
  double surfmin, surfmax, dsurf;
  int bcType;
  int tideLocFirstP, tideLocLengthP;
  int useScalar, scalarAdv, useConstTidePS;
  double tidePS;
  int useWind, useEvap, useRain, inflowLocLength, useSubStep, checkConservation;
  double minDepth, wtfh, CFLl, CFLh;
  double eps;
  int maxIter;
  double offset;
  int inflowI0, inflowI1, inflowJ0, inflowJ1;
  double inflowS;
  double northAngle, rhoa, Cw;
} oracle_cfg;

typedef struct oracle_domain oracle_domain;

enum { ORACLE_PRECOND_JACOBI = 0, ORACLE_PRECOND_SSOR = 1 };
enum { ORACLE_X0_ZERO = 0, ORACLE_X0_SURFACE = 1 };

oracle_domain *oracle_create(const oracle_cfg *cfg, char *errbuf, int errlen);
void oracle_destroy(oracle_domain *d);
const char *oracle_error(const oracle_domain *d);
int oracle_set_tables(oracle_domain *d, int Ne, const double *tables);
int oracle_set_tide(oracle_domain *d, int n, const double *tideP);
/* bc->inflow (kind 1), bc->windspd (2), bc->winddir (3), indexed by tt. */
int oracle_set_series(oracle_domain *d, int kind, int n, const double *values);
void oracle_set_solver(oracle_domain *d, int precond, int x0mode);
int oracle_init(oracle_domain *d, const double *bottom, const double *bottomXP,
                const double *bottomYP, const double *surf0, const double *u0,
                const double *v0, const double *S0, int round_trip_output);
void oracle_explicit(oracle_domain *d, int tt);
void oracle_solve(oracle_domain *d);
double oracle_update(oracle_domain *d, int tt, const double *x);
double oracle_step(oracle_domain *d, int tt);
const double *oracle_solution(const oracle_domain *d);
int oracle_last_iters(const oracle_domain *d);
double oracle_last_accuracy(const oracle_domain *d);
long oracle_field_len(oracle_domain *d, const char *name);
int oracle_get(oracle_domain *d, const char *name, double *out, long n);
int oracle_set(oracle_domain *d, const char *name, const double *in, long n);

#ifdef __cplusplus
}
#endif
#endif
