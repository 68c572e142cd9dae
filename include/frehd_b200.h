/*
 * frehd_b200.h -- C ABI of the B200 implementation of FrehdC's semi-implicit
 * (Casulli) time step with subgrid bathymetry.
 *
 * Everything here is plain C: integers, doubles and pointers to host arrays.
 * Host arrays use the reference model's own linear layout (map.c:45-127):
 *   interior cell (i, j)      -> ii = j*nx + i,            ii in [0, N),  N = nx*ny
 *   ghost ring appended after the interior, N2ct = (nx+2)*(ny+2) entries in total:
 *     [N,        N+nx)        row j = ny   (north / "jP" ghosts)
 *     [N+nx,     N+2nx)       row j = -1   (south / "jM" ghosts)
 *     [N+2nx,    N+2nx+ny)    column i = nx (east / "iP" ghosts)
 *     [N+2nx+ny, N+2nx+2ny)   column i = -1 (west / "iM" ghosts)
 *     N2ct-4 .. N2ct-1        corners (i,j) = (-1,ny), (nx,ny), (nx,-1), (-1,-1)
 * An array documented as "N2ct" carries the ghost ring, "N" is interior only.
 * Subgrid tables are level-major like the reference's all* arrays:
 *   table[N*k + ii] is the value of cell ii at level k (subgrid.c:118-119).
 *
 * The device keeps every domain resident in HBM in a padded 2-D layout and only
 * copies to the host when asked to.  All entry points return a status code
 * (FREHD_OK == 0); none of them aborts the process.
 */
#ifndef FREHD_B200_H
#define FREHD_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
enum frehd_status {
  FREHD_OK = 0,
  FREHD_ERR_INVALID = 1,        /* bad argument, size or null pointer */
  FREHD_ERR_UNSUPPORTED = 2,    /* a Config option this build does not implement */
  FREHD_ERR_CUDA = 3,           /* CUDA runtime error (message: frehd_last_error) */
  FREHD_ERR_NOMEM = 4,          /* device allocation failed */
  FREHD_ERR_CG_NOCONVERGE = 5,  /* CG reached maxIter before ||r|| < eps*||b|| */
  FREHD_ERR_CFL = 6,            /* max CFL > 20; the reference exits here (nsfunctions.c:1226-1231) */
  FREHD_ERR_TIMEOUT = 7,        /* a bounded device-side wait gave up */
  FREHD_ERR_STATE = 8           /* call out of order (e.g. step before geometry is set) */
};

/* Human-readable name of a status code. */
const char *frehd_status_string(int status);
/* Text of the last error raised in this thread (empty when none). */
const char *frehd_last_error(void);
/* Library version string. */
const char *frehd_version(void);
/* Number of CUDA devices visible to the library. */
int frehd_device_count(int *count);

/* ------------------------------------------------------------------ config */
/*
 * The fields of the reference's Config (configuration.h:4-111) that the step
 * reads, with the same names and meaning.  frehd_config_defaults() fills in the
 * values of the shipped data.dat (frehdc5+/data.dat:1-103).
 */
typedef struct frehd_config {
  int nx, ny;                 /* interior cells (NX, NY with one rank) */
  double dx, dy, dt;
  double g, NUx, NUy, Kx, Ky;
  double CDx, CDy, manningN, CDmax, hD, CwT;
  int CDnotN, useThinLayer;
  int useSubgrid, useSubDrag, staggeredV, useminA, useminV;
  double dxf, dyf, subR;      /* fine grid and r = dx/dxf */
  double surfmin, surfmax, dsurf;
  int bcType;                 /* 1: tide on the YP row (j = ny-1) */
  int tideLocFirstP, tideLocLengthP; /* tidal cells (tideLocFirstP + k, ny-1) */
  int useScalar, scalarAdv, useConstTidePS;
  double tidePS;
  int useWind, useEvap, useRain, inflowLocLength, useSubStep, checkConservation;
  double minDepth, wtfh, CFLl, CFLh;
  double eps;                 /* CG stop: ||r||_2 < eps*||b||_2 (rtc.c:53) */
  int maxIter;
  double offset;              /* bathymetry offset -min(z) (bathymetry.c:98-102) */
  /* forcing (configuration.c:53-65,71,78-79) */
  int inflowI0, inflowI1;     /* inflow cells: i in [inflowI0, inflowI1), the data.dat first and
                                 last i-index minus one (configuration.c:57) ... */
  int inflowJ0, inflowJ1;     /* ... and j in [inflowJ0, inflowJ1); inflowLocLength cells */
  double inflowS;             /* scalar concentration of the inflow */
  double northAngle, rhoa, Cw; /* wind (useWind = 1): direction offset in degrees, air
                                  density, wind drag coefficient */
  int nscalar;                /* scalars transported when useScalar = 1, 1 .. FREHD_MAX_SCALARS
                                 (0 counts as 1).  Scalar 0 is the reference's S; the others are
                                 passive tracers with S's transport, boundary and inflow values
                                 (tidePS, inflowS), each one what the reference computes for S
                                 when S starts from that tracer's field. */
} frehd_config;

#define FREHD_MAX_SCALARS 4

void frehd_config_defaults(frehd_config *cfg);

/* ------------------------------------------------------- host pre-processing */
/*
 * Subgrid tables of a deck from its fine bottoms (no GPU needed).  Replaces the
 * reference's MATLAB pre-processor (preProcessing/script_CreateSubAreaWithBlockV16.m
 * with checkBlock = 0) whose output files subgrid.c:2089-2284 reads.
 *   zf      fine bottoms, zf[fj*fpitch + fi], (ny*r) rows of (nx*r) pixels
 *   tables  10*Ne*N doubles: V, Z, Vxp, Vxm, Vyp, Vym, Np, Nm, Op, Om, each level-major
 */
int frehd_build_tables(const double *zf, long fpitch, int nx, int ny, int r,
                       double dxf, double dyf, double surfmin, double dsurf, int Ne,
                       double *tables);
/* Geometry options of the pre-processor.
 * FREHD_GEOM_BLOCK_CHECK: checkBlock = 1 of script_CreateSubAreaWithBlockV16.m:27
 * (ComputeFaceAreaWithBlockCheck.m): each block's wet pixels are reduced to their
 * largest 4-connected cluster and face areas count only pixel pairs wet in both
 * blocks' clusters.  Needs 1 < r <= 8 (r = 1: no effect). */
enum { FREHD_GEOM_BLOCK_CHECK = 1 };
int frehd_build_tables_ex(const double *zf, long fpitch, int nx, int ny, int r,
                          double dxf, double dyf, double surfmin, double dsurf, int Ne,
                          int flags, double *tables);
/* Coarse bottom.dat / bottomXP.dat / bottomYP.dat of a deck (N doubles each). */
int frehd_build_bottoms(const double *zf, long fpitch, int nx, int ny, int r,
                        double *bottom, double *bottomXP, double *bottomYP);

/* ------------------------------------------------------------ one domain */
typedef struct frehd_domain frehd_domain;

/*
 * State of one domain in the reference layout; every pointer may be NULL (skipped).
 * Field names are those of Data (initialize.h:10-21), Sub (subgrid.h:8-29) and
 * Bath (bathymetry.h:7-14).
 */
typedef struct frehd_state {
  /* persistent model state */
  double *surf;              /* N2ct  free surface incl. offset */
  double *uuXP, *vvYP;       /* N2ct  face velocities */
  double *S;                 /* N2ct  scalar */
  double *depth;             /* N     cell depth */
  double *CDXP, *CDYP;       /* N2ct  drag coefficients */
  double *CFLx, *CFLy;       /* N2ct  previous step's CFL numbers (read by advection) */
  double *V, *Z, *Nx, *Oy, *Vx, *Vy, *Zx, *Zy; /* N2ct subgrid geometry at the current level */
  int *ind;                  /* N2ct  persistent subgrid level index */
  /* static bathymetry */
  double *bottomZ, *bottomXP, *bottomYP;      /* N2ct incl. offset */
  /* per-step quantities (download only) */
  double *surfOld;           /* N2ct  */
  double *uuYP, *vvXP;       /* N     interpolated velocities (velocityInterp) */
  double *EnXP, *EnYP;       /* N2ct  explicit velocities after drag inversion */
  double *cellV, *Sm;        /* N     cell volume and scalar mass after the update */
  double *Fuu, *Fvv;         /* N2ct  face flow rates */
  /* face depths of the last updateAllFaceDepth (nsfunctions.c:143-236), N2ct; held
   * only with useWind = 1, whose term reads them (otherwise skipped) */
  double *depthXP, *depthYP;
} frehd_state;

/* Per-domain counters of the last step. */
typedef struct frehd_step_stats {
  int step;                  /* tt of the last completed step */
  int cg_iters;              /* CG iterations of the last solve */
  int status;                /* status of the last step */
  double cg_rel_residual;    /* ||r||/||b|| at exit */
  double max_cflx, max_cfly; /* monitorCFL maxima (nsfunctions.c:1196-1223) */
  int n_cfl_warn;            /* cells with CFL > 2 (the reference prints one line each) */
  double volume;             /* sum of cellV over the domain after the step */
  int cg_fallback;           /* 1: the solve of the assembled matrix stalled (||r|| did not
                                halve in 400 iterations) and was redone with decoupled rows
                                eliminated; laspack would run on to maxIter */
  int cg_noconverge;         /* 1: the solve stopped at maxIter with ||r|| >= eps*||b|| (laspack's
                                CGIter stops there silently, itersolv.c:399-418; the step went on
                                with that solution) */
} frehd_step_stats;

/* Create an empty domain on CUDA device `device`.  Unsupported Config options
 * give FREHD_ERR_UNSUPPORTED.  A domain's device arrays come from the device's
 * default stream-ordered memory pool (cudaMallocAsync on the domain's stream);
 * the first domain on a device sets that pool's release threshold to keep
 * freed memory for reuse. */
int frehd_domain_create(const frehd_config *cfg, int device, frehd_domain **out);
/* Free a domain: waits for the domain's own stream, then returns its memory to
 * the pool in that stream's order (no device-wide synchronisation).  Refused
 * with FREHD_ERR_STATE while the domain is admitted to a batch
 * (frehd_batch_release hands it back first). */
int frehd_domain_destroy(frehd_domain *d);

/* Geometry source, one of the two:
 *   tables: the reference's subgrid tables (10*Ne*N, see frehd_build_tables);
 *   fine bottoms: the r x r fine pixels; level values are evaluated on the device
 *   with the same arithmetic as frehd_build_tables (no tables in HBM). */
int frehd_domain_set_tables(frehd_domain *d, int Ne, const double *tables);
int frehd_domain_set_fine_bottoms(frehd_domain *d, int r, const double *zf, long fpitch);
/* The same with geometry options (FREHD_GEOM_BLOCK_CHECK), evaluated on the device
 * as frehd_build_tables_ex would tabulate them. */
int frehd_domain_set_fine_bottoms_ex(frehd_domain *d, int r, const double *zf, long fpitch,
                                     int flags);

/* Tidal elevation series bc->tideP (initialize.h:28-32), indexed by step tt. */
int frehd_domain_set_tide(frehd_domain *d, int n, const double *tideP);
/* The other boundary series of BC (initialize.h:28-32, read by readBC,
 * initialize.c:345-378), indexed by step tt like tideP; past the end of a series
 * a step reads zero:
 *   FREHD_SERIES_INFLOW      bc->inflow, m^3/s over all inflow cells
 *   FREHD_SERIES_WIND_SPEED  bc->windspd, m/s (useWind = 1)
 *   FREHD_SERIES_WIND_DIR    bc->winddir, degrees from north before northAngle */
enum { FREHD_SERIES_TIDE = 0, FREHD_SERIES_INFLOW = 1, FREHD_SERIES_WIND_SPEED = 2,
       FREHD_SERIES_WIND_DIR = 3 };
int frehd_domain_set_series(frehd_domain *d, int kind, int n, const double *values);
/* Overwrite entries t0 .. t0+n-1 of a series already set (FREHD_SERIES_TIDE is
 * bc->tideP), for forcing that arrives while the model runs.  The copy is queued
 * on the domain's stream, ahead of the steps queued after it, and allocates
 * nothing; from pinned host memory it returns before the copy is done, so the
 * values must stay untouched until the domain's next synchronisation (a
 * FREHD_SERIES_WIND_DIR update waits for its copy). */
int frehd_domain_update_series(frehd_domain *d, int kind, int t0, int n, const double *values);

/* Copy state in the reference layout to/from the device (NULL fields skipped).
 * An upload (and frehd_domain_init, which uploads) also clears the device status
 * a stopped step left behind (FREHD_ERR_CFL, FREHD_ERR_TIMEOUT): after such a
 * step the domain refuses further steps until its state is set again. */
int frehd_domain_upload_state(frehd_domain *d, const frehd_state *st);
int frehd_domain_download_state(frehd_domain *d, frehd_state *st);
/* Scalar s (0 .. nscalar-1; 0 is frehd_state.S) in the layout of the reference's
 * S: Nt = (nx+2)(ny+2) doubles, interior row-major with the ghost ring appended. */
int frehd_domain_upload_scalar(frehd_domain *d, int s, const double *values);
int frehd_domain_download_scalar(frehd_domain *d, int s, double *values);
/* The reference Init's setup of scalar s from its initial field S0 (N doubles,
 * NULL for zeros; initFieldValues, initialize.c:410-430): the interior from S0,
 * zero on the ghost ring and in dry cells (initialize.c:149).  After
 * frehd_domain_init, for the tracers 1 .. nscalar-1. */
int frehd_domain_init_scalar(frehd_domain *d, int s, const double *S0);

/*
 * Run the reference's initialisation sequence on the device (initialize.c:40-155,
 * subgrid path) from the deck's coarse fields (N doubles each, deck datum, the
 * offset is added here as in bathymetry.c:104-121 and initialize.c:401):
 * bottom / bottomXP / bottomYP (bottom.dat, bottomXP.dat, bottomYP.dat), surf0,
 * u0, v0 and S0 (surfic/uuic/vvic/scalaric.dat).  Geometry and the tide series
 * must be set first.  round_trip_output applies the surface round trip through
 * the output datum that DataOutput performs at tt = 0 (fileio.c:65-66,120-121).
 */
int frehd_domain_init(frehd_domain *d, const double *bottom, const double *bottomXP,
                      const double *bottomYP, const double *surf0, const double *u0,
                      const double *v0, const double *S0, int round_trip_output);

/* One complete step tt (oneCompleteStep, nssolve.c:110-118) followed by
 * monitorCFL (nsfunctions.c:1192-1232).  Returns FREHD_ERR_CFL when the max CFL
 * exceeds 20 (the state is left as the reference leaves it before exiting).
 * Returns FREHD_ERR_CG_NOCONVERGE, a warning, when the solve stopped at maxIter
 * before ||r|| < eps*||b||: the step completed with that solution, as the
 * reference's does. */
int frehd_domain_step(frehd_domain *d, int tt);
/* Steps t0 .. t0+nsteps-1 back to back without host synchronisation; the status
 * is checked once at the end.  Stops early (and reports) on CFL > 20; reports
 * FREHD_ERR_CG_NOCONVERGE, after running every step, when any of their solves
 * stopped at maxIter. */
int frehd_domain_run(frehd_domain *d, int t0, int nsteps);

/* Failure-path testing of the bounded device waits (no counterpart in the
 * reference).  The grid-barrier waits of this domain's solves give up after
 * wait_limit_ns (0: the default of 2 s) and then end the step with
 * FREHD_ERR_TIMEOUT; with skip_barrier_rank >= 0, the CTA of that rank in the
 * next solve leaves before its first grid barrier without arriving, so that the
 * other CTAs' wait runs out (skip_barrier_rank = -1: none).  Nothing faults or
 * hangs: every wait is bounded, and no load or partial sum is in flight at that
 * barrier.  frehd_domain_upload_state / frehd_domain_init clear both settings
 * together with the status. */
int frehd_domain_set_wait_test(frehd_domain *d, long long wait_limit_ns, int skip_barrier_rank);

/* Phases of one step, for parity testing against the reference's functions:
 *   FREHD_PHASE_EXPLICIT  solveSourceTerm + matrixCoeffSub/adjust*Boundary (nssolve.c:121-166)
 *   FREHD_PHASE_SOLVE     the free-surface solve (nsfunctions.c:1004-1017)
 *   FREHD_PHASE_UPDATE    getFreeSurface .. enforceTidalBC, updateData, scalarTransport,
 *                         monitorCFL (nssolve.c:169-290, scalar.c:30-57, nsfunctions.c:1192)
 * FREHD_PHASE_UPDATE may take an externally solved surface (x_ext, N doubles in
 * the reference's transposed order k = i*ny + j, as the laspack vector x). */
enum { FREHD_PHASE_EXPLICIT = 1, FREHD_PHASE_SOLVE = 2, FREHD_PHASE_UPDATE = 3 };
int frehd_domain_phase(frehd_domain *d, int phase, int tt, const double *x_ext);

/* Download the assembled system of the last FREHD_PHASE_EXPLICIT in the
 * reference's terms: GnCt/GnXP/GnXM/GnYP/GnYM (row-major, N each) and the
 * right-hand side z (transposed order, N).  NULL pointers skipped. */
int frehd_domain_download_system(frehd_domain *d, double *GnCt, double *GnXP, double *GnXM,
                                 double *GnYP, double *GnYM, double *z);
/* Download the last solution x (transposed order, N). */
int frehd_domain_download_solution(frehd_domain *d, double *x);

int frehd_domain_stats(frehd_domain *d, frehd_step_stats *out);
/* Wait for all work queued on the domain's stream. */
int frehd_domain_sync(frehd_domain *d);

/* ------------------------------------------------------------ output files */
/*
 * The reference's output files written from the device state: one value per
 * line as fprintf("%4.4f \n") prints it (WriteFile, fileio.c:158-181), to
 * <prefix><name>_<tt>.dat, formatted on the GPU with printf's rounding (to
 * nearest, ties to even, on the exact binary value); only the text crosses to
 * the host.
 *   frehd_domain_write_output: the files of DataOutput (fileio.c:62-122) and
 *     SubOutput (fileio.c:125-155) selected by `fields`: uVelocity, vVelocity,
 *     surfaceZ (surf - offset), depth, cdxp and cdyp, scalar (and scalar1 ..
 *     scalar<nscalar-1> for the tracers); SubNx, SubOy, SubVx, SubVy, SubV, SubZ.
 *     Like DataOutput it then round-trips the
 *     interior surface through the output datum (surf = (surf - offset) + offset),
 *     which the next step starts from.
 *   frehd_domain_write_restart: restart_<tt>.dat of writeRestartFile
 *     (fileio.c:192-242): tNEnd, dx, dy, then surf - offset, uu, vv and S.
 *   frehd_format_fixed4: the same formatting of n host values into `out`
 *     (`*len` bytes; `out` may be NULL to ask for the length).
 */
enum { FREHD_OUT_SURFACE = 1, FREHD_OUT_U = 2, FREHD_OUT_V = 4, FREHD_OUT_DEPTH = 8,
       FREHD_OUT_CD = 16, FREHD_OUT_SCALAR = 32, FREHD_OUT_SUB = 64 };
int frehd_domain_write_output(frehd_domain *d, const char *prefix, int tt, int fields);
int frehd_domain_write_restart(frehd_domain *d, const char *prefix, int tt, double tNEnd);
int frehd_format_fixed4(const double *values, long n, char *out, size_t cap, size_t *len);

/* Accumulated device time per kernel (CUDA events on the domain's stream)
 * while profiling is on, and the CG iterations those steps ran. */
typedef struct frehd_kernel_times {
  double explicit_ms, cg_ms, update_geo_ms, update_vel_ms, finish_ms;
  int steps;
  long long cg_iters;
} frehd_kernel_times;
int frehd_domain_set_profiling(frehd_domain *d, int on);  /* on: also resets the sums */
int frehd_domain_kernel_times(frehd_domain *d, frehd_kernel_times *out);
/* The CUDA stream (cudaStream_t) all work of the domain is queued on. */
int frehd_domain_stream(frehd_domain *d, void **stream);

/* Solver start: FREHD_X0_ZERO (default) starts each solve from x = 0 as the
 * reference does (nsfunctions.c:1011); FREHD_X0_SURFACE starts from the current
 * surface (fewer iterations, same residual tolerance, but closed dry cells then
 * end exactly on b/Ct instead of on the CG's side of it, which can change the
 * reference's wet/dry branches). */
enum { FREHD_X0_ZERO = 0, FREHD_X0_SURFACE = 1 };
int frehd_domain_set_solver(frehd_domain *d, int x0_mode);

/* CG schedule.  Both run the reference's Jacobi-PCG to the same stopping rule
 * (itersolv.c:355-456, rtc.c:53) and agree to that tolerance.
 * FREHD_CG_SINGLE_SWEEP (default): one pass over the grid and one global
 * reduction per iteration (Chronopoulos-Gear ordering of the dot products).
 * FREHD_CG_TWO_PHASE: the textbook ordering, two passes and two reductions per
 * iteration, as CGIter does it. */
enum { FREHD_CG_SINGLE_SWEEP = 0, FREHD_CG_TWO_PHASE = 1 };
int frehd_domain_set_cg_schedule(frehd_domain *d, int schedule);

/* Rows the reference decouples (tidal rows, closed dry cells:
 * adjustTidalBoundary nsfunctions.c:887-924, matrixCoeffSub subgrid.c:1061-1078)
 * keep only their diagonal, but their neighbours' rows keep the coupling to
 * them, so the assembled matrix is not symmetric.
 * FREHD_DECOUPLED_AS_ASSEMBLED (default): the CG iterates that matrix, as
 * laspack's CGIter does; results follow the reference's to rounding.
 * FREHD_DECOUPLED_ELIMINATED: the couplings are moved into the right-hand side
 * at the decoupled rows' exact values b/|Ct|, so the iterated system is
 * symmetric positive definite (CG's convergence theory applies); results agree
 * with the reference to the CG tolerance rather than to rounding. */
enum { FREHD_DECOUPLED_AS_ASSEMBLED = 0, FREHD_DECOUPLED_ELIMINATED = 1 };
int frehd_domain_set_decoupled(frehd_domain *d, int mode);

/* Precision of the solve (no counterpart in the reference, which is FP64).
 * FREHD_PRECISION_FP64 (default): the CG in FP64.
 * FREHD_PRECISION_MIXED: iterative refinement; each refinement forms the
 * residual in FP64, solves the scaled system in FP32 (all dot products and
 * norms accumulated in FP64) until its residual fell by eps_inner (e.g. 1e-5),
 * and adds the correction to the FP64 solution.  Stops on the same FP64
 * residual test ||r|| < eps*||b||; a refinement that does not gain a factor 10
 * hands the step to the FP64 solve (cg_fallback = 2).  Single-sweep schedule
 * only; costs 7 FP32 arrays (28 bytes per cell) more device memory.  The
 * stencil kernels stay FP64. */
enum { FREHD_PRECISION_FP64 = 0, FREHD_PRECISION_MIXED = 1 };
int frehd_domain_set_precision(frehd_domain *d, int mode, double eps_inner);

/* The free-surface CG solve alone, for callers that cannot allocate device
 * memory.  No counterpart in the reference (it solves through laspack inside
 * the step, nsfunctions.c:1004-1017); this entry point exists for hosts whose
 * device memory is owned by another runtime's pool, or whose time loop must
 * not allocate after start-up (cudaMalloc/cudaFree synchronise the device).
 * It allocates nothing: no cudaMalloc, no cudaFree, no allocating library call.
 *
 * All arrays are device pointers the caller owns, row-major, cell (i, j) at
 * j*nx + i, in the convention of the domain's device system: Ct the diagonal
 * (negative on a decoupled row, which then holds x = b/|Ct| and has no
 * couplings), Gx[k] the coupling across the east face of cell k, Gy[k] across
 * its north face (0 on the domain edge), b the right-hand side.  Solves to
 * ||r||_2 < eps*||b||_2 or max_iter iterations with the same Jacobi-PCG as
 * the domain step.  x0_from_x = 0 starts from x = 0, else from the x passed in.
 *
 * Limit: nx*ny <= 512*512 cells; larger sizes return FREHD_ERR_INVALID.  The
 * solve's work vectors live in a static device array inside the library
 * (about 8.4 MB, held on every GPU that loads the library until the process
 * exits).  Every call shares it: calls that overlap on the GPU (other streams,
 * other threads without ordering) race; queue them on one stream.  The first
 * call on each device looks up that array's address with that device current;
 * make it before any stream capture.  The array takes device memory when the
 * code that holds it is loaded on the device; with CUDA's default lazy loading
 * that happens at this first call (its address look-up), so a host whose pool
 * reserves the GPU's memory up front makes one call on each device before the
 * reservation (a 1 x 1 solve on its own buffers serves) or sets
 * CUDA_MODULE_LOADING=EAGER.  The address found at the first call is kept for
 * the process: cudaDeviceReset invalidates it, so a host that resets a device
 * must not call this entry point on it again.  With iters and rel_residual
 * both NULL
 * the call only queues work on `stream` (a cudaStream_t; NULL = legacy
 * default); otherwise it waits for the solve and reports them, returning
 * FREHD_ERR_TIMEOUT if a device-side wait gave up. */
int frehd_cg_solve_noalloc(int nx, int ny, const double *Ct, const double *Gx, const double *Gy,
                           const double *b, double *x, double eps, int max_iter, int x0_from_x,
                           void *stream, int *iters, double *rel_residual);

/* ------------------------------------------------------------ batches */
/*
 * Many resident domains stepped together (the batched form; no counterpart in
 * the reference, whose driver runs one domain per process).  A domain is set up
 * with the calls above, then admitted; while admitted, the batch steps it and
 * the single-domain step/state calls refuse it (FREHD_ERR_STATE).  Every
 * frehd_batch_step advances every admitted domain by one step with five kernel
 * launches in total (replayed from a CUDA graph where the driver accepts the
 * capture).  A domain's results do not depend on which other domains share the
 * batch.  The solve of all domains is one cooperative launch in one of two
 * packings (frehd_batch_set_cg_packing):
 *   FREHD_BATCH_CTA_GROUPS (default): a domain's CG runs on
 *     ceil(cells / cells_per_cta) CTAs (at most its tile count) whatever the mix; the
 *     single-CTA solves, largest first, go to whichever CTA is free; admission
 *     also needs free CTAs;
 *   FREHD_BATCH_TILE_LIST: every domain's CG tiles form one list spread over
 *     all CTAs; a domain's sums are added in its own tile order, so its result is
 *     the same in any mix; cells_per_cta is not used, and admission is by memory
 *     alone.
 * The two packings add the solve's partial sums in different orders: their
 * results agree to the solver's rounding, not bit for bit.
 */
typedef struct frehd_batch frehd_batch;
typedef struct frehd_batch_info_t {
  int domains;             /* admitted domains */
  int cg_ctas;             /* CTAs of the batched CG launch */
  int cg_capacity;         /* CTAs the device holds at once for it */
  long tiles;              /* blocks of each stencil kernel per step over all domains (each
                              runs up to four 32 x 8 tiles of one domain) */
  int graph;               /* 1: steps replay a captured CUDA graph */
  long long bytes_used, bytes_budget;
  long long steps;         /* batch steps taken */
} frehd_batch_info_t;

/* Device memory a domain of this configuration holds in FP64, with r x r fine
   bottoms.  The mixed form (frehd_domain_set_precision) adds eight FP32 arrays
   of the padded grid; a batch admits by the bytes a domain actually holds. */
int frehd_domain_footprint(const frehd_config *cfg, int r, long long *bytes);
/* cells_per_cta: cells of a domain per CTA of its CG (the packing granularity):
 * in the CTA-group packing a domain's CG runs on ceil(cells / cells_per_cta) CTAs. */
int frehd_batch_create(int device, long long hbm_budget_bytes, double cells_per_cta,
                       frehd_batch **out);
/* Domains still admitted are handed back to their owners (not destroyed). */
int frehd_batch_destroy(frehd_batch *b);
/* Admit a set-up domain; its next step is tt = t0.  FREHD_ERR_NOMEM when the
 * memory budget or the CG's CTA capacity would be exceeded (the domain stays
 * with the caller). */
int frehd_batch_admit(frehd_batch *b, frehd_domain *d, int t0, int *slot);
/* Hand a domain back (state and last-step statistics readable again). */
int frehd_batch_release(frehd_batch *b, int slot, frehd_domain **d);
/* One step of every admitted domain (queued on the batch's stream). */
int frehd_batch_step(frehd_batch *b);
int frehd_batch_sync(frehd_batch *b);
int frehd_batch_info(frehd_batch *b, frehd_batch_info_t *out);
int frehd_batch_stream(frehd_batch *b, void **stream);
/* Replay steps from a captured CUDA graph (default 1) or launch them directly. */
int frehd_batch_set_graph(frehd_batch *b, int on);
/* Packing of the batched solve (see above); FREHD_ERR_NOMEM when the admitted
 * domains do not fit the CTA groups (the packing then stays the tile list). */
enum { FREHD_BATCH_TILE_LIST = 0, FREHD_BATCH_CTA_GROUPS = 1 };
int frehd_batch_set_cg_packing(frehd_batch *b, int packing);
/* Stencil tiles (32 x 8 cells, consecutive along a row of one domain) each
 * block of the batched stencil kernels runs, 1..8 (default 4): more tiles per
 * block stage the domain's view fewer times, fewer give more blocks to spread
 * over the SMs.  The arithmetic is the same for every value. */
int frehd_batch_set_stencil_tiles(frehd_batch *b, int tiles_per_block);

/* ------------------------------------------------------------ serving */
/*
 * Continuous batching (the served form; the reference's driver loop, FREHD.c,
 * runs one domain to the end instead).  A server owns a batch and one host
 * thread that steps it while it holds domains.  Callers prepare each domain on
 * their own thread (create, geometry, series, init), then submit it for nsteps
 * steps from tt = t0.  Between two batch steps the thread admits waiting
 * domains in submission order while the memory budget and the CG's CTA
 * capacity allow, and releases each domain that has run its steps; poll
 * returns them (the domain's state and statistics are readable again).  A
 * domain that cannot fit even an empty batch completes with FREHD_ERR_NOMEM.
 * The caller keeps ownership of every domain and must not touch one between
 * its submit and the poll that returns it.  Times are seconds on the server's
 * monotonic clock (frehd_server_info_t.clock is "now").
 */
typedef struct frehd_server frehd_server;
typedef struct frehd_server_done {
  long long ticket;          /* from frehd_server_submit */
  frehd_domain *domain;
  int status;                /* FREHD_OK, or the step's or admission's error */
  int steps;                 /* steps the domain ran */
  double t_submit, t_admit, t_done;  /* t_admit < 0: never admitted */
} frehd_server_done;
typedef struct frehd_server_info_t {
  long long submitted, completed;
  int waiting, active, max_active;
  long long batch_steps, cell_steps;
  double clock;              /* the server's clock now */
  int status;                /* FREHD_OK, or the error that stopped the server */
} frehd_server_info_t;

int frehd_server_create(int device, long long hbm_budget_bytes, double cells_per_cta,
                        frehd_server **out);
int frehd_server_submit(frehd_server *s, frehd_domain *d, int t0, int nsteps, long long *ticket);
/* Up to cap completed requests into out (*n of them); waits up to timeout_ms
 * for the first one when none is ready (0: return at once). */
int frehd_server_poll(frehd_server *s, frehd_server_done *out, int cap, int timeout_ms, int *n);
int frehd_server_info(frehd_server *s, frehd_server_info_t *out);
/* Stop the thread; domains still held go back to their owners unfinished. */
int frehd_server_destroy(frehd_server *s);

#ifdef __cplusplus
}
#endif
#endif /* FREHD_B200_H */
