/*
 * frehd_dropin.h -- the drop-in host shim: the reference's own host program
 * (frehdc5+/FREHD.c main and every reference translation unit except
 * nssolve.c) linked with frehdc_b200/dropin/nssolve_b200.c, which runs each
 * time step on a B200 through frehd_b200.h.
 *
 * nssolve_b200.c defines the entry points the reference's nssolve.h declares
 * (frehdc5+/nssolve.h:11-20), with the reference's signatures:
 *   SolveAll          replaces nssolve.c:48-107 (the time loop)
 *   oneCompleteStep   replaces nssolve.c:110-118 (one step; host arrays in, host arrays out)
 *   solveSourceTerm   replaces nssolve.c:121-155
 *   solveFreeSurface  replaces nssolve.c:158-178
 *   updateData        replaces nssolve.c:181-290 (here it also covers scalarTransport,
 *                     which oneCompleteStep calls after it, nssolve.c:116-117)
 * They are declared by the reference's own nssolve.h, which needs laspack's
 * QMatrix/Vector; this header declares only the explicit API below.
 *
 * The structs are the reference's (configuration.h:4-111, initialize.h:10-32,
 * bathymetry.h:7-14, subgrid.h:8-29); the shim reads and writes their arrays
 * in the reference layout and never frees or reallocates them.
 *
 * One device domain per process (the reference keeps one domain per process
 * as well).  All functions return a frehd_status code.
 */
#ifndef FREHD_DROPIN_H
#define FREHD_DROPIN_H

#ifdef __cplusplus
extern "C" {
#endif

struct Data;
struct Sub;
struct Bath;
struct BC;
struct Config;
typedef struct frehd_domain frehd_domain;

/* Create the device domain from the host state left by the reference's Init
 * (initialize.c:40-155): configuration, subgrid tables (sub->allV .. allOm),
 * tide series bc->tideP, bathymetry and the current Data/Sub fields. */
int frehd_gpu_init(struct Data *data, struct Sub *sub, struct Bath *bath, struct BC *bc,
                   struct Config *setting, int device);
/* Steps t0 .. t0+nsteps-1 on the device (oneCompleteStep + monitorCFL each);
 * the host arrays are not touched.  FREHD_ERR_CFL: the device stopped after the
 * step whose max CFL exceeded 20 (frehd_gpu_last_step). */
int frehd_gpu_run(int t0, int nsteps);
/* One step tt on the device (frehd_gpu_run(tt, 1)). */
int frehd_gpu_step(int tt);
/* Copy the device state into the host's Data and Sub arrays (every field the
 * step writes), so the reference's output and monitoring code can read them. */
int frehd_gpu_sync_to_host(struct Data *data, struct Sub *sub);
/* Copy host edits of the persistent state (surf, velocities, scalar, depth,
 * drag, CFL, subgrid fields, ind) to the device. */
int frehd_gpu_sync_from_host(struct Data *data, struct Sub *sub);
/* tt of the last step the device completed. */
int frehd_gpu_last_step(void);
/* Status of the last shim call (FREHD_OK when it succeeded). */
int frehd_gpu_status(void);
/* The device domain (NULL before frehd_gpu_init), for the full frehd_b200.h API. */
frehd_domain *frehd_gpu_domain(void);
/* Release the device domain. */
int frehd_gpu_finalize(void);

#ifdef __cplusplus
}
#endif
#endif
