/*
 * frehd_ref: driver of the unchanged reference model (oracle test
 * infrastructure).  It is linked with the reference's own translation units
 * (frehdc5+ and laspack, compiled from where they lie) and replaces only the
 * program entry: FREHD.c is built with -Dmain=frehd_ref_main so that its
 * ReadInputFile is reused, and main() below repeats FREHD.c:66-110 followed by
 * the body of SolveAll (nssolve.c:48-107) without per-step printing.
 *
 *   frehd_ref run    <deck> <steps> <out.bin>   final state after <steps> steps
 *   frehd_ref phases <deck> <steps> <outdir>    per step, the state at the
 *        phase boundaries of oneCompleteStep (nssolve.c:110-178):
 *        p0 step start, p1 after the explicit terms and matrix assembly
 *        (solveSourceTerm, matrixCoeffSub, adjustMatrixBoundary,
 *        adjustTidalBoundary), p2 the CG solution x, p3 after getFreeSurface ..
 *        monitorCFL.  --at a,b,c limits the dumps to those steps.
 *   frehd_ref time   <deck> <steps>             wall time of the step loop
 *   frehd_ref inject <deck> <tt> <outdir> <state.bin>
 *        initialise from the deck, overwrite the named arrays of the model
 *        with those of state.bin (a dump, possibly edited), then run step tt
 *        with phase dumps (used to drive rarely reached branches).
 *
 * The deck directory must hold data.dat and input/ (relative paths, as the
 * reference expects).  Dumps are little-endian: "FRHDDUMP", int32 version,
 * int32 count, then per array: char name[24], int64 n, int32 type (0 double,
 * 1 int32), int32 pad, data.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "bathymetry.h"
#include "configuration.h"
#include "fileio.h"
#include "initialize.h"
#include "map.h"
#include "nsfunctions.h"
#include "nssolve.h"
#include "scalar.h"
#include "subgrid.h"
#include "utilities.h"

#include "laspack/errhandl.h"
#include "laspack/itersolv.h"
#include "laspack/precond.h"
#include "laspack/qmatrix.h"
#include "laspack/rtc.h"
#include "laspack/vector.h"

void ReadInputFile(char filename[], double *value, char *date, char *inputFolder,
                   char *outputFolder, char *subgridFolder, int N);

static Config *setting;
static Bath *bth;
static Maps *map;
static Data *data;
static IC *ic;
static BC *bc;
static Sub *sub;

typedef struct {
  FILE *f;
  int count;
  long count_pos;
} Dump;

static void dump_open(Dump *d, const char *path) {
  d->f = fopen(path, "wb");
  if (!d->f) {
    fprintf(stderr, "frehd_ref: cannot write %s\n", path);
    exit(2);
  }
  fwrite("FRHDDUMP", 1, 8, d->f);
  int32_t ver = 1;
  fwrite(&ver, 4, 1, d->f);
  d->count_pos = ftell(d->f);
  d->count = 0;
  fwrite(&d->count, 4, 1, d->f);
}

static void dump_arr(Dump *d, const char *name, const void *p, long n, int type) {
  if (!p) return;
  char nm[24];
  memset(nm, 0, sizeof(nm));
  strncpy(nm, name, sizeof(nm) - 1);
  int64_t nn = n;
  int32_t ty = type, pad = 0;
  fwrite(nm, 1, 24, d->f);
  fwrite(&nn, 8, 1, d->f);
  fwrite(&ty, 4, 1, d->f);
  fwrite(&pad, 4, 1, d->f);
  fwrite(p, type == 0 ? 8 : 4, (size_t)n, d->f);
  d->count++;
}

static void dump_close(Dump *d) {
  fseek(d->f, d->count_pos, SEEK_SET);
  int32_t c = d->count;
  fwrite(&c, 4, 1, d->f);
  fclose(d->f);
}

static void dump_state(const char *path, int tt, Vector *x) {
  Dump d;
  const long N = setting->N2ci, T = setting->N2ct;
  dump_open(&d, path);
  int32_t meta[8] = {setting->nx, setting->ny, setting->useSubgrid ? sub->Ne : 0, setting->Nt,
                     tt, 0, 0, 0};
  if (x) meta[5] = GetLastNoIter();
  dump_arr(&d, "meta", meta, 8, 1);
  double acc = x ? GetLastAccuracy() : 0.0;
  dump_arr(&d, "cg_accuracy", &acc, 1, 0);
#define DD(name, n) dump_arr(&d, #name, data->name, n, 0)
  DD(surf, T); DD(surfOld, T); DD(uuXP, T); DD(vvYP, T); DD(uuYP, N); DD(vvXP, N);
  DD(depth, N); DD(depthXP, T); DD(depthYP, T); DD(EnXP, T); DD(EnYP, T);
  DD(DragXP, T); DD(DragYP, T); DD(CDXP, T); DD(CDYP, T);
  DD(GnCt, N); DD(GnXP, N); DD(GnXM, N); DD(GnYP, N); DD(GnYM, N); DD(z, N);
  DD(S, T); DD(Sm, N); DD(cellV, N); DD(Fuu, T); DD(Fvv, T); DD(CFLx, T); DD(CFLy, T);
  DD(rmvCFL, N); DD(wtfXP, T); DD(wtfYP, T); DD(advX, T); DD(advY, T);
  DD(Vloss1, 1); DD(Vloss2, 1); DD(Vloss3, 1); DD(Vloss4, 1);
#undef DD
  if (setting->useSubgrid) {
#define DS(name) dump_arr(&d, #name, sub->name, T, 0)
    DS(V); DS(Z); DS(Vxp); DS(Vyp); DS(Vxm); DS(Vym); DS(Np); DS(Nm); DS(Op); DS(Om);
    DS(Nx); DS(Oy); DS(Vx); DS(Vy); DS(Zx); DS(Zy);
#undef DS
    dump_arr(&d, "ind", sub->ind, T, 1);
    dump_arr(&d, "allSurf", sub->allSurf, sub->Ne, 0);
  }
  dump_arr(&d, "bottomZ", bth->bottomZ, T, 0);
  dump_arr(&d, "bottomXP", bth->bottomXP, T, 0);
  dump_arr(&d, "bottomYP", bth->bottomYP, T, 0);
  dump_arr(&d, "edgeX", bth->edgeX, N, 0);
  dump_arr(&d, "edgeY", bth->edgeY, N, 0);
  dump_arr(&d, "offset", bth->offset, 1, 0);
  dump_arr(&d, "tideP", bc->tideP, setting->Nt, 0);
  if (x) {
    double *xv = (double *)malloc(N * sizeof(double));
    for (long k = 0; k < N; ++k) xv[k] = V_GetCmp(x, (size_t)(k + 1));
    dump_arr(&d, "x", xv, N, 0);
    free(xv);
  }
  dump_close(&d);
}

/* Overwrite model arrays with those of a dump (same names and lengths). */
static void load_state(const char *path) {
  FILE *f = fopen(path, "rb");
  if (!f) {
    fprintf(stderr, "frehd_ref: cannot read %s\n", path);
    exit(2);
  }
  char magic[8];
  int32_t ver, count;
  if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "FRHDDUMP", 8) || fread(&ver, 4, 1, f) != 1 ||
      fread(&count, 4, 1, f) != 1) {
    fprintf(stderr, "frehd_ref: %s is not a dump\n", path);
    exit(2);
  }
  const long N = setting->N2ci, T = setting->N2ct;
  for (int a = 0; a < count; ++a) {
    char nm[24];
    int64_t n;
    int32_t ty, pad;
    if (fread(nm, 1, 24, f) != 24 || fread(&n, 8, 1, f) != 1 || fread(&ty, 4, 1, f) != 1 ||
        fread(&pad, 4, 1, f) != 1) {
      fprintf(stderr, "frehd_ref: truncated dump %s\n", path);
      exit(2);
    }
    size_t esz = ty == 0 ? 8 : 4;
    void *buf = malloc((size_t)n * esz);
    if (fread(buf, esz, (size_t)n, f) != (size_t)n) {
      fprintf(stderr, "frehd_ref: truncated dump %s\n", path);
      exit(2);
    }
    void *dst = NULL;
    long len = -1;
#define M(nm_, ptr_, len_) if (!strcmp(nm, nm_)) { dst = (void *)(ptr_); len = (len_); }
    M("surf", data->surf, T) M("surfOld", data->surfOld, T) M("uuXP", data->uuXP, T)
    M("vvYP", data->vvYP, T) M("uuYP", data->uuYP, N) M("vvXP", data->vvXP, N)
    M("depth", data->depth, N) M("depthXP", data->depthXP, T) M("depthYP", data->depthYP, T)
    M("EnXP", data->EnXP, T) M("EnYP", data->EnYP, T) M("DragXP", data->DragXP, T)
    M("DragYP", data->DragYP, T) M("CDXP", data->CDXP, T) M("CDYP", data->CDYP, T)
    M("S", data->S, T) M("Sm", data->Sm, N) M("cellV", data->cellV, N) M("Fuu", data->Fuu, T)
    M("Fvv", data->Fvv, T) M("CFLx", data->CFLx, T) M("CFLy", data->CFLy, T)
    M("rmvCFL", data->rmvCFL, N) M("wtfXP", data->wtfXP, T) M("wtfYP", data->wtfYP, T)
    M("advX", data->advX, T) M("advY", data->advY, T)
    if (setting->useSubgrid) {
      M("V", sub->V, T) M("Z", sub->Z, T) M("Vxp", sub->Vxp, T) M("Vyp", sub->Vyp, T)
      M("Vxm", sub->Vxm, T) M("Vym", sub->Vym, T) M("Np", sub->Np, T) M("Nm", sub->Nm, T)
      M("Op", sub->Op, T) M("Om", sub->Om, T) M("Nx", sub->Nx, T) M("Oy", sub->Oy, T)
      M("Vx", sub->Vx, T) M("Vy", sub->Vy, T) M("Zx", sub->Zx, T) M("Zy", sub->Zy, T)
      M("ind", sub->ind, T)
    }
#undef M
    if (dst) {
      if (n != len) {
        fprintf(stderr, "frehd_ref: %s has %ld values, expected %ld\n", nm, (long)n, len);
        exit(2);
      }
      memcpy(dst, buf, (size_t)n * esz);
    }
    free(buf);
  }
  fclose(f);
}

static void init_model(const char *deck) {
  if (chdir(deck) != 0) {
    fprintf(stderr, "frehd_ref: cannot enter deck %s\n", deck);
    exit(2);
  }
  int irank = 0, nrank = 1;
  double *value = (double *)malloc(120 * sizeof(double));
  char *date = (char *)malloc(16);
  char *inputFolder = (char *)malloc(100);
  char *outputFolder = (char *)malloc(100);
  char *subgridFolder = (char *)malloc(100);
  ReadInputFile("data.dat", value, date, inputFolder, outputFolder, subgridFolder, 150);
  ReadUserSettings(&setting, value, date, inputFolder, outputFolder, subgridFolder);
  if (setting->useMPI == 1) {
    fprintf(stderr, "frehd_ref: decks with useMPI = 1 are not supported\n");
    exit(2);
  }
  ReadBathymetry(&bth, setting, irank);
  InitBathymetry(bth, setting, irank);
  createMaps(&map, setting);
  Init(&data, &map, &ic, &bc, &sub, bth, setting, irank, nrank);
  /* SolveAll's initial output (nssolve.c:54-55) also round-trips surf through
   * the output datum (fileio.c:65-66,120-121). */
  DataOutput(&data, bth, setting, 0, 0, irank);
  if (setting->useSubgrid != 0) SubOutput(&sub, setting, 0, 0, irank);
}

static int want(int tt, const int *at, int nat) {
  if (nat == 0) return 1;
  for (int k = 0; k < nat; ++k)
    if (at[k] == tt) return 1;
  return 0;
}

static double now(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* One pass of the SolveAll loop body (nssolve.c:71-95) without printing. */
static void solveall_step(int tt) {
  QMatrix A;
  Q_Constr(&A, "A", setting->N2ci, False, Rowws, Normal, True);
  Vector z;
  V_Constr(&z, "z", setting->N2ci, Normal, True);
  Vector x;
  V_Constr(&x, "x", setting->N2ci, Normal, True);
  oneCompleteStep(&data, &sub, map, bc, bth, setting, tt, A, x, z, 0, 1);
  Q_Destr(&A);
  V_Destr(&x);
  V_Destr(&z);
  monitorCFL(&data, bth, 0, setting, tt, 0);
  if (tt % setting->OutItvl == 0) {
    DataOutput(&data, bth, setting, tt, 0, 0);
    if (setting->useSubgrid != 0) SubOutput(&sub, setting, tt, 0, 0);
  }
}

/* oneCompleteStep (nssolve.c:110-178) with dumps between its phases. */
static void phased_step(int tt, const char *outdir, int dumpit) {
  char path[1024];
  QMatrix A;
  Q_Constr(&A, "A", setting->N2ci, False, Rowws, Normal, True);
  Vector z;
  V_Constr(&z, "z", setting->N2ci, Normal, True);
  Vector x;
  V_Constr(&x, "x", setting->N2ci, Normal, True);
  if (dumpit) {
    snprintf(path, sizeof(path), "%s/step%04d_p0.bin", outdir, tt);
    dump_state(path, tt, NULL);
  }
  solveSourceTerm(&data, sub, map, bc, bth, setting, tt, 0, 1);
  if (setting->useSubgrid == 0)
    matrixCoeff(&data, map, setting);
  else
    matrixCoeffSub(&data, map, sub, setting);
  adjustMatrixBoundary(&data, bc, map, setting, 0, 1);
  adjustTidalBoundary(&data, bc, bth, setting, tt, 0, 1);
  if (dumpit) {
    snprintf(path, sizeof(path), "%s/step%04d_p1.bin", outdir, tt);
    dump_state(path, tt, NULL);
  }
  setupMatrix(data, map, setting, A);
  solveMatrix(data, setting, A, x, z);
  if (dumpit) {
    snprintf(path, sizeof(path), "%s/step%04d_p2.bin", outdir, tt);
    dump_state(path, tt, &x);
  }
  getFreeSurface(&data, map, setting, x);
  if (setting->useEvap == 1) evaporation(&data, bc, tt, setting);
  if (setting->useRain == 1) rainfall(&data, bc, tt, setting);
  zeroNegSurf(&data, bth, setting, tt);
  enforceFreeSurfaceBC(&data, map, setting);
  enforceTidalBC(&data, bth, bc, setting, tt, 0, 1);
  updateData(&data, &sub, map, bc, bth, setting, tt, 0, 1);
  if (setting->useScalar == 1) scalarTransport(&data, map, bth, bc, sub, setting, tt, 0, 1);
  Q_Destr(&A);
  V_Destr(&x);
  V_Destr(&z);
  monitorCFL(&data, bth, 0, setting, tt, 0);
  if (dumpit) {
    snprintf(path, sizeof(path), "%s/step%04d_p3.bin", outdir, tt);
    dump_state(path, tt, NULL);
  }
  if (tt % setting->OutItvl == 0) {
    DataOutput(&data, bth, setting, tt, 0, 0);
    if (setting->useSubgrid != 0) SubOutput(&sub, setting, tt, 0, 0);
  }
}

int main(int argc, char **argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s run|phases|time <deck> <steps> [out] [--at a,b]\n", argv[0]);
    return 2;
  }
  const char *mode = argv[1];
  int steps = atoi(argv[3]);
  char out[1024] = {0};
  if (argc > 4 && argv[4][0] != '-') {
    if (argv[4][0] == '/')
      snprintf(out, sizeof(out), "%s", argv[4]);
    else {
      char cwd[900];
      if (!getcwd(cwd, sizeof(cwd))) return 2;
      snprintf(out, sizeof(out), "%s/%s", cwd, argv[4]);
    }
  }
  int at[64], nat = 0;
  for (int k = 4; k < argc; ++k)
    if (!strcmp(argv[k], "--at") && k + 1 < argc) {
      char *s = argv[k + 1];
      while (*s && nat < 64) {
        at[nat++] = (int)strtol(s, &s, 10);
        if (*s == ',') s++;
      }
    }
  init_model(argv[2]);
  if (!strcmp(mode, "inject")) {
    if (argc < 6) {
      fprintf(stderr, "usage: %s inject <deck> <tt> <outdir> <state.bin>\n", argv[0]);
      return 2;
    }
    char st[1024];
    if (argv[5][0] == '/') snprintf(st, sizeof(st), "%s", argv[5]);
    else {
      fprintf(stderr, "frehd_ref: inject wants an absolute state path\n");
      return 2;
    }
    load_state(st);
    phased_step(steps, out, 1);
    return 0;
  }
  if (steps >= setting->Nt) {
    fprintf(stderr, "frehd_ref: steps must be < Nt=%d (BC arrays hold Nt entries)\n", setting->Nt);
    return 2;
  }
  if (!strcmp(mode, "run")) {
    for (int tt = 1; tt <= steps; ++tt) solveall_step(tt);
    if (out[0]) dump_state(out, steps, NULL);
  } else if (!strcmp(mode, "phases")) {
    for (int tt = 1; tt <= steps; ++tt) phased_step(tt, out, want(tt, at, nat));
  } else if (!strcmp(mode, "time")) {
    /* the CG iterations of each step (laspack's count of the last solve, rtc.c:74)
     * are summed outside the timed loop body's work */
    long iters = 0;
    double t0 = now();
    for (int tt = 1; tt <= steps; ++tt) {
      solveall_step(tt);
      iters += GetLastNoIter();
    }
    double t1 = now();
    double cs = (double)setting->N2ci * steps / (t1 - t0);
    printf("{\"steps\": %d, \"cells\": %d, \"seconds\": %.6f, \"cell_steps_per_s\": %.6e, "
           "\"cg_iters_per_step\": %.3f}\n",
           steps, setting->N2ci, t1 - t0, cs, (double)iters / steps);
    if (out[0]) dump_state(out, steps, NULL);
  } else {
    fprintf(stderr, "frehd_ref: unknown mode %s\n", mode);
    return 2;
  }
  return 0;
}
