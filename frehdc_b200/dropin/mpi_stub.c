/* Aborting definitions of the MPI calls the reference host program names, for
 * builds of it without an MPI installation (the drop-in host and the oracle
 * builds).  Both run with useMPI = 0, so none of them is ever called. */
#include <stdio.h>
#include <stdlib.h>

#include "mpi.h"

static int unreachable(const char *f) {
  fprintf(stderr, "frehd host: %s called with useMPI = 0\n", f);
  abort();
  return 1;
}

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return unreachable("MPI_Init"); }
int MPI_Finalize(void) { return unreachable("MPI_Finalize"); }
int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; (void)r; return unreachable("MPI_Comm_rank"); }
int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; (void)s; return unreachable("MPI_Comm_size"); }
int MPI_Type_contiguous(int n, MPI_Datatype o, MPI_Datatype *t) {
  (void)n; (void)o; (void)t; return unreachable("MPI_Type_contiguous");
}
int MPI_Type_commit(MPI_Datatype *t) { (void)t; return unreachable("MPI_Type_commit"); }
int MPI_Type_free(MPI_Datatype *t) { (void)t; return unreachable("MPI_Type_free"); }
int MPI_Sendrecv(const void *a, int b, MPI_Datatype c, int d, int e, void *f, int g,
                 MPI_Datatype h, int i, int j, MPI_Comm k, MPI_Status *l) {
  (void)a; (void)b; (void)c; (void)d; (void)e; (void)f; (void)g; (void)h; (void)i; (void)j;
  (void)k; (void)l;
  return unreachable("MPI_Sendrecv");
}
int MPI_Gather(const void *a, int b, MPI_Datatype c, void *d, int e, MPI_Datatype f, int g,
               MPI_Comm h) {
  (void)a; (void)b; (void)c; (void)d; (void)e; (void)f; (void)g; (void)h;
  return unreachable("MPI_Gather");
}
