/*
 * Minimal MPI declarations so that the reference's mpifunctions.c and FREHD.c
 * compile without an MPI installation (drop-in host and oracle builds).  Both
 * run the reference host with useMPI = 0, where none of these functions is
 * reached; each definition in mpi_stub.c aborts if it ever is.  A build with a
 * real MPI drops this directory from the include path and links libmpi.
 */
#ifndef FREHD_MPI_STUB_H
#define FREHD_MPI_STUB_H

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD ((MPI_Comm)0x44000000)
#define MPI_DOUBLE ((MPI_Datatype)0x4c00080b)
#define MPI_INT ((MPI_Datatype)0x4c000405)
#define MPI_PROC_NULL (-1)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *t);
int MPI_Type_free(MPI_Datatype *t);
int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype stype, int dest, int stag,
                 void *rbuf, int rcount, MPI_Datatype rtype, int src, int rtag,
                 MPI_Comm comm, MPI_Status *status);
int MPI_Gather(const void *sbuf, int scount, MPI_Datatype stype, void *rbuf, int rcount,
               MPI_Datatype rtype, int root, MPI_Comm comm);

#endif
