/*
 * Single-rank stand-in for the MPI interface, used only to compile the
 * reference program into the test oracle (oracle/_ref).  It is test
 * infrastructure: nothing in the product links it.
 *
 * It covers exactly the 16 MPI calls the reference makes (src/comm.cpp,
 * src/universe.cpp, src/main.cpp, src/timer.cpp): with one rank every
 * collective is a copy and point-to-point calls are never reached.
 */
#ifndef MZ_ORACLE_MPI_SHIM_H
#define MZ_ORACLE_MPI_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_NULL      (-1)
#define MPI_COMM_WORLD     (0)
#define MPI_UNDEFINED      (-32766)
#define MPI_STATUS_IGNORE  ((MPI_Status *)0)

#define MPI_CHAR    (1)
#define MPI_INT     (4)
#define MPI_DOUBLE  (8)

#define MPI_SUM     (1)
#define MPI_MAX     (2)
#define MPI_MIN     (3)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Barrier(MPI_Comm comm);
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm *out);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *out);
int MPI_Send(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm comm, MPI_Status *st);
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm comm);
int MPI_Reduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm);
int MPI_Gather(const void *sbuf, int scount, MPI_Datatype st, void *rbuf, int rcount, MPI_Datatype rt,
               int root, MPI_Comm comm);
double MPI_Wtime(void);

#ifdef __cplusplus
}
#endif

#endif
