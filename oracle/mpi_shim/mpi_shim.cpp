// Single-rank MPI stand-in for the test oracle build (see mpi.h).  Every
// datatype constant equals its size in bytes, so a collective over one rank
// is a memcpy of count * datatype bytes.
#include "mpi.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>

extern "C" {

static int g_next_comm = 1;

int MPI_Init(int *, char ***) { return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Abort(MPI_Comm, int code) {
  std::fprintf(stderr, "oracle mpi shim: MPI_Abort(%d)\n", code);
  std::exit(code ? code : 1);
}
int MPI_Barrier(MPI_Comm) { return 0; }
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm *out) {
  *out = (comm == MPI_COMM_NULL) ? MPI_COMM_NULL : g_next_comm++;
  return 0;
}
int MPI_Comm_free(MPI_Comm *comm) { *comm = MPI_COMM_NULL; return 0; }
int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return 0; }
int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return 0; }
int MPI_Comm_split(MPI_Comm, int color, int, MPI_Comm *out) {
  *out = (color == MPI_UNDEFINED) ? MPI_COMM_NULL : g_next_comm++;
  return 0;
}
int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) {
  std::fprintf(stderr, "oracle mpi shim: MPI_Send has no peer with one rank\n");
  std::exit(3);
}
int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) {
  std::fprintf(stderr, "oracle mpi shim: MPI_Recv has no peer with one rank\n");
  std::exit(3);
}
int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
int MPI_Reduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  if (sbuf != rbuf && count > 0) std::memmove(rbuf, sbuf, (size_t)count * (size_t)t);
  return 0;
}
int MPI_Allreduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (sbuf != rbuf && count > 0) std::memmove(rbuf, sbuf, (size_t)count * (size_t)t);
  return 0;
}
int MPI_Gather(const void *sbuf, int scount, MPI_Datatype st, void *rbuf, int, MPI_Datatype, int,
               MPI_Comm) {
  if (sbuf != rbuf && scount > 0) std::memmove(rbuf, sbuf, (size_t)scount * (size_t)st);
  return 0;
}
double MPI_Wtime(void) {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

}  // extern "C"
