/* Single-rank stand-in for the MPI header, used ONLY to compile the
 * reference's own lattice/coupler translation units into the test oracle
 * (oracle/_ref).  Every rank query answers "rank 0 of 1"; reductions with
 * MPI_IN_PLACE are identities; point-to-point calls are never reached on one
 * rank (every face and coupling point is rank-local) and abort if they are.
 *
 * Test infrastructure: nothing in the product links this. */
#ifndef OCTLB_ORACLE_SHIM_MPI_H_
#define OCTLB_ORACLE_SHIM_MPI_H_

#include <cstdio>
#include <cstdlib>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int source, tag, error; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_SUCCESS 0
#define MPI_BYTE 1
#define MPI_INT 2
#define MPI_DOUBLE 3
#define MPI_CHAR 4
#define MPI_MAX 10
#define MPI_SUM 11
#define MPI_TAG_UB 100
#define MPI_IN_PLACE ((void*)1)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)

inline int octlb_shim_mpi_sizeof(MPI_Datatype t) {
  return (t == MPI_BYTE || t == MPI_CHAR) ? 1 : t == MPI_INT ? 4 : 8;
}
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
inline int MPI_Allreduce(const void* in, void* out, int n, MPI_Datatype t,
                         MPI_Op, MPI_Comm) {
  if (in != MPI_IN_PLACE) std::memcpy(out, in, (size_t)n * octlb_shim_mpi_sizeof(t));
  return 0;
}
// Gathers over one rank: the local contribution is the whole result.
inline int MPI_Allgather(const void* in, int n, MPI_Datatype t, void* out, int, MPI_Datatype, MPI_Comm) {
  std::memcpy(out, in, (size_t)n * octlb_shim_mpi_sizeof(t));
  return 0;
}
inline int MPI_Allgatherv(const void* in, int n, MPI_Datatype t, void* out, const int*, const int* displs,
                          MPI_Datatype, MPI_Comm) {
  std::memcpy(static_cast<char*>(out) + (size_t)displs[0] * octlb_shim_mpi_sizeof(t), in,
              (size_t)n * octlb_shim_mpi_sizeof(t));
  return 0;
}
[[noreturn]] inline void octlb_shim_mpi_p2p() {
  std::fprintf(stderr, "oracle MPI shim: point-to-point call on one rank\n");
  std::abort();
}
inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { octlb_shim_mpi_p2p(); }
inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { octlb_shim_mpi_p2p(); }
inline int MPI_Waitall(int n, MPI_Request*, MPI_Status*) { if (n) octlb_shim_mpi_p2p(); return 0; }
inline int MPI_Comm_get_attr(MPI_Comm, int, void*, int* flag) { *flag = 0; return 0; }

#endif
