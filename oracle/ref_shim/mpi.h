// Single-rank stand-in for the MPI names the reference headers mention.
// TEST INFRASTRUCTURE ONLY.
#pragma once
typedef int MPI_Comm; typedef int MPI_Datatype; typedef int MPI_Op;
#define MPI_COMM_WORLD 0
#define MPI_IN_PLACE ((void *)1)
#define MPI_DOUBLE 0
#define MPI_INT 1
#define MPI_UNSIGNED_LONG_LONG 2
#define MPI_LONG_LONG 3
#define MPI_MAX 0
#define MPI_MIN 1
#define MPI_SUM 2
inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
int MPI_Reduce(const void *, void *, int, MPI_Datatype, MPI_Op, int, MPI_Comm);
int MPI_Allreduce(const void *, void *, int, MPI_Datatype, MPI_Op, MPI_Comm);
