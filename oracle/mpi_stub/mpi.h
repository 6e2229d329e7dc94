/*
 * Single-rank stand-in for <mpi.h> so that the reference CPU engine
 * (pyhea/cpp/accelerate.cpp) compiles without an MPI installation.  It gives
 * one rank of size one; the only collective the engine makes, an in-place
 * MPI_Allreduce(MIN) of the logged best fitness (accelerate.cpp:753), is then
 * the identity.  Test infrastructure only.
 */
#ifndef HEA_MPI_STUB_H
#define HEA_MPI_STUB_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 0
#define MPI_MIN 0
#define MPI_IN_PLACE ((void *)1)
static inline int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return 0; }
static inline int MPI_Allreduce(const void *, void *, int, MPI_Datatype, MPI_Op, MPI_Comm) { return 0; }
#endif
