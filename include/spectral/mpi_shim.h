// Single-rank stand-in for the few MPI names the reference's solver interfaces carry
// (constructor arguments of type MPI_Comm, comm() accessors, scalar reductions).
//
// The B200 backend runs one solve per GPU with no domain decomposition, so every
// communicator has size 1.  When the real MPI header is available and
// SPECTRAL_B200_WITH_MPI is defined, it is used instead and only size-1 communicators
// are accepted (the reference's serial FFTW backend has the same rule,
// src/fftw_fft.cpp:8-14).
#pragma once

#ifdef SPECTRAL_B200_WITH_MPI
#include <mpi.h>
#else
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_COMM_WORLD 0
#define MPI_COMM_SELF 1
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_SUCCESS 0

inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Allreduce(const void* in, void* out, int count, MPI_Datatype type, MPI_Op, MPI_Comm) {
  std::memcpy(out, in, (size_t)count * (type == MPI_DOUBLE ? sizeof(double) : sizeof(int)));
  return MPI_SUCCESS;
}
#endif
