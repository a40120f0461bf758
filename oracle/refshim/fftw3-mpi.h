// TEST INFRASTRUCTURE ONLY -- used to compile the reference's own sources into
// oracle/_ref/ (the checker); nothing in the product includes it.
//
// The distributed-FFTW calls of src/fftPair/fftPair.cpp:39-61 and
// src/MPIindex/MPIindex_definitions.hpp:35-48 for one rank: the whole grid is
// local, and a `howmany` transform works on interleaved planes (element
// (k, h) at k*howmany + h: stride howmany, distance 1), which is what FFTW's
// MPI interface specifies for its `howmany` argument.
#pragma once
#include <cstddef>
#include "fftw3.h"
#include "mpi.h"

#define FFTW_MPI_DEFAULT_BLOCK (0)

extern "C" {
void fftw_mpi_init(void);
void fftw_mpi_cleanup(void);
std::ptrdiff_t fftw_mpi_local_size_many(int rnk, const std::ptrdiff_t* n, std::ptrdiff_t howmany,
                                        std::ptrdiff_t block0, MPI_Comm comm, std::ptrdiff_t* local_n0,
                                        std::ptrdiff_t* local_0_start);
fftw_plan fftw_mpi_plan_many_dft(int rnk, const std::ptrdiff_t* n, std::ptrdiff_t howmany,
                                 std::ptrdiff_t block, std::ptrdiff_t tblock, fftw_complex* in,
                                 fftw_complex* out, MPI_Comm comm, int sign, unsigned flags);
}
