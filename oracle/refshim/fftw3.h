// TEST INFRASTRUCTURE ONLY -- used to compile the reference's own sources into
// oracle/_ref/ (the checker); nothing in the product includes it.
//
// The subset of the FFTW3 interface that src/fftPair/fftPair.cpp:39-107 and
// src/initialize.cpp:36-51 call, implemented over the oracle's own
// mixed-radix transform (oracle/oracle_fft.hpp).  Semantics kept from FFTW:
// unnormalised transforms, exponent sign as given, row-major dimensions,
// plans bound to the arrays they were made for, execution out of place or in
// place.
#pragma once
#include <cstddef>

typedef double fftw_complex[2];
typedef struct edus_shim_fftw_plan_s* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

extern "C" {
fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany, fftw_complex* in, const int* inembed,
                             int istride, int idist, fftw_complex* out, const int* onembed, int ostride,
                             int odist, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
int fftw_planner_nthreads(void);
void fftw_cleanup(void);
}
