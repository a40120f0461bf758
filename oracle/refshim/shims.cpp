// TEST INFRASTRUCTURE ONLY -- linked into the reference's own sources to build
// oracle/_ref/EDUS (the checker); nothing in the product links it.
//
// Implementations behind oracle/refshim/{mpi.h, fftw3.h, fftw3-mpi.h, mkl.h}:
// one MPI rank, FFTW's transform semantics over the oracle's mixed-radix FFT,
// and the few dense linear-algebra routines the reference takes from MKL.
// Each routine follows the published semantics of the library call it
// stands in for; none of them is a copy of that library.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <vector>

#include "../oracle_fft.hpp"
#include "../oracle_linalg.hpp"
#include "fftw3-mpi.h"
#include "mkl.h"
#include "mpi.h"

using cd = std::complex<double>;

// ---------------------------------------------------------------------------
// MPI, one rank
namespace {
struct Message {
    int tag;
    std::vector<char> bytes;
};
std::deque<Message>& mailbox() {
    static std::deque<Message> box;
    return box;
}
size_t type_size(MPI_Datatype t) { return (size_t)(t & 0xff); }
int next_comm = 2;
}  // namespace

extern "C" {
int MPI_Init_thread(int*, char***, int required, int* provided) {
    *provided = required;
    return MPI_SUCCESS;
}
int MPI_Query_thread(int* provided) {
    *provided = MPI_THREAD_FUNNELED;
    return MPI_SUCCESS;
}
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm, int* rank) {
    *rank = 0;
    return MPI_SUCCESS;
}
int MPI_Comm_size(MPI_Comm, int* size) {
    *size = 1;
    return MPI_SUCCESS;
}
int MPI_Comm_split(MPI_Comm, int, int, MPI_Comm* newcomm) {
    *newcomm = next_comm++;
    return MPI_SUCCESS;
}
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Send(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm) {
    if (dest != 0) {
        std::fprintf(stderr, "mpi shim: send to rank %d in a one-rank world\n", dest);
        std::abort();
    }
    const char* p = static_cast<const char*>(buf);
    mailbox().push_back(Message{tag, std::vector<char>(p, p + (size_t)count * type_size(type))});
    return MPI_SUCCESS;
}
int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request* req) {
    *req = MPI_REQUEST_NULL;
    return MPI_Send(buf, count, type, dest, tag, comm);  // eager: the payload is copied now
}
int MPI_Recv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm, MPI_Status* status) {
    auto& box = mailbox();
    for (auto it = box.begin(); it != box.end(); ++it) {
        if (it->tag != tag) continue;
        const size_t want = (size_t)count * type_size(type);
        if (it->bytes.size() > want) {
            std::fprintf(stderr, "mpi shim: message of %zu bytes into a buffer of %zu\n", it->bytes.size(), want);
            std::abort();
        }
        std::memcpy(buf, it->bytes.data(), it->bytes.size());
        box.erase(it);
        if (status) {
            status->MPI_SOURCE = source;
            status->MPI_TAG = tag;
            status->MPI_ERROR = 0;
        }
        return MPI_SUCCESS;
    }
    std::fprintf(stderr, "mpi shim: receive with tag %d and no matching send (one rank)\n", tag);
    std::abort();
}
int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request* req) {
    *req = MPI_REQUEST_NULL;
    return MPI_Recv(buf, count, type, source, tag, comm, MPI_STATUS_IGNORE);
}
int MPI_Wait(MPI_Request*, MPI_Status*) { return MPI_SUCCESS; }
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op, int, MPI_Comm) {
    if (sendbuf != MPI_IN_PLACE && sendbuf != recvbuf) std::memcpy(recvbuf, sendbuf, (size_t)count * type_size(type));
    return MPI_SUCCESS;
}
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm) {
    return MPI_Reduce(sendbuf, recvbuf, count, type, op, 0, comm);
}
int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int, MPI_Datatype,
                  MPI_Comm) {
    if (sendbuf != MPI_IN_PLACE && sendbuf != recvbuf)
        std::memcpy(recvbuf, sendbuf, (size_t)sendcount * type_size(sendtype));
    return MPI_SUCCESS;
}
double MPI_Wtime(void) { return omp_get_wtime(); }
}

// ---------------------------------------------------------------------------
// FFTW: a plan is the grid, the batch layout, the two arrays and the sign.
struct edus_shim_fftw_plan_s {
    int rank = 0;
    int n[3] = {1, 1, 1};
    long howmany = 1;
    long stride = 1;  // distance between consecutive grid points of one transform
    long dist = 1;    // distance between the first points of consecutive transforms
    cd* in = nullptr;
    cd* out = nullptr;
    int sign = -1;
    oracle::Fft1d axis[3];
};

namespace {
fftw_plan make_plan(int rank, const long* n, long howmany, long stride, long dist, fftw_complex* in,
                    fftw_complex* out, int sign) {
    if (rank < 1 || rank > 3) {
        std::fprintf(stderr, "fftw shim: rank %d transforms are not supported\n", rank);
        std::abort();
    }
    auto* p = new edus_shim_fftw_plan_s;
    p->rank = rank;
    for (int d = 0; d < rank; ++d) {
        p->n[d] = (int)n[d];
        p->axis[d] = oracle::Fft1d((int)n[d]);
    }
    p->howmany = howmany;
    p->stride = stride;
    p->dist = dist;
    p->in = reinterpret_cast<cd*>(in);
    p->out = reinterpret_cast<cd*>(out);
    p->sign = sign;
    return p;
}
}  // namespace

extern "C" {
fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany, fftw_complex* in, const int* inembed, int istride,
                             int idist, fftw_complex* out, const int* onembed, int ostride, int odist, int sign,
                             unsigned) {
    if (inembed || onembed || istride != ostride || idist != odist) {
        std::fprintf(stderr, "fftw shim: only identical, unembedded input and output layouts are supported\n");
        std::abort();
    }
    long nn[3];
    for (int d = 0; d < rank; ++d) nn[d] = n[d];
    return make_plan(rank, nn, howmany, istride, idist, in, out, sign);
}

fftw_plan fftw_mpi_plan_many_dft(int rnk, const std::ptrdiff_t* n, std::ptrdiff_t howmany, std::ptrdiff_t,
                                 std::ptrdiff_t, fftw_complex* in, fftw_complex* out, MPI_Comm, int sign, unsigned) {
    long nn[3];
    for (int d = 0; d < rnk; ++d) nn[d] = (long)n[d];
    return make_plan(rnk, nn, (long)howmany, (long)howmany, 1, in, out, sign);
}

// Unnormalised multi-dimensional DFT with exponent sign p->sign, row-major grid.
void fftw_execute(const fftw_plan p) {
    long Nk = 1;
    for (int d = 0; d < p->rank; ++d) Nk *= p->n[d];
    if (p->in != p->out) {
#pragma omp parallel for schedule(static)
        for (long h = 0; h < p->howmany; ++h)
            for (long k = 0; k < Nk; ++k) p->out[h * p->dist + k * p->stride] = p->in[h * p->dist + k * p->stride];
    }
    for (int d = 0; d < p->rank; ++d) {
        const int N = p->n[d];
        if (N == 1) continue;
        long inner = 1;  // grid points after axis d
        for (int e = d + 1; e < p->rank; ++e) inner *= p->n[e];
        long outer = 1;
        for (int e = 0; e < d; ++e) outer *= p->n[e];
        const long nlines = outer * inner * p->howmany;
#pragma omp parallel
        {
            std::vector<cd> line(N), work;
#pragma omp for schedule(static)
            for (long l = 0; l < nlines; ++l) {
                const long h = l % p->howmany;
                const long g = l / p->howmany;
                const long o = g / inner, i = g % inner;
                cd* base = p->out + h * p->dist + (o * N * inner + i) * p->stride;
                const long step = inner * p->stride;
                for (int j = 0; j < N; ++j) line[j] = base[j * step];
                p->axis[d].run(line.data(), p->sign, work);
                for (int j = 0; j < N; ++j) base[j * step] = line[j];
            }
        }
    }
}

void fftw_destroy_plan(fftw_plan p) { delete p; }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int) {}
int fftw_planner_nthreads(void) { return omp_get_max_threads(); }
void fftw_cleanup(void) {}
void fftw_mpi_init(void) {}
void fftw_mpi_cleanup(void) {}
std::ptrdiff_t fftw_mpi_local_size_many(int rnk, const std::ptrdiff_t* n, std::ptrdiff_t howmany, std::ptrdiff_t,
                                        MPI_Comm, std::ptrdiff_t* local_n0, std::ptrdiff_t* local_0_start) {
    std::ptrdiff_t total = howmany;
    for (int d = 0; d < rnk; ++d) total *= n[d];
    *local_n0 = n[0];
    *local_0_start = 0;
    return total;
}
}

// ---------------------------------------------------------------------------
// BLAS / LAPACK subset (row-major)
namespace {
template <typename T>
T conj_if(T x, bool c) {
    return x;
}
template <>
cd conj_if<cd>(cd x, bool c) {
    return c ? std::conj(x) : x;
}

// C = alpha op(A) op(B) + beta C, row-major
template <typename T>
void gemm_rm(CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, int m, int n, int k, T alpha, const T* a, int lda, const T* b,
             int ldb, T beta, T* c, int ldc) {
    auto A = [&](int i, int l) {
        return ta == CblasNoTrans ? a[(long)i * lda + l] : conj_if(a[(long)l * lda + i], ta == CblasConjTrans);
    };
    auto B = [&](int l, int j) {
        return tb == CblasNoTrans ? b[(long)l * ldb + j] : conj_if(b[(long)j * ldb + l], tb == CblasConjTrans);
    };
    std::vector<T> row(n);
    for (int i = 0; i < m; ++i) {
        std::fill(row.begin(), row.end(), T(0));
        for (int l = 0; l < k; ++l) {
            const T ail = A(i, l);
            for (int j = 0; j < n; ++j) row[j] += ail * B(l, j);
        }
        for (int j = 0; j < n; ++j) {
            T& cij = c[(long)i * ldc + j];
            cij = (beta == T(0) ? T(0) : beta * cij) + alpha * row[j];
        }
    }
}

void require_row_major(int layout, const char* who) {
    if (layout != CblasRowMajor && layout != LAPACK_ROW_MAJOR) {
        std::fprintf(stderr, "mkl shim: %s supports the row-major layout only\n", who);
        std::abort();
    }
}

// LU with partial pivoting in place (row-major), ipiv 1-based as LAPACK's
template <typename T>
lapack_int getrf(lapack_int m, lapack_int n, T* a, lapack_int lda, lapack_int* ipiv) {
    lapack_int info = 0;
    const int mn = std::min(m, n);
    for (int j = 0; j < mn; ++j) {
        int piv = j;
        double best = std::abs(a[(long)j * lda + j]);
        for (int i = j + 1; i < m; ++i) {
            const double v = std::abs(a[(long)i * lda + j]);
            if (v > best) {
                best = v;
                piv = i;
            }
        }
        ipiv[j] = piv + 1;
        if (best == 0.0) {
            if (info == 0) info = j + 1;
            continue;
        }
        if (piv != j)
            for (int l = 0; l < n; ++l) std::swap(a[(long)j * lda + l], a[(long)piv * lda + l]);
        const T inv = T(1) / a[(long)j * lda + j];
        for (int i = j + 1; i < m; ++i) {
            T& lij = a[(long)i * lda + j];
            lij *= inv;
            for (int l = j + 1; l < n; ++l) a[(long)i * lda + l] -= lij * a[(long)j * lda + l];
        }
    }
    return info;
}

// inverse from the LU factors: solve A X = I column by column
template <typename T>
lapack_int getri(lapack_int n, T* a, lapack_int lda, const lapack_int* ipiv) {
    for (int i = 0; i < n; ++i)
        if (a[(long)i * lda + i] == T(0)) return i + 1;
    std::vector<T> X((size_t)n * n), b(n);
    for (int col = 0; col < n; ++col) {
        for (int i = 0; i < n; ++i) b[i] = (i == col) ? T(1) : T(0);
        for (int i = 0; i < n; ++i) std::swap(b[i], b[ipiv[i] - 1]);
        for (int i = 0; i < n; ++i)
            for (int l = 0; l < i; ++l) b[i] -= a[(long)i * lda + l] * b[l];
        for (int i = n - 1; i >= 0; --i) {
            for (int l = i + 1; l < n; ++l) b[i] -= a[(long)i * lda + l] * b[l];
            b[i] /= a[(long)i * lda + i];
        }
        for (int i = 0; i < n; ++i) X[(size_t)i * n + col] = b[i];
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) a[(long)i * lda + j] = X[(size_t)i * n + j];
    return 0;
}
}  // namespace

void cblas_dgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, MKL_INT m, MKL_INT n, MKL_INT k,
                 double alpha, const double* a, MKL_INT lda, const double* b, MKL_INT ldb, double beta, double* c,
                 MKL_INT ldc) {
    require_row_major(layout, "cblas_dgemm");
    gemm_rm<double>(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

void cblas_zgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, MKL_INT m, MKL_INT n, MKL_INT k,
                 const void* alpha, const void* a, MKL_INT lda, const void* b, MKL_INT ldb, const void* beta, void* c,
                 MKL_INT ldc) {
    require_row_major(layout, "cblas_zgemm");
    gemm_rm<cd>(ta, tb, m, n, k, *static_cast<const cd*>(alpha), static_cast<const cd*>(a), lda,
                static_cast<const cd*>(b), ldb, *static_cast<const cd*>(beta), static_cast<cd*>(c), ldc);
}

void cblas_zgemm_batch_strided(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, MKL_INT m, MKL_INT n,
                               MKL_INT k, const void* alpha, const void* a, MKL_INT lda, MKL_INT stridea,
                               const void* b, MKL_INT ldb, MKL_INT strideb, const void* beta, void* c, MKL_INT ldc,
                               MKL_INT stridec, MKL_INT batch) {
    require_row_major(layout, "cblas_zgemm_batch_strided");
    const cd al = *static_cast<const cd*>(alpha), be = *static_cast<const cd*>(beta);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < batch; ++i)
        gemm_rm<cd>(ta, tb, m, n, k, al, static_cast<const cd*>(a) + (long)i * stridea, lda,
                    static_cast<const cd*>(b) + (long)i * strideb, ldb, be, static_cast<cd*>(c) + (long)i * stridec,
                    ldc);
}

lapack_int LAPACKE_zheevd(int layout, char jobz, char uplo, lapack_int n, MKL_Complex16* a, lapack_int lda,
                          double* w) {
    require_row_major(layout, "LAPACKE_zheevd");
    if (jobz != 'V' || uplo != 'U') {
        std::fprintf(stderr, "mkl shim: LAPACKE_zheevd supports jobz='V', uplo='U' only\n");
        std::abort();
    }
    std::vector<cd> A((size_t)n * n), V((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) A[(size_t)i * n + j] = a[(long)i * lda + j];
    oracle::eigh(n, A.data(), w, V.data());
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) a[(long)i * lda + j] = V[(size_t)i * n + j];
    return 0;
}

lapack_int LAPACKE_dsyev(int layout, char jobz, char uplo, lapack_int n, double* a, lapack_int lda, double* w) {
    require_row_major(layout, "LAPACKE_dsyev");
    if (jobz != 'V' || uplo != 'U') {
        std::fprintf(stderr, "mkl shim: LAPACKE_dsyev supports jobz='V', uplo='U' only\n");
        std::abort();
    }
    std::vector<cd> A((size_t)n * n), V((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) A[(size_t)i * n + j] = a[(long)i * lda + j];
    oracle::eigh(n, A.data(), w, V.data());
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) a[(long)i * lda + j] = V[(size_t)i * n + j].real();
    return 0;
}

lapack_int LAPACKE_dgetrf(int layout, lapack_int m, lapack_int n, double* a, lapack_int lda, lapack_int* ipiv) {
    require_row_major(layout, "LAPACKE_dgetrf");
    return getrf<double>(m, n, a, lda, ipiv);
}
lapack_int LAPACKE_dgetri(int layout, lapack_int n, double* a, lapack_int lda, const lapack_int* ipiv) {
    require_row_major(layout, "LAPACKE_dgetri");
    return getri<double>(n, a, lda, ipiv);
}
lapack_int LAPACKE_zgetrf(int layout, lapack_int m, lapack_int n, MKL_Complex16* a, lapack_int lda,
                          lapack_int* ipiv) {
    require_row_major(layout, "LAPACKE_zgetrf");
    return getrf<cd>(m, n, a, lda, ipiv);
}
lapack_int LAPACKE_zgetri(int layout, lapack_int n, MKL_Complex16* a, lapack_int lda, const lapack_int* ipiv) {
    require_row_major(layout, "LAPACKE_zgetri");
    return getri<cd>(n, a, lda, ipiv);
}

// Full SVD A = U diag(s) V^T (jobu = jobvt = 'A'): V and s from the symmetric
// eigenproblem of A^T A, U's leading columns A v / s, the rest completed to an
// orthonormal basis by Gram-Schmidt.  Singular values descending.
lapack_int LAPACKE_dgesvd(int layout, char jobu, char jobvt, lapack_int m, lapack_int n, double* a, lapack_int lda,
                          double* s, double* u, lapack_int ldu, double* vt, lapack_int ldvt, double*) {
    require_row_major(layout, "LAPACKE_dgesvd");
    if (jobu != 'A' || jobvt != 'A') {
        std::fprintf(stderr, "mkl shim: LAPACKE_dgesvd supports jobu = jobvt = 'A' only\n");
        std::abort();
    }
    std::vector<cd> AtA((size_t)n * n), V((size_t)n * n);
    std::vector<double> lam(n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double acc = 0;
            for (int l = 0; l < m; ++l) acc += a[(long)l * lda + i] * a[(long)l * lda + j];
            AtA[(size_t)i * n + j] = acc;
        }
    oracle::eigh(n, AtA.data(), lam.data(), V.data());
    // descending order
    std::vector<int> ord(n);
    for (int i = 0; i < n; ++i) ord[i] = n - 1 - i;
    const int mn = std::min(m, n);
    for (int i = 0; i < mn; ++i) s[i] = std::sqrt(std::max(lam[ord[i]], 0.0));
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) vt[(long)i * ldvt + j] = V[(size_t)j * n + ord[i]].real();
    const double tol = (mn > 0 ? s[0] : 0.0) * 1e-13 * std::max(m, n);
    std::vector<double> U((size_t)m * m, 0.0);
    int filled = 0;
    for (int i = 0; i < mn; ++i) {
        if (s[i] <= tol) break;
        for (int r = 0; r < m; ++r) {
            double acc = 0;
            for (int l = 0; l < n; ++l) acc += a[(long)r * lda + l] * vt[(long)i * ldvt + l];
            U[(size_t)r * m + i] = acc / s[i];
        }
        ++filled;
    }
    for (int e = 0; filled < m && e < m; ++e) {  // complete with unit vectors
        std::vector<double> v(m, 0.0);
        v[e] = 1.0;
        for (int pass = 0; pass < 2; ++pass)
            for (int c = 0; c < filled; ++c) {
                double d = 0;
                for (int r = 0; r < m; ++r) d += U[(size_t)r * m + c] * v[r];
                for (int r = 0; r < m; ++r) v[r] -= d * U[(size_t)r * m + c];
            }
        double nrm = 0;
        for (int r = 0; r < m; ++r) nrm += v[r] * v[r];
        nrm = std::sqrt(nrm);
        if (nrm < 1e-8) continue;
        for (int r = 0; r < m; ++r) U[(size_t)r * m + filled] = v[r] / nrm;
        ++filled;
    }
    for (int r = 0; r < m; ++r)
        for (int c = 0; c < m; ++c) u[(long)r * ldu + c] = U[(size_t)r * m + c];
    return 0;
}

int mkl_get_max_threads(void) { return 1; }
void mkl_set_num_threads(int) {}
