// TEST INFRASTRUCTURE ONLY -- part of the CPU oracle.  Nothing in the product
// (edus_2.0_b200/) may include, link or call this file.
//
// Mixed-radix FFT used by the oracle in place of FFTW.  It restates the
// transform the reference asks FFTW for:
//   * src/fftPair/fftPair.cpp:39-61  fftw_mpi_plan_many_dft over the k grid,
//     `howmany` = nb*nb interleaved planes (stride howmany, distance 1),
//     unnormalised, sign -1 for k->R and +1 for R->k;
//   * src/fftPair/fftPair.cpp:89-107 the k->R transform is then divided by
//     the number of grid points (sign -1 only).
// The algorithm is the textbook Stockham autosort formulation; any correct
// FFT agrees with FFTW to rounding (~1e-15 relative).
#pragma once
#include <complex>
#include <vector>
#include <cmath>
#include <stdexcept>

namespace oracle {

using cd = std::complex<double>;

struct Fft1d {
    int n = 1;
    std::vector<int> radices;
    std::vector<cd> roots;   // exp(-2 pi i j / n), j = 0..n-1

    explicit Fft1d(int n_ = 1) : n(n_) {
        int m = n;
        for (int r : {4, 2, 3, 5}) {
            while (m % r == 0) { radices.push_back(r); m /= r; }
        }
        // any remaining prime factor is handled by the generic radix loop
        for (int p = 7; m > 1; p += 2) {
            while (m % p == 0) { radices.push_back(p); m /= p; }
        }
        roots.resize(n);
        for (int j = 0; j < n; ++j) {
            long double a = -2.0L * 3.14159265358979323846264338327950288L * j / n;
            roots[j] = cd((double)std::cos(a), (double)std::sin(a));
        }
    }

    // In-place transform of x[0..n) (contiguous). sign = -1 forward, +1 backward.
    void run(cd* x, int sign, std::vector<cd>& work) const {
        if (n == 1) return;
        work.resize(n);
        cd* a = x;
        cd* b = work.data();
        int p = 1;
        cd v[64], y[64];
        for (int R : radices) {
            const int NR = n / R;
            for (int i = 0; i < NR; ++i) {
                const int k = i % p;
                for (int j = 0; j < R; ++j) {
                    cd t = a[i + j * NR];
                    // twiddle exp(sign 2 pi i j k / (p R)) = root[(j k n/(pR)) mod n]
                    long idx = (long)j * k * (n / (p * R)) % n;
                    cd w = roots[idx];
                    if (sign > 0) w = std::conj(w);
                    v[j] = t * w;
                }
                for (int q = 0; q < R; ++q) {
                    cd s = 0.0;
                    for (int m = 0; m < R; ++m) {
                        long idx = (long)m * q % R * (n / R) % n;
                        cd w = roots[idx];
                        if (sign > 0) w = std::conj(w);
                        s += v[m] * w;
                    }
                    y[q] = s;
                }
                const int base = (i / p) * p * R + k;
                for (int q = 0; q < R; ++q) b[base + q * p] = y[q];
            }
            std::swap(a, b);
            p *= R;
        }
        if (a != x) {
            for (int j = 0; j < n; ++j) x[j] = a[j];
        }
    }
};

// Batched 3-D transform of `howmany` interleaved planes:
// element (i0,i1,i2,h) at ((i0*N1+i1)*N2+i2)*howmany + h  (the MPI layout of
// the reference, src/Operator/Operator.hpp:236-238).
struct Fft3dMany {
    int N[3] = {1, 1, 1};
    int howmany = 1;
    Fft1d f[3];

    Fft3dMany() = default;
    Fft3dMany(const int dims[3], int howmany_) : howmany(howmany_) {
        for (int d = 0; d < 3; ++d) { N[d] = dims[d]; f[d] = Fft1d(dims[d]); }
    }

    // out = FFT_sign(in); when sign = -1 the result is divided by N0*N1*N2
    // (fftPair.cpp:98-105).  in and out may alias.
    void run(const cd* in, cd* out, int sign) const {
        const long Nk = (long)N[0] * N[1] * N[2];
        if (in != out) {
            for (long i = 0; i < Nk * howmany; ++i) out[i] = in[i];
        }
        for (int d = 0; d < 3; ++d) {
            if (N[d] == 1) continue;
            // strides in units of elements
            long stride = howmany;
            for (int e = d + 1; e < 3; ++e) stride *= N[e];
            long outer = 1;
            for (int e = 0; e < d; ++e) outer *= N[e];
            long inner = stride;  // number of (i_{d+1..2}, h) combinations
            const long nlines = outer * inner;
#pragma omp parallel
            {
                std::vector<cd> line(N[d]), work;
#pragma omp for schedule(static)
                for (long l = 0; l < nlines; ++l) {
                    long o = l / inner, in_off = l % inner;
                    cd* base = out + o * (long)N[d] * stride + in_off;
                    for (int j = 0; j < N[d]; ++j) line[j] = base[(long)j * stride];
                    f[d].run(line.data(), sign, work);
                    for (int j = 0; j < N[d]; ++j) base[(long)j * stride] = line[j];
                }
            }
        }
        if (sign == -1) {
            const double inv = (double)Nk;
#pragma omp parallel for schedule(static)
            for (long i = 0; i < Nk * howmany; ++i) out[i] /= inv;
        }
    }
};

}  // namespace oracle
