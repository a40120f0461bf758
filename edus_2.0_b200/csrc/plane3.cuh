// Plane transforms spread over many CTAs, for 2-D grids with few band-pair
// planes (a plane per CTA would leave most SMs idle: 4 planes of 120 x 120 for
// two bands).  The same contract as plane_rhs_kernel, in three launches whose
// intermediates stay in L2:
//   rows    CTA (plane, row chunk): k -> R along axis 1 of Rc rows;
//   columns CTA (plane, column chunk): k -> R along axis 0 of Cc columns,
//           the pointwise gradient / self-energy / model terms at the full
//           plane's digit-reversed positions, R -> k along axis 0 of G and H;
//   rows    CTA (plane x {G, H}, row chunk): R -> k along axis 1.
// A stage transforms whole lines of one axis of a [outer][n][inner] sub-array
// (fft_plane.cuh's stage indexing is generic in Nk, n and inner), so the
// sub-plans below reuse the plane's radices, roots and coordinate tables.
// MASK: the radices compiled in (the common set unless the plan needs 11 or 13).
// Reference: Functional_SourceTerm.hpp:15-50, kGradient_definitions.hpp:35-40,
// Coulomb.cpp:150-171, fftPair.cpp:89-107.
#pragma once
#include "kernels.cuh"

namespace edus {

struct Plane3Plan {
    PlanePlan rows;  // axis 1 of [Rc][N1]
    PlanePlan cols;  // axis 0 of [N0][Cc]
    int Rc, Cc;
};

// largest divisor of n that is <= cap
inline int divisor_upto(int n, int cap) {
    for (int d = std::min(n, cap); d >= 1; --d)
        if (n % d == 0) return d;
    return 1;
}

inline Plane3Plan plane3_plan(const PlanePlan& full, int Rc, int Cc) {
    Plane3Plan q;
    q.Rc = Rc;
    q.Cc = Cc;
    q.rows = full;
    q.rows.ax[0].nst = 0;
    q.rows.ax[2].nst = 0;
    q.rows.Nk = Rc * full.ax[1].n;
    q.cols = full;
    q.cols.ax[1].nst = 0;
    q.cols.ax[2].nst = 0;
    q.cols.ax[0].inner = Cc;
    q.cols.ax[0].fd_inner = make_fastdiv(Cc);
    q.cols.Nk = full.ax[0].n * Cc;
    return q;
}

// rows: dst[plane][r][*] = FFT along axis 1 (FWD: k -> R) of src rows of the
// CTA's chunk; with nout = 2 the CTAs alternate between (src, dst) and
// (src2, dst2) (the G and H planes of the inverse pass)
template <bool FWD, int MAXT, int MASK = kRadixAll>
__global__ void __launch_bounds__(MAXT) plane3_rows_kernel(const double2* __restrict__ src, long long src_bstride,
                                                         double2* __restrict__ dst, long long dst_bstride, int P,
                                                         PlanePlan sub, int nout, const double2* __restrict__ roots,
                                                         const double2* __restrict__ src2, double2* __restrict__ dst2) {
    extern __shared__ double2 x3[];
    const int which = blockIdx.x % nout;
    const int plane = blockIdx.x / nout;
    const int b = plane / P, p = plane - (plane / P) * P;
    const int Nk = gridDim.y * sub.Nk;  // whole plane: row chunks x chunk size
    const long long so = (long long)b * src_bstride + (long long)p * Nk + (long long)blockIdx.y * sub.Nk;
    const long long dof = (long long)b * dst_bstride + (long long)p * Nk + (long long)blockIdx.y * sub.Nk;
    const double2* s = which ? src2 : src;
    double2* d = which ? dst2 : dst;
    for (int i = threadIdx.x; i < sub.Nk; i += blockDim.x) x3[i] = __ldg(&s[so + i]);
    __syncthreads();
    if (FWD) plane_forward<1, MASK>(x3, 0, sub, roots);
    else plane_inverse<1, MASK>(x3, 0, sub, roots);
    for (int i = threadIdx.x; i < sub.Nk; i += blockDim.x) d[dof + i] = x3[i];
}

// columns: k -> R along axis 0, pointwise terms, R -> k along axis 0 of G (and H)
template <bool COUL, int MAXT, int MASK = kRadixAll>
__global__ void __launch_bounds__(MAXT) plane3_cols_kernel(
    const double2* __restrict__ S1, long long bstride, double2* __restrict__ SG, double2* __restrict__ SH,
    const double2* __restrict__ rho0p, const double* __restrict__ Wp, double2* __restrict__ diag0,
    const StageField* __restrict__ field, const double2* __restrict__ roots, const double* __restrict__ rpos,
    PlanePlan full, PlanePlan sub, int Cc, int nb, double inv_nk, const int* __restrict__ hpos,
    const double2* __restrict__ hval, int nS) {
    extern __shared__ double2 x3[];
    const int P = nb * nb;
    const int plane = blockIdx.x;
    const int b = plane / P, p = plane - (plane / P) * P;
    const int N0 = full.ax[0].n, N1 = full.ax[1].n, Nk = full.Nk;
    const int c0 = blockIdx.y * Cc;
    const int tot = N0 * Cc;
    double2* X = x3;
    double2* Y = x3 + tot;
    const long long off = (long long)b * bstride + (long long)p * Nk;
    for (int i = threadIdx.x; i < tot; i += blockDim.x) {
        const int r = i / Cc, c = i - (i / Cc) * Cc;
        X[i] = __ldg(&S1[off + (long long)r * N1 + c0 + c]);
    }
    __syncthreads();
    plane_forward<1, MASK>(X, 0, sub, roots);
    const StageField F = field[b];
    const int n = p / nb, m = p - (p / nb) * nb;
    if (COUL && n == m && c0 == 0 && threadIdx.x == 0) diag0[b * nb + n] = cscale(X[0], inv_nk);
    __syncthreads();
    const double* rp0 = rpos + full.ax[0].rposoff;
    const double* rp1 = rpos + full.ax[1].rposoff;
    const double rz = rpos[full.ax[2].rposoff];
    for (int i = threadIdx.x; i < tot; i += blockDim.x) {
        const int q0 = i / Cc, q1 = c0 + (i - (i / Cc) * Cc);
        const int pos = q0 * N1 + q1;
        const double dot = F.g[0] * __ldg(&rp0[q0]) + F.g[1] * __ldg(&rp1[q1]) + F.g[2] * rz;
        const double2 r = cscale(X[i], inv_nk);
        if (COUL) {
            const double2 r0 = __ldg(&rho0p[(long long)p * Nk + pos]);
            const double wv = __ldg(&Wp[(long long)p * Nk + pos]);
            Y[i] = make_double2(-wv * (r.x - r0.x), -wv * (r.y - r0.y));
        }
        X[i] = make_double2(-dot * r.y, dot * r.x);
    }
    __syncthreads();
    if (COUL && nS > 0) {
        // the sparse model H0(R) + E.xi(R) on this chunk's columns
        for (int s2 = threadIdx.x; s2 < nS; s2 += blockDim.x) {
            const int pos = __ldg(&hpos[s2]);
            const int q0 = pos / N1, q1 = pos - (pos / N1) * N1;
            if (q1 < c0 || q1 >= c0 + Cc) continue;
            const int i = q0 * Cc + (q1 - c0);
            double2 v = Y[i];
            const double2 h0 = __ldg(&hval[(long long)p * nS + s2]);
            v.x += h0.x;
            v.y += h0.y;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (F.E[d] != 0.0) {
                    const double2 x = __ldg(&hval[((long long)(d + 1) * P + p) * nS + s2]);
                    v.x += F.E[d] * x.x;
                    v.y += F.E[d] * x.y;
                }
            }
            Y[i] = v;
        }
        __syncthreads();
    }
    if (COUL) plane_inverse<2, MASK>(X, tot, sub, roots);
    else plane_inverse<1, MASK>(X, 0, sub, roots);
    for (int i = threadIdx.x; i < tot; i += blockDim.x) {
        const int r = i / Cc, c = i - (i / Cc) * Cc;
        SG[off + (long long)r * N1 + c0 + c] = X[i];
        if (COUL) SH[off + (long long)r * N1 + c0 + c] = Y[i];
    }
}

}  // namespace edus
