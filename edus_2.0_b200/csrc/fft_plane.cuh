// In-shared-memory FFT of one band-pair plane over the k (or R) grid.
//
// The forward transform (k -> R, sign -1) is an in-place mixed-radix
// decimation-in-frequency pass per axis: natural-order input, output left in
// mixed-radix digit-reversed positions.  The inverse (R -> k, sign +1) is the
// exact reverse flow graph, decimation in time: it consumes the
// digit-reversed positions and leaves natural order.  The pointwise R-space
// work between the two therefore runs on permuted positions; everything the
// pointwise step reads (W, rho0, the R coordinates) is stored in that same
// position order, so no permutation pass ever touches memory.
//
// Radix r stage with sub-length M = L*r (L = M/r) on one line:
//   DIF: y_d = W_M^{a d} sum_b x[a + L b] W_r^{b d},      stored at a + L d
//   DIT: x_b = sum_d W_r^{-b d} (W_M^{-a d} y[a + L d]),   stored at a + L b
// with a in [0, L), over every block of M consecutive positions.
#pragma once
#include <cuda_runtime.h>

namespace edus {

constexpr int kMaxStages = 12;

struct AxisPlan {
    int n;        // length along the axis (1 = axis absent)
    int nst;      // number of radix stages
    int inner;    // element stride of the axis inside the plane
    int rootoff;  // offset of exp(-2 pi i j / n), j < n, in the root table
    int rposoff;  // offset of the R coordinate of each position
    int r[kMaxStages];
    int L[kMaxStages];
};

struct PlanePlan {
    AxisPlan ax[3];
    int Nk;
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// multiply by s*i (s = +1 or -1)
template <int S>
__device__ __forceinline__ double2 cmul_si(double2 a) {
    return S > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

// In-register DFT y_d = sum_b x_b exp(S 2 pi i b d / R), hand-coded radices.
template <int R, int S>
struct Dft;

template <int S>
struct Dft<2, S> {
    __device__ __forceinline__ static void run(double2* v, const double2*, int) {
        double2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <int S>
struct Dft<3, S> {
    __device__ __forceinline__ static void run(double2* v, const double2*, int) {
        const double h = 0.86602540378443864676;  // sqrt(3)/2
        double2 t1 = cadd(v[1], v[2]);
        double2 t2 = make_double2(v[0].x - 0.5 * t1.x, v[0].y - 0.5 * t1.y);
        double2 t3 = cmul_si<S>(cscale(csub(v[1], v[2]), h));
        v[0] = cadd(v[0], t1);
        v[1] = cadd(t2, t3);
        v[2] = csub(t2, t3);
    }
};

template <int S>
struct Dft<4, S> {
    __device__ __forceinline__ static void run(double2* v, const double2*, int) {
        double2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        double2 b0 = cadd(v[1], v[3]), b1 = cmul_si<S>(csub(v[1], v[3]));
        v[0] = cadd(a0, b0);
        v[2] = csub(a0, b0);
        v[1] = cadd(a1, b1);
        v[3] = csub(a1, b1);
    }
};

template <int S>
struct Dft<5, S> {
    __device__ __forceinline__ static void run(double2* v, const double2*, int) {
        const double c1 = 0.30901699437494742410;   // cos(2pi/5)
        const double c2 = -0.80901699437494742410;  // cos(4pi/5)
        const double s1 = 0.95105651629515357212;   // sin(2pi/5)
        const double s2 = 0.58778525229247312917;   // sin(4pi/5)
        double2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        double2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        double2 a1 = make_double2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
        double2 a2 = make_double2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
        double2 b1 = cmul_si<S>(make_double2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
        double2 b2 = cmul_si<S>(make_double2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
        v[0] = cadd(v[0], cadd(t1, t2));
        v[1] = cadd(a1, b1);
        v[4] = csub(a1, b1);
        v[2] = cadd(a2, b2);
        v[3] = csub(a2, b2);
    }
};

template <int S>
struct Dft<8, S> {
    __device__ __forceinline__ static void run(double2* v, const double2*, int) {
        const double r2 = 0.70710678118654752440;
        double2 a[4], b[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            a[j] = cadd(v[j], v[j + 4]);
            b[j] = csub(v[j], v[j + 4]);
        }
        // b_j *= exp(S 2 pi i j / 8)
        b[1] = cscale(cadd(b[1], cmul_si<S>(b[1])), r2);
        b[2] = cmul_si<S>(b[2]);
        b[3] = cscale(csub(cmul_si<S>(b[3]), b[3]), r2);
        Dft<4, S>::run(a, nullptr, 0);
        Dft<4, S>::run(b, nullptr, 0);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            v[2 * m] = a[m];
            v[2 * m + 1] = b[m];
        }
    }
};

// Generic odd radix (7) through the axis root table:
// W_R^{m} = root[m * (n / R)] (conjugated for S = +1).
template <int R, int S>
struct DftGeneric {
    __device__ __forceinline__ static void run(double2* v, const double2* root, int n) {
        double2 y[R];
        const int step = n / R;
#pragma unroll
        for (int d = 0; d < R; ++d) {
            double2 s = v[0];
#pragma unroll
            for (int b = 1; b < R; ++b) {
                double2 w = __ldg(&root[((b * d) % R) * step]);
                if (S > 0) w.y = -w.y;
                s = cadd(s, cmul(v[b], w));
            }
            y[d] = s;
        }
#pragma unroll
        for (int d = 0; d < R; ++d) v[d] = y[d];
    }
};
template <int S>
struct Dft<7, S> : DftGeneric<7, S> {};

// One radix-R stage over every line of axis `ax` of the NBUF planes that
// start at `buf[0]`, `buf[0] + bufstride`, ...  DIF when FWD, DIT otherwise.
template <int R, bool FWD, int NBUF>
__device__ __forceinline__ void stage_R(double2* buf, int bufstride, int Nk, const AxisPlan& ax, int L,
                                        const double2* __restrict__ root) {
    constexpr int S = FWD ? -1 : +1;
    const int n = ax.n;
    const int inner = ax.inner;
    const int M = L * R;
    const int nbfly = n / R;
    const int tw_step = n / M;
    const int ntask = Nk / R;
    for (int t = threadIdx.x; t < ntask; t += blockDim.x) {
        const int in = t % inner;
        const int tmp = t / inner;
        const int bfly = tmp % nbfly;
        const int o = tmp / nbfly;
        const int blk = bfly / L;
        const int a = bfly - blk * L;
        const int base = o * (n * inner) + in + (blk * M + a) * inner;
        const int step = L * inner;
        double2 tw[R];
        tw[0] = make_double2(1.0, 0.0);
#pragma unroll
        for (int d = 1; d < R; ++d) {
            double2 w = __ldg(&root[a * d * tw_step]);
            if (!FWD) w.y = -w.y;
            tw[d] = w;
        }
#pragma unroll
        for (int q = 0; q < NBUF; ++q) {
            double2* X = buf + q * bufstride;
            double2 v[R];
#pragma unroll
            for (int b = 0; b < R; ++b) v[b] = X[base + b * step];
            if (FWD) {
                Dft<R, S>::run(v, root, n);
#pragma unroll
                for (int d = 1; d < R; ++d) v[d] = cmul(v[d], tw[d]);
            } else {
#pragma unroll
                for (int d = 1; d < R; ++d) v[d] = cmul(v[d], tw[d]);
                Dft<R, S>::run(v, root, n);
            }
#pragma unroll
            for (int b = 0; b < R; ++b) X[base + b * step] = v[b];
        }
    }
}

template <bool FWD, int NBUF>
__device__ __forceinline__ void run_stage(double2* buf, int bufstride, int Nk, const AxisPlan& ax, int s,
                                          const double2* __restrict__ roots) {
    const double2* root = roots + ax.rootoff;
    const int L = ax.L[s];
    switch (ax.r[s]) {
        case 2: stage_R<2, FWD, NBUF>(buf, bufstride, Nk, ax, L, root); break;
        case 3: stage_R<3, FWD, NBUF>(buf, bufstride, Nk, ax, L, root); break;
        case 4: stage_R<4, FWD, NBUF>(buf, bufstride, Nk, ax, L, root); break;
        case 5: stage_R<5, FWD, NBUF>(buf, bufstride, Nk, ax, L, root); break;
        case 7: stage_R<7, FWD, NBUF>(buf, bufstride, Nk, ax, L, root); break;
        case 8: stage_R<8, FWD, NBUF>(buf, bufstride, Nk, ax, L, root); break;
        default: break;  // rejected on the host
    }
}

// Forward (k -> R, unnormalised sign -1) transform of the plane(s) in place.
template <int NBUF>
__device__ void plane_forward(double2* buf, int bufstride, const PlanePlan& pl, const double2* __restrict__ roots) {
#pragma unroll 1
    for (int d = 0; d < 3; ++d) {
        const AxisPlan& ax = pl.ax[d];
#pragma unroll 1
        for (int s = 0; s < ax.nst; ++s) {
            run_stage<true, NBUF>(buf, bufstride, pl.Nk, ax, s, roots);
            __syncthreads();
        }
    }
}

// Inverse (R -> k, unnormalised sign +1) transform, exact reverse of plane_forward.
template <int NBUF>
__device__ void plane_inverse(double2* buf, int bufstride, const PlanePlan& pl, const double2* __restrict__ roots) {
#pragma unroll 1
    for (int d = 2; d >= 0; --d) {
        const AxisPlan& ax = pl.ax[d];
#pragma unroll 1
        for (int s = ax.nst - 1; s >= 0; --s) {
            run_stage<false, NBUF>(buf, bufstride, pl.Nk, ax, s, roots);
            __syncthreads();
        }
    }
}

}  // namespace edus
