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

constexpr int kMaxStages = 8;

// Division by a run-time constant d < 2^16 of x < 2^24 without a divide:
// q = (x * m) >> 40 with m = ceil(2^40 / d).  The error of x*m/2^40 against
// x/d is below x/2^40 < 2^-16 < 1/d, so the floor is exact.
struct FastDiv {
    unsigned long long m;
    int d;
};
inline FastDiv make_fastdiv(int d) {
    FastDiv f;
    f.d = d;
    f.m = ((1ull << 40) + (unsigned long long)d - 1ull) / (unsigned long long)d;
    return f;
}
__device__ __forceinline__ int fdiv(int x, const FastDiv& f) {
    return (int)(((unsigned long long)(unsigned)x * f.m) >> 40);
}

struct AxisPlan {
    int n;        // length along the axis (1 = axis absent)
    int nst;      // number of radix stages
    int inner;    // element stride of the axis inside the plane
    int rootoff;  // offset of exp(-2 pi i j / n), j < n, in the root table
    int rposoff;  // offset of the R coordinate of each position
    int r[kMaxStages];
    int L[kMaxStages];
    FastDiv fd_inner;               // divide by inner
    FastDiv fd_nbfly[kMaxStages];   // divide by n / r
    FastDiv fd_L[kMaxStages];       // divide by L
};

struct PlanePlan {
    AxisPlan ax[3];
    int Nk;
    FastDiv fd_n1, fd_n2;  // position -> (q0, q1, q2) in the pointwise stage
};

// Complex helpers for double2 and float2 (the plane kernels run the FFT in
// FP64 for the FP64 forms and in FP32 for the mixed-precision form).
template <typename C>
struct CplxT;
template <>
struct CplxT<double2> {
    using T = double;
};
template <>
struct CplxT<float2> {
    using T = float;
};

__device__ __forceinline__ double2 mkc(double x, double y, double2*) { return make_double2(x, y); }
__device__ __forceinline__ float2 mkc(float x, float y, float2*) { return make_float2(x, y); }
template <typename C>
__device__ __forceinline__ C cmake(typename CplxT<C>::T x, typename CplxT<C>::T y) {
    return mkc(x, y, (C*)nullptr);
}

template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
    return cmake<C>(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { return cmake<C>(a.x + b.x, a.y + b.y); }
template <typename C>
__device__ __forceinline__ C csub(C a, C b) { return cmake<C>(a.x - b.x, a.y - b.y); }
template <typename C>
__device__ __forceinline__ C cscale(C a, typename CplxT<C>::T s) { return cmake<C>(a.x * s, a.y * s); }
// multiply by s*i (s = +1 or -1)
template <int S, typename C>
__device__ __forceinline__ C cmul_si(C a) {
    return S > 0 ? cmake<C>(-a.y, a.x) : cmake<C>(a.y, -a.x);
}
// root table entries are FP64; the FP32 transform rounds them once on use
// (the table may sit in global or in shared memory)
template <typename C>
__device__ __forceinline__ C ldroot(const double2* p) {
    const double2 w = *p;
    return cmake<C>((typename CplxT<C>::T)w.x, (typename CplxT<C>::T)w.y);
}

// In-register DFT y_d = sum_b x_b exp(S 2 pi i b d / R), hand-coded radices.
template <int R, int S, typename C>
struct Dft;

template <int S, typename C>
struct Dft<2, S, C> {
    __device__ __forceinline__ static void run(C* v, const double2*, int) {
        C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <int S, typename C>
struct Dft<3, S, C> {
    __device__ __forceinline__ static void run(C* v, const double2*, int) {
        using T = typename CplxT<C>::T;
        const T h = (T)0.86602540378443864676;  // sqrt(3)/2
        C t1 = cadd(v[1], v[2]);
        C t2 = cmake<C>(v[0].x - (T)0.5 * t1.x, v[0].y - (T)0.5 * t1.y);
        C t3 = cmul_si<S>(cscale(csub(v[1], v[2]), h));
        v[0] = cadd(v[0], t1);
        v[1] = cadd(t2, t3);
        v[2] = csub(t2, t3);
    }
};

template <int S, typename C>
struct Dft<4, S, C> {
    __device__ __forceinline__ static void run(C* v, const double2*, int) {
        C a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        C b0 = cadd(v[1], v[3]), b1 = cmul_si<S>(csub(v[1], v[3]));
        v[0] = cadd(a0, b0);
        v[2] = csub(a0, b0);
        v[1] = cadd(a1, b1);
        v[3] = csub(a1, b1);
    }
};

template <int S, typename C>
struct Dft<5, S, C> {
    __device__ __forceinline__ static void run(C* v, const double2*, int) {
        using T = typename CplxT<C>::T;
        const T c1 = (T)0.30901699437494742410;   // cos(2pi/5)
        const T c2 = (T)-0.80901699437494742410;  // cos(4pi/5)
        const T s1 = (T)0.95105651629515357212;   // sin(2pi/5)
        const T s2 = (T)0.58778525229247312917;   // sin(4pi/5)
        C t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        C t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        C a1 = cmake<C>(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
        C a2 = cmake<C>(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
        C b1 = cmul_si<S>(cmake<C>(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
        C b2 = cmul_si<S>(cmake<C>(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
        v[0] = cadd(v[0], cadd(t1, t2));
        v[1] = cadd(a1, b1);
        v[4] = csub(a1, b1);
        v[2] = cadd(a2, b2);
        v[3] = csub(a2, b2);
    }
};

template <int S, typename C>
struct Dft<8, S, C> {
    __device__ __forceinline__ static void run(C* v, const double2*, int) {
        using T = typename CplxT<C>::T;
        const T r2 = (T)0.70710678118654752440;
        C a[4], b[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            a[j] = cadd(v[j], v[j + 4]);
            b[j] = csub(v[j], v[j + 4]);
        }
        // b_j *= exp(S 2 pi i j / 8)
        b[1] = cscale(cadd(b[1], cmul_si<S>(b[1])), r2);
        b[2] = cmul_si<S>(b[2]);
        b[3] = cscale(csub(cmul_si<S>(b[3]), b[3]), r2);
        Dft<4, S, C>::run(a, nullptr, 0);
        Dft<4, S, C>::run(b, nullptr, 0);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            v[2 * m] = a[m];
            v[2 * m + 1] = b[m];
        }
    }
};

// Generic odd radix (7, 11, 13) through the axis root table,
// W_R^{m} = root[m * (n / R)] = cos(2 pi m / R) - i sin(2 pi m / R).  Inputs
// j and R - j are paired (a_j = x_j + x_{R-j}, b_j = x_j - x_{R-j}), so that
// with theta = 2 pi j d / R
//   y_d     = x_0 + sum_j a_j cos(theta) + S i sum_j b_j sin(theta)
//   y_{R-d} = x_0 + sum_j a_j cos(theta) - S i sum_j b_j sin(theta)
// (half the products of the plain sum, and R + 3 complex registers).
template <int R, int S, typename C>
struct DftGeneric {
    __device__ __forceinline__ static void run(C* v, const double2* root, int n) {
        using T = typename CplxT<C>::T;
        constexpr int H = (R - 1) / 2;
        const int step = n / R;
        C a[H], b[H];
        const C x0 = v[0];
        C y0 = x0;
#pragma unroll
        for (int j = 1; j <= H; ++j) {
            a[j - 1] = cadd(v[j], v[R - j]);
            b[j - 1] = csub(v[j], v[R - j]);
            y0 = cadd(y0, a[j - 1]);
        }
        v[0] = y0;
#pragma unroll
        for (int d = 1; d <= H; ++d) {
            C A = x0, B = cmake<C>((T)0, (T)0);
#pragma unroll
            for (int j = 1; j <= H; ++j) {
                const C w = ldroot<C>(&root[((j * d) % R) * step]);
                const T c = w.x, sn = -w.y;
                A = cmake<C>(fma(a[j - 1].x, c, A.x), fma(a[j - 1].y, c, A.y));
                B = cmake<C>(fma(b[j - 1].x, sn, B.x), fma(b[j - 1].y, sn, B.y));
            }
            const C iB = cmul_si<S>(B);  // S i B
            v[d] = cadd(A, iB);
            v[R - d] = csub(A, iB);
        }
    }
};
template <int S, typename C>
struct Dft<7, S, C> : DftGeneric<7, S, C> {};
template <int S, typename C>
struct Dft<11, S, C> : DftGeneric<11, S, C> {};
template <int S, typename C>
struct Dft<13, S, C> : DftGeneric<13, S, C> {};

// cos(2 pi m / R) and sin(2 pi m / R) for the composite radices (R = 6, 9, 10,
// 12; 0 < m < R, m not a quarter turn), as constants: m is a compile-time
// value wherever these are called (unrolled loops), so the switch folds away.
__device__ __forceinline__ double2 kcossin(int R, int m) {
    const bool neg = 2 * m > R;  // sin(2 pi (R - m) / R) = -sin(2 pi m / R)
    const int q = neg ? R - m : m;
    double c = 0.0, s = 0.0;
    if (R == 6 || (R == 12 && q == 2)) {  // 2 pi / 6
        c = 0.5;
        s = 0.86602540378443864676;
    }
    if ((R == 6 && q == 2) || (R == 9 && q == 3) || (R == 12 && q == 4)) {  // 2 pi / 3
        c = -0.5;
        s = 0.86602540378443864676;
    }
    if (R == 9) {
        if (q == 1) { c = 0.76604444311897803520; s = 0.64278760968653932632; }
        if (q == 2) { c = 0.17364817766693034885; s = 0.98480775301220805936; }
        if (q == 4) { c = -0.93969262078590838405; s = 0.34202014332566873304; }
    }
    if (R == 10) {
        if (q == 1) { c = 0.80901699437494742410; s = 0.58778525229247312917; }
        if (q == 2) { c = 0.30901699437494742410; s = 0.95105651629515357212; }
        if (q == 3) { c = -0.30901699437494742410; s = 0.95105651629515357212; }
        if (q == 4) { c = -0.80901699437494742410; s = 0.58778525229247312917; }
    }
    if (R == 12) {
        if (q == 1) { c = 0.86602540378443864676; s = 0.5; }
        if (q == 5) { c = -0.86602540378443864676; s = 0.5; }
    }
    return make_double2(c, neg ? -s : s);
}

// u * exp(S 2 pi i m / R) for the composite radices' inner twiddles; quarter
// turns are exact (a swap or a sign).
template <int R, int S, typename C>
__device__ __forceinline__ C kroot_mul(C u, int m) {
    using T = typename CplxT<C>::T;
    if ((4 * m) % R == 0) {
        const int k = (4 * m / R) & 3;
        if (k == 1) return cmul_si<S>(u);
        if (k == 2) return cmake<C>(-u.x, -u.y);
        return cmul_si<-S>(u);
    }
    const double2 w = kcossin(R, m);
    return cmul(u, cmake<C>((T)w.x, (T)(S * w.y)));
}

// Composite radix R = R1*R2 entirely in registers (four-step):
//   y[k1 + R1 k2] = sum_n2 W_R2^{n2 k2} W_R^{n2 k1} sum_n1 x[R2 n1 + n2] W_R1^{n1 k1}
// with W_R^m = exp(-2 pi i m / R) (conjugated for S = +1) from constants.
template <int R1, int R2, int S, typename C>
struct DftComposite {
    __device__ __forceinline__ static void run(C* v, const double2* root, int n) {
        constexpr int R = R1 * R2;
        // phase 1, in place: v[R2 k1 + n2] <- W_R^{n2 k1} DFT_R1(v[R2 n1 + n2])_k1
#pragma unroll
        for (int n2 = 0; n2 < R2; ++n2) {
            C u[R1];
#pragma unroll
            for (int n1 = 0; n1 < R1; ++n1) u[n1] = v[R2 * n1 + n2];
            Dft<R1, S, C>::run(u, root, n);
#pragma unroll
            for (int k1 = 0; k1 < R1; ++k1) {
                if (n2 * k1 == 0)
                    v[R2 * k1 + n2] = u[k1];
                else
                    v[R2 * k1 + n2] = kroot_mul<R, S>(u[k1], n2 * k1);
            }
        }
        // phase 2, in place: v[R2 k1 + k2] <- DFT_R2(v[R2 k1 + n2])_k2
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) Dft<R2, S, C>::run(v + R2 * k1, root, n);
        // y[k1 + R1 k2] = v[R2 k1 + k2]: a register permutation
        C y[R];
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1)
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2) y[k1 + R1 * k2] = v[R2 * k1 + k2];
#pragma unroll
        for (int i = 0; i < R; ++i) v[i] = y[i];
    }
};
template <int S, typename C>
struct Dft<6, S, C> : DftComposite<2, 3, S, C> {};
template <int S, typename C>
struct Dft<9, S, C> : DftComposite<3, 3, S, C> {};
template <int S, typename C>
struct Dft<10, S, C> : DftComposite<2, 5, S, C> {};
template <int S, typename C>
struct Dft<12, S, C> : DftComposite<4, 3, S, C> {};

// w[d] = w1^d (conjugated when CONJ), d = 1 .. R-1, by binary powers: each
// entry is at most three products from w1
template <int R, bool CONJ, typename C>
__device__ __forceinline__ void twiddle_powers(C* w, C w1) {
    if (CONJ) w1.y = -w1.y;
    w[1] = w1;
#pragma unroll
    for (int d = 2; d < R; ++d) {
        const int hi = (d & 1) ? d - 1 : d / 2;  // d = hi + lo with lo = 1 (odd d) or hi (even d)
        const int lo = d - hi;
        w[d] = cmul(w[hi], w[lo]);
    }
}

// One radix-R butterfly in registers: DIF (FWD) or DIT, with the stage
// twiddles of butterfly position a (a = 0: none).
template <int R, bool FWD, typename C>
__device__ __forceinline__ void butterfly_R(C* v, int a, int tw_step, int n, const double2* __restrict__ root) {
    constexpr int S = FWD ? -1 : +1;
    if (FWD) {
        Dft<R, S, C>::run(v, root, n);
        if (a != 0) {
            C w[R];
            twiddle_powers<R, false>(w, ldroot<C>(&root[a * tw_step]));
#pragma unroll
            for (int d = 1; d < R; ++d) v[d] = cmul(v[d], w[d]);
        }
    } else {
        if (a != 0) {
            C w[R];
            twiddle_powers<R, true>(w, ldroot<C>(&root[a * tw_step]));
#pragma unroll
            for (int d = 1; d < R; ++d) v[d] = cmul(v[d], w[d]);
        }
        Dft<R, S, C>::run(v, root, n);
    }
}

// One radix-R stage over every line of axis `ax` of the NBUF planes that
// start at `buf[0]`, `buf[0] + bufstride`, ...  DIF when FWD, DIT otherwise.
// BT > 1: a thread takes BT butterflies at once (tasks t, t + T, ...), loads
// all of them before the first DFT and stores after the last, so their
// shared-memory latencies overlap (butterflies of one stage touch disjoint
// elements, so the reordering is safe).
template <int R, bool FWD, int NBUF, typename C, int BT = 1>
__device__ __forceinline__ void stage_R(C* buf, int bufstride, int Nk, const AxisPlan& ax, int s,
                                        const double2* __restrict__ root) {
    const int n = ax.n;
    const int inner = ax.inner;
    const int L = ax.L[s];
    const int M = L * R;
    const int nbfly = n / R;
    const int tw_step = n / M;
    const int ntask = Nk / R;
    const FastDiv fdi = ax.fd_inner, fdb = ax.fd_nbfly[s], fdl = ax.fd_L[s];
    const int step = L * inner;
    if constexpr (BT == 1) {
        for (int t = threadIdx.x; t < ntask; t += blockDim.x) {
            const int tmp = fdiv(t, fdi);
            const int in = t - tmp * inner;
            const int o = fdiv(tmp, fdb);
            const int bfly = tmp - o * nbfly;
            const int blk = fdiv(bfly, fdl);
            const int a = bfly - blk * L;
            const int base = o * (n * inner) + in + (blk * M + a) * inner;
#pragma unroll
            for (int q = 0; q < NBUF; ++q) {
                C* X = buf + q * bufstride;
                C v[R];
#pragma unroll
                for (int b = 0; b < R; ++b) v[b] = X[base + b * step];
                butterfly_R<R, FWD, C>(v, a, tw_step, n, root);
#pragma unroll
                for (int b = 0; b < R; ++b) X[base + b * step] = v[b];
            }
        }
    } else {
        for (int t0 = threadIdx.x; t0 < ntask; t0 += BT * blockDim.x) {
            int base[BT], av[BT];
            bool on[BT];
#pragma unroll
            for (int j = 0; j < BT; ++j) {
                const int t = t0 + j * (int)blockDim.x;
                on[j] = t < ntask;
                const int tt = on[j] ? t : t0;
                const int tmp = fdiv(tt, fdi);
                const int in = tt - tmp * inner;
                const int o = fdiv(tmp, fdb);
                const int bfly = tmp - o * nbfly;
                const int blk = fdiv(bfly, fdl);
                av[j] = bfly - blk * L;
                base[j] = o * (n * inner) + in + (blk * M + av[j]) * inner;
            }
#pragma unroll
            // a task past the end repeats task t0's loads and arithmetic and
            // stores nothing: no branch inside the batch
            for (int q = 0; q < NBUF; ++q) {
                C* X = buf + q * bufstride;
                C v[BT][R];
#pragma unroll
                for (int j = 0; j < BT; ++j)
#pragma unroll
                    for (int b = 0; b < R; ++b) v[j][b] = X[base[j] + b * step];
#pragma unroll
                for (int j = 0; j < BT; ++j) butterfly_R<R, FWD, C>(v[j], av[j], tw_step, n, root);
#pragma unroll
                for (int j = 0; j < BT; ++j)
                    if (on[j]) {
#pragma unroll
                        for (int b = 0; b < R; ++b) X[base[j] + b * step] = v[j][b];
                    }
            }
        }
    }
}

// Radix sets a plane kernel may be specialised for (bit r set = radix r):
// every radix; the common ones (the generic odd radices 11 and 13 need many
// registers, and plans without them run kernels compiled without them); the
// 72-point axes.
constexpr int kRadixCommon = (1 << 2) | (1 << 3) | (1 << 4) | (1 << 5) | (1 << 6) | (1 << 7) | (1 << 8) |
                             (1 << 9) | (1 << 10) | (1 << 12);
constexpr int kRadixAll = kRadixCommon | (1 << 11) | (1 << 13);
constexpr int kRadix89 = (1 << 8) | (1 << 9);

template <bool FWD, int NBUF, int MASK, typename C, int BT = 1>
__device__ __forceinline__ void run_stage(C* buf, int bufstride, int Nk, const AxisPlan& ax, int s,
                                          const double2* __restrict__ roots) {
    const double2* root = roots + ax.rootoff;
    const int r = ax.r[s];
    // only the radices of MASK are compiled in (the host never selects a
    // kernel lacking a radix of its plan)
#define EDUS_STAGE_CASE(R)                                                               \
    if constexpr ((MASK >> R) & 1) {                                                     \
        if (r == R) {                                                                    \
            stage_R<R, FWD, NBUF, C, BT>(buf, bufstride, Nk, ax, s, root);               \
            return;                                                                      \
        }                                                                                \
    }
    EDUS_STAGE_CASE(2)
    EDUS_STAGE_CASE(3)
    EDUS_STAGE_CASE(4)
    EDUS_STAGE_CASE(5)
    EDUS_STAGE_CASE(6)
    EDUS_STAGE_CASE(7)
    EDUS_STAGE_CASE(8)
    EDUS_STAGE_CASE(9)
    EDUS_STAGE_CASE(10)
    EDUS_STAGE_CASE(11)
    EDUS_STAGE_CASE(12)
    EDUS_STAGE_CASE(13)
#undef EDUS_STAGE_CASE
}

// Row-wise stages for 2-D planes (N2 = 1): the unit-stride axis ax[1] of
// rows line0 .. line0 + nl - 1 (each n1 = ax[1].n consecutive elements) in
// one warp, without a CTA barrier: the stages of that axis only touch the
// elements of a row, so a warp that owns whole rows runs them, and the
// pointwise steps between them, alone (__syncwarp between stages).  Lane l
// takes the row-local butterflies l, l + 32, ... in the order of stage_R.
template <int R, bool FWD>
__device__ __forceinline__ void stage_R_rows(double2* X, const AxisPlan& ax, int s, const double2* __restrict__ root,
                                             int line0, int nl) {
    const int n = ax.n;
    const int L = ax.L[s];
    const int M = L * R;
    const int nbfly = n / R;
    const int tw_step = n / M;
    const FastDiv fdb = ax.fd_nbfly[s], fdl = ax.fd_L[s];
    const int lane = threadIdx.x & 31;
    for (int i = lane; i < nl * nbfly; i += 32) {
        const int li = fdiv(i, fdb);
        const int bfly = i - li * nbfly;
        const int blk = fdiv(bfly, fdl);
        const int a = bfly - blk * L;
        const int base = (line0 + li) * n + blk * M + a;
        double2 v[R];
#pragma unroll
        for (int b = 0; b < R; ++b) v[b] = X[base + b * L];
        butterfly_R<R, FWD, double2>(v, a, tw_step, n, root);
#pragma unroll
        for (int b = 0; b < R; ++b) X[base + b * L] = v[b];
    }
}

template <bool FWD, int MASK>
__device__ __forceinline__ void run_stage_rows(double2* X, const AxisPlan& ax, int s, const double2* __restrict__ roots,
                                               int line0, int nl) {
    const double2* root = roots + ax.rootoff;
    const int r = ax.r[s];
#define EDUS_ROWS_CASE(R)                                            \
    if constexpr ((MASK >> R) & 1) {                                 \
        if (r == R) {                                                \
            stage_R_rows<R, FWD>(X, ax, s, root, line0, nl);         \
            return;                                                  \
        }                                                            \
    }
    EDUS_ROWS_CASE(2)
    EDUS_ROWS_CASE(3)
    EDUS_ROWS_CASE(4)
    EDUS_ROWS_CASE(5)
    EDUS_ROWS_CASE(6)
    EDUS_ROWS_CASE(7)
    EDUS_ROWS_CASE(8)
    EDUS_ROWS_CASE(9)
    EDUS_ROWS_CASE(10)
    EDUS_ROWS_CASE(11)
    EDUS_ROWS_CASE(12)
    EDUS_ROWS_CASE(13)
#undef EDUS_ROWS_CASE
}

// The ax[1] part of plane_forward (FWD) or plane_inverse for the warp's rows.
template <bool FWD, int MASK>
__device__ __forceinline__ void rows_transform(double2* X, const PlanePlan& pl, const double2* __restrict__ roots,
                                               int line0, int nl) {
    const AxisPlan& ax = pl.ax[1];
    if (FWD) {
#pragma unroll 1
        for (int s = 0; s < ax.nst; ++s) {
            run_stage_rows<true, MASK>(X, ax, s, roots, line0, nl);
            __syncwarp();
        }
    } else {
#pragma unroll 1
        for (int s = ax.nst - 1; s >= 0; --s) {
            run_stage_rows<false, MASK>(X, ax, s, roots, line0, nl);
            __syncwarp();
        }
    }
}

// The ax[0] part of plane_forward (FWD) or plane_inverse, CTA-wide, each stage
// followed by a CTA barrier.
template <bool FWD, int MASK>
__device__ __forceinline__ void axis0_transform(double2* X, const PlanePlan& pl, const double2* __restrict__ roots) {
    const AxisPlan& ax = pl.ax[0];
    if (FWD) {
#pragma unroll 1
        for (int s = 0; s < ax.nst; ++s) {
            run_stage<true, 1, MASK, double2>(X, 0, pl.Nk, ax, s, roots);
            __syncthreads();
        }
    } else {
#pragma unroll 1
        for (int s = ax.nst - 1; s >= 0; --s) {
            run_stage<false, 1, MASK, double2>(X, 0, pl.Nk, ax, s, roots);
            __syncthreads();
        }
    }
}

// Forward (k -> R, unnormalised sign -1) transform of the plane(s) in place.
template <int NBUF, int MASK, typename C, int BT = 1>
__device__ __forceinline__ void plane_forward(C* buf, int bufstride, const PlanePlan& pl, const double2* __restrict__ roots) {
#pragma unroll 1
    for (int d = 0; d < 3; ++d) {
        const AxisPlan& ax = pl.ax[d];
#pragma unroll 1
        for (int s = 0; s < ax.nst; ++s) {
            run_stage<true, NBUF, MASK, C, BT>(buf, bufstride, pl.Nk, ax, s, roots);
            __syncthreads();
        }
    }
}

// Inverse (R -> k, unnormalised sign +1) transform, exact reverse of plane_forward.
template <int NBUF, int MASK, typename C, int BT = 1>
__device__ __forceinline__ void plane_inverse(C* buf, int bufstride, const PlanePlan& pl, const double2* __restrict__ roots) {
#pragma unroll 1
    for (int d = 2; d >= 0; --d) {
        const AxisPlan& ax = pl.ax[d];
#pragma unroll 1
        for (int s = ax.nst - 1; s >= 0; --s) {
            run_stage<false, NBUF, MASK, C, BT>(buf, bufstride, pl.Nk, ax, s, roots);
            __syncthreads();
        }
    }
}

}  // namespace edus
