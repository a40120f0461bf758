// Kernels of the packed-Hermitian forms (EDUS_PREC_HERM64, EDUS_PREC_MIXED).
//
// The density matrix stays Hermitian when H is, so only the band pairs n <= m
// (Pq = nb (nb+1)/2 "packed planes") are stored and transformed.  The state
// is split rho = rho_ref + delta around a fixed reference (the first state the
// caller sets); with H_ee linear in rho,
//
//   f(rho) = C0 + sum_d E_d K_d + G(delta) - i ( [A, delta] + [E1, rho_ref] )
//   E1     = H_ee,lin(delta)          (-W delta(R), Hartree of delta_nn(R=0))
//   A      = H0' + E.xi + E1,   H0' = H0 + H_ee(rho_ref)
//   C0     = f(rho_ref; E = 0),  K_d = f(rho_ref; E = e_d) - C0
//
// C0, K_d and H0' come from the FP64 full-plane kernels, once.  Everything
// evaluated per right-hand side is then either proportional to delta or to E,
// so storing it in FP32 (EDUS_PREC_MIXED) costs accuracy relative to those
// small quantities only; the state delta, the RK accumulator, the AB history
// and C0, K_d stay FP64, and the matrix products run in FP64 (warp MMAs).
// Packed plane q <-> (n, m), n <= m, row-major over the upper triangle.
#pragma once
#include "kernels.cuh"

namespace edus {

template <typename C>
__device__ __forceinline__ C to_c(double2 v) {
    return cmake<C>((typename CplxT<C>::T)v.x, (typename CplxT<C>::T)v.y);
}
template <typename C>
__device__ __forceinline__ C to_c(float2 v) {
    return cmake<C>((typename CplxT<C>::T)v.x, (typename CplxT<C>::T)v.y);
}
__device__ __forceinline__ double2 to_d(double2 v) { return v; }
__device__ __forceinline__ double2 to_d(float2 v) { return make_double2(v.x, v.y); }

// ---------------------------------------------------------------------------
// Packed plane kernel: one CTA per (packed plane q, solve b).
//   delta(R) = FFT_{-1}(delta_k)/Nk;  G = FFT_{+1}(i (R.E) delta(R));
//   E1(R)   = -W delta(R) (Fock part, HSEX);  E1 = FFT_{+1}(E1(R));
//   delta_nn(R=0) of diagonal planes -> diag0 (Hartree part, added on the diagonal later).
// C is the arithmetic/storage type of the transform (float2 or double2), IT
// the type of the stage input.
template <typename C, typename IT, int MASK, int MAXT, bool COUL>
__global__ void __launch_bounds__(MAXT, (sizeof(C) == 8) ? 2 : 1) plane_packed_kernel(
    const IT* __restrict__ in, long long bstride_in, C* __restrict__ G_out, C* __restrict__ E1_out,
    long long bstride_out, const typename CplxT<C>::T* __restrict__ Wq, double2* __restrict__ diag0,
    const StageField* __restrict__ field, const double2* __restrict__ roots, const double* __restrict__ rpos,
    PlanePlan pl, const int* __restrict__ qnm, int nb, double inv_nk) {
    using T = typename CplxT<C>::T;
    extern __shared__ unsigned char smraw[];
    C* X = reinterpret_cast<C*>(smraw);
    C* Y = X + pl.Nk;
    const int Nk = pl.Nk;
    const int q = blockIdx.x, b = blockIdx.y;
    const int nm = qnm[q];
    const int n = nm >> 16, m = nm & 0xffff;
    const IT* src = in + (long long)b * bstride_in + (long long)q * Nk;
    for (int i = threadIdx.x; i < Nk; i += blockDim.x) X[i] = to_c<C>(src[i]);
    __syncthreads();
    plane_forward<1, MASK>(X, 0, pl, roots);
    const StageField F = field[b];
    if (COUL && n == m && threadIdx.x == 0) diag0[b * nb + n] = make_double2(X[0].x * inv_nk, X[0].y * inv_nk);
    __syncthreads();
    const int n1 = pl.ax[1].n, n2 = pl.ax[2].n;
    const double* rp0 = rpos + pl.ax[0].rposoff;
    const double* rp1 = rpos + pl.ax[1].rposoff;
    const double* rp2 = rpos + pl.ax[2].rposoff;
    const T* wq = Wq + (long long)q * Nk;
    const T inv = (T)inv_nk;
    for (int j = threadIdx.x; j < Nk; j += blockDim.x) {
        const int t = fdiv(j, pl.fd_n2);
        const int q2 = j - t * n2;
        const int q0 = fdiv(t, pl.fd_n1);
        const int q1 = t - q0 * n1;
        const T dot = (T)(F.g[0] * __ldg(&rp0[q0]) + F.g[1] * __ldg(&rp1[q1]) + F.g[2] * __ldg(&rp2[q2]));
        const C r = cscale(X[j], inv);
        X[j] = cmake<C>(-dot * r.y, dot * r.x);
        if (COUL) {
            const T w = __ldg(&wq[j]);
            Y[j] = cmake<C>(-w * r.x, -w * r.y);
        }
    }
    __syncthreads();
    plane_inverse<1, MASK>(X, 0, pl, roots);
    if (COUL) plane_inverse<1, MASK>(Y, 0, pl, roots);
    C* gdst = G_out + (long long)b * bstride_out + (long long)q * Nk;
    for (int i = threadIdx.x; i < Nk; i += blockDim.x) gdst[i] = X[i];
    if (COUL) {
        C* edst = E1_out + (long long)b * bstride_out + (long long)q * Nk;
        for (int i = threadIdx.x; i < Nk; i += blockDim.x) edst[i] = Y[i];
    }
}

// ---------------------------------------------------------------------------
// Packed commutator (FP64 warp MMAs).  Per k point four Hermitian matrices are
// rebuilt in shared memory from their packed planes, as split re/im FP64
// tiles [nbp][pitch]: A, D = delta, E1, Rf = rho_ref.  Only the 8x8 output
// tiles on or above the diagonal are computed (C is anti-Hermitian), and only
// n <= m is written.
struct PackedArgs {
    const void* in;        // stage input delta_s, [B][Pq][Nk] (IT)
    const void* G;         // [B][Pq][Nk] (ST)
    const void* E1;        // [B][Pq][Nk] (ST)
    const void* H0p;       // [Pq][Nk] (ST)  H0 + H_ee(rho_ref)
    const void* xi[3];     // [Pq][Nk] (ST)
    const void* Rref;      // [Pq][Nk] (ST)
    const double2* C0;     // [Pq][Nk]
    const double2* K[3];   // [Pq][Nk]
    const double2* hartree;  // [nb][nb]
    const double2* diag0;    // [B][nb] delta_nn(R=0)
    const StageField* field; // [B]
    const int* qnm;          // [Pq]
    double2* y;              // delta, FP64 [B][Pq][Nk]
    void* aux;               // next stage input (IT of stages 2-4)
    double2* acc;            // RK accumulator, FP64
    double2* out;            // MODE_RHS
    double2* hist[5];        // AB history, FP64
    double c[5];
    int order;
    long long bstride;       // Pq*Nk
    int Nk, nb, Pq, TK;
};

struct PackedGeom {
    int TK, nbp, pitch, tiles, warps_per_k;
    size_t smem;
};

__host__ __device__ inline PackedGeom packed_geometry(int nb) {
    PackedGeom g;
    g.nbp = (nb + 7) & ~7;
    g.pitch = g.nbp + 4;
    g.tiles = g.nbp / 8;
    const int nup = g.tiles * (g.tiles + 1) / 2;
    const size_t per_k = 8 * (size_t)g.nbp * g.pitch * 8;
    g.TK = 1;
    for (int tk = 8; tk >= 1; tk /= 2) {
        const int wpk = 8 / tk;
        if (tk * per_k <= 100 * 1024 && (nup + wpk - 1) / wpk <= 8) {
            g.TK = tk;
            break;
        }
    }
    g.warps_per_k = 8 / g.TK;
    g.smem = g.TK * per_k + (size_t)nb * 16;
    return g;
}

template <typename T>
__device__ __forceinline__ double2 ld2(const T* p, long long i) {
    return to_d(__ldg(reinterpret_cast<const T*>(p) + i));
}

// ST: storage type of the model and intermediate planes; IT: type of the
// stage input (the FP64 state at RK stage 1 and for AB); AT: type of the RK
// stage input written for the next stage.
template <int MODE, bool COUL, typename ST, typename IT, typename AT>
__global__ void __launch_bounds__(256, 2) commutator_packed_kernel(PackedArgs a) {
    extern __shared__ double smd[];
    const int nb = a.nb, Nk = a.Nk, Pq = a.Pq;
    const PackedGeom g = packed_geometry(nb);
    const int TK = g.TK, nbp = g.nbp, pitch = g.pitch;
    const int mat = nbp * pitch;
    double* tiles = smd;  // [TK][8][nbp][pitch]: Ar Ai Dr Di Er Ei Rr Ri
    double2* hh = (double2*)(smd + (size_t)TK * 8 * mat);
    double2* Cs = (double2*)smd;  // [Pq][TK] after the products
    const int b = blockIdx.y;
    const int k0 = blockIdx.x * TK;
    const long long boff = (long long)b * a.bstride;
    const StageField F = a.field[b];
    for (int i = threadIdx.x; i < TK * 8 * mat; i += blockDim.x) tiles[i] = 0.0;
    if (COUL) {
        for (int n = threadIdx.x; n < nb; n += blockDim.x) {
            double2 s = make_double2(0.0, 0.0);
            for (int m = 0; m < nb; ++m) s = cadd(s, cmul(a.hartree[n * nb + m], a.diag0[b * nb + m]));
            hh[n] = s;
        }
    }
    __syncthreads();
    const bool e0 = F.E[0] != 0.0, e1 = F.E[1] != 0.0, e2 = F.E[2] != 0.0;
    const ST* H0p = reinterpret_cast<const ST*>(a.H0p);
    const ST* Rref = reinterpret_cast<const ST*>(a.Rref);
    const ST* E1g = reinterpret_cast<const ST*>(a.E1);
    const IT* ing = reinterpret_cast<const IT*>(a.in);
    const int total = Pq * TK;
    constexpr int U = 2;
    for (int base = threadIdx.x; base < total; base += U * blockDim.x) {
        double2 dv[U], hv[U], x0[U], x1[U], x2[U], ev[U], rv[U];
        bool ok[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int idx = base + u * blockDim.x;
            const int q = idx / TK, kk = idx - (idx / TK) * TK;
            ok[u] = idx < total && k0 + kk < Nk;
            if (ok[u]) {
                const long long e = (long long)q * Nk + k0 + kk;
                dv[u] = ld2(ing, boff + e);
                hv[u] = ld2(H0p, e);
                rv[u] = ld2(Rref, e);
                if (e0) x0[u] = ld2(reinterpret_cast<const ST*>(a.xi[0]), e);
                if (e1) x1[u] = ld2(reinterpret_cast<const ST*>(a.xi[1]), e);
                if (e2) x2[u] = ld2(reinterpret_cast<const ST*>(a.xi[2]), e);
                ev[u] = COUL ? ld2(E1g, boff + e) : make_double2(0.0, 0.0);
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (!ok[u]) continue;
            const int idx = base + u * blockDim.x;
            const int q = idx / TK, kk = idx - (idx / TK) * TK;
            const int nm = a.qnm[q];
            const int i = nm >> 16, j = nm & 0xffff;
            double2 e1v = ev[u];
            if (COUL && i == j) e1v = cadd(e1v, hh[i]);
            double2 av = hv[u];
            if (e0) { av.x += F.E[0] * x0[u].x; av.y += F.E[0] * x0[u].y; }
            if (e1) { av.x += F.E[1] * x1[u].x; av.y += F.E[1] * x1[u].y; }
            if (e2) { av.x += F.E[2] * x2[u].x; av.y += F.E[2] * x2[u].y; }
            av = cadd(av, e1v);
            double* Tt = tiles + (size_t)kk * 8 * mat;
            const double2 vals[4] = {av, dv[u], e1v, rv[u]};
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                Tt[(2 * w) * mat + i * pitch + j] = vals[w].x;
                Tt[(2 * w + 1) * mat + i * pitch + j] = vals[w].y;
                if (i != j) {
                    Tt[(2 * w) * mat + j * pitch + i] = vals[w].x;
                    Tt[(2 * w + 1) * mat + j * pitch + i] = -vals[w].y;
                }
            }
        }
    }
    __syncthreads();
    // C = A D - D A + E1 Rf - Rf E1 on the upper 8x8 tiles
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kk = warp / g.warps_per_k, part = warp - kk * g.warps_per_k;
    const int T = g.tiles;
    const int nup = T * (T + 1) / 2;
    const int per = (nup + g.warps_per_k - 1) / g.warps_per_k;
    const int t0 = part * per, t1 = min(nup, t0 + per);
    constexpr int MAXT = 8;
    double cr[MAXT][2], ci[MAXT][2];
    int tij[MAXT];
#pragma unroll
    for (int t = 0; t < MAXT; ++t) {
        cr[t][0] = cr[t][1] = ci[t][0] = ci[t][1] = 0.0;
        // upper-triangle tile number -> (ti, tj), ti <= tj
        int tt = t0 + t, ti = 0;
        while (tt >= T - ti && ti < T) {
            tt -= T - ti;
            ++ti;
        }
        tij[t] = (ti << 8) | (ti + tt);
    }
    const double* Ar = tiles + (size_t)kk * 8 * mat;
    const double* Ai = Ar + mat;
    const double* Dr = Ar + 2 * mat;
    const double* Di = Ar + 3 * mat;
    const double* Er = Ar + 4 * mat;
    const double* Ei = Ar + 5 * mat;
    const double* Rr = Ar + 6 * mat;
    const double* Ri = Ar + 7 * mat;
    const int ar = lane >> 2, ac = lane & 3;
    if (kk < TK && k0 + kk < Nk) {
        for (int ks = 0; ks < nbp / 4; ++ks) {
            const int kc = ks * 4 + ac;
#pragma unroll
            for (int t = 0; t < MAXT; ++t) {
                if (t0 + t < t1) {
                    const int ti = tij[t] >> 8, tj = tij[t] & 0xff;
                    const int arow = ti * 8 + ar, bcol = tj * 8 + ar;
                    const int ao = arow * pitch + kc, bo = kc * pitch + bcol;
                    // A D - D A
                    double xr = Ar[ao], xi = Ai[ao], yr = Dr[bo], yi = Di[bo];
                    dmma(cr[t][0], cr[t][1], xr, yr);
                    dmma(cr[t][0], cr[t][1], -xi, yi);
                    dmma(ci[t][0], ci[t][1], xr, yi);
                    dmma(ci[t][0], ci[t][1], xi, yr);
                    xr = Dr[ao]; xi = Di[ao]; yr = Ar[bo]; yi = Ai[bo];
                    dmma(cr[t][0], cr[t][1], -xr, yr);
                    dmma(cr[t][0], cr[t][1], xi, yi);
                    dmma(ci[t][0], ci[t][1], -xr, yi);
                    dmma(ci[t][0], ci[t][1], -xi, yr);
                    if (COUL) {
                        // E1 Rf - Rf E1
                        xr = Er[ao]; xi = Ei[ao]; yr = Rr[bo]; yi = Ri[bo];
                        dmma(cr[t][0], cr[t][1], xr, yr);
                        dmma(cr[t][0], cr[t][1], -xi, yi);
                        dmma(ci[t][0], ci[t][1], xr, yi);
                        dmma(ci[t][0], ci[t][1], xi, yr);
                        xr = Rr[ao]; xi = Ri[ao]; yr = Er[bo]; yi = Ei[bo];
                        dmma(cr[t][0], cr[t][1], -xr, yr);
                        dmma(cr[t][0], cr[t][1], xi, yi);
                        dmma(ci[t][0], ci[t][1], -xr, yi);
                        dmma(ci[t][0], ci[t][1], -xi, yr);
                    }
                }
            }
        }
    }
    __syncthreads();  // all fragments read: Cs may overwrite the tiles
    if (kk < TK) {
#pragma unroll
        for (int t = 0; t < MAXT; ++t) {
            if (t0 + t < t1) {
                const int ti = tij[t] >> 8, tj = tij[t] & 0xff;
                const int row = ti * 8 + ar;
#pragma unroll
                for (int qq = 0; qq < 2; ++qq) {
                    const int col = tj * 8 + ac * 2 + qq;
                    if (row < nb && col < nb && row <= col) {
                        // packed index of (row, col), row <= col
                        const int qi = row * nb - (row * (row - 1)) / 2 + (col - row);
                        Cs[qi * TK + kk] = make_double2(cr[t][qq], ci[t][qq]);
                    }
                }
            }
        }
    }
    __syncthreads();
    // epilogue: f = C0 + sum_d E_d K_d + G - i C, then the stage update
    const ST* Gg = reinterpret_cast<const ST*>(a.G);
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int q = idx / TK, kq = idx - (idx / TK) * TK;
        const int k = k0 + kq;
        if (k >= Nk) continue;
        const long long e = (long long)q * Nk + k;
        const double2 c = Cs[idx];
        const double2 gg = ld2(Gg, boff + e);
        double2 f = __ldg(&a.C0[e]);
        if (e0) { const double2 kv = __ldg(&a.K[0][e]); f.x += F.E[0] * kv.x; f.y += F.E[0] * kv.y; }
        if (e1) { const double2 kv = __ldg(&a.K[1][e]); f.x += F.E[1] * kv.x; f.y += F.E[1] * kv.y; }
        if (e2) { const double2 kv = __ldg(&a.K[2][e]); f.x += F.E[2] * kv.x; f.y += F.E[2] * kv.y; }
        f.x += gg.x + c.y;
        f.y += gg.y - c.x;
        {
            // the generator is Hermitian: a diagonal f_nn is real, and its
            // imaginary part is rounding (FP32 in the mixed form) that would
            // otherwise accumulate in rho_nn
            const int nm = __ldg(&a.qnm[q]);
            if ((nm >> 16) == (nm & 0xffff)) f.y = 0.0;
        }
        const long long es = boff + e;
        AT* auxp = reinterpret_cast<AT*>(a.aux);
        if (MODE == MODE_RHS) {
            a.out[es] = f;
        } else if (MODE == MODE_RK1) {
            const double2 yv = a.y[es];
            const double2 av = make_double2(yv.x + a.c[0] * f.x, yv.y + a.c[0] * f.y);
            auxp[es] = to_c<AT>(av);
            a.acc[es] = make_double2(yv.x + a.c[1] * f.x, yv.y + a.c[1] * f.y);
        } else if (MODE == MODE_RK2 || MODE == MODE_RK3) {
            const double2 yv = a.y[es];
            const double2 ac2 = a.acc[es];
            const double2 av = make_double2(yv.x + a.c[0] * f.x, yv.y + a.c[0] * f.y);
            auxp[es] = to_c<AT>(av);
            a.acc[es] = make_double2(ac2.x + a.c[1] * f.x, ac2.y + a.c[1] * f.y);
        } else if (MODE == MODE_RK4) {
            const double2 ac2 = a.acc[es];
            a.y[es] = make_double2(ac2.x + a.c[0] * f.x, ac2.y + a.c[0] * f.y);
        } else if (MODE == MODE_AB) {
            a.hist[0][es] = f;
            double2 yv = a.y[es];
            yv = make_double2(yv.x + a.c[0] * f.x, yv.y + a.c[0] * f.y);
            for (int qh = 1; qh < a.order; ++qh) {
                const double2 fq = a.hist[qh][es];
                yv = make_double2(yv.x + a.c[qh] * fq.x, yv.y + a.c[qh] * fq.y);
            }
            a.y[es] = yv;
        }
    }
}

// ---------------------------------------------------------------------------
// Set-up and conversion kernels of the packed forms.

// dst[q][k] = (ST) src[p(q)][k] for the packed planes of a full [P][Nk] array
template <typename ST>
__global__ void pack_planes(const double2* __restrict__ src, ST* __restrict__ dst, const int* __restrict__ qnm,
                            int nb, int Pq, int Nk) {
    const long long total = (long long)Pq * Nk;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(i / Nk), k = (int)(i - (long long)q * Nk);
        const int nm = qnm[q];
        const int p = (nm >> 16) * nb + (nm & 0xffff);
        dst[i] = to_c<ST>(src[(long long)p * Nk + k]);
    }
}

// real scalar planes (W)
template <typename T>
__global__ void pack_scalar_planes(const double* __restrict__ src, T* __restrict__ dst, const int* __restrict__ qnm,
                                   int nb, int Pq, int Nk) {
    const long long total = (long long)Pq * Nk;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(i / Nk), k = (int)(i - (long long)q * Nk);
        const int nm = qnm[q];
        const int p = (nm >> 16) * nb + (nm & 0xffff);
        dst[i] = (T)src[(long long)p * Nk + k];
    }
}

// delta[q][k] = rho[p(q)][k] - ref[p(q)][k]  (full FP64 planes -> packed FP64)
__global__ void pack_delta(const double2* __restrict__ rho, const double2* __restrict__ ref, double2* __restrict__ delta,
                           const int* __restrict__ qnm, int nb, int Pq, int Nk) {
    const long long total = (long long)Pq * Nk;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(i / Nk), k = (int)(i - (long long)q * Nk);
        const int nm = qnm[q];
        const long long e = (long long)((nm >> 16) * nb + (nm & 0xffff)) * Nk + k;
        delta[i] = csub(rho[e], ref[e]);
    }
}

// rho[p][k] = ref[p][k] + delta of (n, m) (n <= m) or its conjugate (n > m)
__global__ void unpack_delta(const double2* __restrict__ delta, const double2* __restrict__ ref, double2* __restrict__ rho,
                             int nb, int Nk) {
    const int P = nb * nb;
    const long long total = (long long)P * Nk;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(i / Nk), k = (int)(i - (long long)p * Nk);
        const int n = p / nb, m = p - (p / nb) * nb;
        const int lo = n < m ? n : m, hi = n < m ? m : n;
        const int q = lo * nb - (lo * (lo - 1)) / 2 + (hi - lo);
        double2 d = delta[(long long)q * Nk + k];
        if (n > m) d.y = -d.y;
        rho[i] = cadd(ref[i], d);
    }
}

// out = a - b (full FP64 planes)
__global__ void sub_planes(const double2* __restrict__ a, const double2* __restrict__ b, double2* __restrict__ out,
                           long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = csub(a[i], b[i]);
}

// H0' = H0 + H_ee(rho_ref): Fock part from the plain plane kernel (Hee) and
// the Hartree shift of rho_ref on the diagonal.
__global__ void assemble_h0p(const double2* __restrict__ H0, const double2* __restrict__ Hee, double2* __restrict__ out,
                             const double2* __restrict__ hartree, const double2* __restrict__ diag0,
                             const double2* __restrict__ rho0diag, int nb, int Nk, int coul) {
    const int P = nb * nb;
    const long long total = (long long)P * Nk;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(i / Nk);
        double2 h = H0[i];
        if (coul) {
            h = cadd(h, Hee[i]);
            const int n = p / nb;
            if (p == n * nb + n) {
                double2 s = make_double2(0.0, 0.0);
                for (int m = 0; m < nb; ++m) s = cadd(s, cmul(hartree[n * nb + m], csub(diag0[m], rho0diag[m])));
                h = cadd(h, s);
            }
        }
        out[i] = h;
    }
}

}  // namespace edus
