// Persistent, TMA-fed commutator for the fused-Hamiltonian HSEX path
// (12 <= nb <= 24): the same contract as commutator_mma_kernel with FH = true
// (Hee holds H0 + E.xi + Hee; the Hartree diagonal hh is added here).
//
// Each CTA walks tiles of TK = 2 consecutive k points (t = blockIdx.x,
// blockIdx.x + gridDim.x, ...).  Every operand of a tile (the H and rho
// blocks, and G, y, acc of the stage update) is one TMA tensor copy: the
// plane-major array [B][P][Nk] complex is described as the 4-D tensor
// {2 Nk doubles, nb (m), nb (n), B} and the box {2 TK, nb, nb, 1} lands the
// tile as [n][m][kk] complex in shared memory.  While the FP64 tensor-core
// products (mma.sync m8n8k4) of tile t run, the copies of tile t + gridDim.x
// fill the other half of a double buffer, their completion counted by one
// mbarrier per half.  The products give C = H rho - rho H; the Hartree shift
// D = diag(hh) adds (D rho - rho D)_nm = (hh_n - hh_m) rho_nm.  C is staged as
// [p][TK] and the epilogue writes TK*16-byte segments of each plane.
//
// Rows and columns beyond nb (the 8x8 tiles cover nbp = nb rounded up to 8)
// are not in shared memory: the fragment loads return zero for them.  A wait
// on an mbarrier gives up after a bounded number of polls: the CTA then sets
// *status, waits (bounded again) for its copies in flight and returns, and the
// host reports EDUS_ERR_TIMEOUT.
// Reference: BlockMatrix_definitions.hpp:203-226 (commutator),
// Coulomb.cpp:151-159 (Hartree), DESolver.hpp:154-220 (stage updates).
#pragma once
#include <cuda.h>
#include "kernels.cuh"

namespace edus {

struct PipeGeom {
    int TK, nbp, tiles, warps, epi;
    size_t arr_elems;  // complex numbers of one operand block [P][TK]
    size_t arr_bytes;  // its shared-memory footprint, a 128-byte multiple
    size_t buf_bytes;  // one half of the double buffer (5 operand blocks)
    size_t smem;
};

inline bool pipe_supported(int nb) { return nb >= 12 && nb <= 24; }

__host__ __device__ inline PipeGeom pipe_geometry(int nb) {
    PipeGeom g;
    g.TK = 2;
    g.nbp = (nb + 7) & ~7;
    g.tiles = g.nbp / 8;
    g.warps = g.TK * g.tiles * g.tiles;  // one (k, 8x8 tile) job per warp: 8 or 18 warps
    const int threads = g.warps * 32;
    g.epi = (nb * nb * g.TK + threads - 1) / threads;
    g.arr_elems = (size_t)nb * nb * g.TK;
    g.arr_bytes = (g.arr_elems * 16 + 127) & ~(size_t)127;
    g.buf_bytes = 5 * g.arr_bytes;
    // alignment slack, two halves, the staged result [P][TK], hh [nb], two mbarriers
    g.smem = 128 + 2 * g.buf_bytes + g.arr_bytes + (size_t)nb * 16 + 16;
    return g;
}

// Operand tensor maps of one launch (H, rho, G, y, acc), each describing a
// [B][P][Nk] complex array as {2 Nk, nb, nb, B} doubles with box {2 TK, nb, nb, 1}.
struct PipeMaps {
    CUtensorMap m[5];
};

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// true once the phase of parity `parity` has completed; false after `limit` polls
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int limit) {
    for (int i = 0; i < limit; ++i) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int b, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(0), "r"(0), "r"(b), "r"(smem_u32(bar))
        : "memory");
}

template <int MODE, int EPI, int NT>
__global__ void __launch_bounds__(NT, 1)
    commutator_pipe_kernel(StageArgs a, int nbatch, const __grid_constant__ PipeMaps maps, int* status) {
    extern __shared__ unsigned char sraw[];
    const int nb = a.nb, Nk = a.Nk, P = nb * nb;
    const PipeGeom g = pipe_geometry(nb);
    constexpr int TK = 2;
    const int tiles = g.tiles, nbp = g.nbp;
    const size_t arr_bytes = g.arr_bytes;
    unsigned char* base = (unsigned char*)(((unsigned long long)sraw + 127) & ~127ull);
    double2* Cs = (double2*)(base + 2 * g.buf_bytes);                  // [P][TK]
    double2* hh = (double2*)(base + 2 * g.buf_bytes + arr_bytes);      // [nb]
    unsigned long long* bar = (unsigned long long*)(hh + nb);          // [2]
    const int ntk = (Nk + TK - 1) / TK;
    const int ntiles = ntk * nbatch;
    constexpr bool NEED_Y = MODE == MODE_RK1 || MODE == MODE_RK2 || MODE == MODE_RK3 || MODE == MODE_AB;
    constexpr bool NEED_A = MODE == MODE_RK2 || MODE == MODE_RK3 || MODE == MODE_RK4;
    const unsigned tx_bytes = (unsigned)(g.arr_elems * 16) * (3 + (NEED_Y ? 1 : 0) + (NEED_A ? 1 : 0));
    constexpr int kWaitPolls = 1 << 22;

    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    // thread 0 issues every copy of tile t into half h
    auto issue = [&](int t, int h) {
        const int b = t / ntk, k0 = (t - b * ntk) * TK;
        unsigned char* dst = base + h * g.buf_bytes;
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx(&bar[h], tx_bytes);
        const int x = 2 * k0;  // in doubles: 32-byte aligned since k0 is even
        tma_load_4d(dst, &maps.m[0], x, b, &bar[h]);
        tma_load_4d(dst + arr_bytes, &maps.m[1], x, b, &bar[h]);
        tma_load_4d(dst + 2 * arr_bytes, &maps.m[2], x, b, &bar[h]);
        if (NEED_Y) tma_load_4d(dst + 3 * arr_bytes, &maps.m[3], x, b, &bar[h]);
        if (NEED_A) tma_load_4d(dst + 4 * arr_bytes, &maps.m[4], x, b, &bar[h]);
    };

    int pend[2] = {-1, -1};  // thread 0: parity of the phase a pending copy completes
    int t = blockIdx.x;
    if (threadIdx.x == 0 && t < ntiles) {
        issue(t, 0);
        pend[0] = 0;
    }
    int last_b = -1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ar = lane >> 2, ac = lane & 3;
    const double2 zero = make_double2(0.0, 0.0);
    for (int it = 0; t < ntiles; t += gridDim.x, ++it) {
        const int half = it & 1;
        if (threadIdx.x == 0 && t + (int)gridDim.x < ntiles) {
            issue(t + gridDim.x, half ^ 1);
            pend[half ^ 1] = ((it + 1) >> 1) & 1;
        }
        const int b = t / ntk, k0 = (t - b * ntk) * TK;
        const long long boff = (long long)b * a.bstride;
        if (b != last_b) {
            for (int n = threadIdx.x; n < nb; n += NT) {
                double2 s = zero;
                for (int m = 0; m < nb; ++m)
                    s = cadd(s, cmul(__ldg(&a.hartree[n * nb + m]),
                                     csub(__ldg(&a.diag0[b * nb + m]), __ldg(&a.rho0diag[m]))));
                hh[n] = s;
            }
            last_b = b;
        }
        // this half's copies complete its (it/2)-th phase
        const bool ok = mbar_wait(&bar[half], (unsigned)((it >> 1) & 1), kWaitPolls);
        if (__syncthreads_or(!ok)) {  // also makes hh of a new solve visible
            if (threadIdx.x == 0) {
                atomicOr(status, 1);
                for (int h = 0; h < 2; ++h)
                    if (pend[h] >= 0) mbar_wait(&bar[h], (unsigned)pend[h], kWaitPolls);
            }
            return;
        }
        if (threadIdx.x == 0) pend[half] = -1;

        const unsigned char* cur = base + half * g.buf_bytes;
        const double2* Hm = (const double2*)cur;
        const double2* Rm = (const double2*)(cur + arr_bytes);
        const double2* Gs = (const double2*)(cur + 2 * arr_bytes);
        const double2* Ys = (const double2*)(cur + 3 * arr_bytes);
        const double2* As = (const double2*)(cur + 4 * arr_bytes);

        // one job per warp: k point kk, output tile (ti, tj)
        const int kk = warp / (tiles * tiles), tt = warp - kk * tiles * tiles;
        const int ti = tt / tiles, tj = tt - (tt / tiles) * tiles;
        const int arow = ti * 8 + ar, bcol = tj * 8 + ar;
        double cr0 = 0.0, cr1 = 0.0, ci0 = 0.0, ci1 = 0.0;
        for (int ks = 0; ks < nbp / 4; ++ks) {
            const int kc = ks * 4 + ac;
            const bool aok = arow < nb && kc < nb;
            const bool bok = kc < nb && bcol < nb;
            const double2 ha = aok ? Hm[(arow * nb + kc) * TK + kk] : zero;
            const double2 qa = aok ? Rm[(arow * nb + kc) * TK + kk] : zero;
            const double2 rb = bok ? Rm[(kc * nb + bcol) * TK + kk] : zero;
            const double2 hb = bok ? Hm[(kc * nb + bcol) * TK + kk] : zero;
            // H rho
            dmma(cr0, cr1, ha.x, rb.x);
            dmma(cr0, cr1, -ha.y, rb.y);
            dmma(ci0, ci1, ha.x, rb.y);
            dmma(ci0, ci1, ha.y, rb.x);
            // - rho H
            dmma(cr0, cr1, -qa.x, hb.x);
            dmma(cr0, cr1, qa.y, hb.y);
            dmma(ci0, ci1, -qa.x, hb.y);
            dmma(ci0, ci1, -qa.y, hb.x);
        }
        // Hartree shift and staging of C as [p][TK]
        {
            const int row = arow;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int col = tj * 8 + ac * 2 + q;
                if (row < nb && col < nb) {
                    double2 c = make_double2(q ? cr1 : cr0, q ? ci1 : ci0);
                    const int idx = (row * nb + col) * TK + kk;
                    c = cadd(c, cmul(csub(hh[row], hh[col]), Rm[idx]));
                    Cs[idx] = c;
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < EPI; ++u) {
            const int idx = threadIdx.x + u * NT;
            const int p = idx >> 1, kq = idx & 1;
            if (idx >= P * TK || k0 + kq >= Nk) continue;
            const long long e = boff + (long long)p * Nk + k0 + kq;
            const double2 c = Cs[idx];
            const double2 gg = Gs[idx];
            const double2 f = make_double2(gg.x + c.y, gg.y - c.x);  // f = G - i C
            double2 yv = zero, av = zero;
            if (NEED_Y) yv = Ys[idx];
            if (NEED_A) av = As[idx];
            if (MODE == MODE_RHS) {
                a.out[e] = f;
            } else if (MODE == MODE_RK1) {
                a.aux[e] = make_double2(yv.x + a.c[0] * f.x, yv.y + a.c[0] * f.y);
                a.acc[e] = make_double2(yv.x + a.c[1] * f.x, yv.y + a.c[1] * f.y);
            } else if (MODE == MODE_RK2 || MODE == MODE_RK3) {
                a.aux[e] = make_double2(yv.x + a.c[0] * f.x, yv.y + a.c[0] * f.y);
                a.acc[e] = make_double2(av.x + a.c[1] * f.x, av.y + a.c[1] * f.y);
            } else if (MODE == MODE_RK4) {
                a.y[e] = make_double2(av.x + a.c[0] * f.x, av.y + a.c[0] * f.y);
            } else if (MODE == MODE_AB) {
                a.hist[0][e] = f;
                double2 yy = make_double2(yv.x + a.c[0] * f.x, yv.y + a.c[0] * f.y);
                for (int q = 1; q < a.order; ++q) {
                    const double2 fq = a.hist[q][e];
                    yy = make_double2(yy.x + a.c[q] * fq.x, yy.y + a.c[q] * fq.y);
                }
                a.y[e] = yy;
            }
        }
        // the next iteration's copies refill this half: every thread is done with it
        __syncthreads();
    }
}

}  // namespace edus
