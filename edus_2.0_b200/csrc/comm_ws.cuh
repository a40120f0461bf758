// Warp-specialised, TMA-fed persistent commutator for the fused-Hamiltonian
// HSEX path (12 <= nb <= 24): the contract of commutator_mma_kernel with
// FH = true (Hee holds H0 + E.xi + Hee; the Hartree diagonal hh is added
// here), with the
// tensor-core products of tile t overlapping the stage update of tile t - 1 and
// the copies of tiles t + 1, t + 2.
//
// A CTA walks tiles of TK = 2 consecutive k points (t = blockIdx.x,
// blockIdx.x + gridDim.x, ...) with four roles:
//   warp 0      copies H and rho of a tile (TMA) and writes the Hartree
//               shifts hh of its solve into the same stage (lane n keeps
//               hh_n in a register, recomputed when the tile's solve changes:
//               a dot product per tile in this warp would stall the copies);
//   warp 1      copies G, y, acc of a tile (TMA);
//   NM warps    products: a job is one 8x8 output tile (ti, tj) for both k
//               points; job j of the CTA's stream (j = warp, warp + NM, ...)
//               belongs to tile j / tiles^2, so every warp has work in every
//               tile and the four SM sub-partitions get equal shares;
//   NE warps    the stage update from G - i C, y, acc, written to HBM.
// Stages are double buffers handed over by mbarriers only (no CTA-wide
// barrier after set-up): full/empty pairs for the product operands, the
// update operands and the staged commutator C.  Every wait gives up after a
// bounded number of polls; the warp then sets *status and returns, the others
// time out in turn, and the copy warps wait (bounded) for their copies in
// flight before returning.
//
// The product operands are copied with a box wider than the matrix, rows of
// W = nbp + 1 pairs of k points and nbp rows (nbp = nb rounded up to 8): the
// copy fills the margin with zeros, so the 8x8 fragments need no bounds
// tests, and the odd row length spreads the fragment loads over all banks
// once each lane loads both k points of its element in the order set by the
// parity of its row.  The update operands and C are dense [P][TK] arrays.
//
// Per k step and k point the products are 8 m8n8k4 (H rho - rho H from real
// and imaginary parts).  Forming each complex product from three real ones
// (six per k step) gained 2% of this kernel's time: the copies, not the
// products, bound it.
// Reference: BlockMatrix_definitions.hpp:203-226 (commutator),
// Coulomb.cpp:151-159 (Hartree), DESolver.hpp:154-220 (stage updates).
#pragma once
#include "kernels.cuh"
#include "tma.cuh"

namespace edus {

constexpr int kWsStages = 2;

struct WsGeom {
    int TK, nbp, tiles, W, NM, NE, warps, threads, jobs;
    size_t mop_bytes;     // one product operand [nbp][W][TK] complex
    size_t hh_off;        // Hartree shifts [nb] after H and rho
    size_t mstage_bytes;  // H, rho, hh
    size_t arr_bytes;     // one dense [P][TK] block, a 128-byte multiple
    size_t estage_bytes;  // G, y, acc
    size_t off_e, off_c, off_bar, smem;
};

inline bool ws_supported(int nb) { return nb >= 12 && nb <= 24; }

__host__ __device__ inline WsGeom ws_geometry(int nb) {
    WsGeom g;
    g.TK = 2;
    g.nbp = (nb + 7) & ~7;
    g.tiles = g.nbp / 8;
    g.W = g.nbp + 1;
    g.NM = g.tiles == 3 ? 8 : 4;
    g.NE = g.tiles == 3 ? 8 : 4;
    g.warps = 2 + g.NM + g.NE;
    g.threads = 32 * g.warps;
    g.jobs = g.tiles * g.tiles;
    g.mop_bytes = (size_t)g.nbp * g.W * g.TK * 16;  // 24*25*32 = 19200, 16*17*32 = 8704: 128-byte multiples
    g.hh_off = 2 * g.mop_bytes;
    g.mstage_bytes = g.hh_off + (((size_t)nb * 16 + 127) & ~(size_t)127);
    g.arr_bytes = ((size_t)nb * nb * g.TK * 16 + 127) & ~(size_t)127;
    g.estage_bytes = 3 * g.arr_bytes;
    g.off_e = kWsStages * g.mstage_bytes;
    g.off_c = g.off_e + kWsStages * g.estage_bytes;
    g.off_bar = g.off_c + kWsStages * g.arr_bytes;
    g.smem = 128 + g.off_bar + 6 * kWsStages * 8;  // alignment slack, six barriers per stage
    return g;
}

template <int MODE, int TILES>
__global__ void __launch_bounds__(32 * (2 + 2 * (TILES == 3 ? 8 : 4)), 1)
    commutator_ws_kernel(StageArgs a, int nbatch, const __grid_constant__ OperandMaps maps, int* status) {
    extern __shared__ unsigned char sraw[];
    constexpr int TK = 2, S = kWsStages;
    constexpr int NBP = 8 * TILES, W = NBP + 1, JOBS = TILES * TILES;
    constexpr int NM = TILES == 3 ? 8 : 4, NE = NM;
    constexpr int kWaitPolls = 1 << 22;
    constexpr bool NEED_Y = MODE == MODE_RK1 || MODE == MODE_RK2 || MODE == MODE_RK3 || MODE == MODE_AB;
    constexpr bool NEED_A = MODE == MODE_RK2 || MODE == MODE_RK3 || MODE == MODE_RK4;
    const int nb = a.nb, Nk = a.Nk, P = nb * nb;
    const WsGeom g = ws_geometry(nb);
    unsigned char* base = (unsigned char*)(((unsigned long long)sraw + 127) & ~127ull);
    unsigned long long* bar = (unsigned long long*)(base + g.off_bar);
    unsigned long long* full_m = bar;           // product operands landed (1 arrival + bytes)
    unsigned long long* empty_m = bar + S;      // product operands read (one arrival per job)
    unsigned long long* full_e = bar + 2 * S;   // update operands landed
    unsigned long long* empty_e = bar + 3 * S;  // update operands read (one arrival per update warp)
    unsigned long long* full_c = bar + 4 * S;   // C staged (one arrival per job)
    unsigned long long* empty_c = bar + 5 * S;  // C read (one arrival per update warp)
    const int ntk = (Nk + TK - 1) / TK;
    const int ntiles = ntk * nbatch;
    const int nit = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full_m[s], 1);
            mbar_init(&empty_m[s], JOBS);
            mbar_init(&full_e[s], 1);
            mbar_init(&empty_e[s], NE);
            mbar_init(&full_c[s], JOBS);
            mbar_init(&empty_c[s], NE);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    if (warp < 2) {
        // ---- copy warps: warp 0 product operands (+ hh), warp 1 update operands
        const bool prod = warp == 0;
        unsigned long long* full = prod ? full_m : full_e;
        unsigned long long* empty = prod ? empty_m : empty_e;
        const unsigned tx = prod ? (unsigned)(2 * g.mop_bytes)
                                 : (unsigned)((size_t)P * TK * 16) * (1 + (NEED_Y ? 1 : 0) + (NEED_A ? 1 : 0));
        int issued = 0;
        int last_b = -1;
        double2 hreg = make_double2(0.0, 0.0);
        bool ok = true;
        for (int i = 0; i < nit; ++i) {
            const int s = i % S;
            if (i >= S && !warp_wait(&empty[s], (unsigned)((i / S - 1) & 1), kWaitPolls)) {
                ok = false;
                break;
            }
            const int t = blockIdx.x + i * gridDim.x;
            const int b = t / ntk, k0 = (t - b * ntk) * TK;
            const int x = 2 * k0;  // in doubles: 32-byte aligned since k0 is even
            if (prod) {
                unsigned char* dst = base + s * g.mstage_bytes;
                double2* hh = (double2*)(dst + g.hh_off);
                if (b != last_b) {
                    hreg = make_double2(0.0, 0.0);
                    if (lane < nb)
                        for (int m = 0; m < nb; ++m)
                            hreg = cadd(hreg, cmul(__ldg(&a.hartree[lane * nb + m]),
                                                   csub(__ldg(&a.diag0[b * nb + m]), __ldg(&a.rho0diag[m]))));
                    last_b = b;
                }
                if (lane < nb) hh[lane] = hreg;
                __syncwarp();
                if (lane == 0) {
                    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                    mbar_expect_tx(&full[s], tx);
                    tma_load_4d(dst, &maps.m[0], x, b, &full[s]);
                    tma_load_4d(dst + g.mop_bytes, &maps.m[1], x, b, &full[s]);
                }
            } else if (lane == 0) {
                unsigned char* dst = base + g.off_e + s * g.estage_bytes;
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                mbar_expect_tx(&full[s], tx);
                tma_load_4d(dst, &maps.m[2], x, b, &full[s]);
                if (NEED_Y) tma_load_4d(dst + g.arr_bytes, &maps.m[3], x, b, &full[s]);
                if (NEED_A) tma_load_4d(dst + 2 * g.arr_bytes, &maps.m[4], x, b, &full[s]);
            }
            issued = i + 1;
        }
        if (!ok && lane == 0) atomicOr(status, 1);
        // wait for the last copy into each stage: no copy may land after the CTA ends
        for (int i = issued - 1; i >= 0 && i >= issued - S; --i)
            mbar_wait(&full[i % S], (unsigned)((i / S) & 1), kWaitPolls);
        return;
    }

    if (warp < 2 + NM) {
        // ---- product warps
        const int mw = warp - 2;
        const int ar = lane >> 2, ac = lane & 3;
        const bool odd = ar & 1;
        const int k1 = odd ? 1 : 0;
        for (int j = mw;; j += NM) {
            const int i = j / JOBS;
            if (i >= nit) break;
            const int q = j - i * JOBS;
            const int ti = q / TILES, tj = q - (q / TILES) * TILES;
            const int s = i % S;
            if (!warp_wait(&full_m[s], (unsigned)((i / S) & 1), kWaitPolls)) {
                if (lane == 0) atomicOr(status, 1);
                return;
            }
            const unsigned char* ms = base + s * g.mstage_bytes;
            const double2* Hm = (const double2*)ms;  // [NBP][W][TK]
            const double2* Rm = (const double2*)(ms + g.mop_bytes);
            const double2* hh = (const double2*)(ms + g.hh_off);
            const int arow = ti * 8 + ar, bcol = tj * 8 + ar;
            // accumulators per k point: real and imaginary parts of the two C elements
            double c0[2][2], c1[2][2];
#pragma unroll
            for (int kk = 0; kk < 2; ++kk)
#pragma unroll
                for (int r = 0; r < 2; ++r) c0[kk][r] = c1[kk][r] = 0.0;
#pragma unroll
            for (int ks = 0; ks < NBP / 4; ++ks) {
                const int kc = ks * 4 + ac;
                const int ao = (arow * W + kc) * TK, bo = (kc * W + bcol) * TK;
                double2 hA[2], qA[2], rB[2], hB[2];
                {
                    const double2 u0 = Hm[ao + k1], u1 = Hm[ao + (k1 ^ 1)];
                    const double2 v0 = Rm[ao + k1], v1 = Rm[ao + (k1 ^ 1)];
                    const double2 w0 = Rm[bo + k1], w1 = Rm[bo + (k1 ^ 1)];
                    const double2 z0 = Hm[bo + k1], z1 = Hm[bo + (k1 ^ 1)];
                    hA[0] = odd ? u1 : u0;
                    hA[1] = odd ? u0 : u1;
                    qA[0] = odd ? v1 : v0;
                    qA[1] = odd ? v0 : v1;
                    rB[0] = odd ? w1 : w0;
                    rB[1] = odd ? w0 : w1;
                    hB[0] = odd ? z1 : z0;
                    hB[1] = odd ? z0 : z1;
                }
#pragma unroll
                for (int kk = 0; kk < 2; ++kk) {
                    const double2 ha = hA[kk], qa = qA[kk], rb = rB[kk], hb = hB[kk];
                    // H rho
                    dmma(c0[kk][0], c1[kk][0], ha.x, rb.x);
                    dmma(c0[kk][0], c1[kk][0], -ha.y, rb.y);
                    dmma(c0[kk][1], c1[kk][1], ha.x, rb.y);
                    dmma(c0[kk][1], c1[kk][1], ha.y, rb.x);
                    // - rho H
                    dmma(c0[kk][0], c1[kk][0], -qa.x, hb.x);
                    dmma(c0[kk][0], c1[kk][0], qa.y, hb.y);
                    dmma(c0[kk][1], c1[kk][1], -qa.x, hb.y);
                    dmma(c0[kk][1], c1[kk][1], -qa.y, hb.x);
                }
            }
            // the staged C of this tile's slot must have been read
            if (i >= S && !warp_wait(&empty_c[s], (unsigned)((i / S - 1) & 1), kWaitPolls)) {
                if (lane == 0) atomicOr(status, 1);
                return;
            }
            double2* Cs = (double2*)(base + g.off_c + s * g.arr_bytes);
            const int row = arow;
#pragma unroll
            for (int qq = 0; qq < 2; ++qq) {
                const int col = tj * 8 + ac * 2 + qq;
                if (row < nb && col < nb) {
                    const double2 dh = csub(hh[row], hh[col]);
#pragma unroll
                    for (int kk = 0; kk < 2; ++kk) {
                        double2 c = make_double2(qq ? c1[kk][0] : c0[kk][0], qq ? c1[kk][1] : c0[kk][1]);
                        c = cadd(c, cmul(dh, Rm[(row * W + col) * TK + kk]));
                        Cs[(row * nb + col) * TK + kk] = c;
                    }
                }
            }
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&full_c[s]);
                mbar_arrive(&empty_m[s]);
            }
        }
        return;
    }

    // ---- update warps
    const int ew = warp - 2 - NM;
    const double2 zero = make_double2(0.0, 0.0);
    for (int i = 0; i < nit; ++i) {
        const int s = i % S;
        const unsigned par = (unsigned)((i / S) & 1);
        if (!warp_wait(&full_c[s], par, kWaitPolls) || !warp_wait(&full_e[s], par, kWaitPolls)) {
            if (lane == 0) atomicOr(status, 1);
            return;
        }
        const int t = blockIdx.x + i * gridDim.x;
        const int b = t / ntk, k0 = (t - b * ntk) * TK;
        const long long boff = (long long)b * a.bstride;
        const unsigned char* es = base + g.off_e + s * g.estage_bytes;
        const double2* Gs = (const double2*)es;
        const double2* Ys = (const double2*)(es + g.arr_bytes);
        const double2* As = (const double2*)(es + 2 * g.arr_bytes);
        const double2* Cs = (const double2*)(base + g.off_c + s * g.arr_bytes);
        for (int idx = ew * 32 + lane; idx < P * TK; idx += NE * 32) {
            const int p = idx >> 1, kq = idx & 1;
            if (k0 + kq >= Nk) continue;
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
        __syncwarp();
        if (lane == 0) {
            mbar_arrive(&empty_c[s]);
            mbar_arrive(&empty_e[s]);
        }
    }
}

}  // namespace edus
