// Warp-specialised, TMA-fed persistent commutator for the fused-Hamiltonian
// HSEX path (12 <= nb <= 24): the contract of commutator_mma_kernel with
// FH = true (Hee holds H0 + E.xi + Hee; the Hartree diagonal hh is added
// here), with the tensor-core products overlapping the stage update and the
// copies.
//
// A CTA walks update tiles of 4 consecutive k points (u = blockIdx.x,
// blockIdx.x + gridDim.x, ...), each made of two product tiles of 2 k points
// (h = 0, 1).  Four roles:
//   warp 0      copies H and rho of a product tile (TMA) and writes the Hartree
//               shifts hh of its solve into the same stage (lane n keeps hh_n
//               in a register, recomputed when the tile's solve changes: a dot
//               product per tile in this warp would stall the copies);
//   warp 1      copies G, y, acc of an update tile (TMA);
//   NM warps    products: a job is one 8x8 output tile (ti, tj) for both k
//               points of a product tile; job j of the CTA's stream
//               (j = warp, warp + NM, ...) belongs to product tile j / tiles^2,
//               so every warp has work in every tile and the four SM
//               sub-partitions get equal shares;
//   NE warps    the stage update of an update tile from G - i C, y, acc,
//               half by half (the 2 k points of one product tile at a time,
//               so a C slot is free again while the next products run).
// Hand-overs use mbarriers only (no CTA-wide barrier after set-up): SM stages
// of product operands (3 for nb <= 22, 2 above, 4 with 2x2 blocks), one
// update-operand stage and two staged-C slots (one per product tile of an
// update tile, each with its own full/empty pair).  The update operands of tile u + 1 stream in while the
// products of u + 1 run, so one stage hides their copy; their boxes have rows
// of 64 bytes (4 k points), which TMA moves at about 1.5x the rate of 32-byte
// rows.  Every wait gives up after
// a bounded number of polls; the warp then sets *status and returns, the others
// time out in turn, and the copy warps wait (bounded) for their copies in
// flight before returning.
//
// The product operands are copied as nb rows of W pairs of k points, W = nb
// or nb + 1, whichever is odd (the extra column is filled with zeros by the
// copy): the odd row length spreads the fragment loads over all banks once
// each lane loads both k points of its element in the order set by the parity
// of its row.  Fragment rows and columns beyond nb (the 8x8 tiles cover nb
// rounded up to 8) are not loaded: they read as zero.  Update operands are
// dense [P][4]; C is staged per product tile as [k point][row][CW] with CW odd
// and the k-point stride R = 4 (mod 8) 16-byte units, which keeps both the
// fragment-layout stores and the update warps' reads free of bank conflicts.  A product tile past the last k point (Nk = 1 mod 4) is copied
// as zeros and its results are not written.
//
// Each complex product is formed from three real ones,
//   Re(XY) = XrYr - XiYi,  Im(XY) = (Xr + Xi)(Yr + Yi) - XrYr - XiYi,
// so H rho - rho H takes six m8n8k4 per k step and k point instead of eight:
// A = Hr rr - qr hr, B = Hi ri - qi hi, D = (Hr + Hi)(rr + ri) - (qr + qi)(hr + hi)
// accumulate, and C = (A - B, D - A - B).  The rounding differs from the
// four-product form at the 1e-16 level of the operands' magnitudes.
// Reference: BlockMatrix_definitions.hpp:203-226 (commutator),
// Coulomb.cpp:151-159 (Hartree), DESolver.hpp:154-220 (stage updates).
#pragma once
#include "kernels.cuh"
#include "tma.cuh"

namespace edus {

struct WsGeom {
    int TK, TKU, nbp, tiles, W, NM, NE, warps, threads, jobs, SM;
    int CW, CR;           // staged C: row length (odd) and k-point stride (4 mod 8), complex units
    size_t mop_bytes;     // one product operand [nb][W][TK] complex, a 128-byte multiple
    size_t hh_off;        // Hartree shifts [nb] after H and rho
    size_t mstage_bytes;  // H, rho, hh
    size_t arr_bytes;     // one staged C [TK][nb][CW] (k-point stride CR), a 128-byte multiple
    size_t uarr_bytes;    // one update operand [P][TKU], a 128-byte multiple
    size_t off_e, off_c, off_bar, smem;
};

inline bool ws_supported(int nb) { return nb >= 12 && nb <= 24; }

constexpr size_t kWsSmemMax = 232448;  // shared memory a B200 CTA may opt in to

__host__ __device__ inline WsGeom ws_geometry(int nb) {
    WsGeom g;
    g.TK = 2;
    g.TKU = 4;
    g.nbp = (nb + 7) & ~7;
    g.tiles = g.nbp / 8;
    g.W = (nb & 1) ? nb : nb + 1;
    g.NM = g.tiles == 3 ? 8 : 4;
    g.NE = g.tiles == 3 ? 8 : 4;
    g.warps = 2 + g.NM + g.NE;
    g.threads = 32 * g.warps;
    g.jobs = g.tiles * g.tiles;
    g.mop_bytes = ((size_t)nb * g.W * g.TK * 16 + 127) & ~(size_t)127;
    g.hh_off = 2 * g.mop_bytes;
    g.mstage_bytes = g.hh_off + (((size_t)nb * 16 + 127) & ~(size_t)127);
    g.CW = (nb & 1) ? nb : nb + 1;
    g.CR = nb * g.CW + ((4 - nb * g.CW) & 7);
    g.arr_bytes = ((size_t)g.TK * g.CR * 16 + 127) & ~(size_t)127;
    g.uarr_bytes = ((size_t)nb * nb * g.TKU * 16 + 127) & ~(size_t)127;
    for (g.SM = g.tiles == 2 ? 4 : 3;; --g.SM) {
        g.off_e = g.SM * g.mstage_bytes;
        g.off_c = g.off_e + 3 * g.uarr_bytes;
        g.off_bar = g.off_c + 2 * g.arr_bytes;
        g.smem = 128 + g.off_bar + (2 * g.SM + 6) * 8;  // alignment slack, barriers
        if (g.smem <= kWsSmemMax || g.SM == 2) break;
    }
    return g;
}

template <int MODE, int TILES, int SM>
__global__ void __launch_bounds__(32 * (2 + 2 * (TILES == 3 ? 8 : 4)), 1)
    commutator_ws_kernel(StageArgs a, int nbatch, const __grid_constant__ OperandMaps maps, int* status) {
    extern __shared__ unsigned char sraw[];
    constexpr int TK = 2, TKU = 4;
    constexpr int NBP = 8 * TILES, JOBS = TILES * TILES;
    constexpr int NM = TILES == 3 ? 8 : 4, NE = NM;
    constexpr int kWaitPolls = 1 << 22;
    constexpr bool NEED_Y = MODE == MODE_RK1 || MODE == MODE_RK2 || MODE == MODE_RK3 || MODE == MODE_AB;
    constexpr bool NEED_A = MODE == MODE_RK2 || MODE == MODE_RK3 || MODE == MODE_RK4;
    const int nb = a.nb, Nk = a.Nk, P = nb * nb;
    const WsGeom g = ws_geometry(nb);
    const int W = g.W;
    unsigned char* base = (unsigned char*)(((unsigned long long)sraw + 127) & ~127ull);
    unsigned long long* bar = (unsigned long long*)(base + g.off_bar);
    unsigned long long* full_m = bar;            // [SM] product operands landed (1 arrival + bytes)
    unsigned long long* empty_m = bar + SM;      // [SM] product operands read (one arrival per job)
    unsigned long long* full_e = bar + 2 * SM;   // update operands landed
    unsigned long long* empty_e = full_e + 1;    // update operands read (one arrival per update warp)
    unsigned long long* full_c = full_e + 2;     // [2] C slot h staged (one arrival per job)
    unsigned long long* empty_c = full_e + 4;    // [2] C slot h read (one arrival per update warp)
    const int ntu = (Nk + TKU - 1) / TKU;   // update tiles per solve
    const int nut = ntu * nbatch;
    const int nit = (int)blockIdx.x < nut ? (nut - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < SM; ++s) {
            mbar_init(&full_m[s], 1);
            mbar_init(&empty_m[s], JOBS);
        }
        mbar_init(full_e, 1);
        mbar_init(empty_e, NE);
        for (int h = 0; h < 2; ++h) {
            mbar_init(&full_c[h], JOBS);
            mbar_init(&empty_c[h], NE);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    if (warp == 0) {
        // ---- product operands of product tile i = 2 j + h into stage i % SM
        const unsigned tx = (unsigned)((size_t)2 * nb * W * TK * 16);
        int issued = 0, last_b = -1;
        double2 hreg = make_double2(0.0, 0.0);
        bool ok = true;
        for (int i = 0; i < 2 * nit; ++i) {
            const int s = i % SM;
            if (i >= SM && !warp_wait(&empty_m[s], (unsigned)((i / SM - 1) & 1), kWaitPolls)) {
                ok = false;
                break;
            }
            const int u = blockIdx.x + (i >> 1) * gridDim.x;
            const int b = u / ntu, k0 = (u - b * ntu) * TKU + (i & 1) * TK;
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
                mbar_expect_tx(&full_m[s], tx);
                tma_load_4d(dst, &maps.m[0], 2 * k0, b, &full_m[s]);  // x in doubles: 32-byte aligned
                tma_load_4d(dst + g.mop_bytes, &maps.m[1], 2 * k0, b, &full_m[s]);
            }
            issued = i + 1;
        }
        if (!ok && lane == 0) atomicOr(status, 1);
        // wait for the last copy into each stage: no copy may land after the CTA ends
        for (int i = issued - 1; i >= 0 && i >= issued - SM; --i)
            mbar_wait(&full_m[i % SM], (unsigned)((i / SM) & 1), kWaitPolls);
        return;
    }

    if (warp == 1) {
        // ---- update operands of update tile j (one stage)
        const unsigned tx = (unsigned)((size_t)P * TKU * 16) * (1 + (NEED_Y ? 1 : 0) + (NEED_A ? 1 : 0));
        int issued = 0;
        bool ok = true;
        for (int j = 0; j < nit; ++j) {
            if (j >= 1 && !warp_wait(empty_e, (unsigned)((j - 1) & 1), kWaitPolls)) {
                ok = false;
                break;
            }
            const int u = blockIdx.x + j * gridDim.x;
            const int b = u / ntu, x = 2 * (u - b * ntu) * TKU;  // in doubles: 64-byte aligned
            if (lane == 0) {
                unsigned char* dst = base + g.off_e;
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                mbar_expect_tx(full_e, tx);
                tma_load_4d(dst, &maps.m[2], x, b, full_e);
                if (NEED_Y) tma_load_4d(dst + g.uarr_bytes, &maps.m[3], x, b, full_e);
                if (NEED_A) tma_load_4d(dst + 2 * g.uarr_bytes, &maps.m[4], x, b, full_e);
            }
            issued = j + 1;
        }
        if (!ok && lane == 0) atomicOr(status, 1);
        if (issued > 0) mbar_wait(full_e, (unsigned)((issued - 1) & 1), kWaitPolls);
        return;
    }

    if (warp < 2 + NM) {
        // ---- product warps
        const int mw = warp - 2;
        const int ar = lane >> 2, ac = lane & 3;
        const bool odd = ar & 1;
        const int k1 = odd ? 1 : 0;
        for (int jb = mw;; jb += NM) {
            const int i = jb / JOBS;  // product tile
            if (i >= 2 * nit) break;
            const int q = jb - i * JOBS;
            const int ti = q / TILES, tj = q - (q / TILES) * TILES;
            const int s = i % SM, j = i >> 1;
            if (!warp_wait(&full_m[s], (unsigned)((i / SM) & 1), kWaitPolls)) {
                if (lane == 0) atomicOr(status, 1);
                return;
            }
            const unsigned char* ms = base + s * g.mstage_bytes;
            const double2* Hm = (const double2*)ms;  // [nb][W][TK]
            const double2* Rm = (const double2*)(ms + g.mop_bytes);
            const double2* hh = (const double2*)(ms + g.hh_off);
            const int arow = ti * 8 + ar, bcol = tj * 8 + ar;
            // accumulators per k point: A = Re-Re, B = Im-Im, D = sum products
            double c0[2][3], c1[2][3];
#pragma unroll
            for (int kk = 0; kk < 2; ++kk)
#pragma unroll
                for (int r = 0; r < 3; ++r) c0[kk][r] = c1[kk][r] = 0.0;
#pragma unroll
            for (int ks = 0; ks < NBP / 4; ++ks) {
                const int kc = ks * 4 + ac;
                const bool aok = arow < nb && kc < nb, bok = kc < nb && bcol < nb;
                const int ao = aok ? (arow * W + kc) * TK : 0, bo = bok ? (kc * W + bcol) * TK : 0;
                const double2 zero = make_double2(0.0, 0.0);
                double2 hA[2], qA[2], rB[2], hB[2];
                {
                    const double2 u0 = aok ? Hm[ao + k1] : zero, u1 = aok ? Hm[ao + (k1 ^ 1)] : zero;
                    const double2 v0 = aok ? Rm[ao + k1] : zero, v1 = aok ? Rm[ao + (k1 ^ 1)] : zero;
                    const double2 w0 = bok ? Rm[bo + k1] : zero, w1 = bok ? Rm[bo + (k1 ^ 1)] : zero;
                    const double2 z0 = bok ? Hm[bo + k1] : zero, z1 = bok ? Hm[bo + (k1 ^ 1)] : zero;
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
                    dmma(c0[kk][0], c1[kk][0], ha.x, rb.x);
                    dmma(c0[kk][0], c1[kk][0], -qa.x, hb.x);
                    dmma(c0[kk][1], c1[kk][1], ha.y, rb.y);
                    dmma(c0[kk][1], c1[kk][1], -qa.y, hb.y);
                    dmma(c0[kk][2], c1[kk][2], ha.x + ha.y, rb.x + rb.y);
                    dmma(c0[kk][2], c1[kk][2], -(qa.x + qa.y), hb.x + hb.y);
                }
            }
            // this tile's C slot must have been read for the previous update tile
            if (j >= 1 && !warp_wait(&empty_c[i & 1], (unsigned)((j - 1) & 1), kWaitPolls)) {
                if (lane == 0) atomicOr(status, 1);
                return;
            }
            double2* Cs = (double2*)(base + g.off_c + (i & 1) * g.arr_bytes);
            const int row = arow;
#pragma unroll
            for (int qq = 0; qq < 2; ++qq) {
                const int col = tj * 8 + ac * 2 + qq;
                if (row < nb && col < nb) {
                    const double2 dh = csub(hh[row], hh[col]);
#pragma unroll
                    for (int kk = 0; kk < 2; ++kk) {
                        const double xa = qq ? c1[kk][0] : c0[kk][0], xb = qq ? c1[kk][1] : c0[kk][1];
                        const double xd = qq ? c1[kk][2] : c0[kk][2];
                        double2 c = make_double2(xa - xb, xd - xa - xb);
                        c = cadd(c, cmul(dh, Rm[(row * W + col) * TK + kk]));
                        Cs[kk * g.CR + row * g.CW + col] = c;
                    }
                }
            }
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&full_c[i & 1]);
                mbar_arrive(&empty_m[s]);
            }
        }
        return;
    }

    // ---- update warps: half h of update tile j, element (p, kk) at k0 + 2 h + kk
    const int ew = warp - 2 - NM;
    const double2 zero = make_double2(0.0, 0.0);
    const FastDiv fd_nb = {((1ull << 40) + (unsigned long long)nb - 1ull) / (unsigned long long)nb, nb};
    for (int j = 0; j < nit; ++j) {
        const unsigned par = (unsigned)(j & 1);
        const int u = blockIdx.x + j * gridDim.x;
        const int b = u / ntu, k0 = (u - b * ntu) * TKU;
        const long long boff = (long long)b * a.bstride;
        const unsigned char* es = base + g.off_e;
        const double2* Gs = (const double2*)es;  // [P][TKU]
        const double2* Ys = (const double2*)(es + g.uarr_bytes);
        const double2* As = (const double2*)(es + 2 * g.uarr_bytes);
        for (int h = 0; h < 2; ++h) {
            if (!warp_wait(&full_c[h], par, kWaitPolls) || (h == 0 && !warp_wait(full_e, par, kWaitPolls))) {
                if (lane == 0) atomicOr(status, 1);
                return;
            }
            const double2* Cs = (const double2*)(base + g.off_c + h * g.arr_bytes);  // [TK][nb][CW]
            for (int idx = ew * 32 + lane; idx < P * TK; idx += NE * 32) {
                const int p = idx >> 1, kk = idx & 1, kq = 2 * h + kk;
                if (k0 + kq >= Nk) continue;
                const long long e = boff + (long long)p * Nk + k0 + kq;
                const int eu = p * TKU + kq;  // in the update operands [P][TKU]
                const int row = fdiv(p, fd_nb), col = p - row * nb;
                const double2 c = Cs[kk * g.CR + row * g.CW + col];
                const double2 gg = Gs[eu];
                const double2 f = make_double2(gg.x + c.y, gg.y - c.x);  // f = G - i C
                double2 yv = zero, av = zero;
                if (NEED_Y) yv = Ys[eu];
                if (NEED_A) av = As[eu];
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
                    for (int qh = 1; qh < a.order; ++qh) {
                        const double2 fq = a.hist[qh][e];
                        yy = make_double2(yy.x + a.c[qh] * fq.x, yy.y + a.c[qh] * fq.y);
                    }
                    a.y[e] = yy;
                }
            }
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&empty_c[h]);
                if (h == 1) mbar_arrive(empty_e);
            }
        }
    }
}

}  // namespace edus
