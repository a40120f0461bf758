// Device kernels of one right-hand-side evaluation and of the time steppers.
//
// HBM layout (all device arrays): plane-major, [batch][p][k] with p = n*nb+m
// the band pair and k the grid point, complex128 as double2.  A plane is one
// band pair over the whole grid (Nk contiguous complex numbers), so
//   * the plane kernel streams whole planes (one 16-byte vector per thread,
//     fully coalesced) into shared memory for the k<->R transforms, and
//   * the commutator kernel reads a tile of TK consecutive k of every plane:
//     TK*16-byte contiguous segments.
// R-space model arrays (W, rho0) are stored in the digit-reversed position
// order that the in-place forward FFT leaves (see fft_plane.cuh).
#pragma once
#include <cuda_runtime.h>
#include "fft_plane.cuh"
#include "tma.cuh"

namespace edus {

// Field of one solve at one stage: E (Cartesian, a.u.) and g = A^T E, so that
// R.E = g . R_crys for the Gamma-centred crystal coordinates R_crys.
struct StageField {
    double E[3];
    double g[3];
    double ga[3];  // Peierls gauge: A.R = ga . R_crys with A(t) the vector potential
};

// Peierls phases of one stage, per solve b and axis: tab[b * ntab + rposoff_d + q]
// = exp(i ga_d R_d(q)), R_d(q) the Gamma-centred coordinate of position q, so
// that exp(i A.R) = tab[q0] tab[q1] tab[q2] (Simulation.cpp:876-899).
__global__ void peierls_phase_kernel(const StageField* __restrict__ field, const double* __restrict__ rpos,
                                     PlanePlan pl, int ntab, double2* __restrict__ tab) {
    const StageField F = field[blockIdx.x];
    for (int d = 0; d < 3; ++d) {
        const int n = pl.ax[d].n, off = pl.ax[d].rposoff;
        for (int q = threadIdx.x; q < n; q += blockDim.x) {
            double sn, cs;
            sincos(F.ga[d] * rpos[off + q], &sn, &cs);
            tab[(long long)blockIdx.x * ntab + off + q] = make_double2(cs, sn);
        }
    }
}

// exp(i A.R) at plane position j from the per-axis tables of one solve
__device__ __forceinline__ double2 peierls_phase_at(const double2* __restrict__ tb, const PlanePlan& pl, int j) {
    const int t = fdiv(j, pl.fd_n2);
    const int q2 = j - t * pl.ax[2].n;
    const int q0 = fdiv(t, pl.fd_n1);
    const int q1 = t - q0 * pl.ax[1].n;
    return cmul(cmul(__ldg(&tb[pl.ax[0].rposoff + q0]), __ldg(&tb[pl.ax[1].rposoff + q1])),
                __ldg(&tb[pl.ax[2].rposoff + q2]));
}

// Peierls gauge, pointwise: rho(R) -> -W (rho(R) exp(-i A.R) - rho0) exp(+i A.R)
// in place (X holds Nk rho(R)); the gauge-shifted rho enters the self-energy
// and the Hamiltonian leaves with the phase (Functional_SourceTerm.hpp:31-44).
__device__ __forceinline__ void peierls_selfenergy(double2* X, const double2* __restrict__ r0p,
                                                   const double* __restrict__ wp, const double2* __restrict__ tb,
                                                   const PlanePlan& pl, double inv_nk) {
    for (int j = threadIdx.x; j < pl.Nk; j += blockDim.x) {
        const double2 e = peierls_phase_at(tb, pl, j);
        const double2 a = cmul(cscale(X[j], inv_nk), make_double2(e.x, -e.y));
        const double2 r0 = __ldg(&r0p[j]);
        const double wv = __ldg(&wp[j]);
        X[j] = cmul(make_double2(-wv * (a.x - r0.x), -wv * (a.y - r0.y)), e);
    }
}

// Fused Hamiltonian (HSEX only): the model part H0(R) + sum_d E_d xi_d(R) is
// added to the self-energy plane in R before its transform, as the reference
// assembles H in R (Simulation.cpp:296-349), so the plane kernel returns
// H_k = H0_k + E.xi_k + Hee_k and the commutator reads one Hamiltonian array.
// H0(R) and xi(R) of a tight-binding model live on a few lattice vectors: nS
// positions hpos[s] (digit-reversed plane order) with values
// hval[(d * P + p) * nS + s], d = 0 for H0 and 1 + axis for xi.
// In the Peierls gauge (tb != nullptr) the model term is added times its
// phase exp(i A.R) (Simulation.cpp:876-899); pl is read only then.
__device__ __forceinline__ void add_model_R(double2* X, const int* __restrict__ hpos,
                                            const double2* __restrict__ hval, int nS, int p, int P,
                                            const StageField& F, const double2* __restrict__ tb = nullptr,
                                            const PlanePlan* pl = nullptr) {
    for (int s = threadIdx.x; s < nS; s += blockDim.x) {
        const int pos = __ldg(&hpos[s]);
        double2 m = __ldg(&hval[(long long)p * nS + s]);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (F.E[d] != 0.0) {
                const double2 x = __ldg(&hval[((long long)(d + 1) * P + p) * nS + s]);
                m.x += F.E[d] * x.x;
                m.y += F.E[d] * x.y;
            }
        }
        double2 v = X[pos];
        if (tb) m = cmul(m, peierls_phase_at(tb, *pl, pos));
        v.x += m.x;
        v.y += m.y;
        X[pos] = v;
    }
}

// k -> R transform of whole planes (set-up of the fused Hamiltonian):
// dst[p][q] = FFT_{-1}(src[p])[q] / Nk in the digit-reversed position order q.
template <int MASK, int MAXT>
__global__ void __launch_bounds__(MAXT) plane_to_R_kernel(const double2* __restrict__ src, double2* __restrict__ dst,
                                                          const double2* __restrict__ roots, PlanePlan pl,
                                                          double inv_nk) {
    extern __shared__ double2 smem[];
    const int Nk = pl.Nk;
    const long long off = (long long)blockIdx.x * Nk;
    for (int i = threadIdx.x; i < Nk; i += blockDim.x) smem[i] = __ldg(&src[off + i]);
    __syncthreads();
    plane_forward<1, MASK>(smem, 0, pl, roots);
    for (int i = threadIdx.x; i < Nk; i += blockDim.x) dst[off + i] = cscale(smem[i], inv_nk);
}

// ---------------------------------------------------------------------------
// Plane kernel: one CTA per (band pair p, solve b).
//   rho_R  = FFT_{-1}(rho_k) / Nk                      (Operator::go_to_R)
//   G_R    = i (R.E) rho_R                             (kGradient R branch)
//   Hee_R  = -W (rho_R - rho0_R)                       (Coulomb Fock term)
//   G_k    = FFT_{+1}(G_R),  Hee_k = FFT_{+1}(Hee_R)   (Operator::go_to_k)
// and rho_nn(R=0) of diagonal planes is written to diag0 for the Hartree term.
// Reference: Functional_SourceTerm.hpp:15-50, kGradient_definitions.hpp:35-40,
// Coulomb.cpp:150-171, fftPair.cpp:89-107.
template <bool COUL, int MASK, int MAXT>
__global__ void __launch_bounds__(MAXT) plane_rhs_kernel(
    const double2* __restrict__ rho, long long batch_stride_in, double2* __restrict__ G_out,
    double2* __restrict__ Hee_out, long long batch_stride_out, const double2* __restrict__ rho0p,
    const double* __restrict__ Wp, double2* __restrict__ diag0, const StageField* __restrict__ field,
    const double2* __restrict__ roots, const double* __restrict__ rpos, PlanePlan pl, int nb, double inv_nk,
    const int* __restrict__ hpos, const double2* __restrict__ hval, int nS,
    const double2* __restrict__ ptab = nullptr, int ntab = 0) {
    extern __shared__ double2 smem[];
    const int Nk = pl.Nk;
    double2* X = smem;
    double2* Y = smem + Nk;
    const int p = blockIdx.x;
    const int b = blockIdx.y;
    if (ptab) {
        // Peierls gauge: no gradient term; H = (H0 + E.xi + Hee[rho e^{-iA.R}]) e^{iA.R}
        const double2* tb = ptab + (long long)b * ntab;
        const StageField F = field[b];
        double2* hdst = Hee_out + (long long)b * batch_stride_out + (long long)p * Nk;
        if (COUL) {
            const double2* src = rho + (long long)b * batch_stride_in + (long long)p * Nk;
            for (int i = threadIdx.x; i < Nk; i += blockDim.x) X[i] = __ldg(&src[i]);
            __syncthreads();
            plane_forward<1, MASK>(X, 0, pl, roots);
            const int n = p / nb, m = p - (p / nb) * nb;
            if (n == m && threadIdx.x == 0) diag0[b * nb + n] = cscale(X[0], inv_nk);
            __syncthreads();
            peierls_selfenergy(X, rho0p + (long long)p * Nk, Wp + (long long)p * Nk, tb, pl, inv_nk);
        } else {
            for (int i = threadIdx.x; i < Nk; i += blockDim.x) X[i] = make_double2(0.0, 0.0);
        }
        __syncthreads();
        if (nS > 0) {
            add_model_R(X, hpos, hval, nS, p, nb * nb, F, tb, &pl);
            __syncthreads();
        }
        plane_inverse<1, MASK>(X, 0, pl, roots);
        for (int i = threadIdx.x; i < Nk; i += blockDim.x) hdst[i] = X[i];
        return;
    }
    const double2* src = rho + (long long)b * batch_stride_in + (long long)p * Nk;
    for (int i = threadIdx.x; i < Nk; i += blockDim.x) X[i] = __ldg(&src[i]);
    __syncthreads();
    plane_forward<1, MASK>(X, 0, pl, roots);

    const StageField F = field[b];
    const int n = p / nb, m = p - (p / nb) * nb;
    if (COUL && n == m && threadIdx.x == 0) diag0[b * nb + n] = cscale(X[0], inv_nk);
    __syncthreads();  // X[0] is read above before being overwritten below
    const int n1 = pl.ax[1].n, n2 = pl.ax[2].n;
    const double* rp0 = rpos + pl.ax[0].rposoff;
    const double* rp1 = rpos + pl.ax[1].rposoff;
    const double* rp2 = rpos + pl.ax[2].rposoff;
    const double2* r0p = rho0p + (long long)p * Nk;
    const double* wp = Wp + (long long)p * Nk;
    for (int j = threadIdx.x; j < Nk; j += blockDim.x) {
        const int t = fdiv(j, pl.fd_n2);
        const int q2 = j - t * n2;
        const int q0 = fdiv(t, pl.fd_n1);
        const int q1 = t - q0 * n1;
        const double dot = F.g[0] * __ldg(&rp0[q0]) + F.g[1] * __ldg(&rp1[q1]) + F.g[2] * __ldg(&rp2[q2]);
        const double2 r = cscale(X[j], inv_nk);
        X[j] = make_double2(-dot * r.y, dot * r.x);
        if (COUL) {
            const double2 r0 = __ldg(&r0p[j]);
            const double w = __ldg(&wp[j]);
            Y[j] = make_double2(-w * (r.x - r0.x), -w * (r.y - r0.y));
        }
    }
    __syncthreads();
    if (COUL && nS > 0) {
        add_model_R(Y, hpos, hval, nS, p, nb * nb, F);
        __syncthreads();
    }
    // the two inverse transforms run one after the other (fewer live registers)
    plane_inverse<1, MASK>(X, 0, pl, roots);
    if (COUL) plane_inverse<1, MASK>(Y, 0, pl, roots);

    double2* gdst = G_out + (long long)b * batch_stride_out + (long long)p * Nk;
    for (int i = threadIdx.x; i < Nk; i += blockDim.x) gdst[i] = X[i];
    if (COUL) {
        double2* hdst = Hee_out + (long long)b * batch_stride_out + (long long)p * Nk;
        for (int i = threadIdx.x; i < Nk; i += blockDim.x) hdst[i] = Y[i];
    }
}

// ---------------------------------------------------------------------------
// Persistent single-buffer plane kernel: the same contract as plane_rhs_kernel
// with one plane (16 Nk bytes) of shared memory, so two CTAs share an SM and
// one CTA's transforms overlap the other's loads and stores.  Planes of 4096
// points and more come in, and G and H go out, by bulk copies that one thread
// issues; the next copy into the buffer waits for the previous store's reads.  CTA c works on
// planes w = c, c + gridDim.x, ... of the P x B planes.  With HSEX the two
// inverse transforms run in turn from one buffer; rho(R) survives the first
// in the CTA's own slot of `scratch` ([gridDim.x][Nk], written and read back
// by the same thread, so it stays in L2 and needs no fence).
//
// ROWS (2-D grids, N2 = 1, length gauge): warp w owns rows [w lpw, (w+1) lpw)
// of the unit-stride axis ax[1] and runs that axis's stages, the gradient's
// pointwise step, the self-energy pass and the model terms on them alone;
// only the ax[0] stages, which mix rows, are CTA-wide.  The arithmetic is the
// same as without ROWS, in the same order, so the results are bitwise equal;
// a plane then needs 9 CTA barriers instead of 16.
//
// HERM (with ROWS; the Hermitian-plane form): only the band pairs n <= m are
// transformed (upair[i] = n nb + m, nb (nb+1)/2 of them, nplanes = that times
// the solves); G and H of the pair (m, n) are written as the conjugates of
// those of (n, m).  That is the generator for Hermitian rho and H: exact for
// the reference's on odd grids, and its Hermitian part on even ones (the host
// gives the N/2 index coordinate 0 and symmetrises W, as for the packed forms).
template <bool COUL, int MASK, int MAXT, int BT = 1, bool ROWS = false, bool HERM = false>
__global__ void __launch_bounds__(MAXT, 2) plane_rhs_persist_kernel(
    const double2* __restrict__ rho, long long batch_stride_in, double2* __restrict__ G_out,
    double2* __restrict__ Hee_out, long long batch_stride_out, const double2* __restrict__ rho0p,
    const double* __restrict__ Wp, double2* __restrict__ diag0, const StageField* __restrict__ field,
    const double2* __restrict__ roots, const double* __restrict__ rpos, PlanePlan pl, int nb, double inv_nk,
    double2* __restrict__ scratch, int nplanes, const int* __restrict__ hpos, const double2* __restrict__ hval,
    int nS, const int* __restrict__ opos, const double2* __restrict__ oval, int nO,
    const double2* __restrict__ ptab = nullptr, int ntab = 0, int* status = nullptr, int wait_polls = 1 << 22,
    int nroot_s = 0, int nrpos_s = 0, const int* __restrict__ upair = nullptr) {
    static_assert(!HERM || ROWS, "the Hermitian-plane form runs the row-wise kernel");
    extern __shared__ double2 smem[];
    const int Nk = pl.Nk;
    const int P = nb * nb;
    double2* X = smem;
    // the plane arrives by bulk copies (one thread issues them, one instruction
    // per 32 KB), completion counted on the mbarrier after the plane
    unsigned long long* lbar = (unsigned long long*)(X + Nk);
    int nload = 0;
    // small planes load and store per thread: a bulk copy's fixed latency and the
    // barrier round trip cost more than they save there
    const bool bulk = Nk >= 4096;
    if (threadIdx.x == 0) {
        mbar_init(lbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    // the transform roots and the R coordinates, when the host found room for
    // them beside the plane (nroot_s > 0), are read from shared memory
    const double2* rt = roots;
    const double* rq = rpos;
    if (nroot_s > 0) {
        double2* sr = X + Nk + 1;
        double* sq = (double*)(sr + nroot_s);
        for (int i = threadIdx.x; i < nroot_s; i += blockDim.x) sr[i] = __ldg(&roots[i]);
        for (int i = threadIdx.x; i < nrpos_s; i += blockDim.x) sq[i] = __ldg(&rpos[i]);
        rt = sr;
        rq = sq;
    }
    __syncthreads();
    double2* slot = scratch + (long long)blockIdx.x * Nk;
    const int n1 = pl.ax[1].n, n2 = pl.ax[2].n;
    const double* rp0 = rq + pl.ax[0].rposoff;
    const double* rp1 = rq + pl.ax[1].rposoff;
    const double* rp2 = rq + pl.ax[2].rposoff;
    // ROWS: this warp's rows of the unit-stride axis
    const int lane = threadIdx.x & 31;
    const int lpw = (pl.ax[0].n + (int)(blockDim.x >> 5) - 1) / (int)(blockDim.x >> 5);
    const int line0 = (int)(threadIdx.x >> 5) * lpw;
    const int nl = max(0, min(lpw, pl.ax[0].n - line0));
    for (int w = blockIdx.x; w < nplanes; w += gridDim.x) {
        // the solves of one band-pair plane run side by side: rho0 and W, which
        // they share, come from HBM once and from L2 for the others
        const int nbat = nplanes / (HERM ? nb * (nb + 1) / 2 : P);
        const int pi = w / nbat, b = w - (w / nbat) * nbat;
        const int p = HERM ? __ldg(&upair[pi]) : pi;
        // HERM: the transposed pair, whose G and H are the conjugates
        const int pT = (p - (p / nb) * nb) * nb + p / nb;
        if (!ROWS && ptab) {
            // Peierls gauge: no gradient term, two transforms (one without
            // HSEX); H = (H0 + E.xi + Hee[rho e^{-iA.R}]) e^{iA.R}
            const double2* tb = ptab + (long long)b * ntab;
            const StageField F = field[b];
            if (COUL) {
                const double2* src = rho + (long long)b * batch_stride_in + (long long)p * Nk;
                for (int i = threadIdx.x; i < Nk; i += blockDim.x) X[i] = __ldg(&src[i]);
                __syncthreads();
                plane_forward<1, MASK, double2, BT>(X, 0, pl, rt);
                const int n = p / nb, m = p - (p / nb) * nb;
                if (n == m && threadIdx.x == 0) diag0[b * nb + n] = cscale(X[0], inv_nk);
                __syncthreads();
                peierls_selfenergy(X, rho0p + (long long)p * Nk, Wp + (long long)p * Nk, tb, pl, inv_nk);
            } else {
                for (int i = threadIdx.x; i < Nk; i += blockDim.x) X[i] = make_double2(0.0, 0.0);
            }
            __syncthreads();
            if (nS > 0) {
                add_model_R(X, hpos, hval, nS, p, P, F, tb, &pl);
                __syncthreads();
            }
            plane_inverse<1, MASK, double2, BT>(X, 0, pl, rt);
            double2* hdst = Hee_out + (long long)b * batch_stride_out + (long long)p * Nk;
            for (int i = threadIdx.x; i < Nk; i += blockDim.x) hdst[i] = X[i];
            __syncthreads();  // X is reloaded by the next plane
            continue;
        }
        const double2* src = rho + (long long)b * batch_stride_in + (long long)p * Nk;
        if (!bulk) {
            for (int i = threadIdx.x; i < Nk; i += blockDim.x) X[i] = __ldg(&src[i]);
            __syncthreads();
        } else {
            const unsigned bytes = (unsigned)Nk * 16u;
            if (threadIdx.x == 0) {
                bulk_wait_read();  // the previous plane's stores have left X
                mbar_expect_tx(lbar, bytes);
                for (unsigned off = 0; off < bytes; off += 32768u)
                    bulk_load((unsigned char*)X + off, (const unsigned char*)src + off, min(32768u, bytes - off),
                              lbar);
            }
            const bool ok = mbar_wait(lbar, (unsigned)(nload & 1), wait_polls);
            ++nload;
            if (__syncthreads_or(!ok)) {
                // give up: report, and let the copy land (and earlier stores
                // complete) before the CTA ends; these waits keep the full limit
                if (threadIdx.x == 0) {
                    if (status) atomicOr(status, 1);
                    mbar_wait(lbar, (unsigned)((nload - 1) & 1), 1 << 22);
                    bulk_wait_all();
                }
                return;
            }
        }
        const StageField F = field[b];
        if constexpr (ROWS) {
            axis0_transform<true, MASK>(X, pl, rt);
            rows_transform<true, MASK>(X, pl, rt, line0, nl);
            const int n = p / nb, m = p - (p / nb) * nb;
            double2* const dg = (COUL && n == m) ? diag0 + b * nb + n : nullptr;
            const double g2 = F.g[2] * rp2[0];
            for (int idx = lane; idx < nl * n1; idx += 32) {
                const int li = fdiv(idx, pl.fd_n1);
                const int q1 = idx - li * n1;
                const int q0 = line0 + li;
                const int j = q0 * n1 + q1;
                const double dot = F.g[0] * rp0[q0] + F.g[1] * rp1[q1] + g2;
                const double2 r = cscale(X[j], inv_nk);
                if (COUL) {
                    slot[j] = r;
                    if (j == 0 && dg) *dg = r;
                }
                X[j] = make_double2(-dot * r.y, dot * r.x);
            }
            __syncwarp();
            rows_transform<false, MASK>(X, pl, rt, line0, nl);
            __syncthreads();
            axis0_transform<false, MASK>(X, pl, rt);
        } else {
            plane_forward<1, MASK, double2, BT>(X, 0, pl, rt);
            const int n = p / nb, m = p - (p / nb) * nb;
            if (COUL && n == m && threadIdx.x == 0) diag0[b * nb + n] = cscale(X[0], inv_nk);
            __syncthreads();
            for (int j = threadIdx.x; j < Nk; j += blockDim.x) {
                const int t = fdiv(j, pl.fd_n2);
                const int q2 = j - t * n2;
                const int q0 = fdiv(t, pl.fd_n1);
                const int q1 = t - q0 * n1;
                const double dot = F.g[0] * rp0[q0] + F.g[1] * rp1[q1] + F.g[2] * rp2[q2];
                const double2 r = cscale(X[j], inv_nk);
                if (COUL) slot[j] = r;
                X[j] = make_double2(-dot * r.y, dot * r.x);
            }
            __syncthreads();
            plane_inverse<1, MASK, double2, BT>(X, 0, pl, rt);
        }
        double2* gdst = G_out + (long long)b * batch_stride_out + (long long)p * Nk;
        if (!bulk) {
            for (int i = threadIdx.x; i < Nk; i += blockDim.x) gdst[i] = X[i];
        } else {
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            __syncthreads();
            if (threadIdx.x == 0) {
                const unsigned bytes = (unsigned)Nk * 16u;
                for (unsigned off = 0; off < bytes; off += 32768u)
                    bulk_store((unsigned char*)gdst + off, (const unsigned char*)X + off, min(32768u, bytes - off));
                bulk_commit();
            }
        }
        if (HERM && pT != p) {
            // G of (m, n): the conjugate (reads of X beside the bulk store's)
            double2* gT = G_out + (long long)b * batch_stride_out + (long long)pT * Nk;
            for (int i = threadIdx.x; i < Nk; i += blockDim.x) {
                const double2 v = X[i];
                gT[i] = make_double2(v.x, -v.y);
            }
        }
        if (COUL) {
            if (bulk && threadIdx.x == 0) bulk_wait_read();
            __syncthreads();  // the store above has read X before it is refilled
            if (nO > 0) {
                // the Fock term is given (values on nO lattice vectors, zero elsewhere)
                for (int j = threadIdx.x; j < Nk; j += blockDim.x) X[j] = make_double2(0.0, 0.0);
                __syncthreads();
                for (int s2 = threadIdx.x; s2 < nO; s2 += blockDim.x)
                    X[__ldg(&opos[s2])] = __ldg(&oval[(long long)p * nO + s2]);
            } else {
                const double2* r0p = rho0p + (long long)p * Nk;
                const double* wp = Wp + (long long)p * Nk;
                // four positions per thread at once: their twelve global
                // loads are in flight together (ROWS: the warp's rows)
                constexpr int U = 4;
                const int T = ROWS ? 32 : (int)blockDim.x;
                const int jend = ROWS ? (line0 + nl) * n1 : Nk;
                int j = ROWS ? line0 * n1 + lane : (int)threadIdx.x;
                for (; j + (U - 1) * T < jend; j += U * T) {
                    double2 r[U], r0[U];
                    double wv[U];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        r[u] = slot[j + u * T];
                        r0[u] = __ldg(&r0p[j + u * T]);
                        wv[u] = __ldg(&wp[j + u * T]);
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u)
                        X[j + u * T] = make_double2(-wv[u] * (r[u].x - r0[u].x), -wv[u] * (r[u].y - r0[u].y));
                }
                for (; j < jend; j += T) {
                    const double2 r = slot[j];
                    const double2 r0 = __ldg(&r0p[j]);
                    const double wv = __ldg(&wp[j]);
                    X[j] = make_double2(-wv * (r.x - r0.x), -wv * (r.y - r0.y));
                }
            }
            if constexpr (ROWS) {
                if (nO > 0) __syncthreads();  // the CTA-wide scatter above is complete
                __syncwarp();                 // the warp's own self-energy stores
                // the model terms on this warp's rows (add_model_R restricted to them)
                for (int s2 = lane; s2 < nS; s2 += 32) {
                    const int pos = __ldg(&hpos[s2]);
                    if ((unsigned)(fdiv(pos, pl.fd_n1) - line0) >= (unsigned)nl) continue;
                    double2 mv = __ldg(&hval[(long long)p * nS + s2]);
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        if (F.E[d] != 0.0) {
                            const double2 x = __ldg(&hval[((long long)(d + 1) * P + p) * nS + s2]);
                            mv.x += F.E[d] * x.x;
                            mv.y += F.E[d] * x.y;
                        }
                    }
                    double2 v = X[pos];
                    v.x += mv.x;
                    v.y += mv.y;
                    X[pos] = v;
                }
                __syncwarp();
                rows_transform<false, MASK>(X, pl, rt, line0, nl);
                __syncthreads();
                axis0_transform<false, MASK>(X, pl, rt);
            } else {
                __syncthreads();
                if (nS > 0) {
                    add_model_R(X, hpos, hval, nS, p, P, F);
                    __syncthreads();
                }
                plane_inverse<1, MASK, double2, BT>(X, 0, pl, rt);
            }
            double2* hdst = Hee_out + (long long)b * batch_stride_out + (long long)p * Nk;
            if (!bulk) {
                for (int i = threadIdx.x; i < Nk; i += blockDim.x) hdst[i] = X[i];
            } else {
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                __syncthreads();
                if (threadIdx.x == 0) {
                    const unsigned bytes = (unsigned)Nk * 16u;
                    for (unsigned off = 0; off < bytes; off += 32768u)
                        bulk_store((unsigned char*)hdst + off, (const unsigned char*)X + off,
                                   min(32768u, bytes - off));
                    bulk_commit();
                }
            }
            if (HERM && pT != p) {
                double2* hT = Hee_out + (long long)b * batch_stride_out + (long long)pT * Nk;
                for (int i = threadIdx.x; i < Nk; i += blockDim.x) {
                    const double2 v = X[i];
                    hT[i] = make_double2(v.x, -v.y);
                }
            }
        }
        // X is reloaded by the next plane's bulk copy: order this thread's accesses first
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
    }
    if (threadIdx.x == 0) bulk_wait_all();
}

// Plane-kernel variants: the generic one (every radix, up to 512 threads) and
// one specialised for plans made of radices 8 and 9 (72-point axes), which
// fits up to 768 threads.  The thread count is chosen per plan so that the
// butterflies of each stage split into as few, as full, rounds as possible.
struct PlaneLaunch {
    int variant;  // 0 generic (common radices), 1 radix {8,9}, 2 generic with radix 11 or 13
    int threads;
    bool persist;  // persistent single-buffer kernel, two CTAs per SM
};

// The persistent radix-{8,9} plane kernel: most threads a CTA may have, and
// butterflies a thread takes at once in each transform stage.
constexpr int kPersist89Threads = 384;
constexpr int kPersist89Batch = 1;

inline PlaneLaunch plane_launch(const PlanePlan& pl) {
    bool only89 = true;
    for (int d = 0; d < 3; ++d)
        for (int s = 0; s < pl.ax[d].nst; ++s)
            if (pl.ax[d].r[s] != 8 && pl.ax[d].r[s] != 9) only89 = false;
    bool wide = false;
    for (int d = 0; d < 3; ++d)
        for (int s = 0; s < pl.ax[d].nst; ++s)
            if (pl.ax[d].r[s] == 11 || pl.ax[d].r[s] == 13) wide = true;
    PlaneLaunch L;
    L.variant = only89 ? 1 : (wide ? 2 : 0);
    // two single-plane CTAs per SM when a plane leaves room for a second one
    L.persist = (size_t)pl.Nk * 16 <= 110 * 1024;
    const int tmax = L.persist ? (only89 ? kPersist89Threads : 256) : (only89 ? 768 : 512);
    const int bt = (L.persist && only89) ? kPersist89Batch : 1;
    long best = -1;
    L.threads = tmax;
    for (int T = 128; T <= tmax; T += 32) {
        long cost = 0;
        for (int d = 0; d < 3; ++d)
            for (int s = 0; s < pl.ax[d].nst; ++s) {
                const int r = pl.ax[d].r[s];
                const long tasks = pl.Nk / r;
                cost += ((tasks + (long)bt * T - 1) / ((long)bt * T)) * (long)r * bt;
            }
        cost = cost * 4 + 3 * ((pl.Nk + T - 1) / T);  // stages (3 transforms) + load/pointwise/store
        if (best < 0 || cost <= best) {
            best = cost;
            L.threads = T;
        }
    }
    return L;
}

// ---------------------------------------------------------------------------
// Commutator kernel: one CTA per (tile of TK consecutive k, solve b).
//   H_k  = H0_k + sum_d E_d xi_d,k [+ Hee_k + diag(h)],
//          h_n = sum_m Hartree_nm (rho_mm(R=0) - rho0_mm(R=0))
//   f_k  = G_k - i (H_k rho_k - rho_k H_k)
// then the stage epilogue (mode):
//   MODE_RHS : out = f
//   MODE_RK1 : aux = y + h/2 f ; acc = y + h/6 f
//   MODE_RK2 : aux = y + h/2 f ; acc = acc + h/3 f
//   MODE_RK3 : aux = y + h f   ; acc = acc + h/3 f
//   MODE_RK4 : y   = acc + h/6 f
//   MODE_AB  : hist0 = f ; y = y + c0 f + c1 hist1 + ... (order terms, in sequence)
// Reference: BlockMatrix_definitions.hpp:203-226 (commutator), Simulation.cpp:335-347
// (H assembly), Coulomb.cpp:151-159 (Hartree), DESolver.hpp:154-220 (stages).
enum StageMode { MODE_RHS = 0, MODE_RK1 = 1, MODE_RK2 = 2, MODE_RK3 = 3, MODE_RK4 = 4, MODE_AB = 5 };

struct StageArgs {
    const double2* rho;   // stage input, [B][P][Nk]
    const double2* G;     // gradient term in k
    const double2* Hee;   // HSEX self-energy in k (COUL)
    const double2* H0;    // [P][Nk]
    const double2* xi[3]; // [P][Nk]
    const double2* hartree;    // [P]
    const double2* rho0diag;   // [nb]  rho0_nn(R=0)
    const double2* diag0;      // [B][nb] rho_nn(R=0) of the stage input
    const StageField* field;   // [B]
    double2* out;   // MODE_RHS
    double2* y;
    double2* aux;
    double2* acc;
    double2* hist[5];  // AB: hist[0] receives f, hist[i] holds f_{n-i}
    double c[5];       // AB: h*beta_i; RK: c[0] = stage coefficient for aux, c[1] for acc
    int order;
    long long bstride;  // P*Nk
    long long mstride;  // batch stride of H0 and xi: 0 (one model) or P*Nk (a model per solve)
    int Nk, nb, TK;
};

// Launch geometry of the commutator kernel (shared by every caller).
// Each thread computes 2x2 output tiles of one k point and holds at most two
// tiles in registers, so TK (k points per CTA) is the largest power of two
// with TK * tiles <= 2 * threads; threads is 256, or 512 when even TK = 1
// needs more.  Shared memory: H and rho tiles [TK][nbp][nbp+1] (nbp = nb
// rounded up to even; the odd row pitch spreads rows over the banks) and the
// Hartree shift [nb].  The commutator result is staged over the H tiles.
struct CommGeom {
    int TK, threads, nbp, ld;
    size_t smem;
};

__host__ __device__ inline CommGeom comm_geometry(int nb) {
    CommGeom g;
    g.nbp = (nb + 1) & ~1;
    g.ld = g.nbp + 1;
    const int ntile = (g.nbp / 2) * (g.nbp / 2);
    int tk = 64;
    while (tk > 1 && tk * ntile > 512) tk /= 2;
    while (tk > 1 && (2 * (size_t)tk * g.nbp * g.ld + nb) * 16 > 100 * 1024) tk /= 2;
    g.TK = tk;
    g.threads = (tk * ntile > 512) ? 512 : 256;
    g.smem = (2 * (size_t)tk * g.nbp * g.ld + nb) * 16;
    return g;
}

// Stage inputs of a (k tile, solve) into shared memory: H = H0 + sum_d E_d xi_d
// (+ Hee + Hartree diagonal) and rho, element (p, kk) handed to store(i, j, kk, h, r).
// Elements are taken U at a time with every global load issued before any is
// used, so that each thread keeps several loads in flight.
template <bool COUL, bool FH, typename Store>
__device__ __forceinline__ void load_stage_inputs(const StageArgs& a, const StageField& F, const double2* hh, int b,
                                                  int k0, Store store) {
    constexpr int U = 4;
    const int nb = a.nb, P = nb * nb, TK = a.TK, Nk = a.Nk;
    const long long boff = (long long)b * a.bstride;
    const int total = P * TK;
    // with the fused Hamiltonian (FH) the Hee array already holds H0 + E.xi + Hee
    const bool e0 = !FH && F.E[0] != 0.0, e1 = !FH && F.E[1] != 0.0, e2 = !FH && F.E[2] != 0.0;
    for (int base = threadIdx.x; base < total; base += U * blockDim.x) {
        double2 r[U], h[U], x0[U], x1[U], x2[U], he[U];
        long long el[U];
        bool ok[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int idx = base + u * blockDim.x;
            const int p = idx / TK, kk = idx - (idx / TK) * TK;
            ok[u] = idx < total && k0 + kk < Nk;
            el[u] = (long long)p * Nk + k0 + kk;
            if (ok[u]) {
                r[u] = __ldg(&a.rho[boff + el[u]]);
                const long long em = el[u] + (long long)b * a.mstride;
                if (!FH) h[u] = __ldg(&a.H0[em]);
                if (e0) x0[u] = __ldg(&a.xi[0][em]);
                if (e1) x1[u] = __ldg(&a.xi[1][em]);
                if (e2) x2[u] = __ldg(&a.xi[2][em]);
                if (COUL || FH) he[u] = __ldg(&a.Hee[boff + el[u]]);
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int idx = base + u * blockDim.x;
            if (idx >= total) continue;
            const int p = idx / TK, kk = idx - (idx / TK) * TK;
            const int i = p / nb, j = p - (p / nb) * nb;
            double2 hv = make_double2(0.0, 0.0), rv = make_double2(0.0, 0.0);
            if (ok[u]) {
                hv = FH ? make_double2(0.0, 0.0) : h[u];
                rv = r[u];
                if (e0) { hv.x += F.E[0] * x0[u].x; hv.y += F.E[0] * x0[u].y; }
                if (e1) { hv.x += F.E[1] * x1[u].x; hv.y += F.E[1] * x1[u].y; }
                if (e2) { hv.x += F.E[2] * x2[u].x; hv.y += F.E[2] * x2[u].y; }
                if (COUL || FH) hv = cadd(hv, he[u]);
                if (COUL && i == j) hv = cadd(hv, hh[i]);
            }
            store(i, j, kk, hv, rv);
        }
    }
}

// f = G - i C from the staged commutator Cs [P][TK], then the stage update,
// U elements at a time with all loads issued first.
template <int MODE>
__device__ __forceinline__ void stage_epilogue(const StageArgs& a, const double2* Cs, int b, int k0) {
    constexpr int U = 4;
    const int nb = a.nb, P = nb * nb, TK = a.TK, Nk = a.Nk;
    const long long boff = (long long)b * a.bstride;
    const int total = P * TK;
    for (int base = threadIdx.x; base < total; base += U * blockDim.x) {
        double2 g[U], y[U], ac[U];
        long long el[U];
        bool ok[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int idx = base + u * blockDim.x;
            const int p = idx / TK, kk = idx - (idx / TK) * TK;
            ok[u] = idx < total && k0 + kk < Nk;
            el[u] = boff + (long long)p * Nk + k0 + kk;
            if (ok[u]) {
                g[u] = __ldg(&a.G[el[u]]);
                if (MODE == MODE_RK1 || MODE == MODE_RK2 || MODE == MODE_RK3 || MODE == MODE_AB) y[u] = a.y[el[u]];
                if (MODE == MODE_RK2 || MODE == MODE_RK3 || MODE == MODE_RK4) ac[u] = a.acc[el[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (!ok[u]) continue;
            const double2 c = Cs[base + u * blockDim.x];
            const long long e = el[u];
            // f = G - i C
            const double2 f = make_double2(g[u].x + c.y, g[u].y - c.x);
            if (MODE == MODE_RHS) {
                a.out[e] = f;
            } else if (MODE == MODE_RK1) {
                a.aux[e] = make_double2(y[u].x + a.c[0] * f.x, y[u].y + a.c[0] * f.y);
                a.acc[e] = make_double2(y[u].x + a.c[1] * f.x, y[u].y + a.c[1] * f.y);
            } else if (MODE == MODE_RK2 || MODE == MODE_RK3) {
                a.aux[e] = make_double2(y[u].x + a.c[0] * f.x, y[u].y + a.c[0] * f.y);
                a.acc[e] = make_double2(ac[u].x + a.c[1] * f.x, ac[u].y + a.c[1] * f.y);
            } else if (MODE == MODE_RK4) {
                a.y[e] = make_double2(ac[u].x + a.c[0] * f.x, ac[u].y + a.c[0] * f.y);
            } else if (MODE == MODE_AB) {
                a.hist[0][e] = f;
                double2 yy = make_double2(y[u].x + a.c[0] * f.x, y[u].y + a.c[0] * f.y);
                for (int q = 1; q < a.order; ++q) {
                    const double2 fq = a.hist[q][e];
                    yy = make_double2(yy.x + a.c[q] * fq.x, yy.y + a.c[q] * fq.y);
                }
                a.y[e] = yy;
            }
        }
    }
}

// One (k tile, solve) of the CUDA-core commutator: the body of
// commutator_kernel, also run by the sweep's persistent commutator kernel.
// Any blockDim with TK * tiles <= 2 * blockDim works.
template <int MODE, bool COUL, bool FH = false>
__device__ __forceinline__ void commutator_tile(const StageArgs& a, int b, int tile, double2* sm) {
    const int nb = a.nb, TK = a.TK;
    const int nbp = (nb + 1) & ~1, ld = nbp + 1;
    const int tile_stride = nbp * ld;
    double2* Hs = sm;                        // [TK][nbp][ld]
    double2* Rs = sm + TK * tile_stride;     // [TK][nbp][ld]
    double2* hh = Rs + TK * tile_stride;     // [nb] Hartree shift
    double2* Cs = sm;                        // [P][TK], over Hs once the products are done
    const int k0 = tile * TK;
    const StageField F = a.field[b];
    if (COUL) {
        for (int n = threadIdx.x; n < nb; n += blockDim.x) {
            double2 s = make_double2(0.0, 0.0);
            for (int m = 0; m < nb; ++m) {
                const double2 d0 = a.diag0[b * nb + m];
                const double2 r0 = a.rho0diag[m];
                s = cadd(s, cmul(a.hartree[n * nb + m], csub(d0, r0)));
            }
            hh[n] = s;
        }
        __syncthreads();
    }
    load_stage_inputs<COUL, FH>(a, F, hh, b, k0, [&](int i, int j, int kk, double2 h, double2 r) {
        const int o = kk * tile_stride + i * ld + j;
        Hs[o] = h;
        Rs[o] = r;
    });
    __syncthreads();
    // C = H rho - rho H on 2x2 tiles (rows i0, i0+1; columns j0, j0+1) of one
    // k point: per l, 8 shared loads feed 8 complex multiply-adds.
    const int half = nbp / 2;
    const int ntile = half * half;
    const int ntask = TK * ntile;
    double2 acc[2][4];
#pragma unroll
    for (int t = 0; t < 2; ++t)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[t][q] = make_double2(0.0, 0.0);
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        const int task = threadIdx.x + t * blockDim.x;
        if (task < ntask) {
            const int kk = task / ntile, tt = task - (task / ntile) * ntile;
            const int i0 = 2 * (tt / half), j0 = 2 * (tt - (tt / half) * half);
            const double2* H = Hs + kk * tile_stride;
            const double2* R = Rs + kk * tile_stride;
            double2 c00 = make_double2(0.0, 0.0), c01 = c00, c10 = c00, c11 = c00;
            for (int l = 0; l < nb; ++l) {
                const double2 h0 = H[i0 * ld + l], h1 = H[(i0 + 1) * ld + l];
                const double2 r0 = R[l * ld + j0], r1 = R[l * ld + j0 + 1];
                c00.x = fma(h0.x, r0.x, fma(-h0.y, r0.y, c00.x));
                c00.y = fma(h0.x, r0.y, fma(h0.y, r0.x, c00.y));
                c01.x = fma(h0.x, r1.x, fma(-h0.y, r1.y, c01.x));
                c01.y = fma(h0.x, r1.y, fma(h0.y, r1.x, c01.y));
                c10.x = fma(h1.x, r0.x, fma(-h1.y, r0.y, c10.x));
                c10.y = fma(h1.x, r0.y, fma(h1.y, r0.x, c10.y));
                c11.x = fma(h1.x, r1.x, fma(-h1.y, r1.y, c11.x));
                c11.y = fma(h1.x, r1.y, fma(h1.y, r1.x, c11.y));
                const double2 q0 = R[i0 * ld + l], q1 = R[(i0 + 1) * ld + l];
                const double2 g0 = H[l * ld + j0], g1 = H[l * ld + j0 + 1];
                c00.x = fma(-q0.x, g0.x, fma(q0.y, g0.y, c00.x));
                c00.y = fma(-q0.x, g0.y, fma(-q0.y, g0.x, c00.y));
                c01.x = fma(-q0.x, g1.x, fma(q0.y, g1.y, c01.x));
                c01.y = fma(-q0.x, g1.y, fma(-q0.y, g1.x, c01.y));
                c10.x = fma(-q1.x, g0.x, fma(q1.y, g0.y, c10.x));
                c10.y = fma(-q1.x, g0.y, fma(-q1.y, g0.x, c10.y));
                c11.x = fma(-q1.x, g1.x, fma(q1.y, g1.y, c11.x));
                c11.y = fma(-q1.x, g1.y, fma(-q1.y, g1.x, c11.y));
            }
            acc[t][0] = c00;
            acc[t][1] = c01;
            acc[t][2] = c10;
            acc[t][3] = c11;
        }
    }
    __syncthreads();  // every tile read is done: Cs may overwrite Hs
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        const int task = threadIdx.x + t * blockDim.x;
        if (task < ntask) {
            const int kk = task / ntile, tt = task - (task / ntile) * ntile;
            const int i0 = 2 * (tt / half), j0 = 2 * (tt - (tt / half) * half);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int i = i0 + (q >> 1), j = j0 + (q & 1);
                if (i < nb && j < nb) Cs[(i * nb + j) * TK + kk] = acc[t][q];
            }
        }
    }
    __syncthreads();
    stage_epilogue<MODE>(a, Cs, b, k0);
}

template <int MODE, bool COUL, bool FH = false>
__global__ void __launch_bounds__(512) commutator_kernel(StageArgs a) {
    extern __shared__ double2 sm[];
    commutator_tile<MODE, COUL, FH>(a, blockIdx.y, blockIdx.x, sm);
}

// ---------------------------------------------------------------------------
// Tensor-core commutator for nb >= 12: the same contract as commutator_kernel,
// with C = H rho - rho H done by FP64 warp MMAs (mma.sync m8n8k4, 8x8 output
// tiles, K steps of 4).  A complex product is four real products:
//   Re(A B) = Ar Br - Ai Bi,  Im(A B) = Ar Bi + Ai Br,
// so each (tile, K step) issues 8 MMAs (4 for H rho, 4 for -rho H).
// Shared memory per k point: Hr, Hi, Rr, Ri as [nbp][pitch] doubles, nbp = nb
// rounded up to 8 and zero-padded, pitch = nbp + 4 (the fragment rows of a
// half-warp then land on distinct bank groups).  TK k points per CTA, 8 warps,
// 8/TK warps per k point; the result is staged as [p][TK] over the tiles.
struct MmaGeom {
    int TK, nbp, pitch, tiles, warps_per_k;
    size_t smem;
};

__host__ __device__ inline MmaGeom mma_geometry(int nb) {
    MmaGeom g;
    g.nbp = (nb + 7) & ~7;
    g.pitch = g.nbp + 4;
    g.tiles = g.nbp / 8;
    const size_t per_k = 4 * (size_t)g.nbp * g.pitch * 8;
    const int ntile = g.tiles * g.tiles;
    g.TK = 1;
    if (4 * per_k <= 100 * 1024 && (ntile + 1) / 2 <= 8) g.TK = 4;
    else if (2 * per_k <= 160 * 1024 && (ntile + 3) / 4 <= 8) g.TK = 2;
    g.warps_per_k = 8 / g.TK;
    g.smem = g.TK * per_k + (size_t)nb * 16;
    return g;
}

// Which commutator kernel a band count uses (the tensor-core one from 12
// bands up) and its launch geometry.
struct CommLaunch {
    bool mma;
    int TK, threads;
    size_t smem;
};
inline CommLaunch comm_launch(int nb) {
    CommLaunch c;
    c.mma = nb >= 12;
    if (c.mma) {
        const MmaGeom g = mma_geometry(nb);
        c.TK = g.TK;
        c.threads = 256;
        c.smem = g.smem;
    } else {
        const CommGeom g = comm_geometry(nb);
        c.TK = g.TK;
        c.threads = g.threads;
        c.smem = g.smem;
    }
    return c;
}

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// One (k tile, solve) of the FP64 tensor-core commutator: the body of
// commutator_mma_kernel, also run by the sweep's persistent commutator kernel.
// Warps past the first 8 take no product tiles (kk >= TK below).
template <int MODE, bool COUL, bool FH = false, int MAXT = 8>
__device__ __forceinline__ void commutator_mma_tile(const StageArgs& a, int b, int tile, double* smd) {
    const int nb = a.nb, Nk = a.Nk;
    const MmaGeom g = mma_geometry(nb);
    const int TK = g.TK, nbp = g.nbp, pitch = g.pitch;
    const int mat = nbp * pitch;  // doubles per matrix
    double* tiles = smd;          // [TK][4][nbp][pitch]: Hr, Hi, Rr, Ri
    double2* hh = (double2*)(smd + (size_t)TK * 4 * mat);
    double2* Cs = (double2*)smd;  // [P][TK] after the products
    const int k0 = tile * TK;
    const StageField F = a.field[b];
    for (int i = threadIdx.x; i < TK * 4 * mat; i += blockDim.x) tiles[i] = 0.0;
    if (COUL) {
        for (int n = threadIdx.x; n < nb; n += blockDim.x) {
            double2 s = make_double2(0.0, 0.0);
            for (int m = 0; m < nb; ++m) {
                const double2 d0 = a.diag0[b * nb + m];
                const double2 r0 = a.rho0diag[m];
                s = cadd(s, cmul(a.hartree[n * nb + m], csub(d0, r0)));
            }
            hh[n] = s;
        }
    }
    __syncthreads();
    load_stage_inputs<COUL, FH>(a, F, hh, b, k0, [&](int i, int j, int kk, double2 h, double2 r) {
        double* T = tiles + (size_t)kk * 4 * mat + i * pitch + j;
        T[0] = h.x;
        T[mat] = h.y;
        T[2 * mat] = r.x;
        T[3 * mat] = r.y;
    });
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kk = warp / g.warps_per_k, part = warp - kk * g.warps_per_k;
    const int ntile = g.tiles * g.tiles;
    const int per = (ntile + g.warps_per_k - 1) / g.warps_per_k;
    const int t0 = part * per, t1 = min(ntile, t0 + per);
    // MAXT: 8x8 output tiles per warp, at most 8 (nb <= 64); 5 covers nb <= 24
    double cr[MAXT][2], ci[MAXT][2];
#pragma unroll
    for (int t = 0; t < MAXT; ++t) cr[t][0] = cr[t][1] = ci[t][0] = ci[t][1] = 0.0;
    const double* Hr = tiles + (size_t)kk * 4 * mat;
    const double* Hi = Hr + mat;
    const double* Rr = Hr + 2 * mat;
    const double* Ri = Hr + 3 * mat;
    const int ar = lane >> 2, ac = lane & 3;  // A fragment (row, col); B fragment (row = ac, col = ar)
    if (kk < TK && k0 + kk < Nk) {
        for (int ks = 0; ks < nbp / 4; ++ks) {
            const int kc = ks * 4 + ac;
#pragma unroll
            for (int t = 0; t < MAXT; ++t) {
                const int tt = t0 + t;
                if (tt < t1) {
                    const int ti = tt / g.tiles, tj = tt - (tt / g.tiles) * g.tiles;
                    const int arow = ti * 8 + ar;   // output row of the A fragment
                    const int bcol = tj * 8 + ar;   // output column of the B fragment
                    // H rho
                    const double hr = Hr[arow * pitch + kc], hi = Hi[arow * pitch + kc];
                    const double rr = Rr[kc * pitch + bcol], ri = Ri[kc * pitch + bcol];
                    dmma(cr[t][0], cr[t][1], hr, rr);
                    dmma(cr[t][0], cr[t][1], -hi, ri);
                    dmma(ci[t][0], ci[t][1], hr, ri);
                    dmma(ci[t][0], ci[t][1], hi, rr);
                    // - rho H
                    const double qr = Rr[arow * pitch + kc], qi = Ri[arow * pitch + kc];
                    const double gr = Hr[kc * pitch + bcol], gi = Hi[kc * pitch + bcol];
                    dmma(cr[t][0], cr[t][1], -qr, gr);
                    dmma(cr[t][0], cr[t][1], qi, gi);
                    dmma(ci[t][0], ci[t][1], -qr, gi);
                    dmma(ci[t][0], ci[t][1], -qi, gr);
                }
            }
        }
    }
    __syncthreads();  // all fragments read: Cs may overwrite the tiles
    if (kk < TK) {
#pragma unroll
        for (int t = 0; t < MAXT; ++t) {
            const int tt = t0 + t;
            if (tt < t1) {
                const int ti = tt / g.tiles, tj = tt - (tt / g.tiles) * g.tiles;
                const int row = ti * 8 + ar;
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int col = tj * 8 + ac * 2 + q;
                    if (row < nb && col < nb) Cs[(row * nb + col) * TK + kk] = make_double2(cr[t][q], ci[t][q]);
                }
            }
        }
    }
    __syncthreads();
    stage_epilogue<MODE>(a, Cs, b, k0);
}

template <int MODE, bool COUL, bool FH = false>
__global__ void __launch_bounds__(256, 2) commutator_mma_kernel(StageArgs a) {
    extern __shared__ double smd[];
    commutator_mma_tile<MODE, COUL, FH>(a, blockIdx.y, blockIdx.x, smd);
}

// ---------------------------------------------------------------------------
// Layout transposes between the reference's [k][p] and the plane-major [p][k].
__global__ void transpose_kp_to_pk(const double2* __restrict__ src, double2* __restrict__ dst, int Nk, int P) {
    __shared__ double2 tile[32][33];
    const int k0 = blockIdx.x * 32, p0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int k = k0 + r, p = p0 + threadIdx.x;
        if (k < Nk && p < P) tile[r][threadIdx.x] = src[(long long)k * P + p];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int p = p0 + r, k = k0 + threadIdx.x;
        if (k < Nk && p < P) dst[(long long)p * Nk + k] = tile[threadIdx.x][r];
    }
}

__global__ void transpose_pk_to_kp(const double2* __restrict__ src, double2* __restrict__ dst, int Nk, int P) {
    __shared__ double2 tile[32][33];
    const int p0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int p = p0 + r, k = k0 + threadIdx.x;
        if (k < Nk && p < P) tile[r][threadIdx.x] = src[(long long)p * Nk + k];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int k = k0 + r, p = p0 + threadIdx.x;
        if (k < Nk && p < P) dst[(long long)k * P + p] = tile[threadIdx.x][r];
    }
}

// Wannier-gauge population: out[n] = (1/Nk) sum_k Re rho_nn(k), one CTA per n,
// fixed-order tree reduction (deterministic).
__global__ void population_kernel(const double2* __restrict__ rho, int Nk, int nb, double* __restrict__ out) {
    __shared__ double red[256];
    const int n = blockIdx.x;
    const double2* plane = rho + (long long)(n * nb + n) * Nk;
    double s = 0.0;
    for (int k = threadIdx.x; k < Nk; k += blockDim.x) s += plane[k].x;
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[n] = red[0] / (double)Nk;
}

// Non-finite detector over a state array: sets *flag to 1 if any component is
// NaN or Inf.
__global__ void finite_check_kernel(const double2* __restrict__ x, long long n, int* __restrict__ flag) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double2 v = x[i];
        if (!isfinite(v.x) || !isfinite(v.y)) {
            *flag = 1;
            return;
        }
    }
}

}  // namespace edus
