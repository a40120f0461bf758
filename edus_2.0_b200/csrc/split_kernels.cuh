// Split-precision plane kernel (EDUS_PREC_SPLIT32): the right-hand side of
// the full (non-Hermitian, reference-exact) generator with the state split as
// rho = rho_ref + delta.  The map rho -> (G, H) is affine,
//   G(rho)  = sum_d E_d grad_d(rho_ref) + G(delta),
//   H(rho)  = [H0 + Hee(rho_ref)] + E.xi + E1(delta),   E1(delta) = -W delta (R),
// so the terms of rho_ref are computed once per anchor in FP64 and added in
// k space, and only delta goes through the plane transforms, in FP32: their
// rounding error scales with |delta|, not |rho|.  The anchor rho_ref is moved
// to the current state every few steps, which keeps |delta| small.
// The commutator, the stage updates and the state stay FP64.
// Reference: Functional_SourceTerm.hpp:15-50, kGradient_definitions.hpp:35-40,
// Coulomb.cpp:150-171, Simulation.cpp:296-349.
#pragma once
#include "kernels.cuh"

namespace edus {

struct SplitArgs {
    const double2* rho;      // stage input [B][P][Nk]
    const double2* rref;     // anchor [B][P][Nk]
    long long bstride;       // P*Nk
    int nplanes;             // P*B
    double2* G;              // out: gradient term [B][P][Nk]
    double2* H;              // out (HSEX): H0 + E.xi + Hee [B][P][Nk]
    const double2* Gref[3];  // grad_d rho_ref [B][P][Nk] (unit field along d)
    const double2* Hfix;     // H0 + Hee(rho_ref) [B][P][Nk]
    const double2* xi[3];    // [P][Nk]
    const float* W32;        // screened potential, digit-reversed R order [P][Nk]
    const double2* refdiag0; // rho_ref,nn(R=0) [B][nb]
    double2* diag0;          // out: rho_nn(R=0) of the stage input [B][nb]
    const StageField* field; // [B]
    const double2* roots;
    const double* rpos;
    float2* scratch;         // one plane of FP32 per CTA
    int nb;
    double inv_nk;
};

// Persistent: CTA c transforms planes c, c + gridDim.x, ... of the P x B planes,
// one FP32 plane (8 Nk bytes) of shared memory.
template <bool COUL, int MASK, int MAXT>
__global__ void __launch_bounds__(MAXT, 2) plane_split_kernel(SplitArgs a, PlanePlan pl) {
    extern __shared__ float2 sm32[];
    const int Nk = pl.Nk, nb = a.nb, P = nb * nb;
    float2* X = sm32;
    float2* slot = a.scratch + (long long)blockIdx.x * Nk;
    const int n1 = pl.ax[1].n, n2 = pl.ax[2].n;
    const double* rp0 = a.rpos + pl.ax[0].rposoff;
    const double* rp1 = a.rpos + pl.ax[1].rposoff;
    const double* rp2 = a.rpos + pl.ax[2].rposoff;
    const float inv = (float)a.inv_nk;
    for (int w = blockIdx.x; w < a.nplanes; w += gridDim.x) {
        const int b = w / P, p = w - (w / P) * P;
        const long long off = (long long)b * a.bstride + (long long)p * Nk;
        for (int i = threadIdx.x; i < Nk; i += blockDim.x) {
            const double2 r = __ldg(&a.rho[off + i]);
            const double2 q = __ldg(&a.rref[off + i]);
            X[i] = make_float2((float)(r.x - q.x), (float)(r.y - q.y));
        }
        __syncthreads();
        plane_forward<1, MASK>(X, 0, pl, a.roots);
        const StageField F = a.field[b];
        const int n = p / nb, m = p - (p / nb) * nb;
        if (COUL && n == m && threadIdx.x == 0) {
            const double2 r0 = a.refdiag0[b * nb + n];
            a.diag0[b * nb + n] = make_double2(r0.x + (double)X[0].x * a.inv_nk, r0.y + (double)X[0].y * a.inv_nk);
        }
        __syncthreads();
        for (int j = threadIdx.x; j < Nk; j += blockDim.x) {
            const int t = fdiv(j, pl.fd_n2);
            const int q2 = j - t * n2;
            const int q0 = fdiv(t, pl.fd_n1);
            const int q1 = t - q0 * n1;
            const float dot =
                (float)(F.g[0] * __ldg(&rp0[q0]) + F.g[1] * __ldg(&rp1[q1]) + F.g[2] * __ldg(&rp2[q2]));
            const float2 r = make_float2(X[j].x * inv, X[j].y * inv);
            if (COUL) slot[j] = r;
            X[j] = make_float2(-dot * r.y, dot * r.x);
        }
        __syncthreads();
        plane_inverse<1, MASK>(X, 0, pl, a.roots);
        {
            double2* gdst = a.G + off;
            for (int i = threadIdx.x; i < Nk; i += blockDim.x) {
                double2 v = make_double2((double)X[i].x, (double)X[i].y);
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    if (F.E[d] != 0.0) {
                        const double2 gr = __ldg(&a.Gref[d][off + i]);
                        v.x += F.E[d] * gr.x;
                        v.y += F.E[d] * gr.y;
                    }
                }
                gdst[i] = v;
            }
        }
        if (COUL) {
            __syncthreads();  // X is refilled below
            const float* wp = a.W32 + (long long)p * Nk;
            for (int j = threadIdx.x; j < Nk; j += blockDim.x) {
                const float2 r = slot[j];
                const float wv = __ldg(&wp[j]);
                X[j] = make_float2(-wv * r.x, -wv * r.y);
            }
            __syncthreads();
            plane_inverse<1, MASK>(X, 0, pl, a.roots);
            double2* hdst = a.H + off;
            const long long po = (long long)p * Nk;
            for (int i = threadIdx.x; i < Nk; i += blockDim.x) {
                const double2 hf = __ldg(&a.Hfix[off + i]);
                double2 v = make_double2((double)X[i].x + hf.x, (double)X[i].y + hf.y);
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    if (F.E[d] != 0.0) {
                        const double2 x = __ldg(&a.xi[d][po + i]);
                        v.x += F.E[d] * x.x;
                        v.y += F.E[d] * x.y;
                    }
                }
                hdst[i] = v;
            }
        }
        __syncthreads();  // X is reloaded by the next plane
    }
}

// Hfix[b] = H0 + Hee[b] (the anchor's Hamiltonian without the field)
__global__ void add_broadcast_kernel(const double2* __restrict__ H0, const double2* __restrict__ Hee,
                                     double2* __restrict__ out, long long S, int B) {
    const long long total = S * B;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const double2 a = H0[i % S], h = Hee[i];
        out[i] = make_double2(a.x + h.x, a.y + h.y);
    }
}

__global__ void to_float_kernel(const double* __restrict__ src, float* __restrict__ dst, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}

}  // namespace edus
