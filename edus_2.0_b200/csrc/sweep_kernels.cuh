// Kernels that advance a whole sweep of uneven solves (different band counts
// and k grids, independent-particle RHS, FP64, RK4) with one launch per RK
// stage for the plane transforms of every solve (per shared-memory class:
// planes that leave room for two CTAs on an SM, and larger ones) and one
// launch for the commutators and stage updates of every solve (per
// commutator kind: FP64 tensor cores or CUDA cores).
//
// Work items are (shape handle, solve, plane) and (shape handle, solve, k
// tile), ordered by decreasing cost on the host.  The plane kernel is
// persistent: a CTA takes the next item from an atomic counter (largest first
// onto whichever CTA is free).  The commutator kernels run one CTA per item in
// that order (the block scheduler hands items to SMs as they free up), which
// keeps their code at the registers of the per-shape kernels; their
// arguments are one launch parameter.  The solves of small shapes fill the SMs
// that the large ones leave.
// Each item runs the same device code as the shape's own kernels
// (plane_forward / plane_inverse with the gradient of kGradient_definitions.hpp:34-40;
// commutator_tile / commutator_mma_tile with the RK stage epilogue of
// DESolver.hpp:154-187), so a solve's result does not depend on the launch it
// ran in.
#pragma once
#include "kernels.cuh"

namespace edus {

// What a plane item needs from its shape beyond the stage arguments.
struct SweepPlaneDesc {
    const PlanePlan* plan;  // device copy of the shape's plan
    const double2* roots;
    const double* rpos;
    double2* G;             // gradient term out, [B][P][Nk]
    long long S;            // P * Nk (solve stride)
    int Nk;
    double inv_nk;
};

// The next item of this launch for the whole CTA (from `counter`, which the
// host zeroes before the launch).
__device__ __forceinline__ int sweep_fetch(int* counter, int* slot) {
    __syncthreads();  // every thread is done with the previous item (and its shared memory)
    if (threadIdx.x == 0) *slot = atomicAdd(counter, 1);
    __syncthreads();
    return *slot;
}

// Plane items {shape, solve, plane}: rho_R = FFT(rho_k)/Nk, G_R = i (R.E) rho_R,
// G_k = FFT^-1(G_R).  args[shape] are the shape's stage arguments (stage input
// rho, field table of the stage).
template <int MASK, int MAXT>
__global__ void __launch_bounds__(MAXT, MAXT <= 256 ? 2 : 1) sweep_plane_kernel(const SweepPlaneDesc* __restrict__ descs,
                                                           const StageArgs* __restrict__ args,
                                                           const int4* __restrict__ items, int nitems, int* counter) {
    extern __shared__ double2 X[];
    __shared__ int s_item;
    for (;;) {
        const int w = sweep_fetch(counter, &s_item);
        if (w >= nitems) break;
        const int4 it = items[w];
        const SweepPlaneDesc& d = descs[it.x];
        const StageArgs& a = args[it.x];
        const PlanePlan& pl = *d.plan;
        const int Nk = d.Nk;
        const long long off = (long long)it.y * d.S + (long long)it.z * Nk;
        const double2* src = a.rho + off;
        for (int i = threadIdx.x; i < Nk; i += blockDim.x) X[i] = __ldg(&src[i]);
        __syncthreads();
        const StageField F = a.field[it.y];
        const int n1 = pl.ax[1].n, n2 = pl.ax[2].n;
        const double* rp0 = d.rpos + pl.ax[0].rposoff;
        const double* rp1 = d.rpos + pl.ax[1].rposoff;
        const double* rp2 = d.rpos + pl.ax[2].rposoff;
        if (n2 == 1 && pl.ax[0].n > 1 && pl.ax[1].nst > 0) {
            // 2-D plane: row-wise, as plane_rhs_persist_kernel<..., ROWS>
            // (warps own rows of the unit-stride axis; the same arithmetic)
            const int nw = (int)(blockDim.x >> 5);
            const int lpw = (pl.ax[0].n + nw - 1) / nw;
            const int line0 = (int)(threadIdx.x >> 5) * lpw;
            const int nl = max(0, min(lpw, pl.ax[0].n - line0));
            axis0_transform<true, MASK>(X, pl, d.roots);
            rows_transform<true, MASK>(X, pl, d.roots, line0, nl);
            for (int idx = (int)(threadIdx.x & 31); idx < nl * n1; idx += 32) {
                const int li = fdiv(idx, pl.fd_n1);
                const int q1 = idx - li * n1;
                const int q0 = line0 + li;
                const int j = q0 * n1 + q1;
                const double dot = F.g[0] * __ldg(&rp0[q0]) + F.g[1] * __ldg(&rp1[q1]) + F.g[2] * __ldg(&rp2[0]);
                const double2 r = cscale(X[j], d.inv_nk);
                X[j] = make_double2(-dot * r.y, dot * r.x);
            }
            __syncwarp();
            rows_transform<false, MASK>(X, pl, d.roots, line0, nl);
            __syncthreads();
            axis0_transform<false, MASK>(X, pl, d.roots);
        } else {
            plane_forward<1, MASK>(X, 0, pl, d.roots);
            for (int j = threadIdx.x; j < Nk; j += blockDim.x) {
                const int t = fdiv(j, pl.fd_n2);
                const int q2 = j - t * n2;
                const int q0 = fdiv(t, pl.fd_n1);
                const int q1 = t - q0 * n1;
                const double dot =
                    F.g[0] * __ldg(&rp0[q0]) + F.g[1] * __ldg(&rp1[q1]) + F.g[2] * __ldg(&rp2[q2]);
                const double2 r = cscale(X[j], d.inv_nk);
                X[j] = make_double2(-dot * r.y, dot * r.x);
            }
            __syncthreads();
            plane_inverse<1, MASK>(X, 0, pl, d.roots);
        }
        double2* dst = d.G + off;
        for (int i = threadIdx.x; i < Nk; i += blockDim.x) dst[i] = X[i];
    }
}

// The stage arguments of every shape of a fused sweep, as one launch
// parameter: item code reads them from the constant bank, as the per-shape
// kernels read their own StageArgs parameter.
constexpr int kSweepMaxShapes = 64;
struct SweepStageArgs {
    StageArgs a[kSweepMaxShapes];
};

// Commutator items {shape, solve, k tile}: f = G - i[H0 + E.xi, rho] and the
// RK stage update of the shape's arrays, on the FP64 tensor cores (MMA, the
// shapes whose handle uses them) or on CUDA cores (the others): one launch
// per kind over all items, one CTA per item, largest items first (the block
// scheduler hands them out as SMs free up), so that each compiles to the
// registers of the shape's own kernel.  MAXT is at least every shape's
// commutator thread count (256 for fewer than 46 bands); TILES bounds the 8x8
// tiles a warp takes (5 covers 24 bands).
template <int MODE, int MAXT, bool MMA, int TILES = 8>
__global__ void __launch_bounds__(MAXT, MAXT <= 256 ? 2 : 1) sweep_comm_kernel(
    const __grid_constant__ SweepStageArgs args, const int4* __restrict__ items) {
    extern __shared__ double2 sm[];
    const int4 it = items[blockIdx.x];
    const StageArgs& a = args.a[it.x];
    if constexpr (MMA)
        commutator_mma_tile<MODE, false, false, TILES>(a, it.y, it.z, (double*)sm);
    else
        commutator_tile<MODE, false>(a, it.y, it.z, sm);
}

}  // namespace edus
