// edus_rhs_noalloc: one right-hand-side evaluation that allocates no device
// memory.
//
// Who needs it: callers whose device memory is owned by someone else -- a
// framework's caching allocator that reserves the GPU up front, an
// application with a fixed pool sized at start-up, or a time-critical loop
// that cannot take cudaMalloc's implicit device-wide synchronisation.  Such
// callers can still hand us device buffers for the inputs and the output;
// what they cannot do is let us allocate the intermediates.  So this entry
// point keeps its intermediates (plane-major copies of the state and of the
// model, the gradient and self-energy planes, FFT tables) in one fixed array
// that the CUDA module itself carries: `g_noalloc_scratch` below, of
// EDUS_NOALLOC_SCRATCH_BYTES.  Every GPU that loads the library holds that
// array until the process exits.
//
// Rules for users:
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress), sets the kernels' shared-memory limits and copies
//    the k grid's FFT tables from host memory into the array (then waits for
//    that copy); make that first call before any stream capture on that
//    device.  A call whose k grid differs from the previous call's on that
//    device copies the new grid's tables the same way; every other call only
//    queues kernels (the field of the evaluation travels as a kernel
//    argument);
//  * all calls share the one array: calls that overlap on the GPU (different
//    streams, or several host threads) race on it -- serialise them;
//  * problems whose intermediates exceed the array are rejected with
//    EDUS_ERR_UNSUPPORTED; nothing here calls cudaMalloc or cudaFree;
//  * W must be real (the screened potential has no imaginary part): a W_R
//    whose imaginary part is not zero is refused on the device, where the
//    check runs, by an output of NaN (an error code would need a
//    synchronisation).
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>
#include "../../include/edus_gpu.h"
// The handle path's kernels, compiled again here with internal linkage so
// this translation unit carries its own copies.
namespace {
#include "kernels.cuh"
#include "plane_plan.hpp"
}  // namespace

using namespace edus;

// The scratch array.  In host code this name is only a stand-in for the
// symbol: its device address comes from cudaGetSymbolAddress, per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[EDUS_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {nullptr};
int g_smem_set[kMaxDevices] = {0};  // plane-kernel dynamic smem limit already raised to this many bytes
int g_tab_grid[kMaxDevices][3] = {};  // k grid whose FFT tables sit at the front of the array (0: none)
thread_local char* g_errbuf = nullptr;
thread_local int g_errlen = 0;

int nfail(int code, const std::string& msg) {
    if (g_errbuf && g_errlen > 0) std::snprintf(g_errbuf, (size_t)g_errlen, "%s", msg.c_str());
    return code;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// H1[p][k] = H0[k][p] + sum_d E_d xi_d[k][p] (the sequence the commutator
// kernel uses), transposed into the plane layout.
__global__ void prep_hamiltonian(const double2* __restrict__ H0, const double2* __restrict__ xi, double2* __restrict__ H1,
                                 int Nk, int P, double e0, double e1, double e2) {
    const long long S = (long long)Nk * P;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < S; i += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(i / P), p = (int)(i - (long long)(i / P) * P);
        double2 h = H0[i];
        if (e0 != 0.0) { const double2 x = xi[i]; h.x += e0 * x.x; h.y += e0 * x.y; }
        if (e1 != 0.0) { const double2 x = xi[S + i]; h.x += e1 * x.x; h.y += e1 * x.y; }
        if (e2 != 0.0) { const double2 x = xi[2 * S + i]; h.x += e2 * x.x; h.y += e2 * x.y; }
        H1[(long long)p * Nk + k] = h;
    }
}

// W (real part) and rho0 from [R][p] into the plane layout at the
// digit-reversed positions of the plane FFT; rho0_nn(R=0) into r0diag.
__global__ void prep_hsex(const double2* __restrict__ W, const double2* __restrict__ rho0, double* __restrict__ Wp,
                          double2* __restrict__ r0p, double2* __restrict__ r0diag, const int* __restrict__ fq0,
                          const int* __restrict__ fq1, const int* __restrict__ fq2, int N1, int N2, int Nk, int nb,
                          int* __restrict__ status) {
    const int P = nb * nb;
    const long long S = (long long)Nk * P;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < S; i += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(i / Nk), pos = (int)(i - (long long)p * Nk);
        const int q2 = pos % N2, t = pos / N2, q1 = t % N1, q0 = t / N1;
        const long long iR = ((long long)fq0[q0] * N1 + fq1[q1]) * N2 + fq2[q2];
        const double2 w = W[iR * P + p];
        Wp[i] = w.x;
        if (w.y != 0.0) *status = 1;  // refused: the output becomes NaN
        r0p[i] = rho0[iR * P + p];
    }
    if (blockIdx.x == 0)
        for (int n = threadIdx.x; n < nb; n += blockDim.x) r0diag[n] = rho0[n * nb + n];
}

// The evaluation's two stage fields (by value: no host copy), a cleared
// Hartree accumulator and a cleared status word.
__global__ void set_call_state(StageField* __restrict__ field, StageField f0, StageField f1,
                               double2* __restrict__ diag0, int nb, int* __restrict__ status) {
    if (threadIdx.x == 0) {
        field[0] = f0;
        field[1] = f1;
        *status = 0;
    }
    for (int n = threadIdx.x; n < nb; n += blockDim.x) diag0[n] = make_double2(0.0, 0.0);
}

// out[k][p] = src[p][k], or NaN everywhere when the status word is set.
__global__ void transpose_out(const double2* __restrict__ src, double2* __restrict__ dst, int Nk, int P,
                              const int* __restrict__ status) {
    __shared__ double2 tile[32][33];
    const bool refused = *status != 0;
    const int p0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int p = p0 + r, k = k0 + threadIdx.x;
        if (k < Nk && p < P) tile[r][threadIdx.x] = src[(long long)p * Nk + k];
    }
    __syncthreads();
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int k = k0 + r, p = p0 + threadIdx.x;
        if (k < Nk && p < P) dst[(long long)k * P + p] = refused ? make_double2(nan, nan) : tile[threadIdx.x][r];
    }
}

}  // namespace

extern "C" int edus_rhs_noalloc(const int grid[3], int nbands, int coulomb, const double lattice[9],
                                const double efield[3], const double* H0_k, const double* xi_k, const double* W_R,
                                const double* rho0_R, const double* hartree, const double* in_k, double* out_k,
                                void* stream_ptr, char* errbuf, int errlen) {
    g_errbuf = errbuf;
    g_errlen = errlen;
    if (errbuf && errlen > 0) errbuf[0] = '\0';
    if (!grid || !lattice || !efield || !H0_k || !xi_k || !in_k || !out_k)
        return nfail(EDUS_ERR_ARG, "edus_rhs_noalloc: NULL argument");
    if (coulomb && (!W_R || !rho0_R || !hartree))
        return nfail(EDUS_ERR_ARG, "edus_rhs_noalloc: coulomb=1 needs W_R, rho0_R and hartree");
    if (nbands < 1 || nbands > 64) return nfail(EDUS_ERR_ARG, "edus_rhs_noalloc: nbands must be in [1, 64]");
    int N[3];
    for (int d = 0; d < 3; ++d) {
        N[d] = grid[d];
        if (N[d] < 1) return nfail(EDUS_ERR_ARG, "edus_rhs_noalloc: grid dimensions must be >= 1");
    }
    const int Nk = N[0] * N[1] * N[2];
    const int nb = nbands, P = nb * nb;
    const size_t S = (size_t)P * Nk;
    cudaStream_t stream = (cudaStream_t)stream_ptr;

    // FFT plan and tables (host), as in edus_create
    PlanePlan plan{};
    PlaneTables tabs;
    {
        std::string perr;
        if (!build_plane_plan(N, plan, tabs, perr)) return nfail(EDUS_ERR_UNSUPPORTED, "edus_rhs_noalloc: " + perr);
    }
    const std::vector<double2>& roots = tabs.roots;
    const std::vector<double>& rpos = tabs.rpos;
    const std::vector<int>& fqall = tabs.fq;
    const int* fqoff = tabs.fqoff;

    // carve the scratch array
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off = align256(off + bytes);
        return o;
    };
    // the grid's tables first: they stay in place while the grid does not change
    const size_t o_roots = take(roots.size() * sizeof(double2));
    const size_t o_rpos = take(rpos.size() * sizeof(double));
    const size_t o_fq = take(fqall.size() * sizeof(int));
    const size_t o_rho = take(S * sizeof(double2));
    const size_t o_G = take(S * sizeof(double2));
    const size_t o_out = take(S * sizeof(double2));
    const size_t o_H1 = take(S * sizeof(double2));
    const size_t o_Hee = coulomb ? take(S * sizeof(double2)) : 0;
    const size_t o_r0p = coulomb ? take(S * sizeof(double2)) : 0;
    const size_t o_Wp = coulomb ? take(S * sizeof(double)) : 0;
    const size_t o_field = take(2 * sizeof(StageField));
    const size_t o_diag0 = take(nb * sizeof(double2));
    const size_t o_r0diag = take(nb * sizeof(double2));
    const size_t o_status = take(sizeof(int));
    if (off > (size_t)EDUS_NOALLOC_SCRATCH_BYTES)
        return nfail(EDUS_ERR_UNSUPPORTED, "edus_rhs_noalloc: this grid and band count need " + std::to_string(off) +
                                               " bytes of scratch; the built-in array holds " +
                                               std::to_string((size_t)EDUS_NOALLOC_SCRATCH_BYTES) +
                                               " (use edus_create/edus_rhs)");
    const size_t plane_smem = (size_t)Nk * sizeof(double2) * (coulomb ? 2 : 1);
    const CommLaunch cgeo = comm_launch(nb);
    const int tk = cgeo.TK;
    const size_t comm_smem = cgeo.smem;

    // per-device set-up: the array's device address and the kernels' limits
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return nfail(EDUS_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return nfail(EDUS_ERR_UNSUPPORTED, "edus_rhs_noalloc: device ordinal too large");
    int dev_smem = 0;
    cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (plane_smem > (size_t)dev_smem || comm_smem > (size_t)dev_smem)
        return nfail(EDUS_ERR_UNSUPPORTED, "edus_rhs_noalloc: k grid or band count too large for shared memory");
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_addr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p)
                return nfail(EDUS_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_scratch_addr[dev] = p;
        }
        if (g_smem_set[dev] < dev_smem) {
            const int lim = dev_smem;
            if ((e = cudaFuncSetAttribute(plane_rhs_kernel<true, kRadixAll, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim)) != cudaSuccess ||
                (e = cudaFuncSetAttribute(plane_rhs_kernel<false, kRadixAll, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim)) != cudaSuccess ||
                (e = cudaFuncSetAttribute(commutator_kernel<MODE_RHS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim)) != cudaSuccess ||
                (e = cudaFuncSetAttribute(commutator_kernel<MODE_RHS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim)) != cudaSuccess ||
                (e = cudaFuncSetAttribute(commutator_mma_kernel<MODE_RHS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim)) != cudaSuccess ||
                (e = cudaFuncSetAttribute(commutator_mma_kernel<MODE_RHS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim)) != cudaSuccess)
                return nfail(EDUS_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
            g_smem_set[dev] = lim;
        }
        base = (unsigned char*)g_scratch_addr[dev];
    }
    double2* rho_pk = (double2*)(base + o_rho);
    double2* G = (double2*)(base + o_G);
    double2* out_pk = (double2*)(base + o_out);
    double2* H1 = (double2*)(base + o_H1);
    double2* Hee = coulomb ? (double2*)(base + o_Hee) : nullptr;
    double2* r0p = coulomb ? (double2*)(base + o_r0p) : nullptr;
    double* Wp = coulomb ? (double*)(base + o_Wp) : nullptr;
    double2* d_roots = (double2*)(base + o_roots);
    double* d_rpos = (double*)(base + o_rpos);
    int* d_fq = (int*)(base + o_fq);
    StageField* d_field = (StageField*)(base + o_field);
    double2* diag0 = (double2*)(base + o_diag0);
    double2* r0diag = (double2*)(base + o_r0diag);
    int* d_status = (int*)(base + o_status);

    // field: the plane kernel needs g = A^T E for R.E; the Hamiltonian's E.xi
    // is folded into H1 here, so the commutator sees E = 0
    StageField hf[2];
    for (int d = 0; d < 3; ++d) hf[0].E[d] = efield[d];
    for (int c = 0; c < 3; ++c)
        hf[0].g[c] = lattice[0 * 3 + c] * efield[0] + lattice[1 * 3 + c] * efield[1] + lattice[2 * 3 + c] * efield[2];
    for (int d = 0; d < 3; ++d) hf[1].E[d] = hf[1].g[d] = 0.0;

#define NA_CU(expr)                                                                        \
    do {                                                                                   \
        cudaError_t e_ = (expr);                                                           \
        if (e_ != cudaSuccess) return nfail(EDUS_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)
    // the grid's FFT tables: copied only when the device's resident tables are
    // for another grid (first call, or a new grid), and waited for, so that no
    // later call depends on a copy in flight
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (g_tab_grid[dev][0] != N[0] || g_tab_grid[dev][1] != N[1] || g_tab_grid[dev][2] != N[2]) {
            g_tab_grid[dev][0] = 0;
            NA_CU(cudaMemcpyAsync(d_roots, roots.data(), roots.size() * sizeof(double2), cudaMemcpyHostToDevice, stream));
            NA_CU(cudaMemcpyAsync(d_rpos, rpos.data(), rpos.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
            NA_CU(cudaMemcpyAsync(d_fq, fqall.data(), fqall.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
            NA_CU(cudaStreamSynchronize(stream));
            for (int d = 0; d < 3; ++d) g_tab_grid[dev][d] = N[d];
        }
    }
    // the field by value; diag0 is read only after the plane kernel writes it,
    // and is cleared so that a stale value from an earlier call can never leak
    // into this one; the status word starts at zero
    set_call_state<<<1, 64, 0, stream>>>(d_field, hf[0], hf[1], diag0, nb, d_status);
    NA_CU(cudaGetLastError());

    const int nthr = 256;
    const int nblk = (int)std::min<size_t>((S + nthr - 1) / nthr, 148 * 16);
    dim3 tb(32, 8), tg((Nk + 31) / 32, (P + 31) / 32);
    transpose_kp_to_pk<<<tg, tb, 0, stream>>>((const double2*)in_k, rho_pk, Nk, P);
    prep_hamiltonian<<<nblk, nthr, 0, stream>>>((const double2*)H0_k, (const double2*)xi_k, H1, Nk, P, efield[0],
                                                 efield[1], efield[2]);
    if (coulomb)
        prep_hsex<<<nblk, nthr, 0, stream>>>((const double2*)W_R, (const double2*)rho0_R, Wp, r0p, r0diag,
                                             d_fq + fqoff[0], d_fq + fqoff[1], d_fq + fqoff[2], N[1], N[2], Nk, nb,
                                             d_status);
    NA_CU(cudaGetLastError());
    dim3 pg(P, 1);
    if (coulomb)
        plane_rhs_kernel<true, kRadixAll, 512><<<pg, 512, plane_smem, stream>>>(rho_pk, 0, G, Hee, 0, r0p, Wp, diag0,
                                                                                 d_field, d_roots, d_rpos, plan, nb,
                                                                                 1.0 / Nk, nullptr, nullptr, 0);
    else
        plane_rhs_kernel<false, kRadixAll, 512><<<pg, 512, plane_smem, stream>>>(rho_pk, 0, G, Hee, 0, r0p, Wp, diag0,
                                                                                  d_field, d_roots, d_rpos, plan, nb,
                                                                                  1.0 / Nk, nullptr, nullptr, 0);
    NA_CU(cudaGetLastError());
    StageArgs a{};
    a.rho = rho_pk;
    a.G = G;
    a.Hee = Hee;
    a.H0 = H1;
    for (int d = 0; d < 3; ++d) a.xi[d] = H1;  // never read: the commutator's field is zero
    a.hartree = (const double2*)hartree;
    a.rho0diag = r0diag;
    a.diag0 = diag0;
    a.field = d_field + 1;
    a.out = out_pk;
    a.bstride = (long long)S;
    a.Nk = Nk;
    a.nb = nb;
    a.TK = tk;
    dim3 cg((Nk + tk - 1) / tk, 1);
    if (cgeo.mma) {
        if (coulomb)
            commutator_mma_kernel<MODE_RHS, true><<<cg, cgeo.threads, comm_smem, stream>>>(a);
        else
            commutator_mma_kernel<MODE_RHS, false><<<cg, cgeo.threads, comm_smem, stream>>>(a);
    } else {
        if (coulomb)
            commutator_kernel<MODE_RHS, true><<<cg, cgeo.threads, comm_smem, stream>>>(a);
        else
            commutator_kernel<MODE_RHS, false><<<cg, cgeo.threads, comm_smem, stream>>>(a);
    }
    NA_CU(cudaGetLastError());
    dim3 tg2((P + 31) / 32, (Nk + 31) / 32);
    transpose_out<<<tg2, tb, 0, stream>>>(out_pk, (double2*)out_k, Nk, P, d_status);
    NA_CU(cudaGetLastError());
#undef NA_CU
    return EDUS_OK;
}
