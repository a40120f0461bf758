// Host side of the C ABI declared in include/edus_gpu.h.
//
// One handle = one model (H0, xi, W, rho0, Hartree) shared by `batch`
// independent solves, each with its own lasers and density matrix.  All
// device memory is allocated in edus_create / edus_upload_model; the step
// loop allocates nothing.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <stdexcept>
#include "../../include/edus_gpu.h"
#include "kernels.cuh"
#include "packed_kernels.cuh"
#include "comm_ws.cuh"
#include "split_kernels.cuh"
#include "plane3.cuh"
#include "sweep_kernels.cuh"
#include <cudaTypedefs.h>
#include <map>
#include <mutex>
#include "plane_plan.hpp"

using namespace edus;

namespace {

thread_local std::string g_create_error;

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

}  // namespace

struct edus_handle {
    edus_desc d{};
    int N[3] = {1, 1, 1};
    int Nk = 0, nb = 0, P = 0, B = 1;
    size_t S = 0;  // complex numbers per solve (P*Nk)
    cudaStream_t stream = nullptr;
    std::string err;
    bool model_ready = false;
    double t = 0.0;
    double A[9] = {0};  // lattice, row-major, vectors in columns
    PlanePlan plan{};
    int smem_plane = 0, smem_comm = 0, TK = 4, comm_threads = 256;
    bool comm_mma = false;
    // fused Hamiltonian (HSEX): sparse H0(R), xi_d(R) added in the plane kernel
    int* hpos = nullptr;
    double2* hval = nullptr;
    int nS = 0;
    // few planes on a 2-D grid: plane transforms over many CTAs (plane3.cuh)
    bool use3 = false;
    Plane3Plan p3{};
    double2* s3a = nullptr;  // rows pass output, [B][P][Nk]
    double2* s3g = nullptr;  // columns pass: G and H, [B][P][Nk]
    double2* s3h = nullptr;
    // gradient_space "k": finite-difference stencil (edus_set_kgradient)
    int kg_n = 0, kg_cap = 0;
    int* kg_shift = nullptr;     // [n][3]
    double* kg_coef = nullptr;   // [n][4]: b_x, b_y, b_z, w
    // observables: eigenvectors U_k and velocity operator v_d(k), [P][Nk] each
    double2* obsU = nullptr;
    double2* obsV[3] = {nullptr, nullptr, nullptr};
    double* obsacc = nullptr;
    // a model (H0, xi) per solve (edus_upload_model_solve): [B][P][Nk] each
    bool per_solve = false;
    double2* H0b = nullptr;
    double2* xib[3] = {nullptr, nullptr, nullptr};
    // Fock term given by the caller on nO lattice vectors (edus_set_fock_override)
    int* opos = nullptr;
    double2* oval = nullptr;
    int nO = 0, nO_cap = 0;
    // position (digit-reversed plane order) of each frequency index, per axis
    std::vector<int> posof[3];
    // warp-specialised TMA commutator of the fused path (12 <= nb <= 24):
    // CTAs per launch, and its tensor maps keyed by (array, 2 * batch count +
    // box kind): kind 0 the dense box, kind 1 the zero-padded box of the
    // product operands
    bool comm_ws = false;
    int ws_grid = 0;
    // Peierls gauge (edus_set_peierls): per-axis phase tables of the stage
    // ([B][ntab]) and each solve's vector-potential integrator (A, last time)
    bool peierls = false;
    double2* ptab = nullptr;
    int ntab = 0;
    std::vector<double> Avec, Aprev;
    std::map<std::pair<const void*, int>, CUtensorMap> tmaps;
    // split-precision form (EDUS_PREC_SPLIT32): anchor rho_ref and its FP64 terms
    bool split = false, anchored = false;
    int anchor_every = 32, since_anchor = 0;
    double2* sref = nullptr;
    double2* sGref[3] = {nullptr, nullptr, nullptr};
    double2* sHfix = nullptr;
    double2* srefdiag0 = nullptr;
    float* W32 = nullptr;
    float2* split_scratch = nullptr;
    StageField* unit_fields = nullptr;  // [3][B]: E = e_d
    int split_grid = 0, split_threads = 256;
    PlaneLaunch plane_cfg{0, 512, false};
    int plane_grid = 0;            // persistent plane kernel: CTAs per launch
    bool rows_ok = false;          // persistent plane kernel: row-wise variant (2-D grids)
    bool hplanes = false;          // EDUS_PREC_HPLANES: pairs n <= m transformed, (m, n) conjugated
    int Pu = 0;                    // nb (nb + 1) / 2
    int* upair = nullptr;          // [Pu] n nb + m of the pairs n <= m
    int nroot_s = 0, nrpos_s = 0;  // persistent plane kernel: root / coordinate entries it stages in shared memory
    int tab_smem = 0;              // their bytes (0: read from global memory)
    int wait_polls = 1 << 22;      // the plane kernel's bulk-load wait limit (edus_set_wait_limit)
    double2* plane_scratch = nullptr;  // [plane_grid][Nk]: rho(R) between the two inverse transforms
    unsigned long long launches = 0;
    size_t dev_bytes = 0;
    std::vector<std::vector<edus_laser>> lasers;
    // AB ring (DESolver.hpp:47, rotated after each step)
    int index[5] = {0, 1, 2, 3, 4};
    double beta[5] = {0, 0, 0, 0, 0};
    // device buffers
    double2 *H0 = nullptr, *xi[3] = {nullptr, nullptr, nullptr};
    double2* rho0p = nullptr;
    double* Wp = nullptr;
    double2 *hartree = nullptr, *rho0diag = nullptr;
    double2 *y = nullptr, *aux = nullptr, *acc = nullptr, *hist[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    double2 *G = nullptr, *Hee = nullptr, *diag0 = nullptr;
    double2* roots = nullptr;
    double* rpos = nullptr;
    StageField* field = nullptr;   // device table [chunk][stage][B]
    StageField* field_host[2] = {nullptr, nullptr};  // pinned
    cudaEvent_t field_ev[2] = {nullptr, nullptr};
    int field_cur = 0;
    int chunk = 256;
    double2* stage = nullptr;      // [Nk][P] staging for transposes
    double2* tmp_in = nullptr;     // edus_rhs input/output in plane layout
    double2* tmp_out = nullptr;
    double* popbuf = nullptr;
    int* flag = nullptr;
    std::vector<void*> allocs;
    // profiling: event pairs per launch, resolved in edus_get_profile
    bool profiling = false;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof_pending;
    std::vector<cudaEvent_t> prof_pool;
    double prof_ms[2] = {0, 0};
    unsigned long long prof_n[2] = {0, 0};
    // packed-Hermitian forms (HERM64, MIXED)
    bool packed = false, mixed = false;
    int Pq = 0;
    size_t Sq = 0;                      // Pq*Nk
    int* qnm = nullptr;                 // packed plane -> (n << 16) | m
    bool ref_fixed = false;
    double2* ref_full = nullptr;        // rho_ref, FP64 full planes
    void *pH0p = nullptr, *pxi[3] = {nullptr, nullptr, nullptr}, *pRref = nullptr;  // ST planes
    void* pW = nullptr;                 // packed, digit-reversed W (real, ST scalar)
    double2 *pC0 = nullptr, *pK[3] = {nullptr, nullptr, nullptr};
    double2 *py = nullptr, *pacc = nullptr, *phist[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    void *paux = nullptr, *pG = nullptr, *pE1 = nullptr;
    double2* pdiag0 = nullptr;          // [B][nb] delta_nn(R=0)
    StageField* ref_fields = nullptr;   // E = 0, e_x, e_y, e_z
    PackedGeom pgeo{};
    int pplane_threads = 256, pplane_variant = 0;
    size_t pplane_smem = 0;
};

namespace {

int fail(edus_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    else g_create_error = msg;
    return code;
}

#define CU(h, expr)                                                                              \
    do {                                                                                         \
        cudaError_t e_ = (expr);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return fail(h, EDUS_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int dalloc(edus_handle* h, void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(h, EDUS_ERR_NOMEM, std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
    }
    h->allocs.push_back(*p);
    h->dev_bytes += bytes;
    return EDUS_OK;
}

#define ALLOC(h, ptr, bytes)                                      \
    do {                                                          \
        int rc_ = dalloc(h, (void**)&(ptr), (size_t)(bytes));     \
        if (rc_ != EDUS_OK) return rc_;                           \
    } while (0)

void field_at(const std::vector<edus_laser>& ls, const double A[9], double t, StageField& f) {
    // SetOfLaser::operator() (Laser.hpp:143-150) with Laser::operator()
    // (Laser.cpp:131-134), envelope (Laser.cpp:96-104), carrier (Laser.cpp:35-38)
    const double pi = 3.14159265358979323846;
    double E[3] = {0, 0, 0};
    for (const auto& L : ls) {
        double nrm = std::sqrt(L.pol[0] * L.pol[0] + L.pol[1] * L.pol[1] + L.pol[2] * L.pol[2]);
        double pol[3] = {L.pol[0] / nrm, L.pol[1] / nrm, L.pol[2] / nrm};
        // Laser::set_Polarization normalises a second time (Laser.cpp:197-200)
        double n2 = std::sqrt(pol[0] * pol[0] + pol[1] * pol[1] + pol[2] * pol[2]);
        for (int d = 0; d < 3; ++d) pol[d] = pol[d] / n2;
        double a;
        const double amp = std::sqrt(L.intensity);
        if (L.envelope == EDUS_ENVELOPE_SIN2) {
            const double period = 2. * pi / L.omega;
            const double duration = L.cycles * period;
            const double tt = t - L.t0;
            const double env = (tt <= 1.e-07 || tt > duration) ? 0. : std::pow(std::sin(pi * tt / duration), 2.);
            a = amp * env * std::sin(L.omega * (t - L.t0) + L.phase);
        } else {
            const double tt = t - L.t0;
            const double env = std::exp(-2.0 * std::log(2.0) * tt * tt / (L.fwhm * L.fwhm));
            a = amp * env * std::cos(L.omega * tt + L.phase);
        }
        for (int d = 0; d < 3; ++d) E[d] += a * pol[d];
    }
    for (int d = 0; d < 3; ++d) f.E[d] = E[d];
    for (int c = 0; c < 3; ++c) f.g[c] = A[0 * 3 + c] * E[0] + A[1 * 3 + c] * E[1] + A[2 * 3 + c] * E[2];
    for (int c = 0; c < 3; ++c) f.ga[c] = 0.0;
}

// Laser::VectorPotential (Laser.cpp:136-151) for solve b, advanced to t:
// when t - t_prev >= 1e-7, A -= (t - t_prev)/6 (E(t_prev) + 4 E(mid) + E(t)) and
// t_prev = t.  The reference keeps A and t_prev in function statics, starting
// from 0 and 0, shared by all lasers; here each solve integrates the total
// field of its lasers (the same for one laser).
void advance_vecpot(edus_handle* h, int b, double t) {
    const double dT = t - h->Aprev[b];
    if (dT < 1.e-07) return;
    StageField f1, f2, f3;
    field_at(h->lasers[b], h->A, h->Aprev[b], f1);
    field_at(h->lasers[b], h->A, h->Aprev[b] + dT / 2., f2);
    field_at(h->lasers[b], h->A, t, f3);
    for (int d = 0; d < 3; ++d) h->Avec[3 * b + d] -= dT / 6. * (f1.E[d] + 4. * f2.E[d] + f3.E[d]);
    h->Aprev[b] = t;
}

// Peierls gauge at stage time t of solve b: no gradient term (g = 0) and
// ga = A^T A(t), so that A(t).R = ga . R_crys (Simulation.cpp:876-899)
void peierls_field(edus_handle* h, int b, double t, StageField& f) {
    advance_vecpot(h, b, t);
    for (int c = 0; c < 3; ++c) {
        f.g[c] = 0.0;
        f.ga[c] = h->A[0 * 3 + c] * h->Avec[3 * b] + h->A[1 * 3 + c] * h->Avec[3 * b + 1] +
                  h->A[2 * 3 + c] * h->Avec[3 * b + 2];
    }
}

cudaEvent_t prof_event(edus_handle* h) {
    if (!h->prof_pool.empty()) {
        cudaEvent_t e = h->prof_pool.back();
        h->prof_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void prof_begin(edus_handle* h, cudaEvent_t* e0) {
    *e0 = nullptr;
    if (!h->profiling) return;
    *e0 = prof_event(h);
    cudaEventRecord(*e0, h->stream);
}

void prof_end(edus_handle* h, int kind, cudaEvent_t e0) {
    if (!h->profiling || !e0) return;
    cudaEvent_t e1 = prof_event(h);
    cudaEventRecord(e1, h->stream);
    h->prof_pending.push_back({kind, {e0, e1}});
}

void prof_resolve(edus_handle* h) {
    for (auto& pe : h->prof_pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, pe.second.first, pe.second.second) == cudaSuccess) {
            h->prof_ms[pe.first] += ms;
            h->prof_n[pe.first] += 1;
        }
        h->prof_pool.push_back(pe.second.first);
        h->prof_pool.push_back(pe.second.second);
    }
    h->prof_pending.clear();
}

// gradient_space "k" (kGradient_definitions.hpp:18-30): G[b][p][k] =
// sum_i w_i (b_i.E) rho[b][p][k + b_i], k + b_i folded into the grid.  The
// coefficients of the CTA's solve are formed once in shared memory.
__global__ void kgradient_kernel(const double2* __restrict__ rho, long long in_bstride, double2* __restrict__ G,
                                 long long out_bstride, const int* __restrict__ shift, const double* __restrict__ coef,
                                 int n,
                                 const StageField* __restrict__ field, int N0, int N1, int N2, int P) {
    extern __shared__ double kc[];  // [n] coefficients
    int* ks = reinterpret_cast<int*>(kc + n);  // [n][3] shifts
    const int b = blockIdx.y;
    const StageField F = field[b];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        kc[i] = coef[4 * i + 3] * (coef[4 * i] * F.E[0] + coef[4 * i + 1] * F.E[1] + coef[4 * i + 2] * F.E[2]);
        ks[3 * i] = shift[3 * i];
        ks[3 * i + 1] = shift[3 * i + 1];
        ks[3 * i + 2] = shift[3 * i + 2];
    }
    __syncthreads();
    const int Nk = N0 * N1 * N2;
    const long long total = (long long)P * Nk;
    const double2* src = rho + (long long)b * in_bstride;
    double2* dst = G + (long long)b * out_bstride;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(e / Nk), k = (int)(e - (long long)p * Nk);
        const int j2 = k % N2, j1 = (k / N2) % N1, j0 = k / (N1 * N2);
        const double2* plane = src + (long long)p * Nk;
        double2 acc = make_double2(0.0, 0.0);
        for (int i = 0; i < n; ++i) {
            const double c = kc[i];
            if (c == 0.0) continue;
            int a0 = j0 + ks[3 * i], a1 = j1 + ks[3 * i + 1], a2 = j2 + ks[3 * i + 2];
            a0 -= a0 >= N0 ? N0 : 0;
            a1 -= a1 >= N1 ? N1 : 0;
            a2 -= a2 >= N2 ? N2 : 0;
            const double2 v = __ldg(&plane[(a0 * N1 + a1) * N2 + a2]);
            acc.x += c * v.x;
            acc.y += c * v.y;
        }
        dst[e] = acc;
    }
}

template <bool COUL, int MASK, int MAXT>
void launch_plane_variant(edus_handle* h, dim3 grid, const double2* in, long long in_bstride, double2* G,
                          double2* Hee, long long out_bstride, const StageField* field, int nS,
                          const double2* ptab = nullptr) {
    plane_rhs_kernel<COUL, MASK, MAXT><<<grid, h->plane_cfg.threads, h->smem_plane, h->stream>>>(
        in, in_bstride, G, Hee, out_bstride, h->rho0p, h->Wp, h->diag0, field, h->roots, h->rpos, h->plan, h->nb,
        1.0 / h->Nk, h->hpos, h->hval, nS, ptab, h->ntab);
}

template <bool COUL, int MASK, int MAXT, int BT = 1>
void launch_plane_persist(edus_handle* h, int nplanes, const double2* in, long long in_bstride, double2* G,
                          double2* Hee, long long out_bstride, const StageField* field, int nS,
                          const double2* ptab = nullptr) {
    const int grid = std::min(nplanes, h->plane_grid);
    const size_t smem = h->Nk * sizeof(double2) + 16 + h->tab_smem;
    // 2-D grids in the length gauge: the row-wise kernel (warps own rows of
    // the unit-stride axis; fewer CTA barriers, bitwise the same results)
    if (h->hplanes)
        plane_rhs_persist_kernel<COUL, MASK, MAXT, BT, true, true><<<grid, h->plane_cfg.threads, smem, h->stream>>>(
            in, in_bstride, G, Hee, out_bstride, h->rho0p, h->Wp, h->diag0, field, h->roots, h->rpos, h->plan, h->nb,
            1.0 / h->Nk, h->plane_scratch, nplanes, h->hpos, h->hval, nS, h->opos, h->oval, COUL ? h->nO : 0, ptab,
            h->ntab, h->flag, h->wait_polls, h->nroot_s, h->nrpos_s, h->upair);
    else if (h->rows_ok && !ptab)
        plane_rhs_persist_kernel<COUL, MASK, MAXT, BT, true><<<grid, h->plane_cfg.threads, smem, h->stream>>>(
            in, in_bstride, G, Hee, out_bstride, h->rho0p, h->Wp, h->diag0, field, h->roots, h->rpos, h->plan, h->nb,
            1.0 / h->Nk, h->plane_scratch, nplanes, h->hpos, h->hval, nS, h->opos, h->oval, COUL ? h->nO : 0, ptab,
            h->ntab, h->flag, h->wait_polls, h->nroot_s, h->nrpos_s);
    else
        plane_rhs_persist_kernel<COUL, MASK, MAXT, BT><<<grid, h->plane_cfg.threads, smem, h->stream>>>(
            in, in_bstride, G, Hee, out_bstride, h->rho0p, h->Wp, h->diag0, field, h->roots, h->rpos, h->plan, h->nb,
            1.0 / h->Nk, h->plane_scratch, nplanes, h->hpos, h->hval, nS, h->opos, h->oval, COUL ? h->nO : 0, ptab,
            h->ntab, h->flag, h->wait_polls, h->nroot_s, h->nrpos_s);
}

// The three plane3 launches (rows, columns, rows) of one right-hand side.
template <int MASK>
void launch_plane3(edus_handle* h, const double2* in, long long in_bstride, double2* G, double2* Hee,
                   long long out_bstride, const StageField* field, int nbatch, int nS, bool c) {
    const int planes = h->P * nbatch;
    const int N0 = h->N[0], N1 = h->N[1];
    const long long bs = (long long)h->S;
    dim3 gr(planes, N0 / h->p3.Rc), gc(planes, N1 / h->p3.Cc), gi(planes * (c ? 2 : 1), N0 / h->p3.Rc);
    const size_t smr = (size_t)h->p3.Rc * N1 * sizeof(double2);
    const size_t smc = (size_t)N0 * h->p3.Cc * sizeof(double2) * (c ? 2 : 1);
    plane3_rows_kernel<true, 256, MASK><<<gr, 128, smr, h->stream>>>(in, in_bstride, h->s3a, bs, h->P, h->p3.rows,
                                                                     1, h->roots, in, h->s3a);
    if (c)
        plane3_cols_kernel<true, 256, MASK><<<gc, 128, smc, h->stream>>>(
            h->s3a, bs, h->s3g, h->s3h, h->rho0p, h->Wp, h->diag0, field, h->roots, h->rpos, h->plan, h->p3.cols,
            h->p3.Cc, h->nb, 1.0 / h->Nk, h->hpos, h->hval, nS);
    else
        plane3_cols_kernel<false, 256, MASK><<<gc, 128, smc, h->stream>>>(
            h->s3a, bs, h->s3g, h->s3h, h->rho0p, h->Wp, h->diag0, field, h->roots, h->rpos, h->plan, h->p3.cols,
            h->p3.Cc, h->nb, 1.0 / h->Nk, h->hpos, h->hval, 0);
    plane3_rows_kernel<false, 256, MASK><<<gi, 128, smr, h->stream>>>(h->s3g, bs, G, out_bstride, h->P, h->p3.rows,
                                                                      c ? 2 : 1, h->roots, h->s3h, Hee);
}

// fuse: with HSEX and a sparse model, Hee receives the whole Hamiltonian
// H0 + E.xi + Hee (plane kernel) and the commutator reads only it.
int launch_split(edus_handle* h, const double2* in, double2* G, double2* H, const StageField* field, int nbatch) {
    SplitArgs a{};
    a.rho = in;
    a.rref = h->sref;
    a.bstride = (long long)h->S;
    a.nplanes = h->P * nbatch;
    a.G = G;
    a.H = H;
    for (int d = 0; d < 3; ++d) {
        a.Gref[d] = h->sGref[d];
        a.xi[d] = h->xi[d];
    }
    a.Hfix = h->sHfix;
    a.W32 = h->W32;
    a.refdiag0 = h->srefdiag0;
    a.diag0 = h->diag0;
    a.field = field;
    a.roots = h->roots;
    a.rpos = h->rpos;
    a.scratch = h->split_scratch;
    a.nb = h->nb;
    a.inv_nk = 1.0 / h->Nk;
    const int grid = std::min(a.nplanes, h->split_grid);
    const size_t sm = (size_t)h->Nk * sizeof(float2);
    const bool c = h->d.coulomb != 0;
    if (h->plane_cfg.variant == 1) {
        if (c) plane_split_kernel<true, kRadix89, 384><<<grid, h->split_threads, sm, h->stream>>>(a, h->plan);
        else plane_split_kernel<false, kRadix89, 384><<<grid, h->split_threads, sm, h->stream>>>(a, h->plan);
    } else {
        if (c) plane_split_kernel<true, kRadixAll, 256><<<grid, h->split_threads, sm, h->stream>>>(a, h->plan);
        else plane_split_kernel<false, kRadixAll, 256><<<grid, h->split_threads, sm, h->stream>>>(a, h->plan);
    }
    return EDUS_OK;
}

int launch_plane(edus_handle* h, const double2* in, long long in_bstride, double2* G, double2* Hee,
                 long long out_bstride, const StageField* field, int nbatch, bool fuse = true) {
    dim3 grid(h->P, nbatch);
    cudaEvent_t e0;
    prof_begin(h, &e0);
    const bool c = h->d.coulomb != 0;
    const int nS = (fuse && c) ? h->nS : 0;
    // gradient_space "k": the stencil kernel writes G; without HSEX it is the
    // only launch, with HSEX it follows the plane kernel (whose g is zero)
    const bool kmode = h->kg_n > 0 && !h->split && !h->packed;
    auto launch_kgrad = [&]() {
        const long long total = (long long)h->P * h->Nk;
        dim3 kg((unsigned)std::min<long long>((total + 255) / 256, 148LL * 16), nbatch);
        kgradient_kernel<<<kg, 256, h->kg_n * (sizeof(double) + 3 * sizeof(int)), h->stream>>>(
            in, in_bstride, G, out_bstride, h->kg_shift, h->kg_coef, h->kg_n, field, h->N[0], h->N[1], h->N[2], h->P);
        h->launches++;
    };
    if (h->peierls) {
        // Peierls gauge: the stage's phase tables, then H alone (G stays zero)
        peierls_phase_kernel<<<nbatch, 128, 0, h->stream>>>(field, h->rpos, h->plan, h->ntab, h->ptab);
        h->launches++;
        const int np = h->P * nbatch;
        if (h->plane_cfg.persist) {
            if (h->plane_cfg.variant == 1) {
                if (c) launch_plane_persist<true, kRadix89, kPersist89Threads, kPersist89Batch>(h, np, in, in_bstride, G, Hee, out_bstride, field, h->nS, h->ptab);
                else launch_plane_persist<false, kRadix89, kPersist89Threads, kPersist89Batch>(h, np, in, in_bstride, G, Hee, out_bstride, field, h->nS, h->ptab);
            } else {
                if (h->plane_cfg.variant == 2) {
                    if (c) launch_plane_persist<true, kRadixAll, 256>(h, np, in, in_bstride, G, Hee, out_bstride, field, h->nS, h->ptab);
                    else launch_plane_persist<false, kRadixAll, 256>(h, np, in, in_bstride, G, Hee, out_bstride, field, h->nS, h->ptab);
                } else {
                    if (c) launch_plane_persist<true, kRadixCommon, 256>(h, np, in, in_bstride, G, Hee, out_bstride, field, h->nS, h->ptab);
                    else launch_plane_persist<false, kRadixCommon, 256>(h, np, in, in_bstride, G, Hee, out_bstride, field, h->nS, h->ptab);
                }
            }
        } else if (h->plane_cfg.variant == 1) {
            if (c) launch_plane_variant<true, kRadix89, 768>(h, grid, in, in_bstride, G, Hee, out_bstride, field, h->nS, h->ptab);
            else launch_plane_variant<false, kRadix89, 768>(h, grid, in, in_bstride, G, Hee, out_bstride, field, h->nS, h->ptab);
        } else {
            if (h->plane_cfg.variant == 2) {
                if (c) launch_plane_variant<true, kRadixAll, 512>(h, grid, in, in_bstride, G, Hee, out_bstride, field, h->nS, h->ptab);
                else launch_plane_variant<false, kRadixAll, 512>(h, grid, in, in_bstride, G, Hee, out_bstride, field, h->nS, h->ptab);
            } else {
                if (c) launch_plane_variant<true, kRadixCommon, 512>(h, grid, in, in_bstride, G, Hee, out_bstride, field, h->nS, h->ptab);
                else launch_plane_variant<false, kRadixCommon, 512>(h, grid, in, in_bstride, G, Hee, out_bstride, field, h->nS, h->ptab);
            }
        }
        h->launches++;
        CU(h, cudaGetLastError());
        prof_end(h, 0, e0);
        return EDUS_OK;
    }
    if (kmode && !c) {
        launch_kgrad();
        CU(h, cudaGetLastError());
        prof_end(h, 0, e0);
        return EDUS_OK;
    }
    if (h->split && fuse) {
        launch_split(h, in, G, Hee, field, nbatch);
        h->launches++;
        CU(h, cudaGetLastError());
        prof_end(h, 0, e0);
        return EDUS_OK;
    }
    if (h->use3 && h->nO == 0) {
        // rows (k -> R, axis 1), columns (axis 0 both ways + pointwise), rows (R -> k)
        if (h->plane_cfg.variant == 2)
            launch_plane3<kRadixAll>(h, in, in_bstride, G, Hee, out_bstride, field, nbatch, nS, c);
        else
            launch_plane3<kRadixCommon>(h, in, in_bstride, G, Hee, out_bstride, field, nbatch, nS, c);
        h->launches += 3;
        if (kmode) launch_kgrad();
        CU(h, cudaGetLastError());
        prof_end(h, 0, e0);
        return EDUS_OK;
    }
    if (h->plane_cfg.persist) {
        const int np = (h->hplanes ? h->Pu : h->P) * nbatch;
        if (h->plane_cfg.variant == 1) {
            if (c) launch_plane_persist<true, kRadix89, kPersist89Threads, kPersist89Batch>(h, np, in, in_bstride, G, Hee, out_bstride, field, nS);
            else launch_plane_persist<false, kRadix89, kPersist89Threads, kPersist89Batch>(h, np, in, in_bstride, G, Hee, out_bstride, field, nS);
        } else if (h->plane_cfg.variant == 2) {
            if (c) launch_plane_persist<true, kRadixAll, 256>(h, np, in, in_bstride, G, Hee, out_bstride, field, nS);
            else launch_plane_persist<false, kRadixAll, 256>(h, np, in, in_bstride, G, Hee, out_bstride, field, nS);
        } else {
            if (c) launch_plane_persist<true, kRadixCommon, 256>(h, np, in, in_bstride, G, Hee, out_bstride, field, nS);
            else launch_plane_persist<false, kRadixCommon, 256>(h, np, in, in_bstride, G, Hee, out_bstride, field, nS);
        }
    } else if (h->plane_cfg.variant == 1) {
        if (c) launch_plane_variant<true, kRadix89, 768>(h, grid, in, in_bstride, G, Hee, out_bstride, field, nS);
        else launch_plane_variant<false, kRadix89, 768>(h, grid, in, in_bstride, G, Hee, out_bstride, field, nS);
    } else if (h->plane_cfg.variant == 2) {
        if (c) launch_plane_variant<true, kRadixAll, 512>(h, grid, in, in_bstride, G, Hee, out_bstride, field, nS);
        else launch_plane_variant<false, kRadixAll, 512>(h, grid, in, in_bstride, G, Hee, out_bstride, field, nS);
    } else {
        if (c) launch_plane_variant<true, kRadixCommon, 512>(h, grid, in, in_bstride, G, Hee, out_bstride, field, nS);
        else launch_plane_variant<false, kRadixCommon, 512>(h, grid, in, in_bstride, G, Hee, out_bstride, field, nS);
    }
    h->launches++;
    if (kmode) launch_kgrad();
    CU(h, cudaGetLastError());
    prof_end(h, 0, e0);
    return EDUS_OK;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda)
PFN_cuTensorMapEncodeTiled tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(p);
    });
    return fn;
}

// The [nbatch][P][Nk] complex array at `base` as the 4-D tensor
// {2 Nk, nb, nb, nbatch} of doubles, box {2 TKU, nb, nb, 1} (padded = false:
// the update operands, 4 k points) or {2 TK, W, nb, 1} (padded = true: the
// product operands, 2 k points, rows of odd length W; the copy zero-fills a
// column beyond nb).
const CUtensorMap* operand_map(edus_handle* h, const void* base, int nbatch, bool padded) {
    const auto key = std::make_pair(base, 2 * nbatch + (padded ? 1 : 0));
    auto it = h->tmaps.find(key);
    if (it != h->tmaps.end()) return &it->second;
    PFN_cuTensorMapEncodeTiled enc = tensor_map_encoder();
    if (!enc) return nullptr;
    const WsGeom g = ws_geometry(h->nb);
    const cuuint64_t nb = (cuuint64_t)h->nb, Nk = (cuuint64_t)h->Nk;
    const cuuint64_t dims[4] = {2 * Nk, nb, nb, (cuuint64_t)nbatch};
    const cuuint64_t strides[3] = {Nk * 16, nb * Nk * 16, nb * nb * Nk * 16};
    cuuint32_t box[4] = {(cuuint32_t)(2 * g.TKU), (cuuint32_t)nb, (cuuint32_t)nb, 1};
    if (padded) {
        box[0] = (cuuint32_t)(2 * g.TK);
        box[1] = (cuuint32_t)g.W;
    }
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    CUtensorMap m;
    const CUresult r = enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<void*>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return nullptr;
    return &(h->tmaps[key] = m);
}

template <int MODE>
int launch_ws(edus_handle* h, const StageArgs& a, int nbatch) {
    const WsGeom g = ws_geometry(h->nb);
    const int ntiles = ((h->Nk + g.TKU - 1) / g.TKU) * nbatch;  // update tiles
    const int grid = std::min(ntiles, h->ws_grid);
    OperandMaps maps;
    const void* src[5] = {a.Hee, a.rho, a.G, a.y ? (const void*)a.y : (const void*)a.G,
                          a.acc ? (const void*)a.acc : (const void*)a.G};
    for (int i = 0; i < 5; ++i) {
        const CUtensorMap* m = operand_map(h, src[i], nbatch, i < 2);
        if (!m) return fail(h, EDUS_ERR_CUDA, "cuTensorMapEncodeTiled failed for a commutator operand");
        maps.m[i] = *m;
    }
    if (g.tiles == 2)
        commutator_ws_kernel<MODE, 2, 4><<<grid, g.threads, g.smem, h->stream>>>(a, nbatch, maps, h->flag);
    else if (g.SM == 3)
        commutator_ws_kernel<MODE, 3, 3><<<grid, g.threads, g.smem, h->stream>>>(a, nbatch, maps, h->flag);
    else
        commutator_ws_kernel<MODE, 3, 2><<<grid, g.threads, g.smem, h->stream>>>(a, nbatch, maps, h->flag);
    return EDUS_OK;
}

template <int MODE>
int launch_comm_mode(edus_handle* h, const StageArgs& a, int nbatch, bool fuse) {
    dim3 grid((h->Nk + h->TK - 1) / h->TK, nbatch);
    cudaEvent_t e0;
    prof_begin(h, &e0);
    // fused Hamiltonian: Hee holds the whole H (with HSEX and a sparse model,
    // and always in the Peierls gauge)
    const bool fh = fuse && ((h->d.coulomb && (h->nS > 0 || h->split)) || h->peierls);
    if (fh && h->comm_ws) {
        int rc;
        if ((rc = launch_ws<MODE>(h, a, nbatch))) return rc;
    } else if (fh && !h->d.coulomb) {
        if (h->comm_mma)
            commutator_mma_kernel<MODE, false, true><<<grid, h->comm_threads, h->smem_comm, h->stream>>>(a);
        else
            commutator_kernel<MODE, false, true><<<grid, h->comm_threads, h->smem_comm, h->stream>>>(a);
    } else if (h->comm_mma) {
        if (fh)
            commutator_mma_kernel<MODE, true, true><<<grid, h->comm_threads, h->smem_comm, h->stream>>>(a);
        else if (h->d.coulomb)
            commutator_mma_kernel<MODE, true><<<grid, h->comm_threads, h->smem_comm, h->stream>>>(a);
        else
            commutator_mma_kernel<MODE, false><<<grid, h->comm_threads, h->smem_comm, h->stream>>>(a);
    } else {
        if (fh)
            commutator_kernel<MODE, true, true><<<grid, h->comm_threads, h->smem_comm, h->stream>>>(a);
        else if (h->d.coulomb)
            commutator_kernel<MODE, true><<<grid, h->comm_threads, h->smem_comm, h->stream>>>(a);
        else
            commutator_kernel<MODE, false><<<grid, h->comm_threads, h->smem_comm, h->stream>>>(a);
    }
    h->launches++;
    CU(h, cudaGetLastError());
    prof_end(h, 1, e0);
    return EDUS_OK;
}

int launch_comm(edus_handle* h, int mode, const StageArgs& a, int nbatch, bool fuse = true) {
    switch (mode) {
        case MODE_RHS: return launch_comm_mode<MODE_RHS>(h, a, nbatch, fuse);
        case MODE_RK1: return launch_comm_mode<MODE_RK1>(h, a, nbatch, fuse);
        case MODE_RK2: return launch_comm_mode<MODE_RK2>(h, a, nbatch, fuse);
        case MODE_RK3: return launch_comm_mode<MODE_RK3>(h, a, nbatch, fuse);
        case MODE_RK4: return launch_comm_mode<MODE_RK4>(h, a, nbatch, fuse);
        case MODE_AB: return launch_comm_mode<MODE_AB>(h, a, nbatch, fuse);
    }
    return fail(h, EDUS_ERR_ARG, "bad stage mode");
}

// The dynamic shared-memory limit is a process-wide attribute of each kernel:
// every handle sets it to the device's opt-in maximum, so that a handle
// created later (whatever its sizes) never lowers it below what an earlier
// handle launches with.  `bytes` is what this handle needs.
int device_smem_optin(int device) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    return v;
}

template <typename K>
int set_smem(edus_handle* h, K kernel, int bytes) {
    const int lim = device_smem_optin(h->d.device);
    if (bytes > lim)
        return fail(h, EDUS_ERR_UNSUPPORTED,
                    "needs " + std::to_string(bytes) + " B of shared memory per CTA (device: " + std::to_string(lim) + ")");
    CU(h, cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    return EDUS_OK;
}

StageArgs base_args(edus_handle* h) {
    StageArgs a{};
    a.H0 = h->per_solve ? h->H0b : h->H0;
    for (int d = 0; d < 3; ++d) a.xi[d] = h->per_solve ? h->xib[d] : h->xi[d];
    a.mstride = h->per_solve ? (long long)h->S : 0;
    a.Hee = h->Hee;
    a.G = h->G;
    a.hartree = h->hartree;
    a.rho0diag = h->rho0diag;
    a.diag0 = h->diag0;
    a.bstride = (long long)h->S;
    a.Nk = h->Nk;
    a.nb = h->nb;
    a.TK = h->TK;
    return a;
}


// ---------------------------------------------------------------------------
// packed-Hermitian forms: launch helpers

template <typename C, typename IT, bool COUL>
void pplane_t(edus_handle* h, const IT* in, const StageField* field, int nbatch) {
    dim3 grid(h->Pq, nbatch);
    using T = typename CplxT<C>::T;
    const long long bs = (long long)h->Sq;
    if (h->pplane_variant == 1)
        plane_packed_kernel<C, IT, kRadix89, 512, COUL><<<grid, h->pplane_threads, h->pplane_smem, h->stream>>>(
            in, bs, (C*)h->pG, (C*)h->pE1, bs, (const T*)h->pW, h->pdiag0, field, h->roots, h->rpos, h->plan, h->qnm,
            h->nb, 1.0 / h->Nk);
    else
        plane_packed_kernel<C, IT, kRadixAll, 512, COUL><<<grid, h->pplane_threads, h->pplane_smem, h->stream>>>(
            in, bs, (C*)h->pG, (C*)h->pE1, bs, (const T*)h->pW, h->pdiag0, field, h->roots, h->rpos, h->plan, h->qnm,
            h->nb, 1.0 / h->Nk);
}

// in_is_aux: the input is the RK stage input (FP32 in MIXED), else the FP64 state
int launch_pplane(edus_handle* h, const void* in, bool in_is_aux, const StageField* field, int nbatch) {
    cudaEvent_t e0;
    prof_begin(h, &e0);
    const bool c = h->d.coulomb != 0;
    if (h->mixed) {
        if (in_is_aux) {
            if (c) pplane_t<float2, float2, true>(h, (const float2*)in, field, nbatch);
            else pplane_t<float2, float2, false>(h, (const float2*)in, field, nbatch);
        } else {
            if (c) pplane_t<float2, double2, true>(h, (const double2*)in, field, nbatch);
            else pplane_t<float2, double2, false>(h, (const double2*)in, field, nbatch);
        }
    } else {
        if (c) pplane_t<double2, double2, true>(h, (const double2*)in, field, nbatch);
        else pplane_t<double2, double2, false>(h, (const double2*)in, field, nbatch);
    }
    h->launches++;
    CU(h, cudaGetLastError());
    prof_end(h, 0, e0);
    return EDUS_OK;
}

template <int MODE, bool COUL, typename ST, typename IT, typename AT>
void pcomm_t(edus_handle* h, const PackedArgs& a, int nbatch) {
    dim3 grid((h->Nk + h->pgeo.TK - 1) / h->pgeo.TK, nbatch);
    commutator_packed_kernel<MODE, COUL, ST, IT, AT><<<grid, 256, h->pgeo.smem, h->stream>>>(a);
}

template <int MODE, bool COUL>
void pcomm_mode(edus_handle* h, const PackedArgs& a, int nbatch) {
    if (h->mixed) {
        // RK stage 1 and AB read the FP64 state; RK stages 2-4 read the FP32 stage input
        if (MODE == MODE_RK1 || MODE == MODE_AB || MODE == MODE_RHS)
            pcomm_t<MODE, COUL, float2, double2, float2>(h, a, nbatch);
        else
            pcomm_t<MODE, COUL, float2, float2, float2>(h, a, nbatch);
    } else {
        pcomm_t<MODE, COUL, double2, double2, double2>(h, a, nbatch);
    }
}

int launch_pcomm(edus_handle* h, int mode, const PackedArgs& a, int nbatch) {
    cudaEvent_t e0;
    prof_begin(h, &e0);
    const bool c = h->d.coulomb != 0;
#define PC(M)                                          \
    case M:                                            \
        if (c) pcomm_mode<M, true>(h, a, nbatch);      \
        else pcomm_mode<M, false>(h, a, nbatch);       \
        break;
    switch (mode) {
        PC(MODE_RK1) PC(MODE_RK2) PC(MODE_RK3) PC(MODE_RK4) PC(MODE_AB)
        default: return fail(h, EDUS_ERR_ARG, "bad packed stage mode");
    }
#undef PC
    h->launches++;
    CU(h, cudaGetLastError());
    prof_end(h, 1, e0);
    return EDUS_OK;
}

template <typename K>
int set_smem_any(edus_handle* h, K kernel, size_t bytes) {
    return set_smem(h, kernel, (int)bytes);
}

template <int MODE, bool COUL>
int set_pcomm_smem(edus_handle* h) {
    int rc;
    if ((rc = set_smem_any(h, commutator_packed_kernel<MODE, COUL, float2, double2, float2>, h->pgeo.smem))) return rc;
    if ((rc = set_smem_any(h, commutator_packed_kernel<MODE, COUL, float2, float2, float2>, h->pgeo.smem))) return rc;
    if ((rc = set_smem_any(h, commutator_packed_kernel<MODE, COUL, double2, double2, double2>, h->pgeo.smem))) return rc;
    return EDUS_OK;
}

template <typename C, typename IT, bool COUL>
int set_pplane_smem(edus_handle* h) {
    int rc;
    if ((rc = set_smem_any(h, plane_packed_kernel<C, IT, kRadix89, 512, COUL>, h->pplane_smem))) return rc;
    if ((rc = set_smem_any(h, plane_packed_kernel<C, IT, kRadixAll, 512, COUL>, h->pplane_smem))) return rc;
    return EDUS_OK;
}

int packed_setup_smem(edus_handle* h) {
    int rc;
#define SP(M)                                                   \
    if ((rc = set_pcomm_smem<M, true>(h))) return rc;           \
    if ((rc = set_pcomm_smem<M, false>(h))) return rc;
    SP(MODE_RK1) SP(MODE_RK2) SP(MODE_RK3) SP(MODE_RK4) SP(MODE_AB)
#undef SP
    if ((rc = set_pplane_smem<float2, double2, true>(h))) return rc;
    if ((rc = set_pplane_smem<float2, double2, false>(h))) return rc;
    if ((rc = set_pplane_smem<float2, float2, true>(h))) return rc;
    if ((rc = set_pplane_smem<float2, float2, false>(h))) return rc;
    if ((rc = set_pplane_smem<double2, double2, true>(h))) return rc;
    if ((rc = set_pplane_smem<double2, double2, false>(h))) return rc;
    return EDUS_OK;
}

int grid_for(long long n) { return (int)std::min<long long>((n + 255) / 256, 148LL * 8); }

// rho_ref := the full-plane state y[b]; C0, K_d, H0' from the FP64 full-plane
// kernels, then packed (and rounded to the storage type).
// H0(R) and xi_d(R) (k -> R transforms of the uploaded k arrays, as the
// reference's go_to_R, Operator.hpp:566-586) on the lattice vectors where any
// of them is non-zero, for the fused Hamiltonian of the HSEX plane kernel.
// Entries below 1e-13 of an array's largest are transform rounding of zeros
// and are dropped.  More than kMaxSparseR positions (a model dense in R): the
// commutator assembles H from the k arrays instead.
constexpr int kMaxSparseR = 4096;

int build_sparse_model(edus_handle* h) {
    h->nS = 0;
    const int P = h->P, Nk = h->Nk;
    const size_t S = h->S;
    double2* tmp = nullptr;
    CU(h, cudaMalloc((void**)&tmp, 4 * S * sizeof(double2)));
    const double2* src[4] = {h->H0, h->xi[0], h->xi[1], h->xi[2]};
    for (int a = 0; a < 4; ++a)
        plane_to_R_kernel<kRadixAll, 256><<<P, 256, Nk * sizeof(double2), h->stream>>>(src[a], tmp + a * S, h->roots,
                                                                                     h->plan, 1.0 / Nk);
    h->launches += 4;
    std::vector<double2> hv(4 * S);
    const cudaError_t e1 = cudaGetLastError();
    const cudaError_t e2 = cudaMemcpyAsync(hv.data(), tmp, 4 * S * sizeof(double2), cudaMemcpyDeviceToHost, h->stream);
    const cudaError_t e3 = cudaStreamSynchronize(h->stream);
    cudaFree(tmp);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess)
        return fail(h, EDUS_ERR_CUDA, "k -> R transform of the model failed");
    double mx[4] = {0, 0, 0, 0};
    for (int a = 0; a < 4; ++a)
        for (size_t i = 0; i < S; ++i) mx[a] = std::max(mx[a], std::hypot(hv[a * S + i].x, hv[a * S + i].y));
    std::vector<int> pos;
    for (int q = 0; q < Nk; ++q) {
        bool keep = false;
        for (int a = 0; a < 4 && !keep; ++a)
            for (int p = 0; p < P && !keep; ++p) {
                const double2 v = hv[a * S + (size_t)p * Nk + q];
                keep = std::hypot(v.x, v.y) > 1e-13 * mx[a];
            }
        if (keep) pos.push_back(q);
        if ((int)pos.size() > kMaxSparseR) return EDUS_OK;  // dense: unfused path
    }
    const int nS = (int)pos.size();
    if (nS == 0) return EDUS_OK;
    std::vector<double2> vals(4 * (size_t)P * nS);
    for (int a = 0; a < 4; ++a)
        for (int p = 0; p < P; ++p)
            for (int s2 = 0; s2 < nS; ++s2) vals[((size_t)a * P + p) * nS + s2] = hv[a * S + (size_t)p * Nk + pos[s2]];
    int rc;
    if (!h->hpos) {
        if ((rc = dalloc(h, (void**)&h->hpos, kMaxSparseR * sizeof(int)))) return rc;
        if ((rc = dalloc(h, (void**)&h->hval, 4 * (size_t)P * kMaxSparseR * sizeof(double2)))) return rc;
    }
    CU(h, cudaMemcpyAsync(h->hpos, pos.data(), nS * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    CU(h, cudaMemcpyAsync(h->hval, vals.data(), vals.size() * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
    CU(h, cudaStreamSynchronize(h->stream));
    h->nS = nS;
    return EDUS_OK;
}

// Split-precision anchor: rho_ref = the current state of every solve, and its
// FP64 terms grad_d rho_ref (unit field along d), H0 + Hee(rho_ref) and
// rho_ref,nn(R=0), by the FP64 plane kernel.
int anchor_split(edus_handle* h) {
    int rc;
    const size_t SBb = h->S * sizeof(double2) * h->B;
    const long long bs = (long long)h->S;
    CU(h, cudaMemcpyAsync(h->sref, h->y, SBb, cudaMemcpyDeviceToDevice, h->stream));
    const bool prof = h->profiling;
    h->profiling = false;  // keep the anchor out of the per-kernel timings
    for (int d = 0; d < 3; ++d) {
        rc = launch_plane(h, h->sref, bs, h->sGref[d], h->Hee, bs, h->unit_fields + (size_t)d * h->B, h->B, false);
        if (rc) {
            h->profiling = prof;
            return rc;
        }
        if (d == 0 && h->d.coulomb) {
            add_broadcast_kernel<<<grid_for(bs * h->B), 256, 0, h->stream>>>(h->H0, h->Hee, h->sHfix, bs, h->B);
            h->launches++;
            CU(h, cudaMemcpyAsync(h->srefdiag0, h->diag0, (size_t)h->B * h->nb * sizeof(double2),
                                  cudaMemcpyDeviceToDevice, h->stream));
        }
    }
    h->profiling = prof;
    CU(h, cudaGetLastError());
    h->anchored = true;
    h->since_anchor = 0;
    return EDUS_OK;
}

// One CTA per k point: contributions of that k to the Bloch populations
// Re (U^dagger rho U)_nn, the Wannier populations Re rho_nn and tr(v_d rho),
// accumulated in acc[0..nb) (Bloch), acc[nb..2nb) (Wannier), acc[2nb..2nb+6)
// (re, im of d = 0, 1, 2).  Shared memory: rho_k and U_k, [n][m].
// Peierls gauge, observables (Simulation.cpp:447-449, 593-595): the state
// that the populations and the velocity see is rho(R) e^{-iA.R} back in k,
// one plane per CTA: dst = FFT_{+1}(FFT_{-1}(src) e^{-iA.R} / Nk).
template <int MASK, int MAXT>
__global__ void __launch_bounds__(MAXT) peierls_shift_kernel(const double2* __restrict__ src, double2* __restrict__ dst,
                                                             const double2* __restrict__ tb,
                                                             const double2* __restrict__ roots, PlanePlan pl,
                                                             double inv_nk) {
    extern __shared__ double2 xs[];
    const int Nk = pl.Nk;
    const long long off = (long long)blockIdx.x * Nk;
    for (int i = threadIdx.x; i < Nk; i += blockDim.x) xs[i] = __ldg(&src[off + i]);
    __syncthreads();
    plane_forward<1, MASK>(xs, 0, pl, roots);
    for (int j = threadIdx.x; j < Nk; j += blockDim.x) {
        const double2 e = peierls_phase_at(tb, pl, j);
        xs[j] = cmul(cscale(xs[j], inv_nk), make_double2(e.x, -e.y));
    }
    __syncthreads();
    plane_inverse<1, MASK>(xs, 0, pl, roots);
    for (int i = threadIdx.x; i < Nk; i += blockDim.x) dst[off + i] = xs[i];
}

__global__ void observables_kernel(const double2* __restrict__ rho, const double2* __restrict__ U,
                                   const double2* __restrict__ v0, const double2* __restrict__ v1,
                                   const double2* __restrict__ v2, int Nk, int nb, double* __restrict__ acc) {
    extern __shared__ double2 so[];
    const int k = blockIdx.x, P = nb * nb;
    double2* R = so;
    double2* Us = so + P;
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        R[p] = rho[(long long)p * Nk + k];
        Us[p] = U ? U[(long long)p * Nk + k] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    for (int n = threadIdx.x; n < nb; n += blockDim.x) {
        if (U) {
            double bl = 0.0;
            for (int i = 0; i < nb; ++i) {
                double2 t = make_double2(0.0, 0.0);
                for (int j = 0; j < nb; ++j) t = cadd(t, cmul(R[i * nb + j], Us[j * nb + n]));
                const double2 u = Us[i * nb + n];
                bl += u.x * t.x + u.y * t.y;  // Re(conj(u) t)
            }
            atomicAdd(&acc[n], bl);
        }
        atomicAdd(&acc[nb + n], R[n * nb + n].x);
    }
    if (!v0) return;
    const double2* vs[3] = {v0, v1, v2};
    double part[6] = {0, 0, 0, 0, 0, 0};
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        const int n = p / nb, l = p - (p / nb) * nb;
        const double2 r = R[l * nb + n];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double2 c = cmul(vs[d][(long long)p * Nk + k], r);
            part[2 * d] += c.x;
            part[2 * d + 1] += c.y;
        }
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        double v = part[q];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if ((threadIdx.x & 31) == 0) atomicAdd(&acc[2 * nb + q], v);
    }
}

// plane position (digit-reversed order) of the natural R index (j0 N1 + j1) N2 + j2
int position_of(const edus_handle* h, int iR) {
    const int j2 = iR % h->N[2], j1 = (iR / h->N[2]) % h->N[1], j0 = iR / (h->N[1] * h->N[2]);
    return (h->posof[0][j0] * h->N[1] + h->posof[1][j1]) * h->N[2] + h->posof[2][j2];
}

// out[s][p] = planes[p][pos[s]]
__global__ void gather_R_kernel(const double2* __restrict__ planes, const int* __restrict__ pos, int nsel, int P,
                                int Nk, double2* __restrict__ out) {
    const long long total = (long long)nsel * P;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(i / P), p = (int)(i - (long long)s * P);
        out[i] = planes[(long long)p * Nk + pos[s]];
    }
}

// Device status word: a bounded wait that ran out inside a kernel sets it
// (the TMA commutator's operand hand-over, the plane kernel's bulk load).  It
// is cleared once reported, so the handle stays usable: the results of the
// calls since the last check are not to be trusted, later calls are.
int check_status(edus_handle* h) {
    int v = 0;
    CU(h, cudaMemcpyAsync(&v, h->flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CU(h, cudaStreamSynchronize(h->stream));
    if (v) {
        CU(h, cudaMemsetAsync(h->flag, 0, sizeof(int), h->stream));
        return fail(h, EDUS_ERR_TIMEOUT,
                    "a bounded wait in a kernel ran out (commutator_ws_kernel operand hand-over or "
                    "plane_rhs_persist_kernel bulk load): the results since the last synchronising call are invalid");
    }
    return EDUS_OK;
}

int fix_reference(edus_handle* h, int b) {
    int rc;
    const size_t Sb = h->S * sizeof(double2);
    if (!h->tmp_in) {
        if ((rc = dalloc(h, (void**)&h->tmp_in, Sb))) return rc;
        if ((rc = dalloc(h, (void**)&h->tmp_out, Sb))) return rc;
    }
    CU(h, cudaMemcpyAsync(h->ref_full, h->y + (size_t)b * h->S, Sb, cudaMemcpyDeviceToDevice, h->stream));
    StageField rf[4];
    for (int f = 0; f < 4; ++f) {
        for (int d = 0; d < 3; ++d) rf[f].E[d] = (f == d + 1) ? 1.0 : 0.0;
        for (int c = 0; c < 3; ++c) rf[f].g[c] = h->A[0 * 3 + c] * rf[f].E[0] + h->A[1 * 3 + c] * rf[f].E[1] + h->A[2 * 3 + c] * rf[f].E[2];
    }
    CU(h, cudaMemcpyAsync(h->ref_fields, rf, sizeof(rf), cudaMemcpyHostToDevice, h->stream));
    // E = 0: Hee(rho_ref), rho_ref diagonal at R = 0, then C0 = f(rho_ref; 0)
    if ((rc = launch_plane(h, h->ref_full, 0, h->G, h->Hee, 0, h->ref_fields, 1, false))) return rc;
    const int coul = h->d.coulomb ? 1 : 0;
    const long long nS = (long long)h->S;
    assemble_h0p<<<grid_for(nS), 256, 0, h->stream>>>(h->H0, h->Hee, h->tmp_in, h->hartree, h->diag0, h->rho0diag,
                                                       h->nb, h->Nk, coul);
    h->launches++;
    StageArgs a = base_args(h);
    a.rho = h->ref_full;
    a.field = h->ref_fields;
    a.out = h->tmp_out;
    if ((rc = launch_comm(h, MODE_RHS, a, 1, false))) return rc;  // tmp_out = C0 (full)
    const long long nq = (long long)h->Sq;
    pack_planes<double2><<<grid_for(nq), 256, 0, h->stream>>>(h->tmp_out, h->pC0, h->qnm, h->nb, h->Pq, h->Nk);
    h->launches++;
    for (int d = 0; d < 3; ++d) {
        if ((rc = launch_plane(h, h->ref_full, 0, h->G, h->Hee, 0, h->ref_fields + 1 + d, 1, false))) return rc;
        a.field = h->ref_fields + 1 + d;
        a.out = h->stage;
        if ((rc = launch_comm(h, MODE_RHS, a, 1, false))) return rc;  // stage = f(rho_ref; e_d)
        sub_planes<<<grid_for(nS), 256, 0, h->stream>>>(h->stage, h->tmp_out, h->stage, nS);
        pack_planes<double2><<<grid_for(nq), 256, 0, h->stream>>>(h->stage, h->pK[d], h->qnm, h->nb, h->Pq, h->Nk);
        h->launches += 2;
    }
    if (h->mixed) {
        pack_planes<float2><<<grid_for(nq), 256, 0, h->stream>>>(h->tmp_in, (float2*)h->pH0p, h->qnm, h->nb, h->Pq, h->Nk);
        pack_planes<float2><<<grid_for(nq), 256, 0, h->stream>>>(h->ref_full, (float2*)h->pRref, h->qnm, h->nb, h->Pq, h->Nk);
    } else {
        pack_planes<double2><<<grid_for(nq), 256, 0, h->stream>>>(h->tmp_in, (double2*)h->pH0p, h->qnm, h->nb, h->Pq, h->Nk);
        pack_planes<double2><<<grid_for(nq), 256, 0, h->stream>>>(h->ref_full, (double2*)h->pRref, h->qnm, h->nb, h->Pq, h->Nk);
    }
    h->launches += 2;
    CU(h, cudaGetLastError());
    CU(h, cudaStreamSynchronize(h->stream));
    h->ref_fixed = true;
    return EDUS_OK;
}

PackedArgs base_pargs(edus_handle* h) {
    PackedArgs a{};
    a.G = h->pG;
    a.E1 = h->pE1;
    a.H0p = h->pH0p;
    for (int d = 0; d < 3; ++d) {
        a.xi[d] = h->pxi[d];
        a.K[d] = h->pK[d];
    }
    a.Rref = h->pRref;
    a.C0 = h->pC0;
    a.hartree = h->hartree;
    a.diag0 = h->pdiag0;
    a.qnm = h->qnm;
    a.y = h->py;
    a.aux = h->paux;
    a.acc = h->pacc;
    a.bstride = (long long)h->Sq;
    a.Nk = h->Nk;
    a.nb = h->nb;
    a.Pq = h->Pq;
    a.TK = h->pgeo.TK;
    return a;
}

// the state y[b] (full FP64 planes) from rho_ref + delta_b
int unpack_state(edus_handle* h, int b) {
    const long long nS = (long long)h->S;
    unpack_delta<<<grid_for(nS), 256, 0, h->stream>>>(h->py + (size_t)b * h->Sq, h->ref_full, h->y + (size_t)b * h->S,
                                                       h->nb, h->Nk);
    h->launches++;
    CU(h, cudaGetLastError());
    return EDUS_OK;
}

}  // namespace

extern "C" {

const char* edus_last_error(const edus_handle* h) {
    if (!h) return g_create_error.c_str();
    return h->err.c_str();
}

int edus_create(const edus_desc* desc, edus_handle** out) {
    if (!desc || !out) return fail(nullptr, EDUS_ERR_ARG, "edus_create: NULL argument");
    *out = nullptr;
    const edus_desc& d = *desc;
    for (int i = 0; i < 3; ++i)
        if (d.grid[i] < 1) return fail(nullptr, EDUS_ERR_ARG, "grid dimensions must be >= 1");
    if (d.nbands < 1 || d.nbands > 64) return fail(nullptr, EDUS_ERR_ARG, "nbands must be in [1, 64]");
    if (d.solver != EDUS_SOLVER_RK && d.solver != EDUS_SOLVER_AB) return fail(nullptr, EDUS_ERR_ARG, "unknown solver");
    if (d.solver == EDUS_SOLVER_RK && d.order != 4)
        return fail(nullptr, EDUS_ERR_UNSUPPORTED, "RK is implemented for order 4 only (DESolver.hpp:157)");
    if (d.solver == EDUS_SOLVER_AB && d.order != 4 && d.order != 5)
        return fail(nullptr, EDUS_ERR_UNSUPPORTED, "order not implemented for AB (DESolver.hpp:120-124)");
    if (d.precision != EDUS_PREC_FP64 && d.precision != EDUS_PREC_HERM64 && d.precision != EDUS_PREC_MIXED &&
        d.precision != EDUS_PREC_SPLIT32 && d.precision != EDUS_PREC_HPLANES)
        return fail(nullptr, EDUS_ERR_UNSUPPORTED, "precision not supported");
    const bool packed_form = d.precision == EDUS_PREC_HERM64 || d.precision == EDUS_PREC_MIXED;
    const bool herm_planes = d.precision == EDUS_PREC_HPLANES;
    if (packed_form && d.nbands > 32)
        return fail(nullptr, EDUS_ERR_UNSUPPORTED, "the packed-Hermitian forms handle up to 32 bands");
    if (d.batch < 1) return fail(nullptr, EDUS_ERR_ARG, "batch must be >= 1");
    if (!(d.dt > 0.0) || !std::isfinite(d.dt)) return fail(nullptr, EDUS_ERR_ARG, "dt must be positive and finite");

    edus_handle* h = new edus_handle();
    h->d = d;
    for (int i = 0; i < 3; ++i) h->N[i] = d.grid[i];
    h->Nk = d.grid[0] * d.grid[1] * d.grid[2];
    h->nb = d.nbands;
    h->P = d.nbands * d.nbands;
    h->B = d.batch;
    h->S = (size_t)h->P * h->Nk;
    h->lasers.assign(h->B, {});
    auto bail = [&](int rc) {
        std::string m = h->err;
        edus_destroy(h);
        g_create_error = m;
        return rc;
    };
    if (cudaSetDevice(d.device) != cudaSuccess) return bail(fail(h, EDUS_ERR_CUDA, "cudaSetDevice failed"));
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(h, EDUS_ERR_CUDA, "cudaStreamCreate failed"));

    // FFT plan per axis
    PlaneTables tabs;
    {
        std::string perr;
        if (!build_plane_plan(h->N, h->plan, tabs, perr)) return bail(fail(h, EDUS_ERR_UNSUPPORTED, perr));
    }
    for (int ax = 0; ax < 3; ++ax) {
        h->posof[ax].assign(h->N[ax], 0);
        for (int q = 0; q < h->N[ax]; ++q) h->posof[ax][tabs.fq[tabs.fqoff[ax] + q]] = q;
    }
    const std::vector<double2>& roots = tabs.roots;
    std::vector<double>& rpos = tabs.rpos;
    if (packed_form || herm_planes) {
        // The Hermitian forms propagate the Hermitian part of the generator: on an
        // even axis the Gamma-centred index N/2 is -N/2 for both R and -R, so
        // the gradient's i (R.E) is not anti-Hermitian there; its Hermitian
        // part has coordinate 0 on that index.
        for (int ax = 0; ax < 3; ++ax)
            for (int q = 0; q < h->N[ax]; ++q) {
                double& x = rpos[h->plan.ax[ax].rposoff + q];
                if (h->N[ax] % 2 == 0 && x == -0.5 * h->N[ax]) x = 0.0;
            }
    }

    int dev_smem = 0;
    cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, d.device);
    const size_t plane_bytes = (size_t)h->Nk * sizeof(double2) * (d.coulomb ? 2 : 1);
    if (plane_bytes > (size_t)dev_smem)
        return bail(fail(h, EDUS_ERR_UNSUPPORTED,
                         "k grid of " + std::to_string(h->Nk) + " points does not fit one plane" +
                             (d.coulomb ? " pair" : "") + " in shared memory (" + std::to_string(dev_smem) + " B)"));
    h->smem_plane = (int)plane_bytes;
    const CommLaunch cl = comm_launch(h->nb);
    h->comm_mma = cl.mma;
    h->TK = cl.TK;
    h->comm_threads = cl.threads;
    h->smem_comm = (int)cl.smem;
    if (h->smem_comm > dev_smem) return bail(fail(h, EDUS_ERR_UNSUPPORTED, "too many bands for the commutator tile"));
    int rc;
    h->plane_cfg = plane_launch(h->plan);
    {
        int nsm = 0;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, d.device);
        h->plane_grid = 2 * std::max(nsm, 1);
    }
    {
        // the persistent plane kernel keeps the root and coordinate tables
        // beside its plane when two CTAs still fit an SM
        const size_t tb = tabs.roots.size() * sizeof(double2) + ((tabs.rpos.size() * sizeof(double) + 15) & ~(size_t)15);
        if ((size_t)h->Nk * sizeof(double2) + tb <= 110 * 1024) {
            h->nroot_s = (int)tabs.roots.size();
            h->nrpos_s = (int)tabs.rpos.size();
            h->tab_smem = (int)tb;
        }
    }
    {
        const int ps = h->Nk * (int)sizeof(double2) + 16 + h->tab_smem;  // the plane, its load barrier, the tables
        if ((rc = set_smem(h, plane_rhs_persist_kernel<true, kRadix89, kPersist89Threads, kPersist89Batch>, ps))) return bail(rc);
        if ((rc = set_smem(h, plane_rhs_persist_kernel<false, kRadix89, kPersist89Threads, kPersist89Batch>, ps))) return bail(rc);
        if ((rc = set_smem(h, plane_rhs_persist_kernel<true, kRadixAll, 256>, ps))) return bail(rc);
        if ((rc = set_smem(h, plane_rhs_persist_kernel<false, kRadixAll, 256>, ps))) return bail(rc);
        if ((rc = set_smem(h, plane_rhs_persist_kernel<true, kRadixCommon, 256>, ps))) return bail(rc);
        if ((rc = set_smem(h, plane_rhs_persist_kernel<false, kRadixCommon, 256>, ps))) return bail(rc);
        if ((rc = set_smem(h, plane_rhs_persist_kernel<true, kRadix89, kPersist89Threads, kPersist89Batch, true>, ps))) return bail(rc);
        if ((rc = set_smem(h, plane_rhs_persist_kernel<false, kRadix89, kPersist89Threads, kPersist89Batch, true>, ps))) return bail(rc);
        if ((rc = set_smem(h, plane_rhs_persist_kernel<true, kRadixAll, 256, 1, true>, ps))) return bail(rc);
        if ((rc = set_smem(h, plane_rhs_persist_kernel<false, kRadixAll, 256, 1, true>, ps))) return bail(rc);
        if ((rc = set_smem(h, plane_rhs_persist_kernel<true, kRadixCommon, 256, 1, true>, ps))) return bail(rc);
        if ((rc = set_smem(h, plane_rhs_persist_kernel<false, kRadixCommon, 256, 1, true>, ps))) return bail(rc);
        if ((rc = set_smem(h, plane_rhs_persist_kernel<true, kRadix89, kPersist89Threads, kPersist89Batch, true, true>, ps))) return bail(rc);
        if ((rc = set_smem(h, plane_rhs_persist_kernel<false, kRadix89, kPersist89Threads, kPersist89Batch, true, true>, ps))) return bail(rc);
        if ((rc = set_smem(h, plane_rhs_persist_kernel<true, kRadixAll, 256, 1, true, true>, ps))) return bail(rc);
        if ((rc = set_smem(h, plane_rhs_persist_kernel<false, kRadixAll, 256, 1, true, true>, ps))) return bail(rc);
        if ((rc = set_smem(h, plane_rhs_persist_kernel<true, kRadixCommon, 256, 1, true, true>, ps))) return bail(rc);
        if ((rc = set_smem(h, plane_rhs_persist_kernel<false, kRadixCommon, 256, 1, true, true>, ps))) return bail(rc);
        // the row-wise variant: 2-D grids (unit-stride axis ax[1] with stages, several rows)
        h->rows_ok = h->plan.ax[2].n == 1 && h->plan.ax[0].n > 1 && h->plan.ax[1].nst > 0;
        if (herm_planes && !(h->plane_cfg.persist && h->rows_ok))
            return bail(fail(h, EDUS_ERR_UNSUPPORTED,
                             "the Hermitian-plane form needs a 2-D grid whose plane fits the persistent plane "
                             "kernel (at most 7040 k points)"));
    }
    if ((rc = set_smem(h, plane_rhs_kernel<true, kRadixAll, 512>, h->smem_plane))) return bail(rc);
    if ((rc = set_smem(h, plane_rhs_kernel<false, kRadixAll, 512>, h->smem_plane))) return bail(rc);
    if ((rc = set_smem(h, plane_rhs_kernel<true, kRadixCommon, 512>, h->smem_plane))) return bail(rc);
    if ((rc = set_smem(h, plane_rhs_kernel<false, kRadixCommon, 512>, h->smem_plane))) return bail(rc);
    if ((rc = set_smem(h, plane_rhs_kernel<true, kRadix89, 768>, h->smem_plane))) return bail(rc);
    if ((rc = set_smem(h, plane_rhs_kernel<false, kRadix89, 768>, h->smem_plane))) return bail(rc);
    if ((rc = set_smem(h, plane_to_R_kernel<kRadixAll, 256>, h->Nk * (int)sizeof(double2)))) return bail(rc);
    if ((rc = set_smem(h, observables_kernel, 2 * h->P * (int)sizeof(double2)))) return bail(rc);
    if (h->Nk * (int)sizeof(double2) <= dev_smem &&
        (rc = set_smem(h, peierls_shift_kernel<kRadixAll, 256>, h->Nk * (int)sizeof(double2))))
        return bail(rc);
    if ((rc = set_smem(h, kgradient_kernel, 4096 * (int)(sizeof(double) + 3 * sizeof(int))))) return bail(rc);
    // the attribute covers both commutator variants, which the autotuner may swap
    const int smem_cmax = (int)std::max(comm_geometry(h->nb).smem, mma_geometry(h->nb).smem);
#define SETC(M)                                                                                   \
    if ((rc = set_smem(h, commutator_kernel<M, true>, smem_cmax))) return bail(rc);           \
    if ((rc = set_smem(h, commutator_kernel<M, false>, smem_cmax))) return bail(rc);          \
    if ((rc = set_smem(h, commutator_mma_kernel<M, true>, smem_cmax))) return bail(rc);       \
    if ((rc = set_smem(h, commutator_mma_kernel<M, false>, smem_cmax))) return bail(rc);     \
    if ((rc = set_smem(h, commutator_kernel<M, true, true>, smem_cmax))) return bail(rc);     \
    if ((rc = set_smem(h, commutator_mma_kernel<M, true, true>, smem_cmax))) return bail(rc);      \
    if ((rc = set_smem(h, commutator_kernel<M, false, true>, smem_cmax))) return bail(rc);     \
    if ((rc = set_smem(h, commutator_mma_kernel<M, false, true>, smem_cmax))) return bail(rc);
    SETC(MODE_RHS) SETC(MODE_RK1) SETC(MODE_RK2) SETC(MODE_RK3) SETC(MODE_RK4) SETC(MODE_AB)
#undef SETC
    if (d.coulomb && ws_supported(h->nb) && tensor_map_encoder()) {
        const WsGeom wg = ws_geometry(h->nb);
        if ((int)wg.smem <= dev_smem) {
#define SETW(M)                                                                                           \
    if ((rc = set_smem(h, commutator_ws_kernel<M, 3, 3>, (int)wg.smem))) return bail(rc);    \
    if ((rc = set_smem(h, commutator_ws_kernel<M, 3, 2>, (int)wg.smem))) return bail(rc);    \
    if ((rc = set_smem(h, commutator_ws_kernel<M, 2, 4>, (int)wg.smem))) return bail(rc);
            SETW(MODE_RHS) SETW(MODE_RK1) SETW(MODE_RK2) SETW(MODE_RK3) SETW(MODE_RK4) SETW(MODE_AB)
#undef SETW
            int per_sm = 0;
            if (wg.tiles == 2)
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, commutator_ws_kernel<MODE_RK2, 2, 4>,
                                                              wg.threads, wg.smem);
            else if (wg.SM == 3)
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, commutator_ws_kernel<MODE_RK2, 3, 3>,
                                                              wg.threads, wg.smem);
            else
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, commutator_ws_kernel<MODE_RK2, 3, 2>,
                                                              wg.threads, wg.smem);
            int nsm = 0;
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, d.device);
            if (per_sm > 0 && nsm > 0) {
                h->comm_ws = true;
                h->ws_grid = per_sm * nsm;
            }
        }
    }

    const size_t Sb = h->S * sizeof(double2);
    const size_t SBb = Sb * h->B;
#define TRY_ALLOC(ptr, bytes) \
    if ((rc = dalloc(h, (void**)&(ptr), (bytes)))) return bail(rc);
    TRY_ALLOC(h->H0, Sb);
    for (int i = 0; i < 3; ++i) TRY_ALLOC(h->xi[i], Sb);
    TRY_ALLOC(h->y, SBb);
    TRY_ALLOC(h->G, SBb);
    TRY_ALLOC(h->stage, Sb);
    if (d.solver == EDUS_SOLVER_RK) {
        TRY_ALLOC(h->aux, SBb);
        TRY_ALLOC(h->acc, SBb);
    } else {
        for (int i = 0; i < d.order; ++i) {
            TRY_ALLOC(h->hist[i], SBb);
            // zero history (DESolver.cpp:26-29, mdContainers_definitions.hpp:91)
            if (cudaMemsetAsync(h->hist[i], 0, SBb, h->stream) != cudaSuccess)
                return bail(fail(h, EDUS_ERR_CUDA, "cudaMemsetAsync failed"));
        }
        if (d.order == 4) {
            const double b[5] = {55. / 24., -59. / 24., 37. / 24., -3. / 8., 0.};
            std::copy(b, b + 5, h->beta);
        } else {
            const double b[5] = {1901. / 720., -2774. / 720., 2616. / 720., -1274. / 720., 251. / 720.};
            std::copy(b, b + 5, h->beta);
        }
    }
    if (d.coulomb) {
        TRY_ALLOC(h->Hee, SBb);
        TRY_ALLOC(h->rho0p, Sb);
        TRY_ALLOC(h->Wp, (size_t)h->S * sizeof(double));
        TRY_ALLOC(h->hartree, h->P * sizeof(double2));
        TRY_ALLOC(h->rho0diag, h->nb * sizeof(double2));
        TRY_ALLOC(h->diag0, (size_t)h->B * h->nb * sizeof(double2));
    }
    TRY_ALLOC(h->roots, roots.size() * sizeof(double2));
    TRY_ALLOC(h->rpos, rpos.size() * sizeof(double));
    TRY_ALLOC(h->field, (size_t)h->chunk * 4 * h->B * sizeof(StageField));
    if (h->plane_cfg.persist && d.coulomb) TRY_ALLOC(h->plane_scratch, (size_t)h->plane_grid * h->Nk * sizeof(double2));
    {
        // few band-pair planes on a 2-D grid: spread each plane over CTAs
        int nsm = 0;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, d.device);
        const int planes = h->P * h->B;
        if (d.precision == EDUS_PREC_FP64 && h->N[2] == 1 && h->N[1] > 1 && h->Nk >= 1024 && planes < nsm) {
            const int Rc = divisor_upto(h->N[0], std::max(1, planes * h->N[0] / nsm));
            const int Cc = divisor_upto(h->N[1], std::max(1, planes * h->N[1] / nsm));
            h->p3 = plane3_plan(h->plan, Rc, Cc);
            TRY_ALLOC(h->s3a, SBb);
            TRY_ALLOC(h->s3g, SBb);
            if (d.coulomb) TRY_ALLOC(h->s3h, SBb);
            if ((rc = set_smem(h, plane3_rows_kernel<true, 256, kRadixAll>, Rc * h->N[1] * (int)sizeof(double2)))) return bail(rc);
            if ((rc = set_smem(h, plane3_rows_kernel<false, 256, kRadixAll>, Rc * h->N[1] * (int)sizeof(double2)))) return bail(rc);
            if ((rc = set_smem(h, plane3_cols_kernel<true, 256, kRadixAll>, 2 * h->N[0] * Cc * (int)sizeof(double2)))) return bail(rc);
            if ((rc = set_smem(h, plane3_cols_kernel<false, 256, kRadixAll>, h->N[0] * Cc * (int)sizeof(double2)))) return bail(rc);
            if ((rc = set_smem(h, plane3_rows_kernel<true, 256, kRadixCommon>, Rc * h->N[1] * (int)sizeof(double2)))) return bail(rc);
            if ((rc = set_smem(h, plane3_rows_kernel<false, 256, kRadixCommon>, Rc * h->N[1] * (int)sizeof(double2)))) return bail(rc);
            if ((rc = set_smem(h, plane3_cols_kernel<true, 256, kRadixCommon>, 2 * h->N[0] * Cc * (int)sizeof(double2)))) return bail(rc);
            if ((rc = set_smem(h, plane3_cols_kernel<false, 256, kRadixCommon>, h->N[0] * Cc * (int)sizeof(double2)))) return bail(rc);
            h->use3 = true;
        }
    }
    std::vector<int> upair_host;
    if (herm_planes) {
        h->hplanes = true;
        h->Pu = h->nb * (h->nb + 1) / 2;
        for (int n = 0; n < h->nb; ++n)
            for (int m = n; m < h->nb; ++m) upair_host.push_back(n * h->nb + m);
        TRY_ALLOC(h->upair, upair_host.size() * sizeof(int));
    }
    TRY_ALLOC(h->popbuf, h->nb * sizeof(double));
    TRY_ALLOC(h->flag, sizeof(int));
    if (cudaMemsetAsync(h->flag, 0, sizeof(int), h->stream) != cudaSuccess)
        return bail(fail(h, EDUS_ERR_CUDA, "cudaMemsetAsync failed"));
    if (d.precision == EDUS_PREC_SPLIT32) {
        h->split = true;
        for (int dd = 0; dd < 3; ++dd) TRY_ALLOC(h->sGref[dd], SBb);
        TRY_ALLOC(h->sref, SBb);
        TRY_ALLOC(h->unit_fields, 3 * (size_t)h->B * sizeof(StageField));
        if (d.coulomb) {
            TRY_ALLOC(h->sHfix, SBb);
            TRY_ALLOC(h->srefdiag0, (size_t)h->B * h->nb * sizeof(double2));
            TRY_ALLOC(h->W32, (size_t)h->S * sizeof(float));
        }
        const size_t sm = (size_t)h->Nk * sizeof(float2);
        if ((int)sm > dev_smem) return bail(fail(h, EDUS_ERR_UNSUPPORTED, "k grid too large for the split form"));
        int per_sm = 0;
        if (h->plane_cfg.variant == 1) {
            h->split_threads = h->plane_cfg.persist ? h->plane_cfg.threads : 384;
            if ((rc = set_smem(h, plane_split_kernel<true, kRadix89, 384>, (int)sm))) return bail(rc);
            if ((rc = set_smem(h, plane_split_kernel<false, kRadix89, 384>, (int)sm))) return bail(rc);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, plane_split_kernel<true, kRadix89, 384>,
                                                          h->split_threads, sm);
        } else {
            h->split_threads = h->plane_cfg.persist ? h->plane_cfg.threads : 256;
            if ((rc = set_smem(h, plane_split_kernel<true, kRadixAll, 256>, (int)sm))) return bail(rc);
            if ((rc = set_smem(h, plane_split_kernel<false, kRadixAll, 256>, (int)sm))) return bail(rc);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, plane_split_kernel<true, kRadixAll, 256>,
                                                          h->split_threads, sm);
        }
        int nsm = 0;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, d.device);
        h->split_grid = std::max(1, per_sm) * std::max(1, nsm);
        if (d.coulomb) TRY_ALLOC(h->split_scratch, (size_t)h->split_grid * h->Nk * sizeof(float2));
    }
    if (packed_form) {
        h->packed = true;
        h->mixed = d.precision == EDUS_PREC_MIXED;
        h->Pq = h->nb * (h->nb + 1) / 2;
        h->Sq = (size_t)h->Pq * h->Nk;
        const size_t st = h->mixed ? sizeof(float2) : sizeof(double2);
        const size_t sc = h->mixed ? sizeof(float) : sizeof(double);
        const size_t Sq8 = h->Sq * sizeof(double2), SqB8 = Sq8 * h->B;
        TRY_ALLOC(h->qnm, h->Pq * sizeof(int));
        TRY_ALLOC(h->ref_full, Sb);
        TRY_ALLOC(h->pH0p, h->Sq * st);
        for (int i = 0; i < 3; ++i) TRY_ALLOC(h->pxi[i], h->Sq * st);
        TRY_ALLOC(h->pRref, h->Sq * st);
        TRY_ALLOC(h->pC0, Sq8);
        for (int i = 0; i < 3; ++i) TRY_ALLOC(h->pK[i], Sq8);
        TRY_ALLOC(h->py, SqB8);
        TRY_ALLOC(h->pG, h->Sq * st * h->B);
        if (d.coulomb) {
            TRY_ALLOC(h->pE1, h->Sq * st * h->B);
            TRY_ALLOC(h->pW, h->Sq * sc);
            TRY_ALLOC(h->pdiag0, (size_t)h->B * h->nb * sizeof(double2));
        }
        if (d.solver == EDUS_SOLVER_RK) {
            TRY_ALLOC(h->paux, h->Sq * st * h->B);
            TRY_ALLOC(h->pacc, SqB8);
        } else {
            for (int i = 0; i < d.order; ++i) {
                TRY_ALLOC(h->phist[i], SqB8);
                if (cudaMemsetAsync(h->phist[i], 0, SqB8, h->stream) != cudaSuccess)
                    return bail(fail(h, EDUS_ERR_CUDA, "cudaMemsetAsync failed"));
            }
        }
        TRY_ALLOC(h->ref_fields, 4 * sizeof(StageField));
        std::vector<int> qnm;
        for (int n = 0; n < h->nb; ++n)
            for (int m = n; m < h->nb; ++m) qnm.push_back((n << 16) | m);
        if (cudaMemcpyAsync(h->qnm, qnm.data(), qnm.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
            return bail(fail(h, EDUS_ERR_CUDA, "upload of the packed plane map failed"));
        h->pgeo = packed_geometry(h->nb);
        const PlaneLaunch pl = plane_launch(h->plan);
        h->pplane_variant = pl.variant;
        // the packed transform: cost model over 128..512 threads
        {
            long best = -1;
            for (int T = 128; T <= 512; T += 32) {
                long cost = 0;
                for (int ax = 0; ax < 3; ++ax)
                    for (int s2 = 0; s2 < h->plan.ax[ax].nst; ++s2) {
                        const int r = h->plan.ax[ax].r[s2];
                        cost += ((h->Nk / r + T - 1) / T) * (long)r;
                    }
                cost = cost * 4 + 3 * ((h->Nk + T - 1) / T);
                if (best < 0 || cost <= best) {
                    best = cost;
                    h->pplane_threads = T;
                }
            }
        }
        h->pplane_smem = (size_t)h->Nk * st * (d.coulomb ? 2 : 1);
        if (h->pplane_smem > (size_t)dev_smem || h->pgeo.smem > (size_t)dev_smem)
            return bail(fail(h, EDUS_ERR_UNSUPPORTED, "k grid too large for the packed plane kernel"));
        if ((rc = packed_setup_smem(h))) return bail(rc);
    }
#undef TRY_ALLOC
    for (int i = 0; i < 2; ++i) {
        if (cudaMallocHost((void**)&h->field_host[i], (size_t)h->chunk * 4 * h->B * sizeof(StageField)) != cudaSuccess)
            return bail(fail(h, EDUS_ERR_NOMEM, "cudaMallocHost failed"));
        if (cudaEventCreateWithFlags(&h->field_ev[i], cudaEventDisableTiming) != cudaSuccess)
            return bail(fail(h, EDUS_ERR_CUDA, "cudaEventCreate failed"));
        cudaEventRecord(h->field_ev[i], h->stream);
    }
    if (cudaMemcpyAsync(h->roots, roots.data(), roots.size() * sizeof(double2), cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
        cudaMemcpyAsync(h->rpos, rpos.data(), rpos.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
        (h->upair && cudaMemcpyAsync(h->upair, upair_host.data(), upair_host.size() * sizeof(int),
                                     cudaMemcpyHostToDevice, h->stream) != cudaSuccess) ||
        cudaMemsetAsync(h->y, 0, SBb, h->stream) != cudaSuccess || cudaStreamSynchronize(h->stream) != cudaSuccess)
        return bail(fail(h, EDUS_ERR_CUDA, "initial upload failed"));
    *out = h;
    return EDUS_OK;
}

int edus_destroy(edus_handle* h) {
    if (!h) return EDUS_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    prof_resolve(h);
    for (cudaEvent_t e : h->prof_pool) cudaEventDestroy(e);
    for (void* p : h->allocs) cudaFree(p);
    for (int i = 0; i < 2; ++i) {
        if (h->field_host[i]) cudaFreeHost(h->field_host[i]);
        if (h->field_ev[i]) cudaEventDestroy(h->field_ev[i]);
    }
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return EDUS_OK;
}

int edus_upload_model(edus_handle* h, const double* H0_k, const double* xi_k, const double* lattice,
                      const double* W_R, const double* rho0_R, const double* hartree) {
    if (!h) return EDUS_ERR_ARG;
    if (!H0_k || !xi_k || !lattice) return fail(h, EDUS_ERR_ARG, "H0_k, xi_k and lattice are required");
    if (h->d.coulomb && (!W_R || !rho0_R || !hartree))
        return fail(h, EDUS_ERR_ARG, "coulomb=1 needs W_R, rho0_R and hartree");
    CU(h, cudaSetDevice(h->d.device));
    std::memcpy(h->A, lattice, sizeof(h->A));
    const int Nk = h->Nk, P = h->P;
    const size_t Sb = h->S * sizeof(double2);
    dim3 tb(32, 8);
    dim3 tg((Nk + 31) / 32, (P + 31) / 32);
    auto up = [&](const double* src, double2* dst) -> int {
        CU(h, cudaMemcpyAsync(h->stage, src, Sb, cudaMemcpyHostToDevice, h->stream));
        transpose_kp_to_pk<<<tg, tb, 0, h->stream>>>(h->stage, dst, Nk, P);
        h->launches++;
        CU(h, cudaGetLastError());
        return EDUS_OK;
    };
    int rc;
    if ((rc = up(H0_k, h->H0))) return rc;
    for (int d = 0; d < 3; ++d)
        if ((rc = up(xi_k + 2 * h->S * d, h->xi[d]))) return rc;
    if (h->d.coulomb) {
        // R-space arrays go to the digit-reversed positions of the plane FFT
        std::vector<int> fq[3];
        for (int ax = 0; ax < 3; ++ax) {
            std::vector<int> r;
            for (int s = 0; s < h->plan.ax[ax].nst; ++s) r.push_back(h->plan.ax[ax].r[s]);
            dif_positions(h->N[ax], r, fq[ax]);
        }
        // W_R as uploaded; the packed forms take its Hermitian part
        // (W_nm(R) + W_mn(-R)) / 2, which differs from W only on the planes
        // where an even axis sits at its N/2 index (Gamma-centred to -N/2 for
        // both R and -R).  Anywhere else an asymmetry is a model the packed
        // forms cannot represent (e.g. two off-origin Wannier centres under
        // the cumulative r of ModelCoulomb.cpp:76-79).
        std::vector<double> Wuse;
        const bool herm_w = h->packed || h->hplanes;
        if (herm_w) {
            const int nb = h->nb;
            Wuse.assign(h->S, 0.0);
            double mx = 0, dev = 0;
            for (int j0 = 0; j0 < h->N[0]; ++j0)
                for (int j1 = 0; j1 < h->N[1]; ++j1)
                    for (int j2 = 0; j2 < h->N[2]; ++j2) {
                        const int j[3] = {j0, j1, j2};
                        bool nyq = false;
                        for (int ax = 0; ax < 3; ++ax) nyq |= (h->N[ax] % 2 == 0 && 2 * j[ax] == h->N[ax]);
                        const int iR = (j0 * h->N[1] + j1) * h->N[2] + j2;
                        const int mR = (((h->N[0] - j0) % h->N[0]) * h->N[1] + (h->N[1] - j1) % h->N[1]) * h->N[2] +
                                       (h->N[2] - j2) % h->N[2];
                        for (int n = 0; n < nb; ++n)
                            for (int m = 0; m < nb; ++m) {
                                const double a = W_R[2 * (((size_t)iR * nb + n) * nb + m)];
                                const double c = W_R[2 * (((size_t)mR * nb + m) * nb + n)];
                                mx = std::max(mx, std::fabs(a));
                                if (!nyq) dev = std::max(dev, std::fabs(a - c));
                                Wuse[((size_t)iR * nb + n) * nb + m] = 0.5 * (a + c);
                            }
                    }
            if (dev > 1e-12 * std::max(mx, 1e-300))
                return fail(h, EDUS_ERR_UNSUPPORTED,
                            "the Hermitian forms need W_nm(R) = W_mn(-R) (Hermitian self-energy); this model's Wannier "
                            "centres break it (use EDUS_PREC_FP64)");
        }
        std::vector<double> w(h->S);
        std::vector<double2> r0(h->S);
        const int N1 = h->N[1], N2 = h->N[2];
        for (int q0 = 0; q0 < h->N[0]; ++q0)
            for (int q1 = 0; q1 < N1; ++q1)
                for (int q2 = 0; q2 < N2; ++q2) {
                    const int pos = (q0 * N1 + q1) * N2 + q2;
                    const int iR = (fq[0][q0] * N1 + fq[1][q1]) * N2 + fq[2][q2];
                    for (int p = 0; p < P; ++p) {
                        const double* wsrc = W_R + 2 * ((size_t)iR * P + p);
                        if (wsrc[1] != 0.0)
                            return fail(h, EDUS_ERR_ARG, "W_R must be real (the screened potential has no imaginary part)");
                        w[(size_t)p * Nk + pos] = herm_w ? Wuse[(size_t)iR * P + p] : wsrc[0];
                        const double* rsrc = rho0_R + 2 * ((size_t)iR * P + p);
                        r0[(size_t)p * Nk + pos] = make_double2(rsrc[0], rsrc[1]);
                    }
                }
        std::vector<double2> d0(h->nb);
        for (int n = 0; n < h->nb; ++n) d0[n] = make_double2(rho0_R[2 * (n * h->nb + n)], rho0_R[2 * (n * h->nb + n) + 1]);
        CU(h, cudaMemcpyAsync(h->Wp, w.data(), h->S * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        CU(h, cudaMemcpyAsync(h->rho0p, r0.data(), Sb, cudaMemcpyHostToDevice, h->stream));
        CU(h, cudaMemcpyAsync(h->hartree, hartree, P * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
        CU(h, cudaMemcpyAsync(h->rho0diag, d0.data(), h->nb * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
        CU(h, cudaStreamSynchronize(h->stream));  // host vectors go out of scope
    }
    CU(h, cudaStreamSynchronize(h->stream));
    if (h->d.coulomb && (rc = build_sparse_model(h))) return rc;
    if (h->split) {
        // unit fields along x, y, z for the anchor's gradient terms; W in FP32
        std::vector<StageField> uf(3 * (size_t)h->B);
        for (int dd = 0; dd < 3; ++dd)
            for (int b = 0; b < h->B; ++b) {
                StageField& f = uf[(size_t)dd * h->B + b];
                for (int i = 0; i < 3; ++i) f.E[i] = (i == dd) ? 1.0 : 0.0;
                for (int c = 0; c < 3; ++c)
                    f.g[c] = h->A[0 * 3 + c] * f.E[0] + h->A[1 * 3 + c] * f.E[1] + h->A[2 * 3 + c] * f.E[2];
            }
        CU(h, cudaMemcpyAsync(h->unit_fields, uf.data(), uf.size() * sizeof(StageField), cudaMemcpyHostToDevice,
                              h->stream));
        if (h->d.coulomb) {
            to_float_kernel<<<grid_for((long long)h->S), 256, 0, h->stream>>>(h->Wp, h->W32, (long long)h->S);
            h->launches++;
        }
        CU(h, cudaStreamSynchronize(h->stream));
        h->anchored = false;
    }
    if (h->packed) {
        // the packed forms need Hermitian H0, xi and W_nm(R) = W_mn(-R)
        const int nb = h->nb;
        auto herm_ok = [&](const double* X) {
            double mx = 0, dev = 0;
            for (int k = 0; k < Nk; ++k)
                for (int n = 0; n < nb; ++n)
                    for (int m = n; m < nb; ++m) {
                        const double* a = X + 2 * (((size_t)k * nb + n) * nb + m);
                        const double* c = X + 2 * (((size_t)k * nb + m) * nb + n);
                        mx = std::max(mx, std::fabs(a[0]) + std::fabs(a[1]));
                        dev = std::max(dev, std::fabs(a[0] - c[0]) + std::fabs(a[1] + c[1]));
                    }
            return dev <= 1e-12 * std::max(mx, 1e-300);
        };
        if (!herm_ok(H0_k) || !herm_ok(xi_k) || !herm_ok(xi_k + 2 * h->S) || !herm_ok(xi_k + 4 * h->S))
            return fail(h, EDUS_ERR_UNSUPPORTED, "the packed forms need Hermitian H0(k) and xi(k)");
        const long long nq = (long long)h->Sq;
        for (int dd = 0; dd < 3; ++dd) {
            if (h->mixed)
                pack_planes<float2><<<grid_for(nq), 256, 0, h->stream>>>(h->xi[dd], (float2*)h->pxi[dd], h->qnm, nb, h->Pq, Nk);
            else
                pack_planes<double2><<<grid_for(nq), 256, 0, h->stream>>>(h->xi[dd], (double2*)h->pxi[dd], h->qnm, nb, h->Pq, Nk);
            h->launches++;
        }
        if (h->d.coulomb) {
            if (h->mixed)
                pack_scalar_planes<float><<<grid_for(nq), 256, 0, h->stream>>>(h->Wp, (float*)h->pW, h->qnm, nb, h->Pq, Nk);
            else
                pack_scalar_planes<double><<<grid_for(nq), 256, 0, h->stream>>>(h->Wp, (double*)h->pW, h->qnm, nb, h->Pq, Nk);
            h->launches++;
        }
        CU(h, cudaGetLastError());
        CU(h, cudaStreamSynchronize(h->stream));
        h->ref_fixed = false;
    }
    h->model_ready = true;
    return EDUS_OK;
}

int edus_set_kgradient(edus_handle* h, int n, const int* shift, const double* b, const double* w) {
    if (!h || n < 0 || (n > 0 && (!shift || !b || !w))) return EDUS_ERR_ARG;
    if (n == 0) {
        CU(h, cudaStreamSynchronize(h->stream));
        h->kg_n = 0;
        return EDUS_OK;
    }
    if (h->packed || h->split || h->hplanes)
        return fail(h, EDUS_ERR_UNSUPPORTED, "gradient_space \"k\" is implemented for the FP64 form");
    if (n > 4096) return fail(h, EDUS_ERR_ARG, "k-gradient stencil longer than 4096 vectors");
    std::vector<int> sh(3 * (size_t)n);
    std::vector<double> cf(4 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        for (int d = 0; d < 3; ++d) {
            int x = shift[3 * i + d] % h->N[d];
            if (x < 0) x += h->N[d];
            sh[3 * i + d] = x;
            cf[4 * i + d] = b[3 * i + d];
        }
        cf[4 * i + 3] = w[i];
    }
    CU(h, cudaSetDevice(h->d.device));
    CU(h, cudaStreamSynchronize(h->stream));
    int rc;
    if (n > h->kg_cap) {
        if ((rc = dalloc(h, (void**)&h->kg_shift, 3 * (size_t)n * sizeof(int)))) return rc;
        if ((rc = dalloc(h, (void**)&h->kg_coef, 4 * (size_t)n * sizeof(double)))) return rc;
        h->kg_cap = n;
    }
    CU(h, cudaMemcpy(h->kg_shift, sh.data(), sh.size() * sizeof(int), cudaMemcpyHostToDevice));
    CU(h, cudaMemcpy(h->kg_coef, cf.data(), cf.size() * sizeof(double), cudaMemcpyHostToDevice));
    h->kg_n = n;
    return EDUS_OK;
}

int edus_set_peierls(edus_handle* h, int on) {
    if (!h) return EDUS_ERR_ARG;
    CU(h, cudaSetDevice(h->d.device));
    CU(h, cudaStreamSynchronize(h->stream));
    if (!on) {
        h->peierls = false;
        return EDUS_OK;
    }
    if (!h->model_ready) return fail(h, EDUS_ERR_ARG, "edus_upload_model must be called first");
    if (h->packed || h->split || h->hplanes)
        return fail(h, EDUS_ERR_UNSUPPORTED, "the Peierls gauge is implemented for the FP64 form");
    if (h->per_solve) return fail(h, EDUS_ERR_UNSUPPORTED, "the Peierls gauge needs one model for all solves");
    if (h->nO > 0) return fail(h, EDUS_ERR_UNSUPPORTED, "the Peierls gauge does not combine with a Fock override");
    if (h->Nk * sizeof(double2) > (size_t)device_smem_optin(h->d.device))
        return fail(h, EDUS_ERR_UNSUPPORTED, "the Peierls gauge needs a plane (16 Nk bytes) in shared memory");
    int rc;
    if (!h->d.coulomb && h->nS == 0 && (rc = build_sparse_model(h))) return rc;
    if (h->nS == 0)
        return fail(h, EDUS_ERR_UNSUPPORTED,
                    "the Peierls gauge needs H0(R) and xi(R) on at most 4096 lattice vectors");
    const size_t SBb = h->S * sizeof(double2) * h->B;
    if (!h->Hee && (rc = dalloc(h, (void**)&h->Hee, SBb))) return rc;
    if (!h->ptab) {
        h->ntab = h->N[0] + h->N[1] + h->N[2];
        if ((rc = dalloc(h, (void**)&h->ptab, (size_t)h->B * h->ntab * sizeof(double2)))) return rc;
    }
    // no gradient term: the commutators read G = 0
    CU(h, cudaMemsetAsync(h->G, 0, SBb, h->stream));
    CU(h, cudaStreamSynchronize(h->stream));
    h->Avec.assign(3 * (size_t)h->B, 0.0);
    h->Aprev.assign(h->B, 0.0);
    h->peierls = true;
    return EDUS_OK;
}

int edus_vector_potential(edus_handle* h, int b, double t, double* A) {
    if (!h || !A) return EDUS_ERR_ARG;
    if (b < 0 || b >= h->B) return fail(h, EDUS_ERR_ARG, "solve index out of range");
    if ((int)h->Aprev.size() != h->B) {
        h->Avec.assign(3 * (size_t)h->B, 0.0);
        h->Aprev.assign(h->B, 0.0);
    }
    advance_vecpot(h, b, t);
    for (int d = 0; d < 3; ++d) A[d] = h->Avec[3 * b + d];
    return EDUS_OK;
}

int edus_upload_observables(edus_handle* h, const double* U_k, const double* vel_k) {
    if (!h || (!U_k && !vel_k)) return EDUS_ERR_ARG;
    CU(h, cudaSetDevice(h->d.device));
    const size_t Sb = h->S * sizeof(double2);
    int rc;
    dim3 tb(32, 8), tg((h->Nk + 31) / 32, (h->P + 31) / 32);
    auto up = [&](const double* src, double2** dst) -> int {
        int r;
        if (!*dst && (r = dalloc(h, (void**)dst, Sb))) return r;
        CU(h, cudaMemcpyAsync(h->stage, src, Sb, cudaMemcpyHostToDevice, h->stream));
        transpose_kp_to_pk<<<tg, tb, 0, h->stream>>>(h->stage, *dst, h->Nk, h->P);
        h->launches++;
        CU(h, cudaGetLastError());
        CU(h, cudaStreamSynchronize(h->stream));  // h->stage is reused by the next upload
        return EDUS_OK;
    };
    if (U_k && (rc = up(U_k, &h->obsU))) return rc;
    if (vel_k)
        for (int d = 0; d < 3; ++d)
            if ((rc = up(vel_k + 2 * h->S * d, &h->obsV[d]))) return rc;
    if (!h->obsacc && (rc = dalloc(h, (void**)&h->obsacc, (2 * (size_t)h->nb + 6) * sizeof(double)))) return rc;
    return EDUS_OK;
}

int edus_observables(edus_handle* h, int b, int filled, double* pop_bloch, double* pop_wannier, double* vel) {
    if (!h) return EDUS_ERR_ARG;
    if (b < 0 || b >= h->B) return fail(h, EDUS_ERR_ARG, "solve index out of range");
    if (pop_bloch && !h->obsU) return fail(h, EDUS_ERR_ARG, "the Bloch populations need edus_upload_observables(U)");
    if (vel && !h->obsV[0]) return fail(h, EDUS_ERR_ARG, "the velocity needs edus_upload_observables(vel)");
    int rc;
    if (!h->obsacc && (rc = dalloc(h, (void**)&h->obsacc, (2 * (size_t)h->nb + 6) * sizeof(double)))) return rc;
    CU(h, cudaSetDevice(h->d.device));
    if (h->packed && (rc = unpack_state(h, b))) return rc;
    const int nacc = 2 * h->nb + 6;
    const double2* rho = h->y + (size_t)b * h->S;
    if (h->peierls) {
        // the gauge-shifted state at the handle's time, in the transpose buffer
        StageField f;
        field_at(h->lasers[b], h->A, h->t, f);
        peierls_field(h, b, h->t, f);
        CU(h, cudaMemcpyAsync(h->field, &f, sizeof(StageField), cudaMemcpyHostToDevice, h->stream));
        peierls_phase_kernel<<<1, 128, 0, h->stream>>>(h->field, h->rpos, h->plan, h->ntab, h->ptab);
        peierls_shift_kernel<kRadixAll, 256><<<h->P, 256, h->Nk * sizeof(double2), h->stream>>>(
            rho, h->stage, h->ptab, h->roots, h->plan, 1.0 / h->Nk);
        h->launches += 2;
        CU(h, cudaGetLastError());
        rho = h->stage;
    }
    CU(h, cudaMemsetAsync(h->obsacc, 0, nacc * sizeof(double), h->stream));
    observables_kernel<<<h->Nk, 128, 2 * h->P * sizeof(double2), h->stream>>>(
        rho, pop_bloch ? h->obsU : nullptr, vel ? h->obsV[0] : nullptr, h->obsV[1], h->obsV[2],
        h->Nk, h->nb, h->obsacc);
    h->launches++;
    CU(h, cudaGetLastError());
    std::vector<double> a(nacc);
    CU(h, cudaMemcpyAsync(a.data(), h->obsacc, nacc * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CU(h, cudaStreamSynchronize(h->stream));
    const double inv = 1.0 / h->Nk;
    for (int n = 0; n < h->nb; ++n) {
        // Print_Population (Simulation.cpp:439-470): holes of the filled bands in the Bloch gauge
        if (pop_bloch) pop_bloch[n] = n < filled ? 1.0 - a[n] * inv : a[n] * inv;
        if (pop_wannier) pop_wannier[n] = a[h->nb + n] * inv;
    }
    if (vel)
        for (int q = 0; q < 6; ++q) vel[q] = a[2 * h->nb + q] * inv;
    return check_status(h);
}

int edus_efield(edus_handle* h, int b, double t, double* E) {
    if (!h || !E) return EDUS_ERR_ARG;
    if (b < 0 || b >= h->B) return fail(h, EDUS_ERR_ARG, "solve index out of range");
    StageField f;
    field_at(h->lasers[b], h->A, t, f);
    for (int d = 0; d < 3; ++d) E[d] = f.E[d];
    return EDUS_OK;
}

int edus_upload_model_solve(edus_handle* h, int b, const double* H0_k, const double* xi_k) {
    if (!h || !H0_k || !xi_k) return EDUS_ERR_ARG;
    if (b < 0 || b >= h->B) return fail(h, EDUS_ERR_ARG, "solve index out of range");
    if (!h->model_ready) return fail(h, EDUS_ERR_ARG, "edus_upload_model (lattice and shared model) must come first");
    if (h->d.coulomb || h->packed || h->split)
        return fail(h, EDUS_ERR_UNSUPPORTED, "a model per solve is implemented for the FP64 form without HSEX");
    CU(h, cudaSetDevice(h->d.device));
    const size_t Sb = h->S * sizeof(double2);
    int rc;
    if (!h->per_solve) {
        // every solve starts from the shared model
        if ((rc = dalloc(h, (void**)&h->H0b, Sb * h->B))) return rc;
        for (int d = 0; d < 3; ++d)
            if ((rc = dalloc(h, (void**)&h->xib[d], Sb * h->B))) return rc;
        for (int q = 0; q < h->B; ++q) {
            CU(h, cudaMemcpyAsync(h->H0b + (size_t)q * h->S, h->H0, Sb, cudaMemcpyDeviceToDevice, h->stream));
            for (int d = 0; d < 3; ++d)
                CU(h, cudaMemcpyAsync(h->xib[d] + (size_t)q * h->S, h->xi[d], Sb, cudaMemcpyDeviceToDevice,
                                      h->stream));
        }
        h->per_solve = true;
    }
    dim3 tb(32, 8), tg((h->Nk + 31) / 32, (h->P + 31) / 32);
    auto up = [&](const double* src, double2* dst) -> int {
        CU(h, cudaMemcpyAsync(h->stage, src, Sb, cudaMemcpyHostToDevice, h->stream));
        transpose_kp_to_pk<<<tg, tb, 0, h->stream>>>(h->stage, dst, h->Nk, h->P);
        h->launches++;
        CU(h, cudaGetLastError());
        return EDUS_OK;
    };
    if ((rc = up(H0_k, h->H0b + (size_t)b * h->S))) return rc;
    for (int d = 0; d < 3; ++d)
        if ((rc = up(xi_k + 2 * h->S * d, h->xib[d] + (size_t)b * h->S))) return rc;
    CU(h, cudaStreamSynchronize(h->stream));  // the host buffers are the caller's
    return EDUS_OK;
}

int edus_set_lasers(edus_handle* h, int b, int n, const edus_laser* lasers) {
    if (!h) return EDUS_ERR_ARG;
    if (b < 0 || b >= h->B) return fail(h, EDUS_ERR_ARG, "solve index out of range");
    if (n < 0 || (n > 0 && !lasers)) return fail(h, EDUS_ERR_ARG, "bad laser list");
    std::vector<edus_laser> v(lasers, lasers + n);
    for (auto& L : v) {
        const double nrm = std::sqrt(L.pol[0] * L.pol[0] + L.pol[1] * L.pol[1] + L.pol[2] * L.pol[2]);
        if (!(nrm > 0)) return fail(h, EDUS_ERR_ARG, "laser polarisation must be non-zero");
        if (L.envelope == EDUS_ENVELOPE_SIN2 && !(L.omega != 0)) return fail(h, EDUS_ERR_ARG, "sin2 laser needs omega != 0");
        if (L.envelope == EDUS_ENVELOPE_GAUSS && !(L.fwhm > 0)) return fail(h, EDUS_ERR_ARG, "gaussian laser needs fwhm > 0");
        if (L.envelope != EDUS_ENVELOPE_SIN2 && L.envelope != EDUS_ENVELOPE_GAUSS)
            return fail(h, EDUS_ERR_ARG, "unknown envelope");
    }
    h->lasers[b] = v;
    return EDUS_OK;
}

int edus_set_state(edus_handle* h, int b, const double* rho_k) {
    if (!h || !rho_k) return EDUS_ERR_ARG;
    if (b < 0 || b >= h->B) return fail(h, EDUS_ERR_ARG, "solve index out of range");
    CU(h, cudaSetDevice(h->d.device));
    dim3 tb(32, 8), tg((h->Nk + 31) / 32, (h->P + 31) / 32);
    CU(h, cudaMemcpyAsync(h->stage, rho_k, h->S * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
    transpose_kp_to_pk<<<tg, tb, 0, h->stream>>>(h->stage, h->y + (size_t)b * h->S, h->Nk, h->P);
    h->launches++;
    CU(h, cudaGetLastError());
    if (h->packed) {
        if (!h->model_ready) return fail(h, EDUS_ERR_ARG, "the packed forms need edus_upload_model before edus_set_state");
        int rc;
        if (!h->ref_fixed && (rc = fix_reference(h, b))) return rc;
        const long long nq = (long long)h->Sq;
        pack_delta<<<grid_for(nq), 256, 0, h->stream>>>(h->y + (size_t)b * h->S, h->ref_full, h->py + (size_t)b * h->Sq,
                                                        h->qnm, h->nb, h->Pq, h->Nk);
        h->launches++;
        CU(h, cudaGetLastError());
    }
    h->anchored = false;  // split form: the next step anchors at the new state
    CU(h, cudaStreamSynchronize(h->stream));
    return EDUS_OK;
}

int edus_get_state(edus_handle* h, int b, double* rho_k) {
    if (!h || !rho_k) return EDUS_ERR_ARG;
    if (b < 0 || b >= h->B) return fail(h, EDUS_ERR_ARG, "solve index out of range");
    CU(h, cudaSetDevice(h->d.device));
    if (h->packed) {
        int rc;
        if ((rc = unpack_state(h, b))) return rc;
    }
    dim3 tb(32, 8), tg((h->P + 31) / 32, (h->Nk + 31) / 32);
    transpose_pk_to_kp<<<tg, tb, 0, h->stream>>>(h->y + (size_t)b * h->S, h->stage, h->Nk, h->P);
    h->launches++;
    CU(h, cudaGetLastError());
    CU(h, cudaMemcpyAsync(rho_k, h->stage, h->S * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    CU(h, cudaStreamSynchronize(h->stream));
    return check_status(h);
}

int edus_set_time(edus_handle* h, double t) {
    if (!h) return EDUS_ERR_ARG;
    h->t = t;
    return EDUS_OK;
}

int edus_get_time(const edus_handle* h, double* t) {
    if (!h || !t) return EDUS_ERR_ARG;
    *t = h->t;
    return EDUS_OK;
}

int edus_rhs(edus_handle* h, double t, const double* in_k, double* out_k) {
    if (!h || !in_k || !out_k) return EDUS_ERR_ARG;
    if (!h->model_ready) return fail(h, EDUS_ERR_ARG, "edus_upload_model must be called first");
    CU(h, cudaSetDevice(h->d.device));
    if (h->split && !h->anchored) {
        int rc0;
        if ((rc0 = anchor_split(h))) return rc0;
    }
    int rc;
    if (!h->tmp_in) {
        if ((rc = dalloc(h, (void**)&h->tmp_in, h->S * sizeof(double2)))) return rc;
        if ((rc = dalloc(h, (void**)&h->tmp_out, h->S * sizeof(double2)))) return rc;
    }
    // field of solve 0 at time t, in slot 0 of the table (wait for the
    // previous user of the pinned buffer)
    CU(h, cudaEventSynchronize(h->field_ev[0]));
    field_at(h->lasers[0], h->A, t, h->field_host[0][0]);
    if (h->kg_n > 0) h->field_host[0][0].g[0] = h->field_host[0][0].g[1] = h->field_host[0][0].g[2] = 0.0;
    if (h->peierls) peierls_field(h, 0, t, h->field_host[0][0]);
    CU(h, cudaMemcpyAsync(h->field, h->field_host[0], sizeof(StageField), cudaMemcpyHostToDevice, h->stream));
    CU(h, cudaEventRecord(h->field_ev[0], h->stream));
    dim3 tb(32, 8), tg((h->Nk + 31) / 32, (h->P + 31) / 32);
    CU(h, cudaMemcpyAsync(h->stage, in_k, h->S * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
    transpose_kp_to_pk<<<tg, tb, 0, h->stream>>>(h->stage, h->tmp_in, h->Nk, h->P);
    h->launches++;
    if ((rc = launch_plane(h, h->tmp_in, 0, h->G, h->Hee, 0, h->field, 1))) return rc;
    StageArgs a = base_args(h);
    a.rho = h->tmp_in;
    a.field = h->field;
    a.out = h->tmp_out;
    if ((rc = launch_comm(h, MODE_RHS, a, 1))) return rc;
    dim3 tg2((h->P + 31) / 32, (h->Nk + 31) / 32);
    transpose_pk_to_kp<<<tg2, tb, 0, h->stream>>>(h->tmp_out, h->stage, h->Nk, h->P);
    h->launches++;
    CU(h, cudaGetLastError());
    CU(h, cudaMemcpyAsync(out_k, h->stage, h->S * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    CU(h, cudaStreamSynchronize(h->stream));
    return check_status(h);
}

// Host field table of `cnt` steps from the handle's time: stage times as
// DESolver uses them, CurrentTime accumulated by += dt (DESolver.hpp:167-186,
// 205-219); tab[(i * stages + s) * B + b].
static void fill_field_table(edus_handle* h, int cnt, StageField* tab) {
    const int nst = h->d.solver == EDUS_SOLVER_RK ? 4 : 1;
    const double dt = h->d.dt;
    double t = h->t;
    for (int i = 0; i < cnt; ++i) {
        double ts[4] = {t, t + dt / 2., t + dt / 2., t + dt};
        for (int s = 0; s < nst; ++s)
            for (int b = 0; b < h->B; ++b) {
                StageField& f = tab[((size_t)i * nst + s) * h->B + b];
                field_at(h->lasers[b], h->A, ts[s], f);
                if (h->kg_n > 0) f.g[0] = f.g[1] = f.g[2] = 0.0;  // the gradient is the k stencil
                if (h->peierls) peierls_field(h, b, ts[s], f);
            }
        t += dt;
    }
}

// Kernels of `cnt` steps of the full-matrix forms (FP64, SPLIT32) on the
// handle's stream, the field table of those steps being in h->field; advances
// the handle's time and AB ring.
static int launch_plain_steps(edus_handle* h, int cnt) {
    const bool rk = h->d.solver == EDUS_SOLVER_RK;
    const int nst = rk ? 4 : 1;
    const double dt = h->d.dt;
    const int B = h->B;
    const long long bs = (long long)h->S;
    int rc;
    for (int i = 0; i < cnt; ++i) {
        if (h->split && (!h->anchored || h->since_anchor >= h->anchor_every)) {
            if ((rc = anchor_split(h))) return rc;
        }
        h->since_anchor++;
        const StageField* fs = h->field + (size_t)i * nst * B;
        StageArgs a = base_args(h);
        a.y = h->y;
        if (rk) {
            a.aux = h->aux;
            a.acc = h->acc;
            const double c0[4] = {dt / 2., dt / 2., dt, dt / 6.};
            const double c1[4] = {dt / 6., dt / 3., dt / 3., 0.};
            for (int s = 0; s < 4; ++s) {
                const double2* in = (s == 0) ? h->y : h->aux;
                if ((rc = launch_plane(h, in, bs, h->G, h->Hee, bs, fs + (size_t)s * B, B))) return rc;
                a.rho = in;
                a.field = fs + (size_t)s * B;
                a.c[0] = c0[s];
                a.c[1] = c1[s];
                if ((rc = launch_comm(h, MODE_RK1 + s, a, B))) return rc;
            }
        } else {
            if ((rc = launch_plane(h, h->y, bs, h->G, h->Hee, bs, fs, B))) return rc;
            a.rho = h->y;
            a.field = fs;
            a.order = h->d.order;
            for (int q = 0; q < h->d.order; ++q) {
                a.hist[q] = h->hist[h->index[q]];
                a.c[q] = dt * h->beta[q];
            }
            if ((rc = launch_comm(h, MODE_AB, a, B))) return rc;
            // rotate the ring (DESolver.hpp:212-217)
            const int ord = h->d.order;
            int tmp = h->index[ord - 1];
            for (int q = ord - 1; q > 0; --q) h->index[q] = h->index[q - 1];
            h->index[0] = tmp;
        }
        h->t += dt;
    }
    return EDUS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Fused sweep (edus_sweep_step with use_graph = 2).  The handles form two
// groups by plane size: planes above 110 KB (one CTA per SM) and the rest
// (two per SM).  Each group advances on its own stream with, per RK stage,
// one persistent plane launch over every plane of its solves and one
// persistent commutator launch per commutator kind (FP64 tensor cores, CUDA
// cores) over every k tile of its solves (csrc/sweep_kernels.cuh); the two
// groups are independent, so one group's transforms overlap the other's
// commutators.
struct FusedGroup {
    int np = 0, ncm = 0, ncc = 0;   // plane items, tensor-core and CUDA-core tiles
    int off = 0;                    // first item in FusedSweep::items
    size_t sm_p = 0, sm_cm = 0, sm_cc = 0;
    int thr_p = 256, grid_p = 0, grid_cm = 0, grid_cc = 0;
};

struct FusedSweep {
    int n = 0, C = 0;
    bool wide = false;
    PlanePlan* plans = nullptr;
    SweepPlaneDesc* pdesc = nullptr;
    StageArgs* args = nullptr;  // [C][4][n]: handle i at step k of a chunk, stage s
    std::vector<StageArgs> host_args;  // the same on the host (the commutators take them as a parameter)
    int4* items = nullptr;      // per group: planes | tensor-core tiles | CUDA-core tiles
    FusedGroup g[2];            // 0: planes above 110 KB, 1: the others
    int thr_c = 256;
    bool tiles5 = true;         // every tensor-core shape needs at most 5 tiles per warp
    int* count = nullptr;       // [C][4][2][3] work counters, zeroed per chunk
    cudaStream_t s1 = nullptr;  // the second group's stream
    cudaEvent_t fork = nullptr, join = nullptr;
    void release() {
        cudaFree(plans);
        cudaFree(pdesc);
        cudaFree(args);
        cudaFree(items);
        cudaFree(count);
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        if (s1) cudaStreamDestroy(s1);
        plans = nullptr;
        pdesc = nullptr;
        args = nullptr;
        items = nullptr;
        count = nullptr;
        fork = join = nullptr;
        s1 = nullptr;
    }
};

// Planes of at most this many bytes leave room for two CTAs on an SM.
constexpr size_t kSweepSmallPlane = 110 * 1024;

static bool fused_eligible(const edus_handle* h) {
    return h->d.solver == EDUS_SOLVER_RK && !h->d.coulomb && !h->packed && !h->split && !h->hplanes && !h->peierls &&
           h->kg_n == 0 && !h->profiling;
}

static int fused_setup(edus_handle* const* hs, int n, int C, FusedSweep& f) {
    edus_handle* h0 = hs[0];
    if (n > kSweepMaxShapes)
        return fail(h0, EDUS_ERR_UNSUPPORTED,
                    "the fused sweep takes at most " + std::to_string(kSweepMaxShapes) + " handles");
    f.n = n;
    f.C = C;
    std::vector<PlanePlan> plans(n);
    std::vector<StageArgs> args((size_t)C * 4 * n);
    struct Item {
        int4 v;
        double cost;
    };
    std::vector<Item> planes[2], comm_m[2], comm_c[2];
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h0->d.device);
    for (int i = 0; i < n; ++i) {
        edus_handle* h = hs[i];
        plans[i] = h->plan;
        if (plane_launch(h->plan).variant == 2) f.wide = true;
        const double dt = h->d.dt;
        const double c0[4] = {dt / 2., dt / 2., dt, dt / 6.};
        const double c1[4] = {dt / 6., dt / 3., dt / 3., 0.};
        for (int k = 0; k < C; ++k)
            for (int st = 0; st < 4; ++st) {
                StageArgs a = base_args(h);
                a.y = h->y;
                a.aux = h->aux;
                a.acc = h->acc;
                a.rho = st == 0 ? h->y : h->aux;
                a.field = h->field + ((size_t)k * 4 + st) * h->B;
                a.c[0] = c0[st];
                a.c[1] = c1[st];
                args[((size_t)k * 4 + st) * n + i] = a;
            }
        const size_t plane_bytes = (size_t)h->Nk * sizeof(double2);
        const int gi = plane_bytes > kSweepSmallPlane ? 0 : 1;
        FusedGroup& G = f.g[gi];
        G.sm_p = std::max(G.sm_p, plane_bytes);
        const double pcost = (double)h->Nk * std::log2((double)std::max(h->Nk, 2));
        for (int b = 0; b < h->B; ++b)
            for (int p = 0; p < h->P; ++p) planes[gi].push_back({make_int4(i, b, p, 0), pcost});
        const int ntile = (h->Nk + h->TK - 1) / h->TK;
        const double ccost = (double)h->TK * h->nb * h->nb * h->nb;
        auto& cdst = h->comm_mma ? comm_m[gi] : comm_c[gi];
        for (int b = 0; b < h->B; ++b)
            for (int t = 0; t < ntile; ++t) cdst.push_back({make_int4(i, b, t, 0), ccost});
        if (h->comm_mma) {
            const MmaGeom mg = mma_geometry(h->nb);
            if ((mg.tiles * mg.tiles + mg.warps_per_k - 1) / mg.warps_per_k > 5) f.tiles5 = false;
        }
        if (h->comm_mma) G.sm_cm = std::max(G.sm_cm, (size_t)h->smem_comm);
        else G.sm_cc = std::max(G.sm_cc, (size_t)h->smem_comm);
        f.thr_c = std::max(f.thr_c, h->comm_threads);
    }
    f.thr_c = f.thr_c <= 256 ? 256 : 512;
    auto by_cost = [](const Item& x, const Item& y) { return x.cost > y.cost; };
    std::vector<int4> items;
    for (int gi = 0; gi < 2; ++gi) {
        for (auto* v : {&planes[gi], &comm_m[gi], &comm_c[gi]}) std::stable_sort(v->begin(), v->end(), by_cost);
        FusedGroup& G = f.g[gi];
        G.off = (int)items.size();
        G.np = (int)planes[gi].size();
        G.ncm = (int)comm_m[gi].size();
        G.ncc = (int)comm_c[gi].size();
        G.thr_p = gi == 0 ? 512 : 256;
        for (auto* v : {&planes[gi], &comm_m[gi], &comm_c[gi]})
            for (auto& x : *v) items.push_back(x.v);
    }
    auto alloc_copy = [&](void** p, const void* src, size_t bytes) -> int {
        if (cudaMalloc(p, bytes) != cudaSuccess) return fail(h0, EDUS_ERR_CUDA, "fused sweep: cudaMalloc failed");
        if (src && cudaMemcpy(*p, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(h0, EDUS_ERR_CUDA, "fused sweep: upload failed");
        return EDUS_OK;
    };
    int rc;
    if ((rc = alloc_copy((void**)&f.plans, plans.data(), n * sizeof(PlanePlan)))) return rc;
    std::vector<SweepPlaneDesc> pd(n);
    for (int i = 0; i < n; ++i) {
        edus_handle* h = hs[i];
        pd[i] = SweepPlaneDesc{f.plans + i, h->roots, h->rpos, h->G, (long long)h->S, h->Nk, 1.0 / h->Nk};
    }
    if ((rc = alloc_copy((void**)&f.pdesc, pd.data(), n * sizeof(SweepPlaneDesc)))) return rc;
    if ((rc = alloc_copy((void**)&f.args, args.data(), args.size() * sizeof(StageArgs)))) return rc;
    f.host_args = args;
    if ((rc = alloc_copy((void**)&f.items, items.data(), std::max<size_t>(items.size(), 1) * sizeof(int4)))) return rc;
    if ((rc = alloc_copy((void**)&f.count, nullptr, (size_t)C * 4 * 2 * 3 * sizeof(int)))) return rc;
    if (cudaStreamCreateWithFlags(&f.s1, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&f.fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&f.join, cudaEventDisableTiming) != cudaSuccess)
        return fail(h0, EDUS_ERR_CUDA, "fused sweep: stream/event creation failed");
    // kernel attributes (process-wide: the device maximum less the kernel's
    // static shared memory, as for every kernel here)
    const int optin = device_smem_optin(h0->d.device);
    for (const FusedGroup& G : f.g)
        if ((size_t)optin < std::max(G.sm_p, std::max(G.sm_cm, G.sm_cc)) + 64)
            return fail(h0, EDUS_ERR_UNSUPPORTED, "fused sweep: a plane exceeds shared memory");
    auto dyn_max = [optin](auto kernel) {
        cudaFuncAttributes fa{};
        cudaFuncGetAttributes(&fa, kernel);
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
    };
    dyn_max(sweep_plane_kernel<kRadixCommon, 256>);
    dyn_max(sweep_plane_kernel<kRadixCommon, 512>);
    dyn_max(sweep_plane_kernel<kRadixAll, 256>);
    dyn_max(sweep_plane_kernel<kRadixAll, 512>);
#define EDUS_SWEEP_ATTR(M)                             \
    dyn_max(sweep_comm_kernel<M, 256, true, 5>);       \
    dyn_max(sweep_comm_kernel<M, 256, true, 8>);       \
    dyn_max(sweep_comm_kernel<M, 256, false>);         \
    dyn_max(sweep_comm_kernel<M, 512, true, 5>);       \
    dyn_max(sweep_comm_kernel<M, 512, true, 8>);       \
    dyn_max(sweep_comm_kernel<M, 512, false>);
    EDUS_SWEEP_ATTR(MODE_RK1)
    EDUS_SWEEP_ATTR(MODE_RK2)
    EDUS_SWEEP_ATTR(MODE_RK3)
    EDUS_SWEEP_ATTR(MODE_RK4)
#undef EDUS_SWEEP_ATTR
    // grids: as many CTAs as fit on the device at once
    for (FusedGroup& G : f.g) {
        int per = 0;
        if (G.thr_p == 512) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, sweep_plane_kernel<kRadixCommon, 512>, 512, G.sm_p);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, sweep_plane_kernel<kRadixCommon, 256>, 256, G.sm_p);
        G.grid_p = nsm * std::max(per, 1);
        per = 0;
        if (f.thr_c == 256) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, sweep_comm_kernel<MODE_RK1, 256, true, 8>, 256, G.sm_cm);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, sweep_comm_kernel<MODE_RK1, 512, true, 8>, 512, G.sm_cm);
        G.grid_cm = nsm * std::max(per, 1);
        per = 0;
        if (f.thr_c == 256) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, sweep_comm_kernel<MODE_RK1, 256, false>, 256, G.sm_cc);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, sweep_comm_kernel<MODE_RK1, 512, false>, 512, G.sm_cc);
        G.grid_cc = nsm * std::max(per, 1);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(h0, EDUS_ERR_CUDA, std::string("fused sweep set-up: ") + cudaGetErrorString(e));
    return EDUS_OK;
}

// One group's launches for stage `mode` of one step: planes, then the
// commutators of each kind.
template <int MODE>
static int fused_group_stage(const FusedSweep& f, const FusedGroup& G, const StageArgs* a,
                             const SweepStageArgs& pa, int* cnt, cudaStream_t st) {
    int launched = 0;
    const int4* ip = f.items + G.off;
    const int4* im = ip + G.np;
    const int4* ic = im + G.ncm;
    if (G.np) {
        if (G.thr_p == 512) {
            if (f.wide) sweep_plane_kernel<kRadixAll, 512><<<G.grid_p, 512, G.sm_p, st>>>(f.pdesc, a, ip, G.np, cnt);
            else sweep_plane_kernel<kRadixCommon, 512><<<G.grid_p, 512, G.sm_p, st>>>(f.pdesc, a, ip, G.np, cnt);
        } else {
            if (f.wide) sweep_plane_kernel<kRadixAll, 256><<<G.grid_p, 256, G.sm_p, st>>>(f.pdesc, a, ip, G.np, cnt);
            else sweep_plane_kernel<kRadixCommon, 256><<<G.grid_p, 256, G.sm_p, st>>>(f.pdesc, a, ip, G.np, cnt);
        }
        ++launched;
    }
    if (G.ncm) {
        if (f.thr_c == 256) {
            if (f.tiles5) sweep_comm_kernel<MODE, 256, true, 5><<<G.ncm, 256, G.sm_cm, st>>>(pa, im);
            else sweep_comm_kernel<MODE, 256, true, 8><<<G.ncm, 256, G.sm_cm, st>>>(pa, im);
        } else {
            if (f.tiles5) sweep_comm_kernel<MODE, 512, true, 5><<<G.ncm, 512, G.sm_cm, st>>>(pa, im);
            else sweep_comm_kernel<MODE, 512, true, 8><<<G.ncm, 512, G.sm_cm, st>>>(pa, im);
        }
        ++launched;
    }
    if (G.ncc) {
        if (f.thr_c == 256) sweep_comm_kernel<MODE, 256, false><<<G.ncc, 256, G.sm_cc, st>>>(pa, ic);
        else sweep_comm_kernel<MODE, 512, false><<<G.ncc, 512, G.sm_cc, st>>>(pa, ic);
        ++launched;
    }
    return launched;
}

// Kernel launches of one fused step (all groups, four stages).
static int fused_launches_per_step(const FusedSweep& f) {
    int n = 0;
    for (const FusedGroup& G : f.g) n += (G.np ? 1 : 0) + (G.ncm ? 1 : 0) + (G.ncc ? 1 : 0);
    return 4 * n;
}

// `cnt` RK4 steps of every handle of the sweep: group 0 on st, group 1 on
// the sweep's second stream, forked from and joined into st.
static int fused_launch_steps(edus_handle* const* hs, const FusedSweep& f, int cnt, cudaStream_t st) {
    edus_handle* h0 = hs[0];
    if (cudaMemsetAsync(f.count, 0, (size_t)f.C * 4 * 2 * 3 * sizeof(int), st) != cudaSuccess ||
        cudaEventRecord(f.fork, st) != cudaSuccess || cudaStreamWaitEvent(f.s1, f.fork, 0) != cudaSuccess)
        return fail(h0, EDUS_ERR_CUDA, "fused sweep: counter reset / fork failed");
    static SweepStageArgs pa;  // launch parameter, copied at each launch
    for (int k = 0; k < cnt; ++k) {
        for (int s = 0; s < 4; ++s) {
            const StageArgs* a = f.args + ((size_t)k * 4 + s) * f.n;
            const StageArgs* ha = f.host_args.data() + ((size_t)k * 4 + s) * f.n;
            for (int i = 0; i < f.n; ++i) pa.a[i] = ha[i];
            for (int gi = 0; gi < 2; ++gi) {
                int* c = f.count + (((size_t)k * 4 + s) * 2 + gi) * 3;
                const cudaStream_t sg = gi == 0 ? st : f.s1;
                switch (s) {
                    case 0: fused_group_stage<MODE_RK1>(f, f.g[gi], a, pa, c, sg); break;
                    case 1: fused_group_stage<MODE_RK2>(f, f.g[gi], a, pa, c, sg); break;
                    case 2: fused_group_stage<MODE_RK3>(f, f.g[gi], a, pa, c, sg); break;
                    default: fused_group_stage<MODE_RK4>(f, f.g[gi], a, pa, c, sg); break;
                }
            }
        }
        for (int i = 0; i < f.n; ++i) hs[i]->t += hs[i]->d.dt;
        h0->launches += fused_launches_per_step(f);
    }
    if (cudaEventRecord(f.join, f.s1) != cudaSuccess || cudaStreamWaitEvent(st, f.join, 0) != cudaSuccess)
        return fail(h0, EDUS_ERR_CUDA, "fused sweep: join failed");
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(h0, EDUS_ERR_CUDA, std::string("fused sweep launch: ") + cudaGetErrorString(e));
    return EDUS_OK;
}

extern "C" {

// States up to this size step through CUDA graphs when a call covers enough
// steps (edus_step): their steps take tens of microseconds, of which the
// launches are a large part.
constexpr size_t kGraphStepBytes = 16u << 20;
constexpr int kGraphStepMin = 512;

int edus_step(edus_handle* h, int n) {
    if (!h || n < 0) return EDUS_ERR_ARG;
    if (!h->model_ready) return fail(h, EDUS_ERR_ARG, "edus_upload_model must be called first");
    CU(h, cudaSetDevice(h->d.device));
    const bool rk = h->d.solver == EDUS_SOLVER_RK;
    // small RK4 problems in the FP64 form: the same launches, 32 steps per
    // CUDA graph replay (captured once per call)
    if (rk && !h->packed && !h->split && !h->profiling && n >= kGraphStepMin &&
        (size_t)h->S * h->B * sizeof(double2) <= kGraphStepBytes)
        return edus_sweep_step(&h, 1, n, 1);
    const int nst = rk ? 4 : 1;
    const double dt = h->d.dt;
    const int B = h->B;
    int rc;
    for (int s0 = 0; s0 < n; s0 += h->chunk) {
        const int cnt = std::min(h->chunk, n - s0);
        // host field table for this chunk: stage times as DESolver uses them,
        // with CurrentTime accumulated by += dt (DESolver.hpp:167-186, 205-219)
        const int buf = h->field_cur;
        h->field_cur ^= 1;
        CU(h, cudaEventSynchronize(h->field_ev[buf]));
        StageField* tab = h->field_host[buf];
        fill_field_table(h, cnt, tab);
        // the device table of the previous chunk is no longer read once the
        // kernels before this copy (same stream) have run
        CU(h, cudaMemcpyAsync(h->field, tab, (size_t)cnt * nst * B * sizeof(StageField), cudaMemcpyHostToDevice, h->stream));
        CU(h, cudaEventRecord(h->field_ev[buf], h->stream));
        if (h->packed) {
            if (!h->ref_fixed) return fail(h, EDUS_ERR_ARG, "the packed forms need edus_set_state before edus_step");
            for (int i = 0; i < cnt; ++i) {
                const StageField* fs = h->field + (size_t)i * nst * B;
                PackedArgs a = base_pargs(h);
                if (rk) {
                    const double c0[4] = {dt / 2., dt / 2., dt, dt / 6.};
                    const double c1[4] = {dt / 6., dt / 3., dt / 3., 0.};
                    for (int s = 0; s < 4; ++s) {
                        const void* in = (s == 0) ? (const void*)h->py : (const void*)h->paux;
                        if ((rc = launch_pplane(h, in, s != 0, fs + (size_t)s * B, B))) return rc;
                        a.in = in;
                        a.field = fs + (size_t)s * B;
                        a.c[0] = c0[s];
                        a.c[1] = c1[s];
                        if ((rc = launch_pcomm(h, MODE_RK1 + s, a, B))) return rc;
                    }
                } else {
                    if ((rc = launch_pplane(h, h->py, false, fs, B))) return rc;
                    a.in = h->py;
                    a.field = fs;
                    a.order = h->d.order;
                    for (int q = 0; q < h->d.order; ++q) {
                        a.hist[q] = h->phist[h->index[q]];
                        a.c[q] = dt * h->beta[q];
                    }
                    if ((rc = launch_pcomm(h, MODE_AB, a, B))) return rc;
                    const int ord = h->d.order;
                    int tmp = h->index[ord - 1];
                    for (int q = ord - 1; q > 0; --q) h->index[q] = h->index[q - 1];
                    h->index[0] = tmp;
                }
                h->t += dt;
            }
            continue;
        }
        if ((rc = launch_plain_steps(h, cnt))) return rc;
    }
    return EDUS_OK;
}

int edus_sweep_step(edus_handle* const* hs, int n, int steps, int use_graph) {
    if (!hs || n < 1 || steps < 0) return EDUS_ERR_ARG;
    for (int i = 0; i < n; ++i)
        if (!hs[i]) return EDUS_ERR_ARG;
    edus_handle* h0 = hs[0];
    bool graph = use_graph != 0;
    const bool fused = use_graph == 2;
    for (int i = 0; i < n; ++i) {
        edus_handle* h = hs[i];
        if (h->d.device != h0->d.device) return fail(h0, EDUS_ERR_ARG, "a sweep's handles share one device");
        if (!h->model_ready) return fail(h, EDUS_ERR_ARG, "edus_upload_model must be called first");
        if (h->packed || h->split)
            return fail(h, EDUS_ERR_UNSUPPORTED, "a sweep steps the FP64 form (step other forms with edus_step)");
        for (int j = 0; j < i; ++j)
            if (hs[j] == h) return fail(h, EDUS_ERR_ARG, "a handle appears twice in the sweep");
        if (h->d.solver != EDUS_SOLVER_RK || h->profiling) graph = false;
        if (fused && !fused_eligible(h))
            return fail(h, EDUS_ERR_UNSUPPORTED,
                        "the fused sweep steps RK4 independent-particle handles (no HSEX, Peierls, k-space gradient "
                        "or profiling)");
    }
    if (steps == 0) return EDUS_OK;
    CU(h0, cudaSetDevice(h0->d.device));
    constexpr int C = 32;  // steps per captured chunk (<= the field-table capacity)
    cudaStream_t s0 = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join(n, nullptr);
    cudaGraphExec_t exec = nullptr;
    FusedSweep fs;
    int rc = EDUS_OK;
    auto cleanup = [&]() {
        if (s0) cudaStreamSynchronize(s0);
        fs.release();
        if (exec) cudaGraphExecDestroy(exec);
        for (auto& e : join)
            if (e) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        if (s0) cudaStreamDestroy(s0);
    };
    if (cudaStreamCreateWithFlags(&s0, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) != cudaSuccess) {
        cleanup();
        return fail(h0, EDUS_ERR_CUDA, "sweep stream/event creation failed");
    }
    for (auto& e : join)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            cleanup();
            return fail(h0, EDUS_ERR_CUDA, "sweep event creation failed");
        }
    {
        const cudaError_t pend = cudaGetLastError();
        if (pend != cudaSuccess) {
            cleanup();
            return fail(h0, EDUS_ERR_CUDA, std::string("sweep set-up: ") + cudaGetErrorString(pend));
        }
    }
    if (fused && (rc = fused_setup(hs, n, C, fs))) {
        cleanup();
        return rc;
    }
    // every handle's launches of `cnt` steps, forked from and joined into s0
    // (fused: the persistent launches of every handle, on s0)
    auto launch_all = [&](int cnt) -> int {
        {
            const cudaError_t pend = cudaGetLastError();
            if (pend != cudaSuccess) return fail(h0, EDUS_ERR_CUDA, std::string("sweep, before launches: ") + cudaGetErrorString(pend));
        }
        if (fused) return fused_launch_steps(hs, fs, cnt, s0);
        if (cudaEventRecord(fork, s0) != cudaSuccess) return fail(h0, EDUS_ERR_CUDA, "cudaEventRecord failed");
        for (int i = 0; i < n; ++i) {
            edus_handle* h = hs[i];
            if (cudaStreamWaitEvent(h->stream, fork, 0) != cudaSuccess)
                return fail(h, EDUS_ERR_CUDA, "cudaStreamWaitEvent failed");
            int r;
            if ((r = launch_plain_steps(h, cnt))) return r;
            if (cudaEventRecord(join[i], h->stream) != cudaSuccess || cudaStreamWaitEvent(s0, join[i], 0) != cudaSuccess)
                return fail(h, EDUS_ERR_CUDA, "sweep join failed");
        }
        return EDUS_OK;
    };
    for (int done = 0; done < steps && rc == EDUS_OK;) {
        const int cnt = std::min(C, steps - done);
        // field tables of the chunk, uploaded on s0 ahead of the chunk's kernels
        for (int i = 0; i < n && rc == EDUS_OK; ++i) {
            edus_handle* h = hs[i];
            const int nst = h->d.solver == EDUS_SOLVER_RK ? 4 : 1;
            const int buf = h->field_cur;
            h->field_cur ^= 1;
            if (cudaEventSynchronize(h->field_ev[buf]) != cudaSuccess) rc = fail(h, EDUS_ERR_CUDA, "event sync failed");
            StageField* tab = h->field_host[buf];
            fill_field_table(h, cnt, tab);
            if (rc == EDUS_OK &&
                (cudaMemcpyAsync(h->field, tab, (size_t)cnt * nst * h->B * sizeof(StageField), cudaMemcpyHostToDevice,
                                 s0) != cudaSuccess ||
                 cudaEventRecord(h->field_ev[buf], s0) != cudaSuccess))
                rc = fail(h, EDUS_ERR_CUDA, "field table upload failed");
        }
        if (rc) break;
        if (graph && cnt == C) {
            if (!exec) {
                // capture one chunk of every handle once; replays reuse it (the
                // kernels read the field table from the same device buffers)
                std::vector<double> t0(n);
                std::vector<unsigned long long> l0(n);
                for (int i = 0; i < n; ++i) {
                    t0[i] = hs[i]->t;
                    l0[i] = hs[i]->launches;
                }
                cudaGraph_t g = nullptr;
                if (cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
                    rc = fail(h0, EDUS_ERR_CUDA, "cudaStreamBeginCapture failed");
                    break;
                }
                const int r = launch_all(C);
                const cudaError_t ec = cudaStreamEndCapture(s0, &g);
                for (int i = 0; i < n; ++i) {  // the capture ran nothing
                    hs[i]->t = t0[i];
                    hs[i]->launches = l0[i];
                }
                if (r || ec != cudaSuccess || cudaGraphInstantiate(&exec, g, 0) != cudaSuccess) {
                    if (g) cudaGraphDestroy(g);
                    rc = r ? r : fail(h0, EDUS_ERR_CUDA, "capture of the sweep chunk failed");
                    break;
                }
                cudaGraphDestroy(g);
            }
            if (cudaGraphLaunch(exec, s0) != cudaSuccess) {
                rc = fail(h0, EDUS_ERR_CUDA, "cudaGraphLaunch failed");
                break;
            }
            for (int i = 0; i < n; ++i) {
                for (int k = 0; k < C; ++k) hs[i]->t += hs[i]->d.dt;  // as the launches would
                if (!fused) hs[i]->launches += 8LL * C;
            }
            if (fused) h0->launches += (unsigned long long)C * fused_launches_per_step(fs);
        } else {
            rc = launch_all(cnt);
        }
        done += cnt;
    }
    cleanup();
    if (rc) return rc;
    for (int i = 0; i < n; ++i)
        if ((rc = check_status(hs[i]))) return rc;
    return EDUS_OK;
}

int edus_autotune(edus_handle* h, int* plane_threads, int* comm_tensor) {
    if (!h) return EDUS_ERR_ARG;
    if (!h->model_ready) return fail(h, EDUS_ERR_ARG, "edus_upload_model must be called first");
    if (h->packed) return fail(h, EDUS_ERR_UNSUPPORTED, "the packed forms have their own launch geometry");
    CU(h, cudaSetDevice(h->d.device));
    CU(h, cudaStreamSynchronize(h->stream));
    // a field along every axis, on every solve, for the timed launches
    std::vector<StageField> f(h->B);
    for (auto& x : f) {
        for (int i = 0; i < 3; ++i) x.E[i] = 1e-3;
        for (int c = 0; c < 3; ++c) x.g[c] = 1e-3 * (h->A[0 * 3 + c] + h->A[1 * 3 + c] + h->A[2 * 3 + c]);
    }
    StageField* df = nullptr;
    CU(h, cudaMalloc((void**)&df, f.size() * sizeof(StageField)));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const bool prof = h->profiling;
    h->profiling = false;
    int rc = EDUS_OK;
    const long long bs = (long long)h->S;
    auto time_it = [&](auto&& launch) -> float {
        for (int w = 0; w < 2; ++w) launch();
        cudaEventRecord(e0, h->stream);
        for (int r = 0; r < 5; ++r) launch();
        cudaEventRecord(e1, h->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms;
    };
    cudaMemcpy(df, f.data(), f.size() * sizeof(StageField), cudaMemcpyHostToDevice);
    // plane kernel: thread counts, multiples of 32 up to the variant's maximum
    {
        const int tmax = h->plane_cfg.persist ? (h->plane_cfg.variant == 1 ? kPersist89Threads : 256)
                                              : (h->plane_cfg.variant == 1 ? 768 : 512);
        const int keep = h->plane_cfg.threads;
        int best_t = keep;
        float best = 1e30f;
        for (int T = 128; T <= tmax; T += 32) {
            h->plane_cfg.threads = T;
            if (h->split) h->split_threads = T;
            const float ms = time_it([&] { launch_plane(h, h->y, bs, h->G, h->Hee, bs, df, h->B); });
            if (cudaGetLastError() != cudaSuccess) continue;
            if (ms < best) {
                best = ms;
                best_t = T;
            }
        }
        h->plane_cfg.threads = best_t;
        if (h->split) h->split_threads = best_t;
        if (plane_threads) *plane_threads = best_t;
    }
    // commutator: the CUDA-core against the tensor-core kernel (the TMA kernel
    // of the fused HSEX path has one geometry)
    {
        const bool fused = h->d.coulomb && (h->nS > 0 || h->split) && h->comm_ws;
        if (!fused) {
            StageArgs a = base_args(h);
            a.rho = h->y;
            a.field = df;
            a.out = h->stage;
            float best = 1e30f;
            bool best_mma = h->comm_mma;
            for (int mma = 0; mma < 2; ++mma) {
                const CommGeom cg = comm_geometry(h->nb);
                const MmaGeom mg = mma_geometry(h->nb);
                h->comm_mma = mma != 0;
                h->TK = mma ? mg.TK : cg.TK;
                h->comm_threads = mma ? 256 : cg.threads;
                h->smem_comm = (int)(mma ? mg.smem : cg.smem);
                a.TK = h->TK;
                const float ms = time_it([&] { launch_comm(h, MODE_RHS, a, 1); });
                if (cudaGetLastError() != cudaSuccess) continue;
                if (ms < best) {
                    best = ms;
                    best_mma = mma != 0;
                }
            }
            const CommGeom cg = comm_geometry(h->nb);
            const MmaGeom mg = mma_geometry(h->nb);
            h->comm_mma = best_mma;
            h->TK = best_mma ? mg.TK : cg.TK;
            h->comm_threads = best_mma ? 256 : cg.threads;
            h->smem_comm = (int)(best_mma ? mg.smem : cg.smem);
        }
        if (comm_tensor) *comm_tensor = h->comm_mma ? 1 : 0;
    }
    h->profiling = prof;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const cudaError_t e = cudaStreamSynchronize(h->stream);
    cudaFree(df);
    if (e != cudaSuccess) rc = fail(h, EDUS_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(e));
    if (rc == EDUS_OK) rc = check_status(h);
    return rc;
}

int edus_state_rspace(edus_handle* h, int b, int nsel, const int* R_index, double* out) {
    if (!h || nsel < 0 || (nsel > 0 && (!R_index || !out))) return EDUS_ERR_ARG;
    if (b < 0 || b >= h->B) return fail(h, EDUS_ERR_ARG, "solve index out of range");
    if (nsel == 0) return EDUS_OK;
    CU(h, cudaSetDevice(h->d.device));
    int rc;
    if (h->packed && (rc = unpack_state(h, b))) return rc;
    std::vector<int> pos(nsel);
    for (int s = 0; s < nsel; ++s) {
        if (R_index[s] < 0 || R_index[s] >= h->Nk) return fail(h, EDUS_ERR_ARG, "R index out of range");
        pos[s] = position_of(h, R_index[s]);
    }
    double2* tmp = nullptr;
    int* dpos = nullptr;
    double2* dout = nullptr;
    CU(h, cudaMalloc((void**)&tmp, h->S * sizeof(double2)));
    if (cudaMalloc((void**)&dpos, nsel * sizeof(int)) != cudaSuccess ||
        cudaMalloc((void**)&dout, (size_t)nsel * h->P * sizeof(double2)) != cudaSuccess) {
        cudaFree(tmp);
        cudaFree(dpos);
        return fail(h, EDUS_ERR_NOMEM, "edus_state_rspace: allocation failed");
    }
    plane_to_R_kernel<kRadixAll, 256><<<h->P, 256, h->Nk * sizeof(double2), h->stream>>>(
        h->y + (size_t)b * h->S, tmp, h->roots, h->plan, 1.0 / h->Nk);
    cudaMemcpyAsync(dpos, pos.data(), nsel * sizeof(int), cudaMemcpyHostToDevice, h->stream);
    gather_R_kernel<<<grid_for((long long)nsel * h->P), 256, 0, h->stream>>>(tmp, dpos, nsel, h->P, h->Nk, dout);
    h->launches += 2;
    cudaMemcpyAsync(out, dout, (size_t)nsel * h->P * sizeof(double2), cudaMemcpyDeviceToHost, h->stream);
    const cudaError_t e = cudaStreamSynchronize(h->stream);
    cudaFree(tmp);
    cudaFree(dpos);
    cudaFree(dout);
    if (e != cudaSuccess) return fail(h, EDUS_ERR_CUDA, std::string("edus_state_rspace: ") + cudaGetErrorString(e));
    return EDUS_OK;
}

int edus_set_fock_override(edus_handle* h, int nsel, const int* R_index, const double* values) {
    if (!h || nsel < 0 || (nsel > 0 && (!R_index || !values))) return EDUS_ERR_ARG;
    if (nsel == 0) {
        if (h->nO) {
            CU(h, cudaStreamSynchronize(h->stream));
            h->nO = 0;
        }
        return EDUS_OK;
    }
    if (!h->d.coulomb || h->packed || h->split || !h->plane_cfg.persist)
        return fail(h, EDUS_ERR_UNSUPPORTED,
                    "a given Fock term needs the FP64 form with HSEX and a plane that fits two CTAs per SM");
    if (nsel > h->Nk) return fail(h, EDUS_ERR_ARG, "more lattice vectors than grid points");
    CU(h, cudaSetDevice(h->d.device));
    std::vector<int> pos(nsel);
    for (int s = 0; s < nsel; ++s) {
        if (R_index[s] < 0 || R_index[s] >= h->Nk) return fail(h, EDUS_ERR_ARG, "R index out of range");
        pos[s] = position_of(h, R_index[s]);
    }
    // values [nsel][nb][nb] -> [p][nsel]
    std::vector<double2> v((size_t)h->P * nsel);
    for (int s = 0; s < nsel; ++s)
        for (int p = 0; p < h->P; ++p)
            v[(size_t)p * nsel + s] =
                make_double2(values[2 * ((size_t)s * h->P + p)], values[2 * ((size_t)s * h->P + p) + 1]);
    CU(h, cudaStreamSynchronize(h->stream));  // kernels in flight may still read the previous values
    int rc;
    if (nsel > h->nO_cap) {
        if ((rc = dalloc(h, (void**)&h->opos, nsel * sizeof(int)))) return rc;
        if ((rc = dalloc(h, (void**)&h->oval, (size_t)h->P * nsel * sizeof(double2)))) return rc;
        h->nO_cap = nsel;
    }
    CU(h, cudaMemcpyAsync(h->opos, pos.data(), nsel * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    CU(h, cudaMemcpyAsync(h->oval, v.data(), v.size() * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
    CU(h, cudaStreamSynchronize(h->stream));
    h->nO = nsel;
    return EDUS_OK;
}

int edus_set_anchor_interval(edus_handle* h, int steps) {
    if (!h) return EDUS_ERR_ARG;
    if (!h->split) return fail(h, EDUS_ERR_ARG, "the anchor interval belongs to the split-precision form");
    if (steps < 1) return fail(h, EDUS_ERR_ARG, "the anchor interval must be >= 1 step");
    h->anchor_every = steps;
    return EDUS_OK;
}

int edus_synchronize(edus_handle* h) {
    if (!h) return EDUS_ERR_ARG;
    CU(h, cudaSetDevice(h->d.device));
    CU(h, cudaStreamSynchronize(h->stream));
    return check_status(h);
}

int edus_population_wannier(edus_handle* h, int b, double* pop) {
    if (!h || !pop) return EDUS_ERR_ARG;
    if (b < 0 || b >= h->B) return fail(h, EDUS_ERR_ARG, "solve index out of range");
    CU(h, cudaSetDevice(h->d.device));
    if (h->packed) {
        int rc;
        if ((rc = unpack_state(h, b))) return rc;
    }
    population_kernel<<<h->nb, 256, 0, h->stream>>>(h->y + (size_t)b * h->S, h->Nk, h->nb, h->popbuf);
    h->launches++;
    CU(h, cudaGetLastError());
    CU(h, cudaMemcpyAsync(pop, h->popbuf, h->nb * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CU(h, cudaStreamSynchronize(h->stream));
    return EDUS_OK;
}

int edus_get_stream(const edus_handle* h, void** stream) {
    if (!h || !stream) return EDUS_ERR_ARG;
    *stream = (void*)h->stream;
    return EDUS_OK;
}

int edus_set_wait_limit(edus_handle* h, int polls) {
    if (!h) return EDUS_ERR_ARG;
    h->wait_polls = polls >= 0 ? polls : (1 << 22);
    return EDUS_OK;
}

int edus_set_profiling(edus_handle* h, int on) {
    if (!h) return EDUS_ERR_ARG;
    if (on && !h->profiling) {
        CU(h, cudaStreamSynchronize(h->stream));
        prof_resolve(h);
        h->prof_ms[0] = h->prof_ms[1] = 0;
        h->prof_n[0] = h->prof_n[1] = 0;
    }
    h->profiling = on != 0;
    return EDUS_OK;
}

int edus_get_profile(edus_handle* h, int kind, double* total_ms, unsigned long long* launches) {
    if (!h || kind < 0 || kind > 1 || !total_ms || !launches) return EDUS_ERR_ARG;
    CU(h, cudaStreamSynchronize(h->stream));
    prof_resolve(h);
    *total_ms = h->prof_ms[kind];
    *launches = h->prof_n[kind];
    return EDUS_OK;
}

int edus_device_bytes(const edus_handle* h, unsigned long long* bytes) {
    if (!h || !bytes) return EDUS_ERR_ARG;
    *bytes = h->dev_bytes;
    return EDUS_OK;
}

int edus_kernel_launches(const edus_handle* h, unsigned long long* n) {
    if (!h || !n) return EDUS_ERR_ARG;
    *n = h->launches;
    return EDUS_OK;
}

}  // extern "C"
