/*
 * edus_gpu.h -- C ABI of the B200 density-matrix propagator.
 *
 * The library evaluates the right-hand side
 *     d rho_k / dt = E(t).grad_k rho_k - i [H0(k) + E(t).xi(k) + H_ee(k), rho_k]
 * and advances it with RK4 or Adams-Bashforth 4/5 on one GPU.  It replaces
 * the reference's DESolver<Operator<complex<double>>> + SourceTerm pair
 * (gcistaro/EDUS_2.0):
 *     src/DESolver/DESolver.hpp:26-82      DESolver call surface
 *     src/DESolver/DESolver.hpp:154-220    Propagate_RK / Propagate_AB
 *     src/Simulation/Functional_SourceTerm.hpp:10-56   SourceTerm
 *     src/Simulation/Simulation.cpp:163-174            how Simulation wires them
 *
 * Conventions shared with the reference:
 *   - complex numbers are interleaved (re, im) doubles;
 *   - a k-space operator is row-major [k][n][m], k = i2 + N2*(i1 + N1*i0)
 *     (src/MeshGrid/MeshGrid.cpp:117-139, BlockMatrix.hpp:48), exactly the
 *     memory of BlockMatrix<complex<double>>::Values;
 *   - an R-space operator uses the same index with the FFT output index of the
 *     k->R transform; R is Gamma-centred ([-N/2, N/2) per axis,
 *     MeshGrid.cpp:458-486);
 *   - all quantities are in Hartree atomic units.
 *
 * Errors: every entry point returns an int status (EDUS_OK = 0).  No C++
 * exception crosses this boundary.  edus_last_error() gives a message.
 * A handle is not thread-safe; distinct handles may be used from distinct
 * threads.  Work is queued on the handle's own CUDA stream and is complete
 * when a call that returns host data (edus_get_state, edus_rhs,
 * edus_observables) or edus_synchronize returns.
 */
#ifndef EDUS_GPU_H
#define EDUS_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define EDUS_OK 0
#define EDUS_ERR_ARG 1         /* invalid argument or call order */
#define EDUS_ERR_CUDA 2        /* CUDA runtime error (message has details) */
#define EDUS_ERR_TIMEOUT 3     /* a bounded device wait ran out */
#define EDUS_ERR_DIVERGED 4    /* non-finite density matrix detected */
#define EDUS_ERR_UNSUPPORTED 5 /* size or option this build does not handle */
#define EDUS_ERR_NOMEM 6       /* device allocation failed */

/* SolverType, src/Constants.hpp:27 (AB = 0, RK = 1) */
#define EDUS_SOLVER_AB 0
#define EDUS_SOLVER_RK 1

/* Forms of the right-hand side.
 *   FP64   the drop-in form: every band pair, FP64 throughout, no assumption
 *          on the symmetry of rho or H (as the reference).
 *   HERM64 packed-Hermitian form: only band pairs n <= m are stored and
 *          transformed, and the state is split rho = rho_ref + delta around
 *          the first state set; all arithmetic FP64.  It propagates the
 *          Hermitian part of the reference's generator.  The two are equal
 *          on odd grids.  On an even axis the Gamma-centred index N/2 has
 *          coordinate -N/2 for both R and -R, so the reference's gradient
 *          i (R.E) rho(R) and its W_nm(R) there are not Hermitian-preserving.
 *          Their Hermitian parts use coordinate 0 on that index and
 *          (W_nm(R) + W_mn(-R)) / 2.  The difference grows with |rho(R)| on
 *          the N/2 planes; the upload refuses a W that is asymmetric
 *          anywhere else.  Diagonal f_nn are kept real.
 *   MIXED  HERM64 with the per-step intermediates (gradient and self-energy
 *          planes, the model planes, the RK stage input) stored and
 *          transformed in FP32; the state delta, the RK accumulator, the AB
 *          history and the constant terms of the split stay FP64, and the
 *          band-matrix products run in FP64.
 * HERM64 and MIXED need nbands <= 32. */
#define EDUS_PREC_FP64 0
#define EDUS_PREC_HERM64 1
#define EDUS_PREC_MIXED 2
/*   SPLIT32 the full generator of FP64 (every band pair, the reference's own
 *          gradient and self-energy on every grid) with the state split as
 *          rho = rho_ref + delta.  The terms of rho_ref (grad rho_ref,
 *          H0 + Hee(rho_ref), rho_ref,nn(R=0)) are FP64, computed when the
 *          anchor rho_ref is moved to the current state: at the first step,
 *          after edus_set_state and every edus_set_anchor_interval steps
 *          (default 32).  Only delta goes through the plane transforms, in
 *          FP32, so their rounding scales with |delta|.  The commutator, the
 *          stage updates and the state are FP64. */
#define EDUS_PREC_SPLIT32 3
/*   HPLANES the FP64 form's state, commutators and stage updates, with the
 *          k<->R transforms of the band pairs n <= m only: the gradient and
 *          Hamiltonian planes of (m, n) are written as the conjugates of those
 *          of (n, m), as they are for Hermitian rho and H.  On odd grids this
 *          is the reference's generator (to rounding), with 48% fewer
 *          transforms at 22 bands; on even grids it is the generator's
 *          Hermitian part, as for HERM64 (coordinate 0 on the N/2 index, W
 *          symmetrised; the upload refuses a W that is asymmetric elsewhere).
 *          2-D grids of at most 7040 k points, length gauge, R-space
 *          gradient; edus_rhs returns the Hermitian part of f for an input
 *          that is not Hermitian. */
#define EDUS_PREC_HPLANES 4

/* Laser envelopes.  SIN2 is the reference's pulse (src/Laser/Laser.cpp:96-134):
 *   E(t) = sqrt(I) sin^2(pi (t-t0)/(cycles*T)) sin(w (t-t0) + phase) pol,
 *   zero for t-t0 <= 1e-7 or t-t0 > cycles*T.
 * GAUSS is an extension (no reference counterpart):
 *   E(t) = sqrt(I) exp(-2 ln2 (t-t0)^2 / fwhm^2) cos(w (t-t0) + phase) pol,
 *   fwhm being the full width at half maximum of the intensity. */
#define EDUS_ENVELOPE_SIN2 0
#define EDUS_ENVELOPE_GAUSS 1

typedef struct edus_handle edus_handle;

typedef struct {
    int grid[3];     /* N0, N1, N2 of the k grid (= the R grid) */
    int nbands;      /* nb: rows/cols of each block */
    int solver;      /* EDUS_SOLVER_RK or EDUS_SOLVER_AB */
    int order;       /* 4 for RK; 4 or 5 for AB */
    double dt;       /* DESolver::ResolutionTime, a.u. */
    int coulomb;     /* 1: add the HSEX self-energy (Coulomb::EffectiveHamiltonian) */
    int precision;   /* EDUS_PREC_FP64, _HERM64, _MIXED, _SPLIT32 or _HPLANES */
    int batch;       /* independent solves sharing one model (>= 1) */
    int device;      /* CUDA device ordinal */
} edus_desc;

typedef struct {
    double intensity;  /* a.u. (amplitude = sqrt(intensity)) */
    double omega;      /* a.u. */
    double pol[3];     /* Cartesian; normalised by the library */
    double cycles;     /* SIN2: duration in optical periods */
    double t0;         /* SIN2: start time; GAUSS: centre, a.u. */
    double phase;      /* carrier phase, rad */
    double fwhm;       /* GAUSS: intensity FWHM, a.u. */
    int envelope;      /* EDUS_ENVELOPE_* */
} edus_laser;

/* Create a handle and allocate every device buffer it will use.
 * Replaces DESolver::initialize + Operator::initialize_fft
 * (src/DESolver/DESolver.cpp:11-33, src/Operator/Operator.hpp:192-252). */
int edus_create(const edus_desc* desc, edus_handle** out);

/* Release the handle and its device memory. */
int edus_destroy(edus_handle* h);

/* Message of the last failure on this handle (or of the last failed
 * edus_create when h is NULL).  Never NULL. */
const char* edus_last_error(const edus_handle* h);

/* Upload the model (host buffers, caller-owned, copied during the call).
 *   H0_k   [Nk][nb][nb]    H0(k), Simulation::H0_ (Simulation.cpp:99-118)
 *   xi_k   [3][Nk][nb][nb] r_d(k), the Wannier position operator made
 *                          Hermitian (Simulation.cpp:93-97)
 *   lattice[9]             A, row-major, lattice vectors in the COLUMNS,
 *                          bohr (src/Model/Model.hpp:41-44)
 *   W_R    [Nk][nb][nb]    screened potential on the R grid
 *                          (ModelCoulomb::ScreenedPotential_); NULL if coulomb=0
 *   rho0_R [Nk][nb][nb]    ground-state density in R (Coulomb::DM0_); NULL if coulomb=0
 *   hartree[nb][nb]        Coulomb::Hartree (Coulomb.cpp:41-58); NULL if coulomb=0
 * The gradient term uses R.E with R = A R_crys, R_crys Gamma-centred
 * (kGradient_definitions.hpp:35-40). */
int edus_upload_model(edus_handle* h, const double* H0_k, const double* xi_k,
                      const double* lattice, const double* W_R, const double* rho0_R,
                      const double* hartree);

/* A model of its own for solve b (batches of solves whose models differ, such
 * as sweeps over seeded models of one grid and band count): H0_k and xi_k as in
 * edus_upload_model; the lattice stays the handle's.  Solves without a call
 * keep the model of edus_upload_model, which must come first.  FP64 form
 * without HSEX.  No reference counterpart. */
int edus_upload_model_solve(edus_handle* h, int b, const double* H0_k, const double* xi_k);

/* Lasers of solve `b` (0 <= b < batch).  Replaces SetOfLaser
 * (src/Laser/Laser.hpp:128-170).  n may be 0 (no field). */
int edus_set_lasers(edus_handle* h, int b, int n, const edus_laser* lasers);

/* Density matrix of solve b in k, [Nk][nb][nb] (DESolver::get_Function). */
int edus_set_state(edus_handle* h, int b, const double* rho_k);
int edus_get_state(edus_handle* h, int b, double* rho_k);

/* DESolver::CurrentTime.  Like the reference, it starts at 0 whatever the
 * initial time (DESolver.hpp:36, set_InitialTime does not move it). */
int edus_set_time(edus_handle* h, double t);
int edus_get_time(const edus_handle* h, double* t);

/* One SourceTerm evaluation of solve 0 at time t (the field is taken from the
 * lasers of solve 0): out_k = f(t, in_k).  Host buffers [Nk][nb][nb].
 * Replaces Functional_SourceTerm.hpp:10-56. */
int edus_rhs(edus_handle* h, double t, const double* in_k, double* out_k);

/* Advance every solve by n steps (DESolver::Propagate(n), DESolver.hpp:238-242).
 * Asynchronous: returns once the work is queued.  Exception: an RK4 handle in
 * the FP64 form whose state (all solves) is at most 16 MB, profiling off, with
 * n >= 512, steps as edus_sweep_step of that one handle with use_graph 1 (the
 * same launches, 32 steps per CUDA graph replay, for small problems whose
 * steps are dominated by launch overhead) and returns once they are done. */
int edus_step(edus_handle* h, int n);

/* Advance n handles (one device, FP64 form) by `steps` steps together.
 *   use_graph = 0: every handle's kernels run on its own stream, forked from
 *                  and joined into one sweep stream, so solves of different
 *                  grids and band counts share the GPU;
 *   use_graph = 1: the same, and with RK4 handles each chunk of 32 steps of all
 *                  handles is captured once into one CUDA graph and replayed
 *                  (the field tables are refreshed between replays);
 *   use_graph = 2: one persistent launch per RK stage for the plane transforms
 *                  of every solve of every handle (one per shared-memory class:
 *                  planes up to 110 KB, larger planes) and one for all their
 *                  commutators and stage updates; work items (handle, solve,
 *                  plane or k tile) are taken largest first from a counter;
 *                  chunks captured into a CUDA graph.  RK4, independent
 *                  particles, R-space gradient, length gauge (else
 *                  EDUS_ERR_UNSUPPORTED).  A solve's result equals stepping
 *                  its handle alone.
 * Synchronous.  No reference counterpart. */
int edus_sweep_step(edus_handle* const* hs, int n, int steps, int use_graph);

/* Time the launch variants on the handle's own data and keep the fastest:
 * the plane kernel's thread count, and (outside the TMA path) the CUDA-core
 * against the tensor-core commutator.  Either output may be NULL.  Leaves the
 * state unchanged.  No reference counterpart. */
int edus_autotune(edus_handle* h, int* plane_threads, int* comm_tensor);

/* rho(R) of solve b at nsel lattice vectors: out[s][n][m] = rho_nm(R_s) with
 * rho(R) = FFT_{-1}(rho_k) / Nk (Operator::go_to_R, Operator.hpp:566-586) and
 * R_index[s] the natural R index (j0 N1 + j1) N2 + j2.  Synchronous.  No
 * reference counterpart (inputs and training data of the learned self-energy). */
int edus_state_rspace(edus_handle* h, int b, int nsel, const int* R_index, double* out);

/* Replace the Fock term -W (rho(R) - rho0(R)) of every following right-hand
 * side by given values on nsel lattice vectors (values[s][n][m] complex, zero
 * elsewhere); the Hartree term stays exact.  nsel = 0 restores the exact term.
 * FP64 form with HSEX whose plane fits two CTAs per SM.  No reference
 * counterpart (the learned self-energy feeds the propagation through it). */
int edus_set_fock_override(edus_handle* h, int nsel, const int* R_index, const double* values);

/* Learned self-energy network: a multilayer perceptron n_in -> 3 hidden layers
 * of n_hidden (GELU) -> n_out, BF16 weights with FP32 master copies and FP32
 * accumulation, trained on the GPU (mean squared error, Adam).  Batches are
 * row-major [batch][features] FP32 DEVICE buffers.  Parameters are flattened
 * as W0 b0 W1 b1 W2 b2 W3 b3, W_l row-major [in][out] (host FP32 buffers).
 * No reference counterpart. */
typedef struct edus_mlp edus_mlp;
int edus_mlp_create(int n_in, int n_hidden, int n_out, unsigned long long seed, int device, edus_mlp** out);
int edus_mlp_destroy(edus_mlp* m);
const char* edus_mlp_last_error(const edus_mlp* m);
long long edus_mlp_param_count(const edus_mlp* m);
int edus_mlp_set_params(edus_mlp* m, const float* host);
int edus_mlp_get_params(edus_mlp* m, float* host);
int edus_mlp_forward(edus_mlp* m, int batch, const float* x, float* y);
/* loss and the gradient of every parameter (host buffers; either may be NULL) */
int edus_mlp_gradients(edus_mlp* m, int batch, const float* x, const float* target, float* grads_host,
                       float* loss_host);
/* one Adam step on the batch; loss_host (may be NULL) receives the loss before the step */
int edus_mlp_train_step(edus_mlp* m, int batch, const float* x, const float* target, float lr, float* loss_host);

/* Split-precision form: steps between two moves of the anchor rho_ref to the
 * current state (>= 1; default 32).  No reference counterpart. */
int edus_set_anchor_interval(edus_handle* h, int steps);

/* Wait for queued work; reports device-side errors. */
int edus_synchronize(edus_handle* h);

/* gradient_space "k" (kGradient_definitions.hpp:18-30): E.grad_k rho(k) =
 * sum_i w[i] (b_i.E) rho(k + b_i) over n vectors b_i (Cartesian, 1/bohr,
 * b[3i..3i+2]) whose grid offsets are shift[3i..3i+2] (FFT indices, folded);
 * the shells and weights of kGradient.cpp:26-211 are the caller's (one-off
 * set-up).  Replaces the R-space gradient: without HSEX no plane transform
 * runs.  n = 0 restores the R-space gradient.  FP64 form. */
int edus_set_kgradient(edus_handle* h, int n, const int* shift, const double* b, const double* w);

/* Peierls gauge ("peierls": true; Functional_SourceTerm.hpp:15-50,
 * Simulation.cpp:876-899): no gradient term, and the Hamiltonian of a stage at
 * time t is H(R) = (H0(R) + E.xi(R) + Hee[rho(R) e^{-iA.R}](R)) e^{+iA.R},
 * A(t) the vector potential of each solve's lasers integrated as
 * Laser::VectorPotential does (Laser.cpp:136-151: one Simpson step from the
 * previous requested time, from A = 0 at t = 0; every stage time and
 * edus_vector_potential call is a request).  on = 1 resets the integrators;
 * on = 0 returns to the length gauge.  FP64 form, one model for all solves,
 * H0(R) and xi(R) on at most 4096 lattice vectors (tight-binding models). */
int edus_set_peierls(edus_handle* h, int on);

/* Vector potential of solve b advanced to time t (a request, as above), a.u.:
 * Laser::VectorPotential summed over the solve's lasers (SetOfLaser,
 * Laser.hpp:152-158; the reference's accumulator is shared by all lasers, so
 * the two agree for one laser). */
int edus_vector_potential(edus_handle* h, int b, double t, double* A);

/* Observables of Simulation::do_onestep (Simulation.cpp:420-429).  Upload once
 * the eigenvectors U_k [Nk][nb][nb] (columns, SettingUp_EigenSystem) and/or the
 * velocity operator vel_k [3][Nk][nb][nb] (Simulation.cpp:523-576); either may
 * be NULL. */
int edus_upload_observables(edus_handle* h, const double* U_k, const double* vel_k);

/* Observables of solve b's current state (synchronous; any output may be NULL):
 *   pop_bloch[nb]   (1/Nk) sum_k Re (U^dagger rho U)_nn, as 1 - P_n for the
 *                   `filled` lowest bands (Print_Population, bloch)
 *   pop_wannier[nb] (1/Nk) sum_k Re rho_nn (Print_Population, wannier)
 *   vel[6]          re, im of (1/Nk) sum_k tr(v_d rho), d = x, y, z (Print_Velocity) */
int edus_observables(edus_handle* h, int b, int filled, double* pop_bloch, double* pop_wannier, double* vel);

/* E(t) of solve b's lasers, the same field the kernels use (SetOfLaser::operator(),
 * Laser.hpp:143-150). */
int edus_efield(edus_handle* h, int b, double t, double* E);

/* Observables of solve b for the current state, as Simulation::do_onestep
 * prints them (Simulation.cpp:439-470, 583-622):
 *   pop_wannier[nb] = (1/Nk) sum_k Re rho_nn(k).
 * Requires no extra model data. */
int edus_population_wannier(edus_handle* h, int b, double* pop_wannier);

/* The CUDA stream (cudaStream_t) every kernel of this handle runs on. */
int edus_get_stream(const edus_handle* h, void** stream);

/* Poll limit of the plane kernel's wait for its bulk-copied plane (planes of
 * 4096 points and more), in mbarrier try-waits (each of which may itself
 * block for a while); polls < 0 restores the default (2^22, far above any
 * copy).  A wait that runs out sets the handle's status word (the CTA still
 * lets its copies land before it ends), and the next synchronising call
 * returns EDUS_ERR_TIMEOUT and clears the word.  For exercising the failure
 * path: a limit of 0 gives up without waiting.  No reference counterpart. */
int edus_set_wait_limit(edus_handle* h, int polls);

/* Per-kernel timing with CUDA events on the handle's stream (off by default).
 * kind 0 = plane kernel (k<->R transforms + gradient + HSEX), 1 = commutator
 * + stage kernel.  Totals accumulate from the call that enabled profiling;
 * edus_get_profile synchronises the stream. */
int edus_set_profiling(edus_handle* h, int on);
int edus_get_profile(edus_handle* h, int kind, double* total_ms, unsigned long long* launches);

/* ------------------------------------------------------------------------
 * No-allocation variant of edus_rhs.  No counterpart in the reference.
 *
 * For callers that cannot let a library allocate device memory: their GPU
 * memory belongs to another allocator (a framework's caching allocator that
 * reserves the device up front, a fixed pool sized at start-up), or they run
 * a time-critical loop where cudaMalloc's implicit device-wide
 * synchronisation is unacceptable.  The caller passes device buffers for all
 * inputs and the output; the intermediates live in one array built into the
 * library's CUDA module, EDUS_NOALLOC_SCRATCH_BYTES long, which every GPU that
 * loads the library holds until the process exits.  Nothing in this call
 * allocates (no cudaMalloc / cudaFree, no allocating library routine).
 *
 *   grid, nbands, coulomb   as in edus_desc
 *   lattice[9], efield[3]   HOST arrays: A (columns = lattice vectors, bohr)
 *                           and the field E(t) of this evaluation (a.u.)
 *   H0_k, xi_k, W_R, rho0_R, hartree
 *                           DEVICE arrays, layouts of edus_upload_model
 *                           (W_R, rho0_R, hartree may be NULL if coulomb = 0)
 *   in_k, out_k             DEVICE arrays [Nk][nb][nb]: out = f(in)
 *   stream                  cudaStream_t the work is queued on (NULL = legacy)
 *   errbuf, errlen          optional buffer for a message on failure
 * Returns once the work is queued.  The intermediates must fit the array
 * (about 6.5 * Nk * nb^2 * 16 bytes with coulomb, 4 * ... without); larger
 * problems get EDUS_ERR_UNSUPPORTED.  The first call on a device looks up the
 * array's address, raises the kernels' shared-memory limit and copies the k
 * grid's FFT tables from host memory into the array, waiting for that copy:
 * make it before any stream capture on that device.  A call whose grid
 * differs from the previous call's on the device copies its tables the same
 * way; other calls only queue kernels (the field goes as a kernel argument).
 * W_R must be real, as edus_upload_model requires: the check runs on the
 * device, so a W_R with a non-zero imaginary part is refused by an out_k
 * filled with NaN rather than by a return code.  All calls share the array,
 * and each call overwrites what the last one left there: calls that overlap
 * on the GPU (several streams or host threads at once) race and must be
 * serialised by the caller. */
#define EDUS_NOALLOC_SCRATCH_BYTES (64u * 1024u * 1024u)
int edus_rhs_noalloc(const int grid[3], int nbands, int coulomb, const double lattice[9],
                     const double efield[3], const double* H0_k, const double* xi_k,
                     const double* W_R, const double* rho0_R, const double* hartree,
                     const double* in_k, double* out_k, void* stream, char* errbuf, int errlen);

/* Size in bytes of the device memory the handle holds. */
int edus_device_bytes(const edus_handle* h, unsigned long long* bytes);

/* Number of kernel launches this handle has queued since creation. */
int edus_kernel_launches(const edus_handle* h, unsigned long long* n);

#ifdef __cplusplus
}
#endif

#endif /* EDUS_GPU_H */
