// edus_gpu.hpp -- header-only C++ facade over the C ABI of edus_gpu.h with
// the reference's DESolver call surface (src/DESolver/DESolver.hpp:26-82), so
// that Simulation-style host code can hold a GpuDESolver where it held a
// DESolver<Operator<std::complex<double>>>.  Errors become exceptions on this
// (C++) side of the boundary only.
#ifndef EDUS_GPU_HPP
#define EDUS_GPU_HPP

#include <complex>
#include <stdexcept>
#include <string>
#include <vector>

#include "edus_gpu.h"

namespace edus_gpu {

class GpuDESolver {
   public:
    GpuDESolver() = default;
    GpuDESolver(const GpuDESolver&) = delete;
    GpuDESolver& operator=(const GpuDESolver&) = delete;
    ~GpuDESolver() { edus_destroy(h_); }

    // DESolver::initialize(Function, InitialCondition, SourceTerm, type, order):
    // the source term is fixed (the EDUS right-hand side); the model replaces
    // the closure's captured state and rho0_k is the evaluated initial condition.
    void initialize(const int grid[3], int nbands, int solver, int order, double dt, bool coulomb,
                    const std::complex<double>* H0_k, const std::complex<double>* xi_k, const double lattice[9],
                    const std::complex<double>* W_R, const std::complex<double>* rho0_R,
                    const std::complex<double>* hartree, const std::complex<double>* rho0_k, int batch = 1,
                    int device = 0) {
        edus_desc d{};
        for (int i = 0; i < 3; ++i) d.grid[i] = grid[i];
        d.nbands = nbands;
        d.solver = solver;
        d.order = order;
        d.dt = dt;
        d.coulomb = coulomb ? 1 : 0;
        d.precision = EDUS_PREC_FP64;
        d.batch = batch;
        d.device = device;
        edus_destroy(h_);
        h_ = nullptr;
        check(edus_create(&d, &h_), nullptr);
        nk_ = (size_t)grid[0] * grid[1] * grid[2];
        nb_ = nbands;
        dt_cache_ = dt;
        check(edus_upload_model(h_, dp(H0_k), dp(xi_k), lattice, dp(W_R), dp(rho0_R), dp(hartree)), h_);
        for (int b = 0; b < batch; ++b) check(edus_set_state(h_, b, dp(rho0_k)), h_);
    }

    void set_lasers(const std::vector<edus_laser>& lasers, int b = 0) {
        check(edus_set_lasers(h_, b, (int)lasers.size(), lasers.data()), h_);
    }

    // DESolver::set_InitialTime does not move CurrentTime in the reference
    void set_InitialTime(double t) { initial_time_ = t; }
    void set_ResolutionTime(double) {
        throw std::runtime_error("the resolution time is fixed at initialize()");
    }
    double get_CurrentTime() const {
        double t = 0;
        check(edus_get_time(h_, &t), h_);
        return t;
    }
    double get_ResolutionTime() const { return dt_of(); }

    void Propagate() { check(edus_step(h_, 1), h_); }
    void Propagate(const int& nstep) { check(edus_step(h_, nstep), h_); }

    // DESolver::get_Function: the density matrix of solve b in [k][n][m]
    std::vector<std::complex<double>> get_Function(int b = 0) const {
        std::vector<std::complex<double>> out(nk_ * nb_ * nb_);
        check(edus_get_state(h_, b, reinterpret_cast<double*>(out.data())), h_);
        return out;
    }

    // SourceTerm(Output, t, Input) for solve 0
    void SourceTerm(std::complex<double>* out_k, double t, const std::complex<double>* in_k) {
        check(edus_rhs(h_, t, dp(in_k), reinterpret_cast<double*>(out_k)), h_);
    }

    edus_handle* handle() const { return h_; }

   private:
    static const double* dp(const std::complex<double>* p) { return reinterpret_cast<const double*>(p); }
    static void check(int rc, const edus_handle* h) {
        if (rc != EDUS_OK) throw std::runtime_error(std::string("edus_gpu: ") + edus_last_error(h));
    }
    double dt_of() const { return dt_cache_; }

    edus_handle* h_ = nullptr;
    size_t nk_ = 0;
    int nb_ = 0;
    double initial_time_ = 0.0;
    double dt_cache_ = 0.0;
};

}  // namespace edus_gpu

#endif
