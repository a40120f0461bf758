// TEST INFRASTRUCTURE ONLY: the CPU oracle.
//
// This file restates, in plain FP64 C++, the reference EDUS propagation path
// (gcistaro/EDUS_2.0) so the GPU product can be checked against it.  Only the
// tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load the
// shared library built from it; the product never does.
//
// Parity pins (see tests/test_oracle_golden.py):
//   * ci-test/outputs/hBN/{Population,Velocity,Laser,Time}.txt (hBN IPA run),
//   * ci-test/Reference/Struve.txt (Struve H0 table),
//   * the analytic known-answer tests of ci-test/test_DEsolver*.cpp,
//     test_Gradient_R.cpp and test_fft_mpi.cpp restated in Python.
//
// Every function names the reference lines it follows.  Paths are relative
// to the reference project root.
#include <complex>
#include <vector>
#include <array>
#include <string>
#include <fstream>
#include <sstream>
#include <cmath>
#include <cstring>
#include <cstdio>
#include <stdexcept>
#include <algorithm>
#include <memory>
#include "oracle_fft.hpp"
#include "oracle_linalg.hpp"

namespace oracle {

using cd = std::complex<double>;
static const cd im(0., 1.);
// src/Constants.hpp:8-22
static constexpr double pi = 3.14159265358979323846;
static constexpr double Bohr_value = 5.2917721090380 * 1.e-11;
static constexpr double ElectronVolt_value = 1.602176634 * 1.e-19;
static constexpr double Rydberg_value = 2.1798723611035 * 1.e-18;
static constexpr double AtomicUnitOfTime = 2.4188843265857 * 1.e-17;
static constexpr double threshold = 1.e-08;

// src/ConvertUnits.hpp:68-73 : value / Out * In
static double convert(double x, double in_unit, double out_unit) { return x / out_unit * in_unit; }
static const double Angstrom = 1.e-10, AuLength = Bohr_value;
static const double ElectronVoltU = ElectronVolt_value, AuEnergy = 2. * Rydberg_value;

// ---------------------------------------------------------------------------
// Struve H0: src/ModelCoulomb/ModelCoulomb.cpp:7-44 (series for x <= 20,
// asymptotic expansion with the polynomial P0/Q0 fit above).
double struve0(double X) {
    double SH0, A0, BY0, P0, Q0, R, S, T, T2, TA0;
    int K, KM;
    S = 1.0;
    R = 1.0;
    if (X <= 20.0) {
        A0 = 2.0 * X / pi;
        for (K = 1; K < 61; K++) {
            R = -R * X / (2.0 * K + 1.0) * X / (2.0 * K + 1.0);
            S = S + R;
            if (std::fabs(R) < std::fabs(S) * 1.0e-12) break;
        }
        SH0 = A0 * S;
    } else {
        KM = int(0.5 * (X + 1.0));
        if (X >= 50.0) KM = 25;
        for (K = 1; K <= KM; K++) {
            R = -R * std::pow((2.0 * K - 1.0) / X, 2);
            S = S + R;
            if (std::fabs(R) < std::fabs(S) * 1.0e-12) break;
        }
        T = 4.0 / X;
        T2 = T * T;
        P0 = ((((-.37043e-5 * T2 + .173565e-4) * T2 - .487613e-4) * T2 + .17343e-3) * T2 - 0.1753062e-2) * T2 + .3989422793;
        Q0 = T * (((((.32312e-5 * T2 - 0.142078e-4) * T2 + 0.342468e-4) * T2 - 0.869791e-4) * T2 + 0.4564324e-3) * T2 - 0.0124669441);
        TA0 = X - 0.25 * pi;
        BY0 = 2.0 / std::sqrt(X) * (P0 * std::sin(TA0) + Q0 * std::cos(TA0));
        SH0 = 2.0 / (pi * X) * S + BY0;
    }
    return SH0;
}

// ---------------------------------------------------------------------------
// Wannier90 _tb.dat reader: src/Wannier/ReadWannier.cpp:5-153.
// Lines are split on white space (src/StreamFile.cpp); element "m n re im"
// is stored at row m-1, column n-1 (ReadWannier.cpp:23-27).
struct TbModel {
    double UC[3][3];  // rows = lattice vectors, Angstrom
    int nb = 0, nR = 0;
    std::vector<int> R;      // nR*3
    std::vector<cd> H;       // nR*nb*nb, eV
    std::vector<cd> r[3];    // nR*nb*nb, Angstrom
};

static std::vector<std::vector<std::string>> read_tokens(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open " + path);
    std::vector<std::vector<std::string>> out;
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream ss(line);
        std::vector<std::string> tok;
        std::string t;
        while (ss >> t) tok.push_back(t);
        out.push_back(tok);
    }
    return out;
}

TbModel read_tb(const std::string& path) {
    auto lines = read_tokens(path);
    TbModel m;
    size_t li = 1;
    for (int i = 0; i < 3; ++i, ++li) {
        if (lines.at(li).size() != 3) throw std::runtime_error("bad unit cell line");
        for (int j = 0; j < 3; ++j) m.UC[i][j] = std::atof(lines[li][j].c_str());
    }
    m.nb = std::atoi(lines.at(4).at(0).c_str());
    m.nR = std::atoi(lines.at(5).at(0).c_str());
    li = 6;
    int ndeg = 0;
    while (li < lines.size() && !lines[li].empty()) { ndeg += (int)lines[li].size(); ++li; }
    if (ndeg != m.nR) throw std::runtime_error("degeneracy count mismatch");
    while (li < lines.size() && lines[li].empty()) ++li;
    const int nb = m.nb;
    m.R.assign(3 * m.nR, 0);
    m.H.assign((size_t)m.nR * nb * nb, 0.);
    for (int d = 0; d < 3; ++d) m.r[d].assign((size_t)m.nR * nb * nb, 0.);
    // Hamiltonian blocks (ReadWannier.cpp:81-93): R line then lines of 4 tokens
    int idx = 0;
    while (li + 1 < lines.size() && lines[li + 1].size() == 4) {
        for (int d = 0; d < 3; ++d) m.R[3 * idx + d] = (int)std::lround(std::atof(lines[li][d].c_str()));
        ++li;
        while (li < lines.size() && !lines[li].empty()) {
            auto& t = lines[li];
            if (t.size() != 4) throw std::runtime_error("bad H element line");
            int a = std::atoi(t[0].c_str()) - 1, b = std::atoi(t[1].c_str()) - 1;
            m.H[((size_t)idx * nb + a) * nb + b] = cd(std::atof(t[2].c_str()), std::atof(t[3].c_str()));
            ++li;
        }
        ++li;  // blank line
        ++idx;
    }
    if (idx != m.nR) throw std::runtime_error("H block count mismatch");
    // position operator blocks (ReadWannier.cpp:95-108): 8 tokens per line
    idx = 0;
    while (li + 1 < lines.size() && lines[li + 1].size() == 8) {
        ++li;
        while (li < lines.size() && lines[li].size() == 8) {
            auto& t = lines[li];
            int a = std::atoi(t[0].c_str()) - 1, b = std::atoi(t[1].c_str()) - 1;
            for (int d = 0; d < 3; ++d)
                m.r[d][((size_t)idx * nb + a) * nb + b] =
                    cd(std::atof(t[2 + 2 * d].c_str()), std::atof(t[3 + 2 * d].c_str()));
            ++li;
        }
        ++li;
        ++idx;
    }
    if (idx != m.nR) throw std::runtime_error("r block count mismatch");
    return m;
}

// ---------------------------------------------------------------------------
// Lasers: src/Laser/Laser.cpp:35-38 (carrier), :96-104 (sin^2 envelope),
// :131-134 (E = A env carrier pol), :191-200 (amplitude, polarisation).
// envelope 1 (Gaussian, cos carrier) is an extension that the reference lacks;
// it is the pulse shape of the synthetic benchmark workloads.
struct Laser {
    double amplitude = 0, omega = 0, t0 = 0, phase = 0, duration = 0, fwhm = 0;
    double pol[3] = {0, 0, 0};
    int envelope = 0;
    void field(double t, double E[3]) const {
        double a;
        if (envelope == 0) {
            double tt = t - t0;
            double env = (tt <= 1.e-07 || tt > duration) ? 0. : std::pow(std::sin(pi * tt / duration), 2.);
            a = amplitude * env * std::sin(omega * (t - t0) + phase);
        } else {
            double tt = t - t0;
            double env = std::exp(-2.0 * std::log(2.0) * tt * tt / (fwhm * fwhm));
            a = amplitude * env * std::cos(omega * tt + phase);
        }
        for (int d = 0; d < 3; ++d) E[d] = a * pol[d];
    }
};

}  // namespace oracle

using namespace oracle;

extern "C" {

// Laser description passed from the harness (atomic units).  envelope 0 =
// the reference's sin^2 pulse (t0 = start, cycles = duration in periods);
// envelope 1 = Gaussian field envelope exp(-2 ln2 (t-t0)^2 / fwhm^2) (fwhm of
// the intensity) with cos carrier centred at t0.
typedef struct {
    double intensity_au, omega_au, pol[3], cycles, t0_au, phase, fwhm_au;
    int envelope;
} oracle_laser;

typedef struct {
    const char* tb_path;  // full path of the _tb.dat file
    int grid[3];
    int filledbands;
    double dt_au;
    int solver;  // 0 = AB, 1 = RK (src/Constants.hpp:27)
    int order;
    int coulomb;
    double epsilon;
    double r0_au[3];
    int nr0;               // number of r0 components given (1..3)
    int coulomb_fix_centres;  // 0 = reference behaviour (cumulative r), 1 = r = c_n - R - c_m
    // 0 = reference behaviour.  1 = the Hermitian part of the generator on an
    // even grid, where the Gamma-centred index N/2 sits at -N/2 for both R and
    // -R: the gradient uses coordinate 0 there and W_nm(R) becomes
    // (W_nm(R) + W_mn(-R)) / 2.  This is what the packed-Hermitian GPU forms
    // propagate; it differs from the reference only on the N/2 planes.
    int hermitian_nyquist;
    int gradient_k;  // 1: gradient_space "k", the finite-difference gradient of kGradient.cpp
    int peierls;     // 1: "peierls": true, propagation in the Peierls gauge
    int nlasers;
    oracle_laser lasers[8];
} oracle_cfg;

}  // extern "C"

namespace oracle {

struct Sim;
void build_kgradient(Sim& s);
struct Sim {
    int N[3], Nk, nb, P;
    double A[3][3];  // columns = lattice vectors (bohr), src/Model/Model.hpp:41-44
    Fft3dMany fft;
    std::vector<cd> H0k, rk[3], H0R, rR[3];
    std::vector<double> Rcart;   // [Nk][3] Gamma-centred Cartesian R of FFT index
    std::vector<double> Rcrys;   // [Nk][3]
    std::vector<double> Rgrad;   // [Nk][3] Cartesian R used by the k-gradient
    // gradient_space "k": stencil k -> k + b over the shells of kGradient.cpp
    std::vector<std::array<int, 3>> gshift;     // FFT index of b per axis
    std::vector<std::array<double, 3>> gvec;    // b, Cartesian (1/bohr)
    std::vector<double> gw;                     // weight of b's shell
    std::vector<double> eval;    // [Nk][nb]
    std::vector<cd> U;           // [Nk][nb][nb]
    std::vector<cd> vel[3];      // velocity operator in k
    // coulomb
    bool coulomb = false;
    std::vector<cd> W, V, DM0R;
    std::vector<cd> Hartree;
    int origin = 0;
    double r0[3] = {0, 0, 0}, r0_avg = 0, epsilon = 1;
    double min_dist[3] = {100, 0, 0};
    double min_dist_norm = 100;
    std::vector<Laser> lasers;
    // Peierls gauge: the vector potential integrator of Laser::VectorPotential
    bool peierls = false;
    double Avec[3] = {0., 0., 0.};
    double Aprev = 0.;
    std::vector<cd> auxR;
    // solver state
    int solver = 1, order = 4;
    double dt = 0, t = 0;
    std::vector<cd> rho;
    std::array<std::vector<cd>, 5> aux;
    int index[5] = {0, 1, 2, 3, 4};
    double beta[5] = {0, 0, 0, 0, 0};
    int dims = 0;
    // scratch
    std::vector<cd> inR, outR, HR, Hk;

    size_t S() const { return (size_t)Nk * nb * nb; }

    void efield(double time, double E[3]) const {
        // SetOfLaser::operator() sums the lasers (src/Laser/Laser.hpp:143-150)
        E[0] = E[1] = E[2] = 0;
        for (auto& l : lasers) {
            double e[3];
            l.field(time, e);
            for (int d = 0; d < 3; ++d) E[d] += e[d];
        }
    }

    // Laser::VectorPotential (src/Laser/Laser.cpp:136-151): one Simpson step
    // from the previous request, from A = 0 at t = 0.  The reference keeps A
    // and the previous time in function statics shared by all lasers of
    // SetOfLaser::VectorPotential (Laser.hpp:152-158); with one laser that is
    // the integral of the total field, which is what this restates.
    void vector_potential(double time, double out[3]) {
        const double deltaT = time - Aprev;
        if (deltaT >= 1.e-07) {
            double E1[3], E2[3], E3[3];
            efield(Aprev, E1);
            efield(Aprev + deltaT / 2., E2);
            efield(time, E3);
            for (int d = 0; d < 3; ++d) Avec[d] -= deltaT / 6. * (E1[d] + 4. * E2[d] + E3[d]);
            Aprev = time;
        }
        for (int d = 0; d < 3; ++d) out[d] = Avec[d];
    }

    // Simulation::Apply_Peierls_phase (Simulation.cpp:876-899): O(R) *= exp(i sign A(t).R)
    void peierls_phase(cd* OR, double time, int sign) {
        double At[3];
        vector_potential(time, At);
#pragma omp parallel for schedule(static)
        for (int iR = 0; iR < Nk; ++iR) {
            const double* R = &Rcart[3 * (size_t)iR];
            const cd ph = std::exp(im * double(sign) * (At[0] * R[0] + At[1] * R[1] + At[2] * R[2]));
            for (int p = 0; p < P; ++p) OR[(size_t)iR * P + p] *= ph;
        }
    }

    double W_of(const double rc[3]) const {
        // ModelCoulomb::W, src/ModelCoulomb/ModelCoulomb.cpp:139-162
        double rr[3] = {rc[0] / r0[0], rc[1] / r0[1], rc[2] / r0[2]};
        double rn = std::sqrt(rr[0] * rr[0] + rr[1] * rr[1] + rr[2] * rr[2]);
        if (rn < threshold) return W_of(min_dist);
        return pi / (2. * r0_avg * epsilon) * (struve0(rn) - ::y0(rn));
    }
    double V_of(const double rc[3]) const {
        // ModelCoulomb::V, ModelCoulomb.cpp:168-176
        double rn = std::sqrt(rc[0] * rc[0] + rc[1] * rc[1] + rc[2] * rc[2]);
        if (rn < min_dist_norm) return V_of(min_dist);
        return 2. / rn;
    }
};

static void matmul(int n, const cd* a, const cd* b, cd* c, cd alpha, cd beta_) {
    // C = alpha A B + beta C (row major), the role of cblas_zgemm in
    // src/LinearAlgebra/gemm.hpp:20-29
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            cd s = 0.;
            for (int k = 0; k < n; ++k) s += a[i * n + k] * b[k * n + j];
            c[i * n + j] = alpha * s + beta_ * c[i * n + j];
        }
}

Sim* build(const oracle_cfg* cfg) {
    auto sim = std::make_unique<Sim>();
    Sim& s = *sim;
    TbModel m = read_tb(cfg->tb_path);
    s.nb = m.nb;
    s.P = m.nb * m.nb;
    for (int d = 0; d < 3; ++d) s.N[d] = cfg->grid[d];
    s.Nk = s.N[0] * s.N[1] * s.N[2];
    s.dims = (s.N[0] > 1) + (s.N[1] > 1) + (s.N[2] > 1);
    const int nb = s.nb, P = s.P, Nk = s.Nk;
    // lattice: UC^T converted to bohr (Model.hpp:41-44)
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) s.A[i][j] = convert(m.UC[j][i], Angstrom, AuLength);
    // model blocks to a.u. (Model.hpp:54-57)
    for (auto& h : m.H) h = cd(convert(h.real(), ElectronVoltU, AuEnergy), convert(h.imag(), ElectronVoltU, AuEnergy));
    for (int d = 0; d < 3; ++d)
        for (auto& x : m.r[d]) x = cd(convert(x.real(), Angstrom, AuLength), convert(x.imag(), Angstrom, AuLength));
    // Gamma-centred model R (MeshGrid.cpp:458-486).  Model R points must lie in
    // [-N/2, N/2) already; the reference's wrap uses an undefined grid size.
    for (int iR = 0; iR < m.nR; ++iR)
        for (int d = 0; d < 3; ++d) {
            double lo = -s.N[d] / 2., up = s.N[d] / 2.;
            double x = m.R[3 * iR + d];
            if ((x < lo && std::abs(x - lo) > threshold) || x > up || std::abs(x - up) < threshold)
                throw std::runtime_error("model R point outside the Gamma-centred k-grid range");
        }
    // H(k) = sum_R exp(+i 2 pi k.R) H(R), k = i/N (fftPair.cpp:110-142,
    // Simulation.cpp:93-97); r(k) made Hermitian (BlockMatrix_definitions.hpp:258-277)
    s.H0k.assign(s.S(), 0.);
    for (int d = 0; d < 3; ++d) s.rk[d].assign(s.S(), 0.);
    const cd im2pi = im * 2. * pi;
#pragma omp parallel for schedule(static)
    for (int ik = 0; ik < Nk; ++ik) {
        int i0 = ik / (s.N[1] * s.N[2]), i1 = (ik / s.N[2]) % s.N[1], i2 = ik % s.N[2];
        double kc[3] = {double(i0) / s.N[0], double(i1) / s.N[1], double(i2) / s.N[2]};
        for (int iR = 0; iR < m.nR; ++iR) {
            double dot = 0;
            for (int d = 0; d < 3; ++d) dot += kc[d] * m.R[3 * iR + d];
            cd ph = std::exp(1.0 * im2pi * dot);
            for (int p = 0; p < P; ++p) {
                s.H0k[(size_t)ik * P + p] += ph * m.H[(size_t)iR * P + p];
                for (int d = 0; d < 3; ++d) s.rk[d][(size_t)ik * P + p] += ph * m.r[d][(size_t)iR * P + p];
            }
        }
        for (int d = 0; d < 3; ++d) {
            cd* blk = &s.rk[d][(size_t)ik * P];
            for (int i = 0; i < nb; ++i)
                for (int j = i; j < nb; ++j) {
                    cd term = (blk[i * nb + j] + std::conj(blk[j * nb + i])) / 2.;
                    blk[i * nb + j] = term;
                    blk[j * nb + i] = std::conj(term);
                }
        }
    }
    s.fft = Fft3dMany(s.N, P);
    s.H0R.resize(s.S());
    s.fft.run(s.H0k.data(), s.H0R.data(), -1);  // Simulation.cpp:115-118
    for (int d = 0; d < 3; ++d) {
        s.rR[d].resize(s.S());
        s.fft.run(s.rk[d].data(), s.rR[d].data(), -1);
    }
    // Gamma-centred R of each FFT index, Cartesian = A R_crys (Coordinate.cpp:38-49)
    s.Rcart.resize(3 * (size_t)Nk);
    s.Rcrys.resize(3 * (size_t)Nk);
    for (int iR = 0; iR < Nk; ++iR) {
        int j[3] = {iR / (s.N[1] * s.N[2]), (iR / s.N[2]) % s.N[1], iR % s.N[2]};
        double c[3];
        for (int d = 0; d < 3; ++d) {
            double x = j[d], lo = -s.N[d] / 2., up = s.N[d] / 2.;
            while (x < lo && std::abs(x - lo) > threshold) x += s.N[d];
            while (x > up || std::abs(x - up) < threshold) x -= s.N[d];
            c[d] = x;
            s.Rcrys[3 * iR + d] = x;
        }
        for (int a = 0; a < 3; ++a) s.Rcart[3 * iR + a] = s.A[a][0] * c[0] + s.A[a][1] * c[1] + s.A[a][2] * c[2];
    }
    s.Rgrad = s.Rcart;
    s.peierls = cfg->peierls != 0;
    if (cfg->gradient_k) build_kgradient(s);
    if (cfg->hermitian_nyquist) {
        for (int iR = 0; iR < Nk; ++iR) {
            double c[3];
            for (int d = 0; d < 3; ++d) {
                c[d] = s.Rcrys[3 * iR + d];
                if (s.N[d] % 2 == 0 && c[d] == -s.N[d] / 2.) c[d] = 0.;
            }
            for (int a = 0; a < 3; ++a) s.Rgrad[3 * iR + a] = s.A[a][0] * c[0] + s.A[a][1] * c[1] + s.A[a][2] * c[2];
        }
    }
    // lasers (Simulation.cpp:121-144, Laser.cpp)
    for (int il = 0; il < cfg->nlasers; ++il) {
        const oracle_laser& L = cfg->lasers[il];
        Laser l;
        l.t0 = L.t0_au;
        l.amplitude = std::sqrt(L.intensity_au);
        l.omega = L.omega_au;
        double period = 2. * pi / l.omega;
        l.duration = L.cycles * period;
        l.phase = L.phase;
        l.envelope = L.envelope;
        l.fwhm = L.fwhm_au;
        double nrm = std::sqrt(L.pol[0] * L.pol[0] + L.pol[1] * L.pol[1] + L.pol[2] * L.pol[2]);
        double pol[3] = {L.pol[0] / nrm, L.pol[1] / nrm, L.pol[2] / nrm};
        double n2 = std::sqrt(pol[0] * pol[0] + pol[1] * pol[1] + pol[2] * pol[2]);
        for (int d = 0; d < 3; ++d) l.pol[d] = pol[d] / n2;
        s.lasers.push_back(l);
    }
    // eigensystem (Simulation.cpp:263-286)
    s.eval.resize((size_t)Nk * nb);
    s.U.resize(s.S());
#pragma omp parallel for schedule(dynamic)
    for (int ik = 0; ik < Nk; ++ik) eigh(nb, &s.H0k[(size_t)ik * P], &s.eval[(size_t)ik * nb], &s.U[(size_t)ik * P]);
    // initial condition: rho_w = U diag(f) U^H (Functional_InitialCondition.hpp:15-31,
    // Operator.hpp:528-545)
    s.rho.assign(s.S(), 0.);
#pragma omp parallel for schedule(static)
    for (int ik = 0; ik < Nk; ++ik) {
        std::vector<cd> rb(P, 0.), tmp(P, 0.), Ud(P);
        const cd* Uk = &s.U[(size_t)ik * P];
        for (int i = 0; i < nb; ++i)
            for (int j = 0; j < nb; ++j) Ud[i * nb + j] = std::conj(Uk[j * nb + i]);
        for (int b = 0; b < cfg->filledbands && b < nb; ++b) rb[b * nb + b] = 1.;
        matmul(nb, Uk, rb.data(), tmp.data(), 1., 0.);
        matmul(nb, tmp.data(), Ud.data(), &s.rho[(size_t)ik * P], 1., 0.);
    }
    // solver (DESolver.cpp:11-33, DESolver.hpp:109-126)
    s.solver = cfg->solver;
    s.order = cfg->order;
    s.dt = cfg->dt_au;
    s.t = 0.;  // DESolver::CurrentTime starts at 0 whatever InitialTime is
    for (auto& a : s.aux) a.assign(s.S(), 0.);
    if (s.solver == 0) {
        if (s.order == 4) { double b[5] = {55. / 24., -59. / 24., 37. / 24., -3. / 8., 0.}; std::copy(b, b + 5, s.beta); }
        else if (s.order == 5) { double b[5] = {1901. / 720., -2774. / 720., 2616. / 720., -1274. / 720., 251. / 720.}; std::copy(b, b + 5, s.beta); }
        else throw std::runtime_error("order not implemented for AB");
    } else if (s.order != 4) {
        throw std::runtime_error("RK implemented for order 4 only");
    }
    // coulomb (Coulomb.cpp:19-59, ModelCoulomb.cpp:62-134, Simulation.cpp:177-181)
    s.coulomb = cfg->coulomb != 0;
    if (s.coulomb) {
        if (s.dims != 2 && !(s.N[2] == 1)) throw std::runtime_error("Only 2d coulomb is implemented");
        s.epsilon = cfg->epsilon;
        // ModelCoulomb::set_r0 (ModelCoulomb.cpp:187-215)
        s.r0[0] = cfg->r0_au[0];
        if (cfg->nr0 <= 1) { s.r0[1] = s.r0[2] = cfg->r0_au[0]; }
        else if (cfg->nr0 == 2) { s.r0[1] = cfg->r0_au[1]; s.r0[2] = (cfg->r0_au[0] + cfg->r0_au[1]) / 2.; }
        else { s.r0[1] = cfg->r0_au[1]; s.r0[2] = cfg->r0_au[2]; }
        s.r0_avg = (s.r0[0] + s.r0[1] + s.r0[2]) / 3.;
        // wannier centres = diag of r(R=0) of the model (ModelCoulomb.cpp:101-110)
        int iorg = -1;
        for (int iR = 0; iR < m.nR; ++iR)
            if (m.R[3 * iR] == 0 && m.R[3 * iR + 1] == 0 && m.R[3 * iR + 2] == 0) iorg = iR;
        if (iorg < 0) throw std::runtime_error("model has no R=0 block");
        std::vector<std::array<double, 3>> wc(nb);
        for (int n = 0; n < nb; ++n)
            for (int d = 0; d < 3; ++d) wc[n][d] = m.r[d][((size_t)iorg * nb + n) * nb + n].real();
        // minimum non-zero distance (ModelCoulomb.cpp:116-126)
        s.min_dist[0] = 100; s.min_dist[1] = 0; s.min_dist[2] = 0;
        s.min_dist_norm = 100;
        for (int n = 0; n < nb; ++n)
            for (int mm = n + 1; mm < nb; ++mm) {
                double dd[3] = {wc[n][0] - wc[mm][0], wc[n][1] - wc[mm][1], wc[n][2] - wc[mm][2]};
                double dn = std::sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
                if (dn < s.min_dist_norm && dn > 1.e-05) {
                    std::copy(dd, dd + 3, s.min_dist);
                    s.min_dist_norm = dn;
                }
            }
        // potentials on the Gamma-centred master R grid (ModelCoulomb.cpp:62-83),
        // including the cumulative r = r - c_m of line 78 unless fixed
        s.W.assign(s.S(), 0.);
        s.V.assign(s.S(), 0.);
        for (int iR = 0; iR < Nk; ++iR) {
            const double* Rc = &s.Rcart[3 * (size_t)iR];
            for (int n = 0; n < nb; ++n) {
                double r[3] = {wc[n][0] - Rc[0], wc[n][1] - Rc[1], wc[n][2] - Rc[2]};
                for (int mm = 0; mm < nb; ++mm) {
                    double rr[3];
                    if (cfg->coulomb_fix_centres) {
                        for (int d = 0; d < 3; ++d) rr[d] = wc[n][d] - Rc[d] - wc[mm][d];
                    } else {
                        for (int d = 0; d < 3; ++d) { r[d] = r[d] - wc[mm][d]; rr[d] = r[d]; }
                    }
                    s.V[((size_t)iR * nb + n) * nb + mm] = s.V_of(rr);
                    s.W[((size_t)iR * nb + n) * nb + mm] = s.W_of(rr);
                }
            }
        }
        if (cfg->hermitian_nyquist) {
            std::vector<cd> Ws(s.W);
            for (int iR = 0; iR < Nk; ++iR) {
                const int j[3] = {iR / (s.N[1] * s.N[2]), (iR / s.N[2]) % s.N[1], iR % s.N[2]};
                const int mR = (((s.N[0] - j[0]) % s.N[0]) * s.N[1] + (s.N[1] - j[1]) % s.N[1]) * s.N[2] +
                               (s.N[2] - j[2]) % s.N[2];
                for (int n = 0; n < nb; ++n)
                    for (int mm = 0; mm < nb; ++mm)
                        Ws[((size_t)iR * nb + n) * nb + mm] =
                            0.5 * (s.W[((size_t)iR * nb + n) * nb + mm] + s.W[((size_t)mR * nb + mm) * nb + n]);
            }
            s.W.swap(Ws);
        }
        // Hartree_nm = sum_R V_nm(R), symmetrised (Coulomb.cpp:41-58)
        s.Hartree.assign(P, 0.);
        for (int iR = 0; iR < Nk; ++iR)
            for (int p = 0; p < P; ++p) s.Hartree[p] += s.V[(size_t)iR * P + p];
        for (int i = 0; i < nb; ++i)
            for (int j = i + 1; j < nb; ++j) {
                cd v = (s.Hartree[i * nb + j] + s.Hartree[j * nb + i]) / 2.;
                s.Hartree[i * nb + j] = v;
                s.Hartree[j * nb + i] = v;
            }
        s.origin = 0;  // MasterRgrid.find(0,0,0) = index 0
        s.DM0R.resize(s.S());
        s.fft.run(s.rho.data(), s.DM0R.data(), -1);  // Simulation.cpp:180-181
    }
    // velocity operator (Simulation.cpp:523-576): v = -i[r,H0]_k, then the
    // gradient of H0 along axis d in the space of propagation of the gradient
    // (:554-556): gradient_space "R": (R space) += i R_d H0(R) and back to k;
    // gradient_space "k": += sum_b w_b b_d H0(k + b) (kGradient_definitions.hpp:18-30
    // with direction e_d); then / |det A| (2-D) or det (3-D)
    if (s.dims >= 2) {
        double det;
        if (s.dims == 3) {
            det = std::abs(s.A[0][0] * (s.A[1][1] * s.A[2][2] - s.A[1][2] * s.A[2][1]) -
                           s.A[0][1] * (s.A[1][0] * s.A[2][2] - s.A[1][2] * s.A[2][0]) +
                           s.A[0][2] * (s.A[1][0] * s.A[2][1] - s.A[1][1] * s.A[2][0]));
        } else {
            if (s.N[2] > 1) throw std::runtime_error("perpendicular != 2 -> implement me!");
            det = std::abs(s.A[0][0] * s.A[1][1] - s.A[1][0] * s.A[0][1]);
        }
        std::vector<cd> vR(s.S());
        for (int d = 0; d < 3; ++d) {
            s.vel[d].assign(s.S(), 0.);
            for (int ik = 0; ik < Nk; ++ik) {
                cd* o = &s.vel[d][(size_t)ik * P];
                const cd* r = &s.rk[d][(size_t)ik * P];
                const cd* h = &s.H0k[(size_t)ik * P];
                matmul(nb, r, h, o, -im, 0.);
                matmul(nb, h, r, o, im, 1.);
            }
            if (s.gw.empty()) {
                s.fft.run(s.vel[d].data(), vR.data(), -1);
                for (int iR = 0; iR < Nk; ++iR) {
                    double Rd = s.Rcart[3 * (size_t)iR + d];
                    for (int p = 0; p < P; ++p) vR[(size_t)iR * P + p] += 1. * im * Rd * s.H0R[(size_t)iR * P + p];
                }
                s.fft.run(vR.data(), s.vel[d].data(), +1);
            } else {
                for (int ik = 0; ik < Nk; ++ik) {
                    const int j[3] = {ik / (s.N[1] * s.N[2]), (ik / s.N[2]) % s.N[1], ik % s.N[2]};
                    for (size_t i = 0; i < s.gw.size(); ++i) {
                        const double c = s.gw[i] * s.gvec[i][d];
                        if (c == 0.) continue;
                        const int jn[3] = {(j[0] + s.gshift[i][0]) % s.N[0], (j[1] + s.gshift[i][1]) % s.N[1],
                                           (j[2] + s.gshift[i][2]) % s.N[2]};
                        const size_t kn = ((size_t)jn[0] * s.N[1] + jn[1]) * s.N[2] + jn[2];
                        for (int p = 0; p < P; ++p) s.vel[d][(size_t)ik * P + p] += c * s.H0k[kn * P + p];
                    }
                }
            }
            for (auto& x : s.vel[d]) x /= det;
        }
    }
    s.inR.resize(s.S());
    s.outR.resize(s.S());
    s.HR.resize(s.S());
    s.Hk.resize(s.S());
    return sim.release();
}

// Finite-difference k gradient (src/kGradient/kGradient.cpp:26-211, after
// Mostofi et al., CPC 178 (2008) 685): the Gamma-centred k mesh (crystal
// coordinates in [-1/2, 1/2), MeshGrid.cpp:458-486; Cartesian k = B k_crys,
// B = 2 pi A^-T, Model.hpp:46) sorted into shells of equal |b| (k = 0 removed);
// the fewest shells whose matrix A(j, s) = sum_{b in s} b_alpha b_beta (six
// (alpha, beta) pairs) solves A w = q exactly by its pseudo-inverse, q = (1
// per axis with N > 1, 0, 0, 0).  Then E.grad f(k) = sum_s w_s sum_{b in s}
// (b.E) f(k + b).
void build_kgradient(Sim& s) {
    const int Nk = s.Nk;
    // B = 2 pi (A^-1)^T, columns the reciprocal vectors
    const double (&A)[3][3] = s.A;
    const double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                       A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                       A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
    double inv[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const int i1 = (j + 1) % 3, i2 = (j + 2) % 3, j1 = (i + 1) % 3, j2 = (i + 2) % 3;
            inv[i][j] = (A[i1][j1] * A[i2][j2] - A[i1][j2] * A[i2][j1]) / det;
        }
    double B[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) B[i][j] = 2. * pi * inv[j][i];
    std::vector<std::array<double, 3>> kc(Nk);
    std::vector<std::array<int, 3>> kj(Nk);
    std::vector<double> norm(Nk);
    for (int ik = 0; ik < Nk; ++ik) {
        const int j[3] = {ik / (s.N[1] * s.N[2]), (ik / s.N[2]) % s.N[1], ik % s.N[2]};
        double c[3];
        for (int d = 0; d < 3; ++d) {
            double x = (double)j[d] / s.N[d];
            while (x < -0.5 && std::abs(x + 0.5) > threshold) x += 1.;
            while (x > 0.5 || std::abs(x - 0.5) < threshold) x -= 1.;
            c[d] = x;
            kj[ik][d] = j[d];
        }
        for (int a = 0; a < 3; ++a) kc[ik][a] = B[a][0] * c[0] + B[a][1] * c[1] + B[a][2] * c[2];
        norm[ik] = std::sqrt(kc[ik][0] * kc[ik][0] + kc[ik][1] * kc[ik][1] + kc[ik][2] * kc[ik][2]);
    }
    // SortInShells (kGradient.cpp:44-83)
    std::vector<double> knorms;
    for (int ik = 0; ik < Nk; ++ik) {
        bool found = false;
        for (double kn : knorms) found |= std::abs(kn - norm[ik]) < threshold;
        if (!found) knorms.push_back(norm[ik]);
    }
    std::sort(knorms.begin(), knorms.end());
    std::vector<std::vector<int>> shells(knorms.size());
    for (int ik = 0; ik < Nk; ++ik)
        for (size_t sh = 0; sh < knorms.size(); ++sh)
            if (std::abs(knorms[sh] - norm[ik]) < 1.e-07) {
                shells[sh].push_back(ik);
                break;
            }
    if (knorms.empty() || std::abs(knorms[0]) > threshold) throw std::runtime_error("k mesh without k = 0");
    shells.erase(shells.begin());
    // Calculate_nshellsAndweights (kGradient.cpp:86-122)
    const double q[6] = {s.N[0] > 1 ? 1. : 0., s.N[1] > 1 ? 1. : 0., s.N[2] > 1 ? 1. : 0., 0., 0., 0.};
    const int al[6] = {0, 1, 2, 0, 0, 1}, be[6] = {0, 1, 2, 1, 2, 2};
    std::vector<double> w;
    int ns = 0;
    for (ns = 1; ns <= (int)shells.size(); ++ns) {
        std::vector<double> Am(6 * ns, 0.);  // A(j, s)
        for (int j = 0; j < 6; ++j)
            for (int sh = 0; sh < ns; ++sh)
                for (int ik : shells[sh]) Am[j * ns + sh] += kc[ik][al[j]] * kc[ik][be[j]];
        // pseudo-inverse: A^+ = (A^T A)^+ A^T, (A^T A)^+ from its eigen-decomposition
        std::vector<cd> M((size_t)ns * ns), V((size_t)ns * ns);
        std::vector<double> lam(ns);
        for (int a = 0; a < ns; ++a)
            for (int b = 0; b < ns; ++b) {
                double x = 0.;
                for (int j = 0; j < 6; ++j) x += Am[j * ns + a] * Am[j * ns + b];
                M[(size_t)a * ns + b] = x;
            }
        eigh(ns, M.data(), lam.data(), V.data());
        double lmax = 0.;
        for (double l : lam) lmax = std::max(lmax, std::abs(l));
        std::vector<double> Atq(ns, 0.);
        for (int a = 0; a < ns; ++a)
            for (int j = 0; j < 6; ++j) Atq[a] += Am[j * ns + a] * q[j];
        w.assign(ns, 0.);
        for (int e = 0; e < ns; ++e) {
            if (std::abs(lam[e]) <= 1e-12 * lmax) continue;
            double proj = 0.;
            for (int a = 0; a < ns; ++a) proj += V[(size_t)a * ns + e].real() * Atq[a];
            for (int a = 0; a < ns; ++a) w[a] += V[(size_t)a * ns + e].real() * proj / lam[e];
        }
        double res = 0.;
        for (int j = 0; j < 6; ++j) {
            double x = -q[j];
            for (int sh = 0; sh < ns; ++sh) x += Am[j * ns + sh] * w[sh];
            res += x * x;
        }
        if (std::sqrt(res) < threshold) break;
    }
    if (ns > (int)shells.size()) throw std::runtime_error("k gradient: no set of shells solves A w = q");
    s.gshift.clear();
    s.gvec.clear();
    s.gw.clear();
    for (int sh = 0; sh < ns; ++sh)
        for (int ik : shells[sh]) {
            s.gshift.push_back(kj[ik]);
            s.gvec.push_back(kc[ik]);
            s.gw.push_back(w[sh]);
        }
}

// SourceTerm: src/Simulation/Functional_SourceTerm.hpp:10-56
void source_term(Sim& s, cd* out_k, double time, const cd* in_k) {
    const int P = s.P, nb = s.nb;
    const size_t S = s.S();
    s.fft.run(in_k, s.inR.data(), -1);                         // :15 go_to_R
    std::fill(s.outR.begin(), s.outR.end(), cd(0.));           // :16
    double E[3];
    s.efield(time, E);
    // kGradient R branch: out(R) += 1 * i (R.E) in(R)  (kGradient_definitions.hpp:35-40);
    // no gradient term in the Peierls gauge (Functional_SourceTerm.hpp:20)
    const bool grad = !s.peierls;
#pragma omp parallel for schedule(static)
    for (int iR = 0; iR < (grad && s.gw.empty() ? s.Nk : 0); ++iR) {
        const double* Rc = &s.Rgrad[3 * (size_t)iR];
        double dot = Rc[0] * E[0] + Rc[1] * E[1] + Rc[2] * E[2];
        for (int p = 0; p < P; ++p) s.outR[(size_t)iR * P + p] += (1. + 0. * im) * im * dot * s.inR[(size_t)iR * P + p];
    }
    // Calculate_TDHamiltonian in R (Simulation.cpp:296-349)
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)S; ++i) {
        s.HR[i] = 0.;
        s.HR[i] += s.H0R[i] + E[0] * s.rR[0][i] + E[1] * s.rR[1][i] + E[2] * s.rR[2][i];
    }
    // Peierls gauge: the self-energy sees rho(R) e^{-iA.R} (Functional_SourceTerm.hpp:31-38)
    const cd* DM = s.inR.data();
    if (s.peierls) {
        s.auxR = s.inR;
        s.peierls_phase(s.auxR.data(), time, -1);
        DM = s.auxR.data();
    }
    // Coulomb::EffectiveHamiltonian (Coulomb.cpp:134-180)
    if (s.coulomb) {
        const size_t o = (size_t)s.origin * P;
        for (int n = 0; n < nb; ++n)
            for (int m = 0; m < nb; ++m)
                s.HR[o + n * nb + n] += s.Hartree[n * nb + m] * (DM[o + m * nb + m] - s.DM0R[o + m * nb + m]);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)S; ++i) s.HR[i] -= s.W[i] * (DM[i] - s.DM0R[i]);
    }
    // H(R) *= e^{+iA.R} (Functional_SourceTerm.hpp:41-44)
    if (s.peierls) s.peierls_phase(s.HR.data(), time, +1);
    s.fft.run(s.outR.data(), out_k, +1);                       // :49 Output.go_to_k
    if (grad && !s.gw.empty()) {
        // kGradient k branch (kGradient_definitions.hpp:18-30): out(k) += sum w (b.E) in(k + b)
#pragma omp parallel for schedule(static)
        for (int ik = 0; ik < s.Nk; ++ik) {
            const int j[3] = {ik / (s.N[1] * s.N[2]), (ik / s.N[2]) % s.N[1], ik % s.N[2]};
            for (size_t i = 0; i < s.gw.size(); ++i) {
                const double c = s.gw[i] * (s.gvec[i][0] * E[0] + s.gvec[i][1] * E[1] + s.gvec[i][2] * E[2]);
                if (c == 0.) continue;
                const int jn[3] = {(j[0] + s.gshift[i][0]) % s.N[0], (j[1] + s.gshift[i][1]) % s.N[1],
                                   (j[2] + s.gshift[i][2]) % s.N[2]};
                const size_t kn = ((size_t)jn[0] * s.N[1] + jn[1]) * s.N[2] + jn[2];
                for (int p = 0; p < P; ++p) out_k[(size_t)ik * P + p] += c * in_k[kn * P + p];
            }
        }
    }
    s.fft.run(s.HR.data(), s.Hk.data(), +1);                   // :50 H.go_to_k
    // commutator(Out, -i, H, rho, false) (BlockMatrix_definitions.hpp:203-226)
#pragma omp parallel for schedule(static)
    for (int ik = 0; ik < s.Nk; ++ik) {
        cd* o = out_k + (size_t)ik * P;
        const cd* h = &s.Hk[(size_t)ik * P];
        const cd* r = in_k + (size_t)ik * P;
        matmul(nb, h, r, o, -im, 1.);
        matmul(nb, r, h, o, im, 1.);
    }
}

static void sum_with_product(cd* out, double a, const cd* x, double b, const cd* y, size_t n) {
    // DESolver.hpp:10-20
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) out[i] = a * x[i] + b * y[i];
}

// DESolver::Propagate_RK (DESolver.hpp:154-187) / Propagate_AB (:201-220)
void propagate(Sim& s) {
    const size_t S = s.S();
    const double h = s.dt;
    if (s.solver == 1) {
        auto& k = s.aux[0];
        auto& aux = s.aux[1];
        auto& red = s.aux[2];
        cd* y = s.rho.data();
        source_term(s, k.data(), s.t, y);
        sum_with_product(aux.data(), 1., y, h / 2., k.data(), S);
        sum_with_product(red.data(), 1., y, h / 6., k.data(), S);
        source_term(s, k.data(), s.t + h / 2., aux.data());
        sum_with_product(aux.data(), 1., y, h / 2., k.data(), S);
        sum_with_product(red.data(), 1., red.data(), h / 3., k.data(), S);
        source_term(s, k.data(), s.t + h / 2., aux.data());
        sum_with_product(aux.data(), 1., y, h, k.data(), S);
        sum_with_product(red.data(), 1., red.data(), h / 3., k.data(), S);
        source_term(s, k.data(), s.t + h, aux.data());
        sum_with_product(y, 1., red.data(), h / 6., k.data(), S);
        s.t += h;
    } else {
        source_term(s, s.aux[s.index[0]].data(), s.t, s.rho.data());
        for (int i = 0; i < s.order; ++i)
            sum_with_product(s.rho.data(), 1., s.rho.data(), h * s.beta[i], s.aux[s.index[i]].data(), S);
        int tmp = s.index[s.order - 1];
        for (int i = s.order - 1; i > 0; --i) s.index[i] = s.index[i - 1];
        s.index[0] = tmp;
        s.t += h;
    }
}

}  // namespace oracle

extern "C" {

static char g_err[512];

const char* oracle_last_error() { return g_err; }

void* oracle_create(const oracle_cfg* cfg) {
    try {
        return oracle::build(cfg);
    } catch (const std::exception& e) {
        std::snprintf(g_err, sizeof(g_err), "%s", e.what());
        return nullptr;
    }
}

void oracle_destroy(void* h) { delete static_cast<Sim*>(h); }

void oracle_dims(void* h, int* out) {
    Sim& s = *static_cast<Sim*>(h);
    out[0] = s.N[0]; out[1] = s.N[1]; out[2] = s.N[2]; out[3] = s.nb; out[4] = s.Nk; out[5] = s.dims;
}

double oracle_time(void* h) { return static_cast<Sim*>(h)->t; }
void oracle_set_time(void* h, double t) { static_cast<Sim*>(h)->t = t; }

static void copy_out(const std::vector<cd>& v, double* dst) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(cd));
}

// which: 0 H0k, 1-3 xi_k (r_k), 4 W, 5 DM0R, 6 rho (state), 7 U, 8-10 vel_k,
// 11 H0R, 12 V (bare)
int oracle_get_array(void* h, int which, double* dst) {
    Sim& s = *static_cast<Sim*>(h);
    switch (which) {
        case 0: copy_out(s.H0k, dst); return 0;
        case 1: case 2: case 3: copy_out(s.rk[which - 1], dst); return 0;
        case 4: if (s.W.empty()) return -1; copy_out(s.W, dst); return 0;
        case 5: if (s.DM0R.empty()) return -1; copy_out(s.DM0R, dst); return 0;
        case 6: copy_out(s.rho, dst); return 0;
        case 7: copy_out(s.U, dst); return 0;
        case 8: case 9: case 10: if (s.vel[which - 8].empty()) return -1; copy_out(s.vel[which - 8], dst); return 0;
        case 11: copy_out(s.H0R, dst); return 0;
        case 12: if (s.V.empty()) return -1; copy_out(s.V, dst); return 0;
    }
    return -1;
}

void oracle_get_hartree(void* h, double* dst) { copy_out(static_cast<Sim*>(h)->Hartree, dst); }
void oracle_get_rcart(void* h, double* dst) {
    Sim& s = *static_cast<Sim*>(h);
    std::memcpy(dst, s.Rcart.data(), s.Rcart.size() * sizeof(double));
}
void oracle_get_eval(void* h, double* dst) {
    Sim& s = *static_cast<Sim*>(h);
    std::memcpy(dst, s.eval.data(), s.eval.size() * sizeof(double));
}
void oracle_get_lattice(void* h, double* dst) {
    Sim& s = *static_cast<Sim*>(h);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) dst[3 * i + j] = s.A[i][j];
}

void oracle_set_state(void* h, const double* src) {
    Sim& s = *static_cast<Sim*>(h);
    std::memcpy((void*)s.rho.data(), src, s.S() * sizeof(cd));
}

void oracle_efield(void* h, double t, double* E) { static_cast<Sim*>(h)->efield(t, E); }

// one SourceTerm evaluation (the unit-parity hook)
void oracle_rhs(void* h, double t, const double* in_k, double* out_k) {
    Sim& s = *static_cast<Sim*>(h);
    oracle::source_term(s, reinterpret_cast<cd*>(out_k), t, reinterpret_cast<const cd*>(in_k));
}

void oracle_step(void* h, int n) {
    Sim& s = *static_cast<Sim*>(h);
    for (int i = 0; i < n; ++i) oracle::propagate(s);
}

// Observables before a step, as Simulation::do_onestep prints them
// (Simulation.cpp:420-429,439-470,583-622).
// pop_bloch/pop_wannier: nb values each (bloch valence printed as 1 - rho);
// vel: 6 values (re,im of x,y,z).  Returns -1 for vel if not available (1-D).
int oracle_observables(void* h, double* pop_bloch, double* pop_wannier, double* vel) {
    Sim& s = *static_cast<Sim*>(h);
    const int nb = s.nb, P = s.P;
    // Peierls gauge: the observables see rho(R) e^{-iA.R} at CurrentTime
    // (Simulation.cpp:447-449, 593-595)
    const cd* rho = s.rho.data();
    std::vector<cd> shifted;
    if (s.peierls) {
        std::vector<cd> R(s.S());
        shifted.resize(s.S());
        s.fft.run(s.rho.data(), R.data(), -1);
        s.peierls_phase(R.data(), s.t, -1);
        s.fft.run(R.data(), shifted.data(), +1);
        rho = shifted.data();
    }
    std::vector<double> pb(nb, 0.), pw(nb, 0.);
    std::vector<cd> tmp(P), rb(P), Ud(P);
    for (int ik = 0; ik < s.Nk; ++ik) {
        const cd* Uk = &s.U[(size_t)ik * P];
        const cd* r = &rho[(size_t)ik * P];
        for (int i = 0; i < nb; ++i)
            for (int j = 0; j < nb; ++j) Ud[i * nb + j] = std::conj(Uk[j * nb + i]);
        matmul(nb, Ud.data(), r, tmp.data(), 1., 0.);
        matmul(nb, tmp.data(), Uk, rb.data(), 1., 0.);
        for (int n = 0; n < nb; ++n) {
            pb[n] += rb[n * nb + n].real();
            pw[n] += r[n * nb + n].real();
        }
    }
    for (int n = 0; n < nb; ++n) {
        pb[n] /= s.Nk;
        pw[n] /= s.Nk;
        // Print_Population: valence bands printed as 1 - rho_nn (Simulation.cpp:460-462)
        // the filled-band count is not stored here; the caller applies it
        if (pop_bloch) pop_bloch[n] = pb[n];
        if (pop_wannier) pop_wannier[n] = pw[n];
    }
    if (!vel) return 0;
    if (s.vel[0].empty()) return -1;
    for (int d = 0; d < 3; ++d) {
        cd v = 0.;
        for (int ik = 0; ik < s.Nk; ++ik) {
            const cd* a = &s.vel[d][(size_t)ik * P];
            const cd* r = &rho[(size_t)ik * P];
            for (int n = 0; n < nb; ++n)
                for (int k = 0; k < nb; ++k) v += a[n * nb + k] * r[k * nb + n];
        }
        v /= double(s.Nk);
        vel[2 * d] = v.real();
        vel[2 * d + 1] = v.imag();
    }
    return 0;
}

double oracle_struve0(double x) { return oracle::struve0(x); }

// SetOfLaser::VectorPotential at t (advances the integrator, as every request does)
void oracle_vector_potential(void* h, double t, double* out) { static_cast<Sim*>(h)->vector_potential(t, out); }

// standalone FFT of `howmany` interleaved planes on an N0xN1xN2 grid
void oracle_fft(const int* dims, int howmany, const double* in, double* out, int sign) {
    oracle::Fft3dMany f(dims, howmany);
    f.run(reinterpret_cast<const cd*>(in), reinterpret_cast<cd*>(out), sign);
}

void oracle_eigh(int n, const double* A, double* w, double* V) {
    oracle::eigh(n, reinterpret_cast<const cd*>(A), w, reinterpret_cast<cd*>(V));
}

}  // extern "C"
