// Plain-pointer wrappers around the reference's own CPU functions (QSR.cpp), compiled
// together with the reference's QSR.cpp (from the reference tree named by the Makefile's REF)
// by oracle/Makefile into oracle/_ref/.
// TEST INFRASTRUCTURE ONLY: used by tests to pin the FP64 oracle's per-cell math to the
// reference implementation. The reference's main() is renamed at compile time.
#include "QSR.h"

#include <cstring>
#include <vector>

static std::vector<QTensor> to_vec(const double* q, long long n) {
    std::vector<QTensor> v(n);
    std::memcpy(v.data(), q, sizeof(QTensor) * n);
    return v;
}

static DimensionalParams make_params(const double* pr) {
    DimensionalParams p;
    p.a = pr[0]; p.b = pr[1]; p.c = pr[2]; p.T = pr[3]; p.T_star = pr[4];
    p.L1 = pr[5]; p.L2 = pr[6]; p.L3 = pr[7]; p.W = pr[8];
    return p;
}

// Reference signatures at QSR.cpp:179 / 559 / 411 / 10 / 955.
void computeLaplacian(const std::vector<QTensor>& Q, std::vector<QTensor>& laplacianQ, int Nx, int Ny, int Nz,
                      double dx, double dy, double dz);
void computeChemicalPotential(const std::vector<QTensor>& Q, std::vector<QTensor>& mu,
                              const std::vector<QTensor>& laplacianQ, int Nx, int Ny, int Nz, double dx, double dy,
                              double dz, const DimensionalParams& params, double kappa, int modechoice);
double computeRadiality(const std::vector<QTensor>& Q, int Nx, int Ny, int Nz);
void applyWeakAnchoringPenalty(std::vector<QTensor>& mu, const std::vector<QTensor>& Q, int Nx, int Ny, int Nz,
                               const std::vector<bool>& is_shell, double S_shell, double W);
void updateQTensor(std::vector<QTensor>& Q, const std::vector<QTensor>& mu, int Nx, int Ny, int Nz, double dt,
                   const std::vector<bool>& is_shell, double gamma, double W);
void applyBoundaryConditions(std::vector<QTensor>& Q, int Nx, int Ny, int Nz, const std::vector<bool>& is_shell,
                             double S0, double W);

extern "C" {

void ref_laplacian(const double* q, double* lap, int Nx, int Ny, int Nz, double dx, double dy, double dz) {
    const long long n = (long long)Nx * Ny * Nz;
    std::vector<QTensor> Q = to_vec(q, n), L(n);
    computeLaplacian(Q, L, Nx, Ny, Nz, dx, dy, dz);
    std::memcpy(lap, L.data(), sizeof(QTensor) * n);
}

// params: a b c T T_star L1 L2 L3 W
void ref_chem_potential(const double* q, double* mu, int Nx, int Ny, int Nz, double dx, double dy, double dz,
                        const double* params, double kappa, int modechoice) {
    const long long n = (long long)Nx * Ny * Nz;
    std::vector<QTensor> Q = to_vec(q, n), L(n), M(n);
    computeLaplacian(Q, L, Nx, Ny, Nz, dx, dy, dz);
    computeChemicalPotential(Q, M, L, Nx, Ny, Nz, dx, dy, dz, make_params(params), kappa, modechoice);
    std::memcpy(mu, M.data(), sizeof(QTensor) * n);
}

void ref_energy(const double* q, int Nx, int Ny, int Nz, double dx, double dy, double dz, const double* params,
                double kappa, int modechoice, double* bulk, double* elastic) {
    const long long n = (long long)Nx * Ny * Nz;
    std::vector<QTensor> Q = to_vec(q, n);
    EnergyComponents ec = computeEnergyComponents(Q, Nx, Ny, Nz, dx, dy, dz, make_params(params), kappa, modechoice);
    *bulk = ec.bulk;
    *elastic = ec.elastic;
}

// n_steps of the reference CPU time step (QSR.cpp:395-400 chain: Laplacian, chemical
// potential, weak anchoring, update, boundary conditions) on the reference CPU's own droplet
// mask |r - R| < 1, centre N/2 (QSR.cpp:1091-1101), R = min(N)/2 there, or radius_cells when
// that is positive (so that the mask matches a workload's droplet size). Returns wall seconds
// of the stepping loop only.
double ref_run_steps(double* q, int Nx, int Ny, int Nz, double dx, double dy, double dz, const double* params,
                     double kappa, int modechoice, double gamma, double dt, double S_shell, int n_steps,
                     double radius_cells) {
    const long long n = (long long)Nx * Ny * Nz;
    std::vector<QTensor> Q = to_vec(q, n), L(n), M(n);
    std::vector<bool> is_shell(n, false);
    const double R = radius_cells > 0.0 ? radius_cells : std::min({(double)Nx, (double)Ny, (double)Nz}) / 2.0;
    const double cx = Nx / 2.0, cy = Ny / 2.0, cz = Nz / 2.0;
    for (int i = 0; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j)
            for (int k = 0; k < Nz; ++k) {
                const double r = std::sqrt(std::pow(i - cx, 2) + std::pow(j - cy, 2) + std::pow(k - cz, 2));
                if (std::abs(r - R) < 1.0) is_shell[k + Nz * (j + Ny * i)] = true;
            }
    const DimensionalParams P = make_params(params);
    const double t0 = omp_get_wtime();
    for (int s = 0; s < n_steps; ++s) {
        computeLaplacian(Q, L, Nx, Ny, Nz, dx, dy, dz);
        computeChemicalPotential(Q, M, L, Nx, Ny, Nz, dx, dy, dz, P, kappa, modechoice);
        applyWeakAnchoringPenalty(M, Q, Nx, Ny, Nz, is_shell, S_shell, P.W);
        updateQTensor(Q, M, Nx, Ny, Nz, dt, is_shell, gamma, P.W);
        applyBoundaryConditions(Q, Nx, Ny, Nz, is_shell, S_shell, P.W);
    }
    const double t1 = omp_get_wtime();
    std::memcpy(q, Q.data(), sizeof(QTensor) * n);
    return t1 - t0;
}

int ref_max_threads(void) { return omp_get_max_threads(); }

void ref_nematic(const double* q5, double* out4) {
    QTensor t;
    std::memcpy(&t, q5, sizeof(QTensor));
    NematicField nf = calculateNematicField(t);
    out4[0] = nf.S; out4[1] = nf.nx; out4[2] = nf.ny; out4[3] = nf.nz;
}

}  // extern "C"
