/*
 * FP64 CPU oracle for the Landau-de Gennes Q-tensor step -- TEST INFRASTRUCTURE ONLY.
 *
 * This is a CPU restatement of the reference algorithm (Spectre71/LCDrSimulator,
 * QSR.cu and KZM_bulk_ldg.cu) used as the checker in tests/, in the smoke check and
 * in bench.py's cpu_baseline leg. The product (the CUDA library under
 * lcdrsimulator_b200/) never links, loads or calls it.
 *
 * Parity pins: the per-cell math is checked against the reference's own QSR.cpp
 * functions compiled from the reference sources (oracle/ref_shim.cpp), and the
 * whole-step semantics against the reference's FP64 QSR.cu kernels run on a GPU
 * (oracle/ref_cuda_harness.cu -> tests/golden/).
 *
 * Layout: host AoS FP64, 5 doubles per cell (Qxx, Qxy, Qxz, Qyy, Qyz), cell index
 * k + Nz*(j + Ny*i) for the confined solver (QSR.cu:286) and x + Nx*(y + Ny*z) for
 * the periodic bulk solver (KZM_bulk_ldg.cu:161-169).
 */
#ifndef LDG_ORACLE_H
#define LDG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Physical and numerical parameters of the confined droplet solver. */
typedef struct orc_params {
    int Nx, Ny, Nz;
    double dx, dy, dz;
    double a, b, c, T_star;
    int bulk_modechoice;          /* 1 = std, 2 = ravnik (QSR.cu:385-397) */
    double kappa, L1, L2, L3;     /* kappa used only when L1 = L2 = L3 = 0 */
    double W, gamma;
    double droplet_radius_cells;  /* <= 0: reference radius 0.5*(min(N)-1) (QSR.cu:144-162) */
} orc_params;

/* Droplet geometry, field-for-field the reference DropletGeometry (QSR.cu:34-48). */
typedef struct orc_geometry {
    double dx, dy, dz;
    double center_x, center_y, center_z;
    double radius_x, radius_y, radius_z;
    double min_spacing, min_radius, shell_half_thickness, core_radius;
    double delta_eff;             /* shell volume / ellipsoid area (QSR.cu:174-185) */
    long long shell_count;
} orc_geometry;

/* Per-cell classification bits (computed once, in FP64, from the signed distance). */
enum {
    ORC_SHELL  = 1,   /* |sd| <= shell_half_thickness                        (QSR.cu:104-106) */
    ORC_EVOLVE = 2,   /* sd <= (W > 0 ? shell_half_thickness : 0)            (QSR.cu:108-111) */
    ORC_INSIDE = 4,   /* sd <= 0                                             (QSR.cu:100-102) */
    ORC_CORE   = 8,   /* sd < -2*min_spacing (avg_S / max_S / checker set)   (QSR.cu:2288-2300) */
    ORC_RADIAL = 16   /* inside and |r| > 2*min_spacing (radiality set)      (QSR.cu:1002) */
};

typedef struct orc_observables {
    double bulk, elastic, anchoring, total;
    double radiality;   long long radiality_count;
    double avg_S, max_S; long long core_count;
    double checker_rel;
    double checker_even_sum, checker_odd_sum, checker_all_sum;
    long long checker_even_n, checker_odd_n, checker_all_n;
    double defect_density; long long defect_count, defect_plaquettes;
    double xi_grad_proxy; double xi_sum_sq; long long xi_edges;
} orc_observables;

/* Periodic bulk (KZM_bulk_ldg) parameters. */
typedef struct orc_bulk_params {
    int Nx, Ny, Nz;
    double dx, dy, dz;
    double kappa, gamma, dt, q_norm_cap;
    double defects_S_threshold, defects_charge_cutoff;
} orc_bulk_params;

typedef struct orc_bulk_observables {
    double bulk, elastic, total, avg_S, max_S;
    double defect_density_per_plaquette, defect_line_density, xi_grad_proxy;
    long long defect_plaquettes_used, nonzero_defect_plaquettes;
} orc_bulk_observables;

/* ---- confined solver (QSR.cu semantics) ---- */
void orc_bulk_ABC(double a, double b, double c, double T, double T_star, int mode,
                  double* A, double* B, double* C);
double orc_S_eq(double A, double B, double C);
void orc_make_geometry(const orc_params* p, orc_geometry* g);
void orc_classify(const orc_params* p, orc_geometry* g, uint8_t* flags);
void orc_init(const orc_params* p, const orc_geometry* g, int mode, long long seed,
              double S0, double noise_amplitude, double* q);
void orc_laplacian(const orc_params* p, const double* q, double* lap);
void orc_divergence(const orc_params* p, const double* q, double* dcol /* 3 per cell */);
void orc_chem_potential(const orc_params* p, const orc_geometry* g, const uint8_t* flags,
                        const double* q, double T, double S_shell, double* mu);
/* One explicit Euler step (QSR.cu:3234-3249 chain). */
void orc_step_explicit(const orc_params* p, const orc_geometry* g, const uint8_t* flags,
                       double* q, double T, double S_shell, double dt, double q_norm_cap);
/* One semi-implicit IMEX step: RHS + jacobi_iters Jacobi sweeps + strong BC (QSR.cu:2721-2753). */
void orc_step_imex(const orc_params* p, const orc_geometry* g, const uint8_t* flags,
                   double* q, double T, double S_shell, double dt, double L_stab, int jacobi_iters);
void orc_nematic(const double* q, long long n, double* s_n /* 4 per cell: S nx ny nz */);
void orc_observe(const orc_params* p, const orc_geometry* g, const uint8_t* flags,
                 const double* q, double T, double S_shell,
                 int defects_z_slice, double defects_S_threshold, double defects_charge_cutoff,
                 int xi_z_slice, double xi_S_threshold, orc_observables* out);

/* ---- periodic bulk solver (KZM_bulk_ldg.cu semantics) ---- */
void orc_bulk_init(const orc_bulk_params* p, long long seed, double amplitude, double* q);
void orc_bulk_step(const orc_bulk_params* p, const double* q, double* q_next,
                   double A, double B, double C);
void orc_bulk_observe(const orc_bulk_params* p, const double* q, double A, double B, double C,
                      orc_bulk_observables* out);

/* ---- Philox4x32-R counter-based generator (Salmon et al., SC'11): R = 10 (known answers), R = 7 (device noise) ---- */
void orc_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void orc_philox4x32_rounds(const uint32_t ctr[4], const uint32_t key[2], int rounds, uint32_t out[4]);

#ifdef __cplusplus
}
#endif
#endif
