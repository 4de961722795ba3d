// FP64 CPU oracle -- TEST INFRASTRUCTURE ONLY (see ldg_oracle.h).
//
// Restates the reference algorithm cell by cell. Every function cites the reference
// file:line it follows. Parallelised with OpenMP over (i, j) rows; the arithmetic of
// each cell is written in the same order as the reference so that results agree to
// the last few ulps.
#include "ldg_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <random>
#include <vector>

namespace {

constexpr double kPi = 3.14159265358979323846;

struct Idx {
    int Nx, Ny, Nz;
    long long operator()(int i, int j, int k) const {
        return (long long)k + (long long)Nz * ((long long)j + (long long)Ny * (long long)i);
    }
};

// Component c of cell id; c = 5 is Qzz = -(Qxx + Qyy) (QSR.cuh:50-66).
inline double qc(const double* q, long long id, int c) {
    if (c == 5) return -(q[5 * id + 0] + q[5 * id + 3]);
    return q[5 * id + c];
}

// One-sided-at-faces first derivative (QSR.cu:245-273).
inline double deriv1(const double* f, int fstride, int comp, long long id, long long stride,
                     int n, int cur, double inv_2d, double inv_d) {
    auto v = [&](long long x) { return f[fstride * x + comp]; };
    if (cur > 0 && cur < n - 1) return (v(id + stride) - v(id - stride)) * inv_2d;
    if (cur == 0) return (v(id + stride) - v(id)) * inv_d;
    return (v(id) - v(id - stride)) * inv_d;
}

struct Point { double x, y, z, center_radius, signed_distance; };

// sampleDropletGeometry (QSR.cu:70-98): ellipsoid signed-distance proxy (rho - 1)/|grad rho|.
Point sample(const orc_geometry& g, int i, int j, int k) {
    Point p;
    p.x = i * g.dx - g.center_x;
    p.y = j * g.dy - g.center_y;
    p.z = k * g.dz - g.center_z;
    p.center_radius = std::sqrt(p.x * p.x + p.y * p.y + p.z * p.z);
    const double sx = p.x / g.radius_x, sy = p.y / g.radius_y, sz = p.z / g.radius_z;
    const double rho_sq = sx * sx + sy * sy + sz * sz;
    if (rho_sq <= 1e-30) { p.signed_distance = -g.min_radius; return p; }
    const double rho = std::sqrt(rho_sq);
    const double gx = p.x / (g.radius_x * g.radius_x);
    const double gy = p.y / (g.radius_y * g.radius_y);
    const double gz = p.z / (g.radius_z * g.radius_z);
    const double gn = std::sqrt(gx * gx + gy * gy + gz * gz) / rho;
    p.signed_distance = (gn > 1e-30) ? (rho - 1.0) / gn : p.center_radius - g.min_radius;
    return p;
}

// getCenterDirection (QSR.cu:117-128).
void center_dir(const Point& p, double& nx, double& ny, double& nz) {
    if (p.center_radius <= 1e-30) { nx = 1.0; ny = 0.0; nz = 0.0; return; }
    nx = p.x / p.center_radius; ny = p.y / p.center_radius; nz = p.z / p.center_radius;
}

// getSurfaceNormal (QSR.cu:130-142): normal of the ellipsoid level set.
void surface_normal(const orc_geometry& g, const Point& p, double& nx, double& ny, double& nz) {
    const double gx = p.x / (g.radius_x * g.radius_x);
    const double gy = p.y / (g.radius_y * g.radius_y);
    const double gz = p.z / (g.radius_z * g.radius_z);
    const double gn = std::sqrt(gx * gx + gy * gy + gz * gz);
    if (gn <= 1e-30) { center_dir(p, nx, ny, nz); return; }
    nx = gx / gn; ny = gy / gn; nz = gz / gn;
}

// make_uniaxial_qtensor (QSR.cu:60-68).
void uniaxial(double S, double nx, double ny, double nz, double out[5]) {
    out[0] = S * (nx * nx - 1.0 / 3.0);
    out[1] = S * (nx * ny);
    out[2] = S * (nx * nz);
    out[3] = S * (ny * ny - 1.0 / 3.0);
    out[4] = S * (ny * nz);
}

// Bulk molecular field H = A Q - B (Q^2 - trQ2/3 I) + C trQ2 Q on the six tensor entries
// (QSR.cu:399-417), returned as xx, yy, zz, xy, xz, yz.
void bulk_h(const double* q5, double cQ, double cQ2, double cQ3, double h[6]) {
    const double Qxx = q5[0], Qxy = q5[1], Qxz = q5[2], Qyy = q5[3], Qyz = q5[4];
    const double Qzz = -Qxx - Qyy;
    const double trQ2 = Qxx * Qxx + Qyy * Qyy + Qzz * Qzz + 2 * (Qxy * Qxy + Qxz * Qxz + Qyz * Qyz);
    const double q2xx = Qxx * Qxx + Qxy * Qxy + Qxz * Qxz;
    const double q2xy = Qxx * Qxy + Qxy * Qyy + Qxz * Qyz;
    const double q2xz = Qxx * Qxz + Qxy * Qyz + Qxz * Qzz;
    const double q2yy = Qxy * Qxy + Qyy * Qyy + Qyz * Qyz;
    const double q2yz = Qxy * Qxz + Qyy * Qyz + Qyz * Qzz;
    const double q2zz = Qxz * Qxz + Qyz * Qyz + Qzz * Qzz;
    h[0] = cQ * Qxx - cQ2 * (q2xx - trQ2 / 3.0) + cQ3 * trQ2 * Qxx;
    h[1] = cQ * Qyy - cQ2 * (q2yy - trQ2 / 3.0) + cQ3 * trQ2 * Qyy;
    h[2] = cQ * Qzz - cQ2 * (q2zz - trQ2 / 3.0) + cQ3 * trQ2 * Qzz;
    h[3] = cQ * Qxy - cQ2 * q2xy + cQ3 * trQ2 * Qxy;
    h[4] = cQ * Qxz - cQ2 * q2xz + cQ3 * trQ2 * Qxz;
    h[5] = cQ * Qyz - cQ2 * q2yz + cQ3 * trQ2 * Qyz;
}

void force_coeffs(const orc_params* p, double T, double& cQ, double& cQ2, double& cQ3) {
    // computeChemicalPotentialKernel coefficients (QSR.cu:385-397).
    const double dT = T - p->T_star;
    cQ = 3.0 * p->a * dT;
    if (p->bulk_modechoice == 1) { cQ2 = (9.0 * p->b) / 2.0; cQ3 = (9.0 * p->c) / 2.0; }
    else { cQ2 = (27.0 * p->b) / 2.0; cQ3 = 9.0 * p->c; }
}

}  // namespace

// ---------------------------------------------------------------------------------------
// Bulk constants and geometry
// ---------------------------------------------------------------------------------------

extern "C" void orc_bulk_ABC(double a, double b, double c, double T, double T_star, int mode,
                             double* A, double* B, double* C) {
    // bulk_ABC_from_convention (QSR.cu:1363-1378).
    *A = 3.0 * a * (T - T_star);
    if (mode == 1) { *B = (9.0 * b) / 2.0; *C = (9.0 * c) / 2.0; }
    else { *B = (27.0 * b) / 2.0; *C = 9.0 * c; }
}

extern "C" double orc_S_eq(double A, double B, double C) {
    // S_eq_uniaxial_from_ABC (QSR.cu:1391-1418): lower-energy root of 2 C S^2 - B S + 3 A = 0.
    if (!(C > 0.0)) return 0.0;
    const double disc = B * B - 24.0 * A * C;
    if (!(disc > 0.0)) return 0.0;
    const double sd = std::sqrt(disc);
    const double roots[2] = {(B - sd) / (4.0 * C), (B + sd) / (4.0 * C)};
    double best_S = 0.0, best_f = 0.0;
    for (double S : roots) {
        if (!(S > 0.0)) continue;
        const double S2 = S * S;
        const double f = (A / 3.0) * S2 - (2.0 * B / 27.0) * (S2 * S) + (C / 9.0) * (S2 * S2);
        if (f < best_f) { best_f = f; best_S = S; }
    }
    return best_S;
}

extern "C" void orc_make_geometry(const orc_params* p, orc_geometry* g) {
    // makeDropletGeometry (QSR.cu:144-162); the optional radius override replaces the
    // radius index 0.5*(min(N)-1) and keeps the centre at (N-1)/2.
    std::memset(g, 0, sizeof(*g));
    g->dx = p->dx; g->dy = p->dy; g->dz = p->dz;
    g->center_x = 0.5 * ((double)p->Nx - 1.0) * p->dx;
    g->center_y = 0.5 * ((double)p->Ny - 1.0) * p->dy;
    g->center_z = 0.5 * ((double)p->Nz - 1.0) * p->dz;
    double radius_index = 0.5 * ((double)std::min({p->Nx, p->Ny, p->Nz}) - 1.0);
    if (p->droplet_radius_cells > 0.0) radius_index = p->droplet_radius_cells;
    g->radius_x = std::max(radius_index * p->dx, 0.5 * p->dx);
    g->radius_y = std::max(radius_index * p->dy, 0.5 * p->dy);
    g->radius_z = std::max(radius_index * p->dz, 0.5 * p->dz);
    g->min_spacing = std::min({p->dx, p->dy, p->dz});
    g->min_radius = std::min({g->radius_x, g->radius_y, g->radius_z});
    g->shell_half_thickness = g->min_spacing;
    g->core_radius = g->min_spacing;
    g->delta_eff = 2.0 * g->shell_half_thickness;
}

extern "C" void orc_classify(const orc_params* p, orc_geometry* g, uint8_t* flags) {
    // Host shell mask (QSR.cu:2160-2172) plus the per-cell predicates each kernel evaluates
    // (QSR.cu:100-111, 1002, 2288-2300), and delta_eff (QSR.cu:164-185).
    const Idx idx{p->Nx, p->Ny, p->Nz};
    const double band = (p->W > 0.0) ? g->shell_half_thickness : 0.0;
    long long shell = 0;
#pragma omp parallel for collapse(2) reduction(+ : shell)
    for (int i = 0; i < p->Nx; ++i)
        for (int j = 0; j < p->Ny; ++j)
            for (int k = 0; k < p->Nz; ++k) {
                const Point pt = sample(*g, i, j, k);
                uint8_t f = 0;
                if (std::fabs(pt.signed_distance) <= g->shell_half_thickness) { f |= ORC_SHELL; ++shell; }
                if (pt.signed_distance <= band) f |= ORC_EVOLVE;
                if (pt.signed_distance <= 0.0) f |= ORC_INSIDE;
                if (pt.signed_distance < -2.0 * g->min_spacing) f |= ORC_CORE;
                if (pt.signed_distance <= 0.0 && pt.center_radius > 2.0 * g->min_spacing) f |= ORC_RADIAL;
                flags[idx(i, j, k)] = f;
            }
    g->shell_count = shell;
    // estimateEllipsoidSurfaceArea (Knud Thomsen, p = 1.6075) and estimateShellThicknessFromMask.
    const double nominal = 2.0 * g->shell_half_thickness;
    double delta = nominal;
    if (shell > 0) {
        const double pp = 1.6075;
        const double ap = std::pow(g->radius_x, pp), bp = std::pow(g->radius_y, pp), cp = std::pow(g->radius_z, pp);
        const double mean_term = (ap * bp + ap * cp + bp * cp) / 3.0;
        const double area = (mean_term > 0.0) ? 4.0 * kPi * std::pow(mean_term, 1.0 / pp)
                                              : std::numeric_limits<double>::quiet_NaN();
        if (area > 0.0) {
            const double t = (double)shell * g->dx * g->dy * g->dz / area;
            if (std::isfinite(t) && t > 0.0) delta = t;
        }
    }
    g->delta_eff = delta;
}

extern "C" void orc_init(const orc_params* p, const orc_geometry* g, int mode, long long seed,
                         double S0, double noise_amplitude, double* q) {
    // initializeQTensor / initializeIsotropicWithNoise (QSR.cu:1834-1904): std::mt19937 seeded
    // with random_seed, draws in i-j-k order for cells inside the droplet, zero outside.
    const Idx idx{p->Nx, p->Ny, p->Nz};
    const long long n = (long long)p->Nx * p->Ny * p->Nz;
    std::fill(q, q + 5 * n, 0.0);
    std::mt19937 gen = (seed >= 0) ? std::mt19937((std::mt19937::result_type)seed)
                                   : std::mt19937(std::random_device{}());
    if (mode == 2) {
        if (noise_amplitude <= 0.0) return;
        std::normal_distribution<double> dist(0.0, noise_amplitude);
        for (int i = 0; i < p->Nx; ++i)
            for (int j = 0; j < p->Ny; ++j)
                for (int k = 0; k < p->Nz; ++k) {
                    const Point pt = sample(*g, i, j, k);
                    if (pt.signed_distance <= 0.0) {
                        double* c = q + 5 * idx(i, j, k);
                        for (int m = 0; m < 5; ++m) c[m] = dist(gen);
                    }
                }
        return;
    }
    std::uniform_real_distribution<double> dist_theta(0.0, kPi);
    std::uniform_real_distribution<double> dist_phi(0.0, 2.0 * kPi);
    for (int i = 0; i < p->Nx; ++i)
        for (int j = 0; j < p->Ny; ++j)
            for (int k = 0; k < p->Nz; ++k) {
                const Point pt = sample(*g, i, j, k);
                if (!(pt.signed_distance <= 0.0)) continue;
                double S = S0;
                if (pt.center_radius < g->core_radius) S *= (pt.center_radius / g->core_radius);
                double nx, ny, nz;
                if (mode == 0) {
                    const double theta = dist_theta(gen);
                    const double phi = dist_phi(gen);
                    nx = std::sin(theta) * std::cos(phi);
                    ny = std::sin(theta) * std::sin(phi);
                    nz = std::cos(theta);
                } else {
                    center_dir(pt, nx, ny, nz);
                }
                uniaxial(S, nx, ny, nz, q + 5 * idx(i, j, k));
            }
}

// ---------------------------------------------------------------------------------------
// Differential operators
// ---------------------------------------------------------------------------------------

extern "C" void orc_laplacian(const orc_params* p, const double* q, double* lap) {
    // computeLaplacianKernel (QSR.cu:279-323): central 3-point per axis, the shifted interior
    // stencil (f2 - 2 f1 + f0) at the two faces of each axis.
    const int Nx = p->Nx, Ny = p->Ny, Nz = p->Nz;
    const Idx idx{Nx, Ny, Nz};
    const double ix2 = 1.0 / (p->dx * p->dx), iy2 = 1.0 / (p->dy * p->dy), iz2 = 1.0 / (p->dz * p->dz);
#pragma omp parallel for collapse(2)
    for (int i = 0; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j)
            for (int k = 0; k < Nz; ++k) {
                const long long id = idx(i, j, k);
                auto axis = [&](int cur, int n, long long stride, int c, double inv) {
                    const double* b = q + c;
                    auto v = [&](long long x) { return b[5 * x]; };
                    if (cur > 0 && cur < n - 1) return (v(id + stride) - v(id) * 2.0 + v(id - stride)) * inv;
                    if (cur == 0) return (v(id + 2 * stride) - v(id + stride) * 2.0 + v(id)) * inv;
                    return (v(id) - v(id - stride) * 2.0 + v(id - 2 * stride)) * inv;
                };
                for (int c = 0; c < 5; ++c) {
                    const double d2x = axis(i, Nx, (long long)Ny * Nz, c, ix2);
                    const double d2y = axis(j, Ny, Nz, c, iy2);
                    const double d2z = axis(k, Nz, 1, c, iz2);
                    lap[5 * id + c] = d2x + d2y + d2z;
                }
            }
}

extern "C" void orc_divergence(const orc_params* p, const double* q, double* D) {
    // computeDivergenceKernel (QSR.cu:325-371): D_j = d_k Q_kj with one-sided faces.
    const int Nx = p->Nx, Ny = p->Ny, Nz = p->Nz;
    const Idx idx{Nx, Ny, Nz};
    const long long sx = (long long)Ny * Nz, sy = Nz, sz = 1;
    const double i2x = 1.0 / (2.0 * p->dx), i2y = 1.0 / (2.0 * p->dy), i2z = 1.0 / (2.0 * p->dz);
    const double ix = 1.0 / p->dx, iy = 1.0 / p->dy, iz = 1.0 / p->dz;
#pragma omp parallel for collapse(2)
    for (int i = 0; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j)
            for (int k = 0; k < Nz; ++k) {
                const long long id = idx(i, j, k);
                auto dX = [&](int c) { return deriv1(q, 5, c, id, sx, Nx, i, i2x, ix); };
                auto dY = [&](int c) { return deriv1(q, 5, c, id, sy, Ny, j, i2y, iy); };
                auto dZ = [&](int c) { return deriv1(q, 5, c, id, sz, Nz, k, i2z, iz); };
                D[3 * id + 0] = dX(0) + dY(1) + dZ(2);
                D[3 * id + 1] = dX(1) + dY(3) + dZ(4);
                // dQzz/dz on the reconstructed Qzz (QSR.cu:356-368).
                double dzz;
                const double c0 = qc(q, id, 5);
                if (k > 0 && k < Nz - 1) dzz = (qc(q, id + 1, 5) - qc(q, id - 1, 5)) * i2z;
                else if (k == 0) dzz = (qc(q, id + 1, 5) - c0) * iz;
                else dzz = (c0 - qc(q, id - 1, 5)) * iz;
                D[3 * id + 2] = dX(2) + dY(4) + dzz;
            }
}

extern "C" void orc_chem_potential(const orc_params* p, const orc_geometry* g, const uint8_t* flags,
                                   const double* q, double T, double S_shell, double* mu) {
    // mu = bulk + elastic (kappa | L1, L2) projected traceless (QSR.cu:373-472), then the L3
    // contribution on interior cells re-projected (QSR.cu:474-621), then the weak-anchoring
    // penalty on shell cells (QSR.cu:623-652).
    const int Nx = p->Nx, Ny = p->Ny, Nz = p->Nz;
    const Idx idx{Nx, Ny, Nz};
    const long long n = (long long)Nx * Ny * Nz;
    std::vector<double> lap(5 * n);
    orc_laplacian(p, q, lap.data());
    const bool need_D = (p->L2 != 0.0 || p->L3 != 0.0);
    std::vector<double> D;
    if (need_D) { D.resize(3 * n); orc_divergence(p, q, D.data()); }
    double cQ, cQ2, cQ3;
    force_coeffs(p, T, cQ, cQ2, cQ3);
    const long long sx = (long long)Ny * Nz, sy = Nz, sz = 1;
    const double i2x = 1.0 / (2.0 * p->dx), i2y = 1.0 / (2.0 * p->dy), i2z = 1.0 / (2.0 * p->dz);
    const double ix = 1.0 / p->dx, iy = 1.0 / p->dy, iz = 1.0 / p->dz;
    const double ix2 = 1.0 / (p->dx * p->dx), iy2 = 1.0 / (p->dy * p->dy), iz2 = 1.0 / (p->dz * p->dz);
    const double i4xy = 1.0 / (4.0 * p->dx * p->dy), i4xz = 1.0 / (4.0 * p->dx * p->dz),
                 i4yz = 1.0 / (4.0 * p->dy * p->dz);
    const bool all_L_zero = (p->L1 == 0.0 && p->L2 == 0.0 && p->L3 == 0.0);
#pragma omp parallel for collapse(2)
    for (int i = 0; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j)
            for (int k = 0; k < Nz; ++k) {
                const long long id = idx(i, j, k);
                const double* q5 = q + 5 * id;
                const double* L = lap.data() + 5 * id;
                double h[6];  // xx yy zz xy xz yz
                bulk_h(q5, cQ, cQ2, cQ3, h);
                const double lzz = -L[0] - L[3];
                if (all_L_zero) {
                    h[0] -= p->kappa * L[0]; h[1] -= p->kappa * L[3]; h[2] -= p->kappa * lzz;
                    h[3] -= p->kappa * L[1]; h[4] -= p->kappa * L[2]; h[5] -= p->kappa * L[4];
                }
                if (p->L1 != 0.0) {
                    h[0] -= p->L1 * L[0]; h[1] -= p->L1 * L[3]; h[2] -= p->L1 * lzz;
                    h[3] -= p->L1 * L[1]; h[4] -= p->L1 * L[2]; h[5] -= p->L1 * L[4];
                }
                if (p->L2 != 0.0) {
                    const double* Dp = D.data();
                    auto dX = [&](int c) { return deriv1(Dp, 3, c, id, sx, Nx, i, i2x, ix); };
                    auto dY = [&](int c) { return deriv1(Dp, 3, c, id, sy, Ny, j, i2y, iy); };
                    auto dZ = [&](int c) { return deriv1(Dp, 3, c, id, sz, Nz, k, i2z, iz); };
                    const double dDx_dx = dX(0), dDy_dy = dY(1), dDz_dz = dZ(2);
                    const double dDx_dy = dY(0), dDy_dx = dX(1), dDx_dz = dZ(0);
                    const double dDz_dx = dX(2), dDy_dz = dZ(1), dDz_dy = dY(2);
                    h[0] -= p->L2 * dDx_dx; h[1] -= p->L2 * dDy_dy; h[2] -= p->L2 * dDz_dz;
                    h[3] -= p->L2 * (dDy_dx + dDx_dy);
                    h[4] -= p->L2 * (dDz_dx + dDx_dz);
                    h[5] -= p->L2 * (dDz_dy + dDy_dz);
                }
                double corr = (h[0] + h[1] + h[2]) / 3.0;
                double m[5] = {h[0] - corr, h[3], h[4], h[1] - corr, h[5]};

                const bool interior = (i > 0 && i < Nx - 1 && j > 0 && j < Ny - 1 && k > 0 && k < Nz - 1);
                if (p->L3 != 0.0 && interior) {
                    double hx[6] = {m[0], m[3], -(m[0] + m[3]), m[1], m[2], m[4]};
                    double d[6][3];  // [comp 0..5][axis]
                    for (int c = 0; c < 5; ++c) {
                        d[c][0] = (qc(q, id + sx, c) - qc(q, id - sx, c)) * i2x;
                        d[c][1] = (qc(q, id + sy, c) - qc(q, id - sy, c)) * i2y;
                        d[c][2] = (qc(q, id + sz, c) - qc(q, id - sz, c)) * i2z;
                    }
                    for (int a = 0; a < 3; ++a) d[5][a] = -(d[0][a] + d[3][a]);
                    // M_ab = (d_a Q_kl)(d_b Q_kl) (QSR.cu:558-570).
                    auto M = [&](int a, int b) {
                        return d[0][a] * d[0][b] + d[3][a] * d[3][b] + d[5][a] * d[5][b] +
                               2.0 * (d[1][a] * d[1][b] + d[2][a] * d[2][b] + d[4][a] * d[4][b]);
                    };
                    const double Mxx = M(0, 0), Myy = M(1, 1), Mzz = M(2, 2);
                    const double Mxy = M(0, 1), Mxz = M(0, 2), Myz = M(1, 2);
                    hx[0] += 0.5 * p->L3 * Mxx; hx[1] += 0.5 * p->L3 * Myy; hx[2] += 0.5 * p->L3 * Mzz;
                    hx[3] += 0.5 * p->L3 * Mxy; hx[4] += 0.5 * p->L3 * Mxz; hx[5] += 0.5 * p->L3 * Myz;
                    const double Qxx = q5[0], Qxy = q5[1], Qxz = q5[2], Qyy = q5[3], Qyz = q5[4];
                    const double Qzz = -Qxx - Qyy;
                    const double* Dc = D.data() + 3 * id;
                    // B(Q_c) = D . grad Q_c + Q_ab d_a d_b Q_c (QSR.cu:580-603).
                    auto Bc = [&](int c) {
                        const double Qc = qc(q, id, c);
                        const double d2xx = (qc(q, id + sx, c) - 2.0 * Qc + qc(q, id - sx, c)) * ix2;
                        const double d2yy = (qc(q, id + sy, c) - 2.0 * Qc + qc(q, id - sy, c)) * iy2;
                        const double d2zz = (qc(q, id + sz, c) - 2.0 * Qc + qc(q, id - sz, c)) * iz2;
                        const double d2xy = (qc(q, id + sx + sy, c) - qc(q, id + sx - sy, c) -
                                             qc(q, id - sx + sy, c) + qc(q, id - sx - sy, c)) * i4xy;
                        const double d2xz = (qc(q, id + sx + sz, c) - qc(q, id + sx - sz, c) -
                                             qc(q, id - sx + sz, c) + qc(q, id - sx - sz, c)) * i4xz;
                        const double d2yz = (qc(q, id + sy + sz, c) - qc(q, id + sy - sz, c) -
                                             qc(q, id - sy + sz, c) + qc(q, id - sy - sz, c)) * i4yz;
                        const double contract = Qxx * d2xx + Qyy * d2yy + Qzz * d2zz +
                                                2.0 * (Qxy * d2xy + Qxz * d2xz + Qyz * d2yz);
                        return Dc[0] * d[c][0] + Dc[1] * d[c][1] + Dc[2] * d[c][2] + contract;
                    };
                    const double Bxx = Bc(0), Byy = Bc(3), Bzz = -(Bxx + Byy);
                    const double Bxy = Bc(1), Bxz = Bc(2), Byz = Bc(4);
                    hx[0] -= p->L3 * Bxx; hx[1] -= p->L3 * Byy; hx[2] -= p->L3 * Bzz;
                    hx[3] -= p->L3 * Bxy; hx[4] -= p->L3 * Bxz; hx[5] -= p->L3 * Byz;
                    corr = (hx[0] + hx[1] + hx[2]) / 3.0;
                    m[0] = hx[0] - corr; m[3] = hx[1] - corr;
                    m[1] = hx[3]; m[2] = hx[4]; m[4] = hx[5];
                }
                const uint8_t f = flags[id];
                if ((f & ORC_SHELL) && p->W != 0.0 && g->delta_eff > 0.0) {
                    const Point pt = sample(*g, i, j, k);
                    double nx = 1.0, ny = 0.0, nz = 0.0;
                    surface_normal(*g, pt, nx, ny, nz);
                    double Q0[5];
                    uniaxial(S_shell, nx, ny, nz, Q0);
                    const double We = p->W / g->delta_eff;
                    for (int c = 0; c < 5; ++c) m[c] += We * (q5[c] - Q0[c]);
                }
                for (int c = 0; c < 5; ++c) mu[5 * id + c] = m[c];
            }
}

static void strong_bc(const orc_params* p, const orc_geometry* g, const uint8_t* flags, double* q,
                      double S_shell) {
    // applyBoundaryConditionsKernel (QSR.cu:851-867): W <= 0 -> shell cells set to Q0.
    if (p->W > 0.0) return;
    const Idx idx{p->Nx, p->Ny, p->Nz};
#pragma omp parallel for collapse(2)
    for (int i = 0; i < p->Nx; ++i)
        for (int j = 0; j < p->Ny; ++j)
            for (int k = 0; k < p->Nz; ++k) {
                const long long id = idx(i, j, k);
                if (!(flags[id] & ORC_SHELL)) continue;
                const Point pt = sample(*g, i, j, k);
                double nx = 1.0, ny = 0.0, nz = 0.0;
                surface_normal(*g, pt, nx, ny, nz);
                uniaxial(S_shell, nx, ny, nz, q + 5 * id);
            }
}

static inline bool moves(const orc_params* p, uint8_t f) {
    // updateQTensorKernel gates (QSR.cu:705-709).
    if (p->W == 0.0 && (f & ORC_SHELL)) return false;
    return (f & ORC_EVOLVE) != 0;
}

extern "C" void orc_step_explicit(const orc_params* p, const orc_geometry* g, const uint8_t* flags,
                                  double* q, double T, double S_shell, double dt, double q_norm_cap) {
    const long long n = (long long)p->Nx * p->Ny * p->Nz;
    std::vector<double> mu(5 * n);
    orc_chem_potential(p, g, flags, q, T, S_shell, mu.data());
    const double mob = 1.0 / p->gamma;
#pragma omp parallel for
    for (long long id = 0; id < n; ++id) {
        if (!moves(p, flags[id])) continue;
        double* c = q + 5 * id;
        // updateQTensorKernel (QSR.cu:711-731).
        for (int m = 0; m < 5; ++m) c[m] -= mob * mu[5 * id + m] * dt;
        if (q_norm_cap > 0.0) {
            const double Qzz = -c[0] - c[3];
            const double tr = c[0] * c[0] + c[3] * c[3] + Qzz * Qzz + 2.0 * (c[1] * c[1] + c[2] * c[2] + c[4] * c[4]);
            const double qn = std::sqrt(tr > 0.0 ? tr : 0.0);
            if (qn > q_norm_cap && qn > 0.0) {
                const double s = q_norm_cap / qn;
                for (int m = 0; m < 5; ++m) c[m] *= s;
            }
        }
    }
    strong_bc(p, g, flags, q, S_shell);
}

extern "C" void orc_step_imex(const orc_params* p, const orc_geometry* g, const uint8_t* flags,
                              double* q, double T, double S_shell, double dt, double L_stab,
                              int jacobi_iters) {
    const int Nx = p->Nx, Ny = p->Ny, Nz = p->Nz;
    const Idx idx{Nx, Ny, Nz};
    const long long n = (long long)Nx * Ny * Nz;
    std::vector<double> mu(5 * n), lap(5 * n), rhs(5 * n), qa(q, q + 5 * n), qb(5 * n);
    orc_chem_potential(p, g, flags, q, T, S_shell, mu.data());
    orc_laplacian(p, q, lap.data());
    const double mob = 1.0 / p->gamma;
    const double alpha = dt * mob * L_stab;
    // computeRhsSemiImplicitKernel (QSR.cu:734-784).
#pragma omp parallel for
    for (long long id = 0; id < n; ++id) {
        for (int m = 0; m < 5; ++m) {
            rhs[5 * id + m] = moves(p, flags[id])
                ? q[5 * id + m] - (dt * mob) * mu[5 * id + m] - alpha * lap[5 * id + m]
                : q[5 * id + m];
        }
    }
    const double ix2 = 1.0 / (p->dx * p->dx), iy2 = 1.0 / (p->dy * p->dy), iz2 = 1.0 / (p->dz * p->dz);
    const double alpha_j = (dt / p->gamma) * L_stab;  // host alpha (QSR.cu:2728)
    const double denom = 1.0 + 2.0 * alpha_j * (ix2 + iy2 + iz2);
    const long long sx = (long long)Ny * Nz, sy = Nz, sz = 1;
    double* qo = qa.data();
    double* qn = qb.data();
    for (int it = 0; it < jacobi_iters; ++it) {
        // jacobiHelmholtzStepKernel (QSR.cu:786-849).
#pragma omp parallel for collapse(2)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny; ++j)
                for (int k = 0; k < Nz; ++k) {
                    const long long id = idx(i, j, k);
                    const bool face = (i == 0 || j == 0 || k == 0 || i == Nx - 1 || j == Ny - 1 || k == Nz - 1);
                    if (face || !moves(p, flags[id]) || !(denom > 0.0)) {
                        for (int m = 0; m < 5; ++m) qn[5 * id + m] = qo[5 * id + m];
                        continue;
                    }
                    for (int m = 0; m < 5; ++m) {
                        auto v = [&](long long x) { return qo[5 * x + m]; };
                        qn[5 * id + m] = (rhs[5 * id + m] +
                                          alpha_j * (ix2 * (v(id + sx) + v(id - sx)) +
                                                     iy2 * (v(id + sy) + v(id - sy)) +
                                                     iz2 * (v(id + sz) + v(id - sz)))) / denom;
                    }
                }
        std::swap(qo, qn);
    }
    std::copy(qo, qo + 5 * n, q);
    strong_bc(p, g, flags, q, S_shell);
}

// ---------------------------------------------------------------------------------------
// Observables
// ---------------------------------------------------------------------------------------

namespace {
struct NF { double S, nx, ny, nz; };

// calculateNematicFieldDevice (QSR.cu:191-243): shifted power iteration for the largest
// eigenvalue, S = 1.5 lambda_max, director gauge nz >= 0, isotropic cut-off 1e-9.
NF nematic(const double* q5, double iso_cut, NF iso) {
    const double Qxx = q5[0], Qxy = q5[1], Qxz = q5[2], Qyy = q5[3], Qyz = q5[4];
    const double Qzz = -Qxx - Qyy;
    if (std::fabs(Qxx) < iso_cut && std::fabs(Qxy) < iso_cut && std::fabs(Qxz) < iso_cut &&
        std::fabs(Qyy) < iso_cut && std::fabs(Qyz) < iso_cut)
        return iso;
    double nx = Qxx + Qxy + Qxz;
    double ny = Qxy + Qyy + Qyz;
    double nz = Qxz + Qyz - Qxx - Qyy;
    const double n0 = std::sqrt(nx * nx + ny * ny + nz * nz);
    if (n0 > 1e-12) { nx /= n0; ny /= n0; nz /= n0; }
    else { nx = 0.0; ny = 0.0; nz = 1.0; }
    const double r1 = std::fabs(Qxx) + std::fabs(Qxy) + std::fabs(Qxz);
    const double r2 = std::fabs(Qxy) + std::fabs(Qyy) + std::fabs(Qyz);
    const double r3 = std::fabs(Qxz) + std::fabs(Qyz) + std::fabs(Qzz);
    const double alpha = std::max(r1, std::max(r2, r3)) + 1e-12;
    for (int it = 0; it < 15; ++it) {
        const double ax = Qxx * nx + Qxy * ny + Qxz * nz + alpha * nx;
        const double ay = Qxy * nx + Qyy * ny + Qyz * nz + alpha * ny;
        const double az = Qxz * nx + Qyz * ny + Qzz * nz + alpha * nz;
        const double nn = std::sqrt(ax * ax + ay * ay + az * az);
        if (nn < 1e-13) break;
        nx = ax / nn; ny = ay / nn; nz = az / nn;
    }
    const double lam = nx * (Qxx * nx + Qxy * ny + Qxz * nz) + ny * (Qxy * nx + Qyy * ny + Qyz * nz) +
                       nz * (Qxz * nx + Qyz * ny + Qzz * nz);
    const double S = 1.5 * lam;
    if (nz < -1e-10) { nx = -nx; ny = -ny; nz = -nz; }
    return {S, nx, ny, nz};
}

// wrap_to_pi_device (QSR.cu:1027-1035).
inline double wrap_pi(double x) {
    const double two_pi = 2.0 * kPi;
    x = x + kPi;
    x -= std::floor(x / two_pi) * two_pi;
    return x - kPi;
}
}  // namespace

extern "C" void orc_nematic(const double* q, long long n, double* s_n) {
#pragma omp parallel for
    for (long long id = 0; id < n; ++id) {
        const NF f = nematic(q + 5 * id, 1e-9, NF{0.0, 0.0, 0.0, 1.0});
        s_n[4 * id + 0] = f.S; s_n[4 * id + 1] = f.nx; s_n[4 * id + 2] = f.ny; s_n[4 * id + 3] = f.nz;
    }
}

extern "C" void orc_observe(const orc_params* p, const orc_geometry* g, const uint8_t* flags,
                            const double* q, double T, double S_shell,
                            int dz_slice, double dS_thr, double d_cut,
                            int xi_slice, double xi_thr, orc_observables* o) {
    const int Nx = p->Nx, Ny = p->Ny, Nz = p->Nz;
    const Idx idx{Nx, Ny, Nz};
    std::memset(o, 0, sizeof(*o));
    // computeEnergyKernel (QSR.cu:869-992): interior cells, central differences.
    const double dT = T - p->T_star;
    double c2, c3, c4;
    if (p->bulk_modechoice == 1) { c2 = (3.0 * p->a * dT) / 2.0; c3 = (3.0 * p->b) / 2.0; c4 = (9.0 * p->c) / 8.0; }
    else { c2 = (3.0 * p->a * dT) / 2.0; c3 = (9.0 * p->b) / 2.0; c4 = (9.0 * p->c) / 4.0; }
    const double dV = p->dx * p->dy * p->dz;
    const double i2x = 1.0 / (2.0 * p->dx), i2y = 1.0 / (2.0 * p->dy), i2z = 1.0 / (2.0 * p->dz);
    const long long sx = (long long)Ny * Nz, sy = Nz, sz = 1;
    const bool all_L_zero = (p->L1 == 0.0 && p->L2 == 0.0 && p->L3 == 0.0);
    double eb = 0.0, ee = 0.0, ea = 0.0, rad = 0.0, Ssum = 0.0, Smax = 0.0;
    long long radn = 0, coren = 0;
#pragma omp parallel for collapse(2) reduction(+ : eb, ee, ea, rad, Ssum, radn, coren) reduction(max : Smax)
    for (int i = 0; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j)
            for (int k = 0; k < Nz; ++k) {
                const long long id = idx(i, j, k);
                const double* q5 = q + 5 * id;
                const uint8_t f = flags[id];
                const bool interior = (i >= 1 && j >= 1 && k >= 1 && i < Nx - 1 && j < Ny - 1 && k < Nz - 1);
                if (interior) {
                    const double Qxx = q5[0], Qxy = q5[1], Qxz = q5[2], Qyy = q5[3], Qyz = q5[4];
                    const double Qzz = -Qxx - Qyy;
                    const double trQ2 = Qxx * Qxx + Qyy * Qyy + Qzz * Qzz + 2 * (Qxy * Qxy + Qxz * Qxz + Qyz * Qyz);
                    // trQ3 over the full symmetric tensor (QSR.cu:901-913).
                    const double a2xx = Qxx * Qxx + Qxy * Qxy + Qxz * Qxz;
                    const double a2xy = Qxx * Qxy + Qxy * Qyy + Qxz * Qyz;
                    const double a2xz = Qxx * Qxz + Qxy * Qyz + Qxz * Qzz;
                    const double a2yx = Qxy * Qxx + Qyy * Qxy + Qyz * Qxz;
                    const double a2yy = Qxy * Qxy + Qyy * Qyy + Qyz * Qyz;
                    const double a2yz = Qxy * Qxz + Qyy * Qyz + Qyz * Qzz;
                    const double a2zx = Qxz * Qxx + Qyz * Qxy + Qzz * Qxz;
                    const double a2zy = Qxz * Qxy + Qyz * Qyy + Qzz * Qyz;
                    const double a2zz = Qxz * Qxz + Qyz * Qyz + Qzz * Qzz;
                    const double trQ3 = Qxx * a2xx + Qxy * a2yx + Qxz * a2zx + Qxy * a2xy + Qyy * a2yy +
                                        Qyz * a2zy + Qxz * a2xz + Qyz * a2yz + Qzz * a2zz;
                    eb += (c2 * trQ2 - c3 * trQ3 + c4 * trQ2 * trQ2) * dV;
                    double d[6][3];
                    for (int c = 0; c < 5; ++c) {
                        d[c][0] = (q[5 * (id + sx) + c] - q[5 * (id - sx) + c]) * i2x;
                        d[c][1] = (q[5 * (id + sy) + c] - q[5 * (id - sy) + c]) * i2y;
                        d[c][2] = (q[5 * (id + sz) + c] - q[5 * (id - sz) + c]) * i2z;
                    }
                    for (int a = 0; a < 3; ++a) d[5][a] = -(d[0][a] + d[3][a]);
                    auto sq = [&](int c) { return d[c][0] * d[c][0] + d[c][1] * d[c][1] + d[c][2] * d[c][2]; };
                    const double g2 = sq(0) + sq(3) + sq(5) + 2.0 * (sq(1) + sq(2) + sq(4));
                    double fel;
                    if (all_L_zero) {
                        fel = 0.5 * p->kappa * g2;
                    } else {
                        const double f1 = 0.5 * p->L1 * g2;
                        const double dvx = d[0][0] + d[1][1] + d[2][2];
                        const double dvy = d[1][0] + d[3][1] + d[4][2];
                        const double dvz = d[2][0] + d[4][1] + d[5][2];
                        const double f2 = 0.5 * p->L2 * (dvx * dvx + dvy * dvy + dvz * dvz);
                        double f3 = 0.0;
                        if (p->L3 != 0.0) {
                            auto M = [&](int a, int b) {
                                return d[0][a] * d[0][b] + d[3][a] * d[3][b] + d[5][a] * d[5][b] +
                                       2.0 * (d[1][a] * d[1][b] + d[2][a] * d[2][b] + d[4][a] * d[4][b]);
                            };
                            f3 = 0.5 * p->L3 * (Qxx * M(0, 0) + Qyy * M(1, 1) + Qzz * M(2, 2) +
                                                2.0 * (Qxy * M(0, 1) + Qxz * M(0, 2) + Qyz * M(1, 2)));
                        }
                        fel = f1 + f2 + f3;
                    }
                    ee += fel * dV;
                }
                if ((f & ORC_SHELL) && p->W != 0.0 && g->delta_eff > 0.0) {
                    // computeAnchoringEnergyKernel (QSR.cu:654-695).
                    const Point pt = sample(*g, i, j, k);
                    double nx = 1.0, ny = 0.0, nz = 0.0;
                    surface_normal(*g, pt, nx, ny, nz);
                    double Q0[5];
                    uniaxial(S_shell, nx, ny, nz, Q0);
                    const double dxx = q5[0] - Q0[0], dxy = q5[1] - Q0[1], dxz = q5[2] - Q0[2];
                    const double dyy = q5[3] - Q0[3], dyz = q5[4] - Q0[4];
                    const double dzz = (-q5[0] - q5[3]) - (-(Q0[0] + Q0[3]));
                    const double diff2 = dxx * dxx + dyy * dyy + dzz * dzz + 2.0 * (dxy * dxy + dxz * dxz + dyz * dyz);
                    ea += 0.5 * (p->W / g->delta_eff) * diff2 * dV;
                }
                if (f & (ORC_RADIAL | ORC_CORE)) {
                    const NF nf = nematic(q5, 1e-9, NF{0.0, 0.0, 0.0, 1.0});
                    if (f & ORC_RADIAL) {
                        // computeRadialityKernel (QSR.cu:994-1015).
                        const Point pt = sample(*g, i, j, k);
                        double rx, ry, rz;
                        center_dir(pt, rx, ry, rz);
                        rad += std::fabs(nf.nx * rx + nf.ny * ry + nf.nz * rz);
                        ++radn;
                    }
                    if (f & ORC_CORE) {
                        // compute_avg_S_droplet / compute_max_S_droplet (QSR.cu:2285-2321).
                        Ssum += nf.S;
                        ++coren;
                        if (std::isfinite(nf.S)) Smax = std::max(Smax, nf.S);
                    }
                }
            }
    o->bulk = eb; o->elastic = ee; o->anchoring = ea; o->total = eb + ee + ea;
    o->radiality_count = radn;
    o->radiality = (radn > 0) ? rad / radn : 0.0;
    o->core_count = coren;
    o->avg_S = (coren > 0) ? Ssum / coren : 0.0;
    o->max_S = Smax;

    // Checkerboard parity amplitude on the defect slice (QSR.cu:2845-2873).
    o->checker_rel = std::numeric_limits<double>::quiet_NaN();
    {
        const int kz = std::min(std::max(dz_slice, 0), Nz - 1);
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny; ++j) {
                const long long id = idx(i, j, kz);
                if (!(flags[id] & ORC_CORE)) continue;
                const double s = nematic(q + 5 * id, 1e-9, NF{0.0, 0.0, 0.0, 1.0}).S;
                if (!std::isfinite(s) || s <= 0.01) continue;
                o->checker_all_sum += s; o->checker_all_n++;
                if (((i + j) & 1) == 0) { o->checker_even_sum += s; o->checker_even_n++; }
                else { o->checker_odd_sum += s; o->checker_odd_n++; }
            }
        if (o->max_S >= 0.5 && o->checker_even_n > 10 && o->checker_odd_n > 10 && o->checker_all_n > 20 &&
            o->checker_all_sum != 0.0)
            o->checker_rel = std::fabs(o->checker_even_sum - o->checker_odd_sum) / std::fabs(o->checker_all_sum);
    }

    // computeDefectDensity2DProxyKernel (QSR.cu:1114-1176).
    auto nf_at = [&](int i, int j, int k) { return nematic(q + 5 * idx(i, j, k), 1e-9, NF{0.0, 0.0, 0.0, 1.0}); };
    auto ok = [&](const NF& f, double thr) {
        return std::isfinite(f.S) && std::isfinite(f.nx) && std::isfinite(f.ny) && f.S > thr;
    };
    if (dz_slice >= 0 && dz_slice < Nz) {
        for (int i = 0; i < Nx - 1; ++i)
            for (int j = 0; j < Ny - 1; ++j) {
                const NF a = nf_at(i, j, dz_slice), b = nf_at(i + 1, j, dz_slice);
                const NF c = nf_at(i + 1, j + 1, dz_slice), d = nf_at(i, j + 1, dz_slice);
                if (!(ok(a, dS_thr) && ok(b, dS_thr) && ok(c, dS_thr) && ok(d, dS_thr))) continue;
                const double p00 = 2.0 * std::atan2(a.ny, a.nx), p10 = 2.0 * std::atan2(b.ny, b.nx);
                const double p11 = 2.0 * std::atan2(c.ny, c.nx), p01 = 2.0 * std::atan2(d.ny, d.nx);
                const double dsum = wrap_pi(p10 - p00) + wrap_pi(p11 - p10) + wrap_pi(p01 - p11) + wrap_pi(p00 - p01);
                const double s = 0.5 * (dsum * (1.0 / (2.0 * kPi)));
                o->defect_plaquettes++;
                if (std::fabs(s) > d_cut) o->defect_count++;
            }
    }
    o->defect_density = (o->defect_plaquettes > 0) ? (double)o->defect_count / (double)o->defect_plaquettes
                                                   : std::numeric_limits<double>::quiet_NaN();
    // computeXiGradEdgesX/YKernel + compute_xi_grad_proxy_2d (QSR.cu:1042-1106, 2372-2410).
    o->xi_grad_proxy = std::numeric_limits<double>::quiet_NaN();
    if (xi_slice >= 0 && xi_slice < Nz) {
        for (int i = 0; i < Nx - 1; ++i)
            for (int j = 0; j < Ny; ++j) {
                const NF a = nf_at(i, j, xi_slice), b = nf_at(i + 1, j, xi_slice);
                if (!(ok(a, xi_thr) && ok(b, xi_thr))) continue;
                const double dd = wrap_pi(2.0 * std::atan2(b.ny, b.nx) - 2.0 * std::atan2(a.ny, a.nx));
                o->xi_sum_sq += dd * dd; o->xi_edges++;
            }
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny - 1; ++j) {
                const NF a = nf_at(i, j, xi_slice), b = nf_at(i, j + 1, xi_slice);
                if (!(ok(a, xi_thr) && ok(b, xi_thr))) continue;
                const double dd = wrap_pi(2.0 * std::atan2(b.ny, b.nx) - 2.0 * std::atan2(a.ny, a.nx));
                o->xi_sum_sq += dd * dd; o->xi_edges++;
            }
        if (o->xi_edges > 0) {
            const double mean_sq = o->xi_sum_sq / (double)o->xi_edges;
            const double eps = 1e-30;
            const double inv = (mean_sq > 0.0) ? (1.0 / std::sqrt(mean_sq + eps)) : (1.0 / std::sqrt(eps));
            o->xi_grad_proxy = std::min(inv, 0.5 * (double)std::min(Nx, Ny));
        }
    }
}

// ---------------------------------------------------------------------------------------
// Periodic bulk solver (KZM_bulk_ldg.cu)
// ---------------------------------------------------------------------------------------

extern "C" void orc_bulk_init(const orc_bulk_params* p, long long seed, double amplitude, double* q) {
    // KZM_bulk_ldg.cu:874-893: std::mt19937_64(seed), N(0,1) * amplitude, 5 draws per site in
    // memory order (x fastest).
    const long long n = (long long)p->Nx * p->Ny * p->Nz;
    std::mt19937_64 rng((unsigned long long)seed);
    std::normal_distribution<double> gauss(0.0, 1.0);
    for (long long s = 0; s < n; ++s)
        for (int m = 0; m < 5; ++m) q[5 * s + m] = amplitude * gauss(rng);
}

extern "C" void orc_bulk_step(const orc_bulk_params* p, const double* q, double* qn,
                              double A, double B, double C) {
    // updateBulkLdgKernel without noise (KZM_bulk_ldg.cu:351-469): periodic 7-point Laplacian,
    // bulk field, -kappa Laplacian, traceless projection, explicit Euler, optional cap.
    const int Nx = p->Nx, Ny = p->Ny, Nz = p->Nz;
    const double ix2 = 1.0 / (p->dx * p->dx), iy2 = 1.0 / (p->dy * p->dy), iz2 = 1.0 / (p->dz * p->dz);
    const double mob = 1.0 / p->gamma;
    auto fl = [&](int x, int y, int z) { return (long long)x + (long long)Nx * ((long long)y + (long long)Ny * z); };
#pragma omp parallel for collapse(2)
    for (int z = 0; z < Nz; ++z)
        for (int y = 0; y < Ny; ++y)
            for (int x = 0; x < Nx; ++x) {
                const int xp = (x + 1) % Nx, xm = (x + Nx - 1) % Nx;
                const int yp = (y + 1) % Ny, ym = (y + Ny - 1) % Ny;
                const int zp = (z + 1) % Nz, zm = (z + Nz - 1) % Nz;
                const long long id = fl(x, y, z);
                const double* c = q + 5 * id;
                double lap[5];
                for (int m = 0; m < 5; ++m) {
                    lap[m] = (q[5 * fl(xp, y, z) + m] - 2.0 * c[m] + q[5 * fl(xm, y, z) + m]) * ix2 +
                             (q[5 * fl(x, yp, z) + m] - 2.0 * c[m] + q[5 * fl(x, ym, z) + m]) * iy2 +
                             (q[5 * fl(x, y, zp) + m] - 2.0 * c[m] + q[5 * fl(x, y, zm) + m]) * iz2;
                }
                double h[6];
                bulk_h(c, A, B, C, h);
                h[0] -= p->kappa * lap[0]; h[1] -= p->kappa * lap[3]; h[2] += p->kappa * (lap[0] + lap[3]);
                h[3] -= p->kappa * lap[1]; h[4] -= p->kappa * lap[2]; h[5] -= p->kappa * lap[4];
                const double corr = (h[0] + h[1] + h[2]) / 3.0;
                h[0] -= corr; h[1] -= corr;
                double u[5] = {c[0] - mob * p->dt * h[0], c[1] - mob * p->dt * h[3], c[2] - mob * p->dt * h[4],
                               c[3] - mob * p->dt * h[1], c[4] - mob * p->dt * h[5]};
                if (p->q_norm_cap > 0.0) {
                    const double Qzz = -u[0] - u[3];
                    const double tr = u[0] * u[0] + u[3] * u[3] + Qzz * Qzz + 2.0 * (u[1] * u[1] + u[2] * u[2] + u[4] * u[4]);
                    const double qnrm = std::sqrt(std::max(tr, 0.0));
                    if (qnrm > p->q_norm_cap && qnrm > 0.0) {
                        const double s = p->q_norm_cap / qnrm;
                        for (int m = 0; m < 5; ++m) u[m] *= s;
                    }
                }
                for (int m = 0; m < 5; ++m) qn[5 * id + m] = u[m];
            }
}

namespace {
// wrap_to_pi of KZM_bulk_ldg.cu:471-479 (loop form).
inline double wrap_pi_loop(double d) {
    while (d <= -kPi) d += 2.0 * kPi;
    while (d > kPi) d -= 2.0 * kPi;
    return d;
}
bool project_plane(const NF& f, int plane, double& u, double& v) {
    // project_to_plane (KZM_bulk_ldg.cu:481-499).
    if (plane == 0) { u = f.nx; v = f.ny; }
    else if (plane == 1) { u = f.ny; v = f.nz; }
    else { u = f.nx; v = f.nz; }
    const double nrm = std::sqrt(u * u + v * v);
    if (!(nrm > 1e-8)) return false;
    u /= nrm; v /= nrm;
    return true;
}
// plaquette_charge (KZM_bulk_ldg.cu:501-541). Returns 0 = not used, 1 = used, 2 = defect.
int plaquette(const NF& a, const NF& b, const NF& c, const NF& d, int plane, double thr, double cut) {
    if (!(std::isfinite(a.S) && std::isfinite(b.S) && std::isfinite(c.S) && std::isfinite(d.S))) return 0;
    if (!(a.S > thr && b.S > thr && c.S > thr && d.S > thr)) return 0;
    double ua, va, ub, vb, uc, vc, ud, vd;
    if (!project_plane(a, plane, ua, va) || !project_plane(b, plane, ub, vb) ||
        !project_plane(c, plane, uc, vc) || !project_plane(d, plane, ud, vd))
        return 0;
    const double pa = 2.0 * std::atan2(va, ua), pb = 2.0 * std::atan2(vb, ub);
    const double pc = 2.0 * std::atan2(vc, uc), pd = 2.0 * std::atan2(vd, ud);
    const double dsum = wrap_pi_loop(pb - pa) + wrap_pi_loop(pc - pb) + wrap_pi_loop(pd - pc) + wrap_pi_loop(pa - pd);
    const double s = 0.5 * (dsum / (2.0 * kPi));
    return (std::fabs(s) > cut) ? 2 : 1;
}
}  // namespace

extern "C" void orc_bulk_observe(const orc_bulk_params* p, const double* q, double A, double B, double C,
                                 orc_bulk_observables* o) {
    // compute_observables (KZM_bulk_ldg.cu:543-713): forward differences, per-volume energies,
    // three plaquette orientations per site.
    const int Nx = p->Nx, Ny = p->Ny, Nz = p->Nz;
    const long long n = (long long)Nx * Ny * Nz;
    auto fl = [&](int x, int y, int z) { return (long long)x + (long long)Nx * ((long long)y + (long long)Ny * z); };
    const double cv = p->dx * p->dy * p->dz;
    const double tv = cv * (double)Nx * (double)Ny * (double)Nz;
    const double ix = 1.0 / p->dx, iy = 1.0 / p->dy, iz = 1.0 / p->dz;
    std::vector<NF> nf(n);
    double eb = 0.0, ee = 0.0, qi = 0.0, gi = 0.0, Ss = 0.0, Sm = 0.0;
#pragma omp parallel for collapse(2) reduction(+ : eb, ee, qi, gi, Ss) reduction(max : Sm)
    for (int z = 0; z < Nz; ++z)
        for (int y = 0; y < Ny; ++y)
            for (int x = 0; x < Nx; ++x) {
                const long long id = fl(x, y, z);
                const double* c = q + 5 * id;
                const double* px = q + 5 * fl((x + 1) % Nx, y, z);
                const double* py = q + 5 * fl(x, (y + 1) % Ny, z);
                const double* pz = q + 5 * fl(x, y, (z + 1) % Nz);
                const double Qxx = c[0], Qxy = c[1], Qxz = c[2], Qyy = c[3], Qyz = c[4], Qzz = -Qxx - Qyy;
                const double q2xx = Qxx * Qxx + Qxy * Qxy + Qxz * Qxz;
                const double q2xy = Qxx * Qxy + Qxy * Qyy + Qxz * Qyz;
                const double q2xz = Qxx * Qxz + Qxy * Qyz + Qxz * Qzz;
                const double q2yy = Qxy * Qxy + Qyy * Qyy + Qyz * Qyz;
                const double q2yz = Qxy * Qxz + Qyy * Qyz + Qyz * Qzz;
                const double q2zz = Qxz * Qxz + Qyz * Qyz + Qzz * Qzz;
                const double trQ2 = Qxx * Qxx + Qyy * Qyy + Qzz * Qzz + 2.0 * (Qxy * Qxy + Qxz * Qxz + Qyz * Qyz);
                // trQ3 as written at KZM_bulk_ldg.cu:590-593 (uses the symmetric q2 entries).
                const double trQ3 = Qxx * q2xx + Qxy * q2xy + Qxz * q2xz + Qxy * q2xy + Qyy * q2yy + Qyz * q2yz +
                                    Qxz * q2xz + Qyz * q2yz + Qzz * q2zz;
                eb += ((A / 2.0) * trQ2 - (B / 3.0) * trQ3 + (C / 4.0) * trQ2 * trQ2) * cv;
                double d[6][3];
                for (int m = 0; m < 5; ++m) {
                    d[m][0] = (px[m] - c[m]) * ix; d[m][1] = (py[m] - c[m]) * iy; d[m][2] = (pz[m] - c[m]) * iz;
                }
                for (int a = 0; a < 3; ++a) d[5][a] = -(d[0][a] + d[3][a]);
                double g2 = 0.0;
                for (int a = 0; a < 3; ++a)
                    g2 += d[0][a] * d[0][a] + d[3][a] * d[3][a] + d[5][a] * d[5][a];
                double g2o = 0.0;
                for (int a = 0; a < 3; ++a) g2o += d[1][a] * d[1][a] + d[2][a] * d[2][a] + d[4][a] * d[4][a];
                g2 += 2.0 * g2o;
                gi += g2 * cv;
                ee += 0.5 * p->kappa * g2 * cv;
                qi += trQ2 * cv;
                const NF f = nematic(c, 1e-12, NF{0.0, 1.0, 0.0, 0.0});
                nf[id] = f;
                Ss += f.S;
                Sm = std::max(Sm, f.S);
            }
    long long used = 0, defects = 0;
    double line = 0.0;
#pragma omp parallel for collapse(2) reduction(+ : used, defects, line)
    for (int z = 0; z < Nz; ++z)
        for (int y = 0; y < Ny; ++y)
            for (int x = 0; x < Nx; ++x) {
                const int xp = (x + 1) % Nx, yp = (y + 1) % Ny, zp = (z + 1) % Nz;
                const NF& f000 = nf[fl(x, y, z)];
                const NF& f100 = nf[fl(xp, y, z)];
                const NF& f110 = nf[fl(xp, yp, z)];
                const NF& f010 = nf[fl(x, yp, z)];
                const NF& f001 = nf[fl(x, y, zp)];
                const NF& f101 = nf[fl(xp, y, zp)];
                const NF& f011 = nf[fl(x, yp, zp)];
                const double thr = p->defects_S_threshold, cut = p->defects_charge_cutoff;
                int r = plaquette(f000, f100, f110, f010, 0, thr, cut);
                if (r) { ++used; if (r == 2) { ++defects; line += p->dz; } }
                r = plaquette(f000, f010, f011, f001, 1, thr, cut);
                if (r) { ++used; if (r == 2) { ++defects; line += p->dx; } }
                r = plaquette(f000, f100, f101, f001, 2, thr, cut);
                if (r) { ++used; if (r == 2) { ++defects; line += p->dy; } }
            }
    o->bulk = eb / tv;
    o->elastic = ee / tv;
    o->total = o->bulk + o->elastic;
    o->avg_S = Ss / (double)n;
    o->max_S = Sm;
    o->defect_plaquettes_used = used;
    o->nonzero_defect_plaquettes = defects;
    o->defect_density_per_plaquette = (used > 0) ? (double)defects / (double)used
                                                 : std::numeric_limits<double>::quiet_NaN();
    o->defect_line_density = (tv > 0.0) ? line / tv : std::numeric_limits<double>::quiet_NaN();
    o->xi_grad_proxy = (gi > 0.0 && qi > 0.0) ? std::sqrt(qi / gi) : std::numeric_limits<double>::quiet_NaN();
}

// ---------------------------------------------------------------------------------------
// Philox4x32-R (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11): R rounds of two 32x32->64 multiplies with the published constants (R = 10 is the
// paper's default and has published known answers; the device noise uses R = 7).
// ---------------------------------------------------------------------------------------
extern "C" void orc_philox4x32_rounds(const uint32_t ctr[4], const uint32_t key[2], int rounds, uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < rounds; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        const uint32_t n1 = (uint32_t)p1;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        const uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

extern "C" void orc_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    orc_philox4x32_rounds(ctr, key, 10, out);
}
