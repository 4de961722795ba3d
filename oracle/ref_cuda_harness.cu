// Reference FP64 GPU path for whole-run parity pins -- TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own QSR.cu (path given by QSR_REF_SOURCE, from the reference
// tree) into this translation unit with its main() renamed, and drives the reference's
// kernels in the order its time loop launches them (QSR.cu:2708-2753 and 3234-3249),
// with the reference's launch shape. Used only to generate golden fixtures that pin the
// CPU oracle; never linked into the product.
#define main qsr_cuda_reference_main
#include QSR_REF_SOURCE
#undef main

#include <cstring>

namespace {
struct RefState {
    int Nx = 0, Ny = 0, Nz = 0;
    double dx = 0, dy = 0, dz = 0;
    DimensionalParams P{};
    double kappa = 0, gamma = 0.1;
    int modechoice = 1;
    DropletGeometry geom{};
    double delta_eff = 0;
    size_t n = 0;
    QTensor *Q = nullptr, *Qalt = nullptr, *lap = nullptr, *mu = nullptr, *rhs = nullptr;
    bool* shell = nullptr;
    double *Dx = nullptr, *Dy = nullptr, *Dz = nullptr, *eb = nullptr, *ee = nullptr, *ea = nullptr, *rad = nullptr;
    int* cnt = nullptr;
    unsigned *dcount = nullptr, *dplaq = nullptr, *xedges = nullptr;
    double* xsum = nullptr;
    NematicField* nf = nullptr;
    std::vector<unsigned char> h_shell;
} S;

dim3 blk() { return dim3(8, 8, 8); }
dim3 grd() { return dim3((S.Nx + 7) / 8, (S.Ny + 7) / 8, (S.Nz + 7) / 8); }
}  // namespace

extern "C" {

// p: Nx Ny Nz dx dy dz a b c T_star modechoice kappa L1 L2 L3 W gamma radius_cells
int qref_create(const double* p) {
    S.Nx = (int)p[0]; S.Ny = (int)p[1]; S.Nz = (int)p[2];
    S.dx = p[3]; S.dy = p[4]; S.dz = p[5];
    S.P = DimensionalParams{p[6], p[7], p[8], 0.0, p[9], p[12], p[13], p[14], p[15]};
    S.modechoice = (int)p[10];
    S.kappa = p[11];
    if (S.P.L1 != 0 || S.P.L2 != 0 || S.P.L3 != 0) S.kappa = 0.0;  // QSR.cu:2060
    S.gamma = p[16];
    S.geom = makeDropletGeometry(S.Nx, S.Ny, S.Nz, S.dx, S.dy, S.dz);
    if (p[17] > 0.0) {  // optional radius override (not a reference key)
        S.geom.radius_x = std::max(p[17] * S.dx, 0.5 * S.dx);
        S.geom.radius_y = std::max(p[17] * S.dy, 0.5 * S.dy);
        S.geom.radius_z = std::max(p[17] * S.dz, 0.5 * S.dz);
        S.geom.min_radius = std::min({S.geom.radius_x, S.geom.radius_y, S.geom.radius_z});
    }
    if (cudaMemcpyToSymbol(d_droplet_geometry, &S.geom, sizeof(DropletGeometry)) != cudaSuccess) return 1;
    S.n = (size_t)S.Nx * S.Ny * S.Nz;
    S.h_shell.assign(S.n, 0);
    size_t shell_count = 0;
    for (int i = 0; i < S.Nx; ++i)
        for (int j = 0; j < S.Ny; ++j)
            for (int k = 0; k < S.Nz; ++k) {
                const DropletGeometryPoint pt = sampleDropletGeometry(S.geom, i, j, k);
                if (dropletIsInShell(S.geom, pt)) { S.h_shell[k + S.Nz * (j + S.Ny * i)] = 1; ++shell_count; }
            }
    S.delta_eff = estimateShellThicknessFromMask(S.geom, shell_count);
    const size_t qb = S.n * sizeof(QTensor), db = S.n * sizeof(double);
    cudaMalloc(&S.Q, qb); cudaMalloc(&S.Qalt, qb); cudaMalloc(&S.lap, qb); cudaMalloc(&S.mu, qb); cudaMalloc(&S.rhs, qb);
    cudaMalloc(&S.shell, S.n);
    cudaMalloc(&S.Dx, db); cudaMalloc(&S.Dy, db); cudaMalloc(&S.Dz, db);
    cudaMalloc(&S.eb, db); cudaMalloc(&S.ee, db); cudaMalloc(&S.ea, db); cudaMalloc(&S.rad, db);
    cudaMalloc(&S.cnt, S.n * sizeof(int));
    cudaMalloc(&S.dcount, 4); cudaMalloc(&S.dplaq, 4); cudaMalloc(&S.xedges, 4); cudaMalloc(&S.xsum, 8);
    cudaMalloc(&S.nf, S.n * sizeof(NematicField));
    cudaMemcpy(S.shell, S.h_shell.data(), S.n, cudaMemcpyHostToDevice);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

double qref_delta_eff(void) { return S.delta_eff; }

int qref_upload(const double* q) {
    return cudaMemcpy(S.Q, q, S.n * sizeof(QTensor), cudaMemcpyHostToDevice) == cudaSuccess ? 0 : 1;
}

int qref_download(double* q) {
    return cudaMemcpy(q, S.Q, S.n * sizeof(QTensor), cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : 1;
}

}  // extern "C"

namespace {
// The kernels of one step of the reference chain, in its launch order, without a synchronisation.
void launch_step(double T, double S_shell, double dt, double q_norm_cap, int imex, double L_stab, int jacobi_iters) {
    DimensionalParams P = S.P;
    P.T = T;
    const int Nx = S.Nx, Ny = S.Ny, Nz = S.Nz;
    computeLaplacianKernel<<<grd(), blk()>>>(S.Q, S.lap, Nx, Ny, Nz, S.dx, S.dy, S.dz);
    if (P.L2 != 0.0 || P.L3 != 0.0)
        computeDivergenceKernel<<<grd(), blk()>>>(S.Q, S.Dx, S.Dy, S.Dz, Nx, Ny, Nz, S.dx, S.dy, S.dz);
    computeChemicalPotentialKernel<<<grd(), blk()>>>(S.Q, S.mu, S.lap, Nx, Ny, Nz, S.dx, S.dy, S.dz, P, S.kappa,
                                                     S.modechoice, S.Dx, S.Dy, S.Dz);
    if (P.L3 != 0.0)
        computeChemicalPotentialL3Kernel<<<grd(), blk()>>>(S.Q, S.mu, Nx, Ny, Nz, S.dx, S.dy, S.dz, P, S.Dx, S.Dy, S.Dz);
    applyWeakAnchoringPenaltyKernel<<<grd(), blk()>>>(S.mu, S.Q, Nx, Ny, Nz, S.shell, S_shell, P.W, S.delta_eff);
    if (imex && L_stab > 0.0 && jacobi_iters > 0) {
        computeRhsSemiImplicitKernel<<<grd(), blk()>>>(S.Q, S.mu, S.lap, S.rhs, Nx, Ny, Nz, dt, S.gamma, L_stab,
                                                       S.shell, P.W);
        const double alpha = (dt / S.gamma) * L_stab;
        QTensor* qo = S.Q;
        QTensor* qn = S.Qalt;
        for (int it = 0; it < jacobi_iters; ++it) {
            jacobiHelmholtzStepKernel<<<grd(), blk()>>>(S.rhs, qo, qn, Nx, Ny, Nz, alpha, S.dx, S.dy, S.dz, S.shell, P.W);
            std::swap(qo, qn);
        }
        S.Q = qo;
        S.Qalt = qn;
    } else {
        updateQTensorKernel<<<grd(), blk()>>>(S.Q, S.mu, Nx, Ny, Nz, dt, S.shell, S.gamma, P.W, q_norm_cap);
    }
    applyBoundaryConditionsKernel<<<grd(), blk()>>>(S.Q, Nx, Ny, Nz, S.shell, S_shell, P.W);
}
}  // namespace

extern "C" {

// One step of the reference chain. imex != 0 selects the semi-implicit branch (QSR.cu:2721-2749).
int qref_step(double T, double S_shell, double dt, double q_norm_cap, int imex, double L_stab, int jacobi_iters) {
    launch_step(T, S_shell, dt, q_norm_cap, imex, L_stab, jacobi_iters);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}

// n explicit steps of the reference chain back to back (as its time loop launches them between
// log points), timed with CUDA events on the default stream: *ms = elapsed device time.
int qref_time_steps(double T, double S_shell, double dt, int n, float* ms) {
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return 1;
    cudaEventRecord(e0);
    for (int s = 0; s < n; ++s) launch_step(T, S_shell, dt, 0.0, 0, 0.0, 0);
    cudaEventRecord(e1);
    const bool ok = cudaEventSynchronize(e1) == cudaSuccess;
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ok && cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// Observables as the reference's log path computes them (QSR.cu:2323-2410, 2787-2874).
// out: bulk elastic anch radiality avg_S max_S checker_rel defect_density defect_count plaq xi_proxy xi_edges
int qref_observe(double T, double S_shell, int dz_slice, double dS_thr, double d_cut, int xi_slice, double xi_thr,
                 double* out) {
    DimensionalParams P = S.P;
    P.T = T;
    const int Nx = S.Nx, Ny = S.Ny, Nz = S.Nz;
    const size_t n = S.n;
    computeEnergyKernel<<<grd(), blk()>>>(S.Q, S.eb, S.ee, Nx, Ny, Nz, S.dx, S.dy, S.dz, P, S.kappa, S.modechoice);
    computeAnchoringEnergyKernel<<<grd(), blk()>>>(S.Q, S.shell, S.ea, Nx, Ny, Nz, S.dx, S.dy, S.dz, S_shell, P.W,
                                                   S.delta_eff);
    computeRadialityKernel<<<grd(), blk()>>>(S.Q, S.rad, S.cnt, Nx, Ny, Nz);
    std::vector<double> hb(n), he(n), ha(n), hr(n);
    std::vector<int> hc(n);
    cudaMemcpy(hb.data(), S.eb, n * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(he.data(), S.ee, n * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(ha.data(), S.ea, n * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(hr.data(), S.rad, n * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(hc.data(), S.cnt, n * 4, cudaMemcpyDeviceToHost);
    double sb = 0, se = 0, sa = 0, sr = 0;
    long long rc = 0;
    for (size_t i = 0; i < n; ++i) { sb += hb[i]; se += he[i]; sa += ha[i]; sr += hr[i]; rc += hc[i]; }
    out[0] = sb; out[1] = se; out[2] = sa;
    out[3] = (rc > 0) ? sr / rc : 0.0;

    computeNematicFieldKernel<<<grd(), blk()>>>(S.Q, S.nf, Nx, Ny, Nz);
    std::vector<NematicField> nf(n);
    cudaMemcpy(nf.data(), S.nf, n * sizeof(NematicField), cudaMemcpyDeviceToHost);
    const double excl = 2.0 * S.geom.min_spacing;
    double tot = 0, mx = 0;
    long long cnt = 0;
    for (int i = 0; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j)
            for (int k = 0; k < Nz; ++k) {
                const DropletGeometryPoint pt = sampleDropletGeometry(S.geom, i, j, k);
                if (pt.signed_distance < -excl) {
                    const double s = nf[(size_t)k + (size_t)Nz * ((size_t)j + (size_t)Ny * (size_t)i)].S;
                    tot += s; ++cnt;
                    if (std::isfinite(s)) mx = std::max(mx, s);
                }
            }
    out[4] = (cnt > 0) ? tot / cnt : 0.0;
    out[5] = mx;
    double checker = std::numeric_limits<double>::quiet_NaN();
    if (mx >= 0.5) {
        const int kz = std::min(std::max(dz_slice, 0), Nz - 1);
        double es = 0, os = 0, as = 0;
        int en = 0, on = 0, an = 0;
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny; ++j) {
                const DropletGeometryPoint pt = sampleDropletGeometry(S.geom, i, j, kz);
                if (pt.signed_distance >= -excl) continue;
                const double s = nf[(size_t)kz + (size_t)Nz * ((size_t)j + (size_t)Ny * (size_t)i)].S;
                if (!std::isfinite(s) || s <= 0.01) continue;
                as += s; an++;
                if (((i + j) & 1) == 0) { es += s; en++; } else { os += s; on++; }
            }
        if (en > 10 && on > 10 && an > 20 && as != 0.0) checker = std::abs(es - os) / std::abs(as);
    }
    out[6] = checker;

    dim3 t2(16, 16, 1);
    dim3 b2((Nx - 1 + 15) / 16, (Ny - 1 + 15) / 16, 1);
    dim3 bX((Nx - 1 + 15) / 16, (Ny + 15) / 16, 1);
    dim3 bY((Nx + 15) / 16, (Ny - 1 + 15) / 16, 1);
    cudaMemset(S.dcount, 0, 4);
    cudaMemset(S.dplaq, 0, 4);
    computeDefectDensity2DProxyKernel<<<b2, t2>>>(S.Q, Nx, Ny, Nz, dz_slice, dS_thr, d_cut, S.dcount, S.dplaq);
    unsigned dc = 0, dp = 0;
    cudaMemcpy(&dc, S.dcount, 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(&dp, S.dplaq, 4, cudaMemcpyDeviceToHost);
    out[7] = dp > 0 ? double(dc) / double(dp) : std::numeric_limits<double>::quiet_NaN();
    out[8] = dc;
    out[9] = dp;
    cudaMemset(S.xsum, 0, 8);
    cudaMemset(S.xedges, 0, 4);
    computeXiGradEdgesXKernel<<<bX, t2>>>(S.Q, Nx, Ny, Nz, xi_slice, xi_thr, S.xsum, S.xedges);
    computeXiGradEdgesYKernel<<<bY, t2>>>(S.Q, Nx, Ny, Nz, xi_slice, xi_thr, S.xsum, S.xedges);
    double xs = 0;
    unsigned xe = 0;
    cudaMemcpy(&xs, S.xsum, 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(&xe, S.xedges, 4, cudaMemcpyDeviceToHost);
    double xi = std::numeric_limits<double>::quiet_NaN();
    if (xe > 0) {
        const double ms = xs / double(xe);
        const double inv = (ms > 0.0) ? (1.0 / sqrt(ms + 1e-30)) : (1.0 / sqrt(1e-30));
        xi = std::min(inv, 0.5 * double(std::min(Nx, Ny)));
    }
    out[10] = xi;
    out[11] = xe;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}

// ---- host-only wrappers of the reference's step scalars and initialisation (no GPU needed) ----

// estimate_stable_dt_window (QSR.cu:1528-1604). req: dx dy dz gamma a b c T_star modechoice kappa L1 L2
// L3 S_ref_used S0 T_a T_b use_semi_implicit L_stab jacobi_iters. out: min_dx S_scale L_eff_total
// D_total dt_diff_total L_eff_explicit dt_diff bulk_rate dt_bulk dt_max semi_implicit_active.
void qref_dt_window(const double* req, double* out) {
    DtEstimateRequest r;
    r.dx = req[0]; r.dy = req[1]; r.dz = req[2]; r.gamma = req[3];
    r.a = req[4]; r.b = req[5]; r.c = req[6]; r.T_star = req[7]; r.modechoice = (int)req[8];
    r.kappa = req[9]; r.L1 = req[10]; r.L2 = req[11]; r.L3 = req[12];
    r.S_ref_used = req[13]; r.S0 = req[14]; r.T_a = req[15]; r.T_b = req[16];
    r.use_semi_implicit = req[17] != 0.0; r.L_stab = req[18]; r.jacobi_iters = (int)req[19];
    const DtEstimateResult e = estimate_stable_dt_window(r);
    const double v[11] = {e.min_dx, e.S_scale, e.L_eff_total, e.D_total, e.dt_diff_total, e.L_eff_explicit,
                          e.dt_diff, e.bulk_rate, e.dt_bulk, e.dt_max, e.semi_implicit_active ? 1.0 : 0.0};
    std::memcpy(out, v, sizeof(v));
}

// resolve_boundary_shell_order (QSR.cu:1475-1487); custom != 0 selects BoundaryOrderMode::Custom.
double qref_shell_order(int custom, double custom_S, double a, double b, double c, double T, double T_star,
                        int modechoice) {
    return resolve_boundary_shell_order(custom ? BoundaryOrderMode::Custom : BoundaryOrderMode::Equilibrium,
                                        custom_S, a, b, c, T, T_star, modechoice);
}

// initializeQTensor (modes 0, 1) / initializeIsotropicWithNoise (mode 2) (QSR.cu:1841-1904), as main
// dispatches them (QSR.cu:2510-2515), on the reference droplet of an Nx x Ny x Nz grid with the
// optional radius override of qref_create. q: 5 doubles per cell, reference cell order.
void qref_init(int Nx, int Ny, int Nz, double dx, double dy, double dz, double radius_cells, int mode,
               long long seed, double S0, double noise_amplitude, double* q) {
    DropletGeometry g = makeDropletGeometry(Nx, Ny, Nz, dx, dy, dz);
    if (radius_cells > 0.0) {
        g.radius_x = std::max(radius_cells * dx, 0.5 * dx);
        g.radius_y = std::max(radius_cells * dy, 0.5 * dy);
        g.radius_z = std::max(radius_cells * dz, 0.5 * dz);
        g.min_radius = std::min({g.radius_x, g.radius_y, g.radius_z});
    }
    std::vector<QTensor> h;
    if (mode == 2)
        initializeIsotropicWithNoise(h, Nx, Ny, Nz, noise_amplitude, g, seed);
    else
        initializeQTensor(h, Nx, Ny, Nz, S0, mode, g, seed);
    std::memcpy(q, h.data(), h.size() * sizeof(QTensor));
}

// The reference's text writers on a caller's field: saveQTensorToFile (QSR.cu:1818-1832) from 5
// doubles per cell, saveNematicFieldToFile (QSR.cu:1802-1816) from (S, nx, ny, nz) per cell.
void qref_save_qtensor(const double* q, int Nx, int Ny, int Nz, const char* path) {
    std::vector<QTensor> h((size_t)Nx * Ny * Nz);
    std::memcpy(h.data(), q, h.size() * sizeof(QTensor));
    saveQTensorToFile(h, Nx, Ny, Nz, path);
}

void qref_save_nematic(const double* s_n4, int Nx, int Ny, int Nz, const char* path) {
    std::vector<NematicField> h((size_t)Nx * Ny * Nz);
    for (size_t t = 0; t < h.size(); ++t) {
        h[t].S = s_n4[4 * t]; h[t].nx = s_n4[4 * t + 1]; h[t].ny = s_n4[4 * t + 2]; h[t].nz = s_n4[4 * t + 3];
    }
    saveNematicFieldToFile(h, Nx, Ny, Nz, path);
}

void qref_destroy(void) {
    cudaFree(S.Q); cudaFree(S.Qalt); cudaFree(S.lap); cudaFree(S.mu); cudaFree(S.rhs); cudaFree(S.shell);
    cudaFree(S.Dx); cudaFree(S.Dy); cudaFree(S.Dz); cudaFree(S.eb); cudaFree(S.ee); cudaFree(S.ea);
    cudaFree(S.rad); cudaFree(S.cnt); cudaFree(S.dcount); cudaFree(S.dplaq); cudaFree(S.xedges);
    cudaFree(S.xsum); cudaFree(S.nf);
    S = RefState{};
}

}  // extern "C"
