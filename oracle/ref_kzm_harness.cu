// Reference FP64 GPU path of the periodic bulk solver -- TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's KZM_bulk_ldg.cu (path given by KZM_REF_SOURCE) with its main()
// renamed and exposes its update kernel (KZM_bulk_ldg.cu:351-469) and its host observables
// (KZM_bulk_ldg.cu:543-713) through plain pointers, to generate golden fixtures.
#define main kzm_reference_main
#include KZM_REF_SOURCE
#undef main

#include <cstring>

extern "C" {

// p: Nx Ny Nz dx dy dz kappa gamma dt q_norm_cap defects_S_threshold defects_charge_cutoff
static BulkLdgParams make(const double* p) {
    BulkLdgParams b;
    b.Nx = (int)p[0]; b.Ny = (int)p[1]; b.Nz = (int)p[2];
    b.dx = p[3]; b.dy = p[4]; b.dz = p[5];
    b.kappa = p[6]; b.gamma = p[7]; b.dt = p[8]; b.q_norm_cap = p[9];
    b.defects_S_threshold = p[10]; b.defects_charge_cutoff = p[11];
    return b;
}

// Runs n_steps reference updates at fixed (A, B, C) starting at iteration iter0.
int kref_run(const double* p, const double* q_in, double* q_out, int n_steps, double A, double B, double C,
             double noise_sigma, unsigned long long seed, int iter0) {
    const BulkLdgParams b = make(p);
    const size_t n = (size_t)b.Nx * b.Ny * b.Nz;
    QTensor *cur = nullptr, *nxt = nullptr;
    if (cudaMalloc(&cur, n * sizeof(QTensor)) != cudaSuccess) return 1;
    if (cudaMalloc(&nxt, n * sizeof(QTensor)) != cudaSuccess) { cudaFree(cur); return 1; }
    cudaMemcpy(cur, q_in, n * sizeof(QTensor), cudaMemcpyHostToDevice);
    const int bs = 256;
    const int gs = (int)((n + bs - 1) / bs);
    for (int s = 0; s < n_steps; ++s) {
        updateBulkLdgKernel<<<gs, bs>>>(cur, nxt, b, A, B, C, noise_sigma, seed, iter0 + s);
        std::swap(cur, nxt);
    }
    cudaError_t e = cudaMemcpy(q_out, cur, n * sizeof(QTensor), cudaMemcpyDeviceToHost);
    cudaFree(cur);
    cudaFree(nxt);
    return e == cudaSuccess ? 0 : 1;
}

// Device time (*ms) of n_steps reference updates launched back to back after n_warm untimed
// ones, with CUDA events on the default stream (the reference's time loop, KZM_bulk_ldg.cu:951-970).
int kref_time(const double* p, const double* q_in, int n_warm, int n_steps, double A, double B, double C,
              double noise_sigma, unsigned long long seed, float* ms) {
    const BulkLdgParams b = make(p);
    const size_t n = (size_t)b.Nx * b.Ny * b.Nz;
    QTensor *cur = nullptr, *nxt = nullptr;
    if (cudaMalloc(&cur, n * sizeof(QTensor)) != cudaSuccess) return 1;
    if (cudaMalloc(&nxt, n * sizeof(QTensor)) != cudaSuccess) { cudaFree(cur); return 1; }
    cudaMemcpy(cur, q_in, n * sizeof(QTensor), cudaMemcpyHostToDevice);
    const int bs = 256;
    const int gs = (int)((n + bs - 1) / bs);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int s = 0; s < n_warm + n_steps; ++s) {
        if (s == n_warm) cudaEventRecord(e0);
        updateBulkLdgKernel<<<gs, bs>>>(cur, nxt, b, A, B, C, noise_sigma, seed, s);
        std::swap(cur, nxt);
    }
    cudaEventRecord(e1);
    const bool ok = cudaEventSynchronize(e1) == cudaSuccess && cudaGetLastError() == cudaSuccess;
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(cur);
    cudaFree(nxt);
    return ok ? 0 : 2;
}

// The reference's quench loop (KZM_bulk_ldg.cu:917-970) from iteration 0 to total_iters:
// temperature compute_temperature(iter) (pre_equil_iters at T_high, linear ramp over ramp_iters,
// then T_low), bulk coefficients bulk_ABC_from_convention, noise_sigma from noise_strength, one
// updateBulkLdgKernel per iteration with the run's seed. r: a b c T_star modechoice T_high
// T_low pre_equil_iters ramp_iters total_iters noise_strength. Returns the final field and
// the (A, B, C) of the last iteration in abc_out.
int kref_quench(const double* p, const double* r, const double* q_in, double* q_out, unsigned long long seed,
                double* abc_out) {
    BulkLdgParams b = make(p);
    b.a = r[0]; b.b = r[1]; b.c = r[2]; b.T_star = r[3]; b.bulk_modechoice = (int)r[4];
    b.T_high = r[5]; b.T_low = r[6]; b.pre_equil_iters = (int)r[7]; b.ramp_iters = (int)r[8];
    b.total_iters = (int)r[9]; b.noise_strength = r[10];
    const size_t n = (size_t)b.Nx * b.Ny * b.Nz;
    QTensor *cur = nullptr, *nxt = nullptr;
    if (cudaMalloc(&cur, n * sizeof(QTensor)) != cudaSuccess) return 1;
    if (cudaMalloc(&nxt, n * sizeof(QTensor)) != cudaSuccess) { cudaFree(cur); return 1; }
    cudaMemcpy(cur, q_in, n * sizeof(QTensor), cudaMemcpyHostToDevice);
    const int bs = 256;
    const int gs = (int)((n + bs - 1) / bs);
    const double noise_sigma = (b.noise_strength > 0.0) ? std::sqrt(2.0 * (1.0 / b.gamma) * b.noise_strength * b.dt)
                                                        : 0.0;
    double A = 0.0, B = 0.0, C = 0.0;
    for (int iter = 0; iter <= b.total_iters; ++iter) {
        const double T = compute_temperature(b, iter);
        bulk_ABC_from_convention(b.a, b.b, b.c, T, b.T_star, b.bulk_modechoice, A, B, C);
        if (iter == b.total_iters) break;
        updateBulkLdgKernel<<<gs, bs>>>(cur, nxt, b, A, B, C, noise_sigma, seed, iter);
        std::swap(cur, nxt);
    }
    abc_out[0] = A; abc_out[1] = B; abc_out[2] = C;
    cudaError_t e = cudaMemcpy(q_out, cur, n * sizeof(QTensor), cudaMemcpyDeviceToHost);
    cudaFree(cur);
    cudaFree(nxt);
    return e == cudaSuccess ? 0 : 1;
}

// out: bulk elastic total avg_S max_S defect_density line_density xi plaquettes_used defects
void kref_observe(const double* p, const double* q, double A, double B, double C, double* out) {
    const BulkLdgParams b = make(p);
    const size_t n = (size_t)b.Nx * b.Ny * b.Nz;
    std::vector<QTensor> f(n);
    std::memcpy(f.data(), q, n * sizeof(QTensor));
    const BulkLdgObservables o = compute_observables(f, b, A, B, C);
    out[0] = o.bulk; out[1] = o.elastic; out[2] = o.total; out[3] = o.avg_S; out[4] = o.max_S;
    out[5] = o.defect_density_per_plaquette; out[6] = o.defect_line_density; out[7] = o.xi_grad_proxy;
    out[8] = (double)o.defect_plaquettes_used; out[9] = (double)o.nonzero_defect_plaquettes;
}

}  // extern "C"
