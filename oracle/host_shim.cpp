// Plain-pointer exports of the drop-in host programs' step scalars -- TEST INFRASTRUCTURE ONLY.
//
// Compiles the product's lcdrsimulator_b200/host/host_common.hpp (the restatement the qsr_b200
// host program calls) so that tests can compare it number for number with the reference's own
// estimate_stable_dt_window and resolve_boundary_shell_order (QSR.cu:1475-1487, 1528-1604),
// which oracle/ref_cuda_harness.cu exports from the reference build.
#include "host_common.hpp"

#include <algorithm>
#include <string>
#include <vector>

extern "C" {

// Same argument and output order as qref_dt_window in ref_cuda_harness.cu.
void hshim_dt_window(const double* req, double* out) {
    const host::DtResult e = host::estimate_dt(req[0], req[1], req[2], req[3], req[4], req[5], req[6], req[7],
                                               (int)req[8], req[9], req[10], req[11], req[12], req[13], req[14],
                                               req[15], req[16], req[17] != 0.0, req[18], (int)req[19]);
    const double v[11] = {e.min_dx, e.S_scale, e.L_eff_total, e.D_total, e.dt_diff_total, e.L_eff_explicit,
                          e.dt_diff, e.bulk_rate, e.dt_bulk, e.dt_max, e.semi_implicit_active ? 1.0 : 0.0};
    for (int n = 0; n < 11; ++n) out[n] = v[n];
}

double hshim_shell_order(int custom, double custom_S, double a, double b, double c, double T, double T_star,
                         int modechoice) {
    return host::resolve_shell_order(custom != 0, custom_S, a, b, c, T, T_star, modechoice);
}

// The host programs' writers (host_common.hpp) and the warm-start reader, on a caller's field.
int hshim_save_qtensor(const double* q, int Nx, int Ny, int Nz, const char* path) {
    const std::vector<double> v(q, q + 5 * (size_t)Nx * Ny * Nz);
    return host::save_qtensor(v, Nx, Ny, Nz, path) ? 0 : 1;
}

int hshim_save_nematic(const double* s_n4, int Nx, int Ny, int Nz, const char* path) {
    const std::vector<double> v(s_n4, s_n4 + 4 * (size_t)Nx * Ny * Nz);
    return host::save_nematic(v, Nx, Ny, Nz, path) ? 0 : 1;
}

// out3: the file's largest |trace| and |asymmetry| and the largest |Q| entry.
int hshim_load_qtensor(const char* path, int Nx, int Ny, int Nz, double* q, double* out3) {
    std::vector<double> v;
    std::string err;
    host::QtensorFileCheck chk{};
    if (!host::load_qtensor(path, Nx, Ny, Nz, v, err, &chk)) return 1;
    std::copy(v.begin(), v.end(), q);
    out3[0] = chk.max_trace; out3[1] = chk.max_asymmetry; out3[2] = chk.max_entry;
    return 0;
}

}  // extern "C"
