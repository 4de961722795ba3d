// kzm_bulk_ldg_b200 -- drop-in host program for `KZM_bulk_ldg_cuda --config <file>`
// (the reference's KZM_bulk_ldg.cu main): same keys, defaults, validation messages, output
// directory layout, quench_log.dat columns (precision 16), snapshot and summary files. The
// step and the observables run on the GPU through the C ABI (include/ldg_b200.h); the
// Langevin noise uses counter-based Philox keyed by (seed, site, iteration) instead of the
// reference's splitmix64 stream, with the same amplitude sqrt(2 (1/gamma) noise_strength dt).
#include <cmath>
#include <filesystem>
#include <iomanip>
#include <iostream>
#include <limits>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "host_common.hpp"
#include "ldg_b200.h"

namespace fs = std::filesystem;
using namespace host;

namespace {

struct Params {
    int Nx = 64, Ny = 64, Nz = 64;
    double dx = 1e-9, dy = 1e-9, dz = 1e-9;
    double a = 0.044e6, b = 1.413e6, c = 1.153e6, T_star = 308.0;
    int bulk_modechoice = 1;
    double kappa = 6.5e-12, gamma = 0.01;
    double T_high = 315.0, T_low = 290.0, Tc_KZ = 310.2;
    int pre_equil_iters = 200, ramp_iters = 300, total_iters = 1200;
    double dt = 1e-11, init_noise_amplitude = 1e-4, noise_strength = 0.0;
    double defects_S_threshold = 0.1, defects_charge_cutoff = 0.25, q_norm_cap = 0.0;
    long long random_seed = 12345;
    int logFreq = 10, snapshot_mode = 0, snapshotFreq = 100;
};

void check(int rc, const char* what) {
    if (rc != LDG_OK) throw std::runtime_error(std::string(what) + ": " + ldg_last_error());
}

// compute_temperature (KZM_bulk_ldg.cu:315-328).
double temperature(const Params& p, int it) {
    if (it < p.pre_equil_iters) return p.T_high;
    if (it >= p.pre_equil_iters + p.ramp_iters) return p.T_low;
    if (p.ramp_iters <= 0) return p.T_low;
    const double frac = (double)(it - p.pre_equil_iters) / (double)p.ramp_iters;
    return p.T_high + frac * (p.T_low - p.T_high);
}

// estimate_stable_dt (KZM_bulk_ldg.cu:330-349).
double stable_dt(const Params& p) {
    double Ah, Bh, Ch, Al, Bl, Cl;
    bulk_ABC(p.a, p.b, p.c, p.T_high, p.T_star, p.bulk_modechoice, Ah, Bh, Ch);
    bulk_ABC(p.a, p.b, p.c, p.T_low, p.T_star, p.bulk_modechoice, Al, Bl, Cl);
    const double Sl = S_eq(Al, Bl, Cl);
    const double trq2 = 2.0 * Sl * Sl / 3.0;
    const double nonlin = std::abs(Bl) * std::abs(Sl) + std::abs(Cl) * trq2;
    const double lap = 2.0 * p.kappa * (1.0 / (p.dx * p.dx) + 1.0 / (p.dy * p.dy) + 1.0 / (p.dz * p.dz));
    const double local = std::max(std::abs(Ah), std::abs(Al)) + nonlin;
    const double stiff = (1.0 / p.gamma) * (lap + local);
    if (!(stiff > 0.0)) return std::numeric_limits<double>::quiet_NaN();
    return 0.2 / stiff;
}

// Nematic (S, n) of one site for the snapshot writer (KZM_bulk_ldg.cu:207-258).
void nematic(const double* q, double out[4]) {
    const double Qxx = q[0], Qxy = q[1], Qxz = q[2], Qyy = q[3], Qyz = q[4], Qzz = -Qxx - Qyy;
    if (std::fabs(Qxx) < 1e-12 && std::fabs(Qxy) < 1e-12 && std::fabs(Qxz) < 1e-12 && std::fabs(Qyy) < 1e-12 &&
        std::fabs(Qyz) < 1e-12) {
        out[0] = 0.0; out[1] = 1.0; out[2] = 0.0; out[3] = 0.0;
        return;
    }
    double nx = Qxx + Qxy + Qxz, ny = Qxy + Qyy + Qyz, nz = Qxz + Qyz - Qxx - Qyy;
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
    if (nz < -1e-10) { nx = -nx; ny = -ny; nz = -nz; }
    out[0] = 1.5 * lam; out[1] = nx; out[2] = ny; out[3] = nz;
}

// save_qtensor_field (KZM_bulk_ldg.cu:715-730): precision 16, x fastest, with (S, n).
void save_field(const fs::path& path, const std::vector<double>& q, const Params& p) {
    const long long n = (long long)p.Nx * p.Ny * p.Nz;
    std::ofstream out(path);
    out << "# x y z Qxx Qxy Qxz Qyy Qyz S nx ny nz\n";
    const long long chunk = 1 << 15;
    for (long long base = 0; base < n; base += chunk) {
        std::ostringstream ss;
        ss << std::setprecision(16);
        const long long hi = std::min(n, base + chunk);
        for (long long t = base; t < hi; ++t) {
            const int x = (int)(t % p.Nx);
            const int y = (int)((t / p.Nx) % p.Ny);
            const int z = (int)(t / ((long long)p.Nx * p.Ny));
            const double* c = &q[5 * t];
            double nf[4];
            nematic(c, nf);
            ss << x << ' ' << y << ' ' << z << ' ' << c[0] << ' ' << c[1] << ' ' << c[2] << ' ' << c[3] << ' ' << c[4]
               << ' ' << nf[0] << ' ' << nf[1] << ' ' << nf[2] << ' ' << nf[3] << '\n';
        }
        out << ss.str();
    }
}

int run(int argc, char** argv) {
    std::string config_path;
    for (int i = 1; i < argc; ++i) {
        const std::string arg = argv[i] ? argv[i] : "";
        if (arg == "--help" || arg == "-h") {
            std::cout << "kzm_bulk_ldg_b200 options:\n  --config <path>       Run non-interactively using key=value config file\n"
                         "  --help                Show this help\n";
            return 0;
        }
        if (arg == "--config" && i + 1 < argc) config_path = argv[++i];
    }
    Config cfg;
    if (!parse_config(config_path, cfg, true)) throw std::runtime_error("Could not open config file: " + config_path);
    Params p;
    p.Nx = get<int>(cfg, "Nx", p.Nx); p.Ny = get<int>(cfg, "Ny", p.Ny); p.Nz = get<int>(cfg, "Nz", p.Nz);
    p.dx = get<double>(cfg, "dx", p.dx); p.dy = get<double>(cfg, "dy", p.dy); p.dz = get<double>(cfg, "dz", p.dz);
    p.a = get<double>(cfg, "a", p.a); p.b = get<double>(cfg, "b", p.b); p.c = get<double>(cfg, "c", p.c);
    p.T_star = get<double>(cfg, "T_star", p.T_star);
    p.bulk_modechoice = get<int>(cfg, "bulk_modechoice", p.bulk_modechoice);
    p.kappa = get<double>(cfg, "kappa", p.kappa); p.gamma = get<double>(cfg, "gamma", p.gamma);
    p.T_high = get<double>(cfg, "T_high", p.T_high); p.T_low = get<double>(cfg, "T_low", p.T_low);
    p.pre_equil_iters = get<int>(cfg, "pre_equil_iters", p.pre_equil_iters);
    p.ramp_iters = get<int>(cfg, "ramp_iters", p.ramp_iters);
    p.total_iters = get<int>(cfg, "total_iters", p.total_iters);
    p.dt = get<double>(cfg, "dt", p.dt);
    p.init_noise_amplitude = get<double>(cfg, "init_noise_amplitude", p.init_noise_amplitude);
    p.noise_strength = get<double>(cfg, "noise_strength", p.noise_strength);
    p.defects_S_threshold = get<double>(cfg, "defects_S_threshold", p.defects_S_threshold);
    p.defects_charge_cutoff = get<double>(cfg, "defects_charge_cutoff", p.defects_charge_cutoff);
    p.q_norm_cap = get<double>(cfg, "q_norm_cap", p.q_norm_cap);
    p.random_seed = get<long long>(cfg, "random_seed", p.random_seed);
    p.logFreq = std::max(1, get<int>(cfg, "logFreq", p.logFreq));
    p.snapshot_mode = std::max(0, get<int>(cfg, "snapshot_mode", p.snapshot_mode));
    p.snapshotFreq = std::max(1, get<int>(cfg, "snapshotFreq", p.snapshotFreq));
    double Ani, Bni, Cni;
    bulk_ABC(p.a, p.b, p.c, p.T_star, p.T_star, p.bulk_modechoice, Ani, Bni, Cni);
    const double T_NI = T_from_A(A_NI(Bni, Cni), p.a, p.T_star);
    p.Tc_KZ = get<double>(cfg, "Tc_KZ", std::isfinite(T_NI) ? T_NI : p.Tc_KZ);
    // Validation (KZM_bulk_ldg.cu:824-841).
    if (p.Nx <= 1 || p.Ny <= 1 || p.Nz <= 1)
        throw std::runtime_error("Nx, Ny, and Nz must all be greater than 1 for the periodic bulk LdG branch");
    if (p.dx <= 0.0 || p.dy <= 0.0 || p.dz <= 0.0) throw std::runtime_error("dx, dy, and dz must be positive");
    if (p.dt <= 0.0) throw std::runtime_error("dt must be positive");
    if (!(p.gamma > 0.0)) throw std::runtime_error("gamma must be positive");
    if (!(p.kappa >= 0.0)) throw std::runtime_error("kappa must be non-negative");
    if (p.total_iters < p.pre_equil_iters + p.ramp_iters)
        throw std::runtime_error("total_iters must be at least pre_equil_iters + ramp_iters");
    const fs::path out_dir = fs::absolute(trim(get_string(cfg, "out_dir", "output_kzm_bulk_ldg")));
    const bool overwrite = get<bool>(cfg, "overwrite_out_dir", true);
    if (fs::exists(out_dir)) {
        if (!overwrite) throw std::runtime_error("Output directory exists and overwrite_out_dir=false: " + out_dir.string());
        fs::remove_all(out_dir);
    }
    fs::create_directories(out_dir);
    double Al, Bl, Cl;
    bulk_ABC(p.a, p.b, p.c, p.T_low, p.T_star, p.bulk_modechoice, Al, Bl, Cl);
    const double S_eq_low = S_eq(Al, Bl, Cl);
    const double dt_limit = stable_dt(p);
    std::cout << "KZM bulk intermediate branch (3D periodic bulk Landau-de Gennes, B200)\n";
    std::cout << "Grid: " << p.Nx << "x" << p.Ny << "x" << p.Nz << '\n';
    std::cout << "T_high=" << p.T_high << ", T_low=" << p.T_low << ", Tc_KZ=" << p.Tc_KZ;
    if (std::isfinite(T_NI)) std::cout << " (T_NI estimate ~ " << T_NI << ")";
    std::cout << "\ndt=" << p.dt;
    if (std::isfinite(dt_limit)) {
        std::cout << " (rough explicit limit ~ " << dt_limit << ")";
        if (p.dt > dt_limit) std::cout << " [warning: dt exceeds the rough explicit limit]";
    }
    std::cout << '\n';
    unsigned long long seed = 0ull;
    if (p.random_seed < 0) {
        std::random_device rd;
        seed = ((unsigned long long)rd() << 32) ^ (unsigned long long)rd();
    } else {
        seed = (unsigned long long)p.random_seed;
    }
    std::cout << "random_seed=" << seed << '\n';
    // Initial field (KZM_bulk_ldg.cu:874-893).
    const long long n = (long long)p.Nx * p.Ny * p.Nz;
    std::vector<double> field((size_t)(5 * n));
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> gauss(0.0, 1.0);
    for (long long t = 0; t < n; ++t)
        for (int m = 0; m < 5; ++m) field[5 * t + m] = p.init_noise_amplitude * gauss(rng);
    kzm_params kp{p.Nx, p.Ny, p.Nz, p.dx, p.dy, p.dz, p.kappa, p.gamma, p.q_norm_cap, p.defects_S_threshold,
                  p.defects_charge_cutoff};
    kzm_handle* h = nullptr;
    check(kzm_create(&kp, &h), "kzm_create");
    struct Guard { kzm_handle* h; ~Guard() { kzm_destroy(h); } } guard{h};
    check(kzm_upload(h, field.data()), "kzm_upload");
    std::ofstream qlog(out_dir / "quench_log.dat");
    qlog << std::setprecision(16);
    qlog << "iteration,time_s,T_K,dt_s,bulk,elastic,anchoring,total,radiality,avg_S,max_S,"
         << "defect_density_per_plaquette,defect_plaquettes_used,xi_grad_proxy,defect_line_density\n";
    auto should_log = [&](int it) { return it == 0 || it == p.total_iters || (it % p.logFreq == 0); };
    auto should_snap = [&](int it) { return p.snapshot_mode > 0 && (it == p.total_iters || it % p.snapshotFreq == 0); };
    kzm_observables fin{};
    for (int it = 0; it <= p.total_iters; ++it) {
        const double Tc = temperature(p, it);
        double A, B, C;
        bulk_ABC(p.a, p.b, p.c, Tc, p.T_star, p.bulk_modechoice, A, B, C);
        if (should_log(it) || should_snap(it)) {
            check(kzm_observe(h, A, B, C, &fin), "kzm_observe");
            if (should_log(it)) {
                qlog << it << ',' << p.dt * (double)it << ',' << Tc << ',' << p.dt << ',' << fin.bulk << ','
                     << fin.elastic << ',' << 0.0 << ',' << fin.total << ',' << std::numeric_limits<double>::quiet_NaN()
                     << ',' << fin.avg_S << ',' << fin.max_S << ',' << fin.defect_density_per_plaquette << ','
                     << fin.defect_plaquettes_used << ',' << fin.xi_grad_proxy << ',' << fin.defect_line_density << '\n';
            }
            if (should_snap(it)) {
                check(kzm_download(h, field.data()), "kzm_download");
                std::ostringstream name;
                name << "q_tensor_iter_" << std::setw(6) << std::setfill('0') << it << ".dat";
                save_field(out_dir / name.str(), field, p);
            }
        }
        if (it == p.total_iters) break;
        const double sigma = (p.noise_strength > 0.0) ? std::sqrt(2.0 * (1.0 / p.gamma) * p.noise_strength * p.dt) : 0.0;
        kzm_step_args sa{A, B, C, p.dt, sigma, seed, (long long)it};
        check(kzm_step(h, 1, &sa), "kzm_step");
    }
    check(kzm_download(h, field.data()), "kzm_download");
    save_field(out_dir / "q_tensor_final.dat", field, p);
    std::ofstream s(out_dir / "run_summary.txt");
    s << std::setprecision(16);
    s << "Nx=" << p.Nx << "\nNy=" << p.Ny << "\nNz=" << p.Nz << "\ndt=" << p.dt << "\ndt_limit_estimate=" << dt_limit
      << "\nT_high=" << p.T_high << "\nT_low=" << p.T_low << "\nTc_KZ=" << p.Tc_KZ << "\nT_NI_estimate=" << T_NI
      << "\nS_eq_low=" << S_eq_low << "\nbulk_modechoice=" << p.bulk_modechoice
      << "\ndefects_S_threshold=" << p.defects_S_threshold << "\ndefects_charge_cutoff=" << p.defects_charge_cutoff
      << "\npre_equil_iters=" << p.pre_equil_iters << "\nramp_iters=" << p.ramp_iters
      << "\ntotal_iters=" << p.total_iters << "\nfinal_avg_S=" << fin.avg_S << "\nfinal_max_S=" << fin.max_S
      << "\nfinal_defect_density_per_plaquette=" << fin.defect_density_per_plaquette
      << "\nfinal_defect_line_density=" << fin.defect_line_density << "\nfinal_xi_grad_proxy=" << fin.xi_grad_proxy
      << '\n';
    std::cout << "Final avg_S=" << fin.avg_S << ", defect_line_density=" << fin.defect_line_density
              << ", xi_grad_proxy=" << fin.xi_grad_proxy << '\n';
    std::cout << "Output directory: " << out_dir << '\n';
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        return run(argc, argv);
    } catch (const std::exception& e) {
        std::cerr << "KZM_bulk_ldg_cuda ERROR: " << e.what() << std::endl;
        return 1;
    }
}
