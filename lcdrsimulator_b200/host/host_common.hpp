// Shared pieces of the drop-in host programs: the reference's key=value config semantics,
// physics scalars, and the reference's text writers (same bytes, formatted in parallel).
#pragma once

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <sstream>
#include <string>
#include <thread>
#include <type_traits>
#include <unordered_map>
#include <vector>

namespace host {

inline std::string trim(const std::string& s) {
    size_t b = 0, e = s.size();
    while (b < e && std::isspace((unsigned char)s[b])) ++b;
    while (e > b && std::isspace((unsigned char)s[e - 1])) --e;
    return s.substr(b, e - b);
}

inline std::string lower(std::string s) {
    for (char& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

using Config = std::unordered_map<std::string, std::string>;

// key = value, '#' comments, blank lines ignored, last key wins, lines without '=' skipped
// (QSR.cu:1195-1219). A missing file yields an empty config (QSR.cu:1199-1202) unless strict.
inline bool parse_config(const std::string& path, Config& cfg, bool strict) {
    cfg.clear();
    if (path.empty()) return true;
    std::ifstream f(path);
    if (!f) {
        if (strict) return false;
        std::cerr << "[Config] Could not open config file: " << path << std::endl;
        return true;
    }
    std::string line;
    while (std::getline(f, line)) {
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line = line.substr(0, hash);
        line = trim(line);
        if (line.empty()) continue;
        const size_t eq = line.find('=');
        if (eq == std::string::npos) continue;
        const std::string key = trim(line.substr(0, eq));
        if (key.empty()) continue;
        cfg[key] = trim(line.substr(eq + 1));
    }
    return true;
}

// Typed parse (QSR.cu:1221-1253): bool words, integers via long double + llround with range
// check, everything else via operator>>; any failure returns the default.
template <typename T>
T parse_value(const std::string& s, T def) {
    if (s.empty()) return def;
    if constexpr (std::is_same_v<T, bool>) {
        const std::string v = trim(lower(s));
        if (v == "1" || v == "true" || v == "yes" || v == "y" || v == "on") return true;
        if (v == "0" || v == "false" || v == "no" || v == "n" || v == "off") return false;
        return def;
    } else if constexpr (std::is_integral_v<T>) {
        try {
            size_t idx = 0;
            long double v = std::stold(s, &idx);
            while (idx < s.size() && std::isspace((unsigned char)s[idx])) ++idx;
            if (idx != s.size()) return def;
            long double r = std::llround(v);
            if (r < (long double)std::numeric_limits<T>::min() || r > (long double)std::numeric_limits<T>::max())
                return def;
            return (T)r;
        } catch (...) {
            return def;
        }
    } else {
        std::istringstream iss(s);
        T out;
        if (!(iss >> out)) return def;
        return out;
    }
}

template <typename T>
T get(const Config& cfg, const std::string& key, T def) {
    auto it = cfg.find(key);
    if (it == cfg.end()) return def;
    return parse_value<T>(it->second, def);
}

inline std::string get_string(const Config& cfg, const std::string& key, const std::string& def) {
    auto it = cfg.find(key);
    return it == cfg.end() ? def : it->second;
}

// ---- bulk physics scalars (QSR.cu:1358-1438) ----
inline void bulk_ABC(double a, double b, double c, double T, double Ts, int mode, double& A, double& B, double& C) {
    A = 3.0 * a * (T - Ts);
    if (mode == 1) { B = (9.0 * b) / 2.0; C = (9.0 * c) / 2.0; }
    else { B = (27.0 * b) / 2.0; C = 9.0 * c; }
}

inline double bulk_fS(double A, double B, double C, double S) {
    const double S2 = S * S;
    return (A / 3.0) * S2 - (2.0 * B / 27.0) * (S2 * S) + (C / 9.0) * (S2 * S2);
}

inline double S_eq(double A, double B, double C) {
    if (!(C > 0.0)) return 0.0;
    const double disc = B * B - 24.0 * A * C;
    if (!(disc > 0.0)) return 0.0;
    const double sd = std::sqrt(disc);
    double best_S = 0.0, best_f = 0.0;
    for (double S : {(B - sd) / (4.0 * C), (B + sd) / (4.0 * C)}) {
        if (!(S > 0.0)) continue;
        const double f = bulk_fS(A, B, C, S);
        if (f < best_f) { best_f = f; best_S = S; }
    }
    return best_S;
}

inline double A_NI(double B, double C) { return (C > 0.0) ? (B * B) / (27.0 * C) : std::nan(""); }
inline double A_spinN(double B, double C) { return (C > 0.0) ? (B * B) / (24.0 * C) : std::nan(""); }
inline double T_from_A(double A, double a, double Ts) { return (a > 0.0) ? Ts + A / (3.0 * a) : std::nan(""); }

inline double equilibrium_shell_order(double a, double b, double c, double T, double Ts, int mode) {
    double A, B, C;
    bulk_ABC(a, b, c, T, Ts, mode, A, B, C);
    const double s = S_eq(A, B, C);
    return s > 0.0 ? s : 0.0;
}

// Shell order of a step: the custom value, or the equilibrium order max(S_eq(T), 0)
// (resolve_boundary_shell_order, QSR.cu:1475-1487).
inline double resolve_shell_order(bool custom, double custom_S, double a, double b, double c, double T, double Ts,
                                  int mode) {
    return custom ? custom_S : equilibrium_shell_order(a, b, c, T, Ts, mode);
}

struct DtResult {
    double min_dx, S_scale, L_eff_total, D_total, dt_diff_total, L_eff_explicit, dt_diff, bulk_rate, dt_bulk, dt_max;
    bool semi_implicit_active;
};

// estimate_stable_dt_window (QSR.cu:1528-1604).
inline DtResult estimate_dt(double dx, double dy, double dz, double gamma, double a, double b, double c, double Ts,
                     int mode, double kappa, double L1, double L2, double L3, double S_ref_used, double S0, double Ta,
                     double Tb, bool semi, double L_stab, int jacobi) {
    DtResult o{};
    o.min_dx = std::min({dx, dy, dz});
    o.S_scale = std::isfinite(S_ref_used) ? std::abs(S_ref_used) : std::max(std::abs(S0), 0.5);
    const double sa = std::abs(equilibrium_shell_order(a, b, c, Ta, Ts, mode));
    const double sb = std::abs(equilibrium_shell_order(a, b, c, Tb, Ts, mode));
    if (std::isfinite(sa) && sa > 0.0) o.S_scale = std::max(o.S_scale, sa);
    if (std::isfinite(sb) && sb > 0.0) o.S_scale = std::max(o.S_scale, sb);
    o.S_scale = std::max(o.S_scale, 1.0);
    const bool ldg = (L1 != 0.0 || L2 != 0.0 || L3 != 0.0);
    const bool aniso = (L2 != 0.0 || L3 != 0.0);
    o.L_eff_total = ldg ? std::max({std::abs(L1), std::abs(L2), std::abs(L1 + L2), std::abs(L1 + 2.0 * L2),
                                    std::abs(L3) * o.S_scale})
                        : std::abs(kappa);
    if (!(o.L_eff_total > 0.0)) o.L_eff_total = 1e-12;
    o.D_total = o.L_eff_total / gamma;
    if (!(o.D_total > 0.0) || !std::isfinite(o.D_total)) o.D_total = 1e-12;
    o.dt_diff_total = 0.5 * (o.min_dx * o.min_dx) / (6.0 * o.D_total);
    if (aniso) o.dt_diff_total *= 0.25;
    o.L_eff_explicit = o.L_eff_total;
    o.dt_diff = o.dt_diff_total;
    if (semi && L_stab > 0.0 && jacobi > 0) {
        const double L_base = ldg ? L1 : kappa;
        const double Ls = (L_base >= 0.0) ? L_stab : -L_stab;
        const double L_rem = std::abs(L_base - Ls);
        o.L_eff_explicit = ldg ? std::max({L_rem, std::abs(L2), std::abs(L1 + L2), std::abs(L1 + 2.0 * L2),
                                           std::abs(L3) * o.S_scale})
                               : L_rem;
        if (o.L_eff_explicit > 0.0) {
            o.dt_diff = 0.5 * (o.min_dx * o.min_dx) / (6.0 * (o.L_eff_explicit / gamma));
            if (aniso) o.dt_diff *= 0.25;
        } else {
            o.dt_diff = std::numeric_limits<double>::infinity();
        }
        o.semi_implicit_active = true;
    }
    auto rate = [&](double T) {
        double A, B, C;
        bulk_ABC(a, b, c, T, Ts, mode, A, B, C);
        return std::abs(A) + std::abs(B) * o.S_scale + std::abs(C) * o.S_scale * o.S_scale;
    };
    o.bulk_rate = std::max(rate(Ta), rate(Tb));
    o.dt_bulk = (o.bulk_rate > 0.0) ? (0.02 * gamma / o.bulk_rate) : std::numeric_limits<double>::infinity();
    o.dt_max = std::min(o.dt_diff, o.dt_bulk);
    if (!(o.dt_max > 0.0) || !std::isfinite(o.dt_max)) o.dt_max = o.dt_diff;
    return o;
}

// ---- writers ----

// Formats rows [0, n) with fmt_row(i, buf) -> bytes written, in parallel chunks, and writes
// them in order. Output bytes are identical to a serial fprintf loop.
template <class RowFn>
bool write_rows(const std::string& path, const char* header, long long n, int max_row_bytes, RowFn fmt_row) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return false;
    if (header) std::fputs(header, f);
    const int nthreads = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    const long long chunk = 1 << 16;
    std::vector<std::string> bufs(nthreads);
    for (long long base = 0; base < n; base += chunk * nthreads) {
        std::vector<std::thread> ts;
        for (int t = 0; t < nthreads; ++t) {
            ts.emplace_back([&, t]() {
                const long long lo = base + (long long)t * chunk;
                const long long hi = std::min(n, lo + chunk);
                std::string& s = bufs[t];
                s.clear();
                if (lo >= hi) return;
                s.resize((size_t)(hi - lo) * max_row_bytes);
                size_t pos = 0;
                for (long long r = lo; r < hi; ++r) pos += (size_t)fmt_row(r, &s[pos]);
                s.resize(pos);
            });
        }
        for (auto& th : ts) th.join();
        for (auto& s : bufs)
            if (!s.empty()) std::fwrite(s.data(), 1, s.size(), f);
    }
    std::fclose(f);
    return true;
}

// saveNematicFieldToFile (QSR.cu:1802-1816): header "# i j k S nx ny nz", cell order i, j, k.
inline bool save_nematic(const std::vector<double>& snf, int Nx, int Ny, int Nz, const std::string& path) {
    const long long n = (long long)Nx * Ny * Nz;
    return write_rows(path, "# i j k S nx ny nz\n", n, 160, [&](long long t, char* out) {
        const int k = (int)(t % Nz);
        const int j = (int)((t / Nz) % Ny);
        const int i = (int)(t / ((long long)Ny * Nz));
        const double* v = &snf[4 * t];
        return std::snprintf(out, 160, "%d %d %d %.6e %.6e %.6e %.6e\n", i, j, k, v[0], v[1], v[2], v[3]);
    });
}

// saveQTensorToFile (QSR.cu:1818-1832): 9 full-tensor entries, no header.
inline bool save_qtensor(const std::vector<double>& q, int Nx, int Ny, int Nz, const std::string& path) {
    const long long n = (long long)Nx * Ny * Nz;
    return write_rows(path, nullptr, n, 260, [&](long long t, char* out) {
        const int k = (int)(t % Nz);
        const int j = (int)((t / Nz) % Ny);
        const int i = (int)(t / ((long long)Ny * Nz));
        const double* c = &q[5 * t];
        const double zz = -c[0] - c[3];
        return std::snprintf(out, 260, "%d %d %d %.6e %.6e %.6e %.6e %.6e %.6e %.6e %.6e %.6e\n", i, j, k, c[0], c[1],
                             c[2], c[1], c[3], c[4], c[2], c[4], zz);
    });
}

// The traceless/symmetric check of a warm-start file, in FP64: the largest |Qxx + Qyy + Qzz| and
// |Q_ab - Q_ba| over the file's rows, and its largest |Q_ab|.
struct QtensorFileCheck {
    double max_trace = 0.0, max_asymmetry = 0.0, max_entry = 0.0;
};

// Reader of the Qtensor_output_*.dat format (warm start / resume): fills the 5 independent
// components; returns false on a malformed file or a grid mismatch. With `check`, also measures
// how far the file's 9 entries per row are from a traceless symmetric tensor (the stored field
// keeps Qxx, Qxy, Qxz, Qyy, Qyz; Qzz = -(Qxx + Qyy) and the symmetric entries are implied).
inline bool load_qtensor(const std::string& path, int Nx, int Ny, int Nz, std::vector<double>& q, std::string& err,
                         QtensorFileCheck* check = nullptr) {
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) { err = "cannot open " + path; return false; }
    const long long n = (long long)Nx * Ny * Nz;
    q.assign((size_t)(5 * n), 0.0);
    std::vector<char> seen((size_t)n, 0);
    long long rows = 0;
    char line[512];
    while (std::fgets(line, sizeof(line), f)) {
        if (line[0] == '#' || line[0] == '\n') continue;
        int i, j, k;
        double v[9];
        if (std::sscanf(line, "%d %d %d %lf %lf %lf %lf %lf %lf %lf %lf %lf", &i, &j, &k, &v[0], &v[1], &v[2], &v[3],
                        &v[4], &v[5], &v[6], &v[7], &v[8]) != 12) {
            std::fclose(f);
            err = "malformed row " + std::to_string(rows + 1) + " in " + path;
            return false;
        }
        if (i < 0 || j < 0 || k < 0 || i >= Nx || j >= Ny || k >= Nz) {
            std::fclose(f);
            err = "cell index out of the grid in " + path;
            return false;
        }
        const long long t = (long long)k + (long long)Nz * ((long long)j + (long long)Ny * i);
        double* c = &q[5 * t];
        c[0] = v[0]; c[1] = v[1]; c[2] = v[2]; c[3] = v[4]; c[4] = v[5];
        if (check) {
            check->max_trace = std::max(check->max_trace, std::abs(v[0] + v[4] + v[8]));
            check->max_asymmetry = std::max({check->max_asymmetry, std::abs(v[1] - v[3]), std::abs(v[2] - v[6]),
                                             std::abs(v[5] - v[7])});
            for (double x : v) check->max_entry = std::max(check->max_entry, std::abs(x));
        }
        seen[t] = 1;
        ++rows;
    }
    std::fclose(f);
    if (rows != n) {
        err = "expected " + std::to_string(n) + " rows, read " + std::to_string(rows) + " in " + path;
        return false;
    }
    return true;
}

}  // namespace host
