// Confined droplet solver: device kernels and the qsr_* C ABI (include/ldg_b200.h).
//
// Device layout: two FP32 SoA field buffers (ping-pong), one uint8 classification per cell,
// an FP32 SoA right-hand side for the IMEX path, and an FP64 AoS staging buffer for the
// host boundary. One fused kernel per explicit step reads each Q component once per cell
// and writes it once (the reference runs 5-7 separate FP64 AoS passes).
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <new>
#include <random>
#include <vector>

#include "ldg_api_common.h"
#include "ldg_common.cuh"
#include "qsr_tiled.cuh"

using namespace ldg;

namespace {

constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------------------
// Host FP64 geometry: the reference's droplet (QSR.cu:34-185), evaluated once per handle.
// ---------------------------------------------------------------------------------------
struct Geometry {
    double dx, dy, dz, cx, cy, cz, rx, ry, rz, min_spacing, min_radius, shell_half, core_radius;
};

Geometry make_geometry(const qsr_params& p) {
    Geometry g{};
    g.dx = p.dx; g.dy = p.dy; g.dz = p.dz;
    g.cx = 0.5 * ((double)p.Nx - 1.0) * p.dx;
    g.cy = 0.5 * ((double)p.Ny - 1.0) * p.dy;
    g.cz = 0.5 * ((double)p.Nz - 1.0) * p.dz;
    double ridx = 0.5 * ((double)std::min({p.Nx, p.Ny, p.Nz}) - 1.0);
    if (p.droplet_radius_cells > 0.0) ridx = p.droplet_radius_cells;
    g.rx = std::max(ridx * p.dx, 0.5 * p.dx);
    g.ry = std::max(ridx * p.dy, 0.5 * p.dy);
    g.rz = std::max(ridx * p.dz, 0.5 * p.dz);
    g.min_spacing = std::min({p.dx, p.dy, p.dz});
    g.min_radius = std::min({g.rx, g.ry, g.rz});
    g.shell_half = g.min_spacing;
    g.core_radius = g.min_spacing;
    return g;
}

// Signed distance proxy (rho - 1)/|grad rho| and distance from the centre (QSR.cu:70-98).
inline void signed_distance(const Geometry& g, int i, int j, int k, double& sd, double& r) {
    const double x = i * g.dx - g.cx, y = j * g.dy - g.cy, z = k * g.dz - g.cz;
    r = std::sqrt(x * x + y * y + z * z);
    const double sx = x / g.rx, sy = y / g.ry, sz = z / g.rz;
    const double rho_sq = sx * sx + sy * sy + sz * sz;
    if (rho_sq <= 1e-30) { sd = -g.min_radius; return; }
    const double rho = std::sqrt(rho_sq);
    const double gx = x / (g.rx * g.rx), gy = y / (g.ry * g.ry), gz = z / (g.rz * g.rz);
    const double gn = std::sqrt(gx * gx + gy * gy + gz * gz) / rho;
    sd = (gn > 1e-30) ? (rho - 1.0) / gn : r - g.min_radius;
}

// ---------------------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------------------

// Global-memory neighbour accessor for the direct kernels.
struct GAcc {
    const float* __restrict__ q;
    long long id, si, sc;
    int sj;
    __device__ __forceinline__ float operator()(int c, int di, int dj, int dk) const {
        const long long o = id + di * si + (long long)dj * sj + dk;
        if (c < 5) return __ldg(q + c * sc + o);
        return -(__ldg(q + o) + __ldg(q + 3 * sc + o));
    }
};

// Column divergence computed on the fly from the Q accessor (v1 path).
struct GDAcc {
    const GAcc* A;
    const QsrConst* P;
    int i, j, k;
    __device__ __forceinline__ float operator()(int comp, int di, int dj, int dk) const {
        float D[3];
        dcol_at(*A, *P, i, j, k, di, dj, dk, D);
        return D[comp];
    }
};

// One explicit step (RHS=false) or the IMEX right-hand side (RHS=true) for every cell of
// the box. Block (32, 8): k fastest, then j; grid z runs over i.
template <bool kL2, bool kL3, bool kNoise, bool kRHS>
__global__ void __launch_bounds__(256) k_step_direct(const float* __restrict__ q, float* __restrict__ out,
                                                     const uint8_t* __restrict__ flags, QsrConst P) {
    const int k = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 8 + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= P.Nz || j >= P.Ny) return;
    const long long id = (long long)i * P.si + (long long)j * P.sj + k;
    const uint8_t f = flags[id];
    float c[5], o[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) c[m] = __ldg(q + m * P.sc + id);
    if (!kRHS && (f & kFixed)) {
        surface_q0(P, i, j, k, o);
    } else if (f & kMove) {
        GAcc A{q, id, P.si, P.sc, P.sj};
        GDAcc DA{&A, &P, i, j, k};
        float mu[5], lap[5];
        chem_potential<kL2, kL3>(A, DA, P, i, j, k, c, (f & kAnchor) != 0, mu, lap);
        const uint32_t cell = (uint32_t)(k + P.Nz * (j + P.Ny * i));
        if (kRHS) {
            // computeRhsSemiImplicitKernel (QSR.cu:775-783).
#pragma unroll
            for (int m = 0; m < 5; ++m) o[m] = c[m] - P.mob_dt * mu[m] - P.alpha * lap[m];
            if (kNoise) {
                float g[5];
                normals5(cell, P.instance, P.step, P.key0, P.key1, g);
#pragma unroll
                for (int m = 0; m < 5; ++m) o[m] += P.sigma * g[m];
            }
        } else {
            euler_update(P, c, mu, cell, kNoise, o);
        }
    } else {
#pragma unroll
        for (int m = 0; m < 5; ++m) o[m] = c[m];
    }
#pragma unroll
    for (int m = 0; m < 5; ++m) out[m * P.sc + id] = o[m];
}

// One Jacobi sweep of (I - alpha Lap) Q = rhs with faces and non-moving cells held
// (QSR.cu:786-849). LAST also applies the strong-anchoring rewrite (QSR.cu:851-867).
template <bool kLast>
__global__ void __launch_bounds__(256) k_jacobi(const float* __restrict__ rhs, const float* __restrict__ qo,
                                                float* __restrict__ qn, const uint8_t* __restrict__ flags, QsrConst P) {
    const int k = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 8 + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= P.Nz || j >= P.Ny) return;
    const long long id = (long long)i * P.si + (long long)j * P.sj + k;
    const uint8_t f = flags[id];
    float o[5];
    if (kLast && (f & kFixed)) {
        surface_q0(P, i, j, k, o);
    } else {
        const bool face = (i == 0 || j == 0 || k == 0 || i == P.Nx - 1 || j == P.Ny - 1 || k == P.Nz - 1);
        if (face || !(f & kMove)) {
#pragma unroll
            for (int m = 0; m < 5; ++m) o[m] = __ldg(qo + m * P.sc + id);
        } else {
#pragma unroll
            for (int m = 0; m < 5; ++m) {
                const float* b = qo + m * P.sc + id;
                const float s = P.ix2 * (__ldg(b + P.si) + __ldg(b - P.si)) +
                                P.iy2 * (__ldg(b + P.sj) + __ldg(b - P.sj)) + P.iz2 * (__ldg(b + 1) + __ldg(b - 1));
                o[m] = (__ldg(rhs + m * P.sc + id) + P.alpha * s) * P.jdenom_inv;
            }
        }
    }
#pragma unroll
    for (int m = 0; m < 5; ++m) qn[m * P.sc + id] = o[m];
}

// The same sweep over the tiles of the explicit step's work list only (tiles holding moving or
// strongly anchored cells, each over its plane range), writing only moving and strongly anchored
// cells. Every other cell never changes: it holds the same value in both ping-pong buffers, so
// the reference's copy of it (QSR.cu:803-810) is already done. One block of 128 threads per
// visited tile plane (the work list expanded to single planes); each thread updates two
// neighbouring cells (k and k + 1, k even): the centre, i +- 1 and j +- 1 operands and the
// right-hand side of both cells are 8-byte loads, the k-neighbours two 4-byte loads. Each cell's
// arithmetic is the full-box sweep's, operand for operand.
template <bool kLast>
__global__ void __launch_bounds__(128) k_jacobi_tiled(const float* __restrict__ rhs, const float* __restrict__ qo,
                                                       float* __restrict__ qn, const uint8_t* __restrict__ flags,
                                                       const int4* __restrict__ items, QsrConst P) {
    const int4 item = items[blockIdx.x];
    const int i = item.z;
    const int k = item.y + 2 * (int)(threadIdx.x & 15);  // even (tiles start at k0 = 2 mod 4)
    const int j = item.x + (int)(threadIdx.x >> 4);
    if (k < 0 || k >= P.Nz || j >= P.Ny) return;  // the first tile of a row may start at k = -2
    const long long id = (long long)i * P.si + (long long)j * P.sj + k;
    const bool has1 = k + 1 < P.Nz;
    const unsigned f2 = *reinterpret_cast<const unsigned short*>(flags + id);  // both cells' classes
    const uint8_t f[2] = {(uint8_t)(f2 & 0xffu), has1 ? (uint8_t)(f2 >> 8) : (uint8_t)0};
    bool wr[2], st[2];
    const bool ij_face = (j == 0 || j == P.Ny - 1 || i == 0 || i == P.Nx - 1);
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        wr[r] = (f[r] & (kMove | kFixed)) != 0;
        const bool k_face = (k + r == 0) || (k + r == P.Nz - 1);
        st[r] = wr[r] && !(kLast && (f[r] & kFixed)) && (f[r] & kMove) && !ij_face && !k_face;
    }
    if (!wr[0] && !wr[1]) return;
    float o[2][5];
#pragma unroll
    for (int m = 0; m < 5; ++m) {
        const float* b = qo + m * P.sc + id;
        const float2 c = *reinterpret_cast<const float2*>(b);
        o[0][m] = c.x;
        o[1][m] = c.y;
        if (st[0] || st[1]) {  // i and j are interior here (ij_face is false)
            const float2 xp = __ldg(reinterpret_cast<const float2*>(b + P.si));
            const float2 xm = __ldg(reinterpret_cast<const float2*>(b - P.si));
            const float2 yp = __ldg(reinterpret_cast<const float2*>(b + P.sj));
            const float2 ym = __ldg(reinterpret_cast<const float2*>(b - P.sj));
            const float km1 = k >= 1 ? __ldg(b - 1) : 0.0f;
            const float kp2 = k + 2 < P.Nz ? __ldg(b + 2) : 0.0f;
            const float2 rh = __ldg(reinterpret_cast<const float2*>(rhs + m * P.sc + id));
            const float s0 = P.ix2 * (xp.x + xm.x) + P.iy2 * (yp.x + ym.x) + P.iz2 * (c.y + km1);
            const float s1 = P.ix2 * (xp.y + xm.y) + P.iy2 * (yp.y + ym.y) + P.iz2 * (kp2 + c.x);
            if (st[0]) o[0][m] = (rh.x + P.alpha * s0) * P.jdenom_inv;
            if (st[1]) o[1][m] = (rh.y + P.alpha * s1) * P.jdenom_inv;
        }
    }
#pragma unroll
    for (int r = 0; r < 2; ++r)
        if (kLast && wr[r] && (f[r] & kFixed)) surface_q0(P, i, j, k + r, o[r]);
    if (wr[0] && wr[1]) {
#pragma unroll
        for (int m = 0; m < 5; ++m) *reinterpret_cast<float2*>(qn + m * P.sc + id) = make_float2(o[0][m], o[1][m]);
    } else {
#pragma unroll
        for (int r = 0; r < 2; ++r)
            if (wr[r]) {
#pragma unroll
                for (int m = 0; m < 5; ++m) qn[m * P.sc + id + r] = o[r][m];
            }
    }
}

// Host AoS FP64 (reference cell order) <-> device FP32 SoA.
__global__ void k_aos_to_soa(const double* __restrict__ aos, float* __restrict__ a, float* __restrict__ b,
                             int Nx, int Ny, int Nz, int sj, long long si, long long sc, float* __restrict__ la = nullptr,
                             float* __restrict__ lb = nullptr) {
    const long long n = (long long)Nx * Ny * Nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % Nz);
        const long long r = t / Nz;
        const int j = (int)(r % Ny);
        const int i = (int)(r / Ny);
        const long long id = (long long)i * si + (long long)j * sj + k;
#pragma unroll
        for (int m = 0; m < 5; ++m) {
            const double x = aos[5 * t + m];
            const float v = (float)x;
            a[m * sc + id] = v;
            b[m * sc + id] = v;
            if (la) {
                const float r = (float)(x - (double)v);  // low word of compensated storage
                la[m * sc + id] = r;
                lb[m * sc + id] = r;
            }
        }
    }
}

__global__ void k_soa_to_aos(const float* __restrict__ a, double* __restrict__ aos, int Nx, int Ny, int Nz, int sj,
                             long long si, long long sc, const float* __restrict__ lo = nullptr) {
    const long long n = (long long)Nx * Ny * Nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % Nz);
        const long long r = t / Nz;
        const int j = (int)(r % Ny);
        const int i = (int)(r / Ny);
        const long long id = (long long)i * si + (long long)j * sj + k;
#pragma unroll
        for (int m = 0; m < 5; ++m)
            aos[5 * t + m] = (double)a[m * sc + id] + (lo ? (double)lo[m * sc + id] : 0.0);
    }
}

__global__ void k_nematic_out(const float* __restrict__ a, double* __restrict__ out4, int Nx, int Ny, int Nz, int sj,
                              long long si, long long sc) {
    const long long n = (long long)Nx * Ny * Nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % Nz);
        const long long r = t / Nz;
        const int j = (int)(r % Ny);
        const int i = (int)(r / Ny);
        const long long id = (long long)i * si + (long long)j * sj + k;
        double q[5];
#pragma unroll
        for (int m = 0; m < 5; ++m) q[m] = (double)a[m * sc + id];
        const Nematic nf = nematic64(q, 1e-9, Nematic{0.0, 0.0, 0.0, 1.0});
        out4[4 * t + 0] = nf.S;
        out4[4 * t + 1] = nf.nx;
        out4[4 * t + 2] = nf.ny;
        out4[4 * t + 3] = nf.nz;
    }
}

// ---------------------------------------------------------------------------------------
// FP64 observables. Every block writes one partial; a single-block pass sums the partials
// in block order, so results do not depend on scheduling.
// ---------------------------------------------------------------------------------------
struct ObsPartial {
    double bulk, elastic, anch, rad_sum, S_sum, S_max, ce, co, ca, qmax;
    unsigned long long rad_n, core_n, ce_n, co_n, ca_n, nonfinite;
};

struct ObsConst {
    QsrConst P;
    double ix2dummy;
    double i2x, i2y, i2z;
    double c2, c3, c4;         // bulk energy coefficients (QSR.cu:887-899)
    double Liso, L1, L2, L3;   // elastic energy selection (QSR.cu:955-987)
    int all_L_zero;
    double dV, Weff_half;      // cell volume; 0.5*W/delta_eff
    double S_shell;
    double cx, cy, cz, gx, gy, gz;  // FP64 geometry for normals and radial directions (cell units)
    double hx, hy, hz;               // spacing
    int checker_k;
};

constexpr int kObsThreads = 256;

template <class T>
__device__ __forceinline__ T block_sum(T v, T* sh) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    T r = 0;
    if (threadIdx.x == 0)
        for (int x = 0; x < (int)(blockDim.x >> 5); ++x) r += sh[x];
    return r;  // valid in thread 0
}

__device__ __forceinline__ double block_max(double v, double* sh) {
    v = warp_max(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int x = 0; x < (int)(blockDim.x >> 5); ++x) r = fmax(r, sh[x]);
    return r;
}

__global__ void __launch_bounds__(kObsThreads) k_observe_volume(const float* __restrict__ q,
                                                                const uint8_t* __restrict__ flags, ObsConst O,
                                                                ObsPartial* __restrict__ part) {
    const QsrConst& P = O.P;
    const long long n = (long long)P.Nx * P.Ny * P.Nz;
    ObsPartial a{};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % P.Nz);
        const long long r = t / P.Nz;
        const int j = (int)(r % P.Ny);
        const int i = (int)(r / P.Ny);
        const long long id = (long long)i * P.si + (long long)j * P.sj + k;
        const uint8_t f = flags[id];
        double c[5];
        bool finite = true;
#pragma unroll
        for (int m = 0; m < 5; ++m) {
            c[m] = (double)q[m * P.sc + id];
            finite = finite && isfinite(c[m]);
        }
        if (!finite) a.nonfinite++;
        {
            const double zz = -c[0] - c[3];
            const double tr = c[0] * c[0] + c[3] * c[3] + zz * zz + 2.0 * (c[1] * c[1] + c[2] * c[2] + c[4] * c[4]);
            a.qmax = fmax(a.qmax, sqrt(fmax(tr, 0.0)));
        }
        const bool interior = (i >= 1 && j >= 1 && k >= 1 && i < P.Nx - 1 && j < P.Ny - 1 && k < P.Nz - 1);
        if (interior) {
            // computeEnergyKernel (QSR.cu:869-992).
            const double Qxx = c[0], Qxy = c[1], Qxz = c[2], Qyy = c[3], Qyz = c[4], Qzz = -Qxx - Qyy;
            const double trQ2 = Qxx * Qxx + Qyy * Qyy + Qzz * Qzz + 2 * (Qxy * Qxy + Qxz * Qxz + Qyz * Qyz);
            const double a2xx = Qxx * Qxx + Qxy * Qxy + Qxz * Qxz;
            const double a2xy = Qxx * Qxy + Qxy * Qyy + Qxz * Qyz;
            const double a2xz = Qxx * Qxz + Qxy * Qyz + Qxz * Qzz;
            const double a2yy = Qxy * Qxy + Qyy * Qyy + Qyz * Qyz;
            const double a2yz = Qxy * Qxz + Qyy * Qyz + Qyz * Qzz;
            const double a2zz = Qxz * Qxz + Qyz * Qyz + Qzz * Qzz;
            const double trQ3 = Qxx * a2xx + Qyy * a2yy + Qzz * a2zz + 2.0 * (Qxy * a2xy + Qxz * a2xz + Qyz * a2yz);
            a.bulk += (O.c2 * trQ2 - O.c3 * trQ3 + O.c4 * trQ2 * trQ2) * O.dV;
            double d[6][3];
#pragma unroll
            for (int m = 0; m < 5; ++m) {
                const float* b = q + m * P.sc + id;
                d[m][0] = ((double)b[P.si] - (double)b[-P.si]) * O.i2x;
                d[m][1] = ((double)b[P.sj] - (double)b[-P.sj]) * O.i2y;
                d[m][2] = ((double)b[1] - (double)b[-1]) * O.i2z;
            }
#pragma unroll
            for (int x = 0; x < 3; ++x) d[5][x] = -(d[0][x] + d[3][x]);
            auto sq = [&](int m) { return d[m][0] * d[m][0] + d[m][1] * d[m][1] + d[m][2] * d[m][2]; };
            const double g2 = sq(0) + sq(3) + sq(5) + 2.0 * (sq(1) + sq(2) + sq(4));
            double fel;
            if (O.all_L_zero) {
                fel = 0.5 * O.Liso * g2;
            } else {
                const double f1 = 0.5 * O.L1 * g2;
                const double vx = d[0][0] + d[1][1] + d[2][2];
                const double vy = d[1][0] + d[3][1] + d[4][2];
                const double vz = d[2][0] + d[4][1] + d[5][2];
                const double f2 = 0.5 * O.L2 * (vx * vx + vy * vy + vz * vz);
                double f3 = 0.0;
                if (O.L3 != 0.0) {
                    auto M = [&](int x, int y) {
                        return d[0][x] * d[0][y] + d[3][x] * d[3][y] + d[5][x] * d[5][y] +
                               2.0 * (d[1][x] * d[1][y] + d[2][x] * d[2][y] + d[4][x] * d[4][y]);
                    };
                    f3 = 0.5 * O.L3 * (Qxx * M(0, 0) + Qyy * M(1, 1) + Qzz * M(2, 2) +
                                       2.0 * (Qxy * M(0, 1) + Qxz * M(0, 2) + Qyz * M(1, 2)));
                }
                fel = f1 + f2 + f3;
            }
            a.elastic += fel * O.dV;
        }
        const double X = ((double)i - O.cx), Y = ((double)j - O.cy), Z = ((double)k - O.cz);
        if (f & kAnchor) {
            // computeAnchoringEnergyKernel (QSR.cu:654-695).
            const double gx = X * O.gx, gy = Y * O.gy, gz = Z * O.gz;
            const double gn = sqrt(gx * gx + gy * gy + gz * gz);
            double nx = 1.0, ny = 0.0, nz = 0.0;
            if (gn > 0.0) { nx = gx / gn; ny = gy / gn; nz = gz / gn; }
            const double S = O.S_shell;
            const double q0xx = S * (nx * nx - 1.0 / 3.0), q0xy = S * (nx * ny), q0xz = S * (nx * nz);
            const double q0yy = S * (ny * ny - 1.0 / 3.0), q0yz = S * (ny * nz), q0zz = -(q0xx + q0yy);
            const double dxx = c[0] - q0xx, dxy = c[1] - q0xy, dxz = c[2] - q0xz, dyy = c[3] - q0yy, dyz = c[4] - q0yz;
            const double dzz = (-c[0] - c[3]) - q0zz;
            const double diff2 = dxx * dxx + dyy * dyy + dzz * dzz + 2.0 * (dxy * dxy + dxz * dxz + dyz * dyz);
            a.anch += O.Weff_half * diff2 * O.dV;
        }
        if (f & (kRadial | kCore)) {
            const Nematic nf = nematic64(c, 1e-9, Nematic{0.0, 0.0, 0.0, 1.0});
            if (f & kRadial) {
                // computeRadialityKernel (QSR.cu:994-1015): r-hat from the centre.
                const double px = X * O.hx, py = Y * O.hy, pz = Z * O.hz;
                const double rr = sqrt(px * px + py * py + pz * pz);
                double rx = 1.0, ry = 0.0, rz = 0.0;
                if (rr > 1e-30) { rx = px / rr; ry = py / rr; rz = pz / rr; }
                a.rad_sum += fabs(nf.nx * rx + nf.ny * ry + nf.nz * rz);
                a.rad_n++;
            }
            if (f & kCore) {
                a.S_sum += nf.S;
                a.core_n++;
                if (isfinite(nf.S)) a.S_max = fmax(a.S_max, nf.S);
                if (k == O.checker_k && isfinite(nf.S) && nf.S > 0.01) {
                    // Checkerboard sums on the defect slice (QSR.cu:2845-2868).
                    a.ca += nf.S; a.ca_n++;
                    if (((i + j) & 1) == 0) { a.ce += nf.S; a.ce_n++; }
                    else { a.co += nf.S; a.co_n++; }
                }
            }
        }
    }
    __shared__ double shd[kObsThreads / 32];
    __shared__ unsigned long long shu[kObsThreads / 32];
    ObsPartial res{};
    res.bulk = block_sum(a.bulk, shd);
    res.elastic = block_sum(a.elastic, shd);
    res.anch = block_sum(a.anch, shd);
    res.rad_sum = block_sum(a.rad_sum, shd);
    res.S_sum = block_sum(a.S_sum, shd);
    res.ce = block_sum(a.ce, shd);
    res.co = block_sum(a.co, shd);
    res.ca = block_sum(a.ca, shd);
    res.S_max = block_max(a.S_max, shd);
    res.qmax = block_max(a.qmax, shd);
    res.rad_n = block_sum(a.rad_n, shu);
    res.core_n = block_sum(a.core_n, shu);
    res.ce_n = block_sum(a.ce_n, shu);
    res.co_n = block_sum(a.co_n, shu);
    res.ca_n = block_sum(a.ca_n, shu);
    res.nonfinite = block_sum(a.nonfinite, shu);
    if (threadIdx.x == 0) part[blockIdx.x] = res;
}

__global__ void __launch_bounds__(kObsThreads) k_observe_finalize(const ObsPartial* __restrict__ part, int n,
                                                                  ObsPartial* __restrict__ out) {
    ObsPartial a{};
    for (int b = threadIdx.x; b < n; b += blockDim.x) {
        const ObsPartial& p = part[b];
        a.bulk += p.bulk; a.elastic += p.elastic; a.anch += p.anch; a.rad_sum += p.rad_sum; a.S_sum += p.S_sum;
        a.ce += p.ce; a.co += p.co; a.ca += p.ca;
        a.S_max = fmax(a.S_max, p.S_max); a.qmax = fmax(a.qmax, p.qmax);
        a.rad_n += p.rad_n; a.core_n += p.core_n; a.ce_n += p.ce_n; a.co_n += p.co_n; a.ca_n += p.ca_n;
        a.nonfinite += p.nonfinite;
    }
    __shared__ double shd[kObsThreads / 32];
    __shared__ unsigned long long shu[kObsThreads / 32];
    ObsPartial r{};
    r.bulk = block_sum(a.bulk, shd);
    r.elastic = block_sum(a.elastic, shd);
    r.anch = block_sum(a.anch, shd);
    r.rad_sum = block_sum(a.rad_sum, shd);
    r.S_sum = block_sum(a.S_sum, shd);
    r.ce = block_sum(a.ce, shd);
    r.co = block_sum(a.co, shd);
    r.ca = block_sum(a.ca, shd);
    r.S_max = block_max(a.S_max, shd);
    r.qmax = block_max(a.qmax, shd);
    r.rad_n = block_sum(a.rad_n, shu);
    r.core_n = block_sum(a.core_n, shu);
    r.ce_n = block_sum(a.ce_n, shu);
    r.co_n = block_sum(a.co_n, shu);
    r.ca_n = block_sum(a.ca_n, shu);
    r.nonfinite = block_sum(a.nonfinite, shu);
    if (threadIdx.x == 0) *out = r;
}

// Slice nematic field (S, nx, ny) for the 2-D defect and xi proxies.
__global__ void k_slice_nematic(const float* __restrict__ q, QsrConst P, int kz, double* __restrict__ snf) {
    const long long n = (long long)P.Nx * P.Ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(t % P.Ny);
        const int i = (int)(t / P.Ny);
        const long long id = (long long)i * P.si + (long long)j * P.sj + kz;
        double c[5];
#pragma unroll
        for (int m = 0; m < 5; ++m) c[m] = (double)q[m * P.sc + id];
        const Nematic nf = nematic64(c, 1e-9, Nematic{0.0, 0.0, 0.0, 1.0});
        snf[3 * t + 0] = nf.S;
        snf[3 * t + 1] = nf.nx;
        snf[3 * t + 2] = nf.ny;
    }
}

__device__ __forceinline__ double wrap_pi(double x) {
    // wrap_to_pi_device (QSR.cu:1027-1035).
    const double two_pi = 2.0 * kPi;
    x = x + kPi;
    x -= floor(x / two_pi) * two_pi;
    return x - kPi;
}

struct SlicePartial {
    double xi_sum;
    unsigned long long defects, plaq, edges;
};

// Plaquette winding (QSR.cu:1114-1176) and wrapped phase-gradient edges (QSR.cu:1042-1106)
// on one slice, from the slice nematic arrays. mode bit 1: defects, bit 2: xi.
__global__ void __launch_bounds__(kObsThreads) k_slice_metrics(const double* __restrict__ dnf,
                                                               const double* __restrict__ xnf, int Nx, int Ny,
                                                               double dthr, double dcut, double xthr, int mode,
                                                               SlicePartial* __restrict__ part) {
    SlicePartial a{};
    auto ok = [](const double* f, double thr) {
        return isfinite(f[0]) && isfinite(f[1]) && isfinite(f[2]) && f[0] > thr;
    };
    auto psi = [](const double* f) { return 2.0 * atan2(f[2], f[1]); };
    const long long n = (long long)Nx * Ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(t % Ny);
        const int i = (int)(t / Ny);
        if ((mode & 1) && i < Nx - 1 && j < Ny - 1) {
            const double* f00 = dnf + 3 * ((long long)i * Ny + j);
            const double* f10 = dnf + 3 * ((long long)(i + 1) * Ny + j);
            const double* f11 = dnf + 3 * ((long long)(i + 1) * Ny + j + 1);
            const double* f01 = dnf + 3 * ((long long)i * Ny + j + 1);
            if (ok(f00, dthr) && ok(f10, dthr) && ok(f11, dthr) && ok(f01, dthr)) {
                const double p00 = psi(f00), p10 = psi(f10), p11 = psi(f11), p01 = psi(f01);
                const double dsum = wrap_pi(p10 - p00) + wrap_pi(p11 - p10) + wrap_pi(p01 - p11) + wrap_pi(p00 - p01);
                const double s = 0.5 * (dsum * (1.0 / (2.0 * kPi)));
                a.plaq++;
                if (fabs(s) > dcut) a.defects++;
            }
        }
        if (mode & 2) {
            const double* f0 = xnf + 3 * ((long long)i * Ny + j);
            if (i < Nx - 1) {
                const double* f1 = xnf + 3 * ((long long)(i + 1) * Ny + j);
                if (ok(f0, xthr) && ok(f1, xthr)) {
                    const double d = wrap_pi(psi(f1) - psi(f0));
                    a.xi_sum += d * d;
                    a.edges++;
                }
            }
            if (j < Ny - 1) {
                const double* f1 = xnf + 3 * ((long long)i * Ny + j + 1);
                if (ok(f0, xthr) && ok(f1, xthr)) {
                    const double d = wrap_pi(psi(f1) - psi(f0));
                    a.xi_sum += d * d;
                    a.edges++;
                }
            }
        }
    }
    __shared__ double shd[kObsThreads / 32];
    __shared__ unsigned long long shu[kObsThreads / 32];
    SlicePartial r{};
    r.xi_sum = block_sum(a.xi_sum, shd);
    r.defects = block_sum(a.defects, shu);
    r.plaq = block_sum(a.plaq, shu);
    r.edges = block_sum(a.edges, shu);
    if (threadIdx.x == 0) part[blockIdx.x] = r;
}

__global__ void k_slice_finalize(const SlicePartial* __restrict__ part, int n, SlicePartial* __restrict__ out) {
    SlicePartial a{};
    for (int b = threadIdx.x; b < n; b += blockDim.x) {
        a.xi_sum += part[b].xi_sum; a.defects += part[b].defects; a.plaq += part[b].plaq; a.edges += part[b].edges;
    }
    __shared__ double shd[kObsThreads / 32];
    __shared__ unsigned long long shu[kObsThreads / 32];
    SlicePartial r{};
    r.xi_sum = block_sum(a.xi_sum, shd);
    r.defects = block_sum(a.defects, shu);
    r.plaq = block_sum(a.plaq, shu);
    r.edges = block_sum(a.edges, shu);
    if (threadIdx.x == 0) *out = r;
}

constexpr int kObsBlocks = 148 * 8;
constexpr int kSliceBlocks = 148;

}  // namespace

// ---------------------------------------------------------------------------------------
// Handle and C ABI
// ---------------------------------------------------------------------------------------
struct qsr_handle {
    qsr_params p{};
    Geometry g{};
    double delta_eff = 0.0;
    long long shell_cells = 0, evolving_cells = 0, active_cells = 0, written_cells = 0;
    int sj = 0;
    long long si = 0, sc = 0, ncells = 0;
    float* q[2] = {nullptr, nullptr};
    float* lo[2] = {nullptr, nullptr};  // low words of compensated storage (optional)
    float* rhs = nullptr;
    uint8_t* flags = nullptr;
    double* stage = nullptr;       // FP64 AoS staging (5 or 4 doubles per cell)
    bool stage_shared = false;     // staging owned by an ensemble (shared by its droplets)
    ObsPartial* opart = nullptr;   // kObsBlocks + 1
    SlicePartial* spart = nullptr; // kSliceBlocks + 1
    double* snf = nullptr;         // 2 slices x Nx*Ny x 3
    TiledPlan tiled{};             // tiled-kernel launch plan
    int cur = 0;
    bool uploaded = false;
    cudaStream_t stream = nullptr;
    long long launches = 0;
    int device = -1;               // the GPU the handle was created on
};

namespace {

QsrConst make_const(const qsr_handle* h, double T, double S_shell, double dt) {
    const qsr_params& p = h->p;
    QsrConst P{};
    P.Nx = p.Nx; P.Ny = p.Ny; P.Nz = p.Nz;
    P.sj = h->sj; P.si = h->si; P.sc = h->sc;
    P.ix2 = (float)(1.0 / (p.dx * p.dx)); P.iy2 = (float)(1.0 / (p.dy * p.dy)); P.iz2 = (float)(1.0 / (p.dz * p.dz));
    P.i2x = (float)(1.0 / (2.0 * p.dx)); P.i2y = (float)(1.0 / (2.0 * p.dy)); P.i2z = (float)(1.0 / (2.0 * p.dz));
    P.ix = (float)(1.0 / p.dx); P.iy = (float)(1.0 / p.dy); P.iz = (float)(1.0 / p.dz);
    P.i4xy = (float)(1.0 / (4.0 * p.dx * p.dy));
    P.i4xz = (float)(1.0 / (4.0 * p.dx * p.dz));
    P.i4yz = (float)(1.0 / (4.0 * p.dy * p.dz));
    const double dT = T - p.T_star;
    const double cQ = 3.0 * p.a * dT;
    const double cQ2 = (p.bulk_modechoice == 1) ? (9.0 * p.b) / 2.0 : (27.0 * p.b) / 2.0;
    const double cQ3 = (p.bulk_modechoice == 1) ? (9.0 * p.c) / 2.0 : 9.0 * p.c;
    P.cQ = (float)cQ; P.cQ2 = (float)cQ2; P.cQ3 = (float)cQ3;
    const bool all_zero = (p.L1 == 0.0 && p.L2 == 0.0 && p.L3 == 0.0);
    P.Liso = (float)(all_zero ? p.kappa : p.L1);
    P.L2 = (float)p.L2; P.L3 = (float)p.L3;
    P.Weff = (h->delta_eff > 0.0) ? (float)(p.W / h->delta_eff) : 0.0f;
    P.S_shell = (float)S_shell;
    P.mob_dt = (float)((1.0 / p.gamma) * dt);
    P.ci = (float)(0.5 * (p.Nx - 1.0)); P.cj = (float)(0.5 * (p.Ny - 1.0)); P.ck = (float)(0.5 * (p.Nz - 1.0));
    // Surface normal ~ (x/rx^2, y/ry^2, z/rz^2) with x = X dx: scale per axis dx/rx^2 (normalised later),
    // expressed relative to the x axis to stay in FP32 range.
    const double sxn = p.dx / (h->g.rx * h->g.rx);
    P.gnx = 1.0f;
    P.gny = (float)((p.dy / (h->g.ry * h->g.ry)) / sxn);
    P.gnz = (float)((p.dz / (h->g.rz * h->g.rz)) / sxn);
    const double ix2 = 1.0 / (p.dx * p.dx), iy2 = 1.0 / (p.dy * p.dy), iz2 = 1.0 / (p.dz * p.dz);
    P.lap_c = (float)(-2.0 * (ix2 + iy2 + iz2));
    P.L2i2x = (float)(p.L2 / (2.0 * p.dx)); P.L2i2y = (float)(p.L2 / (2.0 * p.dy)); P.L2i2z = (float)(p.L2 / (2.0 * p.dz));
    const double i2[3] = {1.0 / (2.0 * p.dx), 1.0 / (2.0 * p.dy), 1.0 / (2.0 * p.dz)};
    const int ab[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
    for (int m = 0; m < 6; ++m) P.l3m[m] = (float)(0.5 * p.L3 * i2[ab[m][0]] * i2[ab[m][1]]);
    for (int m = 0; m < 6; ++m) P.l2w[m] = (float)(p.L2 * i2[ab[m][0]] * i2[ab[m][1]]);
    return P;
}

int alloc_or_fail(void** ptr, size_t bytes) {
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) {
        set_error(std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
        return LDG_ERR_NOMEM;
    }
    return LDG_OK;
}

template <bool L2, bool L3, bool N, bool R>
void launch_direct(const qsr_handle* h, const float* in, float* out, const QsrConst& P) {
    dim3 blk(32, 8, 1), grd((P.Nz + 31) / 32, (P.Ny + 7) / 8, P.Nx);
    k_step_direct<L2, L3, N, R><<<grd, blk, 0, h->stream>>>(in, out, h->flags, P);
}

template <bool R>
void dispatch_direct(const qsr_handle* h, const float* in, float* out, const QsrConst& P, bool L2, bool L3, bool N) {
    const int key = (L2 ? 1 : 0) | (L3 ? 2 : 0) | (N ? 4 : 0);
    switch (key) {
        case 0: launch_direct<false, false, false, R>(h, in, out, P); break;
        case 1: launch_direct<true, false, false, R>(h, in, out, P); break;
        case 2: launch_direct<false, true, false, R>(h, in, out, P); break;
        case 3: launch_direct<true, true, false, R>(h, in, out, P); break;
        case 4: launch_direct<false, false, true, R>(h, in, out, P); break;
        case 5: launch_direct<true, false, true, R>(h, in, out, P); break;
        case 6: launch_direct<false, true, true, R>(h, in, out, P); break;
        default: launch_direct<true, true, true, R>(h, in, out, P); break;
    }
}

int grid_blocks(long long n, int threads, int cap) {
    long long b = (n + threads - 1) / threads;
    return (int)std::max(1LL, std::min<long long>(b, cap));
}

// Kernel selection: 1 = tiled (default), 0 = direct. LDG_QSR_KERNEL=direct forces the direct path.
int kernel_choice() {
    const char* e = getenv("LDG_QSR_KERNEL");
    if (e && std::strcmp(e, "direct") == 0) return 0;
    return 1;
}

}  // namespace

namespace {

// Enqueues the observables of the current field on stream `st`, with the block results copied
// to R and SR (host memory; pinned for the copies to be asynchronous).
int observe_enqueue(qsr_handle* h, const qsr_observe_args* a, cudaStream_t st, ObsPartial* R, SlicePartial* SR,
                    bool* wd_out, bool* wx_out) {
    const qsr_params& p = h->p;
    ObsConst O{};
    O.P = make_const(h, a->T, a->S_shell, 1.0);
    O.i2x = 1.0 / (2.0 * p.dx); O.i2y = 1.0 / (2.0 * p.dy); O.i2z = 1.0 / (2.0 * p.dz);
    const double dT = a->T - p.T_star;
    if (p.bulk_modechoice == 1) { O.c2 = (3.0 * p.a * dT) / 2.0; O.c3 = (3.0 * p.b) / 2.0; O.c4 = (9.0 * p.c) / 8.0; }
    else { O.c2 = (3.0 * p.a * dT) / 2.0; O.c3 = (9.0 * p.b) / 2.0; O.c4 = (9.0 * p.c) / 4.0; }
    O.all_L_zero = (p.L1 == 0.0 && p.L2 == 0.0 && p.L3 == 0.0);
    O.Liso = p.kappa; O.L1 = p.L1; O.L2 = p.L2; O.L3 = p.L3;
    O.dV = p.dx * p.dy * p.dz;
    O.Weff_half = (h->delta_eff > 0.0) ? 0.5 * (p.W / h->delta_eff) : 0.0;
    O.S_shell = a->S_shell;
    O.cx = 0.5 * (p.Nx - 1.0); O.cy = 0.5 * (p.Ny - 1.0); O.cz = 0.5 * (p.Nz - 1.0);
    // Surface normal ~ (X dx/rx^2, Y dy/ry^2, Z dz/rz^2) in cell units, scaled relative to x.
    const double sx = p.dx / (h->g.rx * h->g.rx);
    O.gx = 1.0;
    O.gy = (p.dy / (h->g.ry * h->g.ry)) / sx;
    O.gz = (p.dz / (h->g.rz * h->g.rz)) / sx;
    O.hx = p.dx; O.hy = p.dy; O.hz = p.dz;
    O.checker_k = std::min(std::max(a->defects_z_slice, 0), p.Nz - 1);
    const float* q = h->q[h->cur];
    k_observe_volume<<<kObsBlocks, kObsThreads, 0, st>>>(q, h->flags, O, h->opart);
    h->launches++;
    LDG_LAUNCHED("k_observe_volume");
    k_observe_finalize<<<1, kObsThreads, 0, st>>>(h->opart, kObsBlocks, h->opart + kObsBlocks);
    h->launches++;
    LDG_LAUNCHED("k_observe_finalize");
    const bool wd = a->want_defects && a->defects_z_slice >= 0 && a->defects_z_slice < p.Nz;
    const bool wx = a->want_xi && a->xi_z_slice >= 0 && a->xi_z_slice < p.Nz;
    const long long nxy = (long long)p.Nx * p.Ny;
    if (wd || wx) {
        double* dnf = h->snf;
        double* xnf = h->snf + 3 * nxy;
        if (wd) {
            k_slice_nematic<<<grid_blocks(nxy, 256, 148 * 4), 256, 0, st>>>(q, O.P, a->defects_z_slice, dnf);
            h->launches++;
        }
        if (wx) {
            if (wd && a->xi_z_slice == a->defects_z_slice) {
                xnf = dnf;
            } else {
                k_slice_nematic<<<grid_blocks(nxy, 256, 148 * 4), 256, 0, st>>>(q, O.P, a->xi_z_slice, xnf);
                h->launches++;
            }
        }
        const int mode = (wd ? 1 : 0) | (wx ? 2 : 0);
        k_slice_metrics<<<kSliceBlocks, kObsThreads, 0, st>>>(dnf, xnf, p.Nx, p.Ny, a->defects_S_threshold,
                                                                     a->defects_charge_cutoff, a->xi_S_threshold, mode,
                                                                     h->spart);
        k_slice_finalize<<<1, kObsThreads, 0, st>>>(h->spart, kSliceBlocks, h->spart + kSliceBlocks);
        h->launches += 2;
        LDG_LAUNCHED("k_slice_metrics");
    }
    LDG_CUDA(cudaMemcpyAsync(R, h->opart + kObsBlocks, sizeof(*R), cudaMemcpyDeviceToHost, st));
    if (wd || wx) LDG_CUDA(cudaMemcpyAsync(SR, h->spart + kSliceBlocks, sizeof(*SR), cudaMemcpyDeviceToHost, st));
    *wd_out = wd;
    *wx_out = wx;
    return LDG_OK;
}

// Fills the observables from the reduced block results.
void observe_finish(const qsr_handle* h, const ObsPartial& R, const SlicePartial& SR, bool wd, bool wx,
                    qsr_observables* o) {
    const qsr_params& p = h->p;
    const double nan = std::numeric_limits<double>::quiet_NaN();
    std::memset(o, 0, sizeof(*o));
    o->bulk = R.bulk; o->elastic = R.elastic; o->anchoring = R.anch;
    o->total = R.bulk + R.elastic + R.anch;
    o->radiality_count = (long long)R.rad_n;
    o->radiality = R.rad_n > 0 ? R.rad_sum / (double)R.rad_n : 0.0;
    o->core_count = (long long)R.core_n;
    o->avg_S = R.core_n > 0 ? R.S_sum / (double)R.core_n : 0.0;
    o->max_S = R.S_max;
    o->checker_rel = nan;
    if (R.S_max >= 0.5 && R.ce_n > 10 && R.co_n > 10 && R.ca_n > 20 && R.ca != 0.0)
        o->checker_rel = std::fabs(R.ce - R.co) / std::fabs(R.ca);
    o->defect_count = (long long)SR.defects;
    o->defect_plaquettes = (long long)SR.plaq;
    o->defect_density = (wd && SR.plaq > 0) ? (double)SR.defects / (double)SR.plaq : nan;
    o->xi_edges = (long long)SR.edges;
    o->xi_grad_proxy = nan;
    if (wx && SR.edges > 0) {
        const double ms = SR.xi_sum / (double)SR.edges;
        const double inv = (ms > 0.0) ? (1.0 / std::sqrt(ms + 1e-30)) : (1.0 / std::sqrt(1e-30));
        o->xi_grad_proxy = std::min(inv, 0.5 * (double)std::min(p.Nx, p.Ny));
    }
    o->max_q_norm = R.qmax;
    o->nonfinite_cells = (long long)R.nonfinite;
}

}  // namespace

extern "C" {

int qsr_create(const qsr_params* params, qsr_handle** out) {
    clear_error();
    LDG_REQUIRE(params && out, LDG_ERR_ARG, "qsr_create: null argument");
    const qsr_params& p = *params;
    LDG_REQUIRE(p.Nx >= 3 && p.Ny >= 3 && p.Nz >= 3, LDG_ERR_ARG, "qsr_create: Nx, Ny, Nz must be >= 3");
    LDG_REQUIRE((long long)p.Nx * p.Ny * p.Nz < (1LL << 32), LDG_ERR_ARG, "qsr_create: grid exceeds 2^32 cells");
    LDG_REQUIRE(p.dx > 0 && p.dy > 0 && p.dz > 0, LDG_ERR_ARG, "qsr_create: spacings must be positive");
    LDG_REQUIRE(p.gamma > 0, LDG_ERR_ARG, "qsr_create: gamma must be positive");
    LDG_REQUIRE(p.bulk_modechoice == 1 || p.bulk_modechoice == 2, LDG_ERR_ARG, "qsr_create: bulk_modechoice must be 1 or 2");
    qsr_handle* h = new (std::nothrow) qsr_handle();
    LDG_REQUIRE(h, LDG_ERR_NOMEM, "qsr_create: host allocation failed");
    h->p = p;
    cudaGetDevice(&h->device);
    h->g = make_geometry(p);
    h->sj = (p.Nz + 3) & ~3;
    h->si = (long long)p.Ny * h->sj;
    h->sc = (long long)p.Nx * h->si;
    h->ncells = (long long)p.Nx * p.Ny * p.Nz;

    // Classification in FP64 on the host (QSR.cu:2160-2187 and the device predicates).
    std::vector<uint8_t> fl((size_t)h->sc, 0);
    const Geometry g = h->g;
    const double band = (p.W > 0.0) ? g.shell_half : 0.0;
    long long shell = 0;
#pragma omp parallel for collapse(2) reduction(+ : shell)
    for (int i = 0; i < p.Nx; ++i)
        for (int j = 0; j < p.Ny; ++j)
            for (int k = 0; k < p.Nz; ++k) {
                double sd, r;
                signed_distance(g, i, j, k, sd, r);
                uint8_t f = 0;
                if (std::fabs(sd) <= g.shell_half) { f |= kShell; ++shell; }
                if (sd <= 0.0) f |= kInside;
                if (sd < -2.0 * g.min_spacing) f |= kCore;
                if (sd <= 0.0 && r > 2.0 * g.min_spacing) f |= kRadial;
                fl[(size_t)i * h->si + (size_t)j * h->sj + k] = f;
                (void)band;
            }
    // delta_eff = shell volume / Knud-Thomsen ellipsoid area (QSR.cu:164-185).
    double delta = 2.0 * g.shell_half;
    if (shell > 0) {
        const double pp = 1.6075;
        const double ap = std::pow(g.rx, pp), bp = std::pow(g.ry, pp), cp = std::pow(g.rz, pp);
        const double mean = (ap * bp + ap * cp + bp * cp) / 3.0;
        const double area = (mean > 0.0) ? 4.0 * kPi * std::pow(mean, 1.0 / pp) : std::numeric_limits<double>::quiet_NaN();
        if (area > 0.0) {
            const double t = (double)shell * g.dx * g.dy * g.dz / area;
            if (std::isfinite(t) && t > 0.0) delta = t;
        }
    }
    h->delta_eff = delta;
    h->shell_cells = shell;
    long long evolving = 0;
#pragma omp parallel for collapse(2) reduction(+ : evolving)
    for (int i = 0; i < p.Nx; ++i)
        for (int j = 0; j < p.Ny; ++j)
            for (int k = 0; k < p.Nz; ++k) {
                double sd, r;
                signed_distance(g, i, j, k, sd, r);
                uint8_t& f = fl[(size_t)i * h->si + (size_t)j * h->sj + k];
                const bool sh = (f & kShell) != 0;
                const bool moves = !(p.W == 0.0 && sh) && (sd <= band);
                if (moves) { f |= kMove; ++evolving; }
                if (p.W <= 0.0 && sh) f |= kFixed;
                if (sh && p.W != 0.0 && delta > 0.0) f |= kAnchor;
            }
    h->evolving_cells = evolving;

    int rc;
    const size_t fbytes = (size_t)h->sc * 5 * sizeof(float);
    if ((rc = alloc_or_fail((void**)&h->q[0], fbytes)) || (rc = alloc_or_fail((void**)&h->q[1], fbytes)) ||
        (rc = alloc_or_fail((void**)&h->flags, (size_t)h->sc)) ||
        (rc = alloc_or_fail((void**)&h->opart, (kObsBlocks + 1) * sizeof(ObsPartial))) ||
        (rc = alloc_or_fail((void**)&h->spart, (kSliceBlocks + 1) * sizeof(SlicePartial))) ||
        (rc = alloc_or_fail((void**)&h->snf, (size_t)2 * p.Nx * p.Ny * 3 * sizeof(double))) ||
        (p.compensated && ((rc = alloc_or_fail((void**)&h->lo[0], fbytes)) ||
                           (rc = alloc_or_fail((void**)&h->lo[1], fbytes))))) {
        qsr_destroy(h);
        return rc;
    }
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMemcpy(h->flags, fl.data(), (size_t)h->sc, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(h->q[0], 0, fbytes);
    if (e == cudaSuccess) e = cudaMemset(h->q[1], 0, fbytes);
    if (e == cudaSuccess && h->lo[0]) e = cudaMemset(h->lo[0], 0, fbytes);
    if (e == cudaSuccess && h->lo[1]) e = cudaMemset(h->lo[1], 0, fbytes);
    if (e != cudaSuccess) {
        set_error(std::string("qsr_create: ") + cudaGetErrorString(e));
        qsr_destroy(h);
        return LDG_ERR_CUDA;
    }
    rc = tiled_plan_build(h->tiled, p.Nx, p.Ny, p.Nz, h->sj, h->si, fl.data(), h->q[0], h->q[1], h->sc);
    if (rc != LDG_OK) {
        qsr_destroy(h);
        return rc;
    }
    h->active_cells = h->tiled.active_cells;
    h->written_cells = h->tiled.written_cells;
    *out = h;
    return LDG_OK;
}

int qsr_geometry(const qsr_handle* h, qsr_geometry_info* o) {
    clear_error();
    LDG_REQUIRE(h && o, LDG_ERR_ARG, "qsr_geometry: null argument");
    o->center_x = h->g.cx; o->center_y = h->g.cy; o->center_z = h->g.cz;
    o->radius_x = h->g.rx; o->radius_y = h->g.ry; o->radius_z = h->g.rz;
    o->min_spacing = h->g.min_spacing;
    o->shell_half_thickness = h->g.shell_half;
    o->delta_eff = h->delta_eff;
    o->shell_cells = h->shell_cells;
    o->evolving_cells = h->evolving_cells;
    o->active_cells = h->tiled.ok ? h->tiled.active_cells : h->active_cells;
    o->written_cells = h->written_cells;
    o->box_cells = h->ncells;
    return LDG_OK;
}

int qsr_initial_field(const qsr_handle* h, int mode, long long seed, double S0, double noise_amplitude,
                      double* q) {
    clear_error();
    LDG_REQUIRE(h && q, LDG_ERR_ARG, "qsr_initial_field: null argument");
    LDG_REQUIRE(mode >= 0 && mode <= 2, LDG_ERR_ARG, "qsr_initial_field: init_mode must be 0, 1 or 2");
    const qsr_params& p = h->p;
    const Geometry& g = h->g;
    const size_t n = (size_t)h->ncells;
    std::fill(q, q + 5 * n, 0.0);
    std::mt19937 gen = (seed >= 0) ? std::mt19937((std::mt19937::result_type)seed) : std::mt19937(std::random_device{}());
    auto id = [&](int i, int j, int k) { return (size_t)k + (size_t)p.Nz * ((size_t)j + (size_t)p.Ny * (size_t)i); };
    if (mode == 2) {
        if (noise_amplitude <= 0.0) return LDG_OK;
        std::normal_distribution<double> dist(0.0, noise_amplitude);
        for (int i = 0; i < p.Nx; ++i)
            for (int j = 0; j < p.Ny; ++j)
                for (int k = 0; k < p.Nz; ++k) {
                    double sd, r;
                    signed_distance(g, i, j, k, sd, r);
                    if (sd <= 0.0)
                        for (int m = 0; m < 5; ++m) q[5 * id(i, j, k) + m] = dist(gen);
                }
        return LDG_OK;
    }
    std::uniform_real_distribution<double> dist_theta(0.0, kPi);
    std::uniform_real_distribution<double> dist_phi(0.0, 2.0 * kPi);
    for (int i = 0; i < p.Nx; ++i)
        for (int j = 0; j < p.Ny; ++j)
            for (int k = 0; k < p.Nz; ++k) {
                double sd, r;
                signed_distance(g, i, j, k, sd, r);
                if (!(sd <= 0.0)) continue;
                double S = S0;
                if (r < g.core_radius) S *= (r / g.core_radius);
                double nx = 1.0, ny = 0.0, nz = 0.0;
                if (mode == 0) {
                    const double theta = dist_theta(gen);
                    const double phi = dist_phi(gen);
                    nx = std::sin(theta) * std::cos(phi);
                    ny = std::sin(theta) * std::sin(phi);
                    nz = std::cos(theta);
                } else if (r > 1e-30) {
                    nx = (i * g.dx - g.cx) / r;
                    ny = (j * g.dy - g.cy) / r;
                    nz = (k * g.dz - g.cz) / r;
                }
                double* c = q + 5 * id(i, j, k);
                c[0] = S * (nx * nx - 1.0 / 3.0);
                c[1] = S * (nx * ny);
                c[2] = S * (nx * nz);
                c[3] = S * (ny * ny - 1.0 / 3.0);
                c[4] = S * (ny * nz);
            }
    return LDG_OK;
}

static int ensure_stage(qsr_handle* h, size_t doubles) {
    if (h->stage) return LDG_OK;
    (void)doubles;
    return alloc_or_fail((void**)&h->stage, (size_t)h->ncells * 5 * sizeof(double));
}

int qsr_upload(qsr_handle* h, const double* q) {
    clear_error();
    LDG_REQUIRE(h && q, LDG_ERR_ARG, "qsr_upload: null argument");
    DeviceGuard device_guard(h->device);
    int rc = ensure_stage(h, 5);
    if (rc) return rc;
    LDG_CUDA(cudaMemcpyAsync(h->stage, q, (size_t)h->ncells * 5 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    h->cur = 0;
    k_aos_to_soa<<<grid_blocks(h->ncells, 256, 148 * 16), 256, 0, h->stream>>>(h->stage, h->q[0], h->q[1], h->p.Nx,
                                                                              h->p.Ny, h->p.Nz, h->sj, h->si, h->sc,
                                                                              h->lo[0], h->lo[1]);
    h->launches++;
    LDG_LAUNCHED("k_aos_to_soa");
    LDG_CUDA(cudaStreamSynchronize(h->stream));
    h->uploaded = true;
    return LDG_OK;
}

int qsr_download(qsr_handle* h, double* q) {
    clear_error();
    LDG_REQUIRE(h && q, LDG_ERR_ARG, "qsr_download: null argument");
    DeviceGuard device_guard(h->device);
    int rc = ensure_stage(h, 5);
    if (rc) return rc;
    k_soa_to_aos<<<grid_blocks(h->ncells, 256, 148 * 16), 256, 0, h->stream>>>(h->q[h->cur], h->stage, h->p.Nx,
                                                                              h->p.Ny, h->p.Nz, h->sj, h->si, h->sc,
                                                                              h->lo[h->cur]);
    h->launches++;
    LDG_LAUNCHED("k_soa_to_aos");
    LDG_CUDA(cudaMemcpyAsync(q, h->stage, (size_t)h->ncells * 5 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    LDG_CUDA(cudaStreamSynchronize(h->stream));
    return tiled_check(h->tiled, h->stream);
}

int qsr_nematic(qsr_handle* h, double* s_n) {
    clear_error();
    LDG_REQUIRE(h && s_n, LDG_ERR_ARG, "qsr_nematic: null argument");
    DeviceGuard device_guard(h->device);
    int rc = ensure_stage(h, 5);
    if (rc) return rc;
    k_nematic_out<<<grid_blocks(h->ncells, 256, 148 * 16), 256, 0, h->stream>>>(h->q[h->cur], h->stage, h->p.Nx,
                                                                               h->p.Ny, h->p.Nz, h->sj, h->si, h->sc);
    h->launches++;
    LDG_LAUNCHED("k_nematic_out");
    LDG_CUDA(cudaMemcpyAsync(s_n, h->stage, (size_t)h->ncells * 4 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    LDG_CUDA(cudaStreamSynchronize(h->stream));
    return LDG_OK;
}

int qsr_step(qsr_handle* h, int n_steps, const qsr_step_args* a) {
    clear_error();
    LDG_REQUIRE(h && a, LDG_ERR_ARG, "qsr_step: null argument");
    DeviceGuard device_guard(h->device);
    LDG_REQUIRE(n_steps >= 0, LDG_ERR_ARG, "qsr_step: n_steps must be >= 0");
    LDG_REQUIRE(h->uploaded, LDG_ERR_STATE, "qsr_step: no field uploaded");
    LDG_REQUIRE(a->dt > 0.0 && std::isfinite(a->dt), LDG_ERR_ARG, "qsr_step: dt must be positive and finite");
    const qsr_params& p = h->p;
    QsrConst P = make_const(h, a->T, a->S_shell, a->dt);
    P.qcap = (float)a->q_norm_cap;
    P.sigma = (float)a->noise_sigma;
    P.key0 = (uint32_t)a->seed;
    P.key1 = (uint32_t)(a->seed >> 32);
    P.instance = 0;
    const bool noise = a->noise_sigma > 0.0;
    const bool L2 = p.L2 != 0.0, L3 = p.L3 != 0.0;
    // The reference falls back to the explicit update when the stabiliser is inactive (QSR.cu:2721).
    const bool imex = a->semi_implicit && a->L_stab > 0.0 && a->jacobi_iters > 0;
    if (imex) {
        if (!h->rhs) {
            int rc = alloc_or_fail((void**)&h->rhs, (size_t)h->sc * 5 * sizeof(float));
            if (rc) return rc;
            LDG_CUDA(cudaMemset(h->rhs, 0, (size_t)h->sc * 5 * sizeof(float)));
        }
        P.alpha = (float)(a->dt * (1.0 / p.gamma) * a->L_stab);
        const double aj = (a->dt / p.gamma) * a->L_stab;  // QSR.cu:2728
        const double denom = 1.0 + 2.0 * aj * (1.0 / (p.dx * p.dx) + 1.0 / (p.dy * p.dy) + 1.0 / (p.dz * p.dz));
        LDG_REQUIRE(denom > 0.0, LDG_ERR_ARG, "qsr_step: non-positive Jacobi denominator");
        P.jdenom_inv = (float)(1.0 / denom);
    }
    const int choice = kernel_choice();
    for (int s = 0; s < n_steps; ++s) {
        P.step = a->step_index + s;
        const float* in = h->q[h->cur];
        float* outb = h->q[1 - h->cur];
        if (!imex) {
            if (choice == 1 && h->tiled.ok) {
                int rc = tiled_step(h->tiled, in, outb, h->flags, P, L2, L3, noise, false, h->stream, h->lo[h->cur],
                                    h->lo[1 - h->cur]);
                if (rc) return rc;
            } else {
                dispatch_direct<false>(h, in, outb, P, L2, L3, noise);
            }
            h->launches++;
            LDG_LAUNCHED("qsr step kernel");
            h->cur = 1 - h->cur;
        } else {
            if (choice == 1 && h->tiled.ok) {
                int rc = tiled_step(h->tiled, in, h->rhs, h->flags, P, L2, L3, noise, true, h->stream);
                if (rc) return rc;
            } else {
                dispatch_direct<true>(h, in, h->rhs, P, L2, L3, noise);
            }
            h->launches++;
            LDG_LAUNCHED("k_step_direct(rhs)");
            dim3 blk(32, 8, 1), grd((p.Nz + 31) / 32, (p.Ny + 7) / 8, p.Nx);
            const bool tiled = choice == 1 && h->tiled.ok;
            int c = h->cur;
            for (int it = 0; it < a->jacobi_iters; ++it) {
                const bool last = (it == a->jacobi_iters - 1);
                if (tiled) {
                    if (h->tiled.n_plane_items > 0) {
                        const int nb = h->tiled.n_plane_items;
                        if (last)
                            k_jacobi_tiled<true><<<nb, 128, 0, h->stream>>>(h->rhs, h->q[c], h->q[1 - c], h->flags,
                                                                             h->tiled.plane_items, P);
                        else
                            k_jacobi_tiled<false><<<nb, 128, 0, h->stream>>>(h->rhs, h->q[c], h->q[1 - c], h->flags,
                                                                              h->tiled.plane_items, P);
                    }
                } else if (last) {
                    k_jacobi<true><<<grd, blk, 0, h->stream>>>(h->rhs, h->q[c], h->q[1 - c], h->flags, P);
                } else {
                    k_jacobi<false><<<grd, blk, 0, h->stream>>>(h->rhs, h->q[c], h->q[1 - c], h->flags, P);
                }
                h->launches++;
                LDG_LAUNCHED("k_jacobi");
                c = 1 - c;
            }
            h->cur = c;
        }
    }
    // Compensated storage is kept by the explicit tiled step only; after other updates the
    // field is its high words.
    if (h->lo[0] && n_steps > 0 && (imex || choice != 1 || !h->tiled.ok)) {
        const size_t fbytes = (size_t)h->sc * 5 * sizeof(float);
        LDG_CUDA(cudaMemsetAsync(h->lo[0], 0, fbytes, h->stream));
        LDG_CUDA(cudaMemsetAsync(h->lo[1], 0, fbytes, h->stream));
    }
    return LDG_OK;
}

int qsr_observe(qsr_handle* h, const qsr_observe_args* a, qsr_observables* o) {
    clear_error();
    LDG_REQUIRE(h && a && o, LDG_ERR_ARG, "qsr_observe: null argument");
    DeviceGuard device_guard(h->device);
    ObsPartial R{};
    SlicePartial SR{};
    bool wd = false, wx = false;
    int rc = observe_enqueue(h, a, h->stream, &R, &SR, &wd, &wx);
    if (rc) return rc;
    LDG_CUDA(cudaStreamSynchronize(h->stream));
    if ((rc = tiled_check(h->tiled, h->stream))) return rc;
    observe_finish(h, R, SR, wd, wx, o);
    return LDG_OK;
}

int qsr_autotune(qsr_handle* h, const qsr_step_args* a, int trial_steps, int* chosen_chunk) {
    clear_error();
    LDG_REQUIRE(h && a, LDG_ERR_ARG, "qsr_autotune: null argument");
    DeviceGuard device_guard(h->device);
    LDG_REQUIRE(trial_steps >= 1, LDG_ERR_ARG, "qsr_autotune: trial_steps must be >= 1");
    LDG_REQUIRE(h->uploaded, LDG_ERR_STATE, "qsr_autotune: no field uploaded");
    LDG_REQUIRE(h->tiled.ok, LDG_ERR_STATE, "qsr_autotune: no tiled plan");
    LDG_CUDA(cudaStreamSynchronize(h->stream));
    // Back up the current field (and its low words) and the launch count; restore both after.
    const size_t fbytes = (size_t)h->sc * 5 * sizeof(float);
    const int planes = h->lo[0] ? 2 : 1;
    float* backup = nullptr;
    int rc = alloc_or_fail((void**)&backup, fbytes * planes);
    if (rc) return rc;
    const int cur0 = h->cur;
    const long long launches0 = h->launches;
    LDG_CUDA(cudaMemcpyAsync(backup, h->q[cur0], fbytes, cudaMemcpyDeviceToDevice, h->stream));
    if (h->lo[0]) LDG_CUDA(cudaMemcpyAsync(backup + h->sc * 5, h->lo[cur0], fbytes, cudaMemcpyDeviceToDevice, h->stream));
    const int candidates[] = {8, 12, 16, 24, 32, 48, 64};
    int best = 0;
    float best_ms = std::numeric_limits<float>::infinity();
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        set_error("qsr_autotune: event creation failed");
        rc = LDG_ERR_CUDA;
    }
    qsr_step_args t = *a;
    for (int c : candidates) {
        if (rc) break;
        if ((rc = tiled_plan_rechunk(h->tiled, c))) break;
        if ((rc = qsr_step(h, 2, &t))) break;
        cudaEventRecord(e0, h->stream);
        if ((rc = qsr_step(h, trial_steps, &t))) break;
        cudaEventRecord(e1, h->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            set_error("qsr_autotune: trial failed");
            rc = LDG_ERR_CUDA;
            break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) { best_ms = ms; best = c; }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    // restore both ping-pong buffers from the backup (frozen cells are identical in both)
    for (int b = 0; b < 2; ++b) {
        cudaMemcpyAsync(h->q[b], backup, fbytes, cudaMemcpyDeviceToDevice, h->stream);
        if (h->lo[0]) cudaMemcpyAsync(h->lo[b], backup + h->sc * 5, fbytes, cudaMemcpyDeviceToDevice, h->stream);
    }
    cudaStreamSynchronize(h->stream);
    cudaFree(backup);
    h->cur = cur0;
    h->launches = launches0;
    if (rc == LDG_OK) rc = tiled_check(h->tiled, h->stream);
    if (rc) return rc;
    if ((rc = tiled_plan_rechunk(h->tiled, best))) return rc;
    if (chosen_chunk) *chosen_chunk = best;
    return LDG_OK;
}

int qsr_sync(qsr_handle* h) {
    clear_error();
    LDG_REQUIRE(h, LDG_ERR_ARG, "qsr_sync: null handle");
    DeviceGuard device_guard(h->device);
    LDG_CUDA(cudaStreamSynchronize(h->stream));
    return tiled_check(h->tiled, h->stream);
}

void* qsr_stream(qsr_handle* h) { return h ? (void*)h->stream : nullptr; }

long long qsr_launch_count(const qsr_handle* h) { return h ? h->launches : 0; }

int qsr_destroy(qsr_handle* h) {
    if (!h) return LDG_OK;
    DeviceGuard device_guard(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    cudaFree(h->q[0]); cudaFree(h->q[1]); cudaFree(h->lo[0]); cudaFree(h->lo[1]); cudaFree(h->rhs); cudaFree(h->flags);
    if (!h->stage_shared) cudaFree(h->stage);
    cudaFree(h->opart); cudaFree(h->spart); cudaFree(h->snf);
    tiled_plan_free(h->tiled);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return LDG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// Ensemble of droplets: every instance is a qsr_handle (geometry, classification, buffers,
// tensor maps, observables); one persistent work-stealing launch per step covers the active
// tiles of all instances, and runs of steps are replayed from a captured CUDA graph.
// ---------------------------------------------------------------------------------------
struct ens_handle {
    ens_params p{};
    int device = -1;                       // the GPU the ensemble was created on
    double* stage = nullptr;               // host-boundary staging shared by all droplets
    void* obs_host = nullptr;              // pinned block results of ens_observe_all
    std::vector<qsr_handle*> inst;
    std::vector<ens_instance> desc;
    std::vector<tiled::EnsInstDev> host_inst;
    CUtensorMap* d_tms = nullptr;          // 2 per instance: input buffer q[0] / q[1]
    tiled::EnsInstDev* d_inst = nullptr;
    tiled::EnsItem* d_items = nullptr;
    int n_items = 0;
    tiled::EnsCtl* d_ctl = nullptr;
    int* d_err = nullptr;
    int chunk = 0;
    int grid = 0;
    size_t smem = 0;
    bool L2 = false, L3 = false, noise = false;
    long long step = 0;
    long long cells = 0, active = 0, written = 0;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    long long launches = 0;
};

namespace {

constexpr int kEnsGraphSteps = 32;

using EnsKernel = void (*)(const CUtensorMap*, const tiled::EnsInstDev*, const tiled::EnsItem*, int, tiled::EnsCtl*,
                           int*);

template <bool kPair>
EnsKernel ens_kernel_t(bool L2, bool L3, bool N) {
    using namespace tiled;
    const int key = (L2 ? 1 : 0) | (L3 ? 2 : 0) | (N ? 4 : 0);
    switch (key) {
        case 0: return k_step_ensemble<false, false, false, kPair>;
        case 1: return k_step_ensemble<true, false, false, kPair>;
        case 2: return k_step_ensemble<false, true, false, kPair>;
        case 3: return k_step_ensemble<true, true, false, kPair>;
        case 4: return k_step_ensemble<false, false, true, kPair>;
        case 5: return k_step_ensemble<true, false, true, kPair>;
        case 6: return k_step_ensemble<false, true, true, kPair>;
        default: return k_step_ensemble<true, true, true, kPair>;
    }
}

// The ensemble runs the two-cell routine unless LDG_QSR_PAIR=0.
EnsKernel ens_kernel(bool L2, bool L3, bool N) {
    return tiled_pair_enabled() ? ens_kernel_t<true>(L2, L3, N) : ens_kernel_t<false>(L2, L3, N);
}
int ens_threads() { return tiled_pair_enabled() ? tiled::PAIR_THREADS : tiled::THREADS; }

void ens_drop_graph(ens_handle* h) {
    if (h->graph) cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
    h->graph_steps = 0;
}

// Work list of all instances split into chunks of `chunk` planes (instance-major, so CTAs that
// run together share halo planes of one droplet in L2), and the persistent grid size.
int ens_rechunk(ens_handle* h, int chunk) {
    std::vector<tiled::EnsItem> items;
    long long active = 0;
    for (size_t n = 0; n < h->inst.size(); ++n) {
        long long a = 0;
        for (const int4& t : tiled_items(h->inst[n]->tiled, chunk, &a))
            items.push_back(tiled::EnsItem{t.x, t.y, t.z, t.w, (int)n, 0, 0, 0});
        active += a;
    }
    h->active = active;
    if (h->d_items) cudaFree(h->d_items);
    h->d_items = nullptr;
    h->n_items = (int)items.size();
    if (h->n_items > 0) {
        int rc = alloc_or_fail((void**)&h->d_items, items.size() * sizeof(tiled::EnsItem));
        if (rc) return rc;
        LDG_CUDA(cudaMemcpy(h->d_items, items.data(), items.size() * sizeof(tiled::EnsItem), cudaMemcpyHostToDevice));
    }
    h->chunk = chunk;
    const EnsKernel k = ens_kernel(h->L2, h->L3, h->noise);
    LDG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->smem));
    int dev = 0, sms = 0, per_sm = 0;
    LDG_CUDA(cudaGetDevice(&dev));
    LDG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    LDG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, ens_threads(), h->smem));
    LDG_REQUIRE(per_sm > 0, LDG_ERR_CUDA, "ensemble: step kernel does not fit on an SM");
    h->grid = std::max(1, std::min(sms * per_sm, h->n_items));
    ens_drop_graph(h);
    return LDG_OK;
}

int ens_launch(ens_handle* h) {
    const EnsKernel k = ens_kernel(h->L2, h->L3, h->noise);
    k<<<h->grid, ens_threads(), h->smem, h->stream>>>(h->d_tms, h->d_inst, h->d_items, h->n_items, h->d_ctl,
                                                      h->d_err);
    LDG_LAUNCHED("k_step_ensemble");
    return LDG_OK;
}

// Captures kEnsGraphSteps launches of the step kernel into a CUDA graph and uploads it, so the
// first ens_step that replays it pays no instantiation cost. Capturing runs no kernel.
int ens_build_graph(ens_handle* h) {
    ens_drop_graph(h);
    if (h->n_items == 0) return LDG_OK;
    cudaGraph_t g = nullptr;
    LDG_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int rc = LDG_OK;
    for (int s = 0; s < kEnsGraphSteps && rc == LDG_OK; ++s) rc = ens_launch(h);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&h->graph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e == cudaSuccess) e = cudaGraphUpload(h->graph, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        ens_drop_graph(h);
        set_error(std::string("ensemble: graph capture failed: ") + cudaGetErrorString(e));
        return LDG_ERR_CUDA;
    }
    h->graph_steps = kEnsGraphSteps;
    return LDG_OK;
}

// Reads and clears the ensemble's device error word.
int ens_check(ens_handle* h) {
    int e = 0;
    LDG_CUDA(cudaMemcpyAsync(&e, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    LDG_CUDA(cudaStreamSynchronize(h->stream));
    if (e != 0) {
        LDG_CUDA(cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream));
        LDG_CUDA(cudaStreamSynchronize(h->stream));
        set_error("ensemble step: a bounded shared-memory pipeline wait gave up");
        return LDG_ERR_TIMEOUT;
    }
    return LDG_OK;
}

// Makes every instance's current buffer the input of the ensemble's next step.
void ens_sync_cur(ens_handle* h) {
    for (qsr_handle* q : h->inst) q->cur = (int)(h->step & 1);
}

// Observables of a droplet at the ensemble's current step: its protocol temperature, its shell
// order, slices Nz/2, thresholds 0.1 / 0.25.
qsr_observe_args ens_default_observe_args(const ens_handle* h, int instance) {
    qsr_observe_args a{};
    const tiled::EnsInstDev& D = h->host_inst[instance];
    a.T = tiled::ens_temperature(D, h->step);
    const double A = D.a3 * (a.T - D.T_star);
    a.S_shell = D.custom_shell ? D.S_custom : std::max(0.0, tiled::ens_S_eq(A, D.B, D.C));
    const int Nz = h->inst[instance]->p.Nz;
    a.defects_z_slice = Nz / 2;
    a.xi_z_slice = Nz / 2;
    a.defects_S_threshold = 0.1;
    a.defects_charge_cutoff = 0.25;
    a.xi_S_threshold = 0.1;
    a.want_defects = 1;
    a.want_xi = 1;
    return a;
}

int ens_set_step(ens_handle* h, long long step) {
    tiled::EnsCtl c{0, 0u, step};
    LDG_CUDA(cudaMemcpyAsync(h->d_ctl, &c, sizeof(c), cudaMemcpyHostToDevice, h->stream));
    LDG_CUDA(cudaStreamSynchronize(h->stream));
    h->step = step;
    ens_sync_cur(h);
    return LDG_OK;
}

}  // namespace

extern "C" {

int ens_destroy(ens_handle* h);

int ens_create(const ens_params* params, int n_instances, const ens_instance* instances, ens_handle** out) {
    clear_error();
    LDG_REQUIRE(params && instances && out, LDG_ERR_ARG, "ens_create: null argument");
    LDG_REQUIRE(n_instances >= 1, LDG_ERR_ARG, "ens_create: need at least one instance");
    const ens_params& p = *params;
    LDG_REQUIRE(p.dt > 0.0 && std::isfinite(p.dt), LDG_ERR_ARG, "ens_create: dt must be positive and finite");
    LDG_REQUIRE(p.protocol == 1 || p.protocol == 2, LDG_ERR_ARG, "ens_create: protocol must be 1 (step) or 2 (ramp)");
    for (int n = 0; n < n_instances; ++n) {
        LDG_REQUIRE(instances[n].N >= 3 && (instances[n].Ny == 0 || instances[n].Ny >= 3) &&
                        (instances[n].Nz == 0 || instances[n].Nz >= 3),
                    LDG_ERR_ARG, "ens_create: instance grid extents must be >= 3");
        LDG_REQUIRE(instances[n].pre_equil_iters >= 0 && instances[n].ramp_iters >= 0, LDG_ERR_ARG,
                    "ens_create: negative protocol length");
        LDG_REQUIRE(instances[n].noise_sigma >= 0.0, LDG_ERR_ARG, "ens_create: negative noise amplitude");
    }
    ens_handle* h = new (std::nothrow) ens_handle();
    LDG_REQUIRE(h, LDG_ERR_NOMEM, "ens_create: host allocation failed");
    h->p = p;
    cudaGetDevice(&h->device);
    h->desc.assign(instances, instances + n_instances);
    h->L2 = p.L2 != 0.0;
    h->L3 = p.L3 != 0.0;
    for (int n = 0; n < n_instances; ++n) {
        const ens_instance& d = instances[n];
        h->noise = h->noise || d.noise_sigma > 0.0;
        if (d.own_material) {
            h->L2 = h->L2 || d.L2 != 0.0;
            h->L3 = h->L3 || d.L3 != 0.0;
        }
    }
    int rc = LDG_OK;
    for (int n = 0; n < n_instances && rc == LDG_OK; ++n) {
        const ens_instance& d = instances[n];
        qsr_params q{};
        q.Nx = d.N;
        q.Ny = d.Ny > 0 ? d.Ny : d.N;
        q.Nz = d.Nz > 0 ? d.Nz : d.N;
        q.dx = p.dx; q.dy = p.dy; q.dz = p.dz;
        q.a = p.a; q.b = p.b; q.c = p.c; q.T_star = p.T_star; q.bulk_modechoice = p.bulk_modechoice;
        q.kappa = p.kappa; q.L1 = p.L1; q.L2 = p.L2; q.L3 = p.L3; q.W = p.W; q.gamma = p.gamma;
        q.droplet_radius_cells = d.droplet_radius_cells;
        if (d.own_material) {
            q.W = d.W; q.L2 = d.L2; q.L3 = d.L3;
        }
        qsr_handle* qh = nullptr;
        rc = qsr_create(&q, &qh);
        if (rc == LDG_OK) h->inst.push_back(qh);
    }
    if (rc != LDG_OK) {
        const std::string msg = ldg_last_error();
        ens_destroy(h);
        set_error(msg);
        return rc;
    }
    // One FP64 staging buffer for the host boundary of every droplet (calls are sequential and
    // each synchronises before returning), allocated here rather than on first use.
    {
        long long maxc = 0;
        for (qsr_handle* q : h->inst) maxc = std::max(maxc, q->ncells);
        rc = alloc_or_fail((void**)&h->stage, (size_t)maxc * 5 * sizeof(double));
        if (rc) {
            ens_destroy(h);
            return rc;
        }
        for (qsr_handle* q : h->inst) {
            q->stage = h->stage;
            q->stage_shared = true;
        }
    }
    // Per-instance descriptors: the static step constants plus the protocol.
    const double a3 = 3.0 * p.a;
    const double B = (p.bulk_modechoice == 1) ? (9.0 * p.b) / 2.0 : (27.0 * p.b) / 2.0;
    const double Cc = (p.bulk_modechoice == 1) ? (9.0 * p.c) / 2.0 : 9.0 * p.c;
    std::vector<CUtensorMap> tms(2 * (size_t)n_instances);
    h->host_inst.resize(n_instances);
    for (int n = 0; n < n_instances; ++n) {
        qsr_handle* qh = h->inst[n];
        const ens_instance& d = instances[n];
        tiled::EnsInstDev& D = h->host_inst[n];
        D.P = make_const(qh, d.T_high, 0.0, p.dt);
        D.P.qcap = (float)p.q_norm_cap;
        D.P.sigma = (float)d.noise_sigma;
        D.P.key0 = (uint32_t)d.seed;
        D.P.key1 = (uint32_t)(d.seed >> 32);
        D.P.instance = 0;
        D.q[0] = qh->q[0];
        D.q[1] = qh->q[1];
        D.flags = qh->flags;
        D.T_high = d.T_high; D.T_low = d.T_low;
        D.pre = d.pre_equil_iters; D.ramp = d.ramp_iters;
        D.protocol = p.protocol;
        D.custom_shell = p.boundary_custom ? 1 : 0;
        D.S_custom = p.boundary_S;
        D.a3 = a3; D.T_star = p.T_star; D.B = B; D.C = Cc;
        tms[2 * n] = qh->tiled.tmap[0];
        tms[2 * n + 1] = qh->tiled.tmap[1];
        h->cells += qh->ncells;
        h->active += qh->active_cells;
        h->written += qh->written_cells;
    }
    using namespace tiled;
    h->smem = tiled_pair_enabled() ? h->inst[0]->tiled.smem_bytes[2]
              : (h->L2 || h->L3)   ? h->inst[0]->tiled.smem_bytes[1]
                                   : h->inst[0]->tiled.smem_bytes[0];
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if ((rc = alloc_or_fail((void**)&h->d_tms, tms.size() * sizeof(CUtensorMap))) ||
        (rc = alloc_or_fail((void**)&h->d_inst, h->host_inst.size() * sizeof(EnsInstDev))) ||
        (rc = alloc_or_fail((void**)&h->d_ctl, sizeof(EnsCtl))) || (rc = alloc_or_fail((void**)&h->d_err, sizeof(int))) ||
        e != cudaSuccess) {
        if (e != cudaSuccess) {
            set_error(std::string("ens_create: ") + cudaGetErrorString(e));
            rc = LDG_ERR_CUDA;
        }
        ens_destroy(h);
        return rc;
    }
    e = cudaMemcpy(h->d_tms, tms.data(), tms.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(h->d_inst, h->host_inst.data(), h->host_inst.size() * sizeof(EnsInstDev), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(h->d_err, 0, sizeof(int));
    if (e != cudaSuccess) {
        set_error(std::string("ens_create: ") + cudaGetErrorString(e));
        ens_destroy(h);
        return LDG_ERR_CUDA;
    }
    if ((rc = ens_rechunk(h, tiled_default_chunk())) || (rc = ens_set_step(h, 0)) || (rc = ens_build_graph(h))) {
        const std::string msg = ldg_last_error();
        ens_destroy(h);
        set_error(msg);
        return rc;
    }
    *out = h;
    return LDG_OK;
}

int ens_initial_fields(ens_handle* h, int init_mode, double S0, double noise_amplitude) {
    clear_error();
    LDG_REQUIRE(h, LDG_ERR_ARG, "ens_initial_fields: null handle");
    DeviceGuard device_guard(h->device);
    LDG_CUDA(cudaStreamSynchronize(h->stream));
    std::vector<double> buf;
    for (size_t n = 0; n < h->inst.size(); ++n) {
        qsr_handle* qh = h->inst[n];
        buf.resize((size_t)qh->ncells * 5);
        int rc = qsr_initial_field(qh, init_mode, (long long)h->desc[n].seed, S0, noise_amplitude, buf.data());
        if (rc == LDG_OK) rc = qsr_upload(qh, buf.data());
        if (rc) return rc;
    }
    ens_sync_cur(h);
    return LDG_OK;
}

int ens_upload(ens_handle* h, int instance, const double* q) {
    clear_error();
    LDG_REQUIRE(h && q, LDG_ERR_ARG, "ens_upload: null argument");
    DeviceGuard device_guard(h->device);
    LDG_REQUIRE(instance >= 0 && instance < (int)h->inst.size(), LDG_ERR_ARG, "ens_upload: instance out of range");
    LDG_CUDA(cudaStreamSynchronize(h->stream));
    // qsr_upload fills both ping-pong buffers, so either parity of the step index reads it.
    const int rc = qsr_upload(h->inst[instance], q);
    ens_sync_cur(h);
    return rc;
}

int ens_download(ens_handle* h, int instance, double* q) {
    clear_error();
    LDG_REQUIRE(h && q, LDG_ERR_ARG, "ens_download: null argument");
    DeviceGuard device_guard(h->device);
    LDG_REQUIRE(instance >= 0 && instance < (int)h->inst.size(), LDG_ERR_ARG, "ens_download: instance out of range");
    int rc = ens_check(h);
    if (rc) return rc;
    ens_sync_cur(h);
    return qsr_download(h->inst[instance], q);
}

int ens_nematic(ens_handle* h, int instance, double* s_n) {
    clear_error();
    LDG_REQUIRE(h && s_n, LDG_ERR_ARG, "ens_nematic: null argument");
    DeviceGuard device_guard(h->device);
    LDG_REQUIRE(instance >= 0 && instance < (int)h->inst.size(), LDG_ERR_ARG, "ens_nematic: instance out of range");
    int rc = ens_check(h);
    if (rc) return rc;
    ens_sync_cur(h);
    return qsr_nematic(h->inst[instance], s_n);
}

int ens_step(ens_handle* h, int n_steps) {
    clear_error();
    LDG_REQUIRE(h, LDG_ERR_ARG, "ens_step: null handle");
    DeviceGuard device_guard(h->device);
    LDG_REQUIRE(n_steps >= 0, LDG_ERR_ARG, "ens_step: n_steps must be >= 0");
    for (qsr_handle* q : h->inst) LDG_REQUIRE(q->uploaded, LDG_ERR_STATE, "ens_step: an instance has no field");
    if (h->n_items == 0) {
        h->step += n_steps;
        return ens_set_step(h, h->step);
    }
    int left = n_steps;
    while (left >= kEnsGraphSteps) {
        if (!h->graph) {
            const int rc = ens_build_graph(h);
            if (rc) return rc;
        }
        LDG_CUDA(cudaGraphLaunch(h->graph, h->stream));
        h->launches += h->graph_steps;
        left -= h->graph_steps;
    }
    for (int s = 0; s < left; ++s) {
        int rc = ens_launch(h);
        if (rc) return rc;
        h->launches++;
    }
    h->step += n_steps;
    ens_sync_cur(h);
    return LDG_OK;
}

int ens_observe(ens_handle* h, int instance, const qsr_observe_args* args, qsr_observables* out) {
    clear_error();
    LDG_REQUIRE(h && out, LDG_ERR_ARG, "ens_observe: null argument");
    DeviceGuard device_guard(h->device);
    LDG_REQUIRE(instance >= 0 && instance < (int)h->inst.size(), LDG_ERR_ARG, "ens_observe: instance out of range");
    int rc = ens_check(h);
    if (rc) return rc;
    ens_sync_cur(h);
    const qsr_observe_args a = args ? *args : ens_default_observe_args(h, instance);
    return qsr_observe(h->inst[instance], &a, out);
}

int ens_observe_all(ens_handle* h, const qsr_observe_args* args, qsr_observables* out) {
    clear_error();
    LDG_REQUIRE(h && out, LDG_ERR_ARG, "ens_observe_all: null argument");
    DeviceGuard device_guard(h->device);
    int rc = ens_check(h);
    if (rc) return rc;
    ens_sync_cur(h);
    const size_t n = h->inst.size();
    if (!h->obs_host) {
        LDG_CUDA(cudaMallocHost((void**)&h->obs_host, n * (sizeof(ObsPartial) + sizeof(SlicePartial))));
    }
    ObsPartial* R = reinterpret_cast<ObsPartial*>(h->obs_host);
    SlicePartial* SR = reinterpret_cast<SlicePartial*>(R + n);
    std::vector<char> wd(n), wx(n);
    std::vector<qsr_observe_args> a(n);
    for (size_t i = 0; i < n; ++i) {
        a[i] = args ? args[i] : ens_default_observe_args(h, (int)i);
        std::memset(&SR[i], 0, sizeof(SlicePartial));
        bool d = false, x = false;
        // every droplet's reductions on the ensemble's stream, after its steps
        if ((rc = observe_enqueue(h->inst[i], &a[i], h->stream, &R[i], &SR[i], &d, &x))) return rc;
        wd[i] = d;
        wx[i] = x;
    }
    LDG_CUDA(cudaStreamSynchronize(h->stream));
    for (size_t i = 0; i < n; ++i) {
        if ((rc = tiled_check(h->inst[i]->tiled, h->stream))) return rc;
        observe_finish(h->inst[i], R[i], SR[i], wd[i] != 0, wx[i] != 0, &out[i]);
    }
    return LDG_OK;
}

long long ens_step_index(const ens_handle* h) { return h ? h->step : -1; }

int ens_geometry(const ens_handle* h, int instance, qsr_geometry_info* out) {
    clear_error();
    LDG_REQUIRE(h && out, LDG_ERR_ARG, "ens_geometry: null argument");
    LDG_REQUIRE(instance >= 0 && instance < (int)h->inst.size(), LDG_ERR_ARG, "ens_geometry: instance out of range");
    return qsr_geometry(h->inst[instance], out);
}

int ens_autotune(ens_handle* h, int trial_steps, int* chosen_chunk) {
    clear_error();
    LDG_REQUIRE(h, LDG_ERR_ARG, "ens_autotune: null handle");
    DeviceGuard device_guard(h->device);
    LDG_REQUIRE(trial_steps >= 1, LDG_ERR_ARG, "ens_autotune: trial_steps must be >= 1");
    for (qsr_handle* q : h->inst) LDG_REQUIRE(q->uploaded, LDG_ERR_STATE, "ens_autotune: an instance has no field");
    LDG_CUDA(cudaStreamSynchronize(h->stream));
    // Back up the current field of every instance (the other buffer differs only in cells
    // the next step rewrites).
    const long long step0 = h->step;
    const int w = (int)(step0 & 1);
    std::vector<float*> backup(h->inst.size(), nullptr);
    int rc = LDG_OK;
    for (size_t n = 0; n < h->inst.size() && rc == LDG_OK; ++n) {
        const size_t bytes = (size_t)h->inst[n]->sc * 5 * sizeof(float);
        rc = alloc_or_fail((void**)&backup[n], bytes);
        if (rc == LDG_OK && cudaMemcpyAsync(backup[n], h->inst[n]->q[w], bytes, cudaMemcpyDeviceToDevice, h->stream) !=
                                cudaSuccess) {
            set_error("ens_autotune: backup copy failed");
            rc = LDG_ERR_CUDA;
        }
    }
    const int candidates[] = {8, 12, 16, 24, 32, 48, 64};
    int best = h->chunk;
    float best_ms = std::numeric_limits<float>::infinity();
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (rc == LDG_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)) {
        set_error("ens_autotune: event creation failed");
        rc = LDG_ERR_CUDA;
    }
    for (int c : candidates) {
        if (rc != LDG_OK) break;
        if ((rc = ens_rechunk(h, c))) break;
        for (int s = 0; s < 2 && rc == LDG_OK; ++s) rc = ens_launch(h);
        if (rc) break;
        cudaEventRecord(e0, h->stream);
        for (int s = 0; s < trial_steps && rc == LDG_OK; ++s) rc = ens_launch(h);
        if (rc) break;
        cudaEventRecord(e1, h->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            set_error("ens_autotune: trial failed");
            rc = LDG_ERR_CUDA;
            break;
        }
        h->launches += 2 + trial_steps;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) { best_ms = ms; best = c; }
        if ((rc = ens_check(h))) break;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    // Restore the fields into both buffers and the step index, whatever happened above.
    for (size_t n = 0; n < h->inst.size(); ++n) {
        if (!backup[n]) continue;
        const size_t bytes = (size_t)h->inst[n]->sc * 5 * sizeof(float);
        cudaMemcpyAsync(h->inst[n]->q[0], backup[n], bytes, cudaMemcpyDeviceToDevice, h->stream);
        cudaMemcpyAsync(h->inst[n]->q[1], backup[n], bytes, cudaMemcpyDeviceToDevice, h->stream);
    }
    cudaStreamSynchronize(h->stream);
    for (float* b : backup) cudaFree(b);
    if (rc != LDG_OK) return rc;
    if ((rc = ens_rechunk(h, best))) return rc;
    if ((rc = ens_set_step(h, step0))) return rc;
    if ((rc = ens_build_graph(h))) return rc;
    if (chosen_chunk) *chosen_chunk = best;
    return LDG_OK;
}

long long ens_cells(const ens_handle* h) { return h ? h->cells : 0; }
long long ens_active_cells(const ens_handle* h) { return h ? h->active : 0; }
long long ens_written_cells(const ens_handle* h) { return h ? h->written : 0; }
void* ens_stream(ens_handle* h) { return h ? (void*)h->stream : nullptr; }
long long ens_launch_count(const ens_handle* h) {
    if (!h) return 0;
    long long n = h->launches;
    for (const qsr_handle* q : h->inst) n += q->launches;
    return n;
}

int ens_destroy(ens_handle* h) {
    if (!h) return LDG_OK;
    DeviceGuard device_guard(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    ens_drop_graph(h);
    for (qsr_handle* q : h->inst) qsr_destroy(q);
    cudaFree(h->stage);
    if (h->obs_host) cudaFreeHost(h->obs_host);
    cudaFree(h->d_tms); cudaFree(h->d_inst); cudaFree(h->d_items); cudaFree(h->d_ctl); cudaFree(h->d_err);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return LDG_OK;
}

}  // extern "C"
