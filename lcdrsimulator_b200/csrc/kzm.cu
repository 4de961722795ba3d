// Periodic bulk LdG solver (KZM_bulk_ldg drop-in): device kernels and the kzm_* C ABI.
//
// Device layout: FP32 SoA, x fastest (the reference's flatten order, KZM_bulk_ldg.cu:161-169),
// rows padded to a multiple of 4 floats. One fused kernel per step: periodic 7-point
// Laplacian, bulk field, traceless projection, Euler, Philox Langevin noise, optional cap.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <new>
#include <string>

#include "ldg_api_common.h"
#include "ldg_common.cuh"

using namespace ldg;

namespace {

constexpr double kPi = 3.14159265358979323846;

struct KzmConst {
    int Nx, Ny, Nz;
    int sy;          // row pitch (x fastest)
    long long sz;    // plane pitch
    long long sc;    // component pitch
    float ix2, iy2, iz2;
    float lap_c;     // -2 (1/dx^2 + 1/dy^2 + 1/dz^2): centre weight of the Laplacian
    float A, B, C, kappa, mob_dt, qcap, sigma;
    uint32_t key0, key1;
    long long step;
};

// One periodic step: block (32, 8) over (x, y), grid z over planes (KZM_bulk_ldg.cu:351-469).
template <bool kNoise>
__global__ void __launch_bounds__(256) k_kzm_step(const float* __restrict__ q, float* __restrict__ out, KzmConst P) {
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= P.Nx || y >= P.Ny) return;
    const int xp = (x + 1 == P.Nx) ? 0 : x + 1, xm = (x == 0) ? P.Nx - 1 : x - 1;
    const int yp = (y + 1 == P.Ny) ? 0 : y + 1, ym = (y == 0) ? P.Ny - 1 : y - 1;
    const int zp = (z + 1 == P.Nz) ? 0 : z + 1, zm = (z == 0) ? P.Nz - 1 : z - 1;
    const long long row = (long long)z * P.sz + (long long)y * P.sy;
    const long long id = row + x;
    const long long oxp = row + xp, oxm = row + xm;
    const long long oyp = (long long)z * P.sz + (long long)yp * P.sy + x;
    const long long oym = (long long)z * P.sz + (long long)ym * P.sy + x;
    const long long ozp = (long long)zp * P.sz + (long long)y * P.sy + x;
    const long long ozm = (long long)zm * P.sz + (long long)y * P.sy + x;
    float c[5], lap[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) {
        const float* b = q + m * P.sc;
        c[m] = __ldg(b + id);
        lap[m] = fmaf(P.ix2, __ldg(b + oxp) + __ldg(b + oxm),
                      fmaf(P.iy2, __ldg(b + oyp) + __ldg(b + oym),
                           fmaf(P.iz2, __ldg(b + ozp) + __ldg(b + ozm), P.lap_c * c[m])));
    }
    float h[6];
    bulk_field(c, P.A, P.B, P.C, h);
    h[0] -= P.kappa * lap[0];
    h[1] -= P.kappa * lap[3];
    h[2] += P.kappa * (lap[0] + lap[3]);
    h[3] -= P.kappa * lap[1];
    h[4] -= P.kappa * lap[2];
    h[5] -= P.kappa * lap[4];
    const float corr = (h[0] + h[1] + h[2]) * (1.0f / 3.0f);
    float u[5] = {c[0] - P.mob_dt * (h[0] - corr), c[1] - P.mob_dt * h[3], c[2] - P.mob_dt * h[4],
                  c[3] - P.mob_dt * (h[1] - corr), c[4] - P.mob_dt * h[5]};
    if (kNoise) {
        float g[5];
        const uint32_t cell = (uint32_t)(x + P.Nx * (y + P.Ny * z));
        normals5(cell, 0u, P.step, P.key0, P.key1, g);
#pragma unroll
        for (int m = 0; m < 5; ++m) u[m] += P.sigma * g[m];
    }
    if (P.qcap > 0.0f) {
        const float zz = -u[0] - u[3];
        const float tr = u[0] * u[0] + u[3] * u[3] + zz * zz + 2.0f * (u[1] * u[1] + u[2] * u[2] + u[4] * u[4]);
        const float qn = sqrtf(fmaxf(tr, 0.0f));
        if (qn > P.qcap && qn > 0.0f) {
            const float s = P.qcap / qn;
#pragma unroll
            for (int m = 0; m < 5; ++m) u[m] *= s;
        }
    }
#pragma unroll
    for (int m = 0; m < 5; ++m) out[m * P.sc + id] = u[m];
}

// The same step as k_kzm_step for a (32 x 8) column tile marching along z over a chunk of
// planes. Each thread keeps its column's planes z-1, z, z+1 in registers and prefetches
// z+2 and z+3; the x/y neighbours come from a shared (34 x 10) tile whose halo holds the
// periodically wrapped values (any N >= 2). Every input value is loaded about once from
// HBM (halo columns from L2) and every site is written once.
constexpr int KTX = 32, KTY = 8, KZC = 32;
template <bool kNoise>
__global__ void __launch_bounds__(KTX* KTY) k_kzm_step_tiled(const float* __restrict__ q, float* __restrict__ out,
                                                             KzmConst P) {
    __shared__ float s[5][KTY + 2][KTX + 2];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x0 = blockIdx.x * KTX, y0 = blockIdx.y * KTY, z0 = blockIdx.z * KZC;
    const int z1 = min(z0 + KZC, P.Nz);
    const int xr = x0 + tx, yr = y0 + ty;
    const bool valid = (xr < P.Nx) && (yr < P.Ny);
    const int x = xr % P.Nx, y = yr % P.Ny;
    const long long row = (long long)y * P.sy;
    const long long rowm = (long long)((y0 + P.Ny - 1) % P.Ny) * P.sy;   // halo row y0-1
    const long long rowp = (long long)((y0 + KTY) % P.Ny) * P.sy;        // halo row y0+KTY
    const int xm = (x0 + P.Nx - 1) % P.Nx, xp = (x0 + KTX) % P.Nx;       // halo columns
    // z stays within [-1, 2 Nz) here (Nz >= 2), so one compare-and-add wraps it.
    auto zw = [&](int z) { return z < 0 ? z + P.Nz : (z >= P.Nz ? z - P.Nz : z); };
    auto load5 = [&](int z, float v[5]) {
        const long long o = (long long)zw(z) * P.sz + row + x;
#pragma unroll
        for (int m = 0; m < 5; ++m) v[m] = __ldg(q + m * P.sc + o);
    };
    float qm[5], qc[5], qp[5], qn[5], qn2[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    load5(z0 - 1, qm);
    load5(z0, qc);
    load5(z0 + 1, qp);
    load5(z0 + 2, qn);
    const uint32_t cell_base = (uint32_t)(x + P.Nx * y);
    for (int z = z0; z < z1; ++z) {
        if (z + 3 < z1 + 1) load5(z + 3, qn2);
        const long long pz = (long long)zw(z) * P.sz;
#pragma unroll
        for (int m = 0; m < 5; ++m) s[m][ty + 1][tx + 1] = qc[m];
        if (ty == 0) {
#pragma unroll
            for (int m = 0; m < 5; ++m) s[m][0][tx + 1] = __ldg(q + m * P.sc + pz + rowm + x);
        }
        if (ty == KTY - 1) {
#pragma unroll
            for (int m = 0; m < 5; ++m) s[m][KTY + 1][tx + 1] = __ldg(q + m * P.sc + pz + rowp + x);
        }
        if (tx == 0) {
#pragma unroll
            for (int m = 0; m < 5; ++m) s[m][ty + 1][0] = __ldg(q + m * P.sc + pz + row + xm);
        }
        if (tx == KTX - 1) {
#pragma unroll
            for (int m = 0; m < 5; ++m) s[m][ty + 1][KTX + 1] = __ldg(q + m * P.sc + pz + row + xp);
        }
        __syncthreads();
        if (valid) {
            float lap[5];
#pragma unroll
            for (int m = 0; m < 5; ++m) {
                const float c = qc[m];
                lap[m] = fmaf(P.ix2, s[m][ty + 1][tx + 2] + s[m][ty + 1][tx],
                              fmaf(P.iy2, s[m][ty + 2][tx + 1] + s[m][ty][tx + 1],
                                   fmaf(P.iz2, qp[m] + qm[m], P.lap_c * c)));
            }
            float h[6];
            bulk_field(qc, P.A, P.B, P.C, h);
            h[0] -= P.kappa * lap[0];
            h[1] -= P.kappa * lap[3];
            h[2] += P.kappa * (lap[0] + lap[3]);
            h[3] -= P.kappa * lap[1];
            h[4] -= P.kappa * lap[2];
            h[5] -= P.kappa * lap[4];
            const float corr = (h[0] + h[1] + h[2]) * (1.0f / 3.0f);
            float u[5] = {qc[0] - P.mob_dt * (h[0] - corr), qc[1] - P.mob_dt * h[3], qc[2] - P.mob_dt * h[4],
                          qc[3] - P.mob_dt * (h[1] - corr), qc[4] - P.mob_dt * h[5]};
            if (kNoise) {
                float g[5];
                normals5(cell_base + (uint32_t)P.Nx * (uint32_t)P.Ny * (uint32_t)z, 0u, P.step, P.key0, P.key1, g);
#pragma unroll
                for (int m = 0; m < 5; ++m) u[m] += P.sigma * g[m];
            }
            if (P.qcap > 0.0f) {
                const float zz = -u[0] - u[3];
                const float tr = u[0] * u[0] + u[3] * u[3] + zz * zz + 2.0f * (u[1] * u[1] + u[2] * u[2] + u[4] * u[4]);
                const float qn_ = sqrtf(fmaxf(tr, 0.0f));
                if (qn_ > P.qcap && qn_ > 0.0f) {
                    const float sc = P.qcap / qn_;
#pragma unroll
                    for (int m = 0; m < 5; ++m) u[m] *= sc;
                }
            }
#pragma unroll
            for (int m = 0; m < 5; ++m) out[m * P.sc + pz + row + x] = u[m];
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < 5; ++m) {
            qm[m] = qc[m];
            qc[m] = qp[m];
            qp[m] = qn[m];
            qn[m] = qn2[m];
        }
    }
}

// Asynchronous-copy variant: every plane of the tile plus its periodically wrapped halo is
// fetched with cp.async (4-byte copies, any wrapped address) into a 5-plane shared ring two
// planes ahead of use, so no thread waits on a global load inside the plane loop; x, y and z
// neighbours all come from shared memory; one CTA barrier per plane.
constexpr int KRING = 5;
constexpr int KPS = (KTY + 2) * (KTX + 2);  // floats per component plane of the ring
__device__ __forceinline__ void cp_async4(float* sdst, const float* gsrc) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(sdst)),
                 "l"(gsrc)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <bool kNoise>
__global__ void __launch_bounds__(KTX* KTY) k_kzm_step_async(const float* __restrict__ q, float* __restrict__ out,
                                                             KzmConst P) {
    extern __shared__ __align__(16) float ring[];  // [KRING][5][KTY+2][KTX+2]
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x0 = blockIdx.x * KTX, y0 = blockIdx.y * KTY, z0 = blockIdx.z * KZC;
    const int z1 = min(z0 + KZC, P.Nz);
    const int xr = x0 + tx, yr = y0 + ty;
    const bool valid = (xr < P.Nx) && (yr < P.Ny);
    const int x = xr % P.Nx, y = yr % P.Ny;
    const long long g_c = (long long)y * P.sy + x;
    const int s_c = (ty + 1) * (KTX + 2) + tx + 1;
    // Flat copy list: the 5 x (KTY+2) x (KTX+2) ring entries of a plane spread over the CTA's
    // threads; each thread's (global in-plane offset, shared offset) pairs are the same for every
    // plane, so they are formed once here (wrapped periodically).
    constexpr int NE = 5 * KPS;
    constexpr int PER = (NE + KTX * KTY - 1) / (KTX * KTY);
    const int tid = ty * KTX + tx;
    long long goff[PER];
    int soff[PER];
#pragma unroll
    for (int t = 0; t < PER; ++t) {
        const int e = tid + t * KTX * KTY;
        const int m = e / KPS, cell = e - m * KPS;
        const int r = cell / (KTX + 2), cc = cell - r * (KTX + 2);
        const int gx = (x0 - 1 + cc + P.Nx) % P.Nx, gy = (y0 - 1 + r + P.Ny) % P.Ny;
        goff[t] = (long long)min(m, 4) * P.sc + (long long)gy * P.sy + gx;
        soff[t] = e;
    }
    auto zw = [&](int z) { return z < 0 ? z + P.Nz : (z >= P.Nz ? z - P.Nz : z); };
    auto issue = [&](int p) {
        float* dst = ring + ((p + KRING) % KRING) * NE;
        const float* src = q + (long long)zw(p) * P.sz;
#pragma unroll
        for (int t = 0; t < PER; ++t)
            if (t < PER - 1 || soff[t] < NE) cp_async4(dst + soff[t], src + goff[t]);
    };
    // Prologue: planes z0-1 .. z0+2, one commit group each.
    for (int p = z0 - 1; p <= z0 + 2; ++p) {
        issue(p);
        cp_async_commit();
    }
    const uint32_t cell_base = (uint32_t)(x + P.Nx * y);
    for (int z = z0; z < z1; ++z) {
        cp_async_wait<1>();  // all groups but the newest (plane z+2): planes z-1 .. z+1 are in
        __syncthreads();     // every thread's copies visible; every thread done with plane z-2
        if (z + 3 <= z1) issue(z + 3);  // into the slot of plane z-2
        cp_async_commit();
        if (valid) {
            const float* pm = ring + ((z - 1 + KRING) % KRING) * 5 * KPS;
            const float* pc = ring + ((z + KRING) % KRING) * 5 * KPS;
            const float* pp = ring + ((z + 1) % KRING) * 5 * KPS;
            float c[5], lap[5];
#pragma unroll
            for (int m = 0; m < 5; ++m) {
                const float* s = pc + m * KPS + s_c;
                c[m] = s[0];
                // sum_a (Q[+1] + Q[-1]) / da^2 - 2 Q sum_a 1/da^2 as one fused chain
                lap[m] = fmaf(P.ix2, s[1] + s[-1],
                              fmaf(P.iy2, s[KTX + 2] + s[-(KTX + 2)],
                                   fmaf(P.iz2, pp[m * KPS + s_c] + pm[m * KPS + s_c], P.lap_c * c[m])));
            }
            float h[6];
            bulk_field(c, P.A, P.B, P.C, h);
            h[0] -= P.kappa * lap[0];
            h[1] -= P.kappa * lap[3];
            h[2] += P.kappa * (lap[0] + lap[3]);
            h[3] -= P.kappa * lap[1];
            h[4] -= P.kappa * lap[2];
            h[5] -= P.kappa * lap[4];
            const float corr = (h[0] + h[1] + h[2]) * (1.0f / 3.0f);
            float u[5] = {c[0] - P.mob_dt * (h[0] - corr), c[1] - P.mob_dt * h[3], c[2] - P.mob_dt * h[4],
                          c[3] - P.mob_dt * (h[1] - corr), c[4] - P.mob_dt * h[5]};
            if (kNoise) {
                float g[5];
                normals5(cell_base + (uint32_t)P.Nx * (uint32_t)P.Ny * (uint32_t)z, 0u, P.step, P.key0, P.key1, g);
#pragma unroll
                for (int m = 0; m < 5; ++m) u[m] += P.sigma * g[m];
            }
            if (P.qcap > 0.0f) {
                const float zz = -u[0] - u[3];
                const float tr = u[0] * u[0] + u[3] * u[3] + zz * zz + 2.0f * (u[1] * u[1] + u[2] * u[2] + u[4] * u[4]);
                const float qn_ = sqrtf(fmaxf(tr, 0.0f));
                if (qn_ > P.qcap && qn_ > 0.0f) {
                    const float sc = P.qcap / qn_;
#pragma unroll
                    for (int m = 0; m < 5; ++m) u[m] *= sc;
                }
            }
            float* o = out + (long long)z * P.sz + g_c;
#pragma unroll
            for (int m = 0; m < 5; ++m) o[m * P.sc] = u[m];
        }
    }
    cp_async_wait<0>();  // no copy into this CTA's shared memory outlives it
}

// Two sites per thread: 128 threads over the same (32 x 8) tile and plane loop as
// k_kzm_step_async, thread (tx, ty) updating rows ty and ty + 4. For Nx a multiple of 4 (so every
// row pitch, plane pitch and component pitch is too) each ring row holds the 40 columns
// x0 - 4 .. x0 + 35 and is fetched as ten 16-byte copies whose sources are 16-byte aligned and
// either wholly inside the box or wholly wrapped (x0 is a multiple of 32): 500 copies per plane
// instead of 1700 four-byte ones. The Laplacian, bulk field and update of both sites run as one
// packed FP32 instruction stream (FFMA2 / FADD2 / FMUL2: per site the same fused operations as
// the one-site kernel); the noise draw, the cap and the stores stay per site.
constexpr int KPT = KTX * KTY / 2;
constexpr int KROW2 = KTX + 8;               // ring row of the two-site kernel: x0 - 4 .. x0 + 35
constexpr int KPS2 = (KTY + 2) * KROW2;      // floats per component plane
constexpr size_t kRingBytes2 = (size_t)KRING * 5 * KPS2 * sizeof(float);
__device__ __forceinline__ void cp_async16(float* sdst, const float* gsrc) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(sdst)),
                 "l"(gsrc)
                 : "memory");
}
template <bool kNoise>
__global__ void __launch_bounds__(KPT) k_kzm_step_pair(const float* __restrict__ q, float* __restrict__ out,
                                                       KzmConst P) {
    extern __shared__ __align__(16) float ring[];  // [KRING][5][KTY+2][KROW2]
    constexpr int ROW = KROW2;
    constexpr int KPS = KPS2;
    const int tid = threadIdx.x;
    const int tx = tid & 31, ty = tid >> 5;
    const int x0 = blockIdx.x * KTX, y0 = blockIdx.y * KTY, z0 = blockIdx.z * KZC;
    const int z1 = min(z0 + KZC, P.Nz);
    const int xr = x0 + tx;
    const int x = xr % P.Nx;
    bool valid[2];
    long long g_c[2];
    uint32_t cell_base[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int yr = y0 + ty + 4 * r;
        valid[r] = (xr < P.Nx) && (yr < P.Ny);
        const int y = yr % P.Ny;
        g_c[r] = (long long)y * P.sy + x;
        cell_base[r] = (uint32_t)(x + P.Nx * y);
    }
    const int s_c = (ty + 1) * ROW + tx + 4;  // row ty; row ty + 4 is 4 * ROW further
    constexpr int NE = 5 * KPS;               // floats per ring plane
    constexpr int NCH = NE / 4;               // 16-byte chunks per ring plane
    constexpr int PER = (NCH + KPT - 1) / KPT;
    long long goff[PER];
#pragma unroll
    for (int t = 0; t < PER; ++t) {
        const int e = min(tid + t * KPT, NCH - 1);
        const int m = e / (KPS / 4), rem = e - m * (KPS / 4);
        const int r = rem / (ROW / 4), c4 = rem - r * (ROW / 4);
        const int gx = (x0 - 4 + 4 * c4 + P.Nx) % P.Nx, gy = (y0 - 1 + r + P.Ny) % P.Ny;
        goff[t] = (long long)m * P.sc + (long long)gy * P.sy + gx;
    }
    auto zw = [&](int z) { return z < 0 ? z + P.Nz : (z >= P.Nz ? z - P.Nz : z); };
    auto issue = [&](int p) {
        float* dst = ring + ((p + KRING) % KRING) * NE;
        const float* src = q + (long long)zw(p) * P.sz;
#pragma unroll
        for (int t = 0; t < PER; ++t)
            if (t < PER - 1 || tid + t * KPT < NCH) cp_async16(dst + 4 * (tid + t * KPT), src + goff[t]);
    };
    for (int p = z0 - 1; p <= z0 + 2; ++p) {
        issue(p);
        cp_async_commit();
    }
    const bool any_valid = valid[0] || valid[1];
    for (int z = z0; z < z1; ++z) {
        cp_async_wait<1>();  // planes z-1 .. z+1 are in
        __syncthreads();     // every thread's copies visible; every thread done with plane z-2
        if (z + 3 <= z1) issue(z + 3);
        cp_async_commit();
        if (any_valid) {
            const float* pm = ring + ((z - 1 + KRING) % KRING) * NE + s_c;
            const float* pc = ring + ((z + KRING) % KRING) * NE + s_c;
            const float* pp = ring + ((z + 1) % KRING) * NE + s_c;
            auto at = [](const float* b, int off) { return mk2(b[off], b[off + 4 * ROW]); };
            F2 c[5], lap[5];
#pragma unroll
            for (int m = 0; m < 5; ++m) {
                const float* sc = pc + m * KPS;
                c[m] = at(sc, 0);
                lap[m] = vfma(P.ix2, at(sc, 1) + at(sc, -1),
                              vfma(P.iy2, at(sc, ROW) + at(sc, -ROW),
                                   vfma(P.iz2, at(pp + m * KPS, 0) + at(pm + m * KPS, 0), P.lap_c * c[m])));
            }
            F2 h[6];
            bulk_field_pair(c, P.A, P.B, P.C, h);
            h[0] = vfma(-P.kappa, lap[0], h[0]);
            h[1] = vfma(-P.kappa, lap[3], h[1]);
            h[2] = vfma(P.kappa, lap[0] + lap[3], h[2]);
            h[3] = vfma(-P.kappa, lap[1], h[3]);
            h[4] = vfma(-P.kappa, lap[2], h[4]);
            h[5] = vfma(-P.kappa, lap[4], h[5]);
            const F2 corr = (1.0f / 3.0f) * (h[0] + h[1] + h[2]);
            const float nmd = -P.mob_dt;
            F2 u[5] = {vfma(nmd, h[0] - corr, c[0]), vfma(nmd, h[3], c[1]), vfma(nmd, h[4], c[2]),
                       vfma(nmd, h[1] - corr, c[3]), vfma(nmd, h[5], c[4])};
            float v[2][5];
#pragma unroll
            for (int m = 0; m < 5; ++m) {
                v[0][m] = u[m].v.x;
                v[1][m] = u[m].v.y;
            }
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                if (!valid[r]) continue;
                if (kNoise) {
                    float g[5];
                    normals5(cell_base[r] + (uint32_t)P.Nx * (uint32_t)P.Ny * (uint32_t)z, 0u, P.step, P.key0,
                             P.key1, g);
#pragma unroll
                    for (int m = 0; m < 5; ++m) v[r][m] = fmaf(P.sigma, g[m], v[r][m]);
                }
                if (P.qcap > 0.0f) {
                    const float zz = -v[r][0] - v[r][3];
                    const float tr = v[r][0] * v[r][0] + v[r][3] * v[r][3] + zz * zz +
                                     2.0f * (v[r][1] * v[r][1] + v[r][2] * v[r][2] + v[r][4] * v[r][4]);
                    const float qn_ = sqrtf(fmaxf(tr, 0.0f));
                    if (qn_ > P.qcap && qn_ > 0.0f) {
                        const float sc = P.qcap / qn_;
#pragma unroll
                        for (int m = 0; m < 5; ++m) v[r][m] *= sc;
                    }
                }
                float* o = out + (long long)z * P.sz + g_c[r];
#pragma unroll
                for (int m = 0; m < 5; ++m) o[m * P.sc] = v[r][m];
            }
        }
    }
    cp_async_wait<0>();  // no copy into this CTA's shared memory outlives it
}

__global__ void k_kzm_from_aos(const double* __restrict__ aos, float* __restrict__ a, KzmConst P) {
    const long long n = (long long)P.Nx * P.Ny * P.Nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % P.Nx);
        const long long r = t / P.Nx;
        const int y = (int)(r % P.Ny);
        const int z = (int)(r / P.Ny);
        const long long id = (long long)z * P.sz + (long long)y * P.sy + x;
#pragma unroll
        for (int m = 0; m < 5; ++m) a[m * P.sc + id] = (float)aos[5 * t + m];
    }
}

__global__ void k_kzm_to_aos(const float* __restrict__ a, double* __restrict__ aos, KzmConst P) {
    const long long n = (long long)P.Nx * P.Ny * P.Nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % P.Nx);
        const long long r = t / P.Nx;
        const int y = (int)(r % P.Ny);
        const int z = (int)(r / P.Ny);
        const long long id = (long long)z * P.sz + (long long)y * P.sy + x;
#pragma unroll
        for (int m = 0; m < 5; ++m) aos[5 * t + m] = (double)a[m * P.sc + id];
    }
}

struct KzmPartial {
    double bulk, elastic, qint, gint, S_sum, S_max, line;
    unsigned long long used, defects;
};

constexpr int kThreads = 256;
constexpr int kBlocks = 148 * 8;

template <class T>
__device__ __forceinline__ T bsum(T v, T* sh) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    T r = 0;
    if (threadIdx.x == 0)
        for (int x = 0; x < (int)(blockDim.x >> 5); ++x) r += sh[x];
    return r;
}

__device__ __forceinline__ double bmax(double v, double* sh) {
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

struct KzmObsConst {
    KzmConst P;
    double A, B, C, kappa, cv, ix, iy, iz;
};

// Pass 1 (KZM_bulk_ldg.cu:564-632): bulk and forward-difference elastic energy, |Q|^2 and
// |grad Q|^2 integrals, nematic (S, n) per site into an FP64 scratch field.
__global__ void __launch_bounds__(kThreads) k_kzm_obs_sites(const float* __restrict__ q, KzmObsConst O,
                                                            double4* __restrict__ nf, KzmPartial* __restrict__ part) {
    const KzmConst& P = O.P;
    const long long n = (long long)P.Nx * P.Ny * P.Nz;
    KzmPartial a{};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % P.Nx);
        const long long r = t / P.Nx;
        const int y = (int)(r % P.Ny);
        const int z = (int)(r / P.Ny);
        const long long id = (long long)z * P.sz + (long long)y * P.sy + x;
        const long long px = (long long)z * P.sz + (long long)y * P.sy + ((x + 1) % P.Nx);
        const long long py = (long long)z * P.sz + (long long)((y + 1) % P.Ny) * P.sy + x;
        const long long pz = (long long)((z + 1) % P.Nz) * P.sz + (long long)y * P.sy + x;
        double c[5], d[6][3];
#pragma unroll
        for (int m = 0; m < 5; ++m) {
            const float* b = q + m * P.sc;
            c[m] = (double)b[id];
            d[m][0] = ((double)b[px] - c[m]) * O.ix;
            d[m][1] = ((double)b[py] - c[m]) * O.iy;
            d[m][2] = ((double)b[pz] - c[m]) * O.iz;
        }
#pragma unroll
        for (int w = 0; w < 3; ++w) d[5][w] = -(d[0][w] + d[3][w]);
        const double Qxx = c[0], Qxy = c[1], Qxz = c[2], Qyy = c[3], Qyz = c[4], Qzz = -Qxx - Qyy;
        const double q2xx = Qxx * Qxx + Qxy * Qxy + Qxz * Qxz;
        const double q2xy = Qxx * Qxy + Qxy * Qyy + Qxz * Qyz;
        const double q2xz = Qxx * Qxz + Qxy * Qyz + Qxz * Qzz;
        const double q2yy = Qxy * Qxy + Qyy * Qyy + Qyz * Qyz;
        const double q2yz = Qxy * Qxz + Qyy * Qyz + Qyz * Qzz;
        const double q2zz = Qxz * Qxz + Qyz * Qyz + Qzz * Qzz;
        const double trQ2 = Qxx * Qxx + Qyy * Qyy + Qzz * Qzz + 2.0 * (Qxy * Qxy + Qxz * Qxz + Qyz * Qyz);
        const double trQ3 = Qxx * q2xx + Qxy * q2xy + Qxz * q2xz + Qxy * q2xy + Qyy * q2yy + Qyz * q2yz +
                            Qxz * q2xz + Qyz * q2yz + Qzz * q2zz;
        a.bulk += ((O.A / 2.0) * trQ2 - (O.B / 3.0) * trQ3 + (O.C / 4.0) * trQ2 * trQ2) * O.cv;
        double g2 = 0.0;
#pragma unroll
        for (int m = 0; m < 6; ++m) {
            const double s = d[m][0] * d[m][0] + d[m][1] * d[m][1] + d[m][2] * d[m][2];
            g2 += (m == 1 || m == 2 || m == 4) ? 2.0 * s : s;
        }
        a.gint += g2 * O.cv;
        a.elastic += 0.5 * O.kappa * g2 * O.cv;
        a.qint += trQ2 * O.cv;
        const Nematic f = nematic64(c, 1e-12, Nematic{0.0, 1.0, 0.0, 0.0});
        nf[t] = make_double4(f.S, f.nx, f.ny, f.nz);
        a.S_sum += f.S;
        a.S_max = fmax(a.S_max, f.S);
    }
    __shared__ double shd[kThreads / 32];
    KzmPartial res{};
    res.bulk = bsum(a.bulk, shd);
    res.elastic = bsum(a.elastic, shd);
    res.qint = bsum(a.qint, shd);
    res.gint = bsum(a.gint, shd);
    res.S_sum = bsum(a.S_sum, shd);
    res.S_max = bmax(a.S_max, shd);
    if (threadIdx.x == 0) part[blockIdx.x] = res;
}

// Pass 1 on a caller-owned device field in the reference layout (AoS FP64, x fastest).
__global__ void __launch_bounds__(kThreads) k_kzm_obs_sites_aos(const double* __restrict__ q, KzmObsConst O,
                                                                double4* __restrict__ nf,
                                                                KzmPartial* __restrict__ part) {
    const KzmConst& P = O.P;
    const long long n = (long long)P.Nx * P.Ny * P.Nz;
    KzmPartial a{};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % P.Nx);
        const long long r = t / P.Nx;
        const int y = (int)(r % P.Ny);
        const int z = (int)(r / P.Ny);
        const long long px = (long long)((x + 1) % P.Nx) + (long long)P.Nx * ((long long)y + (long long)P.Ny * z);
        const long long py = (long long)x + (long long)P.Nx * ((long long)((y + 1) % P.Ny) + (long long)P.Ny * z);
        const long long pz = (long long)x + (long long)P.Nx * ((long long)y + (long long)P.Ny * ((z + 1) % P.Nz));
        double c[5], d[6][3];
#pragma unroll
        for (int m = 0; m < 5; ++m) {
            c[m] = q[5 * t + m];
            d[m][0] = (q[5 * px + m] - c[m]) * O.ix;
            d[m][1] = (q[5 * py + m] - c[m]) * O.iy;
            d[m][2] = (q[5 * pz + m] - c[m]) * O.iz;
        }
#pragma unroll
        for (int w = 0; w < 3; ++w) d[5][w] = -(d[0][w] + d[3][w]);
        const double Qxx = c[0], Qxy = c[1], Qxz = c[2], Qyy = c[3], Qyz = c[4], Qzz = -Qxx - Qyy;
        const double q2xx = Qxx * Qxx + Qxy * Qxy + Qxz * Qxz;
        const double q2xy = Qxx * Qxy + Qxy * Qyy + Qxz * Qyz;
        const double q2xz = Qxx * Qxz + Qxy * Qyz + Qxz * Qzz;
        const double q2yy = Qxy * Qxy + Qyy * Qyy + Qyz * Qyz;
        const double q2yz = Qxy * Qxz + Qyy * Qyz + Qyz * Qzz;
        const double q2zz = Qxz * Qxz + Qyz * Qyz + Qzz * Qzz;
        const double trQ2 = Qxx * Qxx + Qyy * Qyy + Qzz * Qzz + 2.0 * (Qxy * Qxy + Qxz * Qxz + Qyz * Qyz);
        const double trQ3 = Qxx * q2xx + Qxy * q2xy + Qxz * q2xz + Qxy * q2xy + Qyy * q2yy + Qyz * q2yz +
                            Qxz * q2xz + Qyz * q2yz + Qzz * q2zz;
        a.bulk += ((O.A / 2.0) * trQ2 - (O.B / 3.0) * trQ3 + (O.C / 4.0) * trQ2 * trQ2) * O.cv;
        double g2 = 0.0;
#pragma unroll
        for (int m = 0; m < 6; ++m) {
            const double s = d[m][0] * d[m][0] + d[m][1] * d[m][1] + d[m][2] * d[m][2];
            g2 += (m == 1 || m == 2 || m == 4) ? 2.0 * s : s;
        }
        a.gint += g2 * O.cv;
        a.elastic += 0.5 * O.kappa * g2 * O.cv;
        a.qint += trQ2 * O.cv;
        const Nematic f = nematic64(c, 1e-12, Nematic{0.0, 1.0, 0.0, 0.0});
        nf[t] = make_double4(f.S, f.nx, f.ny, f.nz);
        a.S_sum += f.S;
        a.S_max = fmax(a.S_max, f.S);
    }
    __shared__ double shd[kThreads / 32];
    KzmPartial res{};
    res.bulk = bsum(a.bulk, shd);
    res.elastic = bsum(a.elastic, shd);
    res.qint = bsum(a.qint, shd);
    res.gint = bsum(a.gint, shd);
    res.S_sum = bsum(a.S_sum, shd);
    res.S_max = bmax(a.S_max, shd);
    if (threadIdx.x == 0) part[blockIdx.x] = res;
}

__device__ __forceinline__ double wrap_pi_loop(double d) {
    // wrap_to_pi of KZM_bulk_ldg.cu:471-479.
    while (d <= -kPi) d += 2.0 * kPi;
    while (d > kPi) d -= 2.0 * kPi;
    return d;
}

__device__ __forceinline__ bool project_plane(const double4& f, int plane, double& u, double& v) {
    // project_to_plane (KZM_bulk_ldg.cu:481-499).
    if (plane == 0) { u = f.y; v = f.z; }
    else if (plane == 1) { u = f.z; v = f.w; }
    else { u = f.y; v = f.w; }
    const double nrm = sqrt(u * u + v * v);
    if (!(nrm > 1e-8)) return false;
    u /= nrm;
    v /= nrm;
    return true;
}

// plaquette_charge (KZM_bulk_ldg.cu:501-541): 0 unused, 1 used, 2 defect.
__device__ __forceinline__ int plaquette(const double4& a, const double4& b, const double4& c, const double4& d,
                                         int plane, double thr, double cut) {
    if (!(isfinite(a.x) && isfinite(b.x) && isfinite(c.x) && isfinite(d.x))) return 0;
    if (!(a.x > thr && b.x > thr && c.x > thr && d.x > thr)) return 0;
    double ua, va, ub, vb, uc, vc, ud, vd;
    if (!project_plane(a, plane, ua, va) || !project_plane(b, plane, ub, vb) || !project_plane(c, plane, uc, vc) ||
        !project_plane(d, plane, ud, vd))
        return 0;
    const double pa = 2.0 * atan2(va, ua), pb = 2.0 * atan2(vb, ub), pc = 2.0 * atan2(vc, uc), pd = 2.0 * atan2(vd, ud);
    const double dsum = wrap_pi_loop(pb - pa) + wrap_pi_loop(pc - pb) + wrap_pi_loop(pd - pc) + wrap_pi_loop(pa - pd);
    const double s = 0.5 * (dsum / (2.0 * kPi));
    return (fabs(s) > cut) ? 2 : 1;
}

// Pass 2 (KZM_bulk_ldg.cu:634-689): three plaquette orientations per site, line length.
__global__ void __launch_bounds__(kThreads) k_kzm_obs_plaq(const double4* __restrict__ nf, KzmObsConst O, double thr,
                                                           double cut, double dx, double dy, double dz,
                                                           KzmPartial* __restrict__ part) {
    const KzmConst& P = O.P;
    const long long n = (long long)P.Nx * P.Ny * P.Nz;
    KzmPartial a{};
    auto at = [&](int x, int y, int z) { return nf[(long long)x + (long long)P.Nx * ((long long)y + (long long)P.Ny * z)]; };
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % P.Nx);
        const long long r = t / P.Nx;
        const int y = (int)(r % P.Ny);
        const int z = (int)(r / P.Ny);
        const int xp = (x + 1) % P.Nx, yp = (y + 1) % P.Ny, zp = (z + 1) % P.Nz;
        const double4 f000 = nf[t], f100 = at(xp, y, z), f110 = at(xp, yp, z), f010 = at(x, yp, z);
        const double4 f001 = at(x, y, zp), f101 = at(xp, y, zp), f011 = at(x, yp, zp);
        int res = plaquette(f000, f100, f110, f010, 0, thr, cut);
        if (res) { a.used++; if (res == 2) { a.defects++; a.line += dz; } }
        res = plaquette(f000, f010, f011, f001, 1, thr, cut);
        if (res) { a.used++; if (res == 2) { a.defects++; a.line += dx; } }
        res = plaquette(f000, f100, f101, f001, 2, thr, cut);
        if (res) { a.used++; if (res == 2) { a.defects++; a.line += dy; } }
    }
    __shared__ double shd[kThreads / 32];
    __shared__ unsigned long long shu[kThreads / 32];
    KzmPartial res{};
    res.line = bsum(a.line, shd);
    res.used = bsum(a.used, shu);
    res.defects = bsum(a.defects, shu);
    if (threadIdx.x == 0) {
        part[blockIdx.x].line = res.line;
        part[blockIdx.x].used = res.used;
        part[blockIdx.x].defects = res.defects;
    }
}

__global__ void __launch_bounds__(kThreads) k_kzm_obs_final(const KzmPartial* __restrict__ part, int n,
                                                            KzmPartial* __restrict__ out) {
    KzmPartial a{};
    for (int b = threadIdx.x; b < n; b += blockDim.x) {
        const KzmPartial& p = part[b];
        a.bulk += p.bulk; a.elastic += p.elastic; a.qint += p.qint; a.gint += p.gint; a.S_sum += p.S_sum;
        a.S_max = fmax(a.S_max, p.S_max); a.line += p.line; a.used += p.used; a.defects += p.defects;
    }
    __shared__ double shd[kThreads / 32];
    __shared__ unsigned long long shu[kThreads / 32];
    KzmPartial r{};
    r.bulk = bsum(a.bulk, shd);
    r.elastic = bsum(a.elastic, shd);
    r.qint = bsum(a.qint, shd);
    r.gint = bsum(a.gint, shd);
    r.S_sum = bsum(a.S_sum, shd);
    r.S_max = bmax(a.S_max, shd);
    r.line = bsum(a.line, shd);
    r.used = bsum(a.used, shu);
    r.defects = bsum(a.defects, shu);
    if (threadIdx.x == 0) *out = r;
}

int alloc_or_fail(void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        set_error(std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
        return LDG_ERR_NOMEM;
    }
    return LDG_OK;
}

}  // namespace

struct kzm_handle {
    kzm_params p{};
    KzmConst base{};
    long long n = 0;
    float* q[2] = {nullptr, nullptr};
    double* stage = nullptr;
    double4* nf = nullptr;
    KzmPartial* part = nullptr;
    int cur = 0;
    bool uploaded = false;
    cudaStream_t stream = nullptr;
    long long launches = 0;
    int device = -1;  // the GPU the handle was created on
};

extern "C" {

int kzm_create(const kzm_params* params, kzm_handle** out) {
    clear_error();
    LDG_REQUIRE(params && out, LDG_ERR_ARG, "kzm_create: null argument");
    const kzm_params& p = *params;
    // Validation of KZM_bulk_ldg.cu:824-841.
    LDG_REQUIRE(p.Nx > 1 && p.Ny > 1 && p.Nz > 1, LDG_ERR_ARG,
                "Nx, Ny, and Nz must all be greater than 1 for the periodic bulk LdG branch");
    LDG_REQUIRE((long long)p.Nx * p.Ny * p.Nz < (1LL << 32), LDG_ERR_ARG, "kzm_create: grid exceeds 2^32 sites");
    LDG_REQUIRE(p.dx > 0 && p.dy > 0 && p.dz > 0, LDG_ERR_ARG, "dx, dy, and dz must be positive");
    LDG_REQUIRE(p.gamma > 0, LDG_ERR_ARG, "gamma must be positive");
    LDG_REQUIRE(p.kappa >= 0, LDG_ERR_ARG, "kappa must be non-negative");
    kzm_handle* h = new (std::nothrow) kzm_handle();
    LDG_REQUIRE(h, LDG_ERR_NOMEM, "kzm_create: host allocation failed");
    h->p = p;
    cudaGetDevice(&h->device);
    KzmConst& P = h->base;
    P.Nx = p.Nx; P.Ny = p.Ny; P.Nz = p.Nz;
    P.sy = (p.Nx + 3) & ~3;
    P.sz = (long long)p.Ny * P.sy;
    P.sc = (long long)p.Nz * P.sz;
    P.ix2 = (float)(1.0 / (p.dx * p.dx)); P.iy2 = (float)(1.0 / (p.dy * p.dy)); P.iz2 = (float)(1.0 / (p.dz * p.dz));
    P.lap_c = (float)(-2.0 * (1.0 / (p.dx * p.dx) + 1.0 / (p.dy * p.dy) + 1.0 / (p.dz * p.dz)));
    P.kappa = (float)p.kappa;
    P.qcap = (float)p.q_norm_cap;
    h->n = (long long)p.Nx * p.Ny * p.Nz;
    int rc;
    const size_t fb = (size_t)P.sc * 5 * sizeof(float);
    if ((rc = alloc_or_fail((void**)&h->q[0], fb)) || (rc = alloc_or_fail((void**)&h->q[1], fb)) ||
        (rc = alloc_or_fail((void**)&h->part, (kBlocks + 1) * sizeof(KzmPartial)))) {
        kzm_destroy(h);
        return rc;
    }
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMemset(h->q[0], 0, fb);
    if (e == cudaSuccess) e = cudaMemset(h->q[1], 0, fb);
    if (e != cudaSuccess) {
        set_error(std::string("kzm_create: ") + cudaGetErrorString(e));
        kzm_destroy(h);
        return LDG_ERR_CUDA;
    }
    *out = h;
    return LDG_OK;
}

static int kzm_stage(kzm_handle* h) {
    if (h->stage) return LDG_OK;
    return alloc_or_fail((void**)&h->stage, (size_t)h->n * 5 * sizeof(double));
}

int kzm_upload(kzm_handle* h, const double* q) {
    clear_error();
    LDG_REQUIRE(h && q, LDG_ERR_ARG, "kzm_upload: null argument");
    DeviceGuard device_guard(h->device);
    int rc = kzm_stage(h);
    if (rc) return rc;
    LDG_CUDA(cudaMemcpyAsync(h->stage, q, (size_t)h->n * 5 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    h->cur = 0;
    const int blocks = (int)std::min<long long>((h->n + 255) / 256, 148 * 16);
    k_kzm_from_aos<<<blocks, 256, 0, h->stream>>>(h->stage, h->q[0], h->base);
    h->launches++;
    LDG_LAUNCHED("k_kzm_from_aos");
    LDG_CUDA(cudaStreamSynchronize(h->stream));
    h->uploaded = true;
    return LDG_OK;
}

int kzm_download(kzm_handle* h, double* q) {
    clear_error();
    LDG_REQUIRE(h && q, LDG_ERR_ARG, "kzm_download: null argument");
    DeviceGuard device_guard(h->device);
    int rc = kzm_stage(h);
    if (rc) return rc;
    const int blocks = (int)std::min<long long>((h->n + 255) / 256, 148 * 16);
    k_kzm_to_aos<<<blocks, 256, 0, h->stream>>>(h->q[h->cur], h->stage, h->base);
    h->launches++;
    LDG_LAUNCHED("k_kzm_to_aos");
    LDG_CUDA(cudaMemcpyAsync(q, h->stage, (size_t)h->n * 5 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    LDG_CUDA(cudaStreamSynchronize(h->stream));
    return LDG_OK;
}

int kzm_step(kzm_handle* h, int n_steps, const kzm_step_args* a) {
    clear_error();
    LDG_REQUIRE(h && a, LDG_ERR_ARG, "kzm_step: null argument");
    DeviceGuard device_guard(h->device);
    LDG_REQUIRE(n_steps >= 0, LDG_ERR_ARG, "kzm_step: n_steps must be >= 0");
    LDG_REQUIRE(h->uploaded, LDG_ERR_STATE, "kzm_step: no field uploaded");
    LDG_REQUIRE(a->dt > 0.0, LDG_ERR_ARG, "dt must be positive");
    KzmConst P = h->base;
    P.A = (float)a->A; P.B = (float)a->B; P.C = (float)a->C;
    P.mob_dt = (float)((1.0 / h->p.gamma) * a->dt);
    P.sigma = (float)a->noise_sigma;
    P.key0 = (uint32_t)a->seed;
    P.key1 = (uint32_t)(a->seed >> 32);
    // Two-site asynchronous-copy kernel by default; LDG_KZM_KERNEL=async selects the one-site
    // asynchronous-copy kernel, =regs the register-queue tiled kernel, =direct the one-thread-per-
    // site kernel.
    const char* ksel = getenv("LDG_KZM_KERNEL");
    const int kind = !ksel                           ? 3
                     : std::strcmp(ksel, "direct") == 0 ? 0
                     : std::strcmp(ksel, "regs") == 0   ? 1
                     : std::strcmp(ksel, "async") == 0  ? 2
                                                        : 3;
    // the two-site kernel's 16-byte copies need every pitch a multiple of 4 floats
    const int kind_run = (kind == 3 && P.Nx % 4 != 0) ? 2 : kind;
    dim3 blk(32, 8, 1), grd((P.Nx + 31) / 32, (P.Ny + 7) / 8, P.Nz);
    dim3 tgrd((P.Nx + KTX - 1) / KTX, (P.Ny + KTY - 1) / KTY, (P.Nz + KZC - 1) / KZC);
    const size_t ring_bytes = (size_t)KRING * 5 * KPS * sizeof(float);
    for (int s = 0; s < n_steps; ++s) {
        P.step = a->step_index + s;
        const bool noise = a->noise_sigma > 0.0;
        const float* in = h->q[h->cur];
        float* outb = h->q[1 - h->cur];
        if (kind_run == 3) {
            if (noise) k_kzm_step_pair<true><<<tgrd, KPT, kRingBytes2, h->stream>>>(in, outb, P);
            else k_kzm_step_pair<false><<<tgrd, KPT, kRingBytes2, h->stream>>>(in, outb, P);
        } else if (kind_run == 2) {
            if (noise) k_kzm_step_async<true><<<tgrd, blk, ring_bytes, h->stream>>>(in, outb, P);
            else k_kzm_step_async<false><<<tgrd, blk, ring_bytes, h->stream>>>(in, outb, P);
        } else if (kind == 1) {
            if (noise) k_kzm_step_tiled<true><<<tgrd, blk, 0, h->stream>>>(in, outb, P);
            else k_kzm_step_tiled<false><<<tgrd, blk, 0, h->stream>>>(in, outb, P);
        } else if (noise) k_kzm_step<true><<<grd, blk, 0, h->stream>>>(in, outb, P);
        else k_kzm_step<false><<<grd, blk, 0, h->stream>>>(in, outb, P);
        h->launches++;
        LDG_LAUNCHED("k_kzm_step");
        h->cur = 1 - h->cur;
    }
    return LDG_OK;
}

int kzm_observe(kzm_handle* h, double A, double B, double C, kzm_observables* o) {
    clear_error();
    LDG_REQUIRE(h && o, LDG_ERR_ARG, "kzm_observe: null argument");
    DeviceGuard device_guard(h->device);
    if (!h->nf) {
        int rc = alloc_or_fail((void**)&h->nf, (size_t)h->n * sizeof(double4));
        if (rc) return rc;
    }
    const kzm_params& p = h->p;
    KzmObsConst O{};
    O.P = h->base;
    O.A = A; O.B = B; O.C = C; O.kappa = p.kappa;
    O.cv = p.dx * p.dy * p.dz;
    O.ix = 1.0 / p.dx; O.iy = 1.0 / p.dy; O.iz = 1.0 / p.dz;
    k_kzm_obs_sites<<<kBlocks, kThreads, 0, h->stream>>>(h->q[h->cur], O, h->nf, h->part);
    k_kzm_obs_plaq<<<kBlocks, kThreads, 0, h->stream>>>(h->nf, O, p.defects_S_threshold, p.defects_charge_cutoff, p.dx,
                                                       p.dy, p.dz, h->part);
    k_kzm_obs_final<<<1, kThreads, 0, h->stream>>>(h->part, kBlocks, h->part + kBlocks);
    h->launches += 3;
    LDG_LAUNCHED("kzm observables");
    KzmPartial R{};
    LDG_CUDA(cudaMemcpyAsync(&R, h->part + kBlocks, sizeof(R), cudaMemcpyDeviceToHost, h->stream));
    LDG_CUDA(cudaStreamSynchronize(h->stream));
    const double tv = O.cv * (double)p.Nx * (double)p.Ny * (double)p.Nz;
    const double nan = std::numeric_limits<double>::quiet_NaN();
    o->bulk = R.bulk / tv;
    o->elastic = R.elastic / tv;
    o->total = o->bulk + o->elastic;
    o->avg_S = R.S_sum / (double)h->n;
    o->max_S = R.S_max;
    o->defect_plaquettes_used = (long long)R.used;
    o->nonzero_defect_plaquettes = (long long)R.defects;
    o->defect_density_per_plaquette = R.used > 0 ? (double)R.defects / (double)R.used : nan;
    o->defect_line_density = tv > 0.0 ? R.line / tv : nan;
    o->xi_grad_proxy = (R.gint > 0.0 && R.qint > 0.0) ? std::sqrt(R.qint / R.gint) : nan;
    return LDG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// No-allocation observables. Scratch lives in file-scope device arrays of this library:
// the per-site nematic field of at most KZM_NOALLOC_MAX_SITES sites (16 MiB) and one
// partial per reduction block. Every slot a kernel reads is written earlier in the same
// call (all sites of the grid, all kBlocks partials and the final slot), so nothing has to
// start at zero; the arrays keep the last call's contents.
// ---------------------------------------------------------------------------------------
static __device__ __align__(256) double4 g_noalloc_nematic[KZM_NOALLOC_MAX_SITES];
static __device__ __align__(256) KzmPartial g_noalloc_partials[kBlocks + 1];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
double4* g_noalloc_nematic_ptr[kMaxDevices] = {};
KzmPartial* g_noalloc_partials_ptr[kMaxDevices] = {};

// Device addresses of the scratch arrays for the current device, looked up once per device.
int noalloc_scratch(double4** nf, KzmPartial** part) {
    int dev = 0;
    LDG_CUDA(cudaGetDevice(&dev));
    LDG_REQUIRE(dev >= 0 && dev < kMaxDevices, LDG_ERR_ARG, "kzm_observe_device_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_nematic_ptr[dev]) {
        void* a = nullptr;
        void* b = nullptr;
        LDG_CUDA(cudaGetSymbolAddress(&a, g_noalloc_nematic));
        LDG_CUDA(cudaGetSymbolAddress(&b, g_noalloc_partials));
        g_noalloc_nematic_ptr[dev] = static_cast<double4*>(a);
        g_noalloc_partials_ptr[dev] = static_cast<KzmPartial*>(b);
    }
    *nf = g_noalloc_nematic_ptr[dev];
    *part = g_noalloc_partials_ptr[dev];
    return LDG_OK;
}
}  // namespace

extern "C" {

int kzm_observe_device_noalloc(const kzm_params* params, const double* q, double A, double B, double C,
                               void* stream, kzm_observables* o) {
    clear_error();
    LDG_REQUIRE(params && q && o, LDG_ERR_ARG, "kzm_observe_device_noalloc: null argument");
    const kzm_params& p = *params;
    LDG_REQUIRE(p.Nx > 1 && p.Ny > 1 && p.Nz > 1, LDG_ERR_ARG,
                "Nx, Ny, and Nz must all be greater than 1 for the periodic bulk LdG branch");
    LDG_REQUIRE(p.dx > 0 && p.dy > 0 && p.dz > 0, LDG_ERR_ARG, "dx, dy, and dz must be positive");
    const long long n = (long long)p.Nx * p.Ny * p.Nz;
    LDG_REQUIRE(n <= KZM_NOALLOC_MAX_SITES, LDG_ERR_ARG,
                "kzm_observe_device_noalloc: " + std::to_string(n) + " sites exceed the no-allocation scratch limit of " +
                    std::to_string(KZM_NOALLOC_MAX_SITES) + " sites (use kzm_observe for larger grids)");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (st) {
        // the scratch address is the current device's: a stream of another device cannot use it
        int cur = 0, sdev = 0;
        LDG_CUDA(cudaGetDevice(&cur));
        LDG_CUDA(cudaStreamGetDevice(st, &sdev));
        LDG_REQUIRE(sdev == cur, LDG_ERR_ARG,
                    "kzm_observe_device_noalloc: the stream belongs to device " + std::to_string(sdev) +
                        ", not to the current device " + std::to_string(cur));
    }
    double4* nf = nullptr;
    KzmPartial* part = nullptr;
    int rc = noalloc_scratch(&nf, &part);
    if (rc) return rc;
    KzmObsConst O{};
    O.P.Nx = p.Nx; O.P.Ny = p.Ny; O.P.Nz = p.Nz;
    O.A = A; O.B = B; O.C = C; O.kappa = p.kappa;
    O.cv = p.dx * p.dy * p.dz;
    O.ix = 1.0 / p.dx; O.iy = 1.0 / p.dy; O.iz = 1.0 / p.dz;
    k_kzm_obs_sites_aos<<<kBlocks, kThreads, 0, st>>>(q, O, nf, part);
    k_kzm_obs_plaq<<<kBlocks, kThreads, 0, st>>>(nf, O, p.defects_S_threshold, p.defects_charge_cutoff, p.dx, p.dy,
                                                  p.dz, part);
    k_kzm_obs_final<<<1, kThreads, 0, st>>>(part, kBlocks, part + kBlocks);
    LDG_LAUNCHED("kzm_observe_device_noalloc kernels");
    KzmPartial R{};
    LDG_CUDA(cudaMemcpyAsync(&R, part + kBlocks, sizeof(R), cudaMemcpyDeviceToHost, st));
    LDG_CUDA(cudaStreamSynchronize(st));
    const double tv = O.cv * (double)p.Nx * (double)p.Ny * (double)p.Nz;
    const double nan = std::numeric_limits<double>::quiet_NaN();
    o->bulk = R.bulk / tv;
    o->elastic = R.elastic / tv;
    o->total = o->bulk + o->elastic;
    o->avg_S = R.S_sum / (double)n;
    o->max_S = R.S_max;
    o->defect_plaquettes_used = (long long)R.used;
    o->nonzero_defect_plaquettes = (long long)R.defects;
    o->defect_density_per_plaquette = R.used > 0 ? (double)R.defects / (double)R.used : nan;
    o->defect_line_density = tv > 0.0 ? R.line / tv : nan;
    o->xi_grad_proxy = (R.gint > 0.0 && R.qint > 0.0) ? std::sqrt(R.qint / R.gint) : nan;
    return LDG_OK;
}

void* kzm_stream(kzm_handle* h) { return h ? (void*)h->stream : nullptr; }

long long kzm_launch_count(const kzm_handle* h) { return h ? h->launches : 0; }

int kzm_destroy(kzm_handle* h) {
    if (!h) return LDG_OK;
    DeviceGuard device_guard(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    cudaFree(h->q[0]); cudaFree(h->q[1]); cudaFree(h->stage); cudaFree(h->nf); cudaFree(h->part);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return LDG_OK;
}

}  // extern "C"
