// Shared device code of the B200 LdG solver: field layout, per-cell physics written
// against a neighbour accessor, the counter-based noise generator and the FP64 nematic
// eigen-solver used by the reductions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ldg {

// Per-cell classification bits, computed once on the host in FP64 (qsr.cu) from the
// reference predicates (QSR.cu:100-111, 697-709, 851-867, 994-1002, 2288-2300).
enum : uint8_t {
    kMove = 1,     // the update touches the cell: !(W == 0 && shell) && sd <= band
    kFixed = 2,    // strong anchoring: W <= 0 && shell, rewritten to Q0 after the update
    kAnchor = 4,   // weak anchoring penalty: shell && W != 0 && delta_eff > 0
    kShell = 8,    // |sd| <= shell half thickness
    kInside = 16,  // sd <= 0
    kCore = 32,    // sd < -2 min_spacing (avg_S, max_S, checker)
    kRadial = 64,  // inside && |r| > 2 min_spacing (radiality)
};

// Constants of one confined-solver step, passed by value to the kernels. The field is
// FP32 SoA: component c of cell (i, j, k) lives at q[c*sc + i*si + j*sj + k].
struct QsrConst {
    int Nx, Ny, Nz;
    int sj;          // row pitch (>= Nz, multiple of 4)
    long long si;    // plane pitch = Ny*sj
    long long sc;    // component pitch = Nx*si
    float ix2, iy2, iz2;        // 1/d^2
    float i2x, i2y, i2z;        // 1/(2d)
    float ix, iy, iz;           // 1/d
    float i4xy, i4xz, i4yz;     // 1/(4 da db)
    float cQ, cQ2, cQ3;         // bulk force coefficients (QSR.cu:385-397)
    float Liso;                 // kappa if L1 = L2 = L3 = 0, else L1 (QSR.cu:420-438)
    float L2, L3;
    float Weff, S_shell;        // W/delta_eff and the shell order
    float mob_dt;               // dt/gamma
    float qcap;                 // Frobenius cap (0 = off)
    float ci, cj, ck;           // droplet centre in cell units, (N-1)/2
    float gnx, gny, gnz;        // d/r^2 per axis: surface normal ~ (X gnx, Y gny, Z gnz)
    float sigma;                // Langevin amplitude per component (0 = off)
    uint32_t key0, key1;        // Philox key (seed)
    uint32_t instance;          // ensemble instance id (noise counter word)
    long long step;             // global step index (noise counter words)
    // semi-implicit (IMEX) Helmholtz-Jacobi
    float alpha;                // (dt/gamma) L_stab
    float jdenom_inv;           // 1/(1 + 2 alpha sum 1/d^2)
    // products of the constants above, folded on the host so the interior stencils need one
    // fused multiply-add per term
    float lap_c;                // -2 (1/dx^2 + 1/dy^2 + 1/dz^2): centre weight of the Laplacian
    float L2i2x, L2i2y, L2i2z;  // L2/(2d)
    float l3m[6];               // (L3/2) / (4 da db) for M_ab from undivided central differences (xx yy zz xy xz yz)
    float l2w[6];               // L2 / (4 da db) for d_a D_b from undivided second differences (xx yy zz xy xz yz)
};

// ---------------------------------------------------------------------------------------
// Philox4x32 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11) and Box-Muller normals.
// ---------------------------------------------------------------------------------------
// Rounds of the noise generator. The paper reports Philox4x32 with 7 rounds passing TestU01's
// BigCrush (10 is its default safety margin); every noise draw here uses 7.
constexpr int kNoiseRounds = 7;

template <int kRounds>
__device__ __forceinline__ void philox4x32(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c[0]);
        const uint32_t lo0 = 0xD2511F53u * c[0];
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]);
        const uint32_t lo1 = 0xCD9E8D57u * c[2];
        const uint32_t n0 = hi1 ^ c[1] ^ k0;
        const uint32_t n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
}

// Uniform in (0, 1] from a 21-bit integer: (x + 1) 2^-21, formed as one fused multiply-add
// (exact: x is exact in FP32 and the result has at most 22 significant bits).
__device__ __forceinline__ float u21(uint32_t x) {
    return fmaf((float)x, 1.0f / 2097152.0f, 1.0f / 2097152.0f);
}

// Five standard normals for (cell, instance, step) from one Philox4x32-7 block: the four
// 32-bit words give six disjoint 21-bit fields (the low 21 bits of each word, and the high
// 11 bits of words 0|1 and 2|3 joined), i.e. three Box-Muller pairs; the sixth normal is
// not needed. Counter = (cell, instance, step low word, step high word).
// The radius sqrt(-2 ln u) takes ln u from the hardware base-2 logarithm (absolute error at most
// 2^-22 for u in [0.5, 1], 2 ulp below): a normal is off by at most 2e-4 in absolute terms (only
// when |z| < 0.002, i.e. u within 2e-6 of 1) and by less than 1e-5 relative when |z| > 0.05.
__device__ __forceinline__ void normals5(uint32_t cell, uint32_t instance, long long step, uint32_t k0, uint32_t k1,
                                         float g[5]) {
    uint32_t c[4] = {cell, instance, (uint32_t)step, (uint32_t)((unsigned long long)step >> 32)};
    philox4x32<kNoiseRounds>(c, k0, k1);
    constexpr uint32_t M21 = (1u << 21) - 1u;
    const uint32_t f0 = c[0] & M21, f1 = c[1] & M21, f2 = c[2] & M21, f3 = c[3] & M21;
    const uint32_t f4 = ((c[0] >> 21) << 10) | (c[1] >> 22);  // 11 + 10 bits
    const uint32_t f5 = ((c[2] >> 21) << 10) | (c[3] >> 22);
    // angle 2 pi u taken as pi + t with t = 2 pi u - pi in (-pi, pi], where the fast hardware
    // sine/cosine is accurate to ~4e-7: cos(2 pi u) = -cos t, sin(2 pi u) = -sin t
    constexpr float kTwoPi = 6.28318530717958647692f, kPi = 3.14159265358979323846f;
    constexpr float kM2Ln2 = -1.38629436111989061883f;  // -2 ln 2
    // radius sqrt(-2 ln u) = t * rsqrt(t), t = -2 ln 2 log2(u) (the guard keeps t = 0, u = 1, at zero)
    auto radius = [](float u) {
        const float t = kM2Ln2 * __log2f(u);
        return t * rsqrtf(fmaxf(t, 1e-30f));
    };
    float s, co;
    float r = radius(u21(f0));
    __sincosf(fmaf(kTwoPi, u21(f1), -kPi), &s, &co);
    g[0] = -r * co;
    g[1] = -r * s;
    r = radius(u21(f2));
    __sincosf(fmaf(kTwoPi, u21(f3), -kPi), &s, &co);
    g[2] = -r * co;
    g[3] = -r * s;
    r = radius(u21(f4));
    g[4] = -r * __cosf(fmaf(kTwoPi, u21(f5), -kPi));
}

// ---------------------------------------------------------------------------------------
// Stencil physics. `A(c, di, dj, dk)` returns component c (0..4, 5 = Qzz) of the cell at
// offset (di, dj, dk); the face logic below never asks for a cell outside the grid.
// ---------------------------------------------------------------------------------------

// Second derivative along one axis with the reference's shifted stencil at the faces
// (QSR.cu:296-320).
// kFaces = false is the interior form: the caller guarantees 0 < pos < n - 1 for every
// position the stencil is evaluated at, so the face branches are compiled out.
template <int AX, bool kFaces = true, class Acc>
__device__ __forceinline__ float d2_face(const Acc& A, int c, float cv, int pos, int n, float inv) {
    auto at = [&](int s) { return AX == 0 ? A(c, s, 0, 0) : (AX == 1 ? A(c, 0, s, 0) : A(c, 0, 0, s)); };
    if (!kFaces || (pos > 0 && pos < n - 1)) return (at(1) - cv * 2.0f + at(-1)) * inv;
    if (pos == 0) return (at(2) - at(1) * 2.0f + cv) * inv;
    return (cv - at(-1) * 2.0f + at(-2)) * inv;
}

// First derivative along one axis at offset (oi, oj, ok), one-sided first order at the faces
// (QSR.cu:245-273). `pos` is the absolute coordinate of the offset cell along AX.
template <int AX, bool kFaces = true, class Acc>
__device__ __forceinline__ float d1_face(const Acc& A, int c, int oi, int oj, int ok, int pos, int n, float i2, float i1) {
    auto at = [&](int s) {
        return AX == 0 ? A(c, oi + s, oj, ok) : (AX == 1 ? A(c, oi, oj + s, ok) : A(c, oi, oj, ok + s));
    };
    if (!kFaces || (pos > 0 && pos < n - 1)) return (at(1) - at(-1)) * i2;
    if (pos == 0) return (at(1) - at(0)) * i1;
    return (at(0) - at(-1)) * i1;
}

// Column divergence D_j = d_k Q_kj at offset (oi, oj, ok) of cell (i, j, k) (QSR.cu:325-371).
template <bool kFaces = true, class Acc>
__device__ __forceinline__ void dcol_at(const Acc& A, const QsrConst& P, int i, int j, int k, int oi, int oj, int ok,
                                        float D[3]) {
    const int pi = i + oi, pj = j + oj, pk = k + ok;
    D[0] = d1_face<0, kFaces>(A, 0, oi, oj, ok, pi, P.Nx, P.i2x, P.ix) +
           d1_face<1, kFaces>(A, 1, oi, oj, ok, pj, P.Ny, P.i2y, P.iy) +
           d1_face<2, kFaces>(A, 2, oi, oj, ok, pk, P.Nz, P.i2z, P.iz);
    D[1] = d1_face<0, kFaces>(A, 1, oi, oj, ok, pi, P.Nx, P.i2x, P.ix) +
           d1_face<1, kFaces>(A, 3, oi, oj, ok, pj, P.Ny, P.i2y, P.iy) +
           d1_face<2, kFaces>(A, 4, oi, oj, ok, pk, P.Nz, P.i2z, P.iz);
    D[2] = d1_face<0, kFaces>(A, 2, oi, oj, ok, pi, P.Nx, P.i2x, P.ix) +
           d1_face<1, kFaces>(A, 4, oi, oj, ok, pj, P.Ny, P.i2y, P.iy) +
           d1_face<2, kFaces>(A, 5, oi, oj, ok, pk, P.Nz, P.i2z, P.iz);
}

// Bulk molecular field entries xx yy zz xy xz yz (QSR.cu:399-417).
__device__ __forceinline__ void bulk_field(const float q[5], float cQ, float cQ2, float cQ3, float h[6]) {
    const float Qxx = q[0], Qxy = q[1], Qxz = q[2], Qyy = q[3], Qyz = q[4];
    const float Qzz = -Qxx - Qyy;
    const float trQ2 = Qxx * Qxx + Qyy * Qyy + Qzz * Qzz + 2.0f * (Qxy * Qxy + Qxz * Qxz + Qyz * Qyz);
    const float q2xx = Qxx * Qxx + Qxy * Qxy + Qxz * Qxz;
    const float q2xy = Qxx * Qxy + Qxy * Qyy + Qxz * Qyz;
    const float q2xz = Qxx * Qxz + Qxy * Qyz + Qxz * Qzz;
    const float q2yy = Qxy * Qxy + Qyy * Qyy + Qyz * Qyz;
    const float q2yz = Qxy * Qxz + Qyy * Qyz + Qyz * Qzz;
    const float q2zz = Qxz * Qxz + Qyz * Qyz + Qzz * Qzz;
    const float t3 = trQ2 * (1.0f / 3.0f);  // FP32 path: reciprocal multiply (one rounding)
    // cQ Q - cQ2 (Q^2 - tr/3) + cQ3 tr(Q^2) Q with the two linear terms joined: (cQ + cQ3 tr) Q
    const float cg = fmaf(cQ3, trQ2, cQ);
    h[0] = fmaf(-cQ2, q2xx - t3, cg * Qxx);
    h[1] = fmaf(-cQ2, q2yy - t3, cg * Qyy);
    h[2] = fmaf(-cQ2, q2zz - t3, cg * Qzz);
    h[3] = fmaf(-cQ2, q2xy, cg * Qxy);
    h[4] = fmaf(-cQ2, q2xz, cg * Qxz);
    h[5] = fmaf(-cQ2, q2yz, cg * Qyz);
}

// Droplet surface normal at cell (i, j, k) (QSR.cu:130-142), in FP32 from cell units.
__device__ __forceinline__ void surface_q0(const QsrConst& P, int i, int j, int k, float Q0[5]) {
    const float gx = ((float)i - P.ci) * P.gnx, gy = ((float)j - P.cj) * P.gny, gz = ((float)k - P.ck) * P.gnz;
    const float g2 = gx * gx + gy * gy + gz * gz;
    float nx = 1.0f, ny = 0.0f, nz = 0.0f;
    if (g2 > 0.0f) {  // unit normal by one reciprocal square root (2 ulp) instead of three divisions
        const float inv = rsqrtf(g2);
        nx = gx * inv; ny = gy * inv; nz = gz * inv;
    }
    const float S = P.S_shell;
    Q0[0] = S * (nx * nx - 1.0f / 3.0f);
    Q0[1] = S * (nx * ny);
    Q0[2] = S * (nx * nz);
    Q0[3] = S * (ny * ny - 1.0f / 3.0f);
    Q0[4] = S * (ny * nz);
}

// Chemical potential of cell (i, j, k): bulk + elastic (iso | L1, L2) projected traceless,
// then L3 on interior cells re-projected, then the weak-anchoring penalty
// (QSR.cu:373-472, 474-621, 623-652). `lap` returns the Laplacian (IMEX uses it).
// DAcc(c, di, dj, dk) returns the column divergence D_c at a face-neighbour offset.
// kFaces = false: the caller guarantees the cell and all stencil positions are interior.
template <bool kL2, bool kL3, bool kFaces = true, class Acc, class DAcc>
__device__ __forceinline__ void chem_potential(const Acc& A, const DAcc& DA, const QsrConst& P, int i, int j, int k,
                                               const float q[5], bool anchor, float mu[5], float lap[5]) {
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        if (!kFaces) {
            // interior: sum_a (Q[+1] + Q[-1]) / da^2 - 2 Q sum_a 1/da^2
            const float sx = A(c, 1, 0, 0) + A(c, -1, 0, 0);
            const float sy = A(c, 0, 1, 0) + A(c, 0, -1, 0);
            const float sz = A(c, 0, 0, 1) + A(c, 0, 0, -1);
            lap[c] = fmaf(P.ix2, sx, fmaf(P.iy2, sy, fmaf(P.iz2, sz, P.lap_c * q[c])));
        } else {
            const float d2x = d2_face<0, kFaces>(A, c, q[c], i, P.Nx, P.ix2);
            const float d2y = d2_face<1, kFaces>(A, c, q[c], j, P.Ny, P.iy2);
            const float d2z = d2_face<2, kFaces>(A, c, q[c], k, P.Nz, P.iz2);
            lap[c] = d2x + d2y + d2z;
        }
    }
    float h[6];
    bulk_field(q, P.cQ, P.cQ2, P.cQ3, h);
    const float lzz = -lap[0] - lap[3];
    h[0] -= P.Liso * lap[0];
    h[1] -= P.Liso * lap[3];
    h[2] -= P.Liso * lzz;
    h[3] -= P.Liso * lap[1];
    h[4] -= P.Liso * lap[2];
    h[5] -= P.Liso * lap[4];
    if (kL2) {
        // h -= L2 d_a D_b, d_a central with one-sided faces (QSR.cu:436-460). sub() applies one
        // term as a fused multiply-add with L2/(2 da) (central) or L2/da = 2 L2/(2 da) (one-sided).
        auto sub = [&](float& hv, int comp, int ax) {
            const int pos = ax == 0 ? i : (ax == 1 ? j : k);
            const int n = ax == 0 ? P.Nx : (ax == 1 ? P.Ny : P.Nz);
            const float c2 = ax == 0 ? P.L2i2x : (ax == 1 ? P.L2i2y : P.L2i2z);
            auto at = [&](int s) {
                return ax == 0 ? DA(comp, s, 0, 0) : (ax == 1 ? DA(comp, 0, s, 0) : DA(comp, 0, 0, s));
            };
            if (!kFaces || (pos > 0 && pos < n - 1)) hv = fmaf(-c2, at(1) - at(-1), hv);
            else if (pos == 0) hv = fmaf(-2.0f * c2, at(1) - at(0), hv);
            else hv = fmaf(-2.0f * c2, at(0) - at(-1), hv);
        };
        sub(h[0], 0, 0);
        sub(h[1], 1, 1);
        sub(h[2], 2, 2);
        sub(h[3], 1, 0);
        sub(h[3], 0, 1);
        sub(h[4], 2, 0);
        sub(h[4], 0, 2);
        sub(h[5], 2, 1);
        sub(h[5], 1, 2);
    }
    float corr = (h[0] + h[1] + h[2]) * (1.0f / 3.0f);
    mu[0] = h[0] - corr;
    mu[1] = h[3];
    mu[2] = h[4];
    mu[3] = h[1] - corr;
    mu[4] = h[5];
    if (kL3) {
        const bool interior =
            !kFaces || (i > 0 && i < P.Nx - 1 && j > 0 && j < P.Ny - 1 && k > 0 && k < P.Nz - 1);
        if (interior) {
            float hx[6] = {mu[0], mu[3], -(mu[0] + mu[3]), mu[1], mu[2], mu[4]};
            // undivided central differences Q[+1] - Q[-1]; the 1/(2 da) factors are folded into
            // the M_ab weights (P.l3m) and into the divergence below
            float d[6][3];
#pragma unroll
            for (int c = 0; c < 5; ++c) {
                d[c][0] = A(c, 1, 0, 0) - A(c, -1, 0, 0);
                d[c][1] = A(c, 0, 1, 0) - A(c, 0, -1, 0);
                d[c][2] = A(c, 0, 0, 1) - A(c, 0, 0, -1);
            }
#pragma unroll
            for (int a = 0; a < 3; ++a) d[5][a] = -(d[0][a] + d[3][a]);
            auto M = [&](int a, int b) {
                return d[0][a] * d[0][b] + d[3][a] * d[3][b] + d[5][a] * d[5][b] +
                       2.0f * (d[1][a] * d[1][b] + d[2][a] * d[2][b] + d[4][a] * d[4][b]);
            };
            hx[0] = fmaf(P.l3m[0], M(0, 0), hx[0]);
            hx[1] = fmaf(P.l3m[1], M(1, 1), hx[1]);
            hx[2] = fmaf(P.l3m[2], M(2, 2), hx[2]);
            hx[3] = fmaf(P.l3m[3], M(0, 1), hx[3]);
            hx[4] = fmaf(P.l3m[4], M(0, 2), hx[4]);
            hx[5] = fmaf(P.l3m[5], M(1, 2), hx[5]);
            const float Qxx = q[0], Qxy = q[1], Qxz = q[2], Qyy = q[3], Qyz = q[4], Qzz = -q[0] - q[3];
            // D_a / (2 da): pairs with the undivided differences in D . grad Q_c
            const float Dc0 = DA(0, 0, 0, 0) * P.i2x, Dc1 = DA(1, 0, 0, 0) * P.i2y, Dc2 = DA(2, 0, 0, 0) * P.i2z;
            // B(Q_c) = D . grad Q_c + Q_ab d_a d_b Q_c (QSR.cu:580-603), with the Q_ab / (stencil
            // denominator) weights formed once for all five components.
            const float wxx = Qxx * P.ix2, wyy = Qyy * P.iy2, wzz = Qzz * P.iz2;
            const float wxy = 2.0f * Qxy * P.i4xy, wxz = 2.0f * Qxz * P.i4xz, wyz = 2.0f * Qyz * P.i4yz;
            auto Bc = [&](int c) {
                const float Qc2 = 2.0f * (c == 5 ? Qzz : q[c]);
                const float sxx = (A(c, 1, 0, 0) + A(c, -1, 0, 0)) - Qc2;
                const float syy = (A(c, 0, 1, 0) + A(c, 0, -1, 0)) - Qc2;
                const float szz = (A(c, 0, 0, 1) + A(c, 0, 0, -1)) - Qc2;
                const float sxy = (A(c, 1, 1, 0) - A(c, 1, -1, 0)) - (A(c, -1, 1, 0) - A(c, -1, -1, 0));
                const float sxz = (A(c, 1, 0, 1) - A(c, 1, 0, -1)) - (A(c, -1, 0, 1) - A(c, -1, 0, -1));
                const float syz = (A(c, 0, 1, 1) - A(c, 0, 1, -1)) - (A(c, 0, -1, 1) - A(c, 0, -1, -1));
                const float contract = wxx * sxx + wyy * syy + wzz * szz + wxy * sxy + wxz * sxz + wyz * syz;
                return fmaf(Dc0, d[c][0], fmaf(Dc1, d[c][1], fmaf(Dc2, d[c][2], contract)));
            };
            const float Bxx = Bc(0), Byy = Bc(3), Bzz = -(Bxx + Byy);
            const float Bxy = Bc(1), Bxz = Bc(2), Byz = Bc(4);
            hx[0] -= P.L3 * Bxx;
            hx[1] -= P.L3 * Byy;
            hx[2] -= P.L3 * Bzz;
            hx[3] -= P.L3 * Bxy;
            hx[4] -= P.L3 * Bxz;
            hx[5] -= P.L3 * Byz;
            corr = (hx[0] + hx[1] + hx[2]) * (1.0f / 3.0f);
            mu[0] = hx[0] - corr;
            mu[3] = hx[1] - corr;
            mu[1] = hx[3];
            mu[2] = hx[4];
            mu[4] = hx[5];
        }
    }
    if (anchor) {
        float Q0[5];
        surface_q0(P, i, j, k, Q0);
#pragma unroll
        for (int c = 0; c < 5; ++c) mu[c] += P.Weff * (q[c] - Q0[c]);
    }
}

// ---------------------------------------------------------------------------------------
// Packed-pair form of the interior chemical potential. Blackwell issues one FFMA2 / FADD2 /
// FMUL2 for two FP32 lanes, so the stencil arithmetic runs on component pairs: X = (xx, yy),
// Y = (xy, xz); yz stays scalar and zz = -(xx + yy). Same terms and weights as
// chem_potential<kL2, kL3, false>; only the rounding order differs.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a - b as b * (-1) + a (the product is exact, so this is the rounded difference)
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }

// Interior cells (2 <= i, j, k <= N - 3 when L2 is on, else 1 <= .. <= N - 2) read only Q:
//  * the column divergence D_b = d_k Q_kb at the centre (the L3 term's D . grad) from the face
//    neighbours' central differences, as the reference's interior D;
//  * the L2 term d_a D_b (QSR.cu:436-460), the central difference of the reference's central D,
//    which for an interior cell is exactly sum_k S_ak(Q_kb) / (4 da dk): S_ak the undivided
//    mixed (four-corner) second difference for k != a and the wide second difference
//    Q(+2a) - 2 Q + Q(-2a) for k = a. The corner sums are the ones the L3 term needs anyway, so
//    no divergence field is staged.
template <bool kL2, bool kL3, class Acc>
__device__ __forceinline__ void chem_potential_interior_x2(const Acc& A, const QsrConst& P, int i, int j, int k,
                                                           const float q[5], bool anchor, float mu[5], float lap[5]) {
    constexpr bool kMixed = kL2 || kL3;
    auto X = [&](int di, int dj, int dk) { return make_float2(A(0, di, dj, dk), A(3, di, dj, dk)); };
    auto Y = [&](int di, int dj, int dk) { return make_float2(A(1, di, dj, dk), A(2, di, dj, dk)); };
    auto Z = [&](int di, int dj, int dk) { return A(4, di, dj, dk); };  // yz
    const float2 qX = make_float2(q[0], q[3]), qY = make_float2(q[1], q[2]);
    const float qZ = q[4];
    // face neighbours, their sums (Laplacian, pure second derivatives) and undivided central
    // differences (first derivatives)
    const float2 Xpx = X(1, 0, 0), Xmx = X(-1, 0, 0), Xpy = X(0, 1, 0), Xmy = X(0, -1, 0), Xpz = X(0, 0, 1),
                 Xmz = X(0, 0, -1);
    const float2 Ypx = Y(1, 0, 0), Ymx = Y(-1, 0, 0), Ypy = Y(0, 1, 0), Ymy = Y(0, -1, 0), Ypz = Y(0, 0, 1),
                 Ymz = Y(0, 0, -1);
    const float Zpx = Z(1, 0, 0), Zmx = Z(-1, 0, 0), Zpy = Z(0, 1, 0), Zmy = Z(0, -1, 0), Zpz = Z(0, 0, 1),
                Zmz = Z(0, 0, -1);
    const float2 sxX = add2(Xpx, Xmx), syX = add2(Xpy, Xmy), szX = add2(Xpz, Xmz);
    const float2 sxY = add2(Ypx, Ymx), syY = add2(Ypy, Ymy), szY = add2(Ypz, Ymz);
    const float sxZ = Zpx + Zmx, syZ = Zpy + Zmy, szZ = Zpz + Zmz;
    const float2 lapX = fma2(bc2(P.ix2), sxX, fma2(bc2(P.iy2), syX, fma2(bc2(P.iz2), szX, mul2(bc2(P.lap_c), qX))));
    const float2 lapY = fma2(bc2(P.ix2), sxY, fma2(bc2(P.iy2), syY, fma2(bc2(P.iz2), szY, mul2(bc2(P.lap_c), qY))));
    const float lapZ = fmaf(P.ix2, sxZ, fmaf(P.iy2, syZ, fmaf(P.iz2, szZ, P.lap_c * qZ)));
    lap[0] = lapX.x; lap[3] = lapX.y; lap[1] = lapY.x; lap[2] = lapY.y; lap[4] = lapZ;
    float h[6];
    bulk_field(q, P.cQ, P.cQ2, P.cQ3, h);
    // elastic (one-constant or L1): hX = (h_xx, h_yy), hY = (h_xy, h_xz), h_zz, h_yz
    float2 hX = fma2(bc2(-P.Liso), lapX, make_float2(h[0], h[1]));
    float2 hY = fma2(bc2(-P.Liso), lapY, make_float2(h[3], h[4]));
    float hzz = fmaf(P.Liso, lapX.x + lapX.y, h[2]);  // - Liso lap_zz, lap_zz = -(lap_xx + lap_yy)
    float hyz = fmaf(-P.Liso, lapZ, h[5]);
    // undivided mixed second differences (four corners) of every component: (xx, yy), (xy, xz), yz
    float2 mxyX{}, mxzX{}, myzX{}, mxyY{}, mxzY{}, myzY{};
    float mxyZ = 0.0f, mxzZ = 0.0f, myzZ = 0.0f;
    if (kMixed) {
        mxyX = sub2(sub2(X(1, 1, 0), X(1, -1, 0)), sub2(X(-1, 1, 0), X(-1, -1, 0)));
        mxzX = sub2(sub2(X(1, 0, 1), X(1, 0, -1)), sub2(X(-1, 0, 1), X(-1, 0, -1)));
        myzX = sub2(sub2(X(0, 1, 1), X(0, 1, -1)), sub2(X(0, -1, 1), X(0, -1, -1)));
        mxyY = sub2(sub2(Y(1, 1, 0), Y(1, -1, 0)), sub2(Y(-1, 1, 0), Y(-1, -1, 0)));
        mxzY = sub2(sub2(Y(1, 0, 1), Y(1, 0, -1)), sub2(Y(-1, 0, 1), Y(-1, 0, -1)));
        myzY = sub2(sub2(Y(0, 1, 1), Y(0, 1, -1)), sub2(Y(0, -1, 1), Y(0, -1, -1)));
        mxyZ = (Z(1, 1, 0) - Z(1, -1, 0)) - (Z(-1, 1, 0) - Z(-1, -1, 0));
        mxzZ = (Z(1, 0, 1) - Z(1, 0, -1)) - (Z(-1, 0, 1) - Z(-1, 0, -1));
        myzZ = (Z(0, 1, 1) - Z(0, 1, -1)) - (Z(0, -1, 1) - Z(0, -1, -1));
    }
    if (kL2) {
        // wide second differences Q(+2a) - 2 Q + Q(-2a) of the components d_a D_b needs
        const float q2xx = 2.0f * q[0], q2xy = 2.0f * q[1], q2xz = 2.0f * q[2], q2yy = 2.0f * q[3],
                    q2yz = 2.0f * q[4];
        const float wx_xx = (A(0, 2, 0, 0) + A(0, -2, 0, 0)) - q2xx;
        const float wx_xy = (A(1, 2, 0, 0) + A(1, -2, 0, 0)) - q2xy;
        const float wx_xz = (A(2, 2, 0, 0) + A(2, -2, 0, 0)) - q2xz;
        const float wy_yy = (A(3, 0, 2, 0) + A(3, 0, -2, 0)) - q2yy;
        const float wy_xy = (A(1, 0, 2, 0) + A(1, 0, -2, 0)) - q2xy;
        const float wy_yz = (A(4, 0, 2, 0) + A(4, 0, -2, 0)) - q2yz;
        const float wz_xx = (A(0, 0, 0, 2) + A(0, 0, 0, -2)) - q2xx;
        const float wz_yy = (A(3, 0, 0, 2) + A(3, 0, 0, -2)) - q2yy;
        const float wz_xz = (A(2, 0, 0, 2) + A(2, 0, 0, -2)) - q2xz;
        const float wz_yz = (A(4, 0, 0, 2) + A(4, 0, 0, -2)) - q2yz;
        const float wz_zz = -(wz_xx + wz_yy);
        const float mxz_zz = -(mxzX.x + mxzX.y), myz_zz = -(myzX.x + myzX.y);
        const float cxx = P.l2w[0], cyy = P.l2w[1], czz = P.l2w[2], cxy = P.l2w[3], cxz = P.l2w[4], cyz = P.l2w[5];
        // d_x D_x, d_y D_y, d_z D_z
        const float dxDx = fmaf(cxx, wx_xx, fmaf(cxy, mxyY.x, cxz * mxzY.y));
        const float dyDy = fmaf(cxy, mxyY.x, fmaf(cyy, wy_yy, cyz * myzZ));
        const float dzDz = fmaf(cxz, mxzY.y, fmaf(cyz, myzZ, czz * wz_zz));
        // mixed: d_x D_y + d_y D_x, d_x D_z + d_z D_x, d_y D_z + d_z D_y
        const float sxy = fmaf(cxx, wx_xy, fmaf(cxy, mxyX.y, fmaf(cxz, mxzZ,
                          fmaf(cxy, mxyX.x, fmaf(cyy, wy_xy, cyz * myzY.y)))));
        const float sxz = fmaf(cxx, wx_xz, fmaf(cxy, mxyZ, fmaf(cxz, mxz_zz,
                          fmaf(cxz, mxzX.x, fmaf(cyz, myzY.x, czz * wz_xz)))));
        const float syz = fmaf(cxy, mxyY.y, fmaf(cyy, wy_yz, fmaf(cyz, myz_zz,
                          fmaf(cxz, mxzY.x, fmaf(cyz, myzX.y, czz * wz_yz)))));
        hX = fma2(bc2(-1.0f), make_float2(dxDx, dyDy), hX);
        hY = fma2(bc2(-1.0f), make_float2(sxy, sxz), hY);
        hzz -= dzDz;
        hyz -= syz;
    }
    float corr = (hX.x + hX.y + hzz) * (1.0f / 3.0f);
    float2 muX = add2(hX, bc2(-corr));  // (mu_xx, mu_yy)
    float2 muY = hY;                    // (mu_xy, mu_xz)
    float muZ = hyz;                    // mu_yz
    if (kL3) {
        // undivided central differences per axis
        const float2 dXx = sub2(Xpx, Xmx), dXy = sub2(Xpy, Xmy), dXz = sub2(Xpz, Xmz);
        const float2 dYx = sub2(Ypx, Ymx), dYy = sub2(Ypy, Ymy), dYz = sub2(Ypz, Ymz);
        const float dZx = Zpx - Zmx, dZy = Zpy - Zmy, dZz = Zpz - Zmz;
        const float d5x = -(dXx.x + dXx.y), d5y = -(dXy.x + dXy.y), d5z = -(dXz.x + dXz.y);  // zz
        // M_ab = dQ_kl/da dQ_kl/db over all nine entries: xx, yy, zz once, off-diagonals twice
        const float2 dYx2 = add2(dYx, dYx), dYy2 = add2(dYy, dYy), dYz2 = add2(dYz, dYz);
        auto M = [&](float2 xa, float2 xb, float2 ya, float2 yb2, float za, float zb, float va, float vb) {
            const float2 t = fma2(ya, yb2, mul2(xa, xb));
            return fmaf(2.0f * za, zb, fmaf(va, vb, t.x + t.y));
        };
        float hxx = fmaf(P.l3m[0], M(dXx, dXx, dYx, dYx2, dZx, dZx, d5x, d5x), muX.x);
        float hyy = fmaf(P.l3m[1], M(dXy, dXy, dYy, dYy2, dZy, dZy, d5y, d5y), muX.y);
        float hz = fmaf(P.l3m[2], M(dXz, dXz, dYz, dYz2, dZz, dZz, d5z, d5z), -(muX.x + muX.y));
        float hxy = fmaf(P.l3m[3], M(dXx, dXy, dYx, dYy2, dZx, dZy, d5x, d5y), muY.x);
        float hxz = fmaf(P.l3m[4], M(dXx, dXz, dYx, dYz2, dZx, dZz, d5x, d5z), muY.y);
        float hyz3 = fmaf(P.l3m[5], M(dXy, dXz, dYy, dYz2, dZy, dZz, d5y, d5z), muZ);
        // column divergence at the centre: D_x = d_x Q_xx + d_y Q_xy + d_z Q_xz, ... (QSR.cu:325-371)
        const float Dx = fmaf(P.i2x, dXx.x, fmaf(P.i2y, dYy.x, P.i2z * dYz.y));
        const float Dy = fmaf(P.i2x, dYx.x, fmaf(P.i2y, dXy.y, P.i2z * dZz));
        const float Dz = fmaf(P.i2x, dYx.y, fmaf(P.i2y, dZy, P.i2z * d5z));
        // B(Q_c) = D . grad Q_c + Q_ab d_a d_b Q_c (QSR.cu:580-603) on all components at once:
        // weights of the six second derivatives, shared by every component
        const float Qzz = -q[0] - q[3];
        const float2 wxx = bc2(q[0] * P.ix2), wyy = bc2(q[3] * P.iy2), wzz = bc2(Qzz * P.iz2);
        const float2 wxy = bc2(2.0f * q[1] * P.i4xy), wxz = bc2(2.0f * q[2] * P.i4xz), wyz = bc2(2.0f * q[4] * P.i4yz);
        const float2 Dc0 = bc2(Dx * P.i2x), Dc1 = bc2(Dy * P.i2y), Dc2 = bc2(Dz * P.i2z);
        const float2 q2X = add2(qX, qX), q2Y = add2(qY, qY);
        const float2 cX = fma2(wxx, sub2(sxX, q2X), fma2(wyy, sub2(syX, q2X), fma2(wzz, sub2(szX, q2X),
                          fma2(wxy, mxyX, fma2(wxz, mxzX, mul2(wyz, myzX))))));
        const float2 cY = fma2(wxx, sub2(sxY, q2Y), fma2(wyy, sub2(syY, q2Y), fma2(wzz, sub2(szY, q2Y),
                          fma2(wxy, mxyY, fma2(wxz, mxzY, mul2(wyz, myzY))))));
        const float q2Z = 2.0f * qZ;
        const float cZ = fmaf(wxx.x, sxZ - q2Z, fmaf(wyy.x, syZ - q2Z, fmaf(wzz.x, szZ - q2Z,
                         fmaf(wxy.x, mxyZ, fmaf(wxz.x, mxzZ, wyz.x * myzZ)))));
        const float2 BX = fma2(Dc0, dXx, fma2(Dc1, dXy, fma2(Dc2, dXz, cX)));  // (B_xx, B_yy)
        const float2 BY = fma2(Dc0, dYx, fma2(Dc1, dYy, fma2(Dc2, dYz, cY)));  // (B_xy, B_xz)
        const float BZ = fmaf(Dc0.x, dZx, fmaf(Dc1.x, dZy, fmaf(Dc2.x, dZz, cZ)));  // B_yz
        // h -= L3 B, B_zz = -(B_xx + B_yy); re-projected traceless (QSR.cu:611-619)
        const float2 hdX = fma2(bc2(-P.L3), BX, make_float2(hxx, hyy));
        const float2 hdY = fma2(bc2(-P.L3), BY, make_float2(hxy, hxz));
        hz = fmaf(P.L3, BX.x + BX.y, hz);
        hyz3 = fmaf(-P.L3, BZ, hyz3);
        corr = (hdX.x + hdX.y + hz) * (1.0f / 3.0f);
        muX = add2(hdX, bc2(-corr));
        muY = hdY;
        muZ = hyz3;
    }
    mu[0] = muX.x; mu[3] = muX.y; mu[1] = muY.x; mu[2] = muY.y; mu[4] = muZ;
    if (anchor) {
        float Q0[5];
        surface_q0(P, i, j, k, Q0);
#pragma unroll
        for (int c = 0; c < 5; ++c) mu[c] += P.Weff * (q[c] - Q0[c]);
    }
}

// ---------------------------------------------------------------------------------------
// Two cells at once: F2 holds one value of two different cells, and every operation on it is
// one packed instruction (FFMA2 / FADD2 / FMUL2) for both cells. chem_interior_pair is the
// interior chemical potential of chem_potential_interior_x2 written on F2.
// ---------------------------------------------------------------------------------------
struct F2 {
    float2 v;
};
__device__ __forceinline__ F2 mk2(float a, float b) { return F2{make_float2(a, b)}; }
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2{__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return F2{__ffma2_rn(b.v, make_float2(-1.0f, -1.0f), a.v)}; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return F2{__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator*(float s, F2 b) { return F2{__fmul2_rn(make_float2(s, s), b.v)}; }
__device__ __forceinline__ F2 operator-(F2 a) { return F2{__fmul2_rn(a.v, make_float2(-1.0f, -1.0f))}; }
__device__ __forceinline__ F2 vfma(F2 a, F2 b, F2 c) { return F2{__ffma2_rn(a.v, b.v, c.v)}; }
__device__ __forceinline__ F2 vfma(float a, F2 b, F2 c) { return F2{__ffma2_rn(make_float2(a, a), b.v, c.v)}; }

__device__ __forceinline__ void bulk_field_pair(const F2 q[5], float cQ, float cQ2, float cQ3, F2 h[6]) {
    const F2 Qxx = q[0], Qxy = q[1], Qxz = q[2], Qyy = q[3], Qyz = q[4];
    const F2 Qzz = -(Qxx + Qyy);
    const F2 trQ2 = vfma(Qxx, Qxx, vfma(Qyy, Qyy, Qzz * Qzz)) +
                    2.0f * vfma(Qxy, Qxy, vfma(Qxz, Qxz, Qyz * Qyz));
    const F2 q2xx = vfma(Qxx, Qxx, vfma(Qxy, Qxy, Qxz * Qxz));
    const F2 q2xy = vfma(Qxx, Qxy, vfma(Qxy, Qyy, Qxz * Qyz));
    const F2 q2xz = vfma(Qxx, Qxz, vfma(Qxy, Qyz, Qxz * Qzz));
    const F2 q2yy = vfma(Qxy, Qxy, vfma(Qyy, Qyy, Qyz * Qyz));
    const F2 q2yz = vfma(Qxy, Qxz, vfma(Qyy, Qyz, Qyz * Qzz));
    const F2 q2zz = vfma(Qxz, Qxz, vfma(Qyz, Qyz, Qzz * Qzz));
    const F2 t3 = (1.0f / 3.0f) * trQ2;
    const F2 cg = vfma(cQ3, trQ2, mk2(cQ, cQ));
    h[0] = vfma(-cQ2, q2xx - t3, cg * Qxx);
    h[1] = vfma(-cQ2, q2yy - t3, cg * Qyy);
    h[2] = vfma(-cQ2, q2zz - t3, cg * Qzz);
    h[3] = vfma(-cQ2, q2xy, cg * Qxy);
    h[4] = vfma(-cQ2, q2xz, cg * Qxz);
    h[5] = vfma(-cQ2, q2yz, cg * Qyz);
}

// A(c, di, dj, dk) returns an F2 (component c of both cells at that offset; c = 5 is Qzz).
// The terms are formed one stored component at a time (components 0 xx, 1 xy, 2 xz, 3 yy, 4 yz),
// so that only the first differences of every component stay live for M_ab and the divergence:
//  * its face neighbours give its Laplacian and first differences;
//  * its four-corner and wide second differences go straight into the L2 term d_a D_b, which for
//    an interior cell is sum_k S_ak(Q_kb) / (4 da dk) (wide second difference for k = a, four
//    corners for k != a), and into its L3 contraction Q_ab d_a d_b Q_c;
//  * h is projected traceless once at the end (the projection is linear, so projecting after the
//    L1/L2 terms and again after L3, as QSR.cu:462-469 and 611-619 do, gives the same result).
template <bool kL2, bool kL3, class Acc>
__device__ __forceinline__ void chem_interior_pair(const Acc& A, const QsrConst& P, const F2 q[5], F2 mu[5],
                                                   F2 lap[5]) {
    F2 h[6];
    bulk_field_pair(q, P.cQ, P.cQ2, P.cQ3, h);
    const float cxx = P.l2w[0], cyy = P.l2w[1], czz = P.l2w[2], cxy = P.l2w[3], cxz = P.l2w[4], cyz = P.l2w[5];
    // second-derivative weights of the L3 contraction, shared by every component
    const F2 Qzz = -(q[0] + q[3]);
    const F2 wxx = P.ix2 * q[0], wyy = P.iy2 * q[3], wzz = P.iz2 * Qzz;
    const F2 wxy = (2.0f * P.i4xy) * q[1], wxz = (2.0f * P.i4xz) * q[2], wyz = (2.0f * P.i4yz) * q[4];
    F2 d[5][3], contract[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        const F2 px = A(c, 1, 0, 0), mx = A(c, -1, 0, 0), py = A(c, 0, 1, 0), my = A(c, 0, -1, 0);
        const F2 pz = A(c, 0, 0, 1), mz = A(c, 0, 0, -1);
        const F2 sx = px + mx, sy = py + my, sz = pz + mz;
        d[c][0] = px - mx;
        d[c][1] = py - my;
        d[c][2] = pz - mz;
        lap[c] = vfma(P.ix2, sx, vfma(P.iy2, sy, vfma(P.iz2, sz, P.lap_c * q[c])));
        // -Liso lap into h (h_zz takes -Liso lap_zz = Liso (lap_xx + lap_yy))
        if (c == 0) { h[0] = vfma(-P.Liso, lap[c], h[0]); h[2] = vfma(P.Liso, lap[c], h[2]); }
        if (c == 3) { h[1] = vfma(-P.Liso, lap[c], h[1]); h[2] = vfma(P.Liso, lap[c], h[2]); }
        if (c == 1) h[3] = vfma(-P.Liso, lap[c], h[3]);
        if (c == 2) h[4] = vfma(-P.Liso, lap[c], h[4]);
        if (c == 4) h[5] = vfma(-P.Liso, lap[c], h[5]);
        if (kL2 || kL3) {
            const F2 mxy = (A(c, 1, 1, 0) - A(c, 1, -1, 0)) - (A(c, -1, 1, 0) - A(c, -1, -1, 0));
            const F2 mxz = (A(c, 1, 0, 1) - A(c, 1, 0, -1)) - (A(c, -1, 0, 1) - A(c, -1, 0, -1));
            const F2 myz = (A(c, 0, 1, 1) - A(c, 0, 1, -1)) - (A(c, 0, -1, 1) - A(c, 0, -1, -1));
            if (kL2) {
                const F2 q2 = 2.0f * q[c];
                if (c == 0) {  // xx
                    h[0] = vfma(-cxx, (A(0, 2, 0, 0) + A(0, -2, 0, 0)) - q2, h[0]);
                    h[2] = vfma(czz, (A(0, 0, 0, 2) + A(0, 0, 0, -2)) - q2, h[2]);
                    h[3] = vfma(-cxy, mxy, h[3]);
                    h[5] = vfma(cyz, myz, h[5]);
                } else if (c == 3) {  // yy
                    h[1] = vfma(-cyy, (A(3, 0, 2, 0) + A(3, 0, -2, 0)) - q2, h[1]);
                    h[2] = vfma(czz, (A(3, 0, 0, 2) + A(3, 0, 0, -2)) - q2, h[2]);
                    h[3] = vfma(-cxy, mxy, h[3]);
                    h[4] = vfma(cxz, mxz, h[4]);
                } else if (c == 1) {  // xy
                    h[0] = vfma(-cxy, mxy, h[0]);
                    h[1] = vfma(-cxy, mxy, h[1]);
                    h[3] = vfma(-cxx, (A(1, 2, 0, 0) + A(1, -2, 0, 0)) - q2, h[3]);
                    h[3] = vfma(-cyy, (A(1, 0, 2, 0) + A(1, 0, -2, 0)) - q2, h[3]);
                    h[4] = vfma(-cyz, myz, h[4]);
                    h[5] = vfma(-cxz, mxz, h[5]);
                } else if (c == 2) {  // xz
                    h[0] = vfma(-cxz, mxz, h[0]);
                    h[2] = vfma(-cxz, mxz, h[2]);
                    h[3] = vfma(-cyz, myz, h[3]);
                    h[4] = vfma(-cxx, (A(2, 2, 0, 0) + A(2, -2, 0, 0)) - q2, h[4]);
                    h[4] = vfma(-czz, (A(2, 0, 0, 2) + A(2, 0, 0, -2)) - q2, h[4]);
                    h[5] = vfma(-cxy, mxy, h[5]);
                } else {  // yz
                    h[1] = vfma(-cyz, myz, h[1]);
                    h[2] = vfma(-cyz, myz, h[2]);
                    h[3] = vfma(-cxz, mxz, h[3]);
                    h[4] = vfma(-cxy, mxy, h[4]);
                    h[5] = vfma(-cyy, (A(4, 0, 2, 0) + A(4, 0, -2, 0)) - q2, h[5]);
                    h[5] = vfma(-czz, (A(4, 0, 0, 2) + A(4, 0, 0, -2)) - q2, h[5]);
                }
            }
            if (kL3) {
                const F2 q2 = 2.0f * q[c];
                contract[c] = vfma(wxx, sx - q2, vfma(wyy, sy - q2, vfma(wzz, sz - q2,
                              vfma(wxy, mxy, vfma(wxz, mxz, wyz * myz)))));
            }
        }
    }
    if (kL3) {
        F2 d5[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) d5[a] = -(d[0][a] + d[3][a]);
        auto M = [&](int a, int b) {
            const F2 diag = vfma(d[0][a], d[0][b], vfma(d[3][a], d[3][b], d5[a] * d5[b]));
            const F2 off = vfma(d[1][a], d[1][b], vfma(d[2][a], d[2][b], d[4][a] * d[4][b]));
            return vfma(2.0f, off, diag);
        };
        // (L3 / 2) M_ab: h_zz first, as -(hx_xx + hx_yy) of the projected field gets it below
        h[0] = vfma(P.l3m[0], M(0, 0), h[0]);
        h[1] = vfma(P.l3m[1], M(1, 1), h[1]);
        h[2] = vfma(P.l3m[2], M(2, 2), h[2]);
        h[3] = vfma(P.l3m[3], M(0, 1), h[3]);
        h[4] = vfma(P.l3m[4], M(0, 2), h[4]);
        h[5] = vfma(P.l3m[5], M(1, 2), h[5]);
        // centre divergence D_x = d_x Q_xx + d_y Q_xy + d_z Q_xz, ... (QSR.cu:325-371), times 1/(2 da)
        const F2 Dc0 = P.i2x * vfma(P.i2x, d[0][0], vfma(P.i2y, d[1][1], P.i2z * d[2][2]));
        const F2 Dc1 = P.i2y * vfma(P.i2x, d[1][0], vfma(P.i2y, d[3][1], P.i2z * d[4][2]));
        const F2 Dc2 = P.i2z * vfma(P.i2x, d[2][0], vfma(P.i2y, d[4][1], P.i2z * d5[2]));
        F2 B[5];
#pragma unroll
        for (int c = 0; c < 5; ++c) B[c] = vfma(Dc0, d[c][0], vfma(Dc1, d[c][1], vfma(Dc2, d[c][2], contract[c])));
        h[0] = vfma(-P.L3, B[0], h[0]);
        h[1] = vfma(-P.L3, B[3], h[1]);
        h[2] = vfma(P.L3, B[0] + B[3], h[2]);  // - L3 B_zz, B_zz = -(B_xx + B_yy)
        h[3] = vfma(-P.L3, B[1], h[3]);
        h[4] = vfma(-P.L3, B[2], h[4]);
        h[5] = vfma(-P.L3, B[4], h[5]);
    }
    const F2 corr = (1.0f / 3.0f) * (h[0] + h[1] + h[2]);
    mu[0] = h[0] - corr;
    mu[1] = h[3];
    mu[2] = h[4];
    mu[3] = h[1] - corr;
    mu[4] = h[5];
}

// Explicit update with compensated storage: a cell holds hi + lo (two FP32 words). The
// increment -(dt/gamma) mu (+ noise) is added to hi exactly (Knuth's TwoSum) and the rounding
// error carried in lo, so the stored value keeps about 48 significant bits over any number of
// steps while the stencil arithmetic stays FP32. On return out = new hi, lo = new lo.
__device__ __forceinline__ void euler_update_comp(const QsrConst& P, const float q[5], float lo[5], const float mu[5],
                                                  uint32_t cell, bool noise, float out[5]) {
    float d[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) d[c] = -mu[c] * P.mob_dt;
    if (noise) {
        float g[5];
        normals5(cell, P.instance, P.step, P.key0, P.key1, g);
#pragma unroll
        for (int c = 0; c < 5; ++c) d[c] += P.sigma * g[c];
    }
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        const float s = __fadd_rn(q[c], d[c]);
        const float bp = __fsub_rn(s, q[c]);
        const float e = __fadd_rn(__fsub_rn(q[c], __fsub_rn(s, bp)), __fsub_rn(d[c], bp));
        const float t = __fadd_rn(e, lo[c]);
        const float h = __fadd_rn(s, t);
        lo[c] = __fsub_rn(t, __fsub_rn(h, s));
        out[c] = h;
    }
    if (P.qcap > 0.0f) {
        const float zz = -out[0] - out[3];
        const float tr = out[0] * out[0] + out[3] * out[3] + zz * zz +
                         2.0f * (out[1] * out[1] + out[2] * out[2] + out[4] * out[4]);
        const float qn = sqrtf(tr > 0.0f ? tr : 0.0f);
        if (qn > P.qcap && qn > 0.0f) {
            const float sc = P.qcap / qn;
#pragma unroll
            for (int c = 0; c < 5; ++c) { out[c] *= sc; lo[c] *= sc; }
        }
    }
}

// Explicit Euler update with optional Langevin noise and Frobenius cap (QSR.cu:711-731).
__device__ __forceinline__ void euler_update(const QsrConst& P, const float q[5], const float mu[5], uint32_t cell,
                                             bool noise, float out[5]) {
#pragma unroll
    for (int c = 0; c < 5; ++c) out[c] = q[c] - mu[c] * P.mob_dt;
    if (noise) {
        float g[5];
        normals5(cell, P.instance, P.step, P.key0, P.key1, g);
#pragma unroll
        for (int c = 0; c < 5; ++c) out[c] += P.sigma * g[c];
    }
    if (P.qcap > 0.0f) {
        const float zz = -out[0] - out[3];
        const float tr = out[0] * out[0] + out[3] * out[3] + zz * zz +
                         2.0f * (out[1] * out[1] + out[2] * out[2] + out[4] * out[4]);
        const float qn = sqrtf(tr > 0.0f ? tr : 0.0f);
        if (qn > P.qcap && qn > 0.0f) {
            const float s = P.qcap / qn;
#pragma unroll
            for (int c = 0; c < 5; ++c) out[c] *= s;
        }
    }
}

// ---------------------------------------------------------------------------------------
// FP64 nematic eigen-solver (QSR.cu:191-243): shifted power iteration for the largest
// eigenvalue, S = 1.5 lambda, director gauge nz >= 0.
// ---------------------------------------------------------------------------------------
struct Nematic { double S, nx, ny, nz; };

__device__ __forceinline__ Nematic nematic64(const double q[5], double iso_cut, Nematic iso) {
    const double Qxx = q[0], Qxy = q[1], Qxz = q[2], Qyy = q[3], Qyz = q[4];
    const double Qzz = -Qxx - Qyy;
    if (fabs(Qxx) < iso_cut && fabs(Qxy) < iso_cut && fabs(Qxz) < iso_cut && fabs(Qyy) < iso_cut &&
        fabs(Qyz) < iso_cut)
        return iso;
    double nx = Qxx + Qxy + Qxz, ny = Qxy + Qyy + Qyz, nz = Qxz + Qyz - Qxx - Qyy;
    const double n0 = sqrt(nx * nx + ny * ny + nz * nz);
    if (n0 > 1e-12) { nx /= n0; ny /= n0; nz /= n0; }
    else { nx = 0.0; ny = 0.0; nz = 1.0; }
    const double r1 = fabs(Qxx) + fabs(Qxy) + fabs(Qxz);
    const double r2 = fabs(Qxy) + fabs(Qyy) + fabs(Qyz);
    const double r3 = fabs(Qxz) + fabs(Qyz) + fabs(Qzz);
    const double alpha = fmax(r1, fmax(r2, r3)) + 1e-12;
    for (int it = 0; it < 15; ++it) {
        const double ax = Qxx * nx + Qxy * ny + Qxz * nz + alpha * nx;
        const double ay = Qxy * nx + Qyy * ny + Qyz * nz + alpha * ny;
        const double az = Qxz * nx + Qyz * ny + Qzz * nz + alpha * nz;
        const double nn = sqrt(ax * ax + ay * ay + az * az);
        if (nn < 1e-13) break;
        nx = ax / nn; ny = ay / nn; nz = az / nn;
    }
    const double lam = nx * (Qxx * nx + Qxy * ny + Qxz * nz) + ny * (Qxy * nx + Qyy * ny + Qyz * nz) +
                       nz * (Qxz * nx + Qyz * ny + Qzz * nz);
    Nematic r{1.5 * lam, nx, ny, nz};
    if (nz < -1e-10) { r.nx = -nx; r.ny = -ny; r.nz = -nz; }
    return r;
}

// Warp and block reductions (fixed order: deterministic for a fixed launch shape).
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

}  // namespace ldg
