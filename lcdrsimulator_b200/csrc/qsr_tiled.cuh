// Tiled confined-solver step kernel for sm_100a.
//
// A CTA owns a (TJ x TK) column tile of the (j, k) plane and marches along i over a chunk
// of planes. Each plane of the input field arrives in shared memory through one TMA load
// of a 4-D box (k, j, i, component) covering the tile plus a halo of 2 rows and 4 columns
// (the k start stays on a 16-byte boundary), so every Q value is read from HBM about once.
// The ring holds the planes i-2 .. i+2 that the cells of plane i read, plus planes in flight.
// Interior cells read only Q: the L2 term's derivatives of the column divergence are
// evaluated from Q directly (wide and four-corner second differences, which for an interior
// cell equal the reference's central differences of its central divergence), so no divergence
// field is staged and the warps share nothing but the plane ring. Each warp (one tile row)
// therefore marches on its own: it waits only for the TMA of the planes it reads, and when it
// is done with a plane it arrives on that slot's counter; the warp whose arrival completes the
// count issues the load of the plane that reuses the slot. There is no CTA barrier per plane.
// Cells next to a grid face take the reference's face stencils with the divergence evaluated on
// the fly. Per cell the kernel evaluates the chemical potential and the update from shared memory
// and writes only the cells that change (moving and strongly anchored cells): frozen exterior
// cells hold identical values in both ping-pong buffers. Tiles that contain no changing cell are
// never visited (host-built work list). The same per-tile routine drives a persistent,
// work-stealing ensemble kernel over many droplets.
//
// mbarrier waits are bounded: on timeout the kernel records LDG_ERR_TIMEOUT in a device
// word, waits (bounded) for its own TMA loads and returns.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <string>
#include <vector>

#include "ldg_api_common.h"
#include "ldg_common.cuh"

namespace ldg {

namespace tiled {

constexpr int TK = 32;               // tile width along k (one warp per row)
constexpr int TJ = 8;                // tile rows along j (one warp each)
constexpr int THREADS = TK * TJ;
constexpr int NWARP = THREADS / 32;
// Halo rows / columns loaded with each plane: the stencils reach two cells out. The TMA box
// starts at column k0 - HK, which must be a multiple of 4 floats (16 bytes), so tiles start at
// k0 = 2 (mod 4) (the first may start at k0 = -2: its two columns outside the grid are zero
// fill and compute nothing).
constexpr int HJ = 2, HK = 2;
constexpr int RW = TK + 2 * HK;      // 36 floats per smem row
constexpr int ROWS = TJ + 2 * HJ;    // 12 rows
constexpr int CSTR = RW * ROWS;      // floats per component plane
constexpr int PLANE = 5 * CSTR;      // floats per plane (all components)
constexpr int SLOT = (PLANE + 31) / 32 * 32;  // floats per ring slot (TMA destinations 128-byte aligned)
constexpr int LOOK = 2;              // the cells of plane i read planes i-2 .. i+2
// Q ring slots: planes i-2 .. i+2 are read at plane i, the rest are in flight. The L1-only step
// runs three CTAs (24 warps) per SM: 7 slots (~67 KB) and at most 80 registers a thread. The
// L2/L3 steps need more registers (the mixed and wide second differences) and run two CTAs per
// SM with 9 slots (~86 KB, four planes in flight).
// (two cells per thread: 128-thread CTAs, four per SM, 6 slots ~ 52 KB)
template <bool kD, bool kPair = false>
__host__ __device__ constexpr int nq() { return kPair ? 6 : (kD ? 9 : 7); }
constexpr uint32_t PLANE_BYTES = PLANE * 4;
constexpr int CHUNK = 16;            // planes per work item (default; tunable)
constexpr unsigned long long WAIT_NS = 2000000000ull;  // 2 s per wait

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t n) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(n) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}
// One bounded try: the thread may wait in the barrier for a system-dependent time before the
// try returns false. (A suspend-time hint of 1 ms made the two-cell steps 1-2 % slower.)
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
// Waits for the phase with the given parity, giving up after WAIT_NS of wall time.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* b, uint32_t parity) {
    if (mbar_try_wait(b, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (true) {
        if (mbar_try_wait(b, parity)) return true;
        if (global_ns() - t0 > WAIT_NS) return false;
    }
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* tm, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(su32(dst)),
        "l"(tm), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(su32(bar))
        : "memory");
}

// Shared-memory Q accessor centred on local cell (jl, kl) of plane i; planes i-2..i+2.
struct SmemQ {
    const float* pl[5];
    int off;
    __device__ __forceinline__ float operator()(int c, int di, int dj, int dk) const {
        const float* s = pl[di + 2] + off + dj * RW + dk;
        if (c < 5) return s[c * CSTR];
        return -(s[0] + s[3 * CSTR]);
    }
};

// Column divergence D_comp at offset (di, dj, dk) of cell (i, j, k), evaluated on the fly from a
// Q accessor with the reference's face stencils (QSR.cu:325-371): the face path of the tiled kernel.
template <class Acc>
struct FlyD {
    const Acc* A;
    const QsrConst* P;
    int i, j, k;
    __device__ __forceinline__ float operator()(int comp, int di, int dj, int dk) const {
        float D[3];
        dcol_at(*A, *P, i, j, k, di, dj, dk, D);
        return D[comp];
    }
};

// Shared-memory layout of one CTA of the tiled kernels.
struct TileSmem {
    float* sq;          // nq planes of Q (tile + halo, 5 components)
    uint64_t* bar;      // nq mbarriers, one per Q slot (TMA completion)
    unsigned* freed;    // nq counters of warps done with the slot's plane
    int* s_abort;       // set when a bounded wait gave up
    int* s_item;        // work item broadcast (persistent kernel)
};

template <bool kD, bool kPair = false>
__device__ __forceinline__ TileSmem tile_smem(unsigned char* raw) {
    constexpr int NQ = nq<kD, kPair>();
    TileSmem S;
    S.sq = reinterpret_cast<float*>(raw);
    S.bar = reinterpret_cast<uint64_t*>(S.sq + NQ * SLOT);
    S.freed = reinterpret_cast<unsigned*>(S.bar + NQ);
    S.s_abort = reinterpret_cast<int*>(S.freed + NQ);
    S.s_item = S.s_abort + 1;
    return S;
}
template <bool kD, bool kPair = false>
__host__ __device__ constexpr size_t tile_smem_bytes() {
    return (size_t)nq<kD, kPair>() * SLOT * 4 + nq<kD, kPair>() * 8 + nq<kD, kPair>() * 4 + 16;
}

// A warp's arrival on a slot counter: returns the count before it (acquire-release at CTA
// scope, so the warp's reads of the plane happen before the slot is refilled).
__device__ __forceinline__ unsigned arrive_freed(unsigned* ctr) {
    unsigned old;
    asm volatile("atom.acq_rel.cta.shared::cta.add.u32 %0, [%1], 1;" : "=r"(old) : "r"(su32(ctr)) : "memory");
    return old;
}

// One work item: the (TJ x TK) column tile at (j0, k0) over planes [ib, ie). `phase` holds the
// parity of the next phase of every slot barrier (bit s for slot s), so a CTA can run many
// items in a row; every load the item issues is waited for by every warp before it returns.
// Returns false when a bounded wait gave up (the CTA must stop). The caller synchronises the CTA
// before and after an item.
// kComp: compensated storage (explicit steps only): the low words of the input cells are read
// from lo_in and the new low words written to lo_out.
template <bool kL2, bool kL3, bool kNoise, bool kRHS, bool kComp = false>
__device__ __forceinline__ bool process_tile(const CUtensorMap* tm, float* __restrict__ qout,
                                             const uint8_t* __restrict__ flags, int j0, int k0, int ib, int ie,
                                             const QsrConst& P, const TileSmem& S, uint32_t& phase,
                                             int* __restrict__ err, const float* __restrict__ lo_in = nullptr,
                                             float* __restrict__ lo_out = nullptr) {
    constexpr int NQ = nq<kL2 || kL3>();
    float* sq = S.sq;
    uint64_t* bar = S.bar;
    const int base = ib - 2;  // first plane this item loads; slots and phases count from it
    const int tid = threadIdx.x;
    const int kl = tid & 31, jl = tid >> 5;

    // Plane p (p >= base) lives in slot (p - base) % NQ and completes that slot's barrier phase
    // number (p - base) / NQ of this item (every caller has p >= base: unsigned arithmetic).
    auto slot = [&](int p) { return (uint32_t)(p - base) % (uint32_t)NQ; };
    auto parity = [&](int p) { return ((phase >> slot(p)) & 1u) ^ (((uint32_t)(p - base) / (uint32_t)NQ) & 1u); };

    // Planes outside the grid, and planes past the last one this item reads (ie - 1 + LOOK),
    // complete their phase with a plain arrive (no data).
    auto issue = [&](int p) {
        uint64_t* b = &bar[slot(p)];
        if (p >= 0 && p < P.Nx && p < ie + LOOK) {
            fence_proxy_async();
            mbar_expect_tx(b, PLANE_BYTES);
            tma_load_4d(sq + slot(p) * SLOT, tm, k0 - HK, j0 - HJ, p, 0, b);
        } else {
            mbar_arrive(b);
        }
    };
    if (tid == 0)
        for (int p = base; p < base + NQ; ++p) issue(p);
    bool ok = true;
    auto wait_plane = [&](int p) {
        if (!mbar_wait_bounded(&bar[slot(p)], parity(p))) {
            atomicExch(err, LDG_ERR_TIMEOUT);
            *(volatile int*)S.s_abort = 1;
            ok = false;
        }
    };
    // Planes [base, ie + NQ - 2) are issued: the first NQ here, then plane p + NQ when the last
    // warp is done with plane p (after its plane p + 2), for every p <= ie - 3.
    const int issued_end = ie + NQ - 2;

    const int j = j0 + jl, k = k0 + kl;
    const bool in_grid = (j < P.Ny) && (k >= 0) && (k < P.Nz);
    // Interior cells take the Q-only path: every stencil position within the grid away from the
    // faces (the L2 term reaches two cells out: 2 <= pos <= N - 3; otherwise 1 <= pos <= N - 2).
    constexpr int kLo = kL2 ? 2 : 1;
    const bool jk_interior = j >= kLo && j <= P.Ny - 1 - kLo && k >= kLo && k <= P.Nz - 1 - kLo;
    const long long cell0 = (long long)j * P.sj + k;
    uint8_t f_next = in_grid ? __ldg(flags + (long long)ib * P.si + cell0) : 0;
    // Shared-memory planes i-2 .. i+2 of the current step, rolled forward by one plane per step.
    const float* qpl[5];
#pragma unroll
    for (int d = 0; d < 5; ++d) qpl[d] = sq + slot(ib + d - 2) * SLOT;
    int waited_end = base;
    for (int p = base; p <= ib + LOOK - 1; ++p) wait_plane(p);
    waited_end = ib + LOOK;
    for (int i = ib; i < ie; ++i) {
        if (*(volatile int*)S.s_abort) { ok = false; break; }  // another warp gave up
        const uint8_t f = f_next;
        if (in_grid && i + 1 < ie) f_next = __ldg(flags + (long long)(i + 1) * P.si + cell0);
        wait_plane(i + LOOK);
        waited_end = i + LOOK + 1;
        if (!ok) break;
        const bool fixed = in_grid && !kRHS && (f & kFixed);
        const bool move = in_grid && (f & kMove) != 0;
        // The Q-only interior form is taken by a whole warp when none of its computing cells is
        // near a face (exterior cells of a droplet compute nothing, so small droplets use it too).
        const bool warp_interior =
            __all_sync(0xffffffffu, !move || (jk_interior && i >= kLo && i <= P.Nx - 1 - kLo)) != 0;
        if (fixed || move) {
            const long long id = (long long)i * P.si + cell0;
            SmemQ A;
#pragma unroll
            for (int d = 0; d < 5; ++d) A.pl[d] = qpl[d];
            A.off = (jl + HJ) * RW + (kl + HK);
            float c[5], o[5];
#pragma unroll
            for (int m = 0; m < 5; ++m) c[m] = A(m, 0, 0, 0);
            if (fixed) {
                surface_q0(P, i, j, k, o);
                if (kComp) {
#pragma unroll
                    for (int m = 0; m < 5; ++m) lo_out[m * P.sc + id] = 0.0f;
                }
            } else {
                float mu[5], lap[5];
                if (warp_interior) {
                    chem_potential_interior_x2<kL2, kL3>(A, P, i, j, k, c, (f & kAnchor) != 0, mu, lap);
                } else {
                    const FlyD<SmemQ> DA{&A, &P, i, j, k};
                    chem_potential<kL2, kL3, true>(A, DA, P, i, j, k, c, (f & kAnchor) != 0, mu, lap);
                }
                const uint32_t cell = (uint32_t)(k + P.Nz * (j + P.Ny * i));
                if (kRHS) {
#pragma unroll
                    for (int m = 0; m < 5; ++m) o[m] = c[m] - P.mob_dt * mu[m] - P.alpha * lap[m];
                    if (kNoise) {
                        float g[5];
                        normals5(cell, P.instance, P.step, P.key0, P.key1, g);
#pragma unroll
                        for (int m = 0; m < 5; ++m) o[m] += P.sigma * g[m];
                    }
                } else if (kComp) {
                    float lo[5];
#pragma unroll
                    for (int m = 0; m < 5; ++m) lo[m] = __ldg(lo_in + m * P.sc + id);
                    euler_update_comp(P, c, lo, mu, cell, kNoise, o);
#pragma unroll
                    for (int m = 0; m < 5; ++m) lo_out[m * P.sc + id] = lo[m];
                } else {
                    euler_update(P, c, mu, cell, kNoise, o);
                }
            }
#pragma unroll
            for (int m = 0; m < 5; ++m) qout[m * P.sc + id] = o[m];
        }
        // This warp is done with plane i-2: arrive on its slot; the last warp refills the slot with
        // plane i-2+NQ.
        __syncwarp();
        if (kl == 0) {
            const uint32_t s = slot(i - 2);
            if (arrive_freed(&S.freed[s]) % (unsigned)NWARP == (unsigned)NWARP - 1u) issue(i - 2 + NQ);
        }
#pragma unroll
        for (int d = 0; d < 4; ++d) qpl[d] = qpl[d + 1];
        qpl[4] = sq + slot(i + 3) * SLOT;
    }
    // Drain: every load this item issues lands before the slots are reused or released. After
    // an abort some refills are never issued; those waits give up after their bound.
    if (ok) {
        for (int p = waited_end; p < issued_end; ++p) wait_plane(p);
    } else {
        for (int p = waited_end; p < issued_end; ++p)
            if (!mbar_wait_bounded(&bar[slot(p)], parity(p))) break;
    }
    // Advance the per-slot phase parities by the number of loads each slot received.
    const int n_issued = issued_end - base;
#pragma unroll
    for (int s = 0; s < NQ; ++s) {
        const int uses = (n_issued > s) ? (n_issued - s + NQ - 1) / NQ : 0;
        phase ^= (uint32_t)(uses & 1) << s;
    }
    return ok;
}

// Rows of the two cells of a thread in the two-cell kernels: warp w updates tile rows
// PAIR_R0 * w and PAIR_R0 * w + PAIR_DR. Adjacent rows share operands: the centre of one cell
// is a j-neighbour of the other, and their j +- 1 and j +- 2 rows overlap, so the compiler loads
// those shared values once.
constexpr int PAIR_R0 = 2, PAIR_DR = 1;

// Shared-memory accessor of two cells of one plane: local (jl, kl) and (jl + PAIR_DR, kl).
struct SmemQ2 {
    const float* pl[5];
    int off;
    __device__ __forceinline__ F2 operator()(int c, int di, int dj, int dk) const {
        const float* s = pl[di + 2] + off + dj * RW + dk;
        if (c < 5) return mk2(s[c * CSTR], s[c * CSTR + PAIR_DR * RW]);
        return mk2(-(s[0] + s[3 * CSTR]), -(s[PAIR_DR * RW] + s[3 * CSTR + PAIR_DR * RW]));
    }
};
constexpr int PAIR_THREADS = TK * TJ / 2;  // 128: each thread updates two rows of the tile
constexpr int PAIR_NWARP = PAIR_THREADS / 32;

// process_tile for 128 threads, two cells per thread (rows 2w and 2w + 1 of warp w): the interior
// chemical potential of both cells runs as one packed (FFMA2 / FADD2 / FMUL2) instruction stream;
// face cells, the strong-anchoring rewrite and the update run per cell.
template <bool kL2, bool kL3, bool kNoise, bool kRHS, bool kComp = false>
__device__ __forceinline__ bool process_tile_pair(const CUtensorMap* tm, float* __restrict__ qout,
                                                  const uint8_t* __restrict__ flags, int j0, int k0, int ib, int ie,
                                                  const QsrConst& P, const TileSmem& S, uint32_t& phase,
                                                  int* __restrict__ err, const float* __restrict__ lo_in = nullptr,
                                                  float* __restrict__ lo_out = nullptr) {
    constexpr int NQ = nq<kL2 || kL3, true>();
    static_assert(NQ > 2 * LOOK && LOOK == 2, "the ring holds planes i - 2 .. i + 2 and at least one in flight");
    float* sq = S.sq;
    uint64_t* bar = S.bar;
    const int base = ib - 2;
    const int tid = threadIdx.x;
    const int kl = tid & 31, w = tid >> 5;
    auto slot = [&](int p) { return (uint32_t)(p - base) % (uint32_t)NQ; };
    auto parity = [&](int p) { return ((phase >> slot(p)) & 1u) ^ (((uint32_t)(p - base) / (uint32_t)NQ) & 1u); };
    auto issue = [&](int p) {
        uint64_t* b = &bar[slot(p)];
        if (p >= 0 && p < P.Nx && p < ie + LOOK) {
            fence_proxy_async();
            mbar_expect_tx(b, PLANE_BYTES);
            tma_load_4d(sq + slot(p) * SLOT, tm, k0 - HK, j0 - HJ, p, 0, b);
        } else {
            mbar_arrive(b);
        }
    };
    if (tid == 0)
        for (int p = base; p < base + NQ; ++p) issue(p);
    bool ok = true;
    // Waits run in increasing plane order, so each slot's expected parity is tracked by toggling
    // its bit of `par` after every wait on it (no division per plane).
    uint32_t par = phase;
    auto wait_slot = [&](uint32_t sl) {
        if (!mbar_wait_bounded(&bar[sl], (par >> sl) & 1u)) {
            atomicExch(err, LDG_ERR_TIMEOUT);
            *(volatile int*)S.s_abort = 1;
            ok = false;
        }
        par ^= 1u << sl;
    };
    auto wait_plane = [&](int p) { wait_slot(slot(p)); };
    const int issued_end = ie + NQ - 2;
    constexpr int kLo = kL2 ? 2 : 1;
    const int k = k0 + kl;
    int jr[2];
    bool in_grid[2], jk_int[2];
    long long cell0[2];
    uint8_t f_next[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        jr[r] = j0 + PAIR_R0 * w + PAIR_DR * r;
        in_grid[r] = (jr[r] < P.Ny) && (k >= 0) && (k < P.Nz);
        jk_int[r] = jr[r] >= kLo && jr[r] <= P.Ny - 1 - kLo && k >= kLo && k <= P.Nz - 1 - kLo;
        cell0[r] = (long long)jr[r] * P.sj + k;
        f_next[r] = in_grid[r] ? __ldg(flags + (long long)ib * P.si + cell0[r]) : 0;
    }
    const float* qpl[5];
#pragma unroll
    for (int d = 0; d < 5; ++d) qpl[d] = sq + slot(ib + d - 2) * SLOT;
    int waited_end = base;
    for (int p = base; p <= ib + LOOK - 1; ++p) wait_plane(p);
    waited_end = ib + LOOK;
    uint32_t s_w = slot(ib + LOOK);  // slot of plane i + LOOK, advanced by one per plane
    for (int i = ib; i < ie; ++i) {
        if (*(volatile int*)S.s_abort) { ok = false; break; }
        uint8_t f[2];
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            f[r] = f_next[r];
            if (in_grid[r] && i + 1 < ie) f_next[r] = __ldg(flags + (long long)(i + 1) * P.si + cell0[r]);
        }
        wait_slot(s_w);
        waited_end = i + LOOK + 1;
        if (!ok) break;
        bool fixed[2], move[2];
        bool interior = true;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            fixed[r] = in_grid[r] && !kRHS && (f[r] & kFixed);
            move[r] = in_grid[r] && (f[r] & kMove) != 0;
            interior = interior && (!move[r] || (jk_int[r] && i >= kLo && i <= P.Nx - 1 - kLo));
        }
        const bool warp_interior = __all_sync(0xffffffffu, interior) != 0;
        const bool any_move = __any_sync(0xffffffffu, move[0] || move[1]) != 0;
        float mu[2][5], lap[2][5], c[2][5];
        if (any_move) {
            SmemQ A[2];
#pragma unroll
            for (int r = 0; r < 2; ++r) {
#pragma unroll
                for (int d = 0; d < 5; ++d) A[r].pl[d] = qpl[d];
                A[r].off = (PAIR_R0 * w + PAIR_DR * r + HJ) * RW + (kl + HK);
#pragma unroll
                for (int m = 0; m < 5; ++m) c[r][m] = A[r](m, 0, 0, 0);
            }
            if (warp_interior) {
                SmemQ2 A2;
#pragma unroll
                for (int d = 0; d < 5; ++d) A2.pl[d] = qpl[d];
                A2.off = A[0].off;
                F2 q2[5], mu2[5], lap2[5];
#pragma unroll
                for (int m = 0; m < 5; ++m) q2[m] = mk2(c[0][m], c[1][m]);
                chem_interior_pair<kL2, kL3>(A2, P, q2, mu2, lap2);
#pragma unroll
                for (int m = 0; m < 5; ++m) {
                    mu[0][m] = mu2[m].v.x; mu[1][m] = mu2[m].v.y;
                    lap[0][m] = lap2[m].v.x; lap[1][m] = lap2[m].v.y;
                }
                const bool anch0 = move[0] && (f[0] & kAnchor), anch1 = move[1] && (f[1] & kAnchor);
                if (__any_sync(0xffffffffu, anch0 || anch1)) {
#pragma unroll
                    for (int r = 0; r < 2; ++r) {
                        if (r == 0 ? anch0 : anch1) {
                            float Q0[5];
                            surface_q0(P, i, jr[r], k, Q0);
#pragma unroll
                            for (int m = 0; m < 5; ++m) mu[r][m] += P.Weff * (c[r][m] - Q0[m]);
                        }
                    }
                }
            } else {
#pragma unroll
                for (int r = 0; r < 2; ++r)
                    if (move[r]) {
                        const FlyD<SmemQ> DA{&A[r], &P, i, jr[r], k};
                        chem_potential<kL2, kL3, true>(A[r], DA, P, i, jr[r], k, c[r], (f[r] & kAnchor) != 0, mu[r],
                                                       lap[r]);
                    }
            }
        }
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            if (!(fixed[r] || move[r])) continue;
            const long long id = (long long)i * P.si + cell0[r];
            float o[5];
            if (fixed[r]) {
                surface_q0(P, i, jr[r], k, o);
                if (kComp) {
#pragma unroll
                    for (int m = 0; m < 5; ++m) lo_out[m * P.sc + id] = 0.0f;
                }
            } else {
                const uint32_t cell = (uint32_t)(k + P.Nz * (jr[r] + P.Ny * i));
                if (kRHS) {
#pragma unroll
                    for (int m = 0; m < 5; ++m) o[m] = c[r][m] - P.mob_dt * mu[r][m] - P.alpha * lap[r][m];
                    if (kNoise) {
                        float g[5];
                        normals5(cell, P.instance, P.step, P.key0, P.key1, g);
#pragma unroll
                        for (int m = 0; m < 5; ++m) o[m] += P.sigma * g[m];
                    }
                } else if (kComp) {
                    float lo[5];
#pragma unroll
                    for (int m = 0; m < 5; ++m) lo[m] = __ldg(lo_in + m * P.sc + id);
                    euler_update_comp(P, c[r], lo, mu[r], cell, kNoise, o);
#pragma unroll
                    for (int m = 0; m < 5; ++m) lo_out[m * P.sc + id] = lo[m];
                } else {
                    euler_update(P, c[r], mu[r], cell, kNoise, o);
                }
            }
#pragma unroll
            for (int m = 0; m < 5; ++m) qout[m * P.sc + id] = o[m];
        }
        __syncwarp();
        if (kl == 0) {
            // slot of plane i - 2 = slot of plane i + 2 minus four
            const uint32_t sl = s_w + (NQ - 4) >= (uint32_t)NQ ? s_w - 4 : s_w + (NQ - 4);
            if (arrive_freed(&S.freed[sl]) % (unsigned)PAIR_NWARP == (unsigned)PAIR_NWARP - 1u) issue(i - 2 + NQ);
        }
        s_w = (s_w + 1 == (uint32_t)NQ) ? 0u : s_w + 1;  // now the slot of plane i + 3
#pragma unroll
        for (int d = 0; d < 4; ++d) qpl[d] = qpl[d + 1];
        qpl[4] = sq + s_w * SLOT;
    }
    if (ok) {
        for (int p = waited_end; p < issued_end; ++p) wait_plane(p);
    } else {
        for (int p = waited_end; p < issued_end; ++p)
            if (!mbar_wait_bounded(&bar[slot(p)], parity(p))) break;
    }
    const int n_issued = issued_end - base;
#pragma unroll
    for (int sl = 0; sl < NQ; ++sl) {
        const int uses = (n_issued > sl) ? (n_issued - sl + NQ - 1) / NQ : 0;
        phase ^= (uint32_t)(uses & 1) << sl;
    }
    return ok;
}

template <bool kD, bool kPair = false>
__device__ __forceinline__ void tile_smem_init(const TileSmem& S) {
    if (threadIdx.x == 0) {
        for (int s = 0; s < nq<kD, kPair>(); ++s) {
            mbar_init(&S.bar[s], 1);
            S.freed[s] = 0;
        }
        mbar_fence_init();
        *S.s_abort = 0;
    }
    __syncthreads();
}

// Single grid, two cells per thread (128 threads): four CTAs per SM.
template <bool kL2, bool kL3, bool kNoise, bool kRHS, bool kComp = false>
__global__ void __launch_bounds__(PAIR_THREADS, 4)
    k_step_tiled_pair(const __grid_constant__ CUtensorMap tm_in, float* __restrict__ qout,
                      const uint8_t* __restrict__ flags, const int4* __restrict__ items, QsrConst P,
                      int* __restrict__ err, const float* __restrict__ lo_in, float* __restrict__ lo_out) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const TileSmem S = tile_smem<kL2 || kL3, true>(smem_raw);
    tile_smem_init<kL2 || kL3, true>(S);
    const int4 item = items[blockIdx.x];
    uint32_t phase = 0;
    process_tile_pair<kL2, kL3, kNoise, kRHS, kComp>(&tm_in, qout, flags, item.x, item.y, item.z, item.w, P, S, phase,
                                                     err, lo_in, lo_out);
}

// Single grid: one work item per CTA; two CTAs per SM with the L2/L3 terms, three without.
template <bool kL2, bool kL3, bool kNoise, bool kRHS, bool kComp = false>
__global__ void __launch_bounds__(THREADS, (kL2 || kL3) ? 2 : 3)
    k_step_tiled(const __grid_constant__ CUtensorMap tm_in, float* __restrict__ qout, const uint8_t* __restrict__ flags,
                 const int4* __restrict__ items, QsrConst P, int* __restrict__ err, const float* __restrict__ lo_in,
                 float* __restrict__ lo_out) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const TileSmem S = tile_smem<kL2 || kL3>(smem_raw);
    tile_smem_init<kL2 || kL3>(S);
    const int4 item = items[blockIdx.x];
    uint32_t phase = 0;
    process_tile<kL2, kL3, kNoise, kRHS, kComp>(&tm_in, qout, flags, item.x, item.y, item.z, item.w, P, S, phase, err,
                                                lo_in, lo_out);
}

// ---------------------------------------------------------------------------------------
// Ensemble: many independent droplets, one persistent work-stealing launch per step.
// ---------------------------------------------------------------------------------------
struct EnsItem {
    int j0, k0, ib, ie, inst, pad0, pad1, pad2;
};

// Per-instance descriptor. The step index lives on the device (EnsCtl), so the temperature of
// the protocol, the shell order and the noise counter are formed in the kernel and one captured
// CUDA graph can be replayed for any number of steps.
struct EnsInstDev {
    QsrConst P;            // static parts (noise key and stream included); cQ, S_shell, step set per step
    float* q[2];           // ping-pong buffers: input of step s is q[s & 1]
    const uint8_t* flags;
    double T_high, T_low;  // protocol (QSR.cu:2679-2687)
    long long pre, ramp;
    int protocol;          // 1 step, 2 linear ramp
    int custom_shell;      // 1: S_shell = S_custom, 0: equilibrium S_eq(T)
    double S_custom;
    double a3, T_star, B, C;  // A = a3 (T - T_star); B, C of the bulk convention
};

struct EnsCtl {
    int next;            // work-stealing counter (reset by the last CTA of a step)
    unsigned int done;   // CTAs finished in this step
    long long step;      // global step index
};

__host__ __device__ __forceinline__ double ens_temperature(const EnsInstDev& D, long long it) {
    if (it < D.pre) return D.T_high;
    if (D.protocol == 1) return D.T_low;
    const long long t = it - D.pre;
    if (t <= 0) return D.T_high;
    if (t >= D.ramp) return D.T_low;
    return D.T_high + (D.T_low - D.T_high) * ((double)t / (double)D.ramp);
}

// Lower-energy positive root of 2 C S^2 - B S + 3 A = 0 (QSR.cu:1391-1418), FP64.
__host__ __device__ __forceinline__ double ens_S_eq(double A, double B, double C) {
    if (!(C > 0.0)) return 0.0;
    const double disc = B * B - 24.0 * A * C;
    if (!(disc > 0.0)) return 0.0;
    const double sd = sqrt(disc);
    double best_S = 0.0, best_f = 0.0;
    const double roots[2] = {(B - sd) / (4.0 * C), (B + sd) / (4.0 * C)};
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const double S = roots[r];
        if (!(S > 0.0)) continue;
        const double S2 = S * S;
        const double f = (A / 3.0) * S2 - (2.0 * B / 27.0) * (S2 * S) + (C / 9.0) * (S2 * S2);
        if (f < best_f) { best_f = f; best_S = S; }
    }
    return best_S;
}

// kPair: the two-cell routine (128 threads, four CTAs per SM), else one cell per thread.
template <bool kL2, bool kL3, bool kNoise, bool kPair>
__global__ void __launch_bounds__(kPair ? PAIR_THREADS : THREADS, kPair ? 4 : ((kL2 || kL3) ? 2 : 3))
    k_step_ensemble(const CUtensorMap* __restrict__ tms, const EnsInstDev* __restrict__ inst,
                    const EnsItem* __restrict__ items, int n_items, EnsCtl* __restrict__ ctl, int* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const TileSmem S = tile_smem<kL2 || kL3, kPair>(smem_raw);
    tile_smem_init<kL2 || kL3, kPair>(S);
    // Every CTA reads the step index before any CTA of this launch finishes (the last CTA to
    // finish advances it).
    const long long step = *((volatile long long*)&ctl->step);
    const int which = (int)(step & 1);
    uint32_t phase = 0;
    while (true) {
        if (threadIdx.x == 0) *S.s_item = atomicAdd(&ctl->next, 1);
        __syncthreads();
        const int it = *S.s_item;
        // Uniform across the CTA: the item and the abort flag are read between two barriers.
        const bool stop = (it >= n_items) || (*S.s_abort != 0);
        __syncthreads();
        if (stop) break;
        const EnsItem e = items[it];
        const EnsInstDev& D = inst[e.inst];
        QsrConst P = D.P;
        const double T = ens_temperature(D, step);
        const double A = D.a3 * (T - D.T_star);
        P.cQ = (float)A;
        if (!D.custom_shell) {
            const double s = ens_S_eq(A, D.B, D.C);
            P.S_shell = (float)(s > 0.0 ? s : 0.0);
        } else {
            P.S_shell = (float)D.S_custom;
        }
        P.step = step;
        if constexpr (kPair)
            process_tile_pair<kL2, kL3, kNoise, false>(tms + 2 * e.inst + which, D.q[1 - which], D.flags, e.j0, e.k0,
                                                       e.ib, e.ie, P, S, phase, err);
        else
            process_tile<kL2, kL3, kNoise, false>(tms + 2 * e.inst + which, D.q[1 - which], D.flags, e.j0, e.k0, e.ib,
                                                  e.ie, P, S, phase, err);
    }
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned int d = atomicAdd(&ctl->done, 1u);
        if (d == gridDim.x - 1) {
            ctl->next = 0;
            ctl->done = 0;
            ctl->step = step + 1;
            __threadfence();
        }
    }
}

}  // namespace tiled

// One band of TJ rows of the (j, k) plane: for every plane of [ib, ie) the k range [kmin, kmax]
// of its changing cells (kmin > kmax: none).
struct TiledBand {
    int j0 = 0, rows = 0, ib = 0, ie = 0;
    std::vector<int> kmin, kmax;
};

struct TiledPlan {
    bool ok = false;
    long long active_cells = 0;   // cells inside visited tiles at the current chunk (read once per step)
    long long written_cells = 0;  // cells written per step (moving + strongly anchored)
    int n_items = 0;
    int chunk = 0;                // planes per work item (the longest item)
    int4* items = nullptr;        // device work list (j0, k0, i_begin, i_end)
    int n_plane_items = 0;
    int4* plane_items = nullptr;  // the same tiles one plane each (j0, k0, i, i + 1): IMEX sweeps
    int Nz = 0;
    std::vector<TiledBand> bands; // host: the changing cells' extent per row band and plane
    int* err = nullptr;           // device error word
    CUtensorMap tmap[2];
    const float* bufs[2] = {nullptr, nullptr};
    size_t smem_bytes[3] = {0, 0, 0};  // [L1 only, with L2/L3, with L2/L3 two cells per thread]
};

// Work items for chunks of `chunk` planes. In each row band and plane chunk the k tiles start at
// the first changing cell (rounded down to the 4-float TMA alignment) instead of at multiples of
// TK, and each tile's plane range is cut to the planes whose changing cells reach it: every
// changing cell lies in exactly one item, and fewer idle lanes are visited than with a fixed tile
// grid. Items are ordered longest first, and among items of one length with the plane chunk
// slowest (CTAs resident together share halo planes in L2). *active: the cells of the grid inside
// the items' tiles (read once per step).
inline std::vector<int4> tiled_items(const TiledPlan& plan, int chunk, long long* active) {
    using namespace tiled;
    std::vector<int4> items;
    long long act = 0;
    for (const TiledBand& b : plan.bands) {
        for (int ib = b.ib; ib < b.ie; ib += chunk) {
            const int ie = std::min(b.ie, ib + chunk);
            int kmin = INT32_MAX, kmax = -1;
            for (int p = ib; p < ie; ++p)
                if (b.kmin[p - b.ib] <= b.kmax[p - b.ib]) {
                    kmin = std::min(kmin, b.kmin[p - b.ib]);
                    kmax = std::max(kmax, b.kmax[p - b.ib]);
                }
            if (kmax < 0) continue;
            for (int k0 = ((kmin - 2) & ~3) + 2; k0 <= kmax; k0 += TK) {
                int first = -1, last = -1;
                for (int p = ib; p < ie; ++p) {
                    const int lo = b.kmin[p - b.ib], hi = b.kmax[p - b.ib];
                    if (lo <= hi && lo <= k0 + TK - 1 && hi >= k0) {
                        if (first < 0) first = p;
                        last = p;
                    }
                }
                if (first < 0) continue;
                items.push_back(make_int4(b.j0, k0, first, last + 1));
                act += (long long)b.rows * (std::min(plan.Nz, k0 + TK) - std::max(0, k0)) * (last + 1 - first);
            }
        }
    }
    std::stable_sort(items.begin(), items.end(), [](const int4& a, const int4& b) {
        if (a.z != b.z) return a.z < b.z;
        if (a.x != b.x) return a.x < b.x;
        return a.y < b.y;
    });
    // Longest items first (ties keep the order above): CTAs are dispatched in item order, so
    // the short items of the droplet's poles fill the last wave instead of trailing it.
    std::stable_sort(items.begin(), items.end(),
                     [](const int4& a, const int4& b) { return (a.w - a.z) > (b.w - b.z); });
    if (active) *active = act;
    return items;
}

// Kernel choice: LDG_QSR_PAIR=0 always takes one cell per thread, LDG_QSR_PAIR=1 always two;
// otherwise (the default) the ensemble takes two and a single grid chooses by its work list.
inline int tiled_pair_mode() {
    static const int mode = [] {
        const char* e = getenv("LDG_QSR_PAIR");
        return (e && e[0] == '0') ? 0 : ((e && e[0] == '1') ? 1 : 2);
    }();
    return mode;
}
inline bool tiled_pair_enabled() { return tiled_pair_mode() != 0; }

// A single grid takes the two-cell kernel when its work list fills the GPU at least twice over
// (two waves of four 128-thread CTAs per SM); a smaller list finishes sooner with one cell per
// thread, whose 256-thread CTAs bring twice the warps to each item (64^3, R = 28: 0.0102 against
// 0.0123 ms per step).
inline bool tiled_use_pair(const TiledPlan& plan) {
    if (tiled_pair_mode() != 2) return tiled_pair_mode() == 1;
    static const int sms = [] {
        int dev = 0, n = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) !=
                                                      cudaSuccess)
            return 148;
        return n;
    }();
    return plan.n_items >= 2 * 4 * sms;
}

inline int tiled_default_chunk() {
    int chunk = tiled::CHUNK;
    if (const char* e = getenv("LDG_QSR_CHUNK")) chunk = std::min(4096, std::max(8, atoi(e)));
    return chunk;
}

inline int tiled_encode(CUtensorMap* tm, const float* base, int Nx, int Ny, int Nz, int sj, long long si, long long sc) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn) {
            set_error("cuTensorMapEncodeTiled entry point unavailable");
            return LDG_ERR_CUDA;
        }
        encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    cuuint64_t dims[4] = {(cuuint64_t)Nz, (cuuint64_t)Ny, (cuuint64_t)Nx, 5};
    cuuint64_t strides[3] = {(cuuint64_t)sj * 4, (cuuint64_t)si * 4, (cuuint64_t)sc * 4};
    cuuint32_t box[4] = {tiled::RW, tiled::ROWS, 1, 5};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = encode(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void*)base, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
        return LDG_ERR_CUDA;
    }
    return LDG_OK;
}

// Uploads the work list for chunks of `chunk` planes.
inline int tiled_plan_rechunk(TiledPlan& plan, int chunk) {
    long long active = 0;
    const std::vector<int4> items = tiled_items(plan, chunk, &active);
    plan.active_cells = active;
    if (plan.items) cudaFree(plan.items);
    plan.items = nullptr;
    plan.n_items = (int)items.size();
    plan.chunk = chunk;
    if (plan.n_items > 0) {
        LDG_CUDA(cudaMalloc(&plan.items, items.size() * sizeof(int4)));
        LDG_CUDA(cudaMemcpy(plan.items, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice));
    }
    std::vector<int4> planes;
    for (const int4& t : items)
        for (int i = t.z; i < t.w; ++i) planes.push_back(make_int4(t.x, t.y, i, i + 1));
    if (plan.plane_items) cudaFree(plan.plane_items);
    plan.plane_items = nullptr;
    plan.n_plane_items = (int)planes.size();
    if (plan.n_plane_items > 0) {
        LDG_CUDA(cudaMalloc(&plan.plane_items, planes.size() * sizeof(int4)));
        LDG_CUDA(cudaMemcpy(plan.plane_items, planes.data(), planes.size() * sizeof(int4), cudaMemcpyHostToDevice));
    }
    return LDG_OK;
}

// Builds the work list from the host classification and encodes the two tensor maps.
inline int tiled_plan_build(TiledPlan& plan, int Nx, int Ny, int Nz, int sj, long long si, const uint8_t* fl,
                            const float* buf0, const float* buf1, long long sc) {
    using namespace tiled;
    plan = TiledPlan{};
    plan.Nz = Nz;
    const int ntj = (Ny + TJ - 1) / TJ;
    long long written = 0;
    for (int jt = 0; jt < ntj; ++jt) {
        TiledBand b;
        b.j0 = jt * TJ;
        b.rows = std::min(Ny, (jt + 1) * TJ) - b.j0;
        std::vector<int> kmin(Nx, INT32_MAX), kmax(Nx, -1);
        int imin = Nx, imax = -1;
        for (int i = 0; i < Nx; ++i)
            for (int j = b.j0; j < b.j0 + b.rows; ++j)
                for (int k = 0; k < Nz; ++k)
                    if (fl[(size_t)i * si + (size_t)j * sj + k] & (kMove | kFixed)) {
                        kmin[i] = std::min(kmin[i], k);
                        kmax[i] = std::max(kmax[i], k);
                        imin = std::min(imin, i);
                        imax = std::max(imax, i);
                        ++written;
                    }
        if (imax < 0) continue;
        b.ib = imin;
        b.ie = imax + 1;
        b.kmin.assign(kmin.begin() + imin, kmin.begin() + imax + 1);
        b.kmax.assign(kmax.begin() + imin, kmax.begin() + imax + 1);
        plan.bands.push_back(std::move(b));
    }
    plan.written_cells = written;
    int rc = tiled_plan_rechunk(plan, tiled_default_chunk());
    if (rc) return rc;
    LDG_CUDA(cudaMalloc(&plan.err, sizeof(int)));
    LDG_CUDA(cudaMemset(plan.err, 0, sizeof(int)));
    rc = tiled_encode(&plan.tmap[0], buf0, Nx, Ny, Nz, sj, si, sc);
    if (rc) return rc;
    rc = tiled_encode(&plan.tmap[1], buf1, Nx, Ny, Nz, sj, si, sc);
    if (rc) return rc;
    plan.bufs[0] = buf0;
    plan.bufs[1] = buf1;
    plan.smem_bytes[0] = tile_smem_bytes<false>();
    plan.smem_bytes[1] = tile_smem_bytes<true>();
    plan.smem_bytes[2] = tile_smem_bytes<true, true>();
    plan.ok = true;
    return LDG_OK;
}

template <bool L2, bool L3, bool N, bool R, bool K>
inline int tiled_launch_t(const TiledPlan& plan, int which, float* out, const uint8_t* flags, const QsrConst& P,
                          cudaStream_t st, const float* lo_in, float* lo_out) {
    using namespace tiled;
    const size_t smem = plan.smem_bytes[(L2 || L3) ? 1 : 0];
    static bool configured = false;
    if (!configured) {
        LDG_CUDA(cudaFuncSetAttribute(k_step_tiled<L2, L3, N, R, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
        configured = true;
    }
    if (plan.n_items == 0) return LDG_OK;
    if (tiled_use_pair(plan)) {
        const size_t smem2 = plan.smem_bytes[2];
        static bool configured_pair = false;
        if (!configured_pair) {
            LDG_CUDA(cudaFuncSetAttribute(k_step_tiled_pair<L2, L3, N, R, K>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2));
            configured_pair = true;
        }
        k_step_tiled_pair<L2, L3, N, R, K><<<plan.n_items, PAIR_THREADS, smem2, st>>>(plan.tmap[which], out, flags,
                                                                                     plan.items, P, plan.err, lo_in,
                                                                                     lo_out);
        return LDG_OK;
    }
    k_step_tiled<L2, L3, N, R, K><<<plan.n_items, THREADS, smem, st>>>(plan.tmap[which], out, flags, plan.items, P,
                                                                       plan.err, lo_in, lo_out);
    return LDG_OK;
}

template <bool R, bool K>
inline int tiled_dispatch(const TiledPlan& plan, int which, float* out, const uint8_t* flags, const QsrConst& P,
                          bool L2, bool L3, bool noise, cudaStream_t st, const float* lo_in, float* lo_out) {
    const int key = (L2 ? 1 : 0) | (L3 ? 2 : 0) | (noise ? 4 : 0);
    switch (key) {
        case 0: return tiled_launch_t<false, false, false, R, K>(plan, which, out, flags, P, st, lo_in, lo_out);
        case 1: return tiled_launch_t<true, false, false, R, K>(plan, which, out, flags, P, st, lo_in, lo_out);
        case 2: return tiled_launch_t<false, true, false, R, K>(plan, which, out, flags, P, st, lo_in, lo_out);
        case 3: return tiled_launch_t<true, true, false, R, K>(plan, which, out, flags, P, st, lo_in, lo_out);
        case 4: return tiled_launch_t<false, false, true, R, K>(plan, which, out, flags, P, st, lo_in, lo_out);
        case 5: return tiled_launch_t<true, false, true, R, K>(plan, which, out, flags, P, st, lo_in, lo_out);
        case 6: return tiled_launch_t<false, true, true, R, K>(plan, which, out, flags, P, st, lo_in, lo_out);
        default: return tiled_launch_t<true, true, true, R, K>(plan, which, out, flags, P, st, lo_in, lo_out);
    }
}

// One step through the tiled kernel. `in` must be one of the two planned buffers. With lo_out
// set (explicit steps only) the step uses compensated storage: lo_in / lo_out are the low
// words of the input and output buffers.
inline int tiled_step(const TiledPlan& plan, const float* in, float* out, const uint8_t* flags, const QsrConst& P,
                      bool L2, bool L3, bool noise, bool rhs, cudaStream_t st, const float* lo_in = nullptr,
                      float* lo_out = nullptr) {
    const int which = (in == plan.bufs[0]) ? 0 : 1;
    if (rhs) return tiled_dispatch<true, false>(plan, which, out, flags, P, L2, L3, noise, st, nullptr, nullptr);
    if (lo_out) return tiled_dispatch<false, true>(plan, which, out, flags, P, L2, L3, noise, st, lo_in, lo_out);
    return tiled_dispatch<false, false>(plan, which, out, flags, P, L2, L3, noise, st, nullptr, nullptr);
}

// Reads and clears the device error word (LDG_OK when no bounded wait gave up).
inline int tiled_check(const TiledPlan& plan, cudaStream_t st) {
    if (!plan.err) return LDG_OK;
    int e = 0;
    LDG_CUDA(cudaMemcpyAsync(&e, plan.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    LDG_CUDA(cudaStreamSynchronize(st));
    if (e != 0) {
        LDG_CUDA(cudaMemsetAsync(plan.err, 0, sizeof(int), st));
        set_error("tiled step: a bounded shared-memory pipeline wait gave up");
        return LDG_ERR_TIMEOUT;
    }
    return LDG_OK;
}

inline void tiled_plan_free(TiledPlan& plan) {
    if (plan.items) cudaFree(plan.items);
    if (plan.plane_items) cudaFree(plan.plane_items);
    cudaFree(plan.err);
    plan = TiledPlan{};
}

}  // namespace ldg
