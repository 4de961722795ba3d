// BF16 tensor-core (tcgen05) implicit-GEMM 3x3x3 convolutions for the warm-start surrogate.
//
// Activations are NDHWC BF16 (channels innermost), weights [Co][27][Ci] BF16 with the tap
// index t = 9*(dz+1) + 3*(dy+1) + (dx+1). Convolutions are stride 1 with zero padding 1.
//
// Forward (and data gradient, which is the forward of the flipped, transposed weights):
//   GEMM M = 128 output voxels per CTA, N = Co, K = 27 taps x Ci. Each K step is one TMA load
//   of the input box shifted by the tap (the tensor map's zero fill outside the volume is the
//   padding) plus one TMA load of the weights of that tap; both land 128B/64B/32B-swizzled,
//   K-major, exactly as the UMMA descriptors read them. One thread issues tcgen05.mma into a
//   TMEM accumulator of 128 lanes x Co columns; the epilogue reads TMEM with tcgen05.ld and
//   applies bias and leaky ReLU before the BF16 (or FP32) store.
// Weight gradient:
//   GEMM M = 128 rows of (tap, ci), N = Co, K = voxels, both operands MN-major (channels are
//   contiguous per voxel): the A tile stacks 128/Ci taps of the shifted input, the B tile is
//   the output gradient. K is split over CTAs and reduced with FP32 atomics.
//
// Every mbarrier wait is bounded; on timeout the kernel records LDG_ERR_TIMEOUT, waits
// (bounded) for its loads in flight, releases its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "ldg_api_common.h"
#include "sm100_ptx.cuh"

using namespace ldg;
using namespace ldg::sm100;

namespace {

constexpr int BM = 128;     // UMMA M
constexpr int STAGES = 4;
constexpr int KV = 64;      // voxels per weight-gradient K stage

struct BoxDims {
    int bx, by, bz, bn;     // box extent per dimension, each within the tensor's extent
    int tx, ty, tz, tn;     // boxes per dimension (ceil)
    int rows;               // voxels per box = bx * by * bz * bn (<= the GEMM tile's rows)
};

struct FwdArgs {
    int N, D, H, W, Ci, Co;
    BoxDims b;
    int act;       // 0 identity, 1 leaky ReLU (slope 0.01)
    int out_f32;
    int ksteps;    // 27 * cchunks
    int cchunks;   // Ci / CK
    uint32_t tmem_cols;
};

struct WgArgs {
    int N, D, H, W, Ci, Co;
    BoxDims b;             // 64-voxel K boxes
    long long nkb;         // number of K boxes
    int kb_per_cta;
    uint32_t tmem_cols;
};

__device__ __forceinline__ void box_origin(const BoxDims& b, long long t, int& x0, int& y0, int& z0, int& n0) {
    const int xi = (int)(t % b.tx); t /= b.tx;
    const int yi = (int)(t % b.ty); t /= b.ty;
    const int zi = (int)(t % b.tz); t /= b.tz;
    x0 = xi * b.bx; y0 = yi * b.by; z0 = zi * b.bz; n0 = (int)t * b.bn;
}

__device__ __forceinline__ float act_apply(float v, int act) { return (act == 1 && v < 0.0f) ? 0.01f * v : v; }

// ---------------------------------------------------------------------------------------
// Forward / data-gradient kernel
// ---------------------------------------------------------------------------------------
template <int CK>
__global__ void __launch_bounds__(128, 1)
    k_conv3d_fwd(const __grid_constant__ CUtensorMap tmx, const __grid_constant__ CUtensorMap tmw, void* __restrict__ y,
                 const float* __restrict__ bias, FwdArgs a, int* __restrict__ err) {
    constexpr uint32_t ROW = CK * 2;             // bytes per smem row (one voxel or one output channel)
    constexpr uint32_t A_BYTES = BM * ROW;
    constexpr uint32_t SWZ = swizzle_code(ROW);
    constexpr uint32_t SBO = 8 * ROW;            // 8-row core-matrix group stride
    const uint32_t B_BYTES = (uint32_t)a.Co * ROW;
    const uint32_t B_STRIDE = (B_BYTES + 1023u) & ~1023u;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char* sA = base;
    unsigned char* sB = base + STAGES * A_BYTES;
    uint64_t* full = (uint64_t*)(sB + STAGES * B_STRIDE);
    uint64_t* empty = full + STAGES;
    uint64_t* done = empty + STAGES;
    uint32_t* tslot = (uint32_t*)(done + 1);

    const int tid = threadIdx.x, warp = tid >> 5;
    int x0, y0, z0, n0;
    box_origin(a.b, blockIdx.x, x0, y0, z0, n0);

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        fence_mbar_init();
    }
    if (warp == 0) {
        __syncwarp();
        tmem_alloc(tslot, a.tmem_cols);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (tid == 0) {
        // TMA producer
        int issued = 0;
        for (int ks = 0; ks < a.ksteps; ++ks) {
            const int s = ks % STAGES;
            if (ks >= STAGES && !mbar_wait(&empty[s], ((ks / STAGES) - 1) & 1)) {
                atomicExch(err, LDG_ERR_TIMEOUT);
                break;
            }
            const int tap = ks / a.cchunks, cc = ks - tap * a.cchunks;
            const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
            mbar_expect_tx(&full[s], (uint32_t)a.b.rows * ROW + B_BYTES);
            tma_load_5d(sA + s * A_BYTES, &tmx, cc * CK, x0 + dx, y0 + dy, z0 + dz, n0, &full[s]);
            tma_load_3d(sB + s * B_STRIDE, &tmw, cc * CK, tap, 0, &full[s]);
            issued = ks + 1;
        }
        for (int ks = (issued > STAGES ? issued - STAGES : 0); ks < issued; ++ks)
            if (!mbar_wait(&full[ks % STAGES], (ks / STAGES) & 1)) atomicExch(err, LDG_ERR_TIMEOUT);
    } else if (tid == 32) {
        // MMA issuer
        const uint32_t idesc = idesc_bf16(BM, a.Co, false, false);
        for (int ks = 0; ks < a.ksteps; ++ks) {
            const int s = ks % STAGES;
            if (!mbar_wait(&full[s], (ks / STAGES) & 1)) {
                atomicExch(err, LDG_ERR_TIMEOUT);
                break;
            }
            tc_fence_after();
            const uint32_t a0 = smem_u32(sA + s * A_BYTES), b0 = smem_u32(sB + s * B_STRIDE);
#pragma unroll
            for (int k = 0; k < CK / 16; ++k)
                umma_bf16(tmem, smem_desc(a0 + k * 32, 16, SBO, SWZ), smem_desc(b0 + k * 32, 16, SBO, SWZ), idesc,
                          (ks | k) != 0 ? 1u : 0u);
            umma_commit(&empty[s]);
        }
        umma_commit(done);
    }
    // Epilogue: row m of the accumulator is output voxel m of the box; warp w owns lanes 32w..32w+31.
    bool ok = mbar_wait(done, 0);
    ok = __syncthreads_and(ok) != 0;
    tc_fence_after();
    if (!ok && tid == 0) atomicExch(err, LDG_ERR_TIMEOUT);
    const int m = tid;
    const int xi = m % a.b.bx, yi = (m / a.b.bx) % a.b.by, zi = (m / (a.b.bx * a.b.by)) % a.b.bz;
    const int ni = m / (a.b.bx * a.b.by * a.b.bz);
    const int x = x0 + xi, yy = y0 + yi, z = z0 + zi, n = n0 + ni;
    const bool inside = ok && m < a.b.rows && x < a.W && yy < a.H && z < a.D && n < a.N;
    const long long vox = (((long long)n * a.D + z) * a.H + yy) * a.W + x;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < a.Co; c0 += 16) {
        float v[16];
        tmem_ld16(trow + (uint32_t)c0, v);
        if (!inside) continue;
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = act_apply(v[i] + (bias ? bias[c0 + i] : 0.0f), a.act);
        if (a.out_f32) {
            float4* dst = reinterpret_cast<float4*>(static_cast<float*>(y) + vox * a.Co + c0);
#pragma unroll
            for (int q = 0; q < 4; ++q) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        } else {
            uint32_t p[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
                p[q] = *reinterpret_cast<uint32_t*>(&h);
            }
            uint4* dst = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(y) + vox * a.Co + c0);
            dst[0] = make_uint4(p[0], p[1], p[2], p[3]);
            dst[1] = make_uint4(p[4], p[5], p[6], p[7]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, a.tmem_cols);
    }
}

// ---------------------------------------------------------------------------------------
// Weight-gradient kernel
// ---------------------------------------------------------------------------------------
template <int ACA, int ACB>
__global__ void __launch_bounds__(128, 1)
    k_conv3d_wgrad(const __grid_constant__ CUtensorMap tmx, const __grid_constant__ CUtensorMap tmdy,
                   float* __restrict__ dw, WgArgs a, int* __restrict__ err) {
    constexpr uint32_t ROWA = ACA * 2, ROWB = ACB * 2;
    constexpr uint32_t ATOM_A = KV * ROWA;            // ACA channels x 64 voxels
    constexpr uint32_t ATOM_B = KV * ROWB;
    constexpr int NATOM_A = BM / ACA;
    constexpr uint32_t A_BYTES = NATOM_A * ATOM_A;    // 16 KB
    constexpr uint32_t SWZA = swizzle_code(ROWA), SWZB = swizzle_code(ROWB);
    constexpr uint32_t SBOA = 8 * ROWA, SBOB = 8 * ROWB;
    const int natom_b = a.Co / ACB;
    const uint32_t B_BYTES = (uint32_t)natom_b * ATOM_B;
    const uint32_t B_STRIDE = (B_BYTES + 1023u) & ~1023u;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char* sA = base;
    unsigned char* sB = base + STAGES * A_BYTES;
    uint64_t* full = (uint64_t*)(sB + STAGES * B_STRIDE);
    uint64_t* empty = full + STAGES;
    uint64_t* done = empty + STAGES;
    uint32_t* tslot = (uint32_t*)(done + 1);

    const int tid = threadIdx.x, warp = tid >> 5;
    // Row block of this CTA: 128 rows of (tap, ci).
    const bool wide = a.Ci > BM;                       // Ci = 256: two tiles per tap
    const int tap_base = wide ? (int)(blockIdx.x >> 1) : (int)blockIdx.x * (BM / a.Ci);
    const int ci_base = wide ? (int)(blockIdx.x & 1) * BM : 0;
    const long long kb0 = (long long)blockIdx.y * a.kb_per_cta;
    const long long kb1 = (kb0 + a.kb_per_cta < a.nkb) ? kb0 + a.kb_per_cta : a.nkb;
    const int nsteps = (int)(kb1 > kb0 ? kb1 - kb0 : 0);

    // A atoms of this tile that hold a real tap (rows of taps >= 27 are left unloaded and
    // their accumulator rows are discarded).
    int natom_a_valid = 0;
    for (int j = 0; j < NATOM_A; ++j) {
        const int row0 = j * ACA;
        const int tap = wide ? tap_base : tap_base + row0 / a.Ci;
        if (tap < 27) ++natom_a_valid;
    }

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        fence_mbar_init();
    }
    // K rows past the box (volumes smaller than 64 voxels) are never written by the loads and
    // take part in the reduction: zero them once in every stage (a row's 16-byte chunks stay
    // inside the row under the swizzle).
    if (a.b.rows < KV) {
        const uint32_t za = (uint32_t)(KV - a.b.rows) * ROWA, zb = (uint32_t)(KV - a.b.rows) * ROWB;
        for (int s = 0; s < STAGES; ++s) {
            for (int j = 0; j < NATOM_A; ++j) {
                uint4* p = reinterpret_cast<uint4*>(sA + s * A_BYTES + j * ATOM_A + (uint32_t)a.b.rows * ROWA);
                for (uint32_t q = tid; q < za / 16; q += blockDim.x) p[q] = make_uint4(0, 0, 0, 0);
            }
            for (int j = 0; j < natom_b; ++j) {
                uint4* p = reinterpret_cast<uint4*>(sB + s * B_STRIDE + j * ATOM_B + (uint32_t)a.b.rows * ROWB);
                for (uint32_t q = tid; q < zb / 16; q += blockDim.x) p[q] = make_uint4(0, 0, 0, 0);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        __syncwarp();
        tmem_alloc(tslot, a.tmem_cols);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (tid == 0) {
        int issued = 0;
        for (int st = 0; st < nsteps; ++st) {
            const int s = st % STAGES;
            if (st >= STAGES && !mbar_wait(&empty[s], ((st / STAGES) - 1) & 1)) {
                atomicExch(err, LDG_ERR_TIMEOUT);
                break;
            }
            int vx, vy, vz, vn;
            box_origin(a.b, kb0 + st, vx, vy, vz, vn);
            mbar_expect_tx(&full[s], (uint32_t)(natom_a_valid * ACA + a.Co) * (uint32_t)a.b.rows * 2u);
            for (int j = 0; j < NATOM_A; ++j) {
                const int row0 = j * ACA;
                const int tap = wide ? tap_base : tap_base + row0 / a.Ci;
                const int ci = wide ? ci_base + row0 : row0 % a.Ci;
                if (tap >= 27) continue;
                const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
                tma_load_5d(sA + s * A_BYTES + j * ATOM_A, &tmx, ci, vx + dx, vy + dy, vz + dz, vn, &full[s]);
            }
            for (int j = 0; j < natom_b; ++j)
                tma_load_5d(sB + s * B_STRIDE + j * ATOM_B, &tmdy, j * ACB, vx, vy, vz, vn, &full[s]);
            issued = st + 1;
        }
        for (int st = (issued > STAGES ? issued - STAGES : 0); st < issued; ++st)
            if (!mbar_wait(&full[st % STAGES], (st / STAGES) & 1)) atomicExch(err, LDG_ERR_TIMEOUT);
    } else if (tid == 32) {
        const uint32_t idesc = idesc_bf16(BM, a.Co, true, true);
        for (int st = 0; st < nsteps; ++st) {
            const int s = st % STAGES;
            if (!mbar_wait(&full[s], (st / STAGES) & 1)) {
                atomicExch(err, LDG_ERR_TIMEOUT);
                break;
            }
            tc_fence_after();
            const uint32_t a0 = smem_u32(sA + s * A_BYTES), b0 = smem_u32(sB + s * B_STRIDE);
#pragma unroll
            for (int k = 0; k < KV / 16; ++k)
                umma_bf16(tmem, smem_desc(a0 + k * 2 * SBOA, ATOM_A, SBOA, SWZA),
                          smem_desc(b0 + k * 2 * SBOB, ATOM_B, SBOB, SWZB), idesc, (st | k) != 0 ? 1u : 0u);
            umma_commit(&empty[s]);
        }
        umma_commit(done);
    }
    bool ok = mbar_wait(done, 0);
    ok = __syncthreads_and(ok) != 0;
    tc_fence_after();
    if (!ok && tid == 0) atomicExch(err, LDG_ERR_TIMEOUT);
    const int m = tid;
    const int tap = wide ? tap_base : tap_base + m / a.Ci;
    const int ci = wide ? ci_base + m : m % a.Ci;
    const bool valid = ok && nsteps > 0 && tap < 27;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < a.Co; c0 += 16) {
        float v[16];
        tmem_ld16(trow + (uint32_t)c0, v);
        if (!valid) continue;
#pragma unroll
        for (int i = 0; i < 16; ++i) atomicAdd(&dw[((long long)(c0 + i) * 27 + tap) * a.Ci + ci], v[i]);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, a.tmem_cols);
    }
}

// w[co][t][ci] -> wf[ci][26 - t][co]: the data gradient is the forward convolution of the
// output gradient with these weights.
__global__ void k_flip_weights(const __nv_bfloat16* __restrict__ w, __nv_bfloat16* __restrict__ wf, int Ci, int Co) {
    const long long n = (long long)Co * 27 * Ci;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int ci = (int)(i % Ci);
        const int t = (int)((i / Ci) % 27);
        const int co = (int)(i / ((long long)Ci * 27));
        wf[((long long)ci * 27 + (26 - t)) * Co + co] = w[i];
    }
}

// ---------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------
constexpr int kMaxDevices = 64;
int* g_err_dev[kMaxDevices] = {};  // device error word of each GPU (allocated on first use there)
int* g_err = nullptr;              // the current device's word (set by ensure_err)
long long g_launches = 0;
std::mutex g_mu;

int ensure_err() {
    int dev = 0;
    LDG_CUDA(cudaGetDevice(&dev));
    LDG_REQUIRE(dev >= 0 && dev < kMaxDevices, LDG_ERR_ARG, "conv3d: device index out of range");
    if (!g_err_dev[dev]) {
        LDG_CUDA(cudaMalloc(&g_err_dev[dev], sizeof(int)));
        LDG_CUDA(cudaMemset(g_err_dev[dev], 0, sizeof(int)));
    }
    g_err = g_err_dev[dev];
    return LDG_OK;
}

int pow2_floor(int v) {
    int p = 1;
    while (p * 2 <= v) p *= 2;
    return p;
}

BoxDims make_box(int N, int D, int H, int W, int total) {
    BoxDims b{};
    b.bx = std::min(pow2_floor(W), total);
    b.by = std::min(pow2_floor(H), total / b.bx);
    b.bz = std::min(pow2_floor(D), total / (b.bx * b.by));
    b.bn = std::min(N, total / (b.bx * b.by * b.bz));
    b.rows = b.bx * b.by * b.bz * b.bn;
    b.tx = (W + b.bx - 1) / b.bx;
    b.ty = (H + b.by - 1) / b.by;
    b.tz = (D + b.bz - 1) / b.bz;
    b.tn = (N + b.bn - 1) / b.bn;
    return b;
}

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

CUtensorMapSwizzle swizzle_enum(int row_bytes) {
    return row_bytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                            : (row_bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B);
}

// NDHWC BF16 activation map: dims (C, W, H, D, N), box (cbox, bx, by, bz, bn).
int encode_act(CUtensorMap* tm, const void* p, const sg_conv_shape& s, int C, int cbox, const BoxDims& b) {
    auto enc = encoder();
    LDG_REQUIRE(enc, LDG_ERR_CUDA, "cuTensorMapEncodeTiled entry point unavailable");
    cuuint64_t dims[5] = {(cuuint64_t)C, (cuuint64_t)s.W, (cuuint64_t)s.H, (cuuint64_t)s.D, (cuuint64_t)s.N};
    cuuint64_t strides[4] = {(cuuint64_t)C * 2, (cuuint64_t)C * 2 * s.W, (cuuint64_t)C * 2 * s.W * s.H,
                             (cuuint64_t)C * 2 * s.W * s.H * s.D};
    cuuint32_t box[5] = {(cuuint32_t)cbox, (cuuint32_t)b.bx, (cuuint32_t)b.by, (cuuint32_t)b.bz, (cuuint32_t)b.bn};
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    CUresult r = enc(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(p), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_enum(cbox * 2), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("conv3d: activation tensor map encoding failed: " + std::to_string((int)r));
        return LDG_ERR_CUDA;
    }
    return LDG_OK;
}

// Weight map [Co][27][Ci]: dims (Ci, 27, Co), box (ck, 1, Co).
int encode_w(CUtensorMap* tm, const void* p, int Ci, int Co, int ck) {
    auto enc = encoder();
    LDG_REQUIRE(enc, LDG_ERR_CUDA, "cuTensorMapEncodeTiled entry point unavailable");
    cuuint64_t dims[3] = {(cuuint64_t)Ci, 27, (cuuint64_t)Co};
    cuuint64_t strides[2] = {(cuuint64_t)Ci * 2, (cuuint64_t)Ci * 2 * 27};
    cuuint32_t box[3] = {(cuuint32_t)ck, 1, (cuuint32_t)Co};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = enc(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(p), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_enum(ck * 2), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("conv3d: weight tensor map encoding failed: " + std::to_string((int)r));
        return LDG_ERR_CUDA;
    }
    return LDG_OK;
}

bool channels_ok(int c) { return c == 16 || c == 32 || c == 64 || c == 128 || c == 256; }

uint32_t tmem_cols_for(int n) {
    uint32_t c = 32;
    while (c < (uint32_t)n) c *= 2;
    return c;
}

int check_shape(const sg_conv_shape* s, const char* who) {
    LDG_REQUIRE(s, LDG_ERR_ARG, std::string(who) + ": null shape");
    LDG_REQUIRE(s->N >= 1 && s->D >= 1 && s->H >= 1 && s->W >= 1, LDG_ERR_ARG, std::string(who) + ": empty volume");
    LDG_REQUIRE(channels_ok(s->Ci), LDG_ERR_ARG, std::string(who) + ": Ci must be 16, 32, 64, 128 or 256");
    LDG_REQUIRE(s->Co >= 16 && s->Co <= 256 && s->Co % 16 == 0, LDG_ERR_ARG,
                std::string(who) + ": Co must be a multiple of 16 in [16, 256]");
    LDG_REQUIRE((long long)s->N * s->D * s->H * s->W < (1LL << 31), LDG_ERR_ARG, std::string(who) + ": volume too large");
    return LDG_OK;
}

template <int CK>
int launch_fwd(const sg_conv_shape& s, const void* x, const void* w, const float* bias, void* y, int act, int f32,
               cudaStream_t st) {
    FwdArgs a{};
    a.N = s.N; a.D = s.D; a.H = s.H; a.W = s.W; a.Ci = s.Ci; a.Co = s.Co;
    a.b = make_box(s.N, s.D, s.H, s.W, BM);
    a.act = act;
    a.out_f32 = f32;
    a.cchunks = s.Ci / CK;
    a.ksteps = 27 * a.cchunks;
    a.tmem_cols = tmem_cols_for(s.Co);
    CUtensorMap tmx, tmw;
    int rc = encode_act(&tmx, x, s, s.Ci, CK, a.b);
    if (rc) return rc;
    rc = encode_w(&tmw, w, s.Ci, s.Co, CK);
    if (rc) return rc;
    const size_t b_stride = ((size_t)s.Co * CK * 2 + 1023) & ~(size_t)1023;
    const size_t smem = 1024 + STAGES * ((size_t)BM * CK * 2 + b_stride) + (2 * STAGES + 1) * 8 + 16;
    LDG_CUDA(cudaFuncSetAttribute(k_conv3d_fwd<CK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long long tiles = (long long)a.b.tx * a.b.ty * a.b.tz * a.b.tn;
    LDG_REQUIRE(tiles < (1LL << 31), LDG_ERR_ARG, "conv3d: too many tiles");
    k_conv3d_fwd<CK><<<(unsigned)tiles, 128, smem, st>>>(tmx, tmw, y, bias, a, g_err);
    LDG_LAUNCHED("k_conv3d_fwd");
    g_launches++;
    return LDG_OK;
}

template <int ACA, int ACB>
int launch_wgrad(const sg_conv_shape& s, const void* x, const void* dy, float* dw, cudaStream_t st) {
    WgArgs a{};
    a.N = s.N; a.D = s.D; a.H = s.H; a.W = s.W; a.Ci = s.Ci; a.Co = s.Co;
    a.b = make_box(s.N, s.D, s.H, s.W, KV);
    a.nkb = (long long)a.b.tx * a.b.ty * a.b.tz * a.b.tn;
    a.tmem_cols = tmem_cols_for(s.Co);
    const int mtiles = (s.Ci > BM) ? 27 * (s.Ci / BM) : (27 + (BM / s.Ci) - 1) / (BM / s.Ci);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // Split K so the grid covers every SM about twice; at least 8 K boxes per CTA.
    long long splits = std::max(1LL, (2LL * sms + mtiles - 1) / mtiles);
    splits = std::min(splits, std::max(1LL, a.nkb / 8));
    a.kb_per_cta = (int)((a.nkb + splits - 1) / splits);
    splits = (a.nkb + a.kb_per_cta - 1) / a.kb_per_cta;
    CUtensorMap tmx, tmdy;
    BoxDims bk = a.b;
    int rc = encode_act(&tmx, x, s, s.Ci, ACA, bk);
    if (rc) return rc;
    rc = encode_act(&tmdy, dy, s, s.Co, ACB, bk);
    if (rc) return rc;
    const size_t b_stride = ((size_t)s.Co * KV * 2 + 1023) & ~(size_t)1023;
    const size_t smem = 1024 + STAGES * ((size_t)BM * KV * 2 + b_stride) + (2 * STAGES + 1) * 8 + 16;
    LDG_CUDA(cudaFuncSetAttribute(k_conv3d_wgrad<ACA, ACB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    LDG_CUDA(cudaMemsetAsync(dw, 0, (size_t)s.Co * 27 * s.Ci * sizeof(float), st));
    dim3 grid((unsigned)mtiles, (unsigned)splits);
    k_conv3d_wgrad<ACA, ACB><<<grid, 128, smem, st>>>(tmx, tmdy, dw, a, g_err);
    LDG_LAUNCHED("k_conv3d_wgrad");
    g_launches++;
    return LDG_OK;
}

template <int ACA>
int wgrad_dispatch_b(const sg_conv_shape& s, const void* x, const void* dy, float* dw, cudaStream_t st) {
    if (s.Co == 16) return launch_wgrad<ACA, 16>(s, x, dy, dw, st);
    if (s.Co == 32) return launch_wgrad<ACA, 32>(s, x, dy, dw, st);
    LDG_REQUIRE(s.Co % 64 == 0, LDG_ERR_ARG, "conv3d wgrad: Co must be 16, 32 or a multiple of 64");
    return launch_wgrad<ACA, 64>(s, x, dy, dw, st);
}

}  // namespace

extern "C" {

int sg_conv3d_fwd(const sg_conv_shape* s, const void* x, const void* w, const float* bias, void* y, int act,
                  int y_fp32, void* stream) {
    clear_error();
    int rc = check_shape(s, "sg_conv3d_fwd");
    if (rc) return rc;
    LDG_REQUIRE(x && w && y, LDG_ERR_ARG, "sg_conv3d_fwd: null pointer");
    LDG_REQUIRE(act == 0 || act == 1, LDG_ERR_ARG, "sg_conv3d_fwd: act must be 0 or 1");
    std::lock_guard<std::mutex> lk(g_mu);
    if ((rc = ensure_err())) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (s->Ci == 16) return launch_fwd<16>(*s, x, w, bias, y, act, y_fp32, st);
    if (s->Ci == 32) return launch_fwd<32>(*s, x, w, bias, y, act, y_fp32, st);
    return launch_fwd<64>(*s, x, w, bias, y, act, y_fp32, st);
}

int sg_conv3d_wgrad(const sg_conv_shape* s, const void* x, const void* dy, float* dw, void* stream) {
    clear_error();
    int rc = check_shape(s, "sg_conv3d_wgrad");
    if (rc) return rc;
    LDG_REQUIRE(x && dy && dw, LDG_ERR_ARG, "sg_conv3d_wgrad: null pointer");
    std::lock_guard<std::mutex> lk(g_mu);
    if ((rc = ensure_err())) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (s->Ci == 16) return wgrad_dispatch_b<16>(*s, x, dy, dw, st);
    if (s->Ci == 32) return wgrad_dispatch_b<32>(*s, x, dy, dw, st);
    return wgrad_dispatch_b<64>(*s, x, dy, dw, st);
}

int sg_conv3d_flip_weights(const sg_conv_shape* s, const void* w, void* wf, void* stream) {
    clear_error();
    LDG_REQUIRE(s && w && wf, LDG_ERR_ARG, "sg_conv3d_flip_weights: null argument");
    const long long n = (long long)s->Co * 27 * s->Ci;
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 8);
    k_flip_weights<<<std::max(blocks, 1), 256, 0, (cudaStream_t)stream>>>(
        static_cast<const __nv_bfloat16*>(w), static_cast<__nv_bfloat16*>(wf), s->Ci, s->Co);
    LDG_LAUNCHED("k_flip_weights");
    std::lock_guard<std::mutex> lk(g_mu);
    g_launches++;
    return LDG_OK;
}

// Reads and clears the device error word of the conv kernels (synchronises the stream).
int sg_check(void* stream) {
    clear_error();
    std::lock_guard<std::mutex> lk(g_mu);
    int rc = ensure_err();
    if (rc) return rc;
    int e = 0;
    LDG_CUDA(cudaMemcpyAsync(&e, g_err, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    LDG_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    if (e) {
        LDG_CUDA(cudaMemset(g_err, 0, sizeof(int)));
        set_error("conv3d: a bounded pipeline wait gave up");
        return LDG_ERR_TIMEOUT;
    }
    return LDG_OK;
}

long long sg_launch_count(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    return g_launches;
}

}  // extern "C"
