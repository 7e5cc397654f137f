// The warm-start network: a coordinate MLP (inflow parameters and cell
// position -> a converged state of the plain step), trained and evaluated
// on the GPU by this file's kernels.
//
//   gemm_tc_kernel        C[M,N] (fp32) = A[M,K] . B[N,K]^T with bf16 operands
//                         on the 5th-generation tensor cores (tcgen05.mma,
//                         fp32 accumulator in tensor memory), both operands
//                         k-contiguous: X.W^T (forward), dZ.(W^T)^T
//                         (backward, data) and (dZ^T).(H^T)^T (backward,
//                         weights; split over K into partial tiles that
//                         splitk_reduce_kernel adds in a fixed order)
//   gemm_tma_kernel       the same GEMM with the operand tiles brought in by
//                         the tensor memory accelerator (one thread issues
//                         cp.async.bulk.tensor per tile; no cluster
//                         multicast) and, for the forward layers, bias +
//                         GELU applied to the accumulator as it leaves
//                         tensor memory, the hidden layers' Z and H tiles
//                         staged in shared memory and stored by the TMA;
//                         used whenever both operands' rows are 16-byte
//                         aligned
//   transpose_bf16_kernel the transposed operands of the backward GEMMs
//   features_kernel       network inputs: the raw inputs, then sin / cos of
//                         2^f pi s of the last two (the cell position), bf16
//   gather_kernel         a mini-batch of rows of the training set, drawn by
//                         a counter-based hash of (seed, step, row)
//   bias_act_kernel       Z = C + bias, H = GELU(Z) (or Z), H as bf16
//   act_bwd_kernel        dZ = dH * GELU'(Z) (or dH), fp32 and bf16
//   col_sum_*_kernel      bias gradients: column sums in a fixed order
//   mse_kernel            dY = 2 (Y - T) / (M N), squared error per row
//   loss_kernel           mean squared error of the batch (fixed order)
//   adam_kernel           Adam on the fp32 master weights, bf16 copy refreshed
// GELU(x) = x Phi(x) = x/2 (1 + erf(x / sqrt 2)) through CUDA's erff; its
// derivative Phi(x) + x phi(x) through erff and expf.
#include <cuda.h>  // CUtensorMap and its enums (the encoder is looked up at run time)
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/gelios_b200.h"

namespace gelios {
void set_error(const std::string& msg);
}  // namespace gelios

namespace {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// 16-byte asynchronous copy global -> shared; bytes beyond src_bytes are zero
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
// all but the newest TC_STAGES - 1 commit groups have landed
__device__ __forceinline__ void cp_async_wait_ring() { asm volatile("cp.async.wait_group 3;\n" ::); }

// ---- the GEMM on the 5th-generation tensor cores (tcgen05)
// C[M][N] (fp32, rows of ldc) = sum_k A[m][k] B[n][k], A and B bf16 with k
// contiguous (rows of lda / ldb); blockIdx.z: K slice [z kc, (z+1) kc),
// written to C + z c_split.  One 128 x 128 fp32 accumulator tile per CTA
// in tensor memory (128 lanes x 128 columns), K in stages of 64: both
// operand tiles (128 rows x 64 bf16)
// staged by cp.async in the canonical K-major layout without swizzle (core
// matrices of 8 rows x 16 bytes; 16-byte K chunks 128 bytes apart, 8-row
// groups 1024 bytes apart), a ring of four stages (the whole K of a
// 256-wide layer in flight at once).  One thread issues four tcgen05.mma
// (M 128, N 128, K 16) per stage and commits them to the stage's mbarrier,
// which frees the stage for the load of the tile four steps on; the epilogue
// reads the accumulator with tcgen05.ld (warp w: rows 32w..32w+31).  Every
// mbarrier wait is bounded: on expiry the CTA raises `status` and goes on.
constexpr int TC_BM = 128, TC_BN = 128, TC_BK = 64, TC_THREADS = 128;
constexpr int TC_TILE = TC_BM * TC_BK * 2;  // bytes of one operand tile
constexpr int TC_STAGES = 4;
constexpr int TC_SMEM = 2 * TC_STAGES * TC_TILE;  // A and B per stage
constexpr uint32_t TC_LBO = 128, TC_SBO = 1024;
// instruction descriptor of kind::f16: fp32 accumulator (bits 4-5 = 1),
// A and B bf16 (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 = 0),
// N >> 3 in bits 17-22, M >> 4 in bits 24-28
constexpr uint32_t TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_BN >> 3) << 17) |
                              ((uint32_t)(TC_BM >> 4) << 24);

// shared-memory matrix descriptor: start address >> 4 (bits 0-13), leading
// byte offset >> 4 (16-29), stride byte offset >> 4 (32-45), version 1
// (bits 46-47), no swizzle (bits 61-63 = 0)
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((TC_LBO >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((TC_SBO >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
__device__ __forceinline__ uint32_t tc_off(int r, int kc) {
    return static_cast<uint32_t>((r >> 3) * TC_SBO + kc * TC_LBO + (r & 7) * 16);
}
__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait for the phase of the given parity; false if it did not complete
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned parity) {
    for (int i = 0; i < (1 << 22); i++)
        if (mbar_try_wait(b, parity)) return true;
    return false;
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// rows row0.. x k k0..k0+63 of a k-contiguous operand into a canonical tile.
// A warp stages 8 rows x 4 chunks per pass (lane: row lane & 7, chunk
// lane >> 3): each row's 64 bytes are read contiguously, and the 8 rows of
// one chunk fill one 128-byte core matrix (no bank conflict); 4 warps x 8
// passes cover 16 row groups x 2 chunk halves.
template <bool VEC>
__device__ __forceinline__ void tc_load(uint8_t* tile, const __nv_bfloat16* __restrict__ G, int64_t ld, int row0,
                                        int nrows, int k0, int ke) {
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int pass = 0; pass < 8; pass++) {
        const int unit = pass * 4 + warp;  // (row group, chunk half)
        const int r = (unit >> 1) * 8 + (lane & 7), kq = (unit & 1) * 4 + (lane >> 3);
        const int gr = row0 + r;
        const int gk = k0 + kq * 8;
        uint8_t* dst = tile + tc_off(r, kq);
        if (VEC && gr < nrows && gk + 8 <= ke) {
            cp_async16(smem_u32(dst), G + gr * ld + gk, 16);
        } else if (VEC && (gr >= nrows || gk >= ke)) {
            cp_async16(smem_u32(dst), G, 0);
        } else {
            __nv_bfloat16* d = reinterpret_cast<__nv_bfloat16*>(dst);
            for (int e = 0; e < 8; e++) d[e] = (gr < nrows && gk + e < ke) ? G[gr * ld + gk + e] : zero;
        }
    }
}

template <bool AV, bool BV>
__global__ void __launch_bounds__(TC_THREADS) gemm_tc_kernel(int M, int N, int K, int kc,
                                                           const __nv_bfloat16* __restrict__ A, int64_t lda,
                                                           const __nv_bfloat16* __restrict__ B, int64_t ldb,
                                                           float* __restrict__ C, int64_t ldc, int64_t c_split,
                                                           int* __restrict__ status) {
    extern __shared__ __align__(1024) uint8_t tc_smem[];
    __shared__ uint64_t bars[TC_STAGES];
    __shared__ uint32_t tmem_slot;
    uint8_t* sA0 = tc_smem;
    uint8_t* sB0 = tc_smem + TC_STAGES * TC_TILE;
    const int m0 = blockIdx.y * TC_BM, n0 = blockIdx.x * TC_BN;
    const int kb = blockIdx.z * kc, ke = min(K, kb + kc);
    C += blockIdx.z * c_split;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_slot)),
                     "r"(TC_BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < TC_STAGES; i++) mbar_init(&bars[i], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    const int nk = ke > kb ? (ke - kb + TC_BK - 1) / TC_BK : 0;
    bool ok = true;
    // prologue: tiles 0 .. TC_STAGES-2, one commit group each
    for (int j = 0; j < TC_STAGES - 1; j++) {
        if (j < nk) {
            tc_load<AV>(sA0 + j * TC_TILE, A, lda, m0, M, kb + j * TC_BK, ke);
            tc_load<BV>(sB0 + j * TC_TILE, B, ldb, n0, N, kb + j * TC_BK, ke);
        }
        cp_async_commit();
    }
    static_assert(TC_STAGES == 4, "cp_async_wait_ring waits for TC_STAGES - 1 groups");
    for (int it = 0; it < nk; it++) {
        const int s = it % TC_STAGES;
        const int nx = it + TC_STAGES - 1;  // the tile loaded now, into the stage iteration it-1 used
        if (nx < nk) {
            const int sx = nx % TC_STAGES;
            if (it >= 1 && !mbar_wait(&bars[sx], ((it - 1) / TC_STAGES) & 1)) ok = false;
            tc_load<AV>(sA0 + sx * TC_TILE, A, lda, m0, M, kb + nx * TC_BK, ke);
            tc_load<BV>(sB0 + sx * TC_TILE, B, ldb, n0, N, kb + nx * TC_BK, ke);
        }
        cp_async_commit();
        cp_async_wait_ring();
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // staged bytes visible to the tensor cores
        __syncthreads();
        if (threadIdx.x == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(sA0 + s * TC_TILE), b0 = smem_u32(sB0 + s * TC_TILE);
#pragma unroll
            for (int k = 0; k < TC_BK / 16; k++) {
                const uint64_t ad = tc_desc(a0 + k * 2 * TC_LBO), bd = tc_desc(b0 + k * 2 * TC_LBO);
                const uint32_t acc = (it > 0 || k > 0) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(TC_IDESC), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             smem_u32(&bars[s]))
                         : "memory");
        }
    }
    if (nk > 0 && !mbar_wait(&bars[(nk - 1) % TC_STAGES], ((nk - 1) / TC_STAGES) & 1)) ok = false;
    tc_fence_after();
    const int64_t row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < TC_BN; c0 += 16) {
        uint32_t v[16];
        if (nk > 0) {
            const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c0);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];\n"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        } else {
#pragma unroll
            for (int j = 0; j < 16; j++) v[j] = 0u;
        }
        if (row < M) {
            float* dst = C + row * ldc + n0 + c0;
            if (n0 + c0 + 16 <= N && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
#pragma unroll
                for (int j = 0; j < 16; j += 4)
                    *reinterpret_cast<float4*>(dst + j) = make_float4(__uint_as_float(v[j]), __uint_as_float(v[j + 1]),
                                                                      __uint_as_float(v[j + 2]), __uint_as_float(v[j + 3]));
            } else {
#pragma unroll
                for (int j = 0; j < 16; j++)
                    if (n0 + c0 + j < N) dst[j] = __uint_as_float(v[j]);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TC_BN) : "memory");
    }
    if (!ok) atomicOr(status, 1);
}

// out[c][r] = in[r][c] (bf16, rows of ldin -> rows of ldout), 32 x 32 tiles
__global__ void transpose_bf16_kernel(int R, int Cc, const __nv_bfloat16* __restrict__ in, int64_t ldin,
                                      __nv_bfloat16* __restrict__ out, int64_t ldout) {
    __shared__ unsigned short tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int r = r0 + y, c = c0 + threadIdx.x;
        if (r < R && c < Cc) tile[y][threadIdx.x] = __bfloat16_as_ushort(in[r * ldin + c]);
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int c = c0 + y, r = r0 + threadIdx.x;
        if (r < R && c < Cc) out[c * ldout + r] = __ushort_as_bfloat16(tile[threadIdx.x][y]);
    }
}

__global__ void splitk_reduce_kernel(int64_t n, int S, const float* __restrict__ part, float* __restrict__ out) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s = 0.f;
    for (int z = 0; z < S; z++) s += part[z * n + i];
    out[i] = s;
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    const float cdf = 0.5f * (1.f + erff(x * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
    return cdf + x * pdf;
}

// ---- the GEMM with TMA staging
// Per stage and operand one box of 64 k x rows (128 bytes x 128 rows for A,
// x 64 rows for B) loaded with the 128-byte swizzle: row r lands at r * 128
// bytes with its 16-byte chunks permuted by (r mod 8), which is the
// canonical K-major SWIZZLE_128B layout the MMA descriptor names (8-row
// groups 1024 bytes apart; the k-th 16-deep slice of the stage starts 32 k
// bytes into the rows).  Stage buffers are 1024-byte aligned.  Thread 0
// issues the loads (mbarrier expect_tx / complete_tx per stage), waits for
// each stage, issues its four MMAs and commits them to the stage's "empty"
// mbarrier before refilling it.  Out-of-range rows and k are zero-filled by
// the TMA unit.  EPI 0: C (fp32) as gemm_tc_kernel writes it;
// EPI 1: z = C + bias per column, then Z = z, H = bf16(act(z)), Hf = act(z)
// (each output optional, rows of N).
// tile: TM_BN = 64 columns per CTA (256 CTAs for a 8192 x 256 layer, two
// resident per SM: one's epilogue overlaps the other's loads); k-chunk
// stride of the A stage 128 rows x 16 bytes, of the B stage 64 x 16 bytes
constexpr int TM_BN = 64;
constexpr uint32_t TM_SBO = 1024;
constexpr int TM_TILE_B = TM_BN * TC_BK * 2;
// + 1024: the dynamic shared memory base is rounded up to 1024 bytes
constexpr int TM_SMEM = TC_STAGES * (TC_TILE + TM_TILE_B) + 1024;
constexpr uint32_t TM_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TM_BN >> 3) << 17) |
                              ((uint32_t)(TC_BM >> 4) << 24);
// shared-memory matrix descriptor of a K-major SWIZZLE_128B operand: start
// address >> 4 (bits 0-13), leading byte offset 16 (unused for swizzled
// K-major layouts; bits 16-29), stride byte offset 1024 >> 4 (bits 32-45),
// version 1 (bits 46-47), base offset 0 (1024-aligned buffers), layout type
// 2 = SWIZZLE_128B (bits 61-63)
__device__ __forceinline__ uint64_t tm_desc(uint32_t saddr) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (1ull << 16) |
           (static_cast<uint64_t>((TM_SBO >> 4) & 0x3FFFu) << 32) | (1ull << 46) | (2ull << 61);
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::
            "r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// the tile in shared memory -> global memory through the tensor map (rows
// and columns outside the tensor are not written); one bulk group per CTA
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, uint32_t src, int x, int y) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];\n" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(src), "r"(x), "r"(y)
                 : "memory");
}

struct GemmEpilogue {
    const float* bias = nullptr;
    float* Z = nullptr;
    __nv_bfloat16* H = nullptr;
    float* Hf = nullptr;
    int act = 0;
};

// 16 warps: warp w reads TMEM lanes 32 (w % 4) .. (its rows) and the
// columns 16 (w / 4) .. +16 of the tile.
constexpr int TM_THREADS = 512;
template <int EPI>
__global__ void __launch_bounds__(TM_THREADS, 2) gemm_tma_kernel(const __grid_constant__ CUtensorMap tmA,
                                                            const __grid_constant__ CUtensorMap tmB, int M, int N,
                                                            int K, int kc, float* __restrict__ C, int64_t ldc,
                                                            int64_t c_split, GemmEpilogue ep, int* __restrict__ status,
                                                            const __grid_constant__ CUtensorMap tmZ,
                                                            const __grid_constant__ CUtensorMap tmH, int tstore) {
    extern __shared__ __align__(1024) uint8_t tc_smem[];
    __shared__ uint64_t full[TC_STAGES], empty[TC_STAGES];
    __shared__ uint32_t tmem_slot;
    // 1024-byte aligned stage buffers (the swizzle pattern repeats every
    // 1024 bytes and the descriptors assume it starts at the buffer)
    uint8_t* base = tc_smem + ((1024u - (smem_u32(tc_smem) & 1023u)) & 1023u);
    uint8_t* sA0 = base;
    uint8_t* sB0 = base + TC_STAGES * TC_TILE;
    const int m0 = blockIdx.y * TC_BM, n0 = blockIdx.x * TM_BN;
    const int kb = blockIdx.z * kc, ke = min(K, kb + kc);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_slot)),
                     "r"(TM_BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < TC_STAGES; i++) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    const int nk = ke > kb ? (ke - kb + TC_BK - 1) / TC_BK : 0;
    bool ok = true;
    if (threadIdx.x == 0 && nk > 0) {
        auto load = [&](int j) {
            const int st = j % TC_STAGES;
            mbar_expect_tx(&full[st], static_cast<uint32_t>(TC_TILE + TM_TILE_B));
            const uint32_t a = smem_u32(sA0 + st * TC_TILE), b = smem_u32(sB0 + st * TM_TILE_B);
            const int k0 = kb + j * TC_BK;
            tma_load_2d(a, &tmA, k0, m0, &full[st]);
            tma_load_2d(b, &tmB, k0, n0, &full[st]);
        };
        for (int j = 0; j < TC_STAGES && j < nk; j++) load(j);
        for (int it = 0; it < nk; it++) {
            const int st = it % TC_STAGES;
            const unsigned ph = (it / TC_STAGES) & 1;
            if (!mbar_wait(&full[st], ph)) ok = false;
            tc_fence_after();
            const uint32_t a0 = smem_u32(sA0 + st * TC_TILE), b0 = smem_u32(sB0 + st * TM_TILE_B);
#pragma unroll
            for (int k = 0; k < TC_BK / 16; k++) {
                const uint64_t ad = tm_desc(a0 + k * 32);
                const uint64_t bd = tm_desc(b0 + k * 32);
                const uint32_t acc = (it > 0 || k > 0) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(TM_IDESC), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             smem_u32(&empty[st]))
                         : "memory");
            if (it + TC_STAGES < nk) {
                // the stage is free once its MMAs have read it
                if (!mbar_wait(&empty[st], ph)) ok = false;
                load(it + TC_STAGES);
            }
        }
    }
    __syncwarp();
    if (nk > 0 && !mbar_wait(&empty[(nk - 1) % TC_STAGES], ((nk - 1) / TC_STAGES) & 1)) ok = false;
    tc_fence_after();
    const int wl = warp & 3, wc = warp >> 2;
    const int64_t row = m0 + wl * 32 + lane;
    {
        const int c0 = wc * 16;
        uint32_t v[16];
        if (nk > 0) {
            const uint32_t taddr = tmem + (static_cast<uint32_t>(wl * 32) << 16) + static_cast<uint32_t>(c0);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];\n"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        } else {
#pragma unroll
            for (int j = 0; j < 16; j++) v[j] = 0u;
        }
        const int col0 = n0 + c0;
        if (EPI == 1 && tstore) {
            // Z and H of the tile into shared memory in the 128-byte-swizzled
            // layout of the output tensor maps (16-byte chunk c of tile row r
            // at r * 128 + ((c ^ (r & 7)) << 4), so the 8 rows of one store
            // phase fall on 8 different bank groups): Z as two boxes of 32
            // columns, H as one of 64; thread 0 stores them with the TMA
            // below.  The stage buffers are free: the last commit covered
            // every MMA, and every load had landed before its MMA.
            float bv[16];
            const float* bp = ep.bias + col0;
            if (col0 + 16 <= N && (reinterpret_cast<uintptr_t>(bp) & 15) == 0) {
#pragma unroll
                for (int j = 0; j < 16; j += 4) {
                    const float4 q = __ldg(reinterpret_cast<const float4*>(bp + j));
                    bv[j] = q.x;
                    bv[j + 1] = q.y;
                    bv[j + 2] = q.z;
                    bv[j + 3] = q.w;
                }
            } else {
#pragma unroll
                for (int j = 0; j < 16; j++) bv[j] = col0 + j < N ? bp[j] : 0.f;
            }
            float z[16], h[16];
#pragma unroll
            for (int j = 0; j < 16; j++) {
                z[j] = __uint_as_float(v[j]) + bv[j];
                h[j] = ep.act ? gelu(z[j]) : z[j];
            }
            const int r = wl * 32 + lane;
            const uint32_t sw = static_cast<uint32_t>(r & 7);
            uint8_t* zrow = base + (wc >> 1) * (TC_BM * 128) + r * 128;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint32_t ch = static_cast<uint32_t>(4 * (wc & 1) + q);
                *reinterpret_cast<float4*>(zrow + ((ch ^ sw) << 4)) =
                    make_float4(z[4 * q], z[4 * q + 1], z[4 * q + 2], z[4 * q + 3]);
            }
            uint8_t* hrow = base + 2 * (TC_BM * 128) + r * 128;
#pragma unroll
            for (int q = 0; q < 2; q++) {
                __align__(16) __nv_bfloat16 hb[8];
#pragma unroll
                for (int j = 0; j < 8; j++) hb[j] = __float2bfloat16(h[8 * q + j]);
                const uint32_t ch = static_cast<uint32_t>(2 * wc + q);
                *reinterpret_cast<uint4*>(hrow + ((ch ^ sw) << 4)) = *reinterpret_cast<const uint4*>(hb);
            }
            // the generic-proxy writes, visible to the bulk copies
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        } else if (row >= M) {
        } else if (EPI == 0) {
            float* dst = C + blockIdx.z * c_split + row * ldc + col0;
            if (col0 + 16 <= N && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
#pragma unroll
                for (int j = 0; j < 16; j += 4)
                    *reinterpret_cast<float4*>(dst + j) = make_float4(__uint_as_float(v[j]), __uint_as_float(v[j + 1]),
                                                                      __uint_as_float(v[j + 2]), __uint_as_float(v[j + 3]));
            } else {
#pragma unroll
                for (int j = 0; j < 16; j++)
                    if (col0 + j < N) dst[j] = __uint_as_float(v[j]);
            }
        } else {
            float z[16], h[16];
#pragma unroll
            for (int j = 0; j < 16; j++) {
                z[j] = col0 + j < N ? __uint_as_float(v[j]) + ep.bias[col0 + j] : 0.f;
                h[j] = ep.act ? gelu(z[j]) : z[j];
            }
            const int64_t o = row * N + col0;
            const bool full16 = col0 + 16 <= N && (N & 7) == 0;
            if (ep.Z) {
                if (full16 && (N & 3) == 0) {
#pragma unroll
                    for (int j = 0; j < 16; j += 4)
                        *reinterpret_cast<float4*>(ep.Z + o + j) = make_float4(z[j], z[j + 1], z[j + 2], z[j + 3]);
                } else {
                    for (int j = 0; j < 16; j++)
                        if (col0 + j < N) ep.Z[o + j] = z[j];
                }
            }
            if (ep.Hf) {
                for (int j = 0; j < 16; j++)
                    if (col0 + j < N) ep.Hf[o + j] = h[j];
            }
            if (ep.H) {
                if (full16) {
                    __align__(16) __nv_bfloat16 hb[16];
#pragma unroll
                    for (int j = 0; j < 16; j++) hb[j] = __float2bfloat16(h[j]);
                    *reinterpret_cast<uint4*>(ep.H + o) = *reinterpret_cast<const uint4*>(hb);
                    *reinterpret_cast<uint4*>(ep.H + o + 8) = *reinterpret_cast<const uint4*>(hb + 8);
                } else {
                    for (int j = 0; j < 16; j++)
                        if (col0 + j < N) ep.H[o + j] = __float2bfloat16(h[j]);
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TM_BN) : "memory");
    }
    if (EPI == 1 && tstore && threadIdx.x == 0) {
        // x = n0 and n0 + 32: multiples of 32 columns, 128-byte aligned
        tma_store_2d(&tmZ, smem_u32(base), n0, m0);
        if (n0 + 32 < N) tma_store_2d(&tmZ, smem_u32(base + TC_BM * 128), n0 + 32, m0);
        tma_store_2d(&tmH, smem_u32(base + 2 * TC_BM * 128), n0, m0);
        asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
        // the shared memory stays allocated until the copies are complete
        asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
    }
    if (!ok) atomicOr(status, 1);
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// Row of the network input from raw input row x (n_in floats): x, then per
// frequency f < nf: sin(2^f pi s), cos(2^f pi s) for s = x[n_in-2] and for
// s = x[n_in-1].
__device__ __forceinline__ void write_features(const float* __restrict__ x, int n_in, int nf,
                                               __nv_bfloat16* __restrict__ out) {
    for (int j = 0; j < n_in; j++) out[j] = __float2bfloat16(x[j]);
    int o = n_in;
    for (int c = 0; c < 2; c++) {
        const float s = x[n_in - 2 + c];
        float w = 3.14159265358979f;
        for (int f = 0; f < nf; f++) {
            float sn, cs;
            sincosf(w * s, &sn, &cs);
            out[o++] = __float2bfloat16(sn);
            out[o++] = __float2bfloat16(cs);
            w *= 2.f;
        }
    }
}

__global__ void features_kernel(int64_t M, int n_in, int nf, int width, const float* __restrict__ x,
                                __nv_bfloat16* __restrict__ h) {
    const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= M) return;
    write_features(x + r * n_in, n_in, nf, h + r * width);
}

__global__ void gather_kernel(int M, int64_t n_rows, int n_in, int nf, int width, int n_out,
                              const float* __restrict__ X, const float* __restrict__ T, uint64_t key,
                              __nv_bfloat16* __restrict__ h, float* __restrict__ tb) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= M) return;
    const int64_t src = static_cast<int64_t>(mix64(key + static_cast<uint64_t>(r) * 0x9E3779B97F4A7C15ULL) %
                                             static_cast<uint64_t>(n_rows));
    write_features(X + src * n_in, n_in, nf, h + static_cast<int64_t>(r) * width);
    for (int j = 0; j < n_out; j++) tb[static_cast<int64_t>(r) * n_out + j] = T[src * n_out + j];
}

__global__ void bias_act_kernel(int M, int N, const float* __restrict__ C, const float* __restrict__ bias,
                                float* __restrict__ Z, __nv_bfloat16* __restrict__ H, float* __restrict__ Hf, int act) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<int64_t>(M) * N) return;
    const float z = C[i] + bias[i % N];
    if (Z) Z[i] = z;
    const float h = act ? gelu(z) : z;
    if (H) H[i] = __float2bfloat16(h);
    if (Hf) Hf[i] = h;
}

__global__ void act_bwd_kernel(int64_t n, const float* __restrict__ dH, const float* __restrict__ Z,
                               float* __restrict__ dZ, __nv_bfloat16* __restrict__ dZb, int act) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float d = act ? dH[i] * gelu_grad(Z[i]) : dH[i];
    dZ[i] = d;
    dZb[i] = __float2bfloat16(d);
}

// column sums of an M x N matrix: per chunk of kColRows rows, then the
// chunks in order
constexpr int kColRows = 128;
__global__ void col_sum_partial_kernel(int M, int N, const float* __restrict__ X, float* __restrict__ part) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    const int r0 = blockIdx.y * kColRows, r1 = min(M, r0 + kColRows);
    float s = 0.f;
    for (int r = r0; r < r1; r++) s += X[static_cast<int64_t>(r) * N + c];
    part[static_cast<int64_t>(blockIdx.y) * N + c] = s;
}
__global__ void col_sum_final_kernel(int chunks, int N, const float* __restrict__ part, float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    float s = 0.f;
    for (int k = 0; k < chunks; k++) s += part[static_cast<int64_t>(k) * N + c];
    out[c] = s;
}

__global__ void mse_kernel(int M, int N, const float* __restrict__ Y, const float* __restrict__ T,
                           float* __restrict__ dY, float* __restrict__ row_err) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= M) return;
    const float scale = 2.f / (static_cast<float>(M) * N);
    float e = 0.f;
    for (int c = 0; c < N; c++) {
        const float d = Y[static_cast<int64_t>(r) * N + c] - T[static_cast<int64_t>(r) * N + c];
        e += d * d;
        dY[static_cast<int64_t>(r) * N + c] = scale * d;
    }
    row_err[r] = e;
}

// one block of 256 threads: strided partial sums, then a fixed tree
__global__ void loss_kernel(int M, int N, const float* __restrict__ row_err, float* __restrict__ out) {
    __shared__ double s[256];
    double a = 0.0;
    for (int r = threadIdx.x; r < M; r += 256) a += row_err[r];
    s[threadIdx.x] = a;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = static_cast<float>(s[0] / (static_cast<double>(M) * N));
}

__global__ void adam_kernel(int64_t n, float* __restrict__ w, const float* __restrict__ gr, float* __restrict__ m,
                            float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                            __nv_bfloat16* __restrict__ wb) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = gr[i];
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    wb[i] = __float2bfloat16(wi);
}

__global__ void to_bf16_kernel(int64_t n, const float* __restrict__ x, __nv_bfloat16* __restrict__ y) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) y[i] = __float2bfloat16(x[i]);
}

inline unsigned blocks(int64_t n, int t) { return static_cast<unsigned>((n + t - 1) / t); }

struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
    Buf() = default;
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
    Buf(Buf&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; }
    ~Buf() {
        if (p) cudaFree(p);
    }
    bool alloc(size_t n) {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = n;
        return cudaMalloc(&p, n ? n : 16) == cudaSuccess;
    }
    template <typename T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

// number of K slices of length kc
inline int split_count(int K, int kc) { return K > 0 ? (K + kc - 1) / kc : 1; }

inline bool vec_ok(const void* p, int64_t ld) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0 && ld % 8 == 0; }

// status word of the tensor-core GEMM (bit 0: an mbarrier wait expired)
__device__ int g_gemm_status = 0;

template <bool AV, bool BV>
void launch_tc(dim3 grid, int M, int N, int K, int kc, const __nv_bfloat16* A, int64_t lda, const __nv_bfloat16* B,
               int64_t ldb, float* C, int64_t ldc, int64_t c_split, cudaStream_t s) {
    // the shared-memory opt-in is a per-device attribute of the kernel
    static bool attr[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr[dev]) {
        cudaFuncSetAttribute(gemm_tc_kernel<AV, BV>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
        if (dev >= 0 && dev < 64) attr[dev] = true;
    }
    int* st = nullptr;
    cudaGetSymbolAddress(reinterpret_cast<void**>(&st), g_gemm_status);
    gemm_tc_kernel<AV, BV><<<grid, TC_THREADS, TC_SMEM, s>>>(M, N, K, kc, A, lda, B, ldb, C, ldc, c_split, st);
}

// cuTensorMapEncodeTiled, looked up in the driver once (no link against the
// driver library); null where the driver does not offer it
using TensorMapEncode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                     const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                     CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
TensorMapEncode tensor_map_encoder() {
    static TensorMapEncode fn = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<TensorMapEncode>(f);
        else
            cudaGetLastError();
    }
    return fn;
}

// The tensor map of a k-contiguous bf16 operand of `rows` rows of `ld`
// elements, K of them used: boxes of 64 k (128 bytes) x box_rows rows with
// the 128-byte swizzle, zero fill outside.
bool operand_map(CUtensorMap* map, const __nv_bfloat16* X, int64_t ld, int rows, int K, int box_rows) {
    const TensorMapEncode enc = tensor_map_encoder();
    if (!enc || rows <= 0 || K <= 0) return false;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(K), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld) * 2};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(TC_BK), static_cast<cuuint32_t>(box_rows)};
    const cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(X), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The tensor map of a row-major output [rows][N] (fp32 or bf16) for the
// TMA stores of the fused epilogue: boxes of 128 bytes of a row (32 fp32 or
// 64 bf16) x 128 rows, 128-byte swizzle.
bool output_map(CUtensorMap* map, void* X, bool f32, int rows, int N) {
    const TensorMapEncode enc = tensor_map_encoder();
    if (!enc || rows <= 0 || N <= 0) return false;
    const int es = f32 ? 4 : 2;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(N), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(N) * es};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(128 / es), static_cast<cuuint32_t>(TC_BM)};
    const cuuint32_t estr[2] = {1, 1};
    return enc(map, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, X, dims, strides, box,
               estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// address of the GEMM status word on the current device (looked up once)
int* gemm_status_ptr() {
    static int* addr[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!addr[dev]) cudaGetSymbolAddress(reinterpret_cast<void**>(&addr[dev]), g_gemm_status);
    return addr[dev];
}

// The TMA GEMM; false (nothing launched) where an operand cannot be
// described by a tensor map (rows not 16-byte aligned) or the driver offers
// no encoder: the caller then uses gemm_tc_kernel.
template <int EPI>
bool launch_tma(dim3 grid, int M, int N, int K, int kc, const __nv_bfloat16* A, int64_t lda, const __nv_bfloat16* B,
                int64_t ldb, float* C, int64_t ldc, int64_t c_split, const GemmEpilogue& ep, cudaStream_t s) {
    if (!vec_ok(A, lda) || !vec_ok(B, ldb)) return false;
    CUtensorMap ma, mb;
    if (!operand_map(&ma, A, lda, M, K, TC_BM) || !operand_map(&mb, B, ldb, N, K, TM_BN)) return false;
    grid.x = blocks(N, TM_BN);
    static bool attr[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr[dev]) {
        cudaFuncSetAttribute(gemm_tma_kernel<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, TM_SMEM);
        if (dev >= 0 && dev < 64) attr[dev] = true;
    }
    // the fused epilogue of a hidden layer (Z and H, no fp32 activation)
    // leaves the tile through shared memory and the TMA where both outputs
    // can be described by tensor maps (16-byte aligned rows)
    CUtensorMap mz{}, mh{};
    const bool tstore = EPI == 1 && ep.Z && ep.H && !ep.Hf && N % 8 == 0 &&
                        (reinterpret_cast<uintptr_t>(ep.Z) & 15) == 0 && (reinterpret_cast<uintptr_t>(ep.H) & 15) == 0 &&
                        output_map(&mz, ep.Z, true, M, N) && output_map(&mh, ep.H, false, M, N);
    gemm_tma_kernel<EPI><<<grid, TM_THREADS, TM_SMEM, s>>>(ma, mb, M, N, K, kc, C, ldc, c_split, ep,
                                                           gemm_status_ptr(), mz, mh, tstore ? 1 : 0);
    return true;
}

// K slice of a GEMM split `splits` ways (a multiple of the K stage)
inline int tc_split_len(int K, int splits) {
    int kc = (K + splits - 1) / splits;
    return kc > 0 ? (kc + TC_BK - 1) / TC_BK * TC_BK : TC_BK;
}

// C = A . B^T with A [M][lda], B [N][ldb] (k contiguous); see gemm_tc_kernel
void gemm(int M, int N, int K, const __nv_bfloat16* A, int64_t lda, const __nv_bfloat16* B, int64_t ldb, float* C,
          int64_t ldc, cudaStream_t s, int splits = 1, int64_t c_split = 0) {
    if (M <= 0 || N <= 0) return;
    const int kc = tc_split_len(K, splits);
    dim3 grid(blocks(N, TC_BN), blocks(M, TC_BM), split_count(K, kc));
    if (launch_tma<0>(grid, M, N, K, kc, A, lda, B, ldb, C, ldc, c_split, GemmEpilogue{}, s)) return;
    const bool av = vec_ok(A, lda), bv = vec_ok(B, ldb);
    if (av && bv)
        launch_tc<true, true>(grid, M, N, K, kc, A, lda, B, ldb, C, ldc, c_split, s);
    else if (av)
        launch_tc<true, false>(grid, M, N, K, kc, A, lda, B, ldb, C, ldc, c_split, s);
    else if (bv)
        launch_tc<false, true>(grid, M, N, K, kc, A, lda, B, ldb, C, ldc, c_split, s);
    else
        launch_tc<false, false>(grid, M, N, K, kc, A, lda, B, ldb, C, ldc, c_split, s);
}

// reads and clears the GEMM status word (after a synchronisation)
bool gemm_status_ok() {
    int v = 0;
    cudaMemcpyFromSymbol(&v, g_gemm_status, sizeof(int));
    if (v) {
        const int zero = 0;
        cudaMemcpyToSymbol(g_gemm_status, &zero, sizeof(int));
    }
    return v == 0;
}

inline int64_t pad8(int64_t n) { return (n + 7) / 8 * 8; }

void transpose(int R, int Cc, const __nv_bfloat16* in, int64_t ldin, __nv_bfloat16* out, int64_t ldout,
               cudaStream_t s) {
    if (R <= 0 || Cc <= 0) return;
    transpose_bf16_kernel<<<dim3(blocks(Cc, 32), blocks(R, 32)), dim3(32, 8), 0, s>>>(R, Cc, in, ldin, out, ldout);
}

constexpr int kMaxSplit = 32;

}  // namespace

struct gelios_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    int n_in = 0, nf = 0, width = 0, depth = 0, n_out = 0, max_batch = 0;
    int in_w = 0;  // width of the first layer's input (raw inputs + 4 nf features)
    std::vector<int> din, dout;
    std::vector<int64_t> w_off, b_off;
    int64_t n_params = 0;
    int step = 0;
    Buf w32, g32, m, v, wb;
    std::vector<Buf> h;  // bf16 inputs of every layer [max_batch][din]
    std::vector<Buf> z;  // fp32 pre-activations of every hidden layer
    Buf c, y, dh, dz, dzb, tb, rowerr, part, colpart, loss, xin;
    Buf wt, dzt, ht;  // transposes for the backward GEMMs: W_l^T, dZ^T, H_l^T
    Buf X, T;  // training set (fp32 rows)
    int64_t n_rows = 0;
    ~gelios_mlp() {
        if (stream) cudaStreamDestroy(stream);
    }
    int layers() const { return depth + 1; }
};

namespace {
int fail(const char* what) {
    gelios::set_error(what);
    return GELIOS_E_ARG;
}
int cuda_fail(cudaError_t e) {
    gelios::set_error(std::string("CUDA: ") + cudaGetErrorString(e));
    return GELIOS_E_CUDA;
}
#define MLP_TRY(x)                                   \
    do {                                             \
        cudaError_t e_ = (x);                        \
        if (e_ != cudaSuccess) return cuda_fail(e_); \
    } while (0)

// forward pass of M rows whose network inputs are in h[0]; output in y
void forward(gelios_mlp* n, int M) {
    cudaStream_t s = n->stream;
    const __nv_bfloat16* wb = n->wb.as<__nv_bfloat16>();
    for (int l = 0; l < n->layers(); l++) {
        const int di = n->din[l], dO = n->dout[l];
        const bool last = l == n->layers() - 1;
        GemmEpilogue ep;
        ep.bias = n->w32.as<float>() + n->b_off[l];
        ep.Z = last ? nullptr : n->z[l].as<float>();
        ep.H = last ? nullptr : n->h[l + 1].as<__nv_bfloat16>();
        ep.Hf = last ? n->y.as<float>() : nullptr;
        ep.act = last ? 0 : 1;
        // bias and activation applied as the accumulator leaves tensor memory
        // (TMA path), or by bias_act_kernel after the GEMM
        const __nv_bfloat16* A = n->h[l].as<__nv_bfloat16>();
        dim3 grid(blocks(dO, TC_BN), blocks(M, TC_BM), 1);
        if (M > 0 && launch_tma<1>(grid, M, dO, di, tc_split_len(di, 1), A, di, wb + n->w_off[l], di, nullptr, 0, 0,
                                   ep, s))
            continue;
        gemm(M, dO, di, A, di, wb + n->w_off[l], di, n->c.as<float>(), dO, s);
        const int64_t e = static_cast<int64_t>(M) * dO;
        bias_act_kernel<<<blocks(e, 256), 256, 0, s>>>(M, dO, n->c.as<float>(), ep.bias, ep.Z, ep.H, ep.Hf, ep.act);
    }
}

// loss of the batch (targets in tb) into loss[0]; gradients into g32
void backward(gelios_mlp* n, int M) {
    cudaStream_t s = n->stream;
    const int L = n->layers();
    const int64_t eo = static_cast<int64_t>(M) * n->n_out;
    mse_kernel<<<blocks(M, 256), 256, 0, s>>>(M, n->n_out, n->y.as<float>(), n->tb.as<float>(), n->dh.as<float>(),
                                              n->rowerr.as<float>());
    loss_kernel<<<1, 256, 0, s>>>(M, n->n_out, n->rowerr.as<float>(), n->loss.as<float>());
    act_bwd_kernel<<<blocks(eo, 256), 256, 0, s>>>(eo, n->dh.as<float>(), nullptr, n->dz.as<float>(),
                                                   n->dzb.as<__nv_bfloat16>(), 0);
    const __nv_bfloat16* wb = n->wb.as<__nv_bfloat16>();
    float* g = n->g32.as<float>();
    int splits = (M + 255) / 256;
    if (splits > kMaxSplit) splits = kMaxSplit;
    if (splits < 1) splits = 1;
    const int S = split_count(M, tc_split_len(M, splits));
    const int64_t Mp = pad8(M);
    __nv_bfloat16* dzt = n->dzt.as<__nv_bfloat16>();
    __nv_bfloat16* ht = n->ht.as<__nv_bfloat16>();
    for (int l = L - 1; l >= 0; l--) {
        const int di = n->din[l], dO = n->dout[l];
        // dW[dO][di] = dZ^T . H_l (both transposed so k = batch row is
        // contiguous), split over the rows of the batch
        const int64_t wn = static_cast<int64_t>(dO) * di;
        transpose(M, dO, n->dzb.as<__nv_bfloat16>(), dO, dzt, Mp, s);
        transpose(M, di, n->h[l].as<__nv_bfloat16>(), di, ht, Mp, s);
        gemm(dO, di, M, dzt, Mp, ht, Mp, n->part.as<float>(), di, s, splits, wn);
        splitk_reduce_kernel<<<blocks(wn, 256), 256, 0, s>>>(wn, S, n->part.as<float>(), g + n->w_off[l]);
        // db = column sums of dZ
        const int chunks = (M + kColRows - 1) / kColRows;
        col_sum_partial_kernel<<<dim3(blocks(dO, 128), chunks), 128, 0, s>>>(M, dO, n->dz.as<float>(),
                                                                             n->colpart.as<float>());
        col_sum_final_kernel<<<blocks(dO, 128), 128, 0, s>>>(chunks, dO, n->colpart.as<float>(), g + n->b_off[l]);
        if (l == 0) break;
        // dH_l[M][di] = dZ . W_l, then dZ_{l-1} = dH_l * GELU'(Z_{l-1})
        transpose(dO, di, wb + n->w_off[l], di, n->wt.as<__nv_bfloat16>(), pad8(dO), s);
        gemm(M, di, dO, n->dzb.as<__nv_bfloat16>(), dO, n->wt.as<__nv_bfloat16>(), pad8(dO), n->dh.as<float>(), di,
             s);
        const int64_t e = static_cast<int64_t>(M) * di;
        act_bwd_kernel<<<blocks(e, 256), 256, 0, s>>>(e, n->dh.as<float>(), n->z[l - 1].as<float>(),
                                                      n->dz.as<float>(), n->dzb.as<__nv_bfloat16>(), 1);
    }
}
}  // namespace

extern "C" int gelios_mlp_create(gelios_mlp** out, int device, int n_in, int n_fourier, int width, int depth,
                                 int n_out, int max_batch) {
    if (!out) return fail("gelios_mlp_create: null output");
    *out = nullptr;
    if (n_in < 2 || n_in > 256 || n_fourier < 0 || n_fourier > 16 || width < 1 || width > 4096 || depth < 1 ||
        depth > 64 || n_out < 1 || n_out > 4096 || max_batch < 1 || max_batch > (1 << 20))
        return fail("gelios_mlp_create: sizes out of range");
    auto n = std::make_unique<gelios_mlp>();
    n->device = device;
    n->n_in = n_in;
    n->nf = n_fourier;
    n->width = width;
    n->depth = depth;
    n->n_out = n_out;
    n->max_batch = max_batch;
    n->in_w = n_in + 4 * n_fourier;
    MLP_TRY(cudaSetDevice(device));
    MLP_TRY(cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking));
    int64_t off = 0;
    int widest = n->in_w > width ? n->in_w : width;
    if (n_out > widest) widest = n_out;
    for (int l = 0; l <= depth; l++) {
        const int di = l == 0 ? n->in_w : width, dO = l == depth ? n_out : width;
        n->din.push_back(di);
        n->dout.push_back(dO);
        n->w_off.push_back(off);
        off += static_cast<int64_t>(di) * dO;
        n->b_off.push_back(off);
        off += dO;
    }
    n->n_params = off;
    const size_t P = static_cast<size_t>(off);
    const size_t MB = static_cast<size_t>(max_batch), W = static_cast<size_t>(widest);
    bool ok = n->w32.alloc(P * 4) && n->g32.alloc(P * 4) && n->m.alloc(P * 4) && n->v.alloc(P * 4) &&
              n->wb.alloc(P * 2);
    n->h.resize(depth + 1);
    n->z.resize(depth);
    for (int l = 0; l <= depth; l++) ok = ok && n->h[l].alloc(MB * n->din[l] * 2);
    for (int l = 0; l < depth; l++) ok = ok && n->z[l].alloc(MB * width * 4);
    ok = ok && n->c.alloc(MB * W * 4) && n->y.alloc(MB * n_out * 4) && n->dh.alloc(MB * W * 4) &&
         n->dz.alloc(MB * W * 4) && n->dzb.alloc(MB * W * 2) && n->tb.alloc(MB * n_out * 4) &&
         n->rowerr.alloc(MB * 4) && n->part.alloc(static_cast<size_t>(kMaxSplit) * W * W * 4) &&
         n->colpart.alloc(((MB + kColRows - 1) / kColRows) * W * 4) && n->loss.alloc(16) &&
         n->xin.alloc(MB * n_in * 4) && n->wt.alloc(W * pad8(widest) * 2) &&
         n->dzt.alloc(W * pad8(max_batch) * 2) && n->ht.alloc(W * pad8(max_batch) * 2);
    if (!ok) return cuda_fail(cudaErrorMemoryAllocation);
    MLP_TRY(cudaMemsetAsync(n->w32.p, 0, P * 4, n->stream));
    MLP_TRY(cudaMemsetAsync(n->wb.p, 0, P * 2, n->stream));
    MLP_TRY(cudaMemsetAsync(n->m.p, 0, P * 4, n->stream));
    MLP_TRY(cudaMemsetAsync(n->v.p, 0, P * 4, n->stream));
    MLP_TRY(cudaStreamSynchronize(n->stream));
    *out = n.release();
    return GELIOS_OK;
}

extern "C" void gelios_mlp_destroy(gelios_mlp* n) {
    if (!n) return;
    cudaSetDevice(n->device);
    cudaStreamSynchronize(n->stream);
    delete n;
}

extern "C" int64_t gelios_mlp_param_count(const gelios_mlp* n) { return n ? n->n_params : -1; }

extern "C" int gelios_mlp_set_params(gelios_mlp* n, const float* host, int64_t count) {
    if (!n || !host || count != n->n_params) return fail("gelios_mlp_set_params: wrong parameter count");
    MLP_TRY(cudaSetDevice(n->device));
    const size_t P = static_cast<size_t>(n->n_params);
    MLP_TRY(cudaMemcpyAsync(n->w32.p, host, P * 4, cudaMemcpyHostToDevice, n->stream));
    to_bf16_kernel<<<blocks(n->n_params, 256), 256, 0, n->stream>>>(n->n_params, n->w32.as<float>(),
                                                                    n->wb.as<__nv_bfloat16>());
    MLP_TRY(cudaMemsetAsync(n->m.p, 0, P * 4, n->stream));
    MLP_TRY(cudaMemsetAsync(n->v.p, 0, P * 4, n->stream));
    MLP_TRY(cudaGetLastError());
    MLP_TRY(cudaStreamSynchronize(n->stream));
    n->step = 0;
    return GELIOS_OK;
}

extern "C" int gelios_mlp_get_params(const gelios_mlp* n, float* host, int64_t count) {
    if (!n || !host || count != n->n_params) return fail("gelios_mlp_get_params: wrong parameter count");
    MLP_TRY(cudaSetDevice(n->device));
    MLP_TRY(cudaMemcpyAsync(host, n->w32.p, static_cast<size_t>(count) * 4, cudaMemcpyDeviceToHost, n->stream));
    MLP_TRY(cudaStreamSynchronize(n->stream));
    return GELIOS_OK;
}

extern "C" int gelios_mlp_loss_grad(gelios_mlp* n, const float* x, const float* t, int M, double* loss, float* grad) {
    if (!n || !x || !t || M < 1 || M > n->max_batch) return fail("gelios_mlp_loss_grad: bad arguments");
    MLP_TRY(cudaSetDevice(n->device));
    cudaStream_t s = n->stream;
    MLP_TRY(cudaMemcpyAsync(n->xin.p, x, static_cast<size_t>(M) * n->n_in * 4, cudaMemcpyHostToDevice, s));
    MLP_TRY(cudaMemcpyAsync(n->tb.p, t, static_cast<size_t>(M) * n->n_out * 4, cudaMemcpyHostToDevice, s));
    features_kernel<<<blocks(M, 128), 128, 0, s>>>(M, n->n_in, n->nf, n->in_w, n->xin.as<float>(),
                                                   n->h[0].as<__nv_bfloat16>());
    forward(n, M);
    backward(n, M);
    MLP_TRY(cudaGetLastError());
    float l = 0.f;
    MLP_TRY(cudaMemcpyAsync(&l, n->loss.p, 4, cudaMemcpyDeviceToHost, s));
    if (grad)
        MLP_TRY(cudaMemcpyAsync(grad, n->g32.p, static_cast<size_t>(n->n_params) * 4, cudaMemcpyDeviceToHost, s));
    MLP_TRY(cudaStreamSynchronize(s));
    if (!gemm_status_ok()) return cuda_fail(cudaErrorLaunchTimeout);
    if (loss) *loss = l;
    return GELIOS_OK;
}

extern "C" int gelios_mlp_set_data(gelios_mlp* n, const float* x, const float* t, int64_t n_rows) {
    if (!n || !x || !t || n_rows < 1) return fail("gelios_mlp_set_data: bad arguments");
    MLP_TRY(cudaSetDevice(n->device));
    if (!n->X.alloc(static_cast<size_t>(n_rows) * n->n_in * 4) ||
        !n->T.alloc(static_cast<size_t>(n_rows) * n->n_out * 4))
        return cuda_fail(cudaErrorMemoryAllocation);
    MLP_TRY(cudaMemcpyAsync(n->X.p, x, static_cast<size_t>(n_rows) * n->n_in * 4, cudaMemcpyHostToDevice, n->stream));
    MLP_TRY(cudaMemcpyAsync(n->T.p, t, static_cast<size_t>(n_rows) * n->n_out * 4, cudaMemcpyHostToDevice, n->stream));
    MLP_TRY(cudaStreamSynchronize(n->stream));
    n->n_rows = n_rows;
    return GELIOS_OK;
}

extern "C" int gelios_mlp_train(gelios_mlp* n, int iters, int batch, float lr_max, float lr_min, int warmup,
                                uint64_t seed, float* loss_hist) {
    if (!n || iters < 0 || batch < 1 || batch > n->max_batch || !(lr_max >= 0.f) || !(lr_min >= 0.f) || warmup < 0)
        return fail("gelios_mlp_train: bad arguments");
    if (n->n_rows < 1) return fail("gelios_mlp_train: no training set (gelios_mlp_set_data)");
    MLP_TRY(cudaSetDevice(n->device));
    cudaStream_t s = n->stream;
    Buf hist;
    if (!hist.alloc(static_cast<size_t>(iters > 0 ? iters : 1) * 4)) return cuda_fail(cudaErrorMemoryAllocation);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int it = 0; it < iters; it++) {
        const uint64_t key = seed * 0xD1B54A32D192ED03ULL + static_cast<uint64_t>(n->step) * 0x8CB92BA72F3D8DD7ULL;
        gather_kernel<<<blocks(batch, 128), 128, 0, s>>>(batch, n->n_rows, n->n_in, n->nf, n->in_w, n->n_out,
                                                         n->X.as<float>(), n->T.as<float>(), key,
                                                         n->h[0].as<__nv_bfloat16>(), n->tb.as<float>());
        forward(n, batch);
        backward(n, batch);
        MLP_TRY(cudaMemcpyAsync(hist.as<float>() + it, n->loss.p, 4, cudaMemcpyDeviceToDevice, s));
        float lr;
        if (it < warmup) {
            lr = lr_max * static_cast<float>(it + 1) / static_cast<float>(warmup);
        } else {
            const double q = iters > warmup ? static_cast<double>(it - warmup) / (iters - warmup) : 1.0;
            lr = static_cast<float>(lr_min + 0.5 * (lr_max - lr_min) * (1.0 + std::cos(3.14159265358979 * q)));
        }
        n->step++;
        const float c1 = static_cast<float>(1.0 - std::pow(static_cast<double>(b1), n->step));
        const float c2 = static_cast<float>(1.0 - std::pow(static_cast<double>(b2), n->step));
        adam_kernel<<<blocks(n->n_params, 256), 256, 0, s>>>(n->n_params, n->w32.as<float>(), n->g32.as<float>(),
                                                             n->m.as<float>(), n->v.as<float>(), lr, b1, b2, eps, c1,
                                                             c2, n->wb.as<__nv_bfloat16>());
        MLP_TRY(cudaGetLastError());
    }
    if (loss_hist && iters > 0)
        MLP_TRY(cudaMemcpyAsync(loss_hist, hist.p, static_cast<size_t>(iters) * 4, cudaMemcpyDeviceToHost, s));
    MLP_TRY(cudaStreamSynchronize(s));
    if (!gemm_status_ok()) return cuda_fail(cudaErrorLaunchTimeout);
    return GELIOS_OK;
}

extern "C" int gelios_mlp_predict(gelios_mlp* n, const float* x, int64_t M, float* y) {
    if (!n || !x || !y || M < 0) return fail("gelios_mlp_predict: bad arguments");
    MLP_TRY(cudaSetDevice(n->device));
    cudaStream_t s = n->stream;
    for (int64_t r0 = 0; r0 < M; r0 += n->max_batch) {
        const int m = static_cast<int>(M - r0 < n->max_batch ? M - r0 : n->max_batch);
        MLP_TRY(cudaMemcpyAsync(n->xin.p, x + r0 * n->n_in, static_cast<size_t>(m) * n->n_in * 4,
                                cudaMemcpyHostToDevice, s));
        features_kernel<<<blocks(m, 128), 128, 0, s>>>(m, n->n_in, n->nf, n->in_w, n->xin.as<float>(),
                                                       n->h[0].as<__nv_bfloat16>());
        forward(n, m);
        MLP_TRY(cudaGetLastError());
        MLP_TRY(cudaMemcpyAsync(y + r0 * n->n_out, n->y.p, static_cast<size_t>(m) * n->n_out * 4,
                                cudaMemcpyDeviceToHost, s));
    }
    MLP_TRY(cudaStreamSynchronize(s));
    if (!gemm_status_ok()) return cuda_fail(cudaErrorLaunchTimeout);
    return GELIOS_OK;
}

extern "C" int gelios_mlp_gemm_bf16(int M, int N, int K, const void* A, int64_t lda, const void* B, int64_t ldb,
                                    float* C, int64_t ldc, void* stream) {
    if (M < 0 || N < 0 || K < 0 || !A || !B || !C || lda < K || ldb < K || ldc < N)
        return fail("gelios_mlp_gemm_bf16: bad arguments");
    gemm(M, N, K, static_cast<const __nv_bfloat16*>(A), lda, static_cast<const __nv_bfloat16*>(B), ldb, C, ldc,
         static_cast<cudaStream_t>(stream));
    MLP_TRY(cudaGetLastError());
    MLP_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    if (!gemm_status_ok()) return cuda_fail(cudaErrorLaunchTimeout);
    return GELIOS_OK;
}

extern "C" int gelios_mlp_time_layer(int M, int N, int K, int reps, int tma, double* ms) {
    if (M <= 0 || N <= 0 || K <= 0 || reps < 1 || !ms) return fail("gelios_mlp_time_layer: bad arguments");
    const int64_t lda = pad8(K);
    Buf A, B, bias, Z, H, Cf;
    if (!A.alloc(static_cast<size_t>(M) * lda * 2) || !B.alloc(static_cast<size_t>(N) * lda * 2) ||
        !Cf.alloc(tma ? 16 : static_cast<size_t>(M) * N * 4) ||
        !bias.alloc(static_cast<size_t>(N) * 4) || !Z.alloc(static_cast<size_t>(M) * N * 4) ||
        !H.alloc(static_cast<size_t>(M) * N * 2))
        return cuda_fail(cudaErrorMemoryAllocation);
    cudaStream_t s = nullptr;
    MLP_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    std::unique_ptr<CUstream_st, void (*)(cudaStream_t)> guard(s, [](cudaStream_t x) { cudaStreamDestroy(x); });
    // seeded operands (a fixed hash of the index, scaled like a trained layer)
    {
        std::vector<__nv_bfloat16> ha(static_cast<size_t>(M) * lda), hb(static_cast<size_t>(N) * lda);
        std::vector<float> hbias(N);
        auto val = [](uint64_t i) {
            uint64_t z = i * 0x9E3779B97F4A7C15ULL;
            z = (z ^ (z >> 31)) * 0xBF58476D1CE4E5B9ULL;
            return static_cast<float>((z >> 40) & 0xFFFF) / 65536.f - 0.5f;
        };
        for (size_t i = 0; i < ha.size(); i++) ha[i] = __float2bfloat16(val(i));
        for (size_t i = 0; i < hb.size(); i++) hb[i] = __float2bfloat16(0.1f * val(i + ha.size()));
        for (int i = 0; i < N; i++) hbias[i] = 0.01f * val(i + 7);
        MLP_TRY(cudaMemcpyAsync(A.p, ha.data(), ha.size() * 2, cudaMemcpyHostToDevice, s));
        MLP_TRY(cudaMemcpyAsync(B.p, hb.data(), hb.size() * 2, cudaMemcpyHostToDevice, s));
        MLP_TRY(cudaMemcpyAsync(bias.p, hbias.data(), hbias.size() * 4, cudaMemcpyHostToDevice, s));
    }
    GemmEpilogue ep;
    ep.bias = bias.as<float>();
    ep.Z = Z.as<float>();
    ep.H = H.as<__nv_bfloat16>();
    ep.act = 1;
    const dim3 grid(blocks(N, TC_BN), blocks(M, TC_BM), 1);
    const int kc = tc_split_len(K, 1);
    auto layer = [&]() {
        if (tma)
            return launch_tma<1>(grid, M, N, K, kc, A.as<__nv_bfloat16>(), lda, B.as<__nv_bfloat16>(), lda, nullptr, 0,
                                 0, ep, s);
        // the cp.async-staged GEMM, then the bias + activation kernel
        const dim3 g2(blocks(N, TC_BN), blocks(M, TC_BM), 1);
        launch_tc<true, true>(g2, M, N, K, kc, A.as<__nv_bfloat16>(), lda, B.as<__nv_bfloat16>(), lda, Cf.as<float>(),
                              N, 0, s);
        const int64_t e = static_cast<int64_t>(M) * N;
        bias_act_kernel<<<blocks(e, 256), 256, 0, s>>>(M, N, Cf.as<float>(), ep.bias, ep.Z, ep.H, nullptr, 1);
        return true;
    };
    if (!layer()) return fail("gelios_mlp_time_layer: no tensor-map encoder in this driver");
    // the reps launches captured in one CUDA graph, so that the device time
    // per layer is not the host's launch rate
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    MLP_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    for (int r = 0; r < reps; r++) layer();
    MLP_TRY(cudaStreamEndCapture(s, &graph));
    std::unique_ptr<CUgraph_st, void (*)(cudaGraph_t)> gguard(graph, [](cudaGraph_t g) { cudaGraphDestroy(g); });
    MLP_TRY(cudaGraphInstantiate(&exec, graph, 0));
    std::unique_ptr<CUgraphExec_st, void (*)(cudaGraphExec_t)> xguard(exec,
                                                                      [](cudaGraphExec_t x) { cudaGraphExecDestroy(x); });
    MLP_TRY(cudaGraphLaunch(exec, s));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    MLP_TRY(cudaEventCreate(&e0));
    MLP_TRY(cudaEventCreate(&e1));
    MLP_TRY(cudaEventRecord(e0, s));
    MLP_TRY(cudaGraphLaunch(exec, s));
    MLP_TRY(cudaEventRecord(e1, s));
    MLP_TRY(cudaEventSynchronize(e1));
    float t = 0.f;
    MLP_TRY(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    MLP_TRY(cudaGetLastError());
    if (!gemm_status_ok()) return cuda_fail(cudaErrorLaunchTimeout);
    *ms = static_cast<double>(t) / reps;
    return GELIOS_OK;
}
