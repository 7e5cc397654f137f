// The warm-start network: a coordinate MLP (inflow parameters and cell
// position -> a converged state of the plain step), trained and evaluated
// on the GPU by this file's kernels.
//
//   gemm_tn_kernel        C[M,N] (fp32) = A[M,K] . B[N,K]^T with bf16 operands
//                         on the tensor cores (mma.sync m16n8k16, fp32
//                         accumulation), both operands k-contiguous: X.W^T
//                         (forward), dZ.(W^T)^T (backward, data) and
//                         (dZ^T).(H^T)^T (backward, weights; split over K
//                         into partial tiles that splitk_reduce_kernel adds
//                         in a fixed order)
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

// GEMM tiles: 128 x 128 output per block of 8 warps (2 x 4, each warp
// 64 x 32 = 4 x 4 tiles of m16n8), K in steps of 32; operand tiles staged
// in shared memory rows of 40 bf16 (80 bytes: the eight 16-byte rows an
// ldmatrix reads fall in distinct bank groups).
constexpr int BM = 128, BN = 128, BK = 32, SPITCH = BK + 8;
constexpr int kGemmThreads = 256;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// 16-byte asynchronous copy global -> shared; bytes beyond src_bytes are zero
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void ldmatrix_x4(uint32_t (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}

// Rows row0.. (of nrows) x k k0..k0+31 (of ke) of a k-contiguous operand
// (rows of ld elements) into S[128][SPITCH]; zeros outside.  VEC: ld and the
// base are 16-byte aligned, so whole 8-element chunks go by cp.async.
template <bool VEC>
__device__ __forceinline__ void load_tile(__nv_bfloat16 (*S)[SPITCH], const __nv_bfloat16* __restrict__ G, int64_t ld,
                                          int row0, int nrows, int k0, int ke) {
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    for (int c = threadIdx.x; c < BM * (BK / 8); c += kGemmThreads) {
        const int r = c >> 2, kq = (c & 3) * 8;
        const int gr = row0 + r, gk = k0 + kq;
        __nv_bfloat16* dst = &S[r][kq];
        if (VEC && gr < nrows && gk + 8 <= ke) {
            cp_async16(smem_u32(dst), G + gr * ld + gk, 16);
        } else if (VEC && (gr >= nrows || gk >= ke)) {
            cp_async16(smem_u32(dst), G, 0);  // zero fill, nothing read
        } else {
            for (int e = 0; e < 8; e++) dst[e] = (gr < nrows && gk + e < ke) ? G[gr * ld + gk + e] : zero;
        }
    }
}

// C[M][N] (fp32, rows of ldc) = sum_k A[m][k] B[n][k], A and B bf16 with k
// contiguous (rows of lda / ldb).  blockIdx.z: K slice [z kc, (z+1) kc),
// written to C + z c_split.  Two-stage cp.async pipeline, fragments by
// ldmatrix, mma.sync m16n8k16 bf16 -> fp32.
template <bool AV, bool BV>
__global__ void __launch_bounds__(kGemmThreads) gemm_tn_kernel(int M, int N, int K, int kc,
                                                             const __nv_bfloat16* __restrict__ A, int64_t lda,
                                                             const __nv_bfloat16* __restrict__ B, int64_t ldb,
                                                             float* __restrict__ C, int64_t ldc, int64_t c_split) {
    __shared__ __align__(16) __nv_bfloat16 As[2][BM][SPITCH];
    __shared__ __align__(16) __nv_bfloat16 Bs[2][BN][SPITCH];
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int kb = blockIdx.z * kc, ke = min(K, kb + kc);
    C += blockIdx.z * c_split;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = (warp >> 2) * 64, wn = (warp & 3) * 32;
    const int g = lane >> 2, t = lane & 3;
    float acc[4][4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int r = 0; r < 4; r++) acc[i][j][r] = 0.f;
    const int nk = ke > kb ? (ke - kb + BK - 1) / BK : 0;
    if (nk > 0) {
        load_tile<AV>(As[0], A, lda, m0, M, kb, ke);
        load_tile<BV>(Bs[0], B, ldb, n0, N, kb, ke);
    }
    cp_async_commit();
    // lane -> row / k offset of the 8 x 8 matrices of one ldmatrix.x4
    const int a_row = lane & 15, a_k = (lane >> 4) << 3;
    const int b_row = (lane & 7) + ((lane >> 4) << 3), b_k = ((lane >> 3) & 1) << 3;
    for (int it = 0; it < nk; it++) {
        const int cur = it & 1;
        if (it + 1 < nk) {
            load_tile<AV>(As[cur ^ 1], A, lda, m0, M, kb + (it + 1) * BK, ke);
            load_tile<BV>(Bs[cur ^ 1], B, ldb, n0, N, kb + (it + 1) * BK, ke);
        }
        cp_async_commit();
        cp_async_wait1();  // the stage of this iteration has landed
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk += 16) {
            uint32_t a[4][4], b[4][2];
#pragma unroll
            for (int i = 0; i < 4; i++) ldmatrix_x4(a[i], &As[cur][wm + 16 * i + a_row][kk + a_k]);
#pragma unroll
            for (int jp = 0; jp < 2; jp++) {
                uint32_t r[4];
                ldmatrix_x4(r, &Bs[cur][wn + 16 * jp + b_row][kk + b_k]);
                b[2 * jp][0] = r[0];
                b[2 * jp][1] = r[1];
                b[2 * jp + 1][0] = r[2];
                b[2 * jp + 1][1] = r[3];
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++)
                    asm volatile(
                        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
                        "{%8,%9}, {%0,%1,%2,%3};\n"
                        : "+f"(acc[i][j][0]), "+f"(acc[i][j][1]), "+f"(acc[i][j][2]), "+f"(acc[i][j][3])
                        : "r"(a[i][0]), "r"(a[i][1]), "r"(a[i][2]), "r"(a[i][3]), "r"(b[j][0]), "r"(b[j][1]));
        }
        __syncthreads();  // the next iteration refills the other stage, then this one
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int64_t r = m0 + wm + 16 * i + g;
            const int c = n0 + wn + 8 * j + 2 * t;
            if (r < M && c < N) C[r * ldc + c] = acc[i][j][0];
            if (r < M && c + 1 < N) C[r * ldc + c + 1] = acc[i][j][1];
            if (r + 8 < M && c < N) C[(r + 8) * ldc + c] = acc[i][j][2];
            if (r + 8 < M && c + 1 < N) C[(r + 8) * ldc + c + 1] = acc[i][j][3];
        }
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

// K slice length of a split GEMM (a multiple of the K tile) and the number
// of slices
inline int split_len(int K, int splits) {
    int kc = (K + splits - 1) / splits;
    kc = (kc + BK - 1) / BK * BK;
    return kc > 0 ? kc : BK;
}
inline int split_count(int K, int kc) { return K > 0 ? (K + kc - 1) / kc : 1; }

inline bool vec_ok(const void* p, int64_t ld) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0 && ld % 8 == 0; }

// C = A . B^T with A [M][lda], B [N][ldb] (k contiguous); see gemm_tn_kernel
void gemm(int M, int N, int K, const __nv_bfloat16* A, int64_t lda, const __nv_bfloat16* B, int64_t ldb, float* C,
          int64_t ldc, cudaStream_t s, int splits = 1, int64_t c_split = 0) {
    if (M <= 0 || N <= 0) return;
    const int kc = split_len(K, splits);
    dim3 grid(blocks(N, BN), blocks(M, BM), split_count(K, kc));
    const bool av = vec_ok(A, lda), bv = vec_ok(B, ldb);
    if (av && bv)
        gemm_tn_kernel<true, true><<<grid, kGemmThreads, 0, s>>>(M, N, K, kc, A, lda, B, ldb, C, ldc, c_split);
    else if (av)
        gemm_tn_kernel<true, false><<<grid, kGemmThreads, 0, s>>>(M, N, K, kc, A, lda, B, ldb, C, ldc, c_split);
    else if (bv)
        gemm_tn_kernel<false, true><<<grid, kGemmThreads, 0, s>>>(M, N, K, kc, A, lda, B, ldb, C, ldc, c_split);
    else
        gemm_tn_kernel<false, false><<<grid, kGemmThreads, 0, s>>>(M, N, K, kc, A, lda, B, ldb, C, ldc, c_split);
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
        gemm(M, dO, di, n->h[l].as<__nv_bfloat16>(), di, wb + n->w_off[l], di, n->c.as<float>(), dO, s);
        const int64_t e = static_cast<int64_t>(M) * dO;
        const bool last = l == n->layers() - 1;
        bias_act_kernel<<<blocks(e, 256), 256, 0, s>>>(
            M, dO, n->c.as<float>(), n->w32.as<float>() + n->b_off[l], last ? nullptr : n->z[l].as<float>(),
            last ? nullptr : n->h[l + 1].as<__nv_bfloat16>(), last ? n->y.as<float>() : nullptr, last ? 0 : 1);
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
    const int kc = split_len(M, splits), S = split_count(M, kc);
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
    return GELIOS_OK;
}

extern "C" int gelios_mlp_gemm_bf16(int M, int N, int K, const void* A, int64_t lda, const void* B, int64_t ldb,
                                    float* C, int64_t ldc, void* stream) {
    if (M < 0 || N < 0 || K < 0 || !A || !B || !C || lda < K || ldb < K || ldc < N)
        return fail("gelios_mlp_gemm_bf16: bad arguments");
    gemm(M, N, K, static_cast<const __nv_bfloat16*>(A), lda, static_cast<const __nv_bfloat16*>(B), ldb, C, ldc,
         static_cast<cudaStream_t>(stream));
    MLP_TRY(cudaGetLastError());
    return GELIOS_OK;
}
