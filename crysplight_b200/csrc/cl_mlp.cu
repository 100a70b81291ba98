// cl_mlp.cu — the light-response surrogate: a 3 -> 256 -> 256 -> 256 -> 192 SiLU
// MLP trained and evaluated on sm_100a by hand-written kernels.
//
// GEMMs run on the 5th-generation tensor cores: BF16 operands staged in shared
// memory (canonical K-major layout, see cl_umma.cuh), one thread issuing
// tcgen05.mma with the FP32 accumulator in tensor memory, completion through
// tcgen05.commit on an mbarrier (bounded wait), and epilogues fused on the
// TMEM -> register path (bias, SiLU, SiLU', BF16 casts, transposed copies,
// split-K partials).  The 3-wide input layer, the loss, the reductions and
// Adam run on the CUDA cores.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/crysplight_cuda.h"
#include "cl_umma.cuh"

namespace cl {
namespace mlp {

using bf16 = __nv_bfloat16;

constexpr int TILE_M = 128;     // rows per CTA tile (TMEM lanes)
constexpr int TILE_K = 64;      // K elements staged per chunk
constexpr int GEMM_THREADS = 128;
constexpr uint32_t WAIT_BUDGET = 1u << 22;   // polls before a wait gives up
constexpr size_t GEMM_SMEM_BYTES = 100 * 1024;

enum Epi : int {
    EPI_F32 = 0,         // out_f[m][n] = acc
    EPI_BIAS_SILU = 1,   // z = acc + b: out_z = bf16(z), out_h = bf16(silu z), out_ht = transposed
    EPI_BIAS_F32 = 2,    // out_f[m][n] = acc + b
    EPI_DSILU = 3,       // d = acc * silu'(zprev): out_h = bf16(d), out_ht = transposed
    EPI_PARTIAL = 4,     // out_f[split][m][n] = acc (split-K partial)
};

struct GemmArgs {
    const bf16* A; int64_t lda;     // [M][K], K-major
    const bf16* B; int64_t ldb;     // [N][K], K-major
    int M, N, K;                    // M % 128 == 0, N % 32 == 0 && N <= 256, K % 64 == 0
    int k_split;                    // K elements per split (gridDim.y splits)
    const float* bias;
    float* out_f; int64_t ldf;
    bf16* out_h; int64_t ldh;       // [M][N]
    bf16* out_ht; int64_t ldht;     // [N][M]
    bf16* out_z;                    // [M][N], ld = ldh
    const bf16* zprev;              // [M][N], ld = ldh
    unsigned int* err;
};

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z)
{
    const float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// Stage rows [r0, r0+R) x K-chunk [k0, k0+64) of a K-major matrix into the
// canonical layout (16-byte pieces, 8 consecutive threads per row).
__device__ __forceinline__ void stage_tile(uint8_t* smem, const bf16* g, int64_t ld, int r0, int R,
                                           int k0)
{
    const int pieces = R * (TILE_K / 8);
    for (int p = threadIdx.x; p < pieces; p += blockDim.x) {
        const int r = p >> 3, c = p & 7;
        const uint4 v = *reinterpret_cast<const uint4*>(g + (int64_t)(r0 + r) * ld + k0 + 8 * c);
        *reinterpret_cast<uint4*>(smem + umma::tile_offset((uint32_t)r, (uint32_t)(8 * c), (uint32_t)R)) = v;
    }
}

template <int EPI>
__global__ void __launch_bounds__(GEMM_THREADS) gemm_kernel(const __grid_constant__ GemmArgs G)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* sA = smem;                                  // 128 x 64 bf16 = 16 KB
    uint8_t* sB = smem + TILE_M * TILE_K * 2;            // N x 64 bf16 <= 32 KB
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int N = G.N;
    if (warp == 0) umma::tmem_alloc(&tmem_slot, 256);
    if (threadIdx.x == 0) {
        umma::mbar_init(&mbar, 1);
        abort_flag = 0;
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    const uint32_t idesc = umma::make_idesc_bf16(TILE_M, N);
    const uint32_t lbo_a = (TILE_M / 8) * 128, lbo_b = (uint32_t)(N / 8) * 128;
    const uint32_t sa = umma::smem_u32(sA), sb = umma::smem_u32(sB);
    uint32_t phase = 0;

    const int k_begin = blockIdx.y * G.k_split;
    const int k_end = min(G.K, k_begin + G.k_split);
    const int n_tiles = G.M / TILE_M;
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int m0 = tile * TILE_M;
        for (int k0 = k_begin; k0 < k_end; k0 += TILE_K) {
            stage_tile(sA, G.A, G.lda, m0, TILE_M, k0);
            stage_tile(sB, G.B, G.ldb, 0, N, k0);
            umma::fence_async_smem();
            __syncthreads();
            if (threadIdx.x == 0) {
                umma::fence_after_sync();
#pragma unroll
                for (int s = 0; s < TILE_K / 16; ++s) {
                    const uint64_t ad = umma::make_desc(sa + 2 * s * lbo_a, lbo_a, 128);
                    const uint64_t bd = umma::make_desc(sb + 2 * s * lbo_b, lbo_b, 128);
                    umma::mma_bf16(tmem, ad, bd, idesc, (k0 > k_begin || s > 0) ? 1u : 0u);
                }
                umma::commit(&mbar);
            }
            if (!umma::mbar_wait(&mbar, phase, WAIT_BUDGET)) {
                atomicOr(G.err, 1u);
                abort_flag = 1;
            }
            phase ^= 1u;
            __syncthreads();
            if (abort_flag) break;
        }
        if (abort_flag) break;

        // ---- epilogue: warp w owns rows m0 + 32w + lane ----
        umma::fence_after_sync();
        const int row = m0 + 32 * warp + lane;
        for (int c0 = 0; c0 < N; c0 += 32) {
            float v[32];
            umma::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
            if (EPI == EPI_F32 || EPI == EPI_BIAS_F32 || EPI == EPI_PARTIAL) {
                float* o = G.out_f + (EPI == EPI_PARTIAL ? (int64_t)blockIdx.y * G.M * G.ldf : 0) +
                           (int64_t)row * G.ldf + c0;
#pragma unroll
                for (int i = 0; i < 32; i += 4) {
                    float4 q;
                    q.x = v[i] + (EPI == EPI_BIAS_F32 ? G.bias[c0 + i] : 0.0f);
                    q.y = v[i + 1] + (EPI == EPI_BIAS_F32 ? G.bias[c0 + i + 1] : 0.0f);
                    q.z = v[i + 2] + (EPI == EPI_BIAS_F32 ? G.bias[c0 + i + 2] : 0.0f);
                    q.w = v[i + 3] + (EPI == EPI_BIAS_F32 ? G.bias[c0 + i + 3] : 0.0f);
                    *reinterpret_cast<float4*>(o + i) = q;
                }
            } else {
                __align__(16) bf16 h[32];
                __align__(16) bf16 zz[32];
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    float r;
                    if (EPI == EPI_BIAS_SILU) {
                        const float z = v[i] + G.bias[c0 + i];
                        zz[i] = __float2bfloat16_rn(z);
                        r = silu(z);
                    } else {   // EPI_DSILU
                        const float zp = __bfloat162float(G.zprev[(int64_t)row * G.ldh + c0 + i]);
                        r = v[i] * dsilu(zp);
                    }
                    h[i] = __float2bfloat16_rn(r);
                    if (G.out_ht) G.out_ht[(int64_t)(c0 + i) * G.ldht + row] = h[i];
                }
                uint4* dst = reinterpret_cast<uint4*>(G.out_h + (int64_t)row * G.ldh + c0);
#pragma unroll
                for (int i = 0; i < 4; ++i) dst[i] = reinterpret_cast<const uint4*>(h)[i];
                if (EPI == EPI_BIAS_SILU && G.out_z) {
                    uint4* dz = reinterpret_cast<uint4*>(G.out_z + (int64_t)row * G.ldh + c0);
#pragma unroll
                    for (int i = 0; i < 4; ++i) dz[i] = reinterpret_cast<const uint4*>(zz)[i];
                }
            }
        }
        umma::fence_before_sync();
        __syncthreads();          // TMEM reads done before the next tile overwrites it
    }
    if (abort_flag) {
        // give in-flight MMAs one more bounded chance to land before freeing TMEM
        umma::mbar_wait(&mbar, phase, WAIT_BUDGET);
    }
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem, 256);
}

// ---- host launch helper ----
template <int EPI>
int launch_gemm(const GemmArgs& g, int grid_x, int splits, cudaStream_t st)
{
    if (g.M % TILE_M || g.N % 32 || g.N > 256 || g.N < 32 || g.K % TILE_K || splits < 1)
        return CL_ERR_ARG;
    // The request is padded to 100 KB so that at most two CTAs share an SM:
    // each holds 256 of the SM's 512 TMEM columns.
    const size_t need = (size_t)TILE_M * TILE_K * 2 + (size_t)g.N * TILE_K * 2;
    const size_t smem = need > GEMM_SMEM_BYTES ? need : GEMM_SMEM_BYTES;
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(gemm_kernel<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)GEMM_SMEM_BYTES);
        attr_set = true;
    }
    dim3 grid((unsigned)grid_x, (unsigned)splits);
    gemm_kernel<EPI><<<grid, GEMM_THREADS, smem, st>>>(g);
    return cudaGetLastError() == cudaSuccess ? CL_OK : CL_ERR_CUDA;
}


// ===========================================================================
// The MLP: 3 -> 256 -> 256 -> 256 -> 192, SiLU, BF16 weights/activations,
// FP32 accumulation and FP32 master weights with Adam.
// ===========================================================================
constexpr int D_IN = 3, D_H = 256, D_OUT = 192;
constexpr int WGRAD_SPLIT_K = 1024;      // batch rows per weight-gradient split

__device__ __forceinline__ uint32_t hash32(uint32_t a, uint32_t b, uint32_t c)
{
    // Philox4x32-10 with key (c, 0x5eed) on counter (a, b, 0, 0): first word
    uint32_t c0 = a, c1 = b, c2 = 0, c3 = 0, k0 = c, k1 = 0x5eedu;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c1 = (uint32_t)p1; c3 = (uint32_t)p0; c0 = n0; c2 = n2;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    return c0;
}

// Random minibatch (with replacement) from the training set.
__global__ void gather_batch(const float* __restrict__ X, const float* __restrict__ T, int64_t n_all,
                             int B, uint32_t seed, uint32_t step, float* Xb, float* Tb)
{
    const int b = blockIdx.x;
    if (b >= B) return;
    const int64_t i = (int64_t)(hash32((uint32_t)b, step, seed) % (uint32_t)n_all);
    if (threadIdx.x < D_IN) Xb[(int64_t)b * D_IN + threadIdx.x] = X[i * D_IN + threadIdx.x];
    for (int j = threadIdx.x; j < D_OUT; j += blockDim.x) Tb[(int64_t)b * D_OUT + j] = T[i * D_OUT + j];
}

// Layer 1 (K = 3) on the CUDA cores: z = x W1^T + b1, h = silu(z).
__global__ void layer1_fwd(const float* __restrict__ X, const float* __restrict__ W1, const float* __restrict__ b1,
                           int B, bf16* H, bf16* Ht, bf16* Z)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)B * D_H) return;
    const int b = (int)(idx / D_H), j = (int)(idx % D_H);
    const float* x = X + (int64_t)b * D_IN;
    const float z = b1[j] + x[0] * W1[j * D_IN] + x[1] * W1[j * D_IN + 1] + x[2] * W1[j * D_IN + 2];
    const bf16 h = __float2bfloat16_rn(silu(z));
    H[idx] = h;
    if (Z) Z[idx] = __float2bfloat16_rn(z);
    if (Ht) Ht[(int64_t)j * B + b] = h;
}

// Loss 1/(B*192) sum (o - t)^2 and its gradient dO (BF16, row and transposed).
__global__ void loss_grad(const float* __restrict__ O, const float* __restrict__ Tb, int B, float scale,
                          bf16* dO, bf16* dOt, float* loss_acc)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float sq = 0.0f;
    if (idx < (int64_t)B * D_OUT) {
        const int b = (int)(idx / D_OUT), j = (int)(idx % D_OUT);
        const float d = O[idx] - Tb[idx];
        sq = d * d;
        const bf16 g = __float2bfloat16_rn(2.0f * d * scale);
        dO[idx] = g;
        dOt[(int64_t)j * B + b] = g;
    }
    if (loss_acc) {
        for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
        if ((threadIdx.x & 31) == 0 && sq != 0.0f) atomicAdd(loss_acc, sq * scale);
    }
}

// grad_Wt[o][i] = sum_s P[s][i][o]   (P: split-K partials of dW = H^T dZ, [IN][OUT])
__global__ void reduce_wgrad(const float* __restrict__ P, int S, int IN, int OUT, float* gWt)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= IN * OUT) return;
    const int i = idx / OUT, o = idx % OUT;
    float acc = 0.0f;
    for (int s = 0; s < S; ++s) acc += P[((int64_t)s * IN + i) * OUT + o];
    gWt[(int64_t)o * IN + i] = acc;
}

// Row sums of a [R][B] BF16 matrix (bias gradients from transposed gradients);
// with X, also the layer-1 weight gradients g1[r][k] = sum_b G[r][b] X[b][k].
__global__ void row_sums(const bf16* __restrict__ G, int B, float* gb, const float* __restrict__ X, float* g1)
{
    const int r = blockIdx.x;
    float s = 0.0f, w0 = 0.0f, w1 = 0.0f, w2 = 0.0f;
    for (int b = threadIdx.x; b < B; b += blockDim.x) {
        const float g = __bfloat162float(G[(int64_t)r * B + b]);
        s += g;
        if (X) { w0 += g * X[(int64_t)b * 3]; w1 += g * X[(int64_t)b * 3 + 1]; w2 += g * X[(int64_t)b * 3 + 2]; }
    }
    __shared__ float red[4][32];
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        w0 += __shfl_xor_sync(0xffffffffu, w0, o);
        w1 += __shfl_xor_sync(0xffffffffu, w1, o);
        w2 += __shfl_xor_sync(0xffffffffu, w2, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { red[0][w] = s; red[1][w] = w0; red[2][w] = w1; red[3][w] = w2; }
    __syncthreads();
    if (threadIdx.x == 0) {
        float a[4] = {0, 0, 0, 0};
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i)
            for (int q = 0; q < 4; ++q) a[q] += red[q][i];
        gb[r] = a[0];
        if (X) { g1[r * 3] = a[1]; g1[r * 3 + 1] = a[2]; g1[r * 3 + 2] = a[3]; }
    }
}

// Adam on an FP32 master tensor; optional BF16 copies of a [OUT][IN] matrix
// in both layouts ([OUT][IN] for the forward B operand, [IN][OUT] for the
// backward-data B operand).
__global__ void adam_step(float* w, const float* g, float* m, float* v, int n, float lr, float b1,
                          float b2, float eps, float bc1, float bc2, int OUT, int IN, bf16* wt_bf,
                          bf16* w_bf)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi; v[i] = vi;
    const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    w[i] = wi;
    if (wt_bf) {
        const int o = i / IN, k = i % IN;
        const bf16 q = __float2bfloat16_rn(wi);
        wt_bf[i] = q;
        w_bf[(int64_t)k * OUT + o] = q;
    }
}

__global__ void to_bf16_pair(const float* w, int OUT, int IN, bf16* wt_bf, bf16* w_bf)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= OUT * IN) return;
    const int o = i / IN, k = i % IN;
    const bf16 q = __float2bfloat16_rn(w[i]);
    wt_bf[i] = q;
    w_bf[(int64_t)k * OUT + o] = q;
}

}  // namespace mlp
}  // namespace cl

using namespace cl::mlp;

// Parameter block layout (FP32, contiguous): W1[256][3] b1[256] W2t[256][256]
// b2[256] W3t[256][256] b3[256] W4t[192][256] b4[192].
namespace {
constexpr int64_t OFF_W1 = 0, OFF_B1 = OFF_W1 + D_H * D_IN, OFF_W2 = OFF_B1 + D_H,
                  OFF_B2 = OFF_W2 + D_H * D_H, OFF_W3 = OFF_B2 + D_H, OFF_B3 = OFF_W3 + D_H * D_H,
                  OFF_W4 = OFF_B3 + D_H, OFF_B4 = OFF_W4 + D_OUT * D_H, N_PARAMS = OFF_B4 + D_OUT;
}

struct cl_mlp {
    int device = 0;
    int max_batch = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    char err[256] = {0};
    // FP32 master parameters, gradients, Adam moments
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    int64_t adam_t = 0;
    // BF16 weight copies
    bf16 *w2t = nullptr, *w2 = nullptr, *w3t = nullptr, *w3 = nullptr, *w4t = nullptr, *w4 = nullptr;
    // activations and gradients (max_batch rows)
    float *xb = nullptr, *tb = nullptr, *o = nullptr;
    bf16 *h1 = nullptr, *h1t = nullptr, *z1 = nullptr, *h2 = nullptr, *h2t = nullptr, *z2 = nullptr;
    bf16 *h3 = nullptr, *h3t = nullptr, *z3 = nullptr;
    bf16 *dO = nullptr, *dOt = nullptr, *dz3 = nullptr, *dz3t = nullptr, *dz2 = nullptr, *dz2t = nullptr;
    bf16 *dz1 = nullptr, *dz1t = nullptr;
    float* part = nullptr;          // split-K partials
    float* loss = nullptr;          // device accumulator
    unsigned int* derr = nullptr;
    // training set (device pointers owned by the caller)
    const float* data_x = nullptr;
    const float* data_t = nullptr;
    int64_t n_data = 0;
    std::vector<void*> allocs;
};

namespace {

int mlp_fail(cl_mlp* m, int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(m->err, sizeof m->err, fmt, ap);
    va_end(ap);
    return code;
}

template <typename T>
bool dalloc(cl_mlp* m, T** p, size_t count)
{
    void* q = nullptr;
    if (cudaMalloc(&q, count * sizeof(T)) != cudaSuccess) { cudaGetLastError(); return false; }
    m->allocs.push_back(q);
    *p = (T*)q;
    return true;
}

void refresh_bf16(cl_mlp* m, cudaStream_t st)
{
    to_bf16_pair<<<(D_H * D_H + 255) / 256, 256, 0, st>>>(m->p + OFF_W2, D_H, D_H, m->w2t, m->w2);
    to_bf16_pair<<<(D_H * D_H + 255) / 256, 256, 0, st>>>(m->p + OFF_W3, D_H, D_H, m->w3t, m->w3);
    to_bf16_pair<<<(D_OUT * D_H + 255) / 256, 256, 0, st>>>(m->p + OFF_W4, D_OUT, D_H, m->w4t, m->w4);
}

// Forward pass over B rows of m->xb (B % 128 == 0): activations and O.
int forward(cl_mlp* m, int B, bool keep_t, cudaStream_t st)
{
    const int tiles = B / TILE_M;
    const int grid = tiles < 2 * m->num_sms ? tiles : 2 * m->num_sms;
    layer1_fwd<<<(unsigned)(((int64_t)B * D_H + 255) / 256), 256, 0, st>>>(
        m->xb, m->p + OFF_W1, m->p + OFF_B1, B, m->h1, keep_t ? m->h1t : nullptr, m->z1);
    GemmArgs g;
    memset(&g, 0, sizeof g);
    g.err = m->derr;
    g.M = B; g.K = D_H; g.k_split = D_H;
    // layer 2
    g.A = m->h1; g.lda = D_H; g.B = m->w2t; g.ldb = D_H; g.N = D_H;
    g.bias = m->p + OFF_B2; g.out_h = m->h2; g.ldh = D_H; g.out_ht = keep_t ? m->h2t : nullptr; g.ldht = B;
    g.out_z = m->z2;
    int rc = launch_gemm<EPI_BIAS_SILU>(g, grid, 1, st);
    if (rc) return rc;
    // layer 3
    g.A = m->h2; g.B = m->w3t; g.bias = m->p + OFF_B3; g.out_h = m->h3;
    g.out_ht = keep_t ? m->h3t : nullptr; g.out_z = m->z3;
    if ((rc = launch_gemm<EPI_BIAS_SILU>(g, grid, 1, st))) return rc;
    // layer 4 (linear)
    GemmArgs q;
    memset(&q, 0, sizeof q);
    q.err = m->derr;
    q.M = B; q.K = D_H; q.k_split = D_H; q.N = D_OUT;
    q.A = m->h3; q.lda = D_H; q.B = m->w4t; q.ldb = D_H;
    q.bias = m->p + OFF_B4; q.out_f = m->o; q.ldf = D_OUT;
    return launch_gemm<EPI_BIAS_F32>(q, grid, 1, st);
}

// Backward pass for the batch in m->xb / m->tb (forward already run with
// keep_t): gradients into m->g.
int backward(cl_mlp* m, int B, cudaStream_t st)
{
    const int tiles = B / TILE_M;
    const int grid = tiles < 2 * m->num_sms ? tiles : 2 * m->num_sms;
    const float scale = 1.0f / ((float)B * (float)D_OUT);
    loss_grad<<<(unsigned)(((int64_t)B * D_OUT + 255) / 256), 256, 0, st>>>(m->o, m->tb, B, scale, m->dO,
                                                                             m->dOt, m->loss);
    // backward data: dZ3 = (dO W4) * silu'(Z3), dZ2 = (dZ3 W3) * silu'(Z2), dZ1 = (dZ2 W2) * silu'(Z1)
    GemmArgs g;
    memset(&g, 0, sizeof g);
    g.err = m->derr;
    g.M = B; g.N = D_H;
    g.A = m->dO; g.lda = D_OUT; g.K = D_OUT; g.k_split = D_OUT;
    g.B = m->w4; g.ldb = D_OUT;
    g.out_h = m->dz3; g.ldh = D_H; g.out_ht = m->dz3t; g.ldht = B; g.zprev = m->z3;
    int rc = launch_gemm<EPI_DSILU>(g, grid, 1, st);
    if (rc) return rc;
    g.A = m->dz3; g.lda = D_H; g.K = D_H; g.k_split = D_H;
    g.B = m->w3; g.ldb = D_H;
    g.out_h = m->dz2; g.out_ht = m->dz2t; g.zprev = m->z2;
    if ((rc = launch_gemm<EPI_DSILU>(g, grid, 1, st))) return rc;
    g.A = m->dz2; g.B = m->w2;
    g.out_h = m->dz1; g.out_ht = m->dz1t; g.zprev = m->z1;
    if ((rc = launch_gemm<EPI_DSILU>(g, grid, 1, st))) return rc;
    // weight gradients dW = H^T dZ (split-K over the batch) -> grad W^T
    const int splits = (B + WGRAD_SPLIT_K - 1) / WGRAD_SPLIT_K;
    struct WG { const bf16* ht; const bf16* dzt; int OUT; int64_t off_w; int64_t off_b; };
    const WG wg[3] = {{m->h3t, m->dOt, D_OUT, OFF_W4, OFF_B4},
                      {m->h2t, m->dz3t, D_H, OFF_W3, OFF_B3},
                      {m->h1t, m->dz2t, D_H, OFF_W2, OFF_B2}};
    for (int l = 0; l < 3; ++l) {
        GemmArgs w;
        memset(&w, 0, sizeof w);
        w.err = m->derr;
        w.A = wg[l].ht; w.lda = B; w.M = D_H;
        w.B = wg[l].dzt; w.ldb = B; w.N = wg[l].OUT;
        w.K = B; w.k_split = WGRAD_SPLIT_K;
        w.out_f = m->part; w.ldf = wg[l].OUT;
        if ((rc = launch_gemm<EPI_PARTIAL>(w, D_H / TILE_M, splits, st))) return rc;
        reduce_wgrad<<<(D_H * wg[l].OUT + 255) / 256, 256, 0, st>>>(m->part, splits, D_H, wg[l].OUT,
                                                                    m->g + wg[l].off_w);
        row_sums<<<wg[l].OUT, 256, 0, st>>>(wg[l].dzt, B, m->g + wg[l].off_b, nullptr, nullptr);
    }
    // layer 1: bias and weight gradients from dZ1^T and X
    row_sums<<<D_H, 256, 0, st>>>(m->dz1t, B, m->g + OFF_B1, m->xb, m->g + OFF_W1);
    return cudaGetLastError() == cudaSuccess ? CL_OK : CL_ERR_CUDA;
}

void adam(cl_mlp* m, float lr, cudaStream_t st)
{
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    m->adam_t += 1;
    const float bc1 = 1.0f - powf(b1, (float)m->adam_t), bc2 = 1.0f - powf(b2, (float)m->adam_t);
    struct T { int64_t off; int n; int OUT; int IN; bf16* wt; bf16* w; };
    const T ts[8] = {{OFF_W1, D_H * D_IN, 0, 0, nullptr, nullptr},
                     {OFF_B1, D_H, 0, 0, nullptr, nullptr},
                     {OFF_W2, D_H * D_H, D_H, D_H, m->w2t, m->w2},
                     {OFF_B2, D_H, 0, 0, nullptr, nullptr},
                     {OFF_W3, D_H * D_H, D_H, D_H, m->w3t, m->w3},
                     {OFF_B3, D_H, 0, 0, nullptr, nullptr},
                     {OFF_W4, D_OUT * D_H, D_OUT, D_H, m->w4t, m->w4},
                     {OFF_B4, D_OUT, 0, 0, nullptr, nullptr}};
    for (const T& t : ts)
        adam_step<<<(t.n + 255) / 256, 256, 0, st>>>(m->p + t.off, m->g + t.off, m->m + t.off, m->v + t.off,
                                                     t.n, lr, b1, b2, eps, bc1, bc2, t.OUT, t.IN, t.wt, t.w);
}

}  // namespace

extern "C" {

int cl_mlp_param_count(void) { return (int)N_PARAMS; }

int cl_mlp_create(cl_mlp** out, int device, int max_batch)
{
    if (!out || max_batch < TILE_M || max_batch % TILE_M) return CL_ERR_ARG;
    *out = nullptr;
    cl_mlp* m = new (std::nothrow) cl_mlp();
    if (!m) return CL_ERR_OOM;
    m->device = device;
    m->max_batch = max_batch;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaDeviceGetAttribute(&m->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete m;
        return CL_ERR_CUDA;
    }
    const size_t B = (size_t)max_batch;
    const int splits = (max_batch + WGRAD_SPLIT_K - 1) / WGRAD_SPLIT_K;
    bool ok = dalloc(m, &m->p, N_PARAMS) && dalloc(m, &m->g, N_PARAMS) && dalloc(m, &m->m, N_PARAMS) &&
              dalloc(m, &m->v, N_PARAMS) &&
              dalloc(m, &m->w2t, (size_t)D_H * D_H) && dalloc(m, &m->w2, (size_t)D_H * D_H) &&
              dalloc(m, &m->w3t, (size_t)D_H * D_H) && dalloc(m, &m->w3, (size_t)D_H * D_H) &&
              dalloc(m, &m->w4t, (size_t)D_OUT * D_H) && dalloc(m, &m->w4, (size_t)D_OUT * D_H) &&
              dalloc(m, &m->xb, B * D_IN) && dalloc(m, &m->tb, B * D_OUT) && dalloc(m, &m->o, B * D_OUT) &&
              dalloc(m, &m->h1, B * D_H) && dalloc(m, &m->h1t, B * D_H) && dalloc(m, &m->z1, B * D_H) &&
              dalloc(m, &m->h2, B * D_H) && dalloc(m, &m->h2t, B * D_H) && dalloc(m, &m->z2, B * D_H) &&
              dalloc(m, &m->h3, B * D_H) && dalloc(m, &m->h3t, B * D_H) && dalloc(m, &m->z3, B * D_H) &&
              dalloc(m, &m->dO, B * D_OUT) && dalloc(m, &m->dOt, B * D_OUT) &&
              dalloc(m, &m->dz3, B * D_H) && dalloc(m, &m->dz3t, B * D_H) &&
              dalloc(m, &m->dz2, B * D_H) && dalloc(m, &m->dz2t, B * D_H) &&
              dalloc(m, &m->dz1, B * D_H) && dalloc(m, &m->dz1t, B * D_H) &&
              dalloc(m, &m->part, (size_t)splits * D_H * D_H) && dalloc(m, &m->loss, 1) &&
              dalloc(m, &m->derr, 1);
    if (!ok) {
        for (void* q : m->allocs) cudaFree(q);
        delete m;
        return CL_ERR_OOM;
    }
    cudaMemsetAsync(m->m, 0, N_PARAMS * sizeof(float), m->stream);
    cudaMemsetAsync(m->v, 0, N_PARAMS * sizeof(float), m->stream);
    cudaMemsetAsync(m->g, 0, N_PARAMS * sizeof(float), m->stream);
    cudaMemsetAsync(m->derr, 0, sizeof(unsigned int), m->stream);
    cudaMemsetAsync(m->p, 0, N_PARAMS * sizeof(float), m->stream);
    refresh_bf16(m, m->stream);
    cudaStreamSynchronize(m->stream);
    *out = m;
    return CL_OK;
}

void cl_mlp_destroy(cl_mlp* m)
{
    if (!m) return;
    cudaSetDevice(m->device);
    cudaStreamSynchronize(m->stream);
    for (void* q : m->allocs) cudaFree(q);
    cudaStreamDestroy(m->stream);
    delete m;
}

const char* cl_mlp_last_error(const cl_mlp* m) { return m ? m->err : ""; }

// Parameters in the FP32 block layout above (host buffers of cl_mlp_param_count()).
// Setting parameters resets the Adam state.
int cl_mlp_set_params(cl_mlp* m, const float* host)
{
    if (!m || !host) return CL_ERR_ARG;
    cudaSetDevice(m->device);
    cudaMemcpyAsync(m->p, host, N_PARAMS * sizeof(float), cudaMemcpyHostToDevice, m->stream);
    cudaMemsetAsync(m->m, 0, N_PARAMS * sizeof(float), m->stream);
    cudaMemsetAsync(m->v, 0, N_PARAMS * sizeof(float), m->stream);
    m->adam_t = 0;
    refresh_bf16(m, m->stream);
    return cudaStreamSynchronize(m->stream) == cudaSuccess ? CL_OK : CL_ERR_CUDA;
}

int cl_mlp_get_params(cl_mlp* m, float* host)
{
    if (!m || !host) return CL_ERR_ARG;
    cudaSetDevice(m->device);
    cudaMemcpyAsync(host, m->p, N_PARAMS * sizeof(float), cudaMemcpyDeviceToHost, m->stream);
    return cudaStreamSynchronize(m->stream) == cudaSuccess ? CL_OK : CL_ERR_CUDA;
}

// Training set: n rows of inputs x [n][3] and targets t [n][192], FP32 device
// arrays that stay owned by the caller and must outlive the training calls.
int cl_mlp_set_data(cl_mlp* m, const float* d_x, const float* d_t, int64_t n)
{
    if (!m || !d_x || !d_t || n < 1 || n > 0x7fffffff) return CL_ERR_ARG;
    m->data_x = d_x; m->data_t = d_t; m->n_data = n;
    return CL_OK;
}

// `steps` Adam steps on random minibatches of `batch` rows (batch % 128 == 0,
// batch <= max_batch); *loss_out = mean loss over the steps.
int cl_mlp_train(cl_mlp* m, int steps, int batch, float lr, uint32_t seed, uint32_t step0, float* loss_out)
{
    if (!m || steps < 0 || batch < TILE_M || batch % TILE_M || batch > m->max_batch || !m->data_x)
        return CL_ERR_ARG;
    cudaSetDevice(m->device);
    cudaStream_t st = m->stream;
    cudaMemsetAsync(m->loss, 0, sizeof(float), st);
    for (int s = 0; s < steps; ++s) {
        gather_batch<<<batch, 64, 0, st>>>(m->data_x, m->data_t, m->n_data, batch, seed, step0 + (uint32_t)s,
                                          m->xb, m->tb);
        int rc = forward(m, batch, true, st);
        if (!rc) rc = backward(m, batch, st);
        if (rc) return mlp_fail(m, rc, "kernel launch failed: %s", cudaGetErrorString(cudaGetLastError()));
        adam(m, lr, st);
    }
    float loss = 0.0f;
    unsigned int e = 0;
    cudaMemcpyAsync(&loss, m->loss, sizeof loss, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&e, m->derr, sizeof e, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return mlp_fail(m, CL_ERR_CUDA, "%s", cudaGetErrorString(cudaGetLastError()));
    if (e) return mlp_fail(m, CL_ERR_TIMEOUT, "tensor-core completion wait ran out");
    if (loss_out) *loss_out = steps > 0 ? loss / (float)steps : 0.0f;
    return CL_OK;
}

// Inference: out[n][192] (FP32, device) for x[n][3] (FP32, device).
int cl_mlp_forward(cl_mlp* m, const float* d_x, float* d_out, int64_t n)
{
    if (!m || !d_x || !d_out || n < 0) return CL_ERR_ARG;
    cudaSetDevice(m->device);
    cudaStream_t st = m->stream;
    for (int64_t r0 = 0; r0 < n; r0 += m->max_batch) {
        const int rows = (int)((n - r0) < m->max_batch ? (n - r0) : m->max_batch);
        const int B = ((rows + TILE_M - 1) / TILE_M) * TILE_M;
        cudaMemsetAsync(m->xb, 0, (size_t)B * D_IN * sizeof(float), st);
        cudaMemcpyAsync(m->xb, d_x + r0 * D_IN, (size_t)rows * D_IN * sizeof(float), cudaMemcpyDeviceToDevice, st);
        int rc = forward(m, B, false, st);
        if (rc) return mlp_fail(m, rc, "forward launch failed");
        cudaMemcpyAsync(d_out + r0 * D_OUT, m->o, (size_t)rows * D_OUT * sizeof(float), cudaMemcpyDeviceToDevice, st);
    }
    unsigned int e = 0;
    cudaMemcpyAsync(&e, m->derr, sizeof e, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return mlp_fail(m, CL_ERR_CUDA, "%s", cudaGetErrorString(cudaGetLastError()));
    return e ? mlp_fail(m, CL_ERR_TIMEOUT, "tensor-core completion wait ran out") : CL_OK;
}

// Gradient of the loss for one given batch (x [B][3], t [B][192] FP32 device;
// B % 128 == 0): host grad[cl_mlp_param_count()] and the loss.  For tests.
int cl_mlp_gradient(cl_mlp* m, const float* d_x, const float* d_t, int B, float* host_grad, float* loss_out)
{
    if (!m || !d_x || !d_t || !host_grad || B < TILE_M || B % TILE_M || B > m->max_batch) return CL_ERR_ARG;
    cudaSetDevice(m->device);
    cudaStream_t st = m->stream;
    cudaMemcpyAsync(m->xb, d_x, (size_t)B * D_IN * sizeof(float), cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(m->tb, d_t, (size_t)B * D_OUT * sizeof(float), cudaMemcpyDeviceToDevice, st);
    cudaMemsetAsync(m->loss, 0, sizeof(float), st);
    int rc = forward(m, B, true, st);
    if (!rc) rc = backward(m, B, st);
    if (rc) return mlp_fail(m, rc, "launch failed");
    float loss = 0.0f;
    cudaMemcpyAsync(host_grad, m->g, N_PARAMS * sizeof(float), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&loss, m->loss, sizeof loss, cudaMemcpyDeviceToHost, st);
    unsigned int e = 0;
    cudaMemcpyAsync(&e, m->derr, sizeof e, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return mlp_fail(m, CL_ERR_CUDA, "%s", cudaGetErrorString(cudaGetLastError()));
    if (loss_out) *loss_out = loss;
    return e ? mlp_fail(m, CL_ERR_TIMEOUT, "tensor-core completion wait ran out") : CL_OK;
}

}  // extern "C"


extern "C" {

// Diagnostic: C[M][N] (fp32) = A[M][K] * B[N][K]^T with BF16 device operands,
// on the tensor cores (grid_x CTAs in x, `splits` K splits written as partials
// C[split][M][N] when splits > 1).  Returns CL_ERR_TIMEOUT if an mbarrier wait
// ran out.
int cl_umma_gemm_bf16(const void* A, const void* B, float* C, int M, int N, int K, int grid_x,
                      int splits, unsigned int* d_err, void* stream)
{
    if (!A || !B || !C || !d_err || M <= 0 || N <= 0 || K <= 0 || grid_x <= 0) return CL_ERR_ARG;
    GemmArgs g;
    memset(&g, 0, sizeof g);
    g.A = (const bf16*)A; g.lda = K;
    g.B = (const bf16*)B; g.ldb = K;
    g.M = M; g.N = N; g.K = K;
    g.out_f = C; g.ldf = N;
    g.err = d_err;
    if (splits > 1) {
        g.k_split = ((K / splits + TILE_K - 1) / TILE_K) * TILE_K;
        return launch_gemm<EPI_PARTIAL>(g, grid_x, splits, (cudaStream_t)stream);
    }
    g.k_split = K;
    return launch_gemm<EPI_F32>(g, grid_x, 1, (cudaStream_t)stream);
}

}  // extern "C"
