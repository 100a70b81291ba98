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

}  // namespace mlp
}  // namespace cl

using namespace cl::mlp;

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
