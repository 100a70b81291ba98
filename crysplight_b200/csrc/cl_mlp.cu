// cl_mlp.cu — the light-response surrogate: a 3 -> 256 -> 256 -> 256 -> 192 SiLU
// MLP trained and evaluated on sm_100a by hand-written kernels.
//
// GEMMs run on the 5th-generation tensor cores: BF16 operands streamed by TMA
// into a 3- or 4-stage shared-memory ring (128-byte swizzled tiles, K-major,
// or MN-major for the weight gradients, which read the activations and
// gradients as stored), one thread issuing tcgen05.mma into a double-buffered
// FP32 accumulator in tensor memory, and sixteen warps draining it through
// fused epilogues (bias, SiLU, SiLU', the loss and its gradient, bias-gradient
// column sums, the layer-1 gradients, BF16 casts, weight-gradient splits
// added in place).  The 3-wide input layer and Adam run on the CUDA cores.
// The epilogues are element-wise work over the 128 x N accumulator of every
// tile; they are spread over sixteen warps (four per TMEM lane quadrant, each
// taking every fourth 32-column chunk) so that draining a tile keeps pace
// with the tensor cores filling the other accumulator.  Their BF16 outputs
// are staged in shared memory as 32 x 32 tiles and written by TMA stores:
// stored straight from registers, each 16-byte store of a warp touched 32
// rows, and the store queue, not the arithmetic, set the pace.  Column sums
// go through a transposed staging tile into per-CTA shared accumulators (one
// global atomic per column and CTA).  The per-column constants the epilogues
// read (biases, the layer-1 weights) are staged in shared memory once per CTA.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include <atomic>
#include <mutex>

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/crysplight_cuda.h"
#include "cl_umma.cuh"

namespace cl {
namespace mlp {

using bf16 = __nv_bfloat16;

// Programmatic dependent launch: the kernels of a training step are launched
// so that the next one may be scheduled while the previous one drains; each
// kernel allows that at its start (pdl_trigger) and waits for the previous
// kernel's completion and memory (pdl_wait) before its first global access.
// Without the launch attribute both are no-ops.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Launches kernel k with the programmatic-serialization attribute on stream st.
template <typename... P, typename... A>
cudaError_t launch_pdl(void (*k)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, static_cast<P>(args)...);
}

constexpr int TILE_M = 128;     // rows per CTA tile (TMEM lanes)
constexpr int TILE_K = 64;      // K elements per pipeline stage (one 128-byte swizzle row)
#ifndef CL_MLP_EPI_WARPS
#define CL_MLP_EPI_WARPS 16
#endif
constexpr int EPI_WARPS = CL_MLP_EPI_WARPS;   // epilogue warps: warp w drains TMEM lane quadrant w % 4,
                                             // 32-column chunks c with c % (EPI_WARPS/4) == w / 4
constexpr int PRODUCER_WARP = EPI_WARPS;        // TMA producer
constexpr int MMA_WARP = EPI_WARPS + 1;         // MMA issuer / TMEM owner
constexpr int GEMM_THREADS = 32 * (EPI_WARPS + 2);
constexpr uint32_t TMEM_COLS = 512; // two 256-column FP32 accumulators
constexpr uint32_t WAIT_BUDGET = 1u << 22;   // polls before a wait gives up

enum Epi : int {
    EPI_F32 = 0,         // out_f[m][n] = acc
    EPI_BIAS_SILU = 1,   // z = acc + b: out_z = bf16(z), out_h = bf16(silu z)
    EPI_BIAS_F32 = 2,    // out_f[m][n] = acc + b
    EPI_DSILU = 3,       // g = bf16(acc * silu'(zprev)): out_h, colsum += column sums of g
    EPI_PARTIAL = 4,     // out_f[split][m][n] = acc (split-K partial)
    EPI_LOSS = 5,        // o = acc + b, d = o - target: loss += scale d^2, g = bf16(2 scale d) -> out_h, colsum
    EPI_DSILU_L1 = 6,    // as EPI_DSILU with zprev recomputed from x, W1, b1; colsum and gw1 += g, g x
    EPI_WGRAD = 7,       // out_f[n][m] += acc (a K split of a weight gradient, added in place, transposed);
                         // A [K][M] and B [K][N] MN-major (the activations and gradients as stored)
};

// Per epilogue: the BF16 tiles each epilogue warp stages in shared memory per
// 32 x 32 chunk (2 KB each, written out by TMA stores; the transposed tile
// also feeds the column sums), the TMA -> MMA pipeline depth that leaves room
// for them (48 KB per stage for N = 256), and the per-column constants staged
// in shared memory (bias; for EPI_DSILU_L1 also W1 by input component).
template <int EPI>
struct EpiCfg {
    static constexpr int tiles = (EPI == EPI_BIAS_SILU || EPI == EPI_LOSS || EPI == EPI_DSILU) ? 2
                                 : EPI == EPI_DSILU_L1 ? 1 : 0;
    static constexpr int stages = tiles ? 3 : 4;
    static constexpr bool bias = EPI == EPI_BIAS_SILU || EPI == EPI_BIAS_F32 || EPI == EPI_LOSS ||
                                 EPI == EPI_DSILU_L1;
    static constexpr int cst = EPI == EPI_DSILU_L1 ? 4 * 256 : (bias ? 256 : 4);
    // CTA accumulators of the column sums (bias gradient; for EPI_DSILU_L1
    // also the layer-1 weight gradient by input component), flushed once
    static constexpr int acc = EPI == EPI_DSILU_L1 ? 4 * 256 : (tiles >= 2 && EPI != EPI_BIAS_SILU) ? 256 : 4;
};
constexpr uint32_t STAGE_TILE_BYTES = 32 * 64;   // 32 rows x 32 BF16
constexpr uint32_t XS_BYTES = 32 * 3 * 4;        // a warp's 32 input rows (EPI_DSILU_L1)

template <int EPI>
__host__ __device__ constexpr size_t gemm_smem_bytes(int N)
{
    return 1024 + (size_t)EpiCfg<EPI>::stages * ((size_t)TILE_M * 128 + (size_t)N * 128) +
           (size_t)EPI_WARPS * (EpiCfg<EPI>::tiles * STAGE_TILE_BYTES + (EPI == EPI_DSILU_L1 ? XS_BYTES : 0));
}

struct GemmArgs {
    int M, N, K;                    // M % 128 == 0, N % 32 == 0 && 32 <= N <= 256, K % 64 == 0
    int k_split;                    // K elements per split (gridDim.y splits)
    int n_full;                     // row tiles taken whole; the rest go as two N halves each
    const float* bias;
    float* out_f; int64_t ldf;
    bf16* out_h; int64_t ldh;       // [M][N]
    bf16* out_z;                    // [M][N], ld = ldh
    const bf16* zprev;              // [M][N], ld = ldh
    const float* target;            // EPI_LOSS: FP32 rows of N targets
    const int32_t* trow;            // EPI_LOSS: target row of each batch row (nullptr: the same row)
    float scale;
    float* loss;
    float* colsum;                  // [N]
    const float* x; const float* w1; float* gw1;   // EPI_DSILU_L1: x [M][3], W1 [N][3], grad W1 [N][3]
    unsigned int* err;
};

// SiLU and its derivative with the fast exponential and division (results
// are rounded to BF16 afterwards; for z -> -inf, __fdividef by an infinite
// denominator returns 0)
__device__ __forceinline__ float silu(float z) { return __fdividef(z, 1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z)
{
    const float s = __fdividef(1.0f, 1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// Byte offset of 16-byte piece j (0..3) of row r in a 32-row x 64-byte tile
// with the 64-byte swizzle of the TMA stores (piece index XOR bits 7-8 of the
// offset; the tile is 2 KB aligned).  Sixteen-byte stores of 32 rows by 32
// lanes then touch every bank group equally often (no conflicts).
__device__ __forceinline__ uint32_t sw64(uint32_t r, uint32_t j)
{
    return r * 64u + ((j ^ ((r >> 1) & 3u)) << 4);
}

// This lane's row of 32 BF16 (h, 16-byte aligned) into a row-major staging tile.
__device__ __forceinline__ void stage_row(uint8_t* tile, int lane, const bf16* h)
{
#pragma unroll
    for (int j = 0; j < 4; ++j)
        *reinterpret_cast<uint4*>(tile + sw64((uint32_t)lane, (uint32_t)j)) = reinterpret_cast<const uint4*>(h)[j];
}

// This lane's row of 32 BF16 as column `lane` of a transposed staging tile
// (tile row c = column c of the chunk); each store writes one tile row of 64
// bytes across the warp.
__device__ __forceinline__ void stage_col(uint8_t* tile, int lane, const bf16* h)
{
    const uint32_t j = (uint32_t)lane >> 3, e = 2u * ((uint32_t)lane & 7u);
#pragma unroll
    for (int c = 0; c < 32; ++c) *reinterpret_cast<bf16*>(tile + sw64((uint32_t)c, j) + e) = h[c];
}

// Makes this lane's staging writes visible to the TMA unit and joins the warp;
// then lane 0 may issue the stores.
__device__ __forceinline__ void stage_done()
{
    umma::fence_async_smem();
    __syncwarp();
}

// Eight consecutive per-column constants (or row inputs) from shared memory
// (all lanes read the same address: a broadcast).
__device__ __forceinline__ void cst8(const float* c, float* o)
{
    const float4 p = reinterpret_cast<const float4*>(c)[0], q = reinterpret_cast<const float4*>(c)[1];
    o[0] = p.x; o[1] = p.y; o[2] = p.z; o[3] = p.w; o[4] = q.x; o[5] = q.y; o[6] = q.z; o[7] = q.w;
}

// Column sums over the warp's 32 rows, read from the transposed staging tile
// (lane c sums tile row c, rows in order 0..31), added to dst[0..31]; with xs
// (the rows' inputs by component, xs[32 k + r]), also sum g x_k added to
// gw[256 k + c].  dst and gw are the CTA's shared-memory accumulators.
__device__ __forceinline__ void warp_col_sums(const uint8_t* tt, int lane, float* dst, const float* xs, float* gw)
{
    float s = 0.0f, s0 = 0.0f, s1 = 0.0f, s2 = 0.0f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const uint4 q = *reinterpret_cast<const uint4*>(tt + sw64((uint32_t)lane, (uint32_t)j));
        const bf16* g8 = reinterpret_cast<const bf16*>(&q);
        float xa[8], xb[8], xc[8];
        if (xs) { cst8(xs + 8 * j, xa); cst8(xs + 32 + 8 * j, xb); cst8(xs + 64 + 8 * j, xc); }
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const float v = __bfloat162float(g8[e]);
            s += v;
            if (xs) { s0 += v * xa[e]; s1 += v * xb[e]; s2 += v * xc[e]; }
        }
    }
    atomicAdd(dst + lane, s);
    if (xs) {
        atomicAdd(gw + lane, s0);
        atomicAdd(gw + 256 + lane, s1);
        atomicAdd(gw + 512 + lane, s2);
    }
}

// TMA output maps of a GEMM: the row-major output (out_h) and the
// pre-activations (out_z), boxes of 32 x 32 BF16 with the 64-byte swizzle;
// maps of absent outputs are unused copies.
struct OutMaps {
    CUtensorMap h, z;
};

// A unit of work: row tile `tile`, accumulator columns [n0, n0 + nw).  The
// first n_full units are whole tiles; the remaining tiles are split into two
// units of N/2 columns each, so that the last round over the CTAs is half as
// long (512 tiles on 148 SMs: 3.5 tiles' time instead of 4).
struct Unit {
    int tile, n0, nw;
};
__device__ __forceinline__ Unit unit_of(int u, int n_full, int N)
{
    if (u < n_full) return Unit{u, 0, N};
    const int v = u - n_full;
    return Unit{n_full + (v >> 1), (v & 1) * (N >> 1), N >> 1};
}

// Epilogue of one 128 x N tile: the warp owns rows row0 + lane (row0 = tile
// row + 32 (w % 4)) and the 32-column chunks c0 = 32 (half + 4 k).  cst holds
// the bias (and for EPI_DSILU_L1 the columns of W1 at cst + 256 (1 + k)) in
// shared memory; stg is the warp's staging area (EpiCfg::tiles tiles of 2 KB,
// then for EPI_DSILU_L1 its rows' inputs).  BF16 outputs leave through TMA
// stores issued by lane 0; the staging tiles are rewritten only after the
// previous chunk's stores have read them.
template <int EPI>
__device__ __forceinline__ void epilogue(const GemmArgs& G, const OutMaps& om, uint32_t tbase, int row0,
                                         int lane, int half, const float* cst, uint8_t* stg, bool& pending,
                                         float* acc, Unit un, int next_row0, Unit next)
{
    const int N = G.N;
    const int row = row0 + lane;
    // the rows of this warp's next tile, whose epilogue inputs are brought
    // into L2 once this tile is done (next_row0 < 0: no next tile)
    int64_t next_in = -1;
    if ((EPI == EPI_LOSS || EPI == EPI_DSILU) && next_row0 >= 0)
        next_in = EPI == EPI_LOSS && G.trow ? (int64_t)G.trow[next_row0 + lane] : (int64_t)(next_row0 + lane);
    float sq = 0.0f;
    // the loss targets' row: the minibatch row's training-set row
    const int64_t trow_i = EPI == EPI_LOSS ? (G.trow ? (int64_t)G.trow[row] : (int64_t)row) : 0;
    float* xs = reinterpret_cast<float*>(stg + EpiCfg<EPI>::tiles * STAGE_TILE_BYTES);
    float x0 = 0.f, x1 = 0.f, x2 = 0.f;
    if (EPI == EPI_DSILU_L1) {
        x0 = G.x[(int64_t)row * 3]; x1 = G.x[(int64_t)row * 3 + 1]; x2 = G.x[(int64_t)row * 3 + 2];
        xs[lane] = x0; xs[32 + lane] = x1; xs[64 + lane] = x2;
    }
    for (int c0 = un.n0 + 32 * half; c0 < un.n0 + un.nw; c0 += 32 * (EPI_WARPS / 4)) {
        if (EpiCfg<EPI>::tiles) {
            // the previous chunk's TMA stores have read the staging tiles
            if (pending && lane == 0) umma::bulk_wait_read0();
            pending = false;
            __syncwarp();
        }
        // the chunk's pre-activations are requested before the accumulator is
        // read, so that their latency overlaps the tensor-memory load
        uint4 zp4[4];
        if (EPI == EPI_DSILU) {
            const uint4* z4 = reinterpret_cast<const uint4*>(G.zprev + (int64_t)row * G.ldh + c0);
#pragma unroll
            for (int i = 0; i < 4; ++i) zp4[i] = z4[i];
        }
        float v[32];
        umma::tmem_ld32(tbase + (uint32_t)(c0 - un.n0), v);
        // the chunk's loss targets, all requested at once (from L2: prefetched
        // during the previous tile)
        float4 tg[8];
        if (EPI == EPI_LOSS) {
            const float4* t4 = reinterpret_cast<const float4*>(G.target + trow_i * N + c0);
#pragma unroll
            for (int i = 0; i < 8; ++i) tg[i] = t4[i];
        }
        if (EPI == EPI_WGRAD) {
            // column n of the tile is row n of the transposed output: the warp's
            // 32 rows are 32 consecutive floats there (one coalesced reduction)
            float* o = G.out_f + (int64_t)c0 * G.ldf + row;
#pragma unroll
            for (int i = 0; i < 32; ++i) atomicAdd(o + (int64_t)i * G.ldf, v[i]);
        } else if (EPI == EPI_F32 || EPI == EPI_BIAS_F32 || EPI == EPI_PARTIAL) {
            float* o = G.out_f + (EPI == EPI_PARTIAL ? (int64_t)blockIdx.y * G.M * G.ldf : 0) +
                       (int64_t)row * G.ldf + c0;
#pragma unroll
            for (int g = 0; g < 4; ++g) {
                float b[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                if (EPI == EPI_BIAS_F32) cst8(cst + c0 + 8 * g, b);
                float4 q0, q1;
                q0.x = v[8 * g] + b[0]; q0.y = v[8 * g + 1] + b[1]; q0.z = v[8 * g + 2] + b[2]; q0.w = v[8 * g + 3] + b[3];
                q1.x = v[8 * g + 4] + b[4]; q1.y = v[8 * g + 5] + b[5]; q1.z = v[8 * g + 6] + b[6]; q1.w = v[8 * g + 7] + b[7];
                *reinterpret_cast<float4*>(o + 8 * g) = q0;
                *reinterpret_cast<float4*>(o + 8 * g + 4) = q1;
            }
        } else if (EPI == EPI_BIAS_SILU) {
            __align__(16) bf16 h[32];
            __align__(16) bf16 zz[32];
#pragma unroll
            for (int g = 0; g < 4; ++g) {
                float b[8];
                cst8(cst + c0 + 8 * g, b);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const float z = v[8 * g + q] + b[q];
                    zz[8 * g + q] = __float2bfloat16_rn(z);
                    h[8 * g + q] = __float2bfloat16_rn(silu(z));
                }
            }
            stage_row(stg, lane, h);
            if (G.out_z) stage_row(stg + STAGE_TILE_BYTES, lane, zz);
            stage_done();
            if (lane == 0) {
                umma::tma_store_2d(&om.h, c0, row0, stg);
                if (G.out_z) umma::tma_store_2d(&om.z, c0, row0, stg + STAGE_TILE_BYTES);
                umma::bulk_commit();
            }
            pending = true;
        } else {   // EPI_LOSS, EPI_DSILU, EPI_DSILU_L1: a BF16 gradient and its column sums
            __align__(16) bf16 h[32];
            if (EPI == EPI_LOSS) {
#pragma unroll
                for (int g = 0; g < 4; ++g) {
                    float b[8];
                    cst8(cst + c0 + 8 * g, b);
                    const float4 ta = tg[2 * g], tb = tg[2 * g + 1];
                    const float tt[8] = {ta.x, ta.y, ta.z, ta.w, tb.x, tb.y, tb.z, tb.w};
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const float d = (v[8 * g + q] + b[q]) - tt[q];
                        sq += d * d;
                        h[8 * g + q] = __float2bfloat16_rn(2.0f * d * G.scale);
                    }
                }
            } else if (EPI == EPI_DSILU) {
                __align__(16) bf16 zp[32];
#pragma unroll
                for (int i = 0; i < 4; ++i) reinterpret_cast<uint4*>(zp)[i] = zp4[i];
#pragma unroll
                for (int i = 0; i < 32; ++i) h[i] = __float2bfloat16_rn(v[i] * dsilu(__bfloat162float(zp[i])));
            } else {
#pragma unroll
                for (int g = 0; g < 4; ++g) {
                    float b[8], w0[8], w1[8], w2[8];
                    cst8(cst + c0 + 8 * g, b);
                    cst8(cst + 256 + c0 + 8 * g, w0);
                    cst8(cst + 512 + c0 + 8 * g, w1);
                    cst8(cst + 768 + c0 + 8 * g, w2);
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        // the forward's pre-activation, same operations in the same order
                        const float z = b[q] + x0 * w0[q] + x1 * w1[q] + x2 * w2[q];
                        const float zq = __bfloat162float(__float2bfloat16_rn(z));
                        h[8 * g + q] = __float2bfloat16_rn(v[8 * g + q] * dsilu(zq));
                    }
                }
            }
            // the transposed tile serves the column sums; EPI_DSILU_L1 writes no BF16 output
            uint8_t* tt = stg + (EPI == EPI_DSILU_L1 ? 0u : STAGE_TILE_BYTES);
            if (EPI != EPI_DSILU_L1) stage_row(stg, lane, h);
            stage_col(tt, lane, h);
            stage_done();
            if (EPI != EPI_DSILU_L1) {
                if (lane == 0) {
                    if (G.out_h) umma::tma_store_2d(&om.h, c0, row0, stg);
                    umma::bulk_commit();
                }
                pending = true;
            }
            warp_col_sums(tt, lane, acc + c0, EPI == EPI_DSILU_L1 ? xs : nullptr,
                          EPI == EPI_DSILU_L1 ? acc + 256 + c0 : nullptr);
            // the sums have read the tile before the next chunk may rewrite it
            __syncwarp();
        }
    }
    if (EPI == EPI_LOSS) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
        if (lane == 0) atomicAdd(G.loss, sq * G.scale);
    }
    if ((EPI == EPI_LOSS || EPI == EPI_DSILU) && next_in >= 0) {
        for (int c0 = next.n0 + 32 * half; c0 < next.n0 + next.nw; c0 += 32 * (EPI_WARPS / 4)) {
            const void* p = EPI == EPI_LOSS ? (const void*)(G.target + next_in * N + c0)
                                            : (const void*)(G.zprev + next_in * G.ldh + c0);
            asm volatile("prefetch.global.L2 [%0];" :: "l"(p));
        }
    }
}

// C = A B^T on the tensor cores.  A [M][K] and B [N][K] BF16, K-major, read
// through TMA tensor maps (128-byte swizzle, boxes of 64 x 128 rows and 64 x N
// rows).  Persistent over 128-row tiles (blockIdx.x, stride gridDim.x), K split
// over blockIdx.y.  Roles: warp 4 lane 0 streams A/B stages (full/empty
// mbarriers), warp 5 lane 0 issues tcgen05.mma into one of two TMEM
// accumulators and commits, warps 0-3 drain the other accumulator through the
// epilogue.  Every wait is bounded; a wait that runs out sets bit 0 of *err,
// tells the other roles to stop, and the CTA still waits (bounded) for its
// copies and MMAs in flight before freeing TMEM.
template <int EPI>
__global__ void __launch_bounds__(GEMM_THREADS, 1)
    gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                const __grid_constant__ CUtensorMap tmBh, const __grid_constant__ OutMaps om,
                const __grid_constant__ GemmArgs G)
{
    constexpr int STAGES = EpiCfg<EPI>::stages;
    constexpr bool MN = EPI == EPI_WGRAD;   // MN-major operands
    extern __shared__ uint8_t smem_raw[];
    // 1024-byte aligned in the shared window (the swizzle atom); offset from
    // smem_raw so that the compiler still sees shared-memory accesses
    uint8_t* smem = smem_raw + ((1024u - (umma::smem_u32(smem_raw) & 1023u)) & 1023u);
    const int N = G.N;
    const uint32_t a_bytes = TILE_M * 128, stage_bytes = a_bytes + (uint32_t)N * 128;
    uint8_t* stg_all = smem + STAGES * stage_bytes;   // 1024-byte aligned (stage_bytes is)
    __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], acc_full[2], acc_empty[2];
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;
    __shared__ __align__(16) float s_cst[EpiCfg<EPI>::cst];
    __shared__ float s_acc[EpiCfg<EPI>::acc];

    const int split = blockIdx.y;
    const int k_begin = split * G.k_split;
    const int k_end = min(G.K, k_begin + G.k_split);
    const int n_chunks = (k_end - k_begin) / TILE_K;
    const int n_tiles = G.M / TILE_M;
    const int n_units = G.n_full + 2 * (n_tiles - G.n_full);
    pdl_trigger();
    if (n_chunks <= 0 || (int)blockIdx.x >= n_units) return;   // uniform over the CTA

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    volatile int* abort_v = &abort_flag;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) { umma::mbar_init(&full[s], 1); umma::mbar_init(&empty[s], 1); }
        for (int a = 0; a < 2; ++a) { umma::mbar_init(&acc_full[a], 1); umma::mbar_init(&acc_empty[a], EPI_WARPS); }
        abort_flag = 0;
    }
    if (warp == MMA_WARP) umma::tmem_alloc(&tmem_slot, TMEM_COLS);
    if (warp == PRODUCER_WARP && lane == 0) {
        umma::prefetch_tmap(&tmA);
        umma::prefetch_tmap(&tmB);
        if (G.n_full < n_tiles) umma::prefetch_tmap(&tmBh);
        if (EpiCfg<EPI>::tiles > 0 && EPI != EPI_DSILU_L1) {
            umma::prefetch_tmap(&om.h);
            if (EPI == EPI_BIAS_SILU) umma::prefetch_tmap(&om.z);
        }
    }
    // barriers, TMEM and tensor-map prefetches above overlap the previous kernel's tail
    pdl_wait();
    if (EpiCfg<EPI>::bias)
        for (int i = threadIdx.x; i < N; i += blockDim.x) s_cst[i] = G.bias[i];
    if (EPI == EPI_DSILU_L1)
        for (int i = threadIdx.x; i < 3 * N; i += blockDim.x) s_cst[256 * (1 + i % 3) + i / 3] = G.w1[i];
    for (int i = threadIdx.x; i < EpiCfg<EPI>::acc; i += blockDim.x) s_acc[i] = 0.0f;
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = tmem_slot;

    if (warp == PRODUCER_WARP) {
        if (lane == 0) {
            uint32_t it = 0;
            bool ok = true;
            for (int ui = blockIdx.x; ui < n_units && ok; ui += gridDim.x) {
                const Unit un = unit_of(ui, G.n_full, N);
                const int tile = un.tile;
                for (int c = 0; c < n_chunks; ++c, ++it) {
                    const uint32_t s = it % STAGES, r = it / STAGES;
                    if (r > 0 && !umma::mbar_wait_or_abort(&empty[s], (r - 1) & 1u, WAIT_BUDGET, abort_v)) {
                        ok = false;
                        break;
                    }
                    uint8_t* st = smem + s * stage_bytes;
                    umma::mbar_arrive_expect_tx(&full[s], a_bytes + (uint32_t)un.nw * 128u);
                    const int k0 = k_begin + c * TILE_K;
                    if (MN) {
                        // boxes of 64 MN-elements x 64 K-rows, 8 KB apart
                        umma::tma_load_2d(st, &tmA, tile * TILE_M, k0, &full[s]);
                        umma::tma_load_2d(st + 8192, &tmA, tile * TILE_M + 64, k0, &full[s]);
                        for (int q = 0; q < N / 64; ++q)
                            umma::tma_load_2d(st + a_bytes + 8192 * q, &tmB, 64 * q, k0, &full[s]);
                    } else {
                        umma::tma_load_2d(st, &tmA, k0, tile * TILE_M, &full[s]);
                        if (un.nw == N) umma::tma_load_2d(st + a_bytes, &tmB, k0, 0, &full[s]);
                        else umma::tma_load_2d(st + a_bytes, &tmBh, k0, un.n0, &full[s]);
                    }
                }
            }
            if (!ok) { atomicOr(G.err, 1u); *abort_v = 1; }
            // copies still in flight land before the CTA can exit
            for (uint32_t j = it > (uint32_t)STAGES ? it - STAGES : 0u; j < it; ++j)
                umma::mbar_wait(&full[j % STAGES], (j / STAGES) & 1u, WAIT_BUDGET);
        }
    } else if (warp == MMA_WARP) {
        if (lane == 0) {
            const uint32_t idesc_full = umma::make_idesc_bf16(TILE_M, N, MN, MN);
            const uint32_t idesc_half = umma::make_idesc_bf16(TILE_M, N / 2, MN, MN);
            uint32_t it = 0, j = 0;
            bool ok = true;
            for (int ui = blockIdx.x; ui < n_units && ok; ui += gridDim.x, ++j) {
                const uint32_t idesc = ui < G.n_full ? idesc_full : idesc_half;
                const uint32_t a = j & 1u, u = j >> 1;
                if (u > 0 && !umma::mbar_wait_or_abort(&acc_empty[a], (u - 1) & 1u, WAIT_BUDGET, abort_v)) {
                    ok = false;
                    break;
                }
                umma::fence_after_sync();
                const uint32_t d = tmem + a * 256u;
                for (int c = 0; c < n_chunks; ++c, ++it) {
                    const uint32_t s = it % STAGES, r = it / STAGES;
                    if (!umma::mbar_wait_or_abort(&full[s], r & 1u, WAIT_BUDGET, abort_v)) { ok = false; break; }
                    umma::fence_after_sync();
                    const uint32_t sa = umma::smem_u32(smem + s * stage_bytes), sb = sa + a_bytes;
#pragma unroll
                    for (int k = 0; k < TILE_K / 16; ++k) {
                        const uint64_t ad = MN ? umma::make_desc_sw128_mn(sa + 2048u * k, 8192u)
                                               : umma::make_desc_sw128(sa + 32u * k);
                        const uint64_t bd = MN ? umma::make_desc_sw128_mn(sb + 2048u * k, 8192u)
                                               : umma::make_desc_sw128(sb + 32u * k);
                        umma::mma_bf16(d, ad, bd, idesc, (c > 0 || k > 0) ? 1u : 0u);
                    }
                    umma::commit(&empty[s]);
                }
                if (!ok) break;
                umma::commit(&acc_full[a]);
            }
            if (!ok) { atomicOr(G.err, 1u); *abort_v = 1; }
            // the last MMAs complete before TMEM is freed
            if (it > 0) umma::mbar_wait(&empty[(it - 1) % STAGES], ((it - 1) / STAGES) & 1u, WAIT_BUDGET);
        }
    } else {
        uint8_t* stg = stg_all + (size_t)warp * (EpiCfg<EPI>::tiles * STAGE_TILE_BYTES +
                                                (EPI == EPI_DSILU_L1 ? XS_BYTES : 0u));
        bool pending = false;   // TMA stores of this warp not yet known to have read its tiles
        uint32_t j = 0;
        for (int ui = blockIdx.x; ui < n_units; ui += gridDim.x, ++j) {
            const uint32_t a = j & 1u, u = j >> 1;
            const Unit un = unit_of(ui, G.n_full, N);
            if (!umma::mbar_wait_or_abort(&acc_full[a], u & 1u, WAIT_BUDGET, abort_v)) {
                if (lane == 0) atomicOr(G.err, 1u);
                *abort_v = 1;
                break;
            }
            umma::fence_after_sync();
            const int quad = warp & 3;
            const int nu = ui + (int)gridDim.x;
            const Unit next = unit_of(nu < n_units ? nu : ui, G.n_full, N);
            epilogue<EPI>(G, om, tmem + a * 256u + ((uint32_t)(32 * quad) << 16), un.tile * TILE_M + 32 * quad,
                          lane, warp >> 2, s_cst, stg, pending, s_acc, un,
                          nu < n_units ? next.tile * TILE_M + 32 * quad : -1, next);
            umma::fence_before_sync();
            __syncwarp();
            if (lane == 0) umma::mbar_arrive(&acc_empty[a]);
        }
        // the staging tiles stay valid until the TMA stores are complete
        if (EpiCfg<EPI>::tiles && lane == 0) umma::bulk_wait0();
        __syncwarp();
    }
    __syncthreads();
    if (warp == MMA_WARP) {
        umma::fence_after_sync();
        umma::tmem_dealloc(tmem, TMEM_COLS);
    }
    // the CTA's column sums, one global atomic per column
    if (EPI == EPI_LOSS || EPI == EPI_DSILU || EPI == EPI_DSILU_L1) {
        for (int i = threadIdx.x; i < N; i += blockDim.x) atomicAdd(G.colsum + i, s_acc[i]);
        if (EPI == EPI_DSILU_L1)
            for (int i = threadIdx.x; i < 3 * N; i += blockDim.x)
                atomicAdd(G.gw1 + i, s_acc[256 + 256 * (i % 3) + i / 3]);
    }
}

// ---- host side: tensor maps and launches ----
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

bool encoder()
{
    std::call_once(g_encode_once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        cudaGetLastError();
    });
    return g_encode != nullptr;
}

// rows x K BF16 matrix with row stride ld (elements), boxes of 64 x box_rows,
// 128-byte swizzle.
bool make_map(CUtensorMap* m, const bf16* base, int64_t rows, int64_t K, int64_t ld, int box_rows)
{
    if (!encoder() || ((uintptr_t)base & 15) || (ld * 2) % 16 || K % TILE_K) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)(ld * 2)};
    const cuuint32_t box[2] = {(cuuint32_t)TILE_K, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return g_encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// MN-major operand map: a K x MN BF16 matrix stored row by row (row stride ld
// elements), boxes of 64 MN-elements x 64 K-rows with the 128-byte swizzle.
bool make_map_mn(CUtensorMap* m, const bf16* base, int64_t k_rows, int64_t mn, int64_t ld)
{
    if (!encoder() || ((uintptr_t)base & 15) || (ld * 2) % 16 || mn % 64 || k_rows % TILE_K || ld < mn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)mn, (cuuint64_t)k_rows};
    const cuuint64_t strides[1] = {(cuuint64_t)(ld * 2)};
    const cuuint32_t box[2] = {64, 64};
    const cuuint32_t estr[2] = {1, 1};
    return g_encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Store map of a rows x cols BF16 matrix with row stride ld (elements): boxes
// of 32 x 32 with the 64-byte swizzle of the epilogue's staging tiles.
bool make_store_map(CUtensorMap* m, const bf16* base, int64_t rows, int64_t cols, int64_t ld)
{
    if (!encoder() || !base || ((uintptr_t)base & 15) || (ld * 2) % 16 || cols % 32 || rows % 32 || ld < cols)
        return false;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)(ld * 2)};
    const cuuint32_t box[2] = {32, 32};
    const cuuint32_t estr[2] = {1, 1};
    return g_encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                    CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// A [M][K] (row stride lda), B [N][K] (row stride ldb); for EPI_WGRAD A [K][M]
// and B [K][N] (MN-major, N % 64 == 0).
template <int EPI>
int launch_gemm(const GemmArgs& g, const bf16* A, int64_t lda, const bf16* B, int64_t ldb, int grid_x,
                int splits, cudaStream_t st)
{
    if (g.M % TILE_M || g.M <= 0 || g.N % 32 || g.N > 256 || g.N < 32 || g.K % TILE_K || g.K <= 0 ||
        splits < 1 || g.k_split % TILE_K || g.k_split <= 0 || (int64_t)(splits - 1) * g.k_split >= g.K ||
        (int64_t)splits * g.k_split < g.K || grid_x < 1)
        return CL_ERR_ARG;
    CUtensorMap ta, tb;
    if (EPI == EPI_WGRAD) {
        if (g.N % 64 || !make_map_mn(&ta, A, g.K, g.M, lda) || !make_map_mn(&tb, B, g.K, g.N, ldb)) return CL_ERR_ARG;
    } else if (!make_map(&ta, A, g.M, g.K, lda, TILE_M) || !make_map(&tb, B, g.N, g.K, ldb, g.N)) {
        return CL_ERR_ARG;
    }
    // output maps of the staged epilogues (unused ones are copies of ta)
    OutMaps om;
    om.h = om.z = ta;
    if (EpiCfg<EPI>::tiles > 0 && EPI != EPI_DSILU_L1) {
        if (!g.out_h || !make_store_map(&om.h, g.out_h, g.M, g.N, g.ldh)) return CL_ERR_ARG;
        if (EPI == EPI_BIAS_SILU && g.out_z && !make_store_map(&om.z, g.out_z, g.M, g.N, g.ldh)) return CL_ERR_ARG;
    }
    // the shared-memory opt-in is a per-device attribute of the kernel: set it
    // once for every device this process launches on
    static std::atomic<uint64_t> attr_devices{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t bit = 1ull << (dev & 63);
    if (!(attr_devices.load() & bit)) {
        if (cudaFuncSetAttribute(gemm_kernel<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)gemm_smem_bytes<EPI>(256)) != cudaSuccess)
            return CL_ERR_CUDA;
        attr_devices.fetch_or(bit);
    }
    const int tiles = g.M / TILE_M;
    dim3 grid((unsigned)(grid_x < tiles ? grid_x : tiles), (unsigned)splits);
    // a last round that would occupy at most half of the CTAs runs as N halves
    // (two units per tile) on all of them
    GemmArgs ga = g;
    ga.n_full = tiles;
    CUtensorMap tbh = tb;
    const int r = tiles % (int)grid.x;
    if (EPI != EPI_WGRAD && EPI != EPI_PARTIAL && splits == 1 && g.N % 64 == 0 && r > 0 && 2 * r <= (int)grid.x) {
        if (!make_map(&tbh, B, g.N, g.K, ldb, g.N / 2)) return CL_ERR_ARG;
        ga.n_full = tiles - r;
    }
    // at least 116 KB so that one CTA holds an SM: each allocates all 512 TMEM columns
    const size_t smem = gemm_smem_bytes<EPI>(g.N) > 116 * 1024 ? gemm_smem_bytes<EPI>(g.N) : 116 * 1024;
    if (launch_pdl(gemm_kernel<EPI>, grid, dim3(GEMM_THREADS), smem, st, ta, tb, tbh, om, ga) != cudaSuccess)
        return CL_ERR_CUDA;
    return cudaGetLastError() == cudaSuccess ? CL_OK : CL_ERR_CUDA;
}


// ===========================================================================
// The MLP: 3 -> 256 -> 256 -> 256 -> 192, SiLU, BF16 weights/activations,
// FP32 accumulation and FP32 master weights with Adam.
// ===========================================================================
constexpr int D_IN = 3, D_H = 256, D_OUT = 192;
constexpr int WGRAD_MIN_SPLIT_K = 512;   // fewest batch rows per weight-gradient split

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

// Random minibatch (with replacement) from the training set: the inputs are
// copied (Xb), the targets are read in place by the loss epilogue through the
// row indices (rows).
__global__ void __launch_bounds__(256) gather_batch(const float* __restrict__ X, int64_t n_all, int B,
                                                    uint32_t seed, uint32_t step, float* Xb, int32_t* rows)
{
    pdl_trigger();
    pdl_wait();
    const int b = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (b >= B) return;
    const int64_t i = (int64_t)(hash32((uint32_t)b, step, seed) % (uint32_t)n_all);
    rows[b] = (int32_t)i;
    Xb[(int64_t)b * D_IN] = X[i * D_IN];
    Xb[(int64_t)b * D_IN + 1] = X[i * D_IN + 1];
    Xb[(int64_t)b * D_IN + 2] = X[i * D_IN + 2];
}

// Layer 1 (K = 3) on the CUDA cores: h = silu(x W1^T + b1) for 64 rows per
// block; a thread takes two adjacent features of every other row, so that a
// warp stores 128 contiguous bytes of a row per instruction.
constexpr int L1_ROWS = 64;
__global__ void __launch_bounds__(256) layer1_fwd(const float* __restrict__ X, const float* __restrict__ W1,
                                                  const float* __restrict__ b1, bf16* H)
{
    pdl_trigger();
    pdl_wait();
    __shared__ float xs[L1_ROWS * 3];
    const int b0 = blockIdx.x * L1_ROWS;
    for (int i = threadIdx.x; i < L1_ROWS * 3; i += blockDim.x) xs[i] = X[(int64_t)b0 * 3 + i];
    __syncthreads();
    const int j = 2 * (threadIdx.x % (D_H / 2)), r0 = threadIdx.x / (D_H / 2);
    const float wa0 = W1[j * 3], wa1 = W1[j * 3 + 1], wa2 = W1[j * 3 + 2], ba = b1[j];
    const float wb0 = W1[j * 3 + 3], wb1 = W1[j * 3 + 4], wb2 = W1[j * 3 + 5], bb = b1[j + 1];
    __nv_bfloat162* out = reinterpret_cast<__nv_bfloat162*>(H + (int64_t)b0 * D_H + j);
#pragma unroll 4
    for (int r = r0; r < L1_ROWS; r += 2) {
        // same operations, same order as the layer-1 recompute in the backward epilogue
        const float x0 = xs[r * 3], x1 = xs[r * 3 + 1], x2 = xs[r * 3 + 2];
        const float za = ba + x0 * wa0 + x1 * wa1 + x2 * wa2;
        const float zb = bb + x0 * wb0 + x1 * wb1 + x2 * wb2;
        out[(int64_t)r * (D_H / 2)] = __floats2bfloat162_rn(silu(za), silu(zb));
    }
}

// Adam over the whole parameter block in one launch (FP32 master weights;
// the gradient is zeroed as it is read); the three weight matrices of the
// tensor-core layers also get their BF16 copies (W^T as stored for the
// forward B operand, W for the backward-data B operand), described by
// AdamCopies.
struct AdamCopies {
    int64_t off[3]; int n[3]; int OUT[3]; int IN[3];
    bf16* wt[3]; bf16* w[3];
};
__global__ void adam_all(float* __restrict__ w, float* __restrict__ g, float* __restrict__ m,
                         float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float bc1,
                         float bc2, const AdamCopies C)
{
    pdl_trigger();
    pdl_wait();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        g[i] = 0.0f;   // zeroed for the next step's accumulation
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi; v[i] = vi;
        const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        w[i] = wi;
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            const int64_t r = i - C.off[t];
            if (r >= 0 && r < C.n[t]) {
                const int o = (int)(r / C.IN[t]), k = (int)(r % C.IN[t]);
                const bf16 q = __float2bfloat16_rn(wi);
                C.wt[t][r] = q;
                C.w[t][(int64_t)k * C.OUT[t] + o] = q;
            }
        }
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
    int max_ctas = 0;               // cap on the GEMM grid (0: one CTA per SM)
    cudaStream_t stream = nullptr;
    char err[256] = {0};
    // FP32 master parameters, gradients, Adam moments
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    int64_t adam_t = 0;
    // BF16 weight copies
    bf16 *w2t = nullptr, *w2 = nullptr, *w3t = nullptr, *w3 = nullptr, *w4t = nullptr, *w4 = nullptr;
    // activations and gradients (max_batch rows)
    float *xb = nullptr, *o = nullptr;
    int32_t* brow = nullptr;        // training-set row of each minibatch row
    bf16 *h1 = nullptr, *h2 = nullptr, *z2 = nullptr, *h3 = nullptr, *z3 = nullptr;
    bf16 *dO = nullptr, *dz3 = nullptr, *dz2 = nullptr;
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

int grid_for(const cl_mlp* m, int B)
{
    const int tiles = B / TILE_M;
    const int cap = m->max_ctas > 0 && m->max_ctas < m->num_sms ? m->max_ctas : m->num_sms;
    return tiles < cap ? tiles : cap;
}

GemmArgs gemm_args(cl_mlp* m)
{
    GemmArgs g;
    memset(&g, 0, sizeof g);
    g.err = m->derr;
    return g;
}

// Forward pass over B rows of m->xb (B % 128 == 0).  Training (with_loss):
// keeps H and Z for the backward pass and ends in the loss epilogue, which
// reads the targets (rows `trow` of `target`, or its first B rows) and writes
// dO, the b4 gradient and the loss.  Inference: O into m->o.
int forward(cl_mlp* m, int B, bool with_loss, const float* target, const int32_t* trow, cudaStream_t st,
            bool zero_grad = true)
{
    const int grid = grid_for(m, B);
    if (with_loss && zero_grad) cudaMemsetAsync(m->g, 0, N_PARAMS * sizeof(float), st);
    launch_pdl(layer1_fwd, dim3((unsigned)(B / L1_ROWS)), dim3(256), 0, st, (const float*)m->xb,
               (const float*)(m->p + OFF_W1), (const float*)(m->p + OFF_B1), m->h1);
    GemmArgs g = gemm_args(m);
    g.M = B; g.N = D_H; g.K = D_H; g.k_split = D_H;
    g.bias = m->p + OFF_B2; g.out_h = m->h2; g.ldh = D_H;
    g.out_z = with_loss ? m->z2 : nullptr;
    int rc = launch_gemm<EPI_BIAS_SILU>(g, m->h1, D_H, m->w2t, D_H, grid, 1, st);
    if (rc) return rc;
    g.bias = m->p + OFF_B3; g.out_h = m->h3;
    g.out_z = with_loss ? m->z3 : nullptr;
    if ((rc = launch_gemm<EPI_BIAS_SILU>(g, m->h2, D_H, m->w3t, D_H, grid, 1, st))) return rc;
    GemmArgs q = gemm_args(m);
    q.M = B; q.N = D_OUT; q.K = D_H; q.k_split = D_H; q.bias = m->p + OFF_B4;
    if (!with_loss) {
        q.out_f = m->o; q.ldf = D_OUT;
        return launch_gemm<EPI_BIAS_F32>(q, m->h3, D_H, m->w4t, D_H, grid, 1, st);
    }
    q.target = target; q.trow = trow; q.scale = 1.0f / ((float)B * (float)D_OUT); q.loss = m->loss;
    q.out_h = m->dO; q.ldh = D_OUT; q.colsum = m->g + OFF_B4;
    return launch_gemm<EPI_LOSS>(q, m->h3, D_H, m->w4t, D_H, grid, 1, st);
}

// Backward pass after forward(with_loss), which zeroed m->g: bias and layer-1
// gradients accumulate in the epilogues, weight gradients come from the
// split-K GEMMs.
int backward(cl_mlp* m, int B, cudaStream_t st)
{
    const int grid = grid_for(m, B);
    // backward data: dZ3 = (dO W4) * silu'(Z3), dZ2 = (dZ3 W3) * silu'(Z2), dZ1 = (dZ2 W2) * silu'(Z1)
    GemmArgs g = gemm_args(m);
    g.M = B; g.N = D_H; g.K = D_OUT; g.k_split = D_OUT;
    g.out_h = m->dz3; g.ldh = D_H; g.zprev = m->z3; g.colsum = m->g + OFF_B3;
    int rc = launch_gemm<EPI_DSILU>(g, m->dO, D_OUT, m->w4, D_OUT, grid, 1, st);
    if (rc) return rc;
    g.K = D_H; g.k_split = D_H;
    g.out_h = m->dz2; g.zprev = m->z2; g.colsum = m->g + OFF_B2;
    if ((rc = launch_gemm<EPI_DSILU>(g, m->dz3, D_H, m->w3, D_H, grid, 1, st))) return rc;
    GemmArgs l1 = gemm_args(m);
    l1.M = B; l1.N = D_H; l1.K = D_H; l1.k_split = D_H;
    l1.bias = m->p + OFF_B1; l1.x = m->xb; l1.w1 = m->p + OFF_W1;
    l1.colsum = m->g + OFF_B1; l1.gw1 = m->g + OFF_W1;
    if ((rc = launch_gemm<EPI_DSILU_L1>(l1, m->dz2, D_H, m->w2, D_H, grid, 1, st))) return rc;
    // weight gradients dW = H^T dZ (split-K over the batch), each split added
    // in place into grad W^T (zeroed by the forward pass)
    // K splits sized so that the two 128-row tiles of the 256 inputs fill every SM once
    const int per_tile_ctas = m->num_sms / (D_H / TILE_M) > 0 ? m->num_sms / (D_H / TILE_M) : 1;
    int k_split = ((B + per_tile_ctas - 1) / per_tile_ctas + TILE_K - 1) / TILE_K * TILE_K;
    if (k_split < WGRAD_MIN_SPLIT_K) k_split = WGRAD_MIN_SPLIT_K;
    const int splits = (B + k_split - 1) / k_split;
    struct WG { const bf16* h; const bf16* dz; int OUT; int64_t off_w; };
    const WG wg[3] = {{m->h3, m->dO, D_OUT, OFF_W4}, {m->h2, m->dz3, D_H, OFF_W3}, {m->h1, m->dz2, D_H, OFF_W2}};
    for (int l = 0; l < 3; ++l) {
        GemmArgs w = gemm_args(m);
        w.M = D_H; w.N = wg[l].OUT; w.K = B; w.k_split = k_split;
        w.out_f = m->g + wg[l].off_w; w.ldf = D_H;
        if ((rc = launch_gemm<EPI_WGRAD>(w, wg[l].h, D_H, wg[l].dz, wg[l].OUT, D_H / TILE_M, splits, st))) return rc;
    }
    return cudaGetLastError() == cudaSuccess ? CL_OK : CL_ERR_CUDA;
}

void adam(cl_mlp* m, float lr, cudaStream_t st)
{
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    m->adam_t += 1;
    const float bc1 = 1.0f - powf(b1, (float)m->adam_t), bc2 = 1.0f - powf(b2, (float)m->adam_t);
    AdamCopies c;
    const int64_t offs[3] = {OFF_W2, OFF_W3, OFF_W4};
    const int outs[3] = {D_H, D_H, D_OUT};
    bf16* wts[3] = {m->w2t, m->w3t, m->w4t};
    bf16* ws[3] = {m->w2, m->w3, m->w4};
    for (int t = 0; t < 3; ++t) {
        c.off[t] = offs[t]; c.OUT[t] = outs[t]; c.IN[t] = D_H; c.n[t] = outs[t] * D_H;
        c.wt[t] = wts[t]; c.w[t] = ws[t];
    }
    const unsigned grid = (unsigned)((N_PARAMS + 255) / 256);
    launch_pdl(adam_all, dim3(grid), dim3(256), 0, st, m->p, m->g, m->m, m->v, (int64_t)N_PARAMS,
               lr, b1, b2, eps, bc1, bc2, c);
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
    bool ok = dalloc(m, &m->p, N_PARAMS) && dalloc(m, &m->g, N_PARAMS) && dalloc(m, &m->m, N_PARAMS) &&
              dalloc(m, &m->v, N_PARAMS) &&
              dalloc(m, &m->w2t, (size_t)D_H * D_H) && dalloc(m, &m->w2, (size_t)D_H * D_H) &&
              dalloc(m, &m->w3t, (size_t)D_H * D_H) && dalloc(m, &m->w3, (size_t)D_H * D_H) &&
              dalloc(m, &m->w4t, (size_t)D_OUT * D_H) && dalloc(m, &m->w4, (size_t)D_OUT * D_H) &&
              dalloc(m, &m->xb, B * D_IN) && dalloc(m, &m->brow, B) && dalloc(m, &m->o, B * D_OUT) &&
              dalloc(m, &m->h1, B * D_H) &&
              dalloc(m, &m->h2, B * D_H) && dalloc(m, &m->z2, B * D_H) &&
              dalloc(m, &m->h3, B * D_H) && dalloc(m, &m->z3, B * D_H) &&
              dalloc(m, &m->dO, B * D_OUT) && dalloc(m, &m->dz3, B * D_H) && dalloc(m, &m->dz2, B * D_H) &&
              dalloc(m, &m->loss, 1) &&
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

// Cap the number of CTAs of the row-tiled GEMMs (0 = one per SM); with few
// CTAs each one walks many tiles (tests of the persistent pipeline).
int cl_mlp_set_max_ctas(cl_mlp* m, int n)
{
    if (!m || n < 0) return CL_ERR_ARG;
    m->max_ctas = n;
    return CL_OK;
}

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
    // the gradient is zeroed once here and then by each Adam step, so that a
    // step is an unbroken chain of kernels
    cudaMemsetAsync(m->g, 0, N_PARAMS * sizeof(float), st);
    for (int s = 0; s < steps; ++s) {
        launch_pdl(gather_batch, dim3((batch + 255) / 256), dim3(256), 0, st, (const float*)m->data_x,
                   (int64_t)m->n_data, batch, seed, step0 + (uint32_t)s, m->xb, m->brow);
        int rc = forward(m, batch, true, m->data_t, m->brow, st, false);
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
        int rc = forward(m, B, false, nullptr, nullptr, st);
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
    cudaMemsetAsync(m->loss, 0, sizeof(float), st);
    int rc = forward(m, B, true, d_t, nullptr, st);
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
    if (!A || !B || !C || !d_err || M <= 0 || N <= 0 || K <= 0 || grid_x <= 0 || splits < 1) return CL_ERR_ARG;
    GemmArgs g;
    memset(&g, 0, sizeof g);
    g.M = M; g.N = N; g.K = K;
    g.out_f = C; g.ldf = N;
    g.err = d_err;
    if (splits > 1) {
        g.k_split = ((K / splits + TILE_K - 1) / TILE_K) * TILE_K;
        return launch_gemm<EPI_PARTIAL>(g, (const bf16*)A, K, (const bf16*)B, K, grid_x, splits,
                                        (cudaStream_t)stream);
    }
    g.k_split = K;
    return launch_gemm<EPI_F32>(g, (const bf16*)A, K, (const bf16*)B, K, grid_x, 1, (cudaStream_t)stream);
}

}  // extern "C"
