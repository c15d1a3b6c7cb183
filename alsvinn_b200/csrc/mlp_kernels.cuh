// Kernels of the MLP surrogate: the tcgen05 GEMM with its fused epilogues
// and the small CUDA-core kernels around it (input packing, the 256 -> 1
// output head, its loss and backward, column sums for bias gradients, Adam).
#pragma once

#include <cuda.h>

#include "mlp_tc.cuh"

namespace mlpk {

template <int BN>
constexpr int gemm_smem_bytes() {
    return 2 * (kTileM * kChunkK * 2 + BN * kChunkK * 2) + 1024;
}

template <int BN, int EPI>
__device__ __forceinline__ void epilogue16(const GemmArgs& g, long long m, int n, const float* v,
                                           int n_valid) {
    if (EPI == EPI_FORWARD) {
        if (g.z) {
            __align__(16) float z[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                z[i] = v[i] + g.bias[n + i];
            }
            float4* dz = reinterpret_cast<float4*>(g.z + m * g.ldz + n);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                dz[i] = reinterpret_cast<const float4*>(z)[i];
            }
        }
        __align__(16) __nv_bfloat16 hb[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            hb[i] = __float2bfloat16_rn(gelu_half(fmaf(0.5f, v[i], 0.5f * g.bias[n + i])));
        }
        uint4* dh = reinterpret_cast<uint4*>(g.h + m * g.ldh + n);
        dh[0] = reinterpret_cast<const uint4*>(hb)[0];
        dh[1] = reinterpret_cast<const uint4*>(hb)[1];
    } else if (EPI == EPI_BACKWARD) {
        __align__(16) float zin[16];
        const float4* sz = reinterpret_cast<const float4*>(g.zin + m * g.ldz + n);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            reinterpret_cast<float4*>(zin)[i] = sz[i];
        }
        __align__(16) __nv_bfloat16 hb[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            hb[i] = __float2bfloat16_rn(v[i] * gelu_grad(zin[i]));
        }
        uint4* dh = reinterpret_cast<uint4*>(g.h + m * g.ldh + n);
        dh[0] = reinterpret_cast<const uint4*>(hb)[0];
        dh[1] = reinterpret_cast<const uint4*>(hb)[1];
    } else {
        float* dst = g.g + blockIdx.z * g.split_stride + m * g.ldg + n;
        if (n + 16 <= n_valid && (g.ldg & 3) == 0) {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                reinterpret_cast<float4*>(dst)[i] = make_float4(v[4 * i], v[4 * i + 1],
                                                                v[4 * i + 2], v[4 * i + 3]);
            }
        } else {
            for (int i = 0; i < 16; ++i) {
                if (n + i < n_valid) {
                    dst[i] = v[i];
                }
            }
        }
    }
}

// D[128 x BN tile] = A * B^T over K, then the epilogue.  Grid: (M/128, N/BN,
// splits): split z covers K range [z K, (z+1) K) and, with EPI_WGRAD, writes
// its partial product z * split_stride further (summed by sum_splits).
// `n_valid` limits the stored columns of EPI_WGRAD (padded inputs).
template <int BN, int EPI>
__global__ void __launch_bounds__(kThreads) gemm_kernel(GemmArgs g, int n_valid) {
    static_assert(BN == 32 || BN == 64 || BN == 128 || BN == 256, "TMEM columns: power of two");
    extern __shared__ unsigned char smem_raw[];
    __shared__ uint64_t bars[2];
    __shared__ uint64_t drain;
    __shared__ uint32_t tmem_base;
    unsigned char* base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    constexpr int kABytes = kTileM * kChunkK * 2;
    constexpr int kBBytes = BN * kChunkK * 2;
    const unsigned limit = g.wait_limit ? g.wait_limit : kWaitLimit;
    unsigned char* sa[2] = {base, base + kABytes + kBBytes};
    unsigned char* sb[2] = {base + kABytes, base + 2 * kABytes + kBBytes};

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const long long m0 = (long long)blockIdx.x * kTileM;
    const long long n0 = (long long)blockIdx.y * BN;
    const int kb = blockIdx.z * g.K;

    if (warp == 0) {
        tmem_alloc(&tmem_base, BN);
    }
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init(&drain, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    const uint32_t idesc = instr_desc_bf16(kTileM, BN);
    const int nk = g.K / kChunkK;

    int last = -1;          // last chunk whose MMAs were committed
    bool failed = false;
    for (int c = 0; c < nk; ++c) {
        const int s = c & 1;
        bool ok = true;
        if (c >= 2) {
            ok = mbar_wait(&bars[s], unsigned((c - 2) >> 1) & 1u, limit);
        }
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        stage_operand<kTileM>(sa[s], g.a, m0, kb + c * kChunkK);
        stage_operand<BN>(sb[s], g.b, n0, kb + c * kChunkK);
        fence_async_shared();
        __syncthreads();
        if (threadIdx.x == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(sa[s]);
            const uint32_t b0 = smem_u32(sb[s]);
#pragma unroll
            for (int j = 0; j < kChunkK / 16; ++j) {
                mma_bf16(tmem, smem_desc(a0 + j * 256, 128, 1024),
                         smem_desc(b0 + j * 256, 128, 1024), idesc, (c > 0 || j > 0) ? 1u : 0u);
            }
            if (!g.withhold_commit) {
                mma_commit(&bars[s]);
            }
        }
        last = c;
    }
    bool done = false;
    if (last >= 0) {
        done = mbar_wait(&bars[last & 1], unsigned(last >> 1) & 1u, limit);
    }
    if (__syncthreads_or(!done) || failed) {
        if (threadIdx.x == 0) {
            atomicExch(g.error, 1);
            // every MMA issued so far completes before TMEM is freed
            mma_commit(&drain);
        }
        mbar_wait(&drain, 0, kWaitLimit);
    } else {
        tc_fence_after();
        const long long m = m0 + warp * 32 + lane;
        const uint32_t lane_base = tmem + (uint32_t(warp * 32) << 16);
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v[16];
            tmem_load16(lane_base + uint32_t(c0), v);
            epilogue16<BN, EPI>(g, m, int(n0) + c0, v, n_valid);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_free(tmem, BN);
    }
}

// Inference forward layer, persistent and warp-specialised:
// H_out = bf16(gelu(H_in W^T + b)) over 128 x 256 tiles, K = 64 * NK (NK <= 4).
//   warp 0  TMA producer: the whole weight matrix once into shared memory
//           (NK x 32 KB, resident for every tile), then the activation
//           chunks (128 x 64, 16 KB) through a ring of kRing stages;
//   warp 1  MMA issuer: per tile, NK x 4 tcgen05.mma into one of two TMEM
//           accumulators (2 x 256 columns), tcgen05.commit freeing each ring
//           stage and finally marking the accumulator full;
//   warps 4..19  epilogue: warp w reads TMEM lane quarter w % 4 and 64
//           columns, applies bias + GELU and stores BF16 (or, with HEAD,
//           folds the 256 -> 1 output layer in), then releases the
//           accumulator, so the epilogue of tile i overlaps the MMAs of i+1.
// All operands are 128-byte swizzled (the canonical K-major SWIZZLE_128B
// UMMA layout).  Every wait is bounded; a timeout sets the error flag and
// the roles drain and return.
constexpr int kTmaThreads = 640;
constexpr int kRing = 4;
constexpr int kEpiWarp0 = 4;

// Dynamic shared memory of every instantiation: the NK = 4 footprint, so that
// one block per SM owns all 512 TMEM columns whatever NK is.
constexpr int gemm_tma_smem_bytes() {
    return 4 * 256 * kChunkK * 2 + kRing * kTileM * kChunkK * 2 + 1024;
}

__device__ __forceinline__ void named_barrier_sync(int id, int threads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <int NK, bool HEAD>
__global__ void __launch_bounds__(kTmaThreads, 1) gemm_tma_forward(const __grid_constant__ CUtensorMap tmA,
                                                                const __grid_constant__ CUtensorMap tmB,
                                                                GemmArgs g, const float* head_w,
                                                                const float* head_b, float* y,
                                                                long long rows_valid) {
    constexpr int BN = 256;
    constexpr uint32_t kABytes = kTileM * kChunkK * 2;   // one ring stage
    constexpr uint32_t kBBytes = BN * kChunkK * 2;       // one K chunk of the weights
    extern __shared__ unsigned char smem_raw[];
    __shared__ uint64_t b_full;
    __shared__ uint64_t a_full[kRing];
    __shared__ uint64_t a_empty[kRing];
    __shared__ uint64_t t_full[2];
    __shared__ uint64_t t_empty[2];
    __shared__ uint64_t drain;
    __shared__ uint32_t tmem_base;
    __shared__ int abort_flag;
    __shared__ float head_part[2][4][kTileM];
    unsigned char* base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char* sB = base;                       // NK x 32 KB
    unsigned char* sA = base + NK * kBBytes;        // kRing x 16 KB
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int tiles = g.M / kTileM;
    if (warp == 0) {
        tmem_alloc(&tmem_base, 2 * BN);
    }
    if (threadIdx.x == 0) {
        mbar_init(&b_full, 1);
        for (int r = 0; r < kRing; ++r) {
            mbar_init(&a_full[r], 1);
            mbar_init(&a_empty[r], 1);
        }
        for (int k = 0; k < 2; ++k) {
            mbar_init(&t_full[k], 1);
            mbar_init(&t_empty[k], 16);      // one arrival per epilogue warp
        }
        mbar_init(&drain, 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    volatile int* abort_v = &abort_flag;

    if (warp == 0) {
        if (lane == 0) {
            // the weights, once
            mbar_expect_tx(&b_full, NK * kBBytes);
            for (int c = 0; c < NK; ++c) {
                tma_load_2d(sB + c * kBBytes, &tmB, c * kChunkK, 0, &b_full);
            }
            long long it = 0;
            for (int t = blockIdx.x; t < tiles && !*abort_v; t += gridDim.x) {
                for (int c = 0; c < NK; ++c, ++it) {
                    const int slot = int(it % kRing);
                    if (it >= kRing && !mbar_wait(&a_empty[slot], unsigned((it / kRing - 1) & 1))) {
                        *abort_v = 1;
                        break;
                    }
                    mbar_expect_tx(&a_full[slot], kABytes);
                    tma_load_2d(sA + slot * kABytes, &tmA, c * kChunkK, t * kTileM, &a_full[slot]);
                }
            }
            // copies still in flight (an aborted run) land before the block exits
            mbar_wait(&b_full, 0);
            for (int r = 0; r < kRing; ++r) {
                const long long n = it > r ? (it - r + kRing - 1) / kRing : 0;
                if (n > 0) {
                    mbar_wait(&a_full[r], unsigned((n - 1) & 1));
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = instr_desc_bf16(kTileM, BN);
            bool ok = mbar_wait(&b_full, 0);
            long long it = 0;
            int lt = 0;
            for (int t = blockIdx.x; ok && t < tiles && !*abort_v; t += gridDim.x, ++lt) {
                const int acc = lt & 1;
                if (lt >= 2 && !mbar_wait(&t_empty[acc], unsigned(((lt >> 1) - 1) & 1))) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                for (int c = 0; c < NK; ++c, ++it) {
                    const int slot = int(it % kRing);
                    if (!mbar_wait(&a_full[slot], unsigned((it / kRing) & 1))) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a0 = smem_u32(sA + slot * kABytes);
                    const uint32_t b0 = smem_u32(sB + c * kBBytes);
#pragma unroll
                    for (int j = 0; j < kChunkK / 16; ++j) {
                        mma_bf16(tmem + uint32_t(acc * BN), smem_desc_sw128(a0 + j * 32),
                                 smem_desc_sw128(b0 + j * 32), idesc, (c > 0 || j > 0) ? 1u : 0u);
                    }
                    mma_commit(&a_empty[slot]);
                }
                if (!ok) {
                    break;
                }
                mma_commit(&t_full[acc]);
            }
            if (!ok) {
                *abort_v = 1;
            }
            // every MMA this thread issued is complete before TMEM is freed
            mma_commit(&drain);
            mbar_wait(&drain, 0);
        }
    } else if (warp >= kEpiWarp0) {
        const int ew = warp - kEpiWarp0;          // 0..15
        const int quarter = warp & 3;
        const int cg = ew >> 2;
        const int row = quarter * 32 + lane;
        int lt = 0;
        for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++lt) {
            const int acc = lt & 1;
            bool ok = !*abort_v && mbar_wait(&t_full[acc], unsigned((lt >> 1) & 1));
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) {
                *abort_v = 1;
            }
            // even and odd columns summed apart, then added
            float2 hsum2 = make_float2(0.0f, 0.0f);
            if (ok) {
                tc_fence_after();
                const long long m = (long long)t * kTileM + row;
                const uint32_t lane_base = tmem + uint32_t(acc * BN) + (uint32_t(quarter * 32) << 16);
#pragma unroll 1
                for (int c0 = cg * 64; c0 < cg * 64 + 64; c0 += 16) {
                    float v[16];
                    tmem_load16(lane_base + uint32_t(c0), v);
                    if (HEAD) {
#pragma unroll
                        for (int i = 0; i < 16; i += 2) {
                            const float h0 = __bfloat162float(__float2bfloat16_rn(
                                gelu_half(fmaf(0.5f, v[i], 0.5f * g.bias[c0 + i]))));
                            const float h1 = __bfloat162float(__float2bfloat16_rn(
                                gelu_half(fmaf(0.5f, v[i + 1], 0.5f * g.bias[c0 + i + 1]))));
                            hsum2 = __ffma2_rn(make_float2(h0, h1),
                                               make_float2(head_w[c0 + i], head_w[c0 + i + 1]), hsum2);
                        }
                    } else {
                        epilogue16<BN, EPI_FORWARD>(g, m, c0, v, BN);
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&t_empty[acc]);
                }
            }
            if (HEAD) {
                head_part[acc][cg][row] = hsum2.x + hsum2.y;
                named_barrier_sync(1, 16 * 32);
                const int et = ew * 32 + lane;       // 0..511
                if (ok && et < kTileM) {
                    const long long m = (long long)t * kTileM + et;
                    if (m < rows_valid) {
                        y[m] = ((head_part[acc][0][et] + head_part[acc][1][et]) +
                                (head_part[acc][2][et] + head_part[acc][3][et])) + head_b[0];
                    }
                }
            }
            // with HEAD every epilogue warp passes the named barrier once per
            // tile of this block, aborted or not; without it a warp may leave
            if (!HEAD && !ok) {
                break;
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && *abort_v) {
        atomicExch(g.error, 1);
    }
    if (warp == 0) {
        __syncwarp();
        tc_fence_after();
        tmem_free(tmem, 2 * BN);
    }
}

// Inference of the whole network in one persistent kernel: every layer of a
// pair of 128-row tiles runs with the activations kept in shared memory.
//   warp 0  TMA producer, in the MMA warp's order: each tile's packed inputs
//           (128 x 64) into the first K chunk of its activation buffer, and
//           every layer's weight matrix, 64-wide K chunk by chunk (256 x 64,
//           32 KB), through a ring of kFusedRing stages;
//   warp 1  MMA issuer: the tiles alternate layer by layer (tile 0 layer l,
//           tile 1 layer l, tile 0 layer l + 1, ...), each into its own TMEM
//           accumulator (2 x 256 columns), so one tile's MMAs run while the
//           epilogue works on the other; the weights stream from L2 once
//           per tile;
//   warps 4..19  epilogue: bias + GELU of one tile's accumulator, BF16,
//           written straight into the tile's activation buffer in the
//           128-byte swizzled K-major layout the next layer's MMAs read (the
//           layout a SWIZZLE_128B TMA load produces); after the last layer
//           the 256 -> 1 head instead, as gemm_tma_forward<NK, true> folds it.
// Each layer's MMAs are issued chunk by chunk, K step by K step, as
// gemm_tma_forward issues them, and the epilogue rounds at the same points,
// so the results equal the per-layer kernels' bit for bit.  The activations
// never leave the SM: per tile only the packed inputs (16 KB) come from HBM
// and the weights (32 KB + 128 KB per hidden layer) from L2.  Every wait is
// bounded; a timeout sets the error flag and the roles drain and return.
constexpr int kFusedRing = 2;
constexpr int kMaxFusedLayers = 6;
constexpr uint32_t kActBytes = kTileM * 256 * 2;         // one tile's activations (64 KB)
constexpr uint32_t kChunkBytes = kTileM * kChunkK * 2;   // one 64-wide K chunk of a tile (16 KB)
constexpr uint32_t kWChunkBytes = 256 * kChunkK * 2;     // one weight K chunk (32 KB)

constexpr int fused_smem_bytes() {
    return int(2 * kActBytes + kFusedRing * kWChunkBytes) + 1024;
}

struct FusedMaps {
    CUtensorMap x;                       // packed inputs (rows x 64), box 64 x 128
    CUtensorMap w[kMaxFusedLayers];      // layer weights (256 x kpad), box 64 x 256
};

struct FusedArgs {
    const float* bias[kMaxFusedLayers];
    int nk[kMaxFusedLayers];             // 64-wide K chunks of each layer
    int layers;
    const float* head_w;
    const float* head_b;
    float* y;
    long long rows_valid;
    int pairs;                           // tile pairs (rows_pad / 256)
    int* error;                          // set to 1 when a wait gave up
    unsigned wait_limit;                 // polls per wait; 0: kWaitLimit
    int withhold_commit;                 // failure-detection test: the layer
                                         // completions are never committed
};

__global__ void __launch_bounds__(kTmaThreads) mlp_forward_fused(const __grid_constant__ FusedMaps maps,
                                                                 const __grid_constant__ FusedArgs g) {
    constexpr int BN = 256;
    extern __shared__ unsigned char smem_raw[];
    __shared__ uint64_t x_full[2];
    __shared__ uint64_t a_free[2];
    __shared__ uint64_t a_ready[2];
    __shared__ uint64_t b_full[kFusedRing];
    __shared__ uint64_t b_empty[kFusedRing];
    __shared__ uint64_t t_full[2];
    __shared__ uint64_t drain;
    __shared__ uint32_t tmem_base;
    __shared__ int abort_flag;
    __shared__ float head_part[2][4][kTileM];
    // the layers' half biases, then the head's weights (read by every row)
    __shared__ __align__(16) float s_par[kMaxFusedLayers + 1][256];
    unsigned char* base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char* sA = base;                       // 2 tiles x 64 KB of activations
    unsigned char* sB = base + 2 * kActBytes;       // kFusedRing x 32 KB of weights
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int L = g.layers;
    const unsigned limit = g.wait_limit ? g.wait_limit : kWaitLimit;
    if (warp == 0) {
        tmem_alloc(&tmem_base, 2 * BN);
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < 2; ++s) {
            mbar_init(&x_full[s], 1);
            mbar_init(&a_free[s], 1);
            mbar_init(&a_ready[s], 16);      // one arrival per epilogue warp
            mbar_init(&t_full[s], 1);
        }
        for (int r = 0; r < kFusedRing; ++r) {
            mbar_init(&b_full[r], 1);
            mbar_init(&b_empty[r], 1);
        }
        mbar_init(&drain, 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = threadIdx.x; i < (L + 1) * 256; i += blockDim.x) {
        const int l = i >> 8;
        s_par[l][i & 255] = l < L ? 0.5f * g.bias[l][i & 255] : g.head_w[i & 255];
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    volatile int* abort_v = &abort_flag;

    if (warp == 0) {
        if (lane == 0) {
            // in the MMA warp's order: per pair, layer and tile, the tile's
            // inputs (first layer) and the layer's weight chunks
            int it = 0;                // weight chunks issued
            int nx[2] = {0, 0};        // input tiles issued, per tile of the pair
            for (int q = blockIdx.x; q < g.pairs && !*abort_v; q += gridDim.x) {
                for (int l = 0; l < L && !*abort_v; ++l) {
                    for (int s = 0; s < 2 && !*abort_v; ++s) {
                        if (l == 0) {
                            // the previous pair's last MMAs of this tile are done
                            if (nx[s] > 0 &&
                                !mbar_wait(&a_free[s], unsigned((nx[s] - 1) & 1), limit)) {
                                *abort_v = 1;
                                break;
                            }
                            mbar_expect_tx(&x_full[s], kChunkBytes);
                            tma_load_2d(sA + s * kActBytes, &maps.x, 0, (2 * q + s) * kTileM,
                                        &x_full[s]);
                            ++nx[s];
                        }
                        for (int c = 0; c < g.nk[l]; ++c, ++it) {
                            const int slot = it % kFusedRing;
                            if (it >= kFusedRing &&
                                !mbar_wait(&b_empty[slot], unsigned((it / kFusedRing - 1) & 1),
                                           limit)) {
                                *abort_v = 1;
                                break;
                            }
                            mbar_expect_tx(&b_full[slot], kWChunkBytes);
                            tma_load_2d(sB + slot * kWChunkBytes, &maps.w[l], c * kChunkK, 0,
                                        &b_full[slot]);
                        }
                    }
                }
            }
            // copies still in flight (an aborted run) land before the block exits
            for (int r = 0; r < kFusedRing; ++r) {
                const int n = it > r ? (it - r + kFusedRing - 1) / kFusedRing : 0;
                if (n > 0) {
                    mbar_wait(&b_full[r], unsigned((n - 1) & 1));
                }
            }
            for (int s = 0; s < 2; ++s) {
                if (nx[s] > 0) {
                    mbar_wait(&x_full[s], unsigned((nx[s] - 1) & 1));
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // tiles alternate: while the epilogue works on one tile, the
            // other tile's next layer runs on the tensor core
            const uint32_t idesc = instr_desc_bf16(kTileM, BN);
            bool ok = true;
            int it = 0;
            int pi = 0;
            for (int q = blockIdx.x; ok && q < g.pairs && !*abort_v; q += gridDim.x, ++pi) {
                for (int l = 0; ok && l < L; ++l) {
                    const int k = pi * L + l;          // layer passes of each tile
                    for (int s = 0; ok && s < 2; ++s) {
                        if (l == 0) {
                            ok = mbar_wait(&x_full[s], unsigned(pi & 1), limit);
                        }
                        // the epilogue has read this tile's accumulator and
                        // written the layer's input activations
                        if (ok && k > 0) {
                            ok = mbar_wait(&a_ready[s], unsigned((k - 1) & 1), limit);
                        }
                        if (!ok) {
                            break;
                        }
                        tc_fence_after();
                        const uint32_t d = tmem + uint32_t(s * BN);
                        for (int c = 0; c < g.nk[l]; ++c, ++it) {
                            const int slot = it % kFusedRing;
                            if (!mbar_wait(&b_full[slot], unsigned((it / kFusedRing) & 1), limit)) {
                                ok = false;
                                break;
                            }
                            tc_fence_after();
                            const uint32_t b0 = smem_u32(sB + slot * kWChunkBytes);
                            const uint32_t a0 = smem_u32(sA + s * kActBytes + c * kChunkBytes);
#pragma unroll
                            for (int j = 0; j < kChunkK / 16; ++j) {
                                mma_bf16(d, smem_desc_sw128(a0 + j * 32), smem_desc_sw128(b0 + j * 32),
                                         idesc, (c > 0 || j > 0) ? 1u : 0u);
                            }
                            mma_commit(&b_empty[slot]);
                        }
                        if (!ok) {
                            break;
                        }
                        if (!g.withhold_commit) {
                            mma_commit(&t_full[s]);
                        }
                        if (l == L - 1) {
                            mma_commit(&a_free[s]);
                        }
                    }
                }
            }
            if (!ok) {
                *abort_v = 1;
            }
            // every MMA this thread issued is complete before TMEM is freed
            mma_commit(&drain);
            mbar_wait(&drain, 0);
        }
    } else if (warp >= kEpiWarp0) {
        const int ew = warp - kEpiWarp0;          // 0..15
        const int quarter = warp & 3;             // TMEM lanes 32 quarter .. + 31
        const int cg = ew >> 2;                   // columns 64 cg .. + 63
        const int row = quarter * 32 + lane;
        const float* head_w = s_par[L];
        int pi = 0;
        for (int q = blockIdx.x; q < g.pairs; q += gridDim.x, ++pi) {
            for (int l = 0; l < L; ++l) {
                const int k = pi * L + l;
                const bool last = l == L - 1;
                const float* bias = s_par[l];
#pragma unroll 1
                for (int s = 0; s < 2; ++s) {
                    bool ok = !*abort_v && mbar_wait(&t_full[s], unsigned(k & 1), limit);
                    ok = __all_sync(0xffffffffu, ok);
                    if (!ok) {
                        *abort_v = 1;
                    } else {
                        tc_fence_after();
                        const uint32_t lane_base =
                            tmem + uint32_t(s * BN) + (uint32_t(quarter * 32) << 16);
                        // this row of every K chunk: 8-row atoms of 1024 bytes
                        unsigned char* arow = sA + s * kActBytes + (row >> 3) * 1024 + (row & 7) * 128;
                        // head: even and odd columns summed apart, then added
                        float2 hsum2 = make_float2(0.0f, 0.0f);
                        // 16 columns at a time; the next 16 are read from TMEM
                        // while these are computed
                        uint32_t r[2][16];
                        const int sw = (row & 7) << 4;        // this row's 16-byte unit swizzle
                        unsigned char* chunk = arow + cg * kChunkBytes;
                        tmem_load16_start(lane_base + uint32_t(cg * 64), r[0]);
                        // pairs of columns: half pre-activation, GELU and BF16
                        // rounding (each element as the scalar operations round it)
                        if (!last) {
                            // into the next layer's K chunk cg: 16-byte units 2j
                            // and 2j + 1 of this row, swizzled within its 8-row atom
#pragma unroll
                            for (int j = 0; j < 4; ++j) {
                                tmem_load_wait(r[j & 1]);
                                if (j < 3) {
                                    tmem_load16_start(lane_base + uint32_t(cg * 64 + 16 * (j + 1)),
                                                      r[(j + 1) & 1]);
                                }
                                const float* bj = bias + cg * 64 + 16 * j;
                                __nv_bfloat162 hb[8];
#pragma unroll
                                for (int i = 0; i < 8; ++i) {
                                    const float2 acc = make_float2(__uint_as_float(r[j & 1][2 * i]),
                                                                   __uint_as_float(r[j & 1][2 * i + 1]));
                                    const float2 hz = __ffma2_rn(make_float2(0.5f, 0.5f), acc,
                                                                 reinterpret_cast<const float2*>(bj)[i]);
                                    const float2 h = gelu_half2(hz);
                                    hb[i] = __floats2bfloat162_rn(h.x, h.y);
                                }
                                *reinterpret_cast<uint4*>(chunk + (((2 * j) << 4) ^ sw)) =
                                    reinterpret_cast<const uint4*>(hb)[0];
                                *reinterpret_cast<uint4*>(chunk + (((2 * j + 1) << 4) ^ sw)) =
                                    reinterpret_cast<const uint4*>(hb)[1];
                            }
                        } else {
                            // the 256 -> 1 head: the rounded activations times the
                            // head's weights, even and odd columns summed apart
#pragma unroll
                            for (int j = 0; j < 4; ++j) {
                                tmem_load_wait(r[j & 1]);
                                if (j < 3) {
                                    tmem_load16_start(lane_base + uint32_t(cg * 64 + 16 * (j + 1)),
                                                      r[(j + 1) & 1]);
                                }
                                const float* bj = bias + cg * 64 + 16 * j;
                                const float* wj = head_w + cg * 64 + 16 * j;
#pragma unroll
                                for (int i = 0; i < 8; ++i) {
                                    const float2 acc = make_float2(__uint_as_float(r[j & 1][2 * i]),
                                                                   __uint_as_float(r[j & 1][2 * i + 1]));
                                    const float2 hz = __ffma2_rn(make_float2(0.5f, 0.5f), acc,
                                                                 reinterpret_cast<const float2*>(bj)[i]);
                                    const float2 h = gelu_half2(hz);
                                    const __nv_bfloat162 hb = __floats2bfloat162_rn(h.x, h.y);
                                    hsum2 = __ffma2_rn(__bfloat1622float2(hb),
                                                       reinterpret_cast<const float2*>(wj)[i], hsum2);
                                }
                            }
                        }
                        if (last) {
                            head_part[s][cg][row] = hsum2.x + hsum2.y;
                        }
                    }
                    if (last) {
                        // every epilogue warp passes this barrier once per tile, aborted or not
                        named_barrier_sync(1, 16 * 32);
                        const int et = ew * 32 + lane;       // 0..511
                        if (!*abort_v && et < kTileM) {
                            const long long m = (long long)(2 * q + s) * kTileM + et;
                            if (m < g.rows_valid) {
                                g.y[m] = ((head_part[s][0][et] + head_part[s][1][et]) +
                                          (head_part[s][2][et] + head_part[s][3][et])) + g.head_b[0];
                            }
                        }
                    }
                    // the accumulator is read, and this layer's outputs visible to
                    // the tensor core, before the tile's next layer is issued
                    tc_fence_before();
                    fence_async_shared();
                    __syncwarp();
                    if (lane == 0) {
                        mbar_arrive(&a_ready[s]);
                    }
                }
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && *abort_v) {
        atomicExch(g.error, 1);
    }
    if (warp == 0) {
        __syncwarp();
        tc_fence_after();
        tmem_free(tmem, 2 * BN);
    }
}

// x (rows x nin, FP32) -> xb (rows_pad x kpad, BF16), zero padded; one
// 16-byte store of 8 values per work item.
__global__ void pack_inputs(const float* __restrict__ x, long long rows, int nin,
                            __nv_bfloat16* __restrict__ xb, long long rows_pad, int kpad) {
    const int groups = kpad >> 3;
    const long long total = rows_pad * groups;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / groups;
        const int k0 = int(i - r * groups) * 8;
        __align__(16) __nv_bfloat16 v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int k = k0 + j;
            v[j] = __float2bfloat16_rn((r < rows && k < nin) ? x[r * nin + k] : 0.0f);
        }
        *reinterpret_cast<uint4*>(xb + r * kpad + k0) = *reinterpret_cast<const uint4*>(v);
    }
}

// y[r] = sum_i h[r][i] * w[i] + b (one warp per row, FP32).
__global__ void head_forward(const __nv_bfloat16* __restrict__ h, int width,
                             const float* __restrict__ w, const float* __restrict__ b,
                             long long rows, float* __restrict__ y) {
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long r = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); r < rows;
         r += warps) {
        float acc = 0.0f;
        for (int i = lane; i < width; i += 32) {
            acc += __bfloat162float(h[r * width + i]) * w[i];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            acc += __shfl_xor_sync(0xffffffffu, acc, o);
        }
        if (lane == 0) {
            y[r] = acc + b[0];
        }
    }
}

// One training step begins: Adam step counter + 1, loss slot cleared.
__global__ void begin_step(long long* step, float* loss, long long base) {
    const long long t = ++step[0];
    if (loss) {
        loss[t - base - 1] = 0.0f;
    }
}

// MSE head backward: dy = 2 (y - t) / B; dZ = bf16(dy * w * gelu'(Z)); loss
// accumulated into loss[step - base - 1] (block partial sums, atomics).
__global__ void head_backward(const float* __restrict__ y, const float* __restrict__ t, int rows,
                              const float* __restrict__ w, const float* __restrict__ z, int width,
                              float* __restrict__ dy, __nv_bfloat16* __restrict__ dz,
                              const long long* step, float* loss, long long base) {
    __shared__ float part[8];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int r = blockIdx.x * (blockDim.x >> 5) + wib;
    float sq = 0.0f;
    if (r < rows) {
        const float res = y[r] - t[r];
        const float d = 2.0f * res / float(rows);
        sq = res * res;
        if (lane == 0) {
            dy[r] = d;
        }
        for (int i = lane; i < width; i += 32) {
            dz[(long long)r * width + i] =
                __float2bfloat16_rn(d * w[i] * gelu_grad(z[(long long)r * width + i]));
        }
    }
    if (lane == 0) {
        part[wib] = sq;
    }
    __syncthreads();
    if (threadIdx.x == 0 && loss) {
        float s = 0.0f;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            s += part[i];
        }
        atomicAdd(&loss[step[0] - base - 1], s / float(rows));
    }
}

// out[split][n] = sum over rows [split*rows_per_split, ...) of wt[r] * X[r][n]
// (wt null: weights 1), deterministic order; sum_splits adds the splits.
// Block: 32 columns x 8 row groups; grid (columns / 32, splits).
template <typename T>
__global__ void column_sums(const T* __restrict__ x, int rows, int cols, long long ld,
                            const float* __restrict__ wt, float* __restrict__ out,
                            int rows_per_split) {
    __shared__ float part[8][33];
    const int cx = threadIdx.x & 31;
    const int gy = threadIdx.x >> 5;
    const int n = blockIdx.x * 32 + cx;
    const int r0 = blockIdx.y * rows_per_split;
    const int r1 = r0 + rows_per_split < rows ? r0 + rows_per_split : rows;
    out += (long long)blockIdx.y * cols;
    float acc = 0.0f;
    if (n < cols) {
        for (int r = r0 + gy; r < r1; r += 8) {
            float v;
            if constexpr (sizeof(T) == 2) {
                v = __bfloat162float(x[(long long)r * ld + n]);
            } else {
                v = x[(long long)r * ld + n];
            }
            acc += wt ? wt[r] * v : v;
        }
    }
    part[gy][cx] = acc;
    __syncthreads();
    if (gy == 0 && n < cols) {
        float s = 0.0f;
        for (int i = 0; i < 8; ++i) {
            s += part[i][cx];
        }
        out[n] = s;
    }
}

// out[i] = sum over s < splits of partial[s * count + i], in split order.
__global__ void sum_splits(const float* __restrict__ partial, int splits, long long count,
                           float* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int k = 0; k < splits; ++k) {
            s += partial[k * count + i];
        }
        out[i] = s;
    }
}

// One weight matrix of the network in the flat parameter vector and its
// BF16 copy for the tensor cores.
struct Segment {
    long long w_off;    // W (out x in) in the flat vector
    int out, in, kpad;  // kpad: padded K of the BF16 copy
    __nv_bfloat16* wb;  // null for the FP32 head
};

struct AdamArgs {
    float* p;
    const float* g;
    float* m;
    float* v;
    long long n;
    float lr, beta1, beta2, eps;
    const long long* step;
    Segment seg[8];
    int nseg;
};

__global__ void adam_update(AdamArgs a) {
    const long long t = a.step[0];
    const float c1 = 1.0f - powf(a.beta1, float(t));
    const float c2 = 1.0f - powf(a.beta2, float(t));
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.n;
         i += (long long)gridDim.x * blockDim.x) {
        const float gi = a.g[i];
        const float mi = a.beta1 * a.m[i] + (1.0f - a.beta1) * gi;
        const float vi = a.beta2 * a.v[i] + (1.0f - a.beta2) * gi * gi;
        a.m[i] = mi;
        a.v[i] = vi;
        const float pi = a.p[i] - a.lr * (mi / c1) / (sqrtf(vi / c2) + a.eps);
        a.p[i] = pi;
        for (int s = 0; s < a.nseg; ++s) {
            const Segment& sg = a.seg[s];
            const long long rel = i - sg.w_off;
            if (sg.wb && rel >= 0 && rel < (long long)sg.out * sg.in) {
                const long long o = rel / sg.in;
                const int k = int(rel - o * sg.in);
                sg.wb[o * sg.kpad + k] = __float2bfloat16_rn(pi);
            }
        }
    }
}

// BF16 copies of every weight matrix from the flat FP32 vector.
__global__ void cast_weights(const float* __restrict__ p, Segment sg) {
    const long long total = (long long)sg.out * sg.kpad;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long o = i / sg.kpad;
        const int k = int(i - o * sg.kpad);
        sg.wb[i] = __float2bfloat16_rn(k < sg.in ? p[sg.w_off + o * sg.in + k] : 0.0f);
    }
}

// Counter-based U[0,1) draws (splitmix64 finaliser of (seed, index)),
// 24-bit mantissa so every value is exact in FP32.
__global__ void sample_uniform(float* __restrict__ x, long long count, unsigned long long seed) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        x[i] = float(z >> 40) * (1.0f / 16777216.0f);
    }
}

} // namespace mlpk
