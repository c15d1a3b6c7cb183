// BF16 tensor-core GEMM tile for the MLP surrogate (sm_100a, tcgen05).
//
// One CTA of 128 threads computes a 128 x BN tile of D = A * B^T, where
// A is M x K and B is N x K (both read as "K-major" rows of K elements),
// accumulating in FP32 in tensor memory (TMEM).  Operands go from global
// memory through registers into shared memory in the canonical no-swizzle
// K-major UMMA layout: core matrices of 8 rows x 16 bytes (8 BF16 along K),
// the 8 core matrices of a 64-wide K chunk of one 8-row group contiguous
// (1024 bytes), so the descriptor's leading byte offset (next core matrix
// along K) is 128 bytes and its stride byte offset (next 8-row group) is
// 1024 bytes.  Strided staging lets the same kernel read transposed
// operands (dZ^T, H^T, W^T) for the backward pass without extra copies.
//
// Two shared-memory stages: while the tensor core works on chunk c, the
// threads stage chunk c+1; an mbarrier per stage, arrived on by
// tcgen05.commit, says when a stage may be refilled.  Every wait is
// bounded: on timeout the kernel records an error code, waits once more
// (bounded) for its own MMAs, frees its TMEM and returns.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace mlpk {

constexpr int kTileM = 128;
constexpr int kChunkK = 64;
constexpr int kThreads = 128;
constexpr unsigned kWaitLimit = 1u << 22;   // try_wait polls before giving up

enum Epilogue {
    EPI_FORWARD = 0,    // z = acc + bias; Z = z (optional); H = bf16(gelu(z))
    EPI_BACKWARD = 1,   // dZ = bf16(acc * gelu'(Zin))
    EPI_WGRAD = 2,      // G = acc (FP32)
};

struct Operand {
    const __nv_bfloat16* p;
    long long rs;   // element stride between rows (M or N index)
    long long ks;   // element stride along K
};

struct GemmArgs {
    Operand a, b;
    int M, N, K;                // M % 128 == 0, N % BN == 0, K % 64 == 0
    const float* bias;          // EPI_FORWARD
    float* z;                   // EPI_FORWARD (may be null); ld = ldz
    __nv_bfloat16* h;           // EPI_FORWARD / EPI_BACKWARD output; ld = ldh
    const float* zin;           // EPI_BACKWARD: pre-activations; ld = ldz
    float* g;                   // EPI_WGRAD output; ld = ldg
    long long ldz, ldh, ldg;
    long long split_stride;     // EPI_WGRAD: elements between the outputs of K splits
    int* error;                 // set to 1 when a wait gave up
    unsigned wait_limit;        // polls per wait; 0: kWaitLimit
    int withhold_commit;        // failure-detection test: no chunk is committed, so
                                // the waits run out and the error flag is set
};

// GELU in its tanh form (Hendrycks and Gimpel, "Gaussian Error Linear Units",
// 2016): gelu(z) = z/2 (1 + tanh(k (z + a z^3))), k = sqrt(2/pi), a = 0.044715,
// with the hardware tanh (tanh.approx.f32, relative error about 2^-11, below
// the BF16 resolution of the activations it produces).
__device__ __forceinline__ float tanh_hw(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// The argument as z (k + k a z^2) and the value as z/2 + z/2 tanh(u).
__device__ __forceinline__ float gelu_arg(float z) {
    return z * fmaf(0.035677408136300125f, z * z, 0.79788456080286536f);
}

// The GELU of z from hz = z/2: u = hz (2k + 8 k a hz^2) is z (k + k a z^2)
// to the bit (every factor scaled by a power of two), and the value is
// hz + hz tanh(u): four operations around the tanh.  The epilogues form hz
// as fma(1/2, acc, bias/2), which is half of acc + bias exactly.
__device__ __forceinline__ float gelu_half(float hz) {
    const float c = fmaf(8.0f * 0.035677408136300125f, hz * hz, 2.0f * 0.79788456080286536f);
    return fmaf(hz, tanh_hw(hz * c), hz);
}

__device__ __forceinline__ float gelu(float z) {
    return gelu_half(0.5f * z);
}

// gelu_half of two values with the paired FP32 instructions (each component
// rounded as the scalar operation rounds it, so the results are gelu_half's).
__device__ __forceinline__ float2 gelu_half2(float2 hz) {
    const float2 c = __ffma2_rn(make_float2(8.0f * 0.035677408136300125f, 8.0f * 0.035677408136300125f),
                                __fmul2_rn(hz, hz),
                                make_float2(2.0f * 0.79788456080286536f, 2.0f * 0.79788456080286536f));
    const float2 u = __fmul2_rn(hz, c);
    return __ffma2_rn(hz, make_float2(tanh_hw(u.x), tanh_hw(u.y)), hz);
}

__device__ __forceinline__ float gelu_grad(float z) {
    // d/dz: (1 + t)/2 + z/2 (1 - t^2) k (1 + 3 a z^2), t = tanh(u)
    const float t = tanh_hw(gelu_arg(z));
    return 0.5f * (1.0f + t) +
        0.5f * z * (1.0f - t * t) * 0.79788456080286536f * (1.0f + 0.134145f * z * z);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (sm100 format): start address, leading
// and stride byte offsets in 16-byte units, descriptor version 1 at bit 46,
// base offset 0, layout type 0 = no swizzle (bits 61-63).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
        (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1),
// A and B BF16 (bits 7-9 = 1, 10-12 = 1), both K-major, N >> 3 at bit 17,
// M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) |
        (uint32_t(m >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the completion of phase `parity` of `bar`.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity,
                                          unsigned limit = kWaitLimit) {
    for (unsigned i = 0; i < limit; ++i) {
        if (mbar_try_wait(bar, parity)) {
            return true;
        }
    }
    return false;
}

__device__ __forceinline__ void fence_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(dst)), "r"(cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols));
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(bar)) : "memory");
}

// 32 lanes x 32 bits, 16 consecutive columns per thread, without waiting:
// the registers are valid after tmem_load_wait on them.
__device__ __forceinline__ void tmem_load16_start(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// Waits for every TMEM load of this thread; the registers of `r` pass
// through the wait, so no use of them is scheduled before it.
__device__ __forceinline__ void tmem_load_wait(uint32_t* r) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                   "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                   "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
                 :
                 : "memory");
}

// 32 lanes x 32 bits, 16 consecutive columns per thread.
__device__ __forceinline__ void tmem_load16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        v[i] = __uint_as_float(r[i]);
    }
}

// --- TMA (inference path): operands land in shared memory through
// cp.async.bulk.tensor with 128-byte swizzle, the canonical K-major
// SWIZZLE_128B UMMA layout (8 rows x 128 bytes per atom, atoms 1024 bytes
// apart); a K = 16 step advances the descriptor start by 32 bytes.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t(1) << 16) |
        (uint64_t(1024 >> 4) << 32) | (uint64_t(1) << 46) | (uint64_t(2) << 61);
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// 2-D tiled TMA load of box (x = innermost coordinate in elements, y = row)
// into shared memory, completion counted on `bar`.  No multicast.
__device__ __forceinline__ void tma_load_2d(void* dst, const void* tmap, int x, int y,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y),
          "r"(smem_u32(bar))
        : "memory");
}

// Byte offset of element (r, k) of a staged rows x 64 chunk.
__device__ __forceinline__ uint32_t staged_offset(int r, int kc) {
    return uint32_t((r >> 3) * 1024 + kc * 128 + (r & 7) * 16);
}

// Stages rows [row0, row0+ROWS) x K [k0, k0+64) of an operand into `dst`.
template <int ROWS>
__device__ __forceinline__ void stage_operand(unsigned char* dst, const Operand& op, long long row0,
                                              int k0) {
    if (op.ks == 1) {
        // rows of contiguous K: one 16-byte vector per (row, 8-wide K group)
        for (int idx = threadIdx.x; idx < ROWS * 8; idx += kThreads) {
            const int r = idx >> 3;
            const int kc = idx & 7;
            const uint4 v = *reinterpret_cast<const uint4*>(op.p + (row0 + r) * op.rs + k0 + kc * 8);
            *reinterpret_cast<uint4*>(dst + staged_offset(r, kc)) = v;
        }
    } else {
        // transposed operand: consecutive rows are contiguous in memory
        for (int idx = threadIdx.x; idx < ROWS * 8; idx += kThreads) {
            const int r = idx % ROWS;
            const int kc = idx / ROWS;
            const __nv_bfloat16* src = op.p + (row0 + r) * op.rs + (long long)(k0 + kc * 8) * op.ks;
            __align__(16) __nv_bfloat16 e[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                e[j] = src[(long long)j * op.ks];
            }
            *reinterpret_cast<uint4*>(dst + staged_offset(r, kc)) = *reinterpret_cast<uint4*>(e);
        }
    }
}

} // namespace mlpk
