// C ABI of the MLP surrogate (include/als_surrogate.h): parameter layout,
// workspaces, the training step as one captured CUDA graph, inference in
// row chunks.  The kernels are in mlp_kernels.cuh / mlp_tc.cuh.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "als_surrogate.h"
#include "mlp_kernels.cuh"

namespace als {
int report_error(int code, const char* msg);
}

using namespace mlpk;

namespace {

// Rows per inference chunk (a multiple of 256).  The per-layer path keeps
// 0.6 KB of BF16 workspace per chunk row (packed inputs and two activation
// buffers), the whole-network kernel 0.25 KB (two packed-input buffers).
// Measured on the 2^20-row forward call through the per-layer path:
// 65,536 rows 1.84 ms, 262,144 1.39 ms, 1,048,576 1.30 ms; the whole-network
// kernel takes 0.58 ms with 262,144-row chunks, the packing of each chunk
// after the first hidden behind the previous one.
#ifndef ALS_MLP_INFER_CHUNK
#define ALS_MLP_INFER_CHUNK 262144
#endif
constexpr long long kInferChunk = ALS_MLP_INFER_CHUNK;
constexpr int kMaxSplits = 16;             // K splits of a weight gradient, row splits of a column sum

int mlp_fail(int code, const std::string& msg) {
    return als::report_error(code, msg.c_str());
}

#define MLP_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t err_ = (call);                                                      \
        if (err_ != cudaSuccess) {                                                      \
            std::ostringstream os_;                                                     \
            os_ << #call << ": " << cudaGetErrorString(err_);                           \
            return mlp_fail(ALS_E_CUDA, os_.str());                                     \
        }                                                                               \
    } while (0)

struct Layer {
    int in, out, kpad;      // kpad: K of the BF16 copy (multiple of 64)
    long long w_off, b_off; // offsets in the flat vector
    __nv_bfloat16* wb;      // BF16 weights (out x kpad), null for the head
};

int round_up(int v, int m) {
    return (v + m - 1) / m * m;
}

} // namespace

struct als_mlp {
    als_mlp_config cfg;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    std::vector<Layer> layers;      // hidden layers then the head
    long long nparams = 0;
    float* p = nullptr;             // master parameters
    float* g = nullptr;             // gradients
    float* m = nullptr;             // Adam moments
    float* v = nullptr;
    long long* step = nullptr;      // Adam step counter (device)
    int* error = nullptr;           // set by a GEMM whose wait gave up
    unsigned wait_limit = 0;        // als_mlp_test_wait_timeout
    int withhold_commit = 0;
    // training workspace (max_batch rows)
    __nv_bfloat16* xb = nullptr;    // packed inputs (rows x kpad0)
    std::vector<float*> z;          // pre-activations per hidden layer
    std::vector<__nv_bfloat16*> h;  // activations per hidden layer
    __nv_bfloat16* dz[2] = {nullptr, nullptr};
    float* y = nullptr;
    float* dy = nullptr;
    float* loss1 = nullptr;         // loss of a gradient evaluation
    float* split_scratch = nullptr; // K-split partial weight gradients
    float* col_scratch = nullptr;   // row-split partial column sums
    // inference workspace (kInferChunk rows)
    __nv_bfloat16* xi = nullptr;
    __nv_bfloat16* hi[2] = {nullptr, nullptr};
    // tensor maps of the inference operands (width 256): packed inputs, the
    // two activation buffers, every hidden weight matrix
    bool tma = false;
    CUtensorMap tm_x, tm_h[2], tm_w[6];
    // the whole-network inference kernel: its maps over either packed-input
    // buffer (xi, xi2) and the hidden weights; the side stream packs the
    // next chunk's inputs while the network runs on the current one
    bool fused = false;
    FusedMaps fmaps[2];
    CUtensorMap tm_x2;
    __nv_bfloat16* xi2 = nullptr;
    cudaStream_t side = nullptr;
    cudaEvent_t packed[2] = {nullptr, nullptr};
    cudaEvent_t xi_free[2] = {nullptr, nullptr};
    std::vector<void*> allocations;
};

namespace {

template <typename T>
int dev_alloc(als_mlp* s, T** p, size_t count) {
    MLP_CUDA(cudaMalloc((void**)p, count * sizeof(T)));
    MLP_CUDA(cudaMemset(*p, 0, count * sizeof(T)));
    s->allocations.push_back(*p);
    return ALS_OK;
}

#define MLP_TRY(expr)             \
    do {                          \
        int rc_ = (expr);         \
        if (rc_ != ALS_OK) {      \
            return rc_;           \
        }                         \
    } while (0)

// The error flag and wait settings every tcgen05 GEMM of `s` receives.
void arm(const als_mlp* s, GemmArgs& a) {
    a.error = s->error;
    a.wait_limit = s->wait_limit;
    a.withhold_commit = s->withhold_commit;
}

int grid_for(long long work, int threads) {
    long long b = (work + threads - 1) / threads;
    return int(b < 1 ? 1 : (b > 148LL * 16 ? 148LL * 16 : b));
}

template <int BN, int EPI>
int launch_gemm(const GemmArgs& a, int n_valid, cudaStream_t s, int splits = 1) {
    if (a.M % kTileM || a.N % BN || a.K % kChunkK || a.K <= 0 || splits < 1 || splits > 65535) {
        return mlp_fail(ALS_E_INVALID, "GEMM shape is not a multiple of the tile");
    }
    constexpr int smem = gemm_smem_bytes<BN>();   // limit set by configure_kernels()
    dim3 grid(a.M / kTileM, a.N / BN, splits);
    gemm_kernel<BN, EPI><<<grid, kThreads, smem, s>>>(a, n_valid);
    MLP_CUDA(cudaGetLastError());
    return ALS_OK;
}

Operand rows_of(const __nv_bfloat16* p, long long ld) {
    return Operand{p, ld, 1};
}

Operand columns_of(const __nv_bfloat16* p, long long ld) {
    return Operand{p, 1, ld};
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// BF16 matrix rows x cols (row-major, cols contiguous) as a 2-D tensor map
// with a box of box_rows x 64 elements and 128-byte swizzle.
int encode_bf16_map(CUtensorMap* map, const void* base, long long rows, int cols, int box_rows) {
    static EncodeTiledFn encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
                cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) {
            return mlp_fail(ALS_E_CUDA, "cuTensorMapEncodeTiled is not available");
        }
        encode = reinterpret_cast<EncodeTiledFn>(fn);
    }
    const cuuint64_t dims[2] = {cuuint64_t(cols), cuuint64_t(rows)};
    const cuuint64_t strides[1] = {cuuint64_t(cols) * 2};
    const cuuint32_t box[2] = {cuuint32_t(kChunkK), cuuint32_t(box_rows)};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base),
                              dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        return mlp_fail(ALS_E_CUDA, "cuTensorMapEncodeTiled failed");
    }
    return ALS_OK;
}

// Tensor maps of the inference path; only the 256-wide network with K of 64
// (inputs) and 256 (hidden) takes it.
int setup_tma(als_mlp* s) {
    s->tma = false;
    if (s->cfg.width != 256 || s->layers[0].kpad != 64) {
        return ALS_OK;
    }
    MLP_TRY(encode_bf16_map(&s->tm_x, s->xi, kInferChunk, 64, kTileM));
    MLP_TRY(encode_bf16_map(&s->tm_h[0], s->hi[0], kInferChunk, 256, kTileM));
    MLP_TRY(encode_bf16_map(&s->tm_h[1], s->hi[1], kInferChunk, 256, kTileM));
    for (int l = 0; l < s->cfg.hidden; ++l) {
        MLP_TRY(encode_bf16_map(&s->tm_w[l], s->layers[l].wb, 256, s->layers[l].kpad, 256));
    }
    s->tma = true;
    MLP_TRY(encode_bf16_map(&s->tm_x2, s->xi2, kInferChunk, 64, kTileM));
    s->fmaps[0].x = s->tm_x;
    s->fmaps[1].x = s->tm_x2;
    for (int l = 0; l < s->cfg.hidden; ++l) {
        s->fmaps[0].w[l] = s->tm_w[l];
        s->fmaps[1].w[l] = s->tm_w[l];
    }
    s->fused = kInferChunk % (2 * kTileM) == 0;
    return ALS_OK;
}

int sm_count(int* sms) {
    static int cached = 0;
    if (!cached) {
        int dev = 0;
        MLP_CUDA(cudaGetDevice(&dev));
        MLP_CUDA(cudaDeviceGetAttribute(&cached, cudaDevAttrMultiProcessorCount, dev));
    }
    *sms = cached;
    return ALS_OK;
}

// The whole network over `rows_pad` packed rows (a multiple of 256) of
// packed-input buffer `b` (s->xi, s->xi2) in one launch; y[r] for
// r < rows_valid.
int launch_fused_forward(als_mlp* s, int b, long long rows_pad, long long rows_valid, float* y,
                         cudaStream_t st) {
    FusedArgs f = {};
    for (int l = 0; l < s->cfg.hidden; ++l) {
        f.bias[l] = s->p + s->layers[l].b_off;
        f.nk[l] = s->layers[l].kpad / kChunkK;
    }
    const Layer& head = s->layers[s->cfg.hidden];
    f.layers = s->cfg.hidden;
    f.head_w = s->p + head.w_off;
    f.head_b = s->p + head.b_off;
    f.y = y;
    f.rows_valid = rows_valid;
    f.pairs = int(rows_pad / (2 * kTileM));
    f.error = s->error;
    f.wait_limit = s->wait_limit;
    f.withhold_commit = s->withhold_commit;
    int sms = 0;
    MLP_TRY(sm_count(&sms));
    mlp_forward_fused<<<f.pairs < sms ? f.pairs : sms, kTmaThreads, fused_smem_bytes(), st>>>(
        s->fmaps[b], f);
    MLP_CUDA(cudaGetLastError());
    return ALS_OK;
}

template <int NK, bool HEAD>
int launch_tma_forward(const CUtensorMap& a, const CUtensorMap& b, const GemmArgs& g,
                       const float* head_w, const float* head_b, float* y, long long rows_valid,
                       cudaStream_t st) {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        MLP_CUDA(cudaGetDevice(&dev));
        MLP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    }
    const int tiles = g.M / kTileM;
    gemm_tma_forward<NK, HEAD><<<tiles < sms ? tiles : sms, kTmaThreads, gemm_tma_smem_bytes(),
                                 st>>>(a, b, g, head_w, head_b, y, rows_valid);
    MLP_CUDA(cudaGetLastError());
    return ALS_OK;
}

// Forward pass of `rows_pad` rows (multiple of 128) from packed inputs `x`
// through the hidden layers into `hout` (the last activation), storing
// pre-activations when `zs` is given (training), ping-ponging `hbuf`
// otherwise (inference).
int forward_hidden(als_mlp* s, const __nv_bfloat16* x, long long rows_pad,
                   const std::vector<float*>* zs, const std::vector<__nv_bfloat16*>* hs,
                   __nv_bfloat16* const* hbuf, const __nv_bfloat16** hout, cudaStream_t st,
                   float* y_fused = nullptr, long long rows_valid = 0) {
    const int nh = s->cfg.hidden;
    const __nv_bfloat16* in = x;
    long long ld_in = s->layers[0].kpad;
    for (int l = 0; l < nh; ++l) {
        const Layer& L = s->layers[l];
        GemmArgs a = {};
        a.a = rows_of(in, ld_in);
        a.b = rows_of(L.wb, L.kpad);
        a.M = int(rows_pad);
        a.N = L.out;
        a.K = L.kpad;
        a.bias = s->p + L.b_off;
        a.z = zs ? (*zs)[l] : nullptr;
        a.h = hs ? (*hs)[l] : hbuf[l & 1];
        a.ldz = L.out;
        a.ldh = L.out;
        arm(s, a);
        // training batches: narrow N tiles for more CTAs; inference: the
        // whole layer width per CTA, so each activation tile is read once
        if (!zs && s->tma) {
            // inference, 256 wide: TMA-fed tiles (K = 64 inputs, K = 256
            // hidden); the last layer also applies the output head when the
            // caller passes y_fused
            const CUtensorMap& ta = l == 0 ? s->tm_x : s->tm_h[(l - 1) & 1];
            const Layer& head = s->layers[nh];
            const bool fuse = y_fused && l == nh - 1;
            const float* hw = s->p + head.w_off;
            const float* hb = s->p + head.b_off;
            if (L.kpad == 64) {
                MLP_TRY(fuse ? (launch_tma_forward<1, true>(ta, s->tm_w[l], a, hw, hb, y_fused, rows_valid, st))
                             : (launch_tma_forward<1, false>(ta, s->tm_w[l], a, hw, hb, nullptr, 0, st)));
            } else {
                MLP_TRY(fuse ? (launch_tma_forward<4, true>(ta, s->tm_w[l], a, hw, hb, y_fused, rows_valid, st))
                             : (launch_tma_forward<4, false>(ta, s->tm_w[l], a, hw, hb, nullptr, 0, st)));
            }
        } else if (zs || L.out % 128 != 0) {
            MLP_TRY((launch_gemm<64, EPI_FORWARD>(a, L.out, st)));
        } else if (L.out % 256 != 0) {
            MLP_TRY((launch_gemm<128, EPI_FORWARD>(a, L.out, st)));
        } else {
            MLP_TRY((launch_gemm<256, EPI_FORWARD>(a, L.out, st)));
        }
        in = a.h;
        ld_in = L.out;
    }
    *hout = in;
    return ALS_OK;
}

int check_error_flag(als_mlp* s) {
    int e = 0;
    MLP_CUDA(cudaMemcpyAsync(&e, s->error, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    MLP_CUDA(cudaStreamSynchronize(s->stream));
    if (e) {
        cudaMemsetAsync(s->error, 0, sizeof(int), s->stream);
        return mlp_fail(ALS_E_CUDA, "tensor-core GEMM wait timed out");
    }
    return ALS_OK;
}

// The caller's stream waits for nothing of ours and we wait for the caller's
// prior work: work is ordered caller -> ours via an event.
int join_caller(als_mlp* s, void* stream) {
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    MLP_CUDA(cudaEventRecord(s->ev, cs));
    MLP_CUDA(cudaStreamWaitEvent(s->stream, s->ev, 0));
    return ALS_OK;
}

} // namespace

namespace {

// Column sums of a rows x cols matrix (weighted by wt when given) into out:
// row splits on separate blocks, then the splits added in order.
template <typename T>
int col_sums(als_mlp* s, const T* x, int rows, int cols, long long ld, const float* wt, float* out,
             cudaStream_t st) {
    int splits = kMaxSplits;
    if (rows < 8 * splits) {
        splits = std::max(1, rows / 8);
    }
    const int per = (rows + splits - 1) / splits;
    dim3 grid((cols + 31) / 32, splits);
    column_sums<T><<<grid, 256, 0, st>>>(x, rows, cols, ld, wt, s->col_scratch, per);
    sum_splits<<<grid_for(cols, 256), 256, 0, st>>>(s->col_scratch, splits, cols, out);
    MLP_CUDA(cudaGetLastError());
    return ALS_OK;
}

// Largest divisor of the K chunks (K / 64) not above kMaxSplits.
int k_splits(long long K) {
    const long long chunks = K / kChunkK;
    for (int sp = kMaxSplits; sp > 1; --sp) {
        if (chunks % sp == 0) {
            return sp;
        }
    }
    return 1;
}

// Forward + MSE backward of one batch (rows <= max_batch), gradients into
// s->g.  `loss`/`base` select where the loss goes (see head_backward).
int enqueue_gradients(als_mlp* s, const float* x, const float* t, int rows, float* loss,
                      long long base, cudaStream_t st) {
    const int nh = s->cfg.hidden;
    const int W = s->cfg.width;
    const long long rp = round_up(rows, kTileM);
    const Layer& L0 = s->layers[0];
    const Layer& head = s->layers[nh];
    pack_inputs<<<grid_for(rp * (L0.kpad / 8), 256), 256, 0, st>>>(x, rows, s->cfg.inputs, s->xb, rp,
                                                             L0.kpad);
    MLP_CUDA(cudaGetLastError());
    const __nv_bfloat16* last = nullptr;
    MLP_TRY(forward_hidden(s, s->xb, rp, &s->z, &s->h, nullptr, &last, st));
    head_forward<<<grid_for(rows * 32LL, 256), 256, 0, st>>>(last, W, s->p + head.w_off,
                                                              s->p + head.b_off, rows, s->y);
    MLP_CUDA(cudaGetLastError());
    // rows beyond `rows` in the padded batch must not contribute: their
    // dZ rows are zeroed once here (the GEMMs read full 128-row tiles)
    if (rp > rows) {
        for (int k = 0; k < 2; ++k) {
            MLP_CUDA(cudaMemsetAsync(s->dz[k] + (long long)rows * W, 0,
                                     sizeof(__nv_bfloat16) * (rp - rows) * W, st));
        }
    }
    head_backward<<<(rows + 7) / 8, 256, 0, st>>>(s->y, t, rows, s->p + head.w_off, s->z[nh - 1], W,
                                                  s->dy, s->dz[(nh - 1) & 1], s->step, loss, base);
    MLP_CUDA(cudaGetLastError());
    // head gradients: dw = sum_r dy_r h_r, db = sum_r dy_r
    MLP_TRY(col_sums<__nv_bfloat16>(s, last, rows, W, W, s->dy, s->g + head.w_off, st));
    MLP_TRY(col_sums<float>(s, s->dy, rows, 1, 1, nullptr, s->g + head.b_off, st));
    for (int l = nh - 1; l >= 0; --l) {
        const Layer& L = s->layers[l];
        const __nv_bfloat16* dzl = s->dz[l & 1];
        const __nv_bfloat16* hin = l > 0 ? s->h[l - 1] : s->xb;
        const long long ld_in = l > 0 ? s->layers[l - 1].out : L0.kpad;
        // dW = dZ^T H_in : M = out, N = kpad(in), K = rows (padded rows are zero in dZ)
        // K (the batch) split over CTAs; the partial products are added in
        // split order by sum_splits
        const int splits = k_splits(rp);
        GemmArgs a = {};
        a.a = columns_of(dzl, L.out);
        a.b = columns_of(hin, ld_in);
        a.M = L.out;
        a.N = L.kpad;
        a.K = int(rp / splits);
        a.g = s->split_scratch;
        a.ldg = L.in;
        a.split_stride = (long long)L.out * L.in;
        arm(s, a);
        MLP_TRY((launch_gemm<64, EPI_WGRAD>(a, L.in, st, splits)));
        sum_splits<<<grid_for((long long)L.out * L.in, 256), 256, 0, st>>>(
            s->split_scratch, splits, (long long)L.out * L.in, s->g + L.w_off);
        MLP_CUDA(cudaGetLastError());
        MLP_TRY(col_sums<__nv_bfloat16>(s, dzl, rows, L.out, L.out, nullptr, s->g + L.b_off, st));
        if (l > 0) {
            // dZ_{l-1} = (dZ_l W_l) * gelu'(Z_{l-1}) : M = rows, N = in, K = out
            GemmArgs b = {};
            b.a = rows_of(dzl, L.out);
            b.b = columns_of(L.wb, L.kpad);
            b.M = int(rp);
            b.N = L.in;
            b.K = L.out;
            b.zin = s->z[l - 1];
            b.h = s->dz[(l - 1) & 1];
            b.ldz = L.in;
            b.ldh = L.in;
            arm(s, b);
            MLP_TRY((launch_gemm<64, EPI_BACKWARD>(b, L.in, st)));
        }
    }
    return ALS_OK;
}

int refresh_bf16(als_mlp* s, cudaStream_t st) {
    for (int l = 0; l < s->cfg.hidden; ++l) {
        const Layer& L = s->layers[l];
        Segment sg = {L.w_off, L.out, L.in, L.kpad, L.wb};
        cast_weights<<<grid_for((long long)L.out * L.kpad, 256), 256, 0, st>>>(s->p, sg);
        MLP_CUDA(cudaGetLastError());
    }
    return ALS_OK;
}

template <int BN, int EPI>
int configure_one() {
    MLP_CUDA(cudaFuncSetAttribute(gemm_kernel<BN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  gemm_smem_bytes<BN>()));
    return ALS_OK;
}

// Dynamic shared memory limits of every GEMM instantiation, set on the
// current device before any launch (and before any graph capture).
int configure_kernels() {
    MLP_CUDA(cudaFuncSetAttribute(gemm_tma_forward<1, false>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, gemm_tma_smem_bytes()));
    MLP_CUDA(cudaFuncSetAttribute(gemm_tma_forward<1, true>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, gemm_tma_smem_bytes()));
    MLP_CUDA(cudaFuncSetAttribute(gemm_tma_forward<4, false>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, gemm_tma_smem_bytes()));
    MLP_CUDA(cudaFuncSetAttribute(gemm_tma_forward<4, true>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, gemm_tma_smem_bytes()));
    MLP_CUDA(cudaFuncSetAttribute(mlp_forward_fused, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  fused_smem_bytes()));
    MLP_TRY((configure_one<64, EPI_FORWARD>()));
    MLP_TRY((configure_one<128, EPI_FORWARD>()));
    MLP_TRY((configure_one<256, EPI_FORWARD>()));
    MLP_TRY((configure_one<64, EPI_BACKWARD>()));
    MLP_TRY((configure_one<64, EPI_WGRAD>()));
    return ALS_OK;
}

int reset_adam(als_mlp* s, cudaStream_t st) {
    MLP_CUDA(cudaMemsetAsync(s->m, 0, sizeof(float) * s->nparams, st));
    MLP_CUDA(cudaMemsetAsync(s->v, 0, sizeof(float) * s->nparams, st));
    MLP_CUDA(cudaMemsetAsync(s->step, 0, sizeof(long long), st));
    return ALS_OK;
}

// The whole-network path over `rows` rows: chunk i is packed on the side
// stream into buffer i & 1 while chunk i - 1 runs through the network on
// the main stream.
int forward_fused_chunks(als_mlp* s, const float* x_dev, long long rows, float* y_dev,
                         cudaStream_t st) {
    const Layer& L0 = s->layers[0];
    MLP_CUDA(cudaStreamWaitEvent(s->side, s->ev, 0));   // the caller's prior work
    int i = 0;
    for (long long r0 = 0; r0 < rows; r0 += kInferChunk, ++i) {
        const int b = i & 1;
        const long long n = rows - r0 < kInferChunk ? rows - r0 : kInferChunk;
        const long long rp = (n + 2 * kTileM - 1) / (2 * kTileM) * (2 * kTileM);
        if (i >= 2) {
            MLP_CUDA(cudaStreamWaitEvent(s->side, s->xi_free[b], 0));
        }
        pack_inputs<<<grid_for(rp * (L0.kpad / 8), 256), 256, 0, s->side>>>(
            x_dev + r0 * s->cfg.inputs, n, s->cfg.inputs, b ? s->xi2 : s->xi, rp, L0.kpad);
        MLP_CUDA(cudaGetLastError());
        MLP_CUDA(cudaEventRecord(s->packed[b], s->side));
        MLP_CUDA(cudaStreamWaitEvent(st, s->packed[b], 0));
        MLP_TRY(launch_fused_forward(s, b, rp, n, y_dev + r0, st));
        MLP_CUDA(cudaEventRecord(s->xi_free[b], st));
    }
    return ALS_OK;
}

// Inference in chunks of kInferChunk rows: the input packing, then the
// whole-network kernel when it applies and `fused` is set (the packing of
// the next chunk overlapping the current one), else one launch per layer
// (and the head).
int forward_rows(als_mlp* s, const float* x_dev, long long rows, float* y_dev, void* stream,
                 bool fused) {
    if (!s || rows < 0 || (rows > 0 && (!x_dev || !y_dev))) {
        return mlp_fail(ALS_E_INVALID, "invalid argument");
    }
    MLP_CUDA(cudaSetDevice(s->device));
    MLP_TRY(join_caller(s, stream));
    const cudaStream_t st = s->stream;
    const Layer& L0 = s->layers[0];
    const Layer& head = s->layers[s->cfg.hidden];
    if (fused && s->fused) {
        const int rc = forward_fused_chunks(s, x_dev, rows, y_dev, st);
        if (rc != ALS_OK) {
            // no packing of the caller's inputs outlives a failed call
            cudaStreamSynchronize(s->side);
            return rc;
        }
        return check_error_flag(s);
    }
    for (long long r0 = 0; r0 < rows; r0 += kInferChunk) {
        const long long n = rows - r0 < kInferChunk ? rows - r0 : kInferChunk;
        const long long rp = (n + kTileM - 1) / kTileM * kTileM;
        pack_inputs<<<grid_for(rp * (L0.kpad / 8), 256), 256, 0, st>>>(
            x_dev + r0 * s->cfg.inputs, n, s->cfg.inputs, s->xi, rp, L0.kpad);
        MLP_CUDA(cudaGetLastError());
        const __nv_bfloat16* last = nullptr;
        MLP_TRY(forward_hidden(s, s->xi, rp, nullptr, nullptr, s->hi, &last, st,
                               s->tma ? y_dev + r0 : nullptr, n));
        if (!s->tma) {
            head_forward<<<grid_for(n * 32, 256), 256, 0, st>>>(last, s->cfg.width,
                s->p + head.w_off, s->p + head.b_off, n, y_dev + r0);
            MLP_CUDA(cudaGetLastError());
        }
    }
    return check_error_flag(s);
}

} // namespace

extern "C" {

int als_mlp_create(const als_mlp_config* cfg, int device, als_mlp** out) {
    if (!cfg || !out) {
        return mlp_fail(ALS_E_INVALID, "null argument");
    }
    *out = nullptr;
    const als_mlp_config c = *cfg;
    if (c.inputs < 1 || c.inputs > 64 || !(c.width == 64 || c.width == 128 || c.width == 256) ||
        c.hidden < 1 || c.hidden > 6 || c.max_batch < kTileM || c.max_batch % kTileM) {
        return mlp_fail(ALS_E_INVALID, "invalid MLP configuration (inputs 1..64, width 64/128/256, "
                                       "hidden 1..6, max_batch a positive multiple of 128)");
    }
    MLP_CUDA(cudaSetDevice(device));
    als_mlp* s = new als_mlp();
    s->cfg = c;
    s->device = device;
    auto cleanup = [&](int rc) {
        als_mlp_destroy(s);
        return rc;
    };
    long long off = 0;
    for (int l = 0; l <= c.hidden; ++l) {
        Layer L = {};
        L.in = l == 0 ? c.inputs : c.width;
        L.out = l == c.hidden ? 1 : c.width;
        L.kpad = round_up(L.in, kChunkK);
        L.w_off = off;
        off += (long long)L.in * L.out;
        L.b_off = off;
        off += L.out;
        s->layers.push_back(L);
    }
    s->nparams = off;
    bool made = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) == cudaSuccess &&
        cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking) == cudaSuccess &&
        cudaEventCreateWithFlags(&s->ev, cudaEventDisableTiming) == cudaSuccess;
    for (int b = 0; b < 2 && made; ++b) {
        made = cudaEventCreateWithFlags(&s->packed[b], cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&s->xi_free[b], cudaEventDisableTiming) == cudaSuccess;
    }
    if (!made) {
        return cleanup(mlp_fail(ALS_E_CUDA, "stream/event creation failed"));
    }
    int rc = ALS_OK;
    const size_t B = size_t(c.max_batch);
    const size_t Wd = size_t(c.width);
    rc = rc ? rc : dev_alloc(s, &s->p, s->nparams);
    rc = rc ? rc : dev_alloc(s, &s->g, s->nparams);
    rc = rc ? rc : dev_alloc(s, &s->m, s->nparams);
    rc = rc ? rc : dev_alloc(s, &s->v, s->nparams);
    rc = rc ? rc : dev_alloc(s, &s->step, 1);
    rc = rc ? rc : dev_alloc(s, &s->error, 1);
    rc = rc ? rc : dev_alloc(s, &s->loss1, 1);
    for (int l = 0; l < c.hidden && !rc; ++l) {
        rc = dev_alloc(s, &s->layers[l].wb, size_t(s->layers[l].out) * s->layers[l].kpad);
    }
    rc = rc ? rc : dev_alloc(s, &s->xb, B * s->layers[0].kpad);
    s->z.assign(c.hidden, nullptr);
    s->h.assign(c.hidden, nullptr);
    for (int l = 0; l < c.hidden && !rc; ++l) {
        rc = dev_alloc(s, &s->z[l], B * Wd);
        rc = rc ? rc : dev_alloc(s, &s->h[l], B * Wd);
    }
    rc = rc ? rc : dev_alloc(s, &s->dz[0], B * Wd);
    rc = rc ? rc : dev_alloc(s, &s->dz[1], B * Wd);
    rc = rc ? rc : dev_alloc(s, &s->y, B);
    rc = rc ? rc : dev_alloc(s, &s->split_scratch, size_t(kMaxSplits) * Wd * std::max<size_t>(Wd, 64));
    rc = rc ? rc : dev_alloc(s, &s->col_scratch, size_t(kMaxSplits) * Wd);
    rc = rc ? rc : dev_alloc(s, &s->dy, B);
    rc = rc ? rc : dev_alloc(s, &s->xi, size_t(kInferChunk) * s->layers[0].kpad);
    if (c.width == 256) {
        rc = rc ? rc : dev_alloc(s, &s->xi2, size_t(kInferChunk) * s->layers[0].kpad);
    }
    rc = rc ? rc : dev_alloc(s, &s->hi[0], size_t(kInferChunk) * Wd);
    rc = rc ? rc : dev_alloc(s, &s->hi[1], size_t(kInferChunk) * Wd);
    if (rc) {
        return cleanup(rc);
    }
    rc = configure_kernels();
    rc = rc ? rc : setup_tma(s);
    if (rc) {
        return cleanup(rc);
    }
    *out = s;
    return als_mlp_init(s, 0);
}

int als_mlp_destroy(als_mlp* s) {
    if (!s) {
        return ALS_OK;
    }
    cudaSetDevice(s->device);
    if (s->stream) {
        cudaStreamSynchronize(s->stream);
    }
    if (s->side) {
        cudaStreamSynchronize(s->side);
    }
    for (void* p : s->allocations) {
        cudaFree(p);
    }
    for (cudaEvent_t e : {s->ev, s->packed[0], s->packed[1], s->xi_free[0], s->xi_free[1]}) {
        if (e) {
            cudaEventDestroy(e);
        }
    }
    for (cudaStream_t t : {s->stream, s->side}) {
        if (t) {
            cudaStreamDestroy(t);
        }
    }
    delete s;
    return ALS_OK;
}

int als_mlp_param_count(const als_mlp* s, long long* count) {
    if (!s || !count) {
        return mlp_fail(ALS_E_INVALID, "null argument");
    }
    *count = s->nparams;
    return ALS_OK;
}

int als_mlp_init(als_mlp* s, unsigned long long seed) {
    if (!s) {
        return mlp_fail(ALS_E_INVALID, "null handle");
    }
    std::vector<float> host(size_t(s->nparams));
    std::mt19937_64 engine(seed);
    for (const Layer& L : s->layers) {
        const float bound = 1.0f / std::sqrt(float(L.in));
        std::uniform_real_distribution<float> u(-bound, bound);
        for (long long i = 0; i < (long long)L.in * L.out; ++i) {
            host[size_t(L.w_off + i)] = u(engine);
        }
        for (int i = 0; i < L.out; ++i) {
            host[size_t(L.b_off + i)] = u(engine);
        }
    }
    return als_mlp_set_params(s, host.data());
}

int als_mlp_set_params(als_mlp* s, const float* params) {
    if (!s || !params) {
        return mlp_fail(ALS_E_INVALID, "null argument");
    }
    MLP_CUDA(cudaSetDevice(s->device));
    MLP_CUDA(cudaMemcpyAsync(s->p, params, sizeof(float) * s->nparams, cudaMemcpyHostToDevice,
                             s->stream));
    MLP_TRY(refresh_bf16(s, s->stream));
    MLP_TRY(reset_adam(s, s->stream));
    MLP_CUDA(cudaStreamSynchronize(s->stream));
    return ALS_OK;
}

int als_mlp_get_params(const als_mlp* s, float* params) {
    if (!s || !params) {
        return mlp_fail(ALS_E_INVALID, "null argument");
    }
    MLP_CUDA(cudaSetDevice(s->device));
    MLP_CUDA(cudaMemcpyAsync(params, s->p, sizeof(float) * s->nparams, cudaMemcpyDeviceToHost,
                             s->stream));
    MLP_CUDA(cudaStreamSynchronize(s->stream));
    return ALS_OK;
}

int als_mlp_forward(als_mlp* s, const float* x_dev, long long rows, float* y_dev, void* stream) {
    return forward_rows(s, x_dev, rows, y_dev, stream, true);
}

int als_mlp_forward_layers(als_mlp* s, const float* x_dev, long long rows, float* y_dev,
                           void* stream) {
    return forward_rows(s, x_dev, rows, y_dev, stream, false);
}

int als_mlp_gradients(als_mlp* s, const float* x_dev, const float* t_dev, int rows,
                      float* grad_dev, float* loss, void* stream) {
    if (!s || !x_dev || !t_dev || !grad_dev || rows < 1 || rows > s->cfg.max_batch) {
        return mlp_fail(ALS_E_INVALID, "invalid argument (1 <= rows <= max_batch)");
    }
    MLP_CUDA(cudaSetDevice(s->device));
    MLP_TRY(join_caller(s, stream));
    const cudaStream_t st = s->stream;
    // the loss slot is loss1[step - base - 1] with base = step - 1
    long long stepv = 0;
    MLP_CUDA(cudaMemcpyAsync(&stepv, s->step, sizeof(long long), cudaMemcpyDeviceToHost, st));
    MLP_CUDA(cudaStreamSynchronize(st));
    MLP_CUDA(cudaMemsetAsync(s->loss1, 0, sizeof(float), st));
    MLP_TRY(enqueue_gradients(s, x_dev, t_dev, rows, s->loss1, stepv - 1, st));
    MLP_CUDA(cudaMemcpyAsync(grad_dev, s->g, sizeof(float) * s->nparams, cudaMemcpyDeviceToDevice,
                             st));
    float l = 0.0f;
    MLP_CUDA(cudaMemcpyAsync(&l, s->loss1, sizeof(float), cudaMemcpyDeviceToHost, st));
    MLP_TRY(check_error_flag(s));
    if (loss) {
        *loss = l;
    }
    return ALS_OK;
}

int als_mlp_train(als_mlp* s, const float* x_dev, const float* t_dev, int rows, int steps,
                  float lr, float* loss_dev, void* stream) {
    if (!s || !x_dev || !t_dev || rows < 1 || rows > s->cfg.max_batch || steps < 0 ||
        !(lr > 0.0f)) {
        return mlp_fail(ALS_E_INVALID, "invalid argument (1 <= rows <= max_batch, lr > 0)");
    }
    if (steps == 0) {
        return ALS_OK;
    }
    MLP_CUDA(cudaSetDevice(s->device));
    MLP_TRY(join_caller(s, stream));
    const cudaStream_t st = s->stream;
    long long base = 0;
    MLP_CUDA(cudaMemcpyAsync(&base, s->step, sizeof(long long), cudaMemcpyDeviceToHost, st));
    MLP_CUDA(cudaStreamSynchronize(st));

    AdamArgs a = {};
    a.p = s->p;
    a.g = s->g;
    a.m = s->m;
    a.v = s->v;
    a.n = s->nparams;
    a.lr = lr;
    a.beta1 = 0.9f;
    a.beta2 = 0.999f;
    a.eps = 1e-8f;
    a.step = s->step;
    a.nseg = 0;
    for (int l = 0; l < s->cfg.hidden; ++l) {
        const Layer& L = s->layers[l];
        a.seg[a.nseg++] = Segment{L.w_off, L.out, L.in, L.kpad, L.wb};
    }

    // one training step, captured once and replayed
    cudaGraph_t graph = nullptr;
    MLP_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    begin_step<<<1, 1, 0, st>>>(s->step, loss_dev, base);
    int rc = enqueue_gradients(s, x_dev, t_dev, rows, loss_dev, base, st);
    if (rc == ALS_OK) {
        adam_update<<<grid_for(s->nparams, 256), 256, 0, st>>>(a);
    }
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (rc != ALS_OK || ce != cudaSuccess) {
        if (graph) {
            cudaGraphDestroy(graph);
        }
        return rc != ALS_OK ? rc : mlp_fail(ALS_E_CUDA, "graph capture of the training step failed");
    }
    cudaGraphExec_t exec = nullptr;
    if (cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
        cudaGraphDestroy(graph);
        return mlp_fail(ALS_E_CUDA, "graph instantiation of the training step failed");
    }
    cudaError_t le = cudaSuccess;
    for (int k = 0; k < steps && le == cudaSuccess; ++k) {
        le = cudaGraphLaunch(exec, st);
    }
    const cudaError_t se = cudaStreamSynchronize(st);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (le != cudaSuccess || se != cudaSuccess) {
        return mlp_fail(ALS_E_CUDA, std::string("training step: ") +
                                        cudaGetErrorString(le != cudaSuccess ? le : se));
    }
    return check_error_flag(s);
}

int als_mlp_test_wait_timeout(als_mlp* s, unsigned wait_limit, int withhold_commit) {
    if (!s) {
        return mlp_fail(ALS_E_INVALID, "invalid argument");
    }
    s->wait_limit = wait_limit;
    s->withhold_commit = withhold_commit ? 1 : 0;
    return ALS_OK;
}

int als_mlp_sample_uniform(float* x_dev, long long count, unsigned long long seed, void* stream) {
    if (count < 0 || (count > 0 && !x_dev)) {
        return mlp_fail(ALS_E_INVALID, "invalid argument");
    }
    if (count == 0) {
        return ALS_OK;
    }
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    sample_uniform<<<grid_for(count, 256), 256, 0, st>>>(x_dev, count, seed);
    MLP_CUDA(cudaGetLastError());
    MLP_CUDA(cudaStreamSynchronize(st));
    return ALS_OK;
}

} // extern "C"
