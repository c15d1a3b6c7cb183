// Structure-function statistics of ensemble states on the GPU.
//
// Reference: alsuq/src/stats/StructureCube.cpp:39-75 and
// alsfvm/src/functional/StructureCube.cpp (both through
// alsfvm/include/alsfvm/functional/structure_common.hpp:39-160), and
// alsuq/src/stats/StructureBasic.cpp:74-118.  For every variable,
//   cube:  S[h] = sum_cells sum_{q on the cube surface at distance h} |u - u_q|^p / (nx ny nz),
//          h = 1..H-1 (S[0] = 0);
//   basic: S[h] = sum_cells |u - u(x + h e_direction)|^p / (nx ny nz), h = 0..H-1,
// with points outside the interior wrapped (periodic) or clamped (Neumann),
// alsfvm/include/alsfvm/boundary/ValueAtBoundary.hpp:20-110.  The cube
// surface is walked face by face as the reference does (faces normal to x
// exclude the y edges, faces normal to z exclude the x and y edges), so
// every surface point is counted once: 8h points in 2-D, 24h^2 + 2 in 3-D.
//
// One thread per cell, 256 cells per block; per h the block's sum goes
// through a warp shuffle into shared memory, then into a per-tile partial,
// and a second kernel adds the tiles in a fixed order and divides by the
// cell count once (the reference divides every term, so results agree to
// rounding, not bit for bit).  Deterministic for a given launch shape.
#include <cuda_runtime.h>

#include <algorithm>
#include <sstream>
#include <string>

#include "als_b200.h"
#include "scratch.h"

namespace als {
int report_error(int code, const char* msg);
}

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxH = 512;   // 8 warps x 512 doubles of static shared memory

#define ST_CUDA(call)                                                                    \
    do {                                                                                \
        cudaError_t err_ = (call);                                                      \
        if (err_ != cudaSuccess) {                                                      \
            std::ostringstream os_;                                                     \
            os_ << #call << ": " << cudaGetErrorString(err_);                           \
            return als::report_error(ALS_E_CUDA, os_.str().c_str());                    \
        }                                                                               \
    } while (0)

struct StructGeom {
    int n[3];       // interior cells (1 for inactive directions)
    int g[3];       // ghost width per direction (0 for inactive)
    int N[3];       // padded extents
    long long plane;
    int tile[3];    // cells per block and direction
    int tiles[3];
};

// FastPower<p> (alsutils/math/FastPower.hpp) for p = 1..5, pow otherwise
template<int P>
__device__ __forceinline__ double spow(double x, double p) {
    if (P == 1) {
        return x;
    } else if (P == 2) {
        return x * x;
    } else if (P == 3) {
        return x * (x * x);
    } else if (P == 4) {
        return x * (x * (x * x));
    } else if (P == 5) {
        return x * (x * (x * (x * x)));
    }
    return pow(x, p);
}

template<int BC>
__device__ __forceinline__ int bound(int x, int n) {
    if (BC == ALS_BC_PERIODIC) {
        x %= n;
        return x < 0 ? x + n : x;
    }
    return x < 0 ? 0 : (x > n - 1 ? n - 1 : x);
}

template<int BC>
__device__ __forceinline__ int step(int x, int n) {
    // next coordinate along a run of points, given x already bounded and the
    // unbounded coordinate increasing by one
    if (BC == ALS_BC_PERIODIC) {
        return x + 1 == n ? 0 : x + 1;
    }
    return x;   // Neumann: handled by re-clamping the unbounded coordinate
}

template<class T>
__device__ __forceinline__ double load(const T* p, long long i) {
    return double(__ldg(p + i));
}

// Sum over the points of a run along direction `a` (count points starting at
// unbounded coordinate `s`), the other coordinates fixed at padded offset `base`.
template<class T, int BC, int P>
__device__ __forceinline__ double run_sum(const T* u, double uc, long long base, long long stride,
    int s, int count, int n, int g, double p) {
    double acc = 0;
    if (BC == ALS_BC_PERIODIC) {
        int x = bound<BC>(s, n);
        for (int t = 0; t < count; ++t) {
            acc += spow<P>(fabs(uc - load(u, base + (long long)(x + g) * stride)), p);
            x = step<BC>(x, n);
        }
    } else {
        for (int t = 0; t < count; ++t) {
            const int x = bound<BC>(s + t, n);
            acc += spow<P>(fabs(uc - load(u, base + (long long)(x + g) * stride)), p);
        }
    }
    return acc;
}

template<class T, int DIM, int BC, int P, bool CUBE>
__global__ void __launch_bounds__(kThreads) structure_kernel(const T* __restrict__ states,
    long long member_stride, StructGeom G, int nvar, int direction, int H, double p,
    double* __restrict__ partial) {
    __shared__ double part[kWarps][kMaxH];
    const int member = blockIdx.z;
    const int var = blockIdx.y;
    const int tile = blockIdx.x;
    const int tx = tile % G.tiles[0];
    const int ty = (tile / G.tiles[0]) % G.tiles[1];
    const int tz = tile / (G.tiles[0] * G.tiles[1]);
    const int lx = threadIdx.x % G.tile[0];
    const int ly = (threadIdx.x / G.tile[0]) % G.tile[1];
    const int lz = threadIdx.x / (G.tile[0] * G.tile[1]);
    const int i = tx * G.tile[0] + lx;
    const int j = ty * G.tile[1] + ly;
    const int k = tz * G.tile[2] + lz;
    const bool active = i < G.n[0] && j < G.n[1] && k < G.n[2];
    const T* u = states + (long long)member * member_stride + (long long)var * G.plane;
    const long long sx = 1, sy = G.N[0], sz = (long long)G.N[0] * G.N[1];
    double uc = 0;
    if (active) {
        uc = load(u, (k + G.g[2]) * sz + (j + G.g[1]) * sy + (i + G.g[0]));
    }
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int h0 = CUBE ? 1 : 0;
    for (int h = h0; h < H; ++h) {
        double acc = 0;
        if (active) {
            if (!CUBE) {
                const int x = bound<BC>(i + (direction == 0 ? h : 0), G.n[0]);
                const int y = bound<BC>(j + (direction == 1 ? h : 0), G.n[1]);
                const int z = bound<BC>(k + (direction == 2 ? h : 0), G.n[2]);
                acc = spow<P>(fabs(uc - load(u, (z + G.g[2]) * sz + (y + G.g[1]) * sy + (x + G.g[0]))), p);
            } else if (DIM == 1) {
                acc = spow<P>(fabs(uc - load(u, bound<BC>(i - h, G.n[0]) + G.g[0])), p) +
                    spow<P>(fabs(uc - load(u, bound<BC>(i + h, G.n[0]) + G.g[0])), p);
            } else if (DIM == 2) {
                for (int side = -1; side <= 1; side += 2) {
                    // faces normal to x: x = i -+ h, y in [j-h+1, j+h-1]
                    const int x = bound<BC>(i + side * h, G.n[0]);
                    acc += run_sum<T, BC, P>(u, uc, x + G.g[0], sy, j - h + 1, 2 * h - 1, G.n[1],
                        G.g[1], p);
                }
                for (int side = -1; side <= 1; side += 2) {
                    // faces normal to y: y = j -+ h, x in [i-h, i+h]
                    const int y = bound<BC>(j + side * h, G.n[1]);
                    acc += run_sum<T, BC, P>(u, uc, (y + G.g[1]) * sy, sx, i - h, 2 * h + 1,
                        G.n[0], G.g[0], p);
                }
            } else {
                for (int side = -1; side <= 1; side += 2) {
                    // faces normal to x: x = i -+ h, y in [j-h+1, j+h-1], z in [k-h, k+h]
                    const int x = bound<BC>(i + side * h, G.n[0]);
                    for (int zz = k - h; zz <= k + h; ++zz) {
                        const int z = bound<BC>(zz, G.n[2]);
                        acc += run_sum<T, BC, P>(u, uc, (z + G.g[2]) * sz + x + G.g[0], sy,
                            j - h + 1, 2 * h - 1, G.n[1], G.g[1], p);
                    }
                }
                for (int side = -1; side <= 1; side += 2) {
                    // faces normal to y: y = j -+ h, x in [i-h, i+h], z in [k-h, k+h]
                    const int y = bound<BC>(j + side * h, G.n[1]);
                    for (int zz = k - h; zz <= k + h; ++zz) {
                        const int z = bound<BC>(zz, G.n[2]);
                        acc += run_sum<T, BC, P>(u, uc, (z + G.g[2]) * sz + (y + G.g[1]) * sy, sx,
                            i - h, 2 * h + 1, G.n[0], G.g[0], p);
                    }
                }
                for (int side = -1; side <= 1; side += 2) {
                    // faces normal to z: z = k -+ h, x in [i-h+1, i+h-1], y in [j-h+1, j+h-1]
                    const int z = bound<BC>(k + side * h, G.n[2]);
                    for (int yy = j - h + 1; yy <= j + h - 1; ++yy) {
                        const int y = bound<BC>(yy, G.n[1]);
                        acc += run_sum<T, BC, P>(u, uc, (z + G.g[2]) * sz + (y + G.g[1]) * sy, sx,
                            i - h + 1, 2 * h - 1, G.n[0], G.g[0], p);
                    }
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            acc += __shfl_down_sync(0xffffffffu, acc, o);
        }
        if (lane == 0) {
            part[warp][h] = acc;
        }
    }
    __syncthreads();
    const long long row = ((long long)member * nvar + var) * gridDim.x + tile;
    for (int h = threadIdx.x; h < H; h += kThreads) {
        double s = 0;
        if (h >= h0) {
            for (int w = 0; w < kWarps; ++w) {
                s += part[w][h];
            }
        }
        partial[row * H + h] = s;
    }
}

// out[mv][h] = (sum over tiles, in tile order) / cells
__global__ void structure_finish(const double* __restrict__ partial, int tiles, int H, long long rows,
    double cells, double* __restrict__ out) {
    const long long total = rows * H;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long r = t / H;
        const int h = int(t - r * H);
        double s = 0;
        for (int b = 0; b < tiles; ++b) {
            s += partial[(r * tiles + b) * H + h];
        }
        out[t] = s / cells;
    }
}

template<class T, int DIM, int BC, int P, bool CUBE>
cudaError_t launch(const T* states, long long stride, const StructGeom& G, int nvar, int members,
    int direction, int H, double p, double* partial, cudaStream_t s) {
    const int tiles = G.tiles[0] * G.tiles[1] * G.tiles[2];
    dim3 grid(tiles, nvar, members);
    structure_kernel<T, DIM, BC, P, CUBE><<<grid, kThreads, 0, s>>>(states, stride, G, nvar,
        direction, H, p, partial);
    return cudaGetLastError();
}

template<class T, int DIM, int BC, bool CUBE>
cudaError_t by_power(const T* states, long long stride, const StructGeom& G, int nvar,
    int members, int direction, int H, double p, double* partial, cudaStream_t s) {
    if (p == 1.0) {
        return launch<T, DIM, BC, 1, CUBE>(states, stride, G, nvar, members, direction, H, p, partial, s);
    } else if (p == 2.0) {
        return launch<T, DIM, BC, 2, CUBE>(states, stride, G, nvar, members, direction, H, p, partial, s);
    } else if (p == 3.0) {
        return launch<T, DIM, BC, 3, CUBE>(states, stride, G, nvar, members, direction, H, p, partial, s);
    } else if (p == 4.0) {
        return launch<T, DIM, BC, 4, CUBE>(states, stride, G, nvar, members, direction, H, p, partial, s);
    } else if (p == 5.0) {
        return launch<T, DIM, BC, 5, CUBE>(states, stride, G, nvar, members, direction, H, p, partial, s);
    }
    return launch<T, DIM, BC, 0, CUBE>(states, stride, G, nvar, members, direction, H, p, partial, s);
}

template<class T, int DIM>
cudaError_t by_kind(const T* states, long long stride, const StructGeom& G, int nvar, int members,
    int bc, bool cube, int direction, int H, double p, double* partial, cudaStream_t s) {
    if (bc == ALS_BC_PERIODIC) {
        return cube ? by_power<T, DIM, ALS_BC_PERIODIC, true>(states, stride, G, nvar, members, direction, H, p, partial, s)
                    : by_power<T, DIM, ALS_BC_PERIODIC, false>(states, stride, G, nvar, members, direction, H, p, partial, s);
    }
    return cube ? by_power<T, DIM, ALS_BC_NEUMANN, true>(states, stride, G, nvar, members, direction, H, p, partial, s)
                : by_power<T, DIM, ALS_BC_NEUMANN, false>(states, stride, G, nvar, members, direction, H, p, partial, s);
}

template<class T>
cudaError_t dispatch(int dim, const T* states, long long stride, const StructGeom& G, int nvar,
    int members, int bc, bool cube, int direction, int H, double p, double* partial,
    cudaStream_t s) {
    if (dim == 1) {
        return by_kind<T, 1>(states, stride, G, nvar, members, bc, cube, direction, H, p, partial, s);
    } else if (dim == 2) {
        return by_kind<T, 2>(states, stride, G, nvar, members, bc, cube, direction, H, p, partial, s);
    }
    return by_kind<T, 3>(states, stride, G, nvar, members, bc, cube, direction, H, p, partial, s);
}

} // namespace

extern "C" int als_structure_functions(const als_grid* grid, int boundary, int kind,
    int direction, int H, double p, const void* states, int precision, long long member_stride,
    int members, double* out, void* stream) {
    if (!grid || grid->dimension < 1 || grid->dimension > 3 || grid->ghosts < 0 ||
        (boundary != ALS_BC_PERIODIC && boundary != ALS_BC_NEUMANN) ||
        (kind != ALS_STRUCTURE_CUBE && kind != ALS_STRUCTURE_BASIC) || H < 1 || H > kMaxH ||
        !(p > 0) || members < 0 || (members > 0 && (!states || !out)) ||
        (precision != ALS_FP64 && precision != ALS_FP32) ||
        (kind == ALS_STRUCTURE_BASIC && (direction < 0 || direction >= grid->dimension))) {
        return als::report_error(ALS_E_INVALID, "invalid structure-function arguments");
    }
    const int dim = grid->dimension;
    StructGeom G = {};
    for (int d = 0; d < 3; ++d) {
        G.n[d] = d < dim ? grid->n[d] : 1;
        G.g[d] = d < dim ? grid->ghosts : 0;
        if (G.n[d] < 1) {
            return als::report_error(ALS_E_INVALID, "invalid grid size");
        }
        G.N[d] = G.n[d] + 2 * G.g[d];
    }
    G.plane = (long long)G.N[0] * G.N[1] * G.N[2];
    const int nvar = dim + 2;
    if (member_stride < nvar * G.plane) {
        return als::report_error(ALS_E_INVALID, "member stride smaller than a state");
    }
    if (members == 0) {
        return ALS_OK;
    }
    const int shapes[3][3] = {{256, 1, 1}, {16, 16, 1}, {8, 8, 4}};
    for (int d = 0; d < 3; ++d) {
        G.tile[d] = shapes[dim - 1][d];
        G.tiles[d] = (G.n[d] + G.tile[d] - 1) / G.tile[d];
    }
    const long long tiles = (long long)G.tiles[0] * G.tiles[1] * G.tiles[2];
    if (tiles > 0x7fffffffLL) {
        return als::report_error(ALS_E_INVALID, "grid too large");
    }
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    // per-tile partials, members processed in chunks of at most 64 MiB of them
    const long long per_member = tiles * nvar * (long long)H;
    const int chunk = int(std::max<long long>(1, std::min<long long>(
        std::min<long long>(members, 65535), (64LL << 20) / 8 / per_member)));
    double* partial = nullptr;
    ST_CUDA(als::scratch_alloc((void**)&partial, sizeof(double) * per_member * chunk, s));
    const double cells = double(G.n[0]) * G.n[1] * G.n[2];
    cudaError_t err = cudaSuccess;
    for (int m0 = 0; m0 < members && err == cudaSuccess; m0 += chunk) {
        const int mc = std::min(chunk, members - m0);
        if (precision == ALS_FP64) {
            err = dispatch<double>(dim, static_cast<const double*>(states) + m0 * member_stride,
                member_stride, G, nvar, mc, boundary, kind == ALS_STRUCTURE_CUBE, direction, H,
                p, partial, s);
        } else {
            err = dispatch<float>(dim, static_cast<const float*>(states) + m0 * member_stride,
                member_stride, G, nvar, mc, boundary, kind == ALS_STRUCTURE_CUBE, direction, H,
                p, partial, s);
        }
        if (err == cudaSuccess) {
            const long long rows = (long long)mc * nvar;
            const int blocks = int(std::min<long long>((rows * H + 255) / 256, 148LL * 16));
            structure_finish<<<blocks, 256, 0, s>>>(partial, int(tiles), H, rows, cells,
                out + (long long)m0 * nvar * H);
            err = cudaGetLastError();
        }
    }
    als::scratch_free(partial, s);
    if (err != cudaSuccess) {
        return als::report_error(ALS_E_CUDA, cudaGetErrorString(err));
    }
    return ALS_OK;
}
