// Functionals of the solution (alsfvm/src/functional/): maps from a state
// to an observable, accumulated as out += weight * f(U) so that callers can
// integrate them in time (Functional.hpp:41-60,
// TimeIntegrationFunctional.cpp:33-48).  Batched over ensemble members, FP64
// or FP32 states, FP64 results.
//
//   identity            Identity.cpp:25-48           out (interior cells) += w U
//   moment              Moment.cpp:27-37,            out (padded cells) += w U^degree
//                       HostMemory.cpp:293-301
//   log_entropy         LogEntropy.cpp:30-80         out[E] += w sum -rho s/(gamma-1) dV
//   legendre            Legendre.cpp:36-98           out[v] += w sum P_k(x') P_n(y') P_m(u') dV
//   legendre_pointwise  LegendrePointWise.cpp:32-87  out (interior) += w P_degree(u')
//   bv                  BoundedVariation.cpp:24-52,  out[v] += w sum |grad U_v|^p
//                       HostMemory.cpp:325-362
//   bv_direction        alsuq/src/stats/BoundedVariationDirection.cpp:35-70,
//                       HostMemory.cpp:364-401     out[v] += w sum |U(x) - U(x-e_d)|^p
//   structure_2pt       alsuq/src/stats/StructureTwoPoints.cpp:48-92
//                       out[v][h1 + H h2] += w sum (U(x+h1 e)-U)^2 (U(x+h2 e)-U) / cells
//                       (shifts clamped at the last cell; the reference
//                       uses direction1 for both shifts)
//
// Sums over cells (log_entropy, legendre, bv) are reduced in a fixed order
// (per block: strided per-thread sums, then a shared-memory tree; the block
// partials in block order), so they are deterministic and equal the
// reference's sequential sums to rounding.  Legendre polynomials use the
// three-term recurrence (Bonnet) P_{l+1} = ((2l+1) x P_l - l P_{l-1})/(l+1) of
// the boost::math::legendre_p the reference's CPU path calls, with its
// reflection of negative degrees (l -> -l - 1), in FP64: Boost's default
// policy runs the recurrence in long double, so values differ from the
// reference's by a few units of 2^-52 (about 2.5 per degree at most; |P| <= 1).
// An argument outside [-1, 1] is Boost's domain error (an exception in the
// reference); this stream-ordered entry point evaluates the polynomial there.
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "als_b200.h"
#include "scratch.h"

namespace als {
int report_error(int code, const char* msg);
}

namespace {

constexpr int kThreads = 256;
constexpr int kReduceBlocks = 64;   // blocks per member for the sums

struct Geometry {
    int dim;
    int n[3];        // interior cells (1 for inactive directions)
    int N[3];        // padded extents
    int g;
    long long plane; // padded cells per plane
    long long cells; // interior cells
    double origin[3], sides[3], len[3];
    double dV;
};

template<class R>
__device__ __forceinline__ double load(const void* base, long long i) {
    return double(static_cast<const R*>(base)[i]);
}

__device__ __forceinline__ long long padded_index(const Geometry& G, long long c, int* ijk) {
    const int i = int(c % G.n[0]);
    const int j = int((c / G.n[0]) % G.n[1]);
    const int k = int(c / ((long long)G.n[0] * G.n[1]));
    ijk[0] = i;
    ijk[1] = j;
    ijk[2] = k;
    const int px = i + G.g;
    const int py = G.dim > 1 ? j + G.g : 0;
    const int pz = G.dim > 2 ? k + G.g : 0;
    return ((long long)pz * G.N[1] + py) * G.N[0] + px;
}

__device__ __forceinline__ double legendre_p(int l, double x) {
    if (l < 0) {
        l = -l - 1;
    }
    double p0 = 1, p1 = x;
    if (l == 0) {
        return p0;
    }
    for (int m = 1; m < l; ++m) {
        const double next = ((2 * m + 1) * x * p1 - m * p0) / (m + 1);
        p0 = p1;
        p1 = next;
    }
    return p1;
}

// Pointwise functionals: identity, moment, legendre_pointwise.
template<class R>
__global__ void __launch_bounds__(kThreads) pointwise(Geometry G, int kind, int degree, double lo,
    double hi, const void* states, long long member_stride, int members, int nvar, double* out,
    long long out_member_stride, double weight) {
    const long long per_var = kind == ALS_FUNCTIONAL_MOMENT ? G.plane : G.cells;
    const long long total = (long long)members * nvar * per_var;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long c = t % per_var;
        const int v = int((t / per_var) % nvar);
        const int m = int(t / (per_var * nvar));
        const long long base = (long long)m * member_stride + (long long)v * G.plane;
        double* o = out + (long long)m * out_member_stride + (long long)v * per_var + c;
        if (kind == ALS_FUNCTIONAL_MOMENT) {
            // data[i] += factor * pow(other[i], power) over every cell
            *o = *o + weight * pow(load<R>(states, base + c), double(degree));
        } else {
            int ijk[3];
            const double u = load<R>(states, base + padded_index(G, c, ijk));
            if (kind == ALS_FUNCTIONAL_IDENTITY) {
                *o = *o + weight * u;
            } else {
                const double value = (u - lo) / (hi - lo);
                *o = *o + legendre_p(degree, value) * weight;
            }
        }
    }
}

// Block partial sums of a reduced functional: partial[(m * nsum + s) * B + b].
template<class R>
__global__ void __launch_bounds__(kThreads) partial_sums(Geometry G, int kind, int p, int dk,
    int dn, int dm, double lo, double hi, double gamma, int dir, int H, const void* states,
    long long member_stride, int nvar, int nsum, double* partial) {
    const int b = blockIdx.x;
    const int m = blockIdx.y;
    // the sum's index: the variable (legendre, bv, bv_direction), 0
    // (log_entropy), or variable * H^2 + h1 + H h2 (structure_2pt)
    const int sidx = blockIdx.z;
    const long long base = (long long)m * member_stride;
    const long long stride = dir == 0 ? 1 : (dir == 1 ? G.N[0] : (long long)G.N[0] * G.N[1]);
    __shared__ double red[kThreads];
    double acc = 0;
    for (long long c = (long long)b * blockDim.x + threadIdx.x; c < G.cells;
         c += (long long)gridDim.x * blockDim.x) {
        int ijk[3];
        const long long idx = padded_index(G, c, ijk);
        if (kind == ALS_FUNCTIONAL_LOG_ENTROPY) {
            const double rho = load<R>(states, base + idx);
            const double E = load<R>(states, base + (long long)(nvar - 1) * G.plane + idx);
            double msq = 0.0;
            for (int k = 0; k < G.dim; ++k) {
                const double mk = load<R>(states, base + (long long)(1 + k) * G.plane + idx);
                msq += mk * mk;
            }
            const double pressure = (gamma - 1) * (E - 1.0 / (2 * rho) * msq);
            const double s = log(pressure) - gamma * log(rho);
            const double ent = (-rho * s) / (gamma - 1);
            acc += ent * G.dV;
        } else if (kind == ALS_FUNCTIONAL_LEGENDRE) {
            const double x = (G.origin[0] + G.len[0] * ijk[0]) + G.len[0] / 2.0;
            const double y = (G.origin[1] + G.len[1] * ijk[1]) + G.len[1] / 2.0;
            const double xs = 2 * (x - G.origin[0]) / G.sides[0] - 1;
            const double ys = 2 * (y - G.origin[1]) / G.sides[1] - 1;
            const double value = (load<R>(states, base + (long long)sidx * G.plane + idx) - lo) /
                (hi - lo);
            acc += legendre_p(dk, xs) * legendre_p(dn, ys) * legendre_p(dm, value) * G.dV;
        } else if (kind == ALS_FUNCTIONAL_BV_DIRECTION) {
            if (ijk[dir] == 0) {
                continue;
            }
            const long long v0 = base + (long long)sidx * G.plane;
            acc += pow(fabs(load<R>(states, v0 + idx) - load<R>(states, v0 + idx - stride)),
                double(p));
        } else if (kind == ALS_FUNCTIONAL_STRUCTURE_2PT) {
            const int var = sidx / (H * H);
            const int h1 = (sidx % (H * H)) % H;
            const int h2 = (sidx % (H * H)) / H;
            const long long v0 = base + (long long)var * G.plane;
            const double u = load<R>(states, v0 + idx);
            // shifted cells, clamped at the last interior cell along dir
            const int last = G.n[dir] - 1;
            const int s1 = min(ijk[dir] + h1, last) - ijk[dir];
            const int s2 = min(ijk[dir] + h2, last) - ijk[dir];
            const double u1 = load<R>(states, v0 + idx + s1 * stride);
            const double u2 = load<R>(states, v0 + idx + s2 * stride);
            acc += (u1 - u) * (u1 - u) * (u2 - u) / double(G.cells);
        } else {
            // bounded variation: cells after the first along x (and y in 2-D)
            if (ijk[0] == 0 || (G.dim > 1 && ijk[1] == 0)) {
                continue;
            }
            const long long v0 = base + (long long)sidx * G.plane;
            const double u = load<R>(states, v0 + idx);
            const double ux = load<R>(states, v0 + idx - 1);
            const double uy = G.dim > 1 ? load<R>(states, v0 + idx - G.N[0]) : u;
            const double dy = u - uy;
            const double dx = u - ux;
            acc += pow(sqrt(dy * dy + dx * dx), double(p));
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[((long long)m * nsum + sidx) * gridDim.x + b] = red[0];
    }
}

// out slot += weight * (sum of the block partials in block order); sum s
// goes to variable slot0 + s / inner, element s % inner.
__global__ void __launch_bounds__(kThreads) finish_sums(const double* partial, int blocks,
    int members, int nsum, int slot0, int inner, long long per_var, double* out,
    long long out_member_stride, double weight) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= members * nsum) {
        return;
    }
    const int m = t / nsum;
    const int s = t % nsum;
    double sum = 0;
    for (int b = 0; b < blocks; ++b) {
        sum += partial[(long long)t * blocks + b];
    }
    const int v = slot0 + s / inner;
    double* o = out + (long long)m * out_member_stride + (long long)v * per_var + s % inner;
    *o = *o + weight * sum;
}

int blocks_for(long long n) {
    long long b = (n + kThreads - 1) / kThreads;
    if (b < 1) {
        b = 1;
    }
    return int(b < 148LL * 16 ? b : 148LL * 16);
}

long long elements_per_variable(const Geometry& G, int kind, int H) {
    switch (kind) {
    case ALS_FUNCTIONAL_IDENTITY:
    case ALS_FUNCTIONAL_LEGENDRE_POINTWISE:
        return G.cells;
    case ALS_FUNCTIONAL_MOMENT:
        return G.plane;
    case ALS_FUNCTIONAL_STRUCTURE_2PT:
        return (long long)H * H;
    default:
        return 1;
    }
}

int make_geometry(const als_grid* grid, const als_functional_params* p, Geometry& G) {
    if (!grid || grid->dimension < 1 || grid->dimension > 3 || grid->ghosts < 0) {
        return als::report_error(ALS_E_INVALID, "invalid grid");
    }
    std::memset(&G, 0, sizeof(G));
    G.dim = grid->dimension;
    G.g = grid->ghosts;
    G.plane = 1;
    G.cells = 1;
    for (int d = 0; d < 3; ++d) {
        G.n[d] = d < G.dim ? grid->n[d] : 1;
        if (G.n[d] < 1) {
            return als::report_error(ALS_E_INVALID, "invalid grid size");
        }
        G.N[d] = G.n[d] + (d < G.dim ? 2 * G.g : 0);
        G.plane *= G.N[d];
        G.cells *= G.n[d];
        const double lower = p ? p->lower[d] : 0.0;
        const double upper = p ? p->upper[d] : 1.0;
        G.origin[d] = lower;
        G.sides[d] = upper - lower;
        // Grid.cpp:24-41: (top - origin) / n, 1 where a direction has one cell
        G.len[d] = (upper - lower) / double(G.n[d]);
        if (d > 0 && G.n[d] == 1) {
            G.len[d] = 1;
        }
    }
    G.dV = G.len[0] * G.len[1] * G.len[2];
    return ALS_OK;
}

} // namespace

extern "C" {

int als_functional_size2(const als_grid* grid, int kind, const als_functional_params* params,
    long long* elements) {
    Geometry G;
    const int rc = make_geometry(grid, nullptr, G);
    if (rc != ALS_OK) {
        return rc;
    }
    if (!elements || kind < ALS_FUNCTIONAL_IDENTITY || kind > ALS_FUNCTIONAL_STRUCTURE_2PT ||
        (kind == ALS_FUNCTIONAL_STRUCTURE_2PT && (!params || params->number_of_h < 1))) {
        return als::report_error(ALS_E_INVALID, "invalid functional arguments");
    }
    *elements = elements_per_variable(G, kind, params ? params->number_of_h : 0);
    return ALS_OK;
}

int als_functional_size(const als_grid* grid, int kind, long long* elements) {
    return als_functional_size2(grid, kind, nullptr, elements);
}

int als_functional(const als_grid* grid, int kind, const als_functional_params* params,
    const void* states, int precision, long long member_stride, int members, double* out,
    long long out_member_stride, double weight, void* stream) {
    Geometry G;
    int rc = make_geometry(grid, params, G);
    if (rc != ALS_OK) {
        return rc;
    }
    if (!params || !states || !out || members < 1 || member_stride < 0 ||
        out_member_stride < 0 || kind < ALS_FUNCTIONAL_IDENTITY ||
        kind > ALS_FUNCTIONAL_STRUCTURE_2PT || (precision != ALS_FP64 && precision != ALS_FP32)) {
        return als::report_error(ALS_E_INVALID, "invalid functional arguments");
    }
    if ((kind == ALS_FUNCTIONAL_BV_DIRECTION || kind == ALS_FUNCTIONAL_STRUCTURE_2PT) &&
        (params->direction < 0 || params->direction >= G.dim)) {
        return als::report_error(ALS_E_INVALID, "direction outside the grid's dimensions");
    }
    if (kind == ALS_FUNCTIONAL_STRUCTURE_2PT && (params->number_of_h < 1 ||
        params->number_of_h > 64)) {
        return als::report_error(ALS_E_INVALID, "structure_2pt takes 1 <= number_of_h <= 64");
    }
    const int nvar = G.dim + 2;
    const long long per_var = elements_per_variable(G, kind, params->number_of_h);
    if (members > 1 && (member_stride < nvar * G.plane || out_member_stride < nvar * per_var)) {
        return als::report_error(ALS_E_INVALID, "member strides smaller than one member");
    }
    // (the Legendre degrees may be negative: P_{-l-1} = P_l, as in Boost)
    if ((kind == ALS_FUNCTIONAL_MOMENT || kind == ALS_FUNCTIONAL_BV ||
         kind == ALS_FUNCTIONAL_BV_DIRECTION) && params->degree < 0) {
        return als::report_error(ALS_E_INVALID, "negative degree");
    }
    // Legendre.cpp:54-58 / LegendrePointWise.cpp:49-53 accept 2-D grids only;
    // BoundedVariation / HostMemory::getTotalVariation 1-D and 2-D
    if ((kind == ALS_FUNCTIONAL_LEGENDRE || kind == ALS_FUNCTIONAL_LEGENDRE_POINTWISE) &&
        G.dim != 2) {
        return als::report_error(ALS_E_UNSUPPORTED, "the Legendre functionals are two-dimensional");
    }
    if (kind == ALS_FUNCTIONAL_BV && G.dim > 2) {
        return als::report_error(ALS_E_UNSUPPORTED, "bounded variation is 1-D and 2-D");
    }
    if (kind == ALS_FUNCTIONAL_LOG_ENTROPY && !(params->gamma > 1)) {
        return als::report_error(ALS_E_INVALID, "log_entropy needs gamma > 1");
    }
    const cudaStream_t st = (cudaStream_t)stream;
    cudaError_t err = cudaSuccess;
    if (kind == ALS_FUNCTIONAL_IDENTITY || kind == ALS_FUNCTIONAL_MOMENT ||
        kind == ALS_FUNCTIONAL_LEGENDRE_POINTWISE) {
        const int blocks = blocks_for((long long)members * nvar * per_var);
        if (precision == ALS_FP64) {
            pointwise<double><<<blocks, kThreads, 0, st>>>(G, kind, params->degree,
                params->min_value, params->max_value, states, member_stride, members, nvar, out,
                out_member_stride, weight);
        } else {
            pointwise<float><<<blocks, kThreads, 0, st>>>(G, kind, params->degree,
                params->min_value, params->max_value, states, member_stride, members, nvar, out,
                out_member_stride, weight);
        }
        err = cudaGetLastError();
    } else {
        // log_entropy: one sum into the energy slot; legendre, bv,
        // bv_direction: one per variable; structure_2pt: H^2 per variable
        const int H = params->number_of_h;
        const int inner = kind == ALS_FUNCTIONAL_STRUCTURE_2PT ? H * H : 1;
        const int nsum = kind == ALS_FUNCTIONAL_LOG_ENTROPY ? 1 : nvar * inner;
        const int slot0 = kind == ALS_FUNCTIONAL_LOG_ENTROPY ? nvar - 1 : 0;
        if (members > 65535) {
            return als::report_error(ALS_E_INVALID, "at most 65535 members per call");
        }
        long long bl = (G.cells + kThreads - 1) / kThreads;
        int blocks = int(bl < kReduceBlocks ? (bl < 1 ? 1 : bl) : kReduceBlocks);
        // partial sums stay below 512 MB
        while (blocks > 1 && (long long)members * nsum * blocks > (1LL << 26)) {
            blocks /= 2;
        }
        double* partial = nullptr;
        err = als::scratch_alloc((void**)&partial,
            sizeof(double) * size_t(members) * nsum * blocks, st);
        if (err == cudaSuccess) {
            dim3 grid3(blocks, members, nsum);
            if (precision == ALS_FP64) {
                partial_sums<double><<<grid3, kThreads, 0, st>>>(G, kind, params->degree,
                    params->degree_k, params->degree_n, params->degree_m, params->min_value,
                    params->max_value, params->gamma, params->direction, H, states,
                    member_stride, nvar, nsum, partial);
            } else {
                partial_sums<float><<<grid3, kThreads, 0, st>>>(G, kind, params->degree,
                    params->degree_k, params->degree_n, params->degree_m, params->min_value,
                    params->max_value, params->gamma, params->direction, H, states,
                    member_stride, nvar, nsum, partial);
            }
            err = cudaGetLastError();
            if (err == cudaSuccess) {
                finish_sums<<<(members * nsum + kThreads - 1) / kThreads, kThreads, 0, st>>>(
                    partial, blocks, members, nsum, slot0, inner, per_var, out,
                    out_member_stride, weight);
                err = cudaGetLastError();
            }
            const cudaError_t ferr = als::scratch_free(partial, st);
            if (err == cudaSuccess) {
                err = ferr;
            }
        }
    }
    if (err != cudaSuccess) {
        return als::report_error(ALS_E_CUDA, (std::string("functional: ") +
            cudaGetErrorString(err)).c_str());
    }
    return ALS_OK;
}

} // extern "C"
