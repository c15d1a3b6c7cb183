// TeCNO diffusion operator: DiffusionOperator::applyDiffusion of
// TecnoDiffusionCPU<Euler<nsd>, RoeMatrix | RusanovMatrix>
// (alsfvm/src/diffusion/TecnoDiffusionCPU.cpp:23-170) with the TeCNO
// reconstructions "none" and ENO2/3/4 (alsfvm/src/reconstruction/tecno/
// NoReconstruction.cpp:20-44, ENOCPU.cpp:35-267), FP64.
//
// Per direction d the reference makes three passes over the padded volume,
// and so do the kernels here, one launch each (the ENO pass: one launch per
// difference level and per variable, since its difference planes are shared
// by the variables in turn):
//   1. entropy   for cells m with 1 <= m_d <= N_d - 2 (every transverse
//                cell, ghosts included): R^T v(U_m) -> EL[m] and
//                R^T v(U_{m-1}) -> ER[m-1], R the eigenvector matrix at the
//                mean of U_{m-1} and U_m;
//   2. recon     (EL, ER) -> (OL, OR): a copy, or the ENO of that order;
//   3. apply     out[m] += D(m, m+1) - D(m-1, m),
//                D(l, r) = 0.5 R (Lambda (OL[r] - OR[l])) at the mean state.
// The operator object owns EL, ER, OL, OR (initialised to 42, the fill value
// of the reference's HostMemory, HostMemory.cpp:36-37) and the ENO's three
// difference planes (initialised to 0, ENOCPU.cpp:27-33).  The passes leave
// some entries unwritten (the last cells along d) and later reads see what
// earlier passes, variables and calls left there; the reference's results
// depend on that, so these buffers persist between calls exactly as its
// volumes do.  The ENO also rebuilds its stencil values from level-1
// differences at flat offsets +l, -l-1 (ENOCPU.cpp:118-123), i.e. along x
// whatever d is; kept as is.
//
// Numerics follow the reference's expression order (compiled with
// -fmad=false and IEEE division and square root); the entropy variables
// call the device log, so results agree with the reference's to rounding of
// that log, not bit for bit.
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "als_b200.h"
#include "euler_math.cuh"

namespace als {
int report_error(int code, const char* msg);
}

struct als_diffusion {
    als_grid grid;
    int kind = 0;
    int recon = 0;
    int nv = 0;
    int N[3] = {1, 1, 1};
    long long plane = 0;
    double* work = nullptr;   // EL, ER, OL, OR (nv planes each), then 3 difference planes
    int device = 0;
};

namespace {

constexpr int kThreads = 256;

struct Ptrs {
    const double* p[5];
};

struct OutPtrs {
    double* p[5];
};

__device__ __forceinline__ void decode(long long i, const int* N, int* c) {
    c[0] = int(i % N[0]);
    c[1] = int((i / N[0]) % N[1]);
    c[2] = int(i / ((long long)N[0] * N[1]));
}

struct Dims {
    int N[3];
    long long plane;
};

// The conserved state rotated into direction D's frame (Euler.hpp:409-425,
// 506-517), its velocity, pressure and sound speed (computePrimitiveVariables,
// Euler.hpp:290-297).
template<int NSD, int D>
__device__ __forceinline__ void rotated_primitive(const double* U, double gamma, double* u,
    double& p, double& a) {
    double m[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < NSD; ++k) {
        m[k] = U[1 + k];
    }
    if ((NSD == 2 || NSD == 3) && D == 1) {
        const double mx = m[0];
        m[0] = m[1];
        m[1] = -mx;
    } else if (NSD == 3 && D == 2) {
        const double mx = m[0];
        m[0] = m[2];
        m[2] = -mx;
    }
    double dot = m[0] * m[0];
    if (NSD > 1) {
        dot = dot + m[1] * m[1];
    }
    if (NSD > 2) {
        dot = dot + m[2] * m[2];
    }
#pragma unroll
    for (int k = 0; k < NSD; ++k) {
        u[k] = m[k] / U[0];
    }
    p = (gamma - 1) * (U[1 + NSD] - 0.5 * dot / U[0]);
    a = sqrt(gamma * p / U[0]);
}

template<int NSD>
__device__ __forceinline__ double udot(const double* u) {
    double s = u[0] * u[0];
    if (NSD > 1) {
        s = s + u[1] * u[1];
    }
    if (NSD > 2) {
        s = s + u[2] * u[2];
    }
    return s;
}

// R(row, col) of Euler<NSD>::computeEigenVectorMatrix<D>: scaled columns in
// 1-D (Euler.hpp:586-623), plain in 2-D (506-553), normalised in 3-D with
// the column norm's square root in single precision (409-466, mat.hpp:96-110).
template<int NSD, int D>
__device__ __forceinline__ void eigenvectors(const double* U, double gamma, double (&R)[NSD + 2][NSD + 2]) {
    double u[3] = {0, 0, 0}, p, a;
    rotated_primitive<NSD, D>(U, gamma, u, p, a);
    const double H = (U[1 + NSD] + p) / U[0];
    if (NSD == 1) {
        const double rho = U[0];
        const double a1 = sqrt(rho / (2 * gamma));
        const double a2 = sqrt(rho * (gamma - 1) / gamma);
        const double a4 = a1;
        R[0][0] = a1;
        R[0][1] = a2;
        R[0][NSD + 1] = a4;
        R[1][0] = a1 * (u[0] - a);
        R[1][1] = a2 * u[0];
        R[1][NSD + 1] = a4 * (u[0] + a);
        R[NSD + 1][0] = a1 * (H - u[0] * a);
        R[NSD + 1][1] = 0.5 * a2 * udot<NSD>(u);
        R[NSD + 1][NSD + 1] = a4 * (H + u[0] * a);
    } else {
        constexpr int NV = NSD + 2;
#pragma unroll
        for (int r = 0; r < NV; ++r) {
#pragma unroll
            for (int c = 0; c < NV; ++c) {
                R[r][c] = 0;
            }
        }
        // columns: u-a, u, transverse shear(s), u+a
        R[0][0] = 1;
        R[0][1] = 1;
        R[0][NV - 1] = 1;
        R[1][0] = u[0] - a;
        R[1][1] = u[0];
        R[1][NV - 1] = u[0] + a;
#pragma unroll
        for (int k = 1; k < NSD; ++k) {
            R[1 + k][0] = u[k];
            R[1 + k][1] = u[k];
            R[1 + k][1 + k] = 1;
            R[1 + k][NV - 1] = u[k];
            R[NV - 1][1 + k] = u[k];
        }
        R[NV - 1][0] = H - u[0] * a;
        R[NV - 1][1] = 0.5 * udot<NSD>(u);
        R[NV - 1][NV - 1] = H + u[0] * a;
        if (NSD == 3) {
#pragma unroll
            for (int c = 0; c < NV; ++c) {
                double norm = 0;
#pragma unroll
                for (int r = 0; r < NV; ++r) {
                    norm += R[r][c] * R[r][c];
                }
                norm = double(sqrtf(float(norm)));
#pragma unroll
                for (int r = 0; r < NV; ++r) {
                    R[r][c] = R[r][c] / norm;
                }
            }
        }
    }
}

// Eigenvalues u-a, u (NSD times), u+a of the rotated Jacobian
// (Euler.hpp:470-498, 555-580, 646-657).
template<int NSD, int D>
__device__ __forceinline__ void eigenvalues(const double* U, double gamma, double* ev) {
    double u[3] = {0, 0, 0}, p, a;
    rotated_primitive<NSD, D>(U, gamma, u, p, a);
    ev[0] = u[0] - a;
#pragma unroll
    for (int k = 1; k <= NSD; ++k) {
        ev[k] = u[0];
    }
    ev[NSD + 1] = u[0] + a;
}

// v(u) for the entropy -rho s/(gamma-1), s = log p - gamma log rho
// (Euler.hpp:323-348).
template<int NSD>
__device__ __forceinline__ void entropy_variables(const double* U, double gamma, double* v) {
    double dot = U[1] * U[1];
    if (NSD > 1) {
        dot = dot + U[2] * U[2];
    }
    if (NSD > 2) {
        dot = dot + U[3] * U[3];
    }
    double u[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < NSD; ++k) {
        u[k] = U[1 + k] / U[0];
    }
    const double p = (gamma - 1) * (U[1 + NSD] - 0.5 * dot / U[0]);
    const double s = log(p) - gamma * log(U[0]);
    v[0] = (gamma - s) / (gamma - 1) - (U[0] * udot<NSD>(u)) / (2 * p);
#pragma unroll
    for (int k = 0; k < NSD; ++k) {
        v[1 + k] = U[1 + k] / p;
    }
    v[1 + NSD] = -U[0] / p;
}

// y = M x accumulated column by column (mat.hpp:47-60); M = R or R^T.
template<int NV, bool TRANSPOSE>
__device__ __forceinline__ void mat_vec(const double (&R)[NV][NV], const double* x, double* y) {
#pragma unroll
    for (int r = 0; r < NV; ++r) {
        y[r] = 0;
    }
#pragma unroll
    for (int c = 0; c < NV; ++c) {
#pragma unroll
        for (int r = 0; r < NV; ++r) {
            y[r] += (TRANSPOSE ? R[c][r] : R[r][c]) * x[c];
        }
    }
}

// Pass 1 (TecnoDiffusionCPU.cpp:40-58).
template<int NSD, int D>
__global__ void __launch_bounds__(kThreads) entropy_pass(Ptrs U, Dims g, double gamma, double* EL,
    double* ER) {
    constexpr int NV = NSD + 2;
    const long long s = D == 0 ? 1 : (D == 1 ? g.N[0] : (long long)g.N[0] * g.N[1]);
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < g.plane;
         m += (long long)gridDim.x * blockDim.x) {
        int c[3];
        decode(m, g.N, c);
        if (c[D] < 1 || c[D] > g.N[D] - 2) {
            continue;
        }
        double Um[NV], Ul[NV], avg[NV], vm[NV], vl[NV], a[NV], b[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            Um[k] = U.p[k][m];
            Ul[k] = U.p[k][m - s];
        }
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            avg[k] = 0.5 * (Um[k] + Ul[k]);
        }
        double R[NV][NV];
        eigenvectors<NSD, D>(avg, gamma, R);
        entropy_variables<NSD>(Um, gamma, vm);
        entropy_variables<NSD>(Ul, gamma, vl);
        mat_vec<NV, true>(R, vm, a);
        mat_vec<NV, true>(R, vl, b);
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            EL[k * g.plane + m] = a[k];
            ER[k * g.plane + m - s] = b[k];
        }
    }
}

// Undivided differences of one level (ENOCPU.cpp:205-267): out[j - s] =
// a[j] - b[j - s] for cells j with level <= j_d < N_d - level.
__global__ void __launch_bounds__(kThreads) difference_pass(const double* a, const double* b,
    double* out, Dims g, int d, long long s, int level) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < g.plane;
         i += (long long)gridDim.x * blockDim.x) {
        int c[3];
        decode(i, g.N, c);
        if (c[d] < level || c[d] >= g.N[d] - level) {
            continue;
        }
        out[i - s] = a[i] - b[i - s];
    }
}

// The ENO of one variable (ENOCPU.cpp:84-136) for cells
// order-1 <= i_d < N_d - order + 1.
template<int ORDER>
__global__ void __launch_bounds__(kThreads) eno_pass(const double* L, const double* Rt,
    const double* dd, double* OL, double* OR, Dims g, int d, long long s) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < g.plane;
         i += (long long)gridDim.x * blockDim.x) {
        int c[3];
        decode(i, g.N, c);
        if (c[d] < ORDER - 1 || c[d] >= g.N[d] - ORDER + 1) {
            continue;
        }
        int shift = 0;
#pragma unroll
        for (int level = 0; level < ORDER - 1; ++level) {
            if (fabs(dd[level * g.plane + i - s]) < fabs(dd[level * g.plane + i])) {
                ++shift;
            }
        }
        double w[2 * ORDER - 1];
        w[ORDER - 1] = L[i];
#pragma unroll
        for (int l = 0; l < ORDER - 1; ++l) {
            w[ORDER + l] = w[ORDER + l - 1] + dd[i + l];
            w[ORDER - l - 2] = w[ORDER - l - 1] - dd[i - l - 1];
        }
        double uli = 0, uri = 0;
#pragma unroll
        for (int l = 0; l < ORDER; ++l) {
            uli += als::eno_coef<double, ORDER>(shift, l) * w[ORDER - 1 - shift + l];
            uri += als::eno_coef<double, ORDER>(shift + 1, l) * w[ORDER - 1 - shift + l];
        }
        OL[i] = uli;
        OR[i] = uri + (Rt[i] - L[i]);
    }
}

// D(l, r) of TecnoDiffusionCPU.cpp:70-88.
template<int NSD, int D, int KIND>
__device__ __forceinline__ void diffusion_term(const Ptrs& U, const double* OL, const double* OR,
    long long plane, long long l, long long r, double gamma, double* Dv) {
    constexpr int NV = NSD + 2;
    double avg[NV], diff[NV], ev[NV], t[NV], y[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        avg[k] = 0.5 * (U.p[k][r] + U.p[k][l]);
        diff[k] = OL[k * plane + r] - OR[k * plane + l];
    }
    eigenvalues<NSD, D>(avg, gamma, ev);
    if (KIND == ALS_DIFFUSION_TECNOROE) {
        // RoeMatrix.hpp:36-45
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            t[k] = fabs(ev[k]) * diff[k];
        }
    } else {
        // RusanovMatrix.hpp:36-54
        double mx = 0.0;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            mx = fmax(fabs(ev[k]), mx);
        }
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            t[k] = mx * diff[k];
        }
    }
    double R[NV][NV];
    eigenvectors<NSD, D>(avg, gamma, R);
    mat_vec<NV, false>(R, t, y);
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        Dv[k] = 0.5 * y[k];
    }
}

// Pass 3 (TecnoDiffusionCPU.cpp:62-92).
template<int NSD, int D, int KIND>
__global__ void __launch_bounds__(kThreads) apply_pass(Ptrs U, OutPtrs out, Dims g, double gamma,
    const double* OL, const double* OR) {
    constexpr int NV = NSD + 2;
    const long long s = D == 0 ? 1 : (D == 1 ? g.N[0] : (long long)g.N[0] * g.N[1]);
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < g.plane;
         m += (long long)gridDim.x * blockDim.x) {
        int c[3];
        decode(m, g.N, c);
        if (c[D] < 1 || c[D] > g.N[D] - 2) {
            continue;
        }
        double Dr[NV], Dl[NV];
        diffusion_term<NSD, D, KIND>(U, OL, OR, g.plane, m, m + s, gamma, Dr);
        diffusion_term<NSD, D, KIND>(U, OL, OR, g.plane, m - s, m, gamma, Dl);
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            out.p[k][m] = out.p[k][m] + (Dr[k] - Dl[k]);
        }
    }
}

__global__ void __launch_bounds__(kThreads) fill_value(double* p, long long count, double v) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        p[i] = v;
    }
}

int blocks_for(long long n) {
    long long b = (n + kThreads - 1) / kThreads;
    if (b < 1) {
        b = 1;
    }
    return int(b < 148LL * 16 ? b : 148LL * 16);
}

template<int NSD, int D>
cudaError_t run_direction(als_diffusion* h, const Ptrs& U, const OutPtrs& out, cudaStream_t st) {
    Dims g;
    for (int k = 0; k < 3; ++k) {
        g.N[k] = h->N[k];
    }
    g.plane = h->plane;
    const long long vol = (long long)h->nv * h->plane;
    double* EL = h->work;
    double* ER = EL + vol;
    double* OL = ER + vol;
    double* OR = OL + vol;
    double* DD = OR + vol;
    const int blocks = blocks_for(h->plane);
    const double gamma = h->grid.gamma;
    entropy_pass<NSD, D><<<blocks, kThreads, 0, st>>>(U, g, gamma, EL, ER);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        return err;
    }
    if (h->recon == ALS_TECNO_RECON_NONE) {
        // tecno::NoReconstruction copies every cell (NoReconstruction.cpp:20-44)
        err = cudaMemcpyAsync(OL, EL, sizeof(double) * size_t(vol), cudaMemcpyDeviceToDevice, st);
        if (err == cudaSuccess) {
            err = cudaMemcpyAsync(OR, ER, sizeof(double) * size_t(vol), cudaMemcpyDeviceToDevice, st);
        }
    } else {
        const long long s = D == 0 ? 1 : (D == 1 ? g.N[0] : (long long)g.N[0] * g.N[1]);
        for (int v = 0; v < h->nv && err == cudaSuccess; ++v) {
            const double* L = EL + v * h->plane;
            const double* R = ER + v * h->plane;
            for (int level = 1; level < h->recon && err == cudaSuccess; ++level) {
                const double* a = level == 1 ? L : DD + (level - 2) * h->plane;
                const double* b = level == 1 ? R : a;
                difference_pass<<<blocks, kThreads, 0, st>>>(a, b, DD + (level - 1) * h->plane, g,
                    D, s, level);
                err = cudaGetLastError();
            }
            if (err != cudaSuccess) {
                break;
            }
            double* ol = OL + v * h->plane;
            double* orr = OR + v * h->plane;
            switch (h->recon) {
            case ALS_TECNO_RECON_ENO2:
                eno_pass<2><<<blocks, kThreads, 0, st>>>(L, R, DD, ol, orr, g, D, s);
                break;
            case ALS_TECNO_RECON_ENO3:
                eno_pass<3><<<blocks, kThreads, 0, st>>>(L, R, DD, ol, orr, g, D, s);
                break;
            default:
                eno_pass<4><<<blocks, kThreads, 0, st>>>(L, R, DD, ol, orr, g, D, s);
                break;
            }
            err = cudaGetLastError();
        }
    }
    if (err != cudaSuccess) {
        return err;
    }
    if (h->kind == ALS_DIFFUSION_TECNOROE) {
        apply_pass<NSD, D, ALS_DIFFUSION_TECNOROE><<<blocks, kThreads, 0, st>>>(U, out, g, gamma, OL, OR);
    } else {
        apply_pass<NSD, D, ALS_DIFFUSION_TECNORUSANOV><<<blocks, kThreads, 0, st>>>(U, out, g, gamma, OL, OR);
    }
    return cudaGetLastError();
}

int diffusion_ghosts(int recon) {
    // tecno::NoReconstruction: 1 (NoReconstruction.hpp:40-42); ENOCPU<order>: order
    return recon == ALS_TECNO_RECON_NONE ? 1 : recon;
}

bool valid_recon(int recon) {
    return recon == ALS_TECNO_RECON_NONE || recon == ALS_TECNO_RECON_ENO2 ||
        recon == ALS_TECNO_RECON_ENO3 || recon == ALS_TECNO_RECON_ENO4;
}

} // namespace

extern "C" {

int als_diffusion_ghost_cells(int reconstruction) {
    if (!valid_recon(reconstruction)) {
        return als::report_error(ALS_E_INVALID, "unknown TeCNO reconstruction");
    }
    return diffusion_ghosts(reconstruction);
}

int als_diffusion_create(const als_grid* grid, int kind, int reconstruction, als_diffusion** out) {
    if (!out || !grid || grid->dimension < 1 || grid->dimension > 3 ||
        (kind != ALS_DIFFUSION_TECNOROE && kind != ALS_DIFFUSION_TECNORUSANOV) ||
        !valid_recon(reconstruction) || !(grid->gamma > 1)) {
        return als::report_error(ALS_E_INVALID, "invalid diffusion arguments");
    }
    *out = nullptr;
    if (grid->ghosts < diffusion_ghosts(reconstruction)) {
        return als::report_error(ALS_E_INVALID, "planes have fewer ghost cells than the diffusion needs");
    }
    for (int d = 0; d < grid->dimension; ++d) {
        if (grid->n[d] < grid->ghosts) {
            return als::report_error(ALS_E_INVALID,
                "every active direction needs at least `ghosts` interior cells");
        }
    }
    als_diffusion* h = new als_diffusion;
    h->grid = *grid;
    h->kind = kind;
    h->recon = reconstruction;
    h->nv = grid->dimension + 2;
    h->plane = 1;
    for (int d = 0; d < 3; ++d) {
        h->N[d] = d < grid->dimension ? grid->n[d] + 2 * grid->ghosts : 1;
        h->plane *= h->N[d];
    }
    cudaError_t err = cudaGetDevice(&h->device);
    const long long vol = 4LL * h->nv * h->plane;
    if (err == cudaSuccess) {
        err = cudaMalloc(&h->work, sizeof(double) * size_t(vol + 3 * h->plane));
    }
    if (err == cudaSuccess) {
        fill_value<<<blocks_for(vol), kThreads>>>(h->work, vol, 42.0);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) {
        err = cudaMemset(h->work + vol, 0, sizeof(double) * size_t(3 * h->plane));
    }
    if (err == cudaSuccess) {
        err = cudaDeviceSynchronize();
    }
    if (err != cudaSuccess) {
        cudaFree(h->work);
        delete h;
        return als::report_error(ALS_E_CUDA, (std::string("diffusion create: ") +
            cudaGetErrorString(err)).c_str());
    }
    *out = h;
    return ALS_OK;
}

int als_diffusion_apply(als_diffusion* h, const double* const* conserved, double* const* out,
    void* stream) {
    if (!h || !conserved || !out) {
        return als::report_error(ALS_E_INVALID, "invalid diffusion arguments");
    }
    Ptrs U;
    OutPtrs O;
    std::memset(&U, 0, sizeof(U));
    std::memset(&O, 0, sizeof(O));
    for (int v = 0; v < h->nv; ++v) {
        if (!conserved[v] || !out[v]) {
            return als::report_error(ALS_E_INVALID, "null plane");
        }
        U.p[v] = conserved[v];
        O.p[v] = out[v];
    }
    cudaError_t err = cudaSetDevice(h->device);
    const cudaStream_t st = (cudaStream_t)stream;
    // directions in order, each on the output of the previous
    // (TecnoDiffusionCPU.cpp:140-165)
    switch (h->grid.dimension) {
    case 1:
        if (err == cudaSuccess) err = run_direction<1, 0>(h, U, O, st);
        break;
    case 2:
        if (err == cudaSuccess) err = run_direction<2, 0>(h, U, O, st);
        if (err == cudaSuccess) err = run_direction<2, 1>(h, U, O, st);
        break;
    default:
        if (err == cudaSuccess) err = run_direction<3, 0>(h, U, O, st);
        if (err == cudaSuccess) err = run_direction<3, 1>(h, U, O, st);
        if (err == cudaSuccess) err = run_direction<3, 2>(h, U, O, st);
        break;
    }
    if (err != cudaSuccess) {
        return als::report_error(ALS_E_CUDA, (std::string("diffusion apply: ") +
            cudaGetErrorString(err)).c_str());
    }
    return ALS_OK;
}

int als_diffusion_destroy(als_diffusion* h) {
    if (!h) {
        return ALS_OK;
    }
    cudaSetDevice(h->device);
    cudaFree(h->work);
    delete h;
    return ALS_OK;
}

} // extern "C"
