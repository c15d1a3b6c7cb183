// Smaller kernels around the fused stage kernel:
//   * fe_update          ForwardEuler's second half plus step bookkeeping
//   * combine            one Integrator::performSubstep stage combination
//                        for the plug-in path (ForwardEuler.cpp:32-51,
//                        RungeKutta2.cpp:37-67, RungeKutta3.cpp:49-86)
//   * fill_ghosts        Boundary::applyBoundaryConditions (BoundaryCPU.cpp:30-106)
//   * reconstruct_dir    Reconstruction::performReconstruction (ReconstructionCPU.cpp:37-97,
//                        ENOCPU.cpp:41-187) for the plug-in path
//   * region_sums        FP64 sums of every variable over a box of cells, per
//                        member (conservation check, observables)
//   * welford_merge      FP64 mean / M2 of an ensemble, merged chunk by chunk
#pragma once

#include "stage_kernel.cuh"

namespace als {

// One pointer per conserved variable.
template<class R>
struct Planes {
    R* p[kMaxVars];
};

// U^{n+1} = (dt/dx) L + U^n over every padded cell (ghost cells of L and U^n
// are already images, so the result's ghosts are images too), then the
// constraint check and the step bookkeeping of the last block.
template<class R, int NV>
__global__ void __launch_bounds__(256) fe_update(const R* L, R* un, long long plane,
    long long sample_stride, StepState* state, double gamma) {
    const int member = blockIdx.y;
    StepState* st = state + member;
    if (((volatile StepState*)st)->done) {
        return;
    }
    const double dt = step_dt(st);
    const R c = R(dt / st->dx[0]);
    L += (long long)member * sample_stride;
    un += (long long)member * sample_stride;
    bool bad = false;
    long long bad_idx = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane;
         i += (long long)gridDim.x * blockDim.x) {
        R val[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            R x = L[v * plane + i] * c;
            x = x + un[v * plane + i];
            un[v * plane + i] = x;
            val[v] = x;
        }
        if (!bad && !obeys_constraints<R, NV>(val, R(gamma))) {
            bad = true;
            bad_idx = i;
        }
    }
    if (bad) {
        atomicOr(&st->status, 1);
        atomicMin((unsigned long long*)&st->bad_index, (unsigned long long)bad_idx);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned int prev = atomicAdd(&st->arrive, 1u);
        if (prev == gridDim.x - 1) {
            __threadfence();
            ((volatile StepState*)st)->dt = dt;
            finish_step(st);
        }
    }
}

// Stage combination of the plug-in Integrator path, applied to every element
// like the reference's Volume operators: out = L on entry.
//   integrator 0 (FE):  out = c*L + Us
//   integrator 1 (RK2): s0 as FE; s1: ((c*L + Us) + U0) * 0.5
//   integrator 2 (RK3): s0 as FE; s1: ((c*L + Us) * 1/3 + U0) * 3/4;
//                       s2: ((c*L + Us) * 2 + U0) * 1/3
//   integrator 3 (RK4): s0, s1: (c*L) * 0.5 + U0; s2: c*L + U0
//                       (RungeKutta4.cpp:66-78; s3 is combine_rk4_final)
template<class R>
__global__ void __launch_bounds__(256) combine(R* out, const R* us, const R* u0, long long count,
    R c, int integrator, int substep) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        R x = out[i] * c;
        if (integrator == 3) {
            if (substep < 2) {
                x = x * R(0.5);
            }
            out[i] = x + u0[i];
            continue;
        }
        x = x + us[i];
        if (integrator == 2 && substep == 1) {
            x = x * R(1. / 3.);
            x = x + u0[i];
            x = x * R(3. / 4.);
        } else if (integrator == 2 && substep == 2) {
            x = x * R(2);
            x = x + u0[i];
            x = x * R(1. / 3.);
        } else if (integrator == 1 && substep == 1) {
            x = x + u0[i];
            x = x * R(0.5);
        }
        out[i] = x;
    }
}

// RK4's last stage, Volume::addLinearCombination (Volume.cpp:359-370,
// HostMemory.cpp:261-280): out = a1 L + a2 U1 + a3 U2 + a4 U3 + a5 U0,
// summed left to right, with a1 = (1/6)(dt/dx), a2 = a4 = 1/3, a3 = 2/3,
// a5 = -1/3 (RungeKutta4.cpp:80-87).
template<class R>
__global__ void __launch_bounds__(256) combine_rk4_final(R* out, const R* u0, const R* u1,
    const R* u2, const R* u3, long long count, R a1) {
    const R a2 = R(1.0 / 3.0), a3 = R(2.0 / 3.0), a4 = R(1.0 / 3.0), a5 = R(-1.0 / 3.0);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        R x = a1 * out[i];
        x = x + a2 * u1[i];
        x = x + a3 * u2[i];
        x = x + a4 * u3[i];
        x = x + a5 * u0[i];
        out[i] = x;
    }
}

// Maps a padded coordinate to the interior cell whose value it holds after
// the boundary fill (identity for interior cells).
__device__ __forceinline__ int ghost_source(int p, int n, int G, int bc) {
    if (p >= G && p < n + G) {
        return p;
    }
    if (bc == BC_PERIODIC) {
        return p < G ? p + n : p - n;
    }
    return p < G ? 2 * G - 1 - p : 2 * (n + G) - 1 - p;
}

// Padded cells outside the interior box (the ghost shell) of one plane.
// Inactive directions have n = 1 and no ghosts.
__host__ __device__ inline long long ghost_shell_cells(int dim, int n0, int n1, int n2, int G) {
    const long long N0 = n0 + 2LL * G;
    const long long N1 = dim > 1 ? n1 + 2LL * G : 1;
    const long long N2 = dim > 2 ? n2 + 2LL * G : 1;
    const long long inner = (long long)n0 * (dim > 1 ? n1 : 1) * (dim > 2 ? n2 : 1);
    return N0 * N1 * N2 - inner;
}

// Padded coordinates of shell cell k (0 <= k < ghost_shell_cells): first
// the 2G whole z-planes (3-D), then in each interior plane its 2G whole
// rows (2-D and up), then in each interior row its 2G ghost cells.
__device__ __forceinline__ void ghost_shell_cell(long long k, int dim, int n0, int n1, int n2,
    int G, int& x, int& y, int& z) {
    const int Gy = dim > 1 ? G : 0;
    const int Gz = dim > 2 ? G : 0;
    const long long N0 = n0 + 2LL * G;
    const long long N1 = n1 + 2LL * Gy;
    const long long plane2 = N0 * N1;
    const long long outer_z = 2LL * Gz * plane2;
    if (k < outer_z) {
        const long long slab = k / plane2;
        z = slab < Gz ? int(slab) : int(slab) + n2;
        const long long r = k - slab * plane2;
        y = int(r / N0);
        x = int(r - (long long)y * N0);
        return;
    }
    k -= outer_z;
    const long long shell2 = plane2 - (long long)n0 * n1;
    const long long zi = k / shell2;
    z = Gz + int(zi);
    long long r = k - zi * shell2;
    const long long outer_y = 2LL * Gy * N0;
    if (r < outer_y) {
        const long long row = r / N0;
        y = row < Gy ? int(row) : int(row) + n1;
        x = int(r - row * N0);
        return;
    }
    r -= outer_y;
    const long long yi = r / (2 * G);
    y = Gy + int(yi);
    const int c = int(r - yi * 2 * G);
    x = c < G ? c : c + n0;
}

// Every ghost cell takes the value of its source interior cell; sides are
// independent once n >= G, so one pass reproduces the reference's
// side-by-side sequential fill, corners included.  The threads walk the
// ghost shell only (4 x 8,208 cells of a 1024^2 grid's 1,056,784).
// blockIdx.y = member.
template<class R>
__global__ void __launch_bounds__(256) fill_ghosts(Planes<R> planes, int nvar, long long plane,
    long long member_stride, int dim, int n0, int n1, int n2, int G, int bc) {
    const int N0 = n0 + 2 * G;
    const int N1 = dim > 1 ? n1 + 2 * G : 1;
    const long long base = (long long)blockIdx.y * member_stride;
    const long long shell = ghost_shell_cells(dim, n0, n1, n2, G);
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < shell;
         k += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        ghost_shell_cell(k, dim, n0, n1, n2, G, x, y, z);
        const int sx = ghost_source(x, n0, G, bc);
        const int sy = dim > 1 ? ghost_source(y, n1, G, bc) : y;
        const int sz = dim > 2 ? ghost_source(z, n2, G, bc) : z;
        const long long i = ((long long)z * N1 + y) * N0 + x;
        const long long s = ((long long)sz * N1 + sy) * N0 + sx;
        for (int v = 0; v < nvar; ++v) {
            R* p = planes.p[v] + base;
            p[i] = p[s];
        }
    }
    (void)plane;
}

// Stencil values from per-variable planes.
template<class R, int NV>
struct PlaneFetch {
    const Planes<R>* planes;
    long long idx;
    long long s;
    __device__ __forceinline__ R at(int v, int o) const { return planes->p[v][idx + o * s]; }
    __device__ __forceinline__ R dyn(int v, int o) const { return planes->p[v][idx + o * s]; }
};

// Left/right values of every cell the reference reconstructs along `dir`:
// cells [G-1, N-G] along dir, interior across (ReconstructionCPU.cpp:71-96).
template<class R, int NV, int RECON>
__global__ void __launch_bounds__(256) reconstruct_dir(Planes<R> in, Planes<R> left,
    Planes<R> right, int dim, int N0, int N1, int N2, int G, int dir, double gamma) {
    // WENOCPU<3> also reconstructs every cell across the direction, ghosts
    // included (WENOCPU.cpp:100-106); the others only the interior
    const int gt = RECON == RECON_WENO3 ? 0 : G;
    const int e0 = dir == 0 ? N0 - 2 * G + 2 : N0 - 2 * gt;
    const int e1 = dim > 1 ? (dir == 1 ? N1 - 2 * G + 2 : N1 - 2 * gt) : 1;
    const int e2 = dim > 2 ? (dir == 2 ? N2 - 2 * G + 2 : N2 - 2 * gt) : 1;
    const long long count = (long long)e0 * e1 * e2;
    const long long s = dir == 0 ? 1 : (dir == 1 ? N0 : (long long)N0 * N1);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        const int a = int(i % e0);
        const int b = int((i / e0) % e1);
        const int c = int(i / ((long long)e0 * e1));
        const int x = dir == 0 ? a + G - 1 : a + gt;
        const int y = dim > 1 ? (dir == 1 ? b + G - 1 : b + gt) : 0;
        const int z = dim > 2 ? (dir == 2 ? c + G - 1 : c + gt) : 0;
        const long long idx = ((long long)z * N1 + y) * N0 + x;
        PlaneFetch<R, NV> f{&in, idx, s};
        R l[NV], r[NV];
        reconstruct_f<R, NV, RECON>(f, l, r, R(gamma));
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            left.p[v][idx] = l[v];
            right.p[v][idx] = r[v];
        }
    }
}

// FP64 sums of every variable over the padded-coordinate box [lo, hi) of
// each member (one block per member, fixed summation order, so the result is
// reproducible).  out[member * nvar + v].
template<class R>
__global__ void __launch_bounds__(256) region_sums(const R* states, long long plane,
    long long member_stride, int nvar, int N0, int N1, int lo0, int lo1, int lo2, int hi0,
    int hi1, int hi2, double* out) {
    const int member = blockIdx.x;
    const R* base = states + (long long)member * member_stride;
    const int e0 = hi0 - lo0, e1 = hi1 - lo1, e2 = hi2 - lo2;
    const long long count = (long long)e0 * e1 * e2;
    __shared__ double part[kMaxVars][256 / 32];
    double sum[kMaxVars] = {0, 0, 0, 0, 0};
    for (long long i = threadIdx.x; i < count; i += blockDim.x) {
        const int x = lo0 + int(i % e0);
        const int y = lo1 + int((i / e0) % e1);
        const int z = lo2 + int(i / ((long long)e0 * e1));
        const long long idx = ((long long)z * N1 + y) * N0 + x;
        for (int v = 0; v < nvar; ++v) {
            sum[v] += double(base[v * plane + idx]);
        }
    }
    for (int v = 0; v < nvar; ++v) {
        double s = sum[v];
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_down_sync(0xffffffffu, s, o);
        }
        if ((threadIdx.x & 31) == 0) {
            part[v][threadIdx.x >> 5] = s;
        }
    }
    __syncthreads();
    if (threadIdx.x < nvar) {
        double s = 0;
        for (int k = 0; k < 256 / 32; ++k) {
            s += part[threadIdx.x][k];
        }
        out[member * nvar + threadIdx.x] = s;
    }
}

// Merges `members` states (member j at states + j*member_stride) into the
// running FP64 (n_prev, mean, m2) of every element (Chan et al.'s pairwise
// update): chunk mean and chunk M2 in FP64, then
//   n = n_prev + k, d = mean_k - mean, mean += d*k/n, m2 += m2_k + d*d*n_prev*k/n.
template<class R>
__global__ void __launch_bounds__(256) welford_merge(const R* states, long long count,
    int members, long long member_stride, double* mean, double* m2, long long n_prev) {
    const double k = double(members);
    const double n = double(n_prev) + k;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        double s = 0;
        for (int j = 0; j < members; ++j) {
            s += double(states[(long long)j * member_stride + i]);
        }
        const double cm = s / k;
        double cm2 = 0;
        for (int j = 0; j < members; ++j) {
            const double d = double(states[(long long)j * member_stride + i]) - cm;
            cm2 += d * d;
        }
        const double d = cm - mean[i];
        mean[i] = mean[i] + d * (k / n);
        m2[i] = m2[i] + cm2 + d * d * (double(n_prev) * k / n);
    }
}

// Chan's merge of another accumulator (n_b, mean_b, m2_b) into (n_a, mean, m2).
__global__ void __launch_bounds__(256) welford_combine(double* mean, double* m2, long long n_a,
    const double* mean_b, const double* m2_b, long long n_b, long long count) {
    const double n = double(n_a) + double(n_b);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        const double d = mean_b[i] - mean[i];
        mean[i] = mean[i] + d * (double(n_b) / n);
        m2[i] = m2[i] + m2_b[i] + d * d * (double(n_a) * double(n_b) / n);
    }
}

// variance = m2 / n (the biased estimator of MeanVariance, MeanVariance.cpp:55-67).
__global__ void __launch_bounds__(256) welford_finish(const double* mean, const double* m2,
    long long n, long long count, double* mean_out, double* var_out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        if (mean_out) {
            mean_out[i] = mean[i];
        }
        if (var_out) {
            var_out[i] = m2[i] / double(n);
        }
    }
}

} // namespace als
