// Smaller kernels around the fused stage kernel:
//   * fe_update          ForwardEuler's second half plus step bookkeeping
//   * combine            one Integrator::performSubstep stage combination
//                        for the plug-in path (ForwardEuler.cpp:32-51,
//                        RungeKutta2.cpp:37-67, RungeKutta3.cpp:49-86)
//   * fill_ghosts        Boundary::applyBoundaryConditions (BoundaryCPU.cpp:30-106)
//   * reconstruct_dir    Reconstruction::performReconstruction (ReconstructionCPU.cpp:37-97,
//                        ENOCPU.cpp:41-187) for the plug-in path
#pragma once

#include "stage_kernel.cuh"

namespace als {

// U^{n+1} = (dt/dx) L + U^n over every padded cell (ghost cells of L and U^n
// are already images, so the result's ghosts are images too), then the
// constraint check and the step bookkeeping of the last block.
template<class R, int NV>
__global__ void __launch_bounds__(256) fe_update(const R* L, R* un, long long plane,
    long long sample_stride, StepState* state, int member0, double gamma) {
    const int member = member0 + blockIdx.y;
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
            volatile StepState* vs = st;
            vs->dt = dt;
            const double t = vs->t + dt;
            vs->t = t;
            vs->steps = vs->steps + 1;
            vs->ws[0] = 0;
            vs->ws[1] = 0;
            vs->ws[2] = 0;
            vs->arrive = 0;
            if (vs->status != 0 && vs->bad_step < 0) {
                vs->bad_step = vs->steps;
            }
            if (t >= vs->end_time || vs->status != 0 || vs->steps >= vs->max_steps) {
                vs->done = 1;
            }
        }
    }
}

// Stage combination of the plug-in Integrator path, applied to every element
// like the reference's Volume operators: out = L on entry.
//   integrator 0 (FE):  out = c*L + Us
//   integrator 1 (RK2): s0 as FE; s1: ((c*L + Us) + U0) * 0.5
//   integrator 2 (RK3): s0 as FE; s1: ((c*L + Us) * 1/3 + U0) * 3/4;
//                       s2: ((c*L + Us) * 2 + U0) * 1/3
template<class R>
__global__ void __launch_bounds__(256) combine(R* out, const R* us, const R* u0, long long count,
    R c, int integrator, int substep) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        R x = out[i] * c;
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

// Every ghost cell takes the value of its source interior cell; sides are
// independent once n >= G, so one pass reproduces the reference's
// side-by-side sequential fill, corners included.
template<class R>
__global__ void __launch_bounds__(256) fill_ghosts(R* planes, int nvar, long long plane,
    long long sample_stride, int dim, int n0, int n1, int n2, int G, int bc) {
    const int N0 = n0 + 2 * G;
    const int N1 = dim > 1 ? n1 + 2 * G : 1;
    const int N2 = dim > 2 ? n2 + 2 * G : 1;
    planes += (long long)blockIdx.y * sample_stride;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane;
         i += (long long)gridDim.x * blockDim.x) {
        const int x = int(i % N0);
        const int y = int((i / N0) % N1);
        const int z = int(i / ((long long)N0 * N1));
        const int sx = ghost_source(x, n0, G, bc);
        const int sy = dim > 1 ? ghost_source(y, n1, G, bc) : y;
        const int sz = dim > 2 ? ghost_source(z, n2, G, bc) : z;
        if (sx == x && sy == y && sz == z) {
            continue;
        }
        const long long s = ((long long)sz * N1 + sy) * N0 + sx;
        for (int v = 0; v < nvar; ++v) {
            planes[v * plane + i] = planes[v * plane + s];
        }
    }
}

// Left/right values of every cell the reference reconstructs along `dir`:
// cells [G-1, N-G] along dir, interior across (ReconstructionCPU.cpp:71-96).
template<class R, int NV, int RECON>
__global__ void __launch_bounds__(256) reconstruct_dir(const R* in, R* left, R* right,
    long long plane, int dim, int N0, int N1, int N2, int G, int dir) {
    const int e0 = dir == 0 ? N0 - 2 * G + 2 : N0 - 2 * G;
    const int e1 = dim > 1 ? (dir == 1 ? N1 - 2 * G + 2 : N1 - 2 * G) : 1;
    const int e2 = dim > 2 ? (dir == 2 ? N2 - 2 * G + 2 : N2 - 2 * G) : 1;
    const long long count = (long long)e0 * e1 * e2;
    const int s = dir == 0 ? 1 : (dir == 1 ? N0 : N0 * N1);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        const int a = int(i % e0);
        const int b = int((i / e0) % e1);
        const int c = int(i / ((long long)e0 * e1));
        const int x = a + G - (dir == 0 ? 1 : 0);
        const int y = dim > 1 ? b + G - (dir == 1 ? 1 : 0) : 0;
        const int z = dim > 2 ? c + G - (dir == 2 ? 1 : 0) : 0;
        const long long idx = ((long long)z * N1 + y) * N0 + x;
        R l[NV], r[NV];
        reconstruct<R, NV, RECON>(in + idx, (int)plane, s, l, r);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            left[v * plane + idx] = l[v];
            right[v * plane + idx] = r[v];
        }
    }
}

} // namespace als
