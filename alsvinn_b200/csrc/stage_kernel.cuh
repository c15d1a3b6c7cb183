// The fused cell-update stage kernel.
//
// One thread block owns a tile of interior cells.  It stages the tile plus a
// halo of G cells (every variable) in shared memory, then, direction by
// direction, reconstructs every cell the faces need, evaluates each face
// flux exactly once, and accumulates the net flux of its cells in registers.
// The epilogue applies the Runge-Kutta stage combination, writes the result
// and (optionally) the boundary images of the updated cell, so no separate
// ghost-fill pass is needed.
//
// This replaces, per stage, the reference's chain of kernels and host syncs
// (alsfvm/src/numflux/NumericalFluxCUDA.cu:39-160,263-414,
//  alsfvm/src/reconstruction/ReconstructionCUDA.cu:31-100,
//  alsfvm/src/cuda/vector_operations.cu:24-95,233-335,
//  alsfvm/src/boundary/BoundaryCUDA.cu:26-160) while keeping the arithmetic
// of the CPU path (alsfvm/src/numflux/NumericalFluxCPU.cpp:32-221,
// alsfvm/src/integrator/{ForwardEuler,RungeKutta2,RungeKutta3}.cpp).
//
// The first stage of a time step stores the unscaled net flux L(U^n) and
// reduces the face wave speeds; the second stage rebuilds U1 = (dt/dx)L + U^n
// while it loads its halo, so the CFL max never needs a separate pass over
// the state and no stage waits on the host.
#pragma once

#include "euler_math.cuh"
#include "stage_params.h"

namespace als {

// Tile shape (X x Y x Z cells), threads per block T and the most blocks per
// SM the register budget is sized for (B), per dimension.
//
// The kernel is bound by the issue of long dependent FP64 sequences (the
// divide and square-root routines), so occupancy and lane utilisation
// decide its speed.  In 2-D a 32x16 tile needs 544/576 reconstructions and
// 528/544 face fluxes along x/y: with 576 threads every one of these phases
// is a single round (92-100% of the lanes busy), and two such blocks per SM
// give 36 warps.  Measured on KH 1024^2 (ms per RK3 step, FP64, B200):
//   32x16 / 576 threads / 2 blocks (56 regs)   0.420
//   16x16 / 288 threads / 3 blocks (72 regs)   0.438
//   32x8  / 320 threads / 3 blocks (64 regs)   0.454
//   32x8  / 256 threads / 4 blocks (64 regs)   0.490
//   32x16 / 256 threads / 2 blocks (~100 regs) 0.556
//   32x12 / 384 threads / 3 blocks             0.507
//   48x12 / 576 threads / 2 blocks             0.579
// (the first row is 0.433 since the barrier at the end of each direction
// went, 0.430 since the constraint check skips its velocity divisions when
// rho >= 1, 0.407 since the HLL3 star branch forms only the chosen side's
// point flux and interior cells skip the boundary-image code, 0.381 since
// the staging decodes each box position once for all variables).  Keeping
// the tile's U^n in shared memory from the load phase for the epilogue,
// instead of reading it there, ran slower (0.434 vs 0.430; FP32 members 3 %
// slower); so did the per-cell net-flux sums in shared memory (0.390 vs
// 0.381), a 32x14 tile of 512 threads at 64 registers (0.394) and the x
// direction done per warp on a row of a 30x17 tile with warp shuffles
// instead of shared memory and barriers (0.423); so did one block of 576
// threads per SM, with registers to spare and no spills (0.384 vs 0.376).
// All of these are build-time knobs; the FP32 units build with three blocks
// per SM.
#ifndef ALS_TILE2_X
#define ALS_TILE2_X 32
#endif
#ifndef ALS_TILE2_Y
#define ALS_TILE2_Y 16
#endif
#ifndef ALS_STAGE2_THREADS
#define ALS_STAGE2_THREADS 576
#endif
#ifndef ALS_STAGE2_BLOCKS
#define ALS_STAGE2_BLOCKS 2
#endif
// SHAPE 0 is each dimension's default tile.  2-D also builds SHAPE 1, a
// 16 x 16 tile of 288 threads: more halo work per cell than 32 x 16, but
// more resident blocks per SM and finer work items, which can pay on small
// grids or many members; the schedule tuner chooses per grid level
// (als_solver_tune).  Measured alone on KH 1024^2 (FP64, ms per RK3 step):
// 32 x 16 0.407, 16 x 16 0.438.
#ifndef ALS_STAGE2S_BLOCKS
#define ALS_STAGE2S_BLOCKS 3
#endif
template<int DIM, int SHAPE = 0> struct TileShape;
template<> struct TileShape<1, 0> {
    static constexpr int X = 256, Y = 1, Z = 1, T = 256, B = 4;
};
template<> struct TileShape<2, 0> {
    static constexpr int X = ALS_TILE2_X, Y = ALS_TILE2_Y, Z = 1, T = ALS_STAGE2_THREADS,
        B = ALS_STAGE2_BLOCKS;
};
template<> struct TileShape<2, 1> {
    static constexpr int X = 16, Y = 16, Z = 1, T = 288, B = ALS_STAGE2S_BLOCKS;
};
#ifndef ALS_TILE3_X
#define ALS_TILE3_X 8
#endif
#ifndef ALS_TILE3_Y
#define ALS_TILE3_Y 8
#endif
#ifndef ALS_TILE3_Z
#define ALS_TILE3_Z 4
#endif
// 3-D: an 8x8x4 tile needs 320/320/384 reconstructions and 288/288/320
// face fluxes along x/y/z; its FP64 shared memory (90 KB) allows two blocks
// per SM.  Measured on KH 128^3 x 8 members (FP64, ms per RK3 step):
//   8x8x4 / 320 threads / 2 blocks (96 regs)   15.9  (12.4 with the current flux and staging)
//   8x4x4 / 192 threads / 4 blocks             17.2
//   8x8x4 / 384 threads / 2 blocks (80 regs)   17.2
//   8x8x2 / 256 threads / 3 blocks             19.8
//   8x8x4 / 256 threads / 2 blocks             20.1
//   8x8x2 / 192 threads / 4 blocks             21.3
#ifndef ALS_STAGE3_THREADS
#define ALS_STAGE3_THREADS 320
#endif
#ifndef ALS_STAGE3_BLOCKS
#define ALS_STAGE3_BLOCKS 2
#endif
template<> struct TileShape<3, 0> {
    static constexpr int X = ALS_TILE3_X, Y = ALS_TILE3_Y, Z = ALS_TILE3_Z, T = ALS_STAGE3_THREADS,
        B = ALS_STAGE3_BLOCKS;
};
// 3-D shape 1: 16 x 16 columns marching along z over segments of
// ALS_ZMARCH_SEG cells (stage_zmarch.cuh), 288 threads (96 registers at two
// blocks per SM).  KH 128^3 x 8, FP64, ms per RK3 step: 10.59 (segments of
// 16: 10.66; 320 threads: 10.60; 256 threads, 128 registers but two rounds
// per x-y phase: 12.17), against 12.40 for the 8x8x4 boxes.
#ifndef ALS_ZMARCH_SEG
#define ALS_ZMARCH_SEG 32
#endif
#ifndef ALS_ZMARCH_BLOCKS
#define ALS_ZMARCH_BLOCKS 2
#endif
#ifndef ALS_ZMARCH_THREADS
#define ALS_ZMARCH_THREADS 288
#endif
template<> struct TileShape<3, 1> {
    static constexpr int X = 16, Y = 16, Z = ALS_ZMARCH_SEG, T = ALS_ZMARCH_THREADS,
        B = ALS_ZMARCH_BLOCKS;
};

// Shapes built per (dimension, reconstruction, flux): the default for every
// combination; in 2-D the 16 x 16 alternative for WENO2 with HLL, HLL3 and
// Central (the ensemble and benchmark configurations); in 3-D the z-marching
// columns for reconstructions that reach one cell each way (WENO2, ENO2, MC,
// MM, WENOF2, none) with the two-point fluxes.
__host__ __device__ constexpr bool shape_built(int dim, int recon, int flux, int shape) {
    return shape == 0 ||
        (shape == 1 && dim == 2 && recon == RECON_WENO2 &&
            (flux == FLUX_HLL || flux == FLUX_HLL3 || flux == FLUX_CENTRAL)) ||
        (shape == 1 && dim == 3 && recon_ghosts(recon) <= 2 && !stencil_flux(flux));
}
constexpr int kMaxShapes = 2;

template<class R, int DIM, int RECON, int FLUX, int SHAPE = 0>
struct StageLayout {
    static constexpr int NV = DIM + 2;
    static constexpr int G = stage_ghosts(RECON, FLUX);
    static constexpr bool STENCIL = stencil_flux(FLUX);
    static constexpr int TX = TileShape<DIM, SHAPE>::X;
    static constexpr int TY = TileShape<DIM, SHAPE>::Y;
    static constexpr int TZ = TileShape<DIM, SHAPE>::Z;
    static constexpr int BX = TX + 2 * G;
    static constexpr int BY = DIM > 1 ? TY + 2 * G : 1;
    static constexpr int BZ = DIM > 2 ? TZ + 2 * G : 1;
    static constexpr int BOX = BX * BY * BZ;
    static constexpr int CELLS = TX * TY * TZ;
    static constexpr int THREADS = TileShape<DIM, SHAPE>::T;
    static constexpr int CPT = (CELLS + THREADS - 1) / THREADS;  // cells per thread
    // reconstructed cells / faces per direction: the tile extent grows by 2 / 1 along it
    static constexpr int REC0 = (TX + 2) * TY * TZ;
    static constexpr int REC1 = DIM > 1 ? TX * (TY + 2) * TZ : 0;
    static constexpr int REC2 = DIM > 2 ? TX * TY * (TZ + 2) : 0;
    // stencil fluxes read the staged cells directly and need no reconstructed values
    static constexpr int REC = STENCIL ? 0
        : (REC0 > REC1 ? (REC0 > REC2 ? REC0 : REC2) : (REC1 > REC2 ? REC1 : REC2));
    static constexpr int FAC0 = (TX + 1) * TY * TZ;
    static constexpr int FAC1 = DIM > 1 ? TX * (TY + 1) * TZ : 0;
    static constexpr int FAC2 = DIM > 2 ? TX * TY * (TZ + 1) : 0;
    static constexpr int FAC = FAC0 > FAC1 ? (FAC0 > FAC2 ? FAC0 : FAC2) : (FAC1 > FAC2 ? FAC1 : FAC2);
    static constexpr size_t SMEM = sizeof(R) * (size_t(NV) * BOX + size_t(2 * NV) * REC + size_t(NV) * FAC);
    static_assert(THREADS % 32 == 0, "whole warps");
    // resident blocks per SM the shared memory allows (228 KB per SM, 1 KB
    // reserved per block), capped; the register budget is sized to match
    static constexpr int BY_SMEM = int((228 * 1024) / (SMEM + 1024));
    static constexpr int BLOCKS = BY_SMEM < 1 ? 1
        : (BY_SMEM > TileShape<DIM, SHAPE>::B ? TileShape<DIM, SHAPE>::B : BY_SMEM);
};

// dt of the step (Integrator.cpp:20-46) followed by the end-time clamp
// (FixedIntervalWriter.cpp:45-53): dt = min(cfl / sum_d ws_d/dx_d, T - t).
__device__ __forceinline__ double step_dt(const StepState* st) {
    double total = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (st->dx[d] == 0) {
            continue;
        }
        total += __longlong_as_double((long long)st->ws[d]) / st->dx[d];
    }
    double dt = st->cfl / total;
    const double rest = st->end_time - st->t;
    return rest < dt ? rest : dt;
}

// Padded positions that hold a copy of interior cell i along one direction
// (the cell itself first).  Neumann mirrors (Neumann.hpp:24-35), periodic
// wraps (Periodic.hpp:24-42); valid for n >= G.
__device__ __forceinline__ int boundary_images(int i, int n, int G, int bc, int* pos) {
    int c = 0;
    pos[c++] = i + G;
    if (bc == BC_PERIODIC) {
        if (i >= n - G) {
            pos[c++] = i + G - n;
        }
        if (i < G) {
            pos[c++] = i + G + n;
        }
    } else {
        if (i < G) {
            pos[c++] = G - 1 - i;
        }
        if (i >= n - G) {
            pos[c++] = 2 * n + G - 1 - i;
        }
    }
    return c;
}

// The same for subdomain c (of p along the direction) of a split grid: a
// side with a neighbouring subdomain sends the cell to that neighbour's
// ghost layer (step -1 / +1: the member holding the image), a physical side
// takes the boundary condition's image within the subdomain (step 0), as
// CartesianCellExchanger.cpp:51-100 and the boundary do between them.
__device__ __forceinline__ int subdomain_images(int i, int n, int G, int bc, int c, int p,
    int* pos, int* step) {
    int k = 0;
    pos[k] = i + G;
    step[k++] = 0;
    const bool low_neighbour = p > 1 && (c > 0 || bc == BC_PERIODIC);
    const bool high_neighbour = p > 1 && (c < p - 1 || bc == BC_PERIODIC);
    if (i < G) {
        if (low_neighbour || bc == BC_PERIODIC) {
            // the low neighbour's (or, alone along this direction, our own) high ghosts
            pos[k] = i + G + n;
            step[k++] = low_neighbour ? -1 : 0;
        } else {
            pos[k] = G - 1 - i;
            step[k++] = 0;
        }
    }
    if (i >= n - G) {
        if (high_neighbour || bc == BC_PERIODIC) {
            pos[k] = i + G - n;
            step[k++] = high_neighbour ? 1 : 0;
        } else {
            pos[k] = 2 * n + G - 1 - i;
            step[k++] = 0;
        }
    }
    return k;
}

// Simulator::checkConstraints (CPUCellComputer.cpp:80-128, Euler.hpp:269-277):
// all conserved values and p, u finite, rho > 0, p > 0.
template<class R, int NV>
__device__ __forceinline__ bool obeys_constraints(const R* U, R gamma) {
    bool ok = true;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        ok = ok && isfinite(U[v]);
    }
    R dot = U[1] * U[1];
    if (NV > 3) {
        dot = dot + U[2] * U[2];
    }
    if (NV > 4) {
        dot = dot + U[3] * U[3];
    }
    const R ie = U[NV - 1] - R(0.5) * dot / U[0];
    const R p = (gamma - R(1)) * ie;
    // with every U[k] finite and U[0] >= 1 each velocity U[k]/U[0] is at most
    // |U[k]| in magnitude, hence finite: the divisions only decide the answer
    // when U[0] < 1
    if (!(U[0] >= R(1))) {
#pragma unroll
        for (int k = 1; k < NV - 1; ++k) {
            ok = ok && isfinite(U[k] / U[0]);
        }
    }
    return ok && isfinite(p) && (U[0] > R(0)) && (p > R(0));
}

// The stencil flux across the face between staged cells `src` and src + S
// (S: the stride along D): TecnoCombined4 / TecnoCombined6
// (TecnoCombined4.hpp:40-60, TecnoCombined6.hpp:40-65) over the
// entropy-conservative two-point flux, combined per component as the
// reference does, with the largest wave speed of its parts.  The
// reference's six-point stencil {-2, -1, 0, 1, 2, 3} lives in an ivec6
// whose constructor stores 0 as the sixth entry (alsutils/vec6.hpp:36-39):
// its u_{i+3} is u_i, so the last term is F(u_i, u_i), the point flux.
template<class R, int NSD, int FLUX, int D>
__device__ __forceinline__ R stencil_face_flux(const R* src, int box, int S, R gamma, R* F) {
    constexpr int NV = NSD + 2;
    R w = R(0);
    auto pair = [&](int a, int b, R* out) {
        R ua[NV], ub[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            ua[v] = src[v * box + a * S];
            ub[v] = src[v * box + b * S];
        }
        FaceState<R, NSD> A, B;
        make_state<R, NSD, D>(ua, gamma, A);
        make_state<R, NSD, D>(ub, gamma, B);
        w = fmax(w, flux_tecno1<R, NSD, D>(A, B, gamma, out));
    };
    R f01[NV], fm11[NV], f02[NV];
    pair(0, 1, f01);
    pair(-1, 1, fm11);
    pair(0, 2, f02);
    if (FLUX == FLUX_TECNO4) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            F[k] = R(4.0 / 3.0) * f01[k] - R(1.0 / 6.0) * (fm11[k] + f02[k]);
        }
    } else {
        R fm21[NV], fm12[NV], f00[NV];
        pair(-2, 1, fm21);
        pair(-1, 2, fm12);
        pair(0, 0, f00);
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            F[k] = (R(3.0 / 2.0) * f01[k] - R(3.0 / 10.0) * (fm11[k] + f02[k])) +
                R(1.0 / 30.0) * ((fm21[k] + fm12[k]) + f00[k]);
        }
    }
    return w;
}

template<class R>
__device__ __forceinline__ R warp_max(R v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    return v;
}

template<class R, int DIM, int RECON, int FLUX, int SHAPE, int KIND, int D>
__device__ __forceinline__ void stage_direction(const GridDesc& gd, R gamma, const R* box, R* rec,
    R* flx, R (&acc)[StageLayout<R, DIM, RECON, FLUX, SHAPE>::CPT][DIM + 2], R& wmax, int x0, int y0,
    int z0) {
    typedef StageLayout<R, DIM, RECON, FLUX, SHAPE> Lay;
    constexpr int NV = Lay::NV;
    constexpr int G = Lay::G;
    // extents of the reconstructed-cell index space (x fastest), offset -1 along D
    constexpr int E0 = Lay::TX + (D == 0 ? 2 : 0);
    constexpr int E1 = Lay::TY + (D == 1 ? 2 : 0);
    constexpr int RC = E0 * E1 * (Lay::TZ + (D == 2 ? 2 : 0));
    // extents of the face index space, offset -1 along D
    constexpr int F0 = Lay::TX + (D == 0 ? 1 : 0);
    constexpr int F1 = Lay::TY + (D == 1 ? 1 : 0);
    constexpr int FC = F0 * F1 * (Lay::TZ + (D == 2 ? 1 : 0));
    constexpr int S = D == 0 ? 1 : (D == 1 ? Lay::BX : Lay::BX * Lay::BY);
    const int tid = threadIdx.x;

    for (int i = tid; i < (Lay::STENCIL ? 0 : RC); i += Lay::THREADS) {
        const int ex = i % E0;
        const int ey = (i / E0) % E1;
        const int ez = i / (E0 * E1);
        const int bx = ex - (D == 0 ? 1 : 0) + G;
        const int by = DIM > 1 ? ey - (D == 1 ? 1 : 0) + G : 0;
        const int bz = DIM > 2 ? ez - (D == 2 ? 1 : 0) + G : 0;
        const R* src = box + (bz * Lay::BY + by) * Lay::BX + bx;
        R l[NV], r[NV];
        reconstruct<R, NV, RECON>(src, Lay::BOX, S, l, r, gamma);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            rec[v * RC + i] = l[v];
            rec[(NV + v) * RC + i] = r[v];
        }
    }
    __syncthreads();

    const int hiD = D == 0 ? gd.hi[0] : (D == 1 ? gd.hi[1] : gd.hi[2]);
    const int oD = D == 0 ? x0 : (D == 1 ? y0 : z0);
    for (int i = tid; i < FC; i += Lay::THREADS) {
        const int fx = i % F0;
        const int fy = (i / F0) % F1;
        const int fz = i / (F0 * F1);
        R F[NV];
        R w;
        if constexpr (Lay::STENCIL) {
            // the face's left cell, staged at tile cell (fx,fy,fz) - 1 along D
            const int bx = fx - (D == 0 ? 1 : 0) + G;
            const int by = DIM > 1 ? fy - (D == 1 ? 1 : 0) + G : 0;
            const int bz = DIM > 2 ? fz - (D == 2 ? 1 : 0) + G : 0;
            w = stencil_face_flux<R, DIM, FLUX, D>(box + (bz * Lay::BY + by) * Lay::BX + bx,
                Lay::BOX, S, gamma, F);
        } else {
            // face between reconstructed cells (fx,fy,fz) and its +D neighbour in E space
            const int rl = (fz * E1 + fy) * E0 + fx;
            const int rr = rl + (D == 0 ? 1 : (D == 1 ? E0 : E0 * E1));
            R ul[NV], ur[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                ul[v] = rec[(NV + v) * RC + rl];
                ur[v] = rec[v * RC + rr];
            }
            w = face_flux<R, DIM, FLUX, D>(ul, ur, gamma, F);
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            flx[v * FC + i] = F[v];
        }
        if (KIND == KIND_FLUX0) {
            // the face lies between cells oD+f-1 and oD+f of the update region
            const int f = D == 0 ? fx : (D == 1 ? fy : fz);
            bool valid = oD + f - 1 <= hiD - 1;
            if (D != 0) {
                valid = valid && (x0 + fx < gd.hi[0]);
            }
            if (D != 1 && DIM > 1) {
                valid = valid && (y0 + fy < gd.hi[1]);
            }
            if (D != 2 && DIM > 2) {
                valid = valid && (z0 + fz < gd.hi[2]);
            }
            if (valid && wmax < w) {
                wmax = w;
            }
        }
    }
    __syncthreads();

#pragma unroll
    for (int k = 0; k < Lay::CPT; ++k) {
        const int ci = tid + k * Lay::THREADS;
        if (Lay::CELLS % Lay::THREADS != 0 && ci >= Lay::CELLS) {
            continue;
        }
        const int cx = ci % Lay::TX;
        const int cy = (ci / Lay::TX) % Lay::TY;
        const int cz = ci / (Lay::TX * Lay::TY);
        // left face of cell c has face coordinate c (faces are offset by -1)
        const int fl = (cz * F1 + cy) * F0 + cx;
        const int fr = fl + (D == 0 ? 1 : (D == 1 ? F0 : F0 * F1));
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            // out += temp[x+1] + (-temp[x]) with temp = -F (NumericalFluxCPU.cpp:92,113)
            const R tr = -flx[v * FC + fr];
            const R tl = -flx[v * FC + fl];
            acc[k][v] = acc[k][v] + (tr + (-tl));
        }
    }
    // No barrier here: the next direction's reconstruction writes only `rec`,
    // which this phase does not read, and its face phase (which overwrites
    // `flx`) starts after the barrier that ends that reconstruction, which
    // every thread reaches only after finishing this loop.
}

// Advances the time bookkeeping of a member once its last tile of the last
// stage is done (Simulator.cpp:211-213 and checkConstraints).
__device__ __forceinline__ void finish_step(StepState* st) {
    volatile StepState* vs = st;
    const double t = vs->t + vs->dt;
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

// The stage combination of one updated cell (interior coordinates gx, gy,
// gz; its net flux `acc`; `ub`, its value of the stage's input state as
// staged) and its writes: the cell, its boundary images (or, for a split
// grid, the neighbouring subdomains' ghost cells), and, after the last
// stage, the constraint check.
template<class R, int DIM, int NV, int KIND>
__device__ __forceinline__ void update_cell(const StageParams& P, const LevelDesc& L, int member,
    long long base, R c, R gamma, const R* acc, const R* ub, int gx, int gy, int gz, bool& bad,
    long long& bad_idx) {
    constexpr bool LAST = KIND == KIND_RK3_2 || KIND == KIND_RK2_1;
    const GridDesc& gd = L.grid;
    const StepState* st = L.state ? L.state + (L.subdomains ? 0 : member) : nullptr;
    auto unp = [&](int v) { return static_cast<const R*>(L.un[v]) + base; };
    auto outp = [&](int v) { return static_cast<R*>(L.out[v]) + base; };
    const int px = gx + gd.ghosts;
    const int py = DIM > 1 ? gy + gd.ghosts : 0;
    const int pz = DIM > 2 ? gz + gd.ghosts : 0;
    const long long idx = ((long long)pz * gd.N[1] + py) * gd.N[0] + px;
    R val[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        R x = acc[v];
        if (KIND == KIND_RK2_1) {
            // RungeKutta2.cpp:57-63
            x = x * c;
            x = x + ub[v];
            x = x + unp(v)[idx];
            x = x * R(0.5);
        } else if (KIND == KIND_RK3_1) {
            // RungeKutta3.cpp:65-78
            x = x * c;
            x = x + ub[v];
            x = x * R(1. / 3.);
            x = x + unp(v)[idx];
            x = x * R(3. / 4.);
        } else if (KIND == KIND_RK3_2) {
            // RungeKutta3.cpp:65-83
            x = x * c;
            x = x + ub[v];
            x = x * R(2);
            x = x + unp(v)[idx];
            x = x * R(1. / 3.);
        }
        val[v] = x;
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        outp(v)[idx] = val[v];
    }
    // a cell at least G' = gd.ghosts cells from every side of its grid
    // has no boundary image (only the cells of the outer shell do)
    const int gw = gd.ghosts;
    const bool shell = gx < gw || gx >= gd.n[0] - gw ||
        (DIM > 1 && (gy < gw || gy >= gd.n[1] - gw)) ||
        (DIM > 2 && (gz < gw || gz >= gd.n[2] - gw));
    if (P.write_ghosts && shell) {
        int ix[3], iy[3] = {0, 0, 0}, iz[3] = {0, 0, 0};
        int sx[3] = {0, 0, 0}, sy[3] = {0, 0, 0}, sz[3] = {0, 0, 0};
        int nxi, nyi = 1, nzi = 1;
        // this member's subdomain coordinates (subdomains only)
        int c0 = 0, c1 = 0, c2 = 0;
        if (L.subdomains) {
            c0 = member % L.procs[0];
            c1 = (member / L.procs[0]) % L.procs[1];
            c2 = member / (L.procs[0] * L.procs[1]);
            nxi = subdomain_images(gx, gd.n[0], gd.ghosts, P.bc, c0, L.procs[0], ix, sx);
            if (DIM > 1) {
                nyi = subdomain_images(gy, gd.n[1], gd.ghosts, P.bc, c1, L.procs[1], iy, sy);
            }
            if (DIM > 2) {
                nzi = subdomain_images(gz, gd.n[2], gd.ghosts, P.bc, c2, L.procs[2], iz, sz);
            }
        } else {
            nxi = boundary_images(gx, gd.n[0], gd.ghosts, P.bc, ix);
            if (DIM > 1) {
                nyi = boundary_images(gy, gd.n[1], gd.ghosts, P.bc, iy);
            }
            if (DIM > 2) {
                nzi = boundary_images(gz, gd.n[2], gd.ghosts, P.bc, iz);
            }
        }
        if (nxi * nyi * nzi > 1) {
            for (int a = 0; a < nzi; ++a) {
                for (int b = 0; b < nyi; ++b) {
                    for (int e = 0; e < nxi; ++e) {
                        if (a == 0 && b == 0 && e == 0) {
                            continue;
                        }
                        const long long j = ((long long)iz[a] * gd.N[1] + iy[b]) * gd.N[0] + ix[e];
                        // the member holding the image (steps wrap: periodic splits)
                        long long target = base;
                        if (L.subdomains) {
                            const int t0 = (c0 + sx[e] + L.procs[0]) % L.procs[0];
                            const int t1 = (c1 + sy[b] + L.procs[1]) % L.procs[1];
                            const int t2 = (c2 + sz[a] + L.procs[2]) % L.procs[2];
                            target = (long long)(t0 + L.procs[0] * (t1 + L.procs[1] * t2)) *
                                L.member_stride;
                        }
#pragma unroll
                        for (int v = 0; v < NV; ++v) {
                            static_cast<R*>(L.out[v])[target + j] = val[v];
                        }
                    }
                }
            }
        }
    }
    if (LAST && st && !obeys_constraints<R, NV>(val, gamma)) {
        bad = true;
        // subdomains: the member's padded plane offset first
        bad_idx = L.subdomains ? (long long)member * gd.plane + idx : idx;
    }
}

// One work item: tile `tile` of member `member` of level L.
template<class R, int DIM, int RECON, int FLUX, int SHAPE, int KIND>
__device__ __forceinline__ void stage_tile(const StageParams& P, const LevelDesc& L, int tile,
    int member, unsigned char* smem) {
    typedef StageLayout<R, DIM, RECON, FLUX, SHAPE> Lay;
    constexpr int NV = Lay::NV;
    constexpr int G = Lay::G;
    constexpr bool LAST = KIND == KIND_RK3_2 || KIND == KIND_RK2_1;
    const int tid = threadIdx.x;
    const GridDesc& gd = L.grid;
    // subdomains of one grid share member 0's state
    StepState* st = L.state ? L.state + (L.subdomains ? 0 : member) : nullptr;

    R* box = reinterpret_cast<R*>(smem);
    R* rec = box + NV * Lay::BOX;
    R* flx = rec + 2 * NV * Lay::REC;

    const int tx = tile % gd.tiles[0];
    const int ty = (tile / gd.tiles[0]) % gd.tiles[1];
    const int tz = tile / (gd.tiles[0] * gd.tiles[1]);
    const int x0 = gd.lo[0] + tx * Lay::TX;
    const int y0 = gd.lo[1] + ty * Lay::TY;
    const int z0 = gd.lo[2] + tz * Lay::TZ;
    const long long base = (long long)member * L.member_stride;
    // plane pointers are read from the launch parameters where they are
    // used; arrays of them would be held (and spilled) across the kernel
    auto inp = [&](int v) { return static_cast<const R*>(L.in[v]) + base; };
    auto unp = [&](int v) { return static_cast<const R*>(L.un[v]) + base; };
    const R gamma = R(P.gamma);

    R c = R(0);
    if (KIND == KIND_RK2_1 || KIND == KIND_RK3_1) {
        if (st) {
            const double dt = step_dt(st);
            if (tile == 0 && tid == 0 && (member == 0 || !L.subdomains)) {
                st->dt = dt;
            }
            c = R(dt / st->dx[0]);
        } else {
            c = R(P.c_fixed);
        }
    } else if (KIND == KIND_RK3_2) {
        c = st ? R(st->dt / st->dx[0]) : R(P.c_fixed);
    }

    // stage the tile and its halo; U1 = (dt/dx)*L + U^n is formed here for the
    // second stage (RungeKutta{2,3}.cpp: output *= dt/dx; output += U).
    // Planes may carry more ghost cells than the stencil needs (a diffusion
    // operator with a wider stencil sets the width): `sh` skips the extra ones.
    // A box position is decoded once and serves every variable's plane.
    const int sh = gd.ghosts - G;
    for (int b = tid; b < Lay::BOX; b += Lay::THREADS) {
        const int bx = b % Lay::BX;
        const int by = (b / Lay::BX) % Lay::BY;
        const int bz = b / (Lay::BX * Lay::BY);
        const int px = x0 + bx + sh;
        const int py = DIM > 1 ? y0 + by + sh : 0;
        const int pz = DIM > 2 ? z0 + bz + sh : 0;
        const bool inside = px < gd.N[0] && py < gd.N[1] && pz < gd.N[2];
        const long long idx = inside ? ((long long)pz * gd.N[1] + py) * gd.N[0] + px : 0;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            R val = R(0);
            if (inside) {
                if (KIND == KIND_RK2_1 || KIND == KIND_RK3_1) {
                    val = inp(v)[idx] * c;
                    val = val + unp(v)[idx];
                } else {
                    val = inp(v)[idx];
                }
            }
            box[v * Lay::BOX + b] = val;
        }
    }
    __syncthreads();

    R acc[Lay::CPT][NV];
#pragma unroll
    for (int k = 0; k < Lay::CPT; ++k) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            acc[k][v] = R(0);
        }
    }
    R wmax[3] = {R(0), R(0), R(0)};
    stage_direction<R, DIM, RECON, FLUX, SHAPE, KIND, 0>(gd, gamma, box, rec, flx, acc, wmax[0], x0,
        y0, z0);
    if (DIM > 1) {
        stage_direction<R, DIM, RECON, FLUX, SHAPE, KIND, (DIM > 1 ? 1 : 0)>(gd, gamma, box, rec, flx,
            acc, wmax[1], x0, y0, z0);
    }
    if (DIM > 2) {
        stage_direction<R, DIM, RECON, FLUX, SHAPE, KIND, (DIM > 2 ? 2 : 0)>(gd, gamma, box, rec, flx,
            acc, wmax[2], x0, y0, z0);
    }

    bool bad = false;
    long long bad_idx = 0;
#pragma unroll
    for (int k = 0; k < Lay::CPT; ++k) {
        const int ci = tid + k * Lay::THREADS;
        if (Lay::CELLS % Lay::THREADS != 0 && ci >= Lay::CELLS) {
            continue;
        }
        const int cx = ci % Lay::TX;
        const int cy = (ci / Lay::TX) % Lay::TY;
        const int cz = ci / (Lay::TX * Lay::TY);
        const int gx = x0 + cx, gy = y0 + cy, gz = z0 + cz;
        if (gx >= gd.hi[0] || (DIM > 1 && gy >= gd.hi[1]) || (DIM > 2 && gz >= gd.hi[2])) {
            continue;
        }
        const int bidx = ((DIM > 2 ? cz + G : 0) * Lay::BY + (DIM > 1 ? cy + G : 0)) * Lay::BX + cx + G;
        R ub[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            ub[v] = box[v * Lay::BOX + bidx];
        }
        update_cell<R, DIM, NV, KIND>(P, L, member, base, c, gamma, acc[k], ub, gx, gy, gz, bad,
            bad_idx);
    }

    if (KIND == KIND_FLUX0) {
        __shared__ double wsh[3][Lay::THREADS / 32];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const R w = warp_max(wmax[d]);
            if ((tid & 31) == 0) {
                wsh[d][tid >> 5] = double(w);
            }
        }
        __syncthreads();
        if (tid < DIM) {
            double m = 0;
            for (int k = 0; k < Lay::THREADS / 32; ++k) {
                m = fmax(m, wsh[tid][k]);
            }
            unsigned long long* dst = st ? &st->ws[tid] : (L.ws_out + 3 * member + tid);
            atomicMax(dst, (unsigned long long)__double_as_longlong(m));
        }
    }

    if (LAST && st) {
        if (bad) {
            atomicOr(&st->status, 1);
            atomicMin((unsigned long long*)&st->bad_index, (unsigned long long)bad_idx);
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            const unsigned int prev = atomicAdd(&st->arrive, 1u);
            // subdomains: every tile of every member arrives at the shared state
            const unsigned int tiles = unsigned(L.tiles_per_member) *
                (L.subdomains ? unsigned(L.members) : 1u);
            if (prev == tiles - 1) {
                __threadfence();
                finish_step(st);
            }
        }
    }
}

// Work item w of the launch: its level, member and tile, skipping members
// that are done.
template<class R, int DIM, int RECON, int FLUX, int SHAPE, int KIND>
__device__ __forceinline__ void stage_item(const StageParams& P, long long w, unsigned char* smem) {
    int l = 0;
#pragma unroll
    for (int k = 1; k < kMaxLevels; ++k) {
        if (k < P.nlevels && w >= P.level[k].work_begin) {
            l = k;
        }
    }
    const LevelDesc& L = P.level[l];
    const long long local = w - L.work_begin;
    const int member = int(local / L.tiles_per_member);
    const int tile = int(local - (long long)member * L.tiles_per_member);
    if (L.state) {
        const volatile StepState* st = L.state + (L.subdomains ? 0 : member);
        if (st->done) {
            return;
        }
    }
    stage_tile<R, DIM, RECON, FLUX, SHAPE, KIND>(P, L, tile, member, smem);
}

// Two launch modes.  Without a work counter every block takes the work item
// of its index (the hardware hands out blocks as SMs free up).  With one,
// the launch is persistent: a fixed number of resident blocks take items
// from the counter until the list is exhausted, and the last block to
// leave resets the counter for the next launch.
template<class R, int DIM, int RECON, int FLUX, int KIND, int SHAPE = 0>
__global__ void __launch_bounds__((StageLayout<R, DIM, RECON, FLUX, SHAPE>::THREADS),
    (StageLayout<R, DIM, RECON, FLUX, SHAPE>::BLOCKS))
stage_kernel(const StageParams P) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ long long item;
    if (threadIdx.x == 0) {
        item = P.counter ? (long long)atomicAdd(&P.counter[0], 1ull) : (long long)blockIdx.x;
    }
    __syncthreads();
    // one call site, so the tile code is inlined once
    for (long long w = item; w < P.total_work;) {
        stage_item<R, DIM, RECON, FLUX, SHAPE, KIND>(P, w, smem);
        if (!P.counter) {
            break;
        }
        // the next item reuses the shared memory and `item`
        __syncthreads();
        if (threadIdx.x == 0) {
            item = (long long)atomicAdd(&P.counter[0], 1ull);
        }
        __syncthreads();
        w = item;
    }
    if (P.counter && threadIdx.x == 0) {
        __threadfence();
        const unsigned long long prev = atomicAdd(&P.counter[1], 1ull);
        if (prev == gridDim.x - 1) {
            P.counter[0] = 0;
            P.counter[1] = 0;
            __threadfence();
        }
    }
}

} // namespace als
