// Register-marching stage kernel for 1-D and 2-D grids.
//
// Each warp owns a strip of 32 consecutive columns (32 - 2G of them are
// outputs, the others halo) and marches up a segment of TY rows.  Along x
// the stencil neighbours come from warp shuffles; along y every lane keeps a
// sliding window of rows in registers, so every cell is reconstructed and
// every face flux evaluated once per lane with no shared memory and no
// block-wide barrier.  The next row is loaded while the current one is
// computed.  Arithmetic and operation order are those of stage_kernel.cuh
// (the reference's CPU path); only the data movement differs.
#pragma once

#include "stage_kernel.cuh"

namespace als {

constexpr int kMarchThreads = 128;
constexpr unsigned kFullMask = 0xffffffffu;
// minimum resident blocks per SM requested from the register allocator
#ifndef ALS_MARCH_MIN_BLOCKS
#define ALS_MARCH_MIN_BLOCKS 1
#endif

// Stencil values of this lane's row from the neighbouring lanes.
template<class R, int NV>
struct LaneFetch {
    const R* u;
    int lane;
    __device__ __forceinline__ R at(int v, int o) const {
        return __shfl_sync(kFullMask, u[v], lane + o);
    }
    __device__ __forceinline__ R dyn(int v, int o) const {
        return __shfl_sync(kFullMask, u[v], lane + o);
    }
};

// Stencil values along y from the register window (row C is the centre).
template<class R, int NV, int WS, int C>
struct WindowFetch {
    const R (*win)[NV];
    __device__ __forceinline__ R at(int v, int o) const { return win[C + o][v]; }
    __device__ __forceinline__ R dyn(int v, int o) const {
        R r = win[0][v];
#pragma unroll
        for (int k = 1; k < WS; ++k) {
            r = (o == k - C) ? win[k][v] : r;
        }
        return r;
    }
};

template<class R, int DIM, int RECON>
struct MarchShape {
    static constexpr int NV = DIM + 2;
    static constexpr int G = recon_ghosts(RECON);
    static constexpr int OUTX = 32 - 2 * G;        // output columns per warp
    static constexpr int A = G >= 2 ? G - 2 : 0;   // window rows below the output row
    static constexpr int WS = A + G + 1;           // window rows [c-A, c+G]
};

template<class R, int DIM, int RECON, int FLUX, int KIND>
__global__ void __launch_bounds__(kMarchThreads, ALS_MARCH_MIN_BLOCKS)
march_kernel(const StageParams P, const int TY) {
    typedef MarchShape<R, DIM, RECON> S;
    constexpr int NV = S::NV;
    constexpr int G = S::G;
    constexpr int RR = G - 1;
    constexpr int A = S::A;
    constexpr int WS = S::WS;
    constexpr bool LAST = KIND == KIND_RK3_2 || KIND == KIND_RK2_1;
    constexpr bool ONTHEFLY = KIND == KIND_RK2_1 || KIND == KIND_RK3_1;

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int member = P.member0 + blockIdx.y;
    StepState* st = P.state ? P.state + member : nullptr;
    if (st && ((volatile StepState*)st)->done) {
        return;
    }
    const GridDesc& gd = P.grid;
    const long long plane = gd.plane;
    const long long base = (long long)member * P.sample_stride;
    const R* in = static_cast<const R*>(P.in) + base;
    const R* un = static_cast<const R*>(P.un) + base;
    R* out = static_cast<R*>(P.out) + base;
    const R gamma = R(P.gamma);

    R c = R(0);
    if (KIND == KIND_RK2_1 || KIND == KIND_RK3_1) {
        if (st) {
            const double dt = step_dt(st);
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                st->dt = dt;
            }
            c = R(dt / st->dx[0]);
        } else {
            c = R(P.c_fixed);
        }
    } else if (KIND == KIND_RK3_2) {
        c = st ? R(st->dt / st->dx[0]) : R(P.c_fixed);
    }

    const int strips = gd.tiles[0];
    const int segs = gd.tiles[1];
    const int item = blockIdx.x * (kMarchThreads / 32) + warp;
    const bool active = item < strips * segs;
    R wmax[2] = {R(0), R(0)};
    bool bad = false;
    long long bad_idx = 0;

    if (active) {
        const int sx = item % strips;
        const int sy = item / strips;
        const int x0 = gd.lo[0] + sx * S::OUTX;
        const int y0 = DIM == 2 ? gd.lo[1] + sy * TY : 0;
        const int y1 = DIM == 2 ? min(y0 + TY, gd.hi[1]) : 1;
        const int x = x0 - G + lane;          // interior column of this lane
        const int px = x0 + lane;             // padded column
        const bool colok = px < gd.N[0];
        const bool out_lane = lane >= G && lane < 32 - G && x < gd.hi[0];
        const bool face_lane = lane >= G - 1 && lane < 32 - G && x >= gd.lo[0] - 1 && x <= gd.hi[0] - 1;

        auto load_row = [&](int r, R* u) {
            const int py = DIM == 2 ? r + G : 0;
            const bool ok = colok && py >= 0 && py < gd.N[1];
            const long long idx = (long long)py * gd.N[0] + px;
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                R val = R(0);
                if (ok) {
                    if (ONTHEFLY) {
                        val = in[v * plane + idx] * c;
                        val = val + un[v * plane + idx];
                    } else {
                        val = in[v * plane + idx];
                    }
                }
                u[v] = val;
            }
        };

        // x-direction net flux of the row held in u (every lane takes part)
        auto net_x = [&](const R* u, R* net, R& wx) {
            LaneFetch<R, NV> f{u, lane};
            R lx[NV], rx[NV];
            reconstruct_f<R, NV, RECON>(f, lx, rx);
            R lxn[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                lxn[v] = __shfl_down_sync(kFullMask, lx[v], 1);
            }
            R F[NV];
            wx = face_flux<R, DIM, FLUX, 0>(rx, lxn, gamma, F);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                const R Fm = __shfl_up_sync(kFullMask, F[v], 1);
                // out += temp[x+1] + (-temp[x]), temp = -F (NumericalFluxCPU.cpp:92,113)
                const R tr = -F[v];
                const R tl = -Fm;
                net[v] = R(0) + (tr + (-tl));
            }
        };

        // epilogue of one output cell: stage combination, store, boundary images
        auto emit = [&](int yr, const R* acc, const R* ucur) {
            const int py = DIM == 2 ? yr + G : 0;
            const long long idx = (long long)py * gd.N[0] + px;
            R val[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                R xv = acc[v];
                if (KIND == KIND_RK2_1) {
                    xv = xv * c;
                    xv = xv + ucur[v];
                    xv = xv + un[v * plane + idx];
                    xv = xv * R(0.5);
                } else if (KIND == KIND_RK3_1) {
                    xv = xv * c;
                    xv = xv + ucur[v];
                    xv = xv * R(1. / 3.);
                    xv = xv + un[v * plane + idx];
                    xv = xv * R(3. / 4.);
                } else if (KIND == KIND_RK3_2) {
                    xv = xv * c;
                    xv = xv + ucur[v];
                    xv = xv * R(2);
                    xv = xv + un[v * plane + idx];
                    xv = xv * R(1. / 3.);
                }
                val[v] = xv;
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                out[v * plane + idx] = val[v];
            }
            if (P.write_ghosts) {
                int ix[3], iy[3] = {0, 0, 0};
                const int nxi = boundary_images(x, gd.n[0], G, P.bc, ix);
                const int nyi = DIM == 2 ? boundary_images(yr, gd.n[1], G, P.bc, iy) : 1;
                if (nxi * nyi > 1) {
                    for (int b = 0; b < nyi; ++b) {
                        for (int e = 0; e < nxi; ++e) {
                            if (b == 0 && e == 0) {
                                continue;
                            }
                            const long long j = (long long)iy[b] * gd.N[0] + ix[e];
#pragma unroll
                            for (int v = 0; v < NV; ++v) {
                                out[v * plane + j] = val[v];
                            }
                        }
                    }
                }
            }
            if (LAST && st && !bad && !obeys_constraints<R, NV>(val, gamma)) {
                bad = true;
                bad_idx = idx;
            }
        };

        if (DIM == 1) {
            R u[NV];
            load_row(0, u);
            R acc[NV];
            R wx;
            net_x(u, acc, wx);
            if (face_lane && wmax[0] < wx) {
                wmax[0] = wx;
            }
            if (out_lane) {
                emit(0, acc, u);
            }
        } else {
            // right y-reconstruction of row y0-1 (rows y0-1-RR .. y0-1+RR)
            R ryp[NV];
            {
                R tmp[2 * RR + 1][NV];
#pragma unroll
                for (int i = 0; i < 2 * RR + 1; ++i) {
                    load_row(y0 - 1 - RR + i, tmp[i]);
                }
                WindowFetch<R, NV, 2 * RR + 1, RR> f{tmp};
                R l[NV];
                reconstruct_f<R, NV, RECON>(f, l, ryp);
            }
            R win[WS][NV];
#pragma unroll
            for (int i = 0; i < WS; ++i) {
                load_row(y0 - 1 - A + i, win[i]);
            }
            R Gp[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                Gp[v] = R(0);
            }
            const int kend = y1 - y0;
            for (int k = 0; k <= kend; ++k) {
                const int cy = y0 - 1 + k;   // face between rows cy and cy+1
                R nxt[NV];
                if (k < kend) {
                    load_row(cy + G + 1, nxt);
                }
                R ly[NV], ry[NV];
                {
                    WindowFetch<R, NV, WS, A + 1> f{win};
                    reconstruct_f<R, NV, RECON>(f, ly, ry);
                }
                R Gc[NV];
                const R wy = face_flux<R, DIM, FLUX, (DIM == 2 ? 1 : 0)>(ryp, ly, gamma, Gc);
                if (out_lane && cy <= gd.hi[1] - 1 && wmax[1] < wy) {
                    wmax[1] = wy;
                }
                if (k >= 1) {
                    // output row cy: x-direction first, then y (NumericalFluxCPU.cpp:196-209)
                    R acc[NV];
                    R wx;
                    net_x(win[A], acc, wx);
                    if (face_lane && wmax[0] < wx) {
                        wmax[0] = wx;
                    }
#pragma unroll
                    for (int v = 0; v < NV; ++v) {
                        const R tr = -Gc[v];
                        const R tl = -Gp[v];
                        acc[v] = acc[v] + (tr + (-tl));
                    }
                    if (out_lane) {
                        emit(cy, acc, win[A]);
                    }
                }
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    ryp[v] = ry[v];
                    Gp[v] = Gc[v];
                }
                if (k < kend) {
#pragma unroll
                    for (int i = 0; i + 1 < WS; ++i) {
#pragma unroll
                        for (int v = 0; v < NV; ++v) {
                            win[i][v] = win[i + 1][v];
                        }
                    }
#pragma unroll
                    for (int v = 0; v < NV; ++v) {
                        win[WS - 1][v] = nxt[v];
                    }
                }
            }
        }
    }

    if (KIND == KIND_FLUX0) {
        __shared__ double wsh[2][kMarchThreads / 32];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const R w = warp_max(wmax[d]);
            if (lane == 0) {
                wsh[d][warp] = double(w);
            }
        }
        __syncthreads();
        if (threadIdx.x < DIM) {
            double m = 0;
            for (int k = 0; k < kMarchThreads / 32; ++k) {
                m = fmax(m, wsh[threadIdx.x][k]);
            }
            unsigned long long* dst = st ? &st->ws[threadIdx.x] : (P.ws_out + 3 * member + threadIdx.x);
            atomicMax(dst, (unsigned long long)__double_as_longlong(m));
        }
    }

    if (LAST && st) {
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
        }
    }
}

} // namespace als
