// 3-D stage kernel that marches along z (tile shape 1 of the 3-D stage).
//
// A block owns a 16 x 16 column of cells over a segment of ALS_ZMARCH_SEG
// cells along z.  It keeps a ring of three x-y planes (each with its x-y halo of
// G cells, every conserved variable) in shared memory and walks the segment
// plane by plane.  Per plane, the x and y directions reconstruct and
// evaluate their faces like the 2-D kernel; then the thread of each column
// reconstructs the next cell of its column along z and evaluates the z face
// between the two, keeping that face's flux and the next cell's right state
// (in shared memory, private to the column) for the next plane.  So every cell is reconstructed along z once and every
// z face is evaluated once, where the 8 x 8 x 4 tiles of shape 0 reconstruct
// 1.5 cells per cell along z and stage a box of 4.5 times the tile.
//
// The arithmetic and its order are those of stage_kernel (the same
// reconstruction, flux and update_cell; the net flux of a cell adds its x,
// then y, then z contribution), so the two shapes give the same bits.  Built
// for reconstructions whose stencil reaches one cell each way along z
// (WENO2, ENO2, MC, MM, WENOF2, none) and the two-point fluxes.
#pragma once

#include "stage_kernel.cuh"

namespace als {

template<class R, int RECON, int FLUX>
struct ZLayout {
    typedef TileShape<3, 1> Shape;
    static constexpr int NV = 5;
    static constexpr int G = stage_ghosts(RECON, FLUX);
    static constexpr int S = recon_ghosts(RECON) - 1;   // stencil half-width along z
    static constexpr int TX = Shape::X;
    static constexpr int TY = Shape::Y;
    static constexpr int SEG = Shape::Z;
    static constexpr int BX = TX + 2 * G;
    static constexpr int BY = TY + 2 * G;
    static constexpr int PLANE = BX * BY;
    static constexpr int RING = 3;
    static constexpr int COLS = TX * TY;
    static constexpr int THREADS = Shape::T;
    static constexpr int REC = (TX + 2) * TY > TX * (TY + 2) ? (TX + 2) * TY : TX * (TY + 2);
    static constexpr int FAC = (TX + 1) * TY > TX * (TY + 1) ? (TX + 1) * TY : TX * (TY + 1);
    // ring, x-y reconstructions, x-y face fluxes, and per column the right
    // state below the next z face and the flux through the face below
    static constexpr size_t SMEM = sizeof(R) *
        (size_t(NV) * PLANE * RING + size_t(2 * NV) * REC + size_t(NV) * FAC + size_t(2 * NV) * COLS);
    static constexpr int BY_SMEM = int((228 * 1024) / (SMEM + 1024));
    static constexpr int BLOCKS = BY_SMEM < 1 ? 1 : (BY_SMEM > Shape::B ? Shape::B : BY_SMEM);
    static_assert(S == 0 || S == 1, "the ring holds a stencil of one cell each way along z");
    static_assert(COLS <= THREADS && THREADS % 32 == 0, "one thread per column, whole warps");
};

// Values of one column at planes kc-1, kc, kc+1 of the ring (the fetcher of
// reconstruct_f along z; offsets beyond one cell are never asked for).
template<class R>
struct ColumnFetch {
    const R* m;
    const R* c;
    const R* p;
    int vstride;
    __device__ __forceinline__ R at(int v, int o) const {
        return (o < 0 ? m : (o > 0 ? p : c))[v * vstride];
    }
    __device__ __forceinline__ R dyn(int v, int o) const { return at(v, o); }
};

// The x (D = 0) or y (D = 1) direction of plane `pl`: reconstruct every cell
// its faces need, evaluate every face once, and add each column's net flux
// into that column's thread's acc (as stage_direction does for a tile).
template<class R, int RECON, int FLUX, int KIND, int D>
__device__ __forceinline__ void plane_direction(const GridDesc& gd, R gamma, const R* pl, R* rec,
    R* flx, R* acc, R& wmax, int x0, int y0) {
    typedef ZLayout<R, RECON, FLUX> Lay;
    constexpr int NV = Lay::NV;
    constexpr int G = Lay::G;
    constexpr int E0 = Lay::TX + (D == 0 ? 2 : 0);
    constexpr int E1 = Lay::TY + (D == 1 ? 2 : 0);
    constexpr int RC = E0 * E1;
    constexpr int F0 = Lay::TX + (D == 0 ? 1 : 0);
    constexpr int F1 = Lay::TY + (D == 1 ? 1 : 0);
    constexpr int FC = F0 * F1;
    constexpr int ST = D == 0 ? 1 : Lay::BX;
    const int tid = threadIdx.x;

    for (int i = tid; i < RC; i += Lay::THREADS) {
        const int ex = i % E0;
        const int ey = i / E0;
        const int bx = ex - (D == 0 ? 1 : 0) + G;
        const int by = ey - (D == 1 ? 1 : 0) + G;
        R l[NV], r[NV];
        reconstruct<R, NV, RECON>(pl + by * Lay::BX + bx, Lay::PLANE, ST, l, r, gamma);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            rec[v * RC + i] = l[v];
            rec[(NV + v) * RC + i] = r[v];
        }
    }
    __syncthreads();

    const int hiD = D == 0 ? gd.hi[0] : gd.hi[1];
    const int oD = D == 0 ? x0 : y0;
    for (int i = tid; i < FC; i += Lay::THREADS) {
        const int fx = i % F0;
        const int fy = i / F0;
        const int rl = fy * E0 + fx;
        const int rr = rl + (D == 0 ? 1 : E0);
        R ul[NV], ur[NV], F[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            ul[v] = rec[(NV + v) * RC + rl];
            ur[v] = rec[v * RC + rr];
        }
        const R w = face_flux<R, 3, FLUX, D>(ul, ur, gamma, F);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            flx[v * FC + i] = F[v];
        }
        if (KIND == KIND_FLUX0) {
            const int f = D == 0 ? fx : fy;
            bool valid = oD + f - 1 <= hiD - 1;
            if (D != 0) {
                valid = valid && (x0 + fx < gd.hi[0]);
            }
            if (D != 1) {
                valid = valid && (y0 + fy < gd.hi[1]);
            }
            if (valid && wmax < w) {
                wmax = w;
            }
        }
    }
    __syncthreads();

    if (tid < Lay::COLS) {
        const int cx = tid % Lay::TX;
        const int cy = tid / Lay::TX;
        const int fl = cy * F0 + cx;
        const int fr = fl + (D == 0 ? 1 : F0);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const R tr = -flx[v * FC + fr];
            const R tl = -flx[v * FC + fl];
            acc[v] = acc[v] + (tr + (-tl));
        }
    }
    // no barrier: the next writer of flx is the next face phase, behind the
    // barrier that ends the next reconstruction
}

// One work item: columns (tx, ty) over z segment tz of member `member`.
template<class R, int RECON, int FLUX, int KIND>
__device__ __forceinline__ void zmarch_tile(const StageParams& P, const LevelDesc& L, int tile,
    int member, unsigned char* smem) {
    typedef ZLayout<R, RECON, FLUX> Lay;
    constexpr int NV = Lay::NV;
    constexpr int G = Lay::G;
    constexpr bool LAST = KIND == KIND_RK3_2 || KIND == KIND_RK2_1;
    const int tid = threadIdx.x;
    const GridDesc& gd = L.grid;
    StepState* st = L.state ? L.state + (L.subdomains ? 0 : member) : nullptr;

    R* ring = reinterpret_cast<R*>(smem);
    R* rec = ring + Lay::RING * NV * Lay::PLANE;
    R* flx = rec + 2 * NV * Lay::REC;
    // column-private: Rk[v] = zs[v * COLS + col], Fm[v] = zs[(NV + v) * COLS + col]
    R* zs = flx + NV * Lay::FAC;

    const int tx = tile % gd.tiles[0];
    const int ty = (tile / gd.tiles[0]) % gd.tiles[1];
    const int tz = tile / (gd.tiles[0] * gd.tiles[1]);
    const int x0 = gd.lo[0] + tx * Lay::TX;
    const int y0 = gd.lo[1] + ty * Lay::TY;
    const int k0 = gd.lo[2] + tz * Lay::SEG;
    const int k1 = k0 + Lay::SEG < gd.hi[2] ? k0 + Lay::SEG : gd.hi[2];
    const long long base = (long long)member * L.member_stride;
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

    // plane k (interior index along z, -2 <= k <= n + 1) into its ring slot,
    // with the x-y halo; U1 = (dt/dx) L + U^n formed on load as in stage_tile
    const int sh = gd.ghosts - G;
    auto slot = [&](int k) { return ring + ((k - k0 + 3) % 3) * (NV * Lay::PLANE); };
    auto load_plane = [&](int k) {
        R* dst = slot(k);
        const int pz = k + gd.ghosts;
        const bool zin = pz >= 0 && pz < gd.N[2];
        for (int b = tid; b < Lay::PLANE; b += Lay::THREADS) {
            const int bx = b % Lay::BX;
            const int by = b / Lay::BX;
            const int px = x0 + bx + sh;
            const int py = y0 + by + sh;
            const bool inside = zin && px < gd.N[0] && py < gd.N[1];
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
                dst[v * Lay::PLANE + b] = val;
            }
        }
    };

    // this thread's column (threads past the columns help in the x-y phases)
    const bool column = tid < Lay::COLS;
    const int cx = tid % Lay::TX;
    const int cy = (tid / Lay::TX) % Lay::TY;
    const int coff = (cy + G) * Lay::BX + cx + G;
    const bool in_region = column && x0 + cx < gd.hi[0] && y0 + cy < gd.hi[1];
    // reconstruction of cell kc of this column along z
    auto recon_z = [&](int kc, R* l, R* r) {
        ColumnFetch<R> f{slot(kc - 1) + coff, slot(kc) + coff, slot(kc + 1) + coff, Lay::PLANE};
        reconstruct_f<R, NV, RECON>(f, l, r, gamma);
    };

    R wmax[3] = {R(0), R(0), R(0)};
    // the column's right state below the next z face, and the z flux below
    // the current cell, kept in shared memory between planes
    R* Rk = zs + (column ? tid : 0);
    R* Fm = zs + NV * Lay::COLS + (column ? tid : 0);
    {
        load_plane(k0 - 2);
        load_plane(k0 - 1);
        load_plane(k0);
        __syncthreads();
        if (column) {
            R l[NV], r[NV];
            recon_z(k0 - 1, l, r);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                Rk[v * Lay::COLS] = r[v];
            }
        }
        __syncthreads();
        load_plane(k0 + 1);
        __syncthreads();
        if (column) {
            R l[NV], r[NV], rb[NV], F[NV];
            recon_z(k0, l, r);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                rb[v] = Rk[v * Lay::COLS];
            }
            const R w = face_flux<R, 3, FLUX, 2>(rb, l, gamma, F);
            if (KIND == KIND_FLUX0 && in_region && wmax[2] < w) {
                wmax[2] = w;
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                Fm[v * Lay::COLS] = F[v];
                Rk[v * Lay::COLS] = r[v];
            }
        }
    }

    bool bad = false;
    long long bad_idx = 0;
    for (int k = k0; k < k1; ++k) {
        __syncthreads();
        load_plane(k + 2);
        __syncthreads();
        R acc[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            acc[v] = R(0);
        }
        const R* pl = slot(k);
        plane_direction<R, RECON, FLUX, KIND, 0>(gd, gamma, pl, rec, flx, acc, wmax[0], x0, y0);
        plane_direction<R, RECON, FLUX, KIND, 1>(gd, gamma, pl, rec, flx, acc, wmax[1], x0, y0);
        if (column) {
            // z: the face above the cell, between it and the next cell up
            R l[NV], r[NV], rb[NV], Fp[NV];
            recon_z(k + 1, l, r);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                rb[v] = Rk[v * Lay::COLS];
            }
            const R w = face_flux<R, 3, FLUX, 2>(rb, l, gamma, Fp);
            if (KIND == KIND_FLUX0 && in_region && wmax[2] < w) {
                wmax[2] = w;
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                const R tr = -Fp[v];
                const R tl = -Fm[v * Lay::COLS];
                acc[v] = acc[v] + (tr + (-tl));
                Fm[v * Lay::COLS] = Fp[v];
                Rk[v * Lay::COLS] = r[v];
            }
            if (in_region) {
                R ub[NV];
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    ub[v] = pl[v * Lay::PLANE + coff];
                }
                update_cell<R, 3, NV, KIND>(P, L, member, base, c, gamma, acc, ub, x0 + cx, y0 + cy,
                    k, bad, bad_idx);
            }
        }
    }

    if (KIND == KIND_FLUX0) {
        __shared__ double wsh[3][Lay::THREADS / 32];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const R w = warp_max(wmax[d]);
            if ((tid & 31) == 0) {
                wsh[d][tid >> 5] = double(w);
            }
        }
        __syncthreads();
        if (tid < 3) {
            double m = 0;
            for (int q = 0; q < Lay::THREADS / 32; ++q) {
                m = fmax(m, wsh[tid][q]);
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
            const unsigned int tiles = unsigned(L.tiles_per_member) *
                (L.subdomains ? unsigned(L.members) : 1u);
            if (prev == tiles - 1) {
                __threadfence();
                finish_step(st);
            }
        }
    }
}

template<class R, int RECON, int FLUX, int KIND>
__device__ __forceinline__ void zmarch_item(const StageParams& P, long long w, unsigned char* smem) {
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
    zmarch_tile<R, RECON, FLUX, KIND>(P, L, tile, member, smem);
}

// Launch modes as stage_kernel: one block per work item, or persistent
// blocks taking items from the counter.
template<class R, int RECON, int FLUX, int KIND>
__global__ void __launch_bounds__((ZLayout<R, RECON, FLUX>::THREADS),
    (ZLayout<R, RECON, FLUX>::BLOCKS))
zmarch_kernel(const StageParams P) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ long long item;
    if (threadIdx.x == 0) {
        item = P.counter ? (long long)atomicAdd(&P.counter[0], 1ull) : (long long)blockIdx.x;
    }
    __syncthreads();
    for (long long w = item; w < P.total_work;) {
        zmarch_item<R, RECON, FLUX, KIND>(P, w, smem);
        if (!P.counter) {
            break;
        }
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
