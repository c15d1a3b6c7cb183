// Host-side launch of the stage kernel for a run-time (reconstruction, flux,
// kind) triple.  Each translation unit that includes this header
// instantiates the kernels of one (precision, dimension) pair, so the heavy
// instantiations compile in parallel.
#pragma once

#include <cuda_runtime.h>

#include "march_kernel.cuh"
#include "stage_kernel.cuh"

namespace als {

// Rows per warp of the marching kernel: enough warps to fill every SM about
// sixteen warps deep, segments of 4..128 rows.  `rows_hint` > 0 overrides.
inline int march_rows(int rows, int strips, int members, int rows_hint) {
    if (rows_hint > 0) {
        return rows_hint;
    }
    const long long target = 148LL * 16;
    const long long per_seg = (long long)strips * members;
    long long segs = (target + per_seg - 1) / per_seg;
    if (segs < 1) {
        segs = 1;
    }
    long long ty = (rows + segs - 1) / segs;
    ty = ty < 4 ? 4 : (ty > 128 ? 128 : ty);
    return int(ty);
}

template<class R, int DIM, int RECON, int FLUX, int KIND>
cudaError_t launch_march_one(const StageParams& P0, int members, cudaStream_t stream) {
    typedef MarchShape<R, DIM, RECON> S;
    StageParams P = P0;
    const int cols = P.grid.hi[0] - P.grid.lo[0];
    const int rows = DIM == 2 ? P.grid.hi[1] - P.grid.lo[1] : 1;
    const int strips = (cols + S::OUTX - 1) / S::OUTX;
    const int ty = DIM == 2 ? march_rows(rows, strips, members, P.rows_per_warp) : 1;
    const int segs = (rows + ty - 1) / ty;
    P.grid.tiles[0] = strips;
    P.grid.tiles[1] = segs;
    P.grid.tiles[2] = 1;
    const int warps = strips * segs;
    const int wpb = kMarchThreads / 32;
    dim3 grid(unsigned((warps + wpb - 1) / wpb), unsigned(members));
    march_kernel<R, DIM, RECON, FLUX, KIND><<<grid, kMarchThreads, 0, stream>>>(P, ty);
    return cudaGetLastError();
}

template<class R, int DIM, int RECON, int FLUX, int KIND>
cudaError_t launch_stage_one(const StageParams& P, int members, cudaStream_t stream) {
    if constexpr (DIM < 3) {
        // 1-D and 2-D: the register-marching kernel
        return launch_march_one<R, DIM, RECON, FLUX, KIND>(P, members, stream);
    } else {
        // 3-D: shared-memory tiles
        typedef StageLayout<R, DIM, RECON> Lay;
        auto kernel = stage_kernel<R, DIM, RECON, FLUX, KIND>;
        // raising the dynamic shared-memory limit is idempotent and cheap; it is
        // done on every launch so that every device the process uses is covered
        cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
            int(Lay::SMEM));
        if (err != cudaSuccess) {
            return err;
        }
        const unsigned int tiles = unsigned(P.grid.tiles[0]) * P.grid.tiles[1] * P.grid.tiles[2];
        dim3 grid(tiles, unsigned(members));
        kernel<<<grid, kStageThreads, Lay::SMEM, stream>>>(P);
        return cudaGetLastError();
    }
}

template<class R, int DIM, int RECON, int FLUX>
cudaError_t launch_stage_kind(int kind, const StageParams& P, int members, cudaStream_t s) {
    switch (kind) {
    case KIND_FLUX0: return launch_stage_one<R, DIM, RECON, FLUX, KIND_FLUX0>(P, members, s);
    case KIND_RK2_1: return launch_stage_one<R, DIM, RECON, FLUX, KIND_RK2_1>(P, members, s);
    case KIND_RK3_1: return launch_stage_one<R, DIM, RECON, FLUX, KIND_RK3_1>(P, members, s);
    case KIND_RK3_2: return launch_stage_one<R, DIM, RECON, FLUX, KIND_RK3_2>(P, members, s);
    default: return cudaErrorInvalidValue;
    }
}

template<class R, int DIM, int RECON>
cudaError_t launch_stage_flux(int flux, int kind, const StageParams& P, int members, cudaStream_t s) {
    switch (flux) {
    case FLUX_HLL: return launch_stage_kind<R, DIM, RECON, FLUX_HLL>(kind, P, members, s);
    case FLUX_HLL3: return launch_stage_kind<R, DIM, RECON, FLUX_HLL3>(kind, P, members, s);
    case FLUX_CENTRAL: return launch_stage_kind<R, DIM, RECON, FLUX_CENTRAL>(kind, P, members, s);
    default: return cudaErrorInvalidValue;
    }
}

template<class R, int DIM>
cudaError_t launch_stage_dim(int recon, int flux, int kind, const StageParams& P, int members,
    cudaStream_t s) {
    switch (recon) {
    case RECON_NONE: return launch_stage_flux<R, DIM, RECON_NONE>(flux, kind, P, members, s);
    case RECON_WENO2: return launch_stage_flux<R, DIM, RECON_WENO2>(flux, kind, P, members, s);
    case RECON_ENO2: return launch_stage_flux<R, DIM, RECON_ENO2>(flux, kind, P, members, s);
    case RECON_ENO3: return launch_stage_flux<R, DIM, RECON_ENO3>(flux, kind, P, members, s);
    case RECON_ENO4: return launch_stage_flux<R, DIM, RECON_ENO4>(flux, kind, P, members, s);
    default: return cudaErrorInvalidValue;
    }
}

template<class R, int DIM>
size_t stage_smem_dim(int recon) {
    switch (recon) {
    case RECON_NONE: return StageLayout<R, DIM, RECON_NONE>::SMEM;
    case RECON_WENO2: return StageLayout<R, DIM, RECON_WENO2>::SMEM;
    case RECON_ENO2: return StageLayout<R, DIM, RECON_ENO2>::SMEM;
    case RECON_ENO3: return StageLayout<R, DIM, RECON_ENO3>::SMEM;
    default: return StageLayout<R, DIM, RECON_ENO4>::SMEM;
    }
}

// Entry points defined by the per-(precision, dimension) translation units.
cudaError_t launch_stage_f64_1d(int recon, int flux, int kind, const StageParams& P, int members, cudaStream_t s);
cudaError_t launch_stage_f64_2d(int recon, int flux, int kind, const StageParams& P, int members, cudaStream_t s);
cudaError_t launch_stage_f64_3d(int recon, int flux, int kind, const StageParams& P, int members, cudaStream_t s);
cudaError_t launch_stage_f32_1d(int recon, int flux, int kind, const StageParams& P, int members, cudaStream_t s);
cudaError_t launch_stage_f32_2d(int recon, int flux, int kind, const StageParams& P, int members, cudaStream_t s);
cudaError_t launch_stage_f32_3d(int recon, int flux, int kind, const StageParams& P, int members, cudaStream_t s);

} // namespace als
