// Host-side launch of the stage kernel for a run-time (reconstruction, flux,
// kind) triple.  Each translation unit that includes this header
// instantiates the kernels of one (precision, dimension) pair, so the heavy
// instantiations compile in parallel.
#pragma once

#include <cuda_runtime.h>

#include "stage_kernel.cuh"

namespace als {

template<class R, int DIM, int RECON, int FLUX, int KIND>
cudaError_t launch_stage_one(const StageParams& P, int members, cudaStream_t stream) {
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
    kernel<<<grid, Lay::THREADS, Lay::SMEM, stream>>>(P);
    return cudaGetLastError();
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

template<int DIM>
void stage_tile_dim(int* tile) {
    tile[0] = TileShape<DIM>::X;
    tile[1] = TileShape<DIM>::Y;
    tile[2] = TileShape<DIM>::Z;
}

// Entry points defined by the per-(precision, dimension) translation units.
// stage_tile_* report the tile the kernels of that unit were built with, so
// the host always covers the grid with the tiles the kernels expect.
void stage_tile_f64_1d(int* tile);
void stage_tile_f64_2d(int* tile);
void stage_tile_f64_3d(int* tile);
void stage_tile_f32_1d(int* tile);
void stage_tile_f32_2d(int* tile);
void stage_tile_f32_3d(int* tile);
cudaError_t launch_stage_f64_1d(int recon, int flux, int kind, const StageParams& P, int members, cudaStream_t s);
cudaError_t launch_stage_f64_2d(int recon, int flux, int kind, const StageParams& P, int members, cudaStream_t s);
cudaError_t launch_stage_f64_3d(int recon, int flux, int kind, const StageParams& P, int members, cudaStream_t s);
cudaError_t launch_stage_f32_1d(int recon, int flux, int kind, const StageParams& P, int members, cudaStream_t s);
cudaError_t launch_stage_f32_2d(int recon, int flux, int kind, const StageParams& P, int members, cudaStream_t s);
cudaError_t launch_stage_f32_3d(int recon, int flux, int kind, const StageParams& P, int members, cudaStream_t s);

} // namespace als
