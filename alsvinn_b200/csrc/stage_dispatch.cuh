// Host-side launch of the stage kernel for a run-time (reconstruction, flux,
// kind) triple.  Each translation unit that includes this header
// instantiates the kernels of one (precision, dimension) pair, so the heavy
// instantiations compile in parallel.
#pragma once

#include <cuda_runtime.h>

#include "stage_kernel.cuh"

namespace als {

// One block per work item when the launch has no work counter; otherwise a
// persistent launch of as many blocks as can be resident at once (or
// `blocks_per_sm` per SM when > 0, capped by what fits), never more than
// there are work items.
template<class R, int DIM, int RECON, int FLUX, int KIND>
cudaError_t launch_stage_one(const StageParams& P, int blocks_per_sm, cudaStream_t stream) {
    typedef StageLayout<R, DIM, RECON, FLUX> Lay;
    auto kernel = stage_kernel<R, DIM, RECON, FLUX, KIND>;
    // raising the dynamic shared-memory limit is idempotent and cheap; it is
    // done on every launch so that every device the process uses is covered
    cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
        int(Lay::SMEM));
    if (err != cudaSuccess) {
        return err;
    }
    if (P.total_work <= 0) {
        return cudaSuccess;
    }
    if (!P.counter) {
        kernel<<<unsigned(P.total_work), Lay::THREADS, Lay::SMEM, stream>>>(P);
        return cudaGetLastError();
    }
    int device = 0, sms = 0, resident = 0;
    err = cudaGetDevice(&device);
    if (err == cudaSuccess) {
        err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    }
    if (err == cudaSuccess) {
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kernel, Lay::THREADS, Lay::SMEM);
    }
    if (err != cudaSuccess) {
        return err;
    }
    if (resident < 1) {
        resident = 1;
    }
    if (blocks_per_sm > 0 && blocks_per_sm < resident) {
        resident = blocks_per_sm;
    }
    long long blocks = (long long)resident * sms;
    if (blocks > P.total_work) {
        blocks = P.total_work;
    }
    kernel<<<unsigned(blocks), Lay::THREADS, Lay::SMEM, stream>>>(P);
    return cudaGetLastError();
}

template<class R, int DIM, int RECON, int FLUX>
cudaError_t launch_stage_kind(int kind, const StageParams& P, int b, cudaStream_t s) {
    switch (kind) {
    case KIND_FLUX0: return launch_stage_one<R, DIM, RECON, FLUX, KIND_FLUX0>(P, b, s);
    case KIND_RK2_1: return launch_stage_one<R, DIM, RECON, FLUX, KIND_RK2_1>(P, b, s);
    case KIND_RK3_1: return launch_stage_one<R, DIM, RECON, FLUX, KIND_RK3_1>(P, b, s);
    case KIND_RK3_2: return launch_stage_one<R, DIM, RECON, FLUX, KIND_RK3_2>(P, b, s);
    default: return cudaErrorInvalidValue;
    }
}

template<class R, int DIM, int RECON>
cudaError_t launch_stage_flux(int flux, int kind, const StageParams& P, int b, cudaStream_t s) {
    switch (flux) {
    case FLUX_HLL: return launch_stage_kind<R, DIM, RECON, FLUX_HLL>(kind, P, b, s);
    case FLUX_HLL3: return launch_stage_kind<R, DIM, RECON, FLUX_HLL3>(kind, P, b, s);
    case FLUX_CENTRAL: return launch_stage_kind<R, DIM, RECON, FLUX_CENTRAL>(kind, P, b, s);
    default: break;
    }
    // the TeCNO fluxes are built for reconstruction "none" only
    if constexpr (RECON == RECON_NONE) {
        switch (flux) {
        case FLUX_TECNO1: return launch_stage_kind<R, DIM, RECON, FLUX_TECNO1>(kind, P, b, s);
        case FLUX_TECNO4: return launch_stage_kind<R, DIM, RECON, FLUX_TECNO4>(kind, P, b, s);
        case FLUX_TECNO6: return launch_stage_kind<R, DIM, RECON, FLUX_TECNO6>(kind, P, b, s);
        default: break;
        }
    }
    return cudaErrorInvalidValue;
}

template<class R, int DIM>
cudaError_t launch_stage_dim(int recon, int flux, int kind, const StageParams& P, int b,
    cudaStream_t s) {
    switch (recon) {
    case RECON_NONE: return launch_stage_flux<R, DIM, RECON_NONE>(flux, kind, P, b, s);
    case RECON_WENO2: return launch_stage_flux<R, DIM, RECON_WENO2>(flux, kind, P, b, s);
    case RECON_ENO2: return launch_stage_flux<R, DIM, RECON_ENO2>(flux, kind, P, b, s);
    case RECON_ENO3: return launch_stage_flux<R, DIM, RECON_ENO3>(flux, kind, P, b, s);
    case RECON_ENO4: return launch_stage_flux<R, DIM, RECON_ENO4>(flux, kind, P, b, s);
    case RECON_MC: return launch_stage_flux<R, DIM, RECON_MC>(flux, kind, P, b, s);
    case RECON_MM: return launch_stage_flux<R, DIM, RECON_MM>(flux, kind, P, b, s);
    case RECON_WENOF2: return launch_stage_flux<R, DIM, RECON_WENOF2>(flux, kind, P, b, s);
    case RECON_WENO3: return launch_stage_flux<R, DIM, RECON_WENO3>(flux, kind, P, b, s);
    default: return cudaErrorInvalidValue;
    }
}

template<int DIM>
void stage_tile_dim(int* tile) {
    tile[0] = TileShape<DIM>::X;
    tile[1] = TileShape<DIM>::Y;
    tile[2] = TileShape<DIM>::Z;
}

// Entry points defined by the per-(precision, dimension) translation units.
// `blocks_per_sm` (0 = as many as fit) sizes the persistent grid.
// stage_tile_* report the tile the kernels of that unit were built with, so
// the host always covers the grid with the tiles the kernels expect.
cudaError_t launch_stage_f64_1d(int recon, int flux, int kind, const StageParams& P, int blocks_per_sm, cudaStream_t s);
cudaError_t launch_stage_f64_2d(int recon, int flux, int kind, const StageParams& P, int blocks_per_sm, cudaStream_t s);
cudaError_t launch_stage_f64_3d(int recon, int flux, int kind, const StageParams& P, int blocks_per_sm, cudaStream_t s);
cudaError_t launch_stage_f32_1d(int recon, int flux, int kind, const StageParams& P, int blocks_per_sm, cudaStream_t s);
cudaError_t launch_stage_f32_2d(int recon, int flux, int kind, const StageParams& P, int blocks_per_sm, cudaStream_t s);
cudaError_t launch_stage_f32_3d(int recon, int flux, int kind, const StageParams& P, int blocks_per_sm, cudaStream_t s);
void stage_tile_f64_1d(int* tile);
void stage_tile_f64_2d(int* tile);
void stage_tile_f64_3d(int* tile);
void stage_tile_f32_1d(int* tile);
void stage_tile_f32_2d(int* tile);
void stage_tile_f32_3d(int* tile);

} // namespace als
