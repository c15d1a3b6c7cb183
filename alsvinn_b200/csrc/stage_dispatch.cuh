// Host-side launch of the stage kernel for a run-time (reconstruction, flux,
// kind) triple.  Each translation unit that includes this header
// instantiates the kernels of one (precision, dimension) pair, so the heavy
// instantiations compile in parallel.
#pragma once

#include <cuda_runtime.h>

#include "stage_kernel.cuh"
#include "stage_zmarch.cuh"

namespace als {

// One block per work item when the launch has no work counter; otherwise a
// persistent launch of as many blocks as can be resident at once (or
// `blocks_per_sm` per SM when > 0, capped by what fits), never more than
// there are work items.
// The kernel, block size and shared memory of one (shape, kind): the tiled
// stage_kernel, or for 3-D shape 1 the z-marching kernel.
template<class R, int DIM, int RECON, int FLUX, int KIND, int SHAPE>
struct StageLaunch {
    typedef StageLayout<R, DIM, RECON, FLUX, SHAPE> Lay;
    static constexpr int THREADS = Lay::THREADS;
    static constexpr size_t SMEM = Lay::SMEM;
    static decltype(&stage_kernel<R, DIM, RECON, FLUX, KIND, SHAPE>) kernel() {
        return stage_kernel<R, DIM, RECON, FLUX, KIND, SHAPE>;
    }
};
template<class R, int RECON, int FLUX, int KIND>
struct StageLaunch<R, 3, RECON, FLUX, KIND, 1> {
    typedef ZLayout<R, RECON, FLUX> Lay;
    static constexpr int THREADS = Lay::THREADS;
    static constexpr size_t SMEM = Lay::SMEM;
    static decltype(&zmarch_kernel<R, RECON, FLUX, KIND>) kernel() {
        return zmarch_kernel<R, RECON, FLUX, KIND>;
    }
};

template<class R, int DIM, int RECON, int FLUX, int KIND, int SHAPE>
cudaError_t launch_stage_one(const StageParams& P, int blocks_per_sm, cudaStream_t stream) {
    typedef StageLaunch<R, DIM, RECON, FLUX, KIND, SHAPE> Lay;
    auto kernel = Lay::kernel();
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

template<class R, int DIM, int RECON, int FLUX, int SHAPE>
cudaError_t launch_stage_kind(int kind, const StageParams& P, int b, cudaStream_t s) {
    switch (kind) {
    case KIND_FLUX0: return launch_stage_one<R, DIM, RECON, FLUX, KIND_FLUX0, SHAPE>(P, b, s);
    case KIND_RK2_1: return launch_stage_one<R, DIM, RECON, FLUX, KIND_RK2_1, SHAPE>(P, b, s);
    case KIND_RK3_1: return launch_stage_one<R, DIM, RECON, FLUX, KIND_RK3_1, SHAPE>(P, b, s);
    case KIND_RK3_2: return launch_stage_one<R, DIM, RECON, FLUX, KIND_RK3_2, SHAPE>(P, b, s);
    default: return cudaErrorInvalidValue;
    }
}

// The tile shape is a run-time choice among the shapes built for the
// combination (shape_built).
template<class R, int DIM, int RECON, int FLUX>
cudaError_t launch_stage_shape(int shape, int kind, const StageParams& P, int b, cudaStream_t s) {
    if (shape == 0) {
        return launch_stage_kind<R, DIM, RECON, FLUX, 0>(kind, P, b, s);
    }
    if constexpr (shape_built(DIM, RECON, FLUX, 1)) {
        if (shape == 1) {
            return launch_stage_kind<R, DIM, RECON, FLUX, 1>(kind, P, b, s);
        }
    }
    return cudaErrorInvalidValue;
}

template<class R, int DIM, int RECON>
cudaError_t launch_stage_flux(int flux, int kind, int shape, const StageParams& P, int b,
    cudaStream_t s) {
    switch (flux) {
    case FLUX_HLL: return launch_stage_shape<R, DIM, RECON, FLUX_HLL>(shape, kind, P, b, s);
    case FLUX_HLL3: return launch_stage_shape<R, DIM, RECON, FLUX_HLL3>(shape, kind, P, b, s);
    case FLUX_CENTRAL: return launch_stage_shape<R, DIM, RECON, FLUX_CENTRAL>(shape, kind, P, b, s);
    default: break;
    }
    // the TeCNO fluxes are built for reconstruction "none" only
    if constexpr (RECON == RECON_NONE) {
        switch (flux) {
        case FLUX_TECNO1: return launch_stage_shape<R, DIM, RECON, FLUX_TECNO1>(shape, kind, P, b, s);
        case FLUX_TECNO4: return launch_stage_shape<R, DIM, RECON, FLUX_TECNO4>(shape, kind, P, b, s);
        case FLUX_TECNO6: return launch_stage_shape<R, DIM, RECON, FLUX_TECNO6>(shape, kind, P, b, s);
        default: break;
        }
    }
    return cudaErrorInvalidValue;
}

template<class R, int DIM>
cudaError_t launch_stage_dim(int recon, int flux, int kind, int shape, const StageParams& P, int b,
    cudaStream_t s) {
    switch (recon) {
    case RECON_NONE: return launch_stage_flux<R, DIM, RECON_NONE>(flux, kind, shape, P, b, s);
    case RECON_WENO2: return launch_stage_flux<R, DIM, RECON_WENO2>(flux, kind, shape, P, b, s);
    case RECON_ENO2: return launch_stage_flux<R, DIM, RECON_ENO2>(flux, kind, shape, P, b, s);
    case RECON_ENO3: return launch_stage_flux<R, DIM, RECON_ENO3>(flux, kind, shape, P, b, s);
    case RECON_ENO4: return launch_stage_flux<R, DIM, RECON_ENO4>(flux, kind, shape, P, b, s);
    case RECON_MC: return launch_stage_flux<R, DIM, RECON_MC>(flux, kind, shape, P, b, s);
    case RECON_MM: return launch_stage_flux<R, DIM, RECON_MM>(flux, kind, shape, P, b, s);
    case RECON_WENOF2: return launch_stage_flux<R, DIM, RECON_WENOF2>(flux, kind, shape, P, b, s);
    case RECON_WENO3: return launch_stage_flux<R, DIM, RECON_WENO3>(flux, kind, shape, P, b, s);
    default: return cudaErrorInvalidValue;
    }
}

// Tile extents of `shape` (0 0 0 when that shape is not built for the dimension).
template<int DIM>
void stage_tile_dim(int shape, int* tile) {
    tile[0] = tile[1] = tile[2] = 0;
    if (shape == 0) {
        tile[0] = TileShape<DIM, 0>::X;
        tile[1] = TileShape<DIM, 0>::Y;
        tile[2] = TileShape<DIM, 0>::Z;
    }
    if constexpr (DIM >= 2) {
        if (shape == 1) {
            tile[0] = TileShape<DIM, 1>::X;
            tile[1] = TileShape<DIM, 1>::Y;
            tile[2] = TileShape<DIM, 1>::Z;
        }
    }
}

// Entry points defined by the per-(precision, dimension) translation units.
// `shape` selects the tile shape (shape_built), `blocks_per_sm` (0 = as
// many as fit) sizes the persistent grid.  stage_tile_* report the tile of
// a shape as the kernels of that unit were built, so the host always covers
// the grid with the tiles the kernels expect.
cudaError_t launch_stage_f64_1d(int recon, int flux, int kind, int shape, const StageParams& P, int blocks_per_sm, cudaStream_t s);
cudaError_t launch_stage_f64_2d(int recon, int flux, int kind, int shape, const StageParams& P, int blocks_per_sm, cudaStream_t s);
cudaError_t launch_stage_f64_3d(int recon, int flux, int kind, int shape, const StageParams& P, int blocks_per_sm, cudaStream_t s);
cudaError_t launch_stage_f32_1d(int recon, int flux, int kind, int shape, const StageParams& P, int blocks_per_sm, cudaStream_t s);
cudaError_t launch_stage_f32_2d(int recon, int flux, int kind, int shape, const StageParams& P, int blocks_per_sm, cudaStream_t s);
cudaError_t launch_stage_f32_3d(int recon, int flux, int kind, int shape, const StageParams& P, int blocks_per_sm, cudaStream_t s);
void stage_tile_f64_1d(int shape, int* tile);
void stage_tile_f64_2d(int shape, int* tile);
void stage_tile_f64_3d(int shape, int* tile);
void stage_tile_f32_1d(int shape, int* tile);
void stage_tile_f32_2d(int shape, int* tile);
void stage_tile_f32_3d(int shape, int* tile);

} // namespace als
