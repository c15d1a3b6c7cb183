// Stage-kernel instantiations for double precision, 1-D Euler.
#include "stage_dispatch.cuh"

namespace als {
cudaError_t launch_stage_f64_1d(int recon, int flux, int kind, int shape,
    const StageParams& P, int blocks_per_sm, cudaStream_t s) {
    return launch_stage_dim<double, 1>(recon, flux, kind, shape, P, blocks_per_sm, s);
}

void stage_tile_f64_1d(int shape, int* tile) {
    stage_tile_dim<1>(shape, tile);
}
} // namespace als
