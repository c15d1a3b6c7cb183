// Stage-kernel instantiations for float precision, 2-D Euler.
#include "stage_dispatch.cuh"

namespace als {
cudaError_t launch_stage_f32_2d(int recon, int flux, int kind, int shape,
    const StageParams& P, int blocks_per_sm, cudaStream_t s) {
    return launch_stage_dim<float, 2>(recon, flux, kind, shape, P, blocks_per_sm, s);
}

void stage_tile_f32_2d(int shape, int* tile) {
    stage_tile_dim<2>(shape, tile);
}
} // namespace als
