// Stage-kernel instantiations for float precision, 3-D Euler.
#include "stage_dispatch.cuh"

namespace als {
cudaError_t launch_stage_f32_3d(int recon, int flux, int kind, const StageParams& P,
    int members, cudaStream_t s) {
    return launch_stage_dim<float, 3>(recon, flux, kind, P, members, s);
}
} // namespace als
