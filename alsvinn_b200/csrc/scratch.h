// Stream-ordered scratch memory of the library's entry points.
//
// Scratch comes from a memory pool the library owns on each device, whose
// freed memory stays reserved for the next call (release threshold without
// limit).  The device's default pool hands its memory back at every
// synchronisation, so an entry point called once per time step beside a
// host round trip (a functional, a conservation sum) would map its scratch
// afresh on every call.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace als {

// `bytes` of device memory on the current device, ordered on `stream`.
cudaError_t scratch_alloc(void** ptr, size_t bytes, cudaStream_t stream);

// Returns memory from scratch_alloc to the library's pool, ordered on `stream`.
cudaError_t scratch_free(void* ptr, cudaStream_t stream);

} // namespace als
