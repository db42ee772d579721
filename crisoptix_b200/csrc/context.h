// context.h -- identity of the current CUDA context.
//
// Device addresses (a cudaMalloc'd table, the address of a __device__ array)
// belong to the context they were obtained in.  A cache of such addresses
// keyed by device ordinal goes stale when the primary context is destroyed
// (cudaDeviceReset) or when the caller runs in a context of its own, so the
// caches in this library key on the context's process-unique id instead
// (cuCtxGetId, reached through the runtime's driver entry points so the
// library does not link libcuda directly).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace crisb {

// Id of the context current on the calling thread (creating the device's
// primary context first when none is current, as any runtime call would).
// Returns cudaSuccess or the error that prevented the lookup.
cudaError_t current_context_id(unsigned long long* id);

}  // namespace crisb
