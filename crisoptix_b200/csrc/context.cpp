// context.cpp -- current_context_id (context.h).
#include "context.h"

#include <cuda.h>

#include <mutex>

namespace crisb {
namespace {

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

struct DriverFns {
    CtxGetCurrentFn get_current = nullptr;
    CtxGetIdFn get_id = nullptr;
    cudaError_t status = cudaErrorUnknown;
};

const DriverFns& driver_fns() {
    static DriverFns fns;
    static std::once_flag once;
    std::call_once(once, [] {
        void* a = nullptr;
        void* b = nullptr;
        cudaDriverEntryPointQueryResult qa = cudaDriverEntryPointSymbolNotFound,
                                        qb = cudaDriverEntryPointSymbolNotFound;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa);
        if (e == cudaSuccess) e = cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb);
        if (e == cudaSuccess && (qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess || !a || !b))
            e = cudaErrorNotSupported;
        fns.get_current = reinterpret_cast<CtxGetCurrentFn>(a);
        fns.get_id = reinterpret_cast<CtxGetIdFn>(b);
        fns.status = e;
    });
    return fns;
}

}  // namespace

cudaError_t current_context_id(unsigned long long* id) {
    const DriverFns& f = driver_fns();
    if (f.status != cudaSuccess) return f.status;
    CUcontext ctx = nullptr;
    if (f.get_current(&ctx) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
    if (!ctx) {
        // no context yet on this thread: let the runtime make the current
        // device's primary context current (no allocation involved)
        int dev = 0;
        const cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        const cudaError_t e2 = cudaSetDevice(dev);
        if (e2 != cudaSuccess) return e2;
        if (f.get_current(&ctx) != CUDA_SUCCESS || !ctx) return cudaErrorDeviceUninitialized;
    }
    return f.get_id(ctx, id) == CUDA_SUCCESS ? cudaSuccess : cudaErrorDeviceUninitialized;
}

}  // namespace crisb
