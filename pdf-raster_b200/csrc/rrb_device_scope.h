// rrb_device_scope.h — entry points leave the calling thread's CUDA context
// as they found it.
//
// Every public entry point makes its context's device current for the length
// of the call (DeviceScope). On exit the thread's previous current context is
// made current again, so an application that drives another GPU from the same
// thread (a PyTorch process, a renderer with one context per device) is not
// moved to this library's device behind its back. A thread that had no
// current context is left with the library's device current: restoring
// "no device" is not expressible through the runtime API, and binding some
// other device instead would create a context on it.
//
// The driver's cuCtxGetCurrent / cuCtxSetCurrent are looked up through the
// runtime (cudaGetDriverEntryPoint), so the library does not link libcuda and
// still loads on a machine without a GPU driver.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

namespace rrb_host {

struct CtxFns {
    CUresult (*get)(CUcontext*) = nullptr;
    CUresult (*set)(CUcontext) = nullptr;
};

inline const CtxFns& ctx_fns() {
    static const CtxFns fns = [] {
        CtxFns f;
        cudaDriverEntryPointQueryResult q;
        void* g = nullptr;
        void* s = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &g, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPoint("cuCtxSetCurrent", &s, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess) {
            f.get = reinterpret_cast<CUresult (*)(CUcontext*)>(g);
            f.set = reinterpret_cast<CUresult (*)(CUcontext)>(s);
        } else {
            cudaGetLastError();
        }
        return f;
    }();
    return fns;
}

class DeviceScope {
   public:
    explicit DeviceScope(int device) {
        const CtxFns& f = ctx_fns();
        if (f.get && f.get(&prev_) == CUDA_SUCCESS && prev_) saved_ = true;
        status_ = cudaSetDevice(device);
    }
    ~DeviceScope() {
        if (saved_) ctx_fns().set(prev_);
    }
    DeviceScope(const DeviceScope&) = delete;
    DeviceScope& operator=(const DeviceScope&) = delete;
    cudaError_t status() const { return status_; }

   private:
    CUcontext prev_ = nullptr;
    bool saved_ = false;
    cudaError_t status_ = cudaSuccess;
};

}  // namespace rrb_host
