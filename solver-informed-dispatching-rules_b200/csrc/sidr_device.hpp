// sidr_device.hpp -- the calling thread's current device across library calls.
//
// Every entry point that works on a device makes it current with cudaSetDevice.
// DeviceGuard puts the caller's current device back when the call returns, so a
// framework that keeps its own notion of the current device (torch, a serving
// runtime) is not left on another GPU.  It restores only a device whose primary
// context is already active: a thread that never used a device (the runtime
// reports device 0 for it) is not given a context on device 0 by the restore.
#pragma once
#include <cuda_runtime.h>
#include <dlfcn.h>

namespace sidr {

inline bool primary_context_active(int dev) {
    using GetState = int (*)(int, unsigned*, int*);
    using DeviceGet = int (*)(int*, int);
    static GetState get_state = nullptr;
    static DeviceGet device_get = nullptr;
    static bool looked = false;
    if (!looked) {
        // the runtime has loaded the driver library by the time a guard exists
        if (void* h = dlopen("libcuda.so.1", RTLD_NOW | RTLD_NOLOAD)) {
            get_state = (GetState)dlsym(h, "cuDevicePrimaryCtxGetState");
            device_get = (DeviceGet)dlsym(h, "cuDeviceGet");
        }
        looked = true;
    }
    if (!get_state || !device_get) return false;
    int cu_dev = 0;
    if (device_get(&cu_dev, dev) != 0) return false;
    unsigned flags = 0;
    int active = 0;
    return get_state(cu_dev, &flags, &active) == 0 && active != 0;
}

struct DeviceGuard {
    int prev = -1;
    DeviceGuard() {
        if (cudaGetDevice(&prev) != cudaSuccess) {
            cudaGetLastError();
            prev = -1;
        }
    }
    ~DeviceGuard() {
        int now = -1;
        if (prev < 0 || cudaGetDevice(&now) != cudaSuccess || now == prev) return;
        if (primary_context_active(prev)) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;
};

}  // namespace sidr
