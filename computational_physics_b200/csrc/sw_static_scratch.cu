// The scratch array of swb_sweep_static (the sweep that allocates nothing, sw_plain.cu), in a
// translation unit of its own that holds no kernel.  The library is built without relocatable
// device code, so every .cu file becomes its own device module, and a module's __device__
// arrays are reserved on a device when that module loads there.  Here that happens only at the
// first cudaGetSymbolAddress below, i.e. on a device where swb_sweep_static is called: the
// other entry points never reserve these 24 MiB + 1 KiB.

#include <cuda_runtime.h>

#include <mutex>

#include "sw_core.cuh"

// In host code this name is a stand-in for the array, not a device address: the address comes
// from cudaGetSymbolAddress, once per device, with that device current.
static __device__ __align__(256) unsigned char swb_static_scratch[swb::kStaticScratchBytes];

namespace swb {

namespace {

constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mutex;
unsigned char *g_static_base[kStaticMaxDevices] = {};

}  // namespace

int static_scratch_base(int device, unsigned char **base)
{
    if (device < 0 || device >= kStaticMaxDevices)
        return fail(SWB_ERR_ARGUMENT, "device %d out of range", device);
    std::lock_guard<std::mutex> lock(g_static_mutex);
    if (!g_static_base[device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, swb_static_scratch);
        if (e != cudaSuccess)
            return fail(SWB_ERR_CUDA, "cudaGetSymbolAddress(swb_static_scratch) on device %d: %s", device,
                        cudaGetErrorString(e));
        g_static_base[device] = static_cast<unsigned char *>(p);
    }
    *base = g_static_base[device];
    return SWB_OK;
}

}  // namespace swb
