// The nvidia_gpu target device of the reference's device abstraction (added by the drop-in
// build, computational_physics_b200/dropin/build_dropin.py): DeviceName::NVIDIA_GPU's device
// class, its execution context and the device-side spin storage of Lattice<2>.  Everything
// CUDA goes through the C ABI of swb200.h (libswb200.so); this header includes no CUDA header.
//
// Counterparts in the reference: AMD_GPU (utility/device/device_amd_gpu.hpp:15-81),
// HipContext (utility/execution/hip_context.hpp:13-37), SafeCall (utility/hip/hip.cpp),
// GpuPointer (utility/hip/hip.hpp).
#pragma once

#if defined CP_NVIDIA_GPU

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>

#include "swb200.h"
#include "environment/environment.hpp"
#include "execution/context.hpp"

#if !defined(XXX_NAMESPACE)
#define XXX_NAMESPACE cp
#endif

namespace XXX_NAMESPACE
{
    // A non-zero status of the C ABI becomes std::runtime_error with the library's message.
    inline void SwbCall(const int status)
    {
        if (status != SWB_OK)
            throw std::runtime_error(std::string("CUDA error: ") + swb_last_error());
    }

    class NVIDIA_GPU;

    // group_size = number of GPUs, id = GPU id, as for HipContext.
    class CudaContext final : public Context
    {
        private:
            NVIDIA_GPU& device;

        public:
            CudaContext(const std::uint32_t group_size, const std::uint32_t id, NVIDIA_GPU& device) noexcept
                :
                Context(group_size, id), device(device)
            {}

            void Synchronize() override { SwbCall(swb_device_synchronize(static_cast<int>(id))); }

            NVIDIA_GPU& Device() const noexcept { return device; }
    };

    class NVIDIA_GPU final : public AbstractDevice
    {
        public:
            NVIDIA_GPU(const std::uint32_t device_id = 0)
                :
                NVIDIA_GPU(GetEnv("NUM_THREADS_GPU", SmCount(device_id)), device_id)
            {}

            NVIDIA_GPU(const std::uint32_t concurrency, const std::uint32_t device_id)
                :
                AbstractDevice(DeviceName::NVIDIA_GPU, device_id), concurrency(concurrency),
                context(1 /* number of GPUs */, device_id, *this)
            {}

            bool IsOffloadDevice() const noexcept override { return true; }

            std::uint32_t Concurrency() const noexcept override { return concurrency; }

            static constexpr auto Name() noexcept { return DeviceName::NVIDIA_GPU; }

            template <typename T = void>
            static constexpr std::uint32_t WavefrontSize() { return 32; }  // warp size

            template <typename Func, typename ...Args>
            void Execute(Func&& func, Args&&... args)
            {
                func(context, std::forward<Args>(args)...);
            }

            void Synchronize() { context.Synchronize(); }

            CPU& Host() { return host; }

        private:
            static std::uint32_t SmCount(const std::uint32_t device_id)
            {
                std::uint32_t n = 0;
                SwbCall(swb_device_sm_count(static_cast<int>(device_id), &n));
                return n;
            }

            const std::uint32_t concurrency;
            CudaContext context;
            CPU host; /* configured via NUM_THREADS */
    };

    template <>
    struct Device<DeviceName::NVIDIA_GPU>
    {
        using Type = NVIDIA_GPU;
    };

    // Device memory owned by a Lattice<2> (the GpuPointer of the HIP path).
    struct SwbDeviceFree
    {
        int device = 0;
        void operator()(void* p) const noexcept { swb_device_free(device, p); }
    };

    template <typename T>
    using NvGpuPointer = std::unique_ptr<T, SwbDeviceFree>;
}

#undef XXX_NAMESPACE

#endif
