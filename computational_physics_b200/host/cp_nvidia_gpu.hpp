// C++ host mirror of the reference's device / execution / algorithm interface for the new
// nvidia_gpu target (flwende/computational_physics).  Same names, argument meaning and error
// behaviour as the reference; compute goes through the C ABI of include/swb200.h.
//
//   DeviceName::NVIDIA_GPU, NVIDIA_GPU, Device<>  utility/device/device.hpp:11-42,
//                                                 utility/device/device_amd_gpu.hpp:15-81
//   CudaContext                                   utility/execution/hip_context.hpp:18-37
//   GetDevice / DispatchCall                      utility/device/helper.{hpp,cpp}
//   SafeCall (throws std::runtime_error)          utility/hip/hip.cpp:16-24
//   LCG32<NVIDIA_GPU>::State                      random/include/random/lcg32.hpp:99-108
//   Lattice<2>                                    ising/include/lattice.hpp:21-95
//   SwendsenWang_2D<LCG32, NVIDIA_GPU>            ising/include/swendsen_wang.hpp:26-102
//
// There is no CPU target in this build: "cpu" is rejected with the reference's error.
#pragma once

#include <array>
#include <cstdint>
#include <cstdlib>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "swb200.h"

namespace cp
{
    enum class DeviceName : std::uint32_t
    {
        CPU = 1,
        AMD_GPU = 2,
        NVIDIA_GPU = 3
    };

    // SafeCall: non-zero status -> std::runtime_error with the library's message.
    inline void SafeCall(int status)
    {
        if (status != SWB_OK)
            throw std::runtime_error(std::string("CUDA error: ") + swb_last_error());
    }

    template <typename T>
    T GetEnv(const std::string& name, const T& default_value = {})
    {
        const char* value = std::getenv(name.c_str());
        if (!value)
            return default_value;
        try
        {
            return static_cast<T>(std::stoll(value));
        }
        catch (const std::exception&)
        {
            return default_value;
        }
    }

    class Context
    {
        protected:
            const std::uint32_t group_size {};
            const std::uint32_t id {};

        public:
            explicit Context(const std::uint32_t group_size, const std::uint32_t id) noexcept : group_size(group_size), id(id) {}
            virtual ~Context() noexcept = default;
            auto GroupSize() const noexcept { return group_size; }
            auto Id() const noexcept { return id; }
            virtual void Synchronize() = 0;
    };

    class AbstractDevice
    {
        protected:
            DeviceName device_name {};
            std::uint32_t device_id {};

        public:
            virtual ~AbstractDevice() noexcept = default;
            virtual bool IsOffloadDevice() const noexcept = 0;
            virtual std::uint32_t Concurrency() const noexcept = 0;
            constexpr auto Name() const noexcept { return device_name; }
            auto DeviceId() const noexcept { return device_id; }

        protected:
            AbstractDevice(const DeviceName device_name, const std::uint32_t device_id) : device_name(device_name), device_id(device_id) {}
    };

    class NVIDIA_GPU;

    // The meaning of group_size and id is "number of GPUs" and "GPU id" (as HipContext).
    class CudaContext final : public Context
    {
        private:
            NVIDIA_GPU& device;

        public:
            CudaContext(const std::uint32_t group_size, const std::uint32_t id, NVIDIA_GPU& device) noexcept
                : Context(group_size, id), device(device) {}
            void Synchronize() override {}   // work is stream-ordered per lattice; see SwendsenWang_2D
            NVIDIA_GPU& Device() const noexcept { return device; }
    };

    class NVIDIA_GPU final : public AbstractDevice
    {
        public:
            NVIDIA_GPU(const std::uint32_t device_id = 0)
                : NVIDIA_GPU(GetEnv("NUM_THREADS_GPU", 148U), device_id) {}

            NVIDIA_GPU(const std::uint32_t concurrency, const std::uint32_t device_id)
                : AbstractDevice(DeviceName::NVIDIA_GPU, device_id), concurrency(concurrency), context(1, device_id, *this)
            {
                int count = 0;
                SafeCall(swb_device_count(&count));
                if (count <= static_cast<int>(device_id))
                    throw std::runtime_error("CUDA error: no CUDA device " + std::to_string(device_id));
            }

            bool IsOffloadDevice() const noexcept override { return true; }
            std::uint32_t Concurrency() const noexcept override { return concurrency; }
            static constexpr auto Name() noexcept { return DeviceName::NVIDIA_GPU; }

            // Warp size; the tile policy {2 * wf / 8, 8} of ising/src/swendsen_wang.cpp:136 gives 8 x 8.
            template <typename T = void>
            static constexpr std::uint32_t WavefrontSize() { return 32; }

            template <typename Func, typename ...Args>
            void Execute(Func&& func, Args&&... args)
            {
                func(context, std::forward<Args>(args)...);
            }

            void Synchronize() { context.Synchronize(); }

        private:
            const std::uint32_t concurrency;
            CudaContext context;
    };

    template <DeviceName T>
    struct Device;

    template <>
    struct Device<DeviceName::NVIDIA_GPU>
    {
        using Type = NVIDIA_GPU;
    };

    inline std::unique_ptr<AbstractDevice> GetDevice(const std::string& device_name)
    {
        if (device_name == "nvidia_gpu")
            return std::make_unique<NVIDIA_GPU>();
        throw std::runtime_error("Unknown target device.");
    }

    template <typename Func, typename ...Args>
    auto DispatchCall(const std::string& device_name, AbstractDevice& device, Func&& func, Args&&... args)
    {
        if (device_name == "nvidia_gpu")
            return func(static_cast<NVIDIA_GPU&>(device), std::forward<Args>(args)...);
        throw std::runtime_error("Unknown device name.");
    }

    // lcg32 for the nvidia_gpu target: the stream state keeps LCG32_State<W>'s layout.  W is
    // the reference CPU host's SIMD lane count so that results match the CPU path bit for bit
    // (16 with AVX-512); LCG32_WIDTH overrides it (8, 16 or 32).
    template <DeviceName Type>
    class LCG32;

    template <std::uint32_t W>
    struct LCG32_State
    {
        std::uint32_t state[W] {};
        std::uint32_t a[W] {};
        std::uint32_t c[W] {};
        std::uint32_t iteration {};
        static constexpr auto GetShuffleDistance() { return std::uint32_t{15}; }
    };

    template <>
    class LCG32<DeviceName::NVIDIA_GPU>
    {
        public:
            static constexpr std::uint32_t DefaultWaveFrontSize = 16;
            using State = LCG32_State<DefaultWaveFrontSize>;
            static std::uint32_t WaveFrontSize() { return GetEnv("LCG32_WIDTH", DefaultWaveFrontSize); }
    };

    template <std::uint32_t Dimension>
    class Lattice;

    template <std::uint32_t Dimension, template <DeviceName> typename RNG, DeviceName Target>
    class LatticeMonteCarloAlgorithm
    {
        public:
            virtual ~LatticeMonteCarloAlgorithm() noexcept = default;
            virtual void Update(Lattice<Dimension>& lattice, const float temperature) = 0;
    };

    template <template <DeviceName> typename RNG, DeviceName Target>
    class SwendsenWang_2D;

    // Lattice<2>: uint8 0/1 spins on the host, hot start srand48(1) (ising/src/lattice.cpp:113-125);
    // the nvidia_gpu mirror lives in the SwendsenWang_2D handle.
    template <>
    class Lattice<2> final
    {
        public:
            using Spin = std::uint8_t;

        private:
            const std::array<std::uint32_t, 2> extent {};
            const std::size_t num_sites {};
            std::vector<Spin> spins;
            swb_lattice* gpu {};          // device mirror, owned by the strategy
            bool host_current = true;     // host spins up to date
            bool device_current = false;  // device spins up to date

        public:
            Lattice(const std::array<std::uint32_t, 2>& extent);

            auto& Extent() const noexcept { return extent; }
            auto NumSites() const noexcept { return num_sites; }
            Spin* RawPointer() { SyncToHost(); return spins.data(); }

            template <template <template <DeviceName> typename, DeviceName> typename Strategy,
                template <DeviceName> typename RNG, typename Target,
                typename StrategyImplementation = Strategy<RNG, Target::Name()>>
            void Update(const float temperature, Target& target)
            {
                static auto strategy = StrategyImplementation(target);
                strategy.Update(*this, temperature);
            }

            std::pair<double, double> GetEnergyAndMagnetization(NVIDIA_GPU& target);

            // Device mirror hooks (InitializeGpuSpins, ising/src/lattice.cpp:179-194).
            void AttachGpu(swb_lattice* handle);
            swb_lattice* Gpu() const noexcept { return gpu; }
            void MarkDeviceCurrent() { device_current = true; host_current = false; }
            void SyncToHost();
            void EnsureDevice();
    };

    // The drop-in strategy for the nvidia_gpu target.
    template <>
    class SwendsenWang_2D<LCG32, DeviceName::NVIDIA_GPU> : public LatticeMonteCarloAlgorithm<2, LCG32, DeviceName::NVIDIA_GPU>
    {
        using DeviceType = NVIDIA_GPU;

        protected:
            DeviceType& target;
            swb_lattice* handle {};
            std::array<std::uint32_t, 2> tile_size {};

        public:
            SwendsenWang_2D(DeviceType& target) : target(target) {}
            SwendsenWang_2D(SwendsenWang_2D&& other) noexcept : target(other.target), handle(other.handle), tile_size(other.tile_size) { other.handle = nullptr; }
            ~SwendsenWang_2D() { if (handle) swb_destroy(handle); }

            void Update(Lattice<2>& lattice, const float temperature) override;

            // n sweeps with a device-side measurement every measure_every sweeps (the CLI's loop).
            void Update(Lattice<2>& lattice, const float temperature, std::uint32_t n, std::uint32_t measure_every);

            swb_lattice* Handle() const noexcept { return handle; }

        protected:
            void Initialize(Lattice<2>& lattice);
    };
}
