// SwendsenWang_2D for the nvidia_gpu target (added by the drop-in build).  The same plugin
// interface as the reference's template (ising/include/swendsen_wang.hpp:25-100): constructed
// from the target device, Update(lattice, temperature) runs one sweep.  The sweep is the
// B200 engine of libswb200.so (swb_sweep): the lcg32 streams, labels and scratch live in a
// handle the strategy owns, the spins are the lattice's own device array
// (Lattice<2>::RawGpuPointer), attached to the handle.
#pragma once

#if defined CP_NVIDIA_GPU

#include <array>
#include <cstdint>

#include "swb200.h"

#if !defined(XXX_NAMESPACE)
#define XXX_NAMESPACE cp
#endif

namespace XXX_NAMESPACE
{
    template <>
    class SwendsenWang_2D<LCG32, DeviceName::NVIDIA_GPU>
        : public LatticeMonteCarloAlgorithm<2, LCG32, DeviceName::NVIDIA_GPU>
    {
        using DeviceType = NVIDIA_GPU;
        using RngState = LCG32<DeviceName::NVIDIA_GPU>::State;

        protected:
            DeviceType& target;
            std::array<std::uint32_t, 2> tile_size {};
            swb_lattice* handle = nullptr;
            const Lattice<2>::Spin* attached = nullptr;  // the lattice's device spins the handle sweeps

        public:
            SwendsenWang_2D(DeviceType& target) : target(target) {}

            SwendsenWang_2D(const SwendsenWang_2D&) = delete;
            SwendsenWang_2D& operator=(const SwendsenWang_2D&) = delete;

            ~SwendsenWang_2D() override;

            // One sweep: bonds with the lcg32 draws of every tile, labels, boundary merge,
            // resolution and cluster flip, all on the device.
            void Update(Lattice<2>& lattice, const float temperature) override;

            static constexpr std::uint32_t Dimension = 2;

            // The engine's handle (measurement accumulators, stream state).
            swb_lattice* Handle() const noexcept { return handle; }

        protected:
            void Initialize(Lattice<2>& lattice);
    };
}

#undef XXX_NAMESPACE

#endif
