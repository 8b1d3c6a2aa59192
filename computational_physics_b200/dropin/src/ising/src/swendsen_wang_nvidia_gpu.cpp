// SwendsenWang_2D<LCG32, DeviceName::NVIDIA_GPU> (added by the drop-in build): Initialize and
// Update of the nvidia_gpu target over the C ABI of libswb200.so.
#include <iostream>
#include <stdexcept>

#include "environment/environment.hpp"
#include "swendsen_wang.hpp"

#if !defined(XXX_NAMESPACE)
#define XXX_NAMESPACE cp
#endif

namespace XXX_NAMESPACE
{
    SwendsenWang_2D<LCG32, DeviceName::NVIDIA_GPU>::~SwendsenWang_2D()
    {
        swb_destroy(handle);
    }

    // The reference's Initialize for its GPU target (ising/src/swendsen_wang.cpp:41-92): even
    // extents, the GPU tile policy {2 * wavefront / 8, 8} unless TILE_SIZE_X / TILE_SIZE_Y say
    // otherwise, one lcg32 stream per tile seeded i + 1, the label array.
    void SwendsenWang_2D<LCG32, DeviceName::NVIDIA_GPU>::Initialize(Lattice<2>& lattice)
    {
        if (!handle)
        {
            const auto& extent = lattice.Extent();
            if (extent[0] % 2 || extent[1] % 2)
                throw std::runtime_error("SwendsenWang_2D implementation requires evenly sized lattice.");

            std::cout << "Lattice: " << extent[0] << " x " << extent[1] << " (";
            constexpr auto wavefront = DeviceType::WavefrontSize();
            tile_size = {GetEnv("TILE_SIZE_X", 2 * wavefront / 8), GetEnv("TILE_SIZE_Y", 8U)};
            std::cout << "tile size: " << tile_size[0] << " x " << tile_size[1] << ")" << std::endl;

            SwbCall(swb_create(&handle, extent[0], extent[1], tile_size[0], tile_size[1],
                               LCG32<DeviceName::NVIDIA_GPU>::WaveFrontSize, 1 /* seeds i + 1 */,
                               static_cast<int>(target.DeviceId())));
        }
        if (attached != lattice.RawGpuPointer())
        {
            SwbCall(swb_attach_spins(handle, lattice.RawGpuPointer()));
            attached = lattice.RawGpuPointer();
        }
    }

    void SwendsenWang_2D<LCG32, DeviceName::NVIDIA_GPU>::Update(Lattice<2>& lattice, const float temperature)
    {
        Initialize(lattice);
        SwbCall(swb_sweep(handle, temperature, 1, 0));
    }
}
