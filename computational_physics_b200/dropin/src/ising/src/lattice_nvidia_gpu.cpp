// Lattice<2>'s hooks for the nvidia_gpu target (added by the drop-in build): the device copy
// of the spins and the energy / magnetisation measurement.  Counterparts of the AMD_GPU
// specialisations in ising/src/lattice.cpp:69-96; the measurement is a reduction on the device
// instead of a copy of all spins to the host.
#include <iostream>

#include "lattice.hpp"

#if !defined(XXX_NAMESPACE)
#define XXX_NAMESPACE cp
#endif

namespace XXX_NAMESPACE
{
    template <>
    template <>
    std::pair<double, double> Lattice<2>::GetEnergyAndMagnetization<NVIDIA_GPU>(NVIDIA_GPU& gpu)
    {
        double em[2] {};
        SwbCall(swb_spins_energy_magnetization(static_cast<int>(gpu.DeviceId()), extent[0], extent[1],
                                               RawGpuPointer(), em, nullptr, nullptr));
        return {em[0], em[1]};
    }

    template <>
    void Lattice<2>::InitializeGpuSpins(NVIDIA_GPU& gpu)
    {
        if (!nv_gpu_spins.get())
        {
            std::cout << "Initializing GPU spins .. ";

            const int device = static_cast<int>(gpu.DeviceId());
            void* ptr = nullptr;
            SwbCall(swb_device_alloc(device, NumSites() * sizeof(Spin), &ptr));
            nv_gpu_spins = NvGpuPointer<Spin>(static_cast<Spin*>(ptr), SwbDeviceFree{device});
            SwbCall(swb_copy_to_device(device, ptr, RawPointer(), NumSites() * sizeof(Spin)));

            std::cout << "Done." << std::endl;
        }
    }
}
