// Implementation of the nvidia_gpu host mirror declared in cp_nvidia_gpu.hpp.
#include "cp_nvidia_gpu.hpp"

#include <cstdlib>
#include <iostream>

namespace cp
{
    // ising/src/lattice.cpp:113-125: srand48(1), spin = drand48() < 0.5 ? 0 : 1.
    Lattice<2>::Lattice(const std::array<std::uint32_t, 2>& extent)
        : extent(extent), num_sites(static_cast<std::size_t>(extent[0]) * extent[1]), spins(num_sites)
    {
        srand48(1);
        for (std::size_t i = 0; i < num_sites; ++i)
            spins[i] = drand48() < 0.5 ? 0 : 1;
    }

    void Lattice<2>::AttachGpu(swb_lattice* handle)
    {
        gpu = handle;
        SafeCall(swb_set_spins(gpu, spins.data()));
        device_current = true;
        host_current = true;
    }

    void Lattice<2>::SyncToHost()
    {
        if (gpu && !host_current)
        {
            SafeCall(swb_get_spins(gpu, spins.data()));
            host_current = true;
        }
        // A caller may write through RawPointer(): the device copy is refreshed before the next sweep.
        device_current = false;
    }

    void Lattice<2>::EnsureDevice()
    {
        if (gpu && !device_current)
        {
            SafeCall(swb_set_spins(gpu, spins.data()));
            device_current = true;
        }
    }

    std::pair<double, double> Lattice<2>::GetEnergyAndMagnetization(NVIDIA_GPU& target)
    {
        double em[2] {};
        if (gpu)
        {
            if (!device_current)
            {
                SafeCall(swb_set_spins(gpu, spins.data()));
                device_current = true;
            }
            SafeCall(swb_energy_magnetization(gpu, em, nullptr, nullptr));
            return {em[0], em[1]};
        }
        // No mirror yet: reduce on a temporary device lattice (no host reduction path).
        swb_lattice* tmp {};
        SafeCall(swb_create(&tmp, extent[0], extent[1], 8, 8, 16, 1, static_cast<int>(target.DeviceId())));
        int rc = swb_set_spins(tmp, spins.data());
        if (rc == SWB_OK)
            rc = swb_energy_magnetization(tmp, em, nullptr, nullptr);
        swb_destroy(tmp);
        SafeCall(rc);
        return {em[0], em[1]};
    }

    void SwendsenWang_2D<LCG32, DeviceName::NVIDIA_GPU>::Initialize(Lattice<2>& lattice)
    {
        if (handle)
            return;
        const auto& extent = lattice.Extent();
        if (extent[0] % 2 || extent[1] % 2)
            throw std::runtime_error("SwendsenWang_2D implementation requires evenly sized lattice.");
        std::cout << "Lattice: " << extent[0] << " x " << extent[1] << " (";
        const auto wf = NVIDIA_GPU::WavefrontSize();
        tile_size = {GetEnv("TILE_SIZE_X", 2 * wf / 8), GetEnv("TILE_SIZE_Y", 8U)};
        std::cout << "tile size: " << tile_size[0] << " x " << tile_size[1] << ")" << std::endl;
        SafeCall(swb_create(&handle, extent[0], extent[1], tile_size[0], tile_size[1],
                            LCG32<DeviceName::NVIDIA_GPU>::WaveFrontSize(), 1, static_cast<int>(target.DeviceId())));
        lattice.AttachGpu(handle);
    }

    void SwendsenWang_2D<LCG32, DeviceName::NVIDIA_GPU>::Update(Lattice<2>& lattice, const float temperature)
    {
        Update(lattice, temperature, 1, 0);
    }

    void SwendsenWang_2D<LCG32, DeviceName::NVIDIA_GPU>::Update(Lattice<2>& lattice, const float temperature,
                                                               std::uint32_t n, std::uint32_t measure_every)
    {
        Initialize(lattice);
        if (lattice.Gpu() != handle)
            lattice.AttachGpu(handle);
        lattice.EnsureDevice();
        target.Execute([&, this] (CudaContext&)
            {
                SafeCall(swb_sweep(handle, temperature, n, measure_every));
            });
        lattice.MarkDeviceCurrent();
    }
}
