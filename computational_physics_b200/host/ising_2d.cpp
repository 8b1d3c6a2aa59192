// Ising2D command line program for the nvidia_gpu target: same options, defaults and output
// lines as the reference's ising/src/ising_2d.cpp:26-165.
//
//   Ising2D [--extent=N0xN1] [--num_sweeps=S] [--temperature=T] [--algorithm=swendsen_wang]
//           [--rng=lcg32] [--target=nvidia_gpu]
//
// 1000 warmup sweeps, then S sweeps with a measurement every 10 sweeps.  The measurement is a
// device-side reduction accumulated in FP64 on the GPU (the reference copies all spins to the
// host every 10 sweeps, ising/src/lattice.cpp:170-177); the printed quantities are the same:
// ns per spin update (wall time including measurement), E/N, C/N and |M|/N.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <iostream>
#include <stdexcept>
#include <string>

#include "cp_nvidia_gpu.hpp"

using namespace cp;

static constexpr auto N_Warmup = std::uint32_t{1000};
static constexpr auto N_Sep = std::uint32_t{10};

namespace defaults
{
    static constexpr auto N_0 = std::uint32_t{32};
    static constexpr auto N_1 = std::uint32_t{32};
    static constexpr auto Temperature = 2.2691853142130221F;
    static constexpr auto N_Sweeps = std::uint32_t{N_Sep * 10000};
}

int main(int argc, char** argv)
{
    auto n_0 {defaults::N_0};
    auto n_1 {defaults::N_1};
    auto temperature {defaults::Temperature};
    auto n_sweeps {defaults::N_Sweeps};
    auto algorithm = std::string{"swendsen_wang"};
    auto rng_name = std::string{"lcg32"};
    auto target_name = std::string{"nvidia_gpu"};

    if (argc > 1 && (std::string(argv[1]) == "--help" || std::string(argv[1]) == "-h"))
    {
        std::cout << "Usage: " << argv[0] << " [options]" << std::endl
                  << "Options:" << std::endl
                  << "  --help, -h         Show this help message" << std::endl
                  << "  --algorithm        Set algorithm (default: swendsen_wang)" << std::endl
                  << "  --extent=N0xN1     Set lattice dimensions" << std::endl
                  << "  --num_sweeps       Set number of MC sweeps (default: 100000)" << std::endl
                  << "  --rng=<name>       Set RNG type (default: lcg32)" << std::endl
                  << "  --target=<name>    Set target device (default: nvidia_gpu)" << std::endl
                  << "      Supported target devices: nvidia_gpu" << std::endl
                  << "  --temperature      Set temperature (default: 2.2691853)" << std::endl;
        return 0;
    }

    for (int i = 1; i < argc; ++i)
    {
        const auto arg = std::string{argv[i]};
        if (const auto pos = arg.find('='); pos != std::string::npos)
        {
            const auto key = arg.substr(0, pos);
            const auto value = arg.substr(pos + 1);
            if (key == "--extent")
            {
                if (const auto x_pos = value.find('x'); x_pos != std::string::npos)
                {
                    n_0 = std::atoi(value.substr(0, x_pos).c_str());
                    n_1 = std::atoi(value.substr(x_pos + 1).c_str());
                }
            }
            else if (key == "--num_sweeps")
                n_sweeps = std::atoi(value.c_str());
            else if (key == "--temperature")
                temperature = std::atof(value.c_str());
            else if (key == "--algorithm")
                algorithm = value;
            else if (key == "--rng")
                rng_name = value;
            else if (key == "--target")
                target_name = value;
        }
    }

    try
    {
        Lattice<2> lattice({n_0, n_1});
        auto target = GetDevice(target_name);
        std::cout << "Target name: NVIDIA GPU" << std::endl;
        if (rng_name != "lcg32")
            throw std::runtime_error("Unknown RNG name.");
        if (algorithm != "swendsen_wang")
            throw std::runtime_error("Unknown algorithm.");

        std::cout << "WARMUP: " << N_Warmup << " sweeps" << std::endl;
        std::cout << "MEASUREMENT: " << n_sweeps << " sweeps" << std::endl;

        auto& gpu = static_cast<NVIDIA_GPU&>(*target);
        SwendsenWang_2D<LCG32, DeviceName::NVIDIA_GPU> strategy(gpu);
        strategy.Update(lattice, temperature, N_Warmup, 0);
        SafeCall(swb_synchronize(strategy.Handle()));
        SafeCall(swb_reset_accumulators(strategy.Handle()));

        const auto starttime = std::chrono::high_resolution_clock::now();
        strategy.Update(lattice, temperature, n_sweeps - n_sweeps % N_Sep, N_Sep);
        double acc[4] {};
        SafeCall(swb_accumulators(strategy.Handle(), acc));   // waits for the sweeps
        const auto endtime = std::chrono::high_resolution_clock::now();
        const auto elapsed_time_s = std::chrono::duration_cast<std::chrono::microseconds>(endtime - starttime).count() * 1.0E-6;

        std::cout << "Update time per spin: ";
        std::cout << elapsed_time_s * 1.0E9 / (static_cast<std::int64_t>(n_sweeps) * n_0 * n_1) << " ns" << std::endl;

        const auto energy = acc[0], energy_squared = acc[1], magnetization = acc[2];
        const auto samples = n_sweeps / N_Sep;
        const auto heat_capacity = ((energy_squared / samples) - (energy / samples) * (energy / samples)) *
            lattice.NumSites() / (temperature * temperature);

        std::cout << "Internal energy per spin: " << energy / samples << std::endl;
        std::cout << "Heat capacity per spin: " << heat_capacity << std::endl;
        std::cout << "Absolute Magnetization per spin: " << magnetization / samples << std::endl;
    }
    catch (const std::exception& e)
    {
        std::cerr << e.what() << std::endl;
        return 1;
    }
    return 0;
}
