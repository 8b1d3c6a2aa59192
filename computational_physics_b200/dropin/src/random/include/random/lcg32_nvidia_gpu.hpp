// LCG32 for the nvidia_gpu target (added by the drop-in build): the stream state type its
// SwendsenWang_2D specialisation exchanges, as LCG32<DeviceName::AMD_GPU> exposes one
// (random/include/random/lcg32.hpp:99-108).  The lanes are 16 wide, the AVX-512 CPU build's
// lane count, so the GPU streams are bit-identical to the CPU path's; the streams themselves
// live on the device (libswb200.so).
#pragma once

#if defined CP_NVIDIA_GPU

#include "random/lcg32.hpp"

#if !defined(XXX_NAMESPACE)
#define XXX_NAMESPACE cp
#endif

namespace XXX_NAMESPACE
{
    template <>
    class LCG32<DeviceName::NVIDIA_GPU> : public RandomNumberGenerator
    {
        public:
            static constexpr std::uint32_t WaveFrontSize = 16;
            using State = LCG32_State<WaveFrontSize>;
    };
}

#undef XXX_NAMESPACE

#endif
