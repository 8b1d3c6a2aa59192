// Throughput kernel of the lcg32 generator on its own: the equivalent of the reference's
// TestRNG --target program (random/src/test_rng.cpp, random/src/test_rng_amd_gpu.cpp:44-133,
// random/src/test_rng_cpu.cpp).  Many independent streams, stream i seeded seed_base + i as
// LCG32_State::Init does (random/src/lcg32.cpp:27-49); each update of a stream's W lanes
// yields W numbers 2^-32 * (float)u in the order of LCG32<CPU>::NextReal (element k is lane
// k % W after update k / W + 1, random/src/lcg32.cpp:103-129), with the parameter rotation
// before every 15th update (random/src/lcg32.cpp:51-84).
//
// One stream lives in the registers of a W-lane warp segment.  What a program can observe is
// kept: the last 64 numbers of one chosen stream (the reference's 64-number buffer) and an XOR
// of the bits of every number generated, so that no number is dead code.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/swb200.h"
#include "sw_core.cuh"

namespace swb {
namespace {

constexpr uint32_t kRngThreads = 256;
constexpr uint32_t kReport = 64;  // numbers kept of the reported stream

template <int W>
__global__ void __launch_bounds__(kRngThreads) k_lcg32_bench(const uint32_t n_streams, const uint32_t seed_base,
                                                             const uint64_t updates, const uint32_t report_id,
                                                             float *__restrict__ report, unsigned int *checksum)
{
    constexpr uint32_t kLast = kReport / W;  // updates that fill the report buffer
    __shared__ uint32_t init_state[kRngThreads];
    __shared__ uint8_t init_sel[kRngThreads];
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t stream = gid / W, lane = gid % W;
    const bool on = stream < n_streams;
    // LCG32_State::Init of this stream by its lane 0 (W drand48 draws pick the parameter pairs,
    // one more seeds the first lane, every later lane follows by one step of its own pair).
    if (lane == 0 && on) {
        uint64_t x = drand48_seed(seed_base + stream);
        uint32_t s[W];
#pragma unroll
        for (int i = 0; i < W; ++i) {
            x = drand48_step(x);
            s[i] = ((uint32_t)__dmul_rn(1000.0, drand48_value(x))) % 5u;
            init_sel[threadIdx.x + i] = (uint8_t)s[i];
        }
        x = drand48_step(x);
        uint32_t v = lcg_param_a(s[0]) * ((uint32_t)__dmul_rn(4026531839.0, drand48_value(x)) + 1u) + lcg_param_c(s[0]);
        init_state[threadIdx.x] = v;
#pragma unroll
        for (int i = 1; i < W; ++i) {
            v = lcg_param_a(s[i]) * v + lcg_param_c(s[i]);
            init_state[threadIdx.x + i] = v;
        }
    }
    __syncthreads();
    uint32_t st = on ? init_state[threadIdx.x] : 0u, sel = on ? init_sel[threadIdx.x] : 0u;
    uint32_t a = lcg_param_a(sel), c = lcg_param_c(sel);
    uint32_t it = 0, to_rot = kShuffleDistance;  // updates until the next rotation
    float last[kLast];
    uint32_t x = 0;
    for (uint64_t u = 0; u < updates; u += kLast) {
#pragma unroll
        for (uint32_t k = 0; k < kLast; ++k) {
            const bool rot = to_rot == 1;
            if (__any_sync(0xffffffffu, rot)) {
                const uint32_t itn = it + 1;
                const uint32_t src = __shfl_sync(0xffffffffu, st, itn & (W - 1), W);
                const uint32_t from = (lane + src + ((itn & 1u) ? 0u : 1u)) & (W - 1);
                const uint32_t a2 = __shfl_sync(0xffffffffu, a, from, W);
                const uint32_t c2 = __shfl_sync(0xffffffffu, c, from, W);
                if (rot) {
                    a = a2;
                    c = c2;
                }
            }
            it += 1;
            st = a * st + c;
            to_rot = rot ? kShuffleDistance : to_rot - 1;
            const float f = __uint2float_rn(st) * kTwoPowMinus32;  // exact scaling of the rounded u
            x ^= __float_as_uint(f);
            last[k] = f;
        }
    }
    if (on && stream == report_id) {
#pragma unroll
        for (uint32_t k = 0; k < kLast; ++k)
            report[k * W + lane] = last[k];
    }
    x = __reduce_xor_sync(0xffffffffu, on ? x : 0u);
    if ((threadIdx.x & 31) == 0 && x)
        atomicXor(checksum, x);
}

template <int W>
int launch_bench(uint32_t n_streams, uint32_t seed_base, uint64_t updates, uint32_t report_id, float *d_report,
                 unsigned int *d_sum, cudaStream_t st)
{
    const uint64_t threads = (uint64_t)n_streams * W;
    const uint32_t grid = (uint32_t)((threads + kRngThreads - 1) / kRngThreads);
    k_lcg32_bench<W><<<grid, kRngThreads, 0, st>>>(n_streams, seed_base, updates, report_id, d_report, d_sum);
    SWB_LAUNCHED();
    return SWB_OK;
}

}  // namespace
}  // namespace swb

using namespace swb;

extern "C" {

int swb_lcg32_benchmark(uint32_t n_streams, uint32_t lcg_width, uint32_t seed_base, uint64_t updates_per_stream,
                        uint32_t report_id, float *report, uint32_t *checksum, float *ms, int device)
{
    if (!report || !checksum || !ms)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (!(lcg_width == 8 || lcg_width == 16 || lcg_width == 32))
        return fail(SWB_ERR_ARGUMENT, "unsupported lcg32 width %u (8, 16 or 32)", lcg_width);
    const uint64_t per = kReport / lcg_width;
    if (n_streams == 0 || report_id >= n_streams || updates_per_stream < per || updates_per_stream % per)
        return fail(SWB_ERR_ARGUMENT, "need n_streams > report_id and updates a positive multiple of %llu",
                    (unsigned long long)per);
    if ((uint64_t)n_streams * lcg_width > 0xFFFFFFFFull)
        return fail(SWB_ERR_ARGUMENT, "too many streams");
    SWB_CUDA(cudaSetDevice(device));
    cudaStream_t st = nullptr;
    float *d_report = nullptr;
    unsigned int *d_sum = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    auto run = [&]() -> int {
        SWB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        SWB_CUDA(cudaMalloc(&d_report, kReport * sizeof(float)));
        SWB_CUDA(cudaMalloc(&d_sum, sizeof(unsigned int)));
        SWB_CUDA(cudaMemsetAsync(d_sum, 0, sizeof(unsigned int), st));
        for (auto &e : ev)
            SWB_CUDA(cudaEventCreate(&e));
        SWB_CUDA(cudaEventRecord(ev[0], st));
        int rc = SWB_OK;
        switch (lcg_width) {
        case 8: rc = launch_bench<8>(n_streams, seed_base, updates_per_stream, report_id, d_report, d_sum, st); break;
        case 16: rc = launch_bench<16>(n_streams, seed_base, updates_per_stream, report_id, d_report, d_sum, st); break;
        default: rc = launch_bench<32>(n_streams, seed_base, updates_per_stream, report_id, d_report, d_sum, st); break;
        }
        if (rc)
            return rc;
        SWB_CUDA(cudaEventRecord(ev[1], st));
        SWB_CUDA(cudaEventSynchronize(ev[1]));
        SWB_CUDA(cudaEventElapsedTime(ms, ev[0], ev[1]));
        SWB_CUDA(cudaMemcpyAsync(report, d_report, kReport * sizeof(float), cudaMemcpyDeviceToHost, st));
        SWB_CUDA(cudaMemcpyAsync(checksum, d_sum, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
        SWB_CUDA(cudaStreamSynchronize(st));
        return SWB_OK;
    };
    const int rc = run();
    if (st)
        cudaStreamSynchronize(st);
    for (auto &e : ev)
        if (e)
            cudaEventDestroy(e);
    cudaFree(d_report);
    cudaFree(d_sum);
    if (st)
        cudaStreamDestroy(st);
    return rc;
}

}  // extern "C"
