// Swendsen-Wang sweep for the 2D Ising model on one B200 (sm_100a), behind the C ABI of
// include/swb200.h.
//
// One sweep = four kernels on the handle's stream (reference phases in brackets,
// ising/src/swendsen_wang.cpp:94-112):
//
//   k_assign  [AssignLabels + the in-block part of MergeLabels]  one CTA per block of
//             TBX x TBY tiles.  Each tile's lcg32 stream lives in the registers of one
//             W-lane warp segment; the accept bits of every update are warp ballots.
//             Spins of the block plus a one-site halo are staged in shared memory, bond
//             words are formed bit-parallel, and a scanline pass with a lock-free union-find
//             toward the minimum index labels the block in shared memory.  Writes each
//             site's label (block roots: their global index; other sites: the block-local
//             index of their root) and the bond bits of the block's right and bottom edge.
//             A recorded sweep (kDebug) labels tile by tile first, as the reference's
//             AssignLabels does, to dump that stage.
//   k_merge   [MergeLabels across blocks]  atomicMin union on the global label array for
//             the edge bonds recorded by k_assign; each union records the root it linked.
//   k_resolve [ResolveLabels]  every linked root's chain is walked once to the root (the
//             cluster's minimum site index), which becomes its label.
//   k_flip    [ResolveLabels + FlipClusters]  every site reads its block root's label;
//             spin ^= root & 1.  (Without k_resolve, three kernels, k_flip walks the merged
//             roots' chains itself: small lattices of blocks under 128 x 32 sites, see kResolveMinBlocks,
//             and the static-scratch entry point, which has no room for the linked roots.)
//
// k_measure (every measure_every-th sweep) reduces energy and magnetisation on the device
// and accumulates E, E^2, |M| in FP64 (Lattice<2>::GetEnergyAndMagnetization,
// ising/src/lattice.cpp:29-67, and the sums of ising/src/ising_2d.cpp:127-146).
//
// Bit-exactness with the reference CPU path: the stream of tile t is seeded seed_base + t
// and consumed in the reference's order (rows' x-draws, rows' y-draws, then the merge draw
// of tx + ty numbers), the float threshold is evaluated exactly as the reference does, and
// labels are canonical (minimum site index), so bonds, labels and flipped spins match.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/swb200.h"
#include "sw_core.cuh"

namespace swb {

// ------------------------------------------------------------------------------------------
// errors and launch accounting

thread_local std::string g_last_error;
std::atomic<uint64_t> g_launches{0};

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

constexpr uint32_t kAssignThreads = 512;  // at most this many lcg lanes per block

// TXc, TYc make the tile shape a compile-time constant for the common shapes (0 = runtime).
// `dump` is all null in a plain sweep; a recorded sweep runs the same instance with dumps on
// (the tile-local stage only through the runtime-shape instance, which labels tile by tile).
// kMeasure: the instance that also measures the spins it starts from (`meas`), used by the
// sweep after a measured one; a separate instance so the others carry none of its registers.
template <int W, int TXc, int TYc, bool kMeasure, bool kFixedOnly = false>
__global__ void __launch_bounds__(kAssignThreads, 4) k_assign(const Geo g, const uint8_t *__restrict__ spins,
                                                 uint32_t *__restrict__ labels, uint32_t *__restrict__ rng_state,
                                                 uint8_t *__restrict__ rng_sel, uint32_t *__restrict__ rng_iter,
                                                 const uint32_t thr, uint32_t *__restrict__ edge, const AssignDump dump,
                                                 const MeasureArgs meas)
{
    extern __shared__ __align__(16) unsigned char smem[];
    assign_block<W, TXc, TYc, kFixedOnly, true, true, kFixedOnly>(g, blockIdx.x, blockIdx.y, spins, labels, rng_state,
                                                             rng_sel, rng_iter, thr, edge, dump,
                                                             kMeasure ? meas : MeasureArgs{}, smem);
}

__global__ void __launch_bounds__(256) k_merge(const Geo g, const uint32_t *__restrict__ edge, uint32_t *labels,
                                               unsigned int *fault, uint32_t *__restrict__ linked)
{
    merge_block(g, blockIdx.x, blockIdx.y, threadIdx.x, edge, labels, fault, linked);
}

// The linked roots of one block's merge slots (resolve_block), one thread per slot.
__global__ void __launch_bounds__(256) k_resolve(const Geo g, const uint32_t *__restrict__ linked, uint32_t *labels,
                                                 unsigned int *fault)
{
    resolve_block(g, blockIdx.x, blockIdx.y, threadIdx.x, linked, labels, fault);
}

// Resolve + flip, one CTA per block (flip_block).
// Lattices of full 128 x 32 blocks, or of at least kResolveMinBlocks blocks, resolve the
// linked roots in k_resolve; others let k_flip chase them (one launch fewer).  Measured per
// sweep on B200, chasing / resolving: 1024^2 tile 8 x 8 (512 blocks of 128 x 16, twice the
// edge sites per site) 0.0367 / 0.0380 ms; 1024^2 tile 16 x 8 (256 blocks of 128 x 32)
// 0.0356 / 0.0343 ms; 2048^2 0.0632 / 0.0598 ms; 4096^2 0.1733 / 0.1668 ms.
constexpr uint32_t kResolveMinBlocks = 4096;
constexpr uint32_t kResolveBlockSites = 128 * 32;
constexpr uint32_t kFlipThreads = 256;  // 6 CTAs per SM (40 registers), four quads of a 128 x 32 block per thread

template <bool kWriteLabels, bool kResolved>
__global__ void __launch_bounds__(kFlipThreads, 6) k_flip(const Geo g, uint8_t *__restrict__ spins, uint32_t *labels,
                                                       unsigned int *fault)
{
    extern __shared__ __align__(16) unsigned char smem[];
    flip_block<kWriteLabels, 4, kResolved>(g, blockIdx.x, blockIdx.y, spins, labels, fault, smem);
}

__global__ void __launch_bounds__(256) k_measure(const uint32_t L0, const uint32_t L1, const uint8_t *__restrict__ spins,
                                                 Obs *obs, long long *series, const unsigned long long cap,
                                                 const int accumulate)
{
    // work items: 64-site pieces of rows (row_em takes them 16 sites at a time); a thread's
    // partial sums stay far inside int range (at most 3 per site it visits)
    const size_t n = (size_t)L0 * L1;
    const uint32_t per_row = (L0 + 63) / 64, items = per_row * L1;
    int ei = 0, mi = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < items; i += gridDim.x * blockDim.x) {
        const uint32_t y = i / per_row, x0 = (i - y * per_row) * 64;
        row_em(spins, L0, L1, y, x0, min(64u, L0 - x0), ei, mi);
    }
    long long e = ei, m = mi;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        e += __shfl_xor_sync(0xffffffffu, e, o);
        m += __shfl_xor_sync(0xffffffffu, m, o);
    }
    __shared__ long long se[8], sm[8];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        se[w] = e;
        sm[w] = m;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        long long be = 0, bm = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            be += se[k];
            bm += sm[k];
        }
        obs_add_part(obs, series, cap, n, gridDim.x, be, bm, accumulate);
    }
}

// LCG32_State<W>::Init for every tile (random/src/lcg32.cpp:27-49), seeds seed_base + tile.
template <int W>
__global__ void k_rng_init(const uint32_t n_tiles, const uint32_t seed_base, uint32_t *state, uint8_t *sel,
                           uint32_t *iter)
{
    rng_init_tile<W>(n_tiles, seed_base, state, sel, iter);
}

// Hot start of Lattice<2> (ising/src/lattice.cpp:24-26): site i takes drand48 draw i + 1
// after srand48(seed); drand48() < 0.5 iff bit 47 of the 48-bit state is clear.
__global__ void k_hot_start(const size_t n, const uint32_t seed, uint8_t *spins)
{
    hot_start_chunk(n, seed, spins);
}

__global__ void k_fill(const size_t n, const uint8_t v, uint8_t *p)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        p[i] = v;
}

__global__ void k_check_spins(const size_t n, const uint8_t *p, unsigned int *bad)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (p[i] > 1)
            atomicOr(bad, 1u);
}

}  // namespace swb

// ------------------------------------------------------------------------------------------
// the handle

using namespace swb;

struct swb_lattice {
    int device = 0;
    cudaStream_t stream = nullptr;
    Geo g{};
    uint32_t W = 16, seed_base = 1, n_tiles = 0, n_blocks = 0, smem_assign = 0;
    size_t n = 0;
    uint8_t *spins = nullptr;
    uint32_t *labels = nullptr;
    uint32_t *rng_state = nullptr;
    uint8_t *rng_sel = nullptr;
    uint32_t *rng_iter = nullptr;
    uint32_t *edge = nullptr;
    uint32_t *linked = nullptr;  // merge slots: the root each edge union linked (null: flip chases)
    Obs *obs = nullptr;
    long long *series = nullptr;
    unsigned long long series_cap = 0;
    unsigned int *scratch_flag = nullptr;
    unsigned int *fault = nullptr;  // set by a chase that exceeded kChainCap
    int measure_grid = 0;
    uint32_t smem_flip = 0;
    bool spins_attached = false;   // spins point at a caller-owned device buffer (swb_attach_spins)
    bool fused_measure = false;    // the assign phase can measure the spins it starts from
    bool measure_pending = false;  // a sample of the current spins is still to be taken
};

namespace {


int set_device(const swb_lattice *h)
{
    SWB_CUDA(cudaSetDevice(h->device));
    return SWB_OK;
}

template <int W, int TXc, int TYc>
int launch_assign_k(swb_lattice *h, float p_add, const AssignDump &dump, const MeasureArgs &meas)
{
    const Geo &g = h->g;
    // Whole warps: the draws use full-warp shuffles and ballots; surplus lanes have no tile.
    const dim3 grid(g.nbx, g.nby), block((g.TBX * g.TBY * W + 31) / 32 * 32);
    if constexpr (W == 16 && TXc == 16 && TYc == 8) {
        // every block a full 128 x 32 block of 512 threads: the fixed-only instance
        if (g.BX == 128 && g.BY == 32 && g.L0 % 128 == 0 && g.L1 % 32 == 0 && block.x == 512) {
            if (meas.obs)
                k_assign<W, TXc, TYc, true, true><<<grid, block, h->smem_assign, h->stream>>>(
                    g, h->spins, h->labels, h->rng_state, h->rng_sel, h->rng_iter, accept_threshold(p_add), h->edge,
                    dump, meas);
            else
                k_assign<W, TXc, TYc, false, true><<<grid, block, h->smem_assign, h->stream>>>(
                    g, h->spins, h->labels, h->rng_state, h->rng_sel, h->rng_iter, accept_threshold(p_add), h->edge,
                    dump, meas);
            SWB_LAUNCHED();
            return SWB_OK;
        }
    }
    if (meas.obs)
        k_assign<W, TXc, TYc, true><<<grid, block, h->smem_assign, h->stream>>>(
            g, h->spins, h->labels, h->rng_state, h->rng_sel, h->rng_iter, accept_threshold(p_add), h->edge, dump, meas);
    else
        k_assign<W, TXc, TYc, false><<<grid, block, h->smem_assign, h->stream>>>(
            g, h->spins, h->labels, h->rng_state, h->rng_sel, h->rng_iter, accept_threshold(p_add), h->edge, dump, meas);
    SWB_LAUNCHED();
    return SWB_OK;
}

// The instance a plain sweep of this handle runs (compile-time tile shape for the common
// shapes), with `dump` passed through; a dump of the tile-local stage takes the runtime-shape
// instance instead, whose tile-by-tile form computes that stage.
template <int W>
int launch_assign_w(swb_lattice *h, float p_add, const AssignDump &dump, const MeasureArgs &meas)
{
    if (dump.tile_labels)
        return launch_assign_k<W, 0, 0>(h, p_add, dump, meas);
    if constexpr (W == 16) {
        const uint32_t tx = h->g.TX, ty = h->g.TY;
        if (tx == 16 && ty == 8) return launch_assign_k<W, 16, 8>(h, p_add, dump, meas);
        if (tx == 8 && ty == 8) return launch_assign_k<W, 8, 8>(h, p_add, dump, meas);
        if (tx == 32 && ty == 4) return launch_assign_k<W, 32, 4>(h, p_add, dump, meas);
        if (tx == 16 && ty == 16) return launch_assign_k<W, 16, 16>(h, p_add, dump, meas);
        if (tx == 8 && ty == 16) return launch_assign_k<W, 8, 16>(h, p_add, dump, meas);
        if (tx == 32 && ty == 8) return launch_assign_k<W, 32, 8>(h, p_add, dump, meas);
        if (tx == 16 && ty == 4) return launch_assign_k<W, 16, 4>(h, p_add, dump, meas);
    }
    return launch_assign_k<W, 0, 0>(h, p_add, dump, meas);
}

// measure: the assign phase also measures the spins it starts from (only where the block
// labelling uses bond words: fused_measure).
int launch_assign(swb_lattice *h, float p_add, const AssignDump &dump = AssignDump{}, bool measure = false)
{
    const MeasureArgs meas = measure ? MeasureArgs{h->obs, h->series, h->series_cap} : MeasureArgs{};
    switch (h->W) {
    case 8: return launch_assign_w<8>(h, p_add, dump, meas);
    case 16: return launch_assign_w<16>(h, p_add, dump, meas);
    case 32: return launch_assign_w<32>(h, p_add, dump, meas);
    }
    return fail(SWB_ERR_ARGUMENT, "unsupported lcg width %u", h->W);
}

int launch_merge(swb_lattice *h)
{
    const dim3 grid(h->g.nbx, h->g.nby);
    k_merge<<<grid, h->g.BX + h->g.BY, 0, h->stream>>>(h->g, h->edge, h->labels, h->fault, h->linked);
    SWB_LAUNCHED();
    if (h->linked) {
        k_resolve<<<grid, h->g.BX + h->g.BY, 0, h->stream>>>(h->g, h->linked, h->labels, h->fault);
        SWB_LAUNCHED();
    }
    return SWB_OK;
}

int launch_flip(swb_lattice *h, bool write_labels)
{
    const dim3 grid(h->g.nbx, h->g.nby);
    if (h->linked) {
        if (write_labels)
            k_flip<true, true><<<grid, kFlipThreads, h->smem_flip, h->stream>>>(h->g, h->spins, h->labels, h->fault);
        else
            k_flip<false, true><<<grid, kFlipThreads, h->smem_flip, h->stream>>>(h->g, h->spins, h->labels, h->fault);
    } else {
        if (write_labels)
            k_flip<true, false><<<grid, kFlipThreads, h->smem_flip, h->stream>>>(h->g, h->spins, h->labels, h->fault);
        else
            k_flip<false, false><<<grid, kFlipThreads, h->smem_flip, h->stream>>>(h->g, h->spins, h->labels, h->fault);
    }
    SWB_LAUNCHED();
    return SWB_OK;
}

int launch_sweep(swb_lattice *h, float p_add, bool write_labels, const AssignDump &dump = AssignDump{},
                 bool measure = false)
{
    if (int rc = launch_assign(h, p_add, dump, measure))
        return rc;
    if (int rc = launch_merge(h))
        return rc;
    return launch_flip(h, write_labels);
}

int launch_measure(swb_lattice *h, int accumulate)
{
    k_measure<<<h->measure_grid, 256, 0, h->stream>>>(h->g.L0, h->g.L1, h->spins, h->obs, h->series, h->series_cap,
                                                       accumulate);
    SWB_LAUNCHED();
    return SWB_OK;
}

// A measurement of the current spins that swb_sweep left for the next sweep's assign phase to
// make is made now, by k_measure: before anything reads the observables, changes the spins or
// sweeps without measuring.
int flush_measure(swb_lattice *h)
{
    if (!h->measure_pending)
        return SWB_OK;
    h->measure_pending = false;
    return launch_measure(h, 1);
}

bool valid_width(uint32_t W) { return W == 8 || W == 16 || W == 32; }

// Reads the device fault word (after the handle's work so far); non-zero means a label chase
// ran past kChainCap steps, which only corrupt labels can cause.
int check_fault(swb_lattice *h)
{
    unsigned int f = 0;
    SWB_CUDA(cudaMemcpyAsync(&f, h->fault, sizeof(f), cudaMemcpyDeviceToHost, h->stream));
    SWB_CUDA(cudaStreamSynchronize(h->stream));
    if (f)
        return fail(SWB_ERR_STATE, "label union-find fault (word %u: 1 chain over %u steps, 2 union retries, 4 label outside the lattice)", f, kChainCap);
    return SWB_OK;
}

int index_of_pair(uint32_t a, uint32_t c)
{
    for (uint32_t s = 0; s < 5; ++s)
        if (lcg_param_a(s) == a && lcg_param_c(s) == c)
            return (int)s;
    return -1;
}

// One sweep with its stages dumped to host buffers (each may be null).  tile_stage: the
// runtime-shape assign labels tile by tile and dumps the tile-local labels (the reference's
// AssignLabels stage) into `mid`; otherwise the instance a plain sweep runs dumps the labels of
// the bonds inside each block into `mid`.  Both dump the bonds, and the flip stores the
// resolved labels.
int recorded_sweep(swb_lattice *h, float temperature, bool tile_stage, uint8_t *bonds, uint32_t *mid,
                   uint32_t *labels_final)
{
    AssignDump dump{};
    if (bonds)
        SWB_CUDA(cudaMallocAsync(&dump.bonds, h->n, h->stream));
    if (mid || tile_stage)
        SWB_CUDA(cudaMallocAsync(tile_stage ? &dump.tile_labels : &dump.block_labels, h->n * sizeof(uint32_t),
                                 h->stream));
    uint32_t *d_mid = tile_stage ? dump.tile_labels : dump.block_labels;
    int rc = launch_sweep(h, swb_p_add(temperature), true, dump);
    if (rc == SWB_OK) {
        if (bonds)
            SWB_CUDA(cudaMemcpyAsync(bonds, dump.bonds, h->n, cudaMemcpyDeviceToHost, h->stream));
        if (mid)
            SWB_CUDA(cudaMemcpyAsync(mid, d_mid, h->n * 4, cudaMemcpyDeviceToHost, h->stream));
        if (labels_final)
            SWB_CUDA(cudaMemcpyAsync(labels_final, h->labels, h->n * 4, cudaMemcpyDeviceToHost, h->stream));
    }
    if (dump.bonds)
        cudaFreeAsync(dump.bonds, h->stream);
    if (d_mid)
        cudaFreeAsync(d_mid, h->stream);
    SWB_CUDA(cudaStreamSynchronize(h->stream));
    return rc ? rc : check_fault(h);
}

}  // namespace

extern "C" {

const char *swb_version(void) { return "swb200 0.1 (sm_100a)"; }

int swb_device_count(int *count)
{
    if (!count)
        return fail(SWB_ERR_ARGUMENT, "count is NULL");
    *count = 0;
    const cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) {
        *count = 0;
        cudaGetLastError();
    }
    return SWB_OK;
}

const char *swb_last_error(void) { return g_last_error.c_str(); }

uint64_t swb_kernel_launches(void) { return g_launches.load(); }

float swb_p_add(float temperature) { return 1.0f - static_cast<float>(std::exp(-2.0f / temperature)); }

uint32_t swb_accept_threshold(float p_add) { return accept_threshold(p_add); }

int swb_create(swb_lattice **out, uint32_t L0, uint32_t L1, uint32_t tile_x, uint32_t tile_y, uint32_t lcg_width,
               uint32_t seed_base, int device)
{
    if (!out)
        return fail(SWB_ERR_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (L0 == 0 || L1 == 0 || (L0 % 2) || (L1 % 2))
        return fail(SWB_ERR_ARGUMENT, "SwendsenWang_2D implementation requires evenly sized lattice (%u x %u)", L0, L1);
    if ((uint64_t)L0 * L1 > 0x7FFFFFFFull)
        return fail(SWB_ERR_ARGUMENT, "lattice of %u x %u sites exceeds 2^31 - 1 labels", L0, L1);
    if (!(tile_x == 8 || tile_x == 16 || tile_x == 32) || tile_y < 2 || tile_y > 32)
        return fail(SWB_ERR_ARGUMENT, "unsupported tile %u x %u (tile_x in {8,16,32}, 2 <= tile_y <= 32)", tile_x, tile_y);
    if (!valid_width(lcg_width))
        return fail(SWB_ERR_ARGUMENT, "unsupported lcg32 width %u (8, 16 or 32)", lcg_width);
    if (make_geo(L0, L1, tile_x, tile_y, lcg_width, kAssignThreads).nby > kMaxGridY)
        return fail(SWB_ERR_ARGUMENT, "lattice of %u rows needs more than %u block rows", L1, kMaxGridY);
    swb_lattice *h = new swb_lattice();
    h->device = device;
    h->W = lcg_width;
    h->seed_base = seed_base;
    h->g = make_geo(L0, L1, tile_x, tile_y, lcg_width, kAssignThreads);
    h->n = (size_t)L0 * L1;
    h->n_tiles = h->g.n0 * h->g.n1;
    h->n_blocks = h->g.nbx * h->g.nby;
    h->smem_assign = assign_smem(h->g, h->W).total;
    auto cleanup = [&](int rc) {
        swb_destroy(h);
        return rc;
    };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess)
        return cleanup(fail(SWB_ERR_CUDA, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e)));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
#define SWB_TRY(call)                                                                                \
    do {                                                                                             \
        cudaError_t err__ = (call);                                                                  \
        if (err__ != cudaSuccess)                                                                    \
            return cleanup(fail(SWB_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(err__)));   \
    } while (0)
    SWB_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    SWB_TRY(cudaMalloc(&h->spins, h->n + 16));
    SWB_TRY(cudaMalloc(&h->labels, h->n * sizeof(uint32_t) + 16));
    SWB_TRY(cudaMalloc(&h->rng_state, (size_t)h->n_tiles * h->W * sizeof(uint32_t)));
    SWB_TRY(cudaMalloc(&h->rng_sel, (size_t)h->n_tiles * h->W));
    SWB_TRY(cudaMalloc(&h->rng_iter, (size_t)h->n_tiles * sizeof(uint32_t)));
    SWB_TRY(cudaMalloc(&h->edge, (size_t)h->n_blocks * kEdgeWords * sizeof(uint32_t)));
    bool resolve = h->n_blocks >= kResolveMinBlocks || h->g.BX * h->g.BY >= kResolveBlockSites;
    if (const char *e = std::getenv("SWB_RESOLVE_MIN_BLOCKS"))
        resolve = h->n_blocks >= (uint32_t)std::strtoul(e, nullptr, 10);
    if (resolve)
        SWB_TRY(cudaMalloc(&h->linked, (size_t)h->n_blocks * (h->g.BX + h->g.BY) * sizeof(uint32_t)));
    SWB_TRY(cudaMalloc(&h->obs, sizeof(Obs)));
    h->series_cap = 1ull << 17;  // 131072 measurements (2 MiB)
    SWB_TRY(cudaMalloc(&h->series, h->series_cap * 2 * sizeof(long long)));
    SWB_TRY(cudaMalloc(&h->scratch_flag, sizeof(unsigned int)));
    SWB_TRY(cudaMalloc(&h->fault, sizeof(unsigned int)));
    SWB_TRY(cudaMemsetAsync(h->fault, 0, sizeof(unsigned int), h->stream));
    SWB_TRY(cudaMemsetAsync(h->spins, 0, h->n + 16, h->stream));
    SWB_TRY(cudaMemsetAsync(h->obs, 0, sizeof(Obs), h->stream));
    h->smem_flip = flip_smem_bytes(h->g);
    h->fused_measure = (h->g.BX & 31u) == 0 && (h->g.BX & (h->g.BX - 1)) == 0;  // the bond-word labelling
    h->measure_grid = (int)std::min<size_t>((h->n + 255) / 256, (size_t)sms * 8);
    if (h->measure_grid < 1) h->measure_grid = 1;
    switch (h->W) {
    case 8: k_rng_init<8><<<(h->n_tiles + 127) / 128, 128, 0, h->stream>>>(h->n_tiles, seed_base, h->rng_state, h->rng_sel, h->rng_iter); break;
    case 16: k_rng_init<16><<<(h->n_tiles + 127) / 128, 128, 0, h->stream>>>(h->n_tiles, seed_base, h->rng_state, h->rng_sel, h->rng_iter); break;
    default: k_rng_init<32><<<(h->n_tiles + 127) / 128, 128, 0, h->stream>>>(h->n_tiles, seed_base, h->rng_state, h->rng_sel, h->rng_iter); break;
    }
    g_launches.fetch_add(1);
    SWB_TRY(cudaGetLastError());
    SWB_TRY(cudaStreamSynchronize(h->stream));
#undef SWB_TRY
    *out = h;
    return SWB_OK;
}

int swb_destroy(swb_lattice *h)
{
    if (!h)
        return SWB_OK;
    cudaSetDevice(h->device);
    if (h->stream)
        cudaStreamSynchronize(h->stream);
    if (!h->spins_attached)
        cudaFree(h->spins);
    cudaFree(h->labels);
    cudaFree(h->rng_state);
    cudaFree(h->rng_sel);
    cudaFree(h->rng_iter);
    cudaFree(h->edge);
    cudaFree(h->linked);
    cudaFree(h->obs);
    cudaFree(h->series);
    cudaFree(h->scratch_flag);
    cudaFree(h->fault);
    if (h->stream)
        cudaStreamDestroy(h->stream);
    delete h;
    return SWB_OK;
}

int swb_set_spins(swb_lattice *h, const uint8_t *host_spins)
{
    if (!h || !host_spins)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (int rc = set_device(h))
        return rc;
    if (int rc = flush_measure(h))
        return rc;
    SWB_CUDA(cudaMemcpyAsync(h->spins, host_spins, h->n, cudaMemcpyHostToDevice, h->stream));
    SWB_CUDA(cudaMemsetAsync(h->scratch_flag, 0, sizeof(unsigned int), h->stream));
    k_check_spins<<<h->measure_grid, 256, 0, h->stream>>>(h->n, h->spins, h->scratch_flag);
    SWB_LAUNCHED();
    unsigned int bad = 0;
    SWB_CUDA(cudaMemcpyAsync(&bad, h->scratch_flag, sizeof(bad), cudaMemcpyDeviceToHost, h->stream));
    SWB_CUDA(cudaStreamSynchronize(h->stream));
    if (bad)
        return fail(SWB_ERR_ARGUMENT, "spins must be 0 or 1");
    return SWB_OK;
}

int swb_get_spins(swb_lattice *h, uint8_t *host_spins)
{
    if (!h || !host_spins)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (int rc = set_device(h))
        return rc;
    SWB_CUDA(cudaMemcpyAsync(host_spins, h->spins, h->n, cudaMemcpyDeviceToHost, h->stream));
    SWB_CUDA(cudaStreamSynchronize(h->stream));
    return check_fault(h);
}

int swb_hot_start(swb_lattice *h, uint32_t seed)
{
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "NULL handle");
    if (int rc = set_device(h))
        return rc;
    if (int rc = flush_measure(h))
        return rc;
    const size_t chunks = (h->n + 63) / 64;
    k_hot_start<<<(unsigned)((chunks + 255) / 256), 256, 0, h->stream>>>(h->n, seed, h->spins);
    SWB_LAUNCHED();
    return SWB_OK;
}

int swb_cold_start(swb_lattice *h, uint8_t value)
{
    if (!h || value > 1)
        return fail(SWB_ERR_ARGUMENT, "cold start value must be 0 or 1");
    if (int rc = set_device(h))
        return rc;
    if (int rc = flush_measure(h))
        return rc;
    k_fill<<<h->measure_grid, 256, 0, h->stream>>>(h->n, value, h->spins);
    SWB_LAUNCHED();
    return SWB_OK;
}

int swb_sweep(swb_lattice *h, float temperature, uint32_t n_sweeps, uint32_t measure_every)
{
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "NULL handle");
    if (!(temperature > 0.0f) || !std::isfinite(temperature))
        return fail(SWB_ERR_ARGUMENT, "temperature must be positive and finite");
    if (int rc = set_device(h))
        return rc;
    const float p_add = swb_p_add(temperature);
    for (uint32_t s = 1; s <= n_sweeps; ++s) {
        // A pending sample of the spins this sweep starts from is taken by its assign phase
        // (no extra pass over the spins), else by k_measure before the sweep.
        const bool fused = h->measure_pending && h->fused_measure;
        if (!fused)
            if (int rc = flush_measure(h))
                return rc;
        h->measure_pending = false;
        if (int rc = launch_sweep(h, p_add, false, AssignDump{}, fused))
            return rc;
        if (measure_every && (s % measure_every) == 0)
            h->measure_pending = true;
    }
    return SWB_OK;
}

int swb_sweep_recorded(swb_lattice *h, float temperature, uint8_t *bonds, uint32_t *labels_assign,
                       uint32_t *labels_final)
{
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "NULL handle");
    if (!(temperature > 0.0f) || !std::isfinite(temperature))
        return fail(SWB_ERR_ARGUMENT, "temperature must be positive and finite");
    if (int rc = set_device(h))
        return rc;
    if (int rc = flush_measure(h))
        return rc;
    return recorded_sweep(h, temperature, true, bonds, labels_assign, labels_final);
}

int swb_sweep_dumped(swb_lattice *h, float temperature, uint8_t *bonds, uint32_t *labels_block,
                     uint32_t *labels_final)
{
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "NULL handle");
    if (!(temperature > 0.0f) || !std::isfinite(temperature))
        return fail(SWB_ERR_ARGUMENT, "temperature must be positive and finite");
    if (int rc = set_device(h))
        return rc;
    if (int rc = flush_measure(h))
        return rc;
    return recorded_sweep(h, temperature, false, bonds, labels_block, labels_final);
}

int swb_geometry(swb_lattice *h, uint32_t *geometry)
{
    if (!h || !geometry)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    const Geo &g = h->g;
    const uint32_t v[8] = {g.L0, g.L1, g.TX, g.TY, g.BX, g.BY, g.nbx, g.nby};
    std::memcpy(geometry, v, sizeof(v));
    return SWB_OK;
}

int swb_synchronize(swb_lattice *h)
{
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "NULL handle");
    if (int rc = set_device(h))
        return rc;
    SWB_CUDA(cudaStreamSynchronize(h->stream));
    return check_fault(h);
}

int swb_energy_magnetization(swb_lattice *h, double *out, int64_t *e_sum, int64_t *m_sum)
{
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "NULL handle");
    if (int rc = set_device(h))
        return rc;
    if (int rc = flush_measure(h))
        return rc;
    if (int rc = launch_measure(h, 0))
        return rc;
    Obs o;
    SWB_CUDA(cudaMemcpyAsync(&o, h->obs, sizeof(Obs), cudaMemcpyDeviceToHost, h->stream));
    SWB_CUDA(cudaStreamSynchronize(h->stream));
    if (out) {
        out[0] = -(double)o.last_e / (double)h->n;
        out[1] = (double)o.last_m / (double)h->n;
    }
    if (e_sum) *e_sum = o.last_e;
    if (m_sum) *m_sum = o.last_m;
    return SWB_OK;
}

int swb_accumulators(swb_lattice *h, double *out)
{
    if (!h || !out)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (int rc = set_device(h))
        return rc;
    if (int rc = flush_measure(h))
        return rc;
    Obs o;
    SWB_CUDA(cudaMemcpyAsync(&o, h->obs, sizeof(Obs), cudaMemcpyDeviceToHost, h->stream));
    SWB_CUDA(cudaStreamSynchronize(h->stream));
    std::memcpy(out, o.acc, sizeof(o.acc));
    return SWB_OK;
}

int swb_reset_accumulators(swb_lattice *h)
{
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "NULL handle");
    if (int rc = set_device(h))
        return rc;
    h->measure_pending = false;  // a sample requested before the reset is dropped with the others
    SWB_CUDA(cudaMemsetAsync(h->obs, 0, sizeof(Obs), h->stream));
    return SWB_OK;
}

int swb_samples(swb_lattice *h, int64_t *em, uint64_t capacity, uint64_t *count)
{
    if (!h || !count)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (int rc = set_device(h))
        return rc;
    if (int rc = flush_measure(h))
        return rc;
    Obs o;
    SWB_CUDA(cudaMemcpyAsync(&o, h->obs, sizeof(Obs), cudaMemcpyDeviceToHost, h->stream));
    SWB_CUDA(cudaStreamSynchronize(h->stream));
    *count = o.n_samples;
    if (o.n_samples > h->series_cap)
        return fail(SWB_ERR_CAPACITY, "%llu samples recorded, series keeps %llu", o.n_samples, h->series_cap);
    const uint64_t k = o.n_samples < capacity ? o.n_samples : capacity;
    if (k && em) {
        SWB_CUDA(cudaMemcpyAsync(em, h->series, k * 2 * sizeof(long long), cudaMemcpyDeviceToHost, h->stream));
        SWB_CUDA(cudaStreamSynchronize(h->stream));
    }
    return SWB_OK;
}

int swb_rng_shape(swb_lattice *h, uint32_t *n_tiles, uint32_t *lcg_width)
{
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "NULL handle");
    if (n_tiles) *n_tiles = h->n_tiles;
    if (lcg_width) *lcg_width = h->W;
    return SWB_OK;
}

int swb_get_rng(swb_lattice *h, uint32_t *state, uint32_t *a, uint32_t *c, uint32_t *iteration)
{
    if (!h || !state || !a || !c || !iteration)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (int rc = set_device(h))
        return rc;
    const size_t nw = (size_t)h->n_tiles * h->W;
    std::vector<uint8_t> sel(nw);
    SWB_CUDA(cudaMemcpyAsync(state, h->rng_state, nw * 4, cudaMemcpyDeviceToHost, h->stream));
    SWB_CUDA(cudaMemcpyAsync(sel.data(), h->rng_sel, nw, cudaMemcpyDeviceToHost, h->stream));
    SWB_CUDA(cudaMemcpyAsync(iteration, h->rng_iter, (size_t)h->n_tiles * 4, cudaMemcpyDeviceToHost, h->stream));
    SWB_CUDA(cudaStreamSynchronize(h->stream));
    for (size_t i = 0; i < nw; ++i) {
        a[i] = lcg_param_a(sel[i]);
        c[i] = lcg_param_c(sel[i]);
    }
    return SWB_OK;
}

int swb_set_rng(swb_lattice *h, const uint32_t *state, const uint32_t *a, const uint32_t *c,
                const uint32_t *iteration)
{
    if (!h || !state || !a || !c || !iteration)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (int rc = set_device(h))
        return rc;
    const size_t nw = (size_t)h->n_tiles * h->W;
    std::vector<uint8_t> sel(nw);
    for (size_t i = 0; i < nw; ++i) {
        const int s = index_of_pair(a[i], c[i]);
        if (s < 0)
            return fail(SWB_ERR_ARGUMENT, "lane %zu: (a, c) = (%u, %u) is not an lcg32 parameter pair", i, a[i], c[i]);
        sel[i] = (uint8_t)s;
    }
    SWB_CUDA(cudaMemcpyAsync(h->rng_state, state, nw * 4, cudaMemcpyHostToDevice, h->stream));
    SWB_CUDA(cudaMemcpyAsync(h->rng_sel, sel.data(), nw, cudaMemcpyHostToDevice, h->stream));
    SWB_CUDA(cudaMemcpyAsync(h->rng_iter, iteration, (size_t)h->n_tiles * 4, cudaMemcpyHostToDevice, h->stream));
    SWB_CUDA(cudaStreamSynchronize(h->stream));
    return SWB_OK;
}

int swb_device_buffers(swb_lattice *h, void **spins, void **labels)
{
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "NULL handle");
    if (int rc = set_device(h))
        return rc;
    if (int rc = flush_measure(h))  // the caller may change the spins through the pointer
        return rc;
    if (spins) *spins = h->spins;
    if (labels) *labels = h->labels;
    return SWB_OK;
}

int swb_launches_per_sweep(swb_lattice *h, uint32_t *launches)
{
    if (!h || !launches)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    *launches = h->linked ? 4 : 3;
    return SWB_OK;
}

int swb_sweep_timed(swb_lattice *h, float temperature, uint32_t n_sweeps, int per_kernel, float *ms)
{
    if (!h || !ms)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (!(temperature > 0.0f) || !std::isfinite(temperature))
        return fail(SWB_ERR_ARGUMENT, "temperature must be positive and finite");
    if (int rc = set_device(h))
        return rc;
    if (int rc = flush_measure(h))
        return rc;
    const float p_add = swb_p_add(temperature);
    ms[0] = ms[1] = ms[2] = ms[3] = 0.0f;
    cudaEvent_t ev[5];
    for (auto &e : ev)
        SWB_CUDA(cudaEventCreate(&e));
    int rc = SWB_OK;
    SWB_CUDA(cudaEventRecord(ev[0], h->stream));
    for (uint32_t s = 0; s < n_sweeps && rc == SWB_OK; ++s) {
        if (!per_kernel) {
            rc = launch_sweep(h, p_add, false);
            continue;
        }
        SWB_CUDA(cudaEventRecord(ev[1], h->stream));
        if ((rc = launch_assign(h, p_add)))
            break;
        SWB_CUDA(cudaEventRecord(ev[2], h->stream));
        k_merge<<<dim3(h->g.nbx, h->g.nby), h->g.BX + h->g.BY, 0, h->stream>>>(h->g, h->edge, h->labels, h->fault,
                                                                               h->linked);
        SWB_LAUNCHED();
        SWB_CUDA(cudaEventRecord(ev[3], h->stream));
        // resolve + flip: the reference's ResolveLabels and FlipClusters
        if (h->linked) {
            k_resolve<<<dim3(h->g.nbx, h->g.nby), h->g.BX + h->g.BY, 0, h->stream>>>(h->g, h->linked, h->labels,
                                                                                     h->fault);
            SWB_LAUNCHED();
        }
        if ((rc = launch_flip(h, false)))
            break;
        SWB_CUDA(cudaEventRecord(ev[4], h->stream));
        SWB_CUDA(cudaEventSynchronize(ev[4]));
        float t;
        SWB_CUDA(cudaEventElapsedTime(&t, ev[1], ev[2]));
        ms[1] += t;
        SWB_CUDA(cudaEventElapsedTime(&t, ev[2], ev[3]));
        ms[2] += t;
        SWB_CUDA(cudaEventElapsedTime(&t, ev[3], ev[4]));
        ms[3] += t;
    }
    SWB_CUDA(cudaEventRecord(ev[4], h->stream));
    SWB_CUDA(cudaEventSynchronize(ev[4]));
    SWB_CUDA(cudaEventElapsedTime(&ms[0], ev[0], ev[4]));
    for (auto &e : ev)
        cudaEventDestroy(e);
    return rc ? rc : check_fault(h);
}

int swb_attach_spins(swb_lattice *h, void *device_spins)
{
    if (!h || !device_spins)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (reinterpret_cast<uintptr_t>(device_spins) % 16)
        return fail(SWB_ERR_ARGUMENT, "device spins must be 16-byte aligned");
    if (int rc = set_device(h))
        return rc;
    cudaPointerAttributes at{};
    SWB_CUDA(cudaPointerGetAttributes(&at, device_spins));
    if (at.type != cudaMemoryTypeDevice || at.device != h->device)
        return fail(SWB_ERR_ARGUMENT, "spins are not device memory of CUDA device %d", h->device);
    if (int rc = flush_measure(h))
        return rc;
    SWB_CUDA(cudaStreamSynchronize(h->stream));
    if (!h->spins_attached)
        SWB_CUDA(cudaFree(h->spins));
    h->spins = static_cast<uint8_t *>(device_spins);
    h->spins_attached = true;
    return SWB_OK;
}

int swb_device_alloc(int device, size_t bytes, void **ptr)
{
    if (!ptr)
        return fail(SWB_ERR_ARGUMENT, "ptr is NULL");
    *ptr = nullptr;
    SWB_CUDA(cudaSetDevice(device));
    SWB_CUDA(cudaMalloc(ptr, bytes + 16));  // 256-byte aligned; 16 bytes of slack for vector accesses
    return SWB_OK;
}

int swb_device_free(int device, void *ptr)
{
    if (!ptr)
        return SWB_OK;
    SWB_CUDA(cudaSetDevice(device));
    SWB_CUDA(cudaFree(ptr));
    return SWB_OK;
}

int swb_copy_to_device(int device, void *dst, const void *src, size_t bytes)
{
    if ((!dst || !src) && bytes)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    SWB_CUDA(cudaSetDevice(device));
    SWB_CUDA(cudaDeviceSynchronize());  // the engine's streams do not order against this copy
    SWB_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
    SWB_CUDA(cudaDeviceSynchronize());  // a copy from pageable memory may return before it lands
    return SWB_OK;
}

int swb_copy_to_host(int device, void *dst, const void *src, size_t bytes)
{
    if ((!dst || !src) && bytes)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    SWB_CUDA(cudaSetDevice(device));
    SWB_CUDA(cudaDeviceSynchronize());  // the engine's streams do not order against this copy
    SWB_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
    return SWB_OK;
}

int swb_device_synchronize(int device)
{
    SWB_CUDA(cudaSetDevice(device));
    SWB_CUDA(cudaDeviceSynchronize());
    return SWB_OK;
}

int swb_device_sm_count(int device, uint32_t *count)
{
    if (!count)
        return fail(SWB_ERR_ARGUMENT, "count is NULL");
    int v = 0;
    SWB_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device));
    *count = (uint32_t)v;
    return SWB_OK;
}

int swb_spins_energy_magnetization(int device, uint32_t L0, uint32_t L1, const void *device_spins, double *out,
                                   int64_t *e_sum, int64_t *m_sum)
{
    if (!device_spins || L0 == 0 || L1 == 0)
        return fail(SWB_ERR_ARGUMENT, "NULL spins or empty lattice");
    // One small accumulator per device, kept until exit; calls on a device are serialised.
    static std::mutex mu;
    static std::vector<Obs *> acc;
    std::lock_guard<std::mutex> lock(mu);
    SWB_CUDA(cudaSetDevice(device));
    SWB_CUDA(cudaDeviceSynchronize());  // every sweep queued on the engine's streams comes first
    if ((int)acc.size() <= device)
        acc.resize(device + 1, nullptr);
    if (!acc[device]) {
        SWB_CUDA(cudaMalloc(&acc[device], sizeof(Obs)));
        SWB_CUDA(cudaMemset(acc[device], 0, sizeof(Obs)));
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const size_t n = (size_t)L0 * L1;
    const int grid = (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)sms * 8));
    k_measure<<<grid, 256>>>(L0, L1, static_cast<const uint8_t *>(device_spins), acc[device], nullptr, 0, 0);
    SWB_LAUNCHED();
    Obs o;
    SWB_CUDA(cudaMemcpy(&o, acc[device], sizeof(Obs), cudaMemcpyDeviceToHost));
    if (out) {
        out[0] = -(double)o.last_e / (double)n;
        out[1] = (double)o.last_m / (double)n;
    }
    if (e_sum) *e_sum = o.last_e;
    if (m_sum) *m_sum = o.last_m;
    return SWB_OK;
}

int swb_host_alloc(void **ptr, size_t bytes)
{
    if (!ptr)
        return fail(SWB_ERR_ARGUMENT, "ptr is NULL");
    SWB_CUDA(cudaHostAlloc(ptr, bytes ? bytes : 1, cudaHostAllocDefault));
    return SWB_OK;
}

int swb_host_free(void *ptr)
{
    if (ptr)
        SWB_CUDA(cudaFreeHost(ptr));
    return SWB_OK;
}

int swb_update_host(swb_lattice *h, float temperature, const uint8_t *spins_in, uint8_t *spins_out, double *em_out)
{
    if (!h || !spins_in || !spins_out)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (!(temperature > 0.0f) || !std::isfinite(temperature))
        return fail(SWB_ERR_ARGUMENT, "temperature must be positive and finite");
    if (int rc = set_device(h))
        return rc;
    if (int rc = flush_measure(h))
        return rc;
    SWB_CUDA(cudaMemcpyAsync(h->spins, spins_in, h->n, cudaMemcpyHostToDevice, h->stream));
    if (int rc = launch_sweep(h, swb_p_add(temperature), false))
        return rc;
    SWB_CUDA(cudaMemcpyAsync(spins_out, h->spins, h->n, cudaMemcpyDeviceToHost, h->stream));
    if (em_out) {
        if (int rc = launch_measure(h, 0))
            return rc;
        Obs o;
        SWB_CUDA(cudaMemcpyAsync(&o, h->obs, sizeof(Obs), cudaMemcpyDeviceToHost, h->stream));
        SWB_CUDA(cudaStreamSynchronize(h->stream));
        em_out[0] = -(double)o.last_e / (double)h->n;
        em_out[1] = (double)o.last_m / (double)h->n;
    }
    SWB_CUDA(cudaStreamSynchronize(h->stream));
    return SWB_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Sweeps that allocate nothing.
//
// Who cannot allocate: a host that keeps the lattice in device memory it manages itself -- the
// reference's Lattice<2> storage handed over through an FFI, or a serving process whose lattice
// pool already holds its whole HBM budget.  For such a caller a per-sweep cudaMalloc can fail
// (the pool has the memory) and a cudaFree synchronises the whole device, stalling the other
// lattices' streams.  The caller passes its spins and lcg32 streams; the sweep's scratch (label
// array, block edge words, fault word) lives in one file-scope device array (sw_static_scratch.cu), which
// every call on a device shares.

namespace swb {

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace swb

extern "C" {

int swb_sweep_static(void *stream, uint32_t L0, uint32_t L1, uint32_t tile_x, uint32_t tile_y, uint32_t lcg_width,
                     float temperature, uint32_t n_sweeps, uint8_t *spins, uint32_t *rng_state, uint8_t *rng_sel,
                     uint32_t *rng_iter, int wait)
{
    // Every argument is checked before the first CUDA call.
    if (!spins || !rng_state || !rng_sel || !rng_iter)
        return fail(SWB_ERR_ARGUMENT, "NULL buffer");
    if (reinterpret_cast<uintptr_t>(spins) % 16 || reinterpret_cast<uintptr_t>(rng_state) % 4 ||
        reinterpret_cast<uintptr_t>(rng_iter) % 4)
        return fail(SWB_ERR_ARGUMENT, "spins must be 16-byte aligned, rng_state and rng_iter 4-byte aligned");
    if (L0 == 0 || L1 == 0 || (L0 % 2) || (L1 % 2))
        return fail(SWB_ERR_ARGUMENT, "SwendsenWang_2D implementation requires evenly sized lattice (%u x %u)", L0, L1);
    if ((uint64_t)L0 * L1 > kStaticMaxSites)
        return fail(SWB_ERR_CAPACITY, "lattice of %u x %u sites exceeds the static scratch limit of %llu sites", L0, L1,
                    (unsigned long long)kStaticMaxSites);
    if (!(tile_x == 8 || tile_x == 16 || tile_x == 32) || tile_y < 2 || tile_y > 32)
        return fail(SWB_ERR_ARGUMENT, "unsupported tile %u x %u (tile_x in {8,16,32}, 2 <= tile_y <= 32)", tile_x, tile_y);
    if (!valid_width(lcg_width))
        return fail(SWB_ERR_ARGUMENT, "unsupported lcg32 width %u (8, 16 or 32)", lcg_width);
    if (!(temperature > 0.0f) || !std::isfinite(temperature))
        return fail(SWB_ERR_ARGUMENT, "temperature must be positive and finite");
    if (make_geo(L0, L1, tile_x, tile_y, lcg_width, kAssignThreads).nby > kMaxGridY)
        return fail(SWB_ERR_ARGUMENT, "lattice of %u rows needs more than %u block rows", L1, kMaxGridY);

    swb_lattice h;  // a view: caller's buffers plus the static scratch; owns nothing
    h.stream = static_cast<cudaStream_t>(stream);
    h.W = lcg_width;
    h.g = make_geo(L0, L1, tile_x, tile_y, lcg_width, kAssignThreads);
    h.n = (size_t)L0 * L1;
    h.n_tiles = h.g.n0 * h.g.n1;
    h.n_blocks = h.g.nbx * h.g.nby;
    h.smem_assign = assign_smem(h.g, h.W).total;
    h.smem_flip = flip_smem_bytes(h.g);
    const size_t labels_bytes = align256(h.n * sizeof(uint32_t) + 16);
    const size_t edge_bytes = align256((size_t)h.n_blocks * kEdgeWords * sizeof(uint32_t));
    if (labels_bytes + edge_bytes + 256 > kStaticScratchBytes)
        return fail(SWB_ERR_CAPACITY, "lattice %u x %u with tile %u x %u needs %zu bytes of scratch, the static array holds %zu",
                    L0, L1, tile_x, tile_y, labels_bytes + edge_bytes + 256, kStaticScratchBytes);

    SWB_CUDA(cudaGetDevice(&h.device));
    unsigned char *base = nullptr;
    if (int rc = static_scratch_base(h.device, &base))
        return rc;
    h.spins = spins;
    h.rng_state = rng_state;
    h.rng_sel = rng_sel;
    h.rng_iter = rng_iter;
    h.labels = reinterpret_cast<uint32_t *>(base);
    h.edge = reinterpret_cast<uint32_t *>(base + labels_bytes);
    h.fault = reinterpret_cast<unsigned int *>(base + labels_bytes + edge_bytes);

    // The array keeps the previous call's contents.  Labels and edge words are fully written by
    // the assign kernel before they are read; only the fault word must start at zero.
    SWB_CUDA(cudaMemsetAsync(h.fault, 0, sizeof(unsigned int), h.stream));
    const float p_add = swb_p_add(temperature);
    for (uint32_t s = 0; s < n_sweeps; ++s)
        if (int rc = launch_sweep(&h, p_add, false))
            return rc;
    if (wait) {
        unsigned int f = 0;
        SWB_CUDA(cudaMemcpyAsync(&f, h.fault, sizeof(f), cudaMemcpyDeviceToHost, h.stream));
        SWB_CUDA(cudaStreamSynchronize(h.stream));
        if (f)
            return fail(SWB_ERR_STATE, "label union-find fault (word %u: 1 chain over %u steps, 2 union retries, 4 label outside the lattice)", f, kChainCap);
    }
    return SWB_OK;
}

}  // extern "C"
