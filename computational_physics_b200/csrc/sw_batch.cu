// Batched Swendsen-Wang: hundreds of independent periodic lattices of different sizes,
// tiles and temperatures advance together, one kernel launch per sweep phase for all of them.
//
// Work items.  Every active lattice contributes its blocks (TBX x TBY tiles) to one flat list
// of block items (lattice slot, block coordinates), big lattices first.  kb_assign, kb_merge,
// kb_resolve and kb_flip run one CTA per item (a CTA takes items blockIdx.x, blockIdx.x + gridDim.x, ...,
// loading the next item's descriptor while it works on the current one, so a smaller grid
// also covers the list); kb_measure pulls chunks of 4096 sites from a device counter
// (atomicAdd), which kb_assign resets.  A sweep needs no host work and is one CUDA graph: the
// lattices split into two groups whose phase kernels run on two streams side by side; the
// graph is captured once and replayed, and captured again when the lattice set changes.
//
// Per lattice the device keeps spins, labels, lcg32 streams (one per tile, seeded
// seed_base + tile id as the reference's CPU path with one stream per tile), a sweep budget
// (sweeps_left, decremented on the device; lattices at 0 are skipped) and FP64 observable
// accumulators, so jobs with different sweep counts share the same graph replays.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "sw_core.cuh"

namespace swb {

constexpr uint32_t kBatchThreads = 512;        // CTA size of the assign kernel
constexpr uint32_t kMeasureThreads = 256;      // measure: one thread per 16 sites of a 4096-site chunk
constexpr uint32_t kMergeThreads = 160;        // merge, resolve: one thread per block edge site (BX + BY <= 160)
constexpr uint32_t kFlipThreads = 256;         // flip: four quads of a 128 x 32 block per thread
constexpr uint32_t kChunkSites = 4096;         // measure work item
constexpr uint32_t kRoundGroups = 2;           // lattice groups whose sweeps run side by side in a round
constexpr uint32_t kUnlimited = 0xFFFFFFFFu;   // sweeps_left value that never runs out

struct BatchLat {
    Geo g;
    uint8_t *spins;
    uint32_t *labels;
    uint32_t *rng_state;
    uint8_t *rng_sel;
    uint32_t *rng_iter;
    uint32_t *edge;
    uint32_t *linked;         // merge slots: the root each edge union linked
    Obs *obs;
    long long *series;
    unsigned long long series_cap;
    uint32_t thr;             // bond accept threshold, accept_threshold(p_add)
    uint32_t sweeps_left;     // sweeps still to run (kUnlimited: no limit)
    uint32_t swept;           // 1 if this lattice was swept in the current round
    uint32_t measure_every;   // measure after every measure_every-th sweep (0: never)
    uint32_t sweeps_done;     // sweeps completed
    uint32_t measure_base;    // first entry of this lattice's chunks in the round's measure list
};

struct BatchCounters {
    unsigned int measure_next;    // next entry of the measure list (device work counter)
    unsigned int n_active;        // lattices in the work lists
    unsigned int total_chunks;    // measure chunks of all active lattices (the list's capacity)
    unsigned int measure_chunks;  // entries of this round's measure list
};

__device__ __forceinline__ uint32_t next_item(unsigned int *queue, uint32_t *slot)
{
    if (threadIdx.x == 0)
        *slot = atomicAdd(queue, 1u);
    __syncthreads();
    const uint32_t item = *slot;
    __syncthreads();
    return item;
}

// Item k of the flat block list: x = lattice slot, y = byi << 16 | bxi.
__device__ __forceinline__ uint2 load_item(const uint2 *items, uint32_t k, uint32_t total)
{
    return k < total ? items[k] : make_uint2(0, 0);
}

// A block item with what its merge, resolve and flip need, kept beside the item list: those
// kernels start their data loads after one dependent load (the record) instead of two (the
// item, then its lattice's descriptor), and read the lattice's budget in parallel (512-lattice
// mix: resolve + flip 0.083 -> 0.072 ms per round).
struct alignas(16) BlockRec {
    uint32_t lat, bxy, L0, L1;     // lattice slot, byi << 16 | bxi, extent
    uint32_t bxby, nbx, nby, pad;  // BX | BY << 16, blocks per direction
    uint8_t *spins;
    uint32_t *labels;
    uint32_t *edge;
    uint32_t *linked;
};
static_assert(sizeof(BlockRec) == 64, "four 16-byte loads");

__device__ __forceinline__ Geo rec_geo(const BlockRec &r)
{
    Geo g{};
    g.L0 = r.L0;
    g.L1 = r.L1;
    g.BX = r.bxby & 0xFFFFu;
    g.BY = r.bxby >> 16;
    g.nbx = r.nbx;
    g.nby = r.nby;
    return g;
}

template <int W, bool kAllShapes>
__global__ void __launch_bounds__(kBatchThreads, 4) kb_assign(BatchLat *lats, const uint2 *items, const uint32_t total,
                                                              BatchCounters *ctr)
{
    extern __shared__ __align__(16) unsigned char smem[];
    uint2 d = load_item(items, blockIdx.x, total);
    for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
        const uint2 next = load_item(items, item + gridDim.x, total);
        const BatchLat *L = lats + d.x;
        if (L->sweeps_left != 0) {
            const Geo g = L->g;
            assign_block_any<W, kAllShapes>(g, d.y & 0xFFFFu, d.y >> 16, L->spins, L->labels, L->rng_state, L->rng_sel,
                                L->rng_iter, L->thr, L->edge, smem);
            __syncthreads();
        }
        d = next;
    }
}

__global__ void __launch_bounds__(kMergeThreads) kb_merge(const BatchLat *lats, const BlockRec *recs,
                                                          const uint32_t total, unsigned int *fault)
{
    for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
        const BlockRec r = recs[item];
        const Geo g = rec_geo(r);
        const bool active = lats[r.lat].sweeps_left != 0;
        if (threadIdx.x < g.BX + g.BY)
            merge_block(g, r.bxy & 0xFFFFu, r.bxy >> 16, threadIdx.x, r.edge, r.labels, fault, r.linked, active);
    }
}

// ResolveLabels for the roots each block's merge linked (resolve_block).
__global__ void __launch_bounds__(kMergeThreads) kb_resolve(const BatchLat *lats, const BlockRec *recs,
                                                            const uint32_t total, unsigned int *fault)
{
    for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
        const BlockRec r = recs[item];
        const Geo g = rec_geo(r);
        const bool active = lats[r.lat].sweeps_left != 0;
        if (threadIdx.x < g.BX + g.BY)
            resolve_block(g, r.bxy & 0xFFFFu, r.bxy >> 16, threadIdx.x, r.linked, r.labels, fault, active);
    }
}

// Flip of one block (flip_block, after kb_resolve).
__global__ void __launch_bounds__(kFlipThreads, 6) kb_flip(const BatchLat *lats, const BlockRec *recs,
                                                            const uint32_t total, unsigned int *fault)
{
    extern __shared__ __align__(16) unsigned char smem[];
    for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
        const BlockRec r = recs[item];
        // The budget is read beside the data, not ahead of it: a lattice whose budget ran out
        // leaves the lists at the engine's next call, so only the rest of the call in which it
        // finished reads (and does not write) its blocks.
        const bool active = lats[r.lat].sweeps_left != 0;
        flip_block<false, 4, true>(rec_geo(r), r.bxy & 0xFFFFu, r.bxy >> 16, r.spins, r.labels, fault, smem, active);
        if (item + gridDim.x < total)
            __syncthreads();  // the next item reuses the shared memory
    }
}

// Closes a round after every phase kernel of it (before the measurement): each lattice that was
// swept counts the sweep and spends one from its budget.  The kernels of the round read the
// budget only to skip finished lattices, so it changes here, between rounds.
// With chunk_lat (a round that measures), every lattice due for a sample (measure_every divides
// its sweep count) appends its 4096-site chunks to the round's measure list, so kb_measure visits
// only those.
__global__ void kb_end_round(BatchLat *lats, const uint32_t *active, BatchCounters *ctr, uint32_t *chunk_lat)
{
    const uint32_t n = ctr->n_active;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        BatchLat *L = lats + active[k];
        if (L->sweeps_left != 0) {
            L->swept = 1;
            L->sweeps_done += 1;
            if (L->sweeps_left != kUnlimited)
                L->sweeps_left -= 1;
            if (chunk_lat && L->measure_every && L->sweeps_done % L->measure_every == 0) {
                const uint32_t nch = (uint32_t)(((size_t)L->g.L0 * L->g.L1 + kChunkSites - 1) / kChunkSites);
                const uint32_t base = atomicAdd(&ctr->measure_chunks, nch);
                L->measure_base = base;
                for (uint32_t c = 0; c < nch; ++c)
                    chunk_lat[base + c] = active[k];
            }
        }
    }
}

// Energy / magnetisation of the lattices on this round's measure list (kb_end_round): CTAs pull
// 4096-site chunks from a device counter; per lattice int64 sums, the last chunk turns them into
// FP64 accumulators.  A round whose list is empty costs one read per CTA.
__global__ void __launch_bounds__(kMeasureThreads) kb_measure(BatchLat *lats, const uint32_t *chunk_lat,
                                                              BatchCounters *ctr)
{
    __shared__ uint32_t slot;
    __shared__ long long se[kMeasureThreads / 32], sm[kMeasureThreads / 32];
    const uint32_t total = ctr->measure_chunks;
    if (total == 0)
        return;
    while (true) {
        const uint32_t item = next_item(&ctr->measure_next, &slot);
        if (item >= total)
            break;
        BatchLat *L = lats + chunk_lat[item];
        const uint32_t L0 = L->g.L0, L1 = L->g.L1;
        const size_t nsites = (size_t)L0 * L1;
        const uint32_t chunk = item - L->measure_base;
        const uint32_t nchunks = (uint32_t)((nsites + kChunkSites - 1) / kChunkSites);
        const size_t i0 = (size_t)chunk * kChunkSites, i1 = min(i0 + kChunkSites, nsites);
        int ei = 0, mi = 0;
        // 16-site pieces (row_em's unit), cut at row ends: 256 of the CTA's threads per chunk
        for (size_t p = i0 + (size_t)threadIdx.x * 16; p < i1; p += (size_t)blockDim.x * 16) {
            size_t q = p;
            const size_t qe = min(p + 16, i1);
            while (q < qe) {
                const uint32_t y = (uint32_t)(q / L0), x = (uint32_t)(q - (size_t)y * L0);
                const uint32_t cnt = (uint32_t)min((size_t)(L0 - x), qe - q);
                row_em(L->spins, L0, L1, y, x, cnt, ei, mi);
                q += cnt;
            }
        }
        long long e = ei, m = mi;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            e += __shfl_xor_sync(0xffffffffu, e, o);
            m += __shfl_xor_sync(0xffffffffu, m, o);
        }
        if ((threadIdx.x & 31) == 0) {
            se[threadIdx.x >> 5] = e;
            sm[threadIdx.x >> 5] = m;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            long long be = 0, bm = 0;
            for (uint32_t w = 0; w < blockDim.x / 32; ++w) {
                be += se[w];
                bm += sm[w];
            }
            obs_add_part(L->obs, L->series, L->series_cap, nsites, nchunks, be, bm, 1);
        }
        __syncthreads();
    }
}

// Clears the per-round "swept" flags (first node of a round).
__global__ void kb_begin_round(BatchLat *lats, const uint32_t *active, BatchCounters *ctr)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {  // the previous round's measurement is finished
        ctr->measure_next = 0;
        ctr->measure_chunks = 0;
    }
    const uint32_t n = ctr->n_active;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        lats[active[k]].swept = 0;
}

template <int W>
__global__ void kb_rng_init(const uint32_t n_tiles, const uint32_t seed_base, uint32_t *state, uint8_t *sel,
                           uint32_t *iter)
{
    rng_init_tile<W>(n_tiles, seed_base, state, sel, iter);
}

// One lattice's spins and its slice of the contiguous staging buffer (host transfers).
struct StageCopy {
    uint8_t *spins;
    unsigned long long offset;  // byte offset in the staging buffer
    unsigned long long bytes;
};

// Staging buffer -> lattice spins (to_lattice != 0) or back: CTA (x, y) moves piece x (kStagePiece
// bytes) of lattice y of the group; 16-byte moves when both ends and the length allow, else 4-byte
// or single-byte moves.
constexpr uint32_t kStagePiece = 16384;

__global__ void __launch_bounds__(256) kb_stage_copy(const StageCopy *c, uint8_t *stage, const int to_lattice)
{
    const StageCopy d = c[blockIdx.y];
    const size_t p0 = (size_t)blockIdx.x * kStagePiece;
    if (p0 >= d.bytes)
        return;
    const size_t len = min((size_t)kStagePiece, (size_t)d.bytes - p0);
    uint8_t *a = (to_lattice ? d.spins : stage + d.offset) + p0;
    const uint8_t *s = (to_lattice ? stage + d.offset : d.spins) + p0;
    const uintptr_t align = (uintptr_t)a | (uintptr_t)s | (uintptr_t)len;
    if ((align & 15u) == 0) {
        for (size_t i = threadIdx.x; i < len / 16; i += blockDim.x)
            reinterpret_cast<uint4 *>(a)[i] = reinterpret_cast<const uint4 *>(s)[i];
    } else if ((align & 3u) == 0) {
        for (size_t i = threadIdx.x; i < len / 4; i += blockDim.x)
            reinterpret_cast<uint32_t *>(a)[i] = reinterpret_cast<const uint32_t *>(s)[i];
    } else {
        for (size_t i = threadIdx.x; i < len; i += blockDim.x)
            a[i] = s[i];
    }
}

__global__ void kb_hot_start(const size_t n, const uint32_t seed, uint8_t *spins)
{
    hot_start_chunk(n, seed, spins);
}

}  // namespace swb

using namespace swb;

namespace {

struct HostLat {
    bool used = false;
    BatchLat d{};             // host copy of the descriptor
    uint64_t bytes = 0;       // device bytes held
    void *mem = nullptr;      // one allocation for all buffers of the lattice
    uint64_t sched_round = 0; // the engine's round count when d.sweeps_left was last set
};

}  // namespace

struct swb_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t W = 16, capacity = 0;
    uint64_t budget = 0, used = 0;
    std::vector<HostLat> lats;
    BatchLat *d_lats = nullptr;
    uint32_t *d_active = nullptr;
    uint32_t *d_chunk_lat = nullptr;      // the round's measure list: lattice slot per chunk
    uint32_t chunk_lat_cap = 0;
    uint2 *d_items = nullptr;       // flat block list (lattice slot, byi << 16 | bxi)
    BlockRec *d_recs = nullptr;     // the same items as records (merge, resolve, flip)
    uint32_t items_cap = 0;
    uint32_t items_n = 0;           // block items in the list (the phase kernels' grid)
    uint64_t graph_version = ~0ull;  // lists_version the captured graphs were built for
    uint32_t grp_start[kRoundGroups] = {}, grp_count[kRoundGroups] = {};  // item ranges of the round's groups
    cudaStream_t gstream[kRoundGroups] = {};
    cudaEvent_t fork = nullptr, join[kRoundGroups] = {};
    BatchCounters *d_ctr = nullptr;
    unsigned int *d_fault = nullptr;
    uint8_t *d_stage = nullptr;          // contiguous spins of update_host's lattices
    StageCopy *d_copies = nullptr;
    uint64_t stage_cap = 0, copies_cap = 0;
    uint2 *d_io_items = nullptr;         // update_host's block items, grouped
    BlockRec *d_io_recs = nullptr;       // the same as records
    uint64_t io_items_cap = 0;
    cudaStream_t s_in = nullptr, s_out = nullptr;  // update_host's copy streams
    uint64_t lists_version = 0;          // bumped by every rebuild of the work lists
    // update_host's plan for its last id list, reused while the list and the lattice set stay
    struct IoPlan {
        std::vector<uint32_t> ids, gs;
        std::vector<size_t> gi;
        std::vector<StageCopy> copies;
        std::vector<uint64_t> max_bytes;  // largest lattice of each group (the stage copies' grid)
        uint64_t total = 0, version = ~0ull;
    } io;
    std::vector<cudaEvent_t> io_events;
    std::vector<uint32_t> active;   // ids in the work lists
    cudaEvent_t origin = nullptr;           // swb_batch_mark's time origin (recorded at the first mark)
    std::vector<cudaEvent_t> marks;         // swb_batch_mark's events, a ring
    uint32_t next_mark = 0;
    bool lists_dirty = true;
    uint64_t round_count = 0;  // rounds queued so far (every listed lattice with budget left sweeps once)
    bool assign_all_shapes = true;  // an active lattice has a tile only the all-shapes assign compiles
    int grid_measure = 0;
    uint32_t smem_assign = 0, smem_flip = 0;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};   // [measure?]
    uint64_t series_cap = 1u << 16;
};

namespace {

int bset_device(const swb_batch *b)
{
    SWB_CUDA(cudaSetDevice(b->device));
    return SWB_OK;
}

// Non-zero fault word: a label chase ran past kChainCap steps (only corrupt labels can).
int bcheck_fault(swb_batch *b)
{
    unsigned int f = 0;
    SWB_CUDA(cudaMemcpyAsync(&f, b->d_fault, sizeof(f), cudaMemcpyDeviceToHost, b->stream));
    SWB_CUDA(cudaStreamSynchronize(b->stream));
    if (f)
        return fail(SWB_ERR_STATE, "label union-find fault (word %u: 1 chain over %u steps, 2 union retries, 4 label outside the lattice)", f, kChainCap);
    return SWB_OK;
}

uint32_t lattice_chunks(const Geo &g) { return (uint32_t)(((size_t)g.L0 * g.L1 + kChunkSites - 1) / kChunkSites); }

// Device bytes one lattice needs (the admission estimate).
uint64_t lattice_bytes(const Geo &g, uint32_t W, uint64_t series_cap)
{
    const uint64_t n = (uint64_t)g.L0 * g.L1, tiles = (uint64_t)g.n0 * g.n1, blocks = (uint64_t)g.nbx * g.nby;
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    return al(n) + al(4 * n) + al(4 * tiles * W) + al(tiles * W) + al(4 * tiles) + al(4 * kEdgeWords * blocks) +
           al(4 * (uint64_t)(g.BX + g.BY) * blocks) + al(sizeof(Obs)) + al(16 * series_cap);
}

int upload_descriptor(swb_batch *b, uint32_t id)
{
    SWB_CUDA(cudaMemcpyAsync(b->d_lats + id, &b->lats[id].d, sizeof(BatchLat), cudaMemcpyHostToDevice, b->stream));
    return SWB_OK;
}

// Rebuilds the active list and prefix sums (host) and uploads them with the totals.
// The records of a list of block items (BlockRec).
std::vector<BlockRec> make_recs(const swb_batch *b, const std::vector<uint2> &items)
{
    std::vector<BlockRec> recs(items.size());
    for (size_t k = 0; k < items.size(); ++k) {
        const BatchLat &d = b->lats[items[k].x].d;
        BlockRec &r = recs[k];
        r.lat = items[k].x;
        r.bxy = items[k].y;
        r.L0 = d.g.L0;
        r.L1 = d.g.L1;
        r.bxby = d.g.BX | d.g.BY << 16;
        r.nbx = d.g.nbx;
        r.nby = d.g.nby;
        r.pad = 0;
        r.spins = d.spins;
        r.labels = d.labels;
        r.edge = d.edge;
        r.linked = d.linked;
    }
    return recs;
}

// A lattice whose budget the queued rounds have used up (known on the host: every round
// sweeps every listed lattice with budget left once).  It leaves the lists at their next
// rebuild, so rounds launch nothing for it; a server keeps finished jobs until it needs their
// memory.
bool budget_spent(const swb_batch *b, const HostLat &h)
{
    return h.d.sweeps_left != kUnlimited && b->round_count - h.sched_round >= h.d.sweeps_left;
}

int rebuild_lists(swb_batch *b)
{
    for (uint32_t id : b->active)
        if (budget_spent(b, b->lats[id]))
            b->lists_dirty = true;
    if (!b->lists_dirty)
        return SWB_OK;
    b->active.clear();
    for (uint32_t i = 0; i < b->capacity; ++i)
        if (b->lats[i].used && !budget_spent(b, b->lats[i]))
            b->active.push_back(i);
    // big lattices first: their many items start early and balance the tail
    std::stable_sort(b->active.begin(), b->active.end(), [&](uint32_t x, uint32_t y) {
        const Geo &gx = b->lats[x].d.g, &gy = b->lats[y].d.g;
        return (uint64_t)gx.L0 * gx.L1 > (uint64_t)gy.L0 * gy.L1;
    });
    const uint32_t n = (uint32_t)b->active.size();
    b->assign_all_shapes = false;
    for (uint32_t id : b->active) {
        const Geo &g = b->lats[id].d.g;
        const bool lean = (g.TX == 16 && (g.TY == 8 || g.TY == 4)) ||
                          !((g.TX == 8 && (g.TY == 8 || g.TY == 16)) || (g.TX == 32 && (g.TY == 4 || g.TY == 8)) ||
                            (g.TX == 16 && g.TY == 16));
        b->assign_all_shapes |= !lean;
    }
    std::vector<uint32_t> bp(n + 1, 0), cp(n + 1, 0);
    for (uint32_t k = 0; k < n; ++k) {
        const Geo &g = b->lats[b->active[k]].d.g;
        bp[k + 1] = bp[k] + g.nbx * g.nby;
        cp[k + 1] = cp[k] + lattice_chunks(g);
    }
    // lattices to round groups, biggest first onto the lightest group; the items of a group
    // are contiguous, each group's in size order
    std::vector<uint32_t> grp(n, 0);
    uint64_t load[kRoundGroups] = {};
    for (uint32_t k = 0; k < n; ++k) {
        uint32_t best = 0;
        for (uint32_t q = 1; q < kRoundGroups; ++q)
            if (load[q] < load[best])
                best = q;
        grp[k] = best;
        load[best] += bp[k + 1] - bp[k];
    }
    std::vector<uint2> items;
    items.reserve(bp[n]);
    for (uint32_t q = 0; q < kRoundGroups; ++q) {
        b->grp_start[q] = (uint32_t)items.size();
        for (uint32_t k = 0; k < n; ++k) {
            if (grp[k] != q)
                continue;
            const Geo &g = b->lats[b->active[k]].d.g;
            for (uint32_t by = 0; by < g.nby; ++by)
                for (uint32_t bx = 0; bx < g.nbx; ++bx)
                    items.push_back(make_uint2(b->active[k], by << 16 | bx));
        }
        b->grp_count[q] = (uint32_t)items.size() - b->grp_start[q];
    }
    if (items.size() > b->items_cap) {
        // a larger list: the captured graphs hold the old pointer
        SWB_CUDA(cudaStreamSynchronize(b->stream));
        for (auto &ge : b->graph)
            if (ge) {
                cudaGraphExecDestroy(ge);
                ge = nullptr;
            }
        SWB_CUDA(cudaFree(b->d_items));
        b->d_items = nullptr;
        SWB_CUDA(cudaFree(b->d_recs));
        b->d_recs = nullptr;
        const uint32_t cap = std::max<uint32_t>((uint32_t)items.size(), 2 * b->items_cap);
        SWB_CUDA(cudaMalloc(&b->d_items, sizeof(uint2) * cap));
        SWB_CUDA(cudaMalloc(&b->d_recs, sizeof(BlockRec) * cap));
        b->items_cap = cap;
    }
    if (cp[n] > b->chunk_lat_cap) {  // the measure list holds every active lattice's chunks
        SWB_CUDA(cudaStreamSynchronize(b->stream));  // no captured round may still read the old list
        for (auto &ge : b->graph)
            if (ge) {
                cudaGraphExecDestroy(ge);
                ge = nullptr;
            }
        SWB_CUDA(cudaFree(b->d_chunk_lat));
        b->d_chunk_lat = nullptr;
        const uint32_t cap = std::max<uint32_t>(cp[n], 2 * b->chunk_lat_cap);
        SWB_CUDA(cudaMalloc(&b->d_chunk_lat, sizeof(uint32_t) * cap));
        b->chunk_lat_cap = cap;
    }
    b->items_n = (uint32_t)items.size();
    BatchCounters c{};
    c.n_active = n;
    c.total_chunks = cp[n];
    if (n) {
        SWB_CUDA(cudaMemcpyAsync(b->d_items, items.data(), sizeof(uint2) * items.size(), cudaMemcpyHostToDevice,
                                 b->stream));
        const std::vector<BlockRec> recs = make_recs(b, items);
        SWB_CUDA(cudaMemcpyAsync(b->d_recs, recs.data(), sizeof(BlockRec) * recs.size(), cudaMemcpyHostToDevice,
                                 b->stream));
        SWB_CUDA(cudaMemcpyAsync(b->d_active, b->active.data(), n * 4, cudaMemcpyHostToDevice, b->stream));
    }
    SWB_CUDA(cudaMemcpyAsync(b->d_ctr, &c, sizeof(c), cudaMemcpyHostToDevice, b->stream));
    b->lists_dirty = false;
    b->lists_version += 1;
    return SWB_OK;
}

// One CTA per block item (at least one CTA): the hardware scheduler interleaves the phases of
// co-resident CTAs better than a persistent loop does.  `items` / `n` is any list of block
// items: the whole round's, or one group of update_host's pipeline.
int launch_assign_b(swb_batch *b, const uint2 *items, uint32_t n, cudaStream_t st)
{
    const uint32_t grid = std::max(n, 1u);
    switch (b->W) {
    case 8: kb_assign<8, true><<<grid, kBatchThreads, b->smem_assign, st>>>(b->d_lats, items, n, b->d_ctr); break;
    case 16:
        if (b->assign_all_shapes)
            kb_assign<16, true><<<grid, kBatchThreads, b->smem_assign, st>>>(b->d_lats, items, n, b->d_ctr);
        else
            kb_assign<16, false><<<grid, kBatchThreads, b->smem_assign, st>>>(b->d_lats, items, n, b->d_ctr);
        break;
    case 32: kb_assign<32, true><<<grid, kBatchThreads, b->smem_assign, st>>>(b->d_lats, items, n, b->d_ctr); break;
    default: return fail(SWB_ERR_ARGUMENT, "unsupported lcg width %u", b->W);
    }
    SWB_LAUNCHED();
    return SWB_OK;
}

int launch_merge_b(swb_batch *b, const BlockRec *recs, uint32_t n, cudaStream_t st)
{
    kb_merge<<<std::max(n, 1u), kMergeThreads, 0, st>>>(b->d_lats, recs, n, b->d_fault);
    SWB_LAUNCHED();
    return SWB_OK;
}

int launch_resolve_b(swb_batch *b, const BlockRec *recs, uint32_t n, cudaStream_t st)
{
    kb_resolve<<<std::max(n, 1u), kMergeThreads, 0, st>>>(b->d_lats, recs, n, b->d_fault);
    SWB_LAUNCHED();
    return SWB_OK;
}

int launch_flip_b(swb_batch *b, const BlockRec *recs, uint32_t n, cudaStream_t st)
{
    kb_flip<<<std::max(n, 1u), kFlipThreads, b->smem_flip, st>>>(b->d_lats, recs, n, b->d_fault);
    SWB_LAUNCHED();
    return SWB_OK;
}

// The phases of one sweep over a list of block items.
int launch_phases_b(swb_batch *b, const uint2 *items, const BlockRec *recs, uint32_t n, cudaStream_t st)
{
    if (int rc = launch_assign_b(b, items, n, st))
        return rc;
    if (int rc = launch_merge_b(b, recs, n, st))
        return rc;
    if (int rc = launch_resolve_b(b, recs, n, st))
        return rc;
    return launch_flip_b(b, recs, n, st);
}

int launch_end_round(swb_batch *b, cudaStream_t st, bool measure)
{
    kb_end_round<<<4, 128, 0, st>>>(b->d_lats, b->d_active, b->d_ctr, measure ? b->d_chunk_lat : nullptr);
    SWB_LAUNCHED();
    return SWB_OK;
}

// Kernels of one captured round: begin, four phases per non-empty lattice group, end, measure.
uint32_t round_launches(const swb_batch *b, bool measure)
{
    uint32_t n = 2 + (measure ? 1 : 0);
    for (uint32_t q = 0; q < kRoundGroups; ++q)
        n += b->grp_count[q] ? 4 : 0;
    return n;
}

int launch_round(swb_batch *b, bool measure)
{
    kb_begin_round<<<4, 128, 0, b->stream>>>(b->d_lats, b->d_active, b->d_ctr);
    SWB_LAUNCHED();
    // The groups' sweeps run on their own streams: the end of one group's assign overlaps the
    // start of another's merge and flip (lattices are independent), 2 % faster per round than
    // one stream; chaining the assigns did not help (an assign CTA set fills every warp slot).
    if (!b->fork) {
        SWB_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
        for (uint32_t q = 0; q < kRoundGroups; ++q) {
            SWB_CUDA(cudaEventCreateWithFlags(&b->join[q], cudaEventDisableTiming));
            SWB_CUDA(cudaStreamCreateWithFlags(&b->gstream[q], cudaStreamNonBlocking));
        }
    }
    SWB_CUDA(cudaEventRecord(b->fork, b->stream));
    for (uint32_t q = 0; q < kRoundGroups; ++q) {
        if (!b->grp_count[q])
            continue;
        SWB_CUDA(cudaStreamWaitEvent(b->gstream[q], b->fork, 0));
        if (int rc = launch_phases_b(b, b->d_items + b->grp_start[q], b->d_recs + b->grp_start[q], b->grp_count[q],
                                     b->gstream[q]))
            return rc;
        SWB_CUDA(cudaEventRecord(b->join[q], b->gstream[q]));
        SWB_CUDA(cudaStreamWaitEvent(b->stream, b->join[q], 0));
    }
    if (int rc = launch_end_round(b, b->stream, measure))
        return rc;
    if (measure) {
        kb_measure<<<b->grid_measure, kMeasureThreads, 0, b->stream>>>(b->d_lats, b->d_chunk_lat, b->d_ctr);
        SWB_LAUNCHED();
    }
    return SWB_OK;
}

// One round, captured on first use and again after the lattice set changed (rounds() drops
// the graphs then): the grids and item ranges are baked into the graph, the per-lattice state
// (sweep budgets, temperatures, schedules) is read from device memory at every replay.
int round_graph(swb_batch *b, bool measure, cudaGraphExec_t *out)
{
    cudaGraphExec_t &ge = b->graph[measure ? 1 : 0];
    if (!ge) {
        cudaGraph_t g = nullptr;
        SWB_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = launch_round(b, measure);
        const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (rc)
            return rc;
        if (e != cudaSuccess)
            return fail(SWB_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
        const cudaError_t e2 = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        if (e2 != cudaSuccess)
            return fail(SWB_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e2));
    }
    *out = ge;
    return SWB_OK;
}

HostLat *get_lat(swb_batch *b, uint32_t id)
{
    if (!b || id >= b->capacity || !b->lats[id].used)
        return nullptr;
    return &b->lats[id];
}

int rounds(swb_batch *b, uint32_t n_rounds, bool any_measure)
{
    if (int rc = rebuild_lists(b))
        return rc;
    if (b->graph_version != b->lists_version) {  // the graphs' grids follow the item list
        SWB_CUDA(cudaStreamSynchronize(b->stream));
        for (auto &ge : b->graph)
            if (ge) {
                cudaGraphExecDestroy(ge);
                ge = nullptr;
            }
        b->graph_version = b->lists_version;
    }
    cudaGraphExec_t ge;
    if (int rc = round_graph(b, any_measure, &ge))
        return rc;
    for (uint32_t r = 0; r < n_rounds; ++r) {
        SWB_CUDA(cudaGraphLaunch(ge, b->stream));
        g_launches.fetch_add(round_launches(b, any_measure), std::memory_order_relaxed);
        b->round_count += 1;
    }
    return SWB_OK;
}

}  // namespace

extern "C" {

int swb_batch_lattice_bytes(uint32_t L0, uint32_t L1, uint32_t tile_x, uint32_t tile_y, uint32_t lcg_width,
                            uint64_t *bytes)
{
    if (!bytes)
        return fail(SWB_ERR_ARGUMENT, "bytes is NULL");
    const Geo g = make_geo(L0, L1, tile_x, tile_y, lcg_width, kBatchThreads);
    *bytes = lattice_bytes(g, lcg_width, 1u << 16);
    return SWB_OK;
}

int swb_batch_create(swb_batch **out, uint32_t capacity, uint64_t hbm_budget_bytes, uint32_t lcg_width, int device)
{
    if (!out)
        return fail(SWB_ERR_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (capacity == 0 || capacity > (1u << 20))
        return fail(SWB_ERR_ARGUMENT, "capacity must be in [1, 2^20]");
    if (!(lcg_width == 8 || lcg_width == 16 || lcg_width == 32))
        return fail(SWB_ERR_ARGUMENT, "unsupported lcg32 width %u", lcg_width);
    swb_batch *b = new swb_batch();
    b->device = device;
    b->W = lcg_width;
    b->capacity = capacity;
    b->budget = hbm_budget_bytes;
    b->lats.resize(capacity);
    auto cleanup = [&](int rc) {
        swb_batch_destroy(b);
        return rc;
    };
#define SWB_TRY(call)                                                                              \
    do {                                                                                           \
        cudaError_t err__ = (call);                                                                \
        if (err__ != cudaSuccess)                                                                  \
            return cleanup(fail(SWB_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(err__))); \
    } while (0)
    SWB_TRY(cudaSetDevice(device));
    SWB_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    SWB_TRY(cudaMalloc(&b->d_lats, sizeof(BatchLat) * capacity));
    SWB_TRY(cudaMalloc(&b->d_active, 4 * capacity));
    SWB_TRY(cudaMalloc(&b->d_ctr, sizeof(BatchCounters)));
    SWB_TRY(cudaMalloc(&b->d_fault, sizeof(unsigned int)));
    SWB_TRY(cudaMemsetAsync(b->d_fault, 0, sizeof(unsigned int), b->stream));
    SWB_TRY(cudaMemsetAsync(b->d_ctr, 0, sizeof(BatchCounters), b->stream));
    // The assign phase may hold any block up to 128 x 32 sites: size shared memory for it.
    Geo gmax{};
    gmax.BX = 128; gmax.BY = 32;
    b->smem_assign = assign_smem_max(lcg_width, kBatchThreads);
    b->smem_flip = flip_smem_bytes(gmax);
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kb_measure, kMeasureThreads, 0);
    b->grid_measure = sms * std::max(per_sm, 1);  // measure: persistent, pulls chunks
    SWB_TRY(cudaStreamSynchronize(b->stream));
#undef SWB_TRY
    *out = b;
    return SWB_OK;
}

int swb_batch_destroy(swb_batch *b)
{
    if (!b)
        return SWB_OK;
    cudaSetDevice(b->device);
    if (b->stream)
        cudaStreamSynchronize(b->stream);
    for (auto &ge : b->graph)
        if (ge)
            cudaGraphExecDestroy(ge);
    for (auto &l : b->lats)
        if (l.mem)
            cudaFree(l.mem);
    cudaFree(b->d_lats);
    cudaFree(b->d_active);
    cudaFree(b->d_chunk_lat);
    cudaFree(b->d_items);
    cudaFree(b->d_recs);
    cudaFree(b->d_stage);
    cudaFree(b->d_copies);
    cudaFree(b->d_io_items);
    cudaFree(b->d_io_recs);
    for (auto e : b->io_events)
        cudaEventDestroy(e);
    if (b->fork)
        cudaEventDestroy(b->fork);
    for (uint32_t q = 0; q < kRoundGroups; ++q) {
        if (b->join[q])
            cudaEventDestroy(b->join[q]);
        if (b->gstream[q])
            cudaStreamDestroy(b->gstream[q]);
    }
    for (auto e : b->marks)
        cudaEventDestroy(e);
    if (b->origin)
        cudaEventDestroy(b->origin);
    if (b->s_in)
        cudaStreamDestroy(b->s_in);
    if (b->s_out)
        cudaStreamDestroy(b->s_out);
    cudaFree(b->d_ctr);
    cudaFree(b->d_fault);
    if (b->stream)
        cudaStreamDestroy(b->stream);
    delete b;
    return SWB_OK;
}

int swb_batch_add(swb_batch *b, uint32_t L0, uint32_t L1, uint32_t tile_x, uint32_t tile_y, uint32_t block_x,
                  uint32_t block_y, float temperature, uint32_t seed_base, uint32_t *id)
{
    if (!b || !id)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (L0 == 0 || L1 == 0 || (L0 % 2) || (L1 % 2))
        return fail(SWB_ERR_ARGUMENT, "SwendsenWang_2D implementation requires evenly sized lattice (%u x %u)", L0, L1);
    if ((uint64_t)L0 * L1 > 0x7FFFFFFFull)
        return fail(SWB_ERR_ARGUMENT, "lattice of %u x %u sites exceeds 2^31 - 1 labels", L0, L1);
    if (!(tile_x == 8 || tile_x == 16 || tile_x == 32) || tile_y < 2 || tile_y > 32)
        return fail(SWB_ERR_ARGUMENT, "unsupported tile %u x %u", tile_x, tile_y);
    if (!(temperature > 0.0f) || !std::isfinite(temperature))
        return fail(SWB_ERR_ARGUMENT, "temperature must be positive and finite");
    if (int rc = bset_device(b))
        return rc;
    uint32_t slot = b->capacity;
    for (uint32_t i = 0; i < b->capacity; ++i)
        if (!b->lats[i].used) {
            slot = i;
            break;
        }
    if (slot == b->capacity)
        return fail(SWB_ERR_CAPACITY, "all %u lattice slots are in use", b->capacity);
    const Geo g = make_geo(L0, L1, tile_x, tile_y, b->W, kBatchThreads, block_x, block_y);
    if (g.nbx > 0xFFFFu || g.nby > 0xFFFFu)  // block coordinates are 16-bit in the work items
        return fail(SWB_ERR_ARGUMENT, "lattice of %u x %u sites needs more than 65535 blocks in a direction", L0, L1);
    if (assign_smem(g, b->W).total > b->smem_assign)
        return fail(SWB_ERR_ARGUMENT, "block of %u x %u sites needs more shared memory than reserved", g.BX, g.BY);
    const uint64_t bytes = lattice_bytes(g, b->W, b->series_cap);
    if (b->budget && b->used + bytes > b->budget)
        return fail(SWB_ERR_CAPACITY, "lattice needs %llu bytes, %llu of %llu in use", (unsigned long long)bytes,
                    (unsigned long long)b->used, (unsigned long long)b->budget);
    HostLat &h = b->lats[slot];
    void *mem = nullptr;
    SWB_CUDA(cudaMalloc(&mem, bytes));
    const uint64_t n = (uint64_t)L0 * L1, tiles = (uint64_t)g.n0 * g.n1, blocks = (uint64_t)g.nbx * g.nby;
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    char *p = static_cast<char *>(mem);
    BatchLat d{};
    d.g = g;
    d.spins = reinterpret_cast<uint8_t *>(p); p += al(n);
    d.labels = reinterpret_cast<uint32_t *>(p); p += al(4 * n);
    d.rng_state = reinterpret_cast<uint32_t *>(p); p += al(4 * tiles * b->W);
    d.rng_sel = reinterpret_cast<uint8_t *>(p); p += al(tiles * b->W);
    d.rng_iter = reinterpret_cast<uint32_t *>(p); p += al(4 * tiles);
    d.edge = reinterpret_cast<uint32_t *>(p); p += al(4 * kEdgeWords * blocks);
    d.linked = reinterpret_cast<uint32_t *>(p); p += al(4 * (uint64_t)(g.BX + g.BY) * blocks);
    d.obs = reinterpret_cast<Obs *>(p); p += al(sizeof(Obs));
    d.series = reinterpret_cast<long long *>(p);
    d.series_cap = b->series_cap;
    d.thr = accept_threshold(swb_p_add(temperature));
    d.sweeps_left = kUnlimited;
    d.measure_every = 0;
    SWB_CUDA(cudaMemsetAsync(d.spins, 0, n, b->stream));
    SWB_CUDA(cudaMemsetAsync(d.obs, 0, sizeof(Obs), b->stream));
    switch (b->W) {
    case 8: kb_rng_init<8><<<(unsigned)((tiles + 127) / 128), 128, 0, b->stream>>>((uint32_t)tiles, seed_base, d.rng_state, d.rng_sel, d.rng_iter); break;
    case 16: kb_rng_init<16><<<(unsigned)((tiles + 127) / 128), 128, 0, b->stream>>>((uint32_t)tiles, seed_base, d.rng_state, d.rng_sel, d.rng_iter); break;
    default: kb_rng_init<32><<<(unsigned)((tiles + 127) / 128), 128, 0, b->stream>>>((uint32_t)tiles, seed_base, d.rng_state, d.rng_sel, d.rng_iter); break;
    }
    SWB_LAUNCHED();
    h.used = true;
    h.d = d;
    h.bytes = bytes;
    h.mem = mem;
    b->used += bytes;
    b->lists_dirty = true;
    if (int rc = upload_descriptor(b, slot))
        return rc;
    *id = slot;
    return SWB_OK;
}

int swb_batch_remove(swb_batch *b, uint32_t id)
{
    HostLat *h = get_lat(b, id);
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "no lattice %u", id);
    if (int rc = bset_device(b))
        return rc;
    SWB_CUDA(cudaStreamSynchronize(b->stream));
    SWB_CUDA(cudaFree(h->mem));
    b->used -= h->bytes;
    *h = HostLat{};
    b->lists_dirty = true;
    return SWB_OK;
}

int swb_batch_hot_start(swb_batch *b, uint32_t id, uint32_t seed)
{
    HostLat *h = get_lat(b, id);
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "no lattice %u", id);
    if (int rc = bset_device(b))
        return rc;
    const size_t n = (size_t)h->d.g.L0 * h->d.g.L1, chunks = (n + 63) / 64;
    kb_hot_start<<<(unsigned)((chunks + 255) / 256), 256, 0, b->stream>>>(n, seed, h->d.spins);
    SWB_LAUNCHED();
    return SWB_OK;
}

int swb_batch_set_spins(swb_batch *b, uint32_t id, const uint8_t *host_spins)
{
    HostLat *h = get_lat(b, id);
    if (!h || !host_spins)
        return fail(SWB_ERR_ARGUMENT, "no lattice %u or NULL spins", id);
    const size_t n = (size_t)h->d.g.L0 * h->d.g.L1;
    for (size_t i = 0; i < n; ++i)
        if (host_spins[i] > 1)
            return fail(SWB_ERR_ARGUMENT, "spins must be 0 or 1");
    if (int rc = bset_device(b))
        return rc;
    SWB_CUDA(cudaMemcpyAsync(h->d.spins, host_spins, n, cudaMemcpyHostToDevice, b->stream));
    SWB_CUDA(cudaStreamSynchronize(b->stream));
    return SWB_OK;
}

int swb_batch_get_spins(swb_batch *b, uint32_t id, uint8_t *host_spins)
{
    HostLat *h = get_lat(b, id);
    if (!h || !host_spins)
        return fail(SWB_ERR_ARGUMENT, "no lattice %u or NULL spins", id);
    if (int rc = bset_device(b))
        return rc;
    SWB_CUDA(cudaMemcpyAsync(host_spins, h->d.spins, (size_t)h->d.g.L0 * h->d.g.L1, cudaMemcpyDeviceToHost, b->stream));
    SWB_CUDA(cudaStreamSynchronize(b->stream));
    return bcheck_fault(b);
}

int swb_batch_set_temperature(swb_batch *b, uint32_t id, float temperature)
{
    HostLat *h = get_lat(b, id);
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "no lattice %u", id);
    if (!(temperature > 0.0f) || !std::isfinite(temperature))
        return fail(SWB_ERR_ARGUMENT, "temperature must be positive and finite");
    if (int rc = bset_device(b))
        return rc;
    h->d.thr = accept_threshold(swb_p_add(temperature));
    SWB_CUDA(cudaMemcpyAsync(&b->d_lats[id].thr, &h->d.thr, sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream));
    SWB_CUDA(cudaStreamSynchronize(b->stream));
    return SWB_OK;
}

int swb_batch_set_schedule(swb_batch *b, uint32_t id, uint32_t sweeps, uint32_t measure_every)
{
    HostLat *h = get_lat(b, id);
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "no lattice %u", id);
    if (int rc = bset_device(b))
        return rc;
    uint32_t v[2] = {sweeps, measure_every};
    SWB_CUDA(cudaMemcpyAsync(&b->d_lats[id].sweeps_left, &v[0], 4, cudaMemcpyHostToDevice, b->stream));
    SWB_CUDA(cudaMemcpyAsync(&b->d_lats[id].measure_every, &v[1], 4, cudaMemcpyHostToDevice, b->stream));
    SWB_CUDA(cudaStreamSynchronize(b->stream));
    const bool was_spent = budget_spent(b, *h);
    h->d.sweeps_left = sweeps;
    h->d.measure_every = measure_every;
    h->sched_round = b->round_count;
    if (budget_spent(b, *h) != was_spent)  // joins or leaves the lists
        b->lists_dirty = true;
    return SWB_OK;
}

int swb_batch_status(swb_batch *b, uint32_t id, uint32_t *sweeps_left, uint32_t *sweeps_done)
{
    HostLat *h = get_lat(b, id);
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "no lattice %u", id);
    if (int rc = bset_device(b))
        return rc;
    BatchLat d;
    SWB_CUDA(cudaMemcpyAsync(&d, b->d_lats + id, sizeof(d), cudaMemcpyDeviceToHost, b->stream));
    SWB_CUDA(cudaStreamSynchronize(b->stream));
    if (sweeps_left) *sweeps_left = d.sweeps_left;
    if (sweeps_done) *sweeps_done = d.sweeps_done;
    return SWB_OK;
}

int swb_batch_poll(swb_batch *b, uint32_t *sweeps_left, uint32_t *sweeps_done)
{
    if (!b || !sweeps_left)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (int rc = bset_device(b))
        return rc;
    std::vector<BatchLat> d(b->capacity);
    SWB_CUDA(cudaMemcpyAsync(d.data(), b->d_lats, sizeof(BatchLat) * b->capacity, cudaMemcpyDeviceToHost, b->stream));
    SWB_CUDA(cudaStreamSynchronize(b->stream));
    for (uint32_t i = 0; i < b->capacity; ++i) {
        const bool used = b->lats[i].used;
        sweeps_left[i] = used ? d[i].sweeps_left : 0;
        if (sweeps_done)
            sweeps_done[i] = used ? d[i].sweeps_done : 0;
    }
    return SWB_OK;
}

int swb_batch_sweep(swb_batch *b, uint32_t n_rounds, int measure)
{
    if (!b)
        return fail(SWB_ERR_ARGUMENT, "NULL handle");
    if (int rc = bset_device(b))
        return rc;
    return rounds(b, n_rounds, measure != 0);
}

constexpr uint32_t kMarks = 64;  // marks in flight at once

int swb_batch_mark(swb_batch *b, uint32_t *mark)
{
    if (!b || !mark)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (int rc = bset_device(b))
        return rc;
    if (!b->origin) {
        SWB_CUDA(cudaEventCreate(&b->origin));
        SWB_CUDA(cudaEventRecord(b->origin, b->stream));
        b->marks.assign(kMarks, nullptr);
        for (auto &e : b->marks)
            SWB_CUDA(cudaEventCreate(&e));
    }
    const uint32_t m = b->next_mark++;
    SWB_CUDA(cudaEventRecord(b->marks[m % kMarks], b->stream));
    *mark = m;
    return SWB_OK;
}

int swb_batch_mark_query(swb_batch *b, uint32_t mark, int *done, double *ms)
{
    if (!b || !done)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (!b->origin || mark >= b->next_mark || b->next_mark - mark > kMarks)
        return fail(SWB_ERR_ARGUMENT, "mark %u is not one of the last %u marks", mark, kMarks);
    if (int rc = bset_device(b))
        return rc;
    cudaEvent_t e = b->marks[mark % kMarks];
    const cudaError_t q = cudaEventQuery(e);
    if (q == cudaErrorNotReady) {
        *done = 0;
        return SWB_OK;
    }
    SWB_CUDA(q);
    *done = 1;
    if (ms) {
        float t = 0.0f;
        SWB_CUDA(cudaEventElapsedTime(&t, b->origin, e));
        *ms = t;
    }
    return SWB_OK;
}

int swb_batch_synchronize(swb_batch *b)
{
    if (!b)
        return fail(SWB_ERR_ARGUMENT, "NULL handle");
    if (int rc = bset_device(b))
        return rc;
    SWB_CUDA(cudaStreamSynchronize(b->stream));
    return bcheck_fault(b);
}

int swb_batch_sweep_timed(swb_batch *b, uint32_t n_rounds, int per_kernel, float *ms)
{
    if (!b || !ms)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (int rc = bset_device(b))
        return rc;
    if (int rc = rebuild_lists(b))
        return rc;
    ms[0] = ms[1] = ms[2] = ms[3] = 0.0f;
    cudaEvent_t ev[5];
    for (auto &e : ev)
        SWB_CUDA(cudaEventCreate(&e));
    SWB_CUDA(cudaEventRecord(ev[0], b->stream));
    int rc = SWB_OK;
    if (!per_kernel) {
        rc = rounds(b, n_rounds, false);
    } else {
        for (uint32_t r = 0; r < n_rounds && !rc; ++r) {
            kb_begin_round<<<4, 128, 0, b->stream>>>(b->d_lats, b->d_active, b->d_ctr);
            SWB_LAUNCHED();
            SWB_CUDA(cudaEventRecord(ev[1], b->stream));
            if ((rc = launch_assign_b(b, b->d_items, b->items_n, b->stream)))
                break;
            SWB_CUDA(cudaEventRecord(ev[2], b->stream));
            if ((rc = launch_merge_b(b, b->d_recs, b->items_n, b->stream)))
                break;
            SWB_CUDA(cudaEventRecord(ev[3], b->stream));
            // resolve + flip: the reference's ResolveLabels and FlipClusters
            if ((rc = launch_resolve_b(b, b->d_recs, b->items_n, b->stream)))
                break;
            if ((rc = launch_flip_b(b, b->d_recs, b->items_n, b->stream)))
                break;
            SWB_CUDA(cudaEventRecord(ev[4], b->stream));
            if ((rc = launch_end_round(b, b->stream, false)))
                break;
            b->round_count += 1;
            SWB_CUDA(cudaEventSynchronize(ev[4]));
            float t;
            SWB_CUDA(cudaEventElapsedTime(&t, ev[1], ev[2]));
            ms[1] += t;
            SWB_CUDA(cudaEventElapsedTime(&t, ev[2], ev[3]));
            ms[2] += t;
            SWB_CUDA(cudaEventElapsedTime(&t, ev[3], ev[4]));
            ms[3] += t;
        }
    }
    SWB_CUDA(cudaEventRecord(ev[4], b->stream));
    SWB_CUDA(cudaEventSynchronize(ev[4]));
    SWB_CUDA(cudaEventElapsedTime(&ms[0], ev[0], ev[4]));
    for (auto &e : ev)
        cudaEventDestroy(e);
    return rc ? rc : bcheck_fault(b);
}

int swb_batch_accumulators(swb_batch *b, uint32_t id, double *out)
{
    HostLat *h = get_lat(b, id);
    if (!h || !out)
        return fail(SWB_ERR_ARGUMENT, "no lattice %u or NULL out", id);
    if (int rc = bset_device(b))
        return rc;
    Obs o;
    SWB_CUDA(cudaMemcpyAsync(&o, h->d.obs, sizeof(o), cudaMemcpyDeviceToHost, b->stream));
    SWB_CUDA(cudaStreamSynchronize(b->stream));
    std::memcpy(out, o.acc, sizeof(o.acc));
    return SWB_OK;
}

namespace {

// The sample series of lattice h, read on stream st (waited for) after the work already
// ordered before it there.
int read_samples(swb_batch *b, HostLat *h, cudaStream_t st, int64_t *em, uint64_t capacity, uint64_t *count,
                 double *acc)
{
    Obs o;
    SWB_CUDA(cudaMemcpyAsync(&o, h->d.obs, sizeof(o), cudaMemcpyDeviceToHost, st));
    SWB_CUDA(cudaStreamSynchronize(st));
    *count = o.n_samples;
    if (acc)
        std::memcpy(acc, o.acc, sizeof(o.acc));
    if (o.n_samples > h->d.series_cap)
        return fail(SWB_ERR_CAPACITY, "%llu samples recorded, series keeps %llu", o.n_samples, h->d.series_cap);
    const uint64_t k = std::min<uint64_t>(o.n_samples, capacity);
    if (k && em) {
        SWB_CUDA(cudaMemcpyAsync(em, h->d.series, k * 16, cudaMemcpyDeviceToHost, st));
        SWB_CUDA(cudaStreamSynchronize(st));
    }
    (void)b;
    return SWB_OK;
}

}  // namespace

int swb_batch_samples(swb_batch *b, uint32_t id, int64_t *em, uint64_t capacity, uint64_t *count)
{
    HostLat *h = get_lat(b, id);
    if (!h || !count)
        return fail(SWB_ERR_ARGUMENT, "no lattice %u or NULL count", id);
    if (int rc = bset_device(b))
        return rc;
    return read_samples(b, h, b->stream, em, capacity, count, nullptr);
}

int swb_batch_samples_finished(swb_batch *b, uint32_t id, int64_t *em, uint64_t capacity, uint64_t *count,
                               double *acc)
{
    HostLat *h = get_lat(b, id);
    if (!h || !count)
        return fail(SWB_ERR_ARGUMENT, "no lattice %u or NULL count", id);
    if (int rc = bset_device(b))
        return rc;
    if (!b->s_out)
        SWB_CUDA(cudaStreamCreateWithFlags(&b->s_out, cudaStreamNonBlocking));
    return read_samples(b, h, b->s_out, em, capacity, count, acc);
}

int swb_batch_get_rng(swb_batch *b, uint32_t id, uint32_t *state, uint32_t *a, uint32_t *c, uint32_t *iteration)
{
    HostLat *h = get_lat(b, id);
    if (!h || !state || !a || !c || !iteration)
        return fail(SWB_ERR_ARGUMENT, "no lattice %u or NULL argument", id);
    if (int rc = bset_device(b))
        return rc;
    const size_t tiles = (size_t)h->d.g.n0 * h->d.g.n1, nw = tiles * b->W;
    std::vector<uint8_t> sel(nw);
    SWB_CUDA(cudaMemcpyAsync(state, h->d.rng_state, nw * 4, cudaMemcpyDeviceToHost, b->stream));
    SWB_CUDA(cudaMemcpyAsync(sel.data(), h->d.rng_sel, nw, cudaMemcpyDeviceToHost, b->stream));
    SWB_CUDA(cudaMemcpyAsync(iteration, h->d.rng_iter, tiles * 4, cudaMemcpyDeviceToHost, b->stream));
    SWB_CUDA(cudaStreamSynchronize(b->stream));
    for (size_t i = 0; i < nw; ++i) {
        a[i] = lcg_param_a(sel[i]);
        c[i] = lcg_param_c(sel[i]);
    }
    return SWB_OK;
}

int swb_batch_set_rng(swb_batch *b, uint32_t id, const uint32_t *state, const uint32_t *a, const uint32_t *c,
                      const uint32_t *iteration)
{
    HostLat *h = get_lat(b, id);
    if (!h || !state || !a || !c || !iteration)
        return fail(SWB_ERR_ARGUMENT, "no lattice %u or NULL argument", id);
    if (int rc = bset_device(b))
        return rc;
    const size_t tiles = (size_t)h->d.g.n0 * h->d.g.n1, nw = tiles * b->W;
    std::vector<uint8_t> sel(nw);
    for (size_t i = 0; i < nw; ++i) {
        const int k = lcg_pair_index(a[i], c[i]);
        if (k < 0)
            return fail(SWB_ERR_ARGUMENT, "lane %zu: (a, c) = (%u, %u) is not an lcg32 parameter pair", i, a[i], c[i]);
        sel[i] = (uint8_t)k;
    }
    SWB_CUDA(cudaMemcpyAsync(h->d.rng_state, state, nw * 4, cudaMemcpyHostToDevice, b->stream));
    SWB_CUDA(cudaMemcpyAsync(h->d.rng_sel, sel.data(), nw, cudaMemcpyHostToDevice, b->stream));
    SWB_CUDA(cudaMemcpyAsync(h->d.rng_iter, iteration, tiles * 4, cudaMemcpyHostToDevice, b->stream));
    SWB_CUDA(cudaStreamSynchronize(b->stream));
    return SWB_OK;
}

int swb_batch_info(swb_batch *b, uint32_t id, uint32_t *geometry)
{
    HostLat *h = get_lat(b, id);
    if (!h || !geometry)
        return fail(SWB_ERR_ARGUMENT, "no lattice %u or NULL argument", id);
    const Geo &g = h->d.g;
    const uint32_t v[8] = {g.L0, g.L1, g.TX, g.TY, g.TBX, g.TBY, g.n0 * g.n1, g.nbx * g.nby};
    std::memcpy(geometry, v, sizeof(v));
    return SWB_OK;
}

int swb_batch_memory(swb_batch *b, uint64_t *used, uint64_t *budget)
{
    if (!b)
        return fail(SWB_ERR_ARGUMENT, "NULL handle");
    if (used) *used = b->used;
    if (budget) *budget = b->budget;
    return SWB_OK;
}

}  // extern "C"

namespace {

// n_rounds rounds through host buffers: round r copies spins in from side r % 2 (0: spins_in,
// 1: spins_out), sweeps every lattice once and copies the spins out to the other side.
int update_host_rounds(swb_batch *b, uint32_t count, const uint32_t *ids, const uint8_t *const *spins_in,
                       uint8_t *const *spins_out, const uint32_t n_rounds)
{
    if (!b || (count && (!ids || !spins_in || !spins_out)))
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (int rc = bset_device(b))
        return rc;
    if (n_rounds == 0)
        return SWB_OK;
    if (count == 0) {
        if (int rc = rounds(b, n_rounds, false))
            return rc;
        SWB_CUDA(cudaStreamSynchronize(b->stream));
        return SWB_OK;
    }
    // The listed lattices' spins travel through one contiguous device staging buffer, in
    // groups of about equal bytes that form a pipeline: group g's host-to-device copies (one
    // per run of host buffers that follow each other in memory) overlap the sweep of group
    // g - 1 and the device-to-host copies of group g - 2, on three streams.  Lattices that are
    // not listed are swept first, while the first group's spins are still on their way.  Over
    // several rounds the pipeline runs on without a host synchronisation: group g's copies in
    // for round r wait only for its copies out of round r - 1 (the host buffers they read and
    // the staging bytes they overwrite).
    if (int rc = rebuild_lists(b))
        return rc;
    auto &P = b->io;
    const bool same = P.version == b->lists_version && P.ids.size() == count &&
                      std::equal(P.ids.begin(), P.ids.end(), ids);
    if (!same) {
        std::vector<bool> listed(b->capacity, false);
        std::vector<StageCopy> copies(count);
        uint64_t total = 0;
        for (uint32_t k = 0; k < count; ++k) {
            HostLat *h = get_lat(b, ids[k]);
            if (!h)
                return fail(SWB_ERR_ARGUMENT, "no lattice %u", ids[k]);
            if (listed[ids[k]])
                return fail(SWB_ERR_ARGUMENT, "lattice %u listed twice", ids[k]);
            listed[ids[k]] = true;
            copies[k].spins = h->d.spins;
            copies[k].offset = total;
            copies[k].bytes = (uint64_t)h->d.g.L0 * h->d.g.L1;
            total += copies[k].bytes;
        }
        // groups [gs[g], gs[g + 1]) of listed lattices and their block items; the unlisted
        // active lattices' items come first
        constexpr uint32_t kGroups = 8;  // measured on the 512-lattice mix: 6 to 8 groups beat 2, 4, 10, 12 and 16
        const uint32_t G = std::min(count, kGroups);
        std::vector<uint32_t> gs(G + 1, count);
        gs[0] = 0;
        for (uint32_t g = 1, k = 0; g < G; ++g) {
            const uint64_t target = total * g / G;
            while (k < count && copies[k].offset + copies[k].bytes <= target)
                ++k;
            gs[g] = std::min(std::max(k, gs[g - 1] + 1), count - (G - g));  // every group keeps a lattice
        }
        std::vector<uint2> items;
        auto push_items = [&](uint32_t id) {
            const Geo &g = b->lats[id].d.g;
            for (uint32_t by = 0; by < g.nby; ++by)
                for (uint32_t bx = 0; bx < g.nbx; ++bx)
                    items.push_back(make_uint2(id, by << 16 | bx));
        };
        for (uint32_t id : b->active)
            if (!listed[id])
                push_items(id);
        std::vector<size_t> gi(G + 2, 0);
        gi[1] = items.size();
        for (uint32_t g = 0; g < G; ++g) {
            for (uint32_t k = gs[g]; k < gs[g + 1]; ++k)
                push_items(ids[k]);
            gi[g + 2] = items.size();
        }
        if (total > b->stage_cap || count > b->copies_cap || items.size() > b->io_items_cap) {
            SWB_CUDA(cudaStreamSynchronize(b->stream));
            if (total > b->stage_cap) {
                SWB_CUDA(cudaFree(b->d_stage));
                b->d_stage = nullptr;
                SWB_CUDA(cudaMalloc(&b->d_stage, total));
                b->stage_cap = total;
            }
            if (count > b->copies_cap) {
                SWB_CUDA(cudaFree(b->d_copies));
                b->d_copies = nullptr;
                SWB_CUDA(cudaMalloc(&b->d_copies, sizeof(StageCopy) * count));
                b->copies_cap = count;
            }
            if (items.size() > b->io_items_cap) {
                SWB_CUDA(cudaFree(b->d_io_items));
                b->d_io_items = nullptr;
                SWB_CUDA(cudaFree(b->d_io_recs));
                b->d_io_recs = nullptr;
                SWB_CUDA(cudaMalloc(&b->d_io_items, sizeof(uint2) * items.size()));
                SWB_CUDA(cudaMalloc(&b->d_io_recs, sizeof(BlockRec) * items.size()));
                b->io_items_cap = items.size();
            }
        }
        P.version = ~0ull;  // valid again only once the uploads below are queued
        SWB_CUDA(cudaMemcpyAsync(b->d_copies, copies.data(), sizeof(StageCopy) * count, cudaMemcpyHostToDevice,
                                 b->stream));
        SWB_CUDA(cudaMemcpyAsync(b->d_io_items, items.data(), sizeof(uint2) * items.size(), cudaMemcpyHostToDevice,
                                 b->stream));
        const std::vector<BlockRec> recs = make_recs(b, items);
        SWB_CUDA(cudaMemcpyAsync(b->d_io_recs, recs.data(), sizeof(BlockRec) * recs.size(), cudaMemcpyHostToDevice,
                                 b->stream));
        P.ids.assign(ids, ids + count);
        P.gs = std::move(gs);
        P.gi = std::move(gi);
        P.copies = std::move(copies);
        P.total = total;
        P.max_bytes.assign(P.gs.size() - 1, 0);
        for (size_t q = 0; q + 1 < P.gs.size(); ++q)
            for (uint32_t k = P.gs[q]; k < P.gs[q + 1]; ++k)
                P.max_bytes[q] = std::max<uint64_t>(P.max_bytes[q], P.copies[k].bytes);
        P.version = b->lists_version;
    }
    const uint32_t G = (uint32_t)P.gs.size() - 1;
    const auto &gs = P.gs;
    const auto &gi = P.gi;
    const auto &copies = P.copies;
    if (!b->s_in)
        SWB_CUDA(cudaStreamCreateWithFlags(&b->s_in, cudaStreamNonBlocking));
    if (!b->s_out)
        SWB_CUDA(cudaStreamCreateWithFlags(&b->s_out, cudaStreamNonBlocking));
    while (b->io_events.size() < 3 * G) {  // [g]: group g staged; [G + g]: swept; [2G + g]: copied out
        cudaEvent_t e;
        SWB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        b->io_events.push_back(e);
    }
    cudaEvent_t *ev = b->io_events.data();
    auto run = [&]() -> int {
        for (uint32_t r = 0; r < n_rounds; ++r) {
            const uint8_t *const *src = (r & 1) ? spins_out : spins_in;
            uint8_t *const *dst = (r & 1) ? const_cast<uint8_t *const *>(spins_in) : spins_out;
            kb_begin_round<<<4, 128, 0, b->stream>>>(b->d_lats, b->d_active, b->d_ctr);
            SWB_LAUNCHED();
            if (gi[1])
                if (int rc = launch_phases_b(b, b->d_io_items, b->d_io_recs, (uint32_t)gi[1], b->stream))
                    return rc;
            for (uint32_t g = 0; g < G; ++g) {
                if (r)  // the previous round's copies out of this group have landed
                    SWB_CUDA(cudaStreamWaitEvent(b->s_in, ev[2 * G + g], 0));
                for (uint32_t k = gs[g]; k < gs[g + 1];) {
                    uint32_t j = k + 1;
                    while (j < gs[g + 1] && src[j] == src[j - 1] + copies[j - 1].bytes)
                        ++j;
                    SWB_CUDA(cudaMemcpyAsync(b->d_stage + copies[k].offset, src[k],
                                             copies[j - 1].offset + copies[j - 1].bytes - copies[k].offset,
                                             cudaMemcpyHostToDevice, b->s_in));
                    k = j;
                }
                SWB_CUDA(cudaEventRecord(ev[g], b->s_in));
            }
            for (uint32_t g = 0; g < G; ++g) {
                const uint32_t n = gs[g + 1] - gs[g];
                SWB_CUDA(cudaStreamWaitEvent(b->stream, ev[g], 0));
                const dim3 sgrid((uint32_t)((P.max_bytes[g] + kStagePiece - 1) / kStagePiece), n);
                kb_stage_copy<<<sgrid, 256, 0, b->stream>>>(b->d_copies + gs[g], b->d_stage, 1);
                SWB_LAUNCHED();
                if (int rc = launch_phases_b(b, b->d_io_items + gi[g + 1], b->d_io_recs + gi[g + 1],
                                             (uint32_t)(gi[g + 2] - gi[g + 1]), b->stream))
                    return rc;
                kb_stage_copy<<<sgrid, 256, 0, b->stream>>>(b->d_copies + gs[g], b->d_stage, 0);
                SWB_LAUNCHED();
                if (g + 1 == G) {  // every listed and unlisted lattice has swept: close the round
                    if (int rc = launch_end_round(b, b->stream, false))
                        return rc;
                    b->round_count += 1;
                }
                SWB_CUDA(cudaEventRecord(ev[G + g], b->stream));
                SWB_CUDA(cudaStreamWaitEvent(b->s_out, ev[G + g], 0));
                for (uint32_t k = gs[g]; k < gs[g + 1];) {
                    uint32_t j = k + 1;
                    while (j < gs[g + 1] && dst[j] == dst[j - 1] + copies[j - 1].bytes)
                        ++j;
                    SWB_CUDA(cudaMemcpyAsync(dst[k], b->d_stage + copies[k].offset,
                                             copies[j - 1].offset + copies[j - 1].bytes - copies[k].offset,
                                             cudaMemcpyDeviceToHost, b->s_out));
                    k = j;
                }
                SWB_CUDA(cudaEventRecord(ev[2 * G + g], b->s_out));
            }
        }
        SWB_CUDA(cudaStreamSynchronize(b->s_out));
        SWB_CUDA(cudaStreamSynchronize(b->s_in));
        SWB_CUDA(cudaStreamSynchronize(b->stream));
        return SWB_OK;
    };
    const int rc = run();
    if (rc) {  // leave no copy in flight behind an error
        cudaStreamSynchronize(b->s_in);
        cudaStreamSynchronize(b->s_out);
        cudaStreamSynchronize(b->stream);
    }
    return rc ? rc : bcheck_fault(b);
}

}  // namespace

extern "C" {

int swb_batch_update_host(swb_batch *b, uint32_t count, const uint32_t *ids, const uint8_t *const *spins_in,
                          uint8_t *const *spins_out)
{
    return update_host_rounds(b, count, ids, spins_in, spins_out, 1);
}

int swb_batch_update_host_rounds(swb_batch *b, uint32_t count, const uint32_t *ids, uint8_t *const *spins_a,
                                 uint8_t *const *spins_b, uint32_t n_rounds)
{
    return update_host_rounds(b, count, ids, spins_a, spins_b, n_rounds);
}

}  // extern "C"
