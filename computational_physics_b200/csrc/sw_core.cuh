// Shared device code of the Swendsen-Wang engine: lattice geometry, the per-block assign
// phase (lcg32 draws, bonds, shared-memory union-find) and the per-block edge merge.  Used by
// the single-lattice kernels (sw_plain.cu) and the batched kernels (sw_batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <string>
#include <utility>

#include "../../include/swb200.h"
#include "sw_device.cuh"

namespace swb {

// ------------------------------------------------------------------------------------------
// errors and launch accounting (defined in sw_plain.cu)

extern thread_local std::string g_last_error;
extern std::atomic<uint64_t> g_launches;
int fail(int code, const char *fmt, ...);

// swb_sweep_static's scratch: one file-scope device array (sw_static_scratch.cu) holding the
// label array, the block edge words and the fault word of a lattice of at most 2048 x 2048 sites.
constexpr uint64_t kStaticMaxSites = 1ull << 22;               // 2048 x 2048 sites
constexpr size_t kStaticScratchBytes = (24ull << 20) + 1024;   // labels 16 MiB + edge words + fault
// Device address of that array on `device`, which must be current (looked up once per device).
int static_scratch_base(int device, unsigned char **base);

#define SWB_CUDA(call)                                                                          \
    do {                                                                                        \
        cudaError_t err__ = (call);                                                             \
        if (err__ != cudaSuccess)                                                               \
            return ::swb::fail(SWB_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(err__)); \
    } while (0)

#define SWB_LAUNCHED()                                                                           \
    do {                                                                                         \
        ::swb::g_launches.fetch_add(1, std::memory_order_relaxed);                               \
        cudaError_t err__ = cudaGetLastError();                                                  \
        if (err__ != cudaSuccess)                                                                \
            return ::swb::fail(SWB_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(err__)); \
    } while (0)

// ------------------------------------------------------------------------------------------
// geometry

struct Geo {
    uint32_t L0, L1;    // extent
    uint32_t TX, TY;    // tile
    uint32_t TBX, TBY;  // tiles per block
    uint32_t BX, BY;    // block in sites
    uint32_t n0, n1;    // tiles per direction
    uint32_t nbx, nby;  // blocks per direction
};

// Tiles per block: blocks of up to 128 x 32 sites, at most 1024 threads (one per lcg lane).
// tbx / tby (tiles per block) of 0 pick the largest block within 128 x 32 sites and
// max_threads threads; explicit values are clamped to those limits.
inline Geo make_geo(uint32_t L0, uint32_t L1, uint32_t TX, uint32_t TY, uint32_t W, uint32_t max_threads = 1024,
                    uint32_t tbx = 0, uint32_t tby = 0)
{
    Geo g{};
    g.L0 = L0; g.L1 = L1; g.TX = TX; g.TY = TY;
    g.n0 = (L0 + TX - 1) / TX;
    g.n1 = (L1 + TY - 1) / TY;
    g.TBX = 128 / TX;
    g.TBY = TY >= 32 ? 1 : 32 / TY;
    if (tbx && tbx < g.TBX)
        g.TBX = tbx;
    if (tby && tby < g.TBY)
        g.TBY = tby;
    while (g.TBX * g.TBY * W > max_threads && g.TBY > 1)
        g.TBY /= 2;
    while (g.TBX * g.TBY * W > max_threads && g.TBX > 1)
        g.TBX /= 2;
    // Do not make blocks larger than the lattice needs.
    while (g.TBX > 1 && (g.TBX / 2) * TX >= L0)
        g.TBX /= 2;
    while (g.TBY > 1 && (g.TBY / 2) * TY >= L1)
        g.TBY /= 2;
    g.BX = g.TBX * TX;
    g.BY = g.TBY * TY;
    g.nbx = (L0 + g.BX - 1) / g.BX;
    g.nby = (L1 + g.BY - 1) / g.BY;
    return g;
}

// Updates Ks... of a sweep as straight-line code, the rotation before every update k with
// k % 15 == kFirst (the rotating updates of a warp whose tiles share their iteration count).
template <uint32_t kFirst, uint32_t... Ks, class Rotate, class Draw>
__device__ __forceinline__ void draw_sequence(std::integer_sequence<uint32_t, Ks...>, Rotate &rotate, Draw &draw,
                                              const uint32_t it)
{
    ((Ks % kShuffleDistance == kFirst ? rotate(it + Ks + 1, true) : (void)0, draw(Ks)), ...);
}

template <uint32_t V>
struct U32 {  // a compile-time uint32_t passed as a value
    static constexpr uint32_t value = V;
};

constexpr uint32_t kMaxGridY = 65535;  // block rows of a lattice: the kernels' grid y
constexpr uint32_t kEdgeWords = 8;  // per block: [0] right edge rows, [1..4] bottom edge columns
constexpr uint32_t kEdgeE = 6, kEdgeM = 7;  // shared-memory copies of words 6, 7: the block's energy / magnetisation sums

// Label encoding between the assign and flip phases of a sweep.  A block root holds its global
// site index (< 2^31); these are the only entries the merge reads and links.  Every other site
// holds kLocalFlag | the block-local index (yl * BX + xl) of its root, which needs no division
// to resolve and marks the site as a non-root.  Resolved labels (global) are written only by a
// recorded sweep.
constexpr uint32_t kLocalFlag = 0x80000000u;
constexpr uint32_t kLocalMask = 0x0000FFFFu;

// Global site index of a label read at a site of block (bxi, byi).
__device__ __forceinline__ uint32_t label_global(const Geo &g, uint32_t bxi, uint32_t byi, uint32_t v)
{
    if (!(v & kLocalFlag))
        return v;
    const uint32_t r = v & kLocalMask;
    // BX is a power of two unless the caller chose the block shape
    const uint32_t yl = (g.BX & (g.BX - 1)) == 0 ? r >> (__ffs(g.BX) - 1) : r / g.BX;
    return (byi * g.BY + yl) * g.L0 + bxi * g.BX + (r - yl * g.BX);
}

// Observables.  Per-sweep integer sums land in obs->e / obs->m; the last CTA turns them into
// E/N, M/N, accumulates E, E^2, |M| in FP64 and appends (e, m) to the sample series.
struct Obs {
    unsigned long long e, m;       // running int64 sums (two's complement) of this measurement
    unsigned int done;             // CTAs finished
    unsigned int pad;
    long long last_e, last_m;      // sums of the last measurement
    double acc[4];                 // sum E/N, sum (E/N)^2, sum |M/N|, samples
    unsigned long long n_samples;  // samples recorded (may exceed capacity)
};

// LCG32_State<W>::Init (random/src/lcg32.cpp:27-49) of tile t = this thread, seeded seed_base + t:
// drand48 draws pick each lane's (a, c) pair and the first lane's start, the others follow from
// it.  The two double multiplications are rounded as the host's (__dmul_rn).
template <int W>
__device__ __forceinline__ void rng_init_tile(const uint32_t n_tiles, const uint32_t seed_base, uint32_t *state,
                                              uint8_t *sel, uint32_t *iter)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tiles)
        return;
    uint64_t x = drand48_seed(seed_base + t);
    uint32_t s[W];
#pragma unroll
    for (int i = 0; i < W; ++i) {
        x = drand48_step(x);
        s[i] = ((uint32_t)__dmul_rn(1000.0, drand48_value(x))) % 5u;
        sel[(size_t)t * W + i] = (uint8_t)s[i];
    }
    x = drand48_step(x);
    uint32_t v = lcg_param_a(s[0]) * ((uint32_t)__dmul_rn(4026531839.0, drand48_value(x)) + 1u) + lcg_param_c(s[0]);
    state[(size_t)t * W] = v;
#pragma unroll
    for (int i = 1; i < W; ++i) {
        v = lcg_param_a(s[i]) * v + lcg_param_c(s[i]);
        state[(size_t)t * W + i] = v;
    }
    iter[t] = 0;
}

// Hot start of Lattice<2> (ising/src/lattice.cpp:15-27), one 64-site chunk per thread: site i
// takes drand48 draw i + 1 after srand48(seed); drand48() < 0.5 iff bit 47 of the 48-bit state is
// clear.  The chunk's first state comes by jump-ahead; whole chunks store 8 sites at a time.
__device__ __forceinline__ void hot_start_chunk(const size_t n, const uint32_t seed, uint8_t *spins)
{
    constexpr uint32_t kChunk = 64;
    const size_t first = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * kChunk;
    if (first >= n)
        return;
    uint64_t A, C;
    drand48_jump(first, A, C);
    uint64_t x = (A * drand48_seed(seed) + C) & kDrandMask;
    const size_t last = first + kChunk < n ? first + kChunk : n;
    if (last - first == kChunk && (reinterpret_cast<uintptr_t>(spins) & 7u) == 0) {
#pragma unroll
        for (uint32_t q = 0; q < kChunk / 8; ++q) {
            uint64_t v = 0;
#pragma unroll
            for (uint32_t k = 0; k < 8; ++k) {
                x = drand48_step(x);
                v |= (x >> 47) << (8 * k);
            }
            reinterpret_cast<uint64_t *>(spins + first)[q] = v;
        }
        return;
    }
    for (size_t i = first; i < last; ++i) {
        x = drand48_step(x);
        spins[i] = (uint8_t)(x >> 47);
    }
}

// One part of a measurement: adds this part's integer sums (e = sum s (s_right + s_down),
// m = sum s over its sites) and, if it is the last of n_parts, turns the totals into E/N and
// M/N, accumulates E, E^2, |M| in FP64 (with accumulate), appends (e, m) to the series and
// clears the sums for the next measurement.  Called by one thread per part.
__device__ __forceinline__ void obs_add_part(Obs *obs, long long *series, const unsigned long long cap, const size_t n,
                                             const unsigned int n_parts, const long long e, const long long m,
                                             const int accumulate)
{
    atomicAdd(&obs->e, (unsigned long long)e);
    atomicAdd(&obs->m, (unsigned long long)m);
    __threadfence();
    const unsigned int ticket = atomicAdd(&obs->done, 1u);
    if (ticket == n_parts - 1) {
        __threadfence();
        const long long te = (long long)atomicAdd(&obs->e, 0ull);
        const long long tm = (long long)atomicAdd(&obs->m, 0ull);
        obs->last_e = te;
        obs->last_m = tm;
        if (accumulate) {
            const double E = -(double)te / (double)n, M = (double)tm / (double)n;
            obs->acc[0] += E;
            obs->acc[1] += E * E;
            obs->acc[2] += fabs(M);
            obs->acc[3] += 1.0;
            const unsigned long long k = obs->n_samples;
            if (k < cap) {
                series[2 * k] = te;
                series[2 * k + 1] = tm;
            }
            obs->n_samples = k + 1;
        }
        obs->e = 0;
        obs->m = 0;
        obs->done = 0;
    }
}

// A measurement of the spins a sweep starts from, made by its assign phase (obs null: none).
// The blocks of the sweep are its parts.
struct MeasureArgs {
    Obs *obs;
    long long *series;
    unsigned long long cap;
};

// Optional dumps of the assign phase to device buffers (one entry per site, row-major).  All
// null in a plain sweep; set by the recording entry points.  bonds: bit 0 +x, bit 1 +y (every
// bond of the sweep, block edges and the periodic wrap included); block_labels: the minimum
// global site index of the site's component over the bonds inside its block (the labels the
// assign phase hands to the merge); tile_labels: the same inside the site's tile (the
// reference's AssignLabels stage), which only the tile-by-tile form below computes.
struct AssignDump {
    uint8_t *bonds;
    uint32_t *block_labels;
    uint32_t *tile_labels;
};

struct AssignSmem {
    uint32_t parent, draws, slots, edge, bond, sp, plab, pairs, total, pitch;
};

// Pending unions of the scanline labelling (row path): 2048 words shared by the CTA's warps
// (64 per warp at 1024 threads, 128 at 512), one uint16 pair per word.
constexpr uint32_t kPairWords = 2048;

// Updates of every lcg32 lane in one sweep: 2 tile_y - 1 row requests of tile_x numbers and
// the merge request of tile_x + tile_y numbers, W numbers per update.
__host__ __device__ inline uint32_t draw_slots(const Geo &g, uint32_t W)
{
    return (2 * g.TY - 1) * ((g.TX + W - 1) / W) + (g.TX + g.TY + W - 1) / W;
}

__host__ __device__ inline AssignSmem assign_smem(const Geo &g, uint32_t W)
{
    AssignSmem s{};
    const uint32_t ns = g.BX * g.BY, ntb = g.TBX * g.TBY;
    s.pitch = g.BX + 16;  // rows 16-byte aligned for cp.async
    s.slots = draw_slots(g, W);
    s.parent = 0;
    s.draws = s.parent + ns * 4;                                  // [warp][slot] ballot words
    s.edge = s.draws + ((ntb * W + 31) / 32) * s.slots * 4;
    s.bond = s.edge + kEdgeWords * 4;
    s.sp = (s.bond + ns + 15) & ~15u;
    s.plab = (s.sp + (g.BY + 1) * s.pitch + 15) & ~15u;  // uint16 provisional labels (row path)
    s.pairs = (s.plab + 2 * ns + 15) & ~15u;
    s.total = s.pairs + kPairWords * 4;
    return s;
}

// The largest assign_smem of any tile shape with lcg width W (blocks are at most 128 x 32
// sites, so a 128 x 32 lattice has the largest block of each shape).
inline uint32_t assign_smem_max(uint32_t W, uint32_t max_threads)
{
    uint32_t m = 0;
    for (uint32_t tx = 8; tx <= 32; tx *= 2)
        for (uint32_t ty = 2; ty <= 32; ++ty) {
            const uint32_t t = assign_smem(make_geo(128, 32, tx, ty, W, max_threads), W).total;
            m = t > m ? t : m;
        }
    return m;
}

// Accepted draws of a block's tiles, read back from the warps' ballot words: bit k of a request
// word is element k of the request.  Tile tb's lanes are bits (tb * W) % 32 .. + W of warp
// (tb * W) / 32's words; a request starting at update u spans updates u .. u + ceil(n / W).
template <int W>
struct DrawWords {
    const uint32_t *d;
    uint32_t slots;
    __device__ __forceinline__ uint32_t seg(uint32_t tb, uint32_t u) const
    {
        const uint32_t v = d[((tb * W) >> 5) * slots + u] >> ((tb * W) & 31);
        return W == 32 ? v : v & ((1u << (W & 31)) - 1u);
    }
    // elements [0, ur * W) of the request at update u (ur * W <= 32)
    __device__ __forceinline__ uint32_t req(uint32_t tb, uint32_t u, uint32_t ur) const
    {
        uint32_t v = seg(tb, u);
        for (uint32_t s = 1; s < ur; ++s)
            v |= seg(tb, u + s) << (s * W);
        return v;
    }
    // element k of the request at update u
    __device__ __forceinline__ uint32_t bit(uint32_t tb, uint32_t u, uint32_t k) const
    {
        return (seg(tb, u + k / W) >> (k % W)) & 1u;
    }
};

// ------------------------------------------------------------------------------------------
// kernels

// Bit k of the result = bit 0 of byte k of v: multiplying the masked bytes by
// 2^28 + 2^21 + 2^14 + 2^7 lands byte k's bit at bit 28 + k, every cross term below bit 28.
__device__ __forceinline__ uint32_t spin_nibble(uint32_t v)
{
    return ((v & 0x01010101u) * 0x10204080u) >> 28;
}

// Bit k = staged spin byte p[k] (0/1) for k < 32; p is 16-byte aligned in shared memory.
__device__ __forceinline__ uint32_t spin_bits32(const uint8_t *p)
{
    const uint4 a = *reinterpret_cast<const uint4 *>(p), b = *reinterpret_cast<const uint4 *>(p + 16);
    return spin_nibble(a.x) | spin_nibble(a.y) << 4 | spin_nibble(a.z) << 8 | spin_nibble(a.w) << 12 |
           spin_nibble(b.x) << 16 | spin_nibble(b.y) << 20 | spin_nibble(b.z) << 24 | spin_nibble(b.w) << 28;
}

// Energy / magnetisation sums of the `cnt` sites x0 .. x0 + cnt - 1 of row y of an L0 x L1
// periodic lattice: e = sum s (s_right + s_down), m = sum s, s = 2 b - 1.  Rows 16-byte aligned
// (L0 % 16 == 0) and 16-site aligned pieces go 16 sites at a time through bit masks (two 16-byte
// loads, the byte after them, popcounts); anything else site by site.  No per-site division.
__device__ __forceinline__ void row_em(const uint8_t *__restrict__ spins, const uint32_t L0, const uint32_t L1,
                                       const uint32_t y, uint32_t x0, uint32_t cnt, int &e, int &m)
{
    const uint8_t *row = spins + (size_t)y * L0, *down = spins + (size_t)(y + 1 == L1 ? 0 : y + 1) * L0;
    if ((L0 & 15u) == 0) {
        for (; cnt >= 16 && (x0 & 15u) == 0; x0 += 16, cnt -= 16) {
            const uint4 a = *reinterpret_cast<const uint4 *>(row + x0), d = *reinterpret_cast<const uint4 *>(down + x0);
            const uint32_t S = spin_nibble(a.x) | spin_nibble(a.y) << 4 | spin_nibble(a.z) << 8 | spin_nibble(a.w) << 12;
            const uint32_t D = spin_nibble(d.x) | spin_nibble(d.y) << 4 | spin_nibble(d.z) << 8 | spin_nibble(d.w) << 12;
            const uint32_t R = (S >> 1) | ((uint32_t)row[x0 + 16 == L0 ? 0 : x0 + 16] << 15);
            e += 32 - 2 * (__popc(S ^ R) + __popc(S ^ D));
            m += 2 * __popc(S) - 16;
        }
    }
    for (; cnt; ++x0, --cnt) {
        const int v = 2 * row[x0] - 1;
        e += v * ((2 * row[x0 + 1 == L0 ? 0 : x0 + 1] - 1) + (2 * down[x0] - 1));
        m += v;
    }
}

// Labelling of a block whose width is a multiple of 32, from the staged spins (sp) and the
// accepted draws in shared memory: bond bitmasks per 32-site word, then a scanline pass over
// x-runs (below).  The result equals the generic path's: the minimum site index of each
// block-local component.
// Bond words of block (bxi, byi) into shared memory: Xw / Yw [BY][NW] hold the x- and y-bonds
// inside the block, edge_s the bonds that leave it through its last column (word 0, one bit
// per row) and its last row (words 1..NW).  Needs the staged spins and the draw words.
template <int W, int TXc, int TYc>
__device__ __forceinline__ void block_bond_words(const Geo &g, const uint32_t bxi, const uint32_t byi,
                                                 const bool measure, const AssignSmem &L, unsigned char *smem)
{
    const uint32_t TX = TXc ? TXc : g.TX, TY = TYc ? TYc : g.TY;  // compile-time for the common tiles
    const uint32_t Ur = (TX + W - 1) / W, um = (2 * TY - 1) * Ur;  // updates per row request; merge request
    const DrawWords<W> dw{reinterpret_cast<const uint32_t *>(smem + L.draws), L.slots};
    uint32_t *edge_s = reinterpret_cast<uint32_t *>(smem + L.edge);
    const uint8_t *sp = smem + L.sp;
    const uint32_t BX = g.BX, BY = g.BY, NW = BX >> 5, lnw = __ffs(NW) - 1;  // NW is a power of two
    uint32_t *Xw = reinterpret_cast<uint32_t *>(smem + L.bond);
    uint32_t *Yw = Xw + BY * NW;
    const uint32_t tid = threadIdx.x;
    const uint32_t x0 = bxi * BX, y0 = byi * BY;
    const uint32_t bxv = min(BX, g.L0 - x0), byv = min(BY, g.L1 - y0);
    const uint32_t pitch = L.pitch;
    const uint32_t txs = TXc ? (TXc == 8 ? 3 : TXc == 16 ? 4 : 5) : 31 - __clz(TX);  // TX is 8, 16 or 32
    (void)x0; (void)y0;

    // Bond words, bit-parallel: one thread per 32-site word of a row.  Spin bits come from the
    // staged bytes (the word, the word below and the byte to its right: the halo column and
    // row are staged at column bxv and row byv); a bond needs equal spins and an accepted draw.
    // Accept bits per tile: x bonds [0, iimax - 1) from the row's x request, the tile's last
    // column from the merge request's right edge (bit TX + jj); y bonds from the row's y request,
    // or on the tile's last row from the merge request's bottom edge (bits [0, TX)).  Edge bonds
    // go to edge_s (right edge: one bit per row, bottom: the row's words).
    int esum = 0, msum = 0;  // energy / magnetisation of this thread's words (the spins before the flip)
    for (uint32_t i = tid; i < BY * NW; i += blockDim.x) {
        const uint32_t yl = i >> lnw, w = i & (NW - 1);
        uint32_t X = 0, Y = 0;
        if (yl < byv) {
            const uint32_t tby = yl / TY, jj = yl - tby * TY;
            const uint32_t jjmax = min(TY, byv - tby * TY);
            const uint8_t *row = sp + yl * pitch + (w << 5);
            const uint32_t S = spin_bits32(row), D = spin_bits32(row + pitch);
            const uint32_t R = __funnelshift_r(S, (uint32_t)row[32], 1);  // right neighbours
            uint32_t AX = 0, AY = 0;
            constexpr uint32_t kTiles = TXc ? 32 / TXc : 4;
            const uint32_t tiles = TXc ? kTiles : 32 >> txs;
#pragma unroll
            for (uint32_t k = 0; k < kTiles; ++k) {
                const uint32_t c0 = (w << 5) + (k << txs);  // the tile's first column in the block
                if (k < tiles && c0 < bxv) {
                    const uint32_t tb = tby * g.TBX + (c0 >> txs);
                    const uint32_t iimax = min(TX, bxv - c0);
                    const uint32_t tmask = 0xFFFFFFFFu >> (32 - iimax);
                    const uint32_t xb = (dw.req(tb, jj * Ur, Ur) & (tmask >> 1)) | dw.bit(tb, um, TX + jj) << (iimax - 1);
                    const uint32_t yb = dw.req(tb, jj + 1 < jjmax ? (jjmax + jj) * Ur : um, Ur) & tmask;
                    AX |= xb << (k << txs);
                    AY |= yb << (k << txs);
                }
            }
            X = ~(S ^ R) & AX;
            Y = ~(S ^ D) & AY;
            {   // s (s_right + s_down) and s over the word's sites: +1 per equal pair, -1 per unequal one
                const uint32_t nv = min(32u, bxv > (w << 5) ? bxv - (w << 5) : 0u);
                const uint32_t vm = nv == 32 ? 0xFFFFFFFFu : (1u << nv) - 1u;
                esum += 2 * (int)nv - 2 * (__popc((S ^ R) & vm) + __popc((S ^ D) & vm));
                msum += 2 * __popc(S & vm) - (int)nv;
            }
            if (bxv - 1 - (w << 5) < 32u) {  // the block's last column lies in this word
                const uint32_t bit = (bxv - 1) & 31;
                if ((X >> bit) & 1u)
                    atomicOr(edge_s, 1u << yl);
                X &= ~(1u << bit);
            }
            if (yl + 1 == byv) {
                edge_s[1 + w] = Y;
                Y = 0;
            }
        }
        Xw[yl * NW + w] = X;
        Yw[yl * NW + w] = Y;
    }
    if (measure) {  // warp sums into the block's two shared words (zeroed with the edge words)
        esum = __reduce_add_sync(0xffffffffu, esum);
        msum = __reduce_add_sync(0xffffffffu, msum);
        if ((tid & 31) == 0 && (tid >> 5) < ((BY * NW + 31) >> 5)) {
            atomicAdd(reinterpret_cast<int *>(edge_s + kEdgeE), esum);
            atomicAdd(reinterpret_cast<int *>(edge_s + kEdgeM), msum);
        }
    }
}

// Recording only (after the block's labels are stored and its CTA synchronised): every bond of
// the block's sites, and each site's block-local component as a global site index.
template <int W>
__device__ __forceinline__ void dump_block(const Geo &g, const uint32_t bxi, const uint32_t byi,
                                        const uint32_t *labels, const AssignDump &dump, unsigned char *smem)
{
    const AssignSmem L = assign_smem(g, W);
    const uint32_t *edge_s = reinterpret_cast<const uint32_t *>(smem + L.edge);
    const uint32_t BX = g.BX, BY = g.BY, NW = BX >> 5;
    const uint32_t *Xw = reinterpret_cast<const uint32_t *>(smem + L.bond), *Yw = Xw + BY * NW;
    const uint32_t x0 = bxi * BX, y0 = byi * BY;
    const uint32_t bxv = min(BX, g.L0 - x0), byv = min(BY, g.L1 - y0);
    for (uint32_t i = threadIdx.x; i < bxv * byv; i += blockDim.x) {
        const uint32_t yl = i / bxv, xl = i - yl * bxv, w = xl >> 5, k = xl & 31;
        const size_t site = (size_t)(y0 + yl) * g.L0 + x0 + xl;
        if (dump.bonds) {
            const uint32_t xb = xl + 1 == bxv ? (edge_s[0] >> yl) & 1u : (Xw[yl * NW + w] >> k) & 1u;
            const uint32_t yb = yl + 1 == byv ? (edge_s[1 + w] >> k) & 1u : (Yw[yl * NW + w] >> k) & 1u;
            dump.bonds[site] = (uint8_t)(xb | yb << 1);
        }
        if (dump.block_labels)
            dump.block_labels[site] = label_global(g, bxi, byi, labels[site]);
    }
}

// kBX, kBY, kThreads: the block shape and CTA size as compile-time constants (the common full
// 128 x 32 block of 512 threads: the scanline then runs one band per warp with its rows
// unrolled), or 0 for the runtime shape.
template <int W, int TXc, int TYc, bool kMayDump, int kBX = 0, int kBY = 0, int kThreads = 0>
__device__ __forceinline__ void assign_block_labels_rows(const Geo &g, const uint32_t bxi, const uint32_t byi,
                                                         uint32_t *__restrict__ labels, uint32_t *__restrict__ edge,
                                                         const AssignDump &dump, const MeasureArgs &meas,
                                                         unsigned char *smem)
{
    const AssignSmem L = assign_smem(g, W);
    uint32_t *parent = reinterpret_cast<uint32_t *>(smem + L.parent);
    uint32_t *edge_s = reinterpret_cast<uint32_t *>(smem + L.edge);
    const uint32_t BX = kBX ? kBX : g.BX, BY = kBY ? kBY : g.BY;
    const uint32_t NW = BX >> 5, lnw = __ffs(NW) - 1;             // NW is a power of two
    uint32_t *Xw = reinterpret_cast<uint32_t *>(smem + L.bond);  // [BY][NW] x-bonds inside the block
    uint32_t *Yw = Xw + BY * NW;                                  // [BY][NW] y-bonds inside the block
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t nwarps = kThreads ? kThreads / 32 : blockDim.x >> 5;
    const uint32_t x0 = bxi * BX, y0 = byi * BY;
    const uint32_t bxv = min(BX, g.L0 - x0), byv = min(BY, g.L1 - y0);

    // Every site starts as its own root (16-byte stores; parent is at offset 0 and BX*BY is a
    // multiple of 64).
    for (uint32_t i = tid; i < (BX * BY) >> 2; i += blockDim.x)
        reinterpret_cast<uint4 *>(parent)[i] = make_uint4(4 * i, 4 * i + 1, 4 * i + 2, 4 * i + 3);

    block_bond_words<W, TXc, TYc>(g, bxi, byi, meas.obs != nullptr, L, smem);
    __syncthreads();

    // Scanline labelling.  Work item = (32-column strip, band of rows); a warp walks its band
    // top-down with each lane holding the provisional label of the site above.  A run (x-bonded
    // sites of the strip row; its first lane from the gap mask below the lane) takes the label
    // above its leftmost y-bonded site, or with none its own first site as a new label.  Every
    // other y-bond of the run that meets a different label unites the two in the shared
    // union-find (toward the minimum), so each site's root is the minimum of its block-local
    // component.  Seams between strips and bands are united afterwards, then every site
    // resolves its provisional label.
    uint16_t *plab = reinterpret_cast<uint16_t *>(smem + L.plab);
    const uint32_t nb = max(1u, nwarps >> lnw);              // bands
    const uint32_t rb = (nb & (nb - 1)) == 0 ? (BY + nb - 1) >> (__ffs(nb) - 1)  // rows per band
                                             : (BY + nb - 1) / nb;
    const uint32_t below = (1u << lane) - 1u;                // lanes below this one
    // The unions a band needs are queued in the warp's slice of the pair list and run together,
    // one per lane (a union inside the row step would run, divergent, on almost every row).
    // Deferring them changes no provisional label, and the union-find's roots (each set's
    // minimum) do not depend on the order of the unions.
    const uint32_t pcap = kThreads ? kPairWords / (kThreads / 32) : kPairWords / nwarps;  // >= 64
    uint32_t *pl = reinterpret_cast<uint32_t *>(smem + L.pairs) + warp * pcap;
    uint32_t npend = 0;  // queued pairs (warp-uniform)
    auto flush = [&]() {
        __syncwarp();
        for (uint32_t i = lane; i < npend; i += 32) {
            const uint32_t pr = pl[i];
            uf_union(parent, pr & 0xFFFFu, pr >> 16);
        }
        __syncwarp();
        npend = 0;
    };
    // One row of a band: `above` holds the provisional label of the site above, Yup the row
    // above's y-bond word, Xa its x-bond word.
    auto row = [&](const uint32_t X, const uint32_t base, uint32_t &above, const uint32_t Yup, const uint32_t Xa) {
        const uint32_t rs = 32 - __clz(~X & below);  // run start (lane); __clz(0) = 32
        // The first y-bond or run end from the run start (bit 31 always ends a strip run):
        // a y-bond there means the run inherits the label above it.
        const uint32_t pos = __ffs((Yup | ~X | 0x80000000u) & (0xFFFFFFFFu << rs)) - 1;
        const uint32_t rep = __shfl_sync(0xffffffffu, above, pos);
        const uint32_t lab = ((Yup >> pos) & 1u) ? rep : base + rs;
        // A y-bond whose left neighbour is bonded up too, with both rows bonded across, meets
        // the same two runs as that neighbour's: only the leftmost of such a chain unites.
        const uint32_t U = Yup & ~((Yup & X & Xa) << 1);
        const bool need = ((U >> lane) & 1u) && above != lab;
        const uint32_t m = __ballot_sync(0xffffffffu, need);
        if (need)
            pl[npend + __popc(m & below)] = above | lab << 16;
        npend += __popc(m);
        if (npend > pcap - 32)  // room for the next row's pairs
            flush();
        plab[base + lane] = (uint16_t)lab;
        above = lab;
    };
    if constexpr (kBX != 0) {
        // one band per warp, its rows unrolled with compile-time offsets
        static_assert(kBX == 128 && kBY == 32 && kThreads == 512, "the fixed shape is one band per warp");
        constexpr uint32_t kNW = kBX / 32, kRows = kBY / ((kThreads / 32) / kNW);
        const uint32_t sx = warp & (kNW - 1), ya = (warp / kNW) * kRows;
        const uint32_t *xp = Xw + ya * kNW + sx;
        const uint32_t base = ya * kBX + (sx << 5);
        uint32_t above = 0, Yup = 0, Xa = 0;
#pragma unroll
        for (uint32_t r = 0; r < kRows; ++r) {
            const uint32_t X = xp[r * kNW];
            row(X, base + r * kBX, above, Yup, Xa);
            Xa = X;
            Yup = xp[kBY * kNW + r * kNW];
        }
        flush();
    } else {
        for (uint32_t task = warp; task < NW * nb; task += nwarps) {
            const uint32_t sx = task & (NW - 1), band = task >> lnw;
            const uint32_t ya = band * rb, yb = min(BY, ya + rb);
            const uint32_t *xp = Xw + ya * NW + sx;  // this row's x-bond word; xp[BY * NW] its y-bond word
            uint32_t base = ya * BX + (sx << 5);
            uint32_t above = 0, Yup = 0, Xa = 0;     // the band's first row has no bonds up
            for (uint32_t n = yb > ya ? yb - ya : 0; n != 0; --n) {
                const uint32_t X = xp[0];
                row(X, base, above, Yup, Xa);
                Xa = X;
                Yup = xp[BY * NW];
                xp += NW;
                base += BX;
            }
            flush();
        }
    }
    __syncthreads();

    // Seams: y-bonds from the last row of a band into the next band (skipping those whose left
    // neighbour already joins the same runs), and x-bonds from a strip's last column into the
    // next strip.
    for (uint32_t task = warp; task < (nb - 1) * NW; task += nwarps) {
        const uint32_t sx = task & (NW - 1), yl = ((task >> lnw) + 1) * rb - 1;
        if (yl + 1 >= BY)
            continue;
        const uint32_t Y = Yw[yl * NW + sx];
        const uint32_t X = Xw[yl * NW + sx], Xb = Xw[(yl + 1) * NW + sx];
        const uint32_t prevT = sx ? ((Yw[yl * NW + sx - 1] & Xw[yl * NW + sx - 1] & Xw[(yl + 1) * NW + sx - 1]) >> 31) : 0u;
        const uint32_t U = Y & ~(((Y & X & Xb) << 1) | prevT);
        if ((U >> lane) & 1u) {
            const uint32_t l = yl * BX + (sx << 5) + lane;
            uf_union(parent, plab[l], plab[l + BX]);
        }
    }
    for (uint32_t i = tid; i < (BY << lnw); i += blockDim.x) {
        const uint32_t yl = i >> lnw, sx = i & (NW - 1);
        if (sx + 1 < NW && (Xw[i] >> 31)) {
            const uint32_t l = yl * BX + (sx << 5) + 31;
            uf_union(parent, plab[l], plab[l + 1]);
        }
    }
    __syncthreads();

    // Labels: a block root stores its global site index (the merge links these), every other
    // site kLocalFlag | the block-local index of its root.
    if ((g.L0 & 3u) == 0) {
        // four sites per thread: one 8-byte load of provisional labels, four independent finds,
        // one 16-byte store (rows and x0 are 16-byte aligned: L0 and BX are multiples of 4)
        const uint32_t nq = BX >> 2, qs = 31 - __clz(nq);
        for (uint32_t i = tid; i < (byv << qs); i += blockDim.x) {
            const uint32_t yl = i >> qs, x4 = (i & (nq - 1)) << 2;
            if (x4 < bxv) {
                const uint32_t l = yl * BX + x4;
                const uint2 pp = *reinterpret_cast<const uint2 *>(plab + l);
                const uint32_t p[4] = {pp.x & 0xFFFFu, pp.x >> 16, pp.y & 0xFFFFu, pp.y >> 16};
                uint32_t r[4];
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    r[k] = uf_find_halve(parent, p[k]);
                const uint32_t gb = (y0 + yl) * g.L0 + x0 + x4;
                uint4 o;
                o.x = r[0] == l ? gb : (kLocalFlag | r[0]);
                o.y = r[1] == l + 1 ? gb + 1 : (kLocalFlag | r[1]);
                o.z = r[2] == l + 2 ? gb + 2 : (kLocalFlag | r[2]);
                o.w = r[3] == l + 3 ? gb + 3 : (kLocalFlag | r[3]);
                *reinterpret_cast<uint4 *>(labels + (size_t)(y0 + yl) * g.L0 + x0 + x4) = o;
            }
        }
    } else {
        for (uint32_t yl = warp; yl < byv; yl += nwarps) {
            uint32_t *row = labels + (size_t)(y0 + yl) * g.L0 + x0;
            for (uint32_t w = 0; w < NW; ++w) {
                const uint32_t xl = (w << 5) + lane;
                if (xl < bxv) {
                    const uint32_t l = yl * BX + xl;
                    const uint32_t r = uf_find_halve(parent, plab[l]);
                    row[xl] = r == l ? (y0 + yl) * g.L0 + x0 + xl : (kLocalFlag | r);
                }
            }
        }
    }
    if (tid < kEdgeWords)
        edge[((size_t)byi * g.nbx + bxi) * kEdgeWords + tid] = edge_s[tid];
    if (meas.obs && tid == 0)  // the block's sums (complete since the barrier after the bond words)
        obs_add_part(meas.obs, meas.series, meas.cap, (size_t)g.L0 * g.L1, g.nbx * g.nby,
                     reinterpret_cast<const int *>(edge_s)[kEdgeE], reinterpret_cast<const int *>(edge_s)[kEdgeM], 1);
    if (kMayDump && (dump.bonds || dump.block_labels)) {  // recording only
        __syncthreads();
        dump_block<W>(g, bxi, byi, labels, dump, smem);
    }
}

// Block (bxi, byi) of a lattice: lcg32 draws, bonds, union-find in shared memory.  Runs on
// all threads of the CTA (at least TBX * TBY * W of them); smem holds assign_smem(g, W).total bytes.
// kPhaseSeq selects the phase-dispatched draw sequence (below) for full-height tiles of a
// compile-time shape: on B200 it is the faster form inside the batched kernel (whose item loop
// keeps more registers live) and the slower one in the single-lattice kernel.
template <int W, int TXc = 0, int TYc = 0, bool kPhaseSeq = false, bool kMayDump = true, bool kFixedShape = false,
          bool kFixedOnly = false>
__device__ __forceinline__ void assign_block(const Geo &g_in, const uint32_t bxi, const uint32_t byi,
                                             const uint8_t *__restrict__ spins, uint32_t *__restrict__ labels,
                                             uint32_t *__restrict__ rng_state, uint8_t *__restrict__ rng_sel,
                                             uint32_t *__restrict__ rng_iter, const uint32_t thr,
                                             uint32_t *__restrict__ edge, const AssignDump dump,
                                             const MeasureArgs meas, unsigned char *smem)
{
    // kFixedOnly: this block is a full 128 x 32 block of 16 x 8 tiles run by 512 threads (the
    // caller checked), so the block and tile shape are constants here: the shared-memory layout
    // folds to immediates and only the fixed-shape paths are compiled (16384^2 assign 1.36 ->
    // 1.32 ms; 512-lattice mix round 0.337 -> 0.330 ms).
    static_assert(!kFixedOnly || (TXc == 16 && TYc == 8 && W == 16 && kFixedShape), "fixed-only is 16 x 8 tiles, W 16");
    Geo gfix = g_in;
    if constexpr (kFixedOnly) {
        gfix.TX = 16;
        gfix.TY = 8;
        gfix.TBX = 8;
        gfix.TBY = 4;
        gfix.BX = 128;
        gfix.BY = 32;
    }
    const Geo &g = kFixedOnly ? gfix : g_in;
    const AssignSmem L = assign_smem(g, W);
    const uint32_t TX = TXc ? TXc : g.TX, TY = TYc ? TYc : g.TY;  // compile-time for the common tiles
    uint32_t *parent = reinterpret_cast<uint32_t *>(smem + L.parent);
    uint32_t *edge_s = reinterpret_cast<uint32_t *>(smem + L.edge);
    uint8_t *bond = smem + L.bond;
    uint8_t *sp = smem + L.sp;

    const uint32_t tid = threadIdx.x, nthr = kFixedOnly ? 512u : blockDim.x;
    const uint32_t BX = g.BX, BY = g.BY, NS = BX * BY, ntb = g.TBX * g.TBY;
    const uint32_t x0 = bxi * BX, y0 = byi * BY;
    const uint32_t bxv = min(BX, g.L0 - x0), byv = min(BY, g.L1 - y0);
    const uint32_t pitch = L.pitch;

    if (tid < kEdgeWords)
        edge_s[tid] = 0;

    // ---- 1. spins of the block and its halo (column x0+bxv and row y0+byv, periodic).  Rows
    // go global -> shared by cp.async, in flight while the lcg32 draws below run; the strided
    // halo column is one byte per thread, held in a register until then.
    const uint32_t hx = x0 + bxv < g.L0 ? x0 + bxv : 0u;  // column right of the block (periodic)
    uint8_t halo = 0;
    {
        const uint32_t warp = tid >> 5, lane32 = tid & 31, nwarps = nthr >> 5;
        const uint32_t hy = y0 + byv < g.L1 ? y0 + byv : 0u;  // row below the block (periodic)
        const uint32_t vec = (g.L0 % 16 == 0 && BX % 16 == 0) ? 16 : (g.L0 % 4 == 0 ? 4 : 1);
        if (kFixedOnly || (vec == 16 && (BX & (BX - 1)) == 0)) {
            // one 16-byte copy per thread, rows packed across the CTA (a 128-wide row is 8
            // copies, so a warp moves 4 rows at once)
            const uint32_t nv = BX >> 4, vs = 31 - __clz(nv);
            for (uint32_t i = tid; i < ((byv + 1) << vs); i += nthr) {
                const uint32_t yl = i >> vs, v = i & (nv - 1);
                if (v * 16 < bxv) {
                    const uint32_t gy = yl < byv ? y0 + yl : hy;
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(
                                     (uint32_t)__cvta_generic_to_shared(sp + yl * pitch + 16 * v)),
                                 "l"(spins + (size_t)gy * g.L0 + x0 + 16 * v));
                }
            }
        } else {
            for (uint32_t yl = warp; yl <= byv; yl += nwarps) {
                const uint32_t gy = yl < byv ? y0 + yl : hy;
                const uint8_t *row = spins + (size_t)gy * g.L0 + x0;
                uint8_t *dst = sp + yl * pitch;
                if (vec == 16) {
                    for (uint32_t v = lane32; v * 16 < bxv; v += 32)
                        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(
                                         (uint32_t)__cvta_generic_to_shared(dst + 16 * v)),
                                     "l"(row + 16 * v));
                } else if (vec == 4) {
                    for (uint32_t v = lane32; v * 4 < bxv; v += 32)
                        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(
                                         (uint32_t)__cvta_generic_to_shared(dst + 4 * v)),
                                     "l"(row + 4 * v));
                } else {
                    for (uint32_t x = lane32; x < bxv; x += 32)
                        dst[x] = __ldg(row + x);
                }
            }
        }
        if (tid < byv)
            halo = __ldg(spins + (size_t)(y0 + tid) * g.L0 + hx);
    }

    // ---- 2. lcg32 draws of this sweep, one W-lane segment per tile.  Every update's ballot of
    // the accept bits (the whole warp's) goes to shared memory as it is, one word per warp and
    // update; DrawWords reads a tile's requests back.  Row request r (tile_x numbers, x rows
    // then y rows; element k is lane k % W after update k / W + 1 of the request) starts at
    // update r * Ur, the merge request (tile_x + tile_y numbers: bottom edge, then right edge)
    // at update (2 tile_y - 1) * Ur; a tile shorter than tile_y idles through the rows it lacks.
    {
        const uint32_t tb = tid / W, lane = tid % W, lane32 = tid & 31;
        // TBX is a power of two unless the caller chose the block shape
        const uint32_t tbr = (g.TBX & (g.TBX - 1)) == 0 ? tb >> (__ffs(g.TBX) - 1) : tb / g.TBX;
        const uint32_t tgx = bxi * g.TBX + (tb - tbr * g.TBX), tgy = byi * g.TBY + tbr;
        const bool on = tb < ntb && tgx < g.n0 && tgy < g.n1;
        const uint32_t tile = tgy * g.n0 + tgx;
        const uint32_t jjmax = on ? min(TY, g.L1 - tgy * TY) : 0;
        uint32_t *draws = reinterpret_cast<uint32_t *>(smem + L.draws) + (tid >> 5) * L.slots;
        const bool wr = lane32 == 0 && tid < ntb * W;  // one writer per warp that holds tiles
        uint32_t st = 0, sel = 0, it = 0;
        if (on) {
            st = rng_state[(size_t)tile * W + lane];
            sel = rng_sel[(size_t)tile * W + lane];
            it = rng_iter[tile];
        }
        uint32_t a = lcg_param_a(sel), c = lcg_param_c(sel);
        // The parameter rotation of LCG32_State::Update (random/src/lcg32.cpp:51-84): before
        // update itn when itn is a multiple of 15, the (a, c) pairs rotate by
        // state[itn & (W-1)] + (itn odd ? 0 : 1).
        auto rotate = [&](const uint32_t itn, const bool rot) {
            const uint32_t src = __shfl_sync(0xffffffffu, st, itn & (W - 1), W);
            const uint32_t from = (lane + src + ((itn & 1u) ? 0u : 1u)) & (W - 1);
            const uint32_t a2 = __shfl_sync(0xffffffffu, a, from, W);
            const uint32_t c2 = __shfl_sync(0xffffffffu, c, from, W);
            const uint32_t s2 = __shfl_sync(0xffffffffu, sel, from, W);
            if (rot) {
                a = a2;
                c = c2;
                sel = s2;
            }
        };
        bool fast = false;
        if constexpr (TXc != 0 && TYc != 0) {
            constexpr uint32_t kUr = (TXc + W - 1) / W, kRows = (2 * TYc - 1) * kUr;
            constexpr uint32_t kN = kRows + (TXc + TYc + W - 1) / W;  // updates of this sweep
            // Full-height tiles of a compile-time shape (every tile of the warp on the lattice has
            // tile_y rows): the update count is known at every step, nothing is predicated, and
            // the rotating updates come from a mask (update k rotates iff (it + k + 1) % 15 == 0).
            // Segments of tiles off the lattice run along and store nothing.
            if (kN <= 64 && (kFixedOnly || __all_sync(0xffffffffu, !on || jjmax == TYc))) {
                auto draw = [&](const uint32_t k) {  // update k of the sweep and its ballot
                    st = a * st + c;
                    const uint32_t lim = k < kRows ? TXc : TXc + TYc;          // numbers in this request
                    const uint32_t e0 = (k < kRows ? k % kUr : k - kRows) * W;  // its first element here
                    const bool in = e0 + W <= lim || e0 + lane < lim;  // every lane of a full update is in
                    const uint32_t word = __ballot_sync(0xffffffffu, in && lcg_accept(st, thr));
                    if (wr)
                        draws[k] = word;
                };
                // The tiles of a warp normally share their iteration count (every full-height tile
                // makes kN updates a sweep): then the rotating updates sit at compile-time
                // positions, one straight-line sequence per phase it % 15 (kPhaseSeq; tiles off the
                // lattice take the phase of the first tile on it, their results are not stored).
                // Otherwise update k rotates a tile iff bit k of its mask is set.
                bool seq = false;
                if constexpr (kPhaseSeq) {
                    const uint32_t itu = __shfl_sync(0xffffffffu, it, (__ffs(__ballot_sync(0xffffffffu, on)) - 1) & 31);
                    if (__all_sync(0xffffffffu, !on || it == itu)) {
                        auto run = [&](auto phase) {
                            draw_sequence<decltype(phase)::value>(std::make_integer_sequence<uint32_t, kN>{}, rotate, draw, itu);
                        };
                        switch (kShuffleDistance - 1 - itu % kShuffleDistance) {
                        case 0: run(U32<0>{}); break;
                        case 1: run(U32<1>{}); break;
                        case 2: run(U32<2>{}); break;
                        case 3: run(U32<3>{}); break;
                        case 4: run(U32<4>{}); break;
                        case 5: run(U32<5>{}); break;
                        case 6: run(U32<6>{}); break;
                        case 7: run(U32<7>{}); break;
                        case 8: run(U32<8>{}); break;
                        case 9: run(U32<9>{}); break;
                        case 10: run(U32<10>{}); break;
                        case 11: run(U32<11>{}); break;
                        case 12: run(U32<12>{}); break;
                        case 13: run(U32<13>{}); break;
                        default: run(U32<14>{}); break;
                        }
                        seq = true;
                    }
                }
                if (!seq) {
                    const uint64_t rm = (0x1000200040008001ull << (kShuffleDistance - 1 - it % kShuffleDistance)) &
                                        (kN >= 64 ? ~0ull : (1ull << (kN & 63)) - 1);
                    uint64_t wm = __reduce_or_sync(0xffffffffu, (uint32_t)rm);
                    if constexpr (kN > 32)
                        wm |= (uint64_t)__reduce_or_sync(0xffffffffu, (uint32_t)(rm >> 32)) << 32;
#pragma unroll
                    for (uint32_t k = 0; k < kN; ++k) {
                        if ((wm >> k) & 1u)
                            rotate(it + k + 1, (rm >> k) & 1u);
                        draw(k);
                    }
                }
                it += kN;
                fast = true;
            }
        }
        if (!kFixedOnly && !fast) {
            const uint32_t Ur = (TX + W - 1) / W, Um = (TX + TY + W - 1) / W;
            const uint32_t nrow = on ? 2 * jjmax - 1 : 0;
            uint32_t to_rot = kShuffleDistance - it % kShuffleDistance;  // updates until the next rotation
            auto advance = [&](const bool upd) {
                const bool rot = upd && to_rot == 1;
                if (__any_sync(0xffffffffu, rot))
                    rotate(it + 1, rot);
                if (upd) {
                    it += 1;
                    st = a * st + c;
                    to_rot = rot ? kShuffleDistance : to_rot - 1;
                }
            };
            uint32_t u = 0;
            for (uint32_t req = 0; req < 2 * TY - 1; ++req) {
                const bool upd = req < nrow;
                for (uint32_t sub = 0; sub < Ur; ++sub, ++u) {
                    advance(upd);
                    const uint32_t word = __ballot_sync(0xffffffffu, upd && sub * W + lane < TX && lcg_accept(st, thr));
                    if (wr)
                        draws[u] = word;
                }
            }
            for (uint32_t sub = 0; sub < Um; ++sub, ++u) {
                advance(on);
                const uint32_t word = __ballot_sync(0xffffffffu, on && sub * W + lane < TX + TY && lcg_accept(st, thr));
                if (wr)
                    draws[u] = word;
            }
        }
        if (on) {
            rng_state[(size_t)tile * W + lane] = st;
            rng_sel[(size_t)tile * W + lane] = (uint8_t)sel;
            if (lane == 0)
                rng_iter[tile] = it;
        }
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    if (tid < byv)
        sp[tid * pitch + bxv] = halo;
    __syncthreads();

    if constexpr (kFixedOnly) {
        assign_block_labels_rows<W, TXc, TYc, kMayDump, 128, 32, 512>(g, bxi, byi, labels, edge, dump, meas, smem);
        return;
    }
    if (dump.tile_labels == nullptr && (BX & 31u) == 0 && (BX & (BX - 1)) == 0) {
        if constexpr (kFixedShape && TXc != 0) {
            if (BX == 128 && BY == 32 && nthr == 512) {
                assign_block_labels_rows<W, TXc, TYc, kMayDump, 128, 32, 512>(g, bxi, byi, labels, edge, dump, meas,
                                                                               smem);
                return;
            }
        }
        assign_block_labels_rows<W, TXc, TYc, kMayDump>(g, bxi, byi, labels, edge, dump, meas, smem);
        return;
    }

    // ---- 3. bonds (bit 0 +x, bit 1 +y): equal spins and an accepted draw.  The last
    // column / row of a tile bonds through the merge draw: [0, TX) bottom, [TX, TX+TY) right.
    const uint32_t Ur = (TX + W - 1) / W, um = (2 * TY - 1) * Ur;
    const DrawWords<W> dw{reinterpret_cast<const uint32_t *>(smem + L.draws), L.slots};
    for (uint32_t l = tid; l < NS; l += nthr) {
        const uint32_t xl = l % BX, yl = l / BX;
        uint8_t b = 0;
        if (xl < bxv && yl < byv) {
            const uint32_t tbx = xl / TX, tby = yl / TY, tb = tby * g.TBX + tbx;
            const uint32_t ii = xl - tbx * TX, jj = yl - tby * TY;
            const uint32_t iimax = min(TX, bxv - tbx * TX), jjmax = min(TY, byv - tby * TY);
            const uint8_t s = sp[yl * pitch + xl];
            const uint32_t xa = (ii + 1 < iimax) ? dw.bit(tb, jj * Ur, ii) : dw.bit(tb, um, TX + jj);
            const uint32_t ya = (jj + 1 < jjmax) ? dw.bit(tb, (jjmax + jj) * Ur, ii) : dw.bit(tb, um, ii);
            b = (uint8_t)(((xa & 1u) && s == sp[yl * pitch + xl + 1]) | (((ya & 1u) && s == sp[(yl + 1) * pitch + xl]) << 1));
        }
        bond[l] = b;
        parent[l] = l;
    }
    __syncthreads();

    // ---- 4. tile-local components (the reference's AssignLabels result)
    for (uint32_t l = tid; l < NS; l += nthr) {
        const uint8_t b = bond[l];
        if (!b)
            continue;
        const uint32_t xl = l % BX, yl = l / BX;
        const uint32_t tbx = xl / TX, tby = yl / TY;
        const uint32_t ii = xl - tbx * TX, jj = yl - tby * TY;
        const uint32_t iimax = min(TX, bxv - tbx * TX), jjmax = min(TY, byv - tby * TY);
        if ((b & 1) && ii + 1 < iimax)
            uf_union(parent, l, l + 1);
        if ((b & 2) && jj + 1 < jjmax)
            uf_union(parent, l, l + BX);
    }
    __syncthreads();
    if (kMayDump && (dump.bonds || dump.tile_labels)) {  // recording only
        for (uint32_t l = tid; l < NS; l += nthr) {
            const uint32_t xl = l % BX, yl = l / BX;
            if (xl < bxv && yl < byv) {
                const size_t site = (size_t)(y0 + yl) * g.L0 + x0 + xl;
                if (dump.tile_labels) {
                    const uint32_t r = uf_find(parent, l);
                    dump.tile_labels[site] = (y0 + r / BX) * g.L0 + x0 + r % BX;
                }
                if (dump.bonds)
                    dump.bonds[site] = bond[l];
            }
        }
        __syncthreads();
    }

    // ---- 5. bonds between tiles of this block; bonds leaving the block go to k_merge
    for (uint32_t l = tid; l < NS; l += nthr) {
        const uint8_t b = bond[l];
        if (!b)
            continue;
        const uint32_t xl = l % BX, yl = l / BX;
        const uint32_t tbx = xl / TX, tby = yl / TY;
        const uint32_t ii = xl - tbx * TX, jj = yl - tby * TY;
        const uint32_t iimax = min(TX, bxv - tbx * TX), jjmax = min(TY, byv - tby * TY);
        if ((b & 1) && ii + 1 == iimax) {
            if (xl + 1 < bxv)
                uf_union(parent, l, l + 1);
            else
                atomicOr(edge_s, 1u << yl);
        }
        if ((b & 2) && jj + 1 == jjmax) {
            if (yl + 1 < byv)
                uf_union(parent, l, l + BX);
            else
                atomicOr(edge_s + 1 + (xl >> 5), 1u << (xl & 31));
        }
    }
    __syncthreads();

    // ---- 6. labels: a block root stores its global site index, every other site
    // kLocalFlag | the block-local index of its root
    for (uint32_t l = tid; l < NS; l += nthr) {
        const uint32_t xl = l % BX, yl = l / BX;
        if (xl < bxv && yl < byv) {
            const uint32_t r = uf_find(parent, l);
            labels[(size_t)(y0 + yl) * g.L0 + x0 + xl] = r == l ? (y0 + yl) * g.L0 + x0 + xl : (kLocalFlag | r);
            if (kMayDump && dump.block_labels)  // recording only
                dump.block_labels[(size_t)(y0 + yl) * g.L0 + x0 + xl] = (y0 + r / BX) * g.L0 + x0 + r % BX;
        }
    }
    if (tid < kEdgeWords)
        edge[((size_t)byi * g.nbx + bxi) * kEdgeWords + tid] = edge_s[tid];
}

// assign_block with the tile shape as compile-time constants for the common shapes (lcg width
// 16), the runtime form otherwise; full 128 x 32 blocks of 16 x 8 tiles take the fixed-shape
// scanline.  kAllShapes false keeps only 16 x 8 and 16 x 4 (the tiles the B200 table picks):
// every compile-time shape in the kernel costs the 16 x 8 path registers and instruction
// fetches (the 512-lattice mix's assign: 0.271 ms with all seven shapes, 0.245 ms with two).
template <int W, bool kAllShapes = true>
__device__ __forceinline__ void assign_block_any(const Geo &g, const uint32_t bxi, const uint32_t byi,
                                                 const uint8_t *__restrict__ spins, uint32_t *__restrict__ labels,
                                                 uint32_t *__restrict__ rng_state, uint8_t *__restrict__ rng_sel,
                                                 uint32_t *__restrict__ rng_iter, const uint32_t thr,
                                                 uint32_t *__restrict__ edge, unsigned char *smem)
{
#define SWB_TILE(tx, ty)                                                                                              \
    if (g.TX == tx && g.TY == ty) {                                                                                   \
        assign_block<W, tx, ty, true, false, tx == 16 && ty == 8>(g, bxi, byi, spins, labels, rng_state, rng_sel,    \
                                                                 rng_iter, thr, edge, AssignDump{}, MeasureArgs{},   \
                                                                 smem);                                              \
        return;                                                                                                       \
    }
    if constexpr (W == 16) {
        // a full 128 x 32 block of 16 x 8 tiles: the fixed-only form (shape constants folded)
        if (g.TX == 16 && g.TY == 8 && g.BX == 128 && g.BY == 32 && blockDim.x == 512 && (bxi + 1) * 128 <= g.L0 &&
            (byi + 1) * 32 <= g.L1) {
            assign_block<W, 16, 8, true, false, true, true>(g, bxi, byi, spins, labels, rng_state, rng_sel, rng_iter,
                                                            thr, edge, AssignDump{}, MeasureArgs{}, smem);
            return;
        }
        SWB_TILE(16, 8)
        SWB_TILE(16, 4)
        if constexpr (kAllShapes) {
            SWB_TILE(8, 8)
            SWB_TILE(32, 4)
            SWB_TILE(16, 16)
            SWB_TILE(8, 16)
            SWB_TILE(32, 8)
        }
    }
#undef SWB_TILE
    assign_block<W, 0, 0, false, false>(g, bxi, byi, spins, labels, rng_state, rng_sel, rng_iter, thr, edge,
                                        AssignDump{}, MeasureArgs{}, smem);
}

// Unions across the right and bottom edge (periodic) of block (bxi, byi): thread t < BY takes
// row t of the right edge, BY <= t < BY + BX column t - BY of the bottom edge.  With `linked`,
// slot t of the block's BX + BY slots receives the root this thread's union linked (kNoLink
// for none): every block root the merge turns into a non-root appears in exactly one slot.
// With active false (a lattice whose sweep budget is spent) nothing is written; the edge words
// are read all the same, so their load need not wait for the budget's.
__device__ __forceinline__ void merge_block(const Geo &g, const uint32_t bxi, const uint32_t byi, const uint32_t t,
                                            const uint32_t *__restrict__ edge, uint32_t *labels, unsigned int *fault,
                                            uint32_t *__restrict__ linked, const bool active = true)
{
    const uint32_t x0 = bxi * g.BX, y0 = byi * g.BY;
    const uint32_t bxv = min(g.BX, g.L0 - x0), byv = min(g.BY, g.L1 - y0);
    const uint32_t *e = edge + ((size_t)byi * g.nbx + bxi) * kEdgeWords;
    size_t s = 0, nb = 0;
    uint32_t nbx = bxi, nby = byi;  // block of the neighbour site
    bool go = false;
    if (t < g.BY) {
        if (t < byv && ((e[0] >> t) & 1u)) {
            s = (size_t)(y0 + t) * g.L0 + x0 + bxv - 1;
            nb = (size_t)(y0 + t) * g.L0 + (x0 + bxv < g.L0 ? x0 + bxv : 0u);
            nbx = bxi + 1 == g.nbx ? 0 : bxi + 1;
            go = true;
        }
    } else {
        const uint32_t xl = t - g.BY;
        if (xl < bxv && ((e[1 + (xl >> 5)] >> (xl & 31)) & 1u)) {
            s = (size_t)(y0 + byv - 1) * g.L0 + x0 + xl;
            nb = (size_t)(y0 + byv < g.L1 ? y0 + byv : 0u) * g.L0 + x0 + xl;
            nby = byi + 1 == g.nby ? 0 : byi + 1;
            go = true;
        }
    }
    uint32_t link = kNoLink;
    if (go && active) {
        const volatile uint32_t *vl = labels;
        const uint32_t a = label_global(g, bxi, byi, vl[s]), b = label_global(g, nbx, nby, vl[nb]);
        if (a != b)
            link = guf_union_pair(labels, a, b, g.L0 * g.L1, fault);
    }
    if (linked && active)
        linked[((size_t)byi * g.nbx + bxi) * (g.BX + g.BY) + t] = link;
}

// ResolveLabels for the roots the merge linked (slot t of block (bxi, byi), after every merge
// of the sweep): the root's chain is walked to the cluster's root, which is stored in its
// label.  Afterwards every block root's label is its cluster's root, so the flip needs no
// chase; the chases of all blocks are in flight together here instead of behind each flip
// CTA's barrier.
__device__ __forceinline__ void resolve_block(const Geo &g, const uint32_t bxi, const uint32_t byi, const uint32_t t,
                                              const uint32_t *__restrict__ linked, uint32_t *labels,
                                              unsigned int *fault, const bool active = true)
{
    const uint32_t b = linked[((size_t)byi * g.nbx + bxi) * (g.BX + g.BY) + t];
    if (b != kNoLink && active)
        labels[b] = guf_find(labels, b, g.L0 * g.L1, fault);  // the tree's minimum: other finds' atomicMin never undo it
}

// Shared memory of flip_block: the resolved label of every block root.
__host__ __device__ inline uint32_t flip_smem_bytes(const Geo &g)
{
    return g.BX * g.BY * 4;
}

// ResolveLabels + FlipClusters for block (bxi, byi) after the merge.  Block roots (labels
// without kLocalFlag) follow their chain once (guf_find, which also compresses it for the other
// blocks) into shared memory, or with kResolved (resolve_block ran) take their label as it is;
// every site then reads its root's result there and flips iff the cluster's label is odd.
// kWriteLabels stores the resolved global labels (the reference's ResolveLabels output).
// With active false (a lattice whose sweep budget is spent) the block is read but nothing is
// written, so the loads need not wait for the budget's.
template <bool kWriteLabels, int kQuads = 2, bool kResolved = false>
__device__ __forceinline__ void flip_block(const Geo &g, const uint32_t bxi, const uint32_t byi, uint8_t *spins,
                                           uint32_t *labels, unsigned int *fault, unsigned char *smem,
                                           const bool active = true)
{
    const uint32_t BX = g.BX, L0 = g.L0;
    uint32_t *res = reinterpret_cast<uint32_t *>(smem);
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    const uint32_t x0 = bxi * BX, y0 = byi * g.BY;
    const uint32_t bxv = min(BX, L0 - x0), byv = min(g.BY, g.L1 - y0);
    const uint32_t base = y0 * L0 + x0;
    const uint32_t nq = (bxv >> 2) * byv, qrow = bxv >> 2;
    // quads per row: a power of two (32 in a full 128-wide block) takes the shift path below
    const bool qpow2 = qrow && (qrow & (qrow - 1)) == 0;
    if ((L0 & 3u) == 0 && qpow2 && (blockDim.x & (qrow - 1)) == 0 && nq <= kQuads * blockDim.x) {
        // Every thread holds at most kQuads quads (4 labels + 4 spins each) in registers: one
        // round trip for the loads, the merged roots' chains, then the flips.  Quad k of a
        // thread is column xq of row yl0 + k * rstep (whole rows per step).
        const uint32_t lq = __ffs(qrow) - 1;
        const uint32_t rstep = blockDim.x >> lq, yl0 = tid >> lq, xq4 = 4 * (tid & (qrow - 1));
        uint4 lab[kQuads];
        uint32_t spn[kQuads];
#pragma unroll
        for (int k = 0; k < kQuads; ++k) {
            const uint32_t yl = yl0 + k * rstep;
            if (yl < byv) {
                const uint32_t s = base + yl * L0 + xq4;
                lab[k] = *reinterpret_cast<const uint4 *>(labels + s);
                spn[k] = reinterpret_cast<const uint32_t *>(spins)[s >> 2];
            }
        }
#pragma unroll
        for (int k = 0; k < kQuads; ++k) {
            const uint32_t yl = yl0 + k * rstep;
            if (yl < byv) {
                const uint32_t s = base + yl * L0 + xq4, l = yl * BX + xq4;
                const uint32_t v[4] = {lab[k].x, lab[k].y, lab[k].z, lab[k].w};
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (!(v[j] & kLocalFlag))  // a block root: v is its parent (itself unless merged)
                        res[l + j] = kResolved || !active || v[j] == s + j ? v[j]
                                                                            : guf_find(labels, v[j], L0 * g.L1, fault);
            }
        }
        __syncthreads();
        if (!active)
            return;
#pragma unroll
        for (int k = 0; k < kQuads; ++k) {
            const uint32_t yl = yl0 + k * rstep;
            if (yl < byv) {
                const uint32_t s = base + yl * L0 + xq4, l = yl * BX + xq4;
                const uint32_t v[4] = {lab[k].x, lab[k].y, lab[k].z, lab[k].w};
                uint32_t r[4], flip = 0;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    r[j] = res[(v[j] & kLocalFlag) ? (v[j] & kLocalMask) : l + j];
                    flip |= (r[j] & 1u) << (8 * j);
                }
                reinterpret_cast<uint32_t *>(spins)[s >> 2] = spn[k] ^ flip;
                if (kWriteLabels)
                    *reinterpret_cast<uint4 *>(labels + s) = make_uint4(r[0], r[1], r[2], r[3]);
            }
        }
        return;
    }
    for (uint32_t yl = warp; yl < byv; yl += nwarps)
        for (uint32_t xl = lane; xl < bxv; xl += 32) {
            const uint32_t site = base + yl * L0 + xl;
            const uint32_t v = labels[site];
            if (!(v & kLocalFlag))
                res[yl * BX + xl] = kResolved || !active || v == site ? v : guf_find(labels, v, L0 * g.L1, fault);
        }
    __syncthreads();
    if (!active)
        return;
    if ((L0 & 3u) == 0) {
        for (uint32_t yl = warp; yl < byv; yl += nwarps) {
            const uint32_t row = base + yl * L0;
            for (uint32_t q = lane; 4 * q < bxv; q += 32) {
                const uint32_t s = row + 4 * q;
                const uint4 lab = *reinterpret_cast<const uint4 *>(labels + s);
                const uint32_t v[4] = {lab.x, lab.y, lab.z, lab.w};
                uint32_t r[4], flip = 0;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    r[k] = res[(v[k] & kLocalFlag) ? (v[k] & kLocalMask) : yl * BX + 4 * q + k];
                    flip |= (r[k] & 1u) << (8 * k);
                }
                reinterpret_cast<uint32_t *>(spins)[s >> 2] ^= flip;
                if (kWriteLabels)
                    *reinterpret_cast<uint4 *>(labels + s) = make_uint4(r[0], r[1], r[2], r[3]);
            }
        }
    } else {
        for (uint32_t yl = warp; yl < byv; yl += nwarps)
            for (uint32_t xl = lane; xl < bxv; xl += 32) {
                const uint32_t s = base + yl * L0 + xl;
                const uint32_t v = labels[s];
                const uint32_t r = res[(v & kLocalFlag) ? (v & kLocalMask) : yl * BX + xl];
                spins[s] ^= (uint8_t)(r & 1u);
                if (kWriteLabels)
                    labels[s] = r;
            }
    }
}


}  // namespace swb
