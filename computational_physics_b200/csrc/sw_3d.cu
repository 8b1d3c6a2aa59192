// Swendsen-Wang sweep for the 3D Ising model (J = 1, periodic L0 x L1 x L2) on one B200.  The
// reference names the 3D case only (ising/include/swendsen_wang_selflabeling.hpp:20-22); this
// engine extends the 2D conventions: spins uint8 0/1 with site index (z L1 + y) L0 + x, one lcg32
// stream per tile of tx x ty x tz sites seeded seed_base + tile id, the draw order of
// oracle/sw_oracle.c's orc3_sw_sweep (per row: +x requests, then +y, then +z, then one face
// request for the tile's +y, +x and +z faces), the integer accept threshold, labels = minimum
// site index of each cluster, a cluster flips iff its label is odd.
//
// One sweep = four kernels, the 2D split:
//   k3_assign   one CTA per block of tiles: stage the block's spins with a one-site halo, every
//               tile's draws (W-lane warp segments, the 2D rotation rule), bonds, union-find of
//               the bonds inside the block in shared memory; labels in the 2D encoding (block
//               roots: global index; others: kLocalFlag | block-local root) and the block's
//               three outgoing face bitmaps.
//   k3_merge    unions across the +x, +y, +z faces on the global label array (one thread per
//               face site), each recording the root it linked.
//   k3_resolve  every linked root's chain walked to the cluster root.
//   k3_flip     every site reads its root's resolved label and flips iff it is odd.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/swb200.h"
#include "sw_core.cuh"

namespace swb {

constexpr uint32_t k3Threads = 256;  // CTA size of the assign and flip kernels

struct Geo3 {
    uint32_t L0, L1, L2;        // extent
    uint32_t TX, TY, TZ;        // tile
    uint32_t TBX, TBY, TBZ;     // tiles per block
    uint32_t BX, BY, BZ;        // block in sites
    uint32_t n0, n1, n2;        // tiles per direction
    uint32_t nbx, nby, nbz;     // blocks per direction
    uint32_t wx, wy, wz;        // words of the +x, +y, +z face bitmaps per block
};

// Blocks of about 4096 sites whose tiles' lcg lanes fit one CTA (tiles x W <= 256).
inline Geo3 make_geo3(uint32_t L0, uint32_t L1, uint32_t L2, uint32_t TX, uint32_t TY, uint32_t TZ, uint32_t W)
{
    Geo3 g{};
    g.L0 = L0; g.L1 = L1; g.L2 = L2; g.TX = TX; g.TY = TY; g.TZ = TZ;
    g.n0 = (L0 + TX - 1) / TX;
    g.n1 = (L1 + TY - 1) / TY;
    g.n2 = (L2 + TZ - 1) / TZ;
    g.TBX = std::max(1u, 32 / TX);
    g.TBY = std::max(1u, 8 / TY);
    g.TBZ = std::max(1u, 16 / TZ);
    while (g.TBX * g.TBY * g.TBZ * W > k3Threads) {
        if (g.TBZ > 1) g.TBZ /= 2;
        else if (g.TBY > 1) g.TBY /= 2;
        else g.TBX /= 2;
    }
    while (g.TBX > 1 && (g.TBX / 2) * TX >= L0) g.TBX /= 2;
    while (g.TBY > 1 && (g.TBY / 2) * TY >= L1) g.TBY /= 2;
    while (g.TBZ > 1 && (g.TBZ / 2) * TZ >= L2) g.TBZ /= 2;
    g.BX = g.TBX * TX; g.BY = g.TBY * TY; g.BZ = g.TBZ * TZ;
    g.nbx = (L0 + g.BX - 1) / g.BX;
    g.nby = (L1 + g.BY - 1) / g.BY;
    g.nbz = (L2 + g.BZ - 1) / g.BZ;
    g.wx = (g.BY * g.BZ + 31) / 32;
    g.wy = (g.BX * g.BZ + 31) / 32;
    g.wz = (g.BX * g.BY + 31) / 32;
    return g;
}

__host__ __device__ inline uint32_t face_words(const Geo3 &g) { return g.wx + g.wy + g.wz; }
__host__ __device__ inline uint32_t face_sites(const Geo3 &g) { return g.BY * g.BZ + g.BX * g.BZ + g.BX * g.BY; }
__host__ __device__ inline uint32_t block_sites(const Geo3 &g) { return g.BX * g.BY * g.BZ; }
// updates of every lane per sweep (the longest tile): rows for x, y, z, then the face request
__host__ __device__ inline uint32_t draw_updates3(const Geo3 &g, uint32_t W)
{
    const uint32_t ur = (g.TX + W - 1) / W, nface = g.TX * g.TZ + g.TY * g.TZ + g.TX * g.TY;
    return (g.TY * g.TZ + (g.TY - 1) * g.TZ + g.TY * (g.TZ - 1)) * ur + (nface + W - 1) / W;
}

struct Assign3Smem {
    uint32_t parent, acc, box, face, pairs, total;
};

// Pending unions of the fixed-shape assign: a slice of this many words per warp.
constexpr uint32_t k3PairCap = 192;

__host__ __device__ inline Assign3Smem assign3_smem(const Geo3 &g)
{
    Assign3Smem s{};
    const uint32_t ns = block_sites(g);
    s.parent = 0;
    s.acc = ns * 4;                                       // accepted draws: [3][ns] bytes, +x, +y, +z
    s.box = s.acc + 3 * ns;                               // spins of the block and its +1 halo
    s.face = (s.box + (g.BX + 1) * (g.BY + 1) * (g.BZ + 1) + 3) & ~3u;  // face bitmaps
    s.pairs = (s.face + 4 * face_words(g) + 15) & ~15u;
    s.total = s.pairs + 4 * k3PairCap * (k3Threads / 32);
    return s;
}

// Global site index of a label read at a site of block (bxi, byi, bzi).
__device__ __forceinline__ uint32_t label_global3(const Geo3 &g, uint32_t bxi, uint32_t byi, uint32_t bzi, uint32_t v)
{
    if (!(v & kLocalFlag))
        return v;
    const uint32_t r = v & kLocalMask, bxy = g.BX * g.BY;
    const uint32_t zl = r / bxy, yl = (r - zl * bxy) / g.BX, xl = r - zl * bxy - yl * g.BX;
    return ((bzi * g.BZ + zl) * g.L1 + byi * g.BY + yl) * g.L0 + bxi * g.BX + xl;
}

// kFixed: tile 16 x 4 x 4, lcg width 16, and every block a full 32 x 8 x 16 block (the caller
// checked): the block and tile shape are constants, so the site index arithmetic is shifts and
// the loops have fixed trip counts.
template <int W, bool kFixed = false>
__global__ void __launch_bounds__(k3Threads) k3_assign(const Geo3 g_in, const uint8_t *__restrict__ spins,
                                                        uint32_t *__restrict__ labels, uint32_t *__restrict__ rng_state,
                                                        uint8_t *__restrict__ rng_sel, uint32_t *__restrict__ rng_iter,
                                                        const uint32_t thr, uint32_t *__restrict__ faces,
                                                        uint8_t *__restrict__ dump_bonds)
{
    extern __shared__ __align__(16) unsigned char smem[];
    static_assert(!kFixed || W == 16, "the fixed form is lcg width 16");
    Geo3 gfix = g_in;
    if constexpr (kFixed) {
        gfix.TX = 16; gfix.TY = 4; gfix.TZ = 4;
        gfix.TBX = 2; gfix.TBY = 2; gfix.TBZ = 4;
        gfix.BX = 32; gfix.BY = 8; gfix.BZ = 16;
        gfix.wx = 4; gfix.wy = 16; gfix.wz = 8;
    }
    const Geo3 &g = kFixed ? gfix : g_in;
    const Assign3Smem S = assign3_smem(g);
    uint32_t *parent = reinterpret_cast<uint32_t *>(smem + S.parent);
    uint8_t *acc = smem + S.acc, *box = smem + S.box;
    uint32_t *face = reinterpret_cast<uint32_t *>(smem + S.face);
    const uint32_t bxi = blockIdx.x, byi = blockIdx.y, bzi = blockIdx.z;
    const uint32_t BX = g.BX, BY = g.BY, BZ = g.BZ, NS = BX * BY * BZ;
    const uint32_t x0 = bxi * BX, y0 = byi * BY, z0 = bzi * BZ;
    const uint32_t bxv = kFixed ? BX : min(BX, g.L0 - x0), byv = kFixed ? BY : min(BY, g.L1 - y0);
    const uint32_t bzv = kFixed ? BZ : min(BZ, g.L2 - z0);
    const uint32_t tid = threadIdx.x, nthr = kFixed ? k3Threads : blockDim.x;
    const size_t plane = (size_t)g.L0 * g.L1;

    for (uint32_t l = tid; l < NS; l += nthr) {
        parent[l] = l;
        acc[l] = acc[NS + l] = acc[2 * NS + l] = 0;
    }
    for (uint32_t i = tid; i < face_words(g); i += nthr)
        face[i] = 0;
    // spins of the block and the site after it in each direction (periodic); the box is
    // (bxv + 1) x (byv + 1) x (bzv + 1) with pitch BX + 1, BY + 1
    const uint32_t px = BX + 1, pxy = (BX + 1) * (BY + 1);
    for (uint32_t i = tid; i < (bxv + 1) * (byv + 1) * (bzv + 1); i += nthr) {
        const uint32_t zl = i / ((bxv + 1) * (byv + 1)), rem = i - zl * (bxv + 1) * (byv + 1);
        const uint32_t yl = rem / (bxv + 1), xl = rem - yl * (bxv + 1);
        const uint32_t gx = x0 + xl < g.L0 ? x0 + xl : 0, gy = y0 + yl < g.L1 ? y0 + yl : 0;
        const uint32_t gz = z0 + zl < g.L2 ? z0 + zl : 0;
        box[zl * pxy + yl * px + xl] = spins[gz * plane + (size_t)gy * g.L0 + gx];
    }
    __syncthreads();

    // ---- draws: one W-lane segment per tile; every tile runs the longest tile's schedule and a
    // tile that lacks a row idles through it (no update, nothing stored), so that the segment
    // shuffles of the parameter rotation always involve the whole warp.
    {
        const uint32_t TX = g.TX, TY = g.TY, TZ = g.TZ;
        const uint32_t ntb = g.TBX * g.TBY * g.TBZ;
        const uint32_t tb = tid / W, lane = tid % W;
        const uint32_t tbz = tb / (g.TBX * g.TBY), tby = (tb / g.TBX) % g.TBY, tbx = tb % g.TBX;
        const uint32_t tgx = bxi * g.TBX + tbx, tgy = byi * g.TBY + tby, tgz = bzi * g.TBZ + tbz;
        const bool on = tb < ntb && tgx < g.n0 && tgy < g.n1 && tgz < g.n2 && tid < ((ntb * W + 31) & ~31u);
        const uint32_t tile = (tgz * g.n1 + tgy) * g.n0 + tgx;
        const uint32_t iimax = on ? (kFixed ? TX : min(TX, g.L0 - tgx * TX)) : 0;
        const uint32_t jjmax = on ? (kFixed ? TY : min(TY, g.L1 - tgy * TY)) : 0;
        const uint32_t kkmax = on ? (kFixed ? TZ : min(TZ, g.L2 - tgz * TZ)) : 0;
        const uint32_t ox = tbx * TX, oy = tby * TY, oz = tbz * TZ;  // the tile's origin in the block
        uint32_t st = 0, sel = 0, it = 0;
        if (on) {
            st = rng_state[(size_t)tile * W + lane];
            sel = rng_sel[(size_t)tile * W + lane];
            it = rng_iter[tile];
        }
        uint32_t a = lcg_param_a(sel), c = lcg_param_c(sel);
        uint32_t to_rot = kShuffleDistance - it % kShuffleDistance;
        auto advance = [&](const bool upd) {
            const bool rot = upd && to_rot == 1;
            if (__any_sync(0xffffffffu, rot)) {  // the rotation of LCG32_State::Update (random/src/lcg32.cpp:51-84)
                const uint32_t itn = it + 1;
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
            }
            if (upd) {
                it += 1;
                st = a * st + c;
                to_rot = rot ? kShuffleDistance : to_rot - 1;
            }
        };
        const uint32_t ur = (TX + W - 1) / W;
        auto site = [&](uint32_t ii, uint32_t jj, uint32_t kk) { return ((oz + kk) * BY + oy + jj) * BX + ox + ii; };
        // +x rows, +y rows, +z rows: dir 0, 1, 2
        for (uint32_t dir = 0; dir < 3; ++dir) {
            const uint32_t nj = dir == 1 ? TY - 1 : TY, nk = dir == 2 ? TZ - 1 : TZ;
            for (uint32_t kk = 0; kk < nk; ++kk)
                for (uint32_t jj = 0; jj < nj; ++jj) {
                    const bool row = dir == 0 ? (kk < kkmax && jj < jjmax)
                                   : dir == 1 ? (kk < kkmax && jj + 1 < jjmax) : (kk + 1 < kkmax && jj < jjmax);
                    for (uint32_t u = 0; u < ur; ++u) {
                        advance(row);
                        const uint32_t ii = u * W + lane;
                        const bool used = row && ii < TX && (dir == 0 ? ii + 1 < iimax : ii < iimax);
                        if (used && lcg_accept(st, thr))
                            acc[dir * NS + site(ii, jj, kk)] = 1;
                    }
                }
        }
        const uint32_t fy = TX * TZ, fx = TY * TZ, nface = fy + fx + TX * TY;
        for (uint32_t u = 0; u < (nface + W - 1) / W; ++u) {
            advance(on);
            const uint32_t e = u * W + lane;
            if (!on || e >= nface || !lcg_accept(st, thr))
                continue;
            if (e < fy) {  // +y face: the tile's last row
                const uint32_t kk = e / TX, ii = e - kk * TX;
                if (kk < kkmax && ii < iimax)
                    acc[NS + site(ii, jjmax - 1, kk)] = 1;
            } else if (e < fy + fx) {  // +x face: the tile's last column
                const uint32_t kk = (e - fy) / TY, jj = e - fy - kk * TY;
                if (kk < kkmax && jj < jjmax)
                    acc[site(iimax - 1, jj, kk)] = 1;
            } else {  // +z face: the tile's last layer
                const uint32_t jj = (e - fy - fx) / TX, ii = e - fy - fx - jj * TX;
                if (jj < jjmax && ii < iimax)
                    acc[2 * NS + site(ii, jj, kkmax - 1)] = 1;
            }
        }
        if (on) {
            rng_state[(size_t)tile * W + lane] = st;
            rng_sel[(size_t)tile * W + lane] = (uint8_t)sel;
            if (lane == 0)
                rng_iter[tile] = it;
        }
    }
    __syncthreads();

    // ---- bonds (equal spins and an accepted draw); in-block unions, face bits for the merge.
    // The fixed form queues a warp's unions in its slice of a shared list and runs them
    // together, one per lane (inside the loop up to three unions ran, divergent, per site);
    // the union-find's roots (each set's minimum) do not depend on the order of the unions.
    if constexpr (kFixed) {
        const uint32_t lane = tid & 31, below = (1u << lane) - 1u;
        uint32_t *pl = reinterpret_cast<uint32_t *>(smem + S.pairs) + (tid >> 5) * k3PairCap;
        uint32_t npend = 0;  // warp-uniform
        auto flush = [&]() {
            __syncwarp();
            for (uint32_t i = lane; i < npend; i += 32) {
                const uint32_t pr = pl[i];
                uf_union(parent, pr & 0xFFFFu, pr >> 16);
            }
            __syncwarp();
            npend = 0;
        };
        auto queue = [&](const bool u, const uint32_t a, const uint32_t b) {
            const uint32_t m = __ballot_sync(0xffffffffu, u);
            if (u)
                pl[npend + __popc(m & below)] = a | b << 16;
            npend += __popc(m);
        };
        for (uint32_t l = tid; l < NS; l += k3Threads) {  // every site of the block is on the lattice
            const uint32_t zl = l / (BX * BY), yl = (l / BX) % BY, xl = l % BX;
            const uint32_t b0 = zl * pxy + yl * px + xl;
            const uint8_t s = box[b0];
            const uint32_t bond = (acc[l] && s == box[b0 + 1]) | ((acc[NS + l] && s == box[b0 + px]) << 1) |
                                  ((acc[2 * NS + l] && s == box[b0 + pxy]) << 2);
            if (dump_bonds)
                dump_bonds[((size_t)(z0 + zl) * g.L1 + y0 + yl) * g.L0 + x0 + xl] = (uint8_t)bond;
            if ((bond & 1u) && xl + 1 == BX) {
                const uint32_t f = zl * BY + yl;
                atomicOr(face + (f >> 5), 1u << (f & 31));
            }
            if ((bond & 2u) && yl + 1 == BY) {
                const uint32_t f = zl * BX + xl;
                atomicOr(face + g.wx + (f >> 5), 1u << (f & 31));
            }
            if ((bond & 4u) && zl + 1 == BZ) {
                const uint32_t f = yl * BX + xl;
                atomicOr(face + g.wx + g.wy + (f >> 5), 1u << (f & 31));
            }
            queue((bond & 1u) && xl + 1 < BX, l, l + 1);
            queue((bond & 2u) && yl + 1 < BY, l, l + BX);
            queue((bond & 4u) && zl + 1 < BZ, l, l + BX * BY);
            if (npend > k3PairCap - 96)  // room for the next site's three
                flush();
        }
        flush();
    } else
    for (uint32_t l = tid; l < NS; l += nthr) {
        const uint32_t zl = l / (BX * BY), yl = (l / BX) % BY, xl = l % BX;
        if (xl >= bxv || yl >= byv || zl >= bzv)
            continue;
        const uint32_t b0 = zl * pxy + yl * px + xl;
        const uint8_t s = box[b0];
        const uint32_t bond = (acc[l] && s == box[b0 + 1]) | ((acc[NS + l] && s == box[b0 + px]) << 1) |
                              ((acc[2 * NS + l] && s == box[b0 + pxy]) << 2);
        if (dump_bonds)
            dump_bonds[((size_t)(z0 + zl) * g.L1 + y0 + yl) * g.L0 + x0 + xl] = (uint8_t)bond;
        if (bond & 1u) {
            if (xl + 1 < bxv) {
                uf_union(parent, l, l + 1);
            } else {
                const uint32_t f = zl * BY + yl;
                atomicOr(face + (f >> 5), 1u << (f & 31));
            }
        }
        if (bond & 2u) {
            if (yl + 1 < byv) {
                uf_union(parent, l, l + BX);
            } else {
                const uint32_t f = zl * BX + xl;
                atomicOr(face + g.wx + (f >> 5), 1u << (f & 31));
            }
        }
        if (bond & 4u) {
            if (zl + 1 < bzv) {
                uf_union(parent, l, l + BX * BY);
            } else {
                const uint32_t f = yl * BX + xl;
                atomicOr(face + g.wx + g.wy + (f >> 5), 1u << (f & 31));
            }
        }
    }
    __syncthreads();

    // ---- labels: block roots their global index, others kLocalFlag | the block-local root
    for (uint32_t l = tid; l < NS; l += nthr) {
        const uint32_t zl = l / (BX * BY), yl = (l / BX) % BY, xl = l % BX;
        if (xl >= bxv || yl >= byv || zl >= bzv)
            continue;
        const uint32_t r = uf_find(parent, l);
        const uint32_t gs = ((z0 + zl) * g.L1 + y0 + yl) * g.L0 + x0 + xl;
        labels[gs] = r == l ? gs : (kLocalFlag | r);
    }
    const size_t blk = ((size_t)bzi * g.nby + byi) * g.nbx + bxi;
    for (uint32_t i = tid; i < face_words(g); i += nthr)
        faces[blk * face_words(g) + i] = face[i];
}

// Unions across block (bxi, byi, bzi)'s +x, +y and +z faces (periodic), one face site per
// thread; slot t of the block's face_sites slots receives the root the union linked.
__global__ void __launch_bounds__(k3Threads) k3_merge(const Geo3 g, const uint32_t *__restrict__ faces, uint32_t *labels,
                                                       unsigned int *fault, uint32_t *__restrict__ linked)
{
    const uint32_t bxi = blockIdx.x, byi = blockIdx.y, bzi = blockIdx.z;
    const uint32_t BX = g.BX, BY = g.BY, BZ = g.BZ;
    const uint32_t x0 = bxi * BX, y0 = byi * BY, z0 = bzi * BZ;
    const uint32_t bxv = min(BX, g.L0 - x0), byv = min(BY, g.L1 - y0), bzv = min(BZ, g.L2 - z0);
    const size_t blk = ((size_t)bzi * g.nby + byi) * g.nbx + bxi;
    const uint32_t *f = faces + blk * face_words(g);
    const uint32_t nfx = BY * BZ, nfy = BX * BZ, nf = face_sites(g);
    for (uint32_t t = threadIdx.x; t < nf; t += blockDim.x) {
        uint32_t xl, yl, zl, nx, ny, nz, nbx = bxi, nby = byi, nbz = bzi;
        bool go = false;
        if (t < nfx) {
            zl = t / BY; yl = t - zl * BY; xl = bxv - 1;
            go = zl < bzv && yl < byv && ((f[t >> 5] >> (t & 31)) & 1u);
            nx = x0 + bxv < g.L0 ? x0 + bxv : 0; ny = y0 + yl; nz = z0 + zl;
            nbx = bxi + 1 == g.nbx ? 0 : bxi + 1;
        } else if (t < nfx + nfy) {
            const uint32_t u = t - nfx;
            zl = u / BX; xl = u - zl * BX; yl = byv - 1;
            go = zl < bzv && xl < bxv && ((f[g.wx + (u >> 5)] >> (u & 31)) & 1u);
            nx = x0 + xl; ny = y0 + byv < g.L1 ? y0 + byv : 0; nz = z0 + zl;
            nby = byi + 1 == g.nby ? 0 : byi + 1;
        } else {
            const uint32_t u = t - nfx - nfy;
            yl = u / BX; xl = u - yl * BX; zl = bzv - 1;
            go = yl < byv && xl < bxv && ((f[g.wx + g.wy + (u >> 5)] >> (u & 31)) & 1u);
            nx = x0 + xl; ny = y0 + yl; nz = z0 + bzv < g.L2 ? z0 + bzv : 0;
            nbz = bzi + 1 == g.nbz ? 0 : bzi + 1;
        }
        uint32_t link = kNoLink;
        if (go) {
            const volatile uint32_t *vl = labels;
            const size_t s = ((size_t)(z0 + zl) * g.L1 + y0 + yl) * g.L0 + x0 + xl;
            const size_t nb = ((size_t)nz * g.L1 + ny) * g.L0 + nx;
            const uint32_t a = label_global3(g, bxi, byi, bzi, vl[s]), b = label_global3(g, nbx, nby, nbz, vl[nb]);
            if (a != b)
                link = guf_union_pair(labels, a, b, g.L0 * g.L1 * g.L2, fault);
        }
        linked[blk * nf + t] = link;
    }
}

__global__ void __launch_bounds__(k3Threads) k3_resolve(const Geo3 g, const uint32_t *__restrict__ linked, uint32_t *labels,
                                                         unsigned int *fault)
{
    const size_t blk = ((size_t)blockIdx.z * g.nby + blockIdx.y) * g.nbx + blockIdx.x;
    const uint32_t nf = face_sites(g);
    for (uint32_t t = threadIdx.x; t < nf; t += blockDim.x) {
        const uint32_t b = linked[blk * nf + t];
        if (b != kNoLink)
            labels[b] = guf_find(labels, b, g.L0 * g.L1 * g.L2, fault);
    }
}

// Every block root's label is its cluster's root after k3_resolve; every site reads its root's
// and flips iff it is odd.  With write_labels the resolved labels are stored (a dumped sweep).
// kFixed: every block a whole 32 x 8 x 16 block (the assign's fixed form): each thread holds four
// quads of four sites (one 16-byte label load and one 4-byte spin load each) from the first pass
// to the second.
template <bool kFixed = false>
__global__ void __launch_bounds__(k3Threads) k3_flip(const Geo3 g, uint8_t *__restrict__ spins, uint32_t *labels,
                                                      const int write_labels)
{
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t *res = reinterpret_cast<uint32_t *>(smem);
    const uint32_t bxi = blockIdx.x, byi = blockIdx.y, bzi = blockIdx.z;
    if constexpr (kFixed) {
        static_assert(k3Threads == 256, "four quads per thread over 4096 sites");
        const uint32_t x0 = bxi * 32, y0 = byi * 8, z0 = bzi * 16;
        uint4 lab[4];
        uint32_t spn[4];
        size_t site[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t q = threadIdx.x + k * 256, r = q >> 3, x = (q & 7) * 4;  // row r = zl * 8 + yl
            site[k] = ((size_t)(z0 + (r >> 3)) * g.L1 + y0 + (r & 7)) * g.L0 + x0 + x;
            lab[k] = *reinterpret_cast<const uint4 *>(labels + site[k]);
            spn[k] = *reinterpret_cast<const uint32_t *>(spins + site[k]);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t l = (threadIdx.x + k * 256) * 4;
            const uint32_t v[4] = {lab[k].x, lab[k].y, lab[k].z, lab[k].w};
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (!(v[j] & kLocalFlag))
                    res[l + j] = v[j];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t l = (threadIdx.x + k * 256) * 4;
            const uint32_t v[4] = {lab[k].x, lab[k].y, lab[k].z, lab[k].w};
            uint32_t rr[4], flip = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                rr[j] = res[(v[j] & kLocalFlag) ? (v[j] & kLocalMask) : l + j];
                flip |= (rr[j] & 1u) << (8 * j);
            }
            *reinterpret_cast<uint32_t *>(spins + site[k]) = spn[k] ^ flip;
            if (write_labels)
                *reinterpret_cast<uint4 *>(labels + site[k]) = make_uint4(rr[0], rr[1], rr[2], rr[3]);
        }
        return;
    }
    const uint32_t BX = g.BX, BY = g.BY, BZ = g.BZ, NS = BX * BY * BZ;
    const uint32_t x0 = bxi * BX, y0 = byi * BY, z0 = bzi * BZ;
    const uint32_t bxv = min(BX, g.L0 - x0), byv = min(BY, g.L1 - y0), bzv = min(BZ, g.L2 - z0);
    for (uint32_t l = threadIdx.x; l < NS; l += blockDim.x) {
        const uint32_t zl = l / (BX * BY), yl = (l / BX) % BY, xl = l % BX;
        if (xl < bxv && yl < byv && zl < bzv) {
            const uint32_t v = labels[((size_t)(z0 + zl) * g.L1 + y0 + yl) * g.L0 + x0 + xl];
            if (!(v & kLocalFlag))
                res[l] = v;
        }
    }
    __syncthreads();
    for (uint32_t l = threadIdx.x; l < NS; l += blockDim.x) {
        const uint32_t zl = l / (BX * BY), yl = (l / BX) % BY, xl = l % BX;
        if (xl < bxv && yl < byv && zl < bzv) {
            const size_t s = ((size_t)(z0 + zl) * g.L1 + y0 + yl) * g.L0 + x0 + xl;
            const uint32_t v = labels[s];
            const uint32_t r = res[(v & kLocalFlag) ? (v & kLocalMask) : l];
            spins[s] ^= (uint8_t)(r & 1u);
            if (write_labels)
                labels[s] = r;
        }
    }
}

__global__ void __launch_bounds__(256) k3_measure(const Geo3 g, const uint8_t *__restrict__ spins, Obs *obs,
                                                  long long *series, const unsigned long long cap, const int accumulate)
{
    long long e = 0, m = 0;
    const size_t plane = (size_t)g.L0 * g.L1, n = plane * g.L2;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t z = (uint32_t)(i / plane), rem = (uint32_t)(i - (size_t)z * plane);
        const uint32_t y = rem / g.L0, x = rem - y * g.L0;
        const int s = 2 * spins[i] - 1;
        const int rx = 2 * spins[(size_t)z * plane + (size_t)y * g.L0 + (x + 1 == g.L0 ? 0 : x + 1)] - 1;
        const int ry = 2 * spins[(size_t)z * plane + (size_t)(y + 1 == g.L1 ? 0 : y + 1) * g.L0 + x] - 1;
        const int rz = 2 * spins[(size_t)(z + 1 == g.L2 ? 0 : z + 1) * plane + (size_t)y * g.L0 + x] - 1;
        e += s * (rx + ry + rz);
        m += s;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        e += __shfl_xor_sync(0xffffffffu, e, o);
        m += __shfl_xor_sync(0xffffffffu, m, o);
    }
    __shared__ long long se[8], sm[8];
    if ((threadIdx.x & 31) == 0) {
        se[threadIdx.x >> 5] = e;
        sm[threadIdx.x >> 5] = m;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        long long be = 0, bm = 0;
        for (uint32_t k = 0; k < blockDim.x / 32; ++k) {
            be += se[k];
            bm += sm[k];
        }
        obs_add_part(obs, series, cap, n, gridDim.x, be, bm, accumulate);
    }
}

template <int W>
__global__ void k3_rng_init(const uint32_t n_tiles, const uint32_t seed_base, uint32_t *state, uint8_t *sel,
                           uint32_t *iter)
{
    rng_init_tile<W>(n_tiles, seed_base, state, sel, iter);
}

__global__ void k3_hot_start(const size_t n, const uint32_t seed, uint8_t *spins)
{
    hot_start_chunk(n, seed, spins);
}

__global__ void k3_check_spins(const size_t n, const uint8_t *p, unsigned int *bad)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (p[i] > 1)
            atomicOr(bad, 1u);
}

}  // namespace swb

using namespace swb;

struct swb_lattice3 {
    int device = 0;
    cudaStream_t stream = nullptr;
    Geo3 g{};
    uint32_t W = 16, n_tiles = 0, n_blocks = 0, smem_assign = 0;
    size_t n = 0;
    uint8_t *spins = nullptr;
    uint32_t *labels = nullptr, *rng_state = nullptr, *rng_iter = nullptr, *faces = nullptr, *linked = nullptr;
    uint8_t *rng_sel = nullptr;
    Obs *obs = nullptr;
    long long *series = nullptr;
    unsigned long long series_cap = 1ull << 16;
    unsigned int *fault = nullptr, *flag = nullptr;
    int measure_grid = 1;
};

namespace {

int set_device3(const swb_lattice3 *h)
{
    SWB_CUDA(cudaSetDevice(h->device));
    return SWB_OK;
}

int check_fault3(swb_lattice3 *h)
{
    unsigned int f = 0;
    SWB_CUDA(cudaMemcpyAsync(&f, h->fault, sizeof(f), cudaMemcpyDeviceToHost, h->stream));
    SWB_CUDA(cudaStreamSynchronize(h->stream));
    if (f)
        return fail(SWB_ERR_STATE, "label union-find fault (word %u: 1 chain over %u steps, 2 union retries, 4 label outside the lattice)", f, kChainCap);
    return SWB_OK;
}

int launch_sweep3(swb_lattice3 *h, float temperature, uint8_t *dump_bonds, bool write_labels)
{
    const Geo3 &g = h->g;
    const dim3 grid(g.nbx, g.nby, g.nbz);
    const uint32_t thr = accept_threshold(swb_p_add(temperature));
    const bool fixed = h->W == 16 && g.TX == 16 && g.TY == 4 && g.TZ == 4 && g.BX == 32 && g.BY == 8 && g.BZ == 16 &&
                       g.L0 % 32 == 0 && g.L1 % 8 == 0 && g.L2 % 16 == 0;
    if (fixed)
        k3_assign<16, true><<<grid, k3Threads, h->smem_assign, h->stream>>>(g, h->spins, h->labels, h->rng_state,
                                                                            h->rng_sel, h->rng_iter, thr, h->faces,
                                                                            dump_bonds);
    else
    switch (h->W) {
    case 8: k3_assign<8><<<grid, k3Threads, h->smem_assign, h->stream>>>(g, h->spins, h->labels, h->rng_state, h->rng_sel, h->rng_iter, thr, h->faces, dump_bonds); break;
    case 16: k3_assign<16><<<grid, k3Threads, h->smem_assign, h->stream>>>(g, h->spins, h->labels, h->rng_state, h->rng_sel, h->rng_iter, thr, h->faces, dump_bonds); break;
    default: k3_assign<32><<<grid, k3Threads, h->smem_assign, h->stream>>>(g, h->spins, h->labels, h->rng_state, h->rng_sel, h->rng_iter, thr, h->faces, dump_bonds); break;
    }
    SWB_LAUNCHED();
    k3_merge<<<grid, k3Threads, 0, h->stream>>>(g, h->faces, h->labels, h->fault, h->linked);
    SWB_LAUNCHED();
    k3_resolve<<<grid, k3Threads, 0, h->stream>>>(g, h->linked, h->labels, h->fault);
    SWB_LAUNCHED();
    if (fixed)
        k3_flip<true><<<grid, k3Threads, block_sites(g) * 4, h->stream>>>(g, h->spins, h->labels, write_labels ? 1 : 0);
    else
        k3_flip<><<<grid, k3Threads, block_sites(g) * 4, h->stream>>>(g, h->spins, h->labels, write_labels ? 1 : 0);
    SWB_LAUNCHED();
    return SWB_OK;
}

int launch_measure3(swb_lattice3 *h, int accumulate)
{
    k3_measure<<<h->measure_grid, 256, 0, h->stream>>>(h->g, h->spins, h->obs, h->series, h->series_cap, accumulate);
    SWB_LAUNCHED();
    return SWB_OK;
}

bool valid_temperature(float T) { return T > 0.0f && std::isfinite(T); }

}  // namespace

extern "C" {

int swb3_create(swb_lattice3 **out, uint32_t L0, uint32_t L1, uint32_t L2, uint32_t tile_x, uint32_t tile_y,
                uint32_t tile_z, uint32_t lcg_width, uint32_t seed_base, int device)
{
    if (!out)
        return fail(SWB_ERR_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (L0 == 0 || L1 == 0 || L2 == 0 || L0 % 2 || L1 % 2 || (L2 % 2 && L2 != 1))
        return fail(SWB_ERR_ARGUMENT, "SwendsenWang_3D requires even extents (L2 = 1 allowed), got %u x %u x %u", L0, L1,
                    L2);
    if ((uint64_t)L0 * L1 * L2 > 0x7FFFFFFFull)
        return fail(SWB_ERR_ARGUMENT, "lattice of %u x %u x %u sites exceeds 2^31 - 1 labels", L0, L1, L2);
    if (!(tile_x == 8 || tile_x == 16 || tile_x == 32) || tile_y < 1 || tile_y > 8 || tile_z < 1 || tile_z > 8)
        return fail(SWB_ERR_ARGUMENT, "unsupported tile %u x %u x %u (tile_x in {8,16,32}, 1 <= tile_y, tile_z <= 8)",
                    tile_x, tile_y, tile_z);
    if (!(lcg_width == 8 || lcg_width == 16 || lcg_width == 32))
        return fail(SWB_ERR_ARGUMENT, "unsupported lcg32 width %u (8, 16 or 32)", lcg_width);
    const Geo3 g = make_geo3(L0, L1, L2, tile_x, tile_y, tile_z, lcg_width);
    if (g.nby > 65535 || g.nbz > 65535)
        return fail(SWB_ERR_ARGUMENT, "lattice of %u x %u x %u sites needs too many block rows or layers", L0, L1, L2);
    swb_lattice3 *h = new swb_lattice3();
    h->device = device;
    h->W = lcg_width;
    h->g = g;
    h->n = (size_t)L0 * L1 * L2;
    h->n_tiles = g.n0 * g.n1 * g.n2;
    h->n_blocks = g.nbx * g.nby * g.nbz;
    h->smem_assign = assign3_smem(g).total;
    auto cleanup = [&](int rc) {
        swb3_destroy(h);
        return rc;
    };
#define SWB_TRY(call)                                                                              \
    do {                                                                                           \
        cudaError_t err__ = (call);                                                                \
        if (err__ != cudaSuccess)                                                                  \
            return cleanup(fail(SWB_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(err__))); \
    } while (0)
    SWB_TRY(cudaSetDevice(device));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    h->measure_grid = (int)std::max<size_t>(1, std::min<size_t>((h->n + 255) / 256, (size_t)sms * 8));
    SWB_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    SWB_TRY(cudaMalloc(&h->spins, h->n + 16));
    SWB_TRY(cudaMalloc(&h->labels, h->n * 4 + 16));
    SWB_TRY(cudaMalloc(&h->rng_state, (size_t)h->n_tiles * h->W * 4));
    SWB_TRY(cudaMalloc(&h->rng_sel, (size_t)h->n_tiles * h->W));
    SWB_TRY(cudaMalloc(&h->rng_iter, (size_t)h->n_tiles * 4));
    SWB_TRY(cudaMalloc(&h->faces, (size_t)h->n_blocks * face_words(g) * 4));
    SWB_TRY(cudaMalloc(&h->linked, (size_t)h->n_blocks * face_sites(g) * 4));
    SWB_TRY(cudaMalloc(&h->obs, sizeof(Obs)));
    SWB_TRY(cudaMalloc(&h->series, h->series_cap * 16));
    SWB_TRY(cudaMalloc(&h->fault, 4));
    SWB_TRY(cudaMalloc(&h->flag, 4));
    SWB_TRY(cudaMemsetAsync(h->fault, 0, 4, h->stream));
    SWB_TRY(cudaMemsetAsync(h->spins, 0, h->n + 16, h->stream));
    SWB_TRY(cudaMemsetAsync(h->obs, 0, sizeof(Obs), h->stream));
    if (h->smem_assign > 48 * 1024)
        return cleanup(fail(SWB_ERR_ARGUMENT, "block of %u x %u x %u sites needs %u bytes of shared memory", g.BX, g.BY,
                            g.BZ, h->smem_assign));
    const unsigned grid = (h->n_tiles + 127) / 128;
    switch (h->W) {
    case 8: k3_rng_init<8><<<grid, 128, 0, h->stream>>>(h->n_tiles, seed_base, h->rng_state, h->rng_sel, h->rng_iter); break;
    case 16: k3_rng_init<16><<<grid, 128, 0, h->stream>>>(h->n_tiles, seed_base, h->rng_state, h->rng_sel, h->rng_iter); break;
    default: k3_rng_init<32><<<grid, 128, 0, h->stream>>>(h->n_tiles, seed_base, h->rng_state, h->rng_sel, h->rng_iter); break;
    }
    g_launches.fetch_add(1);
    SWB_TRY(cudaGetLastError());
    SWB_TRY(cudaStreamSynchronize(h->stream));
#undef SWB_TRY
    *out = h;
    return SWB_OK;
}

int swb3_destroy(swb_lattice3 *h)
{
    if (!h)
        return SWB_OK;
    cudaSetDevice(h->device);
    if (h->stream)
        cudaStreamSynchronize(h->stream);
    cudaFree(h->spins);
    cudaFree(h->labels);
    cudaFree(h->rng_state);
    cudaFree(h->rng_sel);
    cudaFree(h->rng_iter);
    cudaFree(h->faces);
    cudaFree(h->linked);
    cudaFree(h->obs);
    cudaFree(h->series);
    cudaFree(h->fault);
    cudaFree(h->flag);
    if (h->stream)
        cudaStreamDestroy(h->stream);
    delete h;
    return SWB_OK;
}

int swb3_geometry(swb_lattice3 *h, uint32_t *geometry)
{
    if (!h || !geometry)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    const Geo3 &g = h->g;
    const uint32_t v[12] = {g.L0, g.L1, g.L2, g.TX, g.TY, g.TZ, g.BX, g.BY, g.BZ, g.nbx, g.nby, g.nbz};
    std::memcpy(geometry, v, sizeof(v));
    return SWB_OK;
}

int swb3_set_spins(swb_lattice3 *h, const uint8_t *host_spins)
{
    if (!h || !host_spins)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (int rc = set_device3(h))
        return rc;
    SWB_CUDA(cudaMemcpyAsync(h->spins, host_spins, h->n, cudaMemcpyHostToDevice, h->stream));
    SWB_CUDA(cudaMemsetAsync(h->flag, 0, 4, h->stream));
    k3_check_spins<<<h->measure_grid, 256, 0, h->stream>>>(h->n, h->spins, h->flag);
    SWB_LAUNCHED();
    unsigned int bad = 0;
    SWB_CUDA(cudaMemcpyAsync(&bad, h->flag, 4, cudaMemcpyDeviceToHost, h->stream));
    SWB_CUDA(cudaStreamSynchronize(h->stream));
    if (bad)
        return fail(SWB_ERR_ARGUMENT, "spins must be 0 or 1");
    return SWB_OK;
}

int swb3_get_spins(swb_lattice3 *h, uint8_t *host_spins)
{
    if (!h || !host_spins)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (int rc = set_device3(h))
        return rc;
    SWB_CUDA(cudaMemcpyAsync(host_spins, h->spins, h->n, cudaMemcpyDeviceToHost, h->stream));
    SWB_CUDA(cudaStreamSynchronize(h->stream));
    return check_fault3(h);
}

int swb3_hot_start(swb_lattice3 *h, uint32_t seed)
{
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "NULL handle");
    if (int rc = set_device3(h))
        return rc;
    const size_t chunks = (h->n + 63) / 64;
    k3_hot_start<<<(unsigned)((chunks + 255) / 256), 256, 0, h->stream>>>(h->n, seed, h->spins);
    SWB_LAUNCHED();
    return SWB_OK;
}

int swb3_sweep(swb_lattice3 *h, float temperature, uint32_t n_sweeps, uint32_t measure_every)
{
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "NULL handle");
    if (!valid_temperature(temperature))
        return fail(SWB_ERR_ARGUMENT, "temperature must be positive and finite");
    if (int rc = set_device3(h))
        return rc;
    for (uint32_t s = 1; s <= n_sweeps; ++s) {
        if (int rc = launch_sweep3(h, temperature, nullptr, false))
            return rc;
        if (measure_every && s % measure_every == 0)
            if (int rc = launch_measure3(h, 1))
                return rc;
    }
    return SWB_OK;
}

int swb3_sweep_dumped(swb_lattice3 *h, float temperature, uint8_t *bonds, uint32_t *labels_final)
{
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "NULL handle");
    if (!valid_temperature(temperature))
        return fail(SWB_ERR_ARGUMENT, "temperature must be positive and finite");
    if (int rc = set_device3(h))
        return rc;
    uint8_t *d_bonds = nullptr;
    if (bonds)
        SWB_CUDA(cudaMallocAsync(&d_bonds, h->n, h->stream));
    int rc = launch_sweep3(h, temperature, d_bonds, true);
    if (rc == SWB_OK) {
        if (bonds)
            SWB_CUDA(cudaMemcpyAsync(bonds, d_bonds, h->n, cudaMemcpyDeviceToHost, h->stream));
        if (labels_final)
            SWB_CUDA(cudaMemcpyAsync(labels_final, h->labels, h->n * 4, cudaMemcpyDeviceToHost, h->stream));
    }
    if (d_bonds)
        cudaFreeAsync(d_bonds, h->stream);
    SWB_CUDA(cudaStreamSynchronize(h->stream));
    return rc ? rc : check_fault3(h);
}

int swb3_sweep_timed(swb_lattice3 *h, float temperature, uint32_t n_sweeps, float *ms)
{
    if (!h || !ms)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (!valid_temperature(temperature))
        return fail(SWB_ERR_ARGUMENT, "temperature must be positive and finite");
    if (int rc = set_device3(h))
        return rc;
    cudaEvent_t a, b;
    SWB_CUDA(cudaEventCreate(&a));
    SWB_CUDA(cudaEventCreate(&b));
    SWB_CUDA(cudaEventRecord(a, h->stream));
    int rc = SWB_OK;
    for (uint32_t s = 0; s < n_sweeps && rc == SWB_OK; ++s)
        rc = launch_sweep3(h, temperature, nullptr, false);
    SWB_CUDA(cudaEventRecord(b, h->stream));
    SWB_CUDA(cudaEventSynchronize(b));
    SWB_CUDA(cudaEventElapsedTime(ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return rc ? rc : check_fault3(h);
}

int swb3_energy_magnetization(swb_lattice3 *h, double *out, int64_t *e_sum, int64_t *m_sum)
{
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "NULL handle");
    if (int rc = set_device3(h))
        return rc;
    if (int rc = launch_measure3(h, 0))
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

int swb3_samples(swb_lattice3 *h, int64_t *em, uint64_t capacity, uint64_t *count, double *acc)
{
    if (!h || !count)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (int rc = set_device3(h))
        return rc;
    Obs o;
    SWB_CUDA(cudaMemcpyAsync(&o, h->obs, sizeof(Obs), cudaMemcpyDeviceToHost, h->stream));
    SWB_CUDA(cudaStreamSynchronize(h->stream));
    *count = o.n_samples;
    if (acc)
        std::memcpy(acc, o.acc, sizeof(o.acc));
    if (o.n_samples > h->series_cap)
        return fail(SWB_ERR_CAPACITY, "%llu samples recorded, series keeps %llu", o.n_samples, h->series_cap);
    const uint64_t k = std::min<uint64_t>(o.n_samples, capacity);
    if (k && em) {
        SWB_CUDA(cudaMemcpyAsync(em, h->series, k * 16, cudaMemcpyDeviceToHost, h->stream));
        SWB_CUDA(cudaStreamSynchronize(h->stream));
    }
    return SWB_OK;
}

int swb3_get_rng(swb_lattice3 *h, uint32_t *state, uint32_t *a, uint32_t *c, uint32_t *iteration)
{
    if (!h || !state || !a || !c || !iteration)
        return fail(SWB_ERR_ARGUMENT, "NULL argument");
    if (int rc = set_device3(h))
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

int swb3_rng_shape(swb_lattice3 *h, uint32_t *n_tiles, uint32_t *lcg_width)
{
    if (!h)
        return fail(SWB_ERR_ARGUMENT, "NULL handle");
    if (n_tiles) *n_tiles = h->n_tiles;
    if (lcg_width) *lcg_width = h->W;
    return SWB_OK;
}

}  // extern "C"
