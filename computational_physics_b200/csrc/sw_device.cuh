// Device building blocks of the Swendsen-Wang engine (sm_100a).
//
//  * lcg32 lanes in registers: one thread holds one lane of a tile's stream; a tile's W
//    lanes sit in one W-wide segment of a warp, so the reference's periodic parameter
//    rotation (random/src/lcg32.cpp:51-84) is a segment-local __shfl_sync.
//  * drand48 with jump-ahead, for the bit-exact hot start and stream seeding.
//  * lock-free union-find toward the minimum index (shared or global memory), the
//    reference's atomic-min equivalence rule (ising/src/swendsen_wang_cpu.cpp:107-156).
#pragma once

#include <cstdint>

namespace swb {

// The five Numerical Recipes (a, c) pairs of random/src/lcg32.cpp:17-24, by index.
__host__ __device__ __forceinline__ uint32_t lcg_param_a(uint32_t sel)
{
    return sel == 0 ? 1372383749u : sel == 1 ? 2891336453u : sel == 2 ? 2024337845u : sel == 3 ? 32310901u : 29943829u;
}
__host__ __device__ __forceinline__ uint32_t lcg_param_c(uint32_t sel)
{
    return sel == 0 ? 1289706101u : sel == 1 ? 1640531513u : sel == 2 ? 797082193u : sel == 3 ? 626627237u : 1013904223u;
}

// Index (0..4) of an (a, c) pair among the five, or -1 (host code, for imported streams).
inline int lcg_pair_index(uint32_t a, uint32_t c)
{
    for (uint32_t s = 0; s < 5; ++s)
        if (lcg_param_a(s) == a && lcg_param_c(s) == c)
            return (int)s;
    return -1;
}

constexpr uint32_t kShuffleDistance = 15;          // LCG32_State::ShuffleDistance (lcg32.hpp:43)
constexpr float kTwoPowMinus32 = 2.3283064365386963e-10f;  // the float the reference's literal rounds to

// Accept test of a bond draw.  The reference accepts when (float)u * 2^-32 < p_add, with u
// rounded to nearest (random/src/lcg32.cpp:120-129 and the '< p_add' of its callers).  The
// scaling by 2^-32 is exact and round-to-nearest conversion is monotone in u, so the accepted
// u are exactly the prefix [0, thr) with thr = accept_threshold(p_add): one integer compare.
__device__ __forceinline__ bool lcg_accept(uint32_t u, uint32_t thr)
{
    return u < thr;
}

// Smallest u with (float)u >= p_add * 2^32, by bisection with the same round-to-nearest
// conversion (host code; p_add in [0, 1], so the answer is below 2^32).
inline uint32_t accept_threshold(float p_add)
{
    const float q = p_add * 4294967296.0f;  // exact: power-of-two scaling
    uint64_t lo = 0, hi = 1ull << 32;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (static_cast<float>(static_cast<uint32_t>(mid)) >= q)
            hi = mid;
        else
            lo = mid + 1;
    }
    return static_cast<uint32_t>(lo);
}

// ---- drand48: X' = 0x5DEECE66D X + 0xB mod 2^48 (POSIX), used by LCG32_State::Init and the
// Lattice<2> hot start.
constexpr uint64_t kDrandA = 0x5DEECE66Dull;
constexpr uint64_t kDrandC = 0xBull;
constexpr uint64_t kDrandMask = (1ull << 48) - 1;

__host__ __device__ __forceinline__ uint64_t drand48_seed(uint32_t seed)
{
    return ((uint64_t)seed << 16) | 0x330Eull;
}
__host__ __device__ __forceinline__ uint64_t drand48_step(uint64_t x)
{
    return (kDrandA * x + kDrandC) & kDrandMask;
}
// drand48() as a double: X * 2^-48 exactly.
__host__ __device__ __forceinline__ double drand48_value(uint64_t x)
{
    return (double)x * 0x1p-48;  // exact: x < 2^48
}
// Affine map of k drand48 steps: X_k = A X + C (mod 2^48).
__host__ __device__ inline void drand48_jump(uint64_t k, uint64_t &A, uint64_t &C)
{
    uint64_t a = kDrandA, c = kDrandC;
    A = 1;
    C = 0;
    while (k) {
        if (k & 1) {
            C = (a * C + c) & kDrandMask;
            A = (a * A) & kDrandMask;
        }
        c = (a * c + c) & kDrandMask;
        a = (a * a) & kDrandMask;
        k >>= 1;
    }
}

// ---- union-find toward the minimum index.  After all unions every set's root is its
// smallest member, which is the canonical label.
__device__ __forceinline__ uint32_t uf_find(const volatile uint32_t *p, uint32_t x)
{
    uint32_t y = p[x];
    while (y != x) {
        x = y;
        y = p[x];
    }
    return x;
}

// Find that halves the path on the way (x's parent becomes its grandparent).  The update is
// an atomicMin, which only moves a pointer further toward the root, so it is safe while other
// threads unite; it keeps the trees that concurrent unions build shallow.
__device__ __forceinline__ uint32_t uf_find_halve(uint32_t *p, uint32_t x)
{
    const volatile uint32_t *vp = p;
    uint32_t y = vp[x];
    while (y != x) {
        const uint32_t z = vp[y];
        if (z == y)
            return y;
        atomicMin(p + x, z);
        x = z;
        y = vp[x];
    }
    return x;
}

__device__ __forceinline__ void uf_union(uint32_t *p, uint32_t a, uint32_t b)
{
    while (true) {
        a = uf_find_halve(p, a);
        b = uf_find_halve(p, b);
        if (a == b)
            return;
        if (a > b) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        const uint32_t old = atomicMin(p + b, a);
        if (old == b)
            return;  // b was a root and now hangs below a
        b = old;     // b was re-linked meanwhile: join a with b's new parent
    }
}

// ---- the same on the global label array, which other CTAs change concurrently.  Finds halve
// the path as they go (x's parent becomes its grandparent); the update is an atomicMin, which
// only ever moves a pointer to an ancestor, so it is safe against concurrent unions and keeps
// the trees shallow.  Every loop is capped: parents strictly decrease, so a chain longer than
// kChainCap means corrupt labels; the walk then stops and raises *fault.  Every value read is
// checked against the site count before it is used as an index: a label outside the lattice
// (only corrupt labels hold one) stops the walk too.  Fault bits: 1 chain cap, 2 union retry
// cap, 4 label outside the lattice.
constexpr uint32_t kChainCap = 1u << 22;
constexpr uint32_t kUnionRetryCap = 1u << 16;
constexpr unsigned int kFaultChain = 1u, kFaultRetry = 2u, kFaultRange = 4u;

__device__ __forceinline__ uint32_t guf_find(uint32_t *p, uint32_t x, const uint32_t n_sites, unsigned int *fault)
{
    if (x >= n_sites) {
        atomicOr(fault, kFaultRange);
        return 0;
    }
    const volatile uint32_t *vp = p;
    uint32_t y = vp[x];
    for (uint32_t n = 0; y != x; ++n) {
        if (y >= n_sites || n >= kChainCap) {
            atomicOr(fault, y >= n_sites ? kFaultRange : kFaultChain);
            return x;
        }
        const uint32_t z = vp[y];
        if (z == y)
            return y;
        if (z >= n_sites) {
            atomicOr(fault, kFaultRange);
            return y;
        }
        atomicMin(p + x, z);  // path halving
        x = z;
        y = vp[x];
    }
    return x;
}

constexpr uint32_t kNoLink = 0xFFFFFFFFu;  // guf_union_pair linked no root

// The same union with the two root walks advancing together, one level per step, so the loads
// of both chains are in flight at once.  Each step also points the node it leaves at its
// grandparent (path splitting, by atomicMin as above).  Same caps and fault bits.  Returns the
// root it linked below the other (each root is linked at most once: afterwards it is no root),
// or kNoLink when the two were already one tree.
__device__ __forceinline__ uint32_t guf_union_pair(uint32_t *p, uint32_t a, uint32_t b, const uint32_t n_sites,
                                                   unsigned int *fault)
{
    const volatile uint32_t *vp = p;
    for (uint32_t n = 0; n < kUnionRetryCap; ++n) {
        if (a >= n_sites || b >= n_sites) {  // the arguments, or a parent read by a failed link
            atomicOr(fault, kFaultRange);
            return kNoLink;
        }
        uint32_t ya = vp[a], yb = vp[b];
        for (uint32_t k = 0; ya != a || yb != b; ++k) {
            if (k >= kChainCap || ya >= n_sites || yb >= n_sites) {
                atomicOr(fault, k >= kChainCap ? kFaultChain : kFaultRange);
                return kNoLink;
            }
            const uint32_t za = ya != a ? vp[ya] : ya;
            const uint32_t zb = yb != b ? vp[yb] : yb;
            if (za >= n_sites || zb >= n_sites) {
                atomicOr(fault, kFaultRange);
                return kNoLink;
            }
            if (ya != a) {
                if (za != ya)
                    atomicMin(p + a, za);
                a = ya;
                ya = za;
            }
            if (yb != b) {
                if (zb != yb)
                    atomicMin(p + b, zb);
                b = yb;
                yb = zb;
            }
        }
        if (a == b)
            return kNoLink;
        if (a > b) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        const uint32_t old = atomicMin(p + b, a);
        if (old == b)
            return b;
        b = old;
    }
    atomicOr(fault, kFaultRetry);
    return kNoLink;
}

}  // namespace swb
