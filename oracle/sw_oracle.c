/* Test infrastructure, not product code: the CPU restatement described in sw_oracle.h.
 * Parity of this file with the reference is pinned by tests/test_oracle_golden.py
 * against dumps of the unmodified reference sources (tests/golden/). */
#include "sw_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- drand48 (POSIX): X' = 0x5DEECE66D * X + 0xB mod 2^48; srand48 sets X = seed << 16 | 0x330E. */
void orc_srand48(uint64_t *x, uint32_t seed)
{
    *x = ((uint64_t)seed << 16) | 0x330Eu;
}

double orc_drand48(uint64_t *x)
{
    *x = (0x5DEECE66Dull * *x + 0xBull) & ((1ull << 48) - 1);
    return ldexp((double)*x, -48);
}

/* ising/src/lattice.cpp:24-26 */
void orc_hot_start(uint32_t L0, uint32_t L1, uint32_t seed, uint8_t *spins)
{
    uint64_t x;
    size_t n = (size_t)L0 * L1;
    orc_srand48(&x, seed);
    for (size_t i = 0; i < n; ++i)
        spins[i] = orc_drand48(&x) < 0.5 ? 0 : 1;
}

/* Numerical Recipes LCG parameter pairs (a, c) chosen per lane (random/src/lcg32.cpp:17-24). */
static const uint32_t kParams[5][2] = {
    {1372383749u, 1289706101u},
    {2891336453u, 1640531513u},
    {2024337845u, 797082193u},
    {32310901u, 626627237u},
    {29943829u, 1013904223u},
};

static int valid_width(uint32_t W)
{
    return W >= 2 && W <= 64 && (W & (W - 1)) == 0;
}

/* random/src/lcg32.cpp:27-49 */
void orc_lcg32_init(uint32_t W, uint32_t seed, uint32_t *state, uint32_t *a, uint32_t *c, uint32_t *iteration)
{
    uint64_t x;
    orc_srand48(&x, seed);
    for (uint32_t i = 0; i < W; ++i) {
        uint32_t select = (uint32_t)(1000.0 * orc_drand48(&x)) % 5u;
        a[i] = kParams[select][0];
        c[i] = kParams[select][1];
    }
    state[0] = a[0] * ((uint32_t)(4026531839.0 /* 0xEFFFFFFF */ * orc_drand48(&x)) + 1u) + c[0];
    for (uint32_t i = 1; i < W; ++i)
        state[i] = a[i] * state[i - 1] + c[i];
    *iteration = 0;
}

/* random/src/lcg32.cpp:51-84: every 15th update first rotates the (a, c) pairs by
 * state[iteration & (W-1)] + (iteration odd ? 0 : 1), then every lane steps. */
void orc_lcg32_update(uint32_t W, uint32_t *state, uint32_t *a, uint32_t *c, uint32_t *iteration)
{
    uint32_t m = W - 1, buf[64];
    if ((++*iteration) % 15u == 0) {
        uint32_t shift = state[*iteration & m] + ((*iteration & 1u) ? 0u : 1u);
        for (uint32_t i = 0; i < W; ++i)
            buf[i] = a[(i + shift) & m];
        memcpy(a, buf, W * sizeof(uint32_t));
        for (uint32_t i = 0; i < W; ++i)
            buf[i] = c[(i + shift) & m];
        memcpy(c, buf, W * sizeof(uint32_t));
    }
    for (uint32_t i = 0; i < W; ++i)
        state[i] = a[i] * state[i] + c[i];
}

/* random/src/lcg32.cpp:103-129: element k of a request for n numbers is lane k % W after
 * update k / W + 1 of this request (the tail shorter than W also takes a fresh update);
 * the float is (float)u * 2^-32 with u rounded to nearest. */
void orc_lcg32_next_real(uint32_t W, uint32_t *state, uint32_t *a, uint32_t *c, uint32_t *iteration,
                         uint32_t n, float *out)
{
    for (uint32_t k = 0; k < n; k += W) {
        orc_lcg32_update(W, state, a, c, iteration);
        for (uint32_t l = 0; l < W && k + l < n; ++l)
            out[k + l] = (float)state[l] * 2.3283064365386963e-10f;
    }
}

/* ising/src/swendsen_wang.cpp:100 */
float orc_p_add(float temperature)
{
    return 1.0f - (float)expf(-2.0f / temperature);
}

uint32_t orc_num_tiles(uint32_t L0, uint32_t L1, uint32_t tx, uint32_t ty)
{
    return ((L0 + tx - 1) / tx) * ((L1 + ty - 1) / ty);
}

void orc_rng_init_tiles(uint32_t W, uint32_t n_tiles, uint32_t seed_base,
                        uint32_t *state, uint32_t *a, uint32_t *c, uint32_t *iteration)
{
    for (uint32_t t = 0; t < n_tiles; ++t)
        orc_lcg32_init(W, seed_base + t, state + (size_t)t * W, a + (size_t)t * W, c + (size_t)t * W, iteration + t);
}

/* Union-find toward the minimum index: the root of every set is its smallest element,
 * which is the canonical label the reference converges to (its tile-local min-propagation,
 * swendsen_wang_selflabeling.hpp:106-192, and its atomic-min merge, swendsen_wang_cpu.cpp:125-156). */
static uint32_t uf_find(uint32_t *p, uint32_t x)
{
    while (p[x] != x) {
        p[x] = p[p[x]];
        x = p[x];
    }
    return x;
}

static void uf_union(uint32_t *p, uint32_t a, uint32_t b)
{
    a = uf_find(p, a);
    b = uf_find(p, b);
    if (a < b)
        p[b] = a;
    else if (b < a)
        p[a] = b;
}

int orc_sw_sweep(uint32_t L0, uint32_t L1, uint32_t tx, uint32_t ty, uint32_t W, float p_add,
                 uint8_t *spins, uint32_t *rng_state, uint32_t *rng_a, uint32_t *rng_c, uint32_t *rng_iteration,
                 uint8_t *bonds, uint32_t *labels_assign, uint32_t *labels_final)
{
    if (L0 % 2 || L1 % 2) /* ising/src/swendsen_wang.cpp:47-48 */
        return 1;
    if (!valid_width(W))
        return 2;
    const size_t n = (size_t)L0 * L1;
    const uint32_t n0 = (L0 + tx - 1) / tx, n1 = (L1 + ty - 1) / ty;
    uint8_t *bond = (uint8_t *)calloc(n, 1);
    uint32_t *parent = (uint32_t *)malloc(n * sizeof(uint32_t));
    float *row = (float *)malloc((size_t)(tx + ty) * sizeof(float));
    if (!bond || !parent || !row) {
        free(bond); free(parent); free(row);
        return 3;
    }

    /* Phase 1 random numbers and bonds: per tile, one request of tx numbers per row for
     * the x-bonds (rows 0..jj_max-1), then one per row for the y-bonds (rows 0..jj_max-2)
     * (swendsen_wang_selflabeling.hpp:72-104); then the merge request of tx + ty numbers:
     * [0, tx) bottom edge, [tx, tx + ty) right edge (swendsen_wang_cpu.cpp:68-103).
     * A bond needs equal spins and r < p_add; the last column / row of a tile bonds only
     * through the merge request, to the periodic neighbour. */
    for (uint32_t t = 0; t < n0 * n1; ++t) {
        uint32_t *st = rng_state + (size_t)t * W, *aa = rng_a + (size_t)t * W, *cc = rng_c + (size_t)t * W;
        uint32_t *it = rng_iteration + t;
        const uint32_t j = (t / n0) * ty, i = (t % n0) * tx;
        const uint32_t ii_max = (tx < L0 - i) ? tx : L0 - i;
        const uint32_t jj_max = (ty < L1 - j) ? ty : L1 - j;
        for (uint32_t jj = 0; jj < jj_max; ++jj) {
            orc_lcg32_next_real(W, st, aa, cc, it, tx, row);
            for (uint32_t ii = 0; ii + 1 < ii_max; ++ii) {
                size_t s = (size_t)(j + jj) * L0 + i + ii;
                if (spins[s] == spins[s + 1] && row[ii] < p_add)
                    bond[s] |= 1;
            }
        }
        for (uint32_t jj = 0; jj + 1 < jj_max; ++jj) {
            orc_lcg32_next_real(W, st, aa, cc, it, tx, row);
            for (uint32_t ii = 0; ii < ii_max; ++ii) {
                size_t s = (size_t)(j + jj) * L0 + i + ii;
                if (spins[s] == spins[s + L0] && row[ii] < p_add)
                    bond[s] |= 2;
            }
        }
        orc_lcg32_next_real(W, st, aa, cc, it, tx + ty, row);
        for (uint32_t ii = 0; ii < ii_max; ++ii) {
            size_t s = (size_t)(j + jj_max - 1) * L0 + i + ii;
            size_t s2 = (size_t)((j + jj_max) % L1) * L0 + i + ii;
            if (row[ii] < p_add && spins[s] == spins[s2])
                bond[s] |= 2;
        }
        for (uint32_t jj = 0; jj < jj_max; ++jj) {
            size_t s = (size_t)(j + jj) * L0 + i + ii_max - 1;
            size_t s2 = (size_t)(j + jj) * L0 + (i + ii_max) % L0;
            if (row[tx + jj] < p_add && spins[s] == spins[s2])
                bond[s] |= 1;
        }
    }
    if (bonds)
        memcpy(bonds, bond, n);

    /* Tile-local components (AssignLabels, swendsen_wang_cpu.cpp:14-48): only bonds whose
     * both ends lie in the same tile. */
    for (size_t s = 0; s < n; ++s)
        parent[s] = (uint32_t)s;
    for (uint32_t y = 0; y < L1; ++y) {
        for (uint32_t x = 0; x < L0; ++x) {
            size_t s = (size_t)y * L0 + x;
            if ((bond[s] & 1) && x + 1 < L0 && (x + 1) % tx != 0)
                uf_union(parent, (uint32_t)s, (uint32_t)(s + 1));
            if ((bond[s] & 2) && y + 1 < L1 && (y + 1) % ty != 0)
                uf_union(parent, (uint32_t)s, (uint32_t)(s + L0));
        }
    }
    if (labels_assign)
        for (size_t s = 0; s < n; ++s)
            labels_assign[s] = uf_find(parent, (uint32_t)s);

    /* Cross-tile merge (MergeLabels, swendsen_wang_cpu.cpp:51-105) and resolution
     * (ResolveLabels, :158-180): all remaining bonds. */
    for (uint32_t y = 0; y < L1; ++y) {
        for (uint32_t x = 0; x < L0; ++x) {
            size_t s = (size_t)y * L0 + x;
            if ((bond[s] & 1) && (x + 1 == L0 || (x + 1) % tx == 0))
                uf_union(parent, (uint32_t)s, (uint32_t)((size_t)y * L0 + (x + 1) % L0));
            if ((bond[s] & 2) && (y + 1 == L1 || (y + 1) % ty == 0))
                uf_union(parent, (uint32_t)s, (uint32_t)((size_t)((y + 1) % L1) * L0 + x));
        }
    }
    for (size_t s = 0; s < n; ++s) {
        uint32_t r = uf_find(parent, (uint32_t)s);
        if (labels_final)
            labels_final[s] = r;
        /* FlipClusters (swendsen_wang_cpu.cpp:182-205): flip iff the cluster's label is odd. */
        spins[s] ^= (uint8_t)(r & 1u);
    }
    free(bond);
    free(parent);
    free(row);
    return 0;
}

/* ising/src/lattice.cpp:48-66 */
void orc_energy_magnetization(uint32_t L0, uint32_t L1, const uint8_t *spins, int64_t *e, int64_t *m)
{
    int64_t ee = 0, mm = 0;
    for (uint32_t y = 0; y < L1; ++y) {
        const uint8_t *r = spins + (size_t)y * L0, *d = spins + (size_t)((y + 1) % L1) * L0;
        for (uint32_t x = 0; x < L0; ++x) {
            int s = 2 * r[x] - 1;
            ee += s * ((2 * r[(x + 1) % L0] - 1) + (2 * d[x] - 1));
            mm += s;
        }
    }
    *e = ee;
    *m = mm;
}

void orc_block_labels(uint32_t L0, uint32_t L1, uint32_t BX, uint32_t BY, const uint8_t *bonds, uint32_t *out)
{
    const size_t n = (size_t)L0 * L1;
    for (size_t s = 0; s < n; ++s)
        out[s] = (uint32_t)s;
    for (uint32_t y = 0; y < L1; ++y) {
        for (uint32_t x = 0; x < L0; ++x) {
            size_t s = (size_t)y * L0 + x;
            if ((bonds[s] & 1) && x + 1 < L0 && (x + 1) % BX != 0)
                uf_union(out, (uint32_t)s, (uint32_t)(s + 1));
            if ((bonds[s] & 2) && y + 1 < L1 && (y + 1) % BY != 0)
                uf_union(out, (uint32_t)s, (uint32_t)(s + L0));
        }
    }
    for (size_t s = 0; s < n; ++s)
        out[s] = uf_find(out, (uint32_t)s);
}

/* ---- 3D Swendsen-Wang (this project's extension; the reference names it only in a comment,
 * ising/include/swendsen_wang_selflabeling.hpp:20-22).  Periodic L0 x L1 x L2, site index
 * (z L1 + y) L0 + x, tiles tx x ty x tz in row-major tile order, one lcg32 stream per tile.  Per
 * tile and sweep the draws extend the 2D order: per (kk, jj) row a request of tx numbers for the
 * +x bonds (the row's last site bonds through the face request), then per row with jj + 1 <
 * jj_max one for the +y bonds, then per row with kk + 1 < kk_max one for the +z bonds, then one
 * face request of tx tz + ty tz + tx ty numbers: the +y face (element kk tx + ii, the tile's last
 * row), the +x face (tx tz + kk ty + jj, its last column), the +z face (tx tz + ty tz + jj tx + ii,
 * its last layer), each to the periodic neighbour.  Rows run kk-major, then jj.  A bond needs
 * equal spins and an accepted draw; labels are the minimum site index of each cluster; a
 * cluster flips iff its label is odd.  With L2 = tz = 1 the bonds, labels and flips of a sweep
 * are the 2D sweep's (the face request begins with the 2D merge request; the z bonds join a site
 * to itself), which pins this restatement to the 2D one. */
int orc3_sw_sweep(uint32_t L0, uint32_t L1, uint32_t L2, uint32_t tx, uint32_t ty, uint32_t tz, uint32_t W,
                  float p_add, uint8_t *spins, uint32_t *rng_state, uint32_t *rng_a, uint32_t *rng_c,
                  uint32_t *rng_iteration, uint8_t *bonds, uint32_t *labels_final)
{
    if (L0 % 2 || L1 % 2 || (L2 % 2 && L2 != 1))
        return 1;
    if (!valid_width(W))
        return 2;
    const size_t plane = (size_t)L0 * L1, n = plane * L2;
    const uint32_t n0 = (L0 + tx - 1) / tx, n1 = (L1 + ty - 1) / ty, n2 = (L2 + tz - 1) / tz;
    const uint32_t nface = tx * tz + ty * tz + tx * ty;
    uint8_t *bond = (uint8_t *)calloc(n, 1);
    uint32_t *parent = (uint32_t *)malloc(n * sizeof(uint32_t));
    float *row = (float *)malloc((size_t)(nface > tx ? nface : tx) * sizeof(float));
    if (!bond || !parent || !row) {
        free(bond); free(parent); free(row);
        return 3;
    }
#define SITE(x, y, z) (((size_t)(z) * L1 + (y)) * L0 + (x))
    for (uint32_t t = 0; t < n0 * n1 * n2; ++t) {
        uint32_t *st = rng_state + (size_t)t * W, *aa = rng_a + (size_t)t * W, *cc = rng_c + (size_t)t * W;
        uint32_t *it = rng_iteration + t;
        const uint32_t i = (t % n0) * tx, j = ((t / n0) % n1) * ty, k = (t / (n0 * n1)) * tz;
        const uint32_t ii_max = tx < L0 - i ? tx : L0 - i;
        const uint32_t jj_max = ty < L1 - j ? ty : L1 - j;
        const uint32_t kk_max = tz < L2 - k ? tz : L2 - k;
        for (uint32_t kk = 0; kk < kk_max; ++kk)
            for (uint32_t jj = 0; jj < jj_max; ++jj) {
                orc_lcg32_next_real(W, st, aa, cc, it, tx, row);
                for (uint32_t ii = 0; ii + 1 < ii_max; ++ii) {
                    const size_t s = SITE(i + ii, j + jj, k + kk);
                    if (spins[s] == spins[s + 1] && row[ii] < p_add)
                        bond[s] |= 1;
                }
            }
        for (uint32_t kk = 0; kk < kk_max; ++kk)
            for (uint32_t jj = 0; jj + 1 < jj_max; ++jj) {
                orc_lcg32_next_real(W, st, aa, cc, it, tx, row);
                for (uint32_t ii = 0; ii < ii_max; ++ii) {
                    const size_t s = SITE(i + ii, j + jj, k + kk);
                    if (spins[s] == spins[s + L0] && row[ii] < p_add)
                        bond[s] |= 2;
                }
            }
        for (uint32_t kk = 0; kk + 1 < kk_max; ++kk)
            for (uint32_t jj = 0; jj < jj_max; ++jj) {
                orc_lcg32_next_real(W, st, aa, cc, it, tx, row);
                for (uint32_t ii = 0; ii < ii_max; ++ii) {
                    const size_t s = SITE(i + ii, j + jj, k + kk);
                    if (spins[s] == spins[s + plane] && row[ii] < p_add)
                        bond[s] |= 4;
                }
            }
        orc_lcg32_next_real(W, st, aa, cc, it, nface, row);
        for (uint32_t kk = 0; kk < kk_max; ++kk)
            for (uint32_t ii = 0; ii < ii_max; ++ii) {
                const size_t s = SITE(i + ii, j + jj_max - 1, k + kk);
                const size_t s2 = SITE(i + ii, (j + jj_max) % L1, k + kk);
                if (row[kk * tx + ii] < p_add && spins[s] == spins[s2])
                    bond[s] |= 2;
            }
        for (uint32_t kk = 0; kk < kk_max; ++kk)
            for (uint32_t jj = 0; jj < jj_max; ++jj) {
                const size_t s = SITE(i + ii_max - 1, j + jj, k + kk);
                const size_t s2 = SITE((i + ii_max) % L0, j + jj, k + kk);
                if (row[tx * tz + kk * ty + jj] < p_add && spins[s] == spins[s2])
                    bond[s] |= 1;
            }
        for (uint32_t jj = 0; jj < jj_max; ++jj)
            for (uint32_t ii = 0; ii < ii_max; ++ii) {
                const size_t s = SITE(i + ii, j + jj, k + kk_max - 1);
                const size_t s2 = SITE(i + ii, j + jj, (k + kk_max) % L2);
                if (row[tx * tz + ty * tz + jj * tx + ii] < p_add && spins[s] == spins[s2])
                    bond[s] |= 4;
            }
    }
    if (bonds)
        memcpy(bonds, bond, n);
    for (size_t s = 0; s < n; ++s)
        parent[s] = (uint32_t)s;
    for (uint32_t z = 0; z < L2; ++z)
        for (uint32_t y = 0; y < L1; ++y)
            for (uint32_t x = 0; x < L0; ++x) {
                const size_t s = SITE(x, y, z);
                if (bond[s] & 1)
                    uf_union(parent, (uint32_t)s, (uint32_t)SITE((x + 1) % L0, y, z));
                if (bond[s] & 2)
                    uf_union(parent, (uint32_t)s, (uint32_t)SITE(x, (y + 1) % L1, z));
                if (bond[s] & 4)
                    uf_union(parent, (uint32_t)s, (uint32_t)SITE(x, y, (z + 1) % L2));
            }
    for (size_t s = 0; s < n; ++s) {
        const uint32_t r = uf_find(parent, (uint32_t)s);
        if (labels_final)
            labels_final[s] = r;
        spins[s] ^= (uint8_t)(r & 1u);
    }
#undef SITE
    free(bond);
    free(parent);
    free(row);
    return 0;
}

/* e = sum s (s_x+ + s_y+ + s_z+), m = sum s over the periodic L0 x L1 x L2 lattice, s = 2b - 1. */
void orc3_energy_magnetization(uint32_t L0, uint32_t L1, uint32_t L2, const uint8_t *spins, int64_t *e, int64_t *m)
{
    int64_t ee = 0, mm = 0;
    for (uint32_t z = 0; z < L2; ++z)
        for (uint32_t y = 0; y < L1; ++y)
            for (uint32_t x = 0; x < L0; ++x) {
                const size_t s = ((size_t)z * L1 + y) * L0 + x;
                const int v = 2 * spins[s] - 1;
                const int rx = 2 * spins[((size_t)z * L1 + y) * L0 + (x + 1) % L0] - 1;
                const int ry = 2 * spins[((size_t)z * L1 + (y + 1) % L1) * L0 + x] - 1;
                const int rz = 2 * spins[((size_t)((z + 1) % L2) * L1 + y) * L0 + x] - 1;
                ee += v * (rx + ry + rz);
                mm += v;
            }
    *e = ee;
    *m = mm;
}
