/* Test infrastructure, not product code.
 *
 * CPU restatement of the reference's Swendsen-Wang sweep for the 2D Ising model
 * (flwende/computational_physics), used only as the checker by tests/, by
 * __graft_entry__.smoke() and by the cpu_baseline leg of bench.py.  Every function
 * cites the reference file:line it restates.  The restatement is pinned against the
 * reference itself: tests/golden/ holds stage dumps produced by the unmodified
 * reference CPU sources (oracle/ref_harness.cpp), and tests/test_oracle_golden.py
 * checks this file against them.
 *
 * Conventions shared with the product:
 *   spins   uint8 0/1, row-major, x fastest (ising/include/lattice.hpp:24)
 *   labels  uint32, the minimum global site index of the cluster
 *   bonds   uint8 per site, bit 0 = bond to +x neighbour, bit 1 = bond to +y neighbour
 *   lcg32   one stream per tile (tiles row-major), W lanes; per tile W state words,
 *           W multipliers a, W increments c and one iteration counter
 */
#ifndef SW_ORACLE_H
#define SW_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* POSIX drand48 family (used by random/src/lcg32.cpp:35-43, ising/src/lattice.cpp:24-26). */
void orc_srand48(uint64_t *x, uint32_t seed);
double orc_drand48(uint64_t *x);

/* Lattice<2> hot start: srand48(seed); spin = drand48() < 0.5 ? 0 : 1 (ising/src/lattice.cpp:15-27). */
void orc_hot_start(uint32_t L0, uint32_t L1, uint32_t seed, uint8_t *spins);

/* LCG32_State<W>::Init (random/src/lcg32.cpp:27-49). */
void orc_lcg32_init(uint32_t W, uint32_t seed, uint32_t *state, uint32_t *a, uint32_t *c, uint32_t *iteration);

/* LCG32_State<W>::Update with RANDOM_SHUFFLE_STATE (random/src/lcg32.cpp:51-84). */
void orc_lcg32_update(uint32_t W, uint32_t *state, uint32_t *a, uint32_t *c, uint32_t *iteration);

/* LCG32<CPU>::NextReal(vector of n) (random/src/lcg32.cpp:103-129). */
void orc_lcg32_next_real(uint32_t W, uint32_t *state, uint32_t *a, uint32_t *c, uint32_t *iteration,
                         uint32_t n, float *out);

/* p_add = 1 - exp(-2/T) in float (ising/src/swendsen_wang.cpp:100). */
float orc_p_add(float temperature);

/* Number of tiles of an L0 x L1 lattice with tx x ty tiles (ising/src/swendsen_wang_cpu.cpp:23-25). */
uint32_t orc_num_tiles(uint32_t L0, uint32_t L1, uint32_t tx, uint32_t ty);

/* Initialises the per-tile streams with seeds seed_base + tile id
 * (ising/src/swendsen_wang.cpp:59-73 with one stream per tile). */
void orc_rng_init_tiles(uint32_t W, uint32_t n_tiles, uint32_t seed_base,
                        uint32_t *state, uint32_t *a, uint32_t *c, uint32_t *iteration);

/* One sweep (ising/src/swendsen_wang.cpp:94-112 with the CPU phases of
 * ising/src/swendsen_wang_cpu.cpp and ising/include/swendsen_wang_selflabeling.hpp).
 * spins in/out; rng arrays in/out (n_tiles * W words, n_tiles counters); any of
 * bonds / labels_assign / labels_final may be NULL.  Returns 0, or 1 for odd extents,
 * 2 for an unsupported W, 3 on allocation failure. */
int orc_sw_sweep(uint32_t L0, uint32_t L1, uint32_t tx, uint32_t ty, uint32_t W, float p_add,
                 uint8_t *spins, uint32_t *rng_state, uint32_t *rng_a, uint32_t *rng_c, uint32_t *rng_iteration,
                 uint8_t *bonds, uint32_t *labels_assign, uint32_t *labels_final);

/* Integer sums behind Lattice<2>::GetEnergyAndMagnetization<CPU> (ising/src/lattice.cpp:29-67):
 * e = sum s (s_right + s_down), m = sum s with s = 2b - 1, periodic.  E/N = -e/N, M/N = m/N. */
void orc_energy_magnetization(uint32_t L0, uint32_t L1, const uint8_t *spins, int64_t *e, int64_t *m);

/* Components over the bonds whose two ends lie in the same BX x BY block (blocks tile the
 * lattice from the origin; a bond that wraps around the periodic edge never counts, even when
 * one block spans the lattice): out[s] = the minimum site index of s's component.  This is the
 * intermediate labelling of the GPU path, which merges the tiles of a block before the
 * cross-block merge; it is the reference's AssignLabels (swendsen_wang_cpu.cpp:14-48) with
 * blocks in place of tiles. */
void orc_block_labels(uint32_t L0, uint32_t L1, uint32_t BX, uint32_t BY, const uint8_t *bonds, uint32_t *out);

/* 3D Swendsen-Wang sweep (the draw order is described in sw_oracle.c; L2 = 1 gives the 2D sweep)
 * and its energy / magnetisation sums. */
int orc3_sw_sweep(uint32_t L0, uint32_t L1, uint32_t L2, uint32_t tx, uint32_t ty, uint32_t tz, uint32_t W,
                  float p_add, uint8_t *spins, uint32_t *rng_state, uint32_t *rng_a, uint32_t *rng_c,
                  uint32_t *rng_iteration, uint8_t *bonds, uint32_t *labels_final);
void orc3_energy_magnetization(uint32_t L0, uint32_t L1, uint32_t L2, const uint8_t *spins, int64_t *e, int64_t *m);

#ifdef __cplusplus
}
#endif

#endif
