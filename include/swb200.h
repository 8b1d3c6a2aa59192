/*
 * swb200.h -- C ABI of the B200-native Swendsen-Wang engine for the 2D Ising model.
 *
 * This is the boundary a host program (C, C++, Python ctypes, ...) binds.  It carries
 * only plain pointers and sizes.  Every function returns SWB_OK (0) or a non-zero
 * status; swb_last_error() gives the message of the last failure on the calling thread.
 * Host buffers belong to the caller; device buffers belong to the engine handle.  A
 * handle is driven by one host thread at a time (it owns one CUDA stream).
 *
 * Conventions (identical to the reference flwende/computational_physics):
 *   spins   uint8 0/1, row-major, x fastest            (ising/include/lattice.hpp:24)
 *   labels  uint32, minimum global site index of the cluster
 *   bonds   uint8 per site: bit 0 = +x bond, bit 1 = +y bond (periodic)
 *   lcg32   one stream per tile, tiles row-major, seeded seed_base + tile id; the stream
 *           state is exchanged in the reference's LCG32_State<W> terms: W state words,
 *           W multipliers a, W increments c, one iteration counter per tile
 *           (random/include/random/lcg32.hpp:27-58)
 */
#ifndef SWB200_H
#define SWB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SWB_OK 0
#define SWB_ERR_ARGUMENT 1   /* invalid size, extent, tile, width or pointer            */
#define SWB_ERR_CUDA 2       /* a CUDA runtime call failed                              */
#define SWB_ERR_STATE 3      /* call not valid in the handle's current state            */
#define SWB_ERR_CAPACITY 4   /* request exceeds a configured capacity (samples, budget) */

typedef struct swb_lattice swb_lattice;

/* Library version string. */
const char *swb_version(void);

/* Message of the last failed call on this thread ("" if none). */
const char *swb_last_error(void);

/* Number of visible CUDA devices (0 when there is no GPU or driver). */
int swb_device_count(int *count);

/* Number of kernel launches this process has issued through the library (all handles). */
uint64_t swb_kernel_launches(void);

/* ---- single lattice: the drop-in for SwendsenWang_2D<LCG32, Target>::Update ------------- */

/* Creates an L0 x L1 periodic lattice on CUDA device `device` with tiles tile_x x tile_y
 * and lcg32 streams of `lcg_width` lanes seeded seed_base + tile id.  Replaces
 * SwendsenWang_2D::Initialize (ising/src/swendsen_wang.cpp:41-92): extents must be
 * even (:47-48); at most 2^31 - 1 sites (labels are uint32, swendsen_wang.hpp:28-29, with
 * the top bit used internally).  tile_x in {8, 16, 32},
 * 2 <= tile_y <= 32, lcg_width in {8, 16, 32}.  Spins start all 0.  A lattice of full
 * 128 x 32-site blocks, or of at least 4096 blocks, resolves merged roots in a kernel of
 * their own before the flip, others in the flip; the environment variable
 * SWB_RESOLVE_MIN_BLOCKS, read here, replaces that rule by a block count.  Both forms give
 * identical results. */
int swb_create(swb_lattice **out, uint32_t L0, uint32_t L1, uint32_t tile_x, uint32_t tile_y,
               uint32_t lcg_width, uint32_t seed_base, int device);

/* Releases every device buffer of the handle (reference: GpuPointer deleters,
 * utility/hip/hip.hpp:18-39). */
int swb_destroy(swb_lattice *h);

/* Copies host spins (L0*L1 bytes, 0/1) to the device: Lattice<2>::InitializeGpuSpins
 * (ising/src/lattice.cpp:81-96).  Values other than 0/1 are rejected. */
int swb_set_spins(swb_lattice *h, const uint8_t *host_spins);

/* Copies the device spins to the host (L0*L1 bytes). */
int swb_get_spins(swb_lattice *h, uint8_t *host_spins);

/* Hot start on the device, bit-identical to Lattice<2>'s constructor with srand48(seed)
 * (ising/src/lattice.cpp:15-27; the reference always uses seed 1). */
int swb_hot_start(swb_lattice *h, uint32_t seed);

/* All spins set to `value` (0 or 1): a cold start. */
int swb_cold_start(swb_lattice *h, uint8_t value);

/* p_add = 1 - exp(-2/T) in float, as ising/src/swendsen_wang.cpp:100. */
float swb_p_add(float temperature);

/* The integer form of the bond test: a draw u is accepted iff u < swb_accept_threshold(p_add),
 * which equals the reference's (float)u * 2^-32 < p_add (random/src/lcg32.cpp:120-129). */
uint32_t swb_accept_threshold(float p_add);

/* n_sweeps sweeps at `temperature`: SwendsenWang_2D::Update (ising/src/swendsen_wang.cpp:94-112)
 * -- bond activation + tile labelling, boundary merge, label resolution, cluster flip.  If
 * measure_every > 0, after every measure_every-th sweep the energy and magnetisation are
 * accumulated on the device (E, E^2, |M| in FP64, and the exact integer sums per sample).  The
 * sample of the spins after a sweep is taken by the next sweep's assign phase, which reads those
 * spins anyway, when the next sweep follows on this handle; otherwise (the last sweep of a
 * call, or lattices narrower than 32 sites per block) a reduction kernel takes it before the
 * observables are read, the spins change or an unmeasured sweep runs.  Either way the samples
 * and their order are those of a measurement right after the sweep.
 * Asynchronous on the handle's stream; errors of the launches are reported. */
int swb_sweep(swb_lattice *h, float temperature, uint32_t n_sweeps, uint32_t measure_every);

/* Like swb_sweep with n_sweeps = 1, additionally dumping this sweep's stages to HOST buffers
 * (each may be NULL): bonds (uint8 per site), labels after tile-local labelling
 * (AssignLabels), labels after resolution (ResolveLabels).  The assign phase of this sweep
 * labels tile by tile (the reference's own stage split, ising/src/swendsen_wang.cpp:105-112),
 * a different kernel instance from the one swb_sweep runs; swb_sweep_dumped records that one.
 * Synchronous. */
int swb_sweep_recorded(swb_lattice *h, float temperature, uint8_t *bonds, uint32_t *labels_assign,
                       uint32_t *labels_final);

/* One sweep through the same kernels swb_sweep runs, with their dumps switched on, to HOST
 * buffers (each may be NULL): bonds (as swb_sweep_recorded), labels_block = the minimum global
 * site index of each site's component over the bonds inside its block (swb_geometry gives the
 * block shape; bonds across block edges and the periodic wrap are left to the merge), and the
 * resolved labels (ResolveLabels, ising/src/swendsen_wang_cpu.cpp:160-180).  Synchronous. */
int swb_sweep_dumped(swb_lattice *h, float temperature, uint8_t *bonds, uint32_t *labels_block,
                     uint32_t *labels_final);

/* Geometry of the handle: geometry[0..7] = L0, L1, tile_x, tile_y, block_x, block_y (sites per
 * assign block), blocks in x, blocks in y. */
int swb_geometry(swb_lattice *h, uint32_t *geometry);

/* Waits for all work of the handle. */
int swb_synchronize(swb_lattice *h);

/* Energy and magnetisation per site of the current spins (Lattice<2>::GetEnergyAndMagnetization,
 * ising/src/lattice.cpp:29-79), reduced on the device: out[0] = E/N, out[1] = M/N.
 * The exact integer sums go to e_sum / m_sum when non-NULL. */
int swb_energy_magnetization(swb_lattice *h, double *out, int64_t *e_sum, int64_t *m_sum);

/* Observable accumulators since the last reset: out[0] = sum E/N, out[1] = sum (E/N)^2,
 * out[2] = sum |M/N|, out[3] = number of samples.  Synchronous. */
int swb_accumulators(swb_lattice *h, double *out);

/* Clears the accumulators and the sample series. */
int swb_reset_accumulators(swb_lattice *h);

/* Copies up to `capacity` recorded samples (exact integer sums e, m per measured sweep,
 * interleaved e0, m0, e1, m1, ...) to the host; *count receives the number recorded. */
int swb_samples(swb_lattice *h, int64_t *em, uint64_t capacity, uint64_t *count);

/* Number of tiles and the lane count of the handle's lcg32 streams. */
int swb_rng_shape(swb_lattice *h, uint32_t *n_tiles, uint32_t *lcg_width);

/* Exports / imports the per-tile lcg32 streams in LCG32_State<W> terms (arrays n_tiles*W,
 * n_tiles).  Import rejects (a, c) pairs that are not one of the reference's five
 * parameter pairs (random/src/lcg32.cpp:17-24). */
int swb_get_rng(swb_lattice *h, uint32_t *state, uint32_t *a, uint32_t *c, uint32_t *iteration);
int swb_set_rng(swb_lattice *h, const uint32_t *state, const uint32_t *a, const uint32_t *c,
                const uint32_t *iteration);

/* Device pointers of the spin and label arrays (for zero-copy interop; valid until destroy).
 * Between sweeps the label array holds the engine's internal encoding; resolved labels (the
 * minimum site index of each cluster) are there after swb_sweep_recorded. */
int swb_device_buffers(swb_lattice *h, void **spins, void **labels);

/* Number of kernel launches one plain sweep issues on this handle. */
int swb_launches_per_sweep(swb_lattice *h, uint32_t *launches);

/* n_sweeps sweeps like swb_sweep (no measurement), timed with CUDA events on the handle's
 * stream.  ms[0] = total elapsed; when per_kernel != 0 events bracket every phase and
 * ms[1..3] = summed durations of the assign, merge and resolve + flip kernels.  Synchronous. */
int swb_sweep_timed(swb_lattice *h, float temperature, uint32_t n_sweeps, int per_kernel, float *ms);

/* Page-locked host memory for fast host<->device copies (cudaHostAlloc / cudaFreeHost). */
int swb_host_alloc(void **ptr, size_t bytes);
int swb_host_free(void *ptr);

/* ---- 3D: the Swendsen-Wang sweep of the 3D Ising model ------------------------------------ */
/* No counterpart in the reference, which names the 3D case only
 * (ising/include/swendsen_wang_selflabeling.hpp:20-22).  The 2D conventions extended to a
 * periodic L0 x L1 x L2 lattice: spins uint8 0/1 at (z L1 + y) L0 + x; one lcg32 stream per
 * tile of tile_x x tile_y x tile_z sites (tiles row-major), seeded seed_base + tile id; per tile
 * and sweep the draws are, row by row (z-major), tile_x numbers for the +x bonds, then for the
 * +y bonds of every row but the tile's last, then for the +z bonds of every layer but its last,
 * then one request of tx tz + ty tz + tx ty numbers for its +y, +x and +z faces (the order of
 * oracle/sw_oracle.c orc3_sw_sweep, which L2 = 1 reduces to the 2D sweep); labels are the
 * minimum site index of each cluster and a cluster flips iff its label is odd. */
typedef struct swb_lattice3 swb_lattice3;

/* L0, L1 even, L2 even or 1; tile_x in {8, 16, 32}, 1 <= tile_y, tile_z <= 8; lcg_width in {8,
 * 16, 32}.  Spins start all 0. */
int swb3_create(swb_lattice3 **out, uint32_t L0, uint32_t L1, uint32_t L2, uint32_t tile_x, uint32_t tile_y,
                uint32_t tile_z, uint32_t lcg_width, uint32_t seed_base, int device);
int swb3_destroy(swb_lattice3 *h);
/* geometry[0..11] = L0, L1, L2, tile x, y, z, block x, y, z (sites), blocks in x, y, z. */
int swb3_geometry(swb_lattice3 *h, uint32_t *geometry);
int swb3_set_spins(swb_lattice3 *h, const uint8_t *host_spins);
int swb3_get_spins(swb_lattice3 *h, uint8_t *host_spins);
/* Site i takes drand48 draw i + 1 after srand48(seed), as Lattice<2>'s hot start. */
int swb3_hot_start(swb_lattice3 *h, uint32_t seed);
/* n_sweeps sweeps; with measure_every > 0 e = sum s (s_x+ + s_y+ + s_z+) and m = sum s are
 * recorded after every measure_every-th sweep (E/N = -e / N). */
int swb3_sweep(swb_lattice3 *h, float temperature, uint32_t n_sweeps, uint32_t measure_every);
/* One sweep with its bonds (bit 0 +x, 1 +y, 2 +z) and resolved labels dumped to host buffers
 * (each may be NULL).  Synchronous. */
int swb3_sweep_dumped(swb_lattice3 *h, float temperature, uint8_t *bonds, uint32_t *labels_final);
/* n_sweeps sweeps timed with CUDA events on the handle's stream (ms of all of them). */
int swb3_sweep_timed(swb_lattice3 *h, float temperature, uint32_t n_sweeps, float *ms);
int swb3_energy_magnetization(swb_lattice3 *h, double *out, int64_t *e_sum, int64_t *m_sum);
/* Recorded samples (e, m interleaved) and the accumulators (sum E/N, sum (E/N)^2, sum |M/N|,
 * samples; acc may be NULL). */
int swb3_samples(swb_lattice3 *h, int64_t *em, uint64_t capacity, uint64_t *count, double *acc);
int swb3_rng_shape(swb_lattice3 *h, uint32_t *n_tiles, uint32_t *lcg_width);
int swb3_get_rng(swb_lattice3 *h, uint32_t *state, uint32_t *a, uint32_t *c, uint32_t *iteration);

/* ---- device memory and devices, for host programs that include no CUDA header ----------- */

/* Makes the handle sweep a caller-owned spin array in device memory (L0*L1 bytes, 0/1,
 * 16-byte aligned, on the handle's device) instead of its own, which is released: the
 * reference's Lattice<2> owns its GPU spins and hands them to the strategy
 * (Lattice<2>::InitializeGpuSpins / RawGpuPointer, ising/include/lattice.hpp:77-80,92-94).  The
 * buffer must outlive the handle's use of it; swb_destroy does not free it. */
int swb_attach_spins(swb_lattice *h, void *device_spins);

/* Device memory on CUDA device `device` (256-byte aligned, `bytes` plus 16 bytes of slack) and
 * its release: the hipMalloc / GpuPointer of the reference's GPU lattice storage
 * (ising/src/lattice.cpp:81-96, utility/hip/hip.hpp). */
int swb_device_alloc(int device, size_t bytes, void **ptr);
int swb_device_free(int device, void *ptr);

/* Synchronous host <-> device copies (hipMemcpy in ising/src/lattice.cpp:74,89): each first
 * waits for all work queued on the device (the handles' streams included). */
int swb_copy_to_device(int device, void *dst, const void *src, size_t bytes);
int swb_copy_to_host(int device, void *dst, const void *src, size_t bytes);

/* Waits for all work on the device: HipContext::Synchronize (utility/execution/hip_context.hpp:18-22). */
int swb_device_synchronize(int device);

/* Multiprocessor count: the default of NUM_THREADS_GPU for the GPU device
 * (utility/device/device_amd_gpu.hpp:20). */
int swb_device_sm_count(int device, uint32_t *count);

/* Energy and magnetisation per site of any device spin array (L0 x L1, 0/1), reduced on the
 * device: out[0] = E/N, out[1] = M/N, the integer sums to e_sum / m_sum (each may be NULL).
 * Lattice<2>::GetEnergyAndMagnetization<AMD_GPU> copies the spins to the host for this
 * (ising/src/lattice.cpp:70-79).  Synchronous: it first waits for all work queued on the device,
 * so a lattice swept on a handle's stream is measured after those sweeps; calls on one device
 * are serialised. */
int swb_spins_energy_magnetization(int device, uint32_t L0, uint32_t L1, const void *device_spins, double *out,
                                   int64_t *e_sum, int64_t *m_sum);

/* One sweep through HOST spin buffers, as the reference's Lattice<2> keeps them: copy
 * spins_in to the device, sweep, read the spins back to spins_out and the energy and
 * magnetisation per site to em_out[2] (may be NULL).  Synchronous. */
int swb_update_host(swb_lattice *h, float temperature, const uint8_t *spins_in, uint8_t *spins_out,
                    double *em_out);

/* No counterpart in the reference.  n_sweeps sweeps of a lattice whose buffers the CALLER owns,
 * allocating nothing: for hosts that keep the lattice in device memory they manage themselves
 * (an FFI caller's own lattice storage, a pool holding the whole HBM budget), where a per-call
 * cudaMalloc can fail and a cudaFree would synchronise the device.  Device buffers, on the
 * current device: spins[L0*L1] (0/1, 16-byte aligned), rng_state[n_tiles*W], rng_sel[n_tiles*W]
 * (index 0..4 of the lcg32 parameter pair, random/src/lcg32.cpp:17-24), rng_iter[n_tiles],
 * n_tiles = ceil(L0/tile_x) * ceil(L1/tile_y) -- the layout swb_get_rng exports.  Results equal
 * swb_sweep's on the same state.  The label array, block edge words and fault word live in one
 * static device array of 24 MiB + 1 KiB, so L0*L1 is at most 4,194,304 (2048 x 2048); larger
 * lattices return SWB_ERR_CAPACITY before any CUDA call.  All calls on a device share that array
 * (each call clears its fault word, the kernels overwrite the rest): calls that overlap on the
 * GPU race, so serialise them (one stream, or events).  The first call on each device looks the
 * array's address up (cudaGetSymbolAddress, with that device current); make that first call
 * before any stream capture.  The array is reserved on a device (and held until the process
 * exits) only once this entry point has been called there.  The merged block roots are always
 * resolved by the flip itself (the three-kernel form of swb_sweep; at 2048 x 2048 about 5 %
 * slower than the four-kernel form swb_sweep uses there): the array has no room for the merge
 * slots.  Asynchronous on `stream` (NULL = default stream); with wait != 0 the call
 * synchronises the stream and reports a label union-find fault as SWB_ERR_STATE.  With wait == 0 such
 * a fault is not reported: the next call clears the fault word. */
int swb_sweep_static(void *stream, uint32_t L0, uint32_t L1, uint32_t tile_x, uint32_t tile_y, uint32_t lcg_width,
                     float temperature, uint32_t n_sweeps, uint8_t *spins, uint32_t *rng_state, uint8_t *rng_sel,
                     uint32_t *rng_iter, int wait);

/* ---- the lcg32 generator on its own ---------------------------------------------------- */

/* Throughput kernel of lcg32, the equivalent of the reference's TestRNG --target
 * (random/src/test_rng.cpp, random/src/test_rng_amd_gpu.cpp:44-133): n_streams streams of
 * lcg_width lanes, stream i seeded seed_base + i (LCG32_State::Init), each advanced
 * updates_per_stream times (a positive multiple of 64 / lcg_width); every update yields
 * lcg_width numbers 2^-32 * (float)u in NextReal order (random/src/lcg32.cpp:103-129).
 * report[64] receives the last 64 numbers of stream report_id (the reference's 64-number
 * buffer), *checksum the XOR of the bit patterns of every number generated, *ms the kernel
 * time (CUDA events, stream initialisation included).  Synchronous. */
int swb_lcg32_benchmark(uint32_t n_streams, uint32_t lcg_width, uint32_t seed_base, uint64_t updates_per_stream,
                        uint32_t report_id, float *report, uint32_t *checksum, float *ms, int device);

/* ---- batched lattices: many independent lattices advanced by one kernel launch per sweep
 * phase over all their blocks, replayed as a CUDA graph.  No counterpart in the reference, whose
 * Lattice<2>::Update holds one static strategy per process (ising/include/lattice.hpp:51-57);
 * every lattice still sweeps bit-identically to the single-lattice path with the same
 * extent, tile, lcg width and seeds. ------------------------------------------------------ */

typedef struct swb_batch swb_batch;

/* Creates an empty batch on `device` with room for `capacity` lattices.  hbm_budget_bytes
 * caps the device memory of all lattices together (0 = no cap).  All lattices of a batch
 * use lcg32 streams of `lcg_width` lanes. */
int swb_batch_create(swb_batch **out, uint32_t capacity, uint64_t hbm_budget_bytes, uint32_t lcg_width, int device);
int swb_batch_destroy(swb_batch *b);

/* Device bytes swb_batch_add would reserve for such a lattice (the admission estimate). */
int swb_batch_lattice_bytes(uint32_t L0, uint32_t L1, uint32_t tile_x, uint32_t tile_y, uint32_t lcg_width,
                            uint64_t *bytes);

/* Adds an L0 x L1 lattice with tiles tile_x x tile_y, block_x x block_y tiles per work item
 * (0 = largest that fits), temperature T and streams seeded seed_base + tile id.  Spins start
 * all 0; the lattice sweeps without limit until swb_batch_set_schedule.  Fails with
 * SWB_ERR_CAPACITY when no slot is free or the HBM budget would be exceeded. */
int swb_batch_add(swb_batch *b, uint32_t L0, uint32_t L1, uint32_t tile_x, uint32_t tile_y, uint32_t block_x,
                  uint32_t block_y, float temperature, uint32_t seed_base, uint32_t *id);
int swb_batch_remove(swb_batch *b, uint32_t id);

int swb_batch_hot_start(swb_batch *b, uint32_t id, uint32_t seed);
int swb_batch_set_spins(swb_batch *b, uint32_t id, const uint8_t *host_spins);
int swb_batch_get_spins(swb_batch *b, uint32_t id, uint8_t *host_spins);
int swb_batch_set_temperature(swb_batch *b, uint32_t id, float temperature);

/* Lattice `id` runs `sweeps` more sweeps (0xFFFFFFFF = unlimited) and is measured after every
 * measure_every-th of its sweeps (0 = never), counted on the device. */
int swb_batch_set_schedule(swb_batch *b, uint32_t id, uint32_t sweeps, uint32_t measure_every);
int swb_batch_status(swb_batch *b, uint32_t id, uint32_t *sweeps_left, uint32_t *sweeps_done);

/* sweeps_left / sweeps_done (may be NULL) of every slot, arrays of `capacity` entries (0 for
 * free slots), in one device-to-host copy.  Synchronous. */
int swb_batch_poll(swb_batch *b, uint32_t *sweeps_left, uint32_t *sweeps_done);

/* n_rounds rounds: every lattice with sweeps left sweeps once per round.  measure != 0 adds
 * the measurement phase.  Asynchronous (CUDA graph replays on the batch's stream). */
int swb_batch_sweep(swb_batch *b, uint32_t n_rounds, int measure);

/* Non-blocking progress, for a host loop that keeps the device busy without waiting on it:
 * swb_batch_mark records a point after the work submitted so far (ids count up from 0; the
 * last 64 stay queryable), swb_batch_mark_query tells whether the device has passed it
 * (*done) and, if so, its time in ms since the first mark (*ms, may be NULL), from device
 * events.  No counterpart in the reference, whose GPU path synchronises after every kernel. */
int swb_batch_mark(swb_batch *b, uint32_t *mark);
int swb_batch_mark_query(swb_batch *b, uint32_t mark, int *done, double *ms);
int swb_batch_synchronize(swb_batch *b);

/* Like swb_batch_sweep without measurement, timed with CUDA events: ms[0] total; with
 * per_kernel, ms[1..3] = assign, merge, resolve + flip kernel time summed over rounds.
 * Synchronous. */
int swb_batch_sweep_timed(swb_batch *b, uint32_t n_rounds, int per_kernel, float *ms);

/* Per-lattice observables, as swb_accumulators / swb_samples. */
int swb_batch_accumulators(swb_batch *b, uint32_t id, double *out);
int swb_batch_samples(swb_batch *b, uint32_t id, int64_t *em, uint64_t capacity, uint64_t *count);

/* The same read for a lattice that has finished its sweep budget, without waiting for the
 * batch's other work: valid once a mark (swb_batch_mark) recorded after the lattice's last sweep
 * has been passed (no later round writes its samples); acc[4] (may be NULL) receives its
 * accumulators as swb_batch_accumulators does. */
int swb_batch_samples_finished(swb_batch *b, uint32_t id, int64_t *em, uint64_t capacity, uint64_t *count,
                               double *acc);
int swb_batch_get_rng(swb_batch *b, uint32_t id, uint32_t *state, uint32_t *a, uint32_t *c, uint32_t *iteration);
/* Imports lattice id's lcg32 streams (as swb_set_rng): with the spins, the whole state a
 * preempted job needs to resume bit-identically.  Synchronous. */
int swb_batch_set_rng(swb_batch *b, uint32_t id, const uint32_t *state, const uint32_t *a, const uint32_t *c,
                      const uint32_t *iteration);

/* geometry[8] = L0, L1, tile_x, tile_y, tiles per block x, tiles per block y, tiles, blocks. */
int swb_batch_info(swb_batch *b, uint32_t id, uint32_t *geometry);
int swb_batch_memory(swb_batch *b, uint64_t *used, uint64_t *budget);

/* One round through HOST spin buffers: copy spins_in[k] to lattice ids[k], sweep every
 * lattice once, copy the spins back to spins_out[k].  Buffers that follow each other in host
 * memory (spins_in[k + 1] == spins_in[k] + L0 * L1 of lattice ids[k]; same for spins_out) move
 * in one copy, so one pinned arena for all lattices needs one copy per direction.  Each id at
 * most once.  Synchronous. */
int swb_batch_update_host(swb_batch *b, uint32_t count, const uint32_t *ids, const uint8_t *const *spins_in,
                          uint8_t *const *spins_out);

/* n_rounds rounds of swb_batch_update_host that hand the spins back and forth between two sets
 * of host buffers: round r copies in from spins_a when r is even (spins_b when odd), sweeps
 * every lattice once and copies out to the other set, so after an odd number of rounds the
 * spins are in spins_b, after an even number in spins_a.  Every round moves all listed
 * lattices' spins in and out of the device; the rounds form one pipeline (a group of lattices
 * starts its next round's copy in as soon as its copy out has landed) with one synchronisation
 * at the end.  Synchronous. */
int swb_batch_update_host_rounds(swb_batch *b, uint32_t count, const uint32_t *ids, uint8_t *const *spins_a,
                                 uint8_t *const *spins_b, uint32_t n_rounds);

#ifdef __cplusplus
}
#endif

#endif
