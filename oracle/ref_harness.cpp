// Test infrastructure, not product code.
//
// Stage-dump harness around the UNMODIFIED reference CPU implementation of the
// Swendsen-Wang sweep (flwende/computational_physics).  It is compiled together
// with the reference sources by oracle/Makefile into oracle/_ref/libswref{16,8}.so
// and is only ever loaded by tests, by the golden-fixture generator in
// tests/golden/, and by the reference arm of bench.py.
//
// What it adds on top of the reference:
//   * one lcg32 stream per tile, seeded seed_base + tile_id (the reference seeds
//     its per-thread streams i + 1, ising/src/swendsen_wang.cpp:66-73; running
//     the CPU path with NUM_THREADS = number of tiles gives exactly this), by
//     driving AssignLabels / MergeLabels with a ThreadContext whose thread id is
//     the tile id (ising/src/swendsen_wang_cpu.cpp:16-31, 53-66);
//   * bond masks, which the reference never stores: a copy of each tile's
//     LCG32 is replayed in the reference's own consumption order and the
//     reference's own predicates are applied
//     (ising/include/swendsen_wang_selflabeling.hpp:72-104,
//      ising/src/swendsen_wang_cpu.cpp:79-103);
//   * dumps of the labels after AssignLabels and after ResolveLabels, and of
//     the spins after FlipClusters.
//
// Bond mask encoding per site: bit 0 = bond to the +x neighbour, bit 1 = bond
// to the +y neighbour (both periodic).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <chrono>
#include <memory>
#include <vector>

#include "swendsen_wang.hpp"

using namespace cp;

namespace
{
    using Strategy = SwendsenWang_2D<LCG32, DeviceName::CPU>;

    // Keeps the CPU device (and its thread group) alive for the harness' lifetime.
    CPU& HarnessCpu()
    {
        static CPU cpu(1, 0);
        return cpu;
    }

    class StageHarness : public Strategy
    {
        public:
            using Label = std::uint32_t;

            StageHarness(CPU& cpu) : Strategy(cpu) {}

            void Setup(Lattice<2>& lattice, std::uint32_t tx, std::uint32_t ty, std::uint32_t seed_base)
            {
                Initialize(lattice);
                tile_size = {tx, ty};
                const auto& extent = lattice.Extent();
                n0 = (extent[0] + tx - 1) / tx;
                n1 = (extent[1] + ty - 1) / ty;
                rng_state.clear();
                rng.clear();
                for (std::uint32_t t = 0; t < n0 * n1; ++t)
                    rng_state.emplace_back(seed_base + t);
                for (std::uint32_t t = 0; t < n0 * n1; ++t)
                    rng.emplace_back(new LCG32<DeviceName::CPU>(rng_state[t]));
                stack.resize((2 * tx * ty + tx) * sizeof(Label) + 256);
            }

            std::uint32_t NumTiles() const { return n0 * n1; }

            // Replays the random numbers of one sweep of tile t from a copy of its stream
            // and evaluates the reference's bond predicates on the current spins.
            void DumpBonds(Lattice<2>& lattice, float p_add, std::uint8_t* bonds)
            {
                const auto L0 = lattice.Extent()[0];
                const auto L1 = lattice.Extent()[1];
                const auto tx = tile_size[0];
                const auto ty = tile_size[1];
                std::vector<float> row(tx), edge(tx + ty);
                for (std::uint32_t t = 0; t < n0 * n1; ++t)
                {
                    auto copy = *static_cast<LCG32<DeviceName::CPU>*>(rng[t].get());
                    const auto j = (t / n0) * ty;
                    const auto i = (t % n0) * tx;
                    const auto ii_max = std::min(tx, L0 - i);
                    const auto jj_max = std::min(ty, L1 - j);
                    for (std::uint32_t jj = 0; jj < jj_max; ++jj)
                    {
                        copy.NextReal(row);
                        for (std::uint32_t ii = 0; ii + 1 < ii_max; ++ii)
                            if (lattice[j + jj][i + ii] == lattice[j + jj][i + ii + 1] && row[ii] < p_add)
                                bonds[(j + jj) * L0 + i + ii] |= 1;
                    }
                    for (std::uint32_t jj = 0; jj + 1 < jj_max; ++jj)
                    {
                        copy.NextReal(row);
                        for (std::uint32_t ii = 0; ii < ii_max; ++ii)
                            if ((lattice[j + jj][i + ii] & 1) == (lattice[j + jj + 1][i + ii] & 1) && row[ii] < p_add)
                                bonds[(j + jj) * L0 + i + ii] |= 2;
                    }
                    copy.NextReal(edge);
                    for (std::uint32_t ii = 0; ii < ii_max; ++ii)
                        if (edge[ii] < p_add && lattice[j + jj_max - 1][i + ii] == lattice[(j + jj_max) % L1][i + ii])
                            bonds[(j + jj_max - 1) * L0 + i + ii] |= 2;
                    for (std::uint32_t jj = 0; jj < jj_max; ++jj)
                        if (edge[tx + jj] < p_add && lattice[j + jj][i + ii_max - 1] == lattice[j + jj][(i + ii_max) % L0])
                            bonds[(j + jj) * L0 + i + ii_max - 1] |= 1;
                }
            }

            void Sweep(Lattice<2>& lattice, float temperature, std::uint8_t* bonds,
                       std::uint32_t* labels_assign, std::uint32_t* labels_final)
            {
                const float p_add = 1.0f - static_cast<float>(std::exp(-2.0f / temperature));
                const auto n = lattice.NumSites();
                if (bonds)
                {
                    std::memset(bonds, 0, n);
                    DumpBonds(lattice, p_add, bonds);
                }
                Barrier barrier(1);
                for (std::uint32_t t = 0; t < n0 * n1; ++t)
                {
                    ThreadContext context(n0 * n1, t, barrier);
                    context.StackMemory().Register(reinterpret_cast<std::byte*>(stack.data()), stack.size());
                    AssignLabels(context, lattice, p_add);
                    context.StackMemory().Reset();
                }
                if (labels_assign)
                    std::memcpy(labels_assign, cluster.RawPointer(), n * sizeof(Label));
                for (std::uint32_t t = 0; t < n0 * n1; ++t)
                {
                    ThreadContext context(n0 * n1, t, barrier);
                    MergeLabels(context, lattice, p_add);
                }
                {
                    ThreadContext context(1, 0, barrier);
                    ResolveLabels(context);
                }
                if (labels_final)
                    std::memcpy(labels_final, cluster.RawPointer(), n * sizeof(Label));
                {
                    ThreadContext context(1, 0, barrier);
                    FlipClusters(context, lattice);
                }
            }

            void ExportRng(std::uint32_t* state, std::uint32_t* a, std::uint32_t* c, std::uint32_t* iteration)
            {
                constexpr auto W = CPU::WavefrontSize<std::uint32_t>();
                struct Exposed : LCG32<DeviceName::CPU>
                {
                    const State& S() const { return state; }
                };
                struct ExposedState : LCG32<DeviceName::CPU>::State
                {
                    void Copy(std::uint32_t* s, std::uint32_t* aa, std::uint32_t* cc, std::uint32_t* it) const
                    {
                        std::memcpy(s, this->state, sizeof(this->state));
                        std::memcpy(aa, this->a, sizeof(this->a));
                        std::memcpy(cc, this->c, sizeof(this->c));
                        *it = this->iteration;
                    }
                };
                for (std::uint32_t t = 0; t < n0 * n1; ++t)
                {
                    const auto& st = static_cast<const Exposed*>(static_cast<LCG32<DeviceName::CPU>*>(rng[t].get()))->S();
                    static_cast<const ExposedState&>(st).Copy(state + t * W, a + t * W, c + t * W, iteration + t);
                }
            }

        private:
            std::uint32_t n0 {}, n1 {};
            std::vector<std::uint8_t> stack;
    };

    struct Run
    {
        Lattice<2> lattice;
        StageHarness harness;
        Run(std::uint32_t L0, std::uint32_t L1) : lattice({L0, L1}), harness(HarnessCpu()) {}
    };
}

extern "C"
{
    // Lane count W of the reference's lcg32 in this build (the host's SIMD width for uint32).
    int ref_lcg32_width() { return static_cast<int>(CPU::WavefrontSize<std::uint32_t>()); }

    // p_add exactly as ising/src/swendsen_wang.cpp:100.
    float ref_p_add(float temperature) { return 1.0f - static_cast<float>(std::exp(-2.0f / temperature)); }

    // Hot start of Lattice<2> (ising/src/lattice.cpp:15-27): srand48(1), drand48() < 0.5 ? 0 : 1.
    void ref_hot_start(std::uint32_t L0, std::uint32_t L1, std::uint8_t* spins)
    {
        Lattice<2> lattice({L0, L1});
        std::memcpy(spins, lattice.RawPointer(), lattice.NumSites());
    }

    // LCG32_State<W>::Init (random/src/lcg32.cpp:27-49).
    void ref_lcg32_init(std::uint32_t seed, std::uint32_t* state, std::uint32_t* a, std::uint32_t* c, std::uint32_t* iteration)
    {
        struct S : LCG32<DeviceName::CPU>::State
        {
            S(std::uint32_t seed) : LCG32<DeviceName::CPU>::State(seed) {}
            void Copy(std::uint32_t* s, std::uint32_t* aa, std::uint32_t* cc, std::uint32_t* it) const
            {
                std::memcpy(s, this->state, sizeof(this->state));
                std::memcpy(aa, this->a, sizeof(this->a));
                std::memcpy(cc, this->c, sizeof(this->c));
                *it = this->iteration;
            }
        } s(seed);
        s.Copy(state, a, c, iteration);
    }

    // LCG32<CPU>::NextReal(vector) called repeatedly with chunk sizes sizes[0..k-1]
    // on a stream seeded `seed` (random/src/lcg32.cpp:86-129).  Writes the raw
    // float bit patterns back to back.
    void ref_lcg32_next_real(std::uint32_t seed, const std::uint32_t* sizes, std::uint32_t k, float* out)
    {
        LCG32<DeviceName::CPU> rng(seed);
        std::size_t pos = 0;
        for (std::uint32_t i = 0; i < k; ++i)
        {
            std::vector<float> buffer(sizes[i]);
            rng.NextReal(buffer);
            std::memcpy(out + pos, buffer.data(), sizes[i] * sizeof(float));
            pos += sizes[i];
        }
    }

    // Energy and magnetization per site (ising/src/lattice.cpp:29-67).
    void ref_energy_magnetization(std::uint32_t L0, std::uint32_t L1, const std::uint8_t* spins, double* e, double* m)
    {
        Lattice<2> lattice({L0, L1});
        std::memcpy(lattice.RawPointer(), spins, lattice.NumSites());
        const auto [ee, mm] = lattice.GetEnergyAndMagnetization<DeviceName::CPU>();
        *e = ee;
        *m = mm;
    }

    // Runs n_sweeps sweeps of the reference CPU path on `spins` (in/out) with one lcg32
    // stream per tile (seed_base + tile id) and dumps the stages of the LAST sweep.
    // Any dump pointer may be null.  rng_* (may be null) receive the per-tile lcg32
    // states after the last sweep.
    int ref_sw_run(std::uint32_t L0, std::uint32_t L1, std::uint32_t tx, std::uint32_t ty,
                   std::uint32_t seed_base, float temperature, std::uint32_t n_sweeps,
                   std::uint8_t* spins, std::uint8_t* bonds, std::uint32_t* labels_assign,
                   std::uint32_t* labels_final,
                   std::uint32_t* rng_state, std::uint32_t* rng_a, std::uint32_t* rng_c, std::uint32_t* rng_iteration)
    {
        if (L0 % 2 || L1 % 2 || n_sweeps == 0)
            return 1;
        Run run(L0, L1);
        std::memcpy(run.lattice.RawPointer(), spins, run.lattice.NumSites());
        run.harness.Setup(run.lattice, tx, ty, seed_base);
        for (std::uint32_t s = 0; s < n_sweeps; ++s)
        {
            const bool last = (s + 1 == n_sweeps);
            run.harness.Sweep(run.lattice, temperature, last ? bonds : nullptr,
                              last ? labels_assign : nullptr, last ? labels_final : nullptr);
        }
        std::memcpy(spins, run.lattice.RawPointer(), run.lattice.NumSites());
        if (rng_state && rng_a && rng_c && rng_iteration)
            run.harness.ExportRng(rng_state, rng_a, rng_c, rng_iteration);
        return 0;
    }

    // The reference's own multi-threaded path: SwendsenWang_2D<LCG32, CPU>::Update
    // (ising/src/swendsen_wang.cpp:94-112) on `count` independent lattices, using a
    // CPU device with `num_threads` threads (the NUM_THREADS of the reference).
    // Each lattice gets its own strategy object, so lattices of different sizes can
    // be swept in one process.  Returns the wall seconds spent in the sweeps.
    double ref_cpu_sweep_many(std::uint32_t count, const std::uint32_t* extents, const float* temperatures,
                              std::uint8_t* const* spins, std::uint32_t n_sweeps, std::uint32_t num_threads)
    {
        CPU cpu(num_threads, 0);
        std::vector<std::unique_ptr<Lattice<2>>> lattices;
        std::vector<std::unique_ptr<Strategy>> strategies;
        for (std::uint32_t k = 0; k < count; ++k)
        {
            lattices.emplace_back(new Lattice<2>({extents[k], extents[k]}));
            std::memcpy(lattices.back()->RawPointer(), spins[k], lattices.back()->NumSites());
            strategies.emplace_back(new Strategy(cpu));
            // First Update initialises tile size, labels and lcg32 streams; it is a real sweep.
        }
        const auto t0 = std::chrono::steady_clock::now();
        for (std::uint32_t s = 0; s < n_sweeps; ++s)
            for (std::uint32_t k = 0; k < count; ++k)
                strategies[k]->Update(*lattices[k], temperatures[k]);
        const auto t1 = std::chrono::steady_clock::now();
        for (std::uint32_t k = 0; k < count; ++k)
            std::memcpy(spins[k], lattices[k]->RawPointer(), lattices[k]->NumSites());
        return std::chrono::duration<double>(t1 - t0).count();
    }
}
