// Keyed-Philox replacement for the reference's rng/BRNG.cxx, linked into the
// oracle harness in place of that file so the reference routines draw from
// the same streams as the GPU kernels.
//
// TEST INFRASTRUCTURE ONLY.
//
// The reference API is kept: SetSeed(u, v) sets the 64-bit Philox key to
// u | v << 32 and brng() returns the next draw of the current stream, mapped
// to [0, 1) exactly as rng/BRNG.cxx:33 maps its words.  The harness selects
// the current stream (kind, step, entity) before each reference call.
#include <cstdint>

#include "../../include/dsmc_philox.h"

namespace {
dsmc_stream g_stream;
std::uint64_t g_seed = 0;
std::uint64_t g_draws = 0;
} // namespace

extern "C" void dsmc_ref_rng_select(std::uint32_t kind, std::uint32_t step, std::uint32_t entity)
{
    dsmc_stream_init(&g_stream, g_seed, kind, step, entity);
}

extern "C" std::uint64_t dsmc_ref_rng_draws() { return g_draws; }

extern "C" void dsmc_ref_rng_set_seed64(std::uint64_t seed)
{
    g_seed = seed;
    dsmc_stream_init(&g_stream, g_seed, DSMC_RNG_USER, 0, 0);
}

void SetSeed(unsigned int u, unsigned int v)
{
    dsmc_ref_rng_set_seed64(static_cast<std::uint64_t>(u) | (static_cast<std::uint64_t>(v) << 32));
}

// The reference exposes its generator step; here it is the next 32-bit word
// of the current stream.
unsigned int IntUniform(unsigned int &, unsigned int &)
{
    ++g_draws;
    return dsmc_stream_u32(&g_stream);
}

double brng()
{
    ++g_draws;
    return dsmc_stream_uniform(&g_stream);
}
