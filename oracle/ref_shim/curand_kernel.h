// Host stand-in for the curand Philox state used by the reference's rng.cuh.
// The oracle replaces curand with the PCG32 stream that the B200 renderer uses,
// so the reference's own device code (compiled for the CPU) consumes exactly the
// random numbers the GPU path consumes for the same (iteration, path, pass).
// Stream definition: oracle/pcg32_ref.h.  Test infrastructure only.
#ifndef UPBP_ORACLE_SHIM_CURAND_KERNEL_H
#define UPBP_ORACLE_SHIM_CURAND_KERNEL_H

#include <vector_types.h>
#include "../pcg32_ref.h"

typedef upbp_oracle_pcg32 curandStatePhilox4_32_10_t;

// Which pass the calling thread is running (0 = light, 1 = camera); set by the
// oracle driver before it runs a raygen program.  The reference seeds both
// passes with the same (iteration, path) pair; the B200 renderer separates
// them, and the oracle follows the B200 stream definition.
extern thread_local int g_oracle_rng_pass;
// Light subpaths per iteration, to turn the reference's offset (ioff * L) back
// into an iteration offset.
extern unsigned long long g_oracle_rng_paths_per_iter;

inline void curand_init(unsigned long long seed,
                        unsigned long long subsequence,
                        unsigned long long offset,
                        curandStatePhilox4_32_10_t* state)
{
    unsigned long long ioff = g_oracle_rng_paths_per_iter ? offset / g_oracle_rng_paths_per_iter : 0ull;
    upbp_oracle_pcg32_init(state, seed + ioff, (unsigned int)subsequence, (unsigned int)g_oracle_rng_pass);
}

// curand_uniform returns (0, 1]; the reference maps 1 back to 0.  The PCG32
// value u is in [0, 1), so 0 is reported as 1 and the reference's remap
// recovers u exactly.
inline float curand_uniform(curandStatePhilox4_32_10_t* state)
{
    float u = upbp_oracle_pcg32_uniform(state);
    return u == 0.f ? 1.f : u;
}

inline float4 curand_uniform4(curandStatePhilox4_32_10_t* state)
{
    float4 r;
    r.x = curand_uniform(state);
    r.y = curand_uniform(state);
    r.z = curand_uniform(state);
    r.w = curand_uniform(state);
    return r;
}

#endif
