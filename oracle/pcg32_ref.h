/* Oracle restatement of the random stream used by the B200 renderer.
 *
 * PCG32 (O'Neill 2014, "PCG: A Family of Simple Fast Space-Efficient
 * Statistically Good Algorithms for Random Number Generation", the
 * XSH-RR 64/32 member).  One stream per (iteration, subpath, pass):
 *   seed   = splitmix64(iteration + iteration_offset)
 *   stream = subpath index * 2 + pass        (pass 0 = light, 1 = camera)
 * A uniform float is (next() >> 8) * 2^-24, in [0, 1).
 *
 * The reference seeds curand Philox4x32-10 with (iteration, path index,
 * ioff * L) (gpuupbp/kernel/rng.cuh:42-45); the B200 build keeps the
 * per-(iteration, path) seeding but uses PCG32 per pixel as its spec asks, so
 * image parity with an unmodified reference is statistical.  The oracle
 * compiles the reference's device code against this stream instead, which
 * makes per-path results comparable.  Test infrastructure only.
 */
#ifndef UPBP_ORACLE_PCG32_REF_H
#define UPBP_ORACLE_PCG32_REF_H

#include <stdint.h>

typedef struct {
    uint64_t state;
    uint64_t inc;
} upbp_oracle_pcg32;

static inline uint64_t upbp_oracle_splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

static inline uint32_t upbp_oracle_pcg32_next(upbp_oracle_pcg32* r)
{
    uint64_t old = r->state;
    r->state = old * 6364136223846793005ull + r->inc;
    uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((0u - rot) & 31u));
}

static inline void upbp_oracle_pcg32_init(upbp_oracle_pcg32* r, uint64_t iteration, uint32_t path, uint32_t pass)
{
    uint64_t seed = upbp_oracle_splitmix64(iteration);
    uint64_t stream = ((uint64_t)path << 1) | (uint64_t)(pass & 1u);
    r->state = 0u;
    r->inc = (stream << 1u) | 1u;
    upbp_oracle_pcg32_next(r);
    r->state += seed;
    upbp_oracle_pcg32_next(r);
}

static inline float upbp_oracle_pcg32_uniform(upbp_oracle_pcg32* r)
{
    return (float)(upbp_oracle_pcg32_next(r) >> 8) * (1.0f / 16777216.0f);
}

#endif
