// Vector math, frames and the PCG32 stream shared by every kernel.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define UPBP_HD __host__ __device__ __forceinline__
#define UPBP_D __device__ __forceinline__

namespace upbp {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.318309886183790671538f;
constexpr float kInfinity = 1e36f;     // the reference's INFTY (shared/shared_defs.h)
constexpr float kEpsRay = 1e-3f;       // kernel/defs.cuh EPS_RAY
constexpr float kEpsCosine = 1e-6f;    // kernel/defs.cuh EPS_COSINE
constexpr float kEpsPhong = 1e-3f;     // kernel/defs.cuh EPS_PHONG
constexpr int kThinWallPriority = -1;
constexpr int kGlobalMediumPriority = -2;

UPBP_HD float3 v3(float a) { return make_float3(a, a, a); }
UPBP_HD float3 v3(float a, float b, float c) { return make_float3(a, b, c); }
UPBP_HD float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
UPBP_HD float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
UPBP_HD float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
UPBP_HD float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
UPBP_HD float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
UPBP_HD float3 operator*(float s, float3 a) { return make_float3(a.x * s, a.y * s, a.z * s); }
UPBP_HD float3 operator/(float3 a, float3 b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
UPBP_HD float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
UPBP_HD float3& operator+=(float3& a, float3 b) { a = a + b; return a; }
UPBP_HD float3& operator*=(float3& a, float3 b) { a = a * b; return a; }
UPBP_HD float3& operator*=(float3& a, float s) { a = a * s; return a; }
UPBP_HD float3& operator/=(float3& a, float s) { a = a / s; return a; }
UPBP_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
UPBP_HD float3 cross(float3 a, float3 b)
{
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
UPBP_HD float length(float3 a) { return sqrtf(dot(a, a)); }
UPBP_HD float3 normalize(float3 a) { return a * (1.f / sqrtf(dot(a, a))); }
UPBP_HD float max_component(float3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
UPBP_HD float component(float3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
UPBP_HD float3 xyz(float4 a) { return make_float3(a.x, a.y, a.z); }

UPBP_HD bool is_black_or_negative(float3 a) { return a.x <= 0.f && a.y <= 0.f && a.z <= 0.f; }
UPBP_HD bool is_positive(float a) { return a > 1e-20f; }
UPBP_HD bool is_positive(float3 a) { return is_positive(a.x) && is_positive(a.y) && is_positive(a.z); }
UPBP_HD float luminance(float3 rgb) { return 0.212671f * rgb.x + 0.715160f * rgb.y + 0.072169f * rgb.z; }

/// Orthonormal frame built from its z axis (same construction rule as the
/// reference's shared/frame.h so stored normals rebuild identical frames).
struct Frame {
    float3 x, y, z;
    UPBP_HD void set_from_z(float3 pz)
    {
        z = normalize(pz);
        float3 tmp_x = (fabsf(z.x) > .99f) ? make_float3(0.f, 1.f, 0.f) : make_float3(1.f, 0.f, 0.f);
        y = normalize(cross(z, tmp_x));
        x = cross(y, z);
    }
    UPBP_HD float3 to_world(float3 a) const { return x * a.x + y * a.y + z * a.z; }
    UPBP_HD float3 to_local(float3 a) const { return make_float3(dot(a, x), dot(a, y), dot(a, z)); }
};

// ----------------------------------------------------------------------------
// PCG32 (XSH-RR 64/32).  One stream per (iteration, subpath, pass):
//   seed = splitmix64(iteration + iteration_offset), stream = subpath*2 + pass.
// Uniform floats are (next >> 8) * 2^-24 in [0, 1).

UPBP_HD uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

struct Rng {
    uint64_t state, inc;
    UPBP_HD uint32_t next()
    {
        uint64_t old = state;
        state = old * 6364136223846793005ull + inc;
        uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = (uint32_t)(old >> 59u);
        return (xs >> rot) | (xs << ((0u - rot) & 31u));
    }
    UPBP_HD void init(uint64_t iteration, uint32_t path, uint32_t pass)
    {
        uint64_t seed = splitmix64(iteration);
        uint64_t stream = ((uint64_t)path << 1) | (uint64_t)(pass & 1u);
        state = 0u;
        inc = (stream << 1u) | 1u;
        next();
        state += seed;
        next();
    }
    UPBP_HD float uniform() { return (float)(next() >> 8) * (1.0f / 16777216.0f); }
};

}  // namespace upbp
