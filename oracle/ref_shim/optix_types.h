// Host stand-in for the OptiX 7 type declarations that the reference's shared
// headers and scene loader name (OptixAabb, OptixInstance, handle type, flag
// enums).  Only the names and field layouts the reference reads are declared;
// there is no OptiX runtime behind them.  Test infrastructure: this file is part
// of the oracle that compiles the reference's device code for the CPU.
#ifndef UPBP_ORACLE_SHIM_OPTIX_TYPES_H
#define UPBP_ORACLE_SHIM_OPTIX_TYPES_H

#include <cstdint>
#include <vector_types.h>

typedef unsigned long long OptixTraversableHandle;

struct OptixAabb {
    float minX, minY, minZ;
    float maxX, maxY, maxZ;
};

struct OptixInstance {
    float transform[12];
    unsigned int instanceId;
    unsigned int sbtOffset;
    unsigned int visibilityMask;
    unsigned int flags;
    OptixTraversableHandle traversableHandle;
    unsigned int pad[2];
};

#define OPTIX_SBT_RECORD_ALIGNMENT 16ull
#define OPTIX_SBT_RECORD_HEADER_SIZE ((size_t)32)

enum OptixRayFlags {
    OPTIX_RAY_FLAG_NONE = 0u,
    OPTIX_RAY_FLAG_DISABLE_ANYHIT = 1u << 0,
    OPTIX_RAY_FLAG_ENFORCE_ANYHIT = 1u << 1,
    OPTIX_RAY_FLAG_TERMINATE_ON_FIRST_HIT = 1u << 2,
    OPTIX_RAY_FLAG_DISABLE_CLOSESTHIT = 1u << 3,
};

enum OptixInstanceFlags {
    OPTIX_INSTANCE_FLAG_NONE = 0u,
    OPTIX_INSTANCE_FLAG_DISABLE_TRIANGLE_FACE_CULLING = 1u << 0,
    OPTIX_INSTANCE_FLAG_FLIP_TRIANGLE_FACING = 1u << 1,
    OPTIX_INSTANCE_FLAG_DISABLE_ANYHIT = 1u << 2,
    OPTIX_INSTANCE_FLAG_ENFORCE_ANYHIT = 1u << 3,
};

#endif
