// Host stand-in for the OptiX device API used by the reference's programs.
// Every intrinsic is implemented in oracle/ref_optix_emu.cpp on top of a scalar
// CPU BVH and per-thread traversal state.  Test infrastructure only.
#ifndef UPBP_ORACLE_SHIM_OPTIX_H
#define UPBP_ORACLE_SHIM_OPTIX_H

#include "optix_types.h"

uint3 optixGetLaunchIndex();
void optixTrace(OptixTraversableHandle handle,
                float3 ray_origin,
                float3 ray_direction,
                float tmin,
                float tmax,
                float ray_time,
                unsigned int visibility_mask,
                unsigned int ray_flags,
                unsigned int sbt_offset,
                unsigned int sbt_stride,
                unsigned int miss_sbt_index,
                unsigned int& p0,
                unsigned int& p1);
unsigned int optixGetPayload_0();
unsigned int optixGetPayload_1();
void optixSetPayload_0(unsigned int v);
void optixSetPayload_1(unsigned int v);
void optixTerminateRay();
void optixIgnoreIntersection();
float3 optixGetWorldRayOrigin();
float3 optixGetWorldRayDirection();
float optixGetRayTmin();
float optixGetRayTmax();
unsigned int optixGetPrimitiveIndex();
unsigned int optixGetInstanceIndex();
bool optixReportIntersection(float hit_t, unsigned int hit_kind, unsigned int a0, unsigned int a1, unsigned int a2);
bool optixIsTriangleHit();
float2 optixGetTriangleBarycentrics();
unsigned int optixGetAttribute_0();
unsigned int optixGetAttribute_1();
unsigned int optixGetAttribute_2();
void* optixGetSbtDataPointer();
void optixThrowException(int code);
int optixGetExceptionCode();

#endif
