// Host stand-in for <optix_stubs.h>: opaque declarations of the OptiX host
// types named by the reference's optix_helper.hpp, which the predefined-scene
// loader includes for its sphere-bounds helper.  No OptiX host function is
// called by the oracle.  Test infrastructure only.
#ifndef UPBP_ORACLE_SHIM_OPTIX_STUBS_H
#define UPBP_ORACLE_SHIM_OPTIX_STUBS_H

#include "optix.h"
#include <cuda.h>

typedef struct OptixDeviceContext_t* OptixDeviceContext;
typedef struct OptixModule_t* OptixModule;
typedef struct OptixPipeline_t* OptixPipeline;
typedef struct OptixProgramGroup_t* OptixProgramGroup;
struct OptixAccelBuildOptions { unsigned int buildFlags; unsigned int operation; };
struct OptixBuildInput { unsigned int type; };
struct OptixModuleCompileOptions { int unused; };
struct OptixPipelineCompileOptions { int unused; };
struct OptixProgramGroupOptions { int unused; };
struct OptixShaderBindingTable { CUdeviceptr raygenRecord; };

#endif
