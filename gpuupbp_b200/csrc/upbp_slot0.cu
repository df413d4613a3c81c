// The hot kernels compiled a second time against a fixed parameter bank, for
// the context on launch-parameter slot 0 (upbp_device.cuh explains why), and
// without analytic spheres (upbp_bvh.cuh): a context launches them when it
// holds slot 0 and its scene has no spheres.
// The preprocessor renames the device code's namespace, so these kernels,
// their constant banks and device variables are symbols of their own.
#include <cuda_runtime.h>

#include <type_traits>

#include "upbp_kernel_table.h"

#define UPBP_SLOT0_BANK 1
#define UPBP_NO_SPHERES 1  // used only for scenes without analytic spheres
#define upbp upbp_slot0
#include "upbp_camera_pass.cuh"
#include "upbp_light_pass.cuh"
#undef upbp

namespace upbp_kernels {

const ParamKernels& slot0_kernels()
{
    using namespace upbp_slot0;
    static const ParamKernels k = {
        light_pass_kernel,
        camera_pass_kernel,
        nee_connect_kernel,
        bpt_connect_kernel,
        k_resolve_camera,
        {k_query_keys<false>, k_query_keys<true>},
        {range_search_kernel<kModePb2d>, range_search_kernel<kModeBb1d>, range_search_kernel<kModeBp2d>},
        {{range_eval_kernel<kModePb2d, false>, range_eval_kernel<kModePb2d, true>},
         {range_eval_kernel<kModeBb1d, false>, range_eval_kernel<kModeBb1d, true>},
         {range_eval_kernel<kModeBp2d, false>, range_eval_kernel<kModeBp2d, true>}},
        {{point_merge_kernel<false, false>, point_merge_kernel<false, true>},
         {point_merge_kernel<true, false>, point_merge_kernel<true, true>}},
    };
    return k;
}

cudaError_t slot0_upload_params(const void* params, size_t bytes, cudaStream_t st)
{
    if (bytes != sizeof(upbp_slot0::DeviceParams)) return cudaErrorInvalidValue;
    return cudaMemcpyToSymbolAsync(upbp_slot0::c_slot0, params, bytes, 0, cudaMemcpyHostToDevice, st);
}

cudaError_t slot0_upload_misdbg(const void* bank, size_t bytes, cudaStream_t st)
{
#ifdef UPBP_MIS_DEBUG
    if (bytes != sizeof(upbp_slot0::MisDebug)) return cudaErrorInvalidValue;
    return cudaMemcpyToSymbolAsync(upbp_slot0::c_misdbg, bank, bytes, 0, cudaMemcpyHostToDevice, st);
#else
    (void)bank;
    (void)bytes;
    (void)st;
    return cudaSuccess;
#endif
}

}  // namespace upbp_kernels
