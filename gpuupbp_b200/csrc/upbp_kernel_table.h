// The parameter-reading kernels of one compilation of the device code, as
// host launch handles: upbp_capi.cu's own (reading the slot bank indexed by
// the launch's slot) and upbp_slot0.cu's (reading a fixed bank, for slot 0).
#pragma once

#include <cstddef>

#include <cuda_runtime.h>

namespace upbp_kernels {

using SlotKernel = void (*)(int);
using KeyKernel = void (*)(int, unsigned, unsigned*, unsigned*);

constexpr int kModes = 3;  // PB2D, BB1D, BP2D range modes

struct ParamKernels {
    SlotKernel light_pass, camera_pass, nee_connect, bpt_connect, resolve_camera;
    KeyKernel query_keys[2];       // [segment queries?]
    SlotKernel range_search[kModes];
    SlotKernel range_eval[kModes][2];  // [mode][guided]
    SlotKernel point_merge[2][2];      // [medium][guided]
};

// The slot-0 compilation: its kernels, and the uploads of its fixed banks
// (the launch parameters, and the MIS recording bank of the recording build).
const ParamKernels& slot0_kernels();
cudaError_t slot0_upload_params(const void* params, size_t bytes, cudaStream_t st);
cudaError_t slot0_upload_misdbg(const void* bank, size_t bytes, cudaStream_t st);

}  // namespace upbp_kernels
