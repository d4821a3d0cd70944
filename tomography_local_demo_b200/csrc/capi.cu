// Library information entry points of the C ABI.
#include "mr_common.cuh"

namespace mr {
static thread_local cudaError_t g_last_cuda_error = cudaSuccess;
void set_last_cuda_error(cudaError_t e) { g_last_cuda_error = e; }
}  // namespace mr

extern "C" int mr_abi_version(void) { return MR_ABI_VERSION; }

extern "C" const char* mr_last_cuda_error(void) {
    return mr::g_last_cuda_error == cudaSuccess ? "" : cudaGetErrorString(mr::g_last_cuda_error);
}

extern "C" const char* mr_status_string(int status) {
    switch (status) {
        case MR_OK: return "ok";
        case MR_ERR_INVALID: return "invalid argument";
        case MR_ERR_CUDA: return "CUDA runtime or launch error";
        case MR_ERR_UNSUPPORTED: return "unsupported configuration";
        case MR_ERR_TIMEOUT: return "device-side wait timed out";
        case MR_ERR_SCRATCH_LIMIT: return "request exceeds the fixed device scratch of the no-allocation entry point";
        case MR_ERR_CAPTURE:
            return "first no-allocation call on this device came during stream capture; make it before capturing";
        default: return "unknown status";
    }
}

extern "C" int mr_struct_size(int which) {
    switch (which) {
        case 0: return (int)sizeof(mr_ring);
        case 1: return (int)sizeof(mr_view);
        case 2: return (int)sizeof(mr_grid);
        case 3: return (int)sizeof(mr_tile);
        case 4: return (int)sizeof(mr_filter_view);
        default: return -1;
    }
}

static_assert(sizeof(mr_view) == 64, "mr_view layout");
static_assert(sizeof(mr_grid) == 256, "mr_grid layout");
static_assert(sizeof(mr_tile) == 16, "mr_tile layout");
static_assert(sizeof(mr_filter_view) == 32, "mr_filter_view layout");
