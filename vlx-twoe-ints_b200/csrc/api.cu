// Library-level entry points without a reference counterpart.
#include <cuda_runtime.h>

#include "engine.cuh"
#include "../../include/vlxb.h"

extern "C" {

int vlxb_init(int device)
{
    if (cudaSetDevice(device) != cudaSuccess) return VLXB_ECUDA;
    int rc = vlxb::ensure_pool_configured();
    if (rc) return rc;
    return vlxb::boys_table_device() ? VLXB_OK : VLXB_ECUDA;
}

const char* vlxb_status_string(int status)
{
    switch (status) {
        case VLXB_OK: return "ok";
        case VLXB_EINVAL: return "invalid argument";
        case VLXB_ECUDA: return "CUDA runtime error";
        case VLXB_ENOMEM: return "device memory allocation failed";
        default: return "unknown status";
    }
}

int vlxb_version(void) { return 100; }

}  // extern "C"
