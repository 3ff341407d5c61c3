// Library-internal entry points shared between the C-ABI sources.
#pragma once
#include "at3r.h"
#include <cuda_runtime.h>

extern "C" at3r_status plan_create_impl(const at3r_geom* g, cudaStream_t alloc_stream, at3r_plan** out);
// Sets the calling thread's at3r_last_error() text.
void at3r_set_last_error(const char* msg);
// The library's device memory pool of device `dev` (freed blocks stay cached
// for the next allocation); null if it cannot be created.
cudaMemPool_t at3r_device_pool(int dev);
