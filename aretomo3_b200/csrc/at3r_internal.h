// Library-internal entry points shared between the C-ABI sources.
#pragma once
#include "at3r.h"
#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

extern "C" at3r_status plan_create_impl(const at3r_geom* g, cudaStream_t alloc_stream, at3r_plan** out);
// Device bytes the serving loop holds for a request (workspace on one lane,
// FFT tables, the projections resident on the device, two volume slabs);
// *slab_out (may be null) receives the plan's slab.  0 for invalid sizes.
size_t at3r_estimate_resident_bytes(const at3r_geom* g, int* slab_out);
// One slab of a device-resident series proj[T][ny][nx]: rows [y0, y0 + n)
// into vol_rows[n][Nz][Nx] on `st`, without the per-run bookkeeping.
at3r_status at3r_plan_run_slab(at3r_plan* p, const float* proj, int y0, int n, float* vol_rows, cudaStream_t st);
// Sets the calling thread's at3r_last_error() text.
void at3r_set_last_error(const char* msg);
// The library's device memory pool of device `dev` (freed blocks stay cached
// for the next allocation); null if it cannot be created.
cudaMemPool_t at3r_device_pool(int dev);

// Host <-> device staging shared by the host entry points (csrc/at3r.cu).
namespace at3r {
constexpr size_t kStageBytes = (size_t)64 << 20;   // one pinned staging slot
struct Piece {
    char* dst;
    const char* src;
    size_t bytes;
};
// Whether ptr is page-locked host memory (registered or cudaHostAlloc'd).
bool host_pinned(const void* ptr);
// memcpy of every piece, split over up to 8 host threads.
void parallel_copy(const std::vector<Piece>& pieces);
// Pieces of at most kStageBytes each, in order.
std::vector<Piece> split_pieces(const std::vector<Piece>& in);
// Consecutive pieces that continue each other merged into one.
std::vector<Piece> merge_pieces(const std::vector<Piece>& in);
// A pinned staging set of 4 * kStageBytes from the process-wide pool (null if
// it cannot be allocated); return it with stage_release.
char* stage_acquire();
void stage_release(char* set);
}  // namespace at3r
