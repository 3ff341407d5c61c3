/*
 * at3r — B200-native tomographic reconstruction (WBP and SART) with the
 * semantics of AreTomo3's AreTomo/Recon, behind a C ABI.
 *
 * Geometry: single-axis parallel beam, tilt axis along y, tilt angles in
 * degrees (alpha offset already folded in, as CAlignParam::GetTilts(false)
 * returns them).  Every y-slice (XZ plane) is reconstructed from row y of
 * every tilt image.
 *
 * Sizes (as in the reference):
 *   nx, ny, n_tilts   projection width, height and count
 *   Nx = nx & ~1      volume width (an odd last column is ignored)
 *   Nz = vol_z        volume thickness
 * Data layouts:
 *   projections, device : float proj[n_tilts][ny][nx]  (x fastest)
 *   projections, host   : n_tilts frame pointers, each float[ny][nx]
 *   volume, device      : float vol[ny][Nz][Nx]  — frame y is the XZ slice at
 *                         y with z flipped, exactly the frames that
 *                         CDoWbpRecon::DoIt / CDoSartRecon::DoIt return
 *   volume, host        : ny frame pointers, each float[Nz][Nx]
 *
 * Errors are returned as status codes; nothing aborts the process.  A plan (or
 * a stack, below) is not safe to run from two host threads at once; distinct
 * plans and stacks are independent (no module-global device state).  `stream`
 * is a cudaStream_t (NULL = the legacy default stream).
 */
#ifndef AT3R_H
#define AT3R_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum at3r_status {
    AT3R_OK = 0,
    AT3R_ERR_INVALID_ARGUMENT = 1,
    AT3R_ERR_CUDA = 2,
    AT3R_ERR_OUT_OF_MEMORY = 3,
    AT3R_ERR_UNSUPPORTED = 4,
    AT3R_ERR_TOO_LARGE = 5,
    AT3R_ERR_NO_DEVICE = 6,
    AT3R_ERR_IO = 7
} at3r_status;

typedef enum at3r_method { AT3R_WBP = 0, AT3R_SART = 1 } at3r_method;

/* Storage type of the staged projections (WBP: the filtered sinogram; SART:
 * the weighted sinogram and the residual).  Accumulation is FP32 always. */
typedef enum at3r_storage { AT3R_STORE_F32 = 0, AT3R_STORE_F16 = 1, AT3R_STORE_BF16 = 2 } at3r_storage;

/* How the final complex-to-real inverse FFT of the WBP Fourier crop treats
 * the imaginary parts of its DC and Nyquist bins (the cropped spectrum is
 * not Hermitian there).  cuFFT, which the reference calls, picks per size:
 * most sizes drop them (HERMITIAN); some (e.g. 1200 x 4096) use a
 * half-length packing algorithm that folds them into even/odd samples
 * (PACKED).  MATCH_CUFFT asks the system cuFFT once per size and process
 * which it does (one tiny C2R on a stream of the library's own, with
 * stream-ordered memory), so the output equals the reference's; when
 * libcufft cannot be loaded, plan creation fails with AT3R_ERR_UNSUPPORTED
 * rather than guess, and the caller may name a convention. */
typedef enum at3r_c2r { AT3R_C2R_MATCH_CUFFT = 0, AT3R_C2R_HERMITIAN = 1, AT3R_C2R_PACKED = 2 } at3r_c2r;

typedef struct at3r_geom {
    int nx, ny, n_tilts;
    const float* tilts_deg;   /* [n_tilts]; copied by at3r_plan_create */
    int vol_z;                /* Nz */
    int method;               /* at3r_method */
    /* SART only (CDoSartRecon::DoIt arguments): subsets partition tilts
     * [start_tilt, start_tilt + num_tilts); the first back-projection uses
     * all n_tilts. */
    int start_tilt, num_tilts;
    int iterations, subsets;
    float relax;              /* <= 0: 1/subsets, the reference's rule */
    int storage;              /* at3r_storage */
    int c2r;                  /* at3r_c2r (WBP only) */
    int slab_slices;          /* y-slices per device batch; 0 = automatic */
    int compute_rfactor;      /* SART: accumulate per-iteration residual sums */
    /* SART: seed of the random table of the empty-voxel fill that ends every
     * reconstruction (CTomoSart::DoIt -> GFillEmpty2D, AreTomo/Recon/
     * CTomoSart.cpp:88, MaUtil/GFillEmpty2D.cu:7-143): a voxel left at the
     * -1e30 "empty" value takes the value of the first non-empty voxel along
     * its chain through the table (entry i drawn from subsequence i of
     * cuRAND's XORWOW, MaUtil/GGenRandoms.cu:7-49), else the slice mean.  The
     * reference seeds it with time(0) when it sets up a series;
     * at3r_geom_init does the same, and a fixed seed makes runs repeatable. */
    unsigned long long fill_seed;
} at3r_geom;

typedef struct at3r_plan at3r_plan;

/* Fills g with the reference's defaults for the method (relax = 1/subsets,
 * FP32 storage, cuFFT-matching C2R, automatic slabs, fill seed = time(0)). */
void at3r_geom_init(at3r_geom* g, int method);

/* Validates g, uploads the geometry table and allocates the device workspace
 * on the current device. */
at3r_status at3r_plan_create(const at3r_geom* g, at3r_plan** out);
void at3r_plan_destroy(at3r_plan* plan);

/* Device-resident form: proj and vol are device pointers in the layouts above. */
at3r_status at3r_run_device(at3r_plan* plan, const float* proj, float* vol, void* stream);

/* Host form (the reference's CDoWbpRecon/CDoSartRecon data flow): reads the
 * tilt frames from host memory, writes the volume frames to host memory,
 * overlapping copies with compute; returns after the volume is on the host.
 * Pinned frames are copied directly; pageable ones (plain new[] / malloc, as
 * CTiltSeries allocates them) pass through a pinned staging ring with
 * multi-threaded host copies that overlap the GPU.  destroying a plan waits
 * for the device, as cudaFree does. */
at3r_status at3r_run_host(at3r_plan* plan, const float* const* frames, float* const* vol_frames, void* stream);

/* SART residual sums of the last run: per iteration, sum|raw - fp| and
 * sum|raw| over valid detector samples (FP64).  out holds 2 * iterations. */
at3r_status at3r_get_rfactor(const at3r_plan* plan, double* out, int n);

/* Bytes of device workspace the plan holds. */
size_t at3r_plan_workspace_bytes(const at3r_plan* plan);
/* Per-kernel accounting.  With timing enabled, every kernel launch of a run
 * is bracketed by CUDA events on its stream.  at3r_plan_kernel_stats reports,
 * for kernel kind `kind` of the last run: its name, launches, device
 * milliseconds (0 unless timing was on), algorithmic DRAM bytes (compulsory
 * reads + writes of the data it consumes and produces) and work units
 * (voxel x tilt updates; ray samples for the forward projection).  It
 * returns the number of kinds and waits for the last run's events. */
at3r_status at3r_plan_set_timing(at3r_plan* plan, int enable);
int at3r_plan_kernel_stats(at3r_plan* plan, int kind, const char** name, int64_t* launches, double* ms,
                           double* bytes, double* units);
/* Number of kernel launches issued by the last run. */
int64_t at3r_plan_last_launches(const at3r_plan* plan);
/* Which C2R convention the plan resolved to (AT3R_C2R_HERMITIAN/PACKED). */
int at3r_plan_c2r(const at3r_plan* plan);
/* What the last run met, as bits ORed over its slices (waits for the
 * device): 1 the SART volume held empty (-1e30) voxels, so the forward
 * projection tested every sample and the fill ran; 2 the staged projections
 * held values at or below -5e9 (near the -1e10 "missing" test), so the
 * back-projection tested every sample; 4 the SART residual did; 8 a fill chain
 * found no non-empty voxel and took the slice mean; 16 a back-projection tile
 * gave up waiting for its bulk-copy staging (the AT3R_BP_BULK_STAGING=1
 * option) and was not written.  -1 on a CUDA error. */
int at3r_plan_flags_seen(const at3r_plan* plan);
/* The SART plan's fill table (see at3r_geom.fill_seed): Nx * Nz entries, entry
 * i = Z * Nx + X for the voxel at (X, Z) of a slice before the z flip, as
 * GGenRandoms draws it; n = the capacity in entries.  For checking only: the
 * reconstruction draws the entries it needs as it goes. */
at3r_status at3r_plan_fill_table(const at3r_plan* plan, int* table, size_t n);

/* SART of a device-resident series without allocating device memory.  No
 * counterpart in the reference: it is for callers that cannot allocate when
 * they reconstruct — an application whose own allocator already reserved the
 * device's memory, or a pipeline with other series in flight that a
 * cudaMalloc/cudaFree (which may synchronise the device) would stall.
 * Arguments as in at3r_geom / CDoSartRecon::DoIt; relax <= 0 selects
 * 1/subsets; FP32 storage; proj and vol are device pointers in the layouts
 * above.  Scratch is one 16 MiB array in the library's device image on every
 * GPU that loads the library, held until exit; it must hold
 * 2 * n_tilts * (nx & ~1) floats for at least one y-slice (and n_tilts <=
 * 4096), otherwise AT3R_ERR_TOO_LARGE.  Calls share that array and it keeps
 * the last call's contents: calls that overlap on the GPU race, so serialise
 * them.  Every call looks up the array's device address on the current
 * device (cudaGetSymbolAddress); the first call on a device also does a
 * one-time set-up (a kernel attribute); make that first call before any
 * stream capture.  The per-tilt table travels to the array in kernel
 * parameters, so no host buffer has to outlive the call.
 * Enqueues on `stream` and returns without waiting. */
at3r_status at3r_sart_device_noalloc(const float* proj, int nx, int ny, int n_tilts, const float* tilts_deg,
                                     int vol_z, int start_tilt, int num_tilts, int iterations, int subsets,
                                     float relax, float* vol, void* stream);

/* Plans take their device workspace from a memory pool of the library (one
 * per device) that keeps freed blocks for the next plan, so creating and
 * destroying plans per series costs no device mapping.  This returns the
 * pool's free blocks to the device. */
void at3r_release_cached_memory(void);

/* Volume output stage (replaces CTiltSeries::FlipVol after the reconstruction,
 * DataUtil/CTiltSeries.cpp:286-305, called from CAreTomoMain::mFlipVol,
 * AreTomo/CAreTomoMain.cpp:893-903): the volume as XY frames.  Frame fz of
 * the result is row zr of every XZ frame, fz = flip ? Nz-1-zr : zr, where row
 * zr of an XZ frame holds z = Nz-1-zr; so flip = 1 (the reference's
 * -FlipVol 1) gives frames in z order and flip = 0 (-FlipVol 2) in reverse
 * z order.
 *
 * at3r_run_host_xyz: at3r_run_host, with the volume written as those XY
 * frames into one contiguous host buffer vol_xyz[Nz][ny][Nx] (frame fz at
 * vol_xyz + fz*ny*Nx); the transpose runs on the device per slab and each
 * slab goes out as one strided copy.
 * at3r_volume_xyz: the same transpose on device buffers, vol_xzy[ny][Nz][nx]
 * -> vol_xyz[Nz][ny][nx] (nx = the volume width, even). */
at3r_status at3r_run_host_xyz(at3r_plan* plan, const float* const* frames, float* vol_xyz, int flip, void* stream);
at3r_status at3r_volume_xyz(const float* vol_xzy, int nx, int ny, int vol_z, int flip, float* vol_xyz, void* stream);

/* Projection-alignment re-projection (replaces ProjAlign::CCalcReproj::DoIt,
 * AreTomo/ProjAlign/CCalcReproj.cpp:36-58, with GReproj,
 * AreTomo/ProjAlign/GReproj.cu): the image of tilt proj_idx re-projected from
 * the nearby tilts.  The tilts [range[0], range[1]] that
 * CCalcReproj::mFindProjRange picks (within 20.5 degrees, cos stretch <= 1.2,
 * not skipped, at most 10; skip may be NULL) are back-projected, weighted by
 * the cosine of their angle to tilt proj_idx, onto a (2 nx) x vol_z slice per
 * row, and each slice is projected at tilt proj_idx with nearest-neighbour
 * rays; reproj[ny][nx] holds the mean along each ray, -1e30 where a ray
 * covers less than 80 % of its length.  As in the reference, the caller marks
 * proj_idx itself in skip (CProjAlignMain::mCalcReproj).
 * at3r_reproj_device: proj [n_tilts][ny][nx] and reproj on the device.
 * at3r_reproj_host: host frames (only those of the range are copied) and a
 * host reproj; returns when it is written. */
at3r_status at3r_reproj_range(const float* tilts_deg, const unsigned char* skip, int n_tilts, int proj_idx,
                              int* range);
at3r_status at3r_reproj_device(const float* proj, int nx, int ny, int n_tilts, const float* tilts_deg,
                               const unsigned char* skip, int proj_idx, int vol_z, float* reproj, void* stream);
at3r_status at3r_reproj_host(const float* const* frames, int nx, int ny, int n_tilts, const float* tilts_deg,
                             const unsigned char* skip, int proj_idx, int vol_z, float* reproj, void* stream);

/* Slab autotuner: times the reconstruction of the leading rows (at most two
 * full-capacity slabs) with slab sizes from 4 slices up to the plan's
 * workspace capacity (doubling) on proj / vol (device buffers in the layouts
 * above; those rows of vol are overwritten) and keeps the fastest for the
 * plan.  The
 * choice is cached per problem shape, so later plans of the same shape skip
 * the timing.  *chosen (may be NULL) receives the slab. */
at3r_status at3r_plan_autotune(at3r_plan* plan, const float* proj, float* vol, void* stream, int* chosen);
/* Slices per device batch the plan currently uses. */
int at3r_plan_slab(const at3r_plan* plan);

/* Batched form: a fixed set of plans over device-resident series.  When
 * every plan is WBP with one storage type, the batch runs as waves: wave w
 * holds slab w of every series that has one, and each of the five WBP
 * stages (R-weight, 2x-grid back-projection, row FFT, column crop, inverse
 * rows) is one launch over the whole wave whose persistent CTAs pull blocks
 * — (series, slab, tile) — from a counter across the uneven series, running
 * the same block code as the per-series kernels (results bit-identical to
 * at3r_run_device of each plan).  The branch form captures every plan's own
 * launches (plan i on branch i % branches).  The first at3r_batch_run
 * captures the work into one CUDA graph (by default both forms when both are
 * possible, keeping the one that times faster; at3r_batch_set_mode) and every
 * run replays it as a single graph launch on `stream`.  Plans, buffers and their
 * contents' sizes must stay as given; SART plans must not compute the
 * R-factor and no plan may have timing enabled. */
typedef struct at3r_batch at3r_batch;
at3r_status at3r_batch_create(at3r_plan* const* plans, const float* const* proj, float* const* vol, int n,
                              int branches, at3r_batch** out);
/* Which form the first run captures: AUTO captures both when the wave form
 * is possible, times one launch of each on the device and keeps the faster;
 * BRANCHES / WAVES force one (before the first run). */
enum { AT3R_BATCH_AUTO = 0, AT3R_BATCH_BRANCHES = 1, AT3R_BATCH_WAVES = 2 };
at3r_status at3r_batch_set_mode(at3r_batch* batch, int mode);
at3r_status at3r_batch_run(at3r_batch* batch, void* stream);
/* The form the batch runs (AT3R_BATCH_BRANCHES / _WAVES; 0 before the first
 * run) and, when AUTO timed both, their device milliseconds (else 0). */
int at3r_batch_mode(const at3r_batch* batch, float* ms_waves, float* ms_branches);
void at3r_batch_destroy(at3r_batch* batch);

/* Upper estimate of the device bytes that at3r_plan_create plus one
 * at3r_run_host over the plan hold (workspace, FFT tables, the two slab
 * buffers of the host path); no device needed.  0 for invalid sizes. */
size_t at3r_plan_estimate_bytes(const at3r_geom* g);

/* Serving loop (on the current device).  Series are submitted as they are
 * collected and reconstructed concurrently, with continuous batching at
 * y-slab granularity: a request is admitted as soon as the device bytes it
 * holds (its plan's workspace, its projections kept on the device for the
 * whole request, two volume slabs) fit hbm_budget_bytes beside the admitted
 * ones and fewer than max_inflight requests are active — any queued request
 * that fits may start, so a large request does not hold back smaller ones,
 * and one passed over eight times stops further overtaking until it fits.
 * One engine thread keeps two slabs of every active request queued on that
 * request's own stream, so slabs of different requests interleave on the
 * device, and streams each finished slab's volume rows to the host frames.
 * Frames and volume frames are host buffers as for at3r_run_host (pinned
 * memory moves directly; pageable memory through pinned bounce buffers) and
 * must stay valid until at3r_server_wait returns for the request.  Results
 * equal those of a lone at3r_run_host on the same geometry. */
typedef struct at3r_server at3r_server;
typedef struct at3r_server_opts {
    size_t hbm_budget_bytes;   /* 0 = 90% of the device memory free at creation */
    int max_inflight;          /* requests active at once; 0 = 4 */
} at3r_server_opts;
at3r_status at3r_server_create(const at3r_server_opts* opts, at3r_server** out);
at3r_status at3r_server_submit(at3r_server* server, const at3r_geom* g, const float* const* frames,
                               float* const* vol_frames, int64_t* id);
/* Blocks until request `id` is done; its status; latency from submission to
 * the volume in host memory, and the part of it spent queued.  A request is
 * waited for once: its id is released on return, and a second concurrent
 * wait on the same id returns AT3R_ERR_INVALID_ARGUMENT at once. */
at3r_status at3r_server_wait(at3r_server* server, int64_t id, double* latency_s, double* queued_s);
/* Device bytes currently admitted (by estimate). */
size_t at3r_server_in_use_bytes(at3r_server* server);
/* Waits for every submitted request, then releases the workers. */
void at3r_server_destroy(at3r_server* server);

/* ---- Input stage: the aligned, binned tilt series that Recon reads --------
 * at3r_stack replaces AreTomo/Correct/CCorrTomoStack (Set0..Set4, DoIt,
 * GetCorrectedStack; CCorrTomoStack.cpp:66-222) as CAreTomoMain::
 * mSetupTsCorrection (CAreTomoMain.cpp:595-619) and CCalcVolThick::DoIt
 * (CCalcVolThick.cpp:58-75) set it up, with Fourier cropping; with
 * correct = 0 it is CBinStack::DoFFT (CBinStack.cpp:61-106).  Per tilt:
 *   1. the aligned frame: pixel (X, Y) takes the raw pixel nearest to its
 *      centred coordinates rotated by the frame's tilt axis, moved by the
 *      weighted local patch shift and the global shift, or -1e30 outside the
 *      raw frame (GCorrPatchShift.cu:18-104);
 *   2. the random fill of those pixels (MaUtil/GFillEmpty2D.cu, table of
 *      MaUtil/GGenRandoms.cu drawn once per stack from `seed`);
 *   3. Fourier-crop binning: 2-D R2C normalised by 1/(ax ay), crop, 2-D C2R
 *      (CFourierCropImage.cpp:41-61), or a plain copy when the binned size
 *      equals the aligned size (CFourierCropImage::mCopy).
 * Sizes: the aligned frame is ax x ay = nx x ny, or ny x nx when
 * |sin(size_axis_deg)| > 0.707 (CCorrectUtil::CalcAlignedSize); the binned
 * frame is bx x by = (int)(a / bin) rounded down to even per dimension, or
 * the aligned size when bin == 1 (GFourierResize2D::GetBinnedImgSize).
 * When ax is odd the reference's kernels cover ax - 1 columns and leave the
 * last one unwritten; here it is 0.
 * Layouts: raw frames [n_tilts][ny][nx]; binned frames [n_tilts][by][bx]. */
typedef struct at3r_stack_geom {
    int nx, ny, n_tilts;          /* raw frames */
    int correct;                  /* 1: align (+ fill) before binning; 0: bin the frames as given */
    const float* shifts;          /* [n_tilts][2] global shifts in pixels (CAlignParam::GetShift); NULL = 0 */
    const float* tilt_axes_deg;   /* [n_tilts] frame rotation (CAlignParam::GetTiltAxis); NULL = shift only */
    float size_axis_deg;          /* tilt axis the aligned size follows (CCorrTomoStack::Set1 fTiltAxis) */
    int num_patches;              /* local-alignment patches (Set1 iNumPatches); 0 = none */
    const float* local_params;    /* [n_tilts][5][num_patches]: centre x, centre y, shift x, shift y, good
                                     (CLocalAlignParam::GetParam) */
    int rand_fill;                /* fill empty pixels; CCorrTomoStack forces it with Fourier cropping */
    unsigned long long seed;      /* seed of the fill's random table (the reference seeds with time(0)) */
    float bin;                    /* Fourier-crop binning >= 1 (Set2 fOutBin, CBinStack::DoFFT fBin) */
} at3r_stack_geom;
typedef struct at3r_stack at3r_stack;

/* correct = 1, rand_fill = 1, bin = 1, everything else 0 / NULL. */
void at3r_stack_geom_init(at3r_stack_geom* g);
/* Copies the alignment, draws the random table and plans the binning FFTs
 * on the current device.  AT3R_ERR_TOO_LARGE when a frame dimension exceeds
 * what one CTA's shared-memory FFT holds. */
at3r_status at3r_stack_create(const at3r_stack_geom* g, at3r_stack** out);
void at3r_stack_destroy(at3r_stack* stack);
/* aligned_xy = {ax, ay}, binned_xy = {bx, by} (either may be NULL). */
at3r_status at3r_stack_sizes(const at3r_stack* stack, int* aligned_xy, int* binned_xy);
/* Copies the fill's random table (W * ay entries, W = ax rounded down to
 * even; entry i is the pixel index pixel i's chain starts at) to host
 * memory; n = its capacity in entries.  AT3R_ERR_INVALID_ARGUMENT when the
 * stack has no fill. */
at3r_status at3r_stack_fill_table(const at3r_stack* stack, int* table, size_t n);
/* The C2R convention the binning follows (AT3R_C2R_HERMITIAN / PACKED, as
 * cuFFT treats a 2-D C2R of the binned size; see at3r_c2r). */
int at3r_stack_c2r(const at3r_stack* stack);
/* raw, binned: device buffers in the layouts above. */
at3r_status at3r_stack_run_device(at3r_stack* stack, const float* raw, float* binned, void* stream);
/* frames: n_tilts host frames of nx*ny floats; binned_frames: n_tilts host
 * frames of bx*by floats.  Returns when they are written. */
at3r_status at3r_stack_run_host(at3r_stack* stack, const float* const* frames, float* const* binned_frames,
                                void* stream);

/* ---- Thickness measurement: CCalcVolThick::DoIt (CCalcVolThick.cpp:47-110)
 * The series is aligned and binned by max(20 / pix_size, 20) (at3r_stack with
 * g's shifts and tilt axes, random fill, no local patches), reconstructed by
 * WBP with thickness (int)(bx * 0.8) / 2 * 2, and the standard deviation of a
 * tile of every z plane of the flipped volume (CTiltSeries::FlipVol(true)) is
 * smoothed and searched for the sample's edges (mMeasureStd, mSmooth,
 * mDetectEdges).  tilts_deg: the tilt angles (CAlignParam::GetTilts(false)).
 * profile / profile_smoothed (may be NULL): the vol_z - 1 plane values before
 * and after smoothing, at most profile_cap of them. */
typedef struct at3r_thickness {
    float binning;        /* m_fBinning */
    int binned_xy[2];     /* binned frame size */
    int vol_z;            /* thickness of the low-resolution volume */
    int n_profile;        /* vol_z - 1 */
    int edges[2];         /* sample edges in raw pixels (m_aiSampleEdges); GetLowEdge / GetHighEdge */
    int thickness;        /* edges[1] - edges[0]: CAlignParam::m_iThickness, GetThickness */
    int offset_z;         /* sample centre - volume centre: CAlignParam::m_iOffsetZ */
} at3r_thickness;
at3r_status at3r_thickness_device(const at3r_stack_geom* g, const float* tilts_deg, float pix_size, const float* raw,
                                  float* profile, float* profile_smoothed, int profile_cap, at3r_thickness* result,
                                  void* stream);
at3r_status at3r_thickness_host(const at3r_stack_geom* g, const float* tilts_deg, float pix_size,
                                const float* const* frames, float* profile, float* profile_smoothed,
                                int profile_cap, at3r_thickness* result, void* stream);

/* ---- Volume file: the MRC file CAsyncSaveVol::mSaveVol writes -------------
 * (DataUtil/CAsyncSaveVol.cpp:82-126 through LibSrc/Mrcfile CSaveMrc): the
 * 1024-byte main header — nx, ny, nz, mode 2 (float), sampling equal to the
 * size, cell = size x pix_size, angles 90, axes 1 2 3, min / max / mean 0,
 * and the writer's defaults (extended-header type "AGAR", version 20140,
 * dvid -16224, sub 1, type 5, tilt angles 90, "MAP" and the machine stamp) —
 * with no extended header (CSaveMrc::SetImgSize resets the one asked for
 * before it), then the nz frames of nx x ny floats.  frames: nz host
 * pointers, e.g. the XY frames of at3r_run_host_xyz (nx = Nx, ny = ny, nz =
 * Nz) or the XZ frames of at3r_run_host (nx = Nx, ny = Nz, nz = ny).
 * Frames are written by up to four threads at their offsets.
 * AT3R_ERR_IO when the file cannot be written. */
at3r_status at3r_mrc_write(const char* path, const float* const* frames, int nx, int ny, int nz, float pix_size);

const char* at3r_status_str(at3r_status s);
const char* at3r_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
