/* TEST INFRASTRUCTURE — NOT THE PRODUCT.
 *
 * CPU restatement of AreTomo3's reconstruction path (AreTomo/Recon) used as
 * the checker for the CUDA implementation: the FP64 instantiation is the
 * oracle every GPU result is measured against; the FP32 instantiation (same
 * code, float arithmetic, OpenMP over y-slices) is the timed CPU baseline.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg and
 * reference arm load it.
 *
 * Parity pin: the functions below are checked against outputs of the
 * reference's own CUDA Recon (compiled from the reference sources for sm_100a,
 * oracle/ref/) stored as fixtures in tests/golden/.
 *
 * Conventions (all as in the reference):
 *   nx, ny, T   projection width, height, tilt count; frames[T][ny][nx]
 *   Nx = nx & ~1   volume width and the R-weight FFT length
 *   Nz = volZ      volume thickness
 *   output volume: vol[ny][Nz][Nx], frame y = XZ slice with z flipped
 *   (AreTomo/Recon/CDoWbpRecon.cpp:107-123).
 */
#ifndef AT3R_RECON_ORACLE_H
#define AT3R_RECON_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* How a complex-to-real inverse FFT treats imaginary parts in its DC and
 * Nyquist bins (only reachable through the WBP Fourier crop, whose cropped
 * spectrum is not Hermitian).  0: the real part of the Hermitian-extended
 * inverse (imaginary DC/Nyquist parts dropped); 1: the half-length complex
 * "packing" algorithm, in which they leak into even/odd samples. */
void oracle_set_c2r_mode(int mode);
int oracle_get_c2r_mode(void);

/* Per-tilt cos/sin table as the reference builds it (CTomoBase.cpp:56-65). */
void oracle_cos_sin(const float* tilts_deg, int n_tilts, float* cos_sin);

/* WBP of y-slices [y0, y1).  out: [(y1-y0)][Nz][Nx], z flipped. */
int oracle_wbp_f64(const float* frames, int nx, int ny, int n_tilts, const float* tilts_deg,
                   int vol_z, int y0, int y1, double* out, int n_threads);
int oracle_wbp_f32(const float* frames, int nx, int ny, int n_tilts, const float* tilts_deg,
                   int vol_z, int y0, int y1, float* out, int n_threads);

/* SART of y-slices [y0, y1).  relax <= 0 selects the reference's 1/subsets.
 * rfactor (may be NULL): per-iteration sum|raw - fp| and sum|raw| over the
 * valid detector samples of every subset, as 2*iters doubles. */
int oracle_sart_f64(const float* frames, int nx, int ny, int n_tilts, const float* tilts_deg,
                    int vol_z, int start_tilt, int num_tilts, int iters, int subsets, double relax,
                    int y0, int y1, double* out, double* rfactor, int n_threads);
int oracle_sart_f32(const float* frames, int nx, int ny, int n_tilts, const float* tilts_deg,
                    int vol_z, int start_tilt, int num_tilts, int iters, int subsets, double relax,
                    int y0, int y1, float* out, double* rfactor, int n_threads);

/* The random table of SART's empty-voxel fill (MaUtil/GGenRandoms.cu as
 * GFillEmpty2D::SetSize draws it: Nx * Nz entries for the XZ slice in the
 * reference's voxel order, i = Z * Nx + X before the z flip), e.g. the one a
 * device plan drew; used by oracle_sart_* until replaced.  NULL / n <= 0
 * clears it: empty voxels then take the slice mean. */
void oracle_set_fill_table(const int* table, int n);

/* Projection-alignment re-projection of tilt proj_idx
 * (AreTomo/ProjAlign/CCalcReproj.cpp + GReproj.cu): for every row, the tilts
 * of the range CCalcReproj::mFindProjRange picks (skip flags as the caller
 * passes them; NULL = none) are back-projected onto a (2 nx) x vol_z slice
 * and that slice is forward-projected at tilt proj_idx.  out: [ny][nx], -1e30
 * where a ray covers less than 80 % of its length.  range: the tilt indices
 * used, [first, last]. */
int oracle_reproj_range(const float* tilts_deg, const unsigned char* skip, int n_tilts, int proj_idx, int* range);
int oracle_reproj_f32(const float* frames, int nx, int ny, int n_tilts, const float* tilts_deg,
                      const unsigned char* skip, int proj_idx, int vol_z, float* out, int n_threads);

/* Input stage (AreTomo/Correct/CCorrTomoStack.cpp with Fourier cropping;
 * correct = 0: CBinStack::DoFFT).  sizes = {ax, ay, bx, by}: the aligned
 * (CCorrectUtil::CalcAlignedSize) and binned (GFourierResize2D::
 * GetBinnedImgSize) frame sizes. */
int oracle_stack_sizes(int nx, int ny, int correct, float size_axis_deg, float bin, int* sizes);
/* raw [T][ny][nx] -> out [T][by][bx] in FP64 after the FP32 aligned frame
 * (GCorrPatchShift.cu) and the random fill (GFillEmpty2D.cu) driven by
 * `table` (W * ay entries, W = the width the reference's kernels cover; as
 * GGenRandoms draws it).  shifts [T][2], axes_deg [T] (NULL = 0), local
 * [T][5][num_patches] (may be NULL).  aligned (may be NULL): the filled
 * aligned frames [T][ay][ax]. */
int oracle_stack_f64(const float* raw, int nx, int ny, int n_tilts, int correct, const float* shifts,
                     const float* axes_deg, float size_axis_deg, int num_patches, const float* local,
                     int rand_fill, const int* table, float bin, double* out, float* aligned, int n_threads);
/* The fill alone on one frame img[ay][ax] (columns [0, W) covered). */
int oracle_stack_fill_f32(float* img, int W, int ax, int ay, const int* table);
/* Thickness measurement (AreTomo/Recon/CCalcVolThick.cpp): plane standard
 * deviations of FlipVol(true) of vol[ny][vol_z][Nx] (vol_z - 1 values,
 * mMeasureStd), then smoothing and edge detection (mSmooth, mDetectEdges):
 * result = {low edge, high edge, thickness, z offset} in raw pixels. */
int oracle_thickness_profile(const float* vol, int Nx, int ny, int vol_z, float* profile);
int oracle_thickness_edges(const float* profile, int n, float bin, float* smoothed, int* result);

/* Components, for known-answer tests. */
/* complex FFT of length n, interleaved re/im; sign -1 forward, +1 inverse, unnormalised */
int oracle_fft_f64(const double* in, int n, int sign, double* out);
/* the R-weight filter of one row of length N (even): R2C, x H(k), C2R */
int oracle_rweight_row_f64(const double* in, int n, double* out);
/* the filter's transfer function H(k), k in [0, N/2] */
void oracle_rweight_filter_f64(int n, double* h);
/* 2x grid -> 1x Fourier crop: g[2Nz][2Nx] -> f[Nz][Nx] (not flipped) */
int oracle_fourier_crop_f64(const double* g, int nx_vol, int nz_vol, double* f);
/* inverse real FFT of length n from n/2+1 bins under the current c2r mode */
int oracle_c2r_f64(const double* in_cplx, int n, double* out);

#ifdef __cplusplus
}
#endif
#endif
