/*
 * pkdecon.h -- C ABI of libpkdecon.so, a B200 (sm_100a) implementation of PetaKit5D's
 * Richardson-Lucy deconvolution hot path.
 *
 * Conventions shared by every entry point (they are MATLAB's, so a MEX gateway passes its arrays
 * straight through):
 *   - volumes are column-major [ny nx nz] (y fastest), dims[] = {ny, nx, nz} = size(I) in MATLAB;
 *   - PSFs are float32 column-major with their own dims[];
 *   - bounding boxes are 1-based inclusive [y1 x1 z1 y2 x2 z2] (crop3d_mex.c:54-59 convention);
 *   - every call returns a pk_status; on failure pk_last_error() gives a message (thread-local);
 *   - the caller owns host buffers; the library owns device memory, streams and caches in pk_ctx;
 *   - calls on one pk_ctx are serialised by the library.
 */
#ifndef PKDECON_H
#define PKDECON_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PK_API __attribute__((visibility("default")))
#else
#define PK_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PK_OK = 0,
    PK_ERR_INVALID = 1,      /* bad argument (MATLAB error(...) in the reference) */
    PK_ERR_UNSUPPORTED = 2,  /* size / option this build does not handle */
    PK_ERR_CUDA = 3,         /* CUDA runtime error */
    PK_ERR_NOMEM = 4,        /* device allocation failed or over the memory budget */
    PK_ERR_BUSY = 5,         /* server queue full */
    PK_ERR_TIMEOUT = 6,      /* bounded wait expired */
    PK_ERR_CANCELLED = 7,    /* request cancelled */
    PK_ERR_EMPTY_OTF_MASK = 8, /* omw_backprojector_generation.m:50-52 */
    PK_ERR_INTERNAL = 9       /* an index check of the bounds-checked build (-DPK_CHECK) failed */
} pk_status;

typedef enum { PK_U16 = 0, PK_F32 = 1, PK_F64 = 2 } pk_dtype;

typedef struct pk_ctx pk_ctx;

/* Name/value parameters of decon_lucy_function.m:21-36 and decon_lucy_omw_function.m:12-30. */
typedef struct {
    double background;     /* Background ([] -> 0) */
    double damp_factor;    /* dampFactor, default 1 */
    double scale_factor;   /* scaleFactor, default 1 */
    double decon_offset;   /* deconOffset, default 0 */
    int32_t edge_erosion;  /* EdgeErosion, default 0 */
    int32_t save16bit;     /* save16bit, default 1: output uint16, else float32 */
    int32_t has_bbox;      /* bbox given (non-empty) */
    int64_t bbox[6];       /* 1-based inclusive [y1 x1 z1 y2 x2 z2] */
} pk_decon_params;

/* Fill *p with the reference defaults. */
PK_API void pk_params_default(pk_decon_params* p);

/* ---------------------------------------------------------------- context */
/* Replaces the per-function `persistent` OTF caches of decon_lucy_function.m:61-77 and
 * decon_lucy_omw_function.m:53-73 with an explicit context bound to one device. */
PK_API pk_ctx* pk_ctx_create(int device);
PK_API void pk_ctx_destroy(pk_ctx* ctx);
/* Drop cached OTFs and work buffers (the demo's reset(gpuDevice), demo_RL_deconvolution.m:164-167). */
PK_API pk_status pk_ctx_reset(pk_ctx* ctx);
PK_API const char* pk_last_error(void);
PK_API const char* pk_version(void);

/* The context's CUDA stream (a cudaStream_t); host-buffer calls run on it. */
PK_API void* pk_ctx_stream(pk_ctx* ctx);
/* Number of kernels this context has launched so far. */
PK_API int64_t pk_ctx_kernel_launches(pk_ctx* ctx);
/* Per-kernel-kind device timing: while enabled, every pass launch is bracketed by CUDA events on
 * its stream.  pk_ctx_profile_read writes a JSON object {kind: {"launches", "ms", "bytes"}} where
 * "bytes" is the algorithmic HBM traffic of one launch (minimum bytes the pass must move); it
 * synchronises the recorded events and returns the JSON length (truncated to cap-1). */
PK_API pk_status pk_ctx_profile(pk_ctx* ctx, int32_t enable);
PK_API int32_t pk_ctx_profile_read(pk_ctx* ctx, char* buf, int32_t cap);

/* Autotuner record (no counterpart in the reference).  The first time a single-volume x / z pass of
 * a given transform plan and size class (waves of resident CTAs its tiles make) runs on a context,
 * each kernel variant that can run it (the register-IO kernel and the TMA kernels' tile widths /
 * buffer counts) is timed on scratch buffers of that geometry and the fastest is kept for every
 * later pass of that plan and class, batched and served ones included; choices persist in an
 * on-disk cache (PK_TUNE_FILE, else ~/.cache/pkdecon/tune-v4.txt; PK_TUNE=0 disables the timing).
 * This writes the context's decisions as a JSON list and returns its length (truncated to cap-1). */
PK_API int32_t pk_ctx_tune_read(pk_ctx* ctx, char* buf, int32_t cap);

/* Failure-detection self-test (no counterpart in the reference).  Every wait inside the pass
 * kernels is bounded: a wait that runs out records it in the context's device-wait status word
 * and the kernel returns, and the next call on the context (or the synchronous call itself)
 * returns PK_ERR_TIMEOUT.  This call runs one CTA that waits on a barrier nothing completes,
 * bounded by limit_ns (1e3 .. 1e9), and returns what such a call returns (PK_ERR_TIMEOUT); the
 * context stays usable afterwards. */
PK_API pk_status pk_selftest_device_wait(pk_ctx* ctx, int64_t limit_ns);
/* 1 in the bounds-checked build (built with -DPK_CHECK: index checks in the pass kernels that record a
 * failure and skip the access, the call returning PK_ERR_INTERNAL), else 0 (no counterpart in the
 * reference; a substitute for compute-sanitizer runs). */
PK_API int32_t pk_checked_build(void);

/* Output extent for dims/params: the bbox size when has_bbox, else dims. */
PK_API pk_status pk_output_dims(const int64_t dims[3], const pk_decon_params* p, int64_t out_dims[3]);

/* ---------------------------------------------------------------- the drop-in calls (host buffers) */
/* [J_2, ~, k] = decon_lucy_function(I, PSF, NUMIT, ...)  -- decon_lucy_function.m:1-213.
 * in: host volume of type in_type; out: host buffer of pk_output_dims() voxels, uint16 when
 * params->save16bit else float32.  *iters_run (may be NULL) receives k. */
PK_API pk_status pk_decon_lucy(pk_ctx* ctx, const void* in, pk_dtype in_type, const int64_t dims[3],
                        const float* psf, const int64_t psf_dims[3], int32_t numit,
                        const pk_decon_params* params, void* out, int32_t* iters_run);

/* J = decon_lucy_omw_function(I, PSF_f, PSF_b, NUMIT, ...)  -- decon_lucy_omw_function.m:1-177. */
PK_API pk_status pk_decon_lucy_omw(pk_ctx* ctx, const void* in, pk_dtype in_type, const int64_t dims[3],
                            const float* psf_f, const int64_t psf_f_dims[3],
                            const float* psf_b, const int64_t psf_b_dims[3], int32_t numit,
                            const pk_decon_params* params, void* out);

/* debug = true form of the two calls: decon_lucy_omw_function.m:114-144 (method 1) and
 * decon_lucy_function.m:144-175 (method 0).  Besides `out` (as above) it fills err_mat (column-major,
 * *err_rows x 4 doubles, room for numit x 4): [k, mean((J - I).^2), that / its first value, the
 * reference's stopping measure over every save_step-th iteration], trimmed as the reference trims it
 * (OMW: floor(numit / save_step) rows; RL: the last step index, and RL with numit < 3 * save_step is
 * refused as the reference's trim has no step index then).  If `snapshots` is not NULL, every
 * save_step-th iteration's uint16(J) (full [ny nx nz] volume, before post-processing) is written to
 * it, floor(numit / save_step) volumes one after another -- the reference writes these as
 * Iter_%04d.tif; the caller writes the files. */
PK_API pk_status pk_decon_debug(pk_ctx* ctx, int32_t method, const void* in, pk_dtype in_type, const int64_t dims[3],
                                const float* psf_f, const int64_t psf_f_dims[3],
                                const float* psf_b, const int64_t psf_b_dims[3], int32_t numit,
                                const pk_decon_params* params, int32_t save_step, void* out, double* err_mat,
                                int32_t* err_rows, uint16_t* snapshots);

/* Asynchronous host-buffer call: uploads `in` on a copy stream, deconvolves (method 0 = Biggs RL,
 * 1 = OMW, parameters as pk_decon_lucy / pk_decon_lucy_omw) and downloads into `out` on a second copy
 * stream, then returns at once with a ticket.  Two staging slots are used in turn, so the upload of
 * the next call and the download of the previous one overlap this call's compute (a stream of volumes
 * runs at the slowest of upload, compute and download).  `in` and `out` must stay valid until
 * pk_decon_wait returns; they must be page-locked (pk_host_alloc, cudaHostAlloc) for the copies to
 * overlap.  No counterpart in the reference (its calls are synchronous). */
PK_API pk_status pk_decon_submit(pk_ctx* ctx, int32_t method, const void* in, pk_dtype in_type, const int64_t dims[3],
                                 const float* psf_f, const int64_t psf_f_dims[3], const float* psf_b,
                                 const int64_t psf_b_dims[3], int32_t numit, const pk_decon_params* params, void* out,
                                 int64_t* ticket);
/* Waits for a submitted call (timeout_ms < 0: no limit; PK_ERR_TIMEOUT leaves the ticket valid). */
PK_API pk_status pk_decon_wait(pk_ctx* ctx, int64_t ticket, int32_t timeout_ms);
/* Orders the context's compute stream after everything queued so far on its copy streams (for
 * device-side timing of submitted calls with events on pk_ctx_stream). */
PK_API pk_status pk_ctx_join(pk_ctx* ctx);

/* Device-pointer forms of the two calls (the gateway's mxGPUArray path): `in`/`out` are device
 * pointers, the work is queued on `stream` (a cudaStream_t, NULL = the context's stream) and the
 * call returns without synchronising. */
PK_API pk_status pk_decon_lucy_device(pk_ctx* ctx, const void* d_in, pk_dtype in_type, const int64_t dims[3],
                               const float* psf, const int64_t psf_dims[3], int32_t numit,
                               const pk_decon_params* params, void* d_out, void* stream);
PK_API pk_status pk_decon_lucy_omw_device(pk_ctx* ctx, const void* d_in, pk_dtype in_type, const int64_t dims[3],
                                   const float* psf_f, const int64_t psf_f_dims[3],
                                   const float* psf_b, const int64_t psf_b_dims[3], int32_t numit,
                                   const pk_decon_params* params, void* d_out, void* stream);

/* OMW deconvolution for callers that cannot allocate GPU memory (no counterpart in the reference).
 * Some callers must not call cudaMalloc -- code running under another runtime's device-memory
 * manager, or an allocation-free section such as an acquisition loop -- so this call allocates no
 * device memory and calls no allocating CUDA or library routine: every work buffer, both OTFs, the
 * twiddle tables and the launch descriptors live in one array compiled into the library (about
 * 32.4 MB, held on each GPU that loads the library until exit).  d_in/d_out are device pointers,
 * the PSFs host arrays; the work is queued on `stream` (a cudaStream_t, NULL = default stream) of
 * the calling thread's current device.  Limit: 1,048,576 voxels per volume (larger ones return
 * PK_ERR_UNSUPPORTED); deconOffset, EdgeErosion and NUMIT = 0 return PK_ERR_UNSUPPORTED.  Every
 * call shares the array and leaves its contents behind, so calls that overlap on the GPU race:
 * issue them one after another on one stream.  The first call on a device looks up the array's
 * address; that address is kept for the process, so do not call this entry point on a device
 * after cudaDeviceReset. */
PK_API pk_status pk_decon_lucy_omw_noalloc(const void* d_in, pk_dtype in_type, const int64_t dims[3],
                                           const float* psf_f, const int64_t psf_f_dims[3],
                                           const float* psf_b, const int64_t psf_b_dims[3], int32_t numit,
                                           const pk_decon_params* params, void* d_out, void* stream);

/* ---------------------------------------------------------------- OTF / FFT building blocks */
/* decon_psf2otf(PSF./sum(PSF), dims) (decon_psf2otf.m:1-46), returned as the half spectrum:
 * complex64 (interleaved re,im), column-major [floor(ny/2)+1, nx, nz]. */
PK_API pk_status pk_psf2otf(pk_ctx* ctx, const float* psf, const int64_t psf_dims[3], const int64_t dims[3],
                     float* otf_half);

/* Forward 3D R2C / inverse unnormalised C2R of device float32 volumes (half-spectrum layout as
 * above).  Used by tests of the transform itself. */
PK_API pk_status pk_fft3_r2c_device(pk_ctx* ctx, const float* d_in, const int64_t dims[3], float* d_spec, void* stream);
PK_API pk_status pk_fft3_c2r_device(pk_ctx* ctx, const float* d_spec, const int64_t dims[3], float* d_out, void* stream);

/* ---------------------------------------------------------------- backprojectors */
/* [b_omw, OTF_bp_omw, abs_OTF_c, OTF_mask] = omw_backprojector_generation(psf, alpha, skewed, ...)
 * (omw_backprojector_generation.m:1-166).  skewed: -1 = [] (auto-detect), 0 = false, 1 = true.
 * b_omw: float32 of psf_dims.  Optional outputs (NULL to skip): otf_bp_omw complex64 interleaved,
 * abs_otf_c float32, otf_mask uint8; all of psf_dims (mask z-extent folded back when skewed). */
PK_API pk_status pk_omw_backprojector(pk_ctx* ctx, const float* psf, const int64_t psf_dims[3], double alpha,
                               int32_t skewed, double otf_cum_thresh, double otf_area_thresh,
                               double hann_lo, double hann_hi, double min_int_thresh,
                               float* b_omw, float* otf_bp_omw, float* abs_otf_c, uint8_t* otf_mask);

/* BackProjector's bp_type (third_parties/WBDeconvolution/BackProjector.m:163-231). */
typedef enum {
    PK_BP_TRADITIONAL = 0,        /* 'traditional': the flipped PSF */
    PK_BP_GAUSSIAN = 1,           /* 'gaussian': a Gaussian of the PSF's FWHMs */
    PK_BP_BUTTERWORTH = 2,        /* 'butterworth': the Butterworth filter alone */
    PK_BP_WIENER = 3,             /* 'wiener': Wiener filter of the flipped OTF */
    PK_BP_WIENER_BUTTERWORTH = 4  /* 'wiener-butterworth' */
} pk_bp_type;

/* [PSF_bp, OTF_bp] = BackProjector(PSF_fp, bp_type, alpha, beta, n, resFlag, iRes)
 * (third_parties/WBDeconvolution/BackProjector.m:67-233; called by decon/RLdecon.m for
 * wiener-butterworth back projection).  psf_bp: float64 of psf_dims; otf_bp (NULL to skip):
 * complex128 interleaved.  A bp_type outside pk_bp_type is PK_ERR_INVALID (the reference's
 * "bp_type does not match any back-projector type"). */
PK_API pk_status pk_backprojector(pk_ctx* ctx, const float* psf, const int64_t psf_dims[3], int32_t bp_type,
                                  double alpha, double beta, int32_t n, int32_t res_flag, const double ires[3],
                                  double* psf_bp, double* otf_bp);

/* pk_backprojector with bp_type PK_BP_WIENER_BUTTERWORTH
 * (third_parties/WBDeconvolution/BackProjector.m:67-233, the 'wiener-butterworth' branch). */
PK_API pk_status pk_wb_backprojector(pk_ctx* ctx, const float* psf, const int64_t psf_dims[3], double alpha,
                              double beta, int32_t n, int32_t res_flag, const double ires[3],
                              double* psf_bp, double* otf_bp);

/* ---------------------------------------------------------------- PSF preparation */
/* psf = psf_gen_new(psf, dz_psf, dz_data, medFactor, PSFGenMethod)  (decon/psf_gen_new.m:1-140;
 * called by RLdecon.m:247, RLdecon_large_in_memory.m:107, RLdecon_large_in_place.m:127 and
 * XR_decon_data_wrapper.m:279 for every measured PSF).  psf: float32 [ny nx nz] column-major
 * (nz == 1: a 2D PSF).  method: 0 = 'masked' (the reference default), 1 = 'median'.
 * The output size depends on the PSF (z padding, axial resampling), so out_dims always receives it;
 * with out == NULL nothing else is written, otherwise out (host, out_capacity floats) receives the
 * PSF in float32.  ny * nx * (2 * nz + 8) floats always suffice (the two z paddings add at most
 * nz + 7 slices), so one call with a buffer of that size is enough.  Errors: PK_ERR_INVALID where MATLAB would raise an indexing error (fewer than 5
 * slices or 10 rows, an all-zero result), PK_ERR_UNSUPPORTED for the 2D 'median' method (its call
 * to the undefined `medfilt`) and for 2D border rows with negative values (complex in MATLAB). */
PK_API pk_status pk_psf_gen(pk_ctx* ctx, const float* psf, const int64_t dims[3], double dz_psf, double dz_data,
                            double med_factor, int32_t method, float* out, int64_t out_capacity,
                            int64_t out_dims[3]);

/* ---------------------------------------------------------------- deskew / rotate */
/* volout = deskewRotateFrame3D(vol, angle, dz, xyPixelSize, 'reverse', reverse, 'bbox', bbox,
 * 'objectiveScan', objective_scan, 'xStepThresh', xstep_thresh, 'save16bit', save16bit)
 * (deskew_rotate/deskewRotateFrame3D.m:1-260 with linear interpolation and no resampling, the path
 * RLdecon.m:487-491 takes after deconvolution; the work of volume_deskew_rotate_warp_mex.cpp and
 * skewed_space_interp_volume_deskew_rotate_warp_mex.cpp).  in: uint16 or float32 [ny nx nz]
 * column-major; out: uint16 when save16bit and the input is uint16, else float32.  bbox: NULL (the
 * whole rotated box) or [y1 x1 z1 y2 x2 z2], 1-based inclusive, y2 <= ny.  out_dims always receives
 * the output size; with out == NULL nothing else is done. */
PK_API pk_status pk_deskew_rotate(pk_ctx* ctx, const void* in, pk_dtype in_type, const int64_t dims[3], double angle,
                                  double dz, double xy_pixel_size, int32_t reverse, int32_t objective_scan,
                                  double xstep_thresh, const int64_t* bbox, int32_t save16bit, void* out,
                                  int64_t out_dims[3]);
/* The same on device buffers (d_out holds out_dims voxels), ordered on `stream` (NULL: the context's);
 * a deconvolved volume from pk_decon_*_device can be deskewed without leaving the GPU. */
PK_API pk_status pk_deskew_rotate_device(pk_ctx* ctx, const void* d_in, pk_dtype in_type, const int64_t dims[3],
                                         double angle, double dz, double xy_pixel_size, int32_t reverse,
                                         int32_t objective_scan, double xstep_thresh, const int64_t* bbox,
                                         int32_t save16bit, void* d_out, int64_t out_dims[3], void* stream);

/* ---------------------------------------------------------------- TIFF volumes (host) */
/* getImageSizeMex(path) (io/cpp-tiff/mexSrc/getimagesizemex.cpp): [ny nx nz] of a TIFF (pages, or
 * images=N of an ImageJ raw stack), bits per sample and whether samples are IEEE floats. */
PK_API pk_status pk_tiff_info(const char* path, int64_t dims[3], int32_t* bits, int32_t* is_float);
/* data = parallelReadTiff(path[, range]) (io/cpp-tiff/src/parallelreadtiff.cpp; io/readtiff.m):
 * pages z_range[0]..z_range[1] (1-based inclusive; NULL = all) into out as a column-major
 * [ny nx nz'] array of the file's sample type (out_bytes must hold it).  Classic TIFF or BigTIFF,
 * strips, uncompressed / LZW / Deflate, horizontal predictor; strips decoded on `threads` host
 * threads (0 = all cores).  Read into a pk_host_alloc buffer, the volume is ready for streamed
 * (pinned) uploads. */
PK_API pk_status pk_tiff_read(const char* path, const int64_t* z_range, void* out, int64_t out_bytes, int32_t threads);
/* parallelWriteTiff(path, data) (io/cpp-tiff/src/parallelwritetiff.cpp; io/writetiff.m): a
 * column-major [ny nx nz] array as BigTIFF, one page per z, 512-row strips, LZW (lzw = 1, the
 * writetiff default) or none; bits 8/16/32/64, is_float for single/double. */
PK_API pk_status pk_tiff_write(const char* path, const void* data, const int64_t dims[3], int32_t bits,
                               int32_t is_float, int32_t lzw, int32_t threads);
/* Zarr v2 volumes (io/readzarr.m, io/writezarr.m over io/cpp-zarr/src/parallelreadzarr.cpp,
 * parallelwritezarr.cpp).  An array of shape [ny nx nz] is the MATLAB array [ny nx nz]; chunks in
 * order "F" or "C", keys "i.j.k" or "i/j/k", compressor none, "zlib", "gzip" or "blosc" (the reference's
 * default; lz4, zlib or zstd inside, byte shuffle or none; blosclz, snappy and bit shuffle give
 * PK_ERR_INVALID on the chunk).  pk_zarr_read: the whole array or
 * bbox [y1 x1 z1 y2 x2 z2] (1-based inclusive; NULL = all) into out (column-major, the array's type);
 * missing chunks read as fill_value.  pk_zarr_write: order "F", separator ".", chunks = min(chunks, dims),
 * compressor 0 = none, 1 = zlib, 2 = gzip (level 1), 3 = blosc lz4, 4 = blosc zstd, 5 = blosc zlib (clevel 5,
 * byte shuffle, as zarr.cpp:17 sets); chunks compressed on `threads` host threads. */
PK_API pk_status pk_zarr_info(const char* path, int64_t dims[3], int64_t chunks[3], int32_t* bits, int32_t* is_float);
PK_API pk_status pk_zarr_read(const char* path, const int64_t* bbox, void* out, int64_t out_bytes, int32_t threads);
PK_API pk_status pk_zarr_write(const char* path, const void* data, const int64_t dims[3], int32_t bits,
                               int32_t is_float, const int64_t chunks[3], int32_t compressor, int32_t threads);
/* Writes a region [y1 x1 z1 y2 x2 z2] (1-based inclusive) of an existing order-F Zarr array from a
 * column-major buffer of the region's size; the region must cover whole chunks (it may end at the
 * array's edge) -- the chunk-aligned batches of the large-file runners. */
PK_API pk_status pk_zarr_write_region(const char* path, const void* data, const int64_t bbox[6], int32_t threads);
/* Page-locked host buffers (cudaHostAlloc) for file reads that feed the GPU. */
PK_API pk_status pk_host_alloc(int64_t bytes, void** ptr);
PK_API pk_status pk_host_free(void* ptr);

/* ---------------------------------------------------------------- large-file edge erosion */
/* The large-file runner's edge erosion (decon/RLdecon_large_in_memory.m:146-168, 267-270):
 * mask = im > 0 with the six faces cleared, mask = bwdist(~mask) > erosion - 1 (Euclidean), then
 * out = out .* mask.  im: host uint16/single [ny nx nz]; out (host, out_type, may be NULL) is
 * multiplied in place; mask (host uint8, may be NULL) receives the mask. */
PK_API pk_status pk_edge_erosion_edt(pk_ctx* ctx, const void* im, pk_dtype im_type, const int64_t dims[3],
                                     int32_t erosion, void* out, pk_dtype out_type, uint8_t* mask);

/* ---------------------------------------------------------------- eroded mask */
/* decon_mask_edge_erosion(im > 0, erosion) (decon/decon_mask_edge_erosion.m:1-30) on its own: the
 * eroded-mask file of XR_RLdeconFrame3D.m:205-231.  im: host uint16/single [ny nx nz]; mask (host
 * uint8, ny*nx*nz) receives 0/1.  A full mask loses `erosion` voxels at each face; otherwise the faces
 * are cleared and the mask eroded by strel('disk', erosion-1) per plane and a (2*erosion-1)-long
 * line in z.  A single plane (nz = 1) takes MATLAB's 2-D steps (no z faces, no z erosion). */
PK_API pk_status pk_mask_edge_erosion(pk_ctx* ctx, const void* im, pk_dtype type, const int64_t dims[3],
                                      int32_t erosion, uint8_t* mask);

/* ---------------------------------------------------------------- edge taper */
/* RLdecon.m:351-357: edgetaper(I(:,:,iz), PSF) for every z slice of a host uint16/single [ny nx nz]
 * volume (MATLAB Image Processing Toolbox edgetaper; the reference passes
 * PSF = fspecial('gaussian', nTapering + 30, nTapering)).  psf: host float64, column-major
 * [psf_dims[0] psf_dims[1]], each smaller than the image's y/x size.  out (host, same type and size
 * as in; may equal in) receives J = alpha .* I + (1 - alpha) .* circular blur of I by PSF, alpha from
 * the PSF's autocorrelation (1 inside, 0 at the borders); uint16 by round-half-away, saturated. */
PK_API pk_status pk_edgetaper(pk_ctx* ctx, const void* in, pk_dtype type, const int64_t dims[3], const double* psf,
                              const int64_t psf_dims[2], void* out);

/* ---------------------------------------------------------------- chunking helpers (host) */
/* findGoodFactorNumber(n, direction, allowOddSeven)  -- utils/findGoodFactorNumber.m:1-26. */
PK_API int64_t pk_find_good_factor_number(int64_t n, int32_t direction, int32_t allow_odd_seven);

/* XR_zarrChunkCoordinatesExtraction(volSize, ...) -- stitch/XR_zarrChunkCoordinatesExtraction.m:1-83.
 * Returns the number of chunks; when the three output arrays are non-NULL they receive n*6 int64
 * (1-based inclusive boxes, chunks in y-fastest order). bbox may be NULL. */
PK_API int64_t pk_chunk_coordinates(const int64_t vol_size[3], const int64_t batch_size[3],
                             const int64_t block_size[3], const int64_t* bbox, int32_t same_batch_size,
                             const int64_t border[3], int64_t* batch_bboxes, int64_t* region_bboxes,
                             int64_t* local_bboxes);

/* ---------------------------------------------------------------- batched chunks */
/* One chunk of a batched call: a column-major uint16/float volume with its own PSF pair (psf_b
 * NULL for traditional RL) and its output crop (deconBbox, RLdecon_for_zarr_block.m:146-158). */
typedef struct {
    const void* in;            /* host or device volume (see pk_batch_decon's `device`) */
    int64_t dims[3];
    int32_t psf_id;            /* index into the psf arrays passed to pk_batch_decon */
    int32_t has_bbox;
    int64_t bbox[6];
    void* out;                 /* output buffer (pk_output_dims voxels) */
} pk_chunk;

/* Deconvolve n chunks with OMW (method 1) or Biggs RL (method 0), numit iterations.
 * psf_f[i]/psf_b[i] with dims psf_dims[i] are the PSF pairs referenced by chunk psf_id.
 * pad_good: 1 = pad each chunk (zeros after background removal, at the high end of each axis) to
 * findGoodFactorNumber sizes so chunks share transform sizes; 0 = exact sizes (reference math).
 * device: 1 when chunk in/out are device pointers. */
PK_API pk_status pk_batch_decon(pk_ctx* ctx, int32_t method, int32_t n, const pk_chunk* chunks, pk_dtype in_type,
                         int32_t npsf, const float* const* psf_f, const float* const* psf_b,
                         const int64_t* psf_dims, int32_t numit, const pk_decon_params* params,
                         int32_t pad_good, int32_t device);

/* ---------------------------------------------------------------- serving */
typedef struct pk_server pk_server;

typedef struct {
    int64_t budget_bytes;      /* HBM admission budget for in-flight work buffers */
    int32_t max_batch;         /* max requests advanced together */
    int32_t queue_capacity;    /* max queued (not yet admitted) requests */
    int32_t borrow_inputs;     /* 0: copy each volume at submit; 1: read the caller's buffer (keep it
                                  valid, ideally pinned, until pk_server_wait returns) */
    int32_t device_loop;       /* 0: a host scheduler thread runs rounds of shared pass launches;
                                  1: device-resident loop: a dispatcher kernel takes each admitted
                                  request's whole pass program (a device-launchable graph) from a ring
                                  in page-locked memory and launches it from the device */
    int32_t heartbeat_ms;      /* device loop: a dispatcher returns when the host's heartbeat has
                                  stalled this long (default 2000; the host restarts it with work) */
    int32_t idle_us;           /* device loop: a dispatcher returns after this long without a new
                                  request (default 2000) */
} pk_server_config;

/* Register a PSF pair (psf_b NULL for RL-only) under psf_id; OTFs are cached per (psf_id, size). */
PK_API pk_server* pk_server_create(pk_ctx* ctx, const pk_server_config* cfg);
PK_API pk_status pk_server_add_psf(pk_server* s, int32_t psf_id, const float* psf_f, const float* psf_b,
                            const int64_t psf_dims[3]);
/* Submit a request: host uint16 volume (copied at submit unless borrow_inputs), method 1 = OMW, 0 = RL.
 * Returns a request id (>= 0) or -pk_status. */
PK_API int64_t pk_server_submit(pk_server* s, const uint16_t* vol, const int64_t dims[3], int32_t psf_id,
                         int32_t method, int32_t numit, const pk_decon_params* params);
/* Wait up to timeout_ms for request id; on PK_OK the result is copied to out (pk_output_dims voxels)
 * and *latency_ms receives submit-to-done time. */
PK_API pk_status pk_server_wait(pk_server* s, int64_t id, void* out, int32_t timeout_ms, double* latency_ms);
PK_API pk_status pk_server_cancel(pk_server* s, int64_t id);
/* stats[0..3] = completed, rejected, peak in-flight bytes, rounds run. */
PK_API pk_status pk_server_stats(pk_server* s, int64_t stats[4]);
PK_API void pk_server_destroy(pk_server* s);
/* Device loop: *running = 1 while a dispatcher instance runs, *exit_code = why the last one returned
 * (0 none yet, 1 stopped, 2 launch budget used up, 3 host heartbeat stalled, 4 idle), *instances = dispatcher
 * instances started.  PK_ERR_UNSUPPORTED for a host-scheduler server. */
PK_API pk_status pk_server_loop_status(pk_server* s, int32_t* running, int32_t* exit_code, int64_t* instances);
/* Test hook of the device loop's bounded wait: pause = 1 stops the scheduler's heartbeat (a running
 * dispatcher returns with exit code 3 within heartbeat_ms), 0 resumes it. */
PK_API pk_status pk_server_pause_heartbeat(pk_server* s, int32_t pause);

#ifdef __cplusplus
}
#endif
#endif /* PKDECON_H */
