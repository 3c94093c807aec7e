/*
 * sarbp.h -- C ABI of the B200 (sm_100a) SAR backprojection engine.
 *
 * The engine replaces the reference's GPU focusing call
 *
 *     template <typename T, typename P>
 *     void cuda_focus_SAR_image(const SAR_Aperture<T>&,
 *                               const SAR_ImageFormationParameters<P>&,
 *                               CArray<T>& output_image);
 *
 * (src/gpuBackProjection/cuda_sar_focusing/cuda_sar_focusing.hpp:526-723,
 * declared include/charlotte_sar_api.hpp:256-259, exported as the
 * <float,float> and <double,double> instantiations of
 * libuncc_sar_focusing_gpu.so, src/gpuBackProjection/cuda_sar_focusing/
 * libcuda_sar_focusing.cu:26-32).  That call is one monolithic step: copy
 * the aperture to the GPU, batched inverse FFT (:616-617), 1/N scaling
 * (:618), fftshift (:620), backprojection kernel (:659-670), copy back.
 * Here the same step is split into a reusable plan (device buffers and the
 * FFT plan are created once) and entry points for range compression,
 * backprojection, both together, and the adjoint.  A C++ shim that exports
 * the reference's own template symbols on top of this ABI is built as
 * libsarbp_compat.so.
 *
 * Conventions
 *  - Every entry point returns an int status (SARBP_OK == 0).  Nothing calls
 *    cudaDeviceReset() (the reference does, cuda_sar_focusing.hpp:516).
 *  - Complex data are interleaved (re, im) pairs: complex64 = 2 x float,
 *    complex128 = 2 x double.
 *  - Phase history: complex64 [num_pulses][num_range_samples], frequency
 *    fastest, i.e. SAR_Aperture::sampleData (include/uncc_sar_focusing.hpp:68).
 *  - Images: [nz][nx][ny], x-major inside a z-slice: pixel (ix, iy) at
 *    ix*ny + iy as cpuBackProjection.hpp:87 / cuda_BackProjectionKernels.cuh:
 *    91-92.  complex64 for SARBP_PRECISION_MIXED, complex128 for
 *    SARBP_PRECISION_FP64.
 *  - Pixel ix sits at x0 - wx/2 + ix * wx/(nx-1) (cpuBackProjection.hpp:
 *    55-62); likewise y and z.  nz == 1 is the plane z = z0.
 *  - Stream arguments are cudaStream_t passed as void* (NULL = legacy stream).
 *  - Pointers flagged SARBP_MEMORY_HOST are ordinary host memory; calls that
 *    take or return host memory synchronise the stream before returning.
 *    Calls on device memory are asynchronous; sarbp_plan_check() reads back
 *    kernel-side error flags.
 */
#ifndef SARBP_H
#define SARBP_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SARBP_ABI_VERSION 1

#if defined(__GNUC__)
#define SARBP_API __attribute__((visibility("default")))
#else
#define SARBP_API
#endif

/* Status codes */
enum {
    SARBP_OK = 0,
    SARBP_ERR_INVALID_ARGUMENT = 1, /* a size, flag or grid value is out of range */
    SARBP_ERR_NULL_POINTER = 2,     /* a required pointer is NULL */
    SARBP_ERR_UNSUPPORTED = 3,      /* valid request this library version cannot serve */
    SARBP_ERR_OUT_OF_MEMORY = 4,    /* a device or host allocation failed */
    SARBP_ERR_CUDA = 5,             /* a CUDA runtime call failed */
    SARBP_ERR_CUFFT = 6,            /* a cuFFT call failed */
    SARBP_ERR_NOT_FINITE = 7,       /* non-finite geometry reached a kernel */
    SARBP_ERR_KERNEL_TIMEOUT = 8,   /* a bounded device wait gave up */
    SARBP_ERR_KERNEL_BOUNDS = 9,    /* a checked kernel clamped an index */
    SARBP_ERR_NO_DEVICE = 10        /* no CUDA device available */
};

/* Arithmetic of the backprojection */
enum {
    /* FP64 per-tile geometry and phase reduction, FP32 interpolation,
     * rotation and accumulation; complex64 image. */
    SARBP_PRECISION_MIXED = 0,
    /* everything in FP64 (range compression, geometry, interpolation,
     * rotation, accumulation); complex128 image. */
    SARBP_PRECISION_FP64 = 1
};

/* Range taper applied before zero padding */
enum {
    SARBP_WINDOW_NONE = 0,
    SARBP_WINDOW_HAMMING = 1, /* 0.54 - 0.46 cos(2 pi k / (K-1)) (matlab/formImage3DSAR.m:115-116) */
    SARBP_WINDOW_TAYLOR = 2   /* Taylor window, 5 nearly constant sidelobes at -35 dB: the range
                                 factor of taylorwin(K, 5, -35) in matlab/rangeCompress.m:11 */
};

/* Where a pointer lives */
enum { SARBP_MEMORY_HOST = 0, SARBP_MEMORY_DEVICE = 1 };

/* sarbp_backproject flags */
enum {
    SARBP_ACCUMULATE = 1, /* add into the image instead of overwriting it */
    SARBP_CHECKED = 2     /* bounds-checked kernel variant (tests) */
};

/* Image grid (SAR_ImageFormationParameters N_x_pix, N_y_pix, x0_m, y0_m,
 * Wx_m, Wy_m, include/uncc_sar_focusing.hpp:405-412, plus a z axis). */
typedef struct sarbp_grid {
    int nx, ny, nz;
    double x0, y0, z0;
    double wx, wy, wz;
} sarbp_grid;

typedef struct sarbp_plan_desc {
    int num_range_samples; /* K: frequency samples per pulse */
    int num_pulses;        /* Np: pulses per call (upper bound) */
    int nfft;              /* FFT length >= K (SAR_ImageFormationParameters::N_fft) */
    double max_wr;         /* range-profile extent in metres, c/(2 dF)
                              (SAR_ImageFormationParameters::max_Wy_m, :429) */
    sarbp_grid grid;
    int precision;         /* SARBP_PRECISION_* */
    int window;            /* SARBP_WINDOW_* */
    int device;            /* CUDA ordinal, -1 = current device */
    int reserved[4];       /* zero */
} sarbp_plan_desc;

/* Per-pulse geometry: antenna phase centre (Ant_x/y/z), slant range to the
 * scene centre R0 (slant_range) and start frequency f0 (startF), all double
 * [num_pulses] (SAR_Aperture, include/uncc_sar_focusing.hpp:69-87). */
typedef struct sarbp_geometry {
    const double *ant_x, *ant_y, *ant_z;
    const double *slant_range;
    const double *start_freq;
    int num_pulses;
    int memory; /* SARBP_MEMORY_* for all five arrays */
} sarbp_geometry;

typedef struct sarbp_aperture {
    const void *phase_history; /* complex64 [num_pulses][K] */
    int phase_history_memory;  /* SARBP_MEMORY_* */
    sarbp_geometry geometry;
} sarbp_aperture;

typedef struct sarbp_plan sarbp_plan;

SARBP_API int sarbp_abi_version(void);
SARBP_API const char *sarbp_status_string(int status);

/* Create / destroy a plan.  All device memory and the FFT plan are created
 * here (GPUMemoryManager + cufft_engine, cuda_sar_focusing.hpp:93-348,372-399,
 * done once instead of per call). */
SARBP_API int sarbp_plan_create(const sarbp_plan_desc *desc, sarbp_plan **plan);
SARBP_API int sarbp_plan_destroy(sarbp_plan *plan);
/* Device bytes the plan holds. */
SARBP_API int sarbp_plan_workspace_bytes(const sarbp_plan *plan, size_t *bytes);

/* How the plan runs its forward backprojection: tile (8 tile_mx) x 64 pixels,
 * stage_pulses pulses per shared-memory stage, range-bin window of
 * window_bins entries per (tile, pulse), smem_bytes of dynamic shared memory
 * per CTA, resident_ctas CTAs resident at once on the device, tiles per
 * image, and kernels_per_backproject (2 when a launch's (tile, stage) units
 * are split over the resident CTAs and a fix-up kernel adds the split tiles,
 * else 1).  No counterpart in the reference. */
typedef struct sarbp_plan_info {
    int tile_mx;
    int stage_pulses;
    int window_bins;
    int resident_ctas;
    long long tiles;
    long long smem_bytes;
    int kernels_per_backproject;
    int fused_range_compression; /* 1: one kernel does taper, zero pad, inverse FFT and pair
                                    rows (mixed precision, nfft = R K, K in {256, 512, 1024},
                                    R in {1, 2, 4, 8, 16}); 0: taper kernel, cuFFT, pair-row
                                    kernel */
    int reserved[4];
} sarbp_plan_info;
SARBP_API int sarbp_plan_get_info(const sarbp_plan *plan, sarbp_plan_info *info);

/* Range compression (cuda_sar_focusing.hpp:616-620 plus the zero pad and
 * taper of matlab/bpBasic.m:82, matlab/formImage3DSAR.m:115-116):
 *   rc_p = fftshift(ifft(w .* ph_p, nfft)) for every pulse,
 * kept inside the plan for the next sarbp_backproject. */
SARBP_API int sarbp_range_compress(sarbp_plan *plan, const void *phase_history, int num_pulses, int memory,
                         void *stream);

/* Caller-supplied range weights in place of the plan's taper: complex128
 * [num_range_samples] (interleaved re, im doubles, HOST memory), multiplied
 * into every pulse's samples before the zero pad and inverse FFT -- a
 * taper, a reference function for matched filtering in range, or both
 * (matlab/rangeCompress.m:6-7 takes a caller's taper_window the same way,
 * for the range axis).  NULL restores the plan's desc.window.  The weights
 * fold into the per-sample factor the range-compression kernels already
 * apply (no extra work per sample); sarbp_matched_filter uses them too.
 * Waits for the plan's outstanding submissions; work the caller queued with
 * this plan on its own streams must be complete. */
SARBP_API int sarbp_plan_set_range_weights(sarbp_plan *plan, const double *weights);

/* Copy the plan's range profiles out: complex64 (MIXED) or complex128 (FP64)
 * [num_pulses][nfft]. */
SARBP_API int sarbp_get_range_profiles(sarbp_plan *plan, void *out, int memory, void *stream);

/* Backprojection of the plan's range profiles onto the grid
 * (cuda_BackProjectionKernels.cuh:33-93, cpuBackProjection.hpp:49-93). */
SARBP_API int sarbp_backproject(sarbp_plan *plan, const sarbp_geometry *geometry, void *image, int image_memory,
                      int flags, void *stream);

/* Backprojection of the plan's range profiles for num_hypotheses antenna
 * tracks at once (one launch; SARBP_PRECISION_MIXED plans).  The geometry
 * arrays hold num_hypotheses x num_pulses values, hypothesis-major; images is
 * complex64 [num_hypotheses][nz][nx][ny].  Used for motion-hypothesis batches
 * and search-based autofocus, where the reference evaluates one full image
 * per grid point (src/autofocus/gridSearchErrorFunctions_dft.cuh:258-336). */
SARBP_API int sarbp_backproject_hypotheses(sarbp_plan *plan, const sarbp_geometry *geometry, int num_hypotheses,
                                           void *images, int image_memory, int flags, void *stream);

/* Range compression + backprojection: the reference's cuda_focus_SAR_image. */
SARBP_API int sarbp_focus(sarbp_plan *plan, const sarbp_aperture *aperture, void *image, int image_memory,
                void *stream);

/* Gradient of a real image loss with respect to the per-pulse geometry
 * (the adjoint of the backprojection with respect to antenna position and
 * slant range; no counterpart in the reference, whose autofocus searches a
 * grid instead, src/autofocus/autofocus_gpu.cu:707-1260).  Uses the plan's
 * current range profiles and the same geometry as the forward call.
 * grad_image: dL/dRe(img) + j dL/dIm(img), complex64 on the plan's grid
 * (SARBP_PRECISION_MIXED plans).  Outputs: grad_ant double [3][num_pulses]
 * (rows d/dant_x, d/dant_y, d/dant_z), grad_r0 double [num_pulses] or NULL.
 * flags: SARBP_ACCUMULATE adds into the outputs.  Nothing per pixel-pulse is
 * stored; ranges are recomputed per tile.  The first call allocates the
 * per-tile partial buffer. */
SARBP_API int sarbp_backproject_adjoint(sarbp_plan *plan, const sarbp_geometry *geometry, const void *grad_image,
                                        int grad_memory, double *grad_ant, double *grad_r0, int out_memory,
                                        int flags, void *stream);

/* Pipelined focusing of a stream of apertures held in HOST memory: the
 * reference's cuda_focus_SAR_image (cuda_sar_focusing.hpp:526-723) copies in,
 * computes and copies out one aperture at a time; here submitting aperture
 * t+1 while aperture t computes overlaps t+1's upload and t-1's download with
 * t's kernels (plan-owned streams, two staging slots).
 *
 * sarbp_focus_submit enqueues range compression + backprojection of one
 * aperture whose phase history and geometry are host memory into a host
 * image (complex64 MIXED / complex128 FP64 on the plan's grid) and returns a
 * ticket (1, 2, ...).  Page-locked (pinned) buffers make the copies
 * asynchronous; pageable ones still work, without overlap.  The aperture and
 * image buffers must stay untouched until a wait covering the ticket returns.
 * With two submissions outstanding a third first waits for the oldest.
 * sarbp_focus_wait(plan, ticket) waits for every submission up to ticket
 * (0: all) and returns the first error any of them recorded, once.  The
 * plan's other calls first wait for outstanding submissions (keeping an
 * error they recorded for the next sarbp_focus_wait); work the caller queued
 * on its own streams with device buffers must be complete before a submit. */
SARBP_API int sarbp_focus_submit(sarbp_plan *plan, const sarbp_aperture *aperture, void *image,
                                 unsigned long long *ticket);
SARBP_API int sarbp_focus_wait(sarbp_plan *plan, unsigned long long ticket);

/* Batches of independent scenes of uneven sizes (different K, pulse counts,
 * nfft, grids) focused together: one range-compression launch pair for all
 * scenes (plus one FFT per scene) and ONE backprojection launch whose
 * (tile, pulse-stage) units of all scenes are split evenly over the resident
 * CTAs, captured once as a CUDA graph and replayed per call.  The reference
 * focuses one aperture per call (cuda_sar_focusing.hpp:526-723).
 * descs[i] describes scene i (precision must be SARBP_PRECISION_MIXED; all
 * on descs[0].device).  sarbp_batch_focus takes DEVICE phase histories,
 * geometry and images (complex64 on scene i's grid), num_pulses <= the
 * scene's num_pulses; it is stream-ordered and waits only for the batch's
 * previous call before reusing its scene table.  sarbp_batch_wait waits for
 * the last call, returns kernel-side errors, and (if image_ms is not NULL)
 * stores each image's completion time in ms after the call's start, from the
 * GPU clock.  sarbp_batch_autotune times every instantiated tile shape on
 * the given inputs (each run focuses them), keeps the fastest and returns
 * its time per batch.  Two schedules exist for the backprojection launch:
 * the units of all scenes split evenly over the resident CTAs (every scene
 * completes near the end of the launch), or one CTA per tile in scene order
 * (scenes complete one after another; a tail when few tiles are left).  The
 * default is the split for batches of fewer than four waves of tiles, else
 * one CTA per tile; the autotuner times both with every tile shape. */
typedef struct sarbp_batch sarbp_batch;
typedef struct sarbp_batch_info {
    int num_scenes;
    int tile_mx;
    int stage_pulses;
    int max_window_bins;
    int resident_ctas;
    int graph;              /* 1: calls replay a captured CUDA graph */
    long long tiles;        /* of the last call */
    long long units;        /* (tile, stage) units of the last call */
    long long smem_bytes;
    long long workspace_bytes;
    int per_tile;           /* 1: one CTA per tile in scene order (scenes finish one after
                               another); 0: units split evenly over the resident CTAs */
    int reserved[3];
} sarbp_batch_info;
SARBP_API int sarbp_batch_create(const sarbp_plan_desc *descs, int num_scenes, sarbp_batch **batch);
SARBP_API int sarbp_batch_destroy(sarbp_batch *batch);
SARBP_API int sarbp_batch_focus(sarbp_batch *batch, const sarbp_aperture *apertures, void *const *images,
                                void *stream);
SARBP_API int sarbp_batch_wait(sarbp_batch *batch, double *image_ms);
SARBP_API int sarbp_batch_autotune(sarbp_batch *batch, const sarbp_aperture *apertures, void *const *images,
                                   void *stream, double *best_ms);
SARBP_API int sarbp_batch_get_info(const sarbp_batch *batch, sarbp_batch_info *info);
/* Force a schedule: 1 one CTA per tile, 0 split, -1 automatic (default). */
SARBP_API int sarbp_batch_set_schedule(sarbp_batch *batch, int per_tile);

/* Matched-filter focusing, the reference's other algorithm
 * (cpuBackProjection.hpp:165-228, matlab/mfBasic.m:73-89):
 *     img[q] = sum_p sum_k w_k ph_p[k] exp(+j 4 pi (f0_p + k dF) dR_pq / c)
 * on the plan's grid, with dF = c / (2 max_wr) and the plan's taper w; no
 * 1/nfft scale, so a well-sampled image is nfft times sarbp_focus's (the
 * difference is backprojection's interpolation error).  Every pulse is used,
 * as in MATLAB; the reference's C++ loop skips pulses 0 and 1 (:216-218).
 * K times the work of backprojection: a reference for it on small images.
 * Precision as the plan's (MIXED: FP64 phases, FP32 Horner and sums,
 * complex64 image; FP64: complex128). */
SARBP_API int sarbp_matched_filter(sarbp_plan *plan, const sarbp_aperture *aperture, void *image, int image_memory,
                                   void *stream);

/* The autofocus loss on the device.  Shannon entropy of a complex64 image's
 * normalised intensity, E = -sum p log p with p = |I|^2 / sum |I|^2, the
 * objective the gradient autofocus descends (no counterpart in the
 * reference, whose grid search scores images with a 2-D DFT cost,
 * src/autofocus/gridSearchErrorFunctions_dft.cuh:112-203).  `image` is n
 * complex64 values in device memory; `work` is device memory of
 * sarbp_image_entropy_work_bytes() bytes that keeps the sums for the
 * gradient call; `entropy` (device float, may be NULL) receives E.  Sums in
 * FP64 in a fixed order: repeatable bit for bit.  Asynchronous on `stream`.
 * The gradient call writes grad_image = g * dE/d(Re I) + j g * dE/d(Im I)
 * for the upstream scalar g = *grad_entropy (device float; NULL: 1), from
 * the `work` of the sarbp_image_entropy call on the same image. */
SARBP_API size_t sarbp_image_entropy_work_bytes(void);
SARBP_API int sarbp_image_entropy(const void *image, long long n, void *work, float *entropy, void *stream);
SARBP_API int sarbp_image_entropy_grad(const void *image, long long n, const void *work, const float *grad_entropy,
                                       void *grad_image, void *stream);

/* One call, no plan kept: create, focus, destroy (host or device buffers). */
SARBP_API int sarbp_focus_image(const sarbp_plan_desc *desc, const sarbp_aperture *aperture, void *image,
                      int image_memory);

/* Synchronise the stream, read and clear the plan's device error flags and
 * return the first error they record (SARBP_OK if none). */
SARBP_API int sarbp_plan_check(sarbp_plan *plan, void *stream);

/* Backprojection for callers that cannot allocate device memory when they
 * need an image (a pulse-callback loop that must not stall on cudaMalloc's
 * device-wide synchronisation, an application that owns all GPU memory
 * through its own pool or budget).  No counterpart in the reference.
 * Inputs and output are device memory the caller owns: range profiles
 * complex64 [num_pulses][nfft] (as sarbp_get_range_profiles returns them),
 * geometry (memory must be SARBP_MEMORY_DEVICE), image complex64 on desc's
 * grid.  desc supplies nfft, max_wr, the grid and the device (>= 0: the
 * call runs on that device and restores the caller's current device before
 * returning; -1: the current device); precision must be
 * SARBP_PRECISION_MIXED; flags may be SARBP_ACCUMULATE.  Allocates nothing:
 * its scratch is a fixed 32 MiB file-scope device array per GPU, held until
 * the process exits; requests whose staged rows, num_pulses x (nfft + 2 x
 * (range-window + 2)) 16-byte entries, exceed 2^21 - 1 return
 * SARBP_ERR_UNSUPPORTED.  The first call on a device looks up the array's
 * address (make it before any stream capture).  Calls share the array:
 * overlapping calls on the GPU race.  Synchronous: waits for the stream and
 * returns kernel-side errors. */
SARBP_API int sarbp_backproject_noalloc(const sarbp_plan_desc *desc, const void *range_profiles,
                                        const sarbp_geometry *geometry, void *image, int flags, void *stream);

/* ---- test hooks (failure injection; not for production use) ----------- */

/* The device allocation `after` allocations from now (0: the next one) fails
 * as if the device were out of memory; the hook then disarms itself.
 * after < 0 disarms it.  Counts the allocations of plans and batches in this
 * process (cudaMalloc through the library).  Returns SARBP_OK. */
SARBP_API int sarbp_test_fail_device_alloc(int after);

/* Forward and adjoint kernels of this plan: the producer of pulse `pulse`
 * expects its range-bin window's bytes but issues no copy, so the pulse's
 * stage never completes, the kernels' bounded waits run out (about 2 s) and
 * the call returns SARBP_ERR_KERNEL_TIMEOUT with the device context intact.
 * pulse < 0 turns it off.  Mixed-precision plans only. */
SARBP_API int sarbp_test_drop_window_copy(sarbp_plan *plan, int pulse);

#ifdef __cplusplus
}
#endif

#endif /* SARBP_H */
