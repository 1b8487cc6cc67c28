/*
 * visar-b200: the imgproc stencil-and-warp subset of VISAR's stable C ABI,
 * implemented with CUDA kernels for NVIDIA B200 (sm_100a).
 *
 * Drop-in contract. Every function below keeps the name, signature, constant
 * numbering (OpenCV's), status codes and thread-local error reporting of the
 * VISAR entry point cited beside it (paths relative to the VISAR source
 * tree). Results are bit-exact to VISAR's CPU path for integer outputs and
 * follow its float operation order for f32 outputs.
 *
 * Memory. `visar_image.data` may point to host memory (pageable or pinned)
 * or to CUDA device memory of the current device; the library looks at each
 * pointer (cudaPointerGetAttributes). Host images are staged through device
 * buffers; device images are used in place. Every call is synchronous: when
 * it returns, dst holds the result, as in VISAR.
 */
#ifndef VISAR_B200_H
#define VISAR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* include/visar.h:22-30 */
enum visar_status {
    VISAR_OK = 0,
    VISAR_INVALID_ARGUMENT = -1,
    VISAR_SIZE_MISMATCH = -2,
    VISAR_UNSUPPORTED = -3,
    VISAR_OUT_OF_MEMORY = -4,
    VISAR_INVALID_DATA = -5,
    VISAR_INTERNAL = -6,
};

/* include/visar.h:32 (OpenCV CV_8U .. CV_16F numbering) */
enum visar_depth { VISAR_8U = 0, VISAR_8S = 1, VISAR_16U = 2, VISAR_16S = 3, VISAR_32S = 4, VISAR_32F = 5, VISAR_64F = 6, VISAR_16F = 7 };

/* include/visar.h:34-41, src/capi.zig:38-47. stride is in bytes. */
typedef struct visar_image {
    uint32_t width;
    uint32_t height;
    uint32_t channels;
    uint32_t depth;   /* enum visar_depth */
    size_t stride;    /* bytes between row starts */
    void *data;
} visar_image;

/* include/visar.h:43-47, src/capi.zig:97-119 */
const char *visar_version(void);
const char *visar_build_info(void);
const char *visar_last_error(void);
/* Kept for ABI compatibility: the GPU path has no host thread pool; the value is
   stored and reported back (0 = one per CPU). */
void visar_set_num_threads(int n);
int visar_get_num_threads(void);

/* ---------------------------------------------------------------- imgproc */

/* include/visar.h:50, src/capi.zig:163-171. Codes 0-11, 36-41, 54, 55. */
int visar_cvt_color(const visar_image *src, const visar_image *dst, int code);
/* include/visar.h:54, src/capi.zig:184-191. interpolation 0 nearest, 1 linear,
   2 cubic, 3 area (4 lanczos: unsupported, as in VISAR). */
int visar_resize(const visar_image *src, const visar_image *dst, int interpolation);
/* include/visar.h:55, src/capi.zig:197-206 */
int visar_gaussian_blur(const visar_image *src, const visar_image *dst, int kw, int kh, double sigma_x, double sigma_y, int border);
/* include/visar.h:56, src/capi.zig:208-217 */
int visar_box_filter(const visar_image *src, const visar_image *dst, int kw, int kh, int normalize, int border);
/* include/visar.h:57, src/capi.zig:219-232. dst VISAR_16S (from 8U) or VISAR_32F. */
int visar_sobel(const visar_image *src, const visar_image *dst, int dx, int dy, int ksize, double scale, int border);
/* include/visar.h:68, src/capi.zig:310-322. type 0-4, | 8 OTSU or | 16 TRIANGLE;
   *used (may be NULL) receives the threshold applied. */
int visar_threshold(const visar_image *src, const visar_image *dst, double thresh, double maxval, int type, double *used);
/* include/visar.h:72, src/capi.zig:339-350. op 0-6 (erode .. blackhat), shape 0-2
   (rect, cross, ellipse), kw/kh 1-255, iterations >= 0. */
int visar_morphology(const visar_image *src, const visar_image *dst, int op, int shape, int kw, int kh, int iterations);
/* include/visar.h:75, src/capi.zig:372-380. interpolation 0 nearest, else linear. */
int visar_warp_affine(const visar_image *src, const visar_image *dst, const double m[6], int interpolation, int border, double value);

/* include/visar.h:53, src/capi.zig:176-182 -> src/videoio/frame.zig:169-174.
   BT.601 gray of a BGR or BGRA 8U image shrunk by the integer factor k (1-16)
   with box averaging, in one pass; dst is (width / k) x (height / k), 1 channel,
   leftover columns and rows are ignored. k <= 0: InvalidArgument; k > 16 or
   other shapes: SizeMismatch. */
int visar_gray_downsample(const visar_image *src, const visar_image *dst, int k);

/* include/visar.h:58-60, src/capi.zig:234-249 -> src/imgproc/pyramid.zig:73, :408.
   Types 8U, 16U, 16S, 32F, any channel count. pyr_down: dst ((w+1)/2, (h+1)/2),
   border 1-4 (BORDER_CONSTANT: Unsupported); pyr_up: dst (2w, 2h), border must be
   4 (BORDER_REFLECT_101). */
int visar_pyr_down(const visar_image *src, const visar_image *dst, int border);
int visar_pyr_up(const visar_image *src, const visar_image *dst, int border);

/* include/visar.h:333-341, src/capi_calib3d.zig:186-213 -> src/calib3d/undistort.zig.
   dist: nd = 0, 4, 5 or 8 coefficients (k1 k2 p1 p2 [k3 [k4 k5 k6]]); a NULL dist
   is none (InvalidArgument for any other nd).
   undistort: 8U, 1-4 channels, dst the shape of src; new_k may be NULL (= k).
   init_undistort_rectify_map: VISAR_32F one-channel maps of equal shape; r and
   new_k may be NULL (identity / k); a singular new_k * r is InvalidArgument.
   remap: 8U 1-4 channels through VISAR_32F one-channel maps the size of dst,
   INTER_LINEAR, BORDER_CONSTANT with `value` (rounded, clamped to 0-255). */
int visar_undistort(const visar_image *src, const visar_image *dst, const double k[9], const double *dist, size_t nd,
                    const double *new_k);
int visar_init_undistort_rectify_map(const double k[9], const double *dist, size_t nd, const double *r, const double *new_k,
                                     const visar_image *mapx, const visar_image *mapy);
int visar_remap(const visar_image *src, const visar_image *dst, const visar_image *mapx, const visar_image *mapy,
                double value);

/* The tracker's per-frame tail (demos/track_lib.zig:533-553 in VISAR). */
/* include/visar.h:70, src/capi.zig:326-337 -> src/imgproc/threshold.zig:307-360. 8U one channel;
   method 0 MEAN_C, 1 GAUSSIAN_C; type 0 BINARY, 1 BINARY_INV; odd block_size >= 3. */
int visar_adaptive_threshold(const visar_image *src, const visar_image *dst, double maxval, int method, int type,
                             int block_size, double delta);
/* include/visar.h:76, src/capi.zig:382-386 -> src/imgproc/hist.zig:22-45. 8U one channel. */
int visar_equalize_hist(const visar_image *src, const visar_image *dst);
/* include/visar.h:78, src/capi.zig:529-551 -> src/imgproc/components.zig:408. labels: VISAR_32S image
   of src's size; connectivity 4 (else 8); stats (may be NULL): up to max rows of left, top, width,
   height, area; centroids (may be NULL): up to max rows of cx, cy; *count: labels incl. background.
   stats and centroids are host arrays. */
int visar_connected_components(const visar_image *src, const visar_image *labels, int connectivity, int32_t *stats,
                               double *centroids, size_t max, size_t *count);
/* include/visar.h:191-195, src/capi.zig:446-469 -> src/video/track.zig:17-82. Running-average
   background (learning rate 1 / 2^shift, shift 0-15): mask (8U, frame size) is 255 where the gray
   frame differs from the model by more than threshold; the first frame primes the model. The model
   lives on the device current at create. */
typedef struct visar_background visar_background;
int visar_background_create(uint32_t width, uint32_t height, int shift, visar_background **out);
int visar_background_apply(visar_background *b, const visar_image *frame, const visar_image *mask, int threshold);
void visar_background_free(visar_background *b);

/* Additive exports (Zig API only in VISAR, no C entry point there). */
/* src/imgproc/geometry.zig:586-589 warpPerspective(exec, src, dst, [9]f64, WarpInterp, Border, f64) */
int visar_warp_perspective(const visar_image *src, const visar_image *dst, const double m[9], int interpolation, int border, double value);
/* src/imgproc/filter.zig:909-914 sepFilter2D(exec, gpa, src, dst, kx, ky, border); odd kernel lengths. */
int visar_sep_filter_2d(const visar_image *src, const visar_image *dst, const float *kx, int nkx, const float *ky, int nky, int border);

/* ------------------------------------------------------- device execution */
/* No counterpart in VISAR (its calls run on a host thread pool). */

/* Runs subsequent calls of this thread on `stream` (a cudaStream_t, NULL = the
   library's own stream). Calls stay synchronous unless visar_cuda_set_async(1). */
int visar_cuda_set_stream(void *stream);
/* async = 1: calls on device-resident images return after enqueueing their
   kernels on the thread's stream (host images are always synchronous). */
int visar_cuda_set_async(int async);
/* Number of CUDA kernels the library launched since load (all threads). */
uint64_t visar_cuda_launch_count(void);

/* No counterpart in VISAR. visar_resize(src, dst, INTER_LINEAR) for uint8
   images of 1-4 channels that both live in device memory, allocating no device
   memory: the tap tables go to one 512 KiB buffer reserved statically per
   device. Destination width and height are limited to 16384 (InvalidSize
   beyond); host-resident or overlapping images are refused (InvalidArgument).
   The buffer is shared by every call on a device, so two calls in flight at
   once on one device race; issue them on one stream or one at a time. The
   first call on a device resolves the buffer's address and should come before
   any stream capture on that device. Same stream and async rules as the other
   calls. */
int visar_resize_linear_u8_noalloc(const visar_image *src, const visar_image *dst);

#ifdef __cplusplus
}
#endif

#endif /* VISAR_B200_H */
