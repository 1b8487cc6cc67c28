/*
 * visar-b200 batched form: many images of uneven sizes, channel counts and
 * depths through one pipeline of imgproc stages. No counterpart in VISAR,
 * whose calls take one image each; the arithmetic of every stage is the one
 * of the per-call entry point named beside it (include/visar.h), so each
 * output equals what the per-call drop-in gives for that image.
 *
 * Execution. A plan fixes the images and the stages. Each stage runs as one
 * persistent CUDA kernel per shape class (what selects a kernel: depth,
 * channel count, kernel size, resize mode); its CTAs pull tiles from a
 * device-side queue (an atomic counter over the images' tile prefix sums),
 * so large and small images share one launch. Images a persistent kernel
 * does not cover run through the per-call entry point instead (counted in
 * visar_batch_info.fallback_calls). A plan can be replayed as one CUDA graph.
 *
 * Memory. Every stage output lives in one device pool owned by the plan
 * (rows padded to 256 bytes); inputs are the caller's device images, or
 * plan-owned buffers when visar_image.data is NULL at creation.
 */
#ifndef VISAR_B200_BATCH_H
#define VISAR_B200_BATCH_H

#include <stddef.h>
#include <stdint.h>

#include "visar.h"

#ifdef __cplusplus
extern "C" {
#endif

enum visar_stage_kind {
    /* visar_cvt_color BGR2GRAY (3 channels) / BGRA2GRAY (4 channels); one-channel images pass through. */
    VISAR_STAGE_GRAY = 1,
    /* visar_gaussian_blur: i[0] kw, i[1] kh, i[2] border; d[0] sigma_x, d[1] sigma_y. */
    VISAR_STAGE_GAUSSIAN = 2,
    /* visar_morphology: i[0] op, i[1] shape, i[2] kw, i[3] kh, i[4] iterations. */
    VISAR_STAGE_MORPHOLOGY = 3,
    /* visar_resize: i[0] interpolation; d[0] fx, d[1] fy. The destination is
       (max(1, floor(width * fx)), max(1, floor(height * fy))): for fx = fy = 0.5 the
       (w // 2, h // 2) halving of VISAR's differential tests (tests/py/test_core_vs_opencv.py:229). */
    VISAR_STAGE_RESIZE = 4,
    /* visar_threshold: i[0] type; d[0] thresh, d[1] maxval. */
    VISAR_STAGE_THRESHOLD = 5,
    /* visar_warp_affine, same-size output: i[0] interpolation, i[1] border; d[0..5] the matrix, d[6] the border
       value; per_image (optional): one 6-double matrix per image, replacing d[0..5]. */
    VISAR_STAGE_WARP_AFFINE = 6,
    /* visar_warp_perspective, same-size output: i[0] interpolation, i[1] border; d[0..8] the matrix, d[9] the
       border value; per_image (optional): one 9-double matrix per image. */
    VISAR_STAGE_WARP_PERSPECTIVE = 7,
};

typedef struct visar_stage {
    int kind;               /* enum visar_stage_kind */
    int i[5];
    double d[10];
    const double *per_image;
} visar_stage;

typedef struct visar_batch visar_batch;

typedef struct visar_batch_info {
    size_t images;
    size_t stages;
    size_t launches;        /* persistent kernel launches per run */
    size_t fallback_calls;  /* per-image entry point calls per run */
    size_t pool_bytes;      /* device bytes the plan owns */
    size_t bytes_moved;     /* algorithmic bytes per run: every stage reads its input and writes its output once */
    size_t pixels_in;       /* input pixels per run */
} visar_batch_info;

/* Builds a plan over n images (device memory of one device, or data == NULL
   for a plan-owned input) and nstages stages. Stage parameters are checked
   as the per-call entry points check them. */
int visar_batch_create(const visar_image *inputs, size_t n, const visar_stage *stages, size_t nstages,
                       visar_batch **out);
/* Device view of image i's input (for filling plan-owned inputs). */
int visar_batch_input(const visar_batch *b, size_t i, visar_image *out);
/* Device view of image i after stage `stage` (0-based; the last stage is the result). */
int visar_batch_stage_output(const visar_batch *b, size_t stage, size_t i, visar_image *out);
int visar_batch_output(const visar_batch *b, size_t i, visar_image *out);
/* Runs every stage on the thread's stream (visar_cuda_set_stream, else the
   plan's own stream); synchronous unless visar_cuda_set_async(1). */
int visar_batch_run(visar_batch *b);
/* As visar_batch_run, through a CUDA graph captured on the first call and
   replayed afterwards. Plans with fallback calls run without a graph. */
int visar_batch_run_graph(visar_batch *b);
int visar_batch_get_info(const visar_batch *b, visar_batch_info *info);
void visar_batch_destroy(visar_batch *b);

/* Points input i at another device image of the same width, height,
   channels, depth, row stride and at least the same alignment (e.g. the next
   video frame). As with plan-owned inputs, kernels may read every row of it,
   the last one included, up to its length rounded up to 8 bytes (within the
   stride). Enqueued on the run stream (a one-thread kernel patches the
   device descriptors), so graph replays see it. */
int visar_batch_set_input(visar_batch *b, size_t i, const visar_image *img);
/* Host <-> device copies of all inputs / final outputs, from or to `host[i]`,
   which must match the image's shape; pinned host memory keeps them
   asynchronous. When every host image's rows are contiguous (stride = row
   bytes), each image crosses PCIe as one 1-D copy into (out of) a plan-owned
   device staging buffer and a kernel restrides it into (out of) the pitched
   plan images; 2-D copies of short pitched rows run at about half the link
   rate. The staging buffer and its table are allocated on the first such
   call (and again when the images change). Otherwise one 2-D copy per image.
   Same stream and async rules as visar_batch_run; a plan's uploads (and its
   downloads) share one staging buffer, so they must not overlap on
   different streams. */
int visar_batch_upload(visar_batch *b, const visar_image *host, size_t n);
int visar_batch_download(visar_batch *b, const visar_image *host, size_t n);

/* Per-launch timing: with profiling on, eager runs (visar_batch_run) record
   a CUDA event pair around every persistent launch on the run stream. */
typedef struct visar_batch_launch_stat {
    char name[48];          /* op.depth.channels.kernel (e.g. "gauss.u8.c1.k5") */
    int stage;
    size_t images;
    size_t tiles;
    size_t bytes;           /* algorithmic bytes of the launch */
    int grid;               /* CTAs launched */
    float ms;               /* duration in the last profiled run (0 if none) */
} visar_batch_launch_stat;

int visar_batch_profile(visar_batch *b, int enable);
int visar_batch_launch_stat_get(const visar_batch *b, size_t i, visar_batch_launch_stat *out);

/* Tuning table (written by the autotuner, visar_b200/autotune.py): a flat
   JSON object of "key": integer entries. NULL restores the built-in defaults.
   Plans built afterwards use it. */
int visar_tune_load(const char *json_path);
int visar_tune_set(const char *key, int value);
int visar_tune_get(const char *key, int fallback);

#ifdef __cplusplus
}
#endif

#endif /* VISAR_B200_BATCH_H */
