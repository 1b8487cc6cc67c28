/*
 * visar-b200 served form: a request loop over device-resident images. No
 * counterpart in VISAR (whose calls are synchronous per image).
 *
 * Each request is one device image and a pipeline of 1-16 stages (the
 * visar_stage kinds of visar_batch.h). A scheduler thread admits requests as
 * they arrive while the device pool has room for all of their intermediate
 * results (memory-based admission against pool_bytes), then batches the
 * admitted requests per stage: every scheduling round groups the requests
 * whose next stage is the same and runs each group as one set of persistent
 * tile-queue launches (visar_batch.h's engine), while earlier rounds are
 * still on the GPU. A request's result is the one its pipeline gives through
 * the per-call entry points, whatever it was batched with.
 *
 * Mode VISAR_SERVE_PLAIN runs every request on arrival, stage by stage,
 * through the per-call entry points (no batching): the baseline the batched
 * mode is measured against.
 */
#ifndef VISAR_B200_SERVE_H
#define VISAR_B200_SERVE_H

#include <stddef.h>
#include <stdint.h>

#include "visar_batch.h"

#ifdef __cplusplus
extern "C" {
#endif

enum visar_serve_mode { VISAR_SERVE_BATCHED = 0, VISAR_SERVE_PLAIN = 1 };

typedef struct visar_server_config {
    size_t pool_bytes;   /* device pool for intermediate and final results (0: 64 GiB) */
    int mode;            /* enum visar_serve_mode */
    int max_inflight;    /* scheduling rounds queued on the GPU at once (0: 4; at most 2 while 256 or more requests wait, so that they form larger groups) */
    int streams;         /* streams the stage groups of a round spread over (0: 8) */
} visar_server_config;

typedef struct visar_server visar_server;

typedef struct visar_server_stats {
    uint64_t submitted, completed, released;
    uint64_t rounds;          /* scheduling rounds launched */
    uint64_t launches;        /* persistent launches */
    uint64_t fallback_calls;  /* per-call entry point calls */
    size_t pool_bytes, pool_used, pool_reserved;
    double mean_batch;        /* requests per stage group */
    uint64_t deferred;        /* stage groups put off to a later round for pool or staging memory */
    uint64_t solo;            /* requests run whole through the per-call entry points: new, with no
                                 request sharing their first stage (a round would run them alone) */
    double schedule_s;        /* scheduler thread time spent building and enqueuing rounds, of which: */
    double build_s;           /*   building stage groups (shapes, classes, tables) */
    double upload_s;          /*   staging and enqueuing their descriptor and table copies */
    double launch_s;          /*   enqueuing their launches */
} visar_server_stats;

int visar_server_create(const visar_server_config *cfg, visar_server **out);
/* Queues a request: input is device memory that stays valid and unchanged
   until the request completes; stages are copied. *id identifies it. */
int visar_server_submit(visar_server *s, const visar_image *input, const visar_stage *stages, size_t nstages,
                        uint64_t *id);
/* *done = 1 once the result is ready; out then views it (device memory owned
   by the server until visar_server_release). */
int visar_server_poll(visar_server *s, uint64_t id, int *done, visar_image *out);
int visar_server_wait(visar_server *s, uint64_t id, visar_image *out);
/* Frees a completed request's result. */
int visar_server_release(visar_server *s, uint64_t id);
int visar_server_get_stats(visar_server *s, visar_server_stats *st);
void visar_server_destroy(visar_server *s);

/* Failure handling. When the completion check of a scheduling round returns
   a CUDA error (the context's error is sticky, so the round's results and the
   pool can no longer be trusted), every request that is not yet done
   completes with VISAR_INTERNAL and the CUDA error's name
   (visar_last_error), and every later submission fails the same way; the
   server only has to be destroyed. visar_server_fake_round_error makes the
   next completed round report `cuda_error` (a cudaError_t value) instead of
   what the device said, so callers can test their handling of this path
   without faulting a GPU. */
int visar_server_fake_round_error(visar_server *s, int cuda_error);

/* Load replay: submits n requests at their arrival times (seconds from the
   call, ascending) from a submitting thread, releases each result when it
   completes, and writes each request's latency (ms, submission to completion
   seen by the scheduler) to latency_ms[i]. Returns when all have completed;
   *elapsed_s is the time from the first arrival to the last completion. */
typedef struct visar_trace_request {
    double arrival_s;
    visar_image input;
    const visar_stage *stages;
    size_t nstages;
} visar_trace_request;

int visar_server_run_trace(visar_server *s, const visar_trace_request *reqs, size_t n, double *latency_ms,
                           double *elapsed_s);

#ifdef __cplusplus
}
#endif

#endif /* VISAR_B200_SERVE_H */
