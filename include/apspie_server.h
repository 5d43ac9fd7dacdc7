/*
 * apspie_server.h -- query server over HBM-resident graphs (continuous batching).
 *
 * No reference counterpart: the reference answers one query per process run
 * (test/bfs/run.sh, test/sssp/run.sh, test/mis/run.sh). The server keeps several graphs on
 * one GPU, admits BFS / SSSP / MIS requests against a device-memory budget and runs them
 * on several execution slots whose launches overlap on the device. BFS requests on a graph
 * join a running batched-BFS launch (the graph's engine) at its next level boundary and
 * complete individually as soon as their own search ends; SSSP requests fold into
 * apspie_sssp_batch or run apspie_sssp each; MIS requests share one apspie_mis. Sources
 * without edges are answered by a small fill kernel. Each answer is written by the same
 * kernels as the plain entry points, so it is identical alone or in a mix.
 */
#ifndef APSPIE_SERVER_H
#define APSPIE_SERVER_H

#include <stdint.h>

#include "apspie.h"
#include "apspie_host.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
    APSPIE_QUERY_BFS = 0,  /* d_out: int32[m] depths (-1 unreached) */
    APSPIE_QUERY_SSSP = 1, /* d_out: int32[m] distances (-1 unreached); graph needs int32 weights */
    APSPIE_QUERY_MIS = 2   /* d_out: uint8[m] membership; source ignored */
};

typedef struct apspie_server apspie_server;

typedef struct apspie_server_stats {
    int64_t submitted;
    int64_t completed;
    int64_t failed;
    int64_t launches;         /* kernel launches (batches) issued */
    int64_t batched_queries;  /* requests served by those launches */
    int64_t max_batch_seen;
    int64_t deferred;         /* admission attempts postponed by the memory budget */
    int64_t peak_bytes;       /* largest device footprint admitted */
    int64_t resident_bytes;   /* graphs + per-slot reserved scratch */
    int64_t joined_running;   /* BFS requests posted into an engine launch already on the GPU */
    int64_t trivial;          /* BFS / SSSP requests whose source has no edges (no traversal) */
    int64_t engine_launches;  /* BFS engine launches (each runs until nothing is in flight or waiting) */
    int64_t engine_levels;    /* BFS levels those launches ran, summed */
} apspie_server_stats;

/* device: GPU ordinal; memory_budget_bytes: device bytes the server may hold (graphs,
 * scratch, batch staging); num_slots: concurrent launches (1..16); max_batch: query slots
 * of a BFS engine and requests per SSSP batch (at most 512). */
apspie_status apspie_server_create(int device, int64_t memory_budget_bytes, int32_t num_slots,
                                   int32_t max_batch, apspie_server **out);
/* Uploads a graph (host CSR; int32 weights enable SSSP). symmetric != 0 marks it
 * undirected. MIS priorities are mt19937(mis_seed) outputs per vertex. Before start only. */
apspie_status apspie_server_add_graph(apspie_server *s, const apspie_host_csr *g, int32_t symmetric,
                                      uint32_t mis_seed, int32_t *graph_id);
/* At most max_fold SSSP requests per launch (before start; default max_batch; 1 = every
 * request runs the single-source kernel). */
apspie_status apspie_server_set_sssp_fold(apspie_server *s, int32_t max_fold);
/* BFS requests run the batched kernel only when at least min_batch of them wait on the
 * same graph (before start; default 6); fewer run apspie_bfs each. */
apspie_status apspie_server_set_bfs_min_batch(apspie_server *s, int32_t min_batch);
/* SSSP requests run apspie_sssp_batch only when at least min_batch of them wait on the
 * same graph (before start); fewer run apspie_sssp each. 0 (default) = by graph size:
 * graphs of at most 2^19 vertices from 4 * sqrt(m / 65536) waiting requests (about where
 * one multi-query launch overtakes as many single-source launches on R-MAT graphs: 4 at
 * scale 16, 8 at scale 18), larger graphs never (a slot's multi-query launch holds only
 * its share of the SMs, while single-source queries spread over all slots). */
apspie_status apspie_server_set_sssp_min_batch(apspie_server *s, int32_t min_batch);
/* on != 0 (default): a slot's persistent grid that has the device to itself takes fewer
 * blocks per SM, so that 4096 registers per SM stay free for small kernels of other
 * streams (the answers for sources without edges, the caller's own kernels); 0: it fills
 * the device. Before start. */
apspie_status apspie_server_set_side_room(apspie_server *s, int32_t on);
/* Reserves the slots' scratch and starts the worker thread. */
apspie_status apspie_server_start(apspie_server *s);
/* Queues a request; the answer is written to d_out (device memory of the server's GPU),
 * which must stay valid until the request completes. Thread-safe. */
apspie_status apspie_server_submit(apspie_server *s, int32_t graph_id, int32_t kind, int32_t source,
                                   void *d_out, uint64_t *ticket);
/* Queues n requests at once (request i: graph_ids[i], kinds[i], sources[i], d_outs[i]; its
 * ticket in tickets[i]), under one lock and with one wake-up of the worker. Every request
 * is checked first: if any is invalid, none is queued and the status is the one
 * apspie_server_submit would return for the first invalid request. Thread-safe. */
apspie_status apspie_server_submit_many(apspie_server *s, int32_t n, const int32_t *graph_ids, const int32_t *kinds,
                                        const int32_t *sources, void *const *d_outs, uint64_t *tickets);
/* Blocks until the request completes (timeout_ms < 0: no limit); returns its status and
 * the latency from submit to completion in *latency_ms. A ticket can be waited once. */
apspie_status apspie_server_wait(apspie_server *s, uint64_t ticket, int32_t timeout_ms,
                                 double *latency_ms);
/* Completed requests in completion order, for callers that keep many in flight: blocks
 * until at least one request not yet waited for has completed (or timeout_ms passes:
 * APSPIE_ERR_TIMEOUT; < 0 waits without limit), then reports up to cap of them
 * (tickets[i], statuses[i], latencies_ms[i]; the last two may be NULL) and *count. A ticket
 * reported here cannot be waited for again. */
apspie_status apspie_server_take_completed(apspie_server *s, int32_t timeout_ms, int32_t cap, uint64_t *tickets,
                                           int32_t *statuses, double *latencies_ms, int32_t *count);
/* Non-blocking completion test. */
apspie_status apspie_server_poll(apspie_server *s, uint64_t ticket, int32_t *done);
apspie_status apspie_server_get_stats(apspie_server *s, apspie_server_stats *out);
/* Drains outstanding requests, stops the worker and frees the server. */
void apspie_server_destroy(apspie_server *s);

#ifdef __cplusplus
}
#endif

#endif /* APSPIE_SERVER_H */
