/*
 * fmcs_server.h -- a serving loop for multi-column sort / group requests on one
 * GPU (no reference counterpart: the reference runs one query per process).
 *
 * Continuous batching:
 *   - `slots` execution slots, each a host worker thread with its own
 *     context and CUDA stream, so the work of requests admitted together
 *     overlaps on the device;
 *   - a request is admitted when a slot is free and its estimated device
 *     footprint fits in what is left of the HBM budget; otherwise it waits in
 *     arrival order (a request larger than the whole budget is refused at
 *     submission with FMCS_E_OOM);
 *   - when a slot takes a small request (n <= batch_rows_max) it also takes
 *     the queued small requests with the same columns layout and plan, up to
 *     batch_rows_max rows in total, and runs them as ONE fmcs_run_batch launch;
 *   - columns are resident on the device (device pointers); host pointers
 *     work too, at the cost of their copies.
 * Results are identical to running each request alone (fmcs_run_plan).
 */
#ifndef FMCS_SERVER_H
#define FMCS_SERVER_H

#include "fmcs_capi.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    const void *const *cols;      /* ncols column pointers (device or host) */
    const uint32_t *col_bytes;    /* bytes per value of each column */
    const uint32_t *bw;           /* declared bit width of each column */
    uint32_t ncols;
    const uint32_t *split;        /* bank widths; NULL: the cost model picks the plan */
    uint32_t nbanks;
    const uint64_t *cardinality;  /* distinct values per column, for the cost model (NULL: min(2^bw, n)) */
    uint64_t n;
    int hash;                     /* 0: ORDER BY (sort rounds); 1: GROUP BY (hash rounds) */
    uint32_t *order_out;          /* n entries */
    uint32_t *group_out;          /* n entries, or NULL */
} fmcs_request;

typedef struct {
    int status;                   /* FMCS_OK or an error code */
    uint32_t ngroups;
    uint32_t batched_with;        /* requests that shared the launch (1 = alone) */
    double queue_ms;              /* submission -> admission */
    double run_ms;                /* admission -> results complete */
    double total_ms;              /* submission -> results complete */
} fmcs_result;

typedef struct fmcs_server fmcs_server;

FMCS_API int fmcs_server_create(fmcs_server **server, int device, size_t hbm_budget_bytes, uint32_t slots,
                                uint64_t batch_rows_max);
/* Queue a request (the arrays it points to must stay valid until it completes). */
FMCS_API int fmcs_server_submit(fmcs_server *server, const fmcs_request *req, uint64_t *ticket);
/* Wait for a ticket (timeout_s < 0: no limit).  FMCS_E_TIMEOUT if not done in time. */
FMCS_API int fmcs_server_wait(fmcs_server *server, uint64_t ticket, double timeout_s, fmcs_result *result);
/* Device bytes currently admitted against the budget, and requests queued / running. */
FMCS_API int fmcs_server_load(fmcs_server *server, size_t *admitted_bytes, uint32_t *queued, uint32_t *running);
/* Stop after the admitted work, fail what is still queued, free everything. */
FMCS_API void fmcs_server_destroy(fmcs_server *server);

#ifdef __cplusplus
}
#endif

#endif /* FMCS_SERVER_H */
