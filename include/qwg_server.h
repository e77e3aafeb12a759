/* qwg_server.h - continuous-batching DMC job server on one GPU.
 *
 * No counterpart in the reference: QWalk runs one system per process
 * (program_utils/ooqmc.cpp:40-200, one METHOD section after another).  The
 * server runs many independent DMC jobs (QWalk decks) at once on one device,
 * each a qwg context on its own CUDA stream whose blocks are single graph
 * launches (qwg_dmc_block_async), with:
 *   - admission by device-memory footprint (qwg_footprint) against a budget,
 *     first come first served; a job's walkers stay resident on the device
 *     from admission to retirement;
 *   - continuous batching: each progress call collects every finished block,
 *     immediately enqueues that job's next block, retires finished jobs and
 *     admits queued ones into the freed memory;
 *   - per-block latency: host wall time from the block's enqueue to the
 *     progress call that saw its statistics.
 * A job's results do not depend on what else runs: each context has its own
 * walkers, trial energy and counter-based random stream.
 *
 * Threading: one host thread drives a server.  Admission (context creation,
 * VMC equilibration with single-attempt moves, qwg_dmc_init) runs
 * synchronously inside progress.
 */
#ifndef QWG_SERVER_H
#define QWG_SERVER_H

#include "qwg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct qwg_server qwg_server;

typedef struct {
  const char* deck;        /* QWalk input file (SYSTEM / PSEUDO / TRIALFUNC) */
  int precision;           /* QWG_FP64 or QWG_MIXED */
  int nwalkers;
  int nblocks;             /* DMC blocks to run */
  int vmc_blocks;          /* VMC equilibration blocks before DMC (0: none) */
  int vmc_steps;           /* steps per VMC block */
  double vmc_timestep;
  uint64_t vmc_seed;
  const double* R;         /* initial walkers [nwalkers][nelec][3], host; copied by submit */
  qwg_dmc_params dmc;      /* nstep = steps per block */
} qwg_job_desc;

typedef struct {
  int job;                 /* id returned by qwg_server_submit */
  int block;               /* 0-based block index within the job */
  double latency_ms;       /* enqueue -> statistics seen on the host */
  double queue_ms;         /* submit -> admission (block 0 only, else 0) */
  qwg_block_stats stats;   /* block_ms = device time of the block */
} qwg_block_event;

typedef struct {
  int queued, active, finished, failed;
  unsigned long long bytes_in_use, budget_bytes;
  long long blocks_done;
  double walker_steps;     /* walkers x steps of every finished block */
} qwg_server_status;

/* budget_bytes: device memory the jobs may hold together; max_active: jobs
 * resident at once (0: no limit). */
int qwg_server_create(unsigned long long budget_bytes, int max_active, qwg_server** out);
int qwg_server_destroy(qwg_server* s);
/* Queue a job.  Fails (QWG_ERR_INPUT) when the deck does not parse or the
 * job alone exceeds the budget.  *job receives the job id. */
int qwg_server_submit(qwg_server* s, const qwg_job_desc* job, int* job_id);
/* Non-blocking scheduling pass (see above).  Writes up to max_events block
 * events; *n_events receives how many (events beyond max_events are kept for
 * the next call). */
int qwg_server_progress(qwg_server* s, qwg_block_event* events, int max_events, int* n_events);
int qwg_server_get_status(const qwg_server* s, qwg_server_status* st);
/* Last error of the server (or of a job it ran); valid until the next call. */
const char* qwg_server_last_error(const qwg_server* s);

#ifdef __cplusplus
}
#endif

#endif /* QWG_SERVER_H */
