// Continuous-batching DMC job server (include/qwg_server.h), built only on
// the engine's C-ABI: every job is one qwg context on its own stream.
#include "../../include/qwg_server.h"

#include <chrono>
#include <deque>
#include <string>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

double ms_since(Clock::time_point t0, Clock::time_point t1) {
  return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

struct Job {
  int id = 0;
  std::string deck;
  qwg_job_desc desc{};
  std::vector<double> R;
  unsigned long long bytes = 0;
  qwg_ctx* ctx = nullptr;
  int blocks_done = 0;
  Clock::time_point submitted, admitted, enqueued;
};

}  // namespace

struct qwg_server {
  unsigned long long budget = 0, in_use = 0;
  int max_active = 0;
  int next_id = 0;
  std::deque<Job> queue;
  std::vector<Job> active;
  std::deque<qwg_block_event> pending_events;
  int finished = 0, failed = 0;
  long long blocks_done = 0;
  double walker_steps = 0;
  std::string err;
};

namespace {

// Create the job's context, equilibrate with VMC, start DMC, enqueue block 0.
int admit(qwg_server* s, Job& j) {
  const qwg_job_desc& d = j.desc;
  int rc = qwg_create(j.deck.c_str(), d.precision, d.nwalkers, nullptr, &j.ctx);
  if (rc != QWG_OK) {
    s->err = "job " + std::to_string(j.id) + ": " + qwg_last_error(nullptr);
    return rc;
  }
  auto bail = [&](int code) {
    s->err = "job " + std::to_string(j.id) + ": " + qwg_last_error(j.ctx);
    qwg_destroy(j.ctx);
    j.ctx = nullptr;
    return code;
  };
  if ((rc = qwg_set_walkers(j.ctx, j.R.data(), d.nwalkers)) != QWG_OK) return bail(rc);
  // admission runs inside progress(): equilibrate with single-attempt moves
  // (the split step kernels), which keeps the other jobs' blocks flowing
  if ((rc = qwg_set_vmc_dynamics(j.ctx, 1, 2.0)) != QWG_OK) return bail(rc);
  for (int b = 0; b < d.vmc_blocks; b++) {
    qwg_block_stats st;
    rc = qwg_vmc_block(j.ctx, d.vmc_steps, d.vmc_timestep, d.vmc_seed + (uint64_t)b, d.dmc.deterministic_pp, &st);
    if (rc != QWG_OK) return bail(rc);
  }
  if ((rc = qwg_dmc_init(j.ctx, &d.dmc)) != QWG_OK) return bail(rc);
  j.R.clear();
  j.R.shrink_to_fit();
  j.admitted = Clock::now();
  j.enqueued = j.admitted;
  if ((rc = qwg_dmc_block_async(j.ctx)) != QWG_OK) return bail(rc);
  return QWG_OK;
}

}  // namespace

extern "C" {

int qwg_server_create(unsigned long long budget_bytes, int max_active, qwg_server** out) {
  if (!out || budget_bytes == 0 || max_active < 0) return QWG_ERR_ARG;
  qwg_server* s = new qwg_server();
  s->budget = budget_bytes;
  s->max_active = max_active;
  *out = s;
  return QWG_OK;
}

int qwg_server_destroy(qwg_server* s) {
  if (!s) return QWG_OK;
  for (Job& j : s->active) {
    if (j.ctx) {
      qwg_block_stats st;
      qwg_dmc_block_wait(j.ctx, &st);  // no block left in flight on a freed context
      qwg_destroy(j.ctx);
    }
  }
  delete s;
  return QWG_OK;
}

int qwg_server_submit(qwg_server* s, const qwg_job_desc* d, int* job_id) {
  if (!s || !d || !d->deck || !d->R || d->nwalkers <= 0 || d->nblocks <= 0 || d->dmc.nstep <= 0)
    return QWG_ERR_ARG;
  Job j;
  unsigned long long bytes = 0;
  if (qwg_footprint(d->deck, d->precision, d->nwalkers, &bytes) != QWG_OK) {
    s->err = std::string("qwg_server_submit: deck does not parse or is beyond this build: ") + d->deck;
    return QWG_ERR_INPUT;
  }
  if (bytes > s->budget) {
    s->err = "qwg_server_submit: job needs " + std::to_string(bytes) + " device bytes, budget is " +
             std::to_string(s->budget);
    return QWG_ERR_INPUT;
  }
  qwg_info info;
  char msg[256];
  if (qwg_inspect_deck(d->deck, &info, msg, sizeof msg) != QWG_OK) {
    s->err = std::string("qwg_server_submit: ") + msg;
    return QWG_ERR_INPUT;
  }
  j.id = s->next_id++;
  j.deck = d->deck;
  j.desc = *d;
  j.desc.deck = nullptr;
  j.desc.R = nullptr;
  j.R.assign(d->R, d->R + (size_t)d->nwalkers * info.nelec * 3);
  j.bytes = bytes;
  j.submitted = Clock::now();
  s->queue.push_back(std::move(j));
  if (job_id) *job_id = s->queue.back().id;
  return QWG_OK;
}

int qwg_server_progress(qwg_server* s, qwg_block_event* events, int max_events, int* n_events) {
  if (!s || (max_events > 0 && !events)) return QWG_ERR_ARG;
  int status = QWG_OK;
  // 1. collect finished blocks; enqueue the next block at once
  for (size_t i = 0; i < s->active.size();) {
    Job& j = s->active[i];
    const int r = qwg_dmc_block_ready(j.ctx);
    if (r == 0) { i++; continue; }
    qwg_block_event ev{};
    ev.job = j.id;
    ev.block = j.blocks_done;
    int rc = r < 0 ? r : qwg_dmc_block_wait(j.ctx, &ev.stats);
    const Clock::time_point now = Clock::now();
    if (rc != QWG_OK) {
      s->err = "job " + std::to_string(j.id) + ": " + qwg_last_error(j.ctx);
      status = rc;
      s->failed++;
      qwg_destroy(j.ctx);
      s->in_use -= j.bytes;
      s->active.erase(s->active.begin() + i);
      continue;
    }
    ev.latency_ms = ms_since(j.enqueued, now);
    ev.queue_ms = j.blocks_done == 0 ? ms_since(j.submitted, j.admitted) : 0.0;
    s->pending_events.push_back(ev);
    s->blocks_done++;
    s->walker_steps += (double)ev.stats.nwalkers * ev.stats.nsteps;
    j.blocks_done++;
    if (j.blocks_done < j.desc.nblocks) {
      j.enqueued = Clock::now();
      rc = qwg_dmc_block_async(j.ctx);
      if (rc != QWG_OK) {
        s->err = "job " + std::to_string(j.id) + ": " + qwg_last_error(j.ctx);
        status = rc;
        s->failed++;
        qwg_destroy(j.ctx);
        s->in_use -= j.bytes;
        s->active.erase(s->active.begin() + i);
        continue;
      }
      i++;
    } else {
      qwg_destroy(j.ctx);
      s->in_use -= j.bytes;
      s->finished++;
      s->active.erase(s->active.begin() + i);
    }
  }
  // 2. admit queued jobs, first come first served, while memory allows
  while (!s->queue.empty()) {
    Job& j = s->queue.front();
    if (s->in_use + j.bytes > s->budget) break;
    if (s->max_active > 0 && (int)s->active.size() >= s->max_active) break;
    const int rc = admit(s, j);
    if (rc != QWG_OK) {
      status = rc;
      s->failed++;
      s->queue.pop_front();
      continue;
    }
    s->in_use += j.bytes;
    s->active.push_back(std::move(j));
    s->queue.pop_front();
  }
  int n = 0;
  while (n < max_events && !s->pending_events.empty()) {
    events[n++] = s->pending_events.front();
    s->pending_events.pop_front();
  }
  if (n_events) *n_events = n;
  return status;
}

int qwg_server_get_status(const qwg_server* s, qwg_server_status* st) {
  if (!s || !st) return QWG_ERR_ARG;
  st->queued = (int)s->queue.size();
  st->active = (int)s->active.size();
  st->finished = s->finished;
  st->failed = s->failed;
  st->bytes_in_use = s->in_use;
  st->budget_bytes = s->budget;
  st->blocks_done = s->blocks_done;
  st->walker_steps = s->walker_steps;
  return QWG_OK;
}

const char* qwg_server_last_error(const qwg_server* s) { return s ? s->err.c_str() : ""; }

}  // extern "C"
