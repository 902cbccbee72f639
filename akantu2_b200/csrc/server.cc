// Serving loop: many explicit solves resident on one GPU at once.
//
// A request is a mesh, one material, an initial state and a step count.  It
// waits in a FIFO until the device memory it needs fits in the budget and a
// slot is free.  Requests of at most batch_max_request_elements elements are
// then admitted in batches: a builder thread takes the queue's head and every
// queued request with the same element type, quadrature rule, law and
// precision (up to batch_max_elements elements and batch_max_instances
// requests, within the memory budget) and prepares one batch model for all of
// them (akb_batch_create: one element launch and one node launch per step
// advance every instance, each with its own material, time step and step
// count).  Larger requests, a request with no queued partner of its kind
// (under light load: a model of its own builds and steps faster than a batch
// of one), and every request when batching is off, get a model of their own.
//
// The scheduler thread keeps every running unit (batch or single solve) two
// chunks ahead: a chunk is a solve_step of up to chunk_steps steps (100-step
// graph launches) followed by an event, so the units' kernels overlap on the
// device while the host only polls events.  In a batch, each instance stops
// on the device after its own step count (akb_batch_set_instance_steps);
// right after the chunk in which an instance ends, its displacement (and
// velocity) are copied on the batch's stream into a pinned staging buffer,
// and when that chunk's event has completed the request is handed to a
// builder thread, which copies the result into the caller's buffers and
// reports it, while the rest of the batch goes on.  Chunks end at the next
// instance end rounded up to whole graphs, so a request completes at most 99
// steps of its batch after its own last step.  A batch's model is freed when
// its last request has been reported (stream-ordered frees: no device-wide
// synchronisation).  Each instance of a batch is computed exactly as a
// model of its own would compute it, so a result is the same alone and in
// the mix, bit for bit.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <limits>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "akb_capi.h"
#include "host_common.h"

using namespace akb;

namespace {

enum Phase { QUEUED, BUILDING, STEPPING, FINISHING, DONE };

struct Cohort;

struct Job {
  int64_t id = 0;
  // request (copied at submission)
  int et = 0, rule = 0, precision = 0, dim = 3, law = 0;
  int64_t N = 0, E = 0, steps = 0;
  std::vector<double> X, v0, u0;
  std::vector<int32_t> conn;
  std::vector<uint8_t> blocked;
  std::string mat_type, mat_params;
  double dt_factor = 0.8;
  double *u_out = nullptr, *v_out = nullptr;
  int64_t est_bytes = 0;  // this request's own footprint (reported)
  // run state
  Phase phase = QUEUED;
  akb_model *m = nullptr;
  void *stream = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int head = 0, inflight = 0;
  int64_t left = 0;
  double dt = 0.;
  double t_submit = 0., t_admit = 0., t_start = 0., t_end = 0.;
  int status = AKB_OK;
  std::string message;
  // in a batch: the batch, the instance index, the batch step count at which
  // the instance stops
  Cohort *cohort = nullptr;
  int inst = -1;
  int64_t end_step = 0;
  bool solo = false;  // its batch could not be built: admitted alone
};

// requests advanced together by one batch model
struct Cohort {
  std::vector<Job *> jobs;
  int et = 0, rule = 0, precision = 0, dim = 3, law = 0;
  int64_t N = 0, E = 0, est_bytes = 0;
  akb_model *m = nullptr;
  void *stream = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int head = 0, inflight = 0;
  int64_t enqueued = 0, max_steps = 0;
  std::vector<Job *> chunk_jobs[2];  // results copied after chunk slot k
  size_t next_end = 0;               // jobs sorted by end step: next to enqueue
  std::vector<Job *> by_end;
  double *stage = nullptr;  // pinned: u then v of every instance
  std::vector<int64_t> node_off;
  int unreported = 0;
  int status = AKB_OK;
  std::string message;
};

int law_of(const std::string &type) {
  if (type == "elastic") return 0;
  if (type == "neohookean") return 1;
  if (type == "plastic_linear_isotropic_hardening") return 2;
  return -1;
}

}  // namespace

struct akb_server {
  akb_server_config cfg{};
  std::chrono::steady_clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv_work;   // builders: queue / finish lists changed
  std::condition_variable cv_sched;  // scheduler: ready lists changed
  std::condition_variable cv_done;   // pollers: completion available
  std::deque<Job *> queue, finish, done;
  std::deque<Cohort *> retire;       // batches whose requests are all reported
  std::vector<Job *> ready;
  std::vector<Cohort *> ready_cohorts;
  int64_t reserved = 0;  // device bytes of admitted solves and batches
  int active = 0;        // admitted requests not yet done
  int64_t next_id = 1;
  int64_t n_building = 0, n_running = 0;
  bool stop = false;
  std::thread sched;
  std::vector<std::thread> builders;

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  bool batchable(const Job *j) const {
    return !cfg.no_batching && !j->solo && j->E <= cfg.batch_max_request_elements;
  }
  void builder_loop();
  void scheduler_loop();
  void build(Job *j);
  void build_cohort(Cohort *c);
  void finish_job(Job *j);
  void retire_cohort(Cohort *c);
  void complete(Job *j);  // caller holds mu
  int64_t cohort_bytes(const Cohort *c) const;
  Cohort *take_cohort();  // caller holds mu; the head is batchable
};

namespace {

std::string err_text() {
  const char *e = akb_last_error();
  return e ? std::string(e) : std::string();
}

void release_model(Job *j) {
  for (auto &e : j->ev)
    if (e) {
      cudaEventDestroy(e);
      e = nullptr;
    }
  if (j->m) {
    akb_model_destroy(j->m);
    j->m = nullptr;
  }
}

void release_cohort(Cohort *c) {
  for (auto &e : c->ev)
    if (e) {
      cudaEventDestroy(e);
      e = nullptr;
    }
  if (c->m) {
    akb_model_destroy(c->m);
    c->m = nullptr;
  }
  if (c->stage) {
    cudaFreeHost(c->stage);
    c->stage = nullptr;
  }
}

bool all_finite(const double *x, int64_t n) {
  for (int64_t i = 0; i < n; ++i)
    if (!std::isfinite(x[i])) return false;
  return true;
}

}  // namespace

// a finished or failed request: frees its slot (and, for a request with a
// model of its own, its memory reservation)
void akb_server::complete(Job *j) {
  j->phase = DONE;
  j->t_end = now();
  if (!j->cohort) reserved -= j->est_bytes;
  active--;
  done.push_back(j);
  cv_done.notify_all();
  cv_work.notify_all();
}

int64_t akb_server::cohort_bytes(const Cohort *c) const {
  int64_t b = 0;
  if (akb_estimate_batch_device_bytes(c->et, c->rule, c->N, c->E, (int)c->jobs.size(), c->law,
                                      c->precision, &b) != AKB_OK)
    return std::numeric_limits<int64_t>::max() / 4;
  return b;
}

// the queue's head and the queued requests that can share its batch, in
// arrival order, while the batch fits the limits and the memory budget
Cohort *akb_server::take_cohort() {
  Job *h = queue.front();
  auto *c = new Cohort();
  c->et = h->et;
  c->rule = h->rule;
  c->precision = h->precision;
  c->dim = h->dim;
  c->law = h->law;
  for (auto it = queue.begin(); it != queue.end();) {
    Job *j = *it;
    const bool same = batchable(j) && j->et == c->et && j->rule == c->rule &&
                      j->precision == c->precision && j->law == c->law;
    if (!same || (int)c->jobs.size() >= cfg.batch_max_instances ||
        (!c->jobs.empty() && c->E + j->E > cfg.batch_max_elements) ||
        active + (int)c->jobs.size() >= cfg.max_active) {
      ++it;
      continue;
    }
    c->jobs.push_back(j);
    c->N += j->N;
    c->E += j->E;
    const int64_t need = cohort_bytes(c);
    if (!(reserved == 0 && c->jobs.size() == 1) && reserved + need > cfg.device_bytes) {
      c->jobs.pop_back();
      c->N -= j->N;
      c->E -= j->E;
      if (c->jobs.empty()) break;  // the head waits for memory: no overtaking
      ++it;
      continue;
    }
    it = queue.erase(it);
  }
  c->est_bytes = cohort_bytes(c);
  return c;
}

void akb_server::build(Job *j) {
  int rc = akb_model_create(j->dim, j->et, j->X.data(), j->N, j->conn.data(), j->E, &j->m);
  // short solves (few element-steps) on a high-priority stream: their kernels
  // are scheduled ahead of the long ones', which keeps their latency low
  if (rc == AKB_OK && (double)j->E * (double)j->steps < cfg.short_work) {
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess)
      rc = akb_model_set_stream_priority(j->m, greatest);
  }
  if (rc == AKB_OK) rc = akb_model_add_material(j->m, j->mat_type.c_str(), j->mat_params.c_str());
  if (rc == AKB_OK && j->rule) rc = akb_model_set_quadrature_rule(j->m, j->rule);
  if (rc == AKB_OK) rc = akb_model_init_full(j->m, AKB_EXPLICIT_LUMPED_MASS, j->precision);
  const int64_t nd = j->N * j->dim;
  if (rc == AKB_OK && !j->u0.empty())
    rc = akb_model_set_nodal(j->m, AKB_DISPLACEMENT, j->u0.data(), nd * (int64_t)sizeof(double));
  if (rc == AKB_OK && !j->v0.empty())
    rc = akb_model_set_nodal(j->m, AKB_VELOCITY, j->v0.data(), nd * (int64_t)sizeof(double));
  if (rc == AKB_OK && !j->blocked.empty())
    rc = akb_model_set_nodal(j->m, AKB_BLOCKED_DOFS, j->blocked.data(), nd);
  double dt = 0.;
  if (rc == AKB_OK) rc = akb_model_get_stable_time_step(j->m, &dt);
  if (rc == AKB_OK) {
    j->dt = j->dt_factor * dt;
    rc = akb_model_set_time_step(j->m, j->dt);
  }
  if (rc == AKB_OK && j->steps >= 100) rc = akb_model_prepare_graphs(j->m);
  if (rc == AKB_OK) rc = akb_model_stream(j->m, &j->stream);
  for (auto &e : j->ev)
    if (rc == AKB_OK && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
      rc = AKB_ECUDA;
  // the request's host copies are no longer needed
  std::vector<double>().swap(j->X);
  std::vector<double>().swap(j->v0);
  std::vector<double>().swap(j->u0);
  std::vector<int32_t>().swap(j->conn);
  std::vector<uint8_t>().swap(j->blocked);
  if (rc != AKB_OK) {
    j->status = rc;
    j->message = err_text();
    release_model(j);
  }
  std::lock_guard<std::mutex> lock(mu);
  n_building--;
  if (rc != AKB_OK) {
    complete(j);
    return;
  }
  j->left = j->steps;
  j->phase = STEPPING;
  ready.push_back(j);
  cv_sched.notify_all();
}

void akb_server::build_cohort(Cohort *c) {
  const int ni = (int)c->jobs.size();
  const int d = c->dim;
  std::vector<int64_t> nb_nodes(ni), nb_elems(ni);
  c->node_off.assign(ni + 1, 0);
  for (int k = 0; k < ni; ++k) {
    nb_nodes[k] = c->jobs[k]->N;
    nb_elems[k] = c->jobs[k]->E;
    c->node_off[k + 1] = c->node_off[k] + nb_nodes[k];
  }
  const int64_t N = c->node_off[ni], nd = N * d;
  const int nn = c->et == AKB_TETRAHEDRON_4 ? 4 : (c->et == AKB_HEXAHEDRON_8 ? 8 : 6);
  std::vector<double> X((size_t)nd), u0, v0;
  std::vector<int32_t> conn;
  std::vector<uint8_t> blocked;
  conn.reserve((size_t)c->E * nn);
  bool any_u = false, any_v = false, any_b = false;
  for (int k = 0; k < ni; ++k) {
    Job *j = c->jobs[k];
    std::copy(j->X.begin(), j->X.end(), X.begin() + c->node_off[k] * d);
    conn.insert(conn.end(), j->conn.begin(), j->conn.end());
    any_u |= !j->u0.empty();
    any_v |= !j->v0.empty();
    any_b |= !j->blocked.empty();
  }
  auto gather = [&](bool any, auto member, auto &out) {
    if (!any) return;
    out.assign((size_t)nd, 0);
    for (int k = 0; k < ni; ++k) {
      const auto &src = c->jobs[k]->*member;
      std::copy(src.begin(), src.end(), out.begin() + c->node_off[k] * d);
    }
  };
  gather(any_u, &Job::u0, u0);
  gather(any_v, &Job::v0, v0);
  gather(any_b, &Job::blocked, blocked);
  int rc = akb_batch_create(d, c->et, ni, nb_nodes.data(), nb_elems.data(), X.data(),
                            conn.data(), &c->m);
  for (int k = 0; k < ni && rc == AKB_OK; ++k)
    rc = akb_model_add_material(c->m, c->jobs[k]->mat_type.c_str(), c->jobs[k]->mat_params.c_str());
  std::vector<int32_t> mat_of(ni);
  for (int k = 0; k < ni; ++k) mat_of[k] = k;
  if (rc == AKB_OK) rc = akb_batch_set_instance_materials(c->m, mat_of.data());
  if (rc == AKB_OK && c->rule) rc = akb_model_set_quadrature_rule(c->m, c->rule);
  if (rc == AKB_OK) rc = akb_model_init_full(c->m, AKB_EXPLICIT_LUMPED_MASS, c->precision);
  if (rc == AKB_OK && any_u)
    rc = akb_model_set_nodal(c->m, AKB_DISPLACEMENT, u0.data(), nd * (int64_t)sizeof(double));
  if (rc == AKB_OK && any_v)
    rc = akb_model_set_nodal(c->m, AKB_VELOCITY, v0.data(), nd * (int64_t)sizeof(double));
  if (rc == AKB_OK && any_b) rc = akb_model_set_nodal(c->m, AKB_BLOCKED_DOFS, blocked.data(), nd);
  std::vector<double> dts(ni, 0.);
  if (rc == AKB_OK) rc = akb_batch_get_stable_time_steps(c->m, dts.data());
  if (rc == AKB_OK) {
    for (int k = 0; k < ni; ++k) {
      dts[k] = c->jobs[k]->dt_factor * dts[k];
      c->jobs[k]->dt = dts[k];
    }
    rc = akb_batch_set_time_steps(c->m, dts.data());
  }
  std::vector<int64_t> steps(ni);
  for (int k = 0; k < ni; ++k) {
    Job *j = c->jobs[k];
    steps[k] = j->steps;
    j->cohort = c;
    j->inst = k;
    j->end_step = j->steps;
    c->max_steps = std::max(c->max_steps, j->steps);
  }
  if (rc == AKB_OK) rc = akb_batch_set_instance_steps(c->m, steps.data());
  if (rc == AKB_OK && c->max_steps >= 100) rc = akb_model_prepare_graphs(c->m);
  if (rc == AKB_OK) rc = akb_model_stream(c->m, &c->stream);
  for (auto &e : c->ev)
    if (rc == AKB_OK && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
      rc = AKB_ECUDA;
  if (rc == AKB_OK &&
      cudaHostAlloc((void **)&c->stage, sizeof(double) * (size_t)std::max<int64_t>(2 * nd, 1),
                    cudaHostAllocDefault) != cudaSuccess)
    rc = fail(AKB_ENOMEM, "pinned staging buffer");
  if (rc == AKB_OK)
    for (Job *j : c->jobs) {
      std::vector<double>().swap(j->X);
      std::vector<double>().swap(j->v0);
      std::vector<double>().swap(j->u0);
      std::vector<int32_t>().swap(j->conn);
      std::vector<uint8_t>().swap(j->blocked);
    }
  c->by_end = c->jobs;
  std::stable_sort(c->by_end.begin(), c->by_end.end(),
                   [](const Job *a, const Job *b) { return a->end_step < b->end_step; });
  if (rc != AKB_OK) {
    c->status = rc;
    c->message = err_text();
    release_cohort(c);
  }
  std::lock_guard<std::mutex> lock(mu);
  n_building -= (int64_t)c->jobs.size();
  if (rc != AKB_OK) {
    // one bad request (an inverted element, say) must not fail the others:
    // every request of the batch goes back to the queue's front, to be
    // admitted alone and report its own status
    reserved -= c->est_bytes;
    active -= (int)c->jobs.size();
    for (auto it = c->jobs.rbegin(); it != c->jobs.rend(); ++it) {
      Job *j = *it;
      j->cohort = nullptr;
      j->inst = -1;
      j->solo = true;
      j->dt = 0.;
      j->phase = QUEUED;
      queue.push_front(j);
    }
    delete c;
    cv_work.notify_all();
    return;
  }
  for (Job *j : c->jobs) j->phase = STEPPING;
  c->unreported = ni;
  ready_cohorts.push_back(c);
  cv_sched.notify_all();
}

void akb_server::finish_job(Job *j) {
  int rc = AKB_OK;
  const int64_t nd = j->N * j->dim;
  const int64_t nbytes = nd * (int64_t)sizeof(double);
  if (j->cohort) {
    // the batch's stream has copied this instance's final state to staging
    Cohort *c = j->cohort;
    const double *us = c->stage + c->node_off[j->inst] * j->dim;
    const double *vs = c->stage + c->node_off.back() * j->dim + c->node_off[j->inst] * j->dim;
    if (j->status == AKB_OK && !(all_finite(us, nd) && all_finite(vs, nd))) {
      rc = AKB_ENAN;
      j->message = "non-finite state";
    }
    if (rc == AKB_OK && j->status == AKB_OK) {
      if (j->u_out) std::memcpy(j->u_out, us, (size_t)nbytes);
      if (j->v_out) std::memcpy(j->v_out, vs, (size_t)nbytes);
    }
    if (rc != AKB_OK && j->status == AKB_OK) j->status = rc;
    std::lock_guard<std::mutex> lock(mu);
    complete(j);
    if (--c->unreported == 0) {
      retire.push_back(c);
      cv_work.notify_all();
    }
    return;
  }
  int flags = 0;
  if (j->status == AKB_OK) rc = akb_model_get_status(j->m, &flags);
  if (rc == AKB_OK && j->status == AKB_OK && flags) {
    rc = AKB_ENAN;
    j->message = "non-finite acceleration";
  }
  if (rc == AKB_OK && j->status == AKB_OK && j->u_out)
    rc = akb_model_get_nodal(j->m, AKB_DISPLACEMENT, j->u_out, nbytes);
  if (rc == AKB_OK && j->status == AKB_OK && j->v_out)
    rc = akb_model_get_nodal(j->m, AKB_VELOCITY, j->v_out, nbytes);
  if (rc != AKB_OK && j->status == AKB_OK) {
    j->status = rc;
    if (j->message.empty()) j->message = err_text();
  }
  release_model(j);
  std::lock_guard<std::mutex> lock(mu);
  complete(j);
}

void akb_server::retire_cohort(Cohort *c) {
  release_cohort(c);
  std::lock_guard<std::mutex> lock(mu);
  reserved -= c->est_bytes;
  delete c;
  cv_work.notify_all();
}

void akb_server::builder_loop() {
  cudaSetDevice(cfg.device);
  for (;;) {
    Job *j = nullptr;
    Cohort *c = nullptr, *old = nullptr;
    bool fin = false;
    {
      std::unique_lock<std::mutex> lock(mu);
      cv_work.wait(lock, [&] {
        if (stop || !finish.empty() || !retire.empty()) return true;
        if (queue.empty() || active >= cfg.max_active) return false;
        if (batchable(queue.front())) return true;  // the batch is sized to fit
        return reserved == 0 || reserved + queue.front()->est_bytes <= cfg.device_bytes;
      });
      if (!finish.empty()) {
        j = finish.front();
        finish.pop_front();
        fin = true;
      } else if (!retire.empty()) {
        old = retire.front();
        retire.pop_front();
      } else if (stop) {
        return;
      } else if (batchable(queue.front())) {
        c = take_cohort();
        if (c->jobs.empty()) {
          // nothing fits right now: give the requests back, wait for memory
          for (auto it = c->jobs.rbegin(); it != c->jobs.rend(); ++it) queue.push_front(*it);
          std::stable_sort(queue.begin(), queue.end(),
                           [](const Job *a, const Job *b) { return a->id < b->id; });
          delete c;
          c = nullptr;
          cv_work.wait_for(lock, std::chrono::milliseconds(2));
          continue;
        }
        if (c->jobs.size() == 1 &&
            (reserved == 0 || reserved + c->jobs[0]->est_bytes <= cfg.device_bytes)) {
          // nothing to share a batch with (the load is light): a model of its
          // own, which builds and steps faster than a batch of one
          j = c->jobs[0];
          delete c;
          c = nullptr;
          reserved += j->est_bytes;
          active++;
          n_building++;
          j->phase = BUILDING;
          j->t_admit = now();
        } else {
          reserved += c->est_bytes;
          const double t = now();
          for (Job *jj : c->jobs) {
            jj->phase = BUILDING;
            jj->t_admit = t;
          }
          active += (int)c->jobs.size();
          n_building += (int64_t)c->jobs.size();
        }
      } else {
        j = queue.front();
        queue.pop_front();
        reserved += j->est_bytes;
        active++;
        n_building++;
        j->phase = BUILDING;
        j->t_admit = now();
      }
    }
    if (fin)
      finish_job(j);
    else if (old)
      retire_cohort(old);
    else if (c)
      build_cohort(c);
    else
      build(j);
  }
}

void akb_server::scheduler_loop() {
  cudaSetDevice(cfg.device);
  std::vector<Job *> running;
  std::vector<Cohort *> cohorts;
  const int64_t G = 100;  // steps per captured graph
  for (;;) {
    {
      std::unique_lock<std::mutex> lock(mu);
      if (ready.empty() && running.empty() && ready_cohorts.empty() && cohorts.empty())
        cv_sched.wait(lock, [&] { return stop || !ready.empty() || !ready_cohorts.empty(); });
      for (Job *j : ready) running.push_back(j);
      n_running += (int64_t)ready.size();
      ready.clear();
      for (Cohort *c : ready_cohorts) {
        cohorts.push_back(c);
        n_running += (int64_t)c->jobs.size();
      }
      ready_cohorts.clear();
      if (stop && running.empty() && cohorts.empty()) return;
    }
    bool progress = false;
    std::vector<Job *> leaving;
    for (Job *j : running) {
      while (j->inflight > 0) {
        cudaError_t e = cudaEventQuery(j->ev[j->head]);
        if (e == cudaErrorNotReady) break;
        if (e != cudaSuccess) {
          j->status = AKB_ECUDA;
          j->message = std::string("step chunk: ") + cudaGetErrorString(e);
          j->left = 0;
        }
        j->head = 1 - j->head;
        j->inflight--;
        progress = true;
      }
      while (j->status == AKB_OK && j->inflight < 2 && j->left > 0) {
        const int64_t n = std::min(j->left, cfg.chunk_steps);
        if (j->t_start == 0.) j->t_start = now();
        int rc = akb_model_solve_step(j->m, n);
        if (rc == AKB_OK &&
            cudaEventRecord(j->ev[(j->head + j->inflight) % 2], (cudaStream_t)j->stream) !=
                cudaSuccess)
          rc = AKB_ECUDA;
        if (rc != AKB_OK) {
          j->status = rc;
          j->message = err_text();
          j->left = 0;
          break;
        }
        j->inflight++;
        j->left -= n;
        progress = true;
      }
      if (j->left == 0 && j->inflight == 0) leaving.push_back(j);
    }
    std::vector<Cohort *> drained;
    for (Cohort *c : cohorts) {
      while (c->inflight > 0) {
        cudaError_t e = cudaEventQuery(c->ev[c->head]);
        if (e == cudaErrorNotReady) break;
        if (e != cudaSuccess && c->status == AKB_OK) {
          c->status = AKB_ECUDA;
          c->message = std::string("step chunk: ") + cudaGetErrorString(e);
        }
        for (Job *j : c->chunk_jobs[c->head]) {
          if (c->status != AKB_OK) {
            j->status = c->status;
            j->message = c->message;
          }
          leaving.push_back(j);
        }
        c->chunk_jobs[c->head].clear();
        c->head = 1 - c->head;
        c->inflight--;
        progress = true;
      }
      while (c->inflight < 2 && c->next_end < c->by_end.size()) {
        // up to chunk_steps steps, ending at the next instance end rounded up
        // to whole graphs
        const int64_t target = c->by_end[c->next_end]->end_step;
        int64_t n = std::min<int64_t>(cfg.chunk_steps, c->max_steps - c->enqueued);
        if (target > c->enqueued) {
          const int64_t to_end = ((target - c->enqueued + G - 1) / G) * G;
          n = std::min(n, to_end);
        } else {
          n = 0;  // instances ending now (zero steps): copies only
        }
        const double t = now();
        for (Job *j : c->jobs)
          if (j->t_start == 0.) j->t_start = t;
        int rc = c->status;
        if (rc == AKB_OK && n > 0) rc = akb_model_solve_step(c->m, n);
        if (rc == AKB_OK) c->enqueued += n;
        const int slot = (c->head + c->inflight) % 2;
        // results of the instances that end within this chunk
        while (c->next_end < c->by_end.size() &&
               (rc != AKB_OK || c->by_end[c->next_end]->end_step <= c->enqueued)) {
          Job *j = c->by_end[c->next_end++];
          const int64_t nd = j->N * c->dim;
          const int64_t nbytes = nd * (int64_t)sizeof(double);
          double *us = c->stage + c->node_off[j->inst] * c->dim;
          double *vs = c->stage + c->node_off.back() * c->dim + c->node_off[j->inst] * c->dim;
          if (rc == AKB_OK)
            rc = akb_batch_copy_instance_nodal(c->m, AKB_DISPLACEMENT, j->inst, us, nbytes);
          if (rc == AKB_OK)
            rc = akb_batch_copy_instance_nodal(c->m, AKB_VELOCITY, j->inst, vs, nbytes);
          c->chunk_jobs[slot].push_back(j);
        }
        if (rc == AKB_OK &&
            cudaEventRecord(c->ev[slot], (cudaStream_t)c->stream) != cudaSuccess)
          rc = AKB_ECUDA;
        if (rc != AKB_OK && c->status == AKB_OK) {
          c->status = rc;
          c->message = err_text();
          // the event of this slot may not have been recorded: report at
          // once the requests of this chunk, and all later ones
          while (c->next_end < c->by_end.size()) c->chunk_jobs[slot].push_back(c->by_end[c->next_end++]);
          cudaStreamSynchronize((cudaStream_t)c->stream);
          cudaEventRecord(c->ev[slot], (cudaStream_t)c->stream);
        }
        c->inflight++;
        progress = true;
      }
      if (c->next_end == c->by_end.size() && c->inflight == 0) drained.push_back(c);
    }
    if (!leaving.empty() || !drained.empty()) {
      std::lock_guard<std::mutex> lock(mu);
      for (Job *j : leaving) {
        if (!j->cohort) running.erase(std::find(running.begin(), running.end(), j));
        j->phase = FINISHING;
        finish.push_back(j);
        n_running--;
      }
      // a drained batch stays alive until its last request is reported
      for (Cohort *c : drained) cohorts.erase(std::find(cohorts.begin(), cohorts.end(), c));
      cv_work.notify_all();
      progress = true;
    }
    if (!progress) {
      std::unique_lock<std::mutex> lock(mu);
      cv_sched.wait_for(lock, std::chrono::microseconds(100),
                        [&] { return stop || !ready.empty() || !ready_cohorts.empty(); });
    }
  }
}

extern "C" {

int akb_server_create(const akb_server_config *cfg, akb_server **out) {
  if (!out) return fail(AKB_EINVAL, "null output pointer");
  *out = nullptr;
  akb_server_config c{};
  if (cfg) c = *cfg;
  // more hardware work queues than the default 8, so that independent solves
  // do not serialise behind one another (effective for contexts created
  // after this point)
  setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0);
  if (cudaSetDevice(c.device) != cudaSuccess) return fail(AKB_ECUDA, "cannot select the device");
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess)
    return fail(AKB_ECUDA, "cudaMemGetInfo failed");
  if (c.device_bytes <= 0) c.device_bytes = (int64_t)(0.8 * (double)free_b);
  if (c.max_active <= 0) c.max_active = 64;
  if (c.chunk_steps <= 0) c.chunk_steps = 500;
  if (c.builders <= 0) c.builders = 4;
  if (c.short_work <= 0.) c.short_work = 1e8;
  if (c.batch_max_request_elements <= 0) c.batch_max_request_elements = 1 << 17;
  if (c.batch_max_elements <= 0) c.batch_max_elements = 1 << 23;
  if (c.batch_max_instances <= 0) c.batch_max_instances = 256;
  auto *s = new akb_server();
  s->cfg = c;
  s->t0 = std::chrono::steady_clock::now();
  s->sched = std::thread([s] { s->scheduler_loop(); });
  for (int k = 0; k < c.builders; ++k) s->builders.emplace_back([s] { s->builder_loop(); });
  *out = s;
  return AKB_OK;
}

int akb_server_submit(akb_server *s, const akb_request *r, int64_t *id) {
  if (!s || !r) return fail(AKB_EINVAL, "null argument");
  if (r->element_type < AKB_TETRAHEDRON_4 || r->element_type > AKB_TRIANGLE_6)
    return fail(AKB_EINVAL, "unknown element type");
  if (r->nb_nodes < 0 || r->nb_elements < 0 || r->nb_steps < 0 || !r->material_type ||
      (r->nb_nodes > 0 && !r->nodes) || (r->nb_elements > 0 && !r->connectivity))
    return fail(AKB_EINVAL, "bad request");
  const int law = law_of(r->material_type);
  if (law < 0) return fail(AKB_EMATERIAL, std::string("unknown material type '") + r->material_type + "'");
  auto *j = new Job();
  j->et = r->element_type;
  j->dim = r->element_type == AKB_TRIANGLE_6 ? 2 : 3;
  j->law = law;
  const int nn = r->element_type == AKB_TETRAHEDRON_4 ? 4 : (r->element_type == AKB_HEXAHEDRON_8 ? 8 : 6);
  j->rule = r->quadrature_rule;
  j->precision = r->precision;
  j->N = r->nb_nodes;
  j->E = r->nb_elements;
  j->steps = r->nb_steps;
  const int64_t nd = j->N * j->dim;
  j->X.assign(r->nodes, r->nodes + nd);
  j->conn.assign(r->connectivity, r->connectivity + j->E * nn);
  for (int32_t x : j->conn)
    if (x < 0 || x >= j->N) {
      delete j;
      return fail(AKB_EINVAL, "connectivity refers to a missing node");
    }
  if (r->velocity) j->v0.assign(r->velocity, r->velocity + nd);
  if (r->displacement) j->u0.assign(r->displacement, r->displacement + nd);
  if (r->blocked_dofs) j->blocked.assign(r->blocked_dofs, r->blocked_dofs + nd);
  j->mat_type = r->material_type;
  j->mat_params = r->material_params ? r->material_params : "";
  j->dt_factor = r->dt_factor > 0. ? r->dt_factor : 0.8;
  j->u_out = r->displacement_out;
  j->v_out = r->velocity_out;
  int rc = akb_estimate_device_bytes(j->et, j->rule, j->N, j->E, law, j->precision, &j->est_bytes);
  if (rc != AKB_OK) {
    delete j;
    return rc;
  }
  if (j->est_bytes > s->cfg.device_bytes) {
    const int64_t need = j->est_bytes;
    delete j;
    return fail(AKB_ENOMEM, "the solve needs " + std::to_string(need) +
                                " device bytes, more than the server's budget");
  }
  std::lock_guard<std::mutex> lock(s->mu);
  if (s->stop) {
    delete j;
    return fail(AKB_ESTATE, "the server is shutting down");
  }
  j->id = s->next_id++;
  j->t_submit = s->now();
  s->queue.push_back(j);
  if (id) *id = j->id;
  s->cv_work.notify_all();
  return AKB_OK;
}

int akb_server_poll(akb_server *s, akb_completion *out, int capacity, int *count,
                    double wait_seconds) {
  if (!s || !count || (capacity > 0 && !out)) return fail(AKB_EINVAL, "null argument");
  *count = 0;
  std::unique_lock<std::mutex> lock(s->mu);
  if (s->done.empty() && wait_seconds > 0.)
    s->cv_done.wait_for(lock, std::chrono::duration<double>(wait_seconds),
                        [&] { return !s->done.empty(); });
  while (*count < capacity && !s->done.empty()) {
    Job *j = s->done.front();
    s->done.pop_front();
    akb_completion &c = out[(*count)++];
    std::memset(&c, 0, sizeof(c));
    c.id = j->id;
    c.status = j->status;
    std::snprintf(c.message, sizeof(c.message), "%s", j->message.c_str());
    c.t_submit = j->t_submit;
    c.t_admit = j->t_admit;
    c.t_start = j->t_start;
    c.t_end = j->t_end;
    c.nb_elements = j->E;
    c.nb_steps = j->steps;
    c.dt = j->dt;
    c.device_bytes = j->est_bytes;
    c.batched = j->cohort ? 1 : 0;
    delete j;
  }
  return AKB_OK;
}

int akb_server_get_stats(akb_server *s, akb_server_stats *st) {
  if (!s || !st) return fail(AKB_EINVAL, "null argument");
  std::lock_guard<std::mutex> lock(s->mu);
  st->queued = (int64_t)s->queue.size();
  st->building = s->n_building;
  st->running = s->n_running + (int64_t)s->ready.size();
  for (auto *c : s->ready_cohorts) st->running += (int64_t)c->jobs.size();
  st->finishing = (int64_t)s->finish.size();
  st->completed_unpolled = (int64_t)s->done.size();
  st->device_bytes_reserved = s->reserved;
  st->device_bytes_budget = s->cfg.device_bytes;
  st->now = s->now();
  return AKB_OK;
}

int akb_server_destroy(akb_server *s) {
  if (!s) return AKB_OK;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    // queued solves are dropped; admitted ones run to completion
    for (Job *j : s->queue) delete j;
    s->queue.clear();
  }
  // wait until every admitted solve is done and every batch released
  {
    std::unique_lock<std::mutex> lock(s->mu);
    s->cv_done.wait(lock, [&] { return s->active == 0; });
    s->cv_work.wait(lock, [&] { return s->retire.empty() && s->reserved == 0; });
    s->stop = true;
  }
  s->cv_work.notify_all();
  s->cv_sched.notify_all();
  s->sched.join();
  for (auto &t : s->builders) t.join();
  for (Job *j : s->done) delete j;
  delete s;
  return AKB_OK;
}

}  // extern "C"
