// Serving loop: many explicit solves resident on one GPU at once.
//
// A request is a mesh, one material, an initial state and a step count.  It
// waits in a FIFO until the device memory it needs (akb_estimate_device_bytes)
// fits in the budget and a slot is free; a builder thread then prepares its
// model (mesh tables, lumped mass, stable time step, captured step graph) on
// the model's own stream, and the scheduler thread folds it into the running
// set.  The scheduler keeps every running solve two chunks ahead: a chunk is
// a solve_step of up to chunk_steps steps (100-step graph launches) followed
// by an event, so the solves' kernels overlap on the device while the host
// only polls events.  A solve whose steps are all enqueued and completed is
// handed back to a builder thread, which copies its result into the caller's
// buffers and frees its memory (stream-ordered frees: no device-wide
// synchronisation).  Each solve runs alone on its own model, so its result
// is the same whatever else is running.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
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

struct Job {
  int64_t id = 0;
  // request (copied at submission)
  int et = 0, rule = 0, precision = 0, dim = 3;
  int64_t N = 0, E = 0, steps = 0;
  std::vector<double> X, v0, u0;
  std::vector<int32_t> conn;
  std::vector<uint8_t> blocked;
  std::string mat_type, mat_params;
  double dt_factor = 0.8;
  double *u_out = nullptr, *v_out = nullptr;
  int64_t est_bytes = 0;
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
  std::condition_variable cv_work;   // builders: queue / finish list changed
  std::condition_variable cv_sched;  // scheduler: ready list changed
  std::condition_variable cv_done;   // pollers: completion available
  std::deque<Job *> queue, finish, done;
  std::vector<Job *> ready;
  int64_t reserved = 0;  // device bytes of admitted solves
  int active = 0;        // admitted and not yet done
  int64_t next_id = 1;
  int64_t n_building = 0, n_running = 0;
  bool stop = false;
  std::thread sched;
  std::vector<std::thread> builders;

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  void builder_loop();
  void scheduler_loop();
  void build(Job *j);
  void finish_job(Job *j);
  void complete(Job *j);  // caller holds mu
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

}  // namespace

// a finished or failed job: frees its slot and memory reservation
void akb_server::complete(Job *j) {
  j->phase = DONE;
  j->t_end = now();
  reserved -= j->est_bytes;
  active--;
  done.push_back(j);
  cv_done.notify_all();
  cv_work.notify_all();
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

void akb_server::finish_job(Job *j) {
  int rc = AKB_OK;
  const int64_t nbytes = j->N * j->dim * (int64_t)sizeof(double);
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

void akb_server::builder_loop() {
  cudaSetDevice(cfg.device);
  for (;;) {
    Job *j = nullptr;
    bool fin = false;
    {
      std::unique_lock<std::mutex> lock(mu);
      cv_work.wait(lock, [&] {
        if (stop || !finish.empty()) return true;
        if (queue.empty() || active >= cfg.max_active) return false;
        return reserved == 0 || reserved + queue.front()->est_bytes <= cfg.device_bytes;
      });
      if (!finish.empty()) {
        j = finish.front();
        finish.pop_front();
        fin = true;
      } else if (stop) {
        return;
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
    else
      build(j);
  }
}

void akb_server::scheduler_loop() {
  cudaSetDevice(cfg.device);
  std::vector<Job *> running;
  for (;;) {
    {
      std::unique_lock<std::mutex> lock(mu);
      if (ready.empty() && running.empty())
        cv_sched.wait(lock, [&] { return stop || !ready.empty(); });
      for (Job *j : ready) running.push_back(j);
      n_running += (int64_t)ready.size();
      ready.clear();
      if (stop && running.empty()) return;
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
    if (!leaving.empty()) {
      std::lock_guard<std::mutex> lock(mu);
      for (Job *j : leaving) {
        running.erase(std::find(running.begin(), running.end(), j));
        j->phase = FINISHING;
        finish.push_back(j);
        n_running--;
      }
      cv_work.notify_all();
      progress = true;
    }
    if (!progress) {
      std::unique_lock<std::mutex> lock(mu);
      cv_sched.wait_for(lock, std::chrono::microseconds(100),
                        [&] { return stop || !ready.empty(); });
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
  const int nn = r->element_type == AKB_TETRAHEDRON_4 ? 4 : (r->element_type == AKB_HEXAHEDRON_8 ? 8 : 6);
  j->rule = r->quadrature_rule;
  j->precision = r->precision;
  j->N = r->nb_nodes;
  j->E = r->nb_elements;
  j->steps = r->nb_steps;
  const int64_t nd = j->N * j->dim;
  j->X.assign(r->nodes, r->nodes + nd);
  j->conn.assign(r->connectivity, r->connectivity + j->E * nn);
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
  // wait until every admitted solve is done
  {
    std::unique_lock<std::mutex> lock(s->mu);
    s->cv_done.wait(lock, [&] { return s->active == 0; });
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
