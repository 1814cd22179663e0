// Reconstruction server (include/spimage/serve.h): a native worker thread that
// admits jobs by device-memory footprint, keeps each job resident in its own
// device context on its own stream, and advances all admitted jobs chunk by
// chunk through the SpPhaser API.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <chrono>
#include <condition_variable>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "spimage.h"
#include "spimage/serve.h"
#include "spimage/spb_device.h"

namespace {

thread_local std::string g_err;

int fail(const std::string &msg) {
  g_err = msg;
  return -1;
}

using Clock = std::chrono::steady_clock;

// A device context of one shape and start count, reused across jobs.
struct Slot {
  SpPhaser *ph = nullptr;
  cudaStream_t st = nullptr;
  int nx = 0, ny = 0, nz = 0, starts = 0;
  bool dm = false;
  long long bytes = 0;
  bool busy = false;
  double last_used = 0;
  Image *amp_img = nullptr, *sup_img = nullptr, *model_img = nullptr;
  unsigned *nf_host = nullptr;  // page-locked: the job's sticky non-finite flag after its last checked chunk
};

struct Job {
  long long id = 0;
  spb_job desc{};
  std::vector<float> amp;
  std::vector<int> mask, support;
  int status = 1;
  std::string err;
  double t_submit = -1, t_admit = -1, t_finish = -1;
  long long slots = 0;
  // run state (worker thread only)
  Slot *slot = nullptr;
  SpPhasingAlgorithm *algs[SPB_JOB_MAX_STAGES] = {};
  sp_smap *maps[SPB_JOB_MAX_STAGES + 2] = {};
  SpSupportAlgorithm *sup_alg = nullptr;
  SpSupportArray *sup = nullptr;
  int stage = 0, stage_left = 0;
  long long issued = 0;
  std::deque<cudaEvent_t> inflight;
  std::deque<long long> inflight_slots;  // slots done when the matching event completes
  bool cancel = false;                   // set by spb_server_cancel (under mu)
  // results
  std::vector<float> efourier, sfrac, models;
};

bool has_dm(const spb_job &d) {
  for (int i = 0; i < d.nstages; i++)
    if (d.stage[i].algorithm == SpDiffMap) return true;
  return false;
}

}  // namespace

struct spb_server {
  spb_server_config cfg{};
  Clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  long long next_id = 0;
  std::deque<std::shared_ptr<Job>> pending;
  std::map<long long, std::shared_ptr<Job>> jobs;  // every job not yet released
  std::thread worker;
  int device = 0;
  // worker-only state
  std::list<Slot> slots;
  std::vector<std::shared_ptr<Job>> active;
  std::vector<cudaEvent_t> free_events;
  long long held_bytes = 0;
  // counters (under mu)
  double stats[8] = {};

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
  void run();
  bool admit_one();
  Slot *acquire_slot(const spb_job &d, long long need, bool *no_room);
  void free_slot(Slot *s);
  int start_job(Job &j);
  int issue_chunk(Job &j);
  void finish_job(const std::shared_ptr<Job> &j, int status, const std::string &err);
  void release_job_objects(Job &j);
  cudaEvent_t get_event();
};

// ------------------------------------------------------------------ slots
namespace {

void destroy_slot_objects(Slot &s) {
  if (s.ph) sp_phaser_free(s.ph);
  if (s.st) cudaStreamDestroy(s.st);
  if (s.amp_img) sp_image_free(s.amp_img);
  if (s.sup_img) sp_image_free(s.sup_img);
  if (s.model_img) sp_image_free(s.model_img);
  if (s.nf_host) cudaFreeHost(s.nf_host);
  s = Slot();
}

}  // namespace

void spb_server::free_slot(Slot *s) {
  held_bytes -= s->bytes;
  destroy_slot_objects(*s);
  for (auto it = slots.begin(); it != slots.end(); ++it)
    if (&*it == s) {
      slots.erase(it);
      break;
    }
}

// An idle context for the job (reused, grown for the difference map, or new),
// or nullptr: *no_room when the budget cannot hold it now, else an error.
Slot *spb_server::acquire_slot(const spb_job &d, long long need, bool *no_room) {
  *no_room = false;
  const bool dm = has_dm(d);
  const double budget = cfg.hbm_budget_bytes;
  Slot *reuse = nullptr;
  for (auto &s : slots)
    if (!s.busy && s.nx == d.nx && s.ny == d.ny && s.nz == d.nz && s.starts == d.starts)
      if (!reuse || (dm && s.dm && !reuse->dm)) reuse = &s;
  const long long extra = reuse ? (need > reuse->bytes ? need - reuse->bytes : 0) : need;
  // free idle contexts of other shapes, least recently used first, until the job fits
  while ((double)(held_bytes + extra) > budget) {
    Slot *lru = nullptr;
    for (auto &s : slots)
      if (!s.busy && &s != reuse && (!lru || s.last_used < lru->last_used)) lru = &s;
    if (!lru) break;
    free_slot(lru);
    std::lock_guard<std::mutex> lk(mu);
    stats[5] += 1;
  }
  if ((double)(held_bytes + extra) > budget) {
    *no_room = true;
    return nullptr;
  }
  if (reuse) {
    reuse->busy = true;
    reuse->bytes += extra;
    reuse->dm = reuse->dm || dm;
    held_bytes += extra;
    std::lock_guard<std::mutex> lk(mu);
    stats[6] += 1;
    return reuse;
  }
  slots.emplace_back();
  Slot &s = slots.back();
  s.nx = d.nx;
  s.ny = d.ny;
  s.nz = d.nz;
  s.starts = d.starts;
  s.dm = dm;
  s.bytes = need;
  s.busy = true;
  held_bytes += need;
  s.ph = sp_phaser_alloc();
  cudaError_t e = cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking);
  if (e != cudaSuccess || sp_phaser_set_starts(s.ph, d.starts) != 0) {
    fail(std::string("context set-up: ") + cudaGetErrorString(e));
    free_slot(&s);
    return nullptr;
  }
  s.amp_img = sp_image_alloc(d.nx, d.ny, d.nz);
  s.sup_img = sp_image_alloc(d.nx, d.ny, d.nz);
  if (cudaMallocHost(&s.nf_host, sizeof(unsigned)) != cudaSuccess) {
    s.nf_host = nullptr;
    fail("context set-up: cudaMallocHost failed");
    free_slot(&s);
    return nullptr;
  }
  *s.nf_host = 0;
  std::lock_guard<std::mutex> lk(mu);
  stats[4] += 1;
  if ((double)held_bytes > stats[3]) stats[3] = (double)held_bytes;
  return &s;
}

cudaEvent_t spb_server::get_event() {
  if (!free_events.empty()) {
    cudaEvent_t e = free_events.back();
    free_events.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
  return e;
}

// ------------------------------------------------------------------- jobs
void spb_server::release_job_objects(Job &j) {
  for (auto &a : j.algs)
    if (a) {
      free(a->params);
      free(a);
      a = nullptr;
    }
  for (auto &m : j.maps)
    if (m) {
      spb_smap_free(m);
      m = nullptr;
    }
  if (j.sup_alg) {
    free(j.sup_alg->params);
    free(j.sup_alg);
    j.sup_alg = nullptr;
  }
  if (j.sup) {
    free(j.sup->algorithms);
    free(j.sup);
    j.sup = nullptr;
  }
  for (cudaEvent_t e : j.inflight) free_events.push_back(e);
  j.inflight.clear();
  j.inflight_slots.clear();
}

int spb_server::start_job(Job &j) {
  const spb_job &d = j.desc;
  Slot &s = *j.slot;
  const int n = d.nx * d.ny * d.nz;
  const real k0 = 0;
  for (int i = 0; i < d.nstages; i++) {
    const real beta = d.stage[i].beta;
    switch (d.stage[i].algorithm) {
      case SpHIO:
        j.maps[i] = spb_smap_create(1, &k0, &beta);
        j.algs[i] = sp_phasing_hio_alloc(j.maps[i], (SpPhasingConstraints)d.constraints);
        break;
      case SpRAAR:
        j.maps[i] = spb_smap_create(1, &k0, &beta);
        j.algs[i] = sp_phasing_raar_alloc(j.maps[i], (SpPhasingConstraints)d.constraints);
        break;
      case SpDiffMap:
        j.maps[i] = spb_smap_create(1, &k0, &beta);
        j.algs[i] = sp_phasing_diff_map_alloc(j.maps[i], INFINITY, INFINITY, (SpPhasingConstraints)d.constraints);
        break;
      case SpER:
        j.algs[i] = sp_phasing_er_alloc((SpPhasingConstraints)d.constraints);
        break;
      default:
        return fail("unknown algorithm " + std::to_string(d.stage[i].algorithm));
    }
  }
  if (d.support_period > 0) {
    const real keys[2] = {0, (real)j.slots};
    const real blur[2] = {d.blur_start, d.blur_end};
    const real area = d.support_area;
    j.maps[SPB_JOB_MAX_STAGES] = spb_smap_create(2, keys, blur);
    j.maps[SPB_JOB_MAX_STAGES + 1] = spb_smap_create(1, &k0, &area);
    j.sup_alg = sp_support_area_alloc(j.maps[SPB_JOB_MAX_STAGES], j.maps[SPB_JOB_MAX_STAGES + 1]);
    j.sup = sp_support_array_init(j.sup_alg, d.support_period);
  }
  SpPhaser *ph = s.ph;
  if (sp_phaser_init(ph, j.algs[0], j.sup, SpEngineCUDA)) return fail(std::string("sp_phaser_init: ") + sp_phaser_last_error());
  ph->model_iteration = ph->fmodel_iteration = ph->model_before_projection_iteration = -1;
  ph->model_change_iteration = ph->support_iteration = ph->old_model_iteration = -1;
  for (int i = 0; i < n; i++) {
    s.amp_img->image->data[i] = sp_cinit(j.amp[i], 0);
    s.amp_img->mask->data[i] = j.mask[i] ? 1 : 0;
    s.sup_img->image->data[i] = sp_cinit(j.support[i] ? 1 : 0, 0);
  }
  sp_phaser_set_amplitudes(ph, s.amp_img);
  if (sp_phaser_set_cuda_stream(ph, s.st)) return fail(std::string("stream: ") + sp_phaser_last_error());
  std::vector<unsigned long long> seeds((size_t)d.starts);
  for (int b = 0; b < d.starts; b++) seeds[b] = d.seed + (unsigned long long)b;
  if (sp_phaser_init_models_device(ph, SpModelRandomPhases, seeds.data()))
    return fail(std::string("initial models: ") + sp_phaser_last_error());
  if (sp_phaser_init_support(ph, s.sup_img, 0, 0)) return fail("initial support");
  if (!cfg.no_autotune && sp_phaser_autotune(ph)) return fail(std::string("autotune: ") + sp_phaser_last_error());
  j.stage = 0;
  j.stage_left = d.stage[0].iterations;
  j.issued = 0;
  return 0;
}

// enqueue the next chunk of the job's schedule; 1 issued, 0 nothing left, -1 error
int spb_server::issue_chunk(Job &j) {
  SpPhaser *ph = j.slot->ph;
  while (j.stage_left == 0 && j.stage + 1 < j.desc.nstages) {
    j.stage++;
    j.stage_left = j.desc.stage[j.stage].iterations;
    sp_phaser_set_phasing_algorithm(ph, j.algs[j.stage]);
  }
  if (j.stage_left == 0) return 0;
  const int k = j.stage_left < cfg.chunk_slots ? j.stage_left : cfg.chunk_slots;
  const int rc = sp_phaser_iterate(ph, k);
  if (rc) return fail("sp_phaser_iterate returned " + std::to_string(rc) + ": " + sp_phaser_last_error());
  j.stage_left -= k;
  // every start's model checked for NaN/infinity after the chunk (sticky since the job's first chunk)
  if (spb_ctx_nonfinite_async((spb_ctx *)sp_phaser_device_context(ph), j.issued == 0 ? 1 : 0, j.slot->nf_host))
    return fail(std::string("non-finite check: ") + spb_error_string());
  j.issued += k;
  cudaEvent_t e = get_event();
  if (!e || cudaEventRecord(e, j.slot->st) != cudaSuccess) return fail("cudaEventRecord failed");
  j.inflight.push_back(e);
  j.inflight_slots.push_back(j.issued);
  return 1;
}

void spb_server::finish_job(const std::shared_ptr<Job> &jp, int status, const std::string &err) {
  Job &j = *jp;
  release_job_objects(j);
  if (j.slot) {
    if (status == SPB_JOB_FAILED) {
      cudaStreamSynchronize(j.slot->st);
      free_slot(j.slot);  // its state is unknown after a device or set-up error
    } else {
      // done, cancelled, diverged or out of time: the context is sound once
      // the chunks already queued on its stream have run
      if (status != 0) cudaStreamSynchronize(j.slot->st);
      j.slot->busy = false;
      j.slot->last_used = now();
    }
    j.slot = nullptr;
  }
  std::lock_guard<std::mutex> lk(mu);
  j.status = status;
  j.err = err;
  j.t_finish = now();
  if (status == 0) {
    stats[0] += 1;
    stats[1] += (double)j.desc.starts * (double)j.slots;
  } else {
    stats[7] += 1;
  }
  cv_done.notify_all();
}

// Admits the first pending job (in arrival order) that fits; false when none
// could be admitted.
bool spb_server::admit_one() {
  std::vector<std::shared_ptr<Job>> cand;
  {
    std::lock_guard<std::mutex> lk(mu);
    cand.assign(pending.begin(), pending.end());
  }
  // pending jobs whose time budget ran out end here, whether or not a slot is free
  for (auto &jp : cand) {
    Job &j = *jp;
    if (j.desc.time_budget_s > 0 && now() - j.t_submit > j.desc.time_budget_s) {
      {
        std::lock_guard<std::mutex> lk(mu);
        for (auto it = pending.begin(); it != pending.end(); ++it)
          if (*it == jp) {
            pending.erase(it);
            break;
          }
      }
      finish_job(jp, SPB_JOB_EXPIRED, "time budget of " + std::to_string(j.desc.time_budget_s) +
                                          " s ran out before the job was admitted");
      return true;
    }
  }
  if ((int)active.size() >= cfg.max_active_jobs) return false;
  for (auto &jp : cand) {
    Job &j = *jp;
    const long long need = spb_ctx_footprint(j.desc.nx, j.desc.ny, j.desc.nz, j.desc.starts, has_dm(j.desc));
    auto take = [&]() {
      std::lock_guard<std::mutex> lk(mu);
      for (auto it = pending.begin(); it != pending.end(); ++it)
        if (*it == jp) {
          pending.erase(it);
          break;
        }
    };
    if (need < 0 || (double)need > cfg.hbm_budget_bytes) {
      take();
      finish_job(jp, -1,
                 need < 0 ? std::string("invalid job: ") + spb_error_string()
                          : "job needs " + std::to_string(need) + " device bytes, more than the server's budget");
      return true;
    }
    bool no_room = false;
    Slot *s = acquire_slot(j.desc, need, &no_room);
    if (!s && no_room) continue;
    take();
    if (!s) {
      finish_job(jp, -1, g_err);
      return true;
    }
    j.slot = s;
    {
      std::lock_guard<std::mutex> lk(mu);
      j.t_admit = now();
    }
    if (start_job(j)) {
      finish_job(jp, -1, g_err);
      return true;
    }
    active.push_back(jp);
    std::lock_guard<std::mutex> lk(mu);
    if ((double)active.size() > stats[2]) stats[2] = (double)active.size();
    if ((double)held_bytes > stats[3]) stats[3] = (double)held_bytes;
    return true;
  }
  return false;
}

void spb_server::run() {
  cudaSetDevice(device);
  for (;;) {
    bool progress = false;
    while (admit_one()) progress = true;
    for (size_t i = 0; i < active.size();) {
      std::shared_ptr<Job> jp = active[i];
      Job &j = *jp;
      int err = 0;
      std::string msg;
      while (!j.inflight.empty()) {
        const cudaError_t q = cudaEventQuery(j.inflight.front());
        if (q == cudaErrorNotReady) break;
        if (q != cudaSuccess) {
          err = SPB_JOB_FAILED;
          msg = std::string("device error: ") + cudaGetErrorString(q);
          break;
        }
        const long long done_slots = j.inflight_slots.front();
        free_events.push_back(j.inflight.front());
        j.inflight.pop_front();
        j.inflight_slots.pop_front();
        progress = true;
        // the chunk's check has been copied back with it
        if (*j.slot->nf_host) {
          err = SPB_JOB_NONFINITE;
          msg = "a model holds NaN or infinite values after " + std::to_string(done_slots) + " iteration slots";
          break;
        }
      }
      if (!err) {
        bool cancel;
        {
          std::lock_guard<std::mutex> lk(mu);
          cancel = j.cancel;
        }
        if (cancel) {
          err = SPB_JOB_CANCELLED;
          msg = "cancelled";
        } else if (j.desc.time_budget_s > 0 && now() - j.t_submit > j.desc.time_budget_s) {
          err = SPB_JOB_EXPIRED;
          msg = "time budget of " + std::to_string(j.desc.time_budget_s) + " s ran out";
        }
      }
      while (!err && j.issued < j.slots && (int)j.inflight.size() < cfg.chunks_ahead) {
        const int r = issue_chunk(j);
        if (r < 0) {
          err = SPB_JOB_FAILED;
          msg = g_err;
        }
        if (r <= 0) break;
        progress = true;
      }
      if (!err && j.issued >= j.slots && j.inflight.empty()) {
        // results: per-start Fourier error and support fraction, models if kept
        SpPhaser *ph = j.slot->ph;
        const int nb = j.desc.starts;
        const size_t n = (size_t)j.desc.nx * j.desc.ny * j.desc.nz;
        j.efourier.assign((size_t)nb, 0.0f);
        j.sfrac.assign((size_t)nb, 0.0f);
        if (sp_phaser_starts_efourier(ph, j.efourier.data(), nullptr) ||
            sp_phaser_starts_support_fraction(ph, j.sfrac.data())) {
          err = SPB_JOB_FAILED;
          msg = std::string("results: ") + sp_phaser_last_error();
        } else if (j.desc.keep_models) {
          if (!j.slot->model_img) j.slot->model_img = sp_image_alloc(j.desc.nx, j.desc.ny, j.desc.nz);
          j.models.resize(2 * n * (size_t)nb);
          for (int b = 0; b < nb && !err; b++) {
            if (sp_phaser_start_model(ph, b, j.slot->model_img)) {
              err = SPB_JOB_FAILED;
              msg = std::string("model download: ") + sp_phaser_last_error();
            } else {
              memcpy(j.models.data() + 2 * n * (size_t)b, j.slot->model_img->image->data, sizeof(float) * 2 * n);
            }
          }
        }
        if (!err) {
          finish_job(jp, 0, "");
          active.erase(active.begin() + (long)i);
          progress = true;
          continue;
        }
      }
      if (err) {
        finish_job(jp, err, msg);
        active.erase(active.begin() + (long)i);
        progress = true;
        continue;
      }
      i++;
    }
    std::unique_lock<std::mutex> lk(mu);
    if (stop && pending.empty() && active.empty()) break;
    if (!progress) cv_work.wait_for(lk, std::chrono::microseconds(active.empty() ? 2000 : 40));
  }
}

// ------------------------------------------------------------------- C API
extern "C" const char *spb_server_last_error(void) { return g_err.c_str(); }

extern "C" int spb_server_create(spb_server **out, const spb_server_config *cfg) {
  *out = nullptr;
  int ndev = spb_device_count();
  if (ndev < 1) return fail("no CUDA device available for the reconstruction server");
  spb_server *s = new spb_server();
  if (cfg) s->cfg = *cfg;
  if (cudaGetDevice(&s->device) != cudaSuccess) s->device = 0;
  if (s->cfg.hbm_budget_bytes <= 0) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      delete s;
      return fail("cudaMemGetInfo failed");
    }
    s->cfg.hbm_budget_bytes = 0.6 * (double)fr;
  }
  if (s->cfg.max_active_jobs <= 0) s->cfg.max_active_jobs = 8;
  if (s->cfg.chunk_slots <= 0) s->cfg.chunk_slots = 100;
  if (s->cfg.chunks_ahead <= 0) s->cfg.chunks_ahead = 2;
  s->t0 = Clock::now();
  s->worker = std::thread([s]() { s->run(); });
  *out = s;
  return 0;
}

extern "C" void spb_server_destroy(spb_server *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  for (auto &sl : s->slots) destroy_slot_objects(sl);
  for (cudaEvent_t e : s->free_events) cudaEventDestroy(e);
  delete s;
}

extern "C" long long spb_server_submit(spb_server *s, const spb_job *job) {
  if (!s || !job) return fail("null server or job");
  if (job->nx < 1 || job->ny < 1 || job->nz < 1 || job->starts < 1)
    return fail("invalid job shape or start count");
  if (job->nstages < 1 || job->nstages > SPB_JOB_MAX_STAGES) return fail("a job has 1 to 4 stages");
  if (!job->amplitudes || !job->mask || !job->support) return fail("amplitudes, mask and support are required");
  auto j = std::make_shared<Job>();
  j->desc = *job;
  const size_t n = (size_t)job->nx * job->ny * job->nz;
  for (int i = 0; i < job->nstages; i++) {
    const int a = job->stage[i].algorithm;
    if (a != SpHIO && a != SpRAAR && a != SpDiffMap && a != SpER) return fail("unknown algorithm in a stage");
    if (job->stage[i].iterations < 0) return fail("negative iteration count");
    j->slots += job->stage[i].iterations;
  }
  j->amp.assign(job->amplitudes, job->amplitudes + n);
  j->mask.assign(job->mask, job->mask + n);
  j->support.assign(job->support, job->support + n);
  j->desc.amplitudes = nullptr;
  j->desc.mask = nullptr;
  j->desc.support = nullptr;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return fail("server is shutting down");
    j->id = s->next_id++;
    j->t_submit = s->now();
    s->jobs[j->id] = j;
    s->pending.push_back(j);
  }
  s->cv_work.notify_all();
  return j->id;
}

static void fill_info(const Job &j, spb_job_info *info) {
  if (!info) return;
  info->status = j.status;
  info->starts = j.desc.starts;
  info->slots = j.slots;
  info->t_submit = j.t_submit;
  info->t_admit = j.t_admit;
  info->t_finish = j.t_finish;
}

extern "C" int spb_server_wait(spb_server *s, long long id, double timeout_s, spb_job_info *info) {
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return fail("unknown job id " + std::to_string(id));
  std::shared_ptr<Job> j = it->second;
  auto done = [&]() { return j->status != 1; };
  if (timeout_s < 0) s->cv_done.wait(lk, done);
  else s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done);
  fill_info(*j, info);
  return 0;
}

extern "C" int spb_server_cancel(spb_server *s, long long id) {
  std::shared_ptr<Job> jp;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return fail("unknown job id " + std::to_string(id));
    jp = it->second;
    if (jp->status != SPB_JOB_RUNNING) return fail("job " + std::to_string(id) + " has already ended");
    for (auto p = s->pending.begin(); p != s->pending.end(); ++p)
      if (*p == jp) {  // not admitted yet: ends here
        s->pending.erase(p);
        jp->status = SPB_JOB_CANCELLED;
        jp->err = "cancelled";
        jp->t_finish = s->now();
        s->stats[7] += 1;
        s->cv_done.notify_all();
        return 0;
      }
    jp->cancel = true;  // running: the worker ends it at the next chunk boundary
  }
  s->cv_work.notify_all();
  return 0;
}

extern "C" int spb_server_result(spb_server *s, long long id, float *efourier, float *support_fraction,
                                 float *models) {
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return fail("unknown job id " + std::to_string(id));
  Job &j = *it->second;
  if (j.status == 1) return fail("job " + std::to_string(id) + " has not finished");
  if (j.status < 0) {
    const std::string msg = "job " + std::to_string(id) + " failed: " + j.err;
    s->jobs.erase(it);
    return fail(msg);
  }
  if (efourier) memcpy(efourier, j.efourier.data(), sizeof(float) * j.efourier.size());
  if (support_fraction) memcpy(support_fraction, j.sfrac.data(), sizeof(float) * j.sfrac.size());
  if (models) {
    if (!j.desc.keep_models) return fail("job " + std::to_string(id) + " did not keep its models");
    memcpy(models, j.models.data(), sizeof(float) * j.models.size());
  }
  s->jobs.erase(it);
  return 0;
}

extern "C" int spb_server_stats(spb_server *s, double stats[8]) {
  std::lock_guard<std::mutex> lk(s->mu);
  for (int k = 0; k < 8; k++) stats[k] = s->stats[k];
  return 0;
}

extern "C" const char *spb_server_job_error(spb_server *s, long long id) {
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return "unknown job";
  static thread_local std::string copy;
  copy = it->second->err;
  return copy.c_str();
}
