// Serving loop: tilt series arrive as requests, are admitted against a device
// memory budget, prepared (upload, pre-processing, coarse alignment) and then
// projection-matched in groups of series of any shapes (continuous batching).
//
// The reference aligns exactly one series per process run (Markerfree/src/main/
// Process.cpp:34-92).  Here a pool of worker threads, each with its own stream
// (mf_context), takes tasks from one scheduler function:
//   * admission: queued requests become admitted while the estimated device
//     bytes of all admitted requests stay within the budget;
//   * prepare: an admitted request is uploaded, pre-processed and coarse-aligned
//     (PreProcess, Transform, CalcTIltAxis, FindOffset) on the worker's stream;
//   * match: prepared requests that share the options a group applies to all its
//     series (precision, -p, z shift) are taken together as a group -- of any
//     image sizes, tilt counts and slab thicknesses -- (up to max_group, or fewer
//     when no more such requests are on their way, or when the oldest has waited
//     group_wait_ms) and run through projection matching, the aligned-stack
//     correction and the parameter read-out.
// Work of different workers overlaps on the GPU; a request that arrives while
// others run is admitted as soon as memory frees up.  Each request's result is
// the one it gets when aligned alone (groups keep per-series arithmetic).
//
// The byte estimate does not see everything a worker holds (cuFFT plans, the
// operators of a group's distinct geometries, blocks cached by the stream-ordered
// pool).  When a prepare or a group set-up still finds the device full while
// other requests hold memory, the request is not failed: what it allocated is
// given back, it returns to the head of its queue, the budget drops to what the
// other requests hold (so the scheduler learns where the device really fills),
// and a group that failed is retried at half the size (the size doubles back
// with every group that goes through).  Only a request that
// finds the device full with nothing else on it fails.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>

#include "mf_series.hpp"

using namespace mf;

namespace {

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

enum JobState { kQueued, kAdmitted, kPreparing, kReady, kMatching, kDone };

struct Job {
  int64_t id = 0;
  int nx = 0, ny = 0, nz = 0;
  std::vector<float> angles;
  const float* raw = nullptr;  // caller-owned until the job is done
  float* out = nullptr;        // optional caller-owned aligned stack
  mf_options opt{};
  size_t bytes = 0;
  JobState state = kQueued;
  int rc = MF_OK;
  std::string err;
  mf_series* s = nullptr;
  std::vector<float> sx, sy, rot;
  float angle_offset = 0.0f;
  int passes = 0;
  int64_t mem_wait = -1;  // finished-job count when a group set-up ran out of memory
  double t_submit = 0, t_admit = 0, t_ready = 0, t_done = 0;
};

// Return the blocks the stream-ordered pool caches to the device, once this
// worker's own work has drained.
void return_cached_memory(int gpu, cudaStream_t st) {
  cudaStreamSynchronize(st);
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, gpu) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
  cudaGetLastError();
}

// The device's memory state, appended to an out-of-memory failure.
std::string memory_report(int gpu) {
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  uint64_t reserved = 0, in_use = 0;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, gpu) == cudaSuccess) {
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &in_use);
  }
  cudaGetLastError();
  char b[200];
  snprintf(b, sizeof(b), " [device: %.2f GB free of %.2f; pool %.2f GB reserved, %.2f in use]",
           fr / 1e9, tot / 1e9, reserved / 1e9, in_use / 1e9);
  return b;
}

// Requests that may share a group: the same options of the projection-matching
// stage that a group applies to all its series (any image size, tilt count and
// slab thickness may mix).
std::vector<float> group_key(const Job* j) {
  return {(float)j->opt.precision, (float)(j->opt.align_z != 0), (float)j->opt.nproj,
          j->opt.zshift};
}

// Device bytes a request may hold at its peak: the pre-processed stack, the
// matching buffers (corrected stack, row-FFT scratch, 16-bit copy, operators)
// and a device copy of the aligned output.
size_t estimate_bytes(int nx, int ny, int nz, const mf_options& o) {
  const int bin = std::max(1, std::max((int)((float)nx / 2048.0f + 0.5f),
                                       (int)((float)ny / 2048.0f + 0.5f)));
  const size_t xb = nx / bin / 2 * 2, yb = ny / bin / 2 * 2;
  const size_t stack = (size_t)4 * nx * ny * nz;
  const size_t xo = nx / std::max(1, o.out_bin) / 2 * 2, yo = ny / std::max(1, o.out_bin) / 2 * 2;
  // the stack and its column-major copy (tilt-axis search), the binned working
  // stacks of projection matching, the aligned output and fixed scratch
  return 2 * stack + (size_t)16 * xb * yb * nz + (size_t)4 * xo * yo * nz + ((size_t)64 << 20);
}

}  // namespace

struct mf_server {
  int gpu = 0;
  size_t budget0 = 0, budget = 0, used = 0, peak_used = 0;
  int max_group = 8;
  int group_cap = kMaxGroup;  // lowered when a group set-up runs out of memory
  int64_t done_count = 0, mem_retries = 0;
  double group_wait_s = 0.05;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::map<int64_t, std::unique_ptr<Job>> jobs;
  std::deque<Job*> queued;
  std::vector<Job*> admitted;  // waiting for a prepare task
  std::vector<Job*> ready;     // prepared, waiting for a group
  int preparing = 0;
  int matching = 0;  // groups being matched
  int64_t next_id = 1;
  bool stop = false;
  std::vector<mf_context*> ctxs;
  std::vector<std::thread> threads;
  // statistics
  double first_submit = -1, last_done = -1;
  std::vector<double> latencies;
  int64_t groups = 0, grouped_jobs = 0;

  void admit_locked() {
    while (!queued.empty()) {
      Job* j = queued.front();
      if (used + j->bytes > budget && used > 0) break;  // always admit into an empty device
      queued.pop_front();
      used += j->bytes;
      peak_used = std::max(peak_used, used);
      j->state = kAdmitted;
      j->t_admit = now_s();
      admitted.push_back(j);
    }
  }

  // Next task for a worker: a group of ready jobs, or one job to prepare, or
  // nothing (with the time to wait before asking again).
  bool next_task_locked(std::vector<Job*>* group, Job** prep, double* wait_s) {
    admit_locked();
    *prep = nullptr;
    group->clear();
    *wait_s = 0.25;
    const double t = now_s();
    // ready jobs grouped by the options a group shares, oldest first
    // (a job whose group ran out of memory waits for some job to finish, or for
    // the device to go idle)
    const bool idle = preparing == 0 && matching == 0;
    std::map<std::vector<float>, std::vector<Job*>> by_shape;
    for (Job* j : ready)
      if (j->mem_wait != done_count || idle) by_shape[group_key(j)].push_back(j);
    auto coming = [&](const std::vector<float>& key) {
      for (Job* j : admitted)
        if (group_key(j) == key) return true;
      for (Job* j : queued)
        if (group_key(j) == key) return true;
      return preparing > 0;
    };
    auto take = [&](std::vector<Job*>& v) {
      const int m = std::min((int)v.size(), std::min(max_group, group_cap));
      group->assign(v.begin(), v.begin() + m);
      for (Job* j : *group) {
        j->state = kMatching;
        ready.erase(std::find(ready.begin(), ready.end(), j));
      }
      matching++;
      return true;
    };
    for (auto& kv : by_shape)
      std::sort(kv.second.begin(), kv.second.end(),
                [](Job* a, Job* b) { return a->t_ready < b->t_ready; });
    // 1. a full group, or one whose oldest job has waited too long, runs first
    const double starve_s = 20.0 * group_wait_s;
    for (auto& kv : by_shape)
      if ((int)kv.second.size() >= std::min(max_group, group_cap) ||
          t - kv.second.front()->t_ready >= starve_s)
        return take(kv.second);
    // 2. preparing admitted jobs comes next: it lets more jobs join the
    //    ready groups, so the matching that follows runs on larger groups
    if (!admitted.empty()) {
      *prep = admitted.front();
      admitted.erase(admitted.begin());
      (*prep)->state = kPreparing;
      preparing++;
      return true;
    }
    // 3. with nothing to prepare, a group runs once it has waited the grouping
    //    window or no job of its kind is on the way
    for (auto& kv : by_shape) {
      std::vector<Job*>& v = kv.second;
      const bool waited = t - v.front()->t_ready >= group_wait_s;
      if (waited || !coming(kv.first)) return take(v);
      *wait_s = std::min(*wait_s, std::max(1e-3, group_wait_s - (t - v.front()->t_ready)));
    }
    return false;
  }

  void finish_locked(Job* j, int rc) {
    j->rc = rc;
    if (rc != MF_OK) j->err = mf_last_error();
    if (rc == MF_ERR_NOMEM) {
      char b[160];
      snprintf(b, sizeof(b), " [server: %.2f GB admitted of a %.2f GB budget (%.2f as created)]",
               used / 1e9, budget / 1e9, budget0 / 1e9);
      j->err += b + memory_report(gpu);
    }
    if (j->s) {
      mf_series_destroy(j->s);
      j->s = nullptr;
    }
    j->state = kDone;
    j->t_done = now_s();
    used -= j->bytes;
    done_count++;
    last_done = j->t_done;
    latencies.push_back(j->t_done - j->t_submit);
  }

  void worker(int w) {
    mf_context* ctx = ctxs[w];
    cudaSetDevice(gpu);
    set_alloc_stream(ctx->c.stream);
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
      std::vector<Job*> group;
      Job* prep = nullptr;
      double wait_s = 0.0;
      if (!next_task_locked(&group, &prep, &wait_s)) {
        if (stop && queued.empty() && admitted.empty() && ready.empty() && preparing == 0) break;
        cv_work.wait_for(lk, std::chrono::duration<double>(wait_s));
        continue;
      }
      lk.unlock();
      if (prep) {
        int rc = MF_OK;
        for (int attempt = 0; attempt < 2; ++attempt) {
          rc = mf_series_create(ctx, prep->raw, prep->nx, prep->ny, prep->nz,
                                prep->angles.data(), &prep->s);
          if (rc == MF_OK) {
            prep->s->precision = (mf_precision)prep->opt.precision;
            if (prep->opt.align_z != 0)
              rc = coarse_align(prep->s, prep->opt.pitch_angle, prep->opt.offset);
          }
          if (rc == MF_OK && cudaStreamSynchronize(ctx->c.stream) != cudaSuccess)
            rc = set_error(MF_ERR_CUDA, "stream synchronize failed");
          if (rc != MF_ERR_NOMEM) break;
          // give back what it holds and what the pool caches; with no other request
          // holding memory, try once more before failing
          mf_series_destroy(prep->s);
          prep->s = nullptr;
          return_cached_memory(gpu, ctx->c.stream);
          bool alone;
          {
            std::lock_guard<std::mutex> g(mu);
            alone = used <= prep->bytes;
          }
          if (!alone) break;
        }
        lk.lock();
        preparing--;
        if (rc == MF_OK) {
          prep->state = kReady;
          prep->t_ready = now_s();
          ready.push_back(prep);
        } else if (rc == MF_ERR_NOMEM && used > prep->bytes) {
          // the others hold the memory it needs: back to the head of the queue,
          // admitted again once enough of them have finished
          used -= prep->bytes;
          budget = std::min(budget, used);
          prep->state = kQueued;
          queued.push_front(prep);
          mem_retries++;
        } else {
          finish_locked(prep, rc);
          cv_done.notify_all();
        }
        cv_work.notify_all();
        continue;
      }
      // match a group on this worker's stream; the series move to this context
      int rc = MF_OK;
      std::vector<mf_series*> ss;
      for (Job* j : group) {
        j->s->ctx = ctx;
        ss.push_back(j->s);
      }
      const mf_options& o = group[0]->opt;
      std::vector<int> passes(group.size(), 0), align_z;
      for (Job* j : group) align_z.push_back(j->opt.align_z);
      if (o.align_z != 0) {
        mf_group* g = nullptr;
        rc = group_create(ctx, ss.data(), (int)ss.size(), o.zshift, align_z.data(), o.nproj, &g);
        if (rc == MF_ERR_NOMEM) {
          // set-up allocates everything before any series changes: nothing to undo
          mf_group_destroy(g);  // defined where mf_group is complete
          return_cached_memory(gpu, ctx->c.stream);
          lk.lock();
          size_t gb = 0;
          for (Job* j : group) gb += j->bytes;
          // others that will give memory back: requests being prepared or matched
          const bool others = preparing > 0 || matching > 1;
          if (others || group.size() > 1) {
            if (group.size() > 1) group_cap = std::max(1, (int)group.size() / 2);
            if (used > gb) budget = std::min(budget, used);
            for (Job* j : group) {
              j->state = kReady;
              j->mem_wait = others ? done_count : -1;
              ready.push_back(j);
            }
            matching--;
            mem_retries++;
            cv_work.notify_all();
            continue;
          }
          lk.unlock();
        } else if (rc == MF_OK) {
          rc = group_proj_align(g, passes.data());
          mf_group_destroy(g);  // defined where mf_group is complete
        }
      }
      std::vector<int> rcs(group.size(), rc);
      for (size_t i = 0; i < group.size(); ++i) {
        Job* j = group[i];
        if (rcs[i] == MF_OK && j->out) rcs[i] = mf_correct_stack(j->s, j->opt.out_bin, j->out);
        if (rcs[i] == MF_OK) {
          j->sx = j->s->sx;
          j->sy = j->s->sy;
          j->rot = j->s->rot;
          j->angle_offset = j->s->angle_offset;
          j->passes = passes[i];
        }
      }
      if (cudaStreamSynchronize(ctx->c.stream) != cudaSuccess && rc == MF_OK)
        for (int& r : rcs) r = set_error(MF_ERR_CUDA, "stream synchronize failed");
      lk.lock();
      matching--;
      // a group that went through lets the group size grow back after a shortage
      if (rc == MF_OK && group_cap < kMaxGroup) group_cap = std::min(kMaxGroup, 2 * group_cap);
      groups++;
      grouped_jobs += (int64_t)group.size();
      for (size_t i = 0; i < group.size(); ++i) finish_locked(group[i], rcs[i]);
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }
};

extern "C" {

MF_API int mf_server_create(int gpu, size_t hbm_budget, int max_group, int workers,
                            double group_wait_ms, mf_server** out) {
  if (!out) return set_error(MF_ERR_ARG, "null output pointer");
  *out = nullptr;
  if (max_group < 1 || max_group > kMaxGroup)
    return set_error(MF_ERR_ARG, "max_group must be 1..%d", kMaxGroup);
  if (workers < 1 || workers > 16) return set_error(MF_ERR_ARG, "workers must be 1..16");
  MF_CHECK_CUDA(cudaSetDevice(gpu));
  if (hbm_budget == 0) {
    // 65 % of the free memory once the pool's cached blocks are returned: the rest
    // is left to what the estimate does not count (cuFFT plans and work areas,
    // which cuFFT allocates outside the pool for every shape each worker meets,
    // the coarse stages' transient buffers of the requests being prepared, and
    // group working sets of mixed shapes)
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, gpu) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    size_t fr = 0, tot = 0;
    MF_CHECK_CUDA(cudaMemGetInfo(&fr, &tot));
    hbm_budget = fr / 100 * 65;
  }
  std::unique_ptr<mf_server> s(new mf_server());
  s->gpu = gpu;
  s->budget0 = s->budget = hbm_budget;
  s->max_group = max_group;
  s->group_wait_s = group_wait_ms / 1000.0;
  for (int w = 0; w < workers; ++w) {
    mf_context* c = nullptr;
    int rc = mf_context_create(gpu, &c);
    if (rc != MF_OK) {
      for (mf_context* x : s->ctxs) mf_context_destroy(x);
      return rc;
    }
    s->ctxs.push_back(c);
  }
  for (int w = 0; w < workers; ++w) s->threads.emplace_back(&mf_server::worker, s.get(), w);
  *out = s.release();
  return MF_OK;
}

MF_API int mf_server_submit(mf_server* s, const float* raw, int nx, int ny, int nz,
                            const float* file_angles, const mf_options* opt, float* aligned_out,
                            int64_t* job_id) {
  if (!s || !raw || !file_angles || !opt || !job_id) return set_error(MF_ERR_ARG, "null argument");
  if (nx < 8 || ny < 8 || nz < 2)
    return set_error(MF_ERR_ARG, "stack %d x %d x %d too small (need >= 8 x 8 x 2)", nx, ny, nz);
  if (opt->nproj <= 0) return set_error(MF_ERR_ARG, "nProj must be > 0.");
  if (opt->out_bin < 1) return set_error(MF_ERR_ARG, "output binning must be >= 1");
  if (opt->precision != MF_PREC_FP32 && opt->precision != MF_PREC_BF16 &&
      opt->precision != MF_PREC_FP16)
    return set_error(MF_ERR_ARG, "unknown precision %d", opt->precision);
  std::unique_ptr<Job> j(new Job());
  j->nx = nx;
  j->ny = ny;
  j->nz = nz;
  j->angles.assign(file_angles, file_angles + nz);
  j->raw = raw;
  j->out = aligned_out;
  j->opt = *opt;
  j->bytes = estimate_bytes(nx, ny, nz, *opt);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return set_error(MF_ERR_STATE, "server is shutting down");
    if (j->bytes > s->budget0)
      return set_error(MF_ERR_NOMEM, "request needs about %zu bytes, budget is %zu", j->bytes,
                       s->budget0);
    j->id = s->next_id++;
    j->t_submit = now_s();
    if (s->first_submit < 0) s->first_submit = j->t_submit;
    *job_id = j->id;
    s->queued.push_back(j.get());
    s->jobs[j->id] = std::move(j);
    s->admit_locked();  // admitted now if it fits, not only when a worker asks
  }
  s->cv_work.notify_all();
  return MF_OK;
}

MF_API int mf_server_wait(mf_server* s, int64_t job_id, double timeout_s, mf_align_param* param,
                          int* passes, double* latency_s) {
  if (!s) return set_error(MF_ERR_ARG, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->jobs.find(job_id);
  if (it == s->jobs.end()) return set_error(MF_ERR_ARG, "unknown job %lld", (long long)job_id);
  Job* j = it->second.get();
  const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                      [&] { return j->state == kDone; });
  if (!ok) return set_error(MF_ERR_STATE, "job %lld not finished", (long long)job_id);
  if (j->rc != MF_OK) return set_error(j->rc, "job %lld: %s", (long long)job_id, j->err.c_str());
  if (param) {
    if (!param->shift_x || !param->shift_y || !param->rotate)
      return set_error(MF_ERR_ARG, "null parameter arrays");
    memcpy(param->shift_x, j->sx.data(), sizeof(float) * j->nz);
    memcpy(param->shift_y, j->sy.data(), sizeof(float) * j->nz);
    memcpy(param->rotate, j->rot.data(), sizeof(float) * j->nz);
    param->angle_offset = j->angle_offset;
  }
  if (passes) *passes = j->passes;
  if (latency_s) *latency_s = j->t_done - j->t_submit;
  return MF_OK;
}

MF_API int mf_server_stats(mf_server* s, double* out8) {
  if (!s || !out8) return set_error(MF_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  std::vector<double> l = s->latencies;
  std::sort(l.begin(), l.end());
  auto pct = [&](double q) {
    if (l.empty()) return 0.0;
    size_t i = (size_t)std::min((double)l.size() - 1, std::ceil(q * l.size()) - 1);
    return l[i];
  };
  const double span = (s->last_done > s->first_submit) ? s->last_done - s->first_submit : 0.0;
  out8[0] = (double)l.size();
  out8[1] = span > 0 ? 60.0 * (double)l.size() / span : 0.0;
  out8[2] = pct(0.50);
  out8[3] = pct(0.99);
  out8[4] = (double)s->peak_used;
  out8[5] = (double)s->groups;
  out8[6] = s->groups ? (double)s->grouped_jobs / (double)s->groups : 0.0;
  out8[7] = span;
  return MF_OK;
}

MF_API int mf_server_memory(mf_server* s, size_t* budget0, size_t* budget_now,
                            int64_t* retries) {
  if (!s) return set_error(MF_ERR_ARG, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  if (budget0) *budget0 = s->budget0;
  if (budget_now) *budget_now = s->budget;
  if (retries) *retries = s->mem_retries;
  return MF_OK;
}

MF_API void mf_server_destroy(mf_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (std::thread& t : s->threads) t.join();
  for (mf_context* c : s->ctxs) mf_context_destroy(c);
  delete s;
}

}  // extern "C"
