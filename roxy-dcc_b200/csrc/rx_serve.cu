// Serving loop: render requests of different scenes, resolutions and spp
// admitted as they arrive, with continuous batching.
//
// The reference renders one TaichiRenderer.render() call at a time
// (rendering/taichi_renderer.py:87-191).  Here a host thread owned by the
// server repeats steps: admit queued requests while active slots and the
// device-memory budget allow (a request's accumulator plus, on its scene's
// first use, the scene's BVH and arrays), give every newly admitted request
// its preview frames, spend the rest of the step's path budget on
// refinement frames of the requests admitted earlier, and trace all of it as
// one batch of shared wavefronts.  Requests arriving during a step join the
// next one.  A request's random numbers and frame order are those of a
// render of its own, so its image does not depend on what it was served
// with.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>
#include <vector>

#include "rx_internal.cuh"
#include "rx_runtime.h"

namespace rx {

struct Request {
  int id = -1;
  Scene* sc = nullptr;
  rx_render_params p{};
  int frames = 0, done = 0;
  Accum* acc = nullptr;
  long long bytes = 0;      // accumulator bytes charged at admission
  int state = RX_REQ_QUEUED;
  double t_submit = 0.0, t_admit = -1.0, t_preview = -1.0, t_final = -1.0;
};

struct Server {
  Ctx* ctx = nullptr;
  rx_serve_config cfg{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<int> queue;
  std::vector<int> active;
  std::unordered_map<int, Request> reqs;
  std::unordered_map<Scene*, int> scene_refs;
  long long used = 0, max_used = 0;
  int next_id = 0, max_active_seen = 0;
  long long steps = 0, admitted = 0, completed = 0, failed = 0;
  double busy_s = 0.0;
  bool stop = false;
  Batch* batch = nullptr;
  std::thread th;
  std::chrono::steady_clock::time_point t0;
  std::string last_err;

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

// bytes of a W x H accumulator: four float4 buffers plus counters
static long long accum_need(const rx_render_params& p) { return (long long)p.width * p.height * 64 + 64; }

// bytes of a wave of `paths` paths: seven float4 + three int arrays per path,
// shadow records for one ray per path
static long long wave_need(long long paths) { return paths * (7 * 16 + 3 * 4 + 48); }

static void release_locked(Server* S, Request& r) {
  S->used -= r.bytes;
  r.bytes = 0;
  auto it = S->scene_refs.find(r.sc);
  if (it != S->scene_refs.end() && --it->second == 0) {
    S->used -= (long long)scene_bytes(r.sc);
    S->scene_refs.erase(it);
  }
}

static void serve_loop(Server* S) {
  struct Step {
    int id;
    int frames;
    bool fresh;
  };
  for (;;) {
    std::vector<Step> plan;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_work.wait(lk, [&] { return S->stop || !S->queue.empty() || !S->active.empty(); });
      if (S->stop) return;
      // admission: FIFO while a slot and the memory budget allow
      while (!S->queue.empty() && (int)S->active.size() < S->cfg.max_active) {
        Request& r = S->reqs[S->queue.front()];
        long long need = accum_need(r.p);
        long long scene_new = S->scene_refs.count(r.sc) ? 0 : (long long)scene_bytes(r.sc);
        if (S->used + need + scene_new > S->cfg.hbm_budget) break;
        S->queue.pop_front();
        r.state = RX_REQ_ACTIVE;
        r.t_admit = S->now();
        r.bytes = need;
        S->used += need + scene_new;
        S->scene_refs[r.sc] += 1;
        S->active.push_back(r.id);
        ++S->admitted;
      }
      S->max_used = std::max(S->max_used, S->used);
      S->max_active_seen = std::max(S->max_active_seen, (int)S->active.size());
      // previews of newly admitted requests first, then refinement of the
      // others in admission order within the step's path budget
      long long left = S->cfg.step_paths;
      for (int id : S->active) {
        Request& r = S->reqs[id];
        if (r.done == 0) {
          int f = std::min(r.frames, std::max(S->cfg.preview_frames, 1));
          plan.push_back(Step{id, f, true});
          left -= (long long)f * r.p.width * r.p.height;
        }
      }
      for (int id : S->active) {
        Request& r = S->reqs[id];
        if (r.done == 0 || r.done >= r.frames) continue;
        long long P = (long long)r.p.width * r.p.height;
        if (left < P && !plan.empty()) break;
        int f = (int)std::min<long long>(r.frames - r.done, std::max<long long>(1, left / P));
        plan.push_back(Step{id, f, false});
        left -= (long long)f * P;
      }
    }
    if (plan.empty()) {
      // queued requests wait for memory held by finished, unreleased ones
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_work.wait_for(lk, std::chrono::milliseconds(5));
      continue;
    }
    // device work: the context lock, not the server lock, is held.  A
    // thread waiting in rx_ctx_hold (building a request's scene, say) goes
    // first: the mutex is not fair, and this loop would otherwise re-take
    // it step after step (bounded: at most ~0.5 s of 50-us yields).
    for (int k = 0; k < 10000 && S->ctx->hold_waiters.load() > 0; ++k)
      std::this_thread::sleep_for(std::chrono::microseconds(50));
    std::vector<int> ok(plan.size(), 1);
    int rc = RX_OK;
    double t_start = S->now();
    {
      std::lock_guard<std::recursive_mutex> g(S->ctx->mu);
      cudaSetDevice(S->ctx->device);
      batch_clear(S->batch);
      int n_jobs = 0;
      for (size_t k = 0; k < plan.size(); ++k) {
        Request* r;
        {
          std::lock_guard<std::mutex> lk(S->mu);
          r = &S->reqs[plan[k].id];
        }
        if (!r->acc) {
          r->acc = accum_new(S->ctx, r->p.width, r->p.height);
          if (!r->acc) {
            ok[k] = 0;
            continue;
          }
        }
        int job = -1;
        if (batch_add(S->batch, r->sc, r->acc, &r->p, plan[k].frames, &job) != RX_OK) {
          ok[k] = 0;
          continue;
        }
        ++n_jobs;
      }
      if (n_jobs > 0) rc = batch_render(S->batch);
    }
    double t_end = S->now();
    {
      std::lock_guard<std::mutex> lk(S->mu);
      ++S->steps;
      S->busy_s += t_end - t_start;
      if (rc != RX_OK) S->last_err = S->ctx->err;
      for (size_t k = 0; k < plan.size(); ++k) {
        Request& r = S->reqs[plan[k].id];
        if (!ok[k] || rc != RX_OK) {
          r.state = RX_REQ_FAILED;
          ++S->failed;
        } else {
          r.done += plan[k].frames;
          if (r.t_preview < 0.0) r.t_preview = t_end;
          if (r.done >= r.frames) {
            r.state = RX_REQ_DONE;
            r.t_final = t_end;
            ++S->completed;
          }
        }
        if (r.state == RX_REQ_DONE || r.state == RX_REQ_FAILED)
          S->active.erase(std::remove(S->active.begin(), S->active.end(), r.id), S->active.end());
      }
    }
    S->cv_done.notify_all();
  }
}

Server* serve_new(Ctx* ctx, const rx_serve_config* cfg) {
  Server* S = new Server();
  S->ctx = ctx;
  S->cfg = *cfg;
  S->t0 = std::chrono::steady_clock::now();
  S->batch = batch_new(ctx);
  batch_use_graph(S->batch, false);
  batch_set_config(S->batch, cfg->wave_paths, cfg->extend_block);
  // the shared wave state is reserved up front and allocated now, so the
  // first requests do not wait for it
  long long cap = std::min(cfg->wave_paths, std::max(cfg->step_paths, (long long)1));
  S->used = wave_need(cap);
  S->max_used = S->used;
  {
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    batch_reserve(S->batch, cap);
    // map memory into the stream-ordered pool now (the context keeps freed
    // pool memory), so admitting many requests later allocates accumulators
    // from memory that is already mapped
    long long warm = std::min(cfg->pool_prewarm, cfg->hbm_budget - S->used);
    if (warm > 0) {
      void* p = nullptr;
      if (cudaMallocAsync(&p, (size_t)warm, ctx->stream) == cudaSuccess) cudaFreeAsync(p, ctx->stream);
      else cudaGetLastError();
      cudaStreamSynchronize(ctx->stream);
    }
  }
  S->th = std::thread(serve_loop, S);
  return S;
}

void serve_delete(Server* S) {
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  if (S->th.joinable()) S->th.join();
  std::lock_guard<std::recursive_mutex> g(S->ctx->mu);
  cudaStreamSynchronize(S->ctx->stream);
  for (auto& kv : S->reqs)
    if (kv.second.acc) accum_delete(kv.second.acc);
  batch_delete(S->batch);
  delete S;
}

int serve_submit(Server* S, Scene* sc, const rx_render_params* p, int frames, int* id) {
  Ctx* ctx = S->ctx;
  if (!sc || !p || frames < 1 || p->width <= 0 || p->height <= 0)
    return set_error(ctx, "serve_submit: bad arguments"), RX_ERR_ARG;
  if (p->max_depth < 0 || p->max_depth > 63) return set_error(ctx, "serve_submit: max_depth out of range"), RX_ERR_ARG;
  if (p->direct_light_mode != 0 && p->direct_light_mode != 1)
    return set_error(ctx, "direct_light_mode must be 'one' or 'all'"), RX_ERR_ARG;
  if (sc->n_tris > 0 && sc->n_nodes == 0) return set_error(ctx, "serve_submit: scene has no BVH"), RX_ERR_STATE;
  std::lock_guard<std::mutex> lk(S->mu);
  long long base = wave_need(std::min(S->cfg.wave_paths, std::max(S->cfg.step_paths, (long long)1)));
  if (base + accum_need(*p) + (long long)scene_bytes(sc) > S->cfg.hbm_budget)
    return set_error(ctx, "serve_submit: the request alone exceeds the %lld-byte budget", S->cfg.hbm_budget),
           RX_ERR_CAPACITY;
  Request r;
  r.id = S->next_id++;
  r.sc = sc;
  r.p = *p;
  r.frames = frames;
  r.t_submit = S->now();
  S->reqs[r.id] = r;
  S->queue.push_back(r.id);
  *id = r.id;
  S->cv_work.notify_one();
  return RX_OK;
}

int serve_info(Server* S, int id, rx_request_info* out) {
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return set_error(S->ctx, "serve_info: unknown request %d", id), RX_ERR_ARG;
  const Request& r = it->second;
  out->state = r.state;
  out->frames_done = r.done;
  out->frames = r.frames;
  out->t_submit = r.t_submit;
  out->t_admit = r.t_admit;
  out->t_preview = r.t_preview;
  out->t_final = r.t_final;
  out->bytes = r.bytes;
  return RX_OK;
}

int serve_wait(Server* S, int id, int until_final, double timeout_s) {
  std::unique_lock<std::mutex> lk(S->mu);
  auto pred = [&] {
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return true;
    const Request& r = it->second;
    if (r.state == RX_REQ_DONE || r.state == RX_REQ_FAILED) return true;
    return !until_final && r.done > 0;
  };
  if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred))
    return set_error(S->ctx, "serve_wait: request %d not ready after %.3f s", id, timeout_s), RX_ERR_TIMEOUT;
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return set_error(S->ctx, "serve_wait: unknown request %d", id), RX_ERR_ARG;
  if (it->second.state == RX_REQ_FAILED)
    return set_error(S->ctx, "request %d failed: %s", id, S->last_err.c_str()), RX_ERR_STATE;
  return RX_OK;
}

int serve_read(Server* S, int id, int which, float* host_out) {
  Accum* acc = nullptr;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return set_error(S->ctx, "serve_read: unknown request %d", id), RX_ERR_ARG;
    if (it->second.done == 0 || !it->second.acc)
      return set_error(S->ctx, "serve_read: request %d has no frames yet", id), RX_ERR_STATE;
    acc = it->second.acc;
  }
  // the server thread holds the context lock while a step runs: a read
  // sees the state after the last finished step
  std::lock_guard<std::recursive_mutex> g(S->ctx->mu);
  cudaSetDevice(S->ctx->device);
  return accum_read(acc, which, host_out);
}

int serve_release(Server* S, int id) {
  Accum* acc = nullptr;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return set_error(S->ctx, "serve_release: unknown request %d", id), RX_ERR_ARG;
    Request& r = it->second;
    if (r.state == RX_REQ_QUEUED || r.state == RX_REQ_ACTIVE)
      return set_error(S->ctx, "serve_release: request %d is still being served", id), RX_ERR_STATE;
    if (r.t_admit >= 0.0) release_locked(S, r);
    acc = r.acc;
    S->reqs.erase(it);
  }
  if (acc) {
    std::lock_guard<std::recursive_mutex> g(S->ctx->mu);
    cudaSetDevice(S->ctx->device);
    accum_delete(acc);
  }
  S->cv_work.notify_one();
  return RX_OK;
}

int serve_stats(Server* S, rx_serve_stats* out) {
  std::lock_guard<std::mutex> lk(S->mu);
  out->steps = S->steps;
  out->admitted = S->admitted;
  out->completed = S->completed;
  out->failed = S->failed;
  out->active = (int)S->active.size();
  out->queued = (int)S->queue.size();
  out->max_active_seen = S->max_active_seen;
  out->bytes_in_use = S->used;
  out->max_bytes_in_use = S->max_used;
  out->busy_s = S->busy_s;
  out->uptime_s = S->now();
  return RX_OK;
}

}  // namespace rx
