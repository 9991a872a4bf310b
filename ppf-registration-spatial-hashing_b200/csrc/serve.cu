// Request loop over a resident model library.
//
// A registration request is one scene (host points and normals, copied at
// submission) and the library models to register it against.  Worker threads,
// each with its own context (stream and workspace), take queued requests in
// arrival order and admit them while their estimated device memory fits the
// server's budget; the admitted requests of one worker form a batch whose
// (scene, model) pairs share one batched vote pass (lookup_batch), followed by
// threshold, poses and clustering per pair.  Batches of different workers run
// on different streams, so a request that arrives while others are on the GPU
// is admitted as soon as memory frees and its work overlaps theirs.  Each
// pair has its own lookup state, so a request's result does not depend on
// the requests around it.  There is no counterpart in the reference, whose
// ppf_registration (src/cuda/ppf.cu:29-106) rebuilds every model per call.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>

#include "engine.h"

namespace ppf {

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t ticket = 0;
  std::vector<float> xyz, nxyz;
  uint64_t n = 0;
  uint32_t ref_df = 1;
  std::vector<uint32_t> targets;
  size_t need = 0;  // estimated device bytes while in flight
  Clock::time_point t_submit, t_done;
  // results
  bool done = false;
  ppf_status status = PPF_OK;
  std::string error;
  std::vector<float> poses;
  std::vector<ppf_stats> stats;
};

}  // namespace

struct Server {
  int device = 0;
  std::vector<Model*> models;        // borrowed library
  std::vector<size_t> hints;         // candidate cells of each model's last pass
  size_t budget = 0, in_use = 0;
  uint32_t max_batch = 16;
  std::vector<std::unique_ptr<ppf_context_s>> ctxs;
  std::vector<std::thread> threads;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> queue;
  std::map<uint64_t, std::shared_ptr<Request>> tickets;
  uint64_t next_ticket = 1;
  bool stop = false;

  // Device bytes a request holds while in flight, per target model: the
  // scene as float4 points and normals, and for the expected candidate count
  // c its candidate cells (12 B each, with 25% headroom) and its lookup state
  // (kept votes, about c / 2, at ~230 B each).
  size_t need_bytes(const Request& r) const {
    size_t b = 0;
    for (uint32_t j : r.targets) {
      const size_t c = std::max<size_t>(hints[j], size_t(1) << 20);
      b += 32 * r.n + 15 * c + 115 * c;
    }
    return b;
  }

  void run_batch(Context& ctx, std::vector<std::shared_ptr<Request>>& batch) {
    PPF_CUDA(cudaSetDevice(ctx.device));
    StreamScope scope(ctx.stream);
    std::vector<std::unique_ptr<SceneData>> scenes;
    std::vector<Model*> ms;
    std::vector<const SceneData*> ss;
    std::vector<size_t> caps;
    for (auto& r : batch)
      for (uint32_t j : r->targets) {
        std::unique_ptr<SceneData> s(new SceneData());
        s->n = (uint32_t)r->n;
        s->d_dist = models[j]->t.d_dist;  // each scene takes its model's quantum
        s->ref_df = r->ref_df;
        upload_points(ctx, r->xyz.data(), r->n, s->pts);
        upload_points(ctx, r->nxyz.data(), r->n, s->nrm);
        ms.push_back(models[j]);
        ss.push_back(s.get());
        {
          std::lock_guard<std::mutex> lk(mu);
          caps.push_back(hints[j]);
        }
        scenes.push_back(std::move(s));
      }
    std::vector<LookupState> states(ms.size());
    std::vector<LookupOut> out = lookup_batch(ctx, ms, ss, states.data(), caps.data());
    size_t k = 0;
    std::lock_guard<std::mutex> lk(mu);
    for (auto& r : batch) {
      r->poses.assign(16 * r->targets.size(), 0.f);
      r->stats.assign(r->targets.size(), ppf_stats{});
      for (size_t t = 0; t < r->targets.size(); ++t, ++k) {
        std::memcpy(&r->poses[16 * t], out[k].pose, sizeof(out[k].pose));
        r->stats[t] = out[k].stats;
        if (out[k].status != PPF_OK) r->status = out[k].status;
        hints[r->targets[t]] = out[k].cand_hint;
      }
    }
  }

  void worker(size_t w) {
    Context& ctx = ctxs[w]->c;
    for (;;) {
      std::vector<std::shared_ptr<Request>> batch;
      size_t bytes = 0;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] {
          return (stop && queue.empty()) ||
                 (!queue.empty() && (in_use == 0 || in_use + queue.front()->need <= budget));
        });
        if (queue.empty()) return;  // stopping and drained
        // admit in arrival order while the budget allows; a request larger
        // than the whole budget runs alone once nothing else is in flight
        while (!queue.empty() && batch.size() < max_batch) {
          const size_t need = queue.front()->need;
          if (in_use + need > budget && !(in_use == 0 && batch.empty())) break;
          in_use += need;
          bytes += need;
          batch.push_back(queue.front());
          queue.pop_front();
        }
      }
      std::string err;
      ppf_status st = PPF_OK;
      try {
        run_batch(ctx, batch);
      } catch (const Error& e) {
        st = e.status;
        err = e.what();
      } catch (const std::exception& e) {
        st = PPF_ERR_INTERNAL;
        err = e.what();
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        in_use -= bytes;
        const Clock::time_point now = Clock::now();
        for (auto& r : batch) {
          if (st != PPF_OK) {
            r->status = st;
            r->error = err;
          }
          r->t_done = now;
          r->done = true;
        }
      }
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }
};

Server* server_create(int device, const std::vector<Model*>& models, size_t memory_budget,
                      uint32_t n_workers, uint32_t max_batch) {
  PPF_REQUIRE(!models.empty(), PPF_ERR_INVALID_ARGUMENT, "empty model library");
  PPF_REQUIRE(n_workers >= 1 && n_workers <= 16, PPF_ERR_INVALID_ARGUMENT, "1 to 16 workers");
  std::unique_ptr<Server> s(new Server());
  s->models = models;
  s->hints.resize(models.size());
  for (size_t j = 0; j < models.size(); ++j) {
    PPF_REQUIRE(models[j], PPF_ERR_INVALID_ARGUMENT, "null model in the library");
    s->hints[j] = models[j]->cand_hint;
  }
  // the library's tables may still be in flight on their own contexts' streams
  PPF_CUDA(cudaDeviceSynchronize());
  s->budget = memory_budget;
  s->max_batch = std::max<uint32_t>(1, max_batch);
  for (uint32_t w = 0; w < n_workers; ++w) {
    s->ctxs.emplace_back(new ppf_context_s());
    init_context(s->ctxs.back()->c, device);
  }
  s->device = s->ctxs[0]->c.device;
  for (uint32_t w = 0; w < n_workers; ++w) s->threads.emplace_back(&Server::worker, s.get(), (size_t)w);
  return s.release();
}

uint64_t server_submit(Server* srv, const float* xyz, const float* nxyz, uint64_t n, uint32_t ref_df,
                       const uint32_t* model_ids, uint64_t n_ids) {
  PPF_REQUIRE(xyz && nxyz && n >= 1 && n < (1ull << 31), PPF_ERR_INVALID_ARGUMENT, "bad scene cloud");
  PPF_REQUIRE(model_ids && n_ids >= 1, PPF_ERR_INVALID_ARGUMENT, "no target models");
  PPF_REQUIRE(!is_any_device_pointer(xyz) && !is_any_device_pointer(nxyz), PPF_ERR_INVALID_ARGUMENT,
              "submitted clouds must be host memory");
  auto r = std::make_shared<Request>();
  r->xyz.assign(xyz, xyz + 3 * n);
  r->nxyz.assign(nxyz, nxyz + 3 * n);
  r->n = n;
  r->ref_df = ref_df ? ref_df : 1;
  for (uint64_t i = 0; i < n_ids; ++i) {
    PPF_REQUIRE(model_ids[i] < srv->models.size(), PPF_ERR_INVALID_ARGUMENT, "model id beyond the library");
    r->targets.push_back(model_ids[i]);
  }
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    PPF_REQUIRE(!srv->stop, PPF_ERR_INVALID_ARGUMENT, "server is stopping");
    r->need = srv->need_bytes(*r);
    r->ticket = srv->next_ticket++;
    r->t_submit = Clock::now();
    srv->tickets[r->ticket] = r;
    srv->queue.push_back(r);
  }
  srv->cv_work.notify_one();
  return r->ticket;
}

ppf_status server_wait(Server* srv, uint64_t ticket, float* poses, ppf_stats* stats, double* latency_ms,
                       std::string* error) {
  std::shared_ptr<Request> r;
  {
    std::unique_lock<std::mutex> lk(srv->mu);
    auto it = srv->tickets.find(ticket);
    PPF_REQUIRE(it != srv->tickets.end(), PPF_ERR_INVALID_ARGUMENT, "unknown or already collected ticket");
    r = it->second;
    srv->cv_done.wait(lk, [&] { return r->done; });
    // by key: another waiter on the same ticket may have erased it meanwhile
    srv->tickets.erase(ticket);
  }
  if (poses && !r->poses.empty()) std::memcpy(poses, r->poses.data(), r->poses.size() * sizeof(float));
  if (stats && !r->stats.empty()) std::memcpy(stats, r->stats.data(), r->stats.size() * sizeof(ppf_stats));
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  if (error) *error = r->error;
  return r->status;
}

void server_destroy(Server* srv) {
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->stop = true;
  }
  srv->cv_work.notify_all();
  for (auto& t : srv->threads) t.join();
  delete srv;
}

}  // namespace ppf
