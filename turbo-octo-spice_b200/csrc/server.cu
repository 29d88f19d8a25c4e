// server.cu — a request server over resident catalogues: continuous
// admission of xi requests to worker slots under a device-memory budget, and
// chunk-level scheduling of their sweeps on the GPU.
//
// Each slot owns an engine (its own stream) and a workspace, and runs one
// request at a time on a host thread of its own.  A request is admitted to a
// free slot as soon as one frees up and its workspace fits in the budget
// beside the resident catalogues and the other slots' workspaces
// (admission.h), in the server's order (FIFO, or least estimated work
// first).  Its pair count's dominant kernel runs as a chain of chunks of
// sightline pairs; the server lets at most two chunks be on the GPU at once
// and hands the next chunk to the waiting request that comes first in the
// same order (the shortest-first order uses the remaining work), so the
// requests of different slots overlap on the device: one request's chunks
// run while others expand their sightline pairs or read back results, a
// short request that arrives mid-flight overtakes a long one at its next
// chunk, and the SMs never idle between chunks.  Runs on one catalogue never
// write to it, so any number of slots may count pairs of the same catalogue
// at once.  The results are those of tos_xi_run on the same catalogue: the
// fixed-point sums do not depend on the order in which pairs are added.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cmath>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "admission.h"
#include "engine_internal.h"

namespace tos {
namespace {

struct Request {
  uint64_t id = 0;
  tos_catalog* cat = nullptr;
  tos_grid grid{};
  double scale = 0;
  uint32_t flags = 0;
  uint64_t need = 0;   // workspace estimate (bytes)
  double work = 0;     // estimated pixel pairs (admission order)
  double t_submit = 0; // server clock at submission
  size_t n_rows = 0;   // per-cell or per-group rows returned
  std::vector<tos_xibin> bins, rows;
  tos_xi_stats stats{};
  tos_status status = TOS_OK;
  std::string error;
  tos_request_info info{};
  bool done = false;
};

constexpr double kPi = 3.14159265358979323846;

// Device bytes a run of `cat` on grid g needs in a workspace: the sightline
// pairs are pairs_estimate's, the rest is exact.
// Estimated sightline pairs of a run (uniform sky density over the occupied
// cells, with a 1.5 margin).
double pairs_estimate(const tos_catalog* cat, const tos_grid& g, double scale) {
  const double nc = (double)cat->cells.size(), n = (double)cat->n_los;
  const double cell_sr = cat->cell_sr;
  const double area = std::max(nc * cell_sr, cell_sr);
  const double ang = std::min(max_angular_scale(g, scale), kPi);
  const double disc = 2.0 * kPi * (1.0 - std::cos(ang));
  return 1.5 * 0.5 * n * std::min(n, n * disc / area) + n;
}

uint64_t workspace_estimate(const tos_catalog* cat, const tos_grid& g, double scale, size_t n_rows) {
  const double nb = (double)g.axis[0].nbins * g.axis[1].nbins * g.axis[2].nbins;
  const double nc = (double)cat->cells.size(), n = (double)cat->n_los;
  const double cell_sr = cat->cell_sr;
  const double area = std::max(nc * cell_sr, cell_sr);
  const double ang = std::min(max_angular_scale(g, scale), kPi);
  const double disc = 2.0 * kPi * (1.0 - std::cos(ang));
  const double pairs = pairs_estimate(cat, g, scale);
  const double near_cells = std::min(nc, nc * disc / area + 9.0);
  double bytes = 0;
  bytes += nc * nb * 128.0;                                   // per-cell sums
  bytes += nb * sizeof(tos_xibin) * (1.0 + (double)n_rows);   // results
  bytes += pairs * 20.0;                                      // items (i, j, cos, theta index)
  bytes += n * 24.0;                                          // per primary counts and offsets
  bytes += nc * (near_cells + 12.0) * 4.0;                    // cell neighbours
  bytes += 4192.0 * 8 + 2.0 * 65536 * (g.axis[0].nbins + 1.0) + 1e6;  // counters, tables, cub
  return (uint64_t)bytes;
}


}  // namespace
}  // namespace tos

struct tos_server {
  explicit tos_server(int slots, uint64_t budget) : adm(slots, budget) {}
  int device = 0;
  tos::Admission adm;
  tos_engine* setup = nullptr;                 // catalogue preparation at attach
  std::vector<tos_engine*> engines;            // per slot
  std::vector<std::unique_ptr<tos::Workspace>> ws;
  std::vector<tos::Request*> assigned;         // per slot: the running request
  std::vector<std::thread> threads;
  std::mutex mu;
  std::condition_variable cv_slot, cv_done;
  std::deque<tos::Request*> queue;
  std::unordered_map<uint64_t, std::unique_ptr<tos::Request>> reqs;
  std::unordered_map<const tos_catalog*, uint64_t> attached;  // catalogue -> resident bytes
  std::unordered_map<const tos_catalog*, uint64_t> pending;   // unfinished requests per catalogue
  int policy = tos::kFifo;
  double max_wait_s = 5.0;
  // Sweep scheduler: running requests launch their sweep in chunks, at most
  // kChunksInFlight chunks on the GPU at once (the next one queued behind the
  // running one, so the SMs never idle between chunks); a chunk that may
  // launch goes to the waiting request first in the admission order (FIFO:
  // the oldest; shortest-first: the least remaining work, unless a request
  // has waited max_wait_s since it was submitted).  A short request that
  // arrives while a long one sweeps thus takes the SMs at the long one's next
  // chunk, and every request's expansion and result phases run beside other
  // requests' chunks.
  static constexpr int kChunksInFlight = 2;
  struct ChunkWaiter {
    uint64_t remaining;
    double t_submit;
    uint64_t id;
  };
  std::mutex sched_mu;
  std::condition_variable sched_cv;
  std::vector<ChunkWaiter*> chunk_waiters;
  int chunks_in_flight = 0;

  // Whether w goes before v (sched_mu held).
  bool chunk_before(const ChunkWaiter* w, const ChunkWaiter* v, double t) const {
    if (policy == tos::kShortest) {
      const bool ow = t - w->t_submit > max_wait_s, ov = t - v->t_submit > max_wait_s;
      if (ow != ov) return ow;
      if (!ow && w->remaining != v->remaining) return w->remaining < v->remaining;
    }
    return w->t_submit != v->t_submit ? w->t_submit < v->t_submit : w->id < v->id;
  }

  int acquire_chunk(tos::Request* r, uint64_t remaining) {
    std::unique_lock<std::mutex> lk(sched_mu);
    ChunkWaiter me{remaining, r->t_submit, r->id};
    chunk_waiters.push_back(&me);
    sched_cv.wait(lk, [&] {
      if (chunks_in_flight >= kChunksInFlight) return false;
      const double t = now();
      for (const ChunkWaiter* w : chunk_waiters)
        if (w != &me && chunk_before(w, &me, t)) return false;
      return true;
    });
    chunk_waiters.erase(std::find(chunk_waiters.begin(), chunk_waiters.end(), &me));
    ++chunks_in_flight;
    sched_cv.notify_all();
    return 0;  // the whole GPU: as many CTAs per SM as fit
  }

  void release_chunk() {
    std::lock_guard<std::mutex> lk(sched_mu);
    --chunks_in_flight;
    sched_cv.notify_all();
  }
  uint64_t next_id = 1, completed = 0, peak = 0;
  bool stop = false;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }

  // Start queued requests while a candidate fits (mu held).
  void dispatch() {
    while (!queue.empty()) {
      const double t = now();
      std::vector<tos::QueuedView> view(queue.size());
      for (size_t q = 0; q < queue.size(); ++q) view[q] = {queue[q]->work, t - queue[q]->t_submit};
      std::vector<bool> strict;
      const std::vector<size_t> order = tos::order_queue(view, policy, max_wait_s, &strict);
      size_t pos = queue.size();
      int k = -1;
      for (size_t c = 0; c < order.size(); ++c) {
        k = adm.pick(queue[order[c]]->need);
        if (k >= 0) {
          pos = order[c];
          break;
        }
        if (strict[c]) break;  // not overtaken
      }
      if (k < 0) {
        const int v = adm.trim_victim(queue[order[0]]->need);
        if (v < 0) break;  // wait for a running request to finish
        // an idle slot gives its workspace back (its stream has no work)
        int prev = -1;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        ws[v].reset(new tos::Workspace());
        cudaSetDevice(prev);
        adm.release(v);
        continue;
      }
      tos::Request* r = queue[pos];
      queue.erase(queue.begin() + (long)pos);
      adm.start(k, r->need);
      peak = std::max(peak, adm.in_use());
      r->info.start_s = now();
      r->info.slot = k;
      assigned[k] = r;
      cv_slot.notify_all();
    }
  }

  void worker(int k) {
    cudaSetDevice(device);
    for (;;) {
      tos::Request* r = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_slot.wait(lk, [&] { return stop || assigned[k] != nullptr; });
        if (!assigned[k]) return;  // stopped and idle
        r = assigned[k];
      }
      const size_t nb = (size_t)r->grid.axis[0].nbins * r->grid.axis[1].nbins * r->grid.axis[2].nbins;
      r->bins.assign(nb, tos_xibin{});
      r->rows.assign(r->n_rows * nb, tos_xibin{});
      tos::SweepShare share;
      share.acquire = [this, r](uint64_t remaining) { return acquire_chunk(r, remaining); };
      share.release = [this] { release_chunk(); };
      share.chunks = 16;
      const tos_status s = tos::xi_run_impl(engines[k], r->cat, ws[k].get(), &r->grid, r->scale,
                                            r->flags, nullptr, r->bins.data(),
                                            r->n_rows ? r->rows.data() : nullptr, &r->stats, &share);
      cudaStreamSynchronize(engines[k]->stream);  // chunk callbacks done before `share` goes
      std::string err = (s == TOS_OK) ? std::string() : std::string(tos_last_error());
      const uint64_t held = ws[k]->bytes();
      std::lock_guard<std::mutex> lk(mu);
      r->status = s;
      r->error = err;
      r->info.end_s = now();
      r->done = true;
      assigned[k] = nullptr;
      adm.finish(k, held);
      peak = std::max(peak, adm.in_use());
      if (--pending[r->cat] == 0) pending.erase(r->cat);
      ++completed;
      dispatch();
      cv_done.notify_all();
    }
  }
};

using namespace tos;

extern "C" {

tos_status tos_server_create(int device, int slots, uint64_t memory_budget_bytes, tos_server** out) {
  if (!out) return fail(TOS_ERR_INVALID_ARG, "out is null");
  *out = nullptr;
  if (slots < 1 || slots > 64) return fail(TOS_ERR_INVALID_ARG, "slots must be in [1, 64]");
  std::unique_ptr<tos_server> s(new tos_server(slots, memory_budget_bytes));
  s->device = device;
  TOS_TRY(tos_engine_create(device, &s->setup));
  for (int k = 0; k < slots; ++k) {
    tos_engine* e = nullptr;
    const tos_status st = tos_engine_create(device, &e);
    if (st != TOS_OK) {
      for (tos_engine* x : s->engines) tos_engine_destroy(x);
      tos_engine_destroy(s->setup);
      return st;
    }
    s->engines.push_back(e);
    s->ws.emplace_back(new Workspace());
  }
  s->assigned.assign(slots, nullptr);
  for (int k = 0; k < slots; ++k) s->threads.emplace_back(&tos_server::worker, s.get(), k);
  *out = s.release();
  return TOS_OK;
}

void tos_server_destroy(tos_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (Request* r : s->queue) {  // never started
      r->status = TOS_ERR_INVALID_ARG;
      r->error = "server destroyed before the request started";
      r->done = true;
    }
    s->queue.clear();
    s->cv_slot.notify_all();
    s->cv_done.notify_all();
  }
  for (auto& t : s->threads) t.join();  // running requests finish first
  {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    s->ws.clear();
    cudaSetDevice(prev);
  }
  for (tos_engine* e : s->engines) tos_engine_destroy(e);
  tos_engine_destroy(s->setup);
  delete s;
}

tos_status tos_server_attach(tos_server* s, tos_catalog* cat) {
  if (!s || !cat) return fail(TOS_ERR_INVALID_ARG, "null argument");
  if (cat->device != s->device) return fail(TOS_ERR_INVALID_ARG, "catalogue is on another device");
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->attached.count(cat)) return TOS_OK;
  }
  // the common-grid tables are built once per catalogue, before any request
  {
    std::lock_guard<std::mutex> el(s->setup->mu);
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    tos_status st = TOS_OK;
    for (int w = 0; w < 2 && st == TOS_OK; ++w) st = ensure_grid(s->setup, cat, w, s->setup->stream);
    cudaSetDevice(prev);
    TOS_TRY(st);
  }
  const uint64_t bytes = catalog_data_bytes(cat) + cat->run.bytes();
  std::lock_guard<std::mutex> lk(s->mu);
  if (!s->adm.add_resident(bytes))
    return fail(TOS_ERR_OOM, "catalogue (" + std::to_string(bytes) +
                                 " bytes) does not fit in the server's memory budget");
  s->attached[cat] = bytes;
  return TOS_OK;
}

tos_status tos_server_detach(tos_server* s, tos_catalog* cat) {
  if (!s || !cat) return fail(TOS_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->attached.find(cat);
  if (it == s->attached.end()) return fail(TOS_ERR_INVALID_ARG, "catalogue is not attached");
  if (s->pending.count(cat)) return fail(TOS_ERR_INVALID_ARG, "catalogue has unfinished requests");
  s->adm.remove_resident(it->second);
  s->attached.erase(it);
  s->dispatch();
  return TOS_OK;
}

tos_status tos_server_submit(tos_server* s, tos_catalog* cat, const tos_grid* grid, double scale,
                             uint32_t flags, uint64_t* request_id) {
  if (!s || !cat || !grid || !request_id) return fail(TOS_ERR_INVALID_ARG, "null argument");
  double max_ang = 0;
  TOS_TRY(tos_grid_max_angular_scale(grid, scale, &max_ang));
  if (flags & ~(TOS_XI_SUBSAMPLES | TOS_XI_EXACT | TOS_XI_PER_GROUP))
    return fail(TOS_ERR_INVALID_ARG, "unknown flags");
  if ((flags & TOS_XI_SUBSAMPLES) && (flags & TOS_XI_PER_GROUP))
    return fail(TOS_ERR_INVALID_ARG, "TOS_XI_PER_GROUP and TOS_XI_SUBSAMPLES are exclusive");
  std::unique_ptr<Request> r(new Request());
  r->cat = cat;
  r->grid = *grid;
  r->scale = scale;
  r->flags = flags;
  r->n_rows = (flags & TOS_XI_SUBSAMPLES) ? cat->cells.size()
              : (flags & TOS_XI_PER_GROUP) ? cat->groups.size()
                                           : 0;
  r->need = workspace_estimate(cat, *grid, scale, r->n_rows);
  {
    const double px = (double)cat->n_pix / std::max<double>(1.0, (double)cat->n_los);
    r->work = pairs_estimate(cat, *grid, scale) * px * px;
  }
  r->info.workspace_bytes = r->need;
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return fail(TOS_ERR_INVALID_ARG, "server is shutting down");
  if (!s->attached.count(cat)) return fail(TOS_ERR_INVALID_ARG, "catalogue is not attached");
  if (!s->adm.can_ever_fit(r->need))
    return fail(TOS_ERR_OOM, "request needs about " + std::to_string(r->need) +
                                 " bytes of workspace: more than the budget leaves beside the "
                                 "resident catalogues");
  r->id = s->next_id++;
  r->info.submit_s = s->now();
  r->t_submit = r->info.submit_s;
  r->info.slot = -1;
  *request_id = r->id;
  s->pending[cat]++;
  s->queue.push_back(r.get());
  s->reqs[r->id] = std::move(r);
  s->dispatch();
  return TOS_OK;
}

tos_status tos_server_wait(tos_server* s, uint64_t id, tos_xibin* out_bins, tos_xibin* out_rows,
                           tos_xi_stats* stats, tos_request_info* info) {
  if (!s) return fail(TOS_ERR_INVALID_ARG, "null argument");
  std::unique_ptr<Request> r;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(TOS_ERR_INVALID_ARG, "unknown request id");
    Request* p = it->second.get();
    s->cv_done.wait(lk, [&] { return p->done; });
    r = std::move(it->second);
    s->reqs.erase(it);
  }
  if (info) *info = r->info;
  if (r->status != TOS_OK) return fail(r->status, r->error);
  if (out_bins) std::copy(r->bins.begin(), r->bins.end(), out_bins);
  if (out_rows && r->n_rows) std::copy(r->rows.begin(), r->rows.end(), out_rows);
  if (stats) *stats = r->stats;
  return TOS_OK;
}

tos_status tos_server_set_policy(tos_server* s, int policy, double max_wait_s) {
  if (!s) return fail(TOS_ERR_INVALID_ARG, "null argument");
  if (policy != kFifo && policy != kShortest) return fail(TOS_ERR_INVALID_ARG, "unknown policy");
  if (!(max_wait_s >= 0)) return fail(TOS_ERR_INVALID_ARG, "max_wait_s must be >= 0");
  std::lock_guard<std::mutex> lk(s->mu);
  s->policy = policy;
  s->max_wait_s = max_wait_s;
  s->dispatch();
  return TOS_OK;
}

tos_status tos_server_poll(tos_server* s, uint64_t id, int* done) {
  if (!s || !done) return fail(TOS_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return fail(TOS_ERR_INVALID_ARG, "unknown request id");
  *done = it->second->done ? 1 : 0;
  return TOS_OK;
}

tos_status tos_server_status_get(tos_server* s, tos_server_status* out) {
  if (!s || !out) return fail(TOS_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  out->budget_bytes = s->adm.budget();
  out->resident_bytes = s->adm.resident();
  out->in_use_bytes = s->adm.in_use();
  out->peak_bytes = s->peak;
  out->queued = s->queue.size();
  uint64_t running = 0;
  for (auto* r : s->assigned) running += (r != nullptr);
  out->running = running;
  out->completed = s->completed;
  out->slots = (uint32_t)s->engines.size();
  return TOS_OK;
}

}  // extern "C"
