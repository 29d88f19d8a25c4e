// admission.h — memory-budget admission of requests to worker slots (host
// logic only, no CUDA: unit-tested on its own).
//
// Device memory under the budget is the resident catalogues plus every
// slot's workspace.  A slot keeps its workspace between requests (so a
// steady stream of requests allocates nothing); a request that needs more
// grows it.  A request may start on a free slot k when
//     resident + sum_{s != k} held[s] + max(held[k], need) <= budget.
// Requests start in arrival order (FIFO), or least estimated work first with
// aging (order_queue).  When the first candidate fits on no free slot, idle
// slots give their workspaces back (largest first) until it fits; if it
// still does not fit it waits for running requests to finish.  A request that cannot fit even with every slot empty is refused
// at submission.
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace tos {

// Order in which queued requests are offered to the slots.
enum QueuePolicy {
  kFifo = 0,      // arrival order; the head waits until it fits (no overtaking)
  kShortest = 1,  // smallest estimated work first; a request waiting longer than
                  // max_wait_s goes first (oldest first) and is not overtaken
};

struct QueuedView {
  double work;      // estimated pixel pairs
  double waited_s;  // time in the queue
};

// Candidates to start, in preference order, as positions in the queue
// (arrival order).  The first candidate that fits starts; a candidate marked
// strict in `strict` stops the search when it does not fit.
inline std::vector<size_t> order_queue(const std::vector<QueuedView>& q, int policy,
                                       double max_wait_s, std::vector<bool>* strict) {
  std::vector<size_t> idx(q.size());
  for (size_t k = 0; k < q.size(); ++k) idx[k] = k;
  strict->assign(q.size(), true);
  if (policy == kFifo || q.empty()) {
    idx.resize(q.empty() ? 0 : 1);
    return idx;
  }
  std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
    const bool oa = q[a].waited_s > max_wait_s, ob = q[b].waited_s > max_wait_s;
    if (oa != ob) return oa;                       // waited too long: first
    if (oa) return q[a].waited_s > q[b].waited_s;  // ... oldest first
    return q[a].work < q[b].work;                  // then the least work
  });
  for (size_t k = 0; k < idx.size(); ++k) (*strict)[k] = q[idx[k]].waited_s > max_wait_s;
  return idx;
}

class Admission {
 public:
  Admission(int slots, uint64_t budget) : budget_(budget), held_(slots, 0), busy_(slots, false) {}

  uint64_t budget() const { return budget_; }
  uint64_t resident() const { return resident_; }
  uint64_t held(int k) const { return held_[k]; }
  bool busy(int k) const { return busy_[k]; }
  int slots() const { return (int)held_.size(); }
  uint64_t in_use() const {
    uint64_t t = resident_;
    for (uint64_t h : held_) t += h;
    return t;
  }

  // Resident catalogue bytes: add (false when they do not fit beside the
  // slots' current workspaces) or remove.
  bool add_resident(uint64_t bytes) {
    if (in_use() + bytes > budget_) return false;
    resident_ += bytes;
    return true;
  }
  void remove_resident(uint64_t bytes) { resident_ -= (bytes <= resident_) ? bytes : resident_; }

  // Can a request of `need` bytes ever run (every slot's workspace empty)?
  bool can_ever_fit(uint64_t need) const { return resident_ + need <= budget_; }

  // A free slot that takes `need` bytes now, or -1.  Prefers a slot that
  // already holds enough (no growth), then the one holding the most.
  int pick(uint64_t need) const {
    const uint64_t total = in_use();
    int best = -1;
    for (int k = 0; k < slots(); ++k) {
      if (busy_[k]) continue;
      const uint64_t grown = need > held_[k] ? need : held_[k];
      if (total - held_[k] + grown > budget_) continue;
      if (best < 0) {
        best = k;
        continue;
      }
      const bool k_fits = held_[k] >= need, b_fits = held_[best] >= need;
      if (k_fits != b_fits ? k_fits : held_[k] > held_[best]) best = k;
    }
    return best;
  }

  // The idle slot whose workspace should be given back so that `need` can
  // start, or -1 when trimming idle slots cannot make it fit (then the
  // request waits for a running one to finish).
  int trim_victim(uint64_t need) const {
    uint64_t idle = 0;
    int victim = -1;
    for (int k = 0; k < slots(); ++k) {
      if (busy_[k] || held_[k] == 0) continue;
      idle += held_[k];
      if (victim < 0 || held_[k] > held_[victim]) victim = k;
    }
    if (victim < 0) return -1;
    // after giving back every idle workspace the request runs on an empty slot
    bool free_slot = false;
    for (int k = 0; k < slots(); ++k) free_slot = free_slot || !busy_[k];
    if (!free_slot || in_use() - idle + need > budget_) return -1;
    return victim;
  }

  void start(int k, uint64_t need) {
    busy_[k] = true;
    if (need > held_[k]) held_[k] = need;  // reserved until the run reports its real size
  }
  // The run ended; its workspace now holds `bytes`.
  void finish(int k, uint64_t bytes) {
    busy_[k] = false;
    held_[k] = bytes;
  }
  void release(int k) { held_[k] = 0; }

 private:
  uint64_t budget_;
  uint64_t resident_ = 0;
  std::vector<uint64_t> held_;
  std::vector<bool> busy_;
};

}  // namespace tos
