// Unit test of the server's memory-budget admission policy (admission.h):
// host logic only, built and run by tests/test_admission.py.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "admission.h"

#define CHECK(c)                                                    \
  do {                                                              \
    if (!(c)) {                                                     \
      std::fprintf(stderr, "%s:%d: CHECK(%s) failed\n", __FILE__, __LINE__, #c); \
      std::exit(1);                                                 \
    }                                                               \
  } while (0)

int main() {
  using tos::Admission;
  {  // resident catalogues count against the budget
    Admission a(2, 100);
    CHECK(a.add_resident(60));
    CHECK(!a.add_resident(50));
    CHECK(a.resident() == 60);
    CHECK(a.can_ever_fit(40));
    CHECK(!a.can_ever_fit(41));
    a.remove_resident(60);
    CHECK(a.resident() == 0);
  }
  {  // two slots run at once while both workspaces fit
    Admission a(2, 100);
    CHECK(a.add_resident(20));
    int k = a.pick(30);
    CHECK(k >= 0);
    a.start(k, 30);
    int k2 = a.pick(30);
    CHECK(k2 >= 0 && k2 != k);
    a.start(k2, 30);
    CHECK(a.in_use() == 80);
    CHECK(a.pick(10) < 0);  // no free slot
    a.finish(k, 25);        // real size below the estimate
    CHECK(a.held(k) == 25 && !a.busy(k));
    CHECK(a.pick(25) == k);  // reuses the idle workspace without growth
    CHECK(a.pick(50) == k);  // 20 + 30 + 50 = 100 fits
    CHECK(a.pick(51) < 0);
    CHECK(a.trim_victim(51) < 0);  // the busy slot holds the memory: wait
  }
  {  // the second request waits for memory, not for a slot
    Admission a(3, 100);
    int k = a.pick(70);
    a.start(k, 70);
    CHECK(a.pick(40) < 0);
    CHECK(a.trim_victim(40) < 0);
    a.finish(k, 70);
    // the idle slot holding 70 would have to grow to fit 40? no: it holds
    // enough already, so it takes the request with no growth
    CHECK(a.pick(40) == k);
  }
  {  // idle workspaces are given back for a request that needs the room
    Admission a(2, 100);
    a.start(0, 60);
    a.finish(0, 60);
    a.start(1, 30);  // slot 1 busy with 30
    // a request of 65 cannot grow slot 0 (30 + 65 > 100 needs slot 0 empty: 95)
    CHECK(a.pick(65) == 0);
    a.finish(1, 30);
    // now both idle: 60 + 30 held; a request of 80 fits only after trimming
    CHECK(a.pick(80) < 0);
    const int v = a.trim_victim(80);
    CHECK(v == 0);  // the larger idle workspace goes first
    a.release(v);
    const int k = a.pick(80);  // slot 1 grows its 30 to 80
    CHECK(k == 1);
    a.start(k, 80);
    CHECK(a.in_use() == 80);
  }
  {  // a request larger than the budget never fits
    Admission a(1, 100);
    CHECK(a.add_resident(10));
    CHECK(!a.can_ever_fit(91));
    CHECK(a.pick(91) < 0);
    CHECK(a.trim_victim(91) < 0);
  }
  {  // admission order
    using tos::order_queue;
    std::vector<bool> strict;
    const std::vector<tos::QueuedView> q = {{9e12, 0.5}, {1e10, 0.2}, {4e11, 0.1}, {2e12, 7.0}};
    std::vector<size_t> o = order_queue(q, tos::kFifo, 5.0, &strict);
    CHECK(o.size() == 1 && o[0] == 0 && strict[0]);  // FIFO: the head only
    o = order_queue(q, tos::kShortest, 5.0, &strict);
    CHECK(o.size() == 4);
    CHECK(o[0] == 3 && strict[0]);                    // waited 7 s > 5 s: first, not overtaken
    CHECK(o[1] == 1 && o[2] == 2 && o[3] == 0);       // then least work first
    CHECK(!strict[1] && !strict[2] && !strict[3]);
    o = order_queue({}, tos::kShortest, 5.0, &strict);
    CHECK(o.empty());
  }
  std::puts("admission: ok");
  return 0;
}
