// Stand-in for boost/thread/future.hpp: the old boost packaged_task<R>
// (template argument = result type), shared_future and wait_for_all.
#pragma once
#include <future>
namespace boost {
template <class R>
using shared_future = std::shared_future<R>;
template <class R>
class packaged_task {
 public:
  template <class F>
  explicit packaged_task(F f) : task_(f) {}
  std::future<R> get_future() { return task_.get_future(); }
  void operator()() { task_(); }

 private:
  std::packaged_task<R()> task_;
};
template <class It>
void wait_for_all(It first, It last) {
  for (; first != last; ++first) first->wait();
}
}  // namespace boost
