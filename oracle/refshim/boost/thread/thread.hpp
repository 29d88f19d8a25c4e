// Stand-in for boost/thread/thread.hpp: thread_group over std::thread.
#pragma once
#include <thread>
#include <vector>
namespace boost {
class thread_group {
 public:
  thread_group() = default;
  thread_group(const thread_group&) = delete;
  ~thread_group() { join_all(); }
  template <class F>
  void create_thread(F f) { threads_.emplace_back(f); }
  void join_all() {
    for (auto& t : threads_)
      if (t.joinable()) t.join();
  }

 private:
  std::vector<std::thread> threads_;
};
}  // namespace boost
