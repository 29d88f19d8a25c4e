// Stand-in for boost/asio/io_service.hpp: a FIFO of posted handlers that
// run() drains on any number of threads; run() returns once no work object
// is alive and the queue is empty, as asio's io_service does.
#pragma once
#include <condition_variable>
#include <cstddef>
#include <deque>
#include <functional>
#include <mutex>
namespace boost {
namespace asio {
class io_service {
 public:
  class work {
   public:
    explicit work(io_service& s) : s_(s) {
      std::lock_guard<std::mutex> g(s_.m_);
      ++s_.work_;
    }
    ~work() {
      std::lock_guard<std::mutex> g(s_.m_);
      --s_.work_;
      s_.cv_.notify_all();
    }

   private:
    io_service& s_;
  };
  template <class F>
  void post(F f) {
    std::lock_guard<std::mutex> g(m_);
    q_.emplace_back(std::move(f));
    cv_.notify_one();
  }
  std::size_t run() {
    std::size_t n = 0;
    for (;;) {
      std::function<void()> h;
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return !q_.empty() || work_ == 0; });
        if (q_.empty()) return n;
        h = std::move(q_.front());
        q_.pop_front();
      }
      h();
      ++n;
    }
  }

 private:
  std::mutex m_;
  std::condition_variable cv_;
  std::deque<std::function<void()>> q_;
  long work_ = 0;
};
}  // namespace asio
}  // namespace boost
