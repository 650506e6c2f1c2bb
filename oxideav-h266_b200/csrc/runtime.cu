// Host runtime pieces of the filter chain library: the worker pool that builds
// side information (deblocking plans, SAO / ALF tables) for several pictures
// at once while the GPU filters earlier ones.
#include "internal.h"

namespace h266 {

TaskPool::TaskPool(unsigned threads) {
  for (unsigned t = 0; t < threads; ++t) workers_.emplace_back([this] { loop(); });
}

TaskPool::~TaskPool() {
  wait_all();
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  work_cv_.notify_all();
  for (auto &w : workers_) w.join();
}

void TaskPool::start(size_t n, std::function<void(size_t)> fn) {
  wait_all();  // one job at a time
  {
    std::lock_guard<std::mutex> lk(mu_);
    fn_ = std::move(fn);
    done_.assign(n, 0);
    n_ = n;
    next_ = 0;
    finished_ = 0;
  }
  work_cv_.notify_all();
}

void TaskPool::wait_item(size_t i) {
  std::unique_lock<std::mutex> lk(mu_);
  done_cv_.wait(lk, [&] { return i >= n_ || done_[i]; });
}

void TaskPool::wait_all() {
  std::unique_lock<std::mutex> lk(mu_);
  done_cv_.wait(lk, [&] { return finished_ == n_; });
}

void TaskPool::loop() {
  std::unique_lock<std::mutex> lk(mu_);
  for (;;) {
    work_cv_.wait(lk, [&] { return stop_ || next_ < n_; });
    if (stop_) return;
    const size_t i = next_++;
    lk.unlock();
    fn_(i);
    lk.lock();
    done_[i] = 1;
    ++finished_;
    done_cv_.notify_all();
  }
}

}  // namespace h266
