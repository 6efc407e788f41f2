// Minimal work-sharing thread pool used by the TBB-compatible shim headers.
//
// This is oracle test infrastructure: it lets the unmodified reference CPU
// sources (which include <tbb/...>) compile and run multi-threaded on hosts
// without Intel TBB. It schedules only; the reference's results do not depend
// on which thread runs which chunk because seed chunks, track chunks and
// layers are independent work items in the reference.
//
// Design: one global queue of type-erased tasks served by N-1 worker threads.
// A thread that waits for a group of tasks executes queued tasks itself
// ("help while waiting"), so nested parallel loops cannot deadlock.
#pragma once

#include <atomic>
#include <condition_variable>
#include <cstdlib>
#include <deque>
#include <functional>
#include <memory>
#include <chrono>
#include <mutex>
#include <thread>
#include <vector>

namespace tbbshim {

class Pool {
 public:
  static Pool& instance() {
    static Pool p;
    return p;
  }

  // Number of threads that take part in parallel loops (workers + caller).
  int concurrency() const { return int(m_workers.size()) + 1; }

  // Resize the pool. Must not be called while a parallel loop is running.
  void resize(int n_threads) {
    stop_workers();
    if (n_threads < 1) n_threads = 1;
    m_stop = false;
    for (int i = 0; i < n_threads - 1; ++i)
      m_workers.emplace_back([this] { worker_loop(); });
  }

  void submit(std::function<void()> f) {
    {
      std::lock_guard<std::mutex> lk(m_mtx);
      m_queue.emplace_back(std::move(f));
    }
    m_cv.notify_one();
  }

  // Run one queued task on the calling thread; false if the queue was empty.
  bool run_one() {
    std::function<void()> f;
    {
      std::lock_guard<std::mutex> lk(m_mtx);
      if (m_queue.empty()) return false;
      f = std::move(m_queue.front());
      m_queue.pop_front();
    }
    f();
    return true;
  }

  ~Pool() { stop_workers(); }

 private:
  Pool() {
    int n = 1;
    if (const char* e = std::getenv("MKFIT_REF_THREADS")) n = std::atoi(e);
    resize(n);
  }

  void stop_workers() {
    {
      std::lock_guard<std::mutex> lk(m_mtx);
      m_stop = true;
    }
    m_cv.notify_all();
    for (auto& t : m_workers) t.join();
    m_workers.clear();
  }

  void worker_loop() {
    for (;;) {
      std::function<void()> f;
      {
        std::unique_lock<std::mutex> lk(m_mtx);
        m_cv.wait(lk, [this] { return m_stop || !m_queue.empty(); });
        if (m_stop && m_queue.empty()) return;
        f = std::move(m_queue.front());
        m_queue.pop_front();
      }
      f();
    }
  }

  std::vector<std::thread> m_workers;
  std::deque<std::function<void()>> m_queue;
  std::mutex m_mtx;
  std::condition_variable m_cv;
  bool m_stop = false;
};

// Runs n_tasks calls task(i), i in [0, n_tasks), spread over the pool; returns
// when all have finished. The calling thread runs tasks too.
template <typename F>
void run_tasks(int n_tasks, F&& task) {
  if (n_tasks <= 0) return;
  Pool& pool = Pool::instance();
  if (n_tasks == 1 || pool.concurrency() == 1) {
    for (int i = 0; i < n_tasks; ++i) task(i);
    return;
  }
  // Completion state is shared-owned so a worker that finishes last can still
  // signal after the waiting thread has observed completion and returned.
  struct State {
    std::atomic<int> remaining;
    std::mutex mtx;
    std::condition_variable cv;
  };
  auto st = std::make_shared<State>();
  st->remaining.store(n_tasks);
  for (int i = 1; i < n_tasks; ++i) {
    pool.submit([st, &task, i] {
      task(i);
      if (st->remaining.fetch_sub(1) == 1) {
        std::lock_guard<std::mutex> lk(st->mtx);
        st->cv.notify_all();
      }
    });
  }
  task(0);
  st->remaining.fetch_sub(1);
  // Help with queued work (possibly other loops' tasks) until ours are done.
  while (st->remaining.load() > 0) {
    if (!pool.run_one()) {
      std::unique_lock<std::mutex> lk(st->mtx);
      st->cv.wait_for(lk, std::chrono::microseconds(50),
                      [&] { return st->remaining.load() == 0; });
    }
  }
}

}  // namespace tbbshim
