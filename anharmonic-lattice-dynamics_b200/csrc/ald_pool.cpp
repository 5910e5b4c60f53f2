// Process-wide host worker pool (ald_pool.h).
#include "ald_pool.h"

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

namespace ald {

namespace {

struct Job {
  const std::function<void(int)>* f;
  int ntask;
  std::atomic<int> next{0};  // next task index to hand out
  std::atomic<int> done{0};  // tasks finished
  int active = 0;            // workers inside the job (under the pool's mutex)
};

class Pool {
 public:
  explicit Pool(int nworkers) {
    for (int i = 0; i < nworkers; ++i) workers_.emplace_back([this] { loop(); });
  }
  // never destroyed: the workers wait on cv_ until the process ends
  int width() const { return (int)workers_.size() + 1; }

  void run(int ntask, const std::function<void(int)>& f) {
    Job j;
    j.f = &f;
    j.ntask = ntask;
    {
      std::lock_guard<std::mutex> lk(m_);
      jobs_.push_back(&j);
    }
    cv_.notify_all();
    work(j);
    std::unique_lock<std::mutex> lk(m_);
    remove(&j);
    done_cv_.wait(lk, [&] { return j.active == 0 && j.done.load() == ntask; });
  }

 private:
  static void work(Job& j) {
    for (int i; (i = j.next.fetch_add(1)) < j.ntask;) {
      (*j.f)(i);
      j.done.fetch_add(1);
    }
  }
  void remove(Job* j) {
    auto it = std::find(jobs_.begin(), jobs_.end(), j);
    if (it != jobs_.end()) jobs_.erase(it);
  }
  void loop() {
    std::unique_lock<std::mutex> lk(m_);
    for (;;) {
      cv_.wait(lk, [&] { return !jobs_.empty(); });
      Job* j = jobs_.front();
      if (j->next.load() >= j->ntask) {  // handed out completely: no more work in it
        remove(j);
        continue;
      }
      ++j->active;
      lk.unlock();
      work(*j);
      lk.lock();
      --j->active;
      remove(j);
      done_cv_.notify_all();
    }
  }

  std::mutex m_;
  std::condition_variable cv_, done_cv_;
  std::deque<Job*> jobs_;
  std::vector<std::thread> workers_;
};

Pool& pool() {
  static Pool* p = new Pool((int)std::max(1u, std::min(32u, std::thread::hardware_concurrency())) - 1);
  return *p;
}

}  // namespace

void run_parallel(int ntask, const std::function<void(int)>& f) {
  if (ntask <= 0) return;
  if (ntask == 1) {
    f(0);
    return;
  }
  pool().run(ntask, f);
}

int pool_width() { return pool().width(); }

}  // namespace ald
