// Admission and continuous batching for the serving loop (host logic only, no CUDA).
//
// Requests wait in FIFO order per lane.  A lane's worker takes the longest prefix of its
// queue whose device-memory footprints fit in what the shared budget has left (at most
// max_batch requests), runs them as one batch, then releases their memory.  The memory
// of the other lanes' heads that arrived earlier is kept for them: a request is admitted
// only if it fits beside those heads, so a large request at the head of one lane is not
// starved by a stream of later small ones on the others.  Requests
// that arrive while a batch runs wait for the next one; a request larger than the whole
// budget is refused at submission.  The executor (the GPU in the server, a fake in the
// CPU tests) is a callback.
//
// With a second stage, a lane is a two-step pipeline: the admitting worker runs stage 1
// (in the server: the host-to-device copies) and hands the batch to the lane's second
// thread, which runs stage 2 (the replies and the copies back) and completes it; up to
// `depth` batches per lane are in flight, so batch k+1's copies overlap batch k's work.
#pragma once

#include <stdint.h>

#include <chrono>
#include <condition_variable>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace xpir {

struct Job {
  uint64_t ticket = 0;
  uint32_t lane = 0;
  uint64_t footprint = 0;  // device bytes reserved while the job is admitted
  double t_submit = 0, t_admit = 0, t_done = 0;
  int status = 0;
  bool done = false;
  std::shared_ptr<void> payload;  // executor's data (buffers, request description)
};

struct AdmissionStats {
  uint64_t submitted = 0, completed = 0, batches = 0, max_batch_seen = 0, refused = 0;
  uint64_t peak_in_use = 0;
};

class Admission {
 public:
  // Runs one batch of jobs of one lane; sets each job's status.
  typedef std::function<void(uint32_t lane, std::vector<Job *> &batch)> Executor;

  Admission(uint32_t lanes, uint64_t budget, uint32_t max_batch, Executor exec, Executor stage2 = nullptr,
            uint32_t depth = 2)
      : budget_(budget),
        max_batch_(max_batch ? max_batch : 1),
        depth_(stage2 ? (depth ? depth : 1) : 1),
        exec_(std::move(exec)),
        stage2_(std::move(stage2)),
        queues_(lanes),
        handoff_(lanes),
        inflight_(lanes, 0) {
    for (uint32_t l = 0; l < lanes; l++) workers_.emplace_back([this, l] { run(l); });
    if (stage2_)
      for (uint32_t l = 0; l < lanes; l++) workers_.emplace_back([this, l] { run_stage2(l); });
  }

  ~Admission() { stop(); }

  // Stops the workers once the admitted batches have completed; jobs still queued (never
  // admitted) complete with `cancelled_status`, so that no waiter is left behind.
  void stop(int cancelled_status = -1) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (stopping_) return;
      stopping_ = true;
    }
    cv_.notify_all();
    for (auto &t : workers_)
      if (t.joinable()) t.join();
    std::lock_guard<std::mutex> lk(mu_);
    const double t = now();
    for (auto &q : queues_) {
      for (Job *j : q) {
        j->status = cancelled_status;
        j->t_admit = j->t_done = t;
        j->done = true;
      }
      q.clear();
    }
    done_cv_.notify_all();
  }

  static double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
  }

  // Queues a job; returns its ticket, or 0 if it can never fit the budget or the lane
  // does not exist.
  uint64_t submit(uint32_t lane, uint64_t footprint, std::shared_ptr<void> payload) {
    std::lock_guard<std::mutex> lk(mu_);
    if (lane >= queues_.size() || footprint > budget_ || stopping_) {
      stats_.refused++;
      return 0;
    }
    auto job = std::make_unique<Job>();
    job->ticket = ++next_ticket_;
    job->lane = lane;
    job->footprint = footprint;
    job->t_submit = now();
    job->payload = std::move(payload);
    Job *raw = job.get();
    jobs_[raw->ticket] = std::move(job);
    queues_[lane].push_back(raw);
    stats_.submitted++;
    cv_.notify_all();
    return raw->ticket;
  }

  // Waits for a job (timeout_ms < 0: no limit).  On completion returns the job, which
  // stays owned here until release(); nullptr on timeout or unknown ticket.
  Job *wait(uint64_t ticket, int timeout_ms) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = jobs_.find(ticket);
    if (it == jobs_.end()) return nullptr;
    Job *job = it->second.get();
    auto ready = [&] { return job->done; };
    if (timeout_ms < 0)
      done_cv_.wait(lk, ready);
    else if (!done_cv_.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
      return nullptr;
    return job;
  }

  void release(uint64_t ticket) {
    std::lock_guard<std::mutex> lk(mu_);
    jobs_.erase(ticket);
  }

  AdmissionStats stats() {
    std::lock_guard<std::mutex> lk(mu_);
    return stats_;
  }

  uint64_t in_use() {
    std::lock_guard<std::mutex> lk(mu_);
    return in_use_;
  }

 private:
  void run(uint32_t lane) {
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      // Admit the longest FIFO prefix that fits the remaining budget, once the lane has
      // room for another batch in flight.
      std::vector<Job *> batch;
      cv_.wait(lk, [&] {
        if (stopping_) return true;
        auto &q = queues_[lane];
        return inflight_[lane] < depth_ && !q.empty() && fits(lane, q.front());
      });
      if (stopping_) return;
      auto &q = queues_[lane];
      while (!q.empty() && batch.size() < max_batch_ && fits(lane, q.front())) {
        Job *j = q.front();
        q.pop_front();
        in_use_ += j->footprint;
        j->t_admit = now();
        batch.push_back(j);
      }
      if (in_use_ > stats_.peak_in_use) stats_.peak_in_use = in_use_;
      inflight_[lane]++;
      lk.unlock();
      exec_(lane, batch);
      lk.lock();
      if (stage2_) {
        handoff_[lane].push_back(std::move(batch));
        cv_.notify_all();
      } else {
        complete(lane, batch);
      }
    }
  }

  // With mu_ held: whether job j of `lane` fits in the budget left beside the footprints
  // of the other lanes' heads that were submitted before it.
  bool fits(uint32_t lane, const Job *j) const {
    uint64_t need = j->footprint;
    for (uint32_t l = 0; l < queues_.size(); l++) {
      if (l == lane || queues_[l].empty()) continue;
      const Job *h = queues_[l].front();
      if (h->ticket < j->ticket) {
        if (need > budget_ - h->footprint) return false;  // more than the whole budget
        need += h->footprint;
      }
    }
    return need <= budget_ - in_use_;
  }

  // Stage 2 of a pipelined lane: in admission order, and drained before stop returns.
  void run_stage2(uint32_t lane) {
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      cv_.wait(lk, [&] { return !handoff_[lane].empty() || (stopping_ && inflight_[lane] == 0); });
      if (handoff_[lane].empty()) return;
      std::vector<Job *> batch = std::move(handoff_[lane].front());
      handoff_[lane].pop_front();
      lk.unlock();
      stage2_(lane, batch);
      lk.lock();
      complete(lane, batch);
    }
  }

  // Called with mu_ held: releases the batch's memory and marks its jobs done.
  void complete(uint32_t lane, std::vector<Job *> &batch) {
    const double t = now();
    for (Job *j : batch) {
      in_use_ -= j->footprint;
      j->t_done = t;
      j->done = true;
    }
    inflight_[lane]--;
    stats_.batches++;
    stats_.completed += batch.size();
    if (batch.size() > stats_.max_batch_seen) stats_.max_batch_seen = batch.size();
    done_cv_.notify_all();
    cv_.notify_all();  // memory and a pipeline slot freed: lanes may admit
  }

  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  const uint64_t budget_;
  const uint32_t max_batch_, depth_;
  Executor exec_, stage2_;
  std::vector<std::deque<Job *>> queues_;
  std::vector<std::deque<std::vector<Job *>>> handoff_;
  std::vector<uint32_t> inflight_;
  std::map<uint64_t, std::unique_ptr<Job>> jobs_;
  std::vector<std::thread> workers_;
  uint64_t in_use_ = 0, next_ticket_ = 0;
  bool stopping_ = false;
  AdmissionStats stats_;
};

}  // namespace xpir
