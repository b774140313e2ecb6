// Host-side check of the serving loop's admission and continuous batching
// (xpir_b200/csrc/admission.h), compiled with g++ and driven by a fake executor:
//   1. jobs run in FIFO order per lane and every job completes with the executor's status;
//   2. the bytes admitted at once never exceed the budget;
//   3. a job larger than the whole budget is refused at submission;
//   4. jobs that arrive while a batch runs are admitted together in a later batch
//      (continuous batching), never more than max_batch at a time;
//   5. lanes run concurrently (two lanes' batches overlap in time);
//   6. a head-of-line job that does not fit waits for memory rather than being skipped;
//   7. as a two-stage pipeline (depth 2), stage 1 of a lane's next batch overlaps stage 2
//      of its current one, at most two batches per lane are in flight, stage 2 sees the
//      batches in admission order, and every job completes;
//   8. a job waiting for memory at the head of one lane is not overtaken by jobs submitted
//      after it on another lane;
//   9. stopping runs the admitted jobs to completion and completes the queued ones with
//      the cancellation status.
#include <stdio.h>

#include <atomic>
#include <chrono>
#include <thread>
#include <vector>

#include "../../xpir_b200/csrc/admission.h"

#define CHECK(c)                                                \
  do {                                                          \
    if (!(c)) {                                                 \
      printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c);       \
      return 1;                                                 \
    }                                                           \
  } while (0)

namespace {

struct Trace {
  std::mutex mu;
  std::vector<std::vector<uint64_t>> batches[2];  // tickets per batch, per lane
  std::atomic<uint64_t> in_use{0}, peak{0};
  std::atomic<int> active_lanes{0}, max_active_lanes{0};
};

}  // namespace

int main() {
  using xpir::Admission;
  using xpir::Job;
  Trace tr;
  std::atomic<int> delay_ms{20};
  const uint64_t budget = 1000;
  Admission adm(2, budget, 4, [&](uint32_t lane, std::vector<Job *> &batch) {
    uint64_t bytes = 0;
    std::vector<uint64_t> ids;
    for (Job *j : batch) {
      bytes += j->footprint;
      ids.push_back(j->ticket);
    }
    const uint64_t now = tr.in_use += bytes;
    uint64_t pk = tr.peak.load();
    while (now > pk && !tr.peak.compare_exchange_weak(pk, now)) {
    }
    const int a = ++tr.active_lanes;
    int ma = tr.max_active_lanes.load();
    while (a > ma && !tr.max_active_lanes.compare_exchange_weak(ma, a)) {
    }
    std::this_thread::sleep_for(std::chrono::milliseconds(delay_ms.load()));
    --tr.active_lanes;
    tr.in_use -= bytes;
    {
      std::lock_guard<std::mutex> lk(tr.mu);
      tr.batches[lane].push_back(ids);
    }
    for (Job *j : batch) j->status = (int)(j->ticket % 7);  // executor-chosen status
  });

  // 3. Oversize refusal.
  CHECK(adm.submit(0, budget + 1, nullptr) == 0);
  CHECK(adm.submit(5, 1, nullptr) == 0);  // no such lane

  // 1, 2, 4, 5. A burst on both lanes while the first batches run.
  std::vector<uint64_t> tickets[2];
  for (int i = 0; i < 40; i++)
    for (uint32_t lane = 0; lane < 2; lane++) {
      const uint64_t t = adm.submit(lane, 100 + 37 * (i % 5), nullptr);
      CHECK(t != 0);
      tickets[lane].push_back(t);
    }
  for (uint32_t lane = 0; lane < 2; lane++)
    for (uint64_t t : tickets[lane]) {
      Job *j = adm.wait(t, 20000);
      CHECK(j != nullptr);
      CHECK(j->done);
      CHECK(j->status == (int)(t % 7));
      CHECK(j->t_submit <= j->t_admit && j->t_admit <= j->t_done);
      adm.release(t);
    }
  CHECK(adm.wait(tickets[0][0], 0) == nullptr);  // released: unknown now
  const xpir::AdmissionStats st = adm.stats();
  CHECK(st.completed == 80);
  CHECK(st.refused == 2);
  CHECK(st.peak_in_use <= budget);
  CHECK(tr.peak.load() <= budget);
  CHECK(st.max_batch_seen > 1 && st.max_batch_seen <= 4);  // batching happened, capped
  CHECK(tr.max_active_lanes.load() == 2);                   // lanes overlapped
  CHECK(adm.in_use() == 0);
  {
    std::lock_guard<std::mutex> lk(tr.mu);
    for (int lane = 0; lane < 2; lane++) {
      std::vector<uint64_t> order;
      for (auto &b : tr.batches[lane]) order.insert(order.end(), b.begin(), b.end());
      CHECK(order == tickets[lane]);  // FIFO per lane, each job exactly once
    }
  }

  // 6. Head-of-line blocking by memory: a job needing the whole budget waits until the
  // lane-1 jobs in flight release theirs, and the small job behind it (lane 0) is not
  // admitted ahead of it.
  delay_ms = 50;
  const uint64_t a = adm.submit(1, 600, nullptr);
  std::this_thread::sleep_for(std::chrono::milliseconds(10));
  const uint64_t big = adm.submit(0, budget, nullptr);
  const uint64_t small = adm.submit(0, 10, nullptr);
  CHECK(a && big && small);
  Job *ja = adm.wait(a, 20000);
  Job *jb = adm.wait(big, 20000);
  Job *js = adm.wait(small, 20000);
  CHECK(ja && jb && js);
  CHECK(jb->t_admit >= ja->t_done);  // waited for memory
  CHECK(js->t_admit >= jb->t_admit);  // FIFO: not overtaken
  adm.release(a);
  adm.release(big);
  adm.release(small);

  // 8. Across lanes: a job needing the whole budget at the head of lane 0 is not starved
  // by jobs submitted after it on lanes 1 and 2, whose batches would otherwise overlap so
  // that the budget never empties: none of them is admitted before it.
  {
    Admission three(3, budget, 1, [&](uint32_t, std::vector<Job *> &batch) {
      std::this_thread::sleep_for(std::chrono::milliseconds(15));
      for (Job *j : batch) j->status = 0;
    });
    const uint64_t a1 = three.submit(1, 300, nullptr);
    std::this_thread::sleep_for(std::chrono::milliseconds(7));  // staggered: the lanes' batches interleave
    const uint64_t a2 = three.submit(2, 300, nullptr);
    std::this_thread::sleep_for(std::chrono::milliseconds(2));
    const uint64_t whole = three.submit(0, budget, nullptr);
    std::vector<uint64_t> later;
    for (int i = 0; i < 10; i++) later.push_back(three.submit(1 + i % 2, 300, nullptr));
    Job *jw = three.wait(whole, 20000);
    CHECK(a1 && a2 && jw);
    for (uint64_t t : later) {
      Job *j = three.wait(t, 20000);
      CHECK(j && j->t_admit >= jw->t_admit);
    }
    CHECK(three.stats().peak_in_use <= budget);
    three.stop();
  }

  // 9. Stopping: the admitted job runs to completion, the queued ones complete with the
  // cancellation status, and every waiter returns.
  {
    Admission one(1, budget, 1, [&](uint32_t, std::vector<Job *> &batch) {
      std::this_thread::sleep_for(std::chrono::milliseconds(30));
      for (Job *j : batch) j->status = 3;
    });
    const uint64_t t1 = one.submit(0, 10, nullptr);
    std::this_thread::sleep_for(std::chrono::milliseconds(5));  // t1 admitted
    const uint64_t t2 = one.submit(0, 10, nullptr), t3 = one.submit(0, 10, nullptr);
    one.stop(-5);
    Job *j1 = one.wait(t1, 1000), *j2 = one.wait(t2, 1000), *j3 = one.wait(t3, 1000);
    CHECK(j1 && j2 && j3);
    CHECK(j1->status == 3 && j2->status == -5 && j3->status == -5);
  }

  // Timeout: a job that cannot finish within the wait's limit.
  delay_ms = 300;
  const uint64_t slow = adm.submit(0, 1, nullptr);
  CHECK(adm.wait(slow, 10) == nullptr);
  CHECK(adm.wait(slow, 20000) != nullptr);
  adm.release(slow);
  adm.stop();
  CHECK(adm.submit(0, 1, nullptr) == 0);  // stopped: refused
  const unsigned long long plain_batches = adm.stats().batches;

  // 7. Two-stage pipeline.
  {
    std::mutex mu;
    std::atomic<int> inflight[2] = {{0}, {0}}, max_inflight{0}, overlaps{0};
    std::atomic<int> in_stage2[2] = {{0}, {0}};
    std::vector<uint64_t> order[2];
    Admission pipe(
        2, budget, 3,
        [&](uint32_t lane, std::vector<Job *> &batch) {
          const int f = ++inflight[lane];
          int mx = max_inflight.load();
          while (f > mx && !max_inflight.compare_exchange_weak(mx, f)) {
          }
          if (in_stage2[lane].load()) overlaps++;
          std::this_thread::sleep_for(std::chrono::milliseconds(8));
          for (Job *j : batch) j->status = 1;  // stage 1 done
        },
        [&](uint32_t lane, std::vector<Job *> &batch) {
          in_stage2[lane] = 1;
          std::this_thread::sleep_for(std::chrono::milliseconds(20));
          {
            std::lock_guard<std::mutex> lk(mu);
            for (Job *j : batch) order[lane].push_back(j->ticket);
          }
          for (Job *j : batch) j->status = j->status == 1 ? 2 : -1;
          in_stage2[lane] = 0;
          --inflight[lane];
        },
        2);
    std::vector<uint64_t> t2[2];
    for (int i = 0; i < 30; i++) {
      for (uint32_t lane = 0; lane < 2; lane++) t2[lane].push_back(pipe.submit(lane, 50 + 13 * (i % 4), nullptr));
      std::this_thread::sleep_for(std::chrono::milliseconds(3));
    }
    for (uint32_t lane = 0; lane < 2; lane++)
      for (uint64_t t : t2[lane]) {
        Job *j = pipe.wait(t, 20000);
        CHECK(j && j->status == 2);
        pipe.release(t);
      }
    CHECK(max_inflight.load() <= 2);
    CHECK(overlaps.load() > 0);
    CHECK(pipe.stats().completed == 60 && pipe.stats().peak_in_use <= budget);
    for (int lane = 0; lane < 2; lane++) CHECK(order[lane] == t2[lane]);
    pipe.stop();
  }
  printf("ok %llu batches\n", plain_batches);
  return 0;
}
