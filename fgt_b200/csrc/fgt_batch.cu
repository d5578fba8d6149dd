// fgt_pfgt_batch: many independent point FGTs in one call.
//
// A single pfgt call on a small point set is latency-bound: tens of small
// kernel launches and a few host round trips for the data-dependent sizes of
// the tree levels and lists leave the GPU mostly idle.  The batch keeps
// several instances in flight at once: a persistent pool of host worker
// threads, each with its own CUDA stream and device workspace (the library's
// per-thread stream and arena), takes instances from one work queue, largest
// first (longest-processing-time order), so the instances' kernels overlap on
// the device.  Each instance runs the same pipeline as fgt_pfgt_c, with the
// same results.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "fgt_b200.h"
#include "fgt_common.cuh"
#include "fgt_prims.cuh"

namespace fgt {
namespace {

constexpr int kMaxWorkers = 32;

// Persistent worker threads: run(n, f) calls f(w) on n workers (w = 0..n-1)
// and returns when all have finished.  Threads are created on first use and
// live until the process exits, so their per-thread streams and workspaces
// are reused by later batches.
class WorkerPool {
 public:
  void run(int n, const std::function<void(int)>& f) {
    std::unique_lock<std::mutex> lk(m_);
    while ((int)threads_.size() < n) {
      const int id = (int)threads_.size();
      threads_.emplace_back([this, id] { loop(id); });
      threads_.back().detach();
    }
    job_ = &f;
    want_ = n;
    left_ = n;
    generation_++;
    cv_.notify_all();
    done_.wait(lk, [this] { return left_ == 0; });
    job_ = nullptr;
  }

 private:
  void loop(int id) {
    int seen = 0;
    for (;;) {
      const std::function<void(int)>* job;
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return generation_ != seen; });
        seen = generation_;
        if (id >= want_) continue;
        job = job_;
      }
      (*job)(id);
      std::lock_guard<std::mutex> lk(m_);
      if (--left_ == 0) done_.notify_all();
    }
  }

  std::mutex m_;
  std::condition_variable cv_, done_;
  std::vector<std::thread> threads_;
  const std::function<void(int)>* job_ = nullptr;
  int want_ = 0, left_ = 0, generation_ = 0;
};

WorkerPool& pool() {
  static WorkerPool* p = new WorkerPool();  // never destroyed: its threads outlive main
  return *p;
}
std::mutex g_batch_mutex;  // one batch at a time shares the pool

}  // namespace
}  // namespace fgt

extern "C" int fgt_pfgt_batch(const fgt_opts* opts, int ninst, fgt_instance* inst, int nworkers) {
  using namespace fgt;
  if (ninst < 0 || (ninst > 0 && !inst)) {
    fgt_set_error_message("fgt_pfgt_batch: bad instance array", __FILE__, __LINE__);
    return FGT_ERR_ARG;
  }
  if (ninst == 0) return FGT_OK;
  fgt_opts o;
  fgt_opts_default(&o);
  if (opts) o = *opts;
  // the workers run on their own streams and report no per-call statistics
  o.stream = nullptr;
  o.stats = nullptr;
  o.timing = 0;
  if (o.device < 0) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      (void)cudaGetLastError();
      fgt_set_error_message("no CUDA device", __FILE__, __LINE__);
      for (int i = 0; i < ninst; i++) inst[i].status = FGT_ERR_NODEVICE;
      return FGT_ERR_NODEVICE;
    }
    if (cudaGetDevice(&o.device) != cudaSuccess) o.device = 0;
  }
  // default: 12 workers (the measured throughput of the 512-instance batched
  // workload levels off there: per-instance host round trips and launch
  // serialisation in the runtime bound it), at most the host's threads
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  int nw = nworkers > 0 ? nworkers : std::min(12, hw);
  nw = std::max(1, std::min({nw, kMaxWorkers, ninst}));
  // largest instances first
  std::vector<int> order(ninst);
  for (int i = 0; i < ninst; i++) order[i] = i;
  auto weight = [&](int i) { return (long long)inst[i].ns + (inst[i].ifpghtarg > 0 ? inst[i].nt : 0); };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return weight(a) > weight(b); });
  std::atomic<int> next(0);
  auto run_all = [&](int nwk, const std::function<void(int)>& w) {
    next = 0;
    std::lock_guard<std::mutex> lk(g_batch_mutex);
    if (nwk == 1) w(0);
    else pool().run(nwk, w);
  };
  auto work = [&](int) {
    for (;;) {
      const int k = next.fetch_add(1);
      if (k >= ninst) break;
      fgt_instance& x = inst[order[k]];
      x.status = fgt_pfgt_c(&o, x.nd, x.dim, x.delta, x.eps, x.iperiod, x.bs0, x.cen0, x.ns,
                            x.sources, x.ifcharge, x.charge, x.ifdipole, x.rnormal, x.dipstr,
                            x.ifpgh, x.pot, x.grad, x.hess, x.nt, x.targ, x.ifpghtarg, x.pottarg,
                            x.gradtarg, x.hesstarg);
    }
  };
  // autotuner: the worker count of this batch class (instance count and
  // total points, powers of two), timed over whole batches on the host
  // clock (the instances run on many streams) after a warm-up batch
  if (o.autotune > 0 && nworkers <= 0 && ninst > 1) {
    long long tot = 0;
    for (int i = 0; i < ninst; i++) tot += weight(i);
    int lg = 0, lgi = 0;
    while ((1ll << (lg + 1)) <= tot) lg++;
    while ((1 << (lgi + 1)) <= ninst) lgi++;
    char key[96];
    snprintf(key, sizeof(key), "batch/v1 lg2inst=%d lg2pts=%d", lgi, lg);
    int v = 0;
    if (tune_lookup(key, v)) {
      nw = std::max(1, std::min({v, kMaxWorkers, ninst}));
    } else if (o.autotune >= 2) {
      run_all(nw, work);  // warm-up: streams, workspaces, modules
      double best_t = 1e30;
      int best = nw;
      for (int cand : {4, 8, 12, 16, 24}) {
        const int c = std::max(1, std::min({cand, kMaxWorkers, ninst, hw}));
        const auto t0 = std::chrono::steady_clock::now();
        run_all(c, work);
        cudaDeviceSynchronize();
        const double t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (t < best_t) {
          best_t = t;
          best = c;
        }
      }
      tune_store(key, best);
      nw = best;
    }
  }
  run_all(nw, work);
  for (int i = 0; i < ninst; i++)
    if (inst[i].status != FGT_OK) return inst[i].status;
  return FGT_OK;
}
