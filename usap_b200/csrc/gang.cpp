// Gang scheduling of nodal phases: the concurrent solves of
// usap_batch_partition hand their dense nodal phases to one NodalGang,
// which runs many of them in a single cooperative launch (k_nodal_gang)
// instead of each solve issuing three or four kernel launches per batch.
// A solve that reaches its nodal phase waits; the first waiting thread that
// finds no launch in flight starts one for every waiting phase once all
// solves in progress are waiting or kGangMax are, or once the oldest has
// waited kGangWait and no launch has ended for as long.  A launch returns
// when kGangExitFrac of its phases are finished; the others resume at the
// batch where they stopped, in the next launch, with whatever phases have
// arrived meanwhile.
#include <algorithm>
#include <chrono>
#include <cstring>

#include "job.h"

namespace usap {

namespace {
constexpr auto kGangWait = std::chrono::microseconds(3000);
constexpr double kGangExitFrac = 0.35;
}

NodalGang::NodalGang(int device) : device_(device) {
  USAP_CUDA(cudaSetDevice(device));
  grid_ = nodal_gang_grid(device);
  if (grid_ <= 0) throw Error(USAP_ERR_NO_DEVICE, "device cannot run the cooperative nodal kernel");
  USAP_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
  USAP_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h_jobs_), sizeof(PhaseArgs) * kGangMax));
  USAP_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h_ctl_), sizeof(GangCtl)));
  d_jobs_ = static_cast<PhaseArgs*>(dev_alloc(sizeof(PhaseArgs) * kGangMax, st_));
  d_ctl_ = static_cast<GangCtl*>(dev_alloc(sizeof(GangCtl), st_));
}

NodalGang::~NodalGang() {
  cudaSetDevice(device_);
  if (st_) cudaStreamSynchronize(st_);
  dev_free(d_jobs_, st_);
  dev_free(d_ctl_, st_);
  if (st_) cudaStreamSynchronize(st_);
  if (h_jobs_) cudaFreeHost(h_jobs_);
  if (h_ctl_) cudaFreeHost(h_ctl_);
  if (st_) cudaStreamDestroy(st_);
}

void NodalGang::enter() {
  std::lock_guard<std::mutex> lk(mu_);
  live_++;
}

void NodalGang::leave() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    live_--;
  }
  cv_.notify_all();
}

bool NodalGang::ready_to_launch() const {
  if (busy_ || pending_.empty()) return false;
  const int waiting = static_cast<int>(pending_.size());
  if (waiting >= live_ || waiting >= kGangMax) return true;
  const auto now = std::chrono::steady_clock::now();
  return now - pending_.front()->since > kGangWait && now - last_end_ > kGangWait;
}

void NodalGang::run(const PhaseArgs& pa, cudaStream_t job_stream) {
  Pending me;
  me.pa = pa;
  USAP_CUDA(cudaEventCreateWithFlags(&me.ready, cudaEventDisableTiming));
  USAP_CUDA(cudaEventRecord(me.ready, job_stream));
  std::unique_lock<std::mutex> lk(mu_);
  me.since = std::chrono::steady_clock::now();
  pending_.push_back(&me);
  cv_.notify_all();
  while (!me.done) {
    if (ready_to_launch()) {
      busy_ = true;
      // one launch runs phases of one precision mode: the oldest's, and
      // the others of that mode in arrival order
      const int mode = pending_.front()->pa.a.prec;
      std::vector<Pending*> batch;
      for (auto it = pending_.begin(); it != pending_.end() && batch.size() < static_cast<size_t>(kGangMax);) {
        if ((*it)->pa.a.prec == mode) {
          batch.push_back(*it);
          it = pending_.erase(it);
        } else {
          ++it;
        }
      }
      lk.unlock();
      std::string err;
      try {
        launch(batch);
      } catch (const std::exception& e) {
        err = e.what();
      }
      lk.lock();
      // unfinished phases go back to the front of the queue, still oldest
      std::vector<Pending*> again;
      for (size_t i = 0; i < batch.size(); i++) {
        Pending* p = batch[i];
        if (err.empty() && !h_ctl_->finished[i]) {
          again.push_back(p);
          continue;
        }
        p->error = err;
        p->done = true;
      }
      pending_.insert(pending_.begin(), again.begin(), again.end());
      busy_ = false;
      cv_.notify_all();
      continue;
    }
    cv_.wait_for(lk, std::chrono::microseconds(200));
  }
  lk.unlock();
  cudaEventDestroy(me.ready);
  if (!me.error.empty()) throw Error(USAP_ERR_INTERNAL, "gang nodal kernel: " + me.error);
}

void NodalGang::launch(const std::vector<Pending*>& batch) {
  USAP_CUDA(cudaSetDevice(device_));
  const int K = static_cast<int>(batch.size());
  for (int i = 0; i < K; i++) {
    if (!batch[i]->waited) {   // the job's own queued work precedes its first launch
      USAP_CUDA(cudaStreamWaitEvent(st_, batch[i]->ready, 0));
      batch[i]->waited = true;
    }
    h_jobs_[i] = batch[i]->pa;
  }
  const auto t0 = std::chrono::steady_clock::now();
  USAP_CUDA(cudaMemcpyAsync(d_jobs_, h_jobs_, sizeof(PhaseArgs) * K, cudaMemcpyHostToDevice, st_));
  USAP_CUDA(cudaMemsetAsync(d_ctl_, 0, sizeof(GangCtl), st_));
  const int done_to_exit = std::max(1, static_cast<int>(kGangExitFrac * K + 0.5));
  launch_nodal_gang(d_jobs_, K, d_ctl_, K - done_to_exit + 1, grid_, h_jobs_[0].a.prec, st_);
  USAP_CUDA(cudaMemcpyAsync(h_ctl_, d_ctl_, sizeof(GangCtl), cudaMemcpyDeviceToHost, st_));
  USAP_CUDA(cudaStreamSynchronize(st_));
  launches_++;
  jobs_run_ += K;
  last_end_ = std::chrono::steady_clock::now();
  ms_ += std::chrono::duration<double, std::milli>(last_end_ - t0).count();
  if (h_ctl_->bar_err) throw Error(USAP_ERR_INTERNAL, "a grid barrier timed out");
}

}  // namespace usap
