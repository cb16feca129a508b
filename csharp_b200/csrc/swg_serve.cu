// Serving: query batches against the device-resident sequence set (the database), with
// continuous batching.
//
// A job (one sw_submit_job call) is a batch of queries.  Its life:
//   pending  -> admitted once it gets a query slot per query, room in the query arena for its
//               residues and device memory for its result (nq x database Int16);
//   admitted -> its work items (query, database chunk) are handed out to waves.  A wave is one
//               enqueue of the persistent per-K kernels over items of every admitted job: each
//               job gets an equal share of the wave's time budget, the rest goes to whoever still
//               has items, so a small job admitted while a large one runs finishes in its first
//               wave or two instead of queueing behind it.  Two waves are in flight at a time,
//               on two streams with their own scratch, so the next wave's CTAs take the SMs
//               that the current wave's tail leaves idle;
//   copying  -> its last wave finished: a second thread copies the result to the caller's buffer
//               and frees the job's device memory, slots and arena bytes;
//   done     -> sw_poll reports it and forgets the ticket.
// Jobs that arrive while waves run are admitted at the next wave boundary.
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/swgb200.h"
#include "swg_engine.h"
#include "swg_serve.h"

namespace swg {

namespace {

struct Job {
  int64_t ticket = 0;
  int nq = 0;
  std::vector<uint8_t> residues;
  std::vector<int64_t> offsets;
  int16_t* out = nullptr;
  int64_t ld = 0;
  // admitted state
  std::vector<int> slots;
  int64_t arena_off = -1, arena_bytes = 0;
  int16_t* d_out = nullptr;
  size_t out_bytes = 0;
  std::vector<QueryItem> items;
  size_t next_item = 0;
  int64_t outstanding = 0;  // items handed to waves that have not finished
  // report
  sw_job_info info;
  bool done = false;
};

struct Wave {
  cudaEvent_t ev = nullptr;
  int buf = 0;
  std::vector<std::pair<Job*, int64_t>> parts;  // items of each job in this wave
};

double now_s(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

class ServerImpl : public Server {
 public:
  ~ServerImpl() override { shutdown(); }

  int init(const EngineParams& db, int device, const ServeOptions& opt, std::string* msg) {
    device_ = device;
    opt_ = opt;
    db_count_ = db.nseq;
    t0_ = std::chrono::steady_clock::now();
    cudaSetDevice(device_);
    int rc = 0;
    runner_.reset(QueryRunner::create(db, msg, &rc));
    if (!runner_) return rc ? rc : SW_E_OOM;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    budget_ = opt.memory_bytes ? opt.memory_bytes : free_b / 2;
    const int S = std::max(1, opt.slots);
    if (cudaStreamCreateWithFlags(&st_[0], cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&st_[1], cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&copy_st_, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&up_st_, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&d_arena_, std::max<size_t>(opt.arena_bytes, 64) + 64) != cudaSuccess ||
        cudaMalloc(&d_qoff_, sizeof(int64_t) * S) != cudaSuccess ||
        cudaMalloc(&d_qlen_, sizeof(int32_t) * S) != cudaSuccess ||
        cudaMalloc(&d_qout_, sizeof(int16_t*) * S) != cudaSuccess ||
        cudaMallocHost(&h_qoff_, sizeof(int64_t) * S) != cudaSuccess ||
        cudaMallocHost(&h_qlen_, sizeof(int32_t) * S) != cudaSuccess ||
        cudaMallocHost(&h_qout_, sizeof(int16_t*) * S) != cudaSuccess) {
      cudaGetLastError();
      *msg = "serving buffers";
      return SW_E_OOM;
    }
    std::memset(h_qoff_, 0, sizeof(int64_t) * S);
    std::memset(h_qlen_, 0, sizeof(int32_t) * S);
    std::memset(h_qout_, 0, sizeof(int16_t*) * S);
    for (int s = S - 1; s >= 0; s--) free_slots_.push_back(s);
    arena_free_[0] = (int64_t)std::max<size_t>(opt.arena_bytes, 64);
    for (int b = 0; b < 2; b++)
      if (cudaEventCreateWithFlags(&wave_ev_[b], cudaEventDisableTiming | cudaEventBlockingSync) != cudaSuccess) {
        *msg = "event create";
        return SW_E_CUDA;
      }
    sched_ = std::thread([this] { schedule_loop(); });
    copier_ = std::thread([this] { copy_loop(); });
    return SW_OK;
  }

  int submit(const uint8_t* q, const int64_t* off, int nq, int16_t* out, int64_t ld,
             int64_t* ticket, std::string* msg) override {
    std::unique_ptr<Job> j(new Job());
    j->nq = nq;
    j->offsets.assign(off, off + nq + 1);
    j->residues.assign(q, q + off[nq]);
    j->out = out;
    j->ld = ld;
    std::memset(&j->info, 0, sizeof(j->info));
    j->info.queries = nq;
    j->info.pairs = (int64_t)nq * db_count_;
    for (int i = 0; i < nq; i++) j->info.cells += runner_->query_cells((int)(off[i + 1] - off[i]));
    if (nq > opt_.slots) { *msg = "more queries than serving slots"; return SW_E_UNSUPPORTED; }
    if ((size_t)(off[nq] + 16 * nq) > opt_.arena_bytes) { *msg = "queries exceed the query arena"; return SW_E_UNSUPPORTED; }
    if ((size_t)nq * db_count_ * 2 > budget_) { *msg = "result exceeds the serving memory budget"; return SW_E_UNSUPPORTED; }
    std::lock_guard<std::mutex> lk(mu_);
    if (error_) { *msg = error_msg_; return error_; }
    j->ticket = ++last_ticket_;
    j->info.submit_s = now_s(t0_);
    *ticket = j->ticket;
    stats_.submitted++;
    pending_.push_back(j.get());
    jobs_[j->ticket] = std::move(j);
    cv_sched_.notify_all();
    return SW_OK;
  }

  int poll(int64_t ticket, int timeout_ms, int* done, sw_job_info* info) override {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = jobs_.find(ticket);
    if (it == jobs_.end()) return SW_E_ARG;
    Job* j = it->second.get();
    if (!j->done && timeout_ms > 0)
      cv_done_.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return j->done; });
    *done = j->done ? 1 : 0;
    if (!j->done) return SW_OK;
    if (info) *info = j->info;
    const int st = j->info.status;
    jobs_.erase(it);
    return st;
  }

  void stats(sw_serve_counters* s) override {
    std::lock_guard<std::mutex> lk(mu_);
    *s = stats_;
    s->active = (int32_t)active_.size();
    s->pending = (int32_t)pending_.size();
  }

  void drain() override {
    std::unique_lock<std::mutex> lk(mu_);
    cv_done_.wait(lk, [&] { return pending_.empty() && active_.empty() && copying_.empty(); });
  }

 private:
  // ---- scheduler thread --------------------------------------------------------------------
  void schedule_loop() {
    cudaSetDevice(device_);
    std::deque<Wave> inflight;
    int next_buf = 0;
    for (;;) {
      Wave w;
      {
        std::unique_lock<std::mutex> lk(mu_);
        if (stop_ && inflight.empty()) break;
        if (!stop_) admit_locked();
        if (!stop_ && inflight.size() < 2) form_wave_locked(&w);
        if (w.parts.empty() && inflight.empty()) {
          cv_sched_.wait(lk, [&] { return stop_ || (!pending_.empty() && can_admit_locked(pending_.front())) || has_items_locked(); });
          continue;
        }
      }
      if (!w.parts.empty()) {
        w.buf = next_buf;
        next_buf ^= 1;
        w.ev = wave_ev_[w.buf];
        std::string msg;
        const int rc = launch(w, &msg);
        if (rc) { fail_all(rc, msg); inflight.clear(); continue; }
        inflight.push_back(w);
        continue;
      }
      // two waves queued (or no work to add): wait for the oldest
      Wave& old = inflight.front();
      const cudaError_t e = cudaEventSynchronize(old.ev);
      if (e != cudaSuccess) {
        fail_all(SW_E_CUDA, std::string("serving wave: ") + cudaGetErrorString(e));
        inflight.clear();
        continue;
      }
      std::lock_guard<std::mutex> lk(mu_);
      for (auto& pr : old.parts) {
        Job* j = pr.first;
        j->outstanding -= pr.second;
        if (j->outstanding == 0 && j->next_item == j->items.size()) {
          active_.erase(std::find(active_.begin(), active_.end(), j));
          copying_.push_back(j);
          cv_copy_.notify_all();
        }
      }
      inflight.pop_front();
    }
  }

  bool has_items_locked() const {
    for (Job* j : active_)
      if (j->next_item < j->items.size()) return true;
    return false;
  }

  bool can_admit_locked(const Job* j) const {
    if ((int)free_slots_.size() < j->nq) return false;
    if (in_use_ + (size_t)j->nq * db_count_ * 2 > budget_) return false;
    const int64_t need = arena_need(j);
    for (auto& kv : arena_free_)
      if (kv.second >= need) return true;
    return false;
  }

  static int64_t arena_need(const Job* j) { return ((j->offsets[j->nq] + 16 * j->nq) + 15) / 16 * 16; }

  // First come, first admitted: a job that does not fit holds back the ones behind it.
  void admit_locked() {
    while (!pending_.empty() && can_admit_locked(pending_.front())) {
      Job* j = pending_.front();
      const int64_t need = arena_need(j);
      auto a = arena_free_.begin();
      while (a->second < need) ++a;
      j->arena_off = a->first;
      j->arena_bytes = need;
      if (a->second > need) arena_free_[a->first + need] = a->second - need;
      arena_free_.erase(a);
      j->out_bytes = std::max<size_t>((size_t)j->nq * db_count_ * 2, 2);
      // allocated on the upload stream, which is synchronized below: usable by both wave streams
      if (cudaMallocAsync(reinterpret_cast<void**>(&j->d_out), j->out_bytes, up_st_) != cudaSuccess) {
        cudaGetLastError();
        release_locked(j);
        j->info.status = SW_E_OOM;
        pending_.pop_front();
        finish_locked(j);
        continue;
      }
      in_use_ += (size_t)j->nq * db_count_ * 2;
      // residues into the arena, 16-byte aligned per query; slot tables point at them
      std::vector<uint8_t> packed((size_t)need, (uint8_t)127);
      int64_t p = 0;
      for (int i = 0; i < j->nq; i++) {
        const int slot = free_slots_.back();
        free_slots_.pop_back();
        j->slots.push_back(slot);
        const int64_t len = j->offsets[i + 1] - j->offsets[i];
        std::memcpy(packed.data() + p, j->residues.data() + j->offsets[i], (size_t)len);
        h_qoff_[slot] = j->arena_off + p;
        h_qlen_[slot] = (int32_t)len;
        h_qout_[slot] = j->d_out + (size_t)i * db_count_;
        p += (len + 15) / 16 * 16;
        runner_->plan_query(slot, (int)len, &j->items);
      }
      tables_dirty_ = true;
      // on the upload stream (the wave stream may hold running waves); done before any wave
      // that reads it is enqueued
      if (cudaMemcpyAsync(d_arena_ + j->arena_off, packed.data(), (size_t)need, cudaMemcpyHostToDevice, up_st_) != cudaSuccess ||
          cudaStreamSynchronize(up_st_) != cudaSuccess) {
        cudaGetLastError();
        j->info.status = SW_E_CUDA;
      }
      j->info.admit_s = now_s(t0_);
      pending_.pop_front();
      active_.push_back(j);
      stats_.max_active = std::max<int32_t>(stats_.max_active, (int32_t)active_.size());
      if (j->info.status) j->items.clear();  // the upload failed: report it, free the job
      if (j->items.empty()) {  // an empty database (or a failed job): nothing to compute
        active_.pop_back();
        copying_.push_back(j);
        cv_copy_.notify_all();
      }
    }
  }

  // An equal share of the wave's budget for every admitted job with work left, then the rest
  // in admission order.
  void form_wave_locked(Wave* w) {
    std::vector<Job*> js;
    for (Job* j : active_)
      if (j->next_item < j->items.size()) js.push_back(j);
    if (js.empty()) return;
    const double budget = std::max(1e-4, opt_.wave_seconds);
    const double share = budget / (double)js.size();
    std::vector<int64_t> taken(js.size(), 0);
    double total = 0;
    for (int round = 0; round < 2; round++)
      for (size_t x = 0; x < js.size(); x++) {
        Job* j = js[x];
        double got = 0;
        while (j->next_item < j->items.size()) {
          const double c = j->items[j->next_item].cost;
          if (round == 0 ? (got > 0 && got + c > share) : (total + c > budget)) break;
          wave_items_.push_back(j->items[j->next_item++]);
          got += c;
          total += c;
          taken[x]++;
        }
      }
    for (size_t x = 0; x < js.size(); x++)
      if (taken[x]) {
        w->parts.push_back({js[x], taken[x]});
        js[x]->outstanding += taken[x];
        js[x]->info.waves++;
      }
    stats_.waves++;
  }

  int launch(Wave& w, std::string* msg) {
    const int S = opt_.slots;
    {
      // Entries of slots in use never change, so waves still reading the device tables see the
      // same values; the copy ends before this wave is enqueued and before the mirrors change.
      std::lock_guard<std::mutex> lk(mu_);
      if (tables_dirty_) {
        if (cudaMemcpyAsync(d_qoff_, h_qoff_, sizeof(int64_t) * S, cudaMemcpyHostToDevice, up_st_) != cudaSuccess ||
            cudaMemcpyAsync(d_qlen_, h_qlen_, sizeof(int32_t) * S, cudaMemcpyHostToDevice, up_st_) != cudaSuccess ||
            cudaMemcpyAsync(d_qout_, h_qout_, sizeof(int16_t*) * S, cudaMemcpyHostToDevice, up_st_) != cudaSuccess ||
            cudaStreamSynchronize(up_st_) != cudaSuccess) {
          *msg = "slot table upload";
          return SW_E_CUDA;
        }
        tables_dirty_ = false;
      }
    }
    QueryTables T;
    T.qseq = d_arena_;
    T.qoff = d_qoff_;
    T.qlen = d_qlen_;
    T.qout = d_qout_;
    std::vector<QueryItem> items;
    items.swap(wave_items_);
    int rc = runner_->enqueue(w.buf, items, T, st_[w.buf], msg);
    if (rc) return rc;
    if (cudaEventRecord(w.ev, st_[w.buf]) != cudaSuccess) { *msg = "wave event"; return SW_E_CUDA; }
    return SW_OK;
  }

  // ---- copy thread ---------------------------------------------------------------------------
  void copy_loop() {
    cudaSetDevice(device_);
    for (;;) {
      Job* j = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_copy_.wait(lk, [&] { return stop_copy_ || !copying_.empty(); });
        if (copying_.empty()) break;
        j = copying_.front();
      }
      int status = SW_OK;
      if (j->nq && db_count_ && !j->info.status) {
        cudaError_t e = cudaMemcpy2DAsync(j->out, (size_t)j->ld * 2, j->d_out, (size_t)db_count_ * 2,
                                          (size_t)db_count_ * 2, (size_t)j->nq, cudaMemcpyDeviceToHost, copy_st_);
        if (e == cudaSuccess) e = cudaStreamSynchronize(copy_st_);
        if (e != cudaSuccess) status = SW_E_CUDA;
      }
      if (j->d_out) cudaFreeAsync(j->d_out, copy_st_);
      j->d_out = nullptr;
      std::lock_guard<std::mutex> lk(mu_);
      copying_.pop_front();
      release_locked(j);
      in_use_ -= (size_t)j->nq * db_count_ * 2;
      if (!j->info.status) j->info.status = status;
      finish_locked(j);
      cv_sched_.notify_all();
    }
  }

  void release_locked(Job* j) {
    for (int s : j->slots) {
      h_qlen_[s] = 0;
      free_slots_.push_back(s);
    }
    j->slots.clear();
    if (j->arena_off >= 0) {
      // return the range and merge it with free neighbours
      auto it = arena_free_.emplace(j->arena_off, j->arena_bytes).first;
      auto nx = std::next(it);
      if (nx != arena_free_.end() && it->first + it->second == nx->first) {
        it->second += nx->second;
        arena_free_.erase(nx);
      }
      if (it != arena_free_.begin()) {
        auto pv = std::prev(it);
        if (pv->first + pv->second == it->first) {
          pv->second += it->second;
          arena_free_.erase(it);
        }
      }
      j->arena_off = -1;
    }
  }

  void finish_locked(Job* j) {
    j->info.done_s = now_s(t0_);
    j->done = true;
    stats_.completed++;
    if (!j->info.status) stats_.cells += j->info.cells;
    j->residues.clear();
    j->residues.shrink_to_fit();
    j->items.clear();
    j->items.shrink_to_fit();
    cv_done_.notify_all();
  }

  void fail_all(int rc, const std::string& msg) {
    cudaGetLastError();
    cudaStreamSynchronize(st_[0]);  // nothing may still use the memory the copy thread frees
    cudaStreamSynchronize(st_[1]);
    cudaGetLastError();
    std::lock_guard<std::mutex> lk(mu_);
    error_ = rc;
    error_msg_ = msg;
    for (Job* j : pending_) { j->info.status = rc; finish_locked(j); }
    pending_.clear();
    for (Job* j : active_) {
      j->info.status = rc;
      j->next_item = j->items.size();
      j->outstanding = 0;
      copying_.push_back(j);  // the copy thread frees its memory and reports it
    }
    active_.clear();
    cv_copy_.notify_all();
  }

  void shutdown() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
      cv_sched_.notify_all();
    }
    if (sched_.joinable()) sched_.join();
    {
      std::lock_guard<std::mutex> lk(mu_);
      // admitted jobs whose items were not all handed out end unfinished
      for (Job* j : active_) {
        if (!j->info.status) j->info.status = SW_E_STATE;
        copying_.push_back(j);
      }
      active_.clear();
      for (Job* j : pending_) { j->info.status = SW_E_STATE; finish_locked(j); }
      pending_.clear();
      stop_copy_ = true;
      cv_copy_.notify_all();
    }
    if (copier_.joinable()) copier_.join();
    cudaSetDevice(device_);
    for (cudaStream_t s : st_) if (s) cudaStreamSynchronize(s);
    if (copy_st_) cudaStreamSynchronize(copy_st_);
    runner_.reset();
    for (int b = 0; b < 2; b++) if (wave_ev_[b]) cudaEventDestroy(wave_ev_[b]);
    cudaFree(d_arena_); cudaFree(d_qoff_); cudaFree(d_qlen_); cudaFree(d_qout_);
    cudaFreeHost(h_qoff_); cudaFreeHost(h_qlen_); cudaFreeHost(h_qout_);
    for (cudaStream_t& s : st_) { if (s) cudaStreamDestroy(s); s = nullptr; }
    if (copy_st_) cudaStreamDestroy(copy_st_);
    if (up_st_) cudaStreamDestroy(up_st_);
    copy_st_ = up_st_ = nullptr;
  }

  int device_ = 0;
  ServeOptions opt_;
  int db_count_ = 0;
  size_t budget_ = 0, in_use_ = 0;
  std::chrono::steady_clock::time_point t0_;
  std::unique_ptr<QueryRunner> runner_;
  cudaStream_t st_[2] = {nullptr, nullptr};  // wave streams: the two buffers' waves overlap
  cudaStream_t copy_st_ = nullptr, up_st_ = nullptr;
  cudaEvent_t wave_ev_[2] = {nullptr, nullptr};
  uint8_t* d_arena_ = nullptr;
  int64_t* d_qoff_ = nullptr;
  int32_t* d_qlen_ = nullptr;
  int16_t** d_qout_ = nullptr;
  int64_t* h_qoff_ = nullptr;
  int32_t* h_qlen_ = nullptr;
  int16_t** h_qout_ = nullptr;
  bool tables_dirty_ = true;
  std::vector<QueryItem> wave_items_;

  std::mutex mu_;
  std::condition_variable cv_sched_, cv_copy_, cv_done_;
  bool stop_ = false, stop_copy_ = false;
  int error_ = 0;
  std::string error_msg_;
  int64_t last_ticket_ = 0;
  std::map<int64_t, std::unique_ptr<Job>> jobs_;
  std::deque<Job*> pending_, copying_;
  std::vector<Job*> active_;
  std::vector<int> free_slots_;
  std::map<int64_t, int64_t> arena_free_;  // offset -> bytes
  sw_serve_counters stats_ = {};
  std::thread sched_, copier_;
};

}  // namespace

Server* Server::create(const EngineParams& db, int device, const ServeOptions& opt, std::string* msg, int* rc) {
  ServerImpl* s = new (std::nothrow) ServerImpl();
  if (!s) { *rc = SW_E_OOM; *msg = "server"; return nullptr; }
  if ((*rc = s->init(db, device, opt, msg))) { delete s; return nullptr; }
  return s;
}

}  // namespace swg
