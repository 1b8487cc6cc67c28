// The served form (include/visar_serve.h): a scheduler thread over a device
// pool, admitting requests by their memory needs and batching them per stage
// through the batch engine's stage builder and persistent launches.
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/visar_serve.h"
#include "batch_plan.h"

namespace vb {
namespace sv {

using namespace bt;

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// Best-fit allocator over one device block (256-byte granules).
class DevPool {
 public:
  ~DevPool() {
    if (base_) cudaFree(base_);
  }
  cudaError_t init(size_t cap) {
    cap_ = cap & ~(size_t)255;
    cudaError_t e = cudaMalloc(&base_, cap_);
    if (e != cudaSuccess) {
      base_ = nullptr;
      return e;
    }
    insert_free(0, cap_);
    return cudaSuccess;
  }
  void *alloc(size_t bytes) {
    bytes = std::max<size_t>(256, (bytes + 255) & ~(size_t)255);
    auto it = by_size_.lower_bound(bytes);
    if (it == by_size_.end()) return nullptr;
    const size_t len = it->first, off = it->second;
    by_size_.erase(it);
    by_off_.erase(off);
    if (len > bytes) insert_free(off + bytes, len - bytes);
    sizes_[off] = bytes;
    used_ += bytes;
    return base_ + off;
  }
  void free(void *p) {
    if (!p) return;
    const size_t off = static_cast<uint8_t *>(p) - base_;
    auto it = sizes_.find(off);
    if (it == sizes_.end()) return;
    size_t len = it->second, start = off;
    sizes_.erase(it);
    used_ -= len;
    // Coalesce with the neighbours.
    auto nx = by_off_.find(start + len);
    if (nx != by_off_.end()) {
      len += nx->second;
      erase_free(nx->first, nx->second);
    }
    auto pv = by_off_.lower_bound(start);
    if (pv != by_off_.begin()) {
      --pv;
      if (pv->first + pv->second == start) {
        start = pv->first;
        len += pv->second;
        erase_free(pv->first, pv->second);
      }
    }
    insert_free(start, len);
  }
  size_t cap() const { return cap_; }
  size_t used() const { return used_; }

 private:
  void insert_free(size_t off, size_t len) {
    by_off_[off] = len;
    by_size_.emplace(len, off);
  }
  void erase_free(size_t off, size_t len) {
    by_off_.erase(off);
    auto r = by_size_.equal_range(len);
    for (auto i = r.first; i != r.second; ++i)
      if (i->second == off) {
        by_size_.erase(i);
        break;
      }
  }
  uint8_t *base_ = nullptr;
  size_t cap_ = 0, used_ = 0;
  std::map<size_t, size_t> by_off_;
  std::multimap<size_t, size_t> by_size_;
  std::unordered_map<size_t, size_t> sizes_;
};

// Pinned staging for the descriptors and tables a round uploads: a ring.
// Rounds retire in order, so a round returns everything it took (including
// the end of the ring it skipped when wrapping) by moving the tail.
class Staging {
 public:
  ~Staging() {
    if (base_) cudaFreeHost(base_);
  }
  cudaError_t init(size_t cap) {
    cap_ = cap;
    return cudaHostAlloc(reinterpret_cast<void **>(&base_), cap_, cudaHostAllocDefault);
  }
  // Contiguous space or nullptr; `consumed` grows by what the ring used.
  uint8_t *take(size_t bytes, size_t &consumed) {
    bytes = (bytes + 255) & ~(size_t)255;
    if (used_ == 0) head_ = tail_ = 0;
    size_t off;
    if (head_ >= tail_) {
      if (cap_ - head_ >= bytes) {
        off = head_;
      } else {
        const size_t waste = cap_ - head_;
        if (bytes >= tail_) return nullptr;  // no room before the tail
        used_ += waste;
        consumed += waste;
        off = 0;
      }
    } else {
      if (tail_ - head_ <= bytes) return nullptr;
      off = head_;
    }
    head_ = off + bytes;
    used_ += bytes;
    consumed += bytes;
    return base_ + off;
  }
  size_t head() const { return head_; }
  // A retiring round: everything up to its end position is free again.
  void release(size_t consumed, size_t end) {
    used_ = consumed > used_ ? 0 : used_ - consumed;
    tail_ = end;
  }

 private:
  uint8_t *base_ = nullptr;
  size_t cap_ = 0, head_ = 0, tail_ = 0, used_ = 0;
};

struct Req {
  uint64_t id = 0;
  Buf input, cur;
  bool cur_owned = false;
  std::vector<visar_stage> st;
  std::vector<std::array<double, 9>> mats;
  int next = 0;
  cudaEvent_t ready = nullptr;  // producer of cur (a pending round's event)
  double t_submit = 0, t_done = 0;
  size_t reserve = 0;
  int state = 0;  // 0 queued, 1 admitted, 2 done, 3 released
  int status = VISAR_OK;
  std::string error;  // the failing call's message
  struct Trace *trace = nullptr;  // trace replay: released by the scheduler when done
  size_t trace_i = 0;
};

// A trace replay in progress: the scheduler records each request's latency
// and releases it as soon as it completes (in completion order).
struct Trace {
  double *latency_ms = nullptr;
  size_t done = 0;
  double last_done = 0;
  int rc = VISAR_OK;
  std::string first_error;
};

// Requests waiting or admitted from which a scheduling round keeps at most
// two rounds in flight.
constexpr size_t kBacklog = 256;

struct Round {
  // ev_launch: every launch of the round is done (each stage group runs on
  // a stream of its own and records a group event, in groups); ev_fb: its
  // per-call fallbacks are.
  cudaEvent_t ev_launch = nullptr, ev_fb = nullptr;
  std::vector<cudaEvent_t> groups;
  std::vector<void *> blocks;           // pool blocks freed when the round is done
  std::vector<uint64_t> finishing;      // requests whose last stage ran here
  size_t staging = 0, staging_end = 0;  // staging the round consumed, ring position after it
};

// Output shape of a stage (the rules of build_stage).
void stage_out_shape(const visar_stage &st, const Buf &in, int &w, int &h, int &cn) {
  w = in.v.w;
  h = in.v.h;
  cn = in.v.cn;
  if (st.kind == VISAR_STAGE_GRAY && cn > 1) cn = 1;
  if (st.kind == VISAR_STAGE_RESIZE) {
    w = std::max(1, (int)std::floor((double)in.v.w * st.d[0]));
    h = std::max(1, (int)std::floor((double)in.v.h * st.d[1]));
  }
}

size_t image_bytes(int w, int h, int cn, int depth) { return pitch_of((long long)w * cn * depth_size(depth)) * (size_t)h; }

}  // namespace sv
}  // namespace vb

using namespace vb;
using namespace vb::bt;
using namespace vb::sv;

struct visar_server {
  visar_server_config cfg{};
  int dev = 0;
  DevPool pool;
  Staging staging;
  Plan ctx;  // SM count and counters of the launches being built
  std::vector<cudaStream_t> streams;
  cudaStream_t fb = nullptr;
  int next_stream = 0;
  std::vector<cudaEvent_t> free_events;

  std::mutex mu;
  std::condition_variable cv_done;
  std::unordered_map<uint64_t, std::unique_ptr<Req>> reqs;
  // Submissions wait here under their own lock (a submitter never waits for
  // a scheduling round); the scheduler moves them into reqs / incoming.
  std::mutex mu_in;
  std::vector<std::unique_ptr<Req>> pending;
  std::atomic<uint64_t> n_submitted{0};
  std::deque<uint64_t> incoming;
  std::vector<uint64_t> admitted;  // admitted, stages left
  std::deque<Round> rounds;        // in flight, oldest first
  uint64_t next_id = 1;
  size_t reserved = 0;
  std::atomic<bool> stop{false};
  std::string broken;  // set once a device error was seen: the server only fails requests from then on
  std::atomic<int> fake_round_error{0};  // visar_server_fake_round_error: the next completed round reports it
  std::thread worker;
  visar_server_stats stats{};
  uint64_t groups = 0, grouped = 0;

  cudaEvent_t get_event() {
    if (!free_events.empty()) {
      cudaEvent_t e = free_events.back();
      free_events.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    return e;
  }

  size_t reserve_for(const Req &r) const {
    // Every stage output at once, two temporaries of the largest image, the
    // per-image tables and descriptors.
    size_t total = 64 << 10, big = 0;
    Buf cur = r.input;
    for (const visar_stage &st : r.st) {
      int w, h, cn;
      stage_out_shape(st, cur, w, h, cn);
      const size_t b = image_bytes(w, h, cn, cur.depth);
      total += b + 32 * (size_t)(w + h) + 4096;
      big = std::max(big, std::max(b, image_bytes(cur.v.w, cur.v.h, cur.v.cn, cur.depth)));
      cur.v.w = w;
      cur.v.h = h;
      cur.v.cn = cn;
    }
    return total + 2 * big;
  }

  // Frees a completed request's result (mu held).
  void release_locked(std::unordered_map<uint64_t, std::unique_ptr<Req>>::iterator it) {
    Req &q = *it->second;
    if (q.cur_owned) pool.free(q.cur.v.p);
    reserved -= std::min(reserved, q.reserve);
    reqs.erase(it);
    stats.released++;
  }

  // A request has completed at time t (mu held): trace requests are recorded
  // and released here.
  void finished(uint64_t id, double t) {
    auto it = reqs.find(id);
    if (it == reqs.end()) return;
    Req &q = *it->second;
    q.state = 2;
    q.t_done = t;
    stats.completed++;
    if (Trace *tr = q.trace) {
      if (tr->latency_ms) tr->latency_ms[q.trace_i] = (q.t_done - q.t_submit) * 1e3;
      tr->last_done = std::max(tr->last_done, q.t_done);
      if (q.status != VISAR_OK && tr->rc == VISAR_OK) {
        tr->rc = q.status;
        tr->first_error = q.error;
      }
      tr->done++;
      release_locked(it);
    }
  }

  // A device error was seen (mu held). The context's error is sticky, so no
  // later round can be trusted: every request not yet done completes now
  // with Internal and the CUDA error's name, the rounds in flight are
  // dropped without returning their blocks to the pool, and from here on
  // new submissions fail the same way.
  void fail_all(cudaError_t e) {
    if (broken.empty()) broken = std::string("Internal: ") + cudaGetErrorName(e);
    std::vector<uint64_t> ids;
    for (auto &kv : reqs)
      if (kv.second->state < 2) ids.push_back(kv.first);
    const double t = now_s();
    for (uint64_t id : ids) {
      auto it = reqs.find(id);
      if (it == reqs.end()) continue;
      Req &q = *it->second;
      q.status = VISAR_INTERNAL;
      q.error = broken;
      q.ready = nullptr;
      q.next = (int)q.st.size();
      finished(id, t);
    }
    for (Round &r : rounds) {
      free_events.push_back(r.ev_launch);
      free_events.push_back(r.ev_fb);
      free_events.insert(free_events.end(), r.groups.begin(), r.groups.end());
    }
    rounds.clear();
    incoming.clear();
    admitted.clear();
    cv_done.notify_all();
  }

  // Moves new submissions into the request table (takes mu_in; mu held).
  void take_pending() {
    std::vector<std::unique_ptr<Req>> got;
    {
      std::lock_guard<std::mutex> lk(mu_in);
      got.swap(pending);
    }
    for (auto &q : got) {
      incoming.push_back(q->id);
      const uint64_t id = q->id;
      reqs[id] = std::move(q);
    }
  }

  // Completed rounds: free their memory, finish their requests.
  void poll_rounds() {
    while (!rounds.empty()) {
      Round &r = rounds.front();
      cudaError_t e1 = cudaEventQuery(r.ev_launch);
      const cudaError_t e2 = e1 == cudaSuccess ? cudaEventQuery(r.ev_fb) : e1;
      if (e1 == cudaErrorNotReady || e2 == cudaErrorNotReady) {
        cudaGetLastError();
        break;
      }
      if (const int f = fake_round_error.exchange(0)) e1 = static_cast<cudaError_t>(f);
      if (e1 != cudaSuccess || e2 != cudaSuccess) {
        // A device error is sticky: the round's outputs are undefined and the
        // pool may hold garbage. Fail every request of the round and every
        // request still in flight, and stop admitting work.
        const cudaError_t e = e1 != cudaSuccess ? e1 : e2;
        cudaGetLastError();
        fail_all(e);
        return;
      }
      for (void *p : r.blocks) pool.free(p);
      if (r.staging) staging.release(r.staging, r.staging_end);
      const double t = now_s();
      for (uint64_t id : r.finishing) finished(id, t);
      for (auto &kv : reqs) {
        Req &q = *kv.second;
        if (q.ready == r.ev_launch || q.ready == r.ev_fb ||
            std::find(r.groups.begin(), r.groups.end(), q.ready) != r.groups.end())
          q.ready = nullptr;
      }
      free_events.push_back(r.ev_launch);
      free_events.push_back(r.ev_fb);
      free_events.insert(free_events.end(), r.groups.begin(), r.groups.end());
      rounds.pop_front();
      cv_done.notify_all();
    }
  }

  void admit() {
    const size_t budget = pool.cap() - pool.cap() / 10;
    while (!incoming.empty()) {
      Req &q = *reqs[incoming.front()];
      q.reserve = reserve_for(q);
      if (q.reserve > budget) {  // can never fit the pool
        q.status = VISAR_OUT_OF_MEMORY;
        q.error = "OutOfMemory: request larger than the server pool";
        q.reserve = 0;
        const uint64_t id = q.id;
        incoming.pop_front();
        finished(id, now_s());
        cv_done.notify_all();
        continue;
      }
      if (reserved + q.reserve > budget) break;
      reserved += q.reserve;
      q.state = 1;
      admitted.push_back(q.id);
      incoming.pop_front();
    }
  }

  static void *pool_alloc(void *ctx, size_t bytes) {
    auto *a = static_cast<std::pair<visar_server *, std::vector<void *> *> *>(ctx);
    void *p = a->first->pool.alloc(bytes);
    if (p) a->second->push_back(p);
    return p;
  }

  // Signature of a stage for grouping (warp matrices excluded: per image).
  static std::string stage_key(const visar_stage &st) {
    std::string k(reinterpret_cast<const char *>(&st.kind), sizeof(int));
    k.append(reinterpret_cast<const char *>(st.i), sizeof(st.i));
    const bool warp = st.kind == VISAR_STAGE_WARP_AFFINE || st.kind == VISAR_STAGE_WARP_PERSPECTIVE;
    const int skip = st.kind == VISAR_STAGE_WARP_AFFINE ? 6 : st.kind == VISAR_STAGE_WARP_PERSPECTIVE ? 9 : 0;
    for (int j = warp ? skip : 0; j < 10; j++) k.append(reinterpret_cast<const char *>(&st.d[j]), sizeof(double));
    return k;
  }

  // One scheduling round: every admitted request advances one stage, in
  // groups of equal stages. Each group runs on a stream of its own after the
  // rounds that produced its inputs, so independent groups overlap on the
  // GPU. Returns false when there was nothing to do.
  bool launch_round() {
    if (admitted.empty()) return false;
    std::map<std::string, std::vector<uint64_t>> groups_by;
    for (uint64_t id : admitted) {
      Req &q = *reqs[id];
      groups_by[stage_key(q.st[q.next])].push_back(id);
    }
    Round rd;
    rd.ev_launch = get_event();
    rd.ev_fb = get_event();
    const cudaStream_t ls = streams[next_stream];
    int gstream = next_stream;
    next_stream = (next_stream + 1) % (int)streams.size();
    const cudaStream_t old = thread_stream();
    const int old_async = thread_async();
    std::vector<uint64_t> advanced;
    for (auto &g : groups_by) {
      std::vector<uint64_t> &ids = g.second;
      std::vector<Buf> cur(ids.size()), next;
      std::vector<double> mats;
      visar_stage st = reqs[ids[0]]->st[reqs[ids[0]]->next];
      const bool warp = st.kind == VISAR_STAGE_WARP_AFFINE || st.kind == VISAR_STAGE_WARP_PERSPECTIVE;
      const int nm = st.kind == VISAR_STAGE_WARP_AFFINE ? 6 : 9;
      for (size_t i = 0; i < ids.size(); i++) {
        Req &q = *reqs[ids[i]];
        cur[i] = q.cur;
        cur[i].input = -1;
        if (warp) mats.insert(mats.end(), q.mats[q.next].begin(), q.mats[q.next].begin() + nm);
      }
      if (warp) st.per_image = mats.data();
      std::vector<void *> allocs;
      std::pair<visar_server *, std::vector<void *> *> actx{this, &allocs};
      Builder B{ctx, false, {}, {}};
      B.ext_alloc = &visar_server::pool_alloc;
      B.ext_ctx = &actx;
      Step step;
      const double tb = now_s();
      int rc = build_stage(B, st, cur, next, step);
      // Descriptors, prefix sums and queue counters of the launches.
      std::vector<int *> counters;
      if (rc == VISAR_OK) {
        for (Launch &L : step.launches) {
          std::vector<int> start(L.imgs.size() + 1, 0);
          for (size_t i = 0; i < L.imgs.size(); i++) start[i + 1] = start[i] + L.imgs[i].tiles_x * L.imgs[i].tiles_y;
          L.total = start.back();
          L.d_imgs = B.table(L.imgs);
          L.d_start = B.table(start);
          int *c = static_cast<int *>(pool_alloc(&actx, sizeof(int)));
          if (!L.d_imgs || !L.d_start || !c) {
            rc = VISAR_OUT_OF_MEMORY;
            break;
          }
          counters.push_back(c);
        }
      }
      stats.build_s += now_s() - tb;
      size_t stage_bytes = 0;
      for (const Builder::Upload &u : B.uploads) stage_bytes += (u.data.size() + 255) & ~(size_t)255;
      uint8_t *stg = nullptr;
      size_t consumed = 0;
      if (rc == VISAR_OK && stage_bytes > 0) {
        stg = staging.take(stage_bytes, consumed);
        if (!stg) rc = VISAR_OUT_OF_MEMORY;
      }
      if (rc == VISAR_OUT_OF_MEMORY) {  // retry in a later round
        for (void *p : allocs) pool.free(p);
        stats.deferred++;
        continue;
      }
      if (rc != VISAR_OK) {  // a stage the requests cannot run: fail them
        for (void *p : allocs) pool.free(p);
        for (uint64_t id : ids) {
          Req &q = *reqs[id];
          q.status = rc;
          q.error = visar_last_error();
          q.next = (int)q.st.size();
          rd.finishing.push_back(id);
          advanced.push_back(id);
        }
        continue;
      }
      rd.staging += consumed;
      if (consumed) rd.staging_end = staging.head();
      // Inputs are ready once their producer rounds are.
      std::vector<cudaEvent_t> waits;
      for (uint64_t id : ids)
        if (reqs[id]->ready) waits.push_back(reqs[id]->ready);
      std::sort(waits.begin(), waits.end());
      waits.erase(std::unique(waits.begin(), waits.end()), waits.end());
      cudaEvent_t gev = nullptr;
      if (!step.launches.empty()) {
        const cudaStream_t gs = streams[gstream];
        gstream = (gstream + 1) % (int)streams.size();
        for (cudaEvent_t e : waits) cudaStreamWaitEvent(gs, e, 0);
        const double tu = now_s();
        size_t off = 0;
        for (const Builder::Upload &u : B.uploads) {
          std::memcpy(stg + off, u.data.data(), u.data.size());
          cudaMemcpyAsync(u.dst, stg + off, u.data.size(), cudaMemcpyHostToDevice, gs);
          off += (u.data.size() + 255) & ~(size_t)255;
        }
        const double tl = now_s();
        stats.upload_s += tl - tu;
        for (size_t j = 0; j < step.launches.size(); j++) {
          Launch &L = step.launches[j];
          cudaMemsetAsync(counters[j], 0, sizeof(int), gs);
          ctx.counters = counters[j];
          L.counter = 0;
          const cudaError_t le = run_launch(ctx, L, gs);
          stats.launches++;
          if (le != cudaSuccess) {
            cuda_status(le);
            for (uint64_t id : ids) {
              Req &q = *reqs[id];
              if (q.status == VISAR_OK) {
                q.status = VISAR_INTERNAL;
                q.error = visar_last_error();
              }
            }
          }
        }
        stats.launch_s += now_s() - tl;
        gev = get_event();
        cudaEventRecord(gev, gs);
        cudaStreamWaitEvent(ls, gev, 0);
        rd.groups.push_back(gev);
      } else if (!B.uploads.empty()) {
        size_t off = 0;
        for (const Builder::Upload &u : B.uploads) {
          std::memcpy(stg + off, u.data.data(), u.data.size());
          cudaMemcpyAsync(u.dst, stg + off, u.data.size(), cudaMemcpyHostToDevice, fb);
          off += (u.data.size() + 255) & ~(size_t)255;
        }
      }
      if (!step.fallbacks.empty()) {
        for (cudaEvent_t e : waits) cudaStreamWaitEvent(fb, e, 0);
        set_thread_stream(fb, 1);
        for (const Fallback &f : step.fallbacks) {
          const int frc = run_fallback(f);
          stats.fallback_calls++;
          if (frc != VISAR_OK) {
            for (uint64_t id : ids) {
              Req &q = *reqs[id];
              if (q.cur.v.p == f.s.v.p && q.status == VISAR_OK) {
                q.status = frc;
                q.error = visar_last_error();
              }
            }
          }
        }
        set_thread_stream(old, old_async);
      }
      // Outputs move to their requests; the rest (temporaries, tables,
      // descriptors, counters, the inputs just consumed) go with the round.
      std::vector<void *> outs;
      for (size_t i = 0; i < ids.size(); i++) {
        Req &q = *reqs[ids[i]];
        const bool fell_back = std::any_of(step.fallbacks.begin(), step.fallbacks.end(),
                                           [&](const Fallback &f) { return f.d.v.p == next[i].v.p; });
        if (next[i].v.p != q.cur.v.p) {
          if (q.cur_owned) rd.blocks.push_back(q.cur.v.p);
          q.cur = next[i];
          q.cur_owned = true;
          outs.push_back(next[i].v.p);
        }
        q.ready = fell_back ? rd.ev_fb : gev ? gev : rd.ev_launch;
        q.next++;
        advanced.push_back(ids[i]);
        if (q.next == (int)q.st.size()) rd.finishing.push_back(ids[i]);
      }
      for (void *p : allocs)
        if (std::find(outs.begin(), outs.end(), p) == outs.end()) rd.blocks.push_back(p);
      groups++;
      grouped += ids.size();
    }
    if (advanced.empty()) {
      free_events.push_back(rd.ev_launch);
      free_events.push_back(rd.ev_fb);
      free_events.insert(free_events.end(), rd.groups.begin(), rd.groups.end());
      return false;
    }
    cudaEventRecord(rd.ev_launch, ls);
    cudaEventRecord(rd.ev_fb, fb);
    // Requests with stages left stay admitted.
    std::vector<uint64_t> keep;
    for (uint64_t id : admitted)
      if (reqs[id]->next < (int)reqs[id]->st.size()) keep.push_back(id);
    admitted.swap(keep);
    rounds.push_back(std::move(rd));
    stats.rounds++;
    return true;
  }

  // True when every admitted request is new (no stage run yet) and no two of
  // them share a first stage: a scheduling round would run each alone, so
  // the per-call path (less host work per stage, no round events) serves
  // them sooner.
  bool solo() {
    if (admitted.empty()) return false;
    std::vector<std::string> keys;
    for (uint64_t id : admitted) {
      const Req &q = *reqs[id];
      if (q.next != 0 || q.ready) return false;
      keys.push_back(stage_key(q.st[0]));
    }
    std::sort(keys.begin(), keys.end());
    return std::adjacent_find(keys.begin(), keys.end()) == keys.end();
  }

  // Plain mode (and solo requests): each admitted request runs all its
  // stages now, call by call.
  bool launch_plain(bool solo_reqs = false) {
    if (admitted.empty()) return false;
    Round rd;
    rd.ev_launch = get_event();
    rd.ev_fb = get_event();
    const cudaStream_t old = thread_stream();
    const int old_async = thread_async();
    set_thread_stream(fb, 1);
    for (uint64_t id : admitted) {
      Req &q = *reqs[id];
      bool failed = false;
      for (size_t k = 0; k < q.st.size() && !failed; k++) {
        const visar_stage &st = q.st[k];
        int w, h, cn;
        stage_out_shape(st, q.cur, w, h, cn);
        if ((st.kind == VISAR_STAGE_GRAY && q.cur.v.cn == 1) ||
            (st.kind == VISAR_STAGE_RESIZE && w == q.cur.v.w && h == q.cur.v.h)) {
          continue;  // pass-through, as the batched form
        }
        void *p = pool.alloc(image_bytes(w, h, cn, q.cur.depth));
        if (!p) {
          q.status = VISAR_OUT_OF_MEMORY;
          q.error = "OutOfMemory: server pool";
          failed = true;
          break;
        }
        Fallback f;
        f.st = st;
        f.s = q.cur;
        f.d = Buf{DImg{static_cast<uint8_t *>(p), (long long)pitch_of((long long)w * cn * depth_size(q.cur.depth)), w, h, cn},
                  q.cur.depth};
        std::memset(f.m, 0, sizeof(f.m));
        std::copy(q.mats[k].begin(), q.mats[k].end(), f.m);
        const int rc = run_fallback(f);
        if (!solo_reqs) stats.fallback_calls++;
        if (q.cur_owned) rd.blocks.push_back(q.cur.v.p);
        q.cur = f.d;
        q.cur_owned = true;
        if (rc != VISAR_OK) {
          q.status = rc;
          q.error = visar_last_error();
          failed = true;
        }
      }
      q.next = (int)q.st.size();
      rd.finishing.push_back(id);
      if (solo_reqs) {
        stats.solo++;
        groups++;
        grouped++;
      }
    }
    set_thread_stream(old, old_async);
    admitted.clear();
    cudaEventRecord(rd.ev_launch, fb);
    cudaEventRecord(rd.ev_fb, fb);
    rounds.push_back(std::move(rd));
    stats.rounds++;
    return true;
  }

  void loop() {
    cudaSetDevice(dev);
    while (!stop.load()) {
      bool did = false;
      {
        std::lock_guard<std::mutex> lk(mu);
        take_pending();
        if (!broken.empty() && !incoming.empty()) fail_all(cudaSuccess);
        poll_rounds();
        admit();
        // A long backlog takes fewer rounds in flight, so that more requests
        // gather per round (larger groups); a short one takes the configured
        // number, which keeps the latency of moderate loads low.
        const int limit = incoming.size() + admitted.size() >= kBacklog ? std::min(cfg.max_inflight, 2) : cfg.max_inflight;
        if (broken.empty() && (int)rounds.size() < limit) {
          const double t0 = now_s();
          if (cfg.mode == VISAR_SERVE_PLAIN) did = launch_plain();
          else if (incoming.empty() && solo()) did = launch_plain(true);
          else did = launch_round();
          if (did) stats.schedule_s += now_s() - t0;
        }
      }
      if (!did) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
  }
};

extern "C" {

int visar_server_create(const visar_server_config *cfg, visar_server **out) {
  if (!out) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  *out = nullptr;
  std::unique_ptr<visar_server> s(new (std::nothrow) visar_server);
  if (!s) return report_error(VISAR_OUT_OF_MEMORY, "OutOfMemory");
  if (cfg) s->cfg = *cfg;
  if (s->cfg.pool_bytes == 0) s->cfg.pool_bytes = (size_t)64 << 30;
  if (s->cfg.max_inflight <= 0) s->cfg.max_inflight = 4;
  if (s->cfg.streams <= 0) s->cfg.streams = 8;
  if (s->cfg.mode != VISAR_SERVE_BATCHED && s->cfg.mode != VISAR_SERVE_PLAIN)
    return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument: serve mode");
  cudaError_t e = cudaGetDevice(&s->dev);
  if (e != cudaSuccess) return cuda_status(e);
  if ((e = s->pool.init(s->cfg.pool_bytes)) != cudaSuccess) {
    cudaGetLastError();
    return report_error(VISAR_OUT_OF_MEMORY, "OutOfMemory: server pool");
  }
  if ((e = s->staging.init((size_t)256 << 20)) != cudaSuccess) return cuda_status(e);
  cudaDeviceGetAttribute(&s->ctx.num_sms, cudaDevAttrMultiProcessorCount, s->dev);
  s->streams.resize(s->cfg.streams);
  for (auto &st : s->streams)
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) return cuda_status(e);
  if ((e = cudaStreamCreateWithFlags(&s->fb, cudaStreamNonBlocking)) != cudaSuccess) return cuda_status(e);
  s->stats.pool_bytes = s->pool.cap();
  visar_server *raw = s.get();
  s->worker = std::thread([raw] { raw->loop(); });
  *out = s.release();
  return VISAR_OK;
}

static int submit_req(visar_server *s, const visar_image *input, const visar_stage *stages, size_t nstages,
                      uint64_t *id, Trace *trace, size_t trace_i) {
  if (!s || !input || !input->data || !stages || nstages == 0 || nstages > 16 || !id)
    return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  if (!(input->depth == 0 || input->depth == 2 || input->depth == 3 || input->depth == 5))
    return report_error(VISAR_UNSUPPORTED, "Unsupported");
  if (input->channels == 0 || input->channels > 4) return report_error(VISAR_UNSUPPORTED, "UnsupportedChannels");
  if (input->width == 0 || input->height == 0) return report_error(VISAR_INVALID_ARGUMENT, "InvalidSize");
  std::unique_ptr<Req> q(new Req);
  q->input = Buf{DImg{static_cast<uint8_t *>(input->data), (long long)input->stride, (int)input->width,
                      (int)input->height, (int)input->channels},
                 (int)input->depth};
  q->cur = q->input;
  q->st.assign(stages, stages + nstages);
  q->mats.resize(nstages);
  for (size_t k = 0; k < nstages; k++) {
    q->mats[k].fill(0.0);
    const visar_stage &st = stages[k];
    const int nm = st.kind == VISAR_STAGE_WARP_AFFINE ? 6 : st.kind == VISAR_STAGE_WARP_PERSPECTIVE ? 9 : 0;
    for (int j = 0; j < nm; j++) q->mats[k][j] = st.per_image ? st.per_image[j] : st.d[j];
    q->st[k].per_image = nullptr;
  }
  q->trace = trace;
  q->trace_i = trace_i;
  q->t_submit = now_s();
  std::lock_guard<std::mutex> lk(s->mu_in);
  q->id = s->next_id++;
  *id = q->id;
  s->pending.push_back(std::move(q));
  s->n_submitted++;
  return VISAR_OK;
}

// The request with this id (mu held), or nullptr; *queued = true when it is
// still in the submission queue.
static Req *find_req(visar_server *s, uint64_t id, bool *queued) {
  *queued = false;
  auto it = s->reqs.find(id);
  if (it != s->reqs.end()) return it->second.get();
  std::lock_guard<std::mutex> lk(s->mu_in);
  for (auto &q : s->pending)
    if (q->id == id) *queued = true;
  return nullptr;
}

int visar_server_submit(visar_server *s, const visar_image *input, const visar_stage *stages, size_t nstages,
                        uint64_t *id) {
  return submit_req(s, input, stages, nstages, id, nullptr, 0);
}

int visar_server_poll(visar_server *s, uint64_t id, int *done, visar_image *out) {
  if (!s || !done) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  std::lock_guard<std::mutex> lk(s->mu);
  bool queued;
  Req *r = find_req(s, id, &queued);
  if (queued) {
    *done = 0;
    return VISAR_OK;
  }
  if (!r || r->state == 3 || r->trace) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument: request id");
  Req &q = *r;
  *done = q.state == 2;
  if (*done && out) *out = cimg(q.cur);
  if (*done && q.status != VISAR_OK) return report_error(q.status, q.error.empty() ? "request failed" : q.error.c_str());
  return VISAR_OK;
}

int visar_server_wait(visar_server *s, uint64_t id, visar_image *out) {
  if (!s) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    bool queued;
    Req *r = find_req(s, id, &queued);
    if (queued) {
      s->cv_done.wait_for(lk, std::chrono::milliseconds(1));
      continue;
    }
    if (!r || r->state == 3 || r->trace) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument: request id");
    Req &q = *r;
    if (q.state == 2) {
      if (out) *out = cimg(q.cur);
      return q.status == VISAR_OK ? VISAR_OK : report_error(q.status, q.error.empty() ? "request failed" : q.error.c_str());
    }
    s->cv_done.wait_for(lk, std::chrono::milliseconds(5));
  }
}

int visar_server_release(visar_server *s, uint64_t id) {
  if (!s) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end() || it->second->state != 2 || it->second->trace)
    return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument: request not done");
  s->release_locked(it);
  return VISAR_OK;
}

int visar_server_fake_round_error(visar_server *s, int cuda_error) {
  if (!s || cuda_error <= 0) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  s->fake_round_error.store(cuda_error);
  return VISAR_OK;
}

int visar_server_get_stats(visar_server *s, visar_server_stats *st) {
  if (!s || !st) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  std::lock_guard<std::mutex> lk(s->mu);
  *st = s->stats;
  st->submitted = s->n_submitted.load();
  st->pool_used = s->pool.used();
  st->pool_reserved = s->reserved;
  st->mean_batch = s->groups ? (double)s->grouped / (double)s->groups : 0.0;
  return VISAR_OK;
}

void visar_server_destroy(visar_server *s) {
  if (!s) return;
  s->stop.store(true);
  if (s->worker.joinable()) s->worker.join();
  cudaSetDevice(s->dev);
  for (cudaStream_t st : s->streams) cudaStreamSynchronize(st);
  cudaStreamSynchronize(s->fb);
  for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
  cudaStreamDestroy(s->fb);
  for (Round &r : s->rounds) {
    s->free_events.push_back(r.ev_launch);
    s->free_events.push_back(r.ev_fb);
    s->free_events.insert(s->free_events.end(), r.groups.begin(), r.groups.end());
  }
  for (cudaEvent_t e : s->free_events) cudaEventDestroy(e);
  delete s;
}

int visar_server_run_trace(visar_server *s, const visar_trace_request *reqs, size_t n, double *latency_ms,
                           double *elapsed_s) {
  if (!s || (n > 0 && !reqs)) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  Trace tr;
  tr.latency_ms = latency_ms;
  std::atomic<size_t> submitted{0};
  std::atomic<int> submit_rc{VISAR_OK};
  std::string submit_error;
  const double t0 = now_s();
  tr.last_done = t0;
  std::thread submitter([&] {
    cudaSetDevice(s->dev);
    for (size_t i = 0; i < n; i++) {
      const double due = t0 + reqs[i].arrival_s;
      for (double t = now_s(); t < due; t = now_s())
        if (due - t > 200e-6) std::this_thread::sleep_for(std::chrono::microseconds(50));
      uint64_t id = 0;
      const int rc = submit_req(s, &reqs[i].input, reqs[i].stages, reqs[i].nstages, &id, &tr, i);
      if (rc != VISAR_OK) {
        if (submit_rc.load() == VISAR_OK) submit_error = visar_last_error();
        submit_rc.store(rc);
        if (latency_ms) latency_ms[i] = -1;
        continue;
      }
      submitted++;
    }
  });
  submitter.join();
  {
    std::unique_lock<std::mutex> lk(s->mu);
    while (tr.done < submitted.load()) s->cv_done.wait_for(lk, std::chrono::milliseconds(2));
  }
  if (elapsed_s) *elapsed_s = tr.last_done - (t0 + (n ? reqs[0].arrival_s : 0.0));
  if (submit_rc.load() != VISAR_OK) return report_error(submit_rc.load(), submit_error.c_str());
  return tr.rc == VISAR_OK ? VISAR_OK
                           : report_error(tr.rc, tr.first_error.empty() ? "a request failed" : tr.first_error.c_str());
}

}  // extern "C"
