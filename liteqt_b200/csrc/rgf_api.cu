// rgf_api.cu -- the C ABI declared in include/rgf.h.
//
// Host responsibilities: argument checks, host/device pointer classification
// and staging, building the device task table, sizing the per-CTA workspace,
// launching the persistent solver, and reporting status.  No dense arithmetic
// happens on the host, and there is no CPU fallback: if the CUDA path cannot
// run, the call fails with RGF_E_CUDA / RGF_E_UNSUPPORTED.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "rgf_internal.h"

#if defined(__x86_64__) && defined(__SSE2__)
#include <emmintrin.h>
#endif

using namespace rgf;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define RGF_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(RGF_E_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),    \
                  __FILE__, __LINE__);                                                   \
  } while (0)

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Device buffer that grows and is reused across calls.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int reserve(size_t need) {
    if (need <= bytes) return RGF_OK;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    if (cudaMalloc(&p, need) != cudaSuccess) {
      cudaGetLastError();
      return fail(RGF_E_NOMEM, "cudaMalloc(%zu) failed", need);
    }
    bytes = need;
    return RGF_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
};

// A large host copy with non-temporal (streaming) stores where the host
// has them: the destination lines are not read into the cache before they
// are overwritten, so a byte moved costs two memory transfers, not three.
void stream_copy(char* dst, const char* src, size_t n) {
#if defined(__x86_64__) && defined(__SSE2__)
  if (n >= 4096) {
    const size_t head = (16 - ((uintptr_t)dst & 15)) & 15;
    std::memcpy(dst, src, head);
    dst += head;
    src += head;
    n -= head;
    const size_t body = n & ~size_t(63);
    for (size_t i = 0; i < body; i += 64) {
      const __m128i a = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + i));
      const __m128i b = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + i + 16));
      const __m128i c = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + i + 32));
      const __m128i d = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + i + 48));
      _mm_stream_si128(reinterpret_cast<__m128i*>(dst + i), a);
      _mm_stream_si128(reinterpret_cast<__m128i*>(dst + i + 16), b);
      _mm_stream_si128(reinterpret_cast<__m128i*>(dst + i + 32), c);
      _mm_stream_si128(reinterpret_cast<__m128i*>(dst + i + 48), d);
    }
    _mm_sfence();
    std::memcpy(dst + body, src + body, n - body);
    return;
  }
#endif
  std::memcpy(dst, src, n);
}

// Host threads that share out the memcpy chunks of one bounce piece (below).
// One pool per process: a piece takes it whole (its caller copying too), and
// a caller that finds it taken copies its piece alone, so concurrent copiers
// (one context per host thread) never run more copy threads than the pool's
// plus their own.
class CopyPool {
 public:
  struct Chunk {
    char* dst;
    const char* src;
    size_t bytes;
  };
  static CopyPool& get() {
    static CopyPool* p = new CopyPool();   // never destroyed: its threads outlive static destructors
    return *p;
  }
  // copies every chunk; returns once all are done
  void copy(const std::vector<Chunk>& chunks) {
    std::unique_lock<std::mutex> busy(use_, std::try_to_lock);
    if (!busy.owns_lock() || th_.empty() || chunks.size() < 2) {
      for (const Chunk& c : chunks) stream_copy(c.dst, c.src, c.bytes);
      return;
    }
    {
      std::lock_guard<std::mutex> l(m_);
      list_ = &chunks;
      next_ = 0;
      remaining_ = (int)th_.size();
      gen_++;
    }
    cv_.notify_all();
    take();
    std::unique_lock<std::mutex> l(m_);
    done_cv_.wait(l, [&] { return remaining_ == 0; });
    list_ = nullptr;
  }

 private:
  CopyPool() {
    const unsigned hw = std::thread::hardware_concurrency();
    const int n = (int)std::max(1u, std::min(12u, hw * 3 / 4));
    for (int t = 0; t + 1 < n; t++) th_.emplace_back([this] { worker(); });
  }
  void take() {
    const std::vector<Chunk>& v = *list_;
    for (;;) {
      const size_t i = next_.fetch_add(1);
      if (i >= v.size()) return;
      stream_copy(v[i].dst, v[i].src, v[i].bytes);
    }
  }
  void worker() {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> l(m_);
        cv_.wait(l, [&] { return gen_ != seen; });
        seen = gen_;
      }
      take();
      {
        std::lock_guard<std::mutex> l(m_);
        if (--remaining_ == 0) done_cv_.notify_one();
      }
    }
  }
  std::vector<std::thread> th_;
  std::mutex use_;   // held by the piece the pool works on
  std::mutex m_;
  std::condition_variable cv_, done_cv_;
  uint64_t gen_ = 0;
  int remaining_ = 0;
  const std::vector<Chunk>* list_ = nullptr;
  std::atomic<size_t> next_{0};
};

// Copies between device memory and pageable (not page-locked) host memory at
// the host link's speed.  The driver moves a pageable copy through its own
// pinned buffer with one host thread (about 12 GB/s on the B200 hosts, a
// quarter of the link); here the DMA lands in (or leaves from) pinned bounce
// slots, kSlots x kPiece bytes, and the host side -- pinned slot <-> the
// caller's arrays -- is cut into chunks of at most kChunk bytes that the
// CopyPool copies.
//   enqueue_d2h queues device -> slot copies on `st` (after the work already
//   on it), packing the runs into pieces, and hands each queued piece to the
//   copier's landing thread, which waits for the piece (and every later one
//   that has also landed), writes out their destinations and frees their
//   slots; enqueue_d2h waits for a slot when all are queued.  So the calling
//   thread keeps the link busy while the landed pieces are copied out.
//   finish waits until every queued piece is written out; d2h = enqueue_d2h
//   + finish.  h2d copies host -> device and returns with every source read.
class PageableCopier {
 public:
  struct Copy {
    char* host;
    char* dev;
    size_t bytes;
  };
  static constexpr int kSlots = 16;
  static constexpr size_t kPiece = size_t(8) << 20;
  static constexpr size_t kChunk = size_t(2) << 20;
  static constexpr size_t kSmall = size_t(1) << 20;

  ~PageableCopier() {
    if (th_.joinable()) {
      {
        std::lock_guard<std::mutex> l(m_);
        stop_ = true;
      }
      cv_.notify_all();
      th_.join();
    }
    for (int s = 0; s < kSlots; s++) {
      if (ev_[s]) cudaEventDestroy(ev_[s]);
      if (slot_[s]) cudaFreeHost(slot_[s]);
    }
  }

  cudaError_t enqueue_d2h(const std::vector<Copy>& copies, cudaStream_t st) {
    cudaError_t e = setup();
    if (e != cudaSuccess) return e;
    Piece cur;
    cur.slot = -1;
    size_t fill = 0;
    for (const Copy& c : copies)
      for (size_t at = 0; at < c.bytes;) {
        if (cur.slot < 0) {
          if ((cur.slot = take_slot()) < 0) return error();
          fill = 0;
        }
        const size_t n = std::min(c.bytes - at, kPiece - fill);
        cur.parts.push_back({c.host + at, c.dev + at, n, fill});
        fill = (fill + n + 255) & ~size_t(255);
        at += n;
        if (fill >= kPiece) {
          if ((e = issue(cur, st, true)) != cudaSuccess) return e;
          cur = Piece();
          cur.slot = -1;
        }
      }
    if (cur.slot >= 0 && (e = issue(cur, st, true)) != cudaSuccess) return e;
    return cudaSuccess;
  }
  cudaError_t poll() { return error(); }   // the landing thread's first error, if any
  cudaError_t finish() {
    std::unique_lock<std::mutex> l(m_);
    cv_.wait(l, [&] { return inflight_.empty(); });
    const cudaError_t e = err_;
    err_ = cudaSuccess;
    return e;
  }
  cudaError_t d2h(const std::vector<Copy>& copies, cudaStream_t st) {
    cudaError_t e = enqueue_d2h(copies, st);
    const cudaError_t f = finish();
    return e != cudaSuccess ? e : f;
  }
  cudaError_t h2d(const std::vector<Copy>& copies, cudaStream_t st) {
    cudaError_t e = setup();
    if (e == cudaSuccess) e = finish();   // the landing thread idle, every slot free
    if (e != cudaSuccess) return e;
    // rounds: as many pieces as there are free slots, their sources copied
    // into the slots in one pool pass, then their DMAs queued; a slot is
    // free again once its DMA has read it
    std::vector<Piece> round;
    size_t ci = 0, at = 0;
    std::deque<int> busy_slots;
    std::vector<int> freel;
    {
      std::lock_guard<std::mutex> l(m_);
      freel.swap(free_);
    }
    auto give_back = [&](cudaError_t err) {   // slots return to the free list on an error too
      for (int sl : busy_slots) freel.push_back(sl);
      std::lock_guard<std::mutex> l(m_);
      for (int sl : freel) free_.push_back(sl);
      return err;
    };
    while (ci < copies.size()) {
      while (freel.empty()) {
        if (busy_slots.empty()) return give_back(cudaErrorMemoryAllocation);   // a failed call kept its slots
        if ((e = cudaEventSynchronize(ev_[busy_slots.front()])) != cudaSuccess) return give_back(e);
        freel.push_back(busy_slots.front());
        busy_slots.pop_front();
      }
      round.clear();
      while (!freel.empty() && ci < copies.size()) {
        Piece pc;
        pc.slot = freel.back();
        freel.pop_back();
        size_t fill = 0;
        while (ci < copies.size() && fill < kPiece) {
          const Copy& c = copies[ci];
          const size_t n = std::min(c.bytes - at, kPiece - fill);
          pc.parts.push_back({c.host + at, c.dev + at, n, fill});
          fill = (fill + n + 255) & ~size_t(255);
          at += n;
          if (at == c.bytes) {
            ci++;
            at = 0;
          }
        }
        round.push_back(std::move(pc));
      }
      host_side(round, false);
      for (size_t i = 0; i < round.size(); i++) {
        if ((e = issue(round[i], st, false)) != cudaSuccess) {
          for (size_t k = i; k < round.size(); k++) freel.push_back(round[k].slot);
          return give_back(e);
        }
        busy_slots.push_back(round[i].slot);   // h2d pieces are tracked here, not by the landing thread
      }
    }
    while (!busy_slots.empty()) {
      if ((e = cudaEventSynchronize(ev_[busy_slots.front()])) != cudaSuccess) return give_back(e);
      freel.push_back(busy_slots.front());
      busy_slots.pop_front();
    }
    return give_back(cudaSuccess);
  }

 private:
  struct Part {   // one run of a piece: host range <-> slot offset, device address
    char* host;
    char* dev;
    size_t bytes;
    size_t off;
  };
  struct Piece {
    std::vector<Part> parts;
    int slot;
  };
  cudaError_t setup() {
    if (slot_[0]) return cudaSuccess;
    cudaError_t e = cudaGetDevice(&dev_);
    for (int s = 0; e == cudaSuccess && s < kSlots; s++) {
      e = cudaHostAlloc((void**)&slot_[s], kPiece, cudaHostAllocDefault);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_[s], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
      for (int s = 0; s < kSlots; s++) {
        if (ev_[s]) cudaEventDestroy(ev_[s]);
        if (slot_[s]) cudaFreeHost(slot_[s]);
        ev_[s] = nullptr;
        slot_[s] = nullptr;
      }
      return e;
    }
    for (int s = 0; s < kSlots; s++) free_.push_back(kSlots - 1 - s);
    th_ = std::thread([this] { lander(); });
    return cudaSuccess;
  }
  cudaError_t error() {
    std::lock_guard<std::mutex> l(m_);
    return err_;
  }
  // a free slot (waiting for the landing thread to release one), or -1
  // when none can come back
  int take_slot() {
    std::unique_lock<std::mutex> l(m_);
    cv_.wait(l, [&] { return !free_.empty() || inflight_.empty(); });
    if (free_.empty()) {
      if (err_ == cudaSuccess) err_ = cudaErrorMemoryAllocation;   // a failed call kept its slots
      return -1;
    }
    const int sl = free_.back();
    free_.pop_back();
    return sl;
  }
  // queues the DMA of one piece and records its slot's event; a d2h piece
  // goes to the landing thread, or gives its slot back if it could not be
  // queued
  cudaError_t issue(Piece& pc, cudaStream_t st, bool d2h) {
    char* sl = slot_[pc.slot];
    cudaError_t r = cudaSuccess;
    for (const Part& p : pc.parts) {
      r = d2h ? cudaMemcpyAsync(sl + p.off, p.dev, p.bytes, cudaMemcpyDeviceToHost, st)
              : cudaMemcpyAsync(p.dev, sl + p.off, p.bytes, cudaMemcpyHostToDevice, st);
      if (r != cudaSuccess) break;
    }
    if (r == cudaSuccess) r = cudaEventRecord(ev_[pc.slot], st);
    if (d2h) {
      {
        std::lock_guard<std::mutex> l(m_);
        if (r == cudaSuccess) inflight_.push_back(std::move(pc));
        else free_.push_back(pc.slot);
      }
      cv_.notify_all();
    }
    return r;
  }
  // host side of pieces: slot -> destinations (d2h) or sources -> slot, in
  // chunks shared out by the CopyPool
  void host_side(const std::vector<Piece>& pieces, bool d2h) {
    std::vector<CopyPool::Chunk>& chunks = d2h ? land_chunks_ : h2d_chunks_;
    chunks.clear();
    size_t total = 0;
    for (const Piece& pc : pieces)
      for (const Part& p : pc.parts)
        for (size_t a = 0; a < p.bytes; a += kChunk) {
          const size_t n = std::min(kChunk, p.bytes - a);
          char* sl = slot_[pc.slot] + p.off + a;
          if (d2h) chunks.push_back({p.host + a, sl, n});
          else chunks.push_back({sl, p.host + a, n});
          total += n;
        }
    if (total < kSmall) {
      for (const CopyPool::Chunk& c : chunks) std::memcpy(c.dst, c.src, c.bytes);
      return;
    }
    CopyPool::get().copy(chunks);
  }
  // landing thread: waits for the oldest queued piece, takes it with every
  // later piece that has landed too, writes their destinations and frees
  // their slots
  void lander() {
    bool dev_set = false;
    std::vector<Piece> ready;
    for (;;) {
      {
        std::unique_lock<std::mutex> l(m_);
        cv_.wait(l, [&] { return stop_ || !inflight_.empty(); });
        if (inflight_.empty()) return;   // stop_
        if (!dev_set) {
          cudaSetDevice(dev_);
          dev_set = true;
        }
      }
      // the front piece stays queued (finish waits for it) until written out
      int front;
      {
        std::lock_guard<std::mutex> l(m_);
        front = inflight_.front().slot;
      }
      cudaError_t e = cudaEventSynchronize(ev_[front]);
      size_t take = 1;
      {
        std::lock_guard<std::mutex> l(m_);
        while (take < inflight_.size() && cudaEventQuery(ev_[inflight_[take].slot]) == cudaSuccess) take++;
        ready.clear();
        for (size_t k = 0; k < take; k++) ready.push_back(inflight_[k]);
      }
      if (e == cudaSuccess) host_side(ready, true);
      {
        std::lock_guard<std::mutex> l(m_);
        if (e != cudaSuccess && err_ == cudaSuccess) err_ = e;
        for (size_t k = 0; k < take; k++) {
          free_.push_back(inflight_.front().slot);
          inflight_.pop_front();
        }
      }
      cv_.notify_all();
    }
  }

  char* slot_[kSlots] = {};
  cudaEvent_t ev_[kSlots] = {};
  int dev_ = 0;
  std::mutex m_;
  std::condition_variable cv_;
  bool stop_ = false;
  cudaError_t err_ = cudaSuccess;
  std::vector<int> free_;          // slots without a queued piece
  std::deque<Piece> inflight_;     // queued device -> host pieces, oldest first
  std::vector<CopyPool::Chunk> land_chunks_, h2d_chunks_;
  std::thread th_;                 // the landing thread, started by setup()
};

// The copier of pipelined calls (rgf_opts.pipelined): one thread per context
// follows each call's per-task progress counters (written by the kernel into
// host-mapped memory after each block's outputs) and queues on the copy
// stream the host copies of the blocks that are done, in chunks, while the
// solve runs; once the solve has finished it queues the rest (blocks of tasks
// without a backward sweep, scalars, task info) and records the call's event.
struct PipeJob {
  int slot = 0;
  const volatile int32_t* prog = nullptr;   // host view of the progress counters
  cudaEvent_t solved = nullptr;             // recorded after the solve
  cudaEvent_t freed = nullptr;              // recorded after the call's last copy
  struct Blocks {                           // one block-structured output of one task
    char* host;
    const char* dev;
    size_t blk;                             // bytes per block
    int64_t task;
    int32_t nx;                             // blocks of the output
    int32_t lag;                            // counter value at which its last block is done, minus nx
    bool pageable;                          // host array not page-locked
  };
  struct Copy {
    char* host;
    const char* dev;
    size_t bytes;
    bool pageable;
  };
  std::vector<Blocks> blocks;
  std::vector<Copy> rest;
};

// Follows one solve's progress counters and copies each output block once it
// is written (chunks of kChunk blocks while the solve runs) on the copy
// stream `cs`; pageable destinations go through `pc` (made on first use),
// whose landing thread writes them out.  After the solve: the blocks no
// counter covered and the rest (scalars, task info); returns once every
// pageable destination is written and the page-locked copies are queued,
// after recording j.freed (if any) on `cs`.
cudaError_t run_copy_job(const PipeJob& j, cudaStream_t cs, std::unique_ptr<PageableCopier>& pc) {
  constexpr int32_t kChunk = 8;   // blocks per copy while the solve runs
  std::vector<int32_t> done(j.blocks.size(), 0);
  cudaError_t e = cudaSuccess;
  // copies to pageable arrays are gathered per round (flush below); the
  // others are queued on the copy stream
  std::vector<PageableCopier::Copy> slow;
  auto copy = [&](char* host, const char* dev, size_t bytes, bool pageable) {
    if (pageable) {
      slow.push_back({host, const_cast<char*>(dev), bytes});
      return;
    }
    const cudaError_t r = cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, cs);
    if (r != cudaSuccess && e == cudaSuccess) e = r;
  };
  // pageable runs are queued through the PageableCopier, whose landing
  // thread writes them out as they arrive (finish at the end)
  auto flush = [&] {
    if (!slow.empty()) {
      if (!pc) pc.reset(new PageableCopier());
      const cudaError_t r = pc->enqueue_d2h(slow, cs);
      if (r != cudaSuccess && e == cudaSuccess) e = r;
      slow.clear();
    }
    if (pc) {
      const cudaError_t r = pc->poll();
      if (r != cudaSuccess && e == cudaSuccess) e = r;
    }
  };
  for (;;) {
    const cudaError_t q = cudaEventQuery(j.solved);
    const bool fin = q != cudaErrorNotReady;
    if (q != cudaSuccess && q != cudaErrorNotReady && e == cudaSuccess) e = q;
    for (size_t b = 0; b < j.blocks.size(); b++) {
      const PipeJob::Blocks& o = j.blocks[b];
      int32_t c = j.prog[o.task] - o.lag;
      c = c < 0 ? 0 : (c > o.nx ? o.nx : c);
      if (c > done[b] && (fin || c - done[b] >= kChunk)) {
        const size_t off = (size_t)(o.nx - c) * o.blk;
        copy(o.host + off, o.dev + off, (size_t)(c - done[b]) * o.blk, o.pageable);
        done[b] = c;
      }
    }
    flush();
    if (fin) break;
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  const cudaError_t w = cudaStreamWaitEvent(cs, j.solved, 0);
  if (w != cudaSuccess && e == cudaSuccess) e = w;
  for (size_t b = 0; b < j.blocks.size(); b++) {   // blocks no counter covered
    const PipeJob::Blocks& o = j.blocks[b];
    if (done[b] < o.nx) copy(o.host, o.dev, (size_t)(o.nx - done[b]) * o.blk, o.pageable);
  }
  for (const PipeJob::Copy& r : j.rest) copy(r.host, r.dev, r.bytes, r.pageable);
  flush();
  if (pc) {
    const cudaError_t r = pc->finish();
    if (r != cudaSuccess && e == cudaSuccess) e = r;
  }
  if (j.freed) {
    const cudaError_t f = cudaEventRecord(j.freed, cs);
    if (f != cudaSuccess && e == cudaSuccess) e = f;
  }
  return e;
}

class PipeWorker {
 public:
  PipeWorker(int device, cudaStream_t cs) : dev_(device), cs_(cs), th_([this] { loop(); }) {}
  ~PipeWorker() {
    {
      std::lock_guard<std::mutex> l(m_);
      stop_ = true;
    }
    cv_.notify_all();
    th_.join();
  }
  void push(PipeJob&& j) {
    {
      std::lock_guard<std::mutex> l(m_);
      pending_[j.slot]++;
      pushed_++;
      q_.push_back(std::move(j));
    }
    cv_.notify_all();
  }
  // every job pushed so far has queued its copies
  void drain() {
    std::unique_lock<std::mutex> l(m_);
    cv_.wait(l, [&] { return issued_ == pushed_; });
  }
  // the jobs of staging slot `slot` have queued their copies
  void wait_slot(int slot) {
    std::unique_lock<std::mutex> l(m_);
    cv_.wait(l, [&] { return pending_[slot] == 0; });
  }
  cudaError_t take_error() {
    std::lock_guard<std::mutex> l(m_);
    const cudaError_t e = err_;
    err_ = cudaSuccess;
    return e;
  }

 private:
  void loop() {
    cudaSetDevice(dev_);
    for (;;) {
      PipeJob j;
      {
        std::unique_lock<std::mutex> l(m_);
        cv_.wait(l, [&] { return stop_ || !q_.empty(); });
        if (q_.empty()) return;
        j = std::move(q_.front());
        q_.pop_front();
      }
      const cudaError_t e = run(j);
      {
        std::lock_guard<std::mutex> l(m_);
        if (e != cudaSuccess && err_ == cudaSuccess) err_ = e;
        issued_++;
        pending_[j.slot]--;
      }
      cv_.notify_all();
    }
  }
  cudaError_t run(const PipeJob& j) { return run_copy_job(j, cs_, pc_); }

  int dev_;
  cudaStream_t cs_;
  std::mutex m_;
  std::condition_variable cv_;
  std::deque<PipeJob> q_;
  bool stop_ = false;
  uint64_t pushed_ = 0, issued_ = 0;
  int pending_[2] = {0, 0};
  cudaError_t err_ = cudaSuccess;
  std::unique_ptr<PageableCopier> pc_;   // made by the thread on its first pageable copy
  std::thread th_;   // last member: started once the others exist
};

}  // namespace

struct rgf_ctx {
  rgf_opts opts;
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  DevBuf work, tasks, devs, info, queue, stage;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  rgf_stats stats;
  int8_t variant[kVariantSlots];  // kernel variant per block size (defaults; rgf_autotune may override)
  int8_t ctas[kVariantSlots];     // resident CTAs per SM per block size, 0 = as many as fit
  void* ext_cache = nullptr;      // per-context state of other modules (the FFT form's plans)
  void (*ext_cache_free)(void*) = nullptr;
  // pipelined host outputs (rgf_opts.pipelined): two staging slots used in
  // turn, each with its staging buffer, device and pinned task info, host-
  // mapped progress counters and events (solve done, copies done); the copy
  // stream and the copier thread that follows the counters
  DevBuf pipe_stage[2], pipe_dinfo[2];
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t pipe_free[2] = {nullptr, nullptr}, pipe_solved[2] = {nullptr, nullptr};
  DInfo* pipe_info[2] = {nullptr, nullptr};
  int32_t* pipe_prog[2] = {nullptr, nullptr};   // host-mapped, one counter per task
  int64_t pipe_cap[2] = {0, 0}, pipe_info_n[2] = {0, 0};
  int pipe_sel = 0, pipe_last = -1;
  std::vector<int64_t> pipe_nb[2];   // block size of each task of the call, for the stats
  std::unique_ptr<PipeWorker> worker;
  std::unique_ptr<PageableCopier> pcopy;   // the calling thread's copies to / from pageable arrays
  // synchronous calls whose staged outputs are copied while the solve runs:
  // host-mapped progress counters and the solve's event
  int32_t* sync_prog = nullptr;
  int64_t sync_prog_cap = 0;
  cudaEvent_t sync_solved = nullptr;
};

void* rgf::ctx_ext_cache(rgf_ctx* c) { return c->ext_cache; }
void rgf::ctx_set_ext_cache(rgf_ctx* c, void* cache, void (*free_fn)(void*)) {
  c->ext_cache = cache;
  c->ext_cache_free = free_fn;
}

extern "C" void rgf_opts_default(rgf_opts* o) {
  std::memset(o, 0, sizeof(*o));
  o->struct_size = (int32_t)sizeof(rgf_opts);
  o->device = 0;
  o->eta_dev = 0.0;
  o->eta_lead = 1e-3;
  o->boltz = 8.61734e-05;
  o->sancho_tol = 1e-100;
  o->sancho_nmax = 100;
  o->consistent = 0;
  o->precision = RGF_PREC_FP64;
  o->want_T = 1;
  o->verbose = 0;
  o->zero_copy = 1;
}

extern "C" const char* rgf_last_error(void) { return g_last_error.c_str(); }
extern "C" const char* rgf_version(void) { return "liteqt_b200 rgf 0.1 (sm_100a)"; }

static int check_opts(const rgf_opts* o) {
  if (!o) return fail(RGF_E_ARG, "opts is NULL");
  if (o->struct_size != (int32_t)sizeof(rgf_opts))
    return fail(RGF_E_ARG, "rgf_opts.struct_size %d != %zu (header mismatch)", o->struct_size,
                sizeof(rgf_opts));
  if (o->sancho_nmax < 1 || o->sancho_nmax > 100000) return fail(RGF_E_ARG, "sancho_nmax out of range");
  if (!(o->boltz > 0.0)) return fail(RGF_E_ARG, "boltz must be positive");
  if (o->precision != RGF_PREC_FP64 && o->precision != RGF_PREC_MIXED)
    return fail(RGF_E_ARG, "unknown precision %d", o->precision);
  return RGF_OK;
}

extern "C" int rgf_ctx_create(const rgf_opts* opts, rgf_ctx** out) {
  if (!out) return fail(RGF_E_ARG, "ctx out-pointer is NULL");
  *out = nullptr;
  rgf_opts def;
  if (!opts) {
    rgf_opts_default(&def);
    opts = &def;
  }
  int rc = check_opts(opts);
  if (rc) return rc;
  std::unique_ptr<rgf_ctx> c(new rgf_ctx());
  c->opts = *opts;
  c->device = opts->device;
  RGF_CUDA(cudaSetDevice(c->device));
  RGF_CUDA(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device));
  for (int i = 0; i < kVariantSlots; i++) {
    c->variant[i] = (int8_t)default_variant(i * 8);
    c->ctas[i] = 0;
  }
  RGF_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  RGF_CUDA(cudaEventCreate(&c->ev0));
  RGF_CUDA(cudaEventCreate(&c->ev1));
  std::memset(&c->stats, 0, sizeof(c->stats));
  *out = c.release();
  return RGF_OK;
}

extern "C" int rgf_ctx_destroy(rgf_ctx* c) {
  if (!c) return RGF_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  c->worker.reset();   // queues the copies of every pushed call, then stops
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
  if (c->ext_cache_free) c->ext_cache_free(c->ext_cache);
  for (int b = 0; b < 2; b++) {
    c->pipe_stage[b].release();
    c->pipe_dinfo[b].release();
    if (c->pipe_free[b]) cudaEventDestroy(c->pipe_free[b]);
    if (c->pipe_solved[b]) cudaEventDestroy(c->pipe_solved[b]);
    if (c->pipe_info[b]) cudaFreeHost(c->pipe_info[b]);
    if (c->pipe_prog[b]) cudaFreeHost(c->pipe_prog[b]);
  }
  if (c->sync_prog) cudaFreeHost(c->sync_prog);
  if (c->sync_solved) cudaEventDestroy(c->sync_solved);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  c->work.release();
  c->tasks.release();
  c->devs.release();
  c->info.release();
  c->queue.release();
  c->stage.release();
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  delete c;
  return RGF_OK;
}

extern "C" int rgf_ctx_get_stats(const rgf_ctx* c, rgf_stats* s) {
  if (!c || !s) return fail(RGF_E_ARG, "NULL argument");
  *s = c->stats;
  return RGF_OK;
}

// Waits for every queued solve and output copy of the context (pipelined
// calls), then completes the statistics of the last call.
extern "C" int rgf_ctx_synchronize(rgf_ctx* c) {
  if (!c) return fail(RGF_E_ARG, "ctx is NULL");
  RGF_CUDA(cudaSetDevice(c->device));
  if (c->worker) {
    c->worker->drain();
    const cudaError_t e = c->worker->take_error();
    if (e != cudaSuccess) return fail(RGF_E_CUDA, "pipelined output copies: %s", cudaGetErrorString(e));
  }
  if (c->copy_stream) RGF_CUDA(cudaStreamSynchronize(c->copy_stream));
  const int b = c->pipe_last;
  if (b >= 0) {
    double flops = 0.0, int8_ops = 0.0;
    for (int64_t t = 0; t < c->pipe_info_n[b]; t++) {
      const double nb = (double)c->pipe_nb[b][t];
      flops += 8.0 * nb * nb * nb * (double)(c->pipe_info[b][t].n_gemm + c->pipe_info[b][t].n_inv);
      int8_ops += 8.0 * nb * nb * nb * (double)c->pipe_info[b][t].pad;
    }
    float kms = 0.0f;
    RGF_CUDA(cudaEventElapsedTime(&kms, c->ev0, c->ev1));
    c->stats.last_kernel_ms = kms;
    c->stats.last_flops = flops;
    c->stats.last_int8_ops = int8_ops;
    c->pipe_last = -1;
  }
  return RGF_OK;
}

extern "C" int rgf_ctx_set_opts(rgf_ctx* c, const rgf_opts* o) {
  if (!c) return fail(RGF_E_ARG, "ctx is NULL");
  int rc = check_opts(o);
  if (rc) return rc;
  if (o->device != c->device) return fail(RGF_E_ARG, "cannot change the device of a context");
  c->opts = *o;
  return RGF_OK;
}

namespace {

// Staging of host arrays.  Every host range is registered with its role;
// touching or overlapping ranges are merged into segments (the per-energy
// slices of one host array become one copy), and each segment gets a region
// of one device buffer.
struct Stage {
  struct Item {
    const char* host;
    size_t bytes;
    bool copy_in;   // input, or output whose untouched parts must survive
    bool copy_out;  // output
    bool pageable;  // not page-locked: copied through the PageableCopier
  };
  struct Seg {
    const char* host;
    size_t bytes;
    size_t off;
    bool copy_in, copy_out, pageable;
  };
  // Pinned (page-locked, mapped) host outputs the kernels only write are not
  // staged: the kernels write them through their device mapping, so the
  // device-to-host transfer overlaps the solve instead of following it.
  struct Direct {
    const char* host;
    size_t bytes;
    char* dev;
  };
  std::vector<Item> items;
  std::vector<Seg> segs;
  std::vector<Direct> direct;
  size_t total = 0;
  bool zero_copy = true;

  void add(const void* p, size_t bytes, bool copy_in, bool copy_out, bool write_only = false) {
    if (!p || bytes == 0) return;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
      cudaGetLastError();
      a.type = cudaMemoryTypeUnregistered;
    }
    if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) return;
    if (zero_copy && write_only && copy_out && a.type == cudaMemoryTypeHost && a.devicePointer &&
        a.hostPointer) {
      const char* h = (const char*)p;
      const char* base = (const char*)a.hostPointer;
      if (h >= base) {
        direct.push_back({h, bytes, (char*)a.devicePointer + (h - base)});
        return;
      }
    }
    items.push_back({(const char*)p, bytes, copy_in, copy_out, a.type == cudaMemoryTypeUnregistered});
  }
  void layout() {
    std::vector<Item> v = items;
    std::sort(v.begin(), v.end(), [](const Item& a, const Item& b) { return a.host < b.host; });
    segs.clear();
    for (const Item& it : v) {
      if (!segs.empty() && it.host <= segs.back().host + segs.back().bytes) {
        Seg& s = segs.back();
        const char* end = std::max(s.host + s.bytes, it.host + it.bytes);
        s.bytes = (size_t)(end - s.host);
        s.copy_in = s.copy_in || it.copy_in;
        s.copy_out = s.copy_out || it.copy_out;
        s.pageable = s.pageable || it.pageable;
      } else {
        segs.push_back({it.host, it.bytes, 0, it.copy_in, it.copy_out, it.pageable});
      }
    }
    total = 0;
    for (Seg& s : segs) {
      s.off = total;
      total += (s.bytes + 255) & ~size_t(255);
    }
  }
  // the staged segment holding host address p, or nullptr (device memory,
  // written through its mapping, or NULL)
  const Seg* find(const void* p) const {
    if (!p) return nullptr;
    const char* h = (const char*)p;
    size_t lo = 0, hi = segs.size();
    while (lo < hi) {
      const size_t mid = (lo + hi) / 2;
      if (segs[mid].host <= h) lo = mid + 1; else hi = mid;
    }
    if (lo > 0 && h < segs[lo - 1].host + segs[lo - 1].bytes) return &segs[lo - 1];
    return nullptr;
  }
  // device address of a registered host pointer (or p itself if device / NULL)
  void* resolve(const void* p, char* dbase) const {
    if (!p) return nullptr;
    const char* h = (const char*)p;
    for (const Direct& d : direct)
      if (h >= d.host && h < d.host + d.bytes) return d.dev + (h - d.host);
    size_t lo = 0, hi = segs.size();
    while (lo < hi) {  // last segment with host <= h
      const size_t mid = (lo + hi) / 2;
      if (segs[mid].host <= h) lo = mid + 1; else hi = mid;
    }
    if (lo > 0) {
      const Seg& s = segs[lo - 1];
      if (h < s.host + s.bytes) return dbase + s.off + (size_t)(h - s.host);
    }
    return const_cast<void*>(p);
  }
};

}  // namespace

// The calling thread's copier for pageable host arrays (made on first use).
static PageableCopier& pageable_copier(rgf_ctx* c) {
  if (!c->pcopy) c->pcopy.reset(new PageableCopier());
  return *c->pcopy;
}

// Host -> staging copies of a call's input segments, after the work already
// on st: page-locked ones as stream copies, pageable ones through the
// PageableCopier (its sources are read when this returns).
static int stage_in(rgf_ctx* c, const Stage& sg, char* sbase, cudaStream_t st) {
  std::vector<PageableCopier::Copy> slow;
  for (const auto& s : sg.segs) {
    if (!s.copy_in) continue;
    if (s.pageable) slow.push_back({const_cast<char*>(s.host), sbase + s.off, s.bytes});
    else RGF_CUDA(cudaMemcpyAsync(sbase + s.off, s.host, s.bytes, cudaMemcpyHostToDevice, st));
  }
  if (!slow.empty()) RGF_CUDA(pageable_copier(c).h2d(slow, st));
  return RGF_OK;
}

// Staging -> host copies of a call's output segments, queued on st after the
// solve: the pageable ones are on the host when this returns, the others
// once st has drained.
static int stage_out(rgf_ctx* c, const Stage& sg, char* sbase, cudaStream_t st) {
  std::vector<PageableCopier::Copy> slow;
  for (const auto& s : sg.segs) {
    if (!s.copy_out) continue;
    if (s.pageable) slow.push_back({const_cast<char*>(s.host), sbase + s.off, s.bytes});
    else RGF_CUDA(cudaMemcpyAsync(const_cast<char*>(s.host), sbase + s.off, s.bytes, cudaMemcpyDeviceToHost, st));
  }
  if (!slow.empty()) RGF_CUDA(pageable_copier(c).d2h(slow, st));
  return RGF_OK;
}

// The copies of a solve's staged outputs for run_copy_job: every block-
// structured output by blocks (GRi1 / GLi1 / GGi1 without their last block,
// done one counter step later), and the rest of every output segment.
static void fill_copy_job(PipeJob& j, const rgf_device* devices, const rgf_task* tasks, int64_t n_tasks,
                          const Stage& sg, char* sbase) {
  std::vector<std::pair<const char*, const char*>> covered;   // host ranges copied block by block
  for (int64_t t = 0; t < n_tasks; t++) {
    const rgf_task& k = tasks[t];
    const rgf_device& v = devices[k.device];
    const size_t n2 = (size_t)v.nm * v.nm;
    const void* outs[7] = {k.ldos, k.ndens, k.pdens, k.GRi1, k.GLi1, k.GGi1, k.cur};
    for (int a = 0; a < 7; a++) {
      const Stage::Seg* sgm = sg.find(outs[a]);
      if (!sgm) continue;
      const size_t blk = n2 * (a == 6 ? sizeof(double) : sizeof(rgf_c16));
      char* h = (char*)outs[a];
      // GRi1 / GLi1 / GGi1: blocks 1 .. nx-1, done one counter step later
      const int32_t lag = (a >= 3 && a <= 5) ? 1 : 0;
      const int32_t nblk = (int32_t)v.nx - lag;
      j.blocks.push_back({h, (const char*)sg.resolve(outs[a], sbase), blk, t, nblk, lag, sgm->pageable});
      covered.push_back({h, h + blk * (size_t)nblk});
    }
  }
  std::sort(covered.begin(), covered.end());
  for (const auto& sgm : sg.segs) {   // the rest of every output segment
    if (!sgm.copy_out) continue;
    const char* end = sgm.host + sgm.bytes;
    const char* at = sgm.host;
    for (const auto& r : covered) {
      if (r.second <= at || r.first >= end) continue;
      if (r.first > at)
        j.rest.push_back({(char*)at, sbase + sgm.off + (at - sgm.host), (size_t)(r.first - at), sgm.pageable});
      at = std::max(at, r.second);
      if (at >= end) break;
    }
    if (at < end) j.rest.push_back({(char*)at, sbase + sgm.off + (at - sgm.host), (size_t)(end - at), sgm.pageable});
  }
}

// Kernel parameters common to every launch of a context.
static void fill_params(const rgf_ctx* c, KParams& p) {
  std::memset(&p, 0, sizeof(p));
  p.o.eta_dev = c->opts.eta_dev;
  p.o.eta_lead = c->opts.eta_lead;
  p.o.boltz = c->opts.boltz;
  p.o.sancho_tol = c->opts.sancho_tol;
  p.o.sancho_nmax = c->opts.sancho_nmax;
  p.o.consistent = c->opts.consistent;
  p.o.want_T = c->opts.want_T;
  std::memcpy(p.variant, c->variant, sizeof(p.variant));
}

// Resident CTAs per SM of a launch with this much dynamic shared memory over
// tasks of the block sizes in nb_mask (bit nb/8): the occupancy limit, or the
// smallest count the autotuner chose for one of those block sizes.
static int launch_ctas_per_sm(const rgf_ctx* c, size_t smem, uint64_t nb_mask) {
  int k = solver_blocks_per_sm(smem);
  for (int i = 0; i < kVariantSlots; i++)
    if (((nb_mask >> i) & 1) && c->ctas[i] > 0 && c->ctas[i] < k) k = c->ctas[i];
  return k;
}

// Checks a task list; RGF_OK or the error.
static int validate_batch(const rgf_device* devices, int32_t n_devices, const rgf_task* tasks,
                          int64_t n_tasks) {
  for (int32_t d = 0; d < n_devices; d++) {
    const rgf_device& v = devices[d];
    if (v.nm < 8 || v.nm > kMaxNb || v.nm % 8 != 0)
      return fail(RGF_E_UNSUPPORTED, "device %d: nm=%lld unsupported (multiple of 8 in [8,%d])", d,
                  (long long)v.nm, kMaxNb);
    if (v.nx < 2) return fail(RGF_E_ARG, "device %d: nx=%lld < 2", d, (long long)v.nx);
    if (!v.Hii || !v.H1i) return fail(RGF_E_ARG, "device %d: Hii/H1i is NULL", d);
    if (!(v.temp[0] > 0.0) || !(v.temp[1] > 0.0))
      return fail(RGF_E_ARG, "device %d: temperature must be > 0", d);
  }
  for (int64_t t = 0; t < n_tasks; t++)
    if (tasks[t].device < 0 || tasks[t].device >= n_devices)
      return fail(RGF_E_ARG, "task %lld: device index %d out of range", (long long)t, tasks[t].device);
  return RGF_OK;
}

// Launch geometry of a task list: queue order (descending estimated cost:
// nb^3 x (block operations of the chain + both leads)), slot size, dynamic
// shared memory and the block sizes present.
struct LaunchShape {
  std::vector<int32_t> order;
  int64_t slot = 0;
  size_t smem = 0;
  uint64_t nb_mask = 0;
};
static LaunchShape launch_shape(const rgf_ctx* c, const rgf_device* devices, const rgf_task* tasks,
                                int64_t n_tasks) {
  LaunchShape L;
  L.order.resize(n_tasks);
  std::vector<double> cost(n_tasks);
  for (int64_t t = 0; t < n_tasks; t++) {
    const rgf_device& v = devices[tasks[t].device];
    L.order[t] = (int32_t)t;
    cost[t] = (double)v.nm * v.nm * v.nm * (30.0 * (double)v.nx + 400.0);
    L.slot = std::max<int64_t>(L.slot, slot_elems_for(v.nm, v.nx));
    L.smem = std::max(L.smem, variant_smem(c->variant[v.nm / 8], (int)v.nm));
    L.nb_mask |= 1ull << (v.nm / 8);
  }
  std::stable_sort(L.order.begin(), L.order.end(), [&](int32_t a, int32_t b) { return cost[a] > cost[b]; });
  return L;
}

extern "C" int rgf_solve_batch(rgf_ctx* c, const rgf_device* devices, int32_t n_devices,
                               const rgf_task* tasks, int64_t n_tasks, rgf_task_info* info,
                               void* stream_) {
  if (!c) return fail(RGF_E_ARG, "ctx is NULL");
  if (n_tasks < 0 || (n_tasks > 0 && (!tasks || !devices || n_devices < 1)))
    return fail(RGF_E_ARG, "invalid task list");
  if (n_tasks == 0) return RGF_OK;
  if (n_tasks > (int64_t)INT32_MAX) return fail(RGF_E_ARG, "too many tasks in one batch");
  const bool mixed = c->opts.precision == RGF_PREC_MIXED;
  RGF_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = stream_ ? (cudaStream_t)stream_ : c->stream;
  const bool want_T = c->opts.want_T != 0;

  // ---- validate
  int rc = validate_batch(devices, n_devices, tasks, n_tasks);
  if (rc) return rc;
  if (mixed)
    for (int32_t d = 0; d < n_devices; d++) {
      if (devices[d].nm != 128)
        return fail(RGF_E_UNSUPPORTED, "RGF_PREC_MIXED: device %d has nm=%lld; the mixed form is built for nm=128",
                    d, (long long)devices[d].nm);
      if (devices[d].Sii)
        return fail(RGF_E_UNSUPPORTED, "RGF_PREC_MIXED: device %d has overlap blocks (green_RGF_CMS runs in FP64 "
                    "only)", d);
    }

  // ---- staging of host arrays.  Pipelined calls (no info requested)
  // stage in one of two buffers, taken in turn, and leave before the
  // outputs are on the host; the buffer waits for the copies of the call
  // that used it last.
  const bool pipe = c->opts.pipelined != 0 && info == nullptr;
  Stage sg;
  sg.zero_copy = c->opts.zero_copy != 0 && !pipe;
  for (int32_t d = 0; d < n_devices; d++) {
    const size_t bytes = (size_t)devices[d].nm * devices[d].nm * devices[d].nx * sizeof(rgf_c16);
    sg.add(devices[d].Hii, bytes, true, false);
    sg.add(devices[d].H1i, bytes, true, false);
    sg.add(devices[d].Sii, bytes, true, false);
  }
  for (int64_t t = 0; t < n_tasks; t++) {
    const rgf_task& k = tasks[t];
    const rgf_device& v = devices[k.device];
    const size_t cb = (size_t)v.nm * v.nm * v.nx * sizeof(rgf_c16);
    const size_t rb = (size_t)v.nm * v.nm * v.nx * sizeof(double);
    sg.add(k.sigma_lesser, cb, true, false);
    sg.add(k.sigma_r, cb, true, false);
    // the solver writes these and never reads them back (cur is read-modify-
    // written, so it is always staged)
    sg.add(k.ldos, cb, false, true, true);
    sg.add(k.ndens, cb, false, true, true);
    sg.add(k.pdens, cb, false, true, true);
    // block nx of GRi1 / GLi1 / GGi1 is never written (the reference leaves
    // it untouched): blocks 1 .. nx-1 alone are staged and copied back
    const size_t cb1 = cb - (size_t)v.nm * v.nm * sizeof(rgf_c16);
    sg.add(k.GRi1, cb1, false, true, true);
    sg.add(k.GLi1, cb1, false, true, true);
    sg.add(k.GGi1, cb1, false, true, true);
    sg.add(k.cur, rb, false, true);
    sg.add(k.tr, sizeof(double), false, true, true);
    sg.add(k.tre, sizeof(double), false, true, true);
    if (want_T) sg.add(k.T, sizeof(double), false, true, true);
  }
  sg.layout();
  const int pb = c->pipe_sel;
  if (pipe) {
    if (!c->worker) {
      RGF_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
      for (int b = 0; b < 2; b++) {
        RGF_CUDA(cudaEventCreateWithFlags(&c->pipe_free[b], cudaEventDisableTiming));
        RGF_CUDA(cudaEventCreateWithFlags(&c->pipe_solved[b], cudaEventDisableTiming));
        RGF_CUDA(cudaEventRecord(c->pipe_free[b], c->copy_stream));
      }
      c->worker.reset(new PipeWorker(c->device, c->copy_stream));
    }
    // the call that used this slot has queued its copies (its event is
    // recorded, its solve is done, its counters are no longer read)
    c->worker->wait_slot(pb);
    // buffers that must grow are freed only once their copies are done
    if (c->pipe_stage[pb].bytes < sg.total || c->pipe_cap[pb] < n_tasks)
      RGF_CUDA(cudaEventSynchronize(c->pipe_free[pb]));
    if (c->pipe_cap[pb] < n_tasks) {
      if (c->pipe_info[pb]) cudaFreeHost(c->pipe_info[pb]);
      if (c->pipe_prog[pb]) cudaFreeHost(c->pipe_prog[pb]);
      c->pipe_info[pb] = nullptr;
      c->pipe_prog[pb] = nullptr;
      c->pipe_cap[pb] = 0;
      RGF_CUDA(cudaMallocHost((void**)&c->pipe_info[pb], sizeof(DInfo) * (size_t)n_tasks));
      RGF_CUDA(cudaHostAlloc((void**)&c->pipe_prog[pb], sizeof(int32_t) * (size_t)n_tasks, cudaHostAllocMapped));
      c->pipe_cap[pb] = n_tasks;
    }
    if ((rc = c->pipe_dinfo[pb].reserve(sizeof(DInfo) * n_tasks))) return rc;
    std::memset(c->pipe_prog[pb], 0, sizeof(int32_t) * (size_t)n_tasks);
    RGF_CUDA(cudaStreamWaitEvent(st, c->pipe_free[pb], 0));
  } else if (c->worker) {
    // a call that is not pipelined may write the same host arrays: it
    // follows every queued copy
    c->worker->drain();
    for (int b = 0; b < 2; b++) RGF_CUDA(cudaStreamWaitEvent(st, c->pipe_free[b], 0));
  }
  DevBuf& stg = pipe ? c->pipe_stage[pb] : c->stage;
  rc = stg.reserve(std::max<size_t>(sg.total, 256));
  if (rc) return rc;
  char* sbase = (char*)stg.p;
  if ((rc = stage_in(c, sg, sbase, st))) return rc;

  // ---- device tables
  std::vector<DDev> ddev(n_devices);
  for (int32_t d = 0; d < n_devices; d++) {
    ddev[d].nm = devices[d].nm;
    ddev[d].nx = devices[d].nx;
    ddev[d].Hii = (const double2*)sg.resolve(devices[d].Hii, sbase);
    ddev[d].H1i = (const double2*)sg.resolve(devices[d].H1i, sbase);
    ddev[d].Sii = (const double2*)sg.resolve(devices[d].Sii, sbase);
    for (int i = 0; i < 2; i++) {
      ddev[d].mu[i] = devices[d].mu[i];
      ddev[d].temp[i] = devices[d].temp[i];
    }
  }
  std::vector<DTask> dtask(n_tasks);
  for (int64_t t = 0; t < n_tasks; t++) {
    const rgf_task& k = tasks[t];
    DTask& o = dtask[t];
    o.dev = k.device;
    o.pad = 0;
    o.E = k.E;
    o.sig_lesser = (const double2*)sg.resolve(k.sigma_lesser, sbase);
    o.sig_r = (const double2*)sg.resolve(k.sigma_r, sbase);
    o.ldos = (double2*)sg.resolve(k.ldos, sbase);
    o.ndens = (double2*)sg.resolve(k.ndens, sbase);
    o.pdens = (double2*)sg.resolve(k.pdens, sbase);
    o.GRi1 = (double2*)sg.resolve(k.GRi1, sbase);
    o.GLi1 = (double2*)sg.resolve(k.GLi1, sbase);
    o.GGi1 = (double2*)sg.resolve(k.GGi1, sbase);
    o.cur = (double*)sg.resolve(k.cur, sbase);
    o.tr = (double*)sg.resolve(k.tr, sbase);
    o.tre = (double*)sg.resolve(k.tre, sbase);
    o.T = want_T ? (double*)sg.resolve(k.T, sbase) : nullptr;
  }

  // ---- launch plan: one persistent launch for every block size, longest
  // tasks first, so the launch ends on its shortest tasks
  const LaunchShape shape = launch_shape(c, devices, tasks, n_tasks);
  const std::vector<int32_t>& order = shape.order;
  int64_t slot = shape.slot;
  const size_t smem = shape.smem;
  int grid = c->sm_count * launch_ctas_per_sm(c, smem, shape.nb_mask);
  if (mixed) {
    int64_t nx_max = 2;
    for (int32_t d = 0; d < n_devices; d++) nx_max = std::max<int64_t>(nx_max, devices[d].nx);
    slot = mixed_slot_elems(nx_max);
    grid = c->sm_count;   // one CTA per SM
  }
  if ((int64_t)grid > n_tasks) grid = (int)n_tasks;
  if ((rc = c->work.reserve(sizeof(double2) * (size_t)slot * grid))) return rc;
  if ((rc = c->devs.reserve(sizeof(DDev) * n_devices))) return rc;
  if ((rc = c->tasks.reserve(sizeof(DTask) * n_tasks + sizeof(int32_t) * n_tasks))) return rc;
  if ((rc = c->info.reserve(sizeof(DInfo) * n_tasks))) return rc;
  if ((rc = c->queue.reserve(sizeof(int32_t) * 64))) return rc;
  int32_t* order_d = (int32_t*)((char*)c->tasks.p + sizeof(DTask) * n_tasks);
  RGF_CUDA(cudaMemcpyAsync(c->devs.p, ddev.data(), sizeof(DDev) * n_devices, cudaMemcpyHostToDevice, st));
  RGF_CUDA(cudaMemcpyAsync(c->tasks.p, dtask.data(), sizeof(DTask) * n_tasks, cudaMemcpyHostToDevice, st));
  RGF_CUDA(cudaMemcpyAsync(order_d, order.data(), sizeof(int32_t) * n_tasks, cudaMemcpyHostToDevice, st));
  DInfo* dinfo = pipe ? (DInfo*)c->pipe_dinfo[pb].p : (DInfo*)c->info.p;
  RGF_CUDA(cudaMemsetAsync(dinfo, 0, sizeof(DInfo) * n_tasks, st));
  RGF_CUDA(cudaMemsetAsync(c->queue.p, 0, sizeof(int32_t), st));
  KParams p;
  fill_params(c, p);
  p.devs = (const DDev*)c->devs.p;
  p.tasks = (const DTask*)c->tasks.p;
  p.n_tasks = n_tasks;
  p.order = order_d;
  p.queue = (int32_t*)c->queue.p;
  p.work = (double2*)c->work.p;
  p.slot_elems = slot;
  p.info = dinfo;
  if (pipe) RGF_CUDA(cudaHostGetDevicePointer((void**)&p.progress, c->pipe_prog[pb], 0));
  // a synchronous call with at least kProgressiveBytes of staged outputs
  // copies them as the kernel reports their blocks written, like a
  // pipelined call, and returns once they are on the host
  constexpr size_t kProgressiveBytes = size_t(64) << 20;
  size_t staged_out = 0;
  for (const auto& sgm : sg.segs)
    if (sgm.copy_out) staged_out += sgm.bytes;
  const bool progressive = !pipe && staged_out >= kProgressiveBytes;
  if (progressive) {
    if (!c->copy_stream) RGF_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    if (!c->sync_solved) RGF_CUDA(cudaEventCreateWithFlags(&c->sync_solved, cudaEventDisableTiming));
    if (c->sync_prog_cap < n_tasks) {
      if (c->sync_prog) cudaFreeHost(c->sync_prog);
      c->sync_prog = nullptr;
      c->sync_prog_cap = 0;
      RGF_CUDA(cudaHostAlloc((void**)&c->sync_prog, sizeof(int32_t) * (size_t)n_tasks, cudaHostAllocMapped));
      c->sync_prog_cap = n_tasks;
    }
    std::memset(c->sync_prog, 0, sizeof(int32_t) * (size_t)n_tasks);
    RGF_CUDA(cudaHostGetDevicePointer((void**)&p.progress, c->sync_prog, 0));
  }
  RGF_CUDA(cudaEventRecord(c->ev0, st));
  cudaError_t e = mixed ? launch_mixed(p, grid, st) : launch_solver(p, grid, smem, st);
  if (e != cudaSuccess) return fail(RGF_E_CUDA, "solver launch failed: %s", cudaGetErrorString(e));
  c->stats.launches++;
  RGF_CUDA(cudaEventRecord(c->ev1, st));

  if (pipe) {
    // ---- outputs back: the copier queues them as the blocks are written;
    // the call returns now
    RGF_CUDA(cudaEventRecord(c->pipe_solved[pb], st));
    PipeJob j;
    j.slot = pb;
    j.prog = c->pipe_prog[pb];
    j.solved = c->pipe_solved[pb];
    j.freed = c->pipe_free[pb];
    fill_copy_job(j, devices, tasks, n_tasks, sg, sbase);
    j.rest.push_back({(char*)c->pipe_info[pb], (const char*)dinfo, sizeof(DInfo) * (size_t)n_tasks, false});
    c->worker->push(std::move(j));
    c->pipe_info_n[pb] = n_tasks;
    c->pipe_nb[pb].resize(n_tasks);
    for (int64_t t = 0; t < n_tasks; t++) c->pipe_nb[pb][t] = devices[tasks[t].device].nm;
    c->pipe_last = pb;
    c->pipe_sel ^= 1;
    c->stats.last_tasks = n_tasks;
    return RGF_OK;
  }

  // ---- outputs back
  if (progressive) {
    RGF_CUDA(cudaEventRecord(c->sync_solved, st));
    PipeJob j;
    j.prog = c->sync_prog;
    j.solved = c->sync_solved;
    j.freed = nullptr;
    fill_copy_job(j, devices, tasks, n_tasks, sg, sbase);
    RGF_CUDA(run_copy_job(j, c->copy_stream, c->pcopy));
    RGF_CUDA(cudaStreamSynchronize(c->copy_stream));
  } else if ((rc = stage_out(c, sg, sbase, st))) {
    return rc;
  }
  // the stream is drained before the task info comes back: a copy into
  // pageable memory that waits for a running kernel stalls other host
  // threads' launches (per-thread contexts then run one after another)
  RGF_CUDA(cudaStreamSynchronize(st));
  std::vector<DInfo> hinfo(n_tasks);
  RGF_CUDA(cudaMemcpyAsync(hinfo.data(), c->info.p, sizeof(DInfo) * n_tasks, cudaMemcpyDeviceToHost, st));
  RGF_CUDA(cudaStreamSynchronize(st));
  int worst = 0;
  double flops = 0.0, int8_ops = 0.0;
  for (int64_t t = 0; t < n_tasks; t++) {
    worst |= hinfo[t].status;
    const double nb = (double)devices[tasks[t].device].nm;
    flops += 8.0 * nb * nb * nb * (double)(hinfo[t].n_gemm + hinfo[t].n_inv);
    int8_ops += 8.0 * nb * nb * nb * (double)hinfo[t].pad;   // 4 real nb^3 products per digit pair
  }
  float kms = 0.0f;
  RGF_CUDA(cudaEventElapsedTime(&kms, c->ev0, c->ev1));
  c->stats.last_kernel_ms = kms;
  c->stats.last_flops = flops;
  c->stats.last_int8_ops = int8_ops;
  c->stats.last_tasks = n_tasks;
  if (info) std::memcpy(info, hinfo.data(), sizeof(DInfo) * n_tasks);
  if (c->opts.verbose && worst) {
    for (int64_t t = 0; t < n_tasks; t++) {
      if (hinfo[t].status & RGF_ST_SINGULAR)
        printf(" SEVERE warning: zgetrf failed (singular block), task %lld\n", (long long)t);
      if (hinfo[t].status & RGF_ST_SANCHO_NC)
        printf(" SEVERE warning: nmax reached in sancho!!! task %lld\n", (long long)t);
    }
  }
  if (worst & RGF_ST_BAD_TASK) return fail(RGF_E_ARG, "a task was rejected on the device");
  if (worst & RGF_ST_TIMEOUT) return fail(RGF_E_CUDA, "a tensor-core wait of the mixed form gave up");
  return (worst & ~RGF_ST_REFINE_NC) ? RGF_E_STATUS : RGF_OK;
}

// ------------------------------------------------------------------ blocks
// Batched block products and inverses in either form (device arrays).
static int block_args(rgf_ctx* c, int32_t precision, int64_t nb, int64_t count, std::initializer_list<const void*> ptrs) {
  if (!c) return fail(RGF_E_ARG, "ctx is NULL");
  if (precision != RGF_PREC_FP64 && precision != RGF_PREC_MIXED) return fail(RGF_E_ARG, "unknown precision %d", precision);
  if (count < 0) return fail(RGF_E_ARG, "count < 0");
  if (nb <= 0) return fail(RGF_E_ARG, "nb=%lld", (long long)nb);
  for (const void* p : ptrs)
    if (count > 0 && !is_device_ptr(p)) return fail(RGF_E_ARG, "block arrays must be device memory");
  return RGF_OK;
}

extern "C" int rgf_block_product(rgf_ctx* c, int32_t precision, int64_t nb, int64_t count, const rgf_c16* A,
                               int32_t conj_a, const rgf_c16* B, int32_t conj_b, rgf_c16* C, void* stream_) {
  int rc = block_args(c, precision, nb, count, {A, B, C});
  if (rc) return rc;
  if (nb != 128) return fail(RGF_E_UNSUPPORTED, "rgf_block_product: nb=%lld (built for 128)", (long long)nb);
  if (count == 0) return RGF_OK;
  RGF_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = stream_ ? (cudaStream_t)stream_ : c->stream;
  const int grid = (int)std::min<int64_t>(count, c->sm_count);
  if ((rc = c->work.reserve(sizeof(double2) * 5 * 128 * 128 * (size_t)grid))) return rc;
  if ((rc = c->info.reserve(sizeof(int32_t) * (size_t)count))) return rc;
  RGF_CUDA(cudaMemsetAsync(c->info.p, 0, sizeof(int32_t) * (size_t)count, st));
  const int mode = precision == RGF_PREC_MIXED ? 0 : 1;
  cudaError_t e = launch_block_mixed(mode, 0, (const double2*)A, conj_a, (const double2*)B, conj_b, (double2*)C,
                                     count, (double2*)c->work.p, grid, (int32_t*)c->info.p, st);
  if (e != cudaSuccess) return fail(RGF_E_CUDA, "block product launch failed: %s", cudaGetErrorString(e));
  RGF_CUDA(cudaStreamSynchronize(st));   // see rgf_solve_batch: no pageable copy behind a running kernel
  std::vector<int32_t> h((size_t)count);
  RGF_CUDA(cudaMemcpyAsync(h.data(), c->info.p, sizeof(int32_t) * (size_t)count, cudaMemcpyDeviceToHost, st));
  RGF_CUDA(cudaStreamSynchronize(st));
  for (int32_t v : h)
    if (v & RGF_ST_TIMEOUT) return fail(RGF_E_CUDA, "a tensor-core wait gave up");
  return RGF_OK;
}

extern "C" int rgf_block_inverse(rgf_ctx* c, int32_t precision, int64_t nb, int64_t count, const rgf_c16* X,
                              rgf_c16* Xinv, int32_t* status, void* stream_) {
  int rc = block_args(c, precision, nb, count, {X, Xinv});
  if (rc) return rc;
  const bool mixed = precision == RGF_PREC_MIXED;
  if (mixed ? nb != 128 : (nb != 32 && nb != 64 && nb != 128))
    return fail(RGF_E_UNSUPPORTED, "rgf_block_inverse: nb=%lld not built for this precision", (long long)nb);
  if (count == 0) return RGF_OK;
  RGF_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = stream_ ? (cudaStream_t)stream_ : c->stream;
  const int grid = (int)std::min<int64_t>(count, c->sm_count);
  if ((rc = c->work.reserve(sizeof(double2) * 5 * 128 * 128 * (size_t)grid))) return rc;
  if ((rc = c->info.reserve(sizeof(int32_t) * (size_t)count))) return rc;
  RGF_CUDA(cudaMemsetAsync(c->info.p, 0, sizeof(int32_t) * (size_t)count, st));
  cudaError_t e = mixed ? launch_block_mixed(2, 0, (const double2*)X, 0, nullptr, 0, (double2*)Xinv, count,
                                             (double2*)c->work.p, grid, (int32_t*)c->info.p, st)
                        : launch_block_fp64_inv((int)nb, (const double2*)X, (double2*)Xinv, count,
                                                (double2*)c->work.p, grid, (int32_t*)c->info.p, st);
  if (e != cudaSuccess) return fail(RGF_E_CUDA, "block inverse launch failed: %s", cudaGetErrorString(e));
  RGF_CUDA(cudaStreamSynchronize(st));   // see rgf_solve_batch: no pageable copy behind a running kernel
  std::vector<int32_t> h((size_t)count);
  RGF_CUDA(cudaMemcpyAsync(h.data(), c->info.p, sizeof(int32_t) * (size_t)count, cudaMemcpyDeviceToHost, st));
  RGF_CUDA(cudaStreamSynchronize(st));
  int worst = 0;
  for (int32_t v : h) worst |= v;
  if (status) std::memcpy(status, h.data(), sizeof(int32_t) * (size_t)count);
  if (worst & RGF_ST_TIMEOUT) return fail(RGF_E_CUDA, "a tensor-core wait gave up");
  return (worst & ~RGF_ST_REFINE_NC) ? RGF_E_STATUS : RGF_OK;
}

// ------------------------------------------------------------------ adjoint
extern "C" int rgf_adjoint_energies(rgf_ctx* c, const rgf_device* v, int64_t nen, const double* E,
                                    double* T, double* dTdV, double* dTds, double spindeg,
                                    double* dIdV, double* dIds, rgf_task_info* info, void* stream_) {
  if (!c || !v || !E || nen < 1) return fail(RGF_E_ARG, "invalid argument");
  if (v->nm < 8 || v->nm > kMaxNb || v->nm % 8 != 0)
    return fail(RGF_E_UNSUPPORTED, "nm=%lld unsupported (multiple of 8 in [8,%d])", (long long)v->nm, kMaxNb);
  if (v->nx < 2) return fail(RGF_E_ARG, "nx < 2");
  if (!v->Hii || !v->H1i) return fail(RGF_E_ARG, "Hii/H1i is NULL");
  if (v->Sii) return fail(RGF_E_UNSUPPORTED, "the adjoint is for an orthogonal basis (Sii must be NULL)");
  if (!(v->temp[0] > 0.0) || !(v->temp[1] > 0.0)) return fail(RGF_E_ARG, "temperature must be > 0");
  if ((dIdV || dIds) && nen < 2) return fail(RGF_E_ARG, "the current needs at least two energies");
  RGF_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = stream_ ? (cudaStream_t)stream_ : c->stream;
  const int64_t nx = v->nx, nm = v->nm;
  // staging: H (in), T / dTdV / dTds (out)
  Stage sg;
  const size_t hb = sizeof(rgf_c16) * (size_t)nm * nm * nx;
  sg.add(v->Hii, hb, true, false);
  sg.add(v->H1i, hb, true, false);
  sg.add(T, sizeof(double) * nen, false, true);
  sg.add(dTdV, sizeof(double) * nen * nx, false, true);
  sg.add(dTds, sizeof(double) * nen, false, true);
  sg.layout();
  int rc = c->stage.reserve(std::max<size_t>(sg.total, 256));
  if (rc) return rc;
  char* sbase = (char*)c->stage.p;
  if ((rc = stage_in(c, sg, sbase, st))) return rc;
  // the gradients are always produced on the device (the current needs them)
  const size_t grad_bytes = sizeof(double) * (size_t)nen * (nx + 2);
  double* dT_d = dTdV ? (double*)sg.resolve(dTdV, sbase) : nullptr;
  DDev dd;
  std::memset(&dd, 0, sizeof(dd));
  dd.nm = nm;
  dd.nx = nx;
  dd.Hii = (const double2*)sg.resolve(v->Hii, sbase);
  dd.H1i = (const double2*)sg.resolve(v->H1i, sbase);
  for (int i = 0; i < 2; i++) { dd.mu[i] = v->mu[i]; dd.temp[i] = v->temp[i]; }
  if ((rc = c->devs.reserve(sizeof(DDev)))) return rc;
  if ((rc = c->tasks.reserve(sizeof(DAdj) * nen + grad_bytes))) return rc;
  if ((rc = c->info.reserve(sizeof(DInfo) * nen))) return rc;
  if ((rc = c->queue.reserve(sizeof(int32_t) * 64))) return rc;
  char* tb = (char*)c->tasks.p;
  double* scratch = (double*)(tb + sizeof(DAdj) * nen);  // dTdV (if not given), T, dTds
  if (!dT_d) dT_d = scratch;
  double* T_d = T ? (double*)sg.resolve(T, sbase) : scratch + (size_t)nen * nx;
  double* ds_d = dTds ? (double*)sg.resolve(dTds, sbase) : scratch + (size_t)nen * nx + nen;
  std::vector<DAdj> tasks(nen);
  for (int64_t e = 0; e < nen; e++) {
    DAdj& a = tasks[e];
    a.dev = 0;
    a.pad = 0;
    a.E = E[e];
    a.T = T_d + e;
    a.dTdV = dT_d + e * nx;
    a.dTds = ds_d + e;
  }
  RGF_CUDA(cudaMemcpyAsync(c->devs.p, &dd, sizeof(DDev), cudaMemcpyHostToDevice, st));
  RGF_CUDA(cudaMemcpyAsync(tb, tasks.data(), sizeof(DAdj) * nen, cudaMemcpyHostToDevice, st));
  RGF_CUDA(cudaMemsetAsync(c->info.p, 0, sizeof(DInfo) * nen, st));
  RGF_CUDA(cudaMemsetAsync(c->queue.p, 0, sizeof(int32_t), st));
  const size_t smem = variant_smem(c->variant[nm / 8], (int)nm);
  int grid = c->sm_count * launch_ctas_per_sm(c, smem, 1ull << (nm / 8));
  if ((int64_t)grid > nen) grid = (int)nen;
  const int64_t slot = slot_elems_for(nm, nx);
  if ((rc = c->work.reserve(sizeof(double2) * (size_t)slot * grid))) return rc;
  KParams p;
  fill_params(c, p);
  p.o.want_T = 1;
  p.devs = (const DDev*)c->devs.p;
  p.n_tasks = nen;
  p.queue = (int32_t*)c->queue.p;
  p.work = (double2*)c->work.p;
  p.slot_elems = slot;
  p.info = (DInfo*)c->info.p;
  p.adj = (const DAdj*)tb;
  RGF_CUDA(cudaEventRecord(c->ev0, st));
  cudaError_t e = launch_solver(p, grid, smem, st);
  if (e != cudaSuccess) return fail(RGF_E_CUDA, "adjoint launch failed: %s", cudaGetErrorString(e));
  c->stats.launches++;
  RGF_CUDA(cudaEventRecord(c->ev1, st));
  // current derivatives: weighted energy sums on the device (fixed order)
  std::vector<double> w;
  if (dIdV || dIds) {
    const double kE0 = 1.6022e-19, kHbar = 1.0546e-34, kTpi = 3.14159265359 * 2.0;
    const double dE = E[1] - E[0];
    w.resize(nen);
    for (int64_t k = 0; k < nen; k++) {
      const double fl = 1.0 / (1.0 + std::exp((E[k] - v->mu[0]) / (c->opts.boltz * v->temp[0])));
      const double fr = 1.0 / (1.0 + std::exp((E[k] - v->mu[1]) / (c->opts.boltz * v->temp[1])));
      w[k] = (fl - fr) * dE * kE0 / kTpi / kHbar * kE0 * spindeg;
    }
  }
  if ((rc = stage_out(c, sg, sbase, st))) return rc;
  // the stream is drained before the task info comes back: a copy into
  // pageable memory that waits for a running kernel stalls other host
  // threads' launches (per-thread contexts then run one after another)
  RGF_CUDA(cudaStreamSynchronize(st));
  std::vector<double> hgrad;
  std::vector<double> hds;
  if (dIdV || dIds) {
    hgrad.resize((size_t)nen * nx);
    hds.resize(nen);
    RGF_CUDA(cudaMemcpyAsync(hgrad.data(), dT_d, sizeof(double) * nen * nx, cudaMemcpyDeviceToHost, st));
    RGF_CUDA(cudaMemcpyAsync(hds.data(), ds_d, sizeof(double) * nen, cudaMemcpyDeviceToHost, st));
  }
  std::vector<DInfo> hinfo(nen);
  RGF_CUDA(cudaMemcpyAsync(hinfo.data(), c->info.p, sizeof(DInfo) * nen, cudaMemcpyDeviceToHost, st));
  RGF_CUDA(cudaStreamSynchronize(st));
  float kms = 0.0f;
  RGF_CUDA(cudaEventElapsedTime(&kms, c->ev0, c->ev1));
  c->stats.last_kernel_ms = kms;
  c->stats.last_tasks = nen;
  double flops = 0.0;
  int worst = 0;
  for (int64_t k = 0; k < nen; k++) {
    worst |= hinfo[k].status;
    flops += 8.0 * (double)nm * nm * nm * (double)(hinfo[k].n_gemm + hinfo[k].n_inv);
  }
  c->stats.last_flops = flops;
  // energy sums in a fixed order (energies outermost, as the reference's loops)
  if (dIdV) {
    for (int64_t l = 0; l < nx; l++) dIdV[l] = 0.0;
    for (int64_t k = 0; k < nen; k++)
      for (int64_t l = 0; l < nx; l++) dIdV[l] += w[k] * hgrad[(size_t)k * nx + l];
  }
  if (dIds) {
    *dIds = 0.0;
    for (int64_t k = 0; k < nen; k++) *dIds += w[k] * hds[k];
  }
  if (info) std::memcpy(info, hinfo.data(), sizeof(DInfo) * nen);
  if (worst & RGF_ST_BAD_TASK) return fail(RGF_E_ARG, "a task was rejected on the device");
  return worst ? RGF_E_STATUS : RGF_OK;
}

// ------------------------------------------------------------------ drop-ins
namespace {

// One default context per host thread for the per-energy drop-ins (the
// reference calls them from `!$omp do` threads concurrently).
struct TlsCtx {
  rgf_ctx* ctx = nullptr;
  double boltz = 0.0;
  ~TlsCtx() { if (ctx) rgf_ctx_destroy(ctx); }
};
thread_local TlsCtx g_tls;

// ---- coalescing of concurrent per-energy calls
// The reference calls green_RGF_RS once per energy from `!$omp do` threads
// (green_rgf.f90:2916-2925).  Calls made without a context are queued
// process-wide; the first caller that finds no batch being formed becomes
// the leader: it keeps the queue open while new calls keep arriving (at most
// a few milliseconds), then runs every queued call with its BOLTZ as one
// rgf_solve_batch on a shared context -- one persistent launch, the shared
// Hamiltonian staged once -- and wakes the callers, each of which returns
// once its own outputs are written.  Calls that arrive meanwhile form the
// next batch.  RGF_DROPIN_COALESCE=0 in the environment switches this off
// (each thread then runs its call alone on a context of its own).
struct Pending {
  rgf_device dev;
  rgf_task task;
  double boltz;
  int rc;
  bool done;
};
struct Coalescer {
  std::mutex mu;
  std::condition_variable cv;
  std::vector<Pending*> queue;
  bool forming = false;
  rgf_ctx* ctx[2] = {nullptr, nullptr};   // by BOLTZ: green_RGF_RS / RGF_G
  double ctx_boltz[2] = {0.0, 0.0};
  std::string last_error;
};
Coalescer& coalescer() {
  static Coalescer* c = new Coalescer();   // never destroyed: process-lifetime contexts
  return *c;
}
bool coalescing_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("RGF_DROPIN_COALESCE");
    return !(e && e[0] == '0');
  }();
  return on;
}
bool same_device(const rgf_device& a, const rgf_device& b) {
  return a.nm == b.nm && a.nx == b.nx && a.Hii == b.Hii && a.H1i == b.H1i && a.Sii == b.Sii &&
         a.mu[0] == b.mu[0] && a.mu[1] == b.mu[1] && a.temp[0] == b.temp[0] && a.temp[1] == b.temp[1];
}

// Runs one batch (leader, without the lock): every call of `batch` shares
// `boltz`.
void run_batch(Coalescer& co, std::vector<Pending*>& batch, double boltz) {
  int slot = 0;
  {
    std::lock_guard<std::mutex> g(co.mu);
    for (slot = 0; slot < 2; slot++)
      if (!co.ctx[slot] || co.ctx_boltz[slot] == boltz) break;
  }
  int rc = RGF_OK;
  if (slot == 2) slot = 1;
  if (!co.ctx[slot] || co.ctx_boltz[slot] != boltz) {
    if (co.ctx[slot]) rgf_ctx_destroy(co.ctx[slot]);
    co.ctx[slot] = nullptr;
    rgf_opts o;
    rgf_opts_default(&o);
    o.boltz = boltz;
    o.want_T = 0;
    o.pipelined = 1;   // the batch's host copies run while it solves (synchronised below)
    rc = rgf_ctx_create(&o, &co.ctx[slot]);
    co.ctx_boltz[slot] = boltz;
  }
  if (rc == RGF_OK) {
    std::vector<rgf_device> devs;
    std::vector<rgf_task> tasks;
    tasks.reserve(batch.size());
    for (Pending* p : batch) {
      int d = 0;
      while (d < (int)devs.size() && !same_device(devs[d], p->dev)) d++;
      if (d == (int)devs.size()) devs.push_back(p->dev);
      rgf_task t = p->task;
      t.device = d;
      tasks.push_back(t);
    }
    rc = rgf_solve_batch(co.ctx[slot], devs.data(), (int32_t)devs.size(), tasks.data(), (int64_t)tasks.size(),
                         nullptr, nullptr);
    if (rc == RGF_OK) rc = rgf_ctx_synchronize(co.ctx[slot]);   // every output on the host
    // the batch is complete, so the next one may take the same staging
    // buffer: the context lives as long as the process, and one buffer of
    // the batch's output size is what it then holds instead of two
    co.ctx[slot]->pipe_sel = 0;
  }
  const std::string err = rc ? rgf_last_error() : std::string();
  std::lock_guard<std::mutex> g(co.mu);
  if (rc) co.last_error = err;
  for (Pending* p : batch) {
    p->rc = rc;
    p->done = true;
  }
}

int solve_coalesced(const rgf_device& dev, const rgf_task& task, double boltz) {
  Coalescer& co = coalescer();
  Pending me{dev, task, boltz, RGF_OK, false};
  std::unique_lock<std::mutex> lk(co.mu);
  co.queue.push_back(&me);
  co.cv.notify_all();
  while (!me.done) {
    if (co.forming) {
      co.cv.wait(lk);
      continue;
    }
    co.forming = true;
    // collection window: while calls keep arriving (each within 200 us of
    // the previous), for at most 5 ms
    const auto t0 = std::chrono::steady_clock::now();
    size_t seen = co.queue.size();
    for (;;) {
      co.cv.wait_for(lk, std::chrono::microseconds(200));
      const auto dt = std::chrono::steady_clock::now() - t0;
      if (co.queue.size() == seen || dt > std::chrono::milliseconds(5)) break;
      seen = co.queue.size();
    }
    std::vector<Pending*> batch, rest;
    const double b = co.queue.front()->boltz;
    for (Pending* p : co.queue) (p->boltz == b ? batch : rest).push_back(p);
    co.queue.swap(rest);
    lk.unlock();
    run_batch(co, batch, b);
    lk.lock();
    co.forming = false;
    co.cv.notify_all();
  }
  if (me.rc) g_last_error = co.last_error;
  return me.rc;
}

rgf_ctx* default_ctx(double boltz, int* rc) {
  if (!g_tls.ctx) {
    rgf_opts o;
    rgf_opts_default(&o);
    o.boltz = boltz;
    *rc = rgf_ctx_create(&o, &g_tls.ctx);
    if (*rc) return nullptr;
  }
  if (g_tls.ctx->opts.boltz != boltz) g_tls.ctx->opts.boltz = boltz;
  *rc = RGF_OK;
  return g_tls.ctx;
}

int solve_one(rgf_ctx* ctx, double boltz, const double* temp, const int64_t* nm, const int64_t* nx,
              const double* E, const double* mu, const rgf_c16* Sii, const rgf_c16* Hii, const rgf_c16* H1i,
              const rgf_c16* sl, const rgf_c16* sr, rgf_c16* ndens, rgf_c16* pdens, rgf_c16* ldos,
              double* tr, double* tre, double* cur, rgf_c16* GRi1, rgf_c16* GLi1, rgf_c16* GGi1) {
  if (!temp || !nm || !nx || !E || !mu) return fail(RGF_E_ARG, "NULL scalar argument");
  int rc = RGF_OK;
  double saved_boltz = 0.0;
  if (!ctx && coalescing_enabled()) {
    rgf_device d;
    std::memset(&d, 0, sizeof(d));
    d.nm = *nm;
    d.nx = *nx;
    d.Sii = Sii;
    d.Hii = Hii;
    d.H1i = H1i;
    d.mu[0] = mu[0];
    d.mu[1] = mu[1];
    d.temp[0] = temp[0];
    d.temp[1] = temp[1];
    rgf_task t;
    std::memset(&t, 0, sizeof(t));
    t.E = *E;
    t.sigma_lesser = sl;
    t.sigma_r = sr;
    t.ldos = ldos;
    t.ndens = ndens;
    t.pdens = pdens;
    t.GRi1 = GRi1;
    t.GLi1 = GLi1;
    t.GGi1 = GGi1;
    t.cur = cur;
    t.tr = tr;
    t.tre = tre;
    return solve_coalesced(d, t, boltz);
  }
  if (!ctx) {
    ctx = default_ctx(boltz, &rc);
    if (!ctx) return rc;
  } else {
    saved_boltz = ctx->opts.boltz;
    ctx->opts.boltz = boltz;
  }
  rgf_device d;
  std::memset(&d, 0, sizeof(d));
  d.nm = *nm;
  d.nx = *nx;
  d.Sii = Sii;
  d.Hii = Hii;
  d.H1i = H1i;
  d.mu[0] = mu[0];
  d.mu[1] = mu[1];
  d.temp[0] = temp[0];
  d.temp[1] = temp[1];
  rgf_task t;
  std::memset(&t, 0, sizeof(t));
  t.device = 0;
  t.E = *E;
  t.sigma_lesser = sl;
  t.sigma_r = sr;
  t.ldos = ldos;
  t.ndens = ndens;
  t.pdens = pdens;
  t.GRi1 = GRi1;
  t.GLi1 = GLi1;
  t.GGi1 = GGi1;
  t.cur = cur;
  t.tr = tr;
  t.tre = tre;
  const int keepT = ctx->opts.want_T;
  ctx->opts.want_T = 0;
  rc = rgf_solve_batch(ctx, &d, 1, &t, 1, nullptr, nullptr);
  ctx->opts.want_T = keepT;
  if (saved_boltz != 0.0) ctx->opts.boltz = saved_boltz;
  // the reference has no error return: status bits only mean "SEVERE warning"
  return rc == RGF_E_STATUS ? RGF_OK : rc;
}

}  // namespace

extern "C" int rgf_green_rgf_rs(rgf_ctx* ctx, const double* temp, const int64_t* nm, const int64_t* nx,
                                const double* E, const double* mu, const rgf_c16* Hii,
                                const rgf_c16* H1i, const rgf_c16* sigma_lesser_ph,
                                const rgf_c16* sigma_greater_ph, const rgf_c16* sigma_r_ph,
                                rgf_c16* ndens, rgf_c16* pdens, rgf_c16* ldos, double* tr,
                                double* tre, double* cur, rgf_c16* GRi1, rgf_c16* GLi1,
                                rgf_c16* GGi1) {
  (void)sigma_greater_ph;  // unused by the reference as well
  return solve_one(ctx, 8.61734e-05, temp, nm, nx, E, mu, nullptr, Hii, H1i, sigma_lesser_ph, sigma_r_ph,
                   ndens, pdens, ldos, tr, tre, cur, GRi1, GLi1, GGi1);
}

extern "C" int rgf_green_rgf_cms(rgf_ctx* ctx, const double* temp, const int64_t* nm, const int64_t* nx,
                                 const double* E, const double* mu, const rgf_c16* Sii,
                                 const rgf_c16* Hii, const rgf_c16* H1i,
                                 const rgf_c16* sigma_lesser_ph, const rgf_c16* sigma_greater_ph,
                                 const rgf_c16* sigma_r_ph, rgf_c16* ndens, rgf_c16* pdens,
                                 rgf_c16* ldos, double* tr, double* tre, double* cur, rgf_c16* GRi1,
                                 rgf_c16* GLi1, rgf_c16* GGi1) {
  (void)sigma_greater_ph;  // unused by the reference as well
  if (!Sii) return fail(RGF_E_ARG, "green_RGF_CMS needs the overlap blocks Sii");
  return solve_one(ctx, 8.61734e-05, temp, nm, nx, E, mu, Sii, Hii, H1i, sigma_lesser_ph, sigma_r_ph,
                   ndens, pdens, ldos, tr, tre, cur, GRi1, GLi1, GGi1);
}

extern "C" int rgf_rgf_g(rgf_ctx* ctx, const double* temperature, const int64_t* nm,
                         const int64_t* nx, const double* E, const double* mu, const rgf_c16* Hii,
                         const rgf_c16* H1i, const rgf_c16* sigma_lesser_ph,
                         const rgf_c16* sigma_greater_ph, const rgf_c16* sigma_r_ph, double* tr,
                         double* tre, rgf_c16* ndens, rgf_c16* pdens, rgf_c16* ldos, double* cur,
                         rgf_c16* GRi1, rgf_c16* GLi1, rgf_c16* GGi1) {
  (void)sigma_greater_ph;
  return solve_one(ctx, 8.617333262e-05, temperature, nm, nx, E, mu, nullptr, Hii, H1i, sigma_lesser_ph,
                   sigma_r_ph, ndens, pdens, ldos, tr, tre, cur, GRi1, GLi1, GGi1);
}

extern "C" int rgf_solve_energies(rgf_ctx* ctx, const rgf_device* device, int64_t nen,
                                  const double* E, const rgf_c16* sigma_lesser,
                                  const rgf_c16* sigma_r, rgf_c16* ldos, rgf_c16* ndens,
                                  rgf_c16* pdens, rgf_c16* GRi1, double* cur, double* tr,
                                  double* tre, double* T, rgf_task_info* info, void* stream) {
  if (!ctx || !device || !E || nen < 0) return fail(RGF_E_ARG, "invalid argument");
  const size_t per = (size_t)device->nm * device->nm * device->nx;
  std::vector<rgf_task> tasks(nen);
  for (int64_t e = 0; e < nen; e++) {
    rgf_task& t = tasks[e];
    std::memset(&t, 0, sizeof(t));
    t.device = 0;
    t.E = E[e];
    t.sigma_lesser = sigma_lesser ? sigma_lesser + e * per : nullptr;
    t.sigma_r = sigma_r ? sigma_r + e * per : nullptr;
    t.ldos = ldos ? ldos + e * per : nullptr;
    t.ndens = ndens ? ndens + e * per : nullptr;
    t.pdens = pdens ? pdens + e * per : nullptr;
    t.GRi1 = GRi1 ? GRi1 + e * per : nullptr;
    t.cur = cur ? cur + e * per : nullptr;
    t.tr = tr ? tr + e : nullptr;
    t.tre = tre ? tre + e : nullptr;
    t.T = T ? T + e : nullptr;
  }
  return rgf_solve_batch(ctx, device, 1, tasks.data(), nen, info, stream);
}

// ------------------------------------------------------------------ plans
struct rgf_plan {
  rgf_ctx* ctx = nullptr;
  int64_t n_tasks = 0;
  std::vector<int> task_nb;
  DevBuf work, tasks, devs, info, queue;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~rgf_plan() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    work.release();
    tasks.release();
    devs.release();
    info.release();
    queue.release();
  }
};

extern "C" int rgf_plan_create(rgf_ctx* c, const rgf_device* devices, int32_t n_devices,
                               const rgf_task* tasks, int64_t n_tasks, rgf_plan** out) {
  if (!c || !out) return fail(RGF_E_ARG, "NULL argument");
  *out = nullptr;
  if (n_tasks < 1 || !tasks || !devices || n_devices < 1) return fail(RGF_E_ARG, "invalid task list");
  if (n_tasks > (int64_t)INT32_MAX) return fail(RGF_E_ARG, "too many tasks in one plan");
  if (c->opts.precision != RGF_PREC_FP64)
    return fail(RGF_E_UNSUPPORTED, "precision mode %d is not available in this build", c->opts.precision);
  int rc = validate_batch(devices, n_devices, tasks, n_tasks);
  if (rc) return rc;
  RGF_CUDA(cudaSetDevice(c->device));
  auto dev_ok = [](const void* p) { return !p || is_device_ptr(p); };
  for (int32_t d = 0; d < n_devices; d++)
    if (!dev_ok(devices[d].Hii) || !dev_ok(devices[d].H1i) || !dev_ok(devices[d].Sii))
      return fail(RGF_E_ARG, "device %d: plan arrays must be device memory", d);
  const bool want_T = c->opts.want_T != 0;
  std::vector<DDev> ddev(n_devices);
  for (int32_t d = 0; d < n_devices; d++) {
    ddev[d].nm = devices[d].nm;
    ddev[d].nx = devices[d].nx;
    ddev[d].Hii = (const double2*)devices[d].Hii;
    ddev[d].H1i = (const double2*)devices[d].H1i;
    ddev[d].Sii = (const double2*)devices[d].Sii;
    for (int i = 0; i < 2; i++) {
      ddev[d].mu[i] = devices[d].mu[i];
      ddev[d].temp[i] = devices[d].temp[i];
    }
  }
  std::unique_ptr<rgf_plan> pl(new rgf_plan());
  pl->ctx = c;
  pl->n_tasks = n_tasks;
  pl->task_nb.resize(n_tasks);
  std::vector<DTask> dtask(n_tasks);
  for (int64_t t = 0; t < n_tasks; t++) {
    const rgf_task& k = tasks[t];
    const void* ptrs[] = {k.sigma_lesser, k.sigma_r, k.ldos, k.ndens, k.pdens, k.GRi1, k.GLi1,
                          k.GGi1, k.cur, k.tr, k.tre, want_T ? k.T : nullptr};
    for (const void* q : ptrs)
      if (!dev_ok(q)) return fail(RGF_E_ARG, "task %lld: plan arrays must be device memory", (long long)t);
    DTask& o = dtask[t];
    std::memset(&o, 0, sizeof(o));
    o.dev = k.device;
    o.E = k.E;
    o.sig_lesser = (const double2*)k.sigma_lesser;
    o.sig_r = (const double2*)k.sigma_r;
    o.ldos = (double2*)k.ldos;
    o.ndens = (double2*)k.ndens;
    o.pdens = (double2*)k.pdens;
    o.GRi1 = (double2*)k.GRi1;
    o.GLi1 = (double2*)k.GLi1;
    o.GGi1 = (double2*)k.GGi1;
    o.cur = k.cur;
    o.tr = k.tr;
    o.tre = k.tre;
    o.T = want_T ? k.T : nullptr;
    pl->task_nb[t] = (int)devices[k.device].nm;
  }
  const LaunchShape shape = launch_shape(c, devices, tasks, n_tasks);
  int grid = c->sm_count * launch_ctas_per_sm(c, shape.smem, shape.nb_mask);
  if ((int64_t)grid > n_tasks) grid = (int)n_tasks;
  if ((rc = pl->work.reserve(sizeof(double2) * (size_t)shape.slot * grid))) return rc;
  if ((rc = pl->devs.reserve(sizeof(DDev) * n_devices))) return rc;
  if ((rc = pl->tasks.reserve(sizeof(DTask) * n_tasks + sizeof(int32_t) * n_tasks))) return rc;
  if ((rc = pl->info.reserve(sizeof(DInfo) * n_tasks))) return rc;
  if ((rc = pl->queue.reserve(256))) return rc;
  int32_t* order_d = (int32_t*)((char*)pl->tasks.p + sizeof(DTask) * n_tasks);
  RGF_CUDA(cudaMemcpy(pl->devs.p, ddev.data(), sizeof(DDev) * n_devices, cudaMemcpyHostToDevice));
  RGF_CUDA(cudaMemcpy(pl->tasks.p, dtask.data(), sizeof(DTask) * n_tasks, cudaMemcpyHostToDevice));
  RGF_CUDA(cudaMemcpy(order_d, shape.order.data(), sizeof(int32_t) * n_tasks, cudaMemcpyHostToDevice));
  KParams p;
  fill_params(c, p);
  p.devs = (const DDev*)pl->devs.p;
  p.tasks = (const DTask*)pl->tasks.p;
  p.n_tasks = n_tasks;
  p.order = order_d;
  p.queue = (int32_t*)pl->queue.p;
  p.work = (double2*)pl->work.p;
  p.slot_elems = shape.slot;
  p.info = (DInfo*)pl->info.p;
  solver_blocks_per_sm(shape.smem);  // raises the kernel's shared-memory limit before the capture
  cudaStream_t cs = nullptr;
  RGF_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    cudaError_t e1 = cudaMemsetAsync(pl->queue.p, 0, sizeof(int32_t), cs);
    cudaError_t e2 = cudaMemsetAsync(pl->info.p, 0, sizeof(DInfo) * n_tasks, cs);
    cudaError_t e3 = launch_solver(p, grid, shape.smem, cs, false);
    e = cudaStreamEndCapture(cs, &pl->graph);
    if (e == cudaSuccess) e = e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&pl->exec, pl->graph, 0);
  cudaStreamDestroy(cs);
  if (e != cudaSuccess) return fail(RGF_E_CUDA, "plan capture failed: %s", cudaGetErrorString(e));
  *out = pl.release();
  return RGF_OK;
}

extern "C" int rgf_plan_execute(rgf_plan* pl, rgf_task_info* info, void* stream_) {
  if (!pl || !pl->ctx) return fail(RGF_E_ARG, "plan is NULL");
  rgf_ctx* c = pl->ctx;
  RGF_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = stream_ ? (cudaStream_t)stream_ : c->stream;
  RGF_CUDA(cudaEventRecord(c->ev0, st));
  RGF_CUDA(cudaGraphLaunch(pl->exec, st));
  RGF_CUDA(cudaEventRecord(c->ev1, st));
  c->stats.launches++;
  if (!info) return RGF_OK;
  std::vector<DInfo> h(pl->n_tasks);
  RGF_CUDA(cudaStreamSynchronize(st));   // see rgf_solve_batch: no pageable copy behind a running kernel
  RGF_CUDA(cudaMemcpyAsync(h.data(), pl->info.p, sizeof(DInfo) * pl->n_tasks, cudaMemcpyDeviceToHost, st));
  RGF_CUDA(cudaStreamSynchronize(st));
  int worst = 0;
  double flops = 0.0;
  for (int64_t t = 0; t < pl->n_tasks; t++) {
    worst |= h[t].status;
    const double nb = (double)pl->task_nb[t];
    flops += 8.0 * nb * nb * nb * (double)(h[t].n_gemm + h[t].n_inv);
  }
  float kms = 0.0f;
  RGF_CUDA(cudaEventElapsedTime(&kms, c->ev0, c->ev1));
  c->stats.last_kernel_ms = kms;
  c->stats.last_flops = flops;
  c->stats.last_tasks = pl->n_tasks;
  std::memcpy(info, h.data(), sizeof(DInfo) * pl->n_tasks);
  if (worst & RGF_ST_BAD_TASK) return fail(RGF_E_ARG, "a task was rejected on the device");
  return worst ? RGF_E_STATUS : RGF_OK;
}

extern "C" int rgf_plan_destroy(rgf_plan* pl) {
  if (!pl) return RGF_OK;
  if (pl->ctx) cudaSetDevice(pl->ctx->device);
  cudaDeviceSynchronize();
  delete pl;
  return RGF_OK;
}

// --------------------------------------------------------------- autotuner
extern "C" const char* rgf_variant_name(int32_t v) { return variant_name(v); }

extern "C" int rgf_autotune(rgf_ctx* c, const rgf_device* v, rgf_tune_result* res) {
  if (!c || !v) return fail(RGF_E_ARG, "NULL argument");
  rgf_task dummy;
  std::memset(&dummy, 0, sizeof(dummy));
  int rc = validate_batch(v, 1, &dummy, 1);
  if (rc) return rc;
  RGF_CUDA(cudaSetDevice(c->device));
  const int nb = (int)v->nm;
  const int64_t nxp = std::min<int64_t>(v->nx, 12);
  const size_t blk = (size_t)nb * nb;
  // probe device: the first nxp blocks, on the device
  rgf_device pd = *v;
  pd.nx = nxp;
  void* hbuf = nullptr;
  if (!is_device_ptr(v->Hii) || !is_device_ptr(v->H1i)) {
    RGF_CUDA(cudaMalloc(&hbuf, 2 * sizeof(rgf_c16) * blk * nxp));
    RGF_CUDA(cudaMemcpy(hbuf, v->Hii, sizeof(rgf_c16) * blk * nxp,
                        is_device_ptr(v->Hii) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice));
    RGF_CUDA(cudaMemcpy((rgf_c16*)hbuf + blk * nxp, v->H1i, sizeof(rgf_c16) * blk * nxp,
                        is_device_ptr(v->H1i) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice));
    pd.Hii = (const rgf_c16*)hbuf;
    pd.H1i = (const rgf_c16*)hbuf + blk * nxp;
  }
  struct Cand { int v, k; double us; };
  std::vector<Cand> cands;
  int kmax_all = 1;
  for (int vv = 0; vv < KV_COUNT; vv++) {
    if (!variant_ok(vv, nb)) continue;
    const int occ = solver_blocks_per_sm(variant_smem(vv, nb));
    kmax_all = std::max(kmax_all, occ);
    cands.push_back({vv, 1, 0.0});
    if (occ > 1) cands.push_back({vv, occ, 0.0});
  }
  if (cands.size() > 16) cands.resize(16);
  const int64_t nen_max = (int64_t)c->sm_count * kmax_all;
  void* obuf = nullptr;
  const size_t gbytes = sizeof(rgf_c16) * blk * nxp * nen_max;
  cudaError_t ae = cudaMalloc(&obuf, 2 * gbytes + sizeof(double) * nen_max);
  if (ae != cudaSuccess) {
    cudaGetLastError();
    if (hbuf) cudaFree(hbuf);
    return fail(RGF_E_NOMEM, "autotune: cudaMalloc of the probe outputs failed");
  }
  rgf_c16* ldos = (rgf_c16*)obuf;
  rgf_c16* ndens = (rgf_c16*)((char*)obuf + gbytes);
  double* T = (double*)((char*)obuf + 2 * gbytes);
  const int8_t keep_v = c->variant[nb / 8], keep_k = c->ctas[nb / 8];
  const int32_t keep_T = c->opts.want_T;
  c->opts.want_T = 1;
  rc = RGF_OK;
  for (Cand& cd : cands) {
    c->variant[nb / 8] = (int8_t)cd.v;
    c->ctas[nb / 8] = (int8_t)cd.k;
    const int64_t nen = (int64_t)c->sm_count * cd.k;
    std::vector<double> E(nen);
    for (int64_t i = 0; i < nen; i++) E[i] = -3.0 + 6.0 * ((double)i + 0.5) / (double)nen;
    double best = 1e300;
    for (int rep = 0; rep < 3 && rc == RGF_OK; rep++) {  // first run warms up
      int r = rgf_solve_energies(c, &pd, nen, E.data(), nullptr, nullptr, ldos, ndens, nullptr, nullptr,
                                 nullptr, nullptr, nullptr, T, nullptr, nullptr);
      if (r != RGF_OK && r != RGF_E_STATUS) rc = r;
      if (rep > 0) best = std::min(best, c->stats.last_kernel_ms);
    }
    cd.us = best * 1e3 / (double)nen;
  }
  c->opts.want_T = keep_T;
  cudaFree(obuf);
  if (hbuf) cudaFree(hbuf);
  if (rc != RGF_OK) {
    c->variant[nb / 8] = keep_v;
    c->ctas[nb / 8] = keep_k;
    return rc;
  }
  size_t bi = 0;
  for (size_t i = 1; i < cands.size(); i++)
    if (cands[i].us < cands[bi].us) bi = i;
  c->variant[nb / 8] = (int8_t)cands[bi].v;
  c->ctas[nb / 8] = (int8_t)cands[bi].k;
  if (res) {
    std::memset(res, 0, sizeof(*res));
    res->nb = nb;
    res->variant = cands[bi].v;
    res->ctas_per_sm = cands[bi].k;
    res->n_candidates = (int32_t)cands.size();
    for (size_t i = 0; i < cands.size(); i++) {
      res->cand_variant[i] = cands[i].v;
      res->cand_ctas_per_sm[i] = cands[i].k;
      res->cand_us_per_energy[i] = cands[i].us;
    }
  }
  return RGF_OK;
}

// ------------------------------------------------------------- W solves
extern "C" int rgf_w_solve_batch(rgf_ctx* c, const rgf_w_device* devices, int32_t n_devices,
                                 const rgf_w_task* tasks, int64_t n_tasks, rgf_task_info* info,
                                 void* stream_) {
  if (!c) return fail(RGF_E_ARG, "ctx is NULL");
  if (n_tasks < 0 || (n_tasks > 0 && (!tasks || !devices || n_devices < 1)))
    return fail(RGF_E_ARG, "invalid task list");
  if (n_tasks == 0) return RGF_OK;
  if (n_tasks > (int64_t)INT32_MAX) return fail(RGF_E_ARG, "too many tasks in one batch");
  for (int32_t d = 0; d < n_devices; d++) {
    const rgf_w_device& v = devices[d];
    if (v.nm < 8 || v.nm > kMaxNb || v.nm % 8 != 0)
      return fail(RGF_E_UNSUPPORTED, "device %d: nm=%lld unsupported (multiple of 8 in [8,%d])", d,
                  (long long)v.nm, kMaxNb);
    if (v.nx < 2) return fail(RGF_E_ARG, "device %d: nx=%lld < 2", d, (long long)v.nx);
    if (!v.Vii || !v.V1i) return fail(RGF_E_ARG, "device %d: Vii/V1i is NULL", d);
  }
  for (int64_t t = 0; t < n_tasks; t++) {
    const rgf_w_task& k = tasks[t];
    if (k.device < 0 || k.device >= n_devices)
      return fail(RGF_E_ARG, "task %lld: device index %d out of range", (long long)t, k.device);
    if (!k.PL || !k.PG || !k.PR || !k.WL || !k.WG || !k.WR)
      return fail(RGF_E_ARG, "task %lld: PL/PG/PR and WL/WG/WR are required", (long long)t);
  }
  RGF_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = stream_ ? (cudaStream_t)stream_ : c->stream;
  Stage sg;
  sg.zero_copy = c->opts.zero_copy != 0;
  for (int32_t d = 0; d < n_devices; d++) {
    const size_t bytes = (size_t)devices[d].nm * devices[d].nm * devices[d].nx * sizeof(rgf_c16);
    sg.add(devices[d].Vii, bytes, true, false);
    sg.add(devices[d].V1i, bytes, true, false);
  }
  for (int64_t t = 0; t < n_tasks; t++) {
    const rgf_w_task& k = tasks[t];
    const rgf_w_device& v = devices[k.device];
    const size_t cb = (size_t)v.nm * v.nm * v.nx * sizeof(rgf_c16);
    sg.add(k.PL, cb, true, false);
    sg.add(k.PG, cb, true, false);
    sg.add(k.PR, cb, true, false);
    sg.add(k.WL, cb, false, true);   // accumulated in place while W^< forms: staged
    sg.add(k.WG, cb, false, true);
    sg.add(k.WR, cb, false, true, true);
    sg.add(k.WRi1, cb, true, true, true);  // block nx is left untouched
  }
  sg.layout();
  int rc = c->stage.reserve(std::max<size_t>(sg.total, 256));
  if (rc) return rc;
  char* sbase = (char*)c->stage.p;
  if ((rc = stage_in(c, sg, sbase, st))) return rc;
  std::vector<DDev> ddev(n_devices);
  for (int32_t d = 0; d < n_devices; d++) {
    std::memset(&ddev[d], 0, sizeof(DDev));
    ddev[d].nm = devices[d].nm;
    ddev[d].nx = devices[d].nx;
    ddev[d].Hii = (const double2*)sg.resolve(devices[d].Vii, sbase);
    ddev[d].H1i = (const double2*)sg.resolve(devices[d].V1i, sbase);
  }
  std::vector<DWTask> dt(n_tasks);
  std::vector<int32_t> order(n_tasks);
  std::vector<double> cost(n_tasks);
  int64_t slot = 0;
  size_t smem = 0;
  uint64_t nb_mask = 0;
  for (int64_t t = 0; t < n_tasks; t++) {
    const rgf_w_task& k = tasks[t];
    const rgf_w_device& v = devices[k.device];
    DWTask& o = dt[t];
    o.dev = k.device;
    o.pad = 0;
    o.PL = (const double2*)sg.resolve(k.PL, sbase);
    o.PG = (const double2*)sg.resolve(k.PG, sbase);
    o.PR = (const double2*)sg.resolve(k.PR, sbase);
    o.WL = (double2*)sg.resolve(k.WL, sbase);
    o.WG = (double2*)sg.resolve(k.WG, sbase);
    o.WR = (double2*)sg.resolve(k.WR, sbase);
    o.WRi1 = (double2*)sg.resolve(k.WRi1, sbase);
    order[t] = (int32_t)t;
    cost[t] = (double)v.nm * v.nm * v.nm * (double)v.nx;
    slot = std::max<int64_t>(slot, slot_elems_for(v.nm, v.nx));
    smem = std::max(smem, variant_smem(c->variant[v.nm / 8], (int)v.nm));
    nb_mask |= 1ull << (v.nm / 8);
  }
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return cost[a] > cost[b]; });
  int grid = c->sm_count * launch_ctas_per_sm(c, smem, nb_mask);
  if ((int64_t)grid > n_tasks) grid = (int)n_tasks;
  if ((rc = c->work.reserve(sizeof(double2) * (size_t)slot * grid))) return rc;
  if ((rc = c->devs.reserve(sizeof(DDev) * n_devices))) return rc;
  if ((rc = c->tasks.reserve(sizeof(DWTask) * n_tasks + sizeof(int32_t) * n_tasks))) return rc;
  if ((rc = c->info.reserve(sizeof(DInfo) * n_tasks))) return rc;
  if ((rc = c->queue.reserve(sizeof(int32_t) * 64))) return rc;
  int32_t* order_d = (int32_t*)((char*)c->tasks.p + sizeof(DWTask) * n_tasks);
  RGF_CUDA(cudaMemcpyAsync(c->devs.p, ddev.data(), sizeof(DDev) * n_devices, cudaMemcpyHostToDevice, st));
  RGF_CUDA(cudaMemcpyAsync(c->tasks.p, dt.data(), sizeof(DWTask) * n_tasks, cudaMemcpyHostToDevice, st));
  RGF_CUDA(cudaMemcpyAsync(order_d, order.data(), sizeof(int32_t) * n_tasks, cudaMemcpyHostToDevice, st));
  RGF_CUDA(cudaMemsetAsync(c->info.p, 0, sizeof(DInfo) * n_tasks, st));
  RGF_CUDA(cudaMemsetAsync(c->queue.p, 0, sizeof(int32_t), st));
  KParams p;
  fill_params(c, p);
  p.devs = (const DDev*)c->devs.p;
  p.n_tasks = n_tasks;
  p.order = order_d;
  p.queue = (int32_t*)c->queue.p;
  p.work = (double2*)c->work.p;
  p.slot_elems = slot;
  p.info = (DInfo*)c->info.p;
  p.wtasks = (const DWTask*)c->tasks.p;
  RGF_CUDA(cudaEventRecord(c->ev0, st));
  cudaError_t e = launch_solver(p, grid, smem, st);
  if (e != cudaSuccess) return fail(RGF_E_CUDA, "W launch failed: %s", cudaGetErrorString(e));
  c->stats.launches++;
  RGF_CUDA(cudaEventRecord(c->ev1, st));
  if ((rc = stage_out(c, sg, sbase, st))) return rc;
  // the stream is drained before the task info comes back: a copy into
  // pageable memory that waits for a running kernel stalls other host
  // threads' launches (per-thread contexts then run one after another)
  RGF_CUDA(cudaStreamSynchronize(st));
  std::vector<DInfo> hinfo(n_tasks);
  RGF_CUDA(cudaMemcpyAsync(hinfo.data(), c->info.p, sizeof(DInfo) * n_tasks, cudaMemcpyDeviceToHost, st));
  RGF_CUDA(cudaStreamSynchronize(st));
  int worst = 0;
  double flops = 0.0, int8_ops = 0.0;
  for (int64_t t = 0; t < n_tasks; t++) {
    worst |= hinfo[t].status;
    const double nb = (double)devices[tasks[t].device].nm;
    flops += 8.0 * nb * nb * nb * (double)(hinfo[t].n_gemm + hinfo[t].n_inv);
    int8_ops += 8.0 * nb * nb * nb * (double)hinfo[t].pad;   // 4 real nb^3 products per digit pair
  }
  float kms = 0.0f;
  RGF_CUDA(cudaEventElapsedTime(&kms, c->ev0, c->ev1));
  c->stats.last_kernel_ms = kms;
  c->stats.last_flops = flops;
  c->stats.last_int8_ops = int8_ops;
  c->stats.last_tasks = n_tasks;
  if (info) std::memcpy(info, hinfo.data(), sizeof(DInfo) * n_tasks);
  if (worst & RGF_ST_BAD_TASK) return fail(RGF_E_ARG, "a task was rejected on the device");
  return worst ? RGF_E_STATUS : RGF_OK;
}

extern "C" int rgf_w_solve_energies(rgf_ctx* ctx, const rgf_w_device* device, int64_t nen,
                                    const rgf_c16* PL, const rgf_c16* PG, const rgf_c16* PR,
                                    rgf_c16* WL, rgf_c16* WG, rgf_c16* WR, rgf_c16* WRi1,
                                    rgf_task_info* info, void* stream) {
  if (!ctx || !device || nen < 0 || !PL || !PG || !PR || !WL || !WG || !WR)
    return fail(RGF_E_ARG, "invalid argument");
  const size_t per = (size_t)device->nm * device->nm * device->nx;
  std::vector<rgf_w_task> tasks(nen);
  for (int64_t e = 0; e < nen; e++) {
    rgf_w_task& t = tasks[e];
    std::memset(&t, 0, sizeof(t));
    t.PL = PL + e * per;
    t.PG = PG + e * per;
    t.PR = PR + e * per;
    t.WL = WL + e * per;
    t.WG = WG + e * per;
    t.WR = WR + e * per;
    t.WRi1 = WRi1 ? WRi1 + e * per : nullptr;
  }
  return rgf_w_solve_batch(ctx, device, 1, tasks.data(), nen, info, stream);
}

extern "C" int rgf_green_rgf_calc_w(rgf_ctx* ctx, const int64_t* NBC, const int64_t* nm, const int64_t* nx,
                                    const rgf_c16* Vii, const rgf_c16* V1i, const rgf_c16* PL,
                                    const rgf_c16* PG, const rgf_c16* PR, rgf_c16* WL, rgf_c16* WG,
                                    rgf_c16* WR, const rgf_c16* PL1i, const rgf_c16* PG1i,
                                    const rgf_c16* PR1i, rgf_c16* WLi1, rgf_c16* WGi1, rgf_c16* WRi1) {
  (void)WLi1;  // not written by the reference either
  (void)WGi1;
  if (!NBC || !nm || !nx) return fail(RGF_E_ARG, "NULL scalar argument");
  if (*NBC != 0)
    return fail(RGF_E_UNSUPPORTED, "NBC=%lld: only the NBC = 0 form (every call site) is built", (long long)*NBC);
  if (PL1i || PG1i || PR1i)
    return fail(RGF_E_UNSUPPORTED, "off-diagonal polarization blocks are not supported (no call site passes them)");
  int rc = RGF_OK;
  if (!ctx) {
    ctx = default_ctx(8.61734e-05, &rc);
    if (!ctx) return rc;
  }
  rgf_w_device d;
  d.nm = *nm;
  d.nx = *nx;
  d.Vii = Vii;
  d.V1i = V1i;
  rgf_w_task t;
  std::memset(&t, 0, sizeof(t));
  t.PL = PL;
  t.PG = PG;
  t.PR = PR;
  t.WL = WL;
  t.WG = WG;
  t.WR = WR;
  t.WRi1 = WRi1;
  rc = rgf_w_solve_batch(ctx, &d, 1, &t, 1, nullptr, nullptr);
  return rc == RGF_E_STATUS ? RGF_OK : rc;
}
