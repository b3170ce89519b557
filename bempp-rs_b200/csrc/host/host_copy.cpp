// Dense assembly into host memory with the device-to-host transfer overlapped.
//
// bempp-rs BoundaryAssembler::assemble_into_memory (src/boundary_assemblers.rs:176-214)
// fills a caller-owned column-major host array.  Copying a finished device matrix into
// pageable host memory with one cudaMemcpy runs at the driver's pageable rate and starts
// only after the last kernel.  Here the regular part is assembled in chunks of trial
// tiles (assemble_device); as soon as a chunk's kernels finish, the columns it completed
// are copied by DMA into a pinned staging slot on a copy stream, and host threads move
// the previous slot into the caller's array.  Compute, DMA and host copy overlap; only
// the last group's copy is exposed.
//
// Staging: a process-wide ring of two pinned slots per device (kSlotBytes each) and one
// copy stream, used by one assembly at a time (mutex).  Host copies run on a small
// persistent pool of worker threads, each taking an equal byte share of a group.
// A destination that is itself page-locked skips the staging: the columns go there by
// DMA directly.
#include <sys/mman.h>
#include <unistd.h>
#if defined(__x86_64__)
#include <emmintrin.h>
#endif

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <iterator>
#include <thread>

#include "core.h"

namespace bempp_b200 {

namespace {

constexpr size_t kSlotBytes = size_t(64) << 20;
constexpr size_t kChunkTargetBytes = size_t(48) << 20;  // device bytes per chunk (about)
constexpr int kMaxChunks = 16;
constexpr int64_t kMergeGap = 2;  // columns between two runs still copied as one DMA
constexpr int64_t kMinRun = 16;   // shortest run of finished columns a tx >= sy chunk copies

// Persistent pool running one parallel job at a time.
class CopyPool {
 public:
  static CopyPool& get() {
    static CopyPool pool;
    return pool;
  }
  int size() const { return static_cast<int>(workers_.size()) + 1; }
  // Runs fn(i) for i in [0, size()) on the workers and the calling thread.
  void run(const std::function<void(int)>& fn) {
    {
      std::lock_guard<std::mutex> lock(mu_);
      job_ = &fn;
      pending_ = static_cast<int>(workers_.size());
      ++generation_;
    }
    cv_.notify_all();
    fn(0);
    std::unique_lock<std::mutex> lock(mu_);
    done_cv_.wait(lock, [&] { return pending_ == 0; });
    job_ = nullptr;
  }

 private:
  CopyPool() {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int n = static_cast<int>(std::min(32u, std::max(1u, hw)));
    for (int i = 1; i < n; ++i) workers_.emplace_back([this, i] { loop(i); });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lock(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }
  void loop(int id) {
    uint64_t seen = 0;
    for (;;) {
      const std::function<void(int)>* job;
      {
        std::unique_lock<std::mutex> lock(mu_);
        cv_.wait(lock, [&] { return stop_ || generation_ != seen; });
        if (stop_) return;
        seen = generation_;
        job = job_;
      }
      (*job)(id);
      {
        std::lock_guard<std::mutex> lock(mu_);
        if (--pending_ == 0) done_cv_.notify_one();
      }
    }
  }
  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int)>* job_ = nullptr;
  int pending_ = 0;
  uint64_t generation_ = 0;
  bool stop_ = false;
};

struct Staging {
  void* slot[2] = {nullptr, nullptr};
  cudaStream_t copy = nullptr;
  cudaEvent_t copied[2] = {nullptr, nullptr};
  std::vector<cudaEvent_t> chunk_ready;
  std::mutex mu;
};

std::mutex g_staging_mu;
std::map<int, std::unique_ptr<Staging>> g_staging;

Staging& staging(int device) {
  std::lock_guard<std::mutex> lock(g_staging_mu);
  auto& s = g_staging[device];
  if (!s) {
    auto st = std::make_unique<Staging>();
    for (int i = 0; i < 2; ++i) {
      BEMPP_CUDA(cudaHostAlloc(&st->slot[i], kSlotBytes, cudaHostAllocDefault));
      BEMPP_CUDA(cudaEventCreateWithFlags(&st->copied[i], cudaEventDisableTiming));
    }
    BEMPP_CUDA(cudaStreamCreateWithFlags(&st->copy, cudaStreamNonBlocking));
    s = std::move(st);
  }
  return *s;
}

// One DMA into a staging slot: bytes [src_off, src_off + bytes) of the device matrix,
// which land at the same offsets of the host matrix.
struct Piece {
  size_t src_off, bytes, slot_off;
};
struct Group {
  int chunk = 0;
  std::vector<Piece> pieces;
  size_t bytes = 0;
};

// The DMAs of each chunk into a page-locked destination, as (first column, columns).
// Full tile grid (every chunk the same work): the runs of columns the chunk completes,
// merged across gaps of at most kMergeGap columns (a gap column that is not final yet is
// copied again by a later DMA on the same stream, which lands after this one; a final one
// is copied twice with the same values), fewer, larger copies for ~17 % more bytes.
// Tile pairs tx >= sy only (symmetric operators on one space): the first chunks hold
// most of the work, so the copy stream has time to spare early and none late.  Only
// finished columns are copied, and a run shorter than kMinRun columns waits for a later
// chunk, where the columns beside it may have joined it (the last chunk takes the rest).
ColumnRuns copy_plan(const ColumnRuns& runs, bool triangular) {
  const int n = static_cast<int>(runs.size());
  ColumnRuns plan(n);
  if (!triangular) {
    for (int c = 0; c < n; ++c) {
      const auto& rc = runs[c];
      for (size_t r = 0; r < rc.size();) {
        const int64_t first = rc[r].first;
        int64_t end = rc[r].first + rc[r].second;
        size_t q = r + 1;
        while (q < rc.size() && rc[q].first >= end && rc[q].first - end <= kMergeGap) {
          end = rc[q].first + rc[q].second;
          ++q;
        }
        plan[c].push_back({first, end - first});
        r = q;
      }
    }
    return plan;
  }
  std::vector<std::pair<int64_t, int64_t>> pending, all;
  for (int c = 0; c < n; ++c) {
    // the chunks' runs are disjoint: merge the deferred ones with this chunk's, joining
    // runs that touch
    all.clear();
    std::merge(pending.begin(), pending.end(), runs[c].begin(), runs[c].end(),
               std::back_inserter(all));
    pending.clear();
    for (size_t r = 0; r < all.size();) {
      const int64_t first = all[r].first;
      int64_t end = first + all[r].second;
      size_t q = r + 1;
      while (q < all.size() && all[q].first == end) end += all[q++].second;
      if (end - first >= kMinRun || c + 1 == n)
        plan[c].push_back({first, end - first});
      else
        pending.push_back({first, end - first});
      r = q;
    }
  }
  return plan;
}

std::vector<Group> plan_groups(const ColumnRuns& runs, size_t col_bytes) {
  std::vector<Group> groups;
  for (int c = 0; c < static_cast<int>(runs.size()); ++c) {
    Group g;
    g.chunk = c;
    for (const auto& run : runs[c]) {
      size_t off = static_cast<size_t>(run.first) * col_bytes;
      size_t left = static_cast<size_t>(run.second) * col_bytes;
      while (left > 0) {
        if (g.bytes == kSlotBytes) {
          groups.push_back(std::move(g));
          g = Group();
          g.chunk = c;
        }
        const size_t n = std::min(left, kSlotBytes - g.bytes);
        g.pieces.push_back({off, n, g.bytes});
        g.bytes += n;
        off += n;
        left -= n;
      }
    }
    if (g.bytes > 0) groups.push_back(std::move(g));
  }
  return groups;
}

// memcpy with non-temporal stores: the destination (a large, usually fresh array that
// the caller reads much later) is written without first reading its cache lines, one
// memory pass fewer than a cached copy.  The caller issues the store fence.
void stream_copy(char* dst, const char* src, size_t n) {
#if defined(__x86_64__)
  const size_t head = std::min(n, (16 - reinterpret_cast<uintptr_t>(dst) % 16) % 16);
  std::memcpy(dst, src, head);
  dst += head;
  src += head;
  n -= head;
  const size_t blocks = n / 64;
  for (size_t i = 0; i < blocks; ++i, dst += 64, src += 64) {
    const __m128i a = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src));
    const __m128i b = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + 16));
    const __m128i c = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + 32));
    const __m128i d = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + 48));
    _mm_stream_si128(reinterpret_cast<__m128i*>(dst), a);
    _mm_stream_si128(reinterpret_cast<__m128i*>(dst + 16), b);
    _mm_stream_si128(reinterpret_cast<__m128i*>(dst + 32), c);
    _mm_stream_si128(reinterpret_cast<__m128i*>(dst + 48), d);
  }
  std::memcpy(dst, src, n - 64 * blocks);
#else
  std::memcpy(dst, src, n);
#endif
}

#ifndef MADV_POPULATE_WRITE
#define MADV_POPULATE_WRITE 23  // Linux 5.14+
#endif

// Page faults of one group's destination ranges, taken ahead of the copy while the host
// would otherwise wait for the GPU: madvise(MADV_POPULATE_WRITE) on the pages covering
// each range (pages already present are left as they are; missing ones arrive zeroed),
// or, where the kernel lacks it, a one-byte write at the first address of each page
// inside the range.  Only ranges of groups not yet copied are given; the copy overwrites
// them.
void prefault(const Group& g, void* dst) {
  CopyPool& pool = CopyPool::get();
  const uintptr_t page = static_cast<uintptr_t>(sysconf(_SC_PAGESIZE));
  const int nt = pool.size();
  const size_t share = (g.bytes + nt - 1) / nt;
  pool.run([&](int t) {
    const size_t lo = std::min(g.bytes, share * t), hi = std::min(g.bytes, lo + share);
    for (const Piece& p : g.pieces) {
      const size_t a = std::max(lo, p.slot_off), b = std::min(hi, p.slot_off + p.bytes);
      if (a >= b) continue;
      char* first = static_cast<char*>(dst) + p.src_off + (a - p.slot_off);
      char* last = first + (b - a);
      const uintptr_t p0 = reinterpret_cast<uintptr_t>(first) & ~(page - 1);
      const uintptr_t p1 = (reinterpret_cast<uintptr_t>(last) + page - 1) & ~(page - 1);
      if (madvise(reinterpret_cast<void*>(p0), p1 - p0, MADV_POPULATE_WRITE) == 0) continue;
      for (char* q = first; q < last;) {
        *reinterpret_cast<volatile char*>(q) = 0;
        q = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(q) / page + 1) * page);
      }
    }
  });
}

// Parallel copy of one staged group into the host matrix.
void host_copy(const Group& g, const void* slot, void* dst) {
  CopyPool& pool = CopyPool::get();
  const int nt = pool.size();
  const size_t share = (g.bytes + nt - 1) / nt;
  pool.run([&](int t) {
    const size_t lo = std::min(g.bytes, share * t), hi = std::min(g.bytes, lo + share);
    for (const Piece& p : g.pieces) {
      const size_t a = std::max(lo, p.slot_off), b = std::min(hi, p.slot_off + p.bytes);
      if (a >= b) continue;
      stream_copy(static_cast<char*>(dst) + p.src_off + (a - p.slot_off),
                  static_cast<const char*>(slot) + a, b - a);
    }
#if defined(__x86_64__)
    _mm_sfence();  // this thread's streaming stores are visible before the job ends
#endif
  });
}

void check_stage_timeouts() {
  unsigned n = 0;
  BEMPP_CUDA(take_stage_timeouts(&n));
  if (n)
    throw Error(kIncomplete, std::to_string(n) +
                                 " tile blocks timed out staging their input; their entries "
                                 "were not written");
}

// True when both ends of [p, p + bytes) are page-locked host memory known to CUDA
// (cudaHostAlloc / cudaHostRegister), which the copy engines can write directly.
bool page_locked(const void* p, size_t bytes) {
  const char* ends[2] = {static_cast<const char*>(p), static_cast<const char*>(p) + bytes - 1};
  for (const char* q : ends) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, q) != cudaSuccess) {
      cudaGetLastError();  // pageable memory on older drivers: not an error here
      return false;
    }
    if (at.type != cudaMemoryTypeHost) return false;
  }
  return true;
}

}  // namespace

void assemble_host(BoundaryAssemblerT& a, SpaceT& trial, SpaceT& test, void* data) {
  const size_t nt = static_cast<size_t>(test.ndofs), ns = static_cast<size_t>(trial.ndofs);
  const size_t col_bytes = nt * dtype_size(a.dtype);
  const size_t bytes = col_bytes * ns;
  int device = 0;
  BEMPP_CUDA(cudaGetDevice(&device));
  a.work.alloc(bytes);
  if (!a.stream) BEMPP_CUDA(cudaStreamCreateWithFlags(&a.stream, cudaStreamNonBlocking));

  // compute chunking: ~kChunkTargetBytes of output per chunk
  const bool single = a.dtype == 0 || a.dtype == 2;
  const bool dp0 = test.nbasis == 1 && trial.nbasis == 1 && a.op != kHS;
  int want = static_cast<int>(std::min<size_t>(kMaxChunks, (bytes + kChunkTargetBytes - 1) /
                                                               kChunkTargetBytes));
  if (single && !dp0) want = 1;
  const int nchunks = effective_chunks(trial, want);
  const ColumnRuns& runs = chunk_columns(trial, nchunks);

  if (page_locked(data, bytes)) {
    // A page-locked destination takes each chunk's finished columns straight from the
    // device (one DMA per run of columns on a copy stream): no staging, no host copy.
    if (!a.copy_stream) BEMPP_CUDA(cudaStreamCreateWithFlags(&a.copy_stream, cudaStreamNonBlocking));
    while (a.chunk_ev.size() < static_cast<size_t>(nchunks)) {
      cudaEvent_t e;
      BEMPP_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      a.chunk_ev.push_back(e);
    }
    for (auto& e : a.copy_timing)
      if (!e) BEMPP_CUDA(cudaEventCreate(&e));
    struct Drain {
      cudaStream_t s0, s1;
      ~Drain() {
        cudaStreamSynchronize(s0);
        cudaStreamSynchronize(s1);
      }
    } drain{a.stream, a.copy_stream};
    BEMPP_CUDA(cudaEventRecord(a.copy_timing[0], a.stream));
    assemble_device(a, trial, test, a.work.ptr, a.stream, nchunks, [&](int c) {
      BEMPP_CUDA(cudaEventRecord(a.chunk_ev[c], a.stream));
    });
    BEMPP_CUDA(cudaEventRecord(a.copy_timing[1], a.stream));
    const char* src = static_cast<const char*>(a.work.ptr);
    size_t ncopies = 0;
    // P1 columns finish in short, scattered runs (copy_plan)
    const ColumnRuns plan = copy_plan(runs, a.tx_ge_sy);
    for (int c = 0; c < nchunks; ++c) {
      BEMPP_CUDA(cudaStreamWaitEvent(a.copy_stream, a.chunk_ev[c], 0));
      for (const auto& run : plan[c]) {
        const size_t off = static_cast<size_t>(run.first) * col_bytes;
        BEMPP_CUDA(cudaMemcpyAsync(static_cast<char*>(data) + off, src + off,
                                   static_cast<size_t>(run.second) * col_bytes,
                                   cudaMemcpyDeviceToHost, a.copy_stream));
        ++ncopies;
      }
    }
    BEMPP_CUDA(cudaEventRecord(a.copy_timing[2], a.copy_stream));
    BEMPP_CUDA(cudaStreamSynchronize(a.copy_stream));
    BEMPP_CUDA(cudaStreamSynchronize(a.stream));
    check_stage_timeouts();
    float compute_ms = 0.f, dma_ms = 0.f;
    BEMPP_CUDA(cudaEventElapsedTime(&compute_ms, a.copy_timing[0], a.copy_timing[1]));
    BEMPP_CUDA(cudaEventElapsedTime(&dma_ms, a.copy_timing[0], a.copy_timing[2]));
    a.host_copy_stats = {0.0, 0.0, static_cast<double>(ncopies), static_cast<double>(nchunks),
                         0.0, 0.0, compute_ms, dma_ms};
    return;
  }
  const std::vector<Group> groups = plan_groups(runs, col_bytes);

  // Large destinations are usually fresh, untouched allocations (numpy zeros): ask for
  // transparent huge pages so that the first-touch faults of the host copy are 512x
  // fewer.  A hint only; it changes no contents.
  if (bytes >= (size_t(64) << 20)) {
    const uintptr_t page = static_cast<uintptr_t>(sysconf(_SC_PAGESIZE));
    const uintptr_t lo = (reinterpret_cast<uintptr_t>(data) + page - 1) & ~(page - 1);
    const uintptr_t hi = (reinterpret_cast<uintptr_t>(data) + bytes) & ~(page - 1);
    if (hi > lo) madvise(reinterpret_cast<void*>(lo), hi - lo, MADV_HUGEPAGE);
  }

  Staging& st = staging(device);
  std::lock_guard<std::mutex> lock(st.mu);
  while (st.chunk_ready.size() < static_cast<size_t>(nchunks)) {
    cudaEvent_t e;
    BEMPP_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    st.chunk_ready.push_back(e);
  }
  // Whatever happens below, no DMA into the staging ring outlives this call.
  struct Drain {
    Staging& st;
    cudaStream_t s;
    ~Drain() {
      cudaStreamSynchronize(s);
      cudaStreamSynchronize(st.copy);
    }
  } drain{st, a.stream};

  assemble_device(a, trial, test, a.work.ptr, a.stream, nchunks, [&](int c) {
    BEMPP_CUDA(cudaEventRecord(st.chunk_ready[c], a.stream));
  });

  const char* src = static_cast<const char*>(a.work.ptr);
  auto enqueue = [&](size_t gi) {
    const Group& g = groups[gi];
    const int s = static_cast<int>(gi & 1);
    BEMPP_CUDA(cudaStreamWaitEvent(st.copy, st.chunk_ready[g.chunk], 0));
    for (const Piece& p : g.pieces)
      BEMPP_CUDA(cudaMemcpyAsync(static_cast<char*>(st.slot[s]) + p.slot_off, src + p.src_off,
                                 p.bytes, cudaMemcpyDeviceToHost, st.copy));
    BEMPP_CUDA(cudaEventRecord(st.copied[s], st.copy));
  };
  for (size_t gi = 0; gi < std::min<size_t>(2, groups.size()); ++gi) enqueue(gi);
  using clock = std::chrono::steady_clock;
  double wait_ms = 0.0, copy_ms = 0.0, prefault_ms = 0.0;
  size_t touched = 0;  // groups [0, touched) have been prefaulted or copied
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    const int s = static_cast<int>(gi & 1);
    const auto t0 = clock::now();
    // while this group's data is still on its way, take the page faults of the next ones
    touched = std::max(touched, gi);
    while (touched < groups.size()) {
      const cudaError_t q = cudaEventQuery(st.copied[s]);
      if (q == cudaSuccess) break;
      if (q != cudaErrorNotReady) BEMPP_CUDA(q);
      const auto tp = clock::now();
      prefault(groups[touched++], data);
      prefault_ms += std::chrono::duration<double, std::milli>(clock::now() - tp).count();
    }
    BEMPP_CUDA(cudaEventSynchronize(st.copied[s]));
    const auto t1 = clock::now();
    host_copy(groups[gi], st.slot[s], data);
    copy_ms += std::chrono::duration<double, std::milli>(clock::now() - t1).count();
    wait_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
    if (gi + 2 < groups.size()) enqueue(gi + 2);
  }
  a.host_copy_stats = {wait_ms - prefault_ms, copy_ms, static_cast<double>(groups.size()),
                       static_cast<double>(nchunks), static_cast<double>(CopyPool::get().size()),
                       prefault_ms};
  BEMPP_CUDA(cudaStreamSynchronize(a.stream));
  check_stage_timeouts();
}

}  // namespace bempp_b200
