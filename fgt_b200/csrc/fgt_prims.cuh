// Device primitives: stream-ordered buffers, scans, a stable LSD radix sort,
// sorted-array searches.  All hand-written; no CUB/Thrust.
#pragma once
#include <string>
#include <vector>

#include "fgt_common.cuh"

namespace fgt {

// Per-call device workspace: bump allocation from cached chunks that persist
// across calls (reset at the end of every call; grown with cudaMalloc only
// when a call needs more than any earlier one, then consolidated into one
// chunk of the high-water size).  Removes allocation from the steady state.
struct Arena {
  struct Chunk {
    char* p;
    size_t cap, off;
  };
  std::vector<Chunk> chunks;
  size_t used = 0, high = 0;
  void* alloc(size_t bytes);
  void reset(cudaStream_t s);  // call end: all allocations are dead
  void release_all();
  // Allocation state, and a return to it: buffers allocated after the mark
  // are dead (their device work is stream-ordered before any later use).
  std::vector<size_t> mark() const;
  void rewind(const std::vector<size_t>& m);
};
// Arena of the calling host thread on the current device (created lazily),
// or the arena installed by an ArenaOverride on this thread.
Arena* thread_arena();
// RAII: while alive, this thread's device buffers come from `a` (a plan's
// own arena, which outlives the call).
struct ArenaOverride {
  Arena* prev;
  explicit ArenaOverride(Arena* a);
  ~ArenaOverride();
};
// RAII scope of one library call: resets the arena on exit.
struct ArenaScope {
  Arena* a;
  cudaStream_t s;
  ArenaScope(cudaStream_t st) : a(thread_arena()), s(st) {}
  ~ArenaScope() { a->reset(s); }
};

// Device buffer from the thread's arena (no per-call cudaMalloc).
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = 0;
  DBuf() = default;
  DBuf(size_t count, cudaStream_t st) { alloc(count, st); }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p; n = o.n; s = o.s;
      o.p = nullptr; o.n = 0;
    }
    return *this;
  }
  void alloc(size_t count, cudaStream_t st) {
    release();
    s = st;
    n = count;
    size_t bytes = (count ? count : 1) * sizeof(T);
    p = (T*)thread_arena()->alloc(bytes);
  }
  void zero() {
    if (p) FGT_CUDA(cudaMemsetAsync(p, 0, (n ? n : 1) * sizeof(T), s));
  }
  void release() {  // memory returns to the arena at the end of the call
    p = nullptr;
    n = 0;
  }
  ~DBuf() { release(); }
  T* get() const { return p; }
  operator T*() const { return p; }
};

// On-disk cache of tuned parameters (autotuner): one "key value" line per
// entry in the file named by FGT_TUNE_CACHE, else
// $HOME/.cache/fgt_b200/tune.txt; read once per process, appended to on
// every new entry.  Thread-safe.
bool tune_lookup(const std::string& key, int& value);
void tune_store(const std::string& key, int value);

// Exclusive prefix sum of n int32 values (in == out allowed).  If total is not
// null, the grand total is written to *total (device pointer).
void exclusive_scan_i32(const int* in, int* out, int n, int* total, cudaStream_t s);

// Stable LSD radix sort on the low `bits` bits of 64-bit keys, carrying
// optional 32-bit values.  Results end in keys/vals (tmp buffers of n).
void radix_sort(uint64_t* keys, uint32_t* vals, uint64_t* ktmp, uint32_t* vtmp, int n,
                int bits, cudaStream_t s);

// The same on 32-bit keys (bits <= 32).
void radix_sort_u32(uint32_t* keys, uint32_t* vals, uint32_t* ktmp, uint32_t* vtmp, int n,
                    int bits, cudaStream_t s);

// out[i] = lower_bound(sorted, n, q[i]) for m queries.
void lower_bound_u64(const uint64_t* sorted, int n, const uint64_t* q, int m, int* out,
                     cudaStream_t s);

// Compact the unique values of a sorted uint64 array; returns the count
// (synchronises the stream).
int unique_sorted_u64(const uint64_t* in, int n, uint64_t* out, cudaStream_t s);

// Copy a device int to the host (synchronises the stream).
int fetch_int(const int* d, cudaStream_t s);
// Reads n (<= 16) device ints with one stream synchronisation.
void fetch_ints(const int* const* d, int n, int* h, cudaStream_t s);

__device__ __forceinline__ int dev_lower_bound(const uint64_t* a, int n, uint64_t v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo;
}
// index of v in sorted a, or -1
__device__ __forceinline__ int dev_find(const uint64_t* a, int n, uint64_t v) {
  int i = dev_lower_bound(a, n, v);
  return (i < n && a[i] == v) ? i : -1;
}

}  // namespace fgt
