// Workspace arena, scans, stable LSD radix sort and searches.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include <algorithm>
#include <map>
#include <mutex>

#include "fgt_prims.cuh"

namespace fgt {

namespace {
struct TuneCache {
  std::mutex mu;
  bool loaded = false;
  std::map<std::string, int> kv;
  std::string path;
};
TuneCache& tune_cache() {
  static TuneCache c;
  return c;
}
std::string tune_path() {
  const char* e = getenv("FGT_TUNE_CACHE");
  if (e && *e) return e;
  const char* h = getenv("HOME");
  std::string dir = std::string(h && *h ? h : "/tmp") + "/.cache";
  mkdir(dir.c_str(), 0755);
  dir += "/fgt_b200";
  mkdir(dir.c_str(), 0755);
  return dir + "/tune.txt";
}
void tune_load_locked(TuneCache& c) {
  const std::string p = tune_path();
  if (c.loaded && p == c.path) return;
  c.kv.clear();
  c.path = p;
  c.loaded = true;
  FILE* f = fopen(p.c_str(), "r");
  if (!f) return;
  char line[512];
  while (fgets(line, sizeof(line), f)) {
    char* sp = strrchr(line, ' ');
    if (!sp) continue;
    *sp = 0;
    c.kv[line] = atoi(sp + 1);
  }
  fclose(f);
}
}  // namespace

bool tune_lookup(const std::string& key, int& value) {
  TuneCache& c = tune_cache();
  std::lock_guard<std::mutex> lk(c.mu);
  tune_load_locked(c);
  auto it = c.kv.find(key);
  if (it == c.kv.end()) return false;
  value = it->second;
  return true;
}

void tune_store(const std::string& key, int value) {
  TuneCache& c = tune_cache();
  std::lock_guard<std::mutex> lk(c.mu);
  tune_load_locked(c);
  c.kv[key] = value;
  FILE* f = fopen(c.path.c_str(), "a");
  if (!f) return;  // an unwritable cache only loses the entry
  fprintf(f, "%s %d\n", key.c_str(), value);
  fclose(f);
}

namespace {
std::vector<CheckReader>& check_readers() {
  static std::vector<CheckReader> r;
  return r;
}
}  // namespace
void register_check_reader(CheckReader r) { check_readers().push_back(r); }
unsigned check_sites(cudaStream_t s) {
  unsigned first = 0;
  for (CheckReader r : check_readers()) {
    const unsigned v = r(s);
    if (v && !first) first = v;
  }
  return first;
}

void* Arena::alloc(size_t bytes) {
  bytes = (bytes + 255) & ~size_t(255);
  for (auto& c : chunks)
    if (c.off + bytes <= c.cap) {
      void* p = c.p + c.off;
      c.off += bytes;
      used += bytes;
      high = std::max(high, used);
      return p;
    }
  size_t cap = std::max(bytes, (size_t)256 << 20);
  if (!chunks.empty()) cap = std::max(cap, chunks.back().cap);
  char* p = nullptr;
  if (cudaMalloc((void**)&p, cap) != cudaSuccess) {
    (void)cudaGetLastError();
    fgt_set_error_message("device workspace allocation failed", __FILE__, __LINE__);
    throw Error{FGT_ERR_NOMEM, "device workspace allocation failed"};
  }
  chunks.push_back({p, cap, bytes});
  used += bytes;
  high = std::max(high, used);
  return p;
}

void Arena::reset(cudaStream_t s) {
  if (chunks.size() > 1) {
    // consolidate into one chunk of the high-water size for the next call
    cudaStreamSynchronize(s);
    for (auto& c : chunks) cudaFree(c.p);
    chunks.clear();
    size_t cap = ((size_t)(high * 1.05) + ((size_t)1 << 20)) & ~(((size_t)1 << 20) - 1);
    char* p = nullptr;
    if (cudaMalloc((void**)&p, cap) == cudaSuccess) chunks.push_back({p, cap, 0});
    else (void)cudaGetLastError();
  }
  for (auto& c : chunks) c.off = 0;
  used = 0;
}

std::vector<size_t> Arena::mark() const {
  std::vector<size_t> m;
  for (const auto& c : chunks) m.push_back(c.off);
  m.push_back(used);
  return m;
}

void Arena::rewind(const std::vector<size_t>& m) {
  for (size_t i = 0; i < chunks.size(); i++) chunks[i].off = i + 1 < m.size() ? m[i] : 0;
  used = m.empty() ? 0 : m.back();
}

void Arena::release_all() {
  for (auto& c : chunks) cudaFree(c.p);
  chunks.clear();
  used = high = 0;
}

static thread_local Arena* t_arena_override = nullptr;

ArenaOverride::ArenaOverride(Arena* a) : prev(t_arena_override) { t_arena_override = a; }
ArenaOverride::~ArenaOverride() { t_arena_override = prev; }

Arena* thread_arena() {
  if (t_arena_override) return t_arena_override;
  static thread_local std::map<int, Arena*> arenas;
  int dev = 0;
  cudaGetDevice(&dev);
  auto it = arenas.find(dev);
  if (it != arenas.end()) return it->second;
  Arena* a = new Arena();
  arenas[dev] = a;
  return a;
}

namespace {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ int warp_incl_scan(int v) {
  int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += y;
  }
  return v;
}

// Exclusive block scan of one value per thread; returns block total.
__device__ __forceinline__ int block_excl_scan(int v, int* total) {
  __shared__ int ws[32];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int inc = warp_incl_scan(v);
  if (lane == 31) ws[w] = inc;
  __syncthreads();
  if (w == 0) {
    int x = lane < nw ? ws[lane] : 0;
    int xi = warp_incl_scan(x);
    if (lane < nw) ws[lane] = xi - x;
    if (lane == nw - 1) ws[31] = xi;
  }
  __syncthreads();
  int r = inc - v + ws[w];
  *total = ws[31];
  __syncthreads();
  return r;
}

__global__ void k_scan_reduce(const int* __restrict__ in, int n, int* __restrict__ part) {
  int base = blockIdx.x * SCAN_TILE, s = 0;
  for (int j = 0; j < SCAN_ITEMS; j++) {
    int i = base + threadIdx.x * SCAN_ITEMS + j;
    if (i < n) s += in[i];
  }
  int tot;
  block_excl_scan(s, &tot);
  if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

__global__ void k_scan_apply(const int* in, int* out, int n, const int* __restrict__ part,
                             int* total, int nblocks) {
  int base = blockIdx.x * SCAN_TILE;
  int v[SCAN_ITEMS], s = 0;
  for (int j = 0; j < SCAN_ITEMS; j++) {
    int i = base + threadIdx.x * SCAN_ITEMS + j;
    v[j] = (i < n) ? in[i] : 0;
    s += v[j];
  }
  int tot;
  int ex = block_excl_scan(s, &tot) + (part ? part[blockIdx.x] : 0);
  for (int j = 0; j < SCAN_ITEMS; j++) {
    int i = base + threadIdx.x * SCAN_ITEMS + j;
    if (i < n) out[i] = ex;
    ex += v[j];
  }
  if (total && blockIdx.x == nblocks - 1 && threadIdx.x == SCAN_THREADS - 1) *total = ex;
}

// ---------------------------------------------------------------- radix sort
constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_WARPS = RS_THREADS / 32;

template <typename K>
__global__ void __launch_bounds__(RS_THREADS) k_radix_hist(const K* __restrict__ keys, int n,
                                                           int shift, int* __restrict__ hist,
                                                           int nblocks) {
  __shared__ int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  int base = blockIdx.x * RS_TILE;
  for (int r = 0; r < RS_ITEMS; r++) {
    int i = base + r * RS_THREADS + threadIdx.x;
    if (i < n) atomicAdd(&h[(int)((keys[i] >> shift) & K(255))], 1);
  }
  __syncthreads();
  hist[threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

template <typename K>
__global__ void __launch_bounds__(RS_THREADS)
    k_radix_scatter(const K* __restrict__ kin, const uint32_t* __restrict__ vin,
                    K* __restrict__ kout, uint32_t* __restrict__ vout, int n, int shift,
                    const int* __restrict__ offs, int nblocks) {
  __shared__ int base[256];
  __shared__ int wc[RS_WARPS][256];
  int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  base[tid] = offs[tid * nblocks + blockIdx.x];
  unsigned lt = (1u << lane) - 1u;
  int tbase = blockIdx.x * RS_TILE;
  __syncthreads();
  for (int r = 0; r < RS_ITEMS; r++) {
    int i = tbase + r * RS_THREADS + tid;
    bool valid = i < n;
    K k = valid ? kin[i] : K(0);
    uint32_t v = (valid && vin) ? vin[i] : 0u;
    int d = valid ? (int)((k >> shift) & K(255)) : 256;
    unsigned peers = __match_any_sync(0xffffffffu, d);
    int rank = __popc(peers & lt);
    bool leader = (__ffs(peers) - 1) == lane;
#pragma unroll
    for (int w = 0; w < RS_WARPS; w++) wc[w][tid] = 0;
    __syncthreads();
    if (valid && leader) wc[warp][d] = __popc(peers);
    __syncthreads();
    {
      int run = base[tid];
#pragma unroll
      for (int w = 0; w < RS_WARPS; w++) {
        int c = wc[w][tid];
        wc[w][tid] = run;
        run += c;
      }
      base[tid] = run;
    }
    __syncthreads();
    if (valid) {
      int pos = wc[warp][d] + rank;
      kout[pos] = k;
      if (vout) vout[pos] = v;
    }
    __syncthreads();
  }
}

// k_radix_scatter for 32-bit keys with the tile reordered in shared memory
// first: the tile's items are ranked stably by digit (the same rank as
// k_radix_scatter's), placed in digit order in shared memory, and then
// written out by consecutive threads, so each digit's run of the tile goes
// to consecutive global positions (whole sectors) instead of one scattered
// 4-byte store per item.  Same output as k_radix_scatter.
__global__ void __launch_bounds__(RS_THREADS)
    k_radix_scatter_tile(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                         uint32_t* __restrict__ kout, uint32_t* __restrict__ vout, int n,
                         int shift, const int* __restrict__ offs, int nblocks) {
  __shared__ uint32_t sk[RS_TILE];
  __shared__ uint32_t sv[RS_TILE];
  __shared__ int run[256];    // running count per digit, then the tile's digit start
  __shared__ int gbase[256];  // global start of the tile's run of each digit
  __shared__ int wc[RS_WARPS][256];
  __shared__ int wsum[RS_WARPS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int tbase = blockIdx.x * RS_TILE;
  const int tn = min(RS_TILE, n - tbase);
  run[tid] = 0;
  gbase[tid] = offs[tid * nblocks + blockIdx.x];
  uint32_t key[RS_ITEMS], val[RS_ITEMS];
  int rk[RS_ITEMS];
#pragma unroll
  for (int r = 0; r < RS_ITEMS; r++) {
    const int i = tbase + r * RS_THREADS + tid;
    const bool valid = i < n;
    key[r] = valid ? kin[i] : 0u;
    val[r] = (valid && vin) ? vin[i] : 0u;
  }
  __syncthreads();
  // stable rank of every item among the tile's items of its digit
#pragma unroll
  for (int r = 0; r < RS_ITEMS; r++) {
    const bool valid = tbase + r * RS_THREADS + tid < n;
    const int d = valid ? (int)((key[r] >> shift) & 255u) : 256;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const bool leader = (__ffs(peers) - 1) == lane;
#pragma unroll
    for (int w = 0; w < RS_WARPS; w++) wc[w][tid] = 0;
    __syncthreads();
    if (valid && leader) wc[warp][d] = __popc(peers);
    __syncthreads();
    {
      int c0 = run[tid];
#pragma unroll
      for (int w = 0; w < RS_WARPS; w++) {
        const int c = wc[w][tid];
        wc[w][tid] = c0;
        c0 += c;
      }
      run[tid] = c0;
    }
    __syncthreads();
    rk[r] = valid ? wc[warp][d] + __popc(peers & lt) : 0;
    __syncthreads();
  }
  // exclusive scan of the tile's digit counts: digit starts in the tile
  {
    const int c = run[tid];
    int inc = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += u;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    int wo = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; w++) wo += w < warp ? wsum[w] : 0;
    run[tid] = wo + inc - c;
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RS_ITEMS; r++) {
    if (tbase + r * RS_THREADS + tid < n) {
      const int d = (int)((key[r] >> shift) & 255u);
      const int slot = run[d] + rk[r];
      sk[slot] = key[r];
      sv[slot] = val[r];
    }
  }
  __syncthreads();
  for (int j = tid; j < tn; j += RS_THREADS) {
    const uint32_t k = sk[j];
    const int d = (int)((k >> shift) & 255u);
    const int pos = gbase[d] + (j - run[d]);
    kout[pos] = k;
    if (vout) vout[pos] = sv[j];
  }
}

__global__ void k_lower_bound(const uint64_t* __restrict__ a, int n, const uint64_t* __restrict__ q,
                              int m, int* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    out[i] = dev_lower_bound(a, n, q[i]);
}

__global__ void k_unique_flags(const uint64_t* __restrict__ a, int n, int* __restrict__ f) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    f[i] = (i == 0 || a[i] != a[i - 1]) ? 1 : 0;
}
__global__ void k_unique_scatter(const uint64_t* __restrict__ a, int n, const int* __restrict__ pos,
                                 uint64_t* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (i == 0 || a[i] != a[i - 1]) out[pos[i]] = a[i];
}

}  // namespace

void exclusive_scan_i32(const int* in, int* out, int n, int* total, cudaStream_t s) {
  if (n <= 0) {
    if (total) FGT_CUDA(cudaMemsetAsync(total, 0, sizeof(int), s));
    return;
  }
  int nb = ceil_div(n, SCAN_TILE);
  if (nb == 1) {
    k_scan_apply<<<1, SCAN_THREADS, 0, s>>>(in, out, n, nullptr, total, 1);
    FGT_LAUNCH_CHECK();
    return;
  }
  DBuf<int> part(nb, s);
  k_scan_reduce<<<nb, SCAN_THREADS, 0, s>>>(in, n, part);
  FGT_LAUNCH_CHECK();
  exclusive_scan_i32(part, part, nb, nullptr, s);
  k_scan_apply<<<nb, SCAN_THREADS, 0, s>>>(in, out, n, part, total, nb);
  FGT_LAUNCH_CHECK();
}

namespace {
template <typename K>
void radix_sort_t(K* keys, uint32_t* vals, K* ktmp, uint32_t* vtmp, int n, int bits,
                  cudaStream_t s) {
  if (n <= 1 || bits <= 0) return;
  int nb = ceil_div(n, RS_TILE);
  DBuf<int> hist((size_t)256 * nb, s);
  K *ka = keys, *kb = ktmp;
  uint32_t *va = vals, *vb = vtmp;
  int passes = 0;
  for (int shift = 0; shift < bits; shift += 8) {
    k_radix_hist<K><<<nb, RS_THREADS, 0, s>>>(ka, n, shift, hist, nb);
    FGT_LAUNCH_CHECK();
    exclusive_scan_i32(hist, hist, 256 * nb, nullptr, s);
    if constexpr (sizeof(K) == 4)
      k_radix_scatter_tile<<<nb, RS_THREADS, 0, s>>>(ka, va, kb, vb, n, shift, hist, nb);
    else
      k_radix_scatter<K><<<nb, RS_THREADS, 0, s>>>(ka, va, kb, vb, n, shift, hist, nb);
    FGT_LAUNCH_CHECK();
    std::swap(ka, kb);
    std::swap(va, vb);
    passes++;
  }
  if (passes & 1) {
    FGT_CUDA(cudaMemcpyAsync(keys, ka, sizeof(K) * n, cudaMemcpyDeviceToDevice, s));
    if (vals) FGT_CUDA(cudaMemcpyAsync(vals, va, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
  }
}
}  // namespace

void radix_sort(uint64_t* keys, uint32_t* vals, uint64_t* ktmp, uint32_t* vtmp, int n, int bits,
                cudaStream_t s) {
  radix_sort_t<uint64_t>(keys, vals, ktmp, vtmp, n, bits, s);
}
void radix_sort_u32(uint32_t* keys, uint32_t* vals, uint32_t* ktmp, uint32_t* vtmp, int n,
                    int bits, cudaStream_t s) {
  radix_sort_t<uint32_t>(keys, vals, ktmp, vtmp, n, bits, s);
}

void lower_bound_u64(const uint64_t* sorted, int n, const uint64_t* q, int m, int* out,
                     cudaStream_t s) {
  if (m <= 0) return;
  k_lower_bound<<<grid_for(m, 256), 256, 0, s>>>(sorted, n, q, m, out);
  FGT_LAUNCH_CHECK();
}

int fetch_int(const int* d, cudaStream_t s) {
  int h = 0;
  FGT_CUDA(cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, s));
  FGT_CUDA(cudaStreamSynchronize(s));
  return h;
}

void fetch_ints(const int* const* d, int n, int* h, cudaStream_t s) {
  // a per-thread pinned landing area: the copies queue behind each other
  // and one synchronisation covers them all
  struct Pinned {
    int* p = nullptr;
    ~Pinned() {
      if (p) cudaFreeHost(p);
    }
  };
  static thread_local Pinned buf;
  constexpr int kMax = 16;
  FGT_REQUIRE(n <= kMax, FGT_ERR_UNSUPPORTED, "too many values in one read-back");
  if (!buf.p) FGT_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&buf.p), sizeof(int) * kMax, 0));
  for (int i = 0; i < n; i++)
    FGT_CUDA(cudaMemcpyAsync(buf.p + i, d[i], sizeof(int), cudaMemcpyDeviceToHost, s));
  FGT_CUDA(cudaStreamSynchronize(s));
  for (int i = 0; i < n; i++) h[i] = buf.p[i];
}

int unique_sorted_u64(const uint64_t* in, int n, uint64_t* out, cudaStream_t s) {
  if (n <= 0) return 0;
  DBuf<int> f(n, s), tot(1, s);
  k_unique_flags<<<grid_for(n, 256), 256, 0, s>>>(in, n, f);
  FGT_LAUNCH_CHECK();
  exclusive_scan_i32(f, f, n, tot, s);
  k_unique_scatter<<<grid_for(n, 256), 256, 0, s>>>(in, n, f, out);
  FGT_LAUNCH_CHECK();
  return fetch_int(tot, s);
}

}  // namespace fgt
