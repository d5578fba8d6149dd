// C ABI and host orchestration of the point FGT (pfgt, src/pfgt/pfgt.f:6-409
// and pfgtmain, src/pfgt/pfgt.f:415-1150).  Everything after the host->device
// copy of the inputs runs on the GPU; the host computes only the FP64 scalar
// set-up (cut-off level, root box, expansion length, PW nodes) with the
// reference's formulas.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>  // header-only NVTX v3: no library to link

#include "fgt_pw.cuh"

static thread_local int g_last_status = FGT_OK;
static thread_local std::string g_last_error;

extern "C" void fgt_set_error_message(const char* msg, const char* file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s (%s:%d)", msg ? msg : "error", file ? file : "?", line);
  g_last_error = buf;
}

namespace fgt {

namespace {

// Point gathers run UB points per thread per round (rounds a grid stride
// apart) with all their index and data loads issued before the stores: the
// random reads are latency bound, so the independent loads overlap.
constexpr int UB = 4;

template <typename T, int DIM>
__global__ void k_gather_coords(const double* __restrict__ x, int n,
                                const uint32_t* __restrict__ perm, const int* __restrict__ ref,
                                const double* __restrict__ center, int nboxes,
                                T* __restrict__ off) {
  const int st = gridDim.x * blockDim.x;
  for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += UB * st) {
    size_t o[UB];
    int b[UB];
#pragma unroll
    for (int u = 0; u < UB; u++) {
      const int i = i0 + u * st;
      o[u] = i < n ? perm[i] : 0;
      b[u] = i < n ? ref[i] : 0;
      if (!FGT_DCHECK(o[u] < (size_t)n, 101)) o[u] = 0;
      if (!FGT_DCHECK(b[u] >= 0 && b[u] < nboxes, 102)) b[u] = 0;
    }
    double v[UB][DIM], c[UB][DIM];
#pragma unroll
    for (int u = 0; u < UB; u++)
#pragma unroll
      for (int k = 0; k < DIM; k++) {
        const bool in = i0 + u * st < n;
        v[u][k] = in ? x[o[u] * DIM + k] : 0.0;
        c[u][k] = in ? center[(size_t)b[u] * DIM + k] : 0.0;
      }
#pragma unroll
    for (int u = 0; u < UB; u++) {
      const int i = i0 + u * st;
      if (i < n)
#pragma unroll
        for (int k = 0; k < DIM; k++) off[(size_t)k * n + i] = (T)(v[u][k] - c[u][k]);
    }
  }
}
template <typename T>
void launch_gather_coords(int dim, const double* x, int n, const uint32_t* perm, const int* ref,
                          const double* center, int nboxes, T* off, cudaStream_t s) {
  const int grid = grid_for(n, 256);
  if (dim == 1) k_gather_coords<T, 1><<<grid, 256, 0, s>>>(x, n, perm, ref, center, nboxes, off);
  else if (dim == 2) k_gather_coords<T, 2><<<grid, 256, 0, s>>>(x, n, perm, ref, center, nboxes, off);
  else k_gather_coords<T, 3><<<grid, 256, 0, s>>>(x, n, perm, ref, center, nboxes, off);
  FGT_LAUNCH_CHECK();
}

template <typename T>
__global__ void k_gather_vals(const double* __restrict__ v, int n, int nv,
                              const uint32_t* __restrict__ perm, T* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    size_t o = perm[i];
    if (!FGT_DCHECK(o < (size_t)n, 103)) continue;
    for (int j = 0; j < nv; j++) out[(size_t)j * n + i] = (T)v[o * nv + j];
  }
}

// inv[perm[i]] = i
__global__ void k_invert(const uint32_t* __restrict__ perm, int n, uint32_t* __restrict__ inv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (FGT_DCHECK(perm[i] < (uint32_t)n, 104)) inv[perm[i]] = (uint32_t)i;
}

// out[o] = sorted[inv[o]] for pot/grad/hess in the reference's layouts
// (dreorderi/dreorderiv, src/common/fmmcommon2d.f:29-90).  Gathering by the
// inverse permutation keeps the output writes coalesced; the random accesses
// are reads of whole sectors instead of partial-sector writes.
__global__ void k_gather_out(const double* __restrict__ srt, int n, int nd, int dim, int pgh,
                             const uint32_t* __restrict__ inv, double* __restrict__ pot,
                             double* __restrict__ grad, double* __restrict__ hess) {
  const int nh = dim * (dim + 1) / 2;
  const int st = gridDim.x * blockDim.x;
  for (int o0 = blockIdx.x * blockDim.x + threadIdx.x; o0 < n; o0 += UB * st) {
    size_t iu[UB];
#pragma unroll
    for (int u = 0; u < UB; u++) {
      iu[u] = o0 + u * st < n ? inv[o0 + u * st] : 0;
      if (!FGT_DCHECK(iu[u] < (size_t)n, 105)) iu[u] = 0;
    }
    for (int id = 0; id < nd; id++) {
      double v[UB];
#pragma unroll
      for (int u = 0; u < UB; u++) v[u] = o0 + u * st < n ? srt[(size_t)id * n + iu[u]] : 0.0;
#pragma unroll
      for (int u = 0; u < UB; u++)
        if (o0 + u * st < n) pot[(size_t)(o0 + u * st) * nd + id] = v[u];
      if (pgh >= 2)
        for (int k = 0; k < dim; k++) {
#pragma unroll
          for (int u = 0; u < UB; u++)
            v[u] = o0 + u * st < n ? srt[((size_t)(1 + k) * nd + id) * n + iu[u]] : 0.0;
#pragma unroll
          for (int u = 0; u < UB; u++)
            if (o0 + u * st < n) grad[((size_t)(o0 + u * st) * dim + k) * nd + id] = v[u];
        }
      if (pgh >= 3)
        for (int m = 0; m < nh; m++) {
#pragma unroll
          for (int u = 0; u < UB; u++)
            v[u] = o0 + u * st < n ? srt[((size_t)(1 + dim + m) * nd + id) * n + iu[u]] : 0.0;
#pragma unroll
          for (int u = 0; u < UB; u++)
            if (o0 + u * st < n) hess[((size_t)(o0 + u * st) * nh + m) * nd + id] = v[u];
        }
    }
  }
}

// Sorted outputs SoA [comp*nd + id][n] -> AoS [n][comp*nd + id]: one point's
// components become one contiguous block, so the reorder below reads whole
// sectors at random positions instead of one 8-byte value per component.
// Component order (pot, grad_k, hess_m) x density is the order of the
// reference's per-point blocks of pot(nd,n), grad(nd,dim,n), hess(nd,nh,n).
// Tiles of 64 points through shared memory: component rows are read
// coalesced, the tile's AoS block is written contiguously.
constexpr int AOS_TILE = 64;
constexpr int AOS_MAXC = 96;  // components per point staged (48 KB per block)
__global__ void k_to_aos(const double* __restrict__ srt, int n, int ncomp,
                         double* __restrict__ aos) {
  __shared__ double tile[AOS_TILE * AOS_MAXC];
  if (ncomp > AOS_MAXC) {  // many densities: point by point
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
      for (int c = 0; c < ncomp; c++) aos[(size_t)i * ncomp + c] = srt[(size_t)c * n + i];
    return;
  }
  for (int i0 = blockIdx.x * AOS_TILE; i0 < n; i0 += gridDim.x * AOS_TILE) {
    const int m = min(AOS_TILE, n - i0);
    for (int idx = threadIdx.x; idx < ncomp * AOS_TILE; idx += blockDim.x) {
      const int c = idx / AOS_TILE, p = idx - c * AOS_TILE;
      if (p < m) tile[p * ncomp + c] = srt[(size_t)c * n + i0 + p];
    }
    __syncthreads();
    for (int j = threadIdx.x; j < m * ncomp; j += blockDim.x) aos[(size_t)i0 * ncomp + j] = tile[j];
    __syncthreads();
  }
}

// out[o] = sorted[inv[o]] for pot/grad/hess in the reference's layouts
// (dreorderi/dreorderiv, src/common/fmmcommon2d.f:29-90) from the AoS sorted
// outputs: each point's npot + ngrad + nhess values are contiguous there and
// in every output array.
__global__ void k_gather_out_aos(const double* __restrict__ aos, int n, int npot, int ngrad,
                                 int nhess, const uint32_t* __restrict__ inv,
                                 double* __restrict__ pot, double* __restrict__ grad,
                                 double* __restrict__ hess) {
  const int nc = npot + ngrad + nhess;
  const int st = gridDim.x * blockDim.x;
  for (int o0 = blockIdx.x * blockDim.x + threadIdx.x; o0 < n; o0 += UB * st) {
    size_t iu[UB];
#pragma unroll
    for (int u = 0; u < UB; u++) {
      iu[u] = o0 + u * st < n ? inv[o0 + u * st] : 0;
      if (!FGT_DCHECK(iu[u] < (size_t)n, 106)) iu[u] = 0;
    }
#pragma unroll
    for (int u = 0; u < UB; u++) {
      const size_t o = (size_t)o0 + (size_t)u * st;
      if (o >= (size_t)n) break;
      const double* a = aos + iu[u] * nc;
      for (int c = 0; c < npot; c++) pot[o * npot + c] = a[c];
      for (int c = 0; c < ngrad; c++) grad[o * ngrad + c] = a[npot + c];
      for (int c = 0; c < nhess; c++) hess[o * nhess + c] = a[npot + ngrad + c];
    }
  }
}

// Reorder of one evaluation set's sorted outputs to the caller's layout.
// Up to 7 components per point the gather reads them straight from the SoA
// arrays (a few sectors per point); from 8 on (several densities, hessians)
// the outputs are first transposed to AoS so a point's components are one
// contiguous read (config-3-like calls: nd = 4, pot + grad).
void reorder_outputs(const double* srt, int n, int nd, int dim, int pgh, const uint32_t* inv,
                     double* pot, double* grad, double* hess, cudaStream_t s, int& launches) {
  const int nh = dim * (dim + 1) / 2;
  const int npot = nd, ngrad = pgh >= 2 ? nd * dim : 0, nhess = pgh >= 3 ? nd * nh : 0;
  if (npot + ngrad + nhess < 8) {
    k_gather_out<<<grid_for(n, 256), 256, 0, s>>>(srt, n, nd, dim, pgh, inv, pot, grad, hess);
    FGT_LAUNCH_CHECK();
    launches++;
    return;
  }
  DBuf<double> aos((size_t)n * (npot + ngrad + nhess), s);
  k_to_aos<<<grid_for(n, AOS_TILE * 4, 8), 256, 0, s>>>(srt, n, npot + ngrad + nhess, aos);
  FGT_LAUNCH_CHECK();
  k_gather_out_aos<<<grid_for(n, 256), 256, 0, s>>>(aos, n, npot, ngrad, nhess, inv, pot, grad,
                                                     hess);
  FGT_LAUNCH_CHECK();
  launches += 2;
}

struct DevicePool {
  bool configured = false;
};

void configure_pool(int dev) {
  static std::mutex mu;
  static std::vector<char> done(64, 0);
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 0 || dev >= 64 || done[dev]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  done[dev] = 1;
}

cudaStream_t library_stream(int dev) {
  static thread_local cudaStream_t streams[64] = {0};
  static thread_local bool made[64] = {false};
  if (dev < 0 || dev >= 64) return 0;
  if (!made[dev]) {
    FGT_CUDA(cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking));
    made[dev] = true;
  }
  return streams[dev];
}

// Per-thread side stream for the strength copies of host-buffer calls, and
// its two events (copy may start, copy done).
struct SideStream {
  cudaStream_t s = nullptr;
  cudaEvent_t gate = nullptr, done = nullptr, out = nullptr;
};
SideStream& side_stream(int dev) {
  static thread_local SideStream ss[64];
  SideStream& x = ss[dev < 0 || dev >= 64 ? 0 : dev];
  if (!x.s) {
    FGT_CUDA(cudaStreamCreateWithFlags(&x.s, cudaStreamNonBlocking));
    FGT_CUDA(cudaEventCreateWithFlags(&x.gate, cudaEventDisableTiming));
    FGT_CUDA(cudaEventCreateWithFlags(&x.done, cudaEventDisableTiming));
    FGT_CUDA(cudaEventCreateWithFlags(&x.out, cudaEventDisableTiming));
  }
  return x;
}
// Waits for the side stream when a call leaves (also on error paths), so
// no copy into the call's workspace outlives it.
struct SideSync {
  cudaStream_t s = nullptr;
  ~SideSync() {
    if (s) (void)cudaStreamSynchronize(s);
  }
};

// Phase names of fgt_stats.ms (slots 0..9).
const char* const kPhaseName[10] = {"h2d",       "tree",  "sort_gather", "lists", "form",
                                    "translate", "eval",  "direct",      "scatter", "d2h"};

// Phase boundaries of a call: CUDA events on the call's stream when timing
// is on, and always an NVTX marker "fgt <phase> done" for profilers
// (nothing happens unless a tool is attached).  mark(k) ends phase k.
struct Timer {
  bool on;
  cudaStream_t s;
  std::vector<cudaEvent_t> ev;
  std::vector<int> slot;
  Timer(bool o, cudaStream_t st) : on(o), s(st) {}
  void mark(int phase_slot) {
    if (phase_slot >= 0 && phase_slot < 10) {
      char name[48];
      snprintf(name, sizeof(name), "fgt %s done", kPhaseName[phase_slot]);
      nvtxMarkA(name);
    }
    if (!on) return;
    cudaEvent_t e;
    FGT_CUDA(cudaEventCreate(&e));
    FGT_CUDA(cudaEventRecord(e, s));
    ev.push_back(e);
    slot.push_back(phase_slot);
  }
  void finish(double* ms) {
    if (!on) return;
    FGT_CUDA(cudaStreamSynchronize(s));
    for (size_t i = 1; i < ev.size(); i++) {
      float t = 0;
      cudaEventElapsedTime(&t, ev[i - 1], ev[i]);
      if (slot[i] >= 0 && slot[i] < 12) ms[slot[i]] += t;
    }
    if (ev.size() >= 2) {
      float t = 0;
      cudaEventElapsedTime(&t, ev.front(), ev.back());
      ms[10] = t;
    }
  }
  ~Timer() {
    for (auto e : ev) cudaEventDestroy(e);
  }
};

struct Call {
  int nd, dim, iperiod, ns, nt, ifcharge, ifdipole, ifpgh, ifpghtarg;
  double delta, eps;
  const double *src, *q, *rn, *ds, *trg;  // device pointers
  double *pot, *grad, *hess, *pott, *gradt, *hesst;  // device pointers
  // host-buffer calls: q/rn/ds arrive on a side stream while the tree is
  // built; the strength-dependent part waits for this event
  cudaEvent_t strengths_ready = nullptr;
  // when set: the source outputs are finished (near field and reorder of
  // the sources before those of the targets) when this event completes, so
  // their device-to-host copy overlaps the targets' remaining work
  cudaEvent_t sources_done = nullptr;
};

// Point-dependent part of a call: scalar set-up, tree, lists, sorted FP64
// offsets of every point from its reference box centre, and the inverse leaf
// permutations of the output reorder.  Independent of the strengths and of
// the arithmetic type, so a plan can keep it across calls.
struct Setup {
  int dim = 0, nd = 0, iperiod = 0, ns = 0, nt = 0;
  double delta = 0, eps = 0;
  int npwlevel = 0, ndiv = 0, nlevels = 0, npw = 0, iperiod0 = 0, nlevend = 0;
  double pmax = 0, bs0 = 0, cen0[FGT_MAXDIM] = {0, 0, 0};
  bool periodic_nodes = false, do_pw = false;
  Tree t;
  Lists L;
  DBuf<double> soff, toff;
  DBuf<uint32_t> inv_s, inv_t;
  // packed list-1 sources of the FP32 charge path: record count (-1: not
  // built) and the positions of every list entry's records
  long long near_total = -1;
  DBuf<int> near_pos;
  int launches = 0;
};

// Records of the packed list-1 sources are 64 bytes; above this count (16 GiB,
// and at most an eighth of the device's memory) the near field walks the
// list instead.  The cap depends only on the device, so repeated calls take
// the same path and reuse the same workspace.  FGT_NEAR_PACK_MAX (a record
// count, 0 = never pack) lowers it, e.g. to test the list-walking kernel.
constexpr long long kMaxNearRecords = 1ll << 28;
long long near_pack_max() {
  static std::mutex mu;
  static long long caps[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    (void)cudaGetLastError();
    dev = 0;
  }
  long long cap;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (caps[dev] == 0) {
      size_t free_b = 0, total_b = 0;
      long long c = kMaxNearRecords;
      if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess)
        c = std::min(c, (long long)(total_b / 8 / 64));
      else
        (void)cudaGetLastError();
      caps[dev] = std::max(c, 1ll);
    }
    cap = caps[dev];
  }
  const char* e = getenv("FGT_NEAR_PACK_MAX");
  if (e && *e) {
    char* end = nullptr;
    const long long v = strtoll(e, &end, 10);
    if (end != e && v >= 0) return std::min(v, cap);
  }
  return cap;
}

DirectGeom direct_geom(const Setup& u) {
  DirectGeom g;
  g.dim = u.dim;
  g.nd = u.nd;
  g.iperiod0 = u.iperiod0;
  g.nboxes = u.t.nboxes;
  g.delta = u.delta;
  g.dmax = log(1.0 / u.eps) * u.delta;
  g.bs0 = u.t.boxsize[0];
  g.center = u.t.center;
  g.level = u.t.level;
  return g;
}

// near_lists: build the positions of the packed list-1 sources (FP32, one
// density; used by executions with charges only and pgh <= 2).
void setup_geometry(Setup& u, const Call& c, double* bs0_io, double* cen0_io, const fgt_opts& o,
                    bool near_lists, cudaStream_t s, Timer& tm) {
  const int dim = c.dim;
  u.dim = dim;
  u.nd = c.nd;
  u.iperiod = c.iperiod;
  u.ns = c.ns;
  u.nt = c.nt;
  u.delta = c.delta;
  u.eps = c.eps;
  int launches = 0;
  // --- scalar set-up (pfgt.f:110-140)
  int npwlevel = 0;
  double bs0 = *bs0_io, cen0[FGT_MAXDIM] = {0, 0, 0};
  for (int k = 0; k < dim; k++) cen0[k] = cen0_io[k];
  const bool fixed_root = c.iperiod != 1 && o.root_level >= 0;
  if (fixed_root) {
    // a spatial shard: the root box and cut-off level of the whole point set
    FGT_REQUIRE(bs0 > 0 && isfinite(bs0), FGT_ERR_ARG, "root_level needs bs0 > 0");
    npwlevel = o.root_level;
  } else {
    tree_setup_scalars(dim, c.delta, c.eps, c.iperiod, c.src, c.ns, c.trg, c.nt, &npwlevel, &bs0,
                       cen0, s);
    launches += (c.iperiod != 1) ? 2 : 0;
  }
  if (c.iperiod != 1 && !fixed_root) {
    *bs0_io = bs0;
    for (int k = 0; k < dim; k++) cen0_io[k] = cen0[k];
  }
  u.bs0 = bs0;
  for (int k = 0; k < dim; k++) u.cen0[k] = cen0[k];
  int ndiv = o.ndiv > 0 ? o.ndiv : (dim == 1 ? 20 : (dim == 2 ? 80 : 250));
  // --- tree (pts_tree_mem/build, pts_tree_sort)
  Tree& t = u.t;
  tree_build(t, dim, c.iperiod, npwlevel, ndiv, bs0, cen0, c.src, c.ns, c.trg, c.nt, s);
  launches += 12 + 6 * t.nlevels;
  tm.mark(1);
  const int nlevels = t.nlevels;
  // --- expansion length (pfgt.f:321-334, fgtterms.f:72-141)
  int npw = 0;
  double pmax = 0, pi = 4.0 * atan(1.0);
  auto pwterms = [&](double bsize, int iper) {
    if (iper == 0) {
      double rmax = bsize / sqrt(c.delta), d = sqrt(log(1.0 / c.eps));
      pmax = 2.0 * d;
      double h = 2 * pi / (rmax + d);
      npw = 2 * ((int)(pmax / h) + 1);
    } else {
      npw = 2 * ((int)(bsize * sqrt(log(1.0 / c.eps) / c.delta) / pi) + 1) + 1;
    }
  };
  if (npwlevel <= nlevels) {
    if (npwlevel <= 1) {
      pwterms(2 * t.boxsize[std::max(npwlevel, 0)], c.iperiod);
      if (c.iperiod == 1) npw = npw + 1;
    } else {
      pwterms(2 * t.boxsize[npwlevel], 0);
    }
  }
  if (npw < 4) npw = 4;
  // --- pfgtmain set-up (pfgt.f:611-650)
  int iperiod0 = c.iperiod;
  bool periodic_nodes = false;
  if (npwlevel <= 1 && c.iperiod == 1) {
    periodic_nodes = true;
    iperiod0 = 0;
  }
  int nlevend = nlevels;
  if (npwlevel <= nlevels) nlevend = npwlevel;
  bool do_pw = npwlevel < nlevels;
  // A root smaller than the cut-off with ns <= ndiv forms no expansion; the
  // reference then returns zeros (pfgt.f:649-650, 779).  Compute its direct
  // self interaction instead.
  if (npwlevel < 0 && c.ns <= ndiv) {
    do_pw = false;
    nlevend = 0;
  }
  build_lists(t, npwlevel, iperiod0, nlevend, do_pw, u.L, s);
  launches += do_pw ? 8 : 2;
  tm.mark(3);
  // --- gather (dreorderf, fmmcommon2d.f:3-27) as offsets from reference boxes
  u.soff.alloc((size_t)c.ns * dim, s);
  u.toff.alloc((size_t)std::max(c.nt, 1) * dim, s);
  launch_gather_coords<double>(dim, c.src, c.ns, t.isrc, t.src_ref, t.center, t.nboxes, u.soff, s);
  launches++;
  if (c.nt > 0) {
    launch_gather_coords<double>(dim, c.trg, c.nt, t.itrg, t.trg_ref, t.center, t.nboxes, u.toff, s);
    launches++;
  }
  // inverse leaf permutations for the output reorder
  u.inv_s.alloc(std::max(c.ns, 1), s);
  k_invert<<<grid_for(c.ns, 256), 256, 0, s>>>(t.isrc, c.ns, u.inv_s);
  FGT_LAUNCH_CHECK();
  launches++;
  u.inv_t.alloc(std::max(c.nt, 1), s);
  if (c.nt > 0) {
    k_invert<<<grid_for(c.nt, 256), 256, 0, s>>>(t.itrg, c.nt, u.inv_t);
    FGT_LAUNCH_CHECK();
    launches++;
  }
  u.npwlevel = npwlevel;
  u.iperiod0 = iperiod0;
  if (near_lists && u.L.n_l1 > 0) {
    u.near_total = near_lists_count(direct_geom(u), u.L, t.src_lo, t.src_hi, t.trg_lo, t.trg_hi,
                                    u.soff, c.ns, near_pack_max(), u.near_pos, s);
    launches += 2;
  }
  u.ndiv = ndiv;
  u.nlevels = nlevels;
  u.npw = npw;
  u.pmax = pmax;
  u.periodic_nodes = periodic_nodes;
  u.nlevend = nlevend;
  u.do_pw = do_pw;
  u.launches = launches;
}

// Strength-dependent part of a call on a prepared geometry.
template <typename T>
void execute(const Setup& u, const Call& c, const fgt_opts& o, fgt_stats* st, cudaStream_t s,
             Timer& tm) {
  const int dim = u.dim, nd = u.nd, nhess = dim * (dim + 1) / 2;
  const Tree& t = u.t;
  const Lists& L = u.L;
  int launches = u.launches;
  if (c.strengths_ready) FGT_CUDA(cudaStreamWaitEvent(s, c.strengths_ready, 0));
  DBuf<T> qs, dss, rns;
  if (c.ifcharge) {
    qs.alloc((size_t)c.ns * nd, s);
    k_gather_vals<T><<<grid_for(c.ns, 256), 256, 0, s>>>(c.q, c.ns, nd, t.isrc, qs);
    FGT_LAUNCH_CHECK();
    launches++;
  }
  if (c.ifdipole) {
    dss.alloc((size_t)c.ns * nd, s);
    rns.alloc((size_t)c.ns * dim, s);
    k_gather_vals<T><<<grid_for(c.ns, 256), 256, 0, s>>>(c.ds, c.ns, nd, t.isrc, dss);
    FGT_LAUNCH_CHECK();
    // rnormal(dim,ns) -> SoA [dim][n]
    k_gather_vals<T><<<grid_for(c.ns, 256), 256, 0, s>>>(c.rn, c.ns, dim, t.isrc, rns);
    FGT_LAUNCH_CHECK();
    launches += 2;
  }
  // sorted outputs, FP64
  int ncs = c.ifpgh >= 1 ? (1 + (c.ifpgh >= 2 ? dim : 0) + (c.ifpgh >= 3 ? nhess : 0)) : 0;
  int nct = c.ifpghtarg >= 1 ? (1 + (c.ifpghtarg >= 2 ? dim : 0) + (c.ifpghtarg >= 3 ? nhess : 0)) : 0;
  DBuf<double> outs((size_t)std::max(ncs, 1) * nd * c.ns, s);
  DBuf<double> outt((size_t)std::max(nct, 1) * nd * std::max(c.nt, 1), s);
  outs.zero();
  outt.zero();
  launches += 2;
  SourceSet<T> src;
  src.n = c.ns;
  src.off = u.soff;
  src.q = c.ifcharge ? qs.get() : nullptr;
  src.ds = c.ifdipole ? dss.get() : nullptr;
  src.rn = c.ifdipole ? rns.get() : nullptr;
  src.lo = t.src_lo;
  src.hi = t.src_hi;
  EvalSet<T> es, et;
  es.n = c.ns; es.pgh = c.ifpgh; es.off = u.soff; es.lo = t.src_lo; es.hi = t.src_hi; es.out = outs;
  et.n = c.nt; et.pgh = c.ifpghtarg; et.off = u.toff; et.lo = t.trg_lo; et.hi = t.trg_hi; et.out = outt;
  tm.mark(2);
  // --- plane waves (pfgt.f:700-1073)
  PWWork work;
  PWParams P;
  PWData<T> D;
  PWWork* wk = st ? &work : nullptr;
  const int se = o.small_eval >= 0 ? o.small_eval : -1;
  const bool pw = u.do_pw && L.n_eval > 0;
  // Host-buffer calls finish the sources first and copy their outputs to the
  // host while the targets are evaluated: the two sets are evaluated in two
  // launches (each box's grid is built twice, which the copy hides).
  const bool split_sets = c.sources_done && c.ifpgh >= 1 && c.ifpghtarg >= 1 && c.nt > 0;
  EvalSet<T> none;
  if (pw) {
    pw_setup(P, dim, nd, u.npw, u.pmax, u.periodic_nodes ? 1 : 0, t.boxsize[0], c.delta, c.eps,
             t.boxsize[t.ncutoff], o.spread_width);
    launches += pw_form<T>(P, t, L, src, D, wk, s);
    tm.mark(4);
    launches += pw_translate<T>(P, L, D, wk, s);
    tm.mark(5);
    launches += pw_eval<T>(P, t, L, D, es, split_sets ? none : et, se, wk, s);
    tm.mark(6);
    if (st) {
      st->spread_width = P.w;
      st->grid_cells = P.G;
    }
  }
  // --- direct near field (pfgt.f:1082-1136)
  const DirectGeom g = direct_geom(u);
  double pairs = 0;
  NearPacked packed;
  DBuf<float4> near_rec;
  if constexpr (sizeof(T) == 4) {
    if (u.near_total > 0 && nd == 1 && c.ifcharge && !c.ifdipole && c.ifpgh <= 2 &&
        c.ifpghtarg <= 2) {
      near_rec.alloc((size_t)u.near_total * 4, s);
      near_lists_fill(g, L, src, t.trg_lo, t.trg_hi, u.near_pos, near_rec, s);
      launches++;
      packed.pos = u.near_pos;
      packed.rec = near_rec;
    }
  }
  if (c.sources_done) {
    // sources first, then signal; the targets follow
    launches += direct_near_field<T>(g, L, src, es, st ? &pairs : nullptr, s, &packed);
    if (c.ifpgh >= 1)
      reorder_outputs(outs, c.ns, nd, dim, c.ifpgh, u.inv_s, c.pot, c.grad, c.hess, s, launches);
    FGT_CUDA(cudaEventRecord(c.sources_done, s));
    if (pw && split_sets) launches += pw_eval<T>(P, t, L, D, none, et, se, wk, s);
    launches += direct_near_field<T>(g, L, src, et, st ? &pairs : nullptr, s, &packed);
  } else {
    launches += direct_near_field<T>(g, L, src, et, st ? &pairs : nullptr, s, &packed);
    launches += direct_near_field<T>(g, L, src, es, st ? &pairs : nullptr, s, &packed);
  }
  tm.mark(7);
  // --- back to input order
  if (c.ifpgh >= 1 && !c.sources_done)
    reorder_outputs(outs, c.ns, nd, dim, c.ifpgh, u.inv_s, c.pot, c.grad, c.hess, s, launches);
  if (c.ifpghtarg >= 1 && c.nt > 0)
    reorder_outputs(outt, c.nt, nd, dim, c.ifpghtarg, u.inv_t, c.pott, c.gradt, c.hesst, s,
                    launches);
  tm.mark(8);
  if (st) {
    st->nlevels = u.nlevels;
    st->nboxes = t.nboxes;
    st->npwlevel = u.npwlevel;
    st->npw = u.npw;
    st->ndiv = u.ndiv;
    st->n_form_boxes = L.n_form;
    st->n_eval_boxes = L.n_eval;
    st->n_eval_nufft = work.n_nufft;
    st->flops_form = work.flops_form;
    st->flops_eval = work.flops_eval;
    st->bytes_translate = work.bytes_translate;
    st->pts_form = work.pts_form;
    st->pts_eval_nufft = work.pts_nufft;
    st->pts_eval_modal = work.pts_modal;
    st->slabs_form = work.slabs_form;
    st->slabs_eval = work.slabs_eval;
    {
      // near-field pair arithmetic (charge: 12 pot, 21 +grad, 21+5*nhess +hess)
      auto per = [&](int pgh) {
        double f = pgh >= 3 ? 21 + 5.0 * nhess : (pgh == 2 ? 21 : 12);
        if (c.ifdipole) f += 4.0 * dim + 4;
        return f;
      };
      st->flops_direct = pairs * per(std::max(c.ifpgh, c.ifpghtarg));
    }
    st->n_translations = L.n_trans;
    st->near_pairs = pairs;
    st->n_kernel_launches = launches;
    st->bs0 = u.bs0;
    for (int k = 0; k < dim; k++) st->cen0[k] = u.cen0[k];
  }
}

// ---------------------------------------------------------------- autotuner
// Threshold (evaluation points per box) below which a box is evaluated by
// direct modal sums instead of a grid, when not tuned or given.
int default_small_eval(int dim) { return dim == 3 ? 48 : (dim == 2 ? 8 : 4); }

// Problem class of a call for the tuning cache: dimension, arithmetic,
// requested fields, densities, point count (power of two), cut-off level,
// tree depth and expansion length.
std::string tune_key(const Setup& u, const Call& c, size_t tsize) {
  char k[200];
  long long n = (long long)c.ns + (c.ifpghtarg > 0 ? c.nt : 0);
  int lg = 0;
  while ((1ll << (lg + 1)) <= n) lg++;
  snprintf(k, sizeof(k), "pfgt/v1 dim=%d fp%d pgh=%d,%d nd=%d dip=%d lg2n=%d npwlevel=%d nlevels=%d npw=%d",
           u.dim, (int)(8 * tsize), c.ifpgh, c.ifpghtarg, c.nd, c.ifdipole ? 1 : 0, lg,
           u.npwlevel, u.nlevels, u.npw);
  return k;
}

// Times the strength-dependent part of the call on its prepared geometry
// with each candidate modal-evaluation threshold (the workspace rewound
// after every run, best of two runs each after one warm-up run), stores the
// fastest under `key` and returns it.  The outputs of these runs are
// overwritten by the call's final run.
template <typename T>
int tune_small_eval(const Setup& u, const Call& c, const fgt_opts& o, cudaStream_t s,
                    const std::string& key) {
  static const int c3[] = {0, 16, 32, 48, 64, 96, 128};
  static const int c2[] = {0, 4, 8, 16, 32, 64};
  static const int c1[] = {0, 2, 4, 8, 16};
  const int* cand = u.dim == 3 ? c3 : (u.dim == 2 ? c2 : c1);
  const int ncand = u.dim == 3 ? 7 : (u.dim == 2 ? 6 : 5);
  Arena* ar = thread_arena();
  Timer none(false, s);
  fgt_opts oo = o;
  oo.stats = nullptr;
  oo.timing = 0;
  cudaEvent_t e0, e1;
  FGT_CUDA(cudaEventCreate(&e0));
  FGT_CUDA(cudaEventCreate(&e1));
  int best = default_small_eval(u.dim);
  float best_ms = 1e30f;
  try {
    auto run = [&](int se) {
      const std::vector<size_t> m = ar->mark();
      oo.small_eval = se;
      execute<T>(u, c, oo, nullptr, s, none);
      ar->rewind(m);
    };
    run(-1);  // module loads and workspace growth
    for (int i = 0; i < ncand; i++) {
      float t = 1e30f;
      for (int rep = 0; rep < 2; rep++) {
        FGT_CUDA(cudaEventRecord(e0, s));
        run(cand[i]);
        FGT_CUDA(cudaEventRecord(e1, s));
        FGT_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        FGT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        t = std::min(t, ms);
      }
      if (t < best_ms) {
        best_ms = t;
        best = cand[i];
      }
    }
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  tune_store(key, best);
  return best;
}

template <typename T>
void run_pfgt(const Call& c, double* bs0_io, double* cen0_io, const fgt_opts& o, fgt_stats* st,
              cudaStream_t s, Timer& tm) {
  Setup u;
  // the packed near-field path: FP32, one density, charges only, pgh <= 2
  const bool near = sizeof(T) == 4 && c.nd == 1 && c.ifcharge && !c.ifdipole && c.ifpgh <= 2 &&
                    c.ifpghtarg <= 2;
  setup_geometry(u, c, bs0_io, cen0_io, o, near, s, tm);
  fgt_opts oo = o;
  int tuned = 0;
  if (o.autotune > 0 && o.small_eval < 0 && u.do_pw) {
    const std::string key = tune_key(u, c, sizeof(T));
    int v = 0;
    if (tune_lookup(key, v)) {
      oo.small_eval = v;
      tuned = 1;
    } else if (o.autotune >= 2) {
      oo.small_eval = tune_small_eval<T>(u, c, o, s, key);
      tuned = 1;
    }
  }
  execute<T>(u, c, oo, st, s, tm);
  if (st) {
    st->small_eval_used = oo.small_eval >= 0 ? oo.small_eval : default_small_eval(c.dim);
    st->tuned = tuned;
  }
}

bool fault_requested(const char* what) {
  const char* f = getenv("FGT_FAULT");
  return f && strstr(f, what) != nullptr;
}

// FGT_LOG=1 (any value but "0"): every pfgt call times its phases and
// writes one JSON line to stderr with the tree and list sizes, the per-phase
// device times and the achieved rates of the form, evaluation, near-field
// and translation kernels.  Silent by default.
bool log_requested() {
  const char* f = getenv("FGT_LOG");
  return f && *f && strcmp(f, "0") != 0;
}

void log_call(const fgt_stats& st, int nd, int dim, int ns, int nt, double delta, double eps) {
  static std::mutex mu;
  char ms[512];
  int k = snprintf(ms, sizeof(ms), "{");
  for (int i = 0; i < 10; i++)
    k += snprintf(ms + k, sizeof(ms) - k, "%s\"%s\": %.4f", i ? ", " : "", kPhaseName[i],
                  st.ms[i]);
  snprintf(ms + k, sizeof(ms) - k, ", \"total\": %.4f}", st.ms[10]);
  auto rate = [](double work, double msec) { return msec > 0 ? work / (msec * 1e-3) : 0.0; };
  std::lock_guard<std::mutex> lk(mu);
  fprintf(stderr,
          "{\"fgt\": \"pfgt\", \"nd\": %d, \"dim\": %d, \"ns\": %d, \"nt\": %d, "
          "\"delta\": %.6g, \"eps\": %.6g, \"precision\": \"%s\", \"nlevels\": %d, "
          "\"nboxes\": %d, \"npwlevel\": %d, \"npw\": %d, \"n_form_boxes\": %d, "
          "\"n_eval_boxes\": %d, \"n_translations\": %d, \"near_pairs\": %.6g, "
          "\"kernel_launches\": %d, \"ms\": %s, \"tflops\": {\"form\": %.4g, "
          "\"eval\": %.4g, \"direct\": %.4g}, \"translate_gbs\": %.4g}\n",
          nd, dim, ns, nt, delta, eps, st.precision_used == FGT_PREC_FP64 ? "fp64" : "mixed",
          st.nlevels, st.nboxes, st.npwlevel, st.npw, st.n_form_boxes, st.n_eval_boxes,
          st.n_translations, st.near_pairs, st.n_kernel_launches, ms,
          rate(st.flops_form, st.ms[4]) * 1e-12, rate(st.flops_eval, st.ms[6]) * 1e-12,
          rate(st.flops_direct, st.ms[7]) * 1e-12, rate(st.bytes_translate, st.ms[5]) * 1e-9);
  fflush(stderr);
}

// Device-side failures of a call, read after its last synchronisation:
// a bounded wait that ran out (FGT_ERR_TIMEOUT) and, in the FGT_CHECK build,
// a failed bounds check (FGT_ERR_CHECK, the first failing site named).
void raise_failed_checks(cudaStream_t s) {
  if (near_wait_status(s) == FGT_ERR_TIMEOUT) {
    fgt_set_error_message("a bounded wait of the near-field kernel ran out", __FILE__, __LINE__);
    throw Error{FGT_ERR_TIMEOUT, "a bounded wait of the near-field kernel ran out"};
  }
#ifdef FGT_CHECK
  const unsigned site = check_sites(s);
  if (site) {
    static thread_local char msg[96];
    snprintf(msg, sizeof(msg), "device bounds check failed at site %u", site);
    fgt_set_error_message(msg, __FILE__, __LINE__);
    throw Error{FGT_ERR_CHECK, msg};
  }
#else
  (void)s;
#endif
}

int pfgt_impl(const fgt_opts* opts_in, int nd, int dim, double delta, double eps, int iperiod,
              double* bs0, double* cen0, int ns, const double* sources, int ifcharge,
              const double* charge, int ifdipole, const double* rnormal, const double* dipstr,
              int ifpgh, double* pot, double* grad, double* hess, int nt, const double* targ,
              int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg) {
  fgt_opts o;
  fgt_opts_default(&o);
  if (opts_in) o = *opts_in;
  // argument checks
  FGT_REQUIRE(dim >= 1 && dim <= 3, FGT_ERR_ARG, "dim must be 1, 2 or 3");
  FGT_REQUIRE(nd >= 1, FGT_ERR_ARG, "nd must be >= 1");
  FGT_REQUIRE(delta > 0 && isfinite(delta), FGT_ERR_ARG, "delta must be positive");
  FGT_REQUIRE(eps > 0 && eps < 1, FGT_ERR_ARG, "eps must lie in (0,1)");
  FGT_REQUIRE(ns >= 1, FGT_ERR_ARG, "ns must be >= 1");
  FGT_REQUIRE(nt >= 0, FGT_ERR_ARG, "nt must be >= 0");
  FGT_REQUIRE(iperiod == 0 || iperiod == 1, FGT_ERR_ARG, "iperiod must be 0 or 1");
  FGT_REQUIRE(ifcharge == 1 || ifdipole == 1, FGT_ERR_ARG, "need charges and/or dipoles");
  FGT_REQUIRE(ifpgh >= 0 && ifpgh <= 3 && ifpghtarg >= 0 && ifpghtarg <= 3, FGT_ERR_ARG,
              "ifpgh/ifpghtarg must lie in 0..3");
  FGT_REQUIRE(sources && bs0 && cen0, FGT_ERR_ARG, "null sources/bs0/cen0");
  FGT_REQUIRE(!(ifcharge == 1 && !charge), FGT_ERR_ARG, "null charge");
  FGT_REQUIRE(!(ifdipole == 1 && (!dipstr || !rnormal)), FGT_ERR_ARG, "null dipole arrays");
  FGT_REQUIRE(!(ifpgh >= 1 && !pot) && !(ifpgh >= 2 && !grad) && !(ifpgh >= 3 && !hess),
              FGT_ERR_ARG, "null source output");
  FGT_REQUIRE(!(nt > 0 && !targ), FGT_ERR_ARG, "null targets");
  FGT_REQUIRE(!(nt > 0 && ifpghtarg >= 1 && !pottarg) && !(nt > 0 && ifpghtarg >= 2 && !gradtarg) &&
                  !(nt > 0 && ifpghtarg >= 3 && !hesstarg),
              FGT_ERR_ARG, "null target output");
  FGT_REQUIRE(!(iperiod == 1 && !(*bs0 > 0)), FGT_ERR_ARG, "periodic bs0 must be positive");
  if (fault_requested("launch") || fault_requested("alloc") || fault_requested("queue")) {
    fgt_set_error_message("fault injected by FGT_FAULT", __FILE__, __LINE__);
    return FGT_ERR_INJECTED;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    (void)cudaGetLastError();
    fgt_set_error_message("no CUDA device", __FILE__, __LINE__);
    return FGT_ERR_NODEVICE;
  }
  int dev = o.device;
  if (dev < 0) FGT_CUDA(cudaGetDevice(&dev));
  FGT_CUDA(cudaSetDevice(dev));
  configure_pool(dev);
  cudaStream_t s = o.stream ? (cudaStream_t)o.stream : library_stream(dev);
  ArenaScope arena_scope(s);
  fgt_stats local_stats;
  const bool logging = log_requested();
  fgt_stats* st = o.stats ? o.stats : (logging ? &local_stats : nullptr);
  if (st) memset(st, 0, sizeof(*st));
  Timer tm((o.timing || logging) && st, s);
  int nhess = dim * (dim + 1) / 2;
  int prec = o.precision;
  if (prec == FGT_PREC_AUTO) prec = (eps >= 1e-6 * (1 - 1e-9)) ? FGT_PREC_MIXED : FGT_PREC_FP64;
  Call c;
  c.nd = nd; c.dim = dim; c.iperiod = iperiod; c.ns = ns; c.nt = nt;
  c.ifcharge = ifcharge == 1; c.ifdipole = ifdipole == 1;
  c.ifpgh = ifpgh; c.ifpghtarg = nt > 0 ? ifpghtarg : 0;
  c.delta = delta; c.eps = eps;
  tm.mark(-1);
  // inputs on the device
  DBuf<double> d_src, d_q, d_rn, d_ds, d_trg, d_pot, d_grad, d_hess, d_pt, d_gt, d_ht;
  auto h2d = [&](DBuf<double>& b, const double* h, size_t n) -> const double* {
    if (o.device_ptrs) return h;
    b.alloc(n, s);
    FGT_CUDA(cudaMemcpyAsync(b.get(), h, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    return b.get();
  };
  auto dout = [&](DBuf<double>& b, double* h, size_t n) -> double* {
    if (o.device_ptrs) return h;
    b.alloc(n, s);
    return b.get();
  };
  c.src = h2d(d_src, sources, (size_t)ns * dim);
  c.trg = nt > 0 ? h2d(d_trg, targ, (size_t)nt * dim) : c.src;
  SideSync side_sync;
  SideStream* ssp = nullptr;
  if (o.device_ptrs) {
    c.q = c.ifcharge ? charge : nullptr;
    c.rn = c.ifdipole ? rnormal : nullptr;
    c.ds = c.ifdipole ? dipstr : nullptr;
  } else {
    // strengths are first needed after the tree and lists: copy them on the
    // side stream meanwhile
    SideStream& ss = side_stream(dev);
    ssp = &ss;
    auto side = [&](DBuf<double>& b, const double* h, size_t n) -> const double* {
      b.alloc(n, s);
      FGT_CUDA(cudaMemcpyAsync(b.get(), h, sizeof(double) * n, cudaMemcpyHostToDevice, ss.s));
      return b.get();
    };
    FGT_CUDA(cudaEventRecord(ss.gate, s));
    FGT_CUDA(cudaStreamWaitEvent(ss.s, ss.gate, 0));
    side_sync.s = ss.s;
    c.q = c.ifcharge ? side(d_q, charge, (size_t)ns * nd) : nullptr;
    c.rn = c.ifdipole ? side(d_rn, rnormal, (size_t)ns * dim) : nullptr;
    c.ds = c.ifdipole ? side(d_ds, dipstr, (size_t)ns * nd) : nullptr;
    FGT_CUDA(cudaEventRecord(ss.done, ss.s));
    c.strengths_ready = ss.done;
    c.sources_done = ss.out;
  }
  c.pot = ifpgh >= 1 ? dout(d_pot, pot, (size_t)ns * nd) : nullptr;
  c.grad = ifpgh >= 2 ? dout(d_grad, grad, (size_t)ns * nd * dim) : nullptr;
  c.hess = ifpgh >= 3 ? dout(d_hess, hess, (size_t)ns * nd * nhess) : nullptr;
  c.pott = c.ifpghtarg >= 1 ? dout(d_pt, pottarg, (size_t)nt * nd) : nullptr;
  c.gradt = c.ifpghtarg >= 2 ? dout(d_gt, gradtarg, (size_t)nt * nd * dim) : nullptr;
  c.hesst = c.ifpghtarg >= 3 ? dout(d_ht, hesstarg, (size_t)nt * nd * nhess) : nullptr;
  tm.mark(0);
  if (prec == FGT_PREC_FP64) run_pfgt<double>(c, bs0, cen0, o, st, s, tm);
  else run_pfgt<float>(c, bs0, cen0, o, st, s, tm);
  if (!o.device_ptrs) {
    // source outputs on the side stream once they are final, target outputs
    // on the call's stream
    cudaStream_t so = side_sync.s ? side_sync.s : s;
    if (side_sync.s && c.sources_done) FGT_CUDA(cudaStreamWaitEvent(so, c.sources_done, 0));
    auto d2h = [&](double* h, const DBuf<double>& b, size_t n, cudaStream_t q) {
      if (h && b.p) FGT_CUDA(cudaMemcpyAsync(h, b.get(), sizeof(double) * n, cudaMemcpyDeviceToHost, q));
    };
    if (ifpgh >= 1) d2h(pot, d_pot, (size_t)ns * nd, so);
    if (ifpgh >= 2) d2h(grad, d_grad, (size_t)ns * nd * dim, so);
    if (ifpgh >= 3) d2h(hess, d_hess, (size_t)ns * nd * nhess, so);
    if (c.ifpghtarg >= 1) d2h(pottarg, d_pt, (size_t)nt * nd, s);
    if (c.ifpghtarg >= 2) d2h(gradtarg, d_gt, (size_t)nt * nd * dim, s);
    if (c.ifpghtarg >= 3) d2h(hesstarg, d_ht, (size_t)nt * nd * nhess, s);
    if (so != s && ssp) {  // the call's stream completes after the side copies
      FGT_CUDA(cudaEventRecord(ssp->gate, so));
      FGT_CUDA(cudaStreamWaitEvent(s, ssp->gate, 0));
    }
  }
  tm.mark(9);
  FGT_CUDA(cudaStreamSynchronize(s));
  raise_failed_checks(s);
  if (st) {
    st->precision_used = prec;
    tm.finish(st->ms);
    if (logging) log_call(*st, nd, dim, ns, nt, delta, eps);
  }
  return FGT_OK;
}

}  // namespace

}  // namespace fgt

// A plan: the point-dependent part of pfgt (tree, lists, sorted offsets,
// inverse permutations) kept on the device, in an arena the plan owns, for
// repeated calls with new strengths on the same points.
struct fgt_plan {
  int device = 0;
  int prec = FGT_PREC_MIXED;
  fgt_opts o;
  fgt::Arena* arena = nullptr;
  fgt::Setup u;
};

namespace fgt {
namespace {

fgt_plan* plan_create_impl(const fgt_opts* opts_in, int nd, int dim, double delta, double eps,
                           int iperiod, double* bs0, double* cen0, int ns, const double* sources,
                           int nt, const double* targ) {
  fgt_opts o;
  fgt_opts_default(&o);
  if (opts_in) o = *opts_in;
  FGT_REQUIRE(dim >= 1 && dim <= 3, FGT_ERR_ARG, "dim must be 1, 2 or 3");
  FGT_REQUIRE(nd >= 1, FGT_ERR_ARG, "nd must be >= 1");
  FGT_REQUIRE(delta > 0 && isfinite(delta), FGT_ERR_ARG, "delta must be positive");
  FGT_REQUIRE(eps > 0 && eps < 1, FGT_ERR_ARG, "eps must lie in (0,1)");
  FGT_REQUIRE(ns >= 1, FGT_ERR_ARG, "ns must be >= 1");
  FGT_REQUIRE(nt >= 0, FGT_ERR_ARG, "nt must be >= 0");
  FGT_REQUIRE(iperiod == 0 || iperiod == 1, FGT_ERR_ARG, "iperiod must be 0 or 1");
  FGT_REQUIRE(sources && bs0 && cen0, FGT_ERR_ARG, "null sources/bs0/cen0");
  FGT_REQUIRE(!(nt > 0 && !targ), FGT_ERR_ARG, "null targets");
  FGT_REQUIRE(!(iperiod == 1 && !(*bs0 > 0)), FGT_ERR_ARG, "periodic bs0 must be positive");
  if (fault_requested("launch") || fault_requested("alloc") || fault_requested("queue"))
    throw Error{FGT_ERR_INJECTED, "fault injected by FGT_FAULT"};
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    (void)cudaGetLastError();
    fgt_set_error_message("no CUDA device", __FILE__, __LINE__);
    throw Error{FGT_ERR_NODEVICE, "no CUDA device"};
  }
  int dev = o.device;
  if (dev < 0) FGT_CUDA(cudaGetDevice(&dev));
  FGT_CUDA(cudaSetDevice(dev));
  configure_pool(dev);
  cudaStream_t s = o.stream ? (cudaStream_t)o.stream : library_stream(dev);
  fgt_plan* pl = new fgt_plan();
  pl->device = dev;
  pl->o = o;
  pl->o.stats = nullptr;
  pl->o.timing = 0;
  pl->prec = o.precision == FGT_PREC_AUTO
                 ? ((eps >= 1e-6 * (1 - 1e-9)) ? FGT_PREC_MIXED : FGT_PREC_FP64)
                 : o.precision;
  pl->arena = new Arena();
  try {
    ArenaOverride ov(pl->arena);
    Call c = {};
    c.nd = nd; c.dim = dim; c.iperiod = iperiod; c.ns = ns; c.nt = nt;
    c.delta = delta; c.eps = eps;
    DBuf<double> d_src, d_trg;
    if (o.device_ptrs) {
      c.src = sources;
      c.trg = nt > 0 ? targ : sources;
    } else {
      d_src.alloc((size_t)ns * dim, s);
      FGT_CUDA(cudaMemcpyAsync(d_src.get(), sources, sizeof(double) * ns * dim,
                               cudaMemcpyHostToDevice, s));
      c.src = d_src;
      c.trg = c.src;
      if (nt > 0) {
        d_trg.alloc((size_t)nt * dim, s);
        FGT_CUDA(cudaMemcpyAsync(d_trg.get(), targ, sizeof(double) * nt * dim,
                                 cudaMemcpyHostToDevice, s));
        c.trg = d_trg;
      }
    }
    Timer tm(false, s);
    setup_geometry(pl->u, c, bs0, cen0, o, pl->prec != FGT_PREC_FP64 && nd == 1, s, tm);
    FGT_CUDA(cudaStreamSynchronize(s));
  } catch (...) {
    cudaStreamSynchronize(s);
    pl->arena->release_all();
    delete pl->arena;
    delete pl;
    throw;
  }
  return pl;
}

int plan_execute_impl(fgt_plan* pl, int ifcharge, const double* charge, int ifdipole,
                      const double* rnormal, const double* dipstr, int ifpgh, double* pot,
                      double* grad, double* hess, int ifpghtarg, double* pottarg,
                      double* gradtarg, double* hesstarg) {
  FGT_REQUIRE(pl, FGT_ERR_ARG, "null plan");
  const Setup& u = pl->u;
  const int nd = u.nd, dim = u.dim, ns = u.ns, nt = u.nt, nhess = dim * (dim + 1) / 2;
  FGT_REQUIRE(ifcharge == 1 || ifdipole == 1, FGT_ERR_ARG, "need charges and/or dipoles");
  FGT_REQUIRE(ifpgh >= 0 && ifpgh <= 3 && ifpghtarg >= 0 && ifpghtarg <= 3, FGT_ERR_ARG,
              "ifpgh/ifpghtarg must lie in 0..3");
  FGT_REQUIRE(!(ifcharge == 1 && !charge), FGT_ERR_ARG, "null charge");
  FGT_REQUIRE(!(ifdipole == 1 && (!dipstr || !rnormal)), FGT_ERR_ARG, "null dipole arrays");
  FGT_REQUIRE(!(ifpgh >= 1 && !pot) && !(ifpgh >= 2 && !grad) && !(ifpgh >= 3 && !hess),
              FGT_ERR_ARG, "null source output");
  const int pght = nt > 0 ? ifpghtarg : 0;
  FGT_REQUIRE(!(pght >= 1 && !pottarg) && !(pght >= 2 && !gradtarg) && !(pght >= 3 && !hesstarg),
              FGT_ERR_ARG, "null target output");
  if (fault_requested("launch") || fault_requested("alloc") || fault_requested("queue"))
    throw Error{FGT_ERR_INJECTED, "fault injected by FGT_FAULT"};
  const fgt_opts& o = pl->o;
  FGT_CUDA(cudaSetDevice(pl->device));
  cudaStream_t s = o.stream ? (cudaStream_t)o.stream : library_stream(pl->device);
  ArenaScope arena_scope(s);
  Call c = {};
  c.nd = nd; c.dim = dim; c.iperiod = u.iperiod; c.ns = ns; c.nt = nt;
  c.ifcharge = ifcharge == 1; c.ifdipole = ifdipole == 1;
  c.ifpgh = ifpgh; c.ifpghtarg = pght;
  c.delta = u.delta; c.eps = u.eps;
  DBuf<double> d_q, d_rn, d_ds, d_pot, d_grad, d_hess, d_pt, d_gt, d_ht;
  auto h2d = [&](DBuf<double>& b, const double* h, size_t n) -> const double* {
    if (o.device_ptrs) return h;
    b.alloc(n, s);
    FGT_CUDA(cudaMemcpyAsync(b.get(), h, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    return b.get();
  };
  auto dout = [&](DBuf<double>& b, double* h, size_t n) -> double* {
    if (o.device_ptrs) return h;
    b.alloc(n, s);
    return b.get();
  };
  c.q = c.ifcharge ? h2d(d_q, charge, (size_t)ns * nd) : nullptr;
  c.rn = c.ifdipole ? h2d(d_rn, rnormal, (size_t)ns * dim) : nullptr;
  c.ds = c.ifdipole ? h2d(d_ds, dipstr, (size_t)ns * nd) : nullptr;
  c.pot = ifpgh >= 1 ? dout(d_pot, pot, (size_t)ns * nd) : nullptr;
  c.grad = ifpgh >= 2 ? dout(d_grad, grad, (size_t)ns * nd * dim) : nullptr;
  c.hess = ifpgh >= 3 ? dout(d_hess, hess, (size_t)ns * nd * nhess) : nullptr;
  c.pott = pght >= 1 ? dout(d_pt, pottarg, (size_t)nt * nd) : nullptr;
  c.gradt = pght >= 2 ? dout(d_gt, gradtarg, (size_t)nt * nd * dim) : nullptr;
  c.hesst = pght >= 3 ? dout(d_ht, hesstarg, (size_t)nt * nd * nhess) : nullptr;
  Timer tm(false, s);
  if (pl->prec == FGT_PREC_FP64) execute<double>(u, c, o, nullptr, s, tm);
  else execute<float>(u, c, o, nullptr, s, tm);
  if (!o.device_ptrs) {
    auto d2h = [&](double* h, const DBuf<double>& b, size_t n) {
      if (h && b.p) FGT_CUDA(cudaMemcpyAsync(h, b.get(), sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    };
    if (ifpgh >= 1) d2h(pot, d_pot, (size_t)ns * nd);
    if (ifpgh >= 2) d2h(grad, d_grad, (size_t)ns * nd * dim);
    if (ifpgh >= 3) d2h(hess, d_hess, (size_t)ns * nd * nhess);
    if (pght >= 1) d2h(pottarg, d_pt, (size_t)nt * nd);
    if (pght >= 2) d2h(gradtarg, d_gt, (size_t)nt * nd * dim);
    if (pght >= 3) d2h(hesstarg, d_ht, (size_t)nt * nd * nhess);
  }
  FGT_CUDA(cudaStreamSynchronize(s));
  raise_failed_checks(s);
  return FGT_OK;
}

}  // namespace
}  // namespace fgt

extern "C" {

void fgt_opts_default(fgt_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->precision = FGT_PREC_AUTO;
  o->device_ptrs = 0;
  o->device = -1;
  o->stream = nullptr;
  o->ndiv = 0;
  o->small_eval = -1;
  o->spread_width = 0;
  o->timing = 0;
  o->stats = nullptr;
  o->root_level = -1;
  o->autotune = 0;
}

int fgt_pfgt_c(const fgt_opts* opts, int nd, int dim, double delta, double eps, int iperiod,
               double* bs0, double* cen0, int ns, const double* sources, int ifcharge,
               const double* charge, int ifdipole, const double* rnormal, const double* dipstr,
               int ifpgh, double* pot, double* grad, double* hess, int nt, const double* targ,
               int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg) {
  int st;
  try {
    st = fgt::pfgt_impl(opts, nd, dim, delta, eps, iperiod, bs0, cen0, ns, sources, ifcharge,
                        charge, ifdipole, rnormal, dipstr, ifpgh, pot, grad, hess, nt, targ,
                        ifpghtarg, pottarg, gradtarg, hesstarg);
  } catch (const fgt::Error& e) {
    st = e.code;
  } catch (...) {
    fgt_set_error_message("unexpected host exception", __FILE__, __LINE__);
    st = FGT_ERR_CUDA;
  }
  g_last_status = st;
  return st;
}

void pfgt_(const int* nd, const int* dim, const double* delta, const double* eps,
           const int* iperiod, double* bs0, double* cen0, const int* ns, const double* sources,
           const int* ifcharge, const double* charge, const int* ifdipole, const double* rnormal,
           const double* dipstr, const int* ifpgh, double* pot, double* grad, double* hess,
           const int* nt, const double* targ, const int* ifpghtarg, double* pottarg,
           double* gradtarg, double* hesstarg) {
  int st = fgt_pfgt_c(nullptr, *nd, *dim, *delta, *eps, *iperiod, bs0, cen0, *ns, sources,
                      *ifcharge, charge, *ifdipole, rnormal, dipstr, *ifpgh, pot, grad, hess, *nt,
                      targ, *ifpghtarg, pottarg, gradtarg, hesstarg);
  if (st != FGT_OK) {
    // The Fortran interface has no status argument: poison the requested
    // outputs so a failed call cannot pass for a result.
    double nan = NAN;
    int n = *nd, d = *dim, nh = d * (d + 1) / 2;
    auto fill = [&](double* a, long long cnt) {
      if (a && cnt > 0)
        for (long long i = 0; i < cnt; i++) a[i] = nan;
    };
    if (*ifpgh >= 1) fill(pot, (long long)*ns * n);
    if (*ifpgh >= 2) fill(grad, (long long)*ns * n * d);
    if (*ifpgh >= 3) fill(hess, (long long)*ns * n * nh);
    if (*ifpghtarg >= 1) fill(pottarg, (long long)*nt * n);
    if (*ifpghtarg >= 2) fill(gradtarg, (long long)*nt * n * d);
    if (*ifpghtarg >= 3) fill(hesstarg, (long long)*nt * n * nh);
  }
}

fgt_plan* fgt_plan_create(const fgt_opts* opts, int nd, int dim, double delta, double eps,
                          int iperiod, double* bs0, double* cen0, int ns, const double* sources,
                          int nt, const double* targ, int* status) {
  fgt_plan* pl = nullptr;
  int st = FGT_OK;
  try {
    pl = fgt::plan_create_impl(opts, nd, dim, delta, eps, iperiod, bs0, cen0, ns, sources, nt,
                               targ);
  } catch (const fgt::Error& e) {
    st = e.code;
  } catch (...) {
    fgt_set_error_message("unexpected host exception", __FILE__, __LINE__);
    st = FGT_ERR_CUDA;
  }
  g_last_status = st;
  if (status) *status = st;
  return pl;
}

int fgt_plan_execute(fgt_plan* plan, int ifcharge, const double* charge, int ifdipole,
                     const double* rnormal, const double* dipstr, int ifpgh, double* pot,
                     double* grad, double* hess, int ifpghtarg, double* pottarg,
                     double* gradtarg, double* hesstarg) {
  int st;
  try {
    st = fgt::plan_execute_impl(plan, ifcharge, charge, ifdipole, rnormal, dipstr, ifpgh, pot,
                                grad, hess, ifpghtarg, pottarg, gradtarg, hesstarg);
  } catch (const fgt::Error& e) {
    st = e.code;
  } catch (...) {
    fgt_set_error_message("unexpected host exception", __FILE__, __LINE__);
    st = FGT_ERR_CUDA;
  }
  g_last_status = st;
  return st;
}

void fgt_plan_destroy(fgt_plan* plan) {
  if (!plan) return;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(plan->device);
  if (plan->arena) {
    plan->arena->release_all();  // cudaFree waits for the device work using it
    delete plan->arena;
  }
  delete plan;
  cudaSetDevice(cur);
}

int fgt_last_status(void) { return g_last_status; }

const char* fgt_last_error(void) { return g_last_error.c_str(); }

const char* fgt_version(void) { return "fgt_b200 0.1 (sm_100a)"; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Introspection of the device tree and lists (test support).
namespace {
struct DebugTree {
  fgt::TreeHost th;
  fgt::ListsHost lh;
  std::vector<int> scalars;  // nlevels, nboxes, npwlevel, ncutoff, nleaves, n_form, n_eval, n_trans, n_l1, D
  std::vector<double> dscal; // bs0, cen0[3], boxsize...
};
}  // namespace

extern "C" void* fgt_debug_tree_build(int dim, double delta, double eps, int iperiod, double bs0_in,
                                      const double* cen0_in, int ns, const double* src, int nt,
                                      const double* trg, int ndiv_override) {
  using namespace fgt;
  try {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      (void)cudaGetLastError();
      return nullptr;
    }
    int dev;
    FGT_CUDA(cudaGetDevice(&dev));
    configure_pool(dev);
    cudaStream_t s = library_stream(dev);
    ArenaScope arena_scope(s);
    DBuf<double> dsrc((size_t)ns * dim, s), dtrg((size_t)std::max(nt, 1) * dim, s);
    FGT_CUDA(cudaMemcpyAsync(dsrc.get(), src, sizeof(double) * ns * dim, cudaMemcpyHostToDevice, s));
    if (nt > 0)
      FGT_CUDA(cudaMemcpyAsync(dtrg.get(), trg, sizeof(double) * nt * dim, cudaMemcpyHostToDevice, s));
    int npwlevel = 0;
    double bs0 = bs0_in, cen0[3] = {0, 0, 0};
    for (int k = 0; k < dim; k++) cen0[k] = cen0_in ? cen0_in[k] : 0.0;
    tree_setup_scalars(dim, delta, eps, iperiod, dsrc, ns, nt > 0 ? dtrg.get() : dsrc.get(),
                       nt > 0 ? nt : 0, &npwlevel, &bs0, cen0, s);
    int ndiv = ndiv_override > 0 ? ndiv_override : (dim == 1 ? 20 : (dim == 2 ? 80 : 250));
    Tree t;
    tree_build(t, dim, iperiod, npwlevel, ndiv, bs0, cen0, dsrc, ns, dtrg, nt, s);
    int iperiod0 = (npwlevel <= 1 && iperiod == 1) ? 0 : iperiod;
    int nlevend = t.nlevels;
    if (npwlevel <= t.nlevels) nlevend = npwlevel;
    bool do_pw = npwlevel < t.nlevels;
    if (npwlevel < 0 && ns <= ndiv) {
      do_pw = false;
      nlevend = 0;
    }
    Lists L;
    build_lists(t, npwlevel, iperiod0, nlevend, do_pw, L, s);
    DebugTree* d = new DebugTree();
    tree_download(t, d->th, s);
    lists_download(L, t.nboxes, d->lh, s);
    d->scalars = {t.nlevels, t.nboxes, npwlevel, t.ncutoff, t.nleaves, L.n_form, L.n_eval,
                  L.n_trans, L.n_l1, t.D, nlevend, iperiod0};
    d->dscal = {bs0, cen0[0], cen0[1], cen0[2]};
    for (double b : t.boxsize) d->dscal.push_back(b);
    return d;
  } catch (const fgt::Error&) {
    return nullptr;
  }
}

extern "C" long fgt_debug_tree_get(void* h, const char* name, void* dst, long cap) {
  if (!h || !name) return -1;
  DebugTree* d = (DebugTree*)h;
  auto put = [&](const auto& v) -> long {
    long n = (long)v.size();
    if (dst) memcpy(dst, v.data(), sizeof(v[0]) * (size_t)std::min(n, cap));
    return n;
  };
  std::string s(name);
  if (s == "scalars") return put(d->scalars);
  if (s == "dscalars") return put(d->dscal);
  if (s == "key") return put(d->th.key);
  if (s == "level") return put(d->th.level);
  if (s == "nonleaf") return put(d->th.nonleaf);
  if (s == "parent") return put(d->th.parent);
  if (s == "child0") return put(d->th.child0);
  if (s == "center") return put(d->th.center);
  if (s == "src_lo") return put(d->th.src_lo);
  if (s == "src_hi") return put(d->th.src_hi);
  if (s == "trg_lo") return put(d->th.trg_lo);
  if (s == "trg_hi") return put(d->th.trg_hi);
  if (s == "isrc") return put(d->th.isrc);
  if (s == "itrg") return put(d->th.itrg);
  if (s == "l1_ptr") return put(d->lh.l1_ptr);
  if (s == "l1_src") return put(d->lh.l1_src);
  if (s == "form_box") return put(d->lh.form_box);
  if (s == "eval_box") return put(d->lh.eval_box);
  if (s == "eval_self") return put(d->lh.eval_self);
  if (s == "trans_ptr") return put(d->lh.trans_ptr);
  if (s == "trans_src") return put(d->lh.trans_src);
  if (s == "trans_w") return put(d->lh.trans_w);
  return -1;
}

extern "C" void fgt_debug_tree_free(void* h) { delete (DebugTree*)h; }

// ---------------------------------------------------------------------------
// pfgt_direct drop-in (src/pfgt/pfgt.f:1156-1382), FP64 on the GPU.
extern "C" void pfgt_direct_(const int* nd, const int* dim, const double* delta, const double* dmax,
                             const int* iperiod, const double* shifts, const int* istart,
                             const int* iend, const int* jstart, const int* jend,
                             const double* source, const int* ifcharge, const double* charge,
                             const int* ifdipole, const double* rnormal, const double* dipstr,
                             const double* targ, const int* ifpgh, double* pot, double* grad,
                             double* hess) {
  using namespace fgt;
  int st = FGT_OK;
  try {
    const int n = *nd, d = *dim, pgh = *ifpgh, nh = d * (d + 1) / 2;
    const int is = *istart - 1, ns = *iend - *istart + 1, js = *jstart - 1, nt = *jend - *jstart + 1;
    FGT_REQUIRE(d >= 1 && d <= 3 && n >= 1, FGT_ERR_ARG, "bad nd/dim");
    if (ns > 0 && nt > 0 && pgh >= 1) {
      if (fault_requested("launch") || fault_requested("alloc") || fault_requested("queue"))
        throw Error{FGT_ERR_INJECTED, "fault injected"};
      int ndev = 0;
      if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        (void)cudaGetLastError();
        throw Error{FGT_ERR_NODEVICE, "no CUDA device"};
      }
      int dev;
      FGT_CUDA(cudaGetDevice(&dev));
      configure_pool(dev);
      cudaStream_t s = library_stream(dev);
      ArenaScope arena_scope(s);
      auto up = [&](DBuf<double>& b, const double* h, size_t cnt) {
        b.alloc(cnt, s);
        FGT_CUDA(cudaMemcpyAsync(b.get(), h, sizeof(double) * cnt, cudaMemcpyHostToDevice, s));
        return b.get();
      };
      DBuf<double> bs, bq, brn, bds, bt, bp, bg, bh, bsh;
      const double* ds_ = up(bs, source + (size_t)is * d, (size_t)ns * d);
      const double* dq = *ifcharge == 1 ? up(bq, charge + (size_t)is * n, (size_t)ns * n) : nullptr;
      const double* drn = *ifdipole == 1 ? up(brn, rnormal + (size_t)is * d, (size_t)ns * d) : nullptr;
      const double* dds = *ifdipole == 1 ? up(bds, dipstr + (size_t)is * n, (size_t)ns * n) : nullptr;
      const double* dt = up(bt, targ + (size_t)js * d, (size_t)nt * d);
      const double* dsh = *iperiod == 1 ? up(bsh, shifts, d) : nullptr;
      double* dp = up(bp, pot + (size_t)js * n, (size_t)nt * n) == nullptr ? nullptr : bp.get();
      double* dg = pgh >= 2 ? (up(bg, grad + (size_t)js * n * d, (size_t)nt * n * d), bg.get()) : nullptr;
      double* dh = pgh >= 3 ? (up(bh, hess + (size_t)js * n * nh, (size_t)nt * n * nh), bh.get()) : nullptr;
      direct_all_pairs(n, d, *delta, *dmax, dsh, ns, ds_, dq, drn, dds, nt, dt, pgh, dp, dg, dh, s);
      FGT_CUDA(cudaMemcpyAsync(pot + (size_t)js * n, dp, sizeof(double) * nt * n, cudaMemcpyDeviceToHost, s));
      if (dg) FGT_CUDA(cudaMemcpyAsync(grad + (size_t)js * n * d, dg, sizeof(double) * nt * n * d, cudaMemcpyDeviceToHost, s));
      if (dh) FGT_CUDA(cudaMemcpyAsync(hess + (size_t)js * n * nh, dh, sizeof(double) * nt * n * nh, cudaMemcpyDeviceToHost, s));
      FGT_CUDA(cudaStreamSynchronize(s));
      raise_failed_checks(s);
    }
  } catch (const fgt::Error& e) {
    st = e.code;
  }
  g_last_status = st;
}

// ---------------------------------------------------------------------------
// Self-test of the FGT_CHECK build: the strength gather with a host-crafted
// permutation whose third entry points past the array.  The checked kernel
// records the failure and skips that element; the call then reports
// FGT_ERR_CHECK.  The normal build has no checks: FGT_ERR_UNSUPPORTED.
extern "C" int fgt_check_selftest(void) {
  using namespace fgt;
  int st = FGT_OK;
  try {
#ifndef FGT_CHECK
    FGT_REQUIRE(false, FGT_ERR_UNSUPPORTED, "library built without FGT_CHECK");
#else
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      (void)cudaGetLastError();
      throw Error{FGT_ERR_NODEVICE, "no CUDA device"};
    }
    int dev = 0;
    FGT_CUDA(cudaGetDevice(&dev));
    cudaStream_t s = library_stream(dev);
    ArenaScope arena_scope(s);
    const int n = 4;
    const uint32_t hperm[n] = {0, 1, n + 5, 2};  // entry 2 is out of range
    const double hv[n] = {1, 2, 3, 4};
    DBuf<uint32_t> perm(n, s);
    DBuf<double> v(n, s), out(n, s);
    FGT_CUDA(cudaMemcpyAsync(perm.get(), hperm, sizeof(hperm), cudaMemcpyHostToDevice, s));
    FGT_CUDA(cudaMemcpyAsync(v.get(), hv, sizeof(hv), cudaMemcpyHostToDevice, s));
    k_gather_vals<double><<<1, 32, 0, s>>>(v, n, 1, perm, out);
    FGT_LAUNCH_CHECK();
    FGT_CUDA(cudaStreamSynchronize(s));
    raise_failed_checks(s);
#endif
  } catch (const fgt::Error& e) {
    st = e.code;
  }
  g_last_status = st;
  return st;
}
