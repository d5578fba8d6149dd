// Device tree build: bounding box, path keys, level-synchronous refinement,
// 2:1 level restriction, box tables, sorted point ranges.
#include <math.h>

#include <algorithm>

#include "fgt_tree.cuh"

namespace fgt {

namespace {

struct KeyParams {
  int dim, D;
  double cen0[FGT_MAXDIM];
  double bsh[64];  // bsh[l] = boxsize(l+1)/2: child-centre offset below level l
};

template <int DIM>
__global__ void k_bbox(const double* __restrict__ x, int n, double* __restrict__ part) {
  double lo[DIM], hi[DIM];
#pragma unroll
  for (int k = 0; k < DIM; k++) { lo[k] = INFINITY; hi[k] = -INFINITY; }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
#pragma unroll
    for (int k = 0; k < DIM; k++) {
      double v = x[(size_t)i * DIM + k];
      lo[k] = fmin(lo[k], v);
      hi[k] = fmax(hi[k], v);
    }
  __shared__ double slo[DIM][32], shi[DIM][32];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < DIM; k++) {
    double a = lo[k], b = hi[k];
    for (int o = 16; o; o >>= 1) {
      a = fmin(a, __shfl_xor_sync(0xffffffffu, a, o));
      b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    if (lane == 0) { slo[k][w] = a; shi[k][w] = b; }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < DIM; k++) {
      double a = INFINITY, b = -INFINITY;
      for (int j = 0; j < (int)(blockDim.x >> 5); j++) { a = fmin(a, slo[k][j]); b = fmax(b, shi[k][j]); }
      part[(size_t)blockIdx.x * 2 * DIM + k] = a;
      part[(size_t)blockIdx.x * 2 * DIM + DIM + k] = b;
    }
  }
}

// Full path key of every point (D levels).  The centre recursion
// c_child = c_parent + sign*boxsize(l+1)/2 and the test x - c >= 0 are those
// of tree_refine_boxes (src/common/tree_routs_nd.f:42-45) and
// find_childbox_ind (src/common/pts_tree_nd.f:733-737), so box membership is
// bit-identical to the reference.
template <int DIM>
__global__ void k_point_keys(const double* __restrict__ x, int n, KeyParams p,
                             uint64_t* __restrict__ keys) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double c[DIM], xi[DIM];
#pragma unroll
    for (int k = 0; k < DIM; k++) { c[k] = p.cen0[k]; xi[k] = x[(size_t)i * DIM + k]; }
    uint64_t key = 0;
    for (int l = 0; l < p.D; l++) {
      int dig = 0;
      const double h = p.bsh[l];
#pragma unroll
      for (int k = 0; k < DIM; k++) {
        bool up = (xi[k] - c[k] >= 0);
        dig |= (up ? 1 : 0) << k;
        c[k] = c[k] + (up ? h : -h);
      }
      key = (key << DIM) | (uint64_t)dig;
    }
    keys[i] = key;
  }
}
void launch_point_keys(int dim, const double* x, int n, const KeyParams& p, uint64_t* keys,
                       cudaStream_t s) {
  if (dim == 1) k_point_keys<1><<<grid_for(n, 256), 256, 0, s>>>(x, n, p, keys);
  else if (dim == 2) k_point_keys<2><<<grid_for(n, 256), 256, 0, s>>>(x, n, p, keys);
  else k_point_keys<3><<<grid_for(n, 256), 256, 0, s>>>(x, n, p, keys);
  FGT_LAUNCH_CHECK();
}
void launch_bbox(int dim, const double* x, int n, int gb, double* part, cudaStream_t s) {
  if (dim == 1) k_bbox<1><<<gb, 256, 0, s>>>(x, n, part);
  else if (dim == 2) k_bbox<2><<<gb, 256, 0, s>>>(x, n, part);
  else k_bbox<3><<<gb, 256, 0, s>>>(x, n, part);
  FGT_LAUNCH_CHECK();
}

// Source count of each box of level l from the sorted full keys.
__global__ void k_box_counts(const uint64_t* __restrict__ bk, int nb, int shift,
                             const uint64_t* __restrict__ sk, int ns, int* __restrict__ cnt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
    uint64_t lo = bk[i] << shift, hi = (bk[i] + 1) << shift;
    cnt[i] = dev_lower_bound(sk, ns, hi) - dev_lower_bound(sk, ns, lo);
  }
}

// Source count of each box of level l from the exclusive prefix sums S of
// the per-cell source counts of the full key space (2^(dim*D) cells):
// count = S[(key+1) << shift] - S[key << shift].
__global__ void k_box_counts_dense(const uint64_t* __restrict__ bk, int nb, int shift,
                                   const int* __restrict__ S, int* __restrict__ cnt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
    cnt[i] = S[(bk[i] + 1) << shift] - S[bk[i] << shift];
}

// Per-cell source counts of the full key space; lanes of a warp that hit
// the same cell add once (points arrive in input order, often clustered).
__global__ void k_cell_hist(const uint64_t* __restrict__ keys, int n, int* __restrict__ h) {
  for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
    const int i = i0 + threadIdx.x;
    const unsigned long long k = i < n ? keys[i] : ~0ull;
    const unsigned peers = __match_any_sync(0xffffffffu, k);
    if (i < n && (__ffs(peers) - 1) == (int)(threadIdx.x & 31)) atomicAdd(&h[k], __popc(peers));
  }
}

__global__ void k_flag_gt(const int* __restrict__ cnt, int n, int ndiv, int* __restrict__ f) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    f[i] = cnt[i] > ndiv ? 1 : 0;
}

__global__ void k_compact_u64(const uint64_t* __restrict__ in, const int* __restrict__ flag,
                              const int* __restrict__ pos, int n, uint64_t* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (flag[i]) out[pos[i]] = in[i];
}

__global__ void k_children(const uint64_t* __restrict__ par, int n, int dim,
                           uint64_t* __restrict__ out) {
  int mc = 1 << dim;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n * mc; i += gridDim.x * blockDim.x)
    out[i] = (par[i / mc] << dim) | (uint64_t)(i % mc);
}

__device__ __forceinline__ void key_to_coords(uint64_t key, int l, int dim, uint32_t* c) {
  for (int k = 0; k < dim; k++) c[k] = 0;
  for (int j = 0; j < l; j++) {
    int dig = (int)((key >> (dim * (l - 1 - j))) & ((1u << dim) - 1));
    for (int k = 0; k < dim; k++) c[k] = (c[k] << 1) | ((dig >> k) & 1);
  }
}
__device__ __forceinline__ uint64_t coords_to_key(const uint32_t* c, int l, int dim) {
  uint64_t key = 0;
  for (int j = 0; j < l; j++) {
    int dig = 0;
    for (int k = 0; k < dim; k++) dig |= ((c[k] >> (l - 1 - j)) & 1) << k;
    key = (key << dim) | (uint64_t)dig;
  }
  return key;
}

// Level restriction: every level-(l-1) position whose closure touches a
// non-leaf level-l box must itself be non-leaf (free-space adjacency, as the
// distance tests of pts_tree_fix_lr, src/common/pts_tree_nd.f:783-1035).
// Emits, per non-leaf box, the 2^dim touching level-(l-1) positions (out of
// range positions are replaced by the parent, removed later as duplicates).
__global__ void k_touching_parents(const uint64_t* __restrict__ nl, int n, int l, int dim,
                                   uint64_t* __restrict__ out) {
  int mc = 1 << dim;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n * mc; i += gridDim.x * blockDim.x) {
    int b = i / mc, j = i % mc;
    uint32_t c[FGT_MAXDIM], q[FGT_MAXDIM];
    key_to_coords(nl[b], l, dim, c);
    uint32_t lim = 1u << (l - 1);
    for (int k = 0; k < dim; k++) {
      uint32_t m = c[k] >> 1;
      if ((j >> k) & 1) {
        // the other touching position: m-1 if c even, m+1 if c odd
        long long o = (c[k] & 1) ? (long long)m + 1 : (long long)m - 1;
        q[k] = (o >= 0 && o < (long long)lim) ? (uint32_t)o : m;
      } else {
        q[k] = m;
      }
    }
    out[i] = coords_to_key(q, l - 1, dim);
  }
}

__global__ void k_member(const uint64_t* __restrict__ a, int n, const uint64_t* __restrict__ set,
                         int m, int* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = dev_find(set, m, a[i]) >= 0 ? 1 : 0;
}

struct LevelTables {
  const uint64_t* keys[64];
  int n[64];
  int start[65];
};

__global__ void k_box_tables(int nboxes, int nlevels, int dim, LevelTables lt, KeyParams kp,
                             const uint64_t* __restrict__ key, const int* __restrict__ level,
                             const int* __restrict__ nonleaf, int* __restrict__ parent,
                             int* __restrict__ child0, double* __restrict__ center) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nboxes; b += gridDim.x * blockDim.x) {
    int l = level[b];
    uint64_t k = key[b];
    parent[b] = (l == 0) ? -1 : lt.start[l - 1] + dev_find(lt.keys[l - 1], lt.n[l - 1], k >> dim);
    child0[b] = (nonleaf[b] && l < nlevels)
                    ? lt.start[l + 1] + dev_find(lt.keys[l + 1], lt.n[l + 1], k << dim)
                    : -1;
    double c[FGT_MAXDIM];
    for (int d = 0; d < dim; d++) c[d] = kp.cen0[d];
    for (int j = 0; j < l; j++) {
      int dig = (int)((k >> (dim * (l - 1 - j))) & ((1u << dim) - 1));
      for (int d = 0; d < dim; d++) c[d] = c[d] + (((dig >> d) & 1) ? kp.bsh[j] : -kp.bsh[j]);
    }
    for (int d = 0; d < dim; d++) center[(size_t)b * dim + d] = c[d];
  }
}

__global__ void k_leaf_flags(const int* __restrict__ nonleaf, int n, int* __restrict__ f) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    f[i] = nonleaf[i] ? 0 : 1;
}
__global__ void k_leaf_starts(const uint64_t* __restrict__ key, const int* __restrict__ level,
                              const int* __restrict__ f, const int* __restrict__ pos, int n,
                              int dim, int D, uint64_t* __restrict__ ls,
                              uint32_t* __restrict__ lbox) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (f[i]) {
      ls[pos[i]] = key[i] << (dim * (D - level[i]));
      lbox[pos[i]] = (uint32_t)i;
    }
}

// Reference box of every leaf (by leaf ordinal): the leaf itself when it
// lies at or above the cut-off level, else its ancestor at that level.
__global__ void k_leaf_ref(const uint32_t* __restrict__ lbox, int nl, const int* __restrict__ level,
                           const int* __restrict__ parent, int ncutoff, int* __restrict__ lref) {
  for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < nl; o += gridDim.x * blockDim.x) {
    int b = (int)lbox[o];
    while (level[b] > ncutoff && FGT_DCHECK(parent[b] >= 0, 502)) b = parent[b];
    lref[o] = b;
  }
}
// ref[p] = lref[ordinal of sorted point p]
__global__ void k_point_ref(const uint32_t* __restrict__ ord, int n, const int* __restrict__ lref,
                            int* __restrict__ ref) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    ref[i] = lref[ord[i]];
}

// Leaf ordinal of each point (upper_bound - 1 over sorted leaf start keys);
// doubles as the radix key, the value is the original index.
__global__ void k_point_leaf(const uint64_t* __restrict__ pk, int n,
                             const uint64_t* __restrict__ ls, int nl,
                             uint32_t* __restrict__ ord, uint32_t* __restrict__ idx) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint64_t v = pk[i];
    int lo = 0, hi = nl;  // first start > v
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (ls[mid] <= v) lo = mid + 1; else hi = mid;
    }
    if (!FGT_DCHECK(lo >= 1, 501)) lo = 1;  // every key lies at or after the first leaf
    ord[i] = (uint32_t)(lo - 1);
    idx[i] = (uint32_t)i;
  }
}

// Dense leaf table of the finest cells (small key spaces): the leaves'
// start keys, sorted, cut the 2^(dim*D) cells into the leaves' ranges;
// table[c] = ordinal of the leaf whose range holds cell c.
__global__ void k_cell_leaf(const uint64_t* __restrict__ ls, int nl, long long ncell,
                            uint32_t* __restrict__ table) {
  for (int o = blockIdx.x; o < nl; o += gridDim.x) {
    const long long c0 = (long long)ls[o], c1 = o + 1 < nl ? (long long)ls[o + 1] : ncell;
    for (long long c = c0 + threadIdx.x; c < c1; c += blockDim.x) table[c] = (uint32_t)o;
  }
}
// Leaf ordinal of each point by the dense table (value: the original index).
__global__ void k_point_leaf_dense(const uint64_t* __restrict__ pk, int n,
                                   const uint32_t* __restrict__ table, uint32_t* __restrict__ ord,
                                   uint32_t* __restrict__ idx) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    ord[i] = table[pk[i]];
    idx[i] = (uint32_t)i;
  }
}

// leaf_lo[o] = first sorted position with ordinal >= o, o = 0..nl
__global__ void k_leaf_point_lo(const uint32_t* __restrict__ ord, int n, int nl,
                                int* __restrict__ lo) {
  for (int o = blockIdx.x * blockDim.x + threadIdx.x; o <= nl; o += gridDim.x * blockDim.x) {
    int a = 0, b = n;
    while (a < b) {
      int m = (a + b) >> 1;
      if (ord[m] < (uint32_t)o) a = m + 1; else b = m;
    }
    lo[o] = a;
  }
}

__global__ void k_box_ranges(const uint64_t* __restrict__ key, const int* __restrict__ level,
                             int nboxes, int dim, int D, const uint64_t* __restrict__ ls, int nl,
                             const int* __restrict__ slo, const int* __restrict__ tlo,
                             int* __restrict__ s0, int* __restrict__ s1, int* __restrict__ t0,
                             int* __restrict__ t1) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nboxes; b += gridDim.x * blockDim.x) {
    int sh = dim * (D - level[b]);
    uint64_t lo = key[b] << sh, hi = (key[b] + 1) << sh;
    int a = dev_lower_bound(ls, nl, lo), c = dev_lower_bound(ls, nl, hi);
    s0[b] = slo[a]; s1[b] = slo[c];
    t0[b] = tlo[a]; t1[b] = tlo[c];
  }
}

int bits_for(long long n) {
  int b = 0;
  while ((1ll << b) < n) b++;
  return b;
}

}  // namespace

void tree_setup_scalars(int dim, double delta, double eps, int iperiod, const double* d_src,
                        int ns, const double* d_trg, int nt, int* levcut, double* bs0,
                        double* cen0, cudaStream_t s) {
  if (iperiod != 1) {
    int gb = 4 * kSMs;
    DBuf<double> part((size_t)2 * gb * 2 * dim, s);
    launch_bbox(dim, d_src, ns, gb, part.get(), s);
    launch_bbox(dim, d_trg, nt, gb, part.get() + (size_t)gb * 2 * dim, s);
    std::vector<double> h((size_t)2 * gb * 2 * dim);
    FGT_CUDA(cudaMemcpyAsync(h.data(), part.get(), sizeof(double) * h.size(),
                             cudaMemcpyDeviceToHost, s));
    FGT_CUDA(cudaStreamSynchronize(s));
    double lo[FGT_MAXDIM], hi[FGT_MAXDIM];
    for (int k = 0; k < dim; k++) { lo[k] = INFINITY; hi[k] = -INFINITY; }
    for (int b = 0; b < 2 * gb; b++)
      for (int k = 0; k < dim; k++) {
        lo[k] = std::min(lo[k], h[(size_t)b * 2 * dim + k]);
        hi[k] = std::max(hi[k], h[(size_t)b * 2 * dim + dim + k]);
      }
    // pts_tree_nd.f:1390-1398
    *bs0 = hi[0] - lo[0];
    for (int k = 1; k < dim; k++)
      if (hi[k] - lo[k] > *bs0) *bs0 = hi[k] - lo[k];
    for (int k = 0; k < dim; k++) cen0[k] = (lo[k] + hi[k]) / 2;
  }
  // pts_tree_nd.f:1399-1410
  double dc = sqrt(delta * log(1.0 / eps));
  double dl = log(*bs0 / dc) / log(2.0);
  *levcut = (int)dl;
  if (iperiod == 1) return;
  if (*bs0 < dc) return;
  *levcut = *levcut + 1;
  *bs0 = ldexp(1.0, *levcut) * dc;
}

namespace {
__global__ void k_fill_int(int* __restrict__ a, int n, int v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = v;
}
}  // namespace

void tree_build(Tree& t, int dim, int iperiod, int npwlevel, int ndiv, double bs0,
                const double* cen0, const double* d_src, int ns, const double* d_trg, int nt,
                cudaStream_t s) {
  t.dim = dim;
  t.mc = 1 << dim;
  t.iperiod = iperiod;
  t.npwlevel = npwlevel;
  t.ncutoff = npwlevel > 0 ? npwlevel : 0;
  t.ndiv = ndiv;
  t.ns = ns;
  t.nt = nt;
  t.bs0 = bs0;
  for (int k = 0; k < dim; k++) t.cen0[k] = cen0[k];
  int D = npwlevel >= 0 ? npwlevel + 1 : 0;  // nlmax of pfgt.f:136-140
  FGT_REQUIRE(D * dim <= 63 && D < 63, FGT_ERR_UNSUPPORTED,
              "tree depth exceeds the 63-bit path key (delta too small for the data extent)");
  t.D = D;
  KeyParams kp;
  kp.dim = dim;
  kp.D = D;
  for (int k = 0; k < FGT_MAXDIM; k++) kp.cen0[k] = k < dim ? cen0[k] : 0.0;
  {
    double bs = bs0;
    for (int l = 0; l < 64; l++) {
      double bsc = bs / 2;  // boxsize(l+1)
      kp.bsh[l] = bsc / 2;
      bs = bsc;
    }
  }
  // 1. full keys of sources and targets
  DBuf<uint64_t> skey(ns, s), tkey(nt, s), ksorted, ktmp(std::max(ns, nt), s);
  if (ns > 0) launch_point_keys(dim, d_src, ns, kp, skey, s);
  if (nt > 0) launch_point_keys(dim, d_trg, nt, kp, tkey, s);
  // Source counts per box come from a dense histogram of the full keys
  // (prefix sums over the 2^(dim*D) finest cells) when the key space is
  // small, and not much larger than the point set (clearing and scanning
  // 2^24 cells costs ~0.3 ms, far more than sorting a few thousand keys),
  // else from binary searches in the sorted keys.
  const bool dense =
      dim * D <= 24 && (1ll << (dim * D)) <= 4ll * ((long long)ns + nt) + (1ll << 18);
  DBuf<int> cellsum;
  if (dense) {
    const int ncell = 1 << (dim * D);
    cellsum.alloc((size_t)ncell + 1, s);
    cellsum.zero();
    if (ns > 0) {
      k_cell_hist<<<grid_for(ns, 256), 256, 0, s>>>(skey, ns, cellsum);
      FGT_LAUNCH_CHECK();
    }
    exclusive_scan_i32(cellsum, cellsum, ncell + 1, nullptr, s);
  } else {
    ksorted.alloc(std::max(ns, 1), s);
    if (ns > 0)
      FGT_CUDA(cudaMemcpyAsync(ksorted.get(), skey.get(), sizeof(uint64_t) * ns,
                               cudaMemcpyDeviceToDevice, s));
    radix_sort(ksorted, nullptr, ktmp, nullptr, ns, dim * D, s);
  }

  // 2. refinement on source counts (pts_tree_build, pts_tree_nd.f:520-590)
  std::vector<DBuf<uint64_t>> lk;   // keys of each level
  std::vector<DBuf<uint64_t>> NL;   // non-leaf keys of each level
  std::vector<int> nlk, nnl;
  lk.emplace_back(1, s);
  FGT_CUDA(cudaMemsetAsync(lk[0].get(), 0, sizeof(uint64_t), s));
  nlk.push_back(1);
  int nlevels = 0;
  for (int l = 0; l < D; l++) {
    int nb = nlk[l];
    DBuf<int> cnt(nb, s), flag(nb, s), pos(nb, s), tot(1, s);
    if (dense)
      k_box_counts_dense<<<grid_for(nb, 256), 256, 0, s>>>(lk[l], nb, dim * (D - l), cellsum, cnt);
    else
      k_box_counts<<<grid_for(nb, 256), 256, 0, s>>>(lk[l], nb, dim * (D - l), ksorted, ns, cnt);
    FGT_LAUNCH_CHECK();
    k_flag_gt<<<grid_for(nb, 256), 256, 0, s>>>(cnt, nb, ndiv, flag);
    FGT_LAUNCH_CHECK();
    exclusive_scan_i32(flag, pos, nb, tot, s);
    int nref = fetch_int(tot, s);
    if (nref == 0) break;
    NL.emplace_back(nref, s);
    nnl.push_back(nref);
    k_compact_u64<<<grid_for(nb, 256), 256, 0, s>>>(lk[l], flag, pos, nb, NL[l]);
    FGT_LAUNCH_CHECK();
    lk.emplace_back((size_t)nref * t.mc, s);
    nlk.push_back(nref * t.mc);
    k_children<<<grid_for((long long)nref * t.mc, 256), 256, 0, s>>>(NL[l], nref, dim, lk[l + 1]);
    FGT_LAUNCH_CHECK();
    nlevels = l + 1;
  }
  t.nlevels = nlevels;

  // 3. level restriction (minimal 2:1 balanced refinement)
  for (int l = nlevels - 1; l >= 2; l--) {
    int n = nnl[l], m = nnl[l - 1];
    int tot = n * t.mc + m;
    DBuf<uint64_t> cand(tot, s), ctmp(tot, s);
    k_touching_parents<<<grid_for((long long)n * t.mc, 256), 256, 0, s>>>(NL[l], n, l, dim, cand);
    FGT_LAUNCH_CHECK();
    FGT_CUDA(cudaMemcpyAsync(cand.get() + (size_t)n * t.mc, NL[l - 1].get(),
                             sizeof(uint64_t) * m, cudaMemcpyDeviceToDevice, s));
    radix_sort(cand, nullptr, ctmp, nullptr, tot, dim * (l - 1), s);
    DBuf<uint64_t> uniq(tot, s);
    int nu = unique_sorted_u64(cand, tot, uniq, s);
    NL[l - 1] = std::move(uniq);
    nnl[l - 1] = nu;
  }
  // final level key arrays: children of the (updated) non-leaf sets
  for (int l = 1; l <= nlevels; l++) {
    int n = nnl[l - 1];
    lk[l].alloc((size_t)n * t.mc, s);
    nlk[l] = n * t.mc;
    k_children<<<grid_for((long long)n * t.mc, 256), 256, 0, s>>>(NL[l - 1], n, dim, lk[l]);
    FGT_LAUNCH_CHECK();
  }

  // 4. global box tables
  t.lev_start.assign(nlevels + 2, 0);
  for (int l = 0; l <= nlevels; l++) t.lev_start[l + 1] = t.lev_start[l] + nlk[l];
  int nboxes = t.lev_start[nlevels + 1];
  t.nboxes = nboxes;
  t.boxsize.resize(nlevels + 1);
  t.boxsize[0] = bs0;
  for (int l = 1; l <= nlevels; l++) t.boxsize[l] = t.boxsize[l - 1] / 2;
  t.key.alloc(nboxes, s);
  t.level.alloc(nboxes, s);
  t.nonleaf.alloc(nboxes, s);
  t.parent.alloc(nboxes, s);
  t.child0.alloc(nboxes, s);
  t.center.alloc((size_t)nboxes * dim, s);
  for (int l = 0; l <= nlevels; l++) {
    const int n = t.lev_start[l + 1] - t.lev_start[l];
    if (n > 0) {
      k_fill_int<<<grid_for(n, 256), 256, 0, s>>>(t.level.get() + t.lev_start[l], n, l);
      FGT_LAUNCH_CHECK();
    }
  }
  for (int l = 0; l <= nlevels; l++) {
    FGT_CUDA(cudaMemcpyAsync(t.key.get() + t.lev_start[l], lk[l].get(),
                             sizeof(uint64_t) * nlk[l], cudaMemcpyDeviceToDevice, s));
    if (l < nlevels) {
      k_member<<<grid_for(nlk[l], 256), 256, 0, s>>>(lk[l], nlk[l], NL[l], nnl[l],
                                                      t.nonleaf.get() + t.lev_start[l]);
      FGT_LAUNCH_CHECK();
    } else {
      FGT_CUDA(cudaMemsetAsync(t.nonleaf.get() + t.lev_start[l], 0, sizeof(int) * nlk[l], s));
    }
  }
  FGT_REQUIRE(nlevels < 64, FGT_ERR_UNSUPPORTED, "too many levels");
  LevelTables lt;
  for (int l = 0; l <= nlevels; l++) {
    lt.keys[l] = lk[l].get();
    lt.n[l] = nlk[l];
    lt.start[l] = t.lev_start[l];
  }
  lt.start[nlevels + 1] = t.lev_start[nlevels + 1];
  k_box_tables<<<grid_for(nboxes, 256), 256, 0, s>>>(nboxes, nlevels, dim, lt, kp, t.key,
                                                      t.level, t.nonleaf, t.parent, t.child0,
                                                      t.center);
  FGT_LAUNCH_CHECK();

  // 5. leaves and the final point order (stable by original index)
  DBuf<int> lf(nboxes, s), lpos(nboxes, s), ltot(1, s);
  k_leaf_flags<<<grid_for(nboxes, 256), 256, 0, s>>>(t.nonleaf, nboxes, lf);
  FGT_LAUNCH_CHECK();
  exclusive_scan_i32(lf, lpos, nboxes, ltot, s);
  int nl = fetch_int(ltot, s);
  t.nleaves = nl;
  DBuf<uint64_t> ls(nl, s), lstmp(nl, s);
  DBuf<uint32_t> lbox(nl, s), lbtmp(nl, s);
  k_leaf_starts<<<grid_for(nboxes, 256), 256, 0, s>>>(t.key, t.level, lf, lpos, nboxes, dim, D,
                                                       ls, lbox);
  FGT_LAUNCH_CHECK();
  radix_sort(ls, lbox, lstmp, lbtmp, nl, dim * D, s);
  DBuf<int> lref(std::max(nl, 1), s);
  k_leaf_ref<<<grid_for(nl, 256), 256, 0, s>>>(lbox, nl, t.level, t.parent, t.ncutoff, lref);
  FGT_LAUNCH_CHECK();
  int obits = bits_for(nl);
  DBuf<int> slo(nl + 1, s), tlo(nl + 1, s);
  t.src_ref.alloc(std::max(ns, 1), s);
  t.trg_ref.alloc(std::max(nt, 1), s);
  {
    // leaf ordinals as 32-bit keys (half the key traffic of the sort)
    DBuf<uint32_t> ord(std::max(ns, 1), s);
    DBuf<uint32_t> vtmp(std::max(std::max(ns, nt), 1), s);
    uint32_t* otmp = reinterpret_cast<uint32_t*>(ktmp.get());  // >= max(ns, nt) u32
    t.isrc.alloc(std::max(ns, 1), s);
    DBuf<uint32_t> table;
    if (dense && nl > 0) {  // leaf ordinals by table lookup instead of binary search
      const long long ncell = 1ll << (dim * D);
      table.alloc((size_t)ncell, s);
      k_cell_leaf<<<std::min(nl, kSMs * 16), 256, 0, s>>>(ls, nl, ncell, table);
      FGT_LAUNCH_CHECK();
    }
    auto point_leaf = [&](const uint64_t* keys, int n, uint32_t* o, uint32_t* idx) {
      if (table.p)
        k_point_leaf_dense<<<grid_for(n, 256), 256, 0, s>>>(keys, n, table, o, idx);
      else
        k_point_leaf<<<grid_for(n, 256), 256, 0, s>>>(keys, n, ls, nl, o, idx);
      FGT_LAUNCH_CHECK();
    };
    if (ns > 0) {
      point_leaf(skey, ns, ord, t.isrc);
      radix_sort_u32(ord, t.isrc, otmp, vtmp, ns, obits, s);
    }
    k_leaf_point_lo<<<grid_for(nl + 1, 256), 256, 0, s>>>(ord, ns, nl, slo);
    FGT_LAUNCH_CHECK();
    if (ns > 0) {
      k_point_ref<<<grid_for(ns, 256), 256, 0, s>>>(ord, ns, lref, t.src_ref);
      FGT_LAUNCH_CHECK();
    }
    DBuf<uint32_t> tord(std::max(nt, 1), s);
    t.itrg.alloc(std::max(nt, 1), s);
    if (nt > 0) {
      point_leaf(tkey, nt, tord, t.itrg);
      radix_sort_u32(tord, t.itrg, otmp, vtmp, nt, obits, s);
    }
    k_leaf_point_lo<<<grid_for(nl + 1, 256), 256, 0, s>>>(tord, nt, nl, tlo);
    FGT_LAUNCH_CHECK();
    if (nt > 0) {
      k_point_ref<<<grid_for(nt, 256), 256, 0, s>>>(tord, nt, lref, t.trg_ref);
      FGT_LAUNCH_CHECK();
    }
  }
  t.src_lo.alloc(nboxes, s);
  t.src_hi.alloc(nboxes, s);
  t.trg_lo.alloc(nboxes, s);
  t.trg_hi.alloc(nboxes, s);
  k_box_ranges<<<grid_for(nboxes, 256), 256, 0, s>>>(t.key, t.level, nboxes, dim, D, ls, nl, slo,
                                                      tlo, t.src_lo, t.src_hi, t.trg_lo,
                                                      t.trg_hi);
  FGT_LAUNCH_CHECK();
}

void tree_download(const Tree& t, TreeHost& h, cudaStream_t s) {
  int nb = t.nboxes;
  auto dl = [&](auto& vec, const auto& buf, size_t n) {
    vec.resize(n);
    if (n) FGT_CUDA(cudaMemcpyAsync(vec.data(), buf.get(), sizeof(vec[0]) * n,
                                    cudaMemcpyDeviceToHost, s));
  };
  dl(h.key, t.key, nb);
  dl(h.level, t.level, nb);
  dl(h.nonleaf, t.nonleaf, nb);
  dl(h.parent, t.parent, nb);
  dl(h.child0, t.child0, nb);
  dl(h.src_lo, t.src_lo, nb);
  dl(h.src_hi, t.src_hi, nb);
  dl(h.trg_lo, t.trg_lo, nb);
  dl(h.trg_hi, t.trg_hi, nb);
  dl(h.center, t.center, (size_t)nb * t.dim);
  dl(h.isrc, t.isrc, t.ns);
  dl(h.itrg, t.itrg, t.nt);
  FGT_CUDA(cudaStreamSynchronize(s));
}

}  // namespace fgt
