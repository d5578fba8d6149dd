// Interaction lists (count -> scan -> fill; deterministic, race free).
#include <algorithm>

#include "fgt_lists.cuh"

namespace fgt {

namespace {

struct TV {
  int dim, nlevels, iperiod0, npwlevel, nlevend, ncutoff;
  double bs0, xmin;
  const uint64_t* key;
  const int *level, *nonleaf, *child0, *parent, *src_lo, *src_hi;
  const double* center;
  int lev_start[66];
};

__device__ __forceinline__ void coords_of(const TV& tv, int b, uint32_t* c) {
  int l = tv.level[b];
  uint64_t key = tv.key[b];
  for (int k = 0; k < tv.dim; k++) c[k] = 0;
  for (int j = 0; j < l; j++) {
    int dig = (int)((key >> (tv.dim * (l - 1 - j))) & ((1u << tv.dim) - 1));
    for (int k = 0; k < tv.dim; k++) c[k] = (c[k] << 1) | ((dig >> k) & 1);
  }
}

__device__ __forceinline__ int find_box(const TV& tv, int l, const uint32_t* c) {
  uint64_t key = 0;
  for (int j = 0; j < l; j++) {
    int dig = 0;
    for (int k = 0; k < tv.dim; k++) dig |= ((c[k] >> (l - 1 - j)) & 1) << k;
    key = (key << tv.dim) | (uint64_t)dig;
  }
  int lo = tv.lev_start[l], n = tv.lev_start[l + 1] - lo;
  int i = dev_find(tv.key + lo, n, key);
  return i < 0 ? -1 : lo + i;
}

// Colleagues (same level, closures touching, self included), as computecoll
// (src/common/tree_routs_nd.f:106-242): periodic wrap when `periodic`.
template <typename F>
__device__ __forceinline__ void for_colleagues(const TV& tv, int b, int periodic, F f) {
  int l = tv.level[b];
  uint32_t c[FGT_MAXDIM];
  coords_of(tv, b, c);
  long long n = 1ll << l;
  long long vals[FGT_MAXDIM][3];
  int nv[FGT_MAXDIM];
  for (int k = 0; k < tv.dim; k++) {
    nv[k] = 0;
    for (int o = -1; o <= 1; o++) {
      long long q = (long long)c[k] + o;
      if (periodic) q = ((q % n) + n) % n;
      else if (q < 0 || q >= n) continue;
      bool dup = false;
      for (int j = 0; j < nv[k]; j++) dup |= (vals[k][j] == q);
      if (!dup) vals[k][nv[k]++] = q;
    }
  }
  int tot = 1;
  for (int k = 0; k < tv.dim; k++) tot *= nv[k];
  for (int i = 0; i < tot; i++) {
    uint32_t q[FGT_MAXDIM];
    int r = i;
    for (int k = 0; k < tv.dim; k++) { q[k] = (uint32_t)vals[k][r % nv[k]]; r /= nv[k]; }
    int bb = find_box(tv, l, q);
    if (bb >= 0) f(bb);
  }
}

// Closures of a level-(lc+1) box (coords cf) and a level-lc box (coords cc)
// touch: the distance tests of src/common/tree_routs_nd.f:1181-1213,
// 1226-1245 in units of half the finer box size (periodic minimum image
// when `periodic`).
__device__ __forceinline__ bool touch_levels(const TV& tv, const uint32_t* cf, int lf,
                                             const uint32_t* cc, int periodic) {
  long long P = 2ll << lf;
  for (int k = 0; k < tv.dim; k++) {
    long long d = (long long)(2 * cf[k] + 1) - (long long)(4 * cc[k] + 2);
    if (d < 0) d = -d;
    if (periodic && P - d < d) d = P - d;
    if (d > 3) return false;
  }
  return true;
}

// Modified list 1 of target box T (pfgt_compute_modified_list1,
// src/common/tree_routs_nd.f:1063-1257, restated from the target side).
template <typename F>
__device__ void for_list1(const TV& tv, int T, F add) {
  int l = tv.level[T];
  bool leafT = !tv.nonleaf[T];
  if (l > tv.nlevend) return;
  if (l == 0) {
    if (leafT) add(T);
    return;
  }
  if (!(leafT || l == tv.npwlevel)) return;
  int per = tv.iperiod0;
  // same level: leaf colleagues (self included)
  for_colleagues(tv, T, per, [&](int S) {
    if (!tv.nonleaf[S]) add(S);
  });
  if (!leafT) return;
  uint32_t cT[FGT_MAXDIM];
  coords_of(tv, T, cT);
  // coarser leaf sources adjacent to T (sources at level l-1 >= 1, l-1 < npwlevel)
  if (l - 1 >= 1 && l - 1 < tv.npwlevel) {
    for_colleagues(tv, tv.parent[T], per, [&](int S) {
      if (tv.nonleaf[S]) return;
      uint32_t cS[FGT_MAXDIM];
      coords_of(tv, S, cS);
      if (touch_levels(tv, cT, l, cS, per)) add(S);
    });
  }
  // finer leaf sources: leaf children of non-leaf colleagues touching T
  if (l + 1 <= tv.nlevend) {
    int mc = 1 << tv.dim;
    for_colleagues(tv, T, per, [&](int J) {
      if (!tv.nonleaf[J]) return;
      int c0 = tv.child0[J];
      if (c0 < 0) return;
      for (int j = 0; j < mc; j++) {
        int S = c0 + j;
        if (tv.nonleaf[S]) continue;
        uint32_t cS[FGT_MAXDIM];
        coords_of(tv, S, cS);
        if (touch_levels(tv, cS, l + 1, cT, per)) add(S);
      }
    });
  }
}

__global__ void k_list1_count(TV tv, int nboxes, int* __restrict__ cnt) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nboxes; b += gridDim.x * blockDim.x) {
    int c = 0;
    for_list1(tv, b, [&](int) { c++; });
    cnt[b] = c;
  }
}
__global__ void k_list1_fill(TV tv, int nboxes, const int* __restrict__ ptr, int* __restrict__ out) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nboxes; b += gridDim.x * blockDim.x) {
    int p = ptr[b];
    for_list1(tv, b, [&](int S) { out[p++] = S; });
  }
}

// Plane-wave flags at the cutoff level: form (npts > ndiv, pfgt.f:779) and
// ifpwexp (pfgt_find_pwexp_boxes, src/common/tree_routs_nd.f:1373-1460).
__global__ void k_pw_flags(TV tv, int ndiv, int* __restrict__ fform, int* __restrict__ feval) {
  int lo = tv.lev_start[tv.ncutoff], n = tv.lev_start[tv.ncutoff + 1] - lo;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int b = lo + i;
    fform[i] = (tv.src_hi[b] - tv.src_lo[b] > ndiv) ? 1 : 0;
    int e = 0;
    if (tv.npwlevel <= 0) {
      e = (b == 0);
    } else {
      for_colleagues(tv, b, tv.iperiod0, [&](int J) { e |= tv.nonleaf[J]; });
    }
    feval[i] = e;
  }
}

__global__ void k_compact_idx(const int* __restrict__ f, const int* __restrict__ pos, int n,
                              int base, int* __restrict__ out, int* __restrict__ slot) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (f[i]) out[pos[i]] = base + i;
    if (slot) slot[i] = f[i] ? pos[i] : -1;
  }
}

__device__ __forceinline__ int fnint(double x) { return (int)round(x); }

// PW list of each eval box: non-leaf colleagues other than itself
// (pfgt_compute_listpw, src/common/tree_routs_nd.f:1487-1555) with their
// shift-table index (gnd_find_pwshift_ind, src/bfgt/bfgt_pwrouts.f:1592-1636).
template <bool FILL>
__global__ void k_trans(TV tv, const int* __restrict__ eval_box, int n_eval,
                        const int* __restrict__ form_slot, const int* __restrict__ ptr,
                        int* __restrict__ cnt, int* __restrict__ src, int* __restrict__ widx) {
  int lo = tv.lev_start[tv.ncutoff];
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_eval; e += gridDim.x * blockDim.x) {
    int t = eval_box[e];
    int c = 0, p = FILL ? ptr[e] : 0;
    for_colleagues(tv, t, tv.iperiod0, [&](int s) {
      if (s == t || !tv.nonleaf[s]) return;
      int slot = form_slot[s - lo];
      if (slot < 0) return;  // empty expansion contributes nothing
      if (FILL) {
        int ind = 0, inc = 1;
        for (int d = 0; d < tv.dim; d++) {
          double dx = tv.center[(size_t)t * tv.dim + d] - tv.center[(size_t)s * tv.dim + d];
          int jx = fnint(dx / tv.xmin);
          if (tv.iperiod0 == 1) {
            int jxp1 = fnint((dx - tv.bs0) / tv.xmin);
            int jxm1 = fnint((dx + tv.bs0) / tv.xmin);
            if (abs(jx) > abs(jxp1)) jx = jxp1;
            if (abs(jx) > abs(jxm1)) jx = jxm1;
          }
          ind += (jx + 1) * inc;
          inc *= 3;
        }
        src[p] = slot;
        widx[p] = ind;
        p++;
      }
      c++;
    });
    if (!FILL) cnt[e] = c;
  }
}

TV make_tv(const Tree& t, int npwlevel, int iperiod0, int nlevend) {
  TV tv;
  tv.dim = t.dim;
  tv.nlevels = t.nlevels;
  tv.iperiod0 = iperiod0;
  tv.npwlevel = npwlevel;
  tv.nlevend = nlevend;
  tv.ncutoff = t.ncutoff;
  tv.bs0 = t.bs0;
  tv.xmin = t.boxsize[std::min(t.ncutoff, t.nlevels)];
  tv.key = t.key;
  tv.level = t.level;
  tv.nonleaf = t.nonleaf;
  tv.child0 = t.child0;
  tv.parent = t.parent;
  tv.src_lo = t.src_lo;
  tv.src_hi = t.src_hi;
  tv.center = t.center;
  FGT_REQUIRE(t.nlevels < 64, FGT_ERR_UNSUPPORTED, "too many levels");
  for (int l = 0; l < 66; l++) tv.lev_start[l] = t.lev_start[std::min(l, t.nlevels + 1)];
  return tv;
}

}  // namespace

namespace {
__global__ void k_eval_self(int n_eval, const int* __restrict__ eval_box,
                            const int* __restrict__ fslot, int lo, int* __restrict__ eval_self) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_eval; e += gridDim.x * blockDim.x)
    eval_self[e] = fslot[eval_box[e] - lo];
}
}  // namespace

void build_lists(const Tree& t, int npwlevel, int iperiod0, int nlevend, bool do_pw, Lists& L,
                 cudaStream_t s) {
  TV tv = make_tv(t, npwlevel, iperiod0, nlevend);
  int nb = t.nboxes;
  // direct near field
  L.l1_ptr.alloc(nb + 1, s);
  {
    DBuf<int> cnt(nb, s), tot(1, s);
    k_list1_count<<<grid_for(nb, 128), 128, 0, s>>>(tv, nb, cnt);
    FGT_LAUNCH_CHECK();
    exclusive_scan_i32(cnt, L.l1_ptr, nb, L.l1_ptr.get() + nb, s);
    L.n_l1 = fetch_int(L.l1_ptr.get() + nb, s);
    L.l1_src.alloc(std::max(L.n_l1, 1), s);
    k_list1_fill<<<grid_for(nb, 128), 128, 0, s>>>(tv, nb, L.l1_ptr, L.l1_src);
    FGT_LAUNCH_CHECK();
  }
  L.n_form = L.n_eval = L.n_trans = 0;
  if (!do_pw) return;
  int lo = t.lev_start[t.ncutoff], n = t.lev_start[t.ncutoff + 1] - lo;
  DBuf<int> ff(n, s), fe(n, s), pf(n, s), pe(n, s), tf(1, s), te(1, s), fslot(n, s);
  k_pw_flags<<<grid_for(n, 128), 128, 0, s>>>(tv, t.ndiv, ff, fe);
  FGT_LAUNCH_CHECK();
  exclusive_scan_i32(ff, pf, n, tf, s);
  exclusive_scan_i32(fe, pe, n, te, s);
  L.n_form = fetch_int(tf, s);
  L.n_eval = fetch_int(te, s);
  L.form_box.alloc(std::max(L.n_form, 1), s);
  L.eval_box.alloc(std::max(L.n_eval, 1), s);
  L.eval_self.alloc(std::max(L.n_eval, 1), s);
  k_compact_idx<<<grid_for(n, 256), 256, 0, s>>>(ff, pf, n, lo, L.form_box, fslot);
  FGT_LAUNCH_CHECK();
  k_compact_idx<<<grid_for(n, 256), 256, 0, s>>>(fe, pe, n, lo, L.eval_box, nullptr);
  FGT_LAUNCH_CHECK();
  // eval_self[e] = form slot of eval box e
  if (L.n_eval > 0) {
    k_eval_self<<<grid_for(L.n_eval, 256), 256, 0, s>>>(L.n_eval, L.eval_box, fslot, lo,
                                                         L.eval_self);
    FGT_LAUNCH_CHECK();
  }
  L.trans_ptr.alloc(L.n_eval + 1, s);
  {
    DBuf<int> cnt(std::max(L.n_eval, 1), s);
    if (L.n_eval > 0) {
      k_trans<false><<<grid_for(L.n_eval, 128), 128, 0, s>>>(tv, L.eval_box, L.n_eval, fslot,
                                                             nullptr, cnt, nullptr, nullptr);
      FGT_LAUNCH_CHECK();
    }
    exclusive_scan_i32(cnt, L.trans_ptr, L.n_eval, L.trans_ptr.get() + L.n_eval, s);
    L.n_trans = fetch_int(L.trans_ptr.get() + L.n_eval, s);
    L.trans_src.alloc(std::max(L.n_trans, 1), s);
    L.trans_w.alloc(std::max(L.n_trans, 1), s);
    if (L.n_eval > 0) {
      k_trans<true><<<grid_for(L.n_eval, 128), 128, 0, s>>>(tv, L.eval_box, L.n_eval, fslot,
                                                            L.trans_ptr, nullptr, L.trans_src,
                                                            L.trans_w);
      FGT_LAUNCH_CHECK();
    }
  }
}

void lists_download(const Lists& L, int nboxes, ListsHost& h, cudaStream_t s) {
  auto dl = [&](std::vector<int>& v, const DBuf<int>& b, size_t n) {
    v.resize(n);
    if (n) FGT_CUDA(cudaMemcpyAsync(v.data(), b.get(), sizeof(int) * n, cudaMemcpyDeviceToHost, s));
  };
  dl(h.l1_ptr, L.l1_ptr, nboxes + 1);
  dl(h.l1_src, L.l1_src, L.n_l1);
  dl(h.form_box, L.form_box, L.n_form);
  dl(h.eval_box, L.eval_box, L.n_eval);
  dl(h.eval_self, L.eval_self, L.n_eval);
  if (L.n_eval > 0 || L.trans_ptr.p) dl(h.trans_ptr, L.trans_ptr, L.trans_ptr.p ? L.n_eval + 1 : 0);
  dl(h.trans_src, L.trans_src, L.n_trans);
  dl(h.trans_w, L.trans_w, L.n_trans);
  FGT_CUDA(cudaStreamSynchronize(s));
}

}  // namespace fgt
