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

// ---- modified list 1 of every target box (pfgt_compute_modified_list1,
// src/common/tree_routs_nd.f:1063-1257, restated from the target side):
//   * same level: leaf colleagues (self included);
//   * coarser: leaf colleagues of the parent (levels 1 .. npwlevel-1) whose
//     closure touches the box;
//   * finer: leaf children of non-leaf colleagues touching the box.
// One warp per target box: the candidates of each stage are resolved by the
// lanes at once (one key search per lane), and the kept boxes are emitted in
// candidate order by ballot and prefix count, so count and fill agree.
template <int DIM>
__device__ __forceinline__ void coords_of_d(const TV& tv, int b, uint32_t* c) {
  const int l = tv.level[b];
  const uint64_t key = tv.key[b];
#pragma unroll
  for (int k = 0; k < DIM; k++) c[k] = 0;
  for (int j = 0; j < l; j++) {
    const int dig = (int)((key >> (DIM * (l - 1 - j))) & ((1u << DIM) - 1));
#pragma unroll
    for (int k = 0; k < DIM; k++) c[k] = (c[k] << 1) | ((dig >> k) & 1);
  }
}
template <int DIM>
__device__ __forceinline__ int find_box_d(const TV& tv, int l, const uint32_t* c) {
  uint64_t key = 0;
  for (int j = 0; j < l; j++) {
    int dig = 0;
#pragma unroll
    for (int k = 0; k < DIM; k++) dig |= ((c[k] >> (l - 1 - j)) & 1) << k;
    key = (key << DIM) | (uint64_t)dig;
  }
  const int lo = tv.lev_start[l], n = tv.lev_start[l + 1] - lo;
  const int i = dev_find(tv.key + lo, n, key);
  return i < 0 ? -1 : lo + i;
}
// Closures of a level-(lf) box (coords cf) and a level-(lf-1) box (coords cc)
// touch: the distance tests of src/common/tree_routs_nd.f:1181-1213,
// 1226-1245 in units of half the finer box size (periodic minimum image
// when `periodic`).
template <int DIM>
__device__ __forceinline__ bool touch_levels_d(const uint32_t* cf, int lf, const uint32_t* cc,
                                               int periodic) {
  const long long P = 2ll << lf;
  bool ok = true;
#pragma unroll
  for (int k = 0; k < DIM; k++) {
    long long d = (long long)(2 * cf[k] + 1) - (long long)(4 * cc[k] + 2);
    if (d < 0) d = -d;
    if (periodic && P - d < d) d = P - d;
    ok = ok && d <= 3;
  }
  return ok;
}
// Colleague `i` (in the candidate order of for_colleagues) of box b on this
// lane: the box id, or -1 (no such box, or i >= *tot).
template <int DIM>
__device__ __forceinline__ int colleague_of(const TV& tv, int b, int periodic, int i, int* tot) {
  const int l = tv.level[b];
  uint32_t c[DIM];
  coords_of_d<DIM>(tv, b, c);
  const long long n = 1ll << l;
  uint32_t vals[DIM][3];
  int nv[DIM];
#pragma unroll
  for (int k = 0; k < DIM; k++) {
    nv[k] = 0;
#pragma unroll
    for (int o = -1; o <= 1; o++) {
      long long q = (long long)c[k] + o;
      if (periodic) q = ((q % n) + n) % n;
      else if (q < 0 || q >= n) continue;
      bool dup = false;
#pragma unroll
      for (int j = 0; j < 3; j++) dup |= (j < nv[k] && vals[k][j] == (uint32_t)q);
      if (!dup) {
#pragma unroll
        for (int j = 0; j < 3; j++)
          if (j == nv[k]) vals[k][j] = (uint32_t)q;
        nv[k]++;
      }
    }
  }
  int t = 1;
#pragma unroll
  for (int k = 0; k < DIM; k++) t *= nv[k];
  *tot = t;
  if (i >= t) return -1;
  uint32_t q[DIM];
  int r = i;
#pragma unroll
  for (int k = 0; k < DIM; k++) {
    const int s = r % nv[k];
    q[k] = s == 0 ? vals[k][0] : (s == 1 ? vals[k][1] : vals[k][2]);
    r /= nv[k];
  }
  return find_box_d<DIM>(tv, l, q);
}

template <int DIM, bool FILL>
__global__ void k_list1_warp(TV tv, int nboxes, int* __restrict__ cnt, const int* __restrict__ ptr,
                             int* __restrict__ out) {
  constexpr int MC = 1 << DIM;
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const unsigned lt = (1u << lane) - 1u;
  for (int T = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; T < nboxes; T += nw) {
    const int base = FILL ? ptr[T] : 0;
    int n = 0;
    auto emit = [&](bool keep, int S) {
      const unsigned m = __ballot_sync(0xffffffffu, keep);
      if (FILL && keep) out[base + n + __popc(m & lt)] = S;
      n += __popc(m);
    };
    const int l = tv.level[T];
    const bool leafT = !tv.nonleaf[T];
    if (l <= tv.nlevend) {
      if (l == 0) {
        emit(lane == 0 && leafT, T);
      } else if (leafT || l == tv.npwlevel) {
        const int per = tv.iperiod0;
        // same level: leaf colleagues (self included)
        int tot1;
        const int J = colleague_of<DIM>(tv, T, per, lane, &tot1);
        emit(J >= 0 && !tv.nonleaf[J], J);
        if (leafT) {
          uint32_t cT[DIM];
          coords_of_d<DIM>(tv, T, cT);
          // coarser leaf sources adjacent to T
          if (l - 1 >= 1 && l - 1 < tv.npwlevel) {
            int tot2;
            const int S = colleague_of<DIM>(tv, tv.parent[T], per, lane, &tot2);
            bool keep = false;
            if (S >= 0 && !tv.nonleaf[S]) {
              uint32_t cS[DIM];
              coords_of_d<DIM>(tv, S, cS);
              keep = touch_levels_d<DIM>(cT, l, cS, per);
            }
            emit(keep, S);
          }
          // finer leaf sources: leaf children of non-leaf colleagues touching T
          if (l + 1 <= tv.nlevend) {
            for (int c0 = 0; c0 < tot1 * MC; c0 += 32) {
              const int c = c0 + lane, i = c / MC, j = c % MC;
              const int Ji = __shfl_sync(0xffffffffu, J, i & 31);
              bool keep = false;
              int S = -1;
              if (c < tot1 * MC && Ji >= 0 && tv.nonleaf[Ji] && tv.child0[Ji] >= 0) {
                S = tv.child0[Ji] + j;
                if (!tv.nonleaf[S]) {
                  uint32_t cS[DIM];
                  coords_of_d<DIM>(tv, S, cS);
                  keep = touch_levels_d<DIM>(cS, l + 1, cT, per);
                }
              }
              emit(keep, S);
            }
          }
        }
      }
    }
    if (!FILL && lane == 0) cnt[T] = n;
  }
}

template <bool FILL>
void launch_list1(const TV& tv, int nb, int* cnt, const int* ptr, int* out, cudaStream_t s) {
  const int grid = grid_for((long long)nb * 32, 256);
  if (tv.dim == 1) k_list1_warp<1, FILL><<<grid, 256, 0, s>>>(tv, nb, cnt, ptr, out);
  else if (tv.dim == 2) k_list1_warp<2, FILL><<<grid, 256, 0, s>>>(tv, nb, cnt, ptr, out);
  else k_list1_warp<3, FILL><<<grid, 256, 0, s>>>(tv, nb, cnt, ptr, out);
  FGT_LAUNCH_CHECK();
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
  // direct near field: list lengths; the plane-wave box flags are counted
  // before the one read-back of all three totals
  L.l1_ptr.alloc(nb + 1, s);
  DBuf<int> cnt1(nb, s);
  launch_list1<false>(tv, nb, cnt1, nullptr, nullptr, s);
  exclusive_scan_i32(cnt1, L.l1_ptr, nb, L.l1_ptr.get() + nb, s);
  L.n_form = L.n_eval = L.n_trans = 0;
  const int lo = do_pw ? t.lev_start[t.ncutoff] : 0;
  const int n = do_pw ? t.lev_start[t.ncutoff + 1] - lo : 0;
  DBuf<int> ff, fe, pf, pe, tf, te, fslot;
  if (do_pw) {
    ff.alloc(n, s);
    fe.alloc(n, s);
    pf.alloc(n, s);
    pe.alloc(n, s);
    tf.alloc(1, s);
    te.alloc(1, s);
    fslot.alloc(n, s);
    k_pw_flags<<<grid_for(n, 128), 128, 0, s>>>(tv, t.ndiv, ff, fe);
    FGT_LAUNCH_CHECK();
    exclusive_scan_i32(ff, pf, n, tf, s);
    exclusive_scan_i32(fe, pe, n, te, s);
  }
  {
    const int* src[3] = {L.l1_ptr.get() + nb, tf.get(), te.get()};
    int h[3] = {0, 0, 0};
    fetch_ints(src, do_pw ? 3 : 1, h, s);
    L.n_l1 = h[0];
    L.n_form = h[1];
    L.n_eval = h[2];
  }
  L.l1_src.alloc(std::max(L.n_l1, 1), s);
  launch_list1<true>(tv, nb, nullptr, L.l1_ptr, L.l1_src, s);
  if (!do_pw) return;
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
