// Plane-wave evaluation kernels (K8): per-box grids with interpolation at
// the box's points, and direct modal sums for boxes with few points.
// Included by fgt_pw_eval_f32.cu and fgt_pw_eval_f64.cu, which instantiate
// pw_eval for one arithmetic type each (the two halves compile in parallel).
#pragma once
#include <math.h>

#include <algorithm>
#include <vector>

#include "fgt_pw_dev.cuh"

namespace fgt {

namespace {

// ---------------------------------------------------------------- eval
template <typename T>
struct EvalPtrs {
  const T* loc;      // [n_eval][nd][nexp]
  const int* boxes;  // eval slots handled by this launch
  const int* eval_box;
  int nbox;             // upper bound (grid sizing)
  const int* nbox_dev;  // actual count on the device, or null: nbox
  int* next;            // work counter of the grid kernel (zero at launch)
  // grid kernel: work items (parts of boxes), count on the device, bound
  const WorkItem* items;
  const int* n_items;
  int max_items;
  // two evaluation sets (sources, targets)
  const double* off[2];
  const int* lo[2];
  const int* hi[2];
  double* out[2];
  int n[2], ncomp[2];
  int nd, ncomp_max;
  int cell_bins;  // base cells of the sub-grid for the cell order, 0: bank-class order
  int slab, nslab;  // x-slab grids: planes per slab and slabs per box (1: whole grids)
};

// component factor (complex) of evaluation component c at mode ki[]
template <typename T, int DIM>
__device__ __forceinline__ void eval_factor(const PWArgs<T>& a, int c, const int* ki, T& fr, T& fi) {
  if (c == 0) {
    fr = T(1);
    fi = T(0);
    return;
  }
  if (c <= DIM) {  // i ts(k_d)/sqrt(delta0)
    fr = T(0);
    fi = a.ts[sel3(ki, c - 1)] * a.inv_sqd0;
    return;
  }
  int m = c - 1 - DIM, p, q;
  if (DIM == 1) { p = 0; q = 0; }
  else if (DIM == 2) { p = (m == 2) ? 1 : 0; q = (m == 0) ? 0 : 1; }
  else { p = m < 3 ? m : (m < 5 ? 0 : 1); q = m < 3 ? m : (m == 3 ? 1 : 2); }
  fr = -a.ts[sel3(ki, p)] * a.ts[sel3(ki, q)] * a.inv_sqd0 * a.inv_sqd0;
  fi = T(0);
}

// Grid of evaluation component c of expansion L in buffer B (real values).
template <typename T, int DIM>
__device__ __forceinline__ void build_eval_grid(const PWArgs<T>& a, const T* L, int c, T* B,
                                                const T* tif, const T* tih) {
  const Geo& g = a.g;
  const int K = g.K, NF = 2 * K + 1, NH = K + 1, G = g.G;
  const int nline = DIM == 3 ? NF * NH : (DIM == 2 ? NH : 1);
  if (DIM == 1) {
    for (int l = threadIdx.x; l < G; l += blockDim.x) {
      T acc = T(0);
      for (int k = 0; k < NH; k++) {
        int ki[3] = {k + K, 0, 0};
        T fr, fi;
        eval_factor<T, DIM>(a, c, ki, fr, fi);
        const T f = a.faci[k + K];
        const T lr = L[2 * k] * f, li = L[2 * k + 1] * f;
        const T mr = lr * fr - li * fi, mi = lr * fi + li * fr;
        acc += mr * tih[k * 2 * pad4(G) + l] - mi * tih[k * 2 * pad4(G) + pad4(G) + l];
      }
      B[l] = acc;
    }
    __syncthreads();
    return;
  }
  // expansion times factors at B[kx][ky][kz], then the x pass in place
  for (int m = threadIdx.x; m < g.nexp; m += blockDim.x) {
    int ki[3], pos;
    if (DIM == 3) {
      const int kxi = m / nline, line = m - kxi * nline;
      const int kyi = line / NH, kz = line - kyi * NH;
      ki[0] = kxi;
      ki[1] = kyi;
      ki[2] = kz + K;
      pos = kxi * g.str[0] + kyi * g.str[1] + 2 * kz;
    } else {
      const int kxi = m / NH, ky = m - kxi * NH;
      ki[0] = kxi;
      ki[1] = ky + K;
      pos = kxi * g.str[0] + 2 * ky;
    }
    T f = T(1);
#pragma unroll
    for (int d = 0; d < DIM; d++) f *= a.faci[ki[d]];
    T fr, fi;
    eval_factor<T, DIM>(a, c, ki, fr, fi);
    fr *= f;
    fi *= f;
    const T lr = L[2 * m], li = L[2 * m + 1];
    B[pos] = lr * fr - li * fi;
    B[pos + 1] = lr * fi + li * fr;
  }
  __syncthreads();
  if (DIM == 3) {
    pass_inplace<T, 1>(B, NF * NH, NH, g.str[1], 2, g.str[0], g.str[0], NF, G, tif);
    pass_inplace<T, 1>(B, G * NH, NH, g.str[0], 2, g.str[1], g.str[1], NF, G, tif);
    pass_inplace<T, 2>(B, G * G, G, g.str[0], g.str[1], 2, 1, NH, G, tih);
  } else {
    pass_inplace<T, 1>(B, NH, 1, 2, 0, g.str[0], g.str[0], NF, G, tif);
    pass_inplace<T, 2>(B, G, 1, g.str[0], 0, 2, 1, NH, G, tih);
  }
}

// Thread-per-point interpolation of both evaluation sets in bank-balanced
// order.  DERIV: one potential grid, gradients through the kernel derivative
// (no hessians); otherwise one grid per output component (pot, grad_k,
// hess_kl).
// Threads of a k_eval_comp CTA: more warps share the SM's one grid for the
// 3D FP32 derivative kernel on a shared grid at widths <= 9 (its stencil
// needs fewer registers), 512 otherwise.
#ifndef FGT_EVAL3_THREADS
#define FGT_EVAL3_THREADS 512
#endif
template <typename T, int DIM, int W, bool GB, bool DERIV>
constexpr int eval_threads() {
  if constexpr (std::is_same<T, float>::value && DIM == 3 && W <= 9 && !GB && DERIV)
    return FGT_EVAL3_THREADS;
  // the FP64 derivative stencil needs more than 128 registers per thread
  if constexpr (std::is_same<T, double>::value && DIM == 3 && DERIV) return PW_THREADS / 2;
  return PW_THREADS;
}

template <typename T, int DIM, int W, bool GB, bool DERIV>
__global__ void __launch_bounds__(eval_threads<T, DIM, W, GB, DERIV>())
    k_eval_comp(PWArgs<T> a, EvalPtrs<T> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Geo& g = a.g;
  const int K = g.K, NF = 2 * K + 1, NH = K + 1, G = g.G;
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int Gp = pad4(G);
  // planar rows of 2*Gp (staged or global)
  const T* tif = stage_tw(sm, a.tif, 2 * NF * Gp);
  const T* tih = stage_tw(sm + 2 * NF * Gp, a.tih, 2 * NH * Gp);
  int* ordtmp = reinterpret_cast<int*>(sm + tw_elems_t<T>(G, K));
  int* ordcnt = ordtmp + ORDER_CHUNK;
  unsigned short* perm = reinterpret_cast<unsigned short*>(ordcnt + 32);
  int* bins = reinterpret_cast<int*>(smem_raw + order_offset<T>(G, K));  // NBINS_MAX
  int* bws = bins + NBINS_MAX;                                            // 32
  T* B = GB ? a.gscratch + (size_t)blockIdx.x * g.bufsz
            : reinterpret_cast<T*>(smem_raw + eval_offset<T>(G, K));
  // interpolation reads: shared-space view of the grid (pointer for GB)
  const auto BV = [&]() {
    if constexpr (GB) return static_cast<const T*>(B);
    else return SmemView<T>{(int)(eval_offset<T>(G, K) / sizeof(T))};
  }();
  __syncthreads();
  // shared-space byte address of the grid (shared-memory grid variants)
  const uint32_t grid_saddr =
      (uint32_t)__cvta_generic_to_shared(smem_raw) + (uint32_t)eval_offset<T>(G, K);
  (void)grid_saddr;
  const int n_items = *p.n_items;
  // items (boxes, or parts of large boxes) in decreasing point count, each
  // CTA takes the next one; a part evaluates its share of both point sets
  __shared__ int s_next;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_next = atomicAdd(p.next, 1);
    __syncthreads();
    const int bi = s_next;
    if (bi >= n_items) break;
    const WorkItem it = p.items[bi];
    const int e = it.slot;
    if (!FGT_DCHECK(e >= 0 && e < p.nbox, 301)) continue;
    const int box = p.eval_box[e];
    for (int id = 0; id < p.nd; id++) {
      const T* L = p.loc + ((size_t)e * p.nd + id) * 2 * g.nexp;
      for (int c = 0; c < (DERIV ? 1 : p.ncomp_max); c++) {
        build_eval_grid<T, DIM>(a, L, c, B, tif, tih);
        for (int set = 0; set < 2; set++) {
          // select by value: indexing the parameter arrays with a run-time
          // index would copy them to local memory
          const int ne = set ? p.n[1] : p.n[0];
          if (c >= (set ? p.ncomp[1] : p.ncomp[0]) || ne == 0) continue;
          const double* offs = set ? p.off[1] : p.off[0];
          double* outs = set ? p.out[1] : p.out[0];
          int q0, q1;
          part_range(set ? p.lo[1][box] : p.lo[0][box], set ? p.hi[1][box] : p.hi[0][box],
                     it.part, it.nparts, q0, q1);
          if (!FGT_DCHECK(q0 >= 0 && q0 <= q1 && q1 <= ne, 302)) continue;
          for (int c0 = q0; c0 < q1; c0 += ORDER_CHUNK) {
            const int n = min(ORDER_CHUNK, q1 - c0);
            if (p.cell_bins > 0)
              order_cells<T, DIM, W>(a, offs, ne, c0, n, p.cell_bins, perm, ordtmp, bins, bws);
            else
              order_chunk<T, DIM, W>(a, offs, ne, c0, n, perm, ordtmp, ordcnt);
            // the next point's offsets are loaded while the current one is
            // interpolated; outputs are added with fire-and-forget atomics
            // (one contribution per point here, so the sum is the plain add)
            int pt_n = 0;
            double x_n[DIM];
            if (threadIdx.x < n) {
              pt_n = c0 + perm[threadIdx.x];
#pragma unroll
              for (int k = 0; k < DIM; k++) x_n[k] = offs[(size_t)k * ne + pt_n];
            }
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
              const int pt = pt_n;
              double x[DIM];
#pragma unroll
              for (int k = 0; k < DIM; k++) x[k] = x_n[k] * a.scale_d;
              if (i + (int)blockDim.x < n) {
                pt_n = c0 + perm[i + blockDim.x];
#pragma unroll
                for (int k = 0; k < DIM; k++) x_n[k] = offs[(size_t)k * ne + pt_n];
              }
              if constexpr (DERIV) {
                T v[1 + DIM];
                if constexpr (!GB && DIM == 3 && std::is_same<T, float>::value) {
                  if (!g.wrap)
                    interp_grad_point_s3<W>(a, grid_saddr, x, v);
                  else
                    interp_grad_point<T, DIM, W>(a, BV, x, v);
                } else if constexpr (DIM == 3 && std::is_same<T, double>::value) {
                  if (!g.wrap)
                    interp_grad_point_xr<T, W>(a, BV, x, v);
                  else
                    interp_grad_point<T, DIM, W>(a, BV, x, v);
                } else {
                  interp_grad_point<T, DIM, W>(a, BV, x, v);
                }
                const int nc = set ? p.ncomp[1] : p.ncomp[0];
                atomicAdd(&outs[(size_t)id * ne + pt], (double)v[0]);
                if (nc > 1) {
#pragma unroll
                  for (int d = 0; d < DIM; d++)
                    atomicAdd(&outs[((size_t)(1 + d) * p.nd + id) * ne + pt], (double)v[1 + d]);
                }
              } else {
                const T v = interp_point<T, DIM, W>(a, BV, x);
                atomicAdd(&outs[((size_t)c * p.nd + id) * ne + pt], (double)v);
              }
            }
            __syncthreads();
          }
        }
        __syncthreads();
      }
    }
  }
}

// ------------------------------------------------------ x-slab grids (3D)
// A grid too large for shared memory is cut into slabs of whole x-planes
// (slab_plan).  A work item is (box, point part, slab); its CTA computes the
// slab's planes of the box's grid from the local expansion (the x transform
// evaluated at those planes only, reading the expansion from global
// memory), runs the y and z passes on them (they never leave an x-plane),
// and adds to every point of its part the terms of the interpolation that
// fall on the slab's planes; a point's outputs are the sum of its slabs'
// terms (global atomics, as for the parts of split boxes).

// Sums over stencil cells [jlo, jhi) of one coordinate of the kernel values
// and of their derivatives, in FP64: the function of es_kernel / kernel_val_d
// with the launch's parameters (the same kernel as the T arithmetic), at
// FP64 offsets.
template <typename T>
__device__ __forceinline__ void kernel_sums_d(const PWArgs<T>& a, double x, int jlo, int jhi,
                                              double& ks, double& kd) {
  const double u = x * a.inv_dx_d;
  const double f0 = ceil(u - a.hwdx_d) - u;
  const double ih = (double)a.inv_hw, be = (double)a.beta, bds = be * (double)a.dscale;
  ks = 0.0;
  kd = 0.0;
  for (int j = jlo; j < jhi; j++) {
    const double z = (f0 + (double)j) * ih;
    const double q = 1.0 - z * z;
    const double r = q > 0.0 ? sqrt(q) : 0.0;
    const double e = exp(-be * (z * z) / (1.0 + r));
    ks += e;
    kd += q > 0.0 ? e * bds * z / r : 0.0;
  }
}

// Interpolation terms of one point on the planes [x0, x1) of a slab (slab
// plane xl is grid plane x0 + xl).  DERIV: potential and gradient as
// interp_grad_cells, with the centre cell of the slab's share of the stencil
// as the reference value bref: the T sums run over B - bref and bref's own
// terms (bref times products of kernel and derivative sums) are added back in
// FP64, where a slab's share of the x derivatives, unlike the whole
// stencil's, does not sum to ~0.  Else the potential of one component grid.
// Returns false when the stencil misses the slab.
template <typename T, int W, bool DERIV>
__device__ __forceinline__ bool interp_slab(const PWArgs<T>& a, const T* B, const double* x,
                                            int x0, int x1, double* v) {
  const Geo& g = a.g;
  T f0x;
  int bx = kernel_start<T>(a, x[0], f0x) - g.l0;
  bx = bx < 0 ? 0 : (bx > g.G - W ? g.G - W : bx);
  const int jlo = max(0, x0 - bx), jhi = min(W, x1 - bx);
  if (jlo >= jhi) return false;
  int b1, b2;
  if constexpr (DERIV) {
    T ph[2][W], dph[2][W];  // y and z rows
    b1 = kernel_row_d<T, W>(a, x[1], ph[0], dph[0]) - g.l0;
    b2 = kernel_row_d<T, W>(a, x[2], ph[1], dph[1]) - g.l0;
    b1 = b1 < 0 ? 0 : (b1 > g.G - W ? g.G - W : b1);
    b2 = b2 < 0 ? 0 : (b2 > g.G - W ? g.G - W : b2);
    const T* row0 = B + b1 * g.str[1] + b2;
    const int jm = (jlo + jhi) / 2;
    const T bref = row0[(bx + jm - x0) * g.str[0] + (W / 2) * g.str[1] + W / 2];
    // kernel sums and derivative sums of the three rows (x: the slab's share)
    T ksy = T(0), ksz = T(0), ksx = T(0), kdx = T(0), kdy = T(0), kdz = T(0);
#pragma unroll
    for (int j = 0; j < W; j++) {
      ksy += ph[0][j];
      ksz += ph[1][j];
      kdy += dph[0][j];
      kdz += dph[1][j];
    }
    T pot = T(0), gx = T(0), gy = T(0), gz = T(0);
#pragma unroll 1
    for (int jx = jlo; jx < jhi; jx++) {
      T px, dpx;
      kernel_val_d<T>(a, f0x, jx, px, dpx);
      ksx += px;
      kdx += dpx;
      const T* rx = row0 + (bx + jx - x0) * g.str[0];
      T t0 = T(0), t1 = T(0), t2 = T(0);
#pragma unroll
      for (int jy = 0; jy < W; jy++) {
        const T* ln = rx + jy * g.str[1];
        T s0 = T(0), s1 = T(0);
#pragma unroll
        for (int jz = 0; jz < W; jz++) {
          const T bv = ln[jz] - bref;
          s0 += bv * ph[1][jz];
          s1 += bv * dph[1][jz];
        }
        t0 += ph[0][jy] * s0;
        t1 += dph[0][jy] * s0;
        t2 += ph[0][jy] * s1;
      }
      pot += px * t0;
      gx += dpx * t0;
      gy += px * t1;
      gz += px * t2;
    }
    double Kx, Dx, Ky, Dy, Kz, Dz;
    if constexpr (std::is_same<T, double>::value) {
      Kx = ksx; Dx = kdx; Ky = ksy; Dy = kdy; Kz = ksz; Dz = kdz;
    } else {
      kernel_sums_d<T>(a, x[0], jlo, jhi, Kx, Dx);
      kernel_sums_d<T>(a, x[1], 0, W, Ky, Dy);
      kernel_sums_d<T>(a, x[2], 0, W, Kz, Dz);
    }
    const double br = (double)bref;
    v[0] = (double)pot + br * (Kx * Ky * Kz);
    v[1] = (double)gx + br * (Dx * Ky * Kz);
    v[2] = (double)gy + br * (Kx * Dy * Kz);
    v[3] = (double)gz + br * (Kx * Ky * Dz);
  } else {
    T ph[2][W];
    b1 = kernel_row<T, W>(a, x[1], ph[0]) - g.l0;
    b2 = kernel_row<T, W>(a, x[2], ph[1]) - g.l0;
    b1 = b1 < 0 ? 0 : (b1 > g.G - W ? g.G - W : b1);
    b2 = b2 < 0 ? 0 : (b2 > g.G - W ? g.G - W : b2);
    const T* row0 = B + b1 * g.str[1] + b2;
    T acc = T(0);
#pragma unroll 1
    for (int jx = jlo; jx < jhi; jx++) {
      const T px = es_kernel<T>((f0x + (T)jx) * a.inv_hw, a.beta);
      const T* rx = row0 + (bx + jx - x0) * g.str[0];
      T sx = T(0);
#pragma unroll
      for (int jy = 0; jy < W; jy++) {
        const T* ln = rx + jy * g.str[1];
        T sy = T(0);
#pragma unroll
        for (int jz = 0; jz < W; jz++) sy += ln[jz] * ph[1][jz];
        sx += sy * ph[0][jy];
      }
      acc += sx * px;
    }
    v[0] = (double)acc;
  }
  return true;
}

template <typename T, int W, bool DERIV>
__global__ void __launch_bounds__(PW_THREADS) k_eval_slab(PWArgs<T> a, EvalPtrs<T> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Geo& g = a.g;
  const int K = g.K, NF = 2 * K + 1, NH = K + 1, G = g.G;
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int Gp = pad4(G);
  const T* tif = stage_tw(sm, a.tif, 2 * NF * Gp);
  const T* tih = stage_tw(sm + 2 * NF * Gp, a.tih, 2 * NH * Gp);
  int* ordtmp = reinterpret_cast<int*>(sm + tw_elems_t<T>(G, K));       // ORDER_CHUNK
  int* ordcnt = ordtmp + ORDER_CHUNK;                                    // 32
  unsigned short* perm = reinterpret_cast<unsigned short*>(ordcnt + 32);  // ORDER_CHUNK
  T* B = reinterpret_cast<T*>(smem_raw + order_offset<T>(G, K));       // p.slab planes
  const int C = p.nslab, nline = NF * NH;
  __syncthreads();
  __shared__ int s_next;
  const int n_items = *p.n_items;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_next = atomicAdd(p.next, 1);
    __syncthreads();
    if (s_next >= n_items) break;
    const WorkItem it = p.items[s_next];
    const int e = it.slot;
    if (!FGT_DCHECK(e >= 0 && e < p.nbox && it.nparts % C == 0, 305)) continue;
    const int box = p.eval_box[e];
    const int x0 = (it.part % C) * p.slab, x1 = min(G, x0 + p.slab), np_ = x1 - x0;
    if (!FGT_DCHECK(np_ > 0 && np_ <= p.slab, 306)) continue;
    for (int id = 0; id < p.nd; id++) {
      const T* L = p.loc + ((size_t)e * p.nd + id) * 2 * g.nexp;
      for (int c = 0; c < (DERIV ? 1 : p.ncomp_max); c++) {
        // the x transform at the slab's planes (factors as build_eval_grid)
        for (int o = threadIdx.x; o < np_ * nline; o += blockDim.x) {
          const int xl = o / nline, line = o - xl * nline;
          const int kyi = line / NH, kz = line - kyi * NH;
          const T fyz = a.faci[kyi] * a.faci[kz + K];
          const T* tw = tif + x0 + xl;
          T re = T(0), im = T(0);
          for (int kx = 0; kx < NF; kx++, tw += 2 * Gp) {
            const int m = kx * nline + line;
            const int ki[3] = {kx, kyi, kz + K};
            T fr, fi;
            eval_factor<T, 3>(a, c, ki, fr, fi);
            const T f = a.faci[kx] * fyz;
            fr *= f;
            fi *= f;
            const T lr = L[2 * m], li = L[2 * m + 1];
            const T vr = lr * fr - li * fi, vi = lr * fi + li * fr;
            const T tr = tw[0], ti = tw[Gp];
            re += vr * tr - vi * ti;
            im += vr * ti + vi * tr;
          }
          T* bo = B + xl * g.str[0] + kyi * g.str[1] + 2 * kz;
          bo[0] = re;
          bo[1] = im;
        }
        __syncthreads();
        pass_inplace<T, 1>(B, np_ * NH, NH, g.str[0], 2, g.str[1], g.str[1], NF, G, tif);
        pass_inplace<T, 2>(B, np_ * G, G, g.str[0], g.str[1], 2, 1, NH, G, tih);
        for (int set = 0; set < 2; set++) {
          const int ne = set ? p.n[1] : p.n[0];
          if (c >= (set ? p.ncomp[1] : p.ncomp[0]) || ne == 0) continue;
          const double* offs = set ? p.off[1] : p.off[0];
          double* outs = set ? p.out[1] : p.out[0];
          const int nc = set ? p.ncomp[1] : p.ncomp[0];
          int q0, q1;
          part_range(set ? p.lo[1][box] : p.lo[0][box], set ? p.hi[1][box] : p.hi[0][box],
                     it.part / C, it.nparts / C, q0, q1);
          if (!FGT_DCHECK(q0 >= 0 && q0 <= q1 && q1 <= ne, 307)) continue;
          for (int c0 = q0; c0 < q1; c0 += ORDER_CHUNK) {
            const int n = min(ORDER_CHUNK, q1 - c0);
            order_chunk<T, 3, W>(a, offs, ne, c0, n, perm, ordtmp, ordcnt);
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
              const int pt = c0 + perm[i];
              double x[3];
#pragma unroll
              for (int k = 0; k < 3; k++) x[k] = offs[(size_t)k * ne + pt] * a.scale_d;
              double v[4];
              if (!interp_slab<T, W, DERIV>(a, B, x, x0, x1, v)) continue;
              if constexpr (DERIV) {
                atomicAdd(&outs[(size_t)id * ne + pt], v[0]);
                if (nc > 1) {
#pragma unroll
                  for (int d = 0; d < 3; d++)
                    atomicAdd(&outs[((size_t)(1 + d) * p.nd + id) * ne + pt], v[1 + d]);
                }
              } else {
                atomicAdd(&outs[((size_t)c * p.nd + id) * ne + pt], v[0]);
              }
            }
            __syncthreads();
          }
        }
        __syncthreads();
      }
    }
  }
}

// Direct modal evaluation for boxes with few points (at most pmax points of
// both evaluation sets together), one CTA per box:
//   u(x) = Re sum_m w(m) L_m e^{i k_m . x},  w = 1 on the kz = 0 plane and 2
// elsewhere (Hermitian half space).  The phase factors e^{i k x_d} of the
// box's points are computed once (FP64 sincos, stored as T, point index
// fastest).  Mode rows (kx, ky) are summed over the last dimension.  Lanes
// are (point, row subgroup) pairs for up to 32 points at a time, so a thread
// accumulates one point over many rows in registers and the lanes of a warp
// read at most 32/npoints distinct expansion rows per load; the partials of
// all threads are added once per box in FP64.
template <typename T, int DIM>
__global__ void __launch_bounds__(MODAL_THREADS) k_eval_modal(PWArgs<T> a, EvalPtrs<T> p,
                                                              int pmax) {
  constexpr int NHS = DIM * (DIM + 1) / 2, NCM = 1 + DIM + NHS;
  constexpr int NW = MODAL_THREADS / 32;
  const Geo& g = a.g;
  const int K = g.K, NF = 2 * K + 1, NH = K + 1, NE = DIM * NF;
  const int nrows = g.nexp / NH;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* red = reinterpret_cast<double*>(smem_raw);        // [NW][32][NCM]
  T* E = reinterpret_cast<T*>(red + (size_t)NW * 32 * NCM);  // [NE][pmax] complex
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nbox = p.nbox_dev ? *p.nbox_dev : p.nbox;
  for (int bi = blockIdx.x; bi < nbox; bi += gridDim.x) {
    const int e = p.boxes[bi];
    const int box = p.eval_box[e];
    const int n0 = p.n[0] > 0 && p.ncomp[0] > 0 ? p.hi[0][box] - p.lo[0][box] : 0;
    const int n1 = p.n[1] > 0 && p.ncomp[1] > 0 ? p.hi[1][box] - p.lo[1][box] : 0;
    const int np = n0 + n1;  // <= pmax by the box split
    const int ncmax = max(n0 ? p.ncomp[0] : 0, n1 ? p.ncomp[1] : 0);
    __syncthreads();
    for (int i = threadIdx.x; i < np * NE; i += blockDim.x) {
      const int r = i / np, pi = i - r * np, d = r / NF, k = r - d * NF - K;
      const int set = pi < n0 ? 0 : 1;
      const int pt = set ? p.lo[1][box] + pi - n0 : p.lo[0][box] + pi;
      const double* offs = set ? p.off[1] : p.off[0];
      const int ne = set ? p.n[1] : p.n[0];
      const double x = offs[(size_t)d * ne + pt] * a.scale_d;
      double sn, cs;
      sincos(x * (double)k, &sn, &cs);
      E[2 * ((size_t)r * pmax + pi)] = (T)cs;
      E[2 * ((size_t)r * pmax + pi) + 1] = (T)sn;
    }
    __syncthreads();
    for (int id = 0; id < p.nd; id++) {
      const T* L = p.loc + ((size_t)e * p.nd + id) * 2 * g.nexp;
      // one row partition for every point of the box, so that equal points
      // (a source that is also a target) get bitwise equal sums
      const int nsub = 32 / max(1, min(32, np));
      for (int p0 = 0; p0 < np; p0 += 32) {
        const int npg = min(32, np - p0);
        const int pi = p0 + lane % npg, sub = lane / npg;
        const bool act = sub < nsub;
        const T* Ex = E + 2 * (size_t)pi;  // + 2 * pmax * r for row r of E
        const T* El = E + 2 * ((size_t)((DIM - 1) * NF + K) * pmax + pi);
        T v[NCM];
#pragma unroll
        for (int c = 0; c < NCM; c++) v[c] = T(0);
        if (act) {
          for (int r = warp * nsub + sub; r < nrows; r += NW * nsub) {
            int ki[3] = {0, 0, 0};
            if (DIM == 3) {
              ki[0] = r / NF;
              ki[1] = r - ki[0] * NF;
            } else if (DIM == 2) {
              ki[0] = r;
            }
            const T* Lr = L + 2 * (size_t)r * NH;
            T s0r = T(0), s0i = T(0), s1r = T(0), s1i = T(0), s2r = T(0), s2i = T(0);
#pragma unroll 4
            for (int kz = 0; kz < NH; kz++) {
              const T w = kz == 0 ? T(1) : T(2);
              const T lr = __ldg(Lr + 2 * kz) * w, li = __ldg(Lr + 2 * kz + 1) * w;
              const T er = El[2 * (size_t)kz * pmax], ei = El[2 * (size_t)kz * pmax + 1];
              const T tr = lr * er - li * ei, ti = lr * ei + li * er;
              s0r += tr;
              s0i += ti;
              if (ncmax > 1) {
                const T t = a.ts[K + kz];
                s1r += t * tr;
                s1i += t * ti;
                if (ncmax > 1 + DIM) {
                  s2r += t * t * tr;
                  s2i += t * t * ti;
                }
              }
            }
            T pr = T(1), pim = T(0);  // phase of the row in the other dimensions
#pragma unroll
            for (int d = 0; d < DIM - 1; d++) {
              const size_t o = 2 * (size_t)(d * NF + ki[d]) * pmax;
              const T cr = Ex[o], ci = Ex[o + 1];
              const T nr = pr * cr - pim * ci;
              pim = pr * ci + pim * cr;
              pr = nr;
            }
            const T t0r = pr * s0r - pim * s0i, t0i = pr * s0i + pim * s0r;
            v[0] += t0r;
            if (ncmax > 1) {
              const T t1r = pr * s1r - pim * s1i, t1i = pr * s1i + pim * s1r;
#pragma unroll
              for (int d = 0; d < DIM - 1; d++) v[1 + d] -= t0i * a.ts[ki[d]];
              v[DIM] -= t1i;
              if (ncmax > 1 + DIM) {
                const T t2r = pr * s2r - pim * s2i;
#pragma unroll
                for (int hm = 0; hm < NHS; hm++) {
                  int pp, qq;
                  if (DIM == 1) { pp = 0; qq = 0; }
                  else if (DIM == 2) { pp = (hm == 2) ? 1 : 0; qq = (hm == 0) ? 0 : 1; }
                  else { pp = hm < 3 ? hm : (hm < 5 ? 0 : 1); qq = hm < 3 ? hm : (hm == 3 ? 1 : 2); }
                  const bool lp = pp == DIM - 1, lq = qq == DIM - 1;
                  T h;
                  if (lp && lq) h = t2r;
                  else if (lp) h = t1r * a.ts[sel3(ki, qq)];
                  else if (lq) h = t1r * a.ts[sel3(ki, pp)];
                  else h = t0r * a.ts[sel3(ki, pp)] * a.ts[sel3(ki, qq)];
                  v[1 + DIM + hm] -= h;
                }
              }
            }
          }
        }
#pragma unroll
        for (int c = 0; c < NCM; c++) red[((size_t)warp * 32 + lane) * NCM + c] = (double)v[c];
        __syncthreads();
        const double s1 = (double)a.inv_sqd0, s2 = s1 * s1;
        for (int i = threadIdx.x; i < npg * NCM; i += blockDim.x) {
          const int q = i / NCM, c = i - q * NCM, pj = p0 + q;
          const int set = pj < n0 ? 0 : 1;
          if (c >= (set ? p.ncomp[1] : p.ncomp[0])) continue;
          double v2 = 0;
          for (int w = 0; w < NW; w++)
            for (int sb = 0; sb < nsub; sb++) v2 += red[((size_t)w * 32 + sb * npg + q) * NCM + c];
          v2 *= c == 0 ? 1.0 : (c <= DIM ? s1 : s2);
          const int ne = set ? p.n[1] : p.n[0];
          const int pt = set ? p.lo[1][box] + pj - n0 : p.lo[0][box] + pj;
          double* outs = set ? p.out[1] : p.out[0];
          outs[((size_t)c * p.nd + id) * ne + pt] += v2;
        }
        __syncthreads();
      }
    }
  }
}

// FP32 modal evaluation (potential, or potential + gradient) of the boxes
// with few points: the sums of k_eval_modal, with the box's expansion
// streamed through shared memory in chunks of whole rows (register
// prefetch of the next chunk while the current one is summed), stored as
// (w lr, w lr, -w li, w li) so that one 128-bit broadcast load and two packed
// FP32x2 FMAs against the point's (er, ei) and (ei, er) give the complex
// product of a mode; the point's factors are one 8-byte load per mode (the
// shared-memory traffic of the loop is mostly these per-lane loads).  Rows,
// lanes and the FP64 reduction as in k_eval_modal.
constexpr int MODAL_CHUNK = 1024;  // modes per staged chunk (whole rows)
template <int DIM>
__host__ __device__ constexpr int modal32_ncg() { return 1 + DIM; }
template <int DIM>
size_t modal32_smem(int K, int pmax) {
  const int NF = 2 * K + 1, NH = K + 1;
  return sizeof(double) * (MODAL_THREADS / 32) * 32 * modal32_ncg<DIM>() +
         sizeof(float4) * ((size_t)NH * pmax + 2 * MODAL_CHUNK) +
         sizeof(float2) * ((size_t)(DIM - 1) * NF * pmax + NH);
}

template <int DIM, bool GRAD>
__global__ void __launch_bounds__(MODAL_THREADS) k_eval_modal32(PWArgs<float> a, EvalPtrs<float> p,
                                                                int pmax) {
  constexpr int NCG = modal32_ncg<DIM>();
  constexpr int NW = MODAL_THREADS / 32;
  const Geo& g = a.g;
  const int K = g.K, NF = 2 * K + 1, NH = K + 1;
  const int nrows = g.nexp / NH;
  const int rpc = max(1, MODAL_CHUNK / NH);  // rows per chunk
  const int nch = (nrows + rpc - 1) / rpc;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* red = reinterpret_cast<double*>(smem_raw);                 // [NW][32][NCG]
  // [NH][pmax] (cos, sin) of the last dimension (in a region sized for float4)
  float2* Ez = reinterpret_cast<float2*>(red + (size_t)NW * 32 * NCG);
  float4* Lb = reinterpret_cast<float4*>(Ez) + (size_t)NH * pmax;     // [2][MODAL_CHUNK]
  float2* Exy = reinterpret_cast<float2*>(Lb + 2 * MODAL_CHUNK);      // [(DIM-1) NF][pmax]
  float2* T2 = Exy + (size_t)(DIM - 1) * NF * pmax;                   // [NH] (t, t)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int kz = threadIdx.x; kz < NH; kz += blockDim.x) T2[kz] = make_float2(a.ts[K + kz], a.ts[K + kz]);
  const int nbox = p.nbox_dev ? *p.nbox_dev : p.nbox;
  for (int bi = blockIdx.x; bi < nbox; bi += gridDim.x) {
    const int e = p.boxes[bi];
    const int box = p.eval_box[e];
    const int n0 = p.n[0] > 0 && p.ncomp[0] > 0 ? p.hi[0][box] - p.lo[0][box] : 0;
    const int n1 = p.n[1] > 0 && p.ncomp[1] > 0 ? p.hi[1][box] - p.lo[1][box] : 0;
    const int np = n0 + n1;  // <= pmax by the box split
    __syncthreads();
    // phase factors e^{i k x_d}: FP64 sincos, stored as FP32
    for (int i = threadIdx.x; i < np * DIM * NF; i += blockDim.x) {
      const int r = i / np, pi = i - r * np, d = r / NF, k = r - d * NF - K;
      if (d == DIM - 1 && k < 0) continue;
      const int set = pi < n0 ? 0 : 1;
      const int pt = set ? p.lo[1][box] + pi - n0 : p.lo[0][box] + pi;
      const double* offs = set ? p.off[1] : p.off[0];
      const int ne = set ? p.n[1] : p.n[0];
      const double x = offs[(size_t)d * ne + pt] * a.scale_d;
      double sn, cs;
      sincos(x * (double)k, &sn, &cs);
      const float c = (float)cs, sv = (float)sn;
      if (d == DIM - 1) Ez[(size_t)k * pmax + pi] = make_float2(c, sv);
      else Exy[(size_t)r * pmax + pi] = make_float2(c, sv);
    }
    for (int id = 0; id < p.nd; id++) {
      const float2* L = reinterpret_cast<const float2*>(p.loc + ((size_t)e * p.nd + id) * 2 * g.nexp);
      const int nsub = 32 / max(1, min(32, np));
      const int S = NW * nsub;  // row streams
      for (int p0 = 0; p0 < np; p0 += 32) {
        const int npg = min(32, np - p0);
        const int pi = p0 + lane % npg, sub = lane / npg;
        const bool act = sub < nsub;
        const int rs = warp * nsub + sub;
        float v[NCG];
#pragma unroll
        for (int c = 0; c < NCG; c++) v[c] = 0.f;
        // chunk 0 to shared memory; later chunks prefetched into registers
        float2 pf[MODAL_CHUNK / MODAL_THREADS];
        auto fetch = [&](int c) {
          const int m0 = c * rpc * NH, m1 = min(g.nexp, m0 + rpc * NH);
#pragma unroll
          for (int j = 0; j < MODAL_CHUNK / MODAL_THREADS; j++) {
            const int m = m0 + threadIdx.x + j * MODAL_THREADS;
            pf[j] = m < m1 ? __ldg(L + m) : make_float2(0.f, 0.f);
          }
        };
        auto stage = [&](int c, float4* buf) {
          const int m0 = c * rpc * NH;
#pragma unroll
          for (int j = 0; j < MODAL_CHUNK / MODAL_THREADS; j++) {
            const int mm = threadIdx.x + j * MODAL_THREADS;
            const float w = ((m0 + mm) % NH) == 0 ? 1.f : 2.f;
            buf[mm] = make_float4(w * pf[j].x, w * pf[j].x, -w * pf[j].y, w * pf[j].y);
          }
        };
        __syncthreads();
        fetch(0);
        stage(0, Lb);
        __syncthreads();
        for (int c = 0; c < nch; c++) {
          if (c + 1 < nch) fetch(c + 1);
          const float4* Lc = Lb + (c & 1) * MODAL_CHUNK;
          const int r0 = c * rpc, r1 = min(nrows, r0 + rpc);
          if (act) {
            for (int r = r0 + ((rs - r0) % S + S) % S; r < r1; r += S) {
              const float4* Lr = Lc + (size_t)(r - r0) * NH;
              const float2* Ep = Ez + pi;
              float2 s0 = make_float2(0.f, 0.f), s1 = make_float2(0.f, 0.f);
#pragma unroll 4
              for (int kz = 0; kz < NH; kz++) {
                const float4 L4 = Lr[kz];
                const float2 e2 = Ep[(size_t)kz * pmax];
                float2 pr = __fmul2_rn(make_float2(L4.x, L4.y), e2);
                pr = __ffma2_rn(make_float2(L4.z, L4.w), make_float2(e2.y, e2.x), pr);
                s0 = __fadd2_rn(s0, pr);
                if (GRAD) s1 = __ffma2_rn(T2[kz], pr, s1);
              }
              int ki[2] = {0, 0};
              if (DIM == 3) {
                ki[0] = r / NF;
                ki[1] = r - ki[0] * NF;
              } else if (DIM == 2) {
                ki[0] = r;
              }
              float pr = 1.f, pim = 0.f;  // phase of the row in the other dimensions
#pragma unroll
              for (int d = 0; d < DIM - 1; d++) {
                const float2 cc = Exy[(size_t)(d * NF + ki[d]) * pmax + pi];
                const float nr = pr * cc.x - pim * cc.y;
                pim = pr * cc.y + pim * cc.x;
                pr = nr;
              }
              const float t0r = pr * s0.x - pim * s0.y, t0i = pr * s0.y + pim * s0.x;
              v[0] += t0r;
              if (GRAD) {
                const float t1i = pr * s1.y + pim * s1.x;
#pragma unroll
                for (int d = 0; d < DIM - 1; d++) v[1 + d] -= t0i * a.ts[ki[d]];
                v[DIM] -= t1i;
              }
            }
          }
          if (c + 1 < nch) stage(c + 1, Lb + ((c + 1) & 1) * MODAL_CHUNK);
          __syncthreads();
        }
#pragma unroll
        for (int c = 0; c < NCG; c++) red[((size_t)warp * 32 + lane) * NCG + c] = (double)v[c];
        __syncthreads();
        const double s1 = (double)a.inv_sqd0;
        for (int i = threadIdx.x; i < npg * NCG; i += blockDim.x) {
          const int q = i / NCG, c = i - q * NCG, pj = p0 + q;
          const int set = pj < n0 ? 0 : 1;
          if (c >= (set ? p.ncomp[1] : p.ncomp[0])) continue;
          double v2 = 0;
          for (int w = 0; w < NW; w++)
            for (int sb = 0; sb < nsub; sb++) v2 += red[((size_t)w * 32 + sb * npg + q) * NCG + c];
          v2 *= c == 0 ? 1.0 : s1;
          const int ne = set ? p.n[1] : p.n[0];
          const int pt = set ? p.lo[1][box] + pj - n0 : p.lo[0][box] + pj;
          double* outs = set ? p.out[1] : p.out[0];
          outs[((size_t)c * p.nd + id) * ne + pt] += v2;
        }
      }
    }
  }
}

// Evaluation of small 2D boxes, one warp per box (see small2_layout): the
// grid boxes boxes[first..*nbox_dev) of the longest-processing-time order,
// which hold at most SMALL2_MAX points.  Potential only, or potential and
// gradient through the kernel derivative (DERIV); same sums as k_eval_comp.
template <typename T, int W, bool DERIV>
__global__ void __launch_bounds__(256) k_eval_small2(PWArgs<T> a, EvalPtrs<T> p,
                                                     const int* __restrict__ first,
                                                     int* __restrict__ next) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Geo& g = a.g;
  const int K = g.K, NF = 2 * K + 1, NH = K + 1, G = g.G, Gp = pad4(G);
  T* sm = reinterpret_cast<T*>(smem_raw);
  const T* tif = stage_tw(sm, a.tif, 2 * NF * Gp);
  const T* tih = stage_tw(sm + 2 * NF * Gp, a.tih, 2 * NH * Gp);
  const Small2Layout lay = small2_layout(G, K);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* R1 = reinterpret_cast<T*>(smem_raw + tw_bytes16<T>(G, K)) + (size_t)warp * lay.per_warp;
  T* R2 = R1 + lay.r1;
  Geo gw = g;  // the warp's real grid: rows of SA values, y contiguous
  gw.str[0] = lay.SA;
  gw.str[1] = 1;
  __syncthreads();
  const int f0 = *first, nbox = *p.nbox_dev;
  for (;;) {
    int bi = 0;
    if (lane == 0) bi = atomicAdd(next, 1);
    bi = __shfl_sync(0xffffffffu, bi, 0) + f0;
    if (bi >= nbox) break;
    const int e = p.boxes[bi];
    if (!FGT_DCHECK(e >= 0 && e < p.nbox, 303)) continue;
    const int box = p.eval_box[e];
    for (int id = 0; id < p.nd; id++) {
      const T* L = p.loc + ((size_t)e * p.nd + id) * 2 * g.nexp;
      for (int m = lane; m < g.nexp; m += 32) {
        const int kxi = m / NH, ky = m - kxi * NH;
        const T f = a.faci[kxi] * a.faci[ky + K];
        R1[kxi * lay.SC + 2 * ky] = L[2 * m] * f;
        R1[kxi * lay.SC + 2 * ky + 1] = L[2 * m + 1] * f;
      }
      __syncwarp();
      warp_pass_c2c<T>(R1, lay.SC, NF, G, NH, tif, [&](int x, int ky, T re, T im) {
        R2[x * lay.SC + 2 * ky] = re;
        R2[x * lay.SC + 2 * ky + 1] = im;
      });
      __syncwarp();
      warp_pass_c2r<T>(R2, lay.SC, R1, lay.SA, G, NH, tih);
      __syncwarp();
      const T* B = R1;
      for (int set = 0; set < 2; set++) {
        const int ne = set ? p.n[1] : p.n[0];
        const int nc = set ? p.ncomp[1] : p.ncomp[0];
        if (nc == 0 || ne == 0) continue;
        const double* offs = set ? p.off[1] : p.off[0];
        double* outs = set ? p.out[1] : p.out[0];
        const int q0 = set ? p.lo[1][box] : p.lo[0][box];
        const int q1 = set ? p.hi[1][box] : p.hi[0][box];
        if (!FGT_DCHECK(q0 >= 0 && q0 <= q1 && q1 <= ne, 304)) continue;
        for (int q = q0 + lane; q < q1; q += 32) {
          double x[2];
          x[0] = offs[q] * a.scale_d;
          x[1] = offs[(size_t)ne + q] * a.scale_d;
          T ph[2][W];
          int sc[2];
          if constexpr (DERIV) {
            T dph[2][W], v[3];
            sc[0] = kernel_row_d<T, W>(a, x[0], ph[0], dph[0]);
            sc[1] = kernel_row_d<T, W>(a, x[1], ph[1], dph[1]);
            interp_grad_cells<T, 2, W>(B, LinIdx<2, W>(gw, sc), ph, dph, v);
            outs[(size_t)id * ne + q] += (double)v[0];
            if (nc > 1) {
              outs[((size_t)1 * p.nd + id) * ne + q] += (double)v[1];
              outs[((size_t)2 * p.nd + id) * ne + q] += (double)v[2];
            }
          } else {
            sc[0] = kernel_row<T, W>(a, x[0], ph[0]);
            sc[1] = kernel_row<T, W>(a, x[1], ph[1]);
            outs[(size_t)id * ne + q] += (double)interp_cells<T, 2, W>(B, LinIdx<2, W>(gw, sc), ph);
          }
        }
      }
      __syncwarp();
    }
  }
}

// First entry of a list sorted by k_lpt_keys (ascending keys = descending
// point counts) whose box holds at most `limit` points.
__global__ void k_first_at_most_e(const uint64_t* __restrict__ keys, int n, int limit,
                                  int* __restrict__ out) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    constexpr uint64_t MAXC = (1ull << (LPT_BITS - 1)) - 1;
    const uint64_t v = MAXC - (uint64_t)limit;  // count <= limit  <=>  key >= v
    int lo = 0, hi = n;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (keys[mid] < v) lo = mid + 1; else hi = mid;
    }
    *out = lo;
  }
}

// box partition by evaluation-point count
__global__ void k_eval_split(int n_eval, const int* __restrict__ eval_box, const int* __restrict__ lo0,
                             const int* __restrict__ hi0, const int* __restrict__ lo1,
                             const int* __restrict__ hi1, int thr, int* __restrict__ big,
                             unsigned long long* __restrict__ cnt) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_eval; e += gridDim.x * blockDim.x) {
    int b = eval_box[e];
    int n = (lo0 ? hi0[b] - lo0[b] : 0) + (lo1 ? hi1[b] - lo1[b] : 0);
    big[e] = n > thr ? 1 : 0;
    atomicAdd(&cnt[n > thr ? 0 : 1], (unsigned long long)n);
  }
}
__global__ void k_split_fill(int n, const int* __restrict__ f, const int* __restrict__ pos,
                             int* __restrict__ big_list, int* __restrict__ small_list,
                             const int* __restrict__ nbig, int* __restrict__ counts) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    counts[0] = *nbig;
    counts[1] = n - *nbig;
  }
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    if (f[e]) big_list[pos[e]] = e;
    else small_list[e - pos[e]] = e;
  }
}

template <typename T, int DIM, int W, bool DERIV>
int launch_eval_k(PWArgs<T>& a, const EvalPtrs<T>& ep, DBuf<T>& gs, cudaStream_t s) {
  size_t fix = eval_offset<T>(a.g.G, a.g.K);
  size_t need = fix + sizeof(T) * (size_t)a.g.bufsz;
  int grid = std::max(1, std::min(ep.max_items, kSMs));
  bool gb = need > (size_t)MAXSMEM;
  EvalPtrs<T> epk = ep;
  {  // cell order when the sub-grid's base cells fit the bins
    const long nb = a.g.G - W + 1;
    long nbins = 1;
    for (int d = 0; d < DIM; d++) nbins *= nb;
    // order_cells spreads the bins over whole rounds of the CTA's threads
    const long nthr = eval_threads<T, DIM, W, false, DERIV>();
    const long padded = (nbins + nthr - 1) / nthr * nthr;
    epk.cell_bins =
        (sizeof(T) == 4 && !a.g.wrap && nb > 0 && padded <= NBINS_MAX) ? (int)nbins : 0;
  }
  if constexpr (DIM == 3) {
    if (gb && ep.nslab > 1) {  // x-slab grids
      const size_t ss = order_offset<T>(a.g.G, a.g.K) + sizeof(T) * (size_t)a.g.str[0] * ep.slab;
      auto k = k_eval_slab<T, W, DERIV>;
      set_smem(k, ss);
      k<<<grid, PW_THREADS, ss, s>>>(a, epk);
      FGT_LAUNCH_CHECK();
      return 1;
    }
  }
  if (gb) {
    gs.alloc((size_t)grid * a.g.bufsz, s);
    a.gscratch = gs;
  }
  size_t sm = gb ? fix : need;
  if (gb) {
    auto k = k_eval_comp<T, DIM, W, true, DERIV>;
    set_smem(k, sm);
    k<<<grid, eval_threads<T, DIM, W, true, DERIV>(), sm, s>>>(a, epk);
  } else {
    auto k = k_eval_comp<T, DIM, W, false, DERIV>;
    set_smem(k, sm);
    k<<<grid, eval_threads<T, DIM, W, false, DERIV>(), sm, s>>>(a, epk);
  }
  FGT_LAUNCH_CHECK();
  return 1;
}

template <typename T>
int small2_eval_warps(const Geo& g, size_t& smem) {
  const Small2Layout lay = small2_layout(g.G, g.K);
  const size_t fix = tw_bytes16<T>(g.G, g.K);
  const size_t per = sizeof(T) * (size_t)lay.per_warp;
  if (fix + per > (size_t)MAXSMEM) return 0;
  const int nw = (int)std::min<size_t>(8, ((size_t)MAXSMEM - fix) / per);
  smem = fix + per * nw;
  return nw;
}
template <typename T, int W, bool DERIV>
void launch_eval_small2(PWArgs<T>& a, const EvalPtrs<T>& ep, const int* first, int* next,
                        cudaStream_t s) {
  size_t smem = 0;
  const int nw = small2_eval_warps<T>(a.g, smem);
  auto k = k_eval_small2<T, W, DERIV>;
  set_smem(k, smem);
  // as many 8-warp CTAs per SM as the shared memory allows (the warps of a
  // CTA share only the staged tables; more CTAs hide more latency)
  const int per_sm = std::max(1, std::min(8, (int)((size_t)(228 * 1024) / (smem + 1024))));
  k<<<kSMs * per_sm, 32 * nw, smem, s>>>(a, ep, first, next);
  FGT_LAUNCH_CHECK();
}
template <typename T>
void eval_small2_w(int w, bool deriv, PWArgs<T>& a, const EvalPtrs<T>& ep, const int* first,
                   int* next, cudaStream_t s) {
#define FGT_S2(WW)                                                              \
  case WW:                                                                      \
    if (deriv) launch_eval_small2<T, WW, true>(a, ep, first, next, s);          \
    else launch_eval_small2<T, WW, false>(a, ep, first, next, s);               \
    return;
  switch (w) {
    FGT_S2(6) FGT_S2(7) FGT_S2(8) FGT_S2(9) FGT_S2(10) FGT_S2(12) FGT_S2(14) FGT_S2(16)
    default: FGT_REQUIRE(false, FGT_ERR_UNSUPPORTED, "no evaluation kernel for this width");
  }
#undef FGT_S2
}

// deriv: gradients through the kernel derivative (widths 8..16 only)
template <typename T, int DIM, int W>
int launch_eval(PWArgs<T>& a, const EvalPtrs<T>& ep, bool deriv, DBuf<T>& gs, cudaStream_t s) {
  if constexpr (W % 2 == 1) {  // odd widths: FP32 derivative evaluation only
    FGT_REQUIRE(deriv && sizeof(T) == 4, FGT_ERR_UNSUPPORTED, "odd kernel width outside the FP32 gradient path");
    if constexpr (sizeof(T) == 4) return launch_eval_k<T, DIM, W, true>(a, ep, gs, s);
    return 0;
  } else {
    if constexpr (W >= 8) {
      if (deriv) return launch_eval_k<T, DIM, W, true>(a, ep, gs, s);
    }
    FGT_REQUIRE(!deriv, FGT_ERR_UNSUPPORTED, "derivative evaluation needs a kernel width >= 7");
    return launch_eval_k<T, DIM, W, false>(a, ep, gs, s);
  }
}

template <typename T, int DIM>
int eval_w(int w, PWArgs<T>& a, const EvalPtrs<T>& ep, bool deriv, DBuf<T>& gs, cudaStream_t s) {
  switch (w) {
    case 6: return launch_eval<T, DIM, 6>(a, ep, deriv, gs, s);
    case 7: return launch_eval<T, DIM, 7>(a, ep, deriv, gs, s);
    case 8: return launch_eval<T, DIM, 8>(a, ep, deriv, gs, s);
    case 9: return launch_eval<T, DIM, 9>(a, ep, deriv, gs, s);
    case 10: return launch_eval<T, DIM, 10>(a, ep, deriv, gs, s);
    case 12: return launch_eval<T, DIM, 12>(a, ep, deriv, gs, s);
    case 14: return launch_eval<T, DIM, 14>(a, ep, deriv, gs, s);
    case 16: return launch_eval<T, DIM, 16>(a, ep, deriv, gs, s);
    default: FGT_REQUIRE(false, FGT_ERR_UNSUPPORTED, "no evaluation kernel for this width");
  }
  return 0;
}
template <typename T>
int eval_dim(int dim, int w, PWArgs<T>& a, const EvalPtrs<T>& ep, bool deriv, DBuf<T>& gs,
             cudaStream_t s) {
  if (dim == 1) return eval_w<T, 1>(w, a, ep, deriv, gs, s);
  if (dim == 2) return eval_w<T, 2>(w, a, ep, deriv, gs, s);
  return eval_w<T, 3>(w, a, ep, deriv, gs, s);
}

}  // namespace

template <typename T>
int pw_eval(const PWParams& P, const Tree& t, const Lists& L, const PWData<T>& D,
            const EvalSet<T>& e0, const EvalSet<T>& e1, int small_eval, PWWork* work,
            cudaStream_t s) {
  // both evaluation sets (sources, targets) share the grid of every box
  const bool u0 = e0.pgh > 0 && e0.n > 0, u1 = e1.pgh > 0 && e1.n > 0;
  if (!(u0 || u1) || L.n_eval <= 0) return 0;
  const int pgh_max = std::max(u0 ? e0.pgh : 0, u1 ? e1.pgh : 0);
  // Grids of the evaluation: potential only (width w); potential and
  // gradient from one grid through the kernel derivative, whose aliasing
  // error at width w+2 is below that of the potential at width w; one grid
  // per output component (pot, grad_k, hess_kl) at width w when hessians are
  // requested or w+2 exceeds the widest kernel.
  // FP32: width w+1 (its aliasing error, ~1e-7 at eps = 1e-6, stays below
  // the FP32 rounding of the sums); FP64: w+2
  // The evaluation kernels exist for widths 6..10, 12, 14 and 16 (odd
  // widths 7 and 9 for the FP32 derivative only): an odd width above 9
  // (FP32 at eps < 1e-6) is rounded up to the next even one.
  int wgrad = P.w + (sizeof(T) == 4 ? 1 : 2);
  if (wgrad > 9 && (wgrad & 1)) wgrad++;
  const bool deriv = pgh_max == 2 && wgrad <= 16;
  const int mode = deriv ? 1 : 2;
  PWParams Pe = P;
  if (deriv) pw_grid(Pe, wgrad, true);
  PWArgs<T> a;
  DevTables<T> tb;
  make_args<T>(Pe, a, tb, s, false, 1);
  int launches = 0;
  // boxes with at most thr evaluation points use the modal sums; thr is
  // capped by the modal kernel's shared memory (per point: FP64 partials of
  // every warp and the phase factors)
  const int ncm = 1 + P.dim + P.dim * (P.dim + 1) / 2;
  const size_t modal_fix = sizeof(double) * MODAL_THREADS * ncm;
  const size_t modal_pt = sizeof(T) * 2 * (size_t)P.dim * (2 * P.K + 1);
  const int thr = std::min(small_eval >= 0 ? small_eval : (P.dim == 3 ? 48 : (P.dim == 2 ? 8 : 4)),
                           (int)((MAXSMEM - modal_fix) / modal_pt));
  DBuf<int> big(L.n_eval, s), pos(L.n_eval, s), tot(1, s);
  DBuf<unsigned long long> cnt(2, s);
  cnt.zero();
  k_eval_split<<<grid_for(L.n_eval, 256), 256, 0, s>>>(
      L.n_eval, L.eval_box, u0 ? e0.lo : nullptr, u0 ? e0.hi : nullptr, u1 ? e1.lo : nullptr,
      u1 ? e1.hi : nullptr, thr, big, cnt);
  FGT_LAUNCH_CHECK();
  exclusive_scan_i32(big, pos, L.n_eval, tot, s);
  // both lists sized for all eval boxes; the counts stay on the device
  DBuf<int> lbig(L.n_eval, s), lsmall(L.n_eval, s), counts(2, s);
  k_split_fill<<<grid_for(L.n_eval, 256), 256, 0, s>>>(L.n_eval, big, pos, lbig, lsmall, tot,
                                                        counts);
  FGT_LAUNCH_CHECK();
  launches += 3;
  int nh = P.dim * (P.dim + 1) / 2;
  auto ncomp = [&](int pgh) { return pgh <= 0 ? 0 : 1 + (pgh >= 2 ? P.dim : 0) + (pgh >= 3 ? nh : 0); };
  EvalPtrs<T> ep;
  ep.nbox_dev = nullptr;
  ep.next = nullptr;
  ep.loc = D.loc;
  ep.eval_box = L.eval_box;
  ep.nd = P.nd;
  const EvalSet<T>* es[2] = {&e0, &e1};
  bool us[2] = {u0, u1};
  for (int i = 0; i < 2; i++) {
    ep.off[i] = us[i] ? es[i]->off : nullptr;
    ep.lo[i] = us[i] ? es[i]->lo : nullptr;
    ep.hi[i] = us[i] ? es[i]->hi : nullptr;
    ep.out[i] = us[i] ? es[i]->out : nullptr;
    ep.n[i] = us[i] ? es[i]->n : 0;
    ep.ncomp[i] = us[i] ? ncomp(es[i]->pgh) : 0;
  }
  ep.ncomp_max = std::max(ep.ncomp[0], ep.ncomp[1]);
  ep.items = nullptr;
  ep.n_items = nullptr;
  ep.max_items = 0;
  // grids too large for shared memory: x-slabs (3D without wrap-around)
  SlabPlan sp;
  if (eval_offset<T>(a.g.G, a.g.K) + sizeof(T) * (size_t)a.g.bufsz > (size_t)MAXSMEM)
    sp = slab_plan(a.g, sizeof(T), order_offset<T>(a.g.G, a.g.K));
  ep.slab = sp.planes;
  ep.nslab = sp.nslab;
  if (work) work->slabs_eval = sp.nslab;
  ItemList il;
  DBuf<int> first2(1, s), next2(1, s);
  DBuf<T> gs;
  {
    // longest-processing-time order of the grid boxes (by point count)
    DBuf<uint64_t> okey(L.n_eval, s), otmp(L.n_eval, s);
    DBuf<uint32_t> vtmp(L.n_eval, s);
    DBuf<int> next(1, s);
    next.zero();
    k_lpt_keys<<<grid_for(L.n_eval, 256), 256, 0, s>>>(
        L.n_eval, counts.get(), L.eval_box, lbig, u0 ? e0.lo : e1.lo, u0 ? e0.hi : e1.hi,
        (u0 && u1) ? e1.lo : nullptr, (u0 && u1) ? e1.hi : nullptr, okey,
        reinterpret_cast<uint32_t*>(lbig.get()));
    FGT_LAUNCH_CHECK();
    radix_sort(okey, reinterpret_cast<uint32_t*>(lbig.get()), otmp, vtmp, L.n_eval, LPT_BITS, s);
    ep.boxes = lbig;
    ep.nbox = L.n_eval;
    ep.nbox_dev = counts.get();
    ep.next = next;
    // 2D: grid boxes with at most SMALL2_MAX points (a suffix of the order)
    // go to the warp-per-box kernel, the rest to the CTA kernel
    size_t sm2 = 0;
    const bool small2 = P.dim == 2 && !a.g.wrap && (deriv || ep.ncomp_max == 1) &&
                        small2_eval_warps<T>(a.g, sm2) > 0;
    if (small2) {
      next2.zero();
      k_first_at_most_e<<<1, 32, 0, s>>>(okey, L.n_eval, SMALL2_MAX, first2);
      FGT_LAUNCH_CHECK();
    }
    // boxes above the split threshold become several items
    const long long npts = (u0 ? (long long)e0.n : 0) + (u1 ? (long long)e1.n : 0);
    build_items(il, L.n_eval, small2 ? first2.get() : counts.get(),
                reinterpret_cast<const uint32_t*>(lbig.get()),
                L.eval_box, u0 ? e0.lo : e1.lo, u0 ? e0.hi : e1.hi, (u0 && u1) ? e1.lo : nullptr,
                (u0 && u1) ? e1.hi : nullptr, npts, eval_split_threshold(npts), false, s,
                sp.nslab);
    ep.items = il.items;
    ep.n_items = il.n_items;
    ep.max_items = il.max_items;
    launches += 6 + eval_dim<T>(P.dim, Pe.w, a, ep, deriv, gs, s);
    if (small2) {
      eval_small2_w<T>(Pe.w, deriv, a, ep, first2, next2, s);
      launches += 2;
    }
  }
  {
    ep.boxes = lsmall;
    ep.nbox = L.n_eval;
    ep.nbox_dev = counts.get() + 1;
    int grid = std::max(1, std::min(L.n_eval, kSMs * 8));
    size_t sm = modal_fix + modal_pt * (size_t)std::max(thr, 1);
    bool done = false;
    if constexpr (sizeof(T) == 4) {
      // FP32 without hessians: the staged-expansion kernel
      if (ep.ncomp_max <= 1 + P.dim && P.K + 1 <= MODAL_CHUNK) {
        const bool grad = ep.ncomp_max > 1;
        const int pm = std::max(thr, 1);
        auto go = [&](auto kern, size_t smb) {
          set_smem(kern, smb);
          kern<<<grid, MODAL_THREADS, smb, s>>>(a, ep, pm);
        };
        if (P.dim == 1) {
          const size_t smb = modal32_smem<1>(P.K, pm);
          if (grad) go(k_eval_modal32<1, true>, smb); else go(k_eval_modal32<1, false>, smb);
        } else if (P.dim == 2) {
          const size_t smb = modal32_smem<2>(P.K, pm);
          if (grad) go(k_eval_modal32<2, true>, smb); else go(k_eval_modal32<2, false>, smb);
        } else {
          const size_t smb = modal32_smem<3>(P.K, pm);
          if (grad) go(k_eval_modal32<3, true>, smb); else go(k_eval_modal32<3, false>, smb);
        }
        done = true;
      }
    }
    if (done) {
    } else if (P.dim == 1) {
      set_smem(k_eval_modal<T, 1>, sm);
      k_eval_modal<T, 1><<<grid, MODAL_THREADS, sm, s>>>(a, ep, thr);
    } else if (P.dim == 2) {
      set_smem(k_eval_modal<T, 2>, sm);
      k_eval_modal<T, 2><<<grid, MODAL_THREADS, sm, s>>>(a, ep, thr);
    } else {
      set_smem(k_eval_modal<T, 3>, sm);
      k_eval_modal<T, 3><<<grid, MODAL_THREADS, sm, s>>>(a, ep, thr);
    }
    FGT_LAUNCH_CHECK();
    launches++;
  }
  if (work) {
    unsigned long long h[2] = {0, 0};
    int hc[2] = {0, 0};
    FGT_CUDA(cudaMemcpyAsync(h, cnt.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    FGT_CUDA(cudaMemcpyAsync(hc, counts.get(), sizeof(hc), cudaMemcpyDeviceToHost, s));
    FGT_CUDA(cudaStreamSynchronize(s));
    const int nbig = hc[0];
    work->n_nufft += nbig;
    const double wd = pow((double)Pe.w, P.dim);
    const double grids = mode == 2 ? ep.ncomp_max : 1;
    // derivative mode: value and derivative sums along the last dimension
    const double fl_pt = mode == 1 ? 4.0 * wd : 2.0 * wd * grids;
    work->pts_nufft = (double)h[0];
    work->pts_modal = (double)h[1];
    work->flops_eval = (double)P.nd * (nbig * grids * pw_pass_flops(Pe) + (double)h[0] * fl_pt) +
                       (double)P.nd * ep.ncomp_max * (double)h[1] * P.nexp * 8.0;
    work->w_eval = Pe.w;
    work->G_eval = Pe.G;
  }
  return launches;
}

}  // namespace fgt
