// Plane-wave form (K6) and translate (K7) kernels and the host set-up of
// the plane-wave grids; shared device helpers are in fgt_pw_dev.cuh.
#include <math.h>

#include <algorithm>
#include <utility>
#include <vector>

#include "fgt_pw_dev.cuh"

namespace fgt {

namespace {

// ---------------------------------------------------------------- form
struct FormIO {
  int n_form, ns, nd, ncomp;  // ncomp: charge (1) and/or dipole (dim)
  int has_q, has_dip;
  const int *form_box, *s_lo, *s_hi;
  const WorkItem* items;  // form items, most sources first
  const int* n_items;     // item count (device)
  int max_items;          // upper bound of the item count (grid sizing)
  int slab, nslab;        // x-slab grids: planes per slab and slabs per box (1: whole grids)
  int* next;              // work counter (zero at launch)
};

template <typename T>
struct FormPtrs {
  const double* off;     // sorted SoA FP64 offsets
  const T *q, *ds, *rn;  // sorted SoA
  T* mp;                 // [n_form][nd][nexp] complex
  T* partial;            // [partial slots][nd][nexp] complex: parts of split boxes
};

// ------------------------------------------------ block-tiled spreading (3D)
// The box's points are counting-sorted by 4x4x4 block of stencil base cells.
// A warp takes one block at a time and accumulates all of its points into a
// register tile of (4+W-1)^3 cells: lane l owns the tile columns (tx,ty) =
// l, l+32, ... with all TILE z cells.  Per point the warp reads the point's
// three shifted kernel rows (zero outside the stencil) from shared memory and
// does NCOL*TILE FMAs per lane; the tile is flushed once per block with one
// shared-memory atomic per non-zero cell, instead of W^3 atomics per point.
constexpr int TB = 4;           // block edge (base cells)
constexpr int NBLK_MAX = 1024;  // blocks per box
constexpr int PB = 8;           // points per warp batch
constexpr int TP = 12;          // padded kernel row (TILE <= TP - 1)
// points sorted per round: FP32 8192; FP64 2048 (its ~200 KB grid leaves
// little shared memory)
template <typename T>
__host__ __device__ constexpr int fch() {
  return sizeof(T) == 4 ? 8192 : 2048;
}

constexpr int RD = 10;  // FP64 kernel row: one tile row (TILE <= RD - 1) + a zero

// byte offset of the grid buffer in the tiled form kernel; every part is a
// multiple of 16 bytes, so the kernel-row buffer is float4 aligned.  The
// FP64 variant's row buffer holds three rows of RD doubles per warp.
template <typename T>
__host__ __device__ constexpr size_t tiled_offset(int G, int K) {
  return tw_bytes16<T>(G, K) + sizeof(int) * (2 * NBLK_MAX + 32) + sizeof(int) * fch<T>() +
         sizeof(unsigned short) * fch<T>() +
         (sizeof(T) == 4 ? sizeof(float) * (PW_THREADS / 32) * PB * 3 * TP
                         : sizeof(double) * (PW_THREADS / 32) * 3 * RD);
}

// Exclusive scan of cnt[0..n) into off[0..n) for n <= 2 * blockDim.x;
// ws holds blockDim.x / 32 ints.  Ends with a block barrier.
__device__ __forceinline__ void block_scan(const int* cnt, int* off, int n, int* ws) {
  const int t = threadIdx.x, lane = t & 31, w = t >> 5, nw = blockDim.x >> 5;
  const int v0 = 2 * t < n ? cnt[2 * t] : 0, v1 = 2 * t + 1 < n ? cnt[2 * t + 1] : 0;
  const int s = v0 + v1;
  int inc = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += u;
  }
  if (lane == 31) ws[w] = inc;
  __syncthreads();
  if (w == 0) {
    const int x = lane < nw ? ws[lane] : 0;
    int ix = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, ix, o);
      if (lane >= o) ix += u;
    }
    if (lane < nw) ws[lane] = ix - x;
  }
  __syncthreads();
  const int ex = ws[w] + inc - s;
  if (2 * t < n) off[2 * t] = ex;
  if (2 * t + 1 < n) off[2 * t + 1] = ex + v0;
  __syncthreads();
}

template <typename T, int W>
__device__ __forceinline__ int base_cell(const PWArgs<T>& a, double xs) {
  const double u = xs * a.inv_dx_d;
  const int b = (int)ceil(u - a.hwdx_d) - a.g.l0;
  return b < 0 ? 0 : (b > a.g.G - W ? a.g.G - W : b);
}

// Spread points c0..c0+n-1 (n <= FCH) of one strength set into B.
// sq: charges (is_q) or dipole strengths, sr: dipole direction component.
template <typename T, int W>
__device__ void spread_tiled(const PWArgs<T>& a, T* B, const double* __restrict__ off, int ns,
                             const T* __restrict__ sq, const T* __restrict__ sr, bool is_q, int c0,
                             int n, int* cnt, int* boff, int* misc, int* tmp,
                             unsigned short* perm, T* rows) {
  constexpr int TILE = TB + W - 1, NCOL = (TILE * TILE + 31) / 32, NP2 = TP / 2;
  static_assert(TILE <= TP - 1, "tile row too long");
  static_assert(std::is_same<T, float>::value, "tiled spreading is the FP32 path");
  const Geo& g = a.g;
  const int nbd = (g.G - W + 1 + TB - 1) / TB, nblk = nbd * nbd * nbd;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) cnt[i] = 0;
  if (threadIdx.x == 0) misc[0] = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    int blk = 0;
#pragma unroll
    for (int d = 0; d < 3; d++)
      blk = blk * nbd + base_cell<T, W>(a, off[(size_t)d * ns + c0 + i] * a.scale_d) / TB;
    const int r = atomicAdd(&cnt[blk], 1);
    tmp[i] = (r << 10) | blk;
  }
  __syncthreads();
  block_scan(cnt, boff, nblk, misc + 1);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int v = tmp[i];
    perm[boff[v & (NBLK_MAX - 1)] + (v >> 10)] = (unsigned short)i;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T* R = rows + warp * (PB * 3 * TP);
  int cx[NCOL], cy[NCOL];  // slots past the tile read the zero entry TP-1
#pragma unroll
  for (int j = 0; j < NCOL; j++) {
    const int c = lane + 32 * j;
    cx[j] = c < TILE * TILE ? c / TILE : TP - 1;
    cy[j] = c < TILE * TILE ? c % TILE : TP - 1;
  }
  for (;;) {
    int bi = 0;
    if (lane == 0) bi = atomicAdd(&misc[0], 1);
    bi = __shfl_sync(0xffffffffu, bi, 0);
    if (bi >= nblk) break;
    const int nb = cnt[bi];
    if (nb == 0) continue;
    const int start = boff[bi];
    int org[3];
    org[2] = (bi % nbd) * TB;
    org[1] = ((bi / nbd) % nbd) * TB;
    org[0] = (bi / (nbd * nbd)) * TB;
    // z cells in pairs (packed FP32x2 FMAs); TILE <= TP - 1 cells in TP/2 pairs
    float2 acc[NCOL][NP2];
#pragma unroll
    for (int j = 0; j < NCOL; j++)
#pragma unroll
      for (int i = 0; i < NP2; i++) acc[j][i] = make_float2(0.f, 0.f);
    for (int k0 = 0; k0 < nb; k0 += PB) {
      const int np = min(PB, nb - k0);
      if (lane < 3 * PB) {
        const int pp = lane % PB, d = lane / PB;
        if (pp < np) {
          T* row = R + (pp * 3 + d) * TP;
          const int pt = c0 + perm[start + k0 + pp];
          T ph[W];
          const double x = off[(size_t)d * ns + pt] * a.scale_d;
          const int i0 = kernel_row<T, W>(a, x, ph);
          int b = i0 - g.l0;
          b = b < 0 ? 0 : (b > g.G - W ? g.G - W : b);
          const int o = b - org[d];
          const T sc = d == 0 ? (is_q ? sq[pt] : sq[pt] * sr[pt]) : T(1);
#pragma unroll
          for (int t = 0; t < TP; t++) row[t] = T(0);
#pragma unroll
          for (int j = 0; j < W; j++) row[o + j] = ph[j] * sc;
        }
      }
      __syncwarp();
#pragma unroll 1
      for (int pq = 0; pq < np; pq++) {
        const float* row = R + pq * 3 * TP;
        const float4* rv = reinterpret_cast<const float4*>(row + 2 * TP);
        float2 rz[NP2];
#pragma unroll
        for (int i = 0; i < NP2 / 2; i++) {
          const float4 q4 = rv[i];
          rz[2 * i] = make_float2(q4.x, q4.y);
          rz[2 * i + 1] = make_float2(q4.z, q4.w);
        }
#pragma unroll
        for (int j = 0; j < NCOL; j++) {
          const float v = row[cx[j]] * row[TP + cy[j]];
          const float2 vv = make_float2(v, v);
#pragma unroll
          for (int i = 0; i < NP2; i++) acc[j][i] = __ffma2_rn(vv, rz[i], acc[j][i]);
        }
      }
      __syncwarp();
    }
#pragma unroll
    for (int j = 0; j < NCOL; j++) {
      const int x = org[0] + cx[j], y = org[1] + cy[j];
      if (lane + 32 * j < TILE * TILE && x < g.G && y < g.G) {
        float* col = B + x * g.str[0] + y * g.str[1] + org[2];
#pragma unroll
        for (int i = 0; i < NP2; i++) {
          const int t = 2 * i;
          if (t < TILE && org[2] + t < g.G && acc[j][i].x != 0.f) atomicAdd(col + t, acc[j][i].x);
          if (t + 1 < TILE && org[2] + t + 1 < g.G && acc[j][i].y != 0.f)
            atomicAdd(col + t + 1, acc[j][i].y);
        }
      }
    }
  }
  __syncthreads();
}

// FP64 block-tiled spreading (3D, eps >= ~1e-6): as spread_tiled, with
// blocks of TBD^3 base cells and a register tile of (TBD+W-1)^3 FP64 cells
// (lane l owns the tile columns l, l+32, ... with all TILE z cells).  Per
// point, lane t < 3 RD writes entry t % RD of the point's kernel row t / RD
// in tile coordinates (zero outside the stencil, the x row times the
// strength) to the warp's row buffer, and every lane reads its values as
// broadcasts: no shuffles and no edge selects.  The flush adds every
// non-zero tile cell with one atomic: ~TILE^3/(points per block) atomics
// per point instead of W^3.
template <int W, int TBD>
__device__ void spread_tiled_d(const PWArgs<double>& a, double* B, const double* __restrict__ off,
                               int ns, const double* __restrict__ sq,
                               const double* __restrict__ sr, bool is_q, int c0, int n, int* cnt,
                               int* boff, int* misc, int* tmp, unsigned short* perm,
                               double* rows) {
  constexpr int TILE = TBD + W - 1, NCOL = (TILE * TILE + 31) / 32;
  static_assert(TILE <= RD - 1 && 3 * RD <= 32, "one row entry per lane, a zero at RD - 1");
  const Geo& g = a.g;
  const int nbd = (g.G - W + 1 + TBD - 1) / TBD, nblk = nbd * nbd * nbd;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) cnt[i] = 0;
  if (threadIdx.x == 0) misc[0] = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    int blk = 0;
#pragma unroll
    for (int d = 0; d < 3; d++)
      blk = blk * nbd + base_cell<double, W>(a, off[(size_t)d * ns + c0 + i] * a.scale_d) / TBD;
    const int r = atomicAdd(&cnt[blk], 1);
    tmp[i] = (r << 10) | blk;
  }
  __syncthreads();
  block_scan(cnt, boff, nblk, misc + 1);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int v = tmp[i];
    perm[boff[v & (NBLK_MAX - 1)] + (v >> 10)] = (unsigned short)i;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  double* R = rows + (threadIdx.x >> 5) * 3 * RD;
  // slots past the tile read entry RD - 1 of the rows, which stays zero
  int cx[NCOL], cy[NCOL];
#pragma unroll
  for (int j = 0; j < NCOL; j++) {
    const int c = lane + 32 * j;
    cx[j] = c < TILE * TILE ? c / TILE : RD - 1;
    cy[j] = c < TILE * TILE ? c % TILE : RD - 1;
  }
  const int kd = lane / RD, kq = lane - kd * RD;  // this lane's row entry
  for (;;) {
    int bi = 0;
    if (lane == 0) bi = atomicAdd(&misc[0], 1);
    bi = __shfl_sync(0xffffffffu, bi, 0);
    if (bi >= nblk) break;
    const int nb = cnt[bi];
    if (nb == 0) continue;
    const int start = boff[bi];
    int org[3];
    org[2] = (bi % nbd) * TBD;
    org[1] = ((bi / nbd) % nbd) * TBD;
    org[0] = (bi / (nbd * nbd)) * TBD;
    double acc[NCOL][TILE];
#pragma unroll
    for (int j = 0; j < NCOL; j++)
#pragma unroll
      for (int t = 0; t < TILE; t++) acc[j][t] = 0.0;
    for (int k = 0; k < nb; k++) {
      const int pt = c0 + perm[start + k];
      // this lane's row entry: kernel value at stencil offset kq - o[kd] of
      // dimension kd (zero outside the stencil; the x row carries the strength)
      double v = 0.0;
      if (lane < 3 * RD) {
        const double x = off[(size_t)kd * ns + pt] * a.scale_d;
        double f0;
        int b = kernel_start<double>(a, x, f0) - g.l0;
        b = b < 0 ? 0 : (b > g.G - W ? g.G - W : b);
        int j = kq - (b - (kd == 0 ? org[0] : (kd == 1 ? org[1] : org[2])));
        if (!FGT_DCHECK(kq != RD - 1 || j >= W, 208)) j = W;  // entry RD - 1 stays zero
        if (j >= 0 && j < W) {
          v = es_kernel<double>((f0 + (double)j) * a.inv_hw, a.beta);
          if (kd == 0) v *= is_q ? sq[pt] : sq[pt] * sr[pt];
        }
        R[lane] = v;
      }
      __syncwarp();
      double pz[TILE];
#pragma unroll
      for (int t = 0; t < TILE; t++) pz[t] = R[2 * RD + t];
#pragma unroll
      for (int j = 0; j < NCOL; j++) {
        const double pxy = R[cx[j]] * R[RD + cy[j]];
#pragma unroll
        for (int t = 0; t < TILE; t++) acc[j][t] = fma(pxy, pz[t], acc[j][t]);
      }
      __syncwarp();
    }
#pragma unroll
    for (int j = 0; j < NCOL; j++) {
      const int x = org[0] + cx[j], y = org[1] + cy[j];
      if (lane + 32 * j < TILE * TILE && x < g.G && y < g.G) {
        double* col = B + x * g.str[0] + y * g.str[1] + org[2];
#pragma unroll
        for (int t = 0; t < TILE; t++)
          if (org[2] + t < g.G && acc[j][t] != 0.0) atomicAdd(col + t, acc[j][t]);
      }
    }
  }
  __syncthreads();
}
constexpr int TB_D = 2;  // FP64 block edge (register tile of 3 x 9 columns, no spills)

template <typename T, int DIM, int W, bool GB, bool TILED>
__global__ void __launch_bounds__(PW_THREADS) k_form(PWArgs<T> a, FormIO io, FormPtrs<T> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Geo& g = a.g;
  const int K = g.K, NF = 2 * K + 1, NH = K + 1, G = g.G;
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int NFp = pad4(NF), NHp = pad4(NH);
  // G*NF and G*NH complex, planar rows of 2*NFp / 2*NHp (staged or global)
  const T* twf = stage_tw(sm, a.twf, 2 * G * NFp);
  const T* twh = stage_tw(sm + 2 * G * NFp, a.twh, 2 * G * NHp);
  // atomic-spreading scratch
  int* ordtmp = reinterpret_cast<int*>(sm + tw_elems_t<T>(G, K));  // ORDER_CHUNK
  int* ordcnt = ordtmp + ORDER_CHUNK;                        // 32
  unsigned short* perm = reinterpret_cast<unsigned short*>(ordcnt + 32);  // ORDER_CHUNK
  // tiled-spreading scratch
  int* tcnt = reinterpret_cast<int*>(smem_raw + tw_bytes16<T>(G, K));  // NBLK_MAX
  int* toff = tcnt + NBLK_MAX;                             // NBLK_MAX
  int* tmisc = toff + NBLK_MAX;                            // 32
  int* ttmp = tmisc + 32;                                  // fch
  unsigned short* tperm = reinterpret_cast<unsigned short*>(ttmp + fch<T>());  // fch
  T* trows = reinterpret_cast<T*>(tperm + fch<T>());  // FP32: warps * PB * 3 * TP
  T* B = GB ? a.gscratch + (size_t)blockIdx.x * g.bufsz
            : reinterpret_cast<T*>(smem_raw + (TILED ? tiled_offset<T>(G, K)
                                                     : order_offset<T>(G, K)));
  __syncthreads();
  // items in decreasing source count, each CTA takes the next one; the
  // parts of a split box write partial expansions, summed by k_form_reduce
  __shared__ int s_next;
  const int n_items = *io.n_items;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_next = atomicAdd(io.next, 1);
    __syncthreads();
    if (s_next >= n_items) break;
    const WorkItem it = io.items[s_next];
    const int fb = it.slot;
    if (!FGT_DCHECK(fb >= 0 && fb < io.n_form, 201)) continue;
    const int box = io.form_box[fb];
    int p0, p1;
    part_range(io.s_lo[box], io.s_hi[box], it.part, it.nparts, p0, p1);
    if (!FGT_DCHECK(p0 >= 0 && p0 <= p1 && p1 <= io.ns, 202)) continue;
    T* mp_base = it.pslot >= 0 ? p.partial + (size_t)it.pslot * io.nd * 2 * g.nexp
                               : p.mp + (size_t)fb * io.nd * 2 * g.nexp;
    for (int id = 0; id < io.nd; id++) {
      T* mp = mp_base + (size_t)id * 2 * g.nexp;
      int first = 1;
      for (int comp = 0; comp < io.ncomp; comp++) {
        // comp 0 = charge when present; the others are dipole directions
        const bool is_q = io.has_q && comp == 0;
        const int dd = is_q ? -1 : comp - io.has_q;
        for (int i = threadIdx.x; i < g.bufsz; i += blockDim.x) B[i] = T(0);
        __syncthreads();
        if constexpr (TILED) {
          const T* sq = is_q ? p.q + (size_t)id * io.ns : p.ds + (size_t)id * io.ns;
          const T* sr = is_q ? nullptr : p.rn + (size_t)dd * io.ns;
          for (int c0 = p0; c0 < p1; c0 += fch<T>()) {
            if constexpr (std::is_same<T, double>::value)
              spread_tiled_d<W, TB_D>(a, B, p.off, io.ns, sq, sr, is_q, c0, min(fch<T>(), p1 - c0),
                                      tcnt, toff, tmisc, ttmp, tperm, trows);
            else
              spread_tiled<T, W>(a, B, p.off, io.ns, sq, sr, is_q, c0, min(fch<T>(), p1 - c0),
                                 tcnt, toff, tmisc, ttmp, tperm, trows);
          }
        } else {
          for (int c0 = p0; c0 < p1; c0 += ORDER_CHUNK) {
            const int n = min(ORDER_CHUNK, p1 - c0);
            order_chunk<T, DIM, W>(a, p.off, io.ns, c0, n, perm, ordtmp, ordcnt);
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
              const int pt = c0 + perm[i];
              double x[DIM];
#pragma unroll
              for (int k = 0; k < DIM; k++) x[k] = p.off[(size_t)k * io.ns + pt] * a.scale_d;
              const T str = is_q ? p.q[(size_t)id * io.ns + pt]
                                 : p.ds[(size_t)id * io.ns + pt] * p.rn[(size_t)dd * io.ns + pt];
              spread_point<T, DIM, W>(a, B, x, str);
            }
            __syncthreads();
          }
        }
        // passes on the last and middle dimensions
        if (DIM == 3) {
          pass_inplace<T, 0>(B, G * G, G, g.str[0], g.str[1], 1, 2, G, NH, twh);
          pass_inplace<T, 1>(B, G * NH, NH, g.str[0], 2, g.str[1], g.str[1], G, NF, twf);
          pass_inplace<T, 1>(B, NF * NH, NH, g.str[1], 2, g.str[0], g.str[0], G, NF, twf);
        } else if (DIM == 2) {
          pass_inplace<T, 0>(B, G, 1, g.str[0], 0, 1, 2, G, NH, twh);
          pass_inplace<T, 1>(B, NH, 1, 2, 0, g.str[0], g.str[0], G, NF, twf);
        }
        // expansion: the x pass's modes (1D: the pass along x here) with
        // weights and deconvolution
        const int nline = DIM == 3 ? NF * NH : (DIM == 2 ? NH : 1);
        const int nko = DIM == 1 ? NH : NF;
        for (int o = threadIdx.x; o < nko * nline; o += blockDim.x) {
          const int kxi = o / nline, line = o - kxi * nline;
          int lb, kyi = 0, kz = 0;
          if (DIM == 3) {
            kyi = line / NH;
            kz = line - kyi * NH;
            lb = kyi * g.str[1] + 2 * kz;
          } else if (DIM == 2) {
            kz = line;
            lb = 2 * line;
          } else {
            lb = 0;
          }
          T re = T(0), im = T(0);
          if (DIM == 1) {
            for (int l = 0; l < G; l++) {
              const T gv = B[l];
              re += gv * twh[l * 2 * NHp + kxi];
              im += gv * twh[l * 2 * NHp + NHp + kxi];
            }
          } else {
            re = B[kxi * g.str[0] + lb];
            im = B[kxi * g.str[0] + lb + 1];
          }
          int ki[3];
          if (DIM == 3) { ki[0] = kxi; ki[1] = kyi; ki[2] = kz + K; }
          else if (DIM == 2) { ki[0] = kxi; ki[1] = kz + K; }
          else { ki[0] = kxi + K; }
          T f = T(1);
#pragma unroll
          for (int d = 0; d < DIM; d++) f *= a.facf[ki[d]];
          T vr = re * f, vi = im * f;
          if (!is_q) {  // * (-i) ts(k_d) / sqrt(delta0)
            const T cc = a.ts[sel3(ki, dd)] * a.inv_sqd0;
            const T tr = vi * cc, ti = -vr * cc;
            vr = tr;
            vi = ti;
          }
          const int m = (DIM == 1) ? kxi : kxi * nline + line;
          if (first) {
            mp[2 * m] = vr;
            mp[2 * m + 1] = vi;
          } else {
            mp[2 * m] += vr;
            mp[2 * m + 1] += vi;
          }
        }
        first = 0;
        __syncthreads();
      }
    }
  }
}

// ------------------------------------------------------ x-slab grids (3D)
// A grid too large for shared memory (eps <= 1e-9 with plane waves) is cut
// into slabs of whole x-planes (slab_plan).  A work item is (box, point part,
// slab); its CTA holds the slab in shared memory, spreads every point of its
// part into the planes that the point's stencil shares with the slab
// (shared-memory atomics), runs the z and y passes of the form on the slab's
// planes (they never leave an x-plane), and adds the slab's terms of the x
// transform, times the weights of the expansion, to the box's expansion with
// global atomics (the expansions are zeroed before the launch).  No grid
// leaves shared memory; the slabs of a box run on different SMs.

// Spread one point into the planes [x0, x1) of a slab (plane xl of the slab
// is grid plane x0 + xl).
template <typename T, int W>
__device__ __forceinline__ void spread_point_slab(const PWArgs<T>& a, T* B, const double* x, T str,
                                                  int x0, int x1) {
  const Geo& g = a.g;
  T ph[2][W];  // y and z rows; the x values are computed as the x loop reaches them
  int b[3];
  T f0x;
  b[0] = kernel_start<T>(a, x[0], f0x) - g.l0;
  b[1] = kernel_row<T, W>(a, x[1], ph[0]) - g.l0;
  b[2] = kernel_row<T, W>(a, x[2], ph[1]) - g.l0;
#pragma unroll
  for (int d = 0; d < 3; d++) b[d] = b[d] < 0 ? 0 : (b[d] > g.G - W ? g.G - W : b[d]);
  const int jlo = max(0, x0 - b[0]), jhi = min(W, x1 - b[0]);
  T* by = B + b[1] * g.str[1] + b[2];
#pragma unroll 1
  for (int jx = jlo; jx < jhi; jx++) {
    T* bx = by + (b[0] + jx - x0) * g.str[0];
    const T vx = str * es_kernel<T>((f0x + (T)jx) * a.inv_hw, a.beta);
#pragma unroll
    for (int jy = 0; jy < W; jy++) {
      T* bxy = bx + jy * g.str[1];
      const T vxy = vx * ph[0][jy];
#pragma unroll
      for (int jz = 0; jz < W; jz++) atomicAdd(bxy + jz, vxy * ph[1][jz]);
    }
  }
}

template <typename T, int W>
__global__ void __launch_bounds__(PW_THREADS) k_form_slab(PWArgs<T> a, FormIO io, FormPtrs<T> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Geo& g = a.g;
  const int K = g.K, NF = 2 * K + 1, NH = K + 1, G = g.G;
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int NFp = pad4(NF), NHp = pad4(NH);
  const T* twf = stage_tw(sm, a.twf, 2 * G * NFp);
  const T* twh = stage_tw(sm + 2 * G * NFp, a.twh, 2 * G * NHp);
  int* ordtmp = reinterpret_cast<int*>(sm + tw_elems_t<T>(G, K));  // ORDER_CHUNK
  int* ordcnt = ordtmp + ORDER_CHUNK;                               // 32
  unsigned short* perm = reinterpret_cast<unsigned short*>(ordcnt + 32);  // ORDER_CHUNK
  T* B = reinterpret_cast<T*>(smem_raw + order_offset<T>(G, K));  // io.slab planes
  const int C = io.nslab, nline = NF * NH;
  __syncthreads();
  __shared__ int s_next;
  const int n_items = *io.n_items;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_next = atomicAdd(io.next, 1);
    __syncthreads();
    if (s_next >= n_items) break;
    const WorkItem it = io.items[s_next];
    const int fb = it.slot;
    if (!FGT_DCHECK(fb >= 0 && fb < io.n_form && it.nparts % C == 0, 206)) continue;
    const int box = io.form_box[fb];
    const int x0 = (it.part % C) * io.slab, x1 = min(G, x0 + io.slab), np_ = x1 - x0;
    int p0, p1;
    part_range(io.s_lo[box], io.s_hi[box], it.part / C, it.nparts / C, p0, p1);
    if (!FGT_DCHECK(p0 >= 0 && p0 <= p1 && p1 <= io.ns && np_ > 0 && np_ <= io.slab, 207))
      continue;
    for (int id = 0; id < io.nd; id++) {
      T* mp = p.mp + ((size_t)fb * io.nd + id) * 2 * g.nexp;
      for (int comp = 0; comp < io.ncomp; comp++) {
        const bool is_q = io.has_q && comp == 0;
        const int dd = is_q ? -1 : comp - io.has_q;
        for (int i = threadIdx.x; i < np_ * g.str[0]; i += blockDim.x) B[i] = T(0);
        __syncthreads();
        for (int c0 = p0; c0 < p1; c0 += ORDER_CHUNK) {
          const int n = min(ORDER_CHUNK, p1 - c0);
          order_chunk<T, 3, W>(a, p.off, io.ns, c0, n, perm, ordtmp, ordcnt);
          for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const int pt = c0 + perm[i];
            double x[3];
#pragma unroll
            for (int k = 0; k < 3; k++) x[k] = p.off[(size_t)k * io.ns + pt] * a.scale_d;
            const T str = is_q ? p.q[(size_t)id * io.ns + pt]
                               : p.ds[(size_t)id * io.ns + pt] * p.rn[(size_t)dd * io.ns + pt];
            spread_point_slab<T, W>(a, B, x, str, x0, x1);
          }
          __syncthreads();
        }
        // passes along z (real -> half complex) and y on the slab's planes
        pass_inplace<T, 0>(B, np_ * G, G, g.str[0], g.str[1], 1, 2, G, NH, twh);
        pass_inplace<T, 1>(B, np_ * NH, NH, g.str[0], 2, g.str[1], g.str[1], G, NF, twf);
        // the slab's terms of the x transform, weights and deconvolution
        // (as k_form's expansion step), added to the box's expansion
        for (int o = threadIdx.x; o < NF * nline; o += blockDim.x) {
          const int kxi = o / nline, line = o - kxi * nline;
          const int kyi = line / NH, kz = line - kyi * NH;
          const T* bl = B + kyi * g.str[1] + 2 * kz;
          const T* tw = twf + (size_t)x0 * 2 * NFp + kxi;
          T re = T(0), im = T(0);
          for (int xl = 0; xl < np_; xl++, bl += g.str[0], tw += 2 * NFp) {
            const T br = bl[0], bi = bl[1], tr = tw[0], ti = tw[NFp];
            re += br * tr - bi * ti;
            im += br * ti + bi * tr;
          }
          const int ki[3] = {kxi, kyi, kz + K};
          const T f = a.facf[ki[0]] * a.facf[ki[1]] * a.facf[ki[2]];
          T vr = re * f, vi = im * f;
          if (!is_q) {  // * (-i) ts(k_d) / sqrt(delta0)
            const T cc = a.ts[sel3(ki, dd)] * a.inv_sqd0;
            const T tr = vi * cc, ti = -vr * cc;
            vr = tr;
            vi = ti;
          }
          atomicAdd(mp + 2 * o, vr);
          atomicAdd(mp + 2 * o + 1, vi);
        }
        __syncthreads();
      }
    }
  }
}

// Form of small 2D boxes, one warp per box (see small2_layout): the boxes
// order[first..n_form) of the longest-processing-time order, which all hold
// at most SMALL2_MAX sources.  Same sums as k_form for DIM = 2.
template <typename T, int W>
__global__ void __launch_bounds__(256) k_form_small2(PWArgs<T> a, FormIO io, FormPtrs<T> p,
                                                     const uint32_t* __restrict__ order,
                                                     const int* __restrict__ first,
                                                     int* __restrict__ next) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Geo& g = a.g;
  const int K = g.K, NF = 2 * K + 1, NH = K + 1, G = g.G;
  T* sm = reinterpret_cast<T*>(smem_raw);
  const T* twf = stage_tw(sm, a.twf, 2 * G * pad4(NF));
  const T* twh = stage_tw(sm + 2 * G * pad4(NF), a.twh, 2 * G * pad4(NH));
  const Small2Layout lay = small2_layout(G, K);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* A = reinterpret_cast<T*>(smem_raw + tw_bytes16<T>(G, K)) + (size_t)warp * lay.per_warp;
  T* Cb = A + lay.r1;
  __syncthreads();
  const int f0 = *first;
  for (;;) {
    int bi = 0;
    if (lane == 0) bi = atomicAdd(next, 1);
    bi = __shfl_sync(0xffffffffu, bi, 0) + f0;
    if (bi >= io.n_form) break;
    const int fb = (int)order[bi];
    if (!FGT_DCHECK(fb >= 0 && fb < io.n_form, 203)) continue;
    const int box = io.form_box[fb];
    const int p0 = io.s_lo[box], p1 = io.s_hi[box];
    if (!FGT_DCHECK(p0 >= 0 && p0 <= p1 && p1 <= io.ns && p1 - p0 <= SMALL2_MAX, 204)) continue;
    for (int id = 0; id < io.nd; id++) {
      T* mp = p.mp + ((size_t)fb * io.nd + id) * 2 * g.nexp;
      for (int comp = 0; comp < io.ncomp; comp++) {
        const bool is_q = io.has_q && comp == 0;
        const int dd = is_q ? -1 : comp - io.has_q;
        for (int i = lane; i < G * lay.SA; i += 32) A[i] = T(0);
        __syncwarp();
        // points in batches of 32: lane j prepares point j (stencil base,
        // kernel offsets, strength), then the warp adds them one by one
        for (int c0 = p0; c0 < p1; c0 += 32) {
          const int nb = min(32, p1 - c0);
          int bx = 0, by = 0;
          T fx = T(0), fy = T(0), st = T(0);
          if (lane < nb) {
            const int pt = c0 + lane;
            const double x = p.off[pt] * a.scale_d, y = p.off[(size_t)io.ns + pt] * a.scale_d;
            bx = kernel_start<T>(a, x, fx) - g.l0;
            by = kernel_start<T>(a, y, fy) - g.l0;
            // cells beyond the sub-grid carry zero weight (points lie
            // inside it), so the clamp only keeps the stencil in bounds
            bx = bx < 0 ? 0 : (bx > G - W ? G - W : bx);
            by = by < 0 ? 0 : (by > G - W ? G - W : by);
            st = is_q ? p.q[(size_t)id * io.ns + pt]
                      : p.ds[(size_t)id * io.ns + pt] * p.rn[(size_t)dd * io.ns + pt];
          }
          for (int j = 0; j < nb; j++) {
            const int jbx = __shfl_sync(0xffffffffu, bx, j), jby = __shfl_sync(0xffffffffu, by, j);
            const T jfx = __shfl_sync(0xffffffffu, fx, j), jfy = __shfl_sync(0xffffffffu, fy, j);
            const T jst = __shfl_sync(0xffffffffu, st, j);
            T v = T(0);
            if (lane < 2 * W) {
              const int k = lane < W ? lane : lane - W;
              v = es_kernel<T>(((lane < W ? jfx : jfy) + (T)k) * a.inv_hw, a.beta);
            }
#pragma unroll
            for (int cc = 0; cc < (W * W + 31) / 32; cc++) {
              const int c = cc * 32 + lane;
              const int cx = c < W * W ? c / W : 0, cy = c < W * W ? c % W : 0;
              const T px = __shfl_sync(0xffffffffu, v, cx);
              const T py = __shfl_sync(0xffffffffu, v, W + cy);
              if (c < W * W) A[(jbx + cx) * lay.SA + jby + cy] += jst * px * py;
            }
            __syncwarp();
          }
        }
        warp_pass_r2c<T>(A, lay.SA, Cb, lay.SC, G, NH, twh);
        __syncwarp();
        const bool first_c = comp == 0;
        warp_pass_c2c<T>(Cb, lay.SC, G, NF, NH, twf, [&](int kxi, int ky, T re, T im) {
          const int ki[3] = {kxi, ky + K, 0};
          const T f = a.facf[kxi] * a.facf[ky + K];
          T vr = re * f, vi = im * f;
          if (!is_q) {  // * (-i) ts(k_d) / sqrt(delta0)
            const T cf = a.ts[sel3(ki, dd)] * a.inv_sqd0;
            const T tr = vi * cf, ti = -vr * cf;
            vr = tr;
            vi = ti;
          }
          const int m = kxi * NH + ky;
          if (first_c) {
            mp[2 * m] = vr;
            mp[2 * m + 1] = vi;
          } else {
            mp[2 * m] += vr;
            mp[2 * m + 1] += vi;
          }
        });
        __syncwarp();
      }
    }
  }
}

// First entry of a list sorted by k_lpt_keys (ascending keys = descending
// point counts) whose box holds at most `limit` points.
__global__ void k_first_at_most(const uint64_t* __restrict__ keys, int n, int limit,
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

// mp of every split form box = sum of its parts' partial expansions, in part
// order (deterministic).  One thread per (split box, density, mode).
template <typename T>
__global__ void k_form_reduce(const SplitRec* __restrict__ rec, const int* __restrict__ n_split,
                              int nd, int nexp, const T* __restrict__ partial, T* __restrict__ mp) {
  using V = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
  const long long per = (long long)nd * nexp;
  const long long total = (long long)(*n_split) * per;
  const V* pv = reinterpret_cast<const V*>(partial);
  V* mv = reinterpret_cast<V*>(mp);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const SplitRec r = rec[i / per];
    const long long j = i % per;
    V acc;
    acc.x = T(0);
    acc.y = T(0);
    for (int q = 0; q < r.nparts; q++) {
      const V v = pv[(long long)(r.pslot + q) * per + j];
      acc.x += v.x;
      acc.y += v.y;
    }
    mv[(long long)r.slot * per + j] = acc;
  }
}

// ---------------------------------------------------------------- translate
constexpr int TRANS_MPT = 4;
// Local expansion of every eval box: its own form expansion plus the
// diagonal translations W[w] * M[s] of its list (gnd_shiftpw,
// src/pfgt/bfgt_pwrouts.f:1555-1636), one mode per thread, complex values
// as 8- or 16-byte vectors.
template <typename T>
__global__ void k_translate(int n_eval, int n_form, int nsh, int nexp, int nd, int ge,
                            const int* __restrict__ self,
                            const int* __restrict__ ptr, const int* __restrict__ src,
                            const int* __restrict__ widx, const T* __restrict__ mp,
                            const T* __restrict__ wtab, T* __restrict__ loc) {
  using V = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
  constexpr int MPT = TRANS_MPT;  // modes per thread, blockDim apart
  const V* mpv = reinterpret_cast<const V*>(mp);
  const V* wv = reinterpret_cast<const V*>(wtab);
  V* lv = reinterpret_cast<V*>(loc);
  const int e0 = blockIdx.y * ge, e1 = min(n_eval, e0 + ge);
  const int m0 = blockIdx.x * blockDim.x * MPT + threadIdx.x;
  bool ok[MPT];
#pragma unroll
  for (int i = 0; i < MPT; i++) ok[i] = m0 + i * (int)blockDim.x < nexp;
  for (int e = e0; e < e1; e++) {
    const int sf = self[e], j0 = ptr[e], j1 = ptr[e + 1];
    for (int id = 0; id < nd; id++) {
      V acc[MPT];
      const V* sp = mpv + ((size_t)(sf >= 0 ? sf : 0) * nd + id) * nexp + m0;
#pragma unroll
      for (int i = 0; i < MPT; i++) {
        acc[i].x = T(0);
        acc[i].y = T(0);
        if (sf >= 0 && ok[i]) acc[i] = __ldg(sp + i * blockDim.x);
      }
      for (int j = j0; j < j1; j++) {
        if (!FGT_DCHECK(src[j] >= 0 && src[j] < n_form && widx[j] >= 0 && widx[j] < nsh, 205))
          continue;
        const V* ap = mpv + ((size_t)src[j] * nd + id) * nexp + m0;
        const V* wp = wv + (size_t)widx[j] * nexp + m0;
        V av[MPT], w[MPT];
#pragma unroll
        for (int i = 0; i < MPT; i++) {
          if (ok[i]) {
            av[i] = __ldg(ap + i * blockDim.x);
            w[i] = __ldg(wp + i * blockDim.x);
          } else {
            av[i].x = av[i].y = w[i].x = w[i].y = T(0);
          }
        }
#pragma unroll
        for (int i = 0; i < MPT; i++) {
          acc[i].x += av[i].x * w[i].x - av[i].y * w[i].y;
          acc[i].y += av[i].x * w[i].y + av[i].y * w[i].x;
        }
      }
      V* op = lv + ((size_t)e * nd + id) * nexp + m0;
#pragma unroll
      for (int i = 0; i < MPT; i++)
        if (ok[i]) op[i * blockDim.x] = acc[i];
    }
  }
}

// W[s][m] = prod_d exp(i ts(k_d) xmin s_d) (gnd_mk_full_translation_matrices,
// src/pfgt/pfgt_nufftrouts.f:336-424), s_d = s/3^d % 3 - 1.
template <typename T>
__global__ void k_wtab(int dim, int K, int nexp, const double* __restrict__ ts, double xmin,
                       T* __restrict__ w) {
  int nsh = dim == 1 ? 3 : (dim == 2 ? 9 : 27);
  int NF = 2 * K + 1, NH = K + 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nsh * nexp; i += gridDim.x * blockDim.x) {
    int s = i / nexp, m = i - s * nexp;
    int ki[3];
    if (dim == 3) { ki[0] = m / (NF * NH); ki[1] = (m / NH) % NF; ki[2] = m % NH + K; }
    else if (dim == 2) { ki[0] = m / NH; ki[1] = m % NH + K; }
    else { ki[0] = m + K; }
    double ph = 0;
    int r = s;
    for (int d = 0; d < dim; d++) {
      int sd = r % 3 - 1;
      r /= 3;
      ph += ts[ki[d]] * xmin * sd;
    }
    double sn, cs;
    sincos(ph, &sn, &cs);
    w[2 * (size_t)i] = (T)cs;
    w[2 * (size_t)i + 1] = (T)sn;
  }
}

__global__ void k_count_points(int n, const int* __restrict__ box, const int* __restrict__ lo,
                               const int* __restrict__ hi, unsigned long long* __restrict__ cnt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    atomicAdd(cnt, (unsigned long long)(hi[box[i]] - lo[box[i]]));
}

template <typename T, int DIM, int W>
int launch_form(PWArgs<T>& a, const FormIO& io, const FormPtrs<T>& fp, DBuf<T>& gs, cudaStream_t s) {
  size_t fix = fixed_smem(a, W, 1);
  size_t need = fix + sizeof(T) * (size_t)a.g.bufsz;
  int grid = std::max(1, std::min(io.max_items, kSMs));
  if constexpr (std::is_same<T, float>::value && DIM == 3 && TB + W - 1 <= TP - 1) {
    const int nbd = (a.g.G - W + 1 + TB - 1) / TB;
    const size_t tneed = tiled_offset<T>(a.g.G, a.g.K) + sizeof(T) * (size_t)a.g.bufsz;
    if (!a.g.wrap && nbd * nbd * nbd <= NBLK_MAX && tneed <= (size_t)MAXSMEM) {
      auto k = k_form<T, DIM, W, false, true>;
      set_smem(k, tneed);
      k<<<grid, PW_THREADS, tneed, s>>>(a, io, fp);
      FGT_LAUNCH_CHECK();
      return 1;
    }
  }
  if constexpr (std::is_same<T, double>::value && DIM == 3 && W <= 8) {
    const int nbd = (a.g.G - W + 1 + TB_D - 1) / TB_D;
    const size_t tneed = tiled_offset<T>(a.g.G, a.g.K) + sizeof(T) * (size_t)a.g.bufsz;
    if (!a.g.wrap && nbd * nbd * nbd <= NBLK_MAX && tneed <= (size_t)MAXSMEM) {
      auto k = k_form<T, DIM, W, false, true>;
      set_smem(k, tneed);
      k<<<grid, PW_THREADS, tneed, s>>>(a, io, fp);
      FGT_LAUNCH_CHECK();
      return 1;
    }
  }
  if (need <= (size_t)MAXSMEM) {
    auto k = k_form<T, DIM, W, false, false>;
    set_smem(k, need);
    k<<<grid, PW_THREADS, need, s>>>(a, io, fp);
  } else if (DIM == 3 && io.nslab > 1) {
    // x-slab grids (the expansions were zeroed by the caller)
    const size_t sm = fix + sizeof(T) * (size_t)a.g.str[0] * io.slab;
    auto k = k_form_slab<T, W>;
    set_smem(k, sm);
    k<<<grid, PW_THREADS, sm, s>>>(a, io, fp);
  } else {
    gs.alloc((size_t)grid * a.g.bufsz, s);
    a.gscratch = gs;
    auto k = k_form<T, DIM, W, true, false>;
    set_smem(k, fix);
    k<<<grid, PW_THREADS, fix, s>>>(a, io, fp);
  }
  FGT_LAUNCH_CHECK();
  return 1;
}

template <typename T, int DIM>
int form_w(int w, PWArgs<T>& a, const FormIO& io, const FormPtrs<T>& fp, DBuf<T>& gs, cudaStream_t s) {
  switch (w) {
    case 6: return launch_form<T, DIM, 6>(a, io, fp, gs, s);
    case 8: return launch_form<T, DIM, 8>(a, io, fp, gs, s);
    case 10: return launch_form<T, DIM, 10>(a, io, fp, gs, s);
    case 12: return launch_form<T, DIM, 12>(a, io, fp, gs, s);
    case 14: return launch_form<T, DIM, 14>(a, io, fp, gs, s);
    case 16: return launch_form<T, DIM, 16>(a, io, fp, gs, s);
    default: FGT_REQUIRE(false, FGT_ERR_UNSUPPORTED, "no form kernel for this width");
  }
  return 0;
}
// Shared memory of k_form_small2 and its warps per CTA (0: does not fit).
template <typename T>
int small2_warps(const Geo& g, size_t& smem) {
  const Small2Layout lay = small2_layout(g.G, g.K);
  const size_t fix = tw_bytes16<T>(g.G, g.K);
  const size_t per = sizeof(T) * (size_t)lay.per_warp;
  if (fix + per > (size_t)MAXSMEM) return 0;
  const int nw = (int)std::min<size_t>(8, ((size_t)MAXSMEM - fix) / per);
  smem = fix + per * nw;
  return nw;
}

template <typename T, int W>
void launch_form_small2(PWArgs<T>& a, const FormIO& io, const FormPtrs<T>& fp,
                        const uint32_t* order, const int* first, int* next, cudaStream_t s) {
  size_t smem = 0;
  const int nw = small2_warps<T>(a.g, smem);
  auto k = k_form_small2<T, W>;
  set_smem(k, smem);
  // as many 8-warp CTAs per SM as the shared memory allows (the warps of a
  // CTA share only the staged tables; more CTAs hide more latency)
  const int per_sm = std::max(1, std::min(8, (int)((size_t)(228 * 1024) / (smem + 1024))));
  k<<<kSMs * per_sm, 32 * nw, smem, s>>>(a, io, fp, order, first, next);
  FGT_LAUNCH_CHECK();
}
template <typename T>
void form_small2_w(int w, PWArgs<T>& a, const FormIO& io, const FormPtrs<T>& fp,
                   const uint32_t* order, const int* first, int* next, cudaStream_t s) {
  switch (w) {
    case 6: return launch_form_small2<T, 6>(a, io, fp, order, first, next, s);
    case 8: return launch_form_small2<T, 8>(a, io, fp, order, first, next, s);
    case 10: return launch_form_small2<T, 10>(a, io, fp, order, first, next, s);
    case 12: return launch_form_small2<T, 12>(a, io, fp, order, first, next, s);
    case 14: return launch_form_small2<T, 14>(a, io, fp, order, first, next, s);
    case 16: return launch_form_small2<T, 16>(a, io, fp, order, first, next, s);
    default: FGT_REQUIRE(false, FGT_ERR_UNSUPPORTED, "no form kernel for this width");
  }
}

void legendre(int nq, std::vector<double>& xq, std::vector<double>& wq) {
  const double pi = 4.0 * atan(1.0);
  xq.resize(nq);
  wq.resize(nq);
  for (int i = 0; i < nq; i++) {  // Newton on the Legendre polynomial
    double x = cos(pi * (i + 0.75) / (nq + 0.5)), dp = 1;
    for (int it = 0; it < 100; it++) {
      double p0 = 1, p1 = x;
      for (int j = 2; j <= nq; j++) {
        double p2 = ((2 * j - 1) * x * p1 - (j - 1) * p0) / j;
        p0 = p1;
        p1 = p2;
      }
      dp = nq * (x * p1 - p0) / (x * x - 1);
      double dxn = p1 / dp;
      x -= dxn;
      if (fabs(dxn) < 1e-16) break;
    }
    double p0 = 1, p1 = x;
    for (int j = 2; j <= nq; j++) {
      double p2 = ((2 * j - 1) * x * p1 - (j - 1) * p0) / j;
      p0 = p1;
      p1 = p2;
    }
    dp = nq * (x * p1 - p0) / (x * x - 1);
    xq[i] = x;
    wq[i] = 2 / ((1 - x * x) * dp * dp);
  }
}

}  // namespace

// ------------------------------------------------------------------ host set-up
void pw_grid(PWParams& P, int w, bool exact_w) {
  const double pi = 4.0 * atan(1.0);
  const int K = P.K, NF = 2 * K + 1;
  w = exact_w ? std::max(4, std::min(16, w)) : supported_w(std::max(4, std::min(16, w)));
  P.w = w;
  P.beta = 0.97 * pi * (1 - 1.0 / (2 * 2.0)) * w;
  P.halfw = w * P.dx / 2;
  double xmax = (P.boxsize_cut / 2) * (P.hpw / P.sqd0) * (1 + 1e-6) + 1e-12;
  int lmin = (int)ceil((-xmax - P.halfw) / P.dx);
  int lmax = (int)ceil((xmax - P.halfw) / P.dx) + w - 1;
  P.l0 = lmin;
  P.G = lmax - lmin + 1;
  P.wrap = false;
  if (P.G >= P.nf) {
    P.wrap = true;
    P.G = P.nf;
    P.l0 = 0;
  }
  // every in-place pass round needs one whole line per thread group
  FGT_REQUIRE(std::max(P.G, NF) <= PW_THREADS, FGT_ERR_UNSUPPORTED,
              "plane-wave expansion too long for the spreading kernels");
  // Fourier transform of the kernel, Gauss-Legendre on [-halfw, halfw]
  P.phihat.assign(NF, 0);
  // 200-point Gauss-Legendre rule, computed once per process
  static const std::pair<std::vector<double>, std::vector<double>> gl = [] {
    std::pair<std::vector<double>, std::vector<double>> r;
    legendre(200, r.first, r.second);
    return r;
  }();
  const std::vector<double>& xq = gl.first;
  const std::vector<double>& wq = gl.second;
  for (int k = -K; k <= K; k++) {
    double acc = 0;
    for (size_t i = 0; i < xq.size(); i++) {
      double z = xq[i];
      double ph = exp(P.beta * (sqrt(std::max(0.0, 1 - z * z)) - 1));
      acc += wq[i] * P.halfw * ph * cos(k * z * P.halfw);
    }
    P.phihat[k + K] = acc;
  }
}

void pw_setup(PWParams& P, int dim, int nd, int npw, double pmax, int periodic_nodes, double bs0,
              double delta, double eps, double boxsize_cut, int spread_width) {
  const double pi = 4.0 * atan(1.0);
  P.dim = dim;
  P.nd = nd;
  P.K = npw / 2;
  const int K = P.K, NF = 2 * K + 1;
  P.nexp = dim == 3 ? NF * NF * (K + 1) : (dim == 2 ? NF * (K + 1) : K + 1);
  double h;
  P.ts.assign(NF, 0);
  P.wsym.assign(NF, 0);
  std::vector<double> ws(NF);
  if (periodic_nodes) {
    // get_periodic_pwnodes, src/common/fgtterms.f:191-211 (delta0 = 1)
    h = 2 * pi / bs0;
    double w = sqrt(pi * delta) / bs0, hw = h * sqrt(delta) / 2;
    for (int k = -K; k <= K; k++) ws[k + K] = w * exp(-(hw * k) * (hw * k));
    P.delta0 = 1.0;
  } else {
    // get_pwnodes (trapezoid), src/common/fgtterms.f:151-179
    h = pmax / K;
    double w = h / (2.0 * sqrt(pi));
    for (int k = -K; k <= K; k++) {
      double t = k * h;
      ws[k + K] = w * exp(-t * t / 4);
    }
    P.delta0 = delta;
  }
  for (int k = -K; k <= K; k++) P.ts[k + K] = k * h;
  for (int k = -K + 1; k <= K - 1; k++) P.wsym[k + K] = ws[k + K];
  P.wsym[0] = P.wsym[2 * K] = ws[0] / 2;  // split the k=-K term over +-K
  P.hpw = h;
  P.sqd0 = sqrt(P.delta0);
  P.boxsize_cut = boxsize_cut;
  P.xmin = boxsize_cut / P.sqd0;
  // spreading grid (upsampling 2 over the 2K+1 modes), ES kernel
  P.nf = 2 * NF;
  P.dx = 2 * pi / P.nf;
  int w = spread_width > 0 ? spread_width : (int)ceil(log10(1.0 / eps)) + 2;
  pw_grid(P, w);
}

// ------------------------------------------------------------------ drivers
double pw_pass_flops(const PWParams& P) {
  const double G = P.G, NF = 2 * P.K + 1, NH = P.K + 1;
  double fma;
  if (P.dim == 3) fma = G * G * NH * G * 2 + G * NH * NF * G * 4 + NF * NH * NF * G * 4;
  else if (P.dim == 2) fma = G * NH * G * 2 + NH * NF * G * 4;
  else fma = NH * G * 2;
  return 2 * fma;
}

template <typename T>
int pw_form(const PWParams& P, const Tree& t, const Lists& L, const SourceSet<T>& src,
            PWData<T>& D, PWWork* work, cudaStream_t s) {
  if (L.n_form <= 0) {
    D.mp.alloc(2, s);
    return 0;
  }
  PWArgs<T> a;
  DevTables<T> tb;
  make_args<T>(P, a, tb, s, false, 0);
  D.mp.alloc((size_t)L.n_form * P.nd * 2 * P.nexp, s);
  FormIO io;
  io.n_form = L.n_form;
  io.ns = src.n;
  io.nd = P.nd;
  io.has_q = src.q != nullptr;
  io.has_dip = src.ds != nullptr;
  io.ncomp = (io.has_q ? 1 : 0) + (io.has_dip ? P.dim : 0);
  io.form_box = L.form_box;
  io.s_lo = src.lo;
  io.s_hi = src.hi;
  // longest-processing-time order of the form boxes (by source count) and a
  // work counter: the boxes' costs vary by several times, so a fixed
  // round-robin assignment leaves CTAs idle at the end.  Boxes above the
  // split threshold are cut into parts of about thr sources.
  DBuf<uint64_t> okey(std::max(L.n_form, 1), s), otmp(std::max(L.n_form, 1), s);
  DBuf<uint32_t> oval(std::max(L.n_form, 1), s), vtmp(std::max(L.n_form, 1), s);
  DBuf<int> next(1, s);
  next.zero();
  if (L.n_form > 0) {
    k_lpt_keys<<<grid_for(L.n_form, 256), 256, 0, s>>>(L.n_form, nullptr, L.form_box, nullptr,
                                                       src.lo, src.hi, nullptr, nullptr, okey,
                                                       oval);
    FGT_LAUNCH_CHECK();
    radix_sort(okey, oval, otmp, vtmp, L.n_form, LPT_BITS, s);
  }
  const int thr = form_split_threshold(src.n);
  // 2D: boxes with at most SMALL2_MAX sources (a suffix of the order) go to
  // the warp-per-box kernel, the rest to the CTA kernel
  size_t sm2 = 0;
  const bool small2 = P.dim == 2 && !a.g.wrap && small2_warps<T>(a.g, sm2) > 0;
  DBuf<int> first(1, s), next2(1, s);
  if (small2) {
    next2.zero();
    k_first_at_most<<<1, 32, 0, s>>>(okey, L.n_form, SMALL2_MAX, first);
    FGT_LAUNCH_CHECK();
  }
  // FP32 grids too large for shared memory: x-slabs (3D without
  // wrap-around).  FP64 keeps the global-memory grid: its shared-memory
  // atomics are no faster than global ones (the slab form of the FP64
  // eps = 1e-9 cell took 101 ms against 88 ms).
  SlabPlan sp;
  if (sizeof(T) == 4 &&
      sizeof(T) * (size_t)a.g.bufsz + order_offset<T>(a.g.G, a.g.K) > (size_t)MAXSMEM)
    sp = slab_plan(a.g, sizeof(T), order_offset<T>(a.g.G, a.g.K));
  if (sp.nslab > 1) D.mp.zero();
  if (work) work->slabs_form = sp.nslab;
  ItemList il;
  build_items(il, L.n_form, small2 ? first.get() : nullptr, oval, L.form_box, src.lo, src.hi,
              nullptr, nullptr, src.n, thr, true, s, sp.nslab);
  io.items = il.items;
  io.n_items = il.n_items;
  io.max_items = il.max_items;
  io.slab = sp.planes;
  io.nslab = sp.nslab;
  io.next = next;
  FormPtrs<T> fp;
  fp.off = src.off;
  fp.q = src.q;
  fp.ds = src.ds;
  fp.rn = src.rn;
  fp.mp = D.mp;
  DBuf<T> part((size_t)std::max(il.max_partial, 1) * P.nd * 2 * P.nexp, s);
  fp.partial = part;
  DBuf<T> gs;
  int n;
  if (P.dim == 1) n = form_w<T, 1>(P.w, a, io, fp, gs, s);
  else if (P.dim == 2) n = form_w<T, 2>(P.w, a, io, fp, gs, s);
  else n = form_w<T, 3>(P.w, a, io, fp, gs, s);
  if (small2) {
    form_small2_w<T>(P.w, a, io, fp, oval, first, next2, s);
    n += 2;
  }
  k_form_reduce<T><<<kSMs * 4, 256, 0, s>>>(il.split, il.n_split, P.nd, P.nexp, part, D.mp);
  FGT_LAUNCH_CHECK();
  n += 6;
  if (work) {
    DBuf<unsigned long long> c(1, s);
    c.zero();
    k_count_points<<<grid_for(L.n_form, 256), 256, 0, s>>>(L.n_form, L.form_box, src.lo, src.hi, c);
    FGT_LAUNCH_CHECK();
    unsigned long long h = 0;
    FGT_CUDA(cudaMemcpyAsync(&h, c.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    FGT_CUDA(cudaStreamSynchronize(s));
    const double wd = pow((double)P.w, P.dim), tr = (double)io.ncomp * P.nd;
    work->pts_form = (double)h;
    work->flops_form = tr * (L.n_form * pw_pass_flops(P) + (double)h * 2 * wd);
    n++;
  }
  return n;
}

template <typename T>
int pw_translate(const PWParams& P, const Lists& L, PWData<T>& D, PWWork* work, cudaStream_t s) {
  int nsh = P.dim == 1 ? 3 : (P.dim == 2 ? 9 : 27);
  D.wtab.alloc((size_t)nsh * 2 * P.nexp, s);
  DBuf<double> ts64(P.ts.size(), s);
  double* hts = static_cast<double*>(pinned_stage(2, sizeof(double) * P.ts.size()));
  std::copy(P.ts.begin(), P.ts.end(), hts);
  FGT_CUDA(cudaMemcpyAsync(ts64.get(), hts, sizeof(double) * P.ts.size(), cudaMemcpyHostToDevice,
                           s));
  pinned_stage_used(2, s);
  k_wtab<T><<<grid_for((long long)nsh * P.nexp, 256), 256, 0, s>>>(P.dim, P.K, P.nexp, ts64,
                                                                   P.xmin, D.wtab);
  FGT_LAUNCH_CHECK();
  D.loc.alloc((size_t)std::max(L.n_eval, 1) * P.nd * 2 * P.nexp, s);
  if (work)
    work->bytes_translate = (double)sizeof(T) * 2 * P.nexp * P.nd *
                            ((double)L.n_trans + 2.0 * L.n_eval);
  if (L.n_eval == 0) return 1;
  // a thread runs TRANS_MPT modes of TGE consecutive eval boxes, which
  // share most of their source expansions: the repeated reads hit L1
  constexpr int TGE = 4;
  int gx = std::max(1, ceil_div(P.nexp, 256 * TRANS_MPT));
  for (int e0 = 0; e0 < L.n_eval; e0 += 65535 * TGE) {
    int ne = std::min(65535 * TGE, L.n_eval - e0);
    dim3 grid(gx, ceil_div(ne, TGE));
    k_translate<T><<<grid, 256, 0, s>>>(ne, L.n_form, nsh, P.nexp, P.nd, TGE, L.eval_self.get() + e0,
                                        L.trans_ptr.get() + e0, L.trans_src, L.trans_w, D.mp,
                                        D.wtab, D.loc.get() + (size_t)e0 * P.nd * 2 * P.nexp);
    FGT_LAUNCH_CHECK();
  }
  return 2;
}

template int pw_form<float>(const PWParams&, const Tree&, const Lists&, const SourceSet<float>&,
                            PWData<float>&, PWWork*, cudaStream_t);
template int pw_form<double>(const PWParams&, const Tree&, const Lists&, const SourceSet<double>&,
                             PWData<double>&, PWWork*, cudaStream_t);
template int pw_translate<float>(const PWParams&, const Lists&, PWData<float>&, PWWork*,
                                 cudaStream_t);
template int pw_translate<double>(const PWParams&, const Lists&, PWData<double>&, PWWork*,
                                  cudaStream_t);

}  // namespace fgt
