// Device helpers shared by the plane-wave form/translate kernels (K6, K7,
// fgt_pw.cu) and the evaluation kernels (K8, fgt_pw_eval_impl.cuh).
//
// Per box, one CTA keeps the whole spreading sub-grid in shared memory (a
// global-memory slice per CTA when it does not fit): spread (ES kernel,
// Barnett-Magland-af Klinteberg 2019) -> in-place pruned DFT passes along the
// last, middle and first dimension -> deconvolution and PW weights fused into
// the pass that writes the expansion.  Only the sub-grid the box's points can
// reach is stored: for boxes of the cut-off size the scaled coordinates lie
// in [-pi/3, pi/3], about a third of the 2*pi period.
//
// 3D FP32 spreading accumulates blocks of points in register tiles
// (spread_tiled); the other spreading variants and the interpolation are
// thread-per-point.  Interpolation visits each box's points sorted by
// stencil base cell (order_cells: a warp reads few distinct addresses);
// thread-per-point spreading and the periodic full grids use a bank-balanced
// order (order_chunk: 32 distinct banks per stencil offset).
#pragma once
#include <math.h>

#include <algorithm>
#include <type_traits>
#include <vector>

#include "fgt_prims.cuh"
#include "fgt_pw.cuh"

namespace fgt {

namespace {

constexpr int PW_THREADS = 512;
constexpr int MODAL_THREADS = 256;
constexpr int ORDER_CHUNK = 2048;  // points ordered per round (u16 indices)
constexpr int MAXSMEM = 227 * 1024;

struct Geo {
  int dim, K, G, l0, nf, wrap, nexp, nd;
  int S[3], str[3];  // buffer extents and strides (T units) per dim
  int bufsz;
};

template <typename T>
struct PWArgs {
  Geo g;
  T halfw_over_dx, inv_hw, beta, dscale;  // inv_hw = dx / halfw
  double scale_d, inv_dx_d, hwdx_d;  // FP64 positions (points are FP64 offsets)
  const T* twf;   // [G][2K+1] fwd full (planar rows, see pad4)
  const T* twh;   // [G][K+1]  fwd half
  const T* tif;   // [2K+1][G] inv full
  const T* tih;   // [K+1][G]  inv half (with 1/2/2/.. weights)
  const T* facf;  // [2K+1] dx*wsym/phihat
  const T* faci;  // [2K+1] dx/phihat
  const T* ts;    // [2K+1] ts(k)
  T inv_sqd0;
  T* gscratch;  // global buffer slices when the grid does not fit in smem
};

// Twiddle tables are planar per input index l: row l holds the real parts
// of the nout outputs, zero-padded to a multiple of 4, then the imaginary
// parts (so a thread's 4 consecutive outputs are two 128-bit loads).
__host__ __device__ constexpr int pad4(int n) { return (n + 3) & ~3; }
// elements of the staged tables of either kernel: form G x (2K+1) and
// G x (K+1), evaluation (2K+1) x G and (K+1) x G, complex, planar rows
__host__ __device__ constexpr size_t tw_elems(int G, int K) {
  return 2 * (size_t)((size_t)G * (pad4(2 * K + 1) + pad4(K + 1)) > (size_t)pad4(G) * (3 * K + 2)
                          ? (size_t)G * (pad4(2 * K + 1) + pad4(K + 1))
                          : (size_t)pad4(G) * (3 * K + 2));
}

// Where the kernels read the twiddle tables: staged in shared memory (FP32),
// or from global memory through the L1 cache (FP64: the 8-byte grids of the
// eps = 1e-6 cells, ~200 KB, only fit in shared memory without the tables).
template <typename T>
__host__ __device__ constexpr bool tw_in_smem() {
  return sizeof(T) == 4;
}
template <typename T>
__host__ __device__ constexpr size_t tw_elems_t(int G, int K) {
  return tw_in_smem<T>() ? tw_elems(G, K) : 0;
}
// twiddle tables in shared memory, rounded up to 16 bytes (scratch or grids follow)
template <typename T>
__host__ __device__ constexpr size_t tw_bytes16(int G, int K) {
  return ((size_t)sizeof(T) * tw_elems_t<T>(G, K) + 15) & ~(size_t)15;
}

// byte offset of the grid buffer in shared memory: twiddles, then the
// ordering scratch (ORDER_CHUNK ints + 32 counters + ORDER_CHUNK u16)
template <typename T>
__host__ __device__ constexpr size_t order_offset(int G, int K) {
  return (((size_t)sizeof(T) * tw_elems_t<T>(G, K) + sizeof(int) * (ORDER_CHUNK + 32) +
           sizeof(unsigned short) * ORDER_CHUNK) + 15) &
         ~(size_t)15;
}

// ---------------------------------------------------------------- passes
// In-place line transforms over whole lines per round (a line is read
// completely before any of its outputs is written).
// MODE 0: real -> half complex (fwd, last dim), MODE 1: complex -> complex,
// MODE 2: half complex -> real (inv, last dim).
template <typename T, int MODE>
__device__ __forceinline__ void pass_inplace(T* B, int nl, int nb, int SA, int SB, int ein,
                                             int eout, int nin, int nout, const T* __restrict__ tw) {
  constexpr int LG = 2;
  static_assert(LG == 2, "two line pointers below");
  const int np = pad4(nout);  // twiddle row: np real parts, then np imaginary parts
  if constexpr (std::is_same<T, float>::value) {
    // FP32: a thread owns LG lines x 4 consecutive outputs; the twiddles of
    // its outputs are two 128-bit loads per input (real parts, imaginary
    // parts), and the accumulators are FP32x2 pairs of neighbouring outputs,
    // (re_k, re_k+1) += (xr, xr)(tr_k, tr_k+1) - (xi, xi)(ti_k, ti_k+1),
    // (im_k, im_k+1) += (xr, xr)(ti_k, ti_k+1) + (xi, xi)(tr_k, tr_k+1).
    // Lines past nl and outputs past nout compute on clamped or zero-padded
    // data and are not stored.
    const int nkg = np / 4;
    const int ngroups = blockDim.x / nkg;
    const int t = threadIdx.x, lg = t / nkg, kg = t - lg * nkg;
    const bool act_t = lg < ngroups;
    const int lpr = ngroups * LG;
    const float4* twr = reinterpret_cast<const float4*>(tw) + kg;  // + l * (np / 2) per row
    const int rstep = np / 2;                                       // float4 per row
    for (int r0 = 0; r0 < nl; r0 += lpr) {
      float2 ar[LG][2], ai[LG][2];
      int base[LG];
      bool lact[LG];
#pragma unroll
      for (int g = 0; g < LG; g++) {
        const int line = r0 + lg * LG + g;
        lact[g] = act_t && line < nl;
        const int lc = lact[g] ? line : 0;
        base[g] = (lc / nb) * SA + (lc % nb) * SB;
#pragma unroll
        for (int j = 0; j < 2; j++) {
          ar[g][j] = make_float2(0.f, 0.f);
          ai[g][j] = make_float2(0.f, 0.f);
        }
      }
      if (act_t) {
        const float4* tp = twr;
        const float* bp0 = B + base[0];
        const float* bp1 = B + base[LG - 1];
#pragma unroll 2
        for (int l = 0; l < nin; l++, tp += rstep, bp0 += ein, bp1 += ein) {
          const float4 TR = tp[0], TI = tp[np / 4];  // real row, imaginary row
          const float2 tr01 = make_float2(TR.x, TR.y), tr23 = make_float2(TR.z, TR.w);
          const float2 ti01 = make_float2(TI.x, TI.y), ti23 = make_float2(TI.z, TI.w);
#pragma unroll
          for (int g = 0; g < LG; g++) {
            const float* bp = g == 0 ? bp0 : bp1;
            if (MODE == 0) {
              const float gv = bp[0];
              const float2 gg = make_float2(gv, gv);
              ar[g][0] = __ffma2_rn(gg, tr01, ar[g][0]);
              ar[g][1] = __ffma2_rn(gg, tr23, ar[g][1]);
              ai[g][0] = __ffma2_rn(gg, ti01, ai[g][0]);
              ai[g][1] = __ffma2_rn(gg, ti23, ai[g][1]);
            } else {
              const float2 x = *reinterpret_cast<const float2*>(bp);
              const float2 xr = make_float2(x.x, x.x), nxi = make_float2(-x.y, -x.y);
              ar[g][0] = __ffma2_rn(nxi, ti01, __ffma2_rn(xr, tr01, ar[g][0]));
              ar[g][1] = __ffma2_rn(nxi, ti23, __ffma2_rn(xr, tr23, ar[g][1]));
              if (MODE == 1) {
                const float2 xi = make_float2(x.y, x.y);
                ai[g][0] = __ffma2_rn(xi, tr01, __ffma2_rn(xr, ti01, ai[g][0]));
                ai[g][1] = __ffma2_rn(xi, tr23, __ffma2_rn(xr, ti23, ai[g][1]));
              }
            }
          }
        }
      }
      __syncthreads();
#pragma unroll
      for (int g = 0; g < LG; g++) {
        if (!lact[g]) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int k = 4 * kg + j;
          if (k >= nout) break;
          const float re = (j & 1) ? ar[g][j >> 1].y : ar[g][j >> 1].x;
          if (MODE == 2) {
            B[base[g] + k * eout] = re;
          } else {
            const float im = (j & 1) ? ai[g][j >> 1].y : ai[g][j >> 1].x;
            B[base[g] + k * eout] = re;
            B[base[g] + k * eout + 1] = im;
          }
        }
      }
      __syncthreads();
    }
    return;
  }
  // FP64: LG lines x KG outputs per thread, outputs interleaved over the lanes
  constexpr int KG = 2;
  const int nkg = (nout + KG - 1) / KG;
  const int ngroups = blockDim.x / nkg;
  const int t = threadIdx.x, lg = t / nkg, kg = t - lg * nkg;
  const bool act_t = lg < ngroups;
  const int lpr = ngroups * LG;
  for (int r0 = 0; r0 < nl; r0 += lpr) {
    T re[LG][KG], im[LG][KG];
    int base[LG];
    bool lact[LG];
#pragma unroll
    for (int g = 0; g < LG; g++) {
      const int line = r0 + lg * LG + g;
      lact[g] = act_t && line < nl;
      base[g] = lact[g] ? (line / nb) * SA + (line % nb) * SB : 0;
#pragma unroll
      for (int j = 0; j < KG; j++) re[g][j] = im[g][j] = T(0);
    }
    if (act_t) {
      for (int l = 0; l < nin; l++) {
        T tr[KG], ti[KG];
#pragma unroll
        for (int j = 0; j < KG; j++) {
          const int k = kg + j * nkg;  // interleaved: neighbouring lanes, neighbouring modes
          const bool ok = k < nout;
          tr[j] = ok ? tw[(size_t)l * 2 * np + k] : T(0);
          ti[j] = ok ? tw[(size_t)l * 2 * np + np + k] : T(0);
        }
#pragma unroll
        for (int g = 0; g < LG; g++) {
          if (!lact[g]) continue;
          if (MODE == 0) {
            const T gv = B[base[g] + l * ein];
#pragma unroll
            for (int j = 0; j < KG; j++) {
              re[g][j] += gv * tr[j];
              im[g][j] += gv * ti[j];
            }
          } else {
            const T xr = B[base[g] + l * ein], xi = B[base[g] + l * ein + 1];
#pragma unroll
            for (int j = 0; j < KG; j++) {
              re[g][j] += xr * tr[j] - xi * ti[j];
              if (MODE == 1) im[g][j] += xr * ti[j] + xi * tr[j];
            }
          }
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int g = 0; g < LG; g++) {
      if (!lact[g]) continue;
#pragma unroll
      for (int j = 0; j < KG; j++) {
        const int k = kg + j * nkg;  // interleaved: neighbouring lanes, neighbouring modes
        if (k >= nout) break;
        if (MODE == 2) {
          B[base[g] + k * eout] = re[g][j];
        } else {
          B[base[g] + k * eout] = re[g][j];
          B[base[g] + k * eout + 1] = im[g][j];
        }
      }
    }
    __syncthreads();
  }
}

// ES kernel exp(beta (sqrt(1 - z^2) - 1)) with the exponent written as
// -beta z^2 / (1 + sqrt(1 - z^2)): no cancellation near the peak, where the
// direct form loses beta * 2^-24 of relative accuracy in FP32.
template <typename T>
__device__ __forceinline__ T es_kernel(T z, T beta) {
  const T q = T(1) - z * z;
  const T r = q > T(0) ? q * Real<T>::rsqrt_(q) : T(0);
  return Real<T>::expm(Real<T>::div12(beta * (z * z), T(1) + r));
}

__device__ __forceinline__ int pmod(int a, int n) {
  int c = a % n;
  return c < 0 ? c + n : c;
}

// ki[i] for a run-time i without demoting ki to local memory
__device__ __forceinline__ int sel3(const int* ki, int i) {
  return i == 0 ? ki[0] : (i == 1 ? ki[1] : ki[2]);
}

// Stencil cell offsets (T units) along each dimension.  Lin: the sub-grid
// case, cells base..base+W-1 (offsets fold into address immediates); Tab:
// the periodic full grid, cells wrap modulo nf (one modulo per dimension).
template <int DIM, int W>
struct LinIdx {
  int o[DIM];
  int str0, str1;
  __device__ __forceinline__ LinIdx(const Geo& g, const int* s) : str0(g.str[0]), str1(g.str[1]) {
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      int b = s[d] - g.l0;
      b = b < 0 ? 0 : (b > g.G - W ? g.G - W : b);
      o[d] = b * g.str[d];
    }
  }
  __device__ __forceinline__ int x(int j) const { return o[0] + j * (DIM == 1 ? 1 : str0); }
  __device__ __forceinline__ int y(int j) const { return o[1] + j * (DIM == 2 ? 1 : str1); }
  __device__ __forceinline__ int z(int j) const { return o[DIM - 1] + j; }
};
template <int DIM, int W>
struct TabIdx {
  int o[DIM][W];
  __device__ __forceinline__ TabIdx(const Geo& g, const int* s) {
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      int c = pmod(s[d], g.nf);
#pragma unroll
      for (int j = 0; j < W; j++) {
        o[d][j] = c * g.str[d];
        c = c + 1 == g.nf ? 0 : c + 1;
      }
    }
  }
  __device__ __forceinline__ int x(int j) const { return o[0][j]; }
  __device__ __forceinline__ int y(int j) const { return o[1][j]; }
  __device__ __forceinline__ int z(int j) const { return o[DIM - 1][j]; }
};

// Calls body(x offset, weight) for the W cells of a stencil's outer dimension
// with every register-array index a compile-time constant, so the kernel
// values never go to local memory: fully unrolled for W <= U, otherwise a
// rolled loop over rotating registers.
template <typename T, int W, int U, class IX, class F>
__device__ __forceinline__ void outer_cells(const IX& ix, const T* ph0, F&& body) {
  if constexpr (W <= U) {
#pragma unroll
    for (int j = 0; j < W; j++) body(ix.x(j), ph0[j]);
  } else {
    int xo[W];
    T pw[W];
#pragma unroll
    for (int j = 0; j < W; j++) {
      xo[j] = ix.x(j);
      pw[j] = ph0[j];
    }
#pragma unroll 1
    for (int j = 0; j < W; j++) {
      body(xo[0], pw[0]);
#pragma unroll
      for (int k = 0; k + 1 < W; k++) {
        xo[k] = xo[k + 1];
        pw[k] = pw[k + 1];
      }
    }
  }
}

// Read-only view of a grid in dynamic shared memory by 32-bit element offset:
// indexing the __shared__ array directly keeps every load a shared-space load
// with the stencil offsets in the address immediate.  The global-memory grid
// variants use a plain pointer, which supports the same + and [].
template <typename T>
struct SmemView {
  int base;  // element offset from the start of dynamic shared memory
  __device__ __forceinline__ SmemView operator+(int k) const { return SmemView{base + k}; }
  __device__ __forceinline__ T operator[](int i) const {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    return reinterpret_cast<const T*>(smem_raw)[base + i];
  }
};

template <typename T, int DIM, int W, class IX, class GV>
__device__ __forceinline__ T interp_cells(const GV& B, const IX& ix, const T (*ph)[W]) {
  T acc = T(0);
  if constexpr (DIM == 1) {
#pragma unroll
    for (int j = 0; j < W; j++) acc += B[ix.x(j)] * ph[0][j];
  } else if constexpr (DIM == 2) {
    outer_cells<T, W, 16>(ix, ph[0], [&](int xo, T p0) {
      const auto bx = B + xo;
      T sy = T(0);
#pragma unroll
      for (int jy = 0; jy < W; jy++) sy += bx[ix.z(jy)] * ph[1][jy];
      acc += sy * p0;
    });
  } else {
    outer_cells<T, W, 8>(ix, ph[0], [&](int xo, T p0) {
      const auto bx = B + xo;
      T sx = T(0);
#pragma unroll
      for (int jy = 0; jy < W; jy++) {
        const auto bxy = bx + ix.y(jy);
        T sy = T(0);
#pragma unroll
        for (int jz = 0; jz < W; jz++) sy += bxy[ix.z(jz)] * ph[2][jz];
        sx += sy * ph[1][jy];
      }
      acc += sx * p0;
    });
  }
  return acc;
}

template <typename T, int DIM, int W, class IX>
__device__ __forceinline__ void spread_cells(T* B, const IX& ix, const T (*ph)[W], T str) {
  if constexpr (DIM == 1) {
#pragma unroll
    for (int j = 0; j < W; j++) atomicAdd(B + ix.x(j), str * ph[0][j]);
  } else if constexpr (DIM == 2) {
    outer_cells<T, W, 16>(ix, ph[0], [&](int xo, T p0) {
      T* bx = B + xo;
      const T v = str * p0;
#pragma unroll
      for (int jy = 0; jy < W; jy++) atomicAdd(bx + ix.z(jy), v * ph[1][jy]);
    });
  } else {
    outer_cells<T, W, 8>(ix, ph[0], [&](int xo, T p0) {
      T* bx = B + xo;
      const T vx = str * p0;
#pragma unroll
      for (int jy = 0; jy < W; jy++) {
        T* bxy = bx + ix.y(jy);
        const T vxy = vx * ph[1][jy];
#pragma unroll
        for (int jz = 0; jz < W; jz++) atomicAdd(bxy + ix.z(jz), vxy * ph[2][jz]);
      }
    });
  }
}

// Thread-per-point interpolation (component grids of the hessian path).
template <typename T, int W>
__device__ __forceinline__ int kernel_row(const PWArgs<T>& a, double x, T* phi) {
  const double u = x * a.inv_dx_d;
  const int i0 = (int)ceil(u - a.hwdx_d);
  const T f0 = (T)((double)i0 - u);
#pragma unroll
  for (int j = 0; j < W; j++) phi[j] = es_kernel<T>((f0 + (T)j) * a.inv_hw, a.beta);
  return i0;
}

template <typename T, int DIM, int W, class GV>
__device__ __forceinline__ T interp_point(const PWArgs<T>& a, const GV& B, const double* x) {
  T ph[DIM][W];
  int s[DIM];
#pragma unroll
  for (int d = 0; d < DIM; d++) s[d] = kernel_row<T, W>(a, x[d], ph[d]);
  if (a.g.wrap) return interp_cells<T, DIM, W>(B, TabIdx<DIM, W>(a.g, s), ph);
  return interp_cells<T, DIM, W>(B, LinIdx<DIM, W>(a.g, s), ph);
}

template <typename T, int DIM, int W>
__device__ __forceinline__ void spread_point(const PWArgs<T>& a, T* B, const double* x, T str) {
  T ph[DIM][W];
  int s[DIM];
#pragma unroll
  for (int d = 0; d < DIM; d++) s[d] = kernel_row<T, W>(a, x[d], ph[d]);
  if (a.g.wrap)
    spread_cells<T, DIM, W>(B, TabIdx<DIM, W>(a.g, s), ph, str);
  else
    spread_cells<T, DIM, W>(B, LinIdx<DIM, W>(a.g, s), ph, str);
}

// Kernel values and their derivatives with respect to the point's original
// coordinate: d/dx phi((x_c - x)/halfw) = phi * beta * z / (sqrt(1-z^2) halfw),
// times the coordinate scale (a.dscale = scale / halfw).  Zero at |z| = 1.
template <typename T>
__device__ __forceinline__ void kernel_val_d(const PWArgs<T>& a, T f0, int j, T& phi, T& dphi) {
  const T z = (f0 + (T)j) * a.inv_hw;
  const T q = T(1) - z * z;
  const T rq = q > T(0) ? Real<T>::rsqrt_(q) : T(0);
  const T e = Real<T>::expm(Real<T>::div12(a.beta * (z * z), T(1) + q * rq));
  phi = e;
  dphi = e * (a.beta * a.dscale) * z * rq;
}
// First stencil cell of a coordinate and the offset f0 = i0 - x/dx of the
// kernel argument (cell j of the stencil is at f0 + j grid spacings).
template <typename T>
__device__ __forceinline__ int kernel_start(const PWArgs<T>& a, double x, T& f0) {
  const double u = x * a.inv_dx_d;
  const int i0 = (int)ceil(u - a.hwdx_d);
  f0 = (T)((double)i0 - u);
  return i0;
}
template <typename T, int W>
__device__ __forceinline__ int kernel_row_d(const PWArgs<T>& a, double x, T* phi, T* dphi) {
  T f0;
  const int i0 = kernel_start<T>(a, x, f0);
#pragma unroll
  for (int j = 0; j < W; j++) kernel_val_d<T>(a, f0, j, phi[j], dphi[j]);
  return i0;
}

// outer_cells with a second weight row (value and derivative along x)
template <typename T, int W, int U, class IX, class F>
__device__ __forceinline__ void outer_cells2(const IX& ix, const T* p0, const T* q0, F&& body) {
  if constexpr (W <= U) {
#pragma unroll
    for (int j = 0; j < W; j++) body(ix.x(j), p0[j], q0[j]);
  } else {
    int xo[W];
    T pw[W], qw[W];
#pragma unroll
    for (int j = 0; j < W; j++) {
      xo[j] = ix.x(j);
      pw[j] = p0[j];
      qw[j] = q0[j];
    }
#pragma unroll 1
    for (int j = 0; j < W; j++) {
      body(xo[0], pw[0], qw[0]);
#pragma unroll
      for (int k = 0; k + 1 < W; k++) {
        xo[k] = xo[k + 1];
        pw[k] = pw[k + 1];
        qw[k] = qw[k + 1];
      }
    }
  }
}

// Value and derivative sums of one stencil line in the last dimension,
// sum_j (B_j - bref) ph_j and sum_j (B_j - bref) dph_j.  FP32: cells in
// pairs with packed FP32x2 add/FMA (two lanes of arithmetic per instruction
// on sm_100), the last cell of an odd width alone.
template <typename T, int W, class IX, class GV>
__device__ __forceinline__ void line_sums(const GV& bl, const IX& ix, T bref, const T* ph,
                                          const T* dph, T& s0, T& s1) {
  if constexpr (std::is_same<T, float>::value) {
    float2 a0 = make_float2(0.f, 0.f), a1 = make_float2(0.f, 0.f);
    const float2 nb = make_float2(-bref, -bref);
#pragma unroll
    for (int j = 0; j + 1 < W; j += 2) {
      const float2 b = __fadd2_rn(make_float2(bl[ix.z(j)], bl[ix.z(j + 1)]), nb);
      a0 = __ffma2_rn(b, make_float2(ph[j], ph[j + 1]), a0);
      a1 = __ffma2_rn(b, make_float2(dph[j], dph[j + 1]), a1);
    }
    s0 = a0.x + a0.y;
    s1 = a1.x + a1.y;
    if constexpr (W % 2 == 1) {  // last cell of an odd width
      const float b = bl[ix.z(W - 1)] - bref;
      s0 += b * ph[W - 1];
      s1 += b * dph[W - 1];
    }
  } else {
    s0 = T(0);
    s1 = T(0);
#pragma unroll
    for (int j = 0; j < W; j++) {
      const T b = bl[ix.z(j)] - bref;
      s0 += b * ph[j];
      s1 += b * dph[j];
    }
  }
}

// Potential and gradient of one grid at one point: v[0] = pot, v[1+d] = d/dx_d.
// The sums run over B - Bref (Bref = the stencil's centre cell): the
// derivative stencils sum to the derivative of the kernel's partition of
// unity, which is at the aliasing level, so dropping Bref from them changes
// nothing, while the smaller summands keep the FP32 sums from cancelling
// when the field varies slowly over the stencil.  The potential adds Bref
// times the product of the kernel row sums back.
template <typename T, int DIM, int W, class IX, class GV>
__device__ __forceinline__ void interp_grad_cells(const GV& B, const IX& ix, const T (*ph)[W],
                                                  const T (*dph)[W], T* v) {
  T ksum = T(1);
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    T sd = T(0);
#pragma unroll
    for (int j = 0; j < W; j++) sd += ph[d][j];
    ksum *= sd;
  }
  if constexpr (DIM == 1) {
    const T bref = B[ix.x(W / 2)];
    T s0 = T(0), s1 = T(0);
#pragma unroll
    for (int j = 0; j < W; j++) {
      const T b = B[ix.x(j)] - bref;
      s0 += b * ph[0][j];
      s1 += b * dph[0][j];
    }
    v[0] = s0 + bref * ksum;
    v[1] = s1;
  } else if constexpr (DIM == 2) {
    const T bref = B[ix.x(W / 2) + ix.z(W / 2)];
    T pot = T(0), gx = T(0), gy = T(0);
    outer_cells2<T, W, 16>(ix, ph[0], dph[0], [&](int xo, T px, T dpx) {
      T s0, s1;
      line_sums<T, W>(B + xo, ix, bref, ph[1], dph[1], s0, s1);
      pot += px * s0;
      gx += dpx * s0;
      gy += px * s1;
    });
    v[0] = pot + bref * ksum;
    v[1] = gx;
    v[2] = gy;
  } else {
    const T bref = B[ix.x(W / 2) + ix.y(W / 2) + ix.z(W / 2)];
    T pot = T(0), gx = T(0), gy = T(0), gz = T(0);
    outer_cells2<T, W, 8>(ix, ph[0], dph[0], [&](int xo, T px, T dpx) {
      const auto bx = B + xo;
      T t0 = T(0), t1 = T(0), t2 = T(0);
#pragma unroll
      for (int jy = 0; jy < W; jy++) {
        T s0, s1;
        line_sums<T, W>(bx + ix.y(jy), ix, bref, ph[2], dph[2], s0, s1);
        t0 += ph[1][jy] * s0;
        t1 += dph[1][jy] * s0;
        t2 += ph[1][jy] * s1;
      }
      pot += px * t0;
      gx += dpx * t0;
      gy += px * t1;
      gz += px * t2;
    });
    v[0] = pot + bref * ksum;
    v[1] = gx;
    v[2] = gy;
    v[3] = gz;
  }
}

// ------------------------------------------- 3D FP32 stencil on a shared grid
// Compile-time loop: f(std::integral_constant<int, i>) for i = B .. E-1.
template <int B, int E, class F>
__device__ __forceinline__ void static_for(F&& f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    static_for<B + 1, E>(f);
  }
}
// Shared-space load at a 32-bit shared address plus a compile-time byte
// offset: one address register per stencil line, the cell offsets in the
// load's immediate.
template <int OFF>
__device__ __forceinline__ float lds_f32(uint32_t a) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1+%2];" : "=f"(v) : "r"(a), "n"(OFF));
  return v;
}
__device__ __forceinline__ float lds_f32(uint32_t a) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
  return v;
}

// line_sums for a line of a grid in shared memory starting at byte address la.
template <int W>
__device__ __forceinline__ void line_sums_smem(uint32_t la, float bref, const float* ph,
                                               const float* dph, float& s0, float& s1) {
  const float2 nb = make_float2(-bref, -bref);
  float2 a0, a1;
  {
    const float2 b = __fadd2_rn(make_float2(lds_f32<0>(la), lds_f32<4>(la)), nb);
    a0 = __fmul2_rn(b, make_float2(ph[0], ph[1]));
    a1 = __fmul2_rn(b, make_float2(dph[0], dph[1]));
  }
  static_for<1, W / 2>([&](auto P) {
    constexpr int j = 2 * decltype(P)::value;
    const float2 b = __fadd2_rn(make_float2(lds_f32<4 * j>(la), lds_f32<4 * j + 4>(la)), nb);
    a0 = __ffma2_rn(b, make_float2(ph[j], ph[j + 1]), a0);
    a1 = __ffma2_rn(b, make_float2(dph[j], dph[j + 1]), a1);
  });
  if constexpr (W % 2 == 1) {
    const float b = lds_f32<4 * (W - 1)>(la) - bref;
    a0.x = fmaf(b, ph[W - 1], a0.x);
    a1.x = fmaf(b, dph[W - 1], a1.x);
  }
  s0 = a0.x + a0.y;
  s1 = a1.x + a1.y;
}

// interp_grad_point for a 3D FP32 grid in shared memory without wrap-around
// (grid at shared byte address gb): the same sums over B - Bref, with the
// stencil addresses advanced by one add per line and the x weights computed
// as the rolled x loop reaches them (no register rotation).
template <int W>
__device__ __forceinline__ void interp_grad_point_s3(const PWArgs<float>& a, uint32_t gb,
                                                     const double* x, float* v) {
  const Geo& g = a.g;
  float ph[2][W], dph[2][W];  // y and z rows
  float f0x;
  int s[3];
  s[0] = kernel_start<float>(a, x[0], f0x);
  s[1] = kernel_row_d<float, W>(a, x[1], ph[0], dph[0]);
  s[2] = kernel_row_d<float, W>(a, x[2], ph[1], dph[1]);
  const LinIdx<3, W> ix(g, s);
  const uint32_t str0 = 4u * (uint32_t)g.str[0], str1 = 4u * (uint32_t)g.str[1];
  const uint32_t a0 = gb + 4u * (uint32_t)(ix.o[0] + ix.o[1] + ix.o[2]);
  const float bref = lds_f32(a0 + (W / 2) * (str0 + str1) + 4u * (W / 2));
  float ksy = 0.f, ksz = 0.f;
#pragma unroll
  for (int j = 0; j < W; j++) ksy += ph[0][j];
#pragma unroll
  for (int j = 0; j < W; j++) ksz += ph[1][j];
  float pot = 0.f, gx = 0.f, gy = 0.f, gz = 0.f, ksx = 0.f;
  uint32_t ax = a0;
#pragma unroll 1
  for (int jx = 0; jx < W; jx++, ax += str0) {
    float px, dpx;
    kernel_val_d<float>(a, f0x, jx, px, dpx);
    ksx += px;
    float t0 = 0.f, t1 = 0.f, t2 = 0.f;
    uint32_t ay = ax;
#pragma unroll
    for (int jy = 0; jy < W; jy++, ay += str1) {
      float s0, s1;
      line_sums_smem<W>(ay, bref, ph[1], dph[1], s0, s1);
      t0 += ph[0][jy] * s0;
      t1 += dph[0][jy] * s0;
      t2 += ph[0][jy] * s1;
    }
    pot += px * t0;
    gx += dpx * t0;
    gy += px * t1;
    gz += px * t2;
  }
  v[0] = pot + bref * ((ksx * ksy) * ksz);
  v[1] = gx;
  v[2] = gy;
  v[3] = gz;
}

// interp_grad_point for 3D grids without wrap-around, with the x weights
// computed as the rolled x loop reaches them: only the y and z rows (values
// and derivatives) stay in registers, so the FP64 stencil fits the 128
// registers of a 512-thread CTA.  Same sums as interp_grad_cells.
template <typename T, int W, class GV>
__device__ __forceinline__ void interp_grad_point_xr(const PWArgs<T>& a, const GV& B,
                                                     const double* x, T* v) {
  T ph[2][W], dph[2][W];  // y and z rows
  T f0x;
  int s[3];
  s[0] = kernel_start<T>(a, x[0], f0x);
  s[1] = kernel_row_d<T, W>(a, x[1], ph[0], dph[0]);
  s[2] = kernel_row_d<T, W>(a, x[2], ph[1], dph[1]);
  const LinIdx<3, W> ix(a.g, s);
  const T bref = B[ix.x(W / 2) + ix.y(W / 2) + ix.z(W / 2)];
  T ksy = T(0), ksz = T(0), ksx = T(0);
#pragma unroll
  for (int j = 0; j < W; j++) {
    ksy += ph[0][j];
    ksz += ph[1][j];
  }
  T pot = T(0), gx = T(0), gy = T(0), gz = T(0);
#pragma unroll 1
  for (int jx = 0; jx < W; jx++) {
    T px, dpx;
    kernel_val_d<T>(a, f0x, jx, px, dpx);
    ksx += px;
    const auto bx = B + ix.x(jx);
    T t0 = T(0), t1 = T(0), t2 = T(0);
#pragma unroll
    for (int jy = 0; jy < W; jy++) {
      T s0, s1;
      line_sums<T, W>(bx + ix.y(jy), ix, bref, ph[1], dph[1], s0, s1);
      t0 += ph[0][jy] * s0;
      t1 += dph[0][jy] * s0;
      t2 += ph[0][jy] * s1;
    }
    pot += px * t0;
    gx += dpx * t0;
    gy += px * t1;
    gz += px * t2;
  }
  v[0] = pot + bref * ((ksx * ksy) * ksz);
  v[1] = gx;
  v[2] = gy;
  v[3] = gz;
}

template <typename T, int DIM, int W, class GV>
__device__ __forceinline__ void interp_grad_point(const PWArgs<T>& a, const GV& B, const double* x,
                                                  T* v) {
  T ph[DIM][W], dph[DIM][W];
  int s[DIM];
#pragma unroll
  for (int d = 0; d < DIM; d++) s[d] = kernel_row_d<T, W>(a, x[d], ph[d], dph[d]);
  if (a.g.wrap)
    interp_grad_cells<T, DIM, W>(B, TabIdx<DIM, W>(a.g, s), ph, dph, v);
  else
    interp_grad_cells<T, DIM, W>(B, LinIdx<DIM, W>(a.g, s), ph, dph, v);
}

// Bank-balanced processing order of a chunk of points.  Thread-per-point
// stencils touch B[base_p + offset] for the same offset in every lane at
// once; ordering the chunk by (rank within bank class, bank class) with
// class = base_p mod NCLASS puts NCLASS different classes into every run of
// NCLASS consecutive points, so those accesses hit distinct banks.
template <typename T, int DIM, int W>
__device__ __forceinline__ void order_chunk(const PWArgs<T>& a, const double* off, int ne, int q0,
                                            int n, unsigned short* perm, int* tmp, int* cnt) {
  constexpr int NCLASS = sizeof(T) == 4 ? 32 : 16;  // 4-byte banks
  const Geo& g = a.g;
  if (threadIdx.x < NCLASS) cnt[threadIdx.x] = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    int base = 0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      const double u = off[(size_t)d * ne + q0 + i] * a.scale_d * a.inv_dx_d;
      const int i0 = (int)ceil(u - a.hwdx_d);
      int b = g.wrap ? pmod(i0, g.nf) : i0 - g.l0;
      if (!g.wrap) b = b < 0 ? 0 : (b > g.G - W ? g.G - W : b);
      base += b * g.str[d];
    }
    const int cls = base & (NCLASS - 1);
    const int rank = atomicAdd(&cnt[cls], 1);
    tmp[i] = rank * NCLASS + cls;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int rank = tmp[i] / NCLASS, cls = tmp[i] % NCLASS;
    int pos = 0;
#pragma unroll 8
    for (int c = 0; c < NCLASS; c++) {
      const int k = cnt[c];
      pos += k < rank ? k : rank;
      pos += (c < cls && k > rank) ? 1 : 0;
    }
    perm[pos] = (unsigned short)i;
  }
  __syncthreads();
}

// Processing order of a chunk of points sorted by stencil base cell: a
// counting sort over the (G-W+1)^DIM base cells of the sub-grid (nbins <=
// NBINS_MAX).  Points that share a base cell become consecutive, so the lanes
// of a warp read few distinct addresses at every stencil offset (equal
// addresses are broadcast); distinct cells in a warp are neighbours in memory
// and fall into different banks.  Bin k lives at slot (k % per) * blockDim +
// k / per, so each thread's serial pass over its `per` consecutive bins reads
// consecutive words across the block.  ws: 32 ints.
constexpr int NBINS_MAX = 8192;

template <typename T, int DIM, int W>
__device__ __forceinline__ void order_cells(const PWArgs<T>& a, const double* off, int ne, int q0,
                                            int n, int nbins, unsigned short* perm, int* tmp,
                                            int* bins, int* ws) {
  const Geo& g = a.g;
  const int nb = g.G - W + 1, bd = blockDim.x, t = threadIdx.x;
  const int per = (nbins + bd - 1) / bd;
  auto slot = [&](int k) { return (k % per) * bd + k / per; };
  for (int i = t; i < per * bd; i += bd) bins[i] = 0;
  __syncthreads();
  for (int i = t; i < n; i += bd) {
    int key = 0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      const double u = off[(size_t)d * ne + q0 + i] * a.scale_d * a.inv_dx_d;
      int b = (int)ceil(u - a.hwdx_d) - g.l0;
      b = b < 0 ? 0 : (b > g.G - W ? g.G - W : b);
      key = key * nb + b;
    }
    const int r = atomicAdd(&bins[slot(key)], 1);
    tmp[i] = key | (r << 13);
  }
  __syncthreads();
  // exclusive scan over the bins in key order
  int sum = 0;
  for (int i = 0; i < per; i++) sum += bins[i * bd + t];
  const int lane = t & 31, w = t >> 5, nw = bd >> 5;
  int inc = sum;
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
  int ex = ws[w] + inc - sum;
  for (int i = 0; i < per; i++) {
    const int c = bins[i * bd + t];
    bins[i * bd + t] = ex;
    ex += c;
  }
  __syncthreads();
  for (int i = t; i < n; i += bd) {
    const int v = tmp[i];
    perm[bins[slot(v & (NBINS_MAX - 1))] + (v >> 13)] = (unsigned short)i;
  }
  __syncthreads();
}

// byte offset of the grid buffer in the evaluation kernel: the ordering
// scratch of order_offset, then the cell-order bins and scan workspace
template <typename T>
__host__ __device__ constexpr size_t eval_offset(int G, int K) {
  // FP32: the cell-order bins; FP64 grids use the bank-class order (no bins)
  return order_offset<T>(G, K) + (sizeof(T) == 4 ? sizeof(int) * (NBINS_MAX + 32) : 0);
}

// Keys of a longest-processing-time order: entry i of a box list (list[i]
// indexes `box`; the identity when list is null) gets key MAXC - cost, with
// cost = points of the box in one or two evaluation sets, so an ascending
// sort puts the most expensive boxes first.  Entries at or beyond *count
// (when count is given) sort after all others.
constexpr int LPT_BITS = 25;
__global__ void k_lpt_keys(int n, const int* __restrict__ count, const int* __restrict__ box,
                           const int* __restrict__ list, const int* __restrict__ lo0,
                           const int* __restrict__ hi0, const int* __restrict__ lo1,
                           const int* __restrict__ hi1, uint64_t* __restrict__ keys,
                           uint32_t* __restrict__ vals) {
  const int m = count ? *count : n;
  constexpr uint64_t MAXC = (1ull << (LPT_BITS - 1)) - 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int e = list ? list[i] : i;
    vals[i] = (uint32_t)e;
    if (i >= m) {
      keys[i] = 1ull << (LPT_BITS - 1);
      continue;
    }
    const int b = box[e];
    long long c = (long long)(hi0[b] - lo0[b]) + (lo1 ? (long long)(hi1[b] - lo1[b]) : 0);
    c = c < 0 ? 0 : (c > (long long)MAXC ? (long long)MAXC : c);
    keys[i] = MAXC - (uint64_t)c;
  }
}

// Work items of the form and grid-evaluation kernels.  A box whose point
// count exceeds the split threshold is cut into `nparts` contiguous point
// ranges of about equal size, each a separate item, so one large box (at a
// cut-off level 0 the root box holds every point) keeps every SM busy
// instead of one.  The items of a box are consecutive and follow the
// longest-processing-time order of the boxes.  pslot: slot of the item's
// partial expansion (form items of split boxes), -1 otherwise.
struct WorkItem {
  int slot, part, nparts, pslot;
};
// A split form box: its form slot, first partial slot and part count.
struct SplitRec {
  int slot, pslot, nparts;
};

// Part count of entry i of a sorted slot list (entries at or beyond *count
// get 0): ceil(points / thr) point parts when the box holds more than thr
// points, else 1, times nslab grid slabs (x-slab grids: every part of a box
// spreads or interpolates into one slab).  nsplit[i] = part count of boxes
// split into point parts with partial expansions (no slabs), 0 otherwise.
__global__ void k_item_parts(int n, const int* __restrict__ count, const uint32_t* __restrict__ order,
                             const int* __restrict__ box, const int* __restrict__ lo0,
                             const int* __restrict__ hi0, const int* __restrict__ lo1,
                             const int* __restrict__ hi1, int thr, int nslab,
                             int* __restrict__ nparts, int* __restrict__ nsplit) {
  const int m = count ? *count : n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int np = 0;
    if (i < m) {
      const int b = box[order[i]];
      const long long c =
          (long long)(hi0[b] - lo0[b]) + (lo1 ? (long long)(hi1[b] - lo1[b]) : 0);
      np = c > thr ? (int)((c + thr - 1) / thr) : 1;
    }
    nparts[i] = np * nslab;
    nsplit[i] = (nslab == 1 && np > 1) ? np : 0;
  }
}

// Items of every entry (offsets from exclusive scans of nparts and nsplit);
// split boxes are also listed in `split` (order of the list unspecified; each
// record carries its own slots, so results do not depend on it).  With
// nslab > 1, part p is slab p % nslab of point part p / nslab, and no item
// has a partial slot (the slab kernels add into the box's expansion).
__global__ void k_item_fill(int n, const int* __restrict__ count, const uint32_t* __restrict__ order,
                            const int* __restrict__ nparts, const int* __restrict__ ioff,
                            const int* __restrict__ poff, int nslab, WorkItem* __restrict__ items,
                            SplitRec* __restrict__ split, int* __restrict__ nsplit_total) {
  const int m = count ? *count : n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const int np = nparts[i], slot = (int)order[i], o = ioff[i];
    for (int p = 0; p < np; p++) {
      WorkItem w;
      w.slot = slot;
      w.part = p;
      w.nparts = np;
      w.pslot = (nslab == 1 && np > 1) ? poff[i] + p : -1;
      items[o + p] = w;
    }
    if (nslab == 1 && np > 1 && split) {
      const int k = atomicAdd(nsplit_total, 1);
      SplitRec r;
      r.slot = slot;
      r.pslot = poff[i];
      r.nparts = np;
      split[k] = r;
    }
  }
}

// Split thresholds (points per part) of the form and grid-evaluation
// kernels for a call with n points in the set: about two parts per SM when
// every point sits in one box, never below the size at which the per-part
// grid transforms stop being small against the spreading or interpolation.
inline int form_split_threshold(long long n) {
  return (int)std::max<long long>(8192, (n + 2 * kSMs - 1) / (2 * kSMs));
}
inline int eval_split_threshold(long long n) {
  return (int)std::max<long long>(8192, (n + 2 * kSMs - 1) / (2 * kSMs));
}

// Work items of a sorted slot list (host side, all sizes stay on the device).
// n: list length bound; count: actual length on the device (or null = n);
// npts_bound: upper bound of the points over all listed boxes; thr: split
// threshold; nslab: grid slabs per box (1: whole grids).  Items and split
// records live in the call's workspace.
struct ItemList {
  DBuf<WorkItem> items;
  DBuf<SplitRec> split;
  DBuf<int> n_items, n_split, n_partial;
  int max_items = 0, max_partial = 0;
};
inline void build_items(ItemList& il, int n, const int* count, const uint32_t* order,
                        const int* box, const int* lo0, const int* hi0, const int* lo1,
                        const int* hi1, long long npts_bound, int thr, bool want_split,
                        cudaStream_t s, int nslab = 1) {
  // every split box holds more than thr points and has at most 2*points/thr
  // parts; every other box has one
  const long long extra = 2 * (npts_bound / std::max(thr, 1)) + 1;
  il.max_items = (int)std::min<long long>(((long long)n + extra) * nslab, 1ll << 30);
  il.max_partial = (int)std::min<long long>(extra, 1ll << 30);
  DBuf<int> np(std::max(n, 1), s), ns(std::max(n, 1), s), ioff(std::max(n, 1), s),
      poff(std::max(n, 1), s);
  il.items.alloc(std::max(il.max_items, 1), s);
  il.n_items.alloc(1, s);
  il.n_partial.alloc(1, s);
  il.n_split.alloc(1, s);
  il.n_split.zero();
  if (want_split) il.split.alloc(std::max(il.max_partial, 1), s);
  if (n <= 0) {
    il.n_items.zero();
    il.n_partial.zero();
    return;
  }
  k_item_parts<<<grid_for(n, 256), 256, 0, s>>>(n, count, order, box, lo0, hi0, lo1, hi1, thr,
                                                 nslab, np, ns);
  FGT_LAUNCH_CHECK();
  exclusive_scan_i32(np, ioff, n, il.n_items, s);
  exclusive_scan_i32(ns, poff, n, il.n_partial, s);
  k_item_fill<<<grid_for(n, 256), 256, 0, s>>>(n, count, order, np, ioff, poff, nslab, il.items,
                                                want_split ? il.split.get() : nullptr, il.n_split);
  FGT_LAUNCH_CHECK();
}

// x-slab grids (3D, no wrap-around): a grid too large for shared memory is
// cut into nslab slabs of at most `planes` whole x-planes (each plane holds
// str[0] elements), sized so that `fixed` bytes of scratch plus one slab fit
// in SLAB_SMEM bytes of shared memory.  The passes along z and y stay inside
// an x-plane; only the x transform and the stencils' x extent cross slabs.
constexpr size_t SLAB_SMEM = 216 * 1024;
struct SlabPlan {
  int planes = 0, nslab = 1;
  size_t smem = 0;
};
inline SlabPlan slab_plan(const Geo& g, size_t tsize, size_t fixed) {
  SlabPlan r;
  const size_t plane = tsize * (size_t)g.str[0];
  if (g.dim != 3 || g.wrap || fixed + plane > SLAB_SMEM) return r;
  const int pmax = (int)((SLAB_SMEM - fixed) / plane);
  r.nslab = (g.G + pmax - 1) / pmax;
  r.planes = (g.G + r.nslab - 1) / r.nslab;
  r.smem = fixed + plane * (size_t)r.planes;
  return r;
}

// Point range [q0, q1) of part `part` of `nparts` of [lo, hi).
__device__ __forceinline__ void part_range(int lo, int hi, int part, int nparts, int& q0, int& q1) {
  if (nparts <= 1) {
    q0 = lo;
    q1 = hi;
    return;
  }
  const int chunk = (hi - lo + nparts - 1) / nparts;
  q0 = min(hi, lo + part * chunk);
  q1 = min(hi, q0 + chunk);
}

// ------------------------------------------------ small 2D boxes, one warp each
// A 2D box of the cut-off level with a few hundred points needs only
// ~1e5 FMAs of spreading and passes: one CTA per box spends most of its time
// in block barriers and shared-memory atomics.  These kernels give each box
// to one warp: spreading walks the box's points in order with the lanes
// owning the stencil's cells (plain read-modify-writes, no atomics), and the
// line transforms are warp-wide register-blocked sums.  Per warp: the real
// grid A (G rows of SA values, SA odd so lane-per-row accesses hit distinct
// banks) and half-complex grids of SC values per row.  Region R1 holds the
// real grid (form: spreading target; evaluation: the grid interpolated) or,
// in the evaluation, first the modes (2K+1 rows); region R2 holds the G rows
// of the half-complex intermediate of the two line passes.
constexpr int SMALL2_MAX = 2048;  // points per box handled by a warp
struct Small2Layout {
  int SA, SC, r1, per_warp;  // r1, per_warp in elements
};
__host__ __device__ inline Small2Layout small2_layout(int G, int K) {
  Small2Layout l;
  l.SA = G | 1;
  l.SC = (2 * (K + 1)) | 1;
  const int a = G * l.SA, b = (2 * K + 1) * l.SC;
  l.r1 = ((a > b ? a : b) + 3) & ~3;
  l.per_warp = (l.r1 + G * l.SC + 3) & ~3;
  return l;
}

// Pass along the last dimension, real -> half complex (form):
// C[r][2k..2k+1] = sum_y A[r][y] tw[y][k], k < NH, lane r < G.
template <typename T>
__device__ __forceinline__ void warp_pass_r2c(const T* A, int SA, T* C, int SC, int G, int NH,
                                              const T* tw) {
  const int np = pad4(NH), lane = threadIdx.x & 31;
  for (int r = lane; r < G; r += 32) {
    const T* a = A + r * SA;
    for (int k0 = 0; k0 < NH; k0 += 4) {
      T re[4] = {T(0), T(0), T(0), T(0)}, im[4] = {T(0), T(0), T(0), T(0)};
      const T* t = tw + k0;
      for (int y = 0; y < G; y++, t += 2 * np) {
        const T g = a[y];
#pragma unroll
        for (int j = 0; j < 4; j++) {
          re[j] += g * t[j];
          im[j] += g * t[np + j];
        }
      }
#pragma unroll
      for (int j = 0; j < 4; j++)
        if (k0 + j < NH) {
          C[r * SC + 2 * (k0 + j)] = re[j];
          C[r * SC + 2 * (k0 + j) + 1] = im[j];
        }
    }
  }
}

// Pass along the last dimension, half complex -> real (evaluation):
// A[r][y] = sum_k Re(C[r][k] tw[k][y]), y < G, lane r < G.
template <typename T>
__device__ __forceinline__ void warp_pass_c2r(const T* C, int SC, T* A, int SA, int G, int NH,
                                              const T* tw) {
  const int np = pad4(G), lane = threadIdx.x & 31;
  for (int r = lane; r < G; r += 32) {
    const T* c = C + r * SC;
    for (int y0 = 0; y0 < G; y0 += 4) {
      T acc[4] = {T(0), T(0), T(0), T(0)};
      const T* t = tw + y0;
      for (int k = 0; k < NH; k++, t += 2 * np) {
        const T cr = c[2 * k], ci = c[2 * k + 1];
#pragma unroll
        for (int j = 0; j < 4; j++) acc[j] += cr * t[j] - ci * t[np + j];
      }
#pragma unroll
      for (int j = 0; j < 4; j++)
        if (y0 + j < G) A[r * SA + y0 + j] = acc[j];
    }
  }
}

// Complex pass along the first dimension over the NH columns of C:
// out(o, k) = sum_i C[i][k] tw[i][o], o < nout, i < nin; the lanes take
// (column, group of 4 outputs) pairs and hand every finished group to
// emit(o, k, re, im).
template <typename T, class F>
__device__ __forceinline__ void warp_pass_c2c(const T* C, int SC, int nin, int nout, int NH,
                                              const T* tw, F&& emit) {
  const int np = pad4(nout), ng = (nout + 3) / 4, lane = threadIdx.x & 31;
  for (int pr = lane; pr < NH * ng; pr += 32) {
    const int k = pr / ng, o0 = (pr - k * ng) * 4;
    T re[4] = {T(0), T(0), T(0), T(0)}, im[4] = {T(0), T(0), T(0), T(0)};
    const T* c = C + 2 * k;
    const T* t = tw + o0;
    for (int i = 0; i < nin; i++, c += SC, t += 2 * np) {
      const T xr = c[0], xi = c[1];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        re[j] += xr * t[j] - xi * t[np + j];
        im[j] += xr * t[np + j] + xi * t[j];
      }
    }
#pragma unroll
    for (int j = 0; j < 4; j++)
      if (o0 + j < nout) emit(o0 + j, k, re[j], im[j]);
  }
}

template <typename T>
__device__ __forceinline__ void load_tw(T* dst, const T* src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}
// A twiddle table for the kernel: staged at `smem` (FP32) or read in place.
template <typename T>
__device__ __forceinline__ const T* stage_tw(T* smem, const T* src, int n) {
  if constexpr (tw_in_smem<T>()) {
    load_tw(smem, src, n);
    return smem;
  } else {
    return src;
  }
}

int supported_w(int w) {
  const int ws[] = {6, 8, 10, 12, 14, 16};
  for (int v : ws)
    if (w <= v) return v;
  return 16;
}

template <typename T>
struct DevTables {
  DBuf<T> all;  // twf, twh, tif, tih, facf, faci, ts back to back
};

// Pinned host staging of small host-computed tables, per host thread and
// slot (0: form tables, 1: evaluation tables, 2: translation nodes).  The
// tables go to the device with one asynchronous copy (a pageable source would
// make the copy wait for the stream); a slot is rewritten only by a later
// call, after that call's final stream synchronisation.
// Event recorded after the last asynchronous copy out of a staging slot; the
// slot is rewritten only once that copy has run (one call can stage the same
// slot twice, e.g. the two evaluation launches of a host-buffer call).
inline cudaEvent_t& pinned_stage_event(int slot) {
  static thread_local cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  return ev[slot];
}
inline void pinned_stage_used(int slot, cudaStream_t s) {
  cudaEvent_t& e = pinned_stage_event(slot);
  if (!e) FGT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  FGT_CUDA(cudaEventRecord(e, s));
}
inline void* pinned_stage(int slot, size_t bytes) {
  static thread_local void* buf[3] = {nullptr, nullptr, nullptr};
  static thread_local size_t cap[3] = {0, 0, 0};
  if (cudaEvent_t e = pinned_stage_event(slot)) FGT_CUDA(cudaEventSynchronize(e));
  if (cap[slot] < bytes) {
    if (buf[slot]) cudaFreeHost(buf[slot]);
    buf[slot] = nullptr;
    cap[slot] = 0;
    const size_t want = std::max(bytes, (size_t)1 << 20);
    FGT_CUDA(cudaHostAlloc(&buf[slot], want, cudaHostAllocDefault));
    cap[slot] = want;
  }
  return buf[slot];
}

template <typename T>
void make_args(const PWParams& P, PWArgs<T>& a, DevTables<T>& tb, cudaStream_t s, bool pad,
               int slot) {
  Geo& g = a.g;
  g.dim = P.dim;
  g.K = P.K;
  g.G = P.G;
  g.l0 = P.l0;
  g.nf = P.nf;
  g.wrap = P.wrap ? 1 : 0;
  g.nexp = P.nexp;
  g.nd = P.nd;
  const int K = P.K, NF = 2 * K + 1, NH = K + 1, G = P.G;
  int S[3] = {1, 1, 1};
  if (P.dim == 3) {
    S[0] = std::max(G, NF);
    S[1] = std::max(G, NF);
    S[2] = std::max(G, 2 * NH);
  } else if (P.dim == 2) {
    S[0] = std::max(G, NF);
    S[1] = std::max(G, 2 * NH);
  } else {
    S[0] = std::max(G, 2 * NH);
  }
  // even last extent: every complex element (re, im) of the passes starts
  // at an even element offset, as the FP32 passes' 8-byte loads require
  S[P.dim - 1] += S[P.dim - 1] & 1;
  if (pad && sizeof(T) == 4 && P.dim >= 2) {
    int& last = S[P.dim - 1];
    while ((last - P.w) % 32 != 0 || (last & 1)) last++;
  }
  g.bufsz = 1;
  for (int d = 0; d < P.dim; d++) g.bufsz *= S[d];
  for (int d = 0; d < 3; d++) g.S[d] = S[d];
  g.str[P.dim - 1] = 1;
  for (int d = P.dim - 2; d >= 0; d--) g.str[d] = g.str[d + 1] * S[d + 1];
  a.scale_d = P.hpw / P.sqd0;
  a.inv_dx_d = 1.0 / P.dx;
  a.hwdx_d = P.halfw / P.dx;
  a.halfw_over_dx = (T)(P.halfw / P.dx);
  a.inv_hw = (T)(P.dx / P.halfw);
  a.beta = (T)P.beta;
  a.dscale = (T)(a.inv_dx_d * a.scale_d / a.hwdx_d);
  a.inv_sqd0 = (T)(1.0 / P.sqd0);
  // planar rows: [l][re of nout padded | im of nout padded]
  const int NFp = pad4(NF), NHp = pad4(NH), Gp = pad4(G);
  const size_t ntwf = 2 * (size_t)G * NFp, ntwh = 2 * (size_t)G * NHp, ntif = 2 * (size_t)NF * Gp,
               ntih = 2 * (size_t)NH * Gp, total = ntwf + ntwh + ntif + ntih + 3 * (size_t)NF;
  T* h = static_cast<T*>(pinned_stage(slot, sizeof(T) * total));
  std::fill(h, h + total, T(0));
  T *twf = h, *twh = twf + ntwf, *tif = twh + ntwh, *tih = tif + ntif;
  T *facf = tih + ntih, *faci = facf + NF, *ts = faci + NF;
  for (int l = 0; l < G; l++) {
    double xl = (double)(P.l0 + l) * P.dx;
    for (int k = -K; k <= K; k++) {
      double c = cos(k * xl), sn = sin(k * xl);
      twf[(size_t)l * 2 * NFp + k + K] = (T)c;
      twf[(size_t)l * 2 * NFp + NFp + k + K] = (T)(-sn);
      tif[(size_t)(k + K) * 2 * Gp + l] = (T)c;
      tif[(size_t)(k + K) * 2 * Gp + Gp + l] = (T)sn;
      if (k >= 0) {
        twh[(size_t)l * 2 * NHp + k] = (T)c;
        twh[(size_t)l * 2 * NHp + NHp + k] = (T)(-sn);
        double f = k == 0 ? 1.0 : 2.0;
        tih[(size_t)k * 2 * Gp + l] = (T)(f * c);
        tih[(size_t)k * 2 * Gp + Gp + l] = (T)(f * sn);
      }
    }
  }
  for (int k = 0; k < NF; k++) {
    facf[k] = (T)(P.dx * P.wsym[k] / P.phihat[k]);
    faci[k] = (T)(P.dx / P.phihat[k]);
    ts[k] = (T)P.ts[k];
  }
  tb.all.alloc(total, s);
  FGT_CUDA(cudaMemcpyAsync(tb.all.get(), h, sizeof(T) * total, cudaMemcpyHostToDevice, s));
  pinned_stage_used(slot, s);
  T* d = tb.all.get();
  a.twf = d;
  a.twh = d + ntwf;
  a.tif = a.twh + ntwh;
  a.tih = a.tif + ntif;
  a.facf = a.tih + ntih;
  a.faci = a.facf + NF;
  a.ts = a.faci + NF;
  a.gscratch = nullptr;
}

template <typename T>
size_t fixed_smem(const PWArgs<T>& a, int, int) {
  return order_offset<T>(a.g.G, a.g.K);
}

template <typename KernelT>
void set_smem(KernelT k, size_t bytes) {
  FGT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

}  // namespace

// flops of the in-place passes of one grid (used for the work counters)
double pw_pass_flops(const PWParams& P);

}  // namespace fgt
