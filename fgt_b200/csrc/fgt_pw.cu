// Plane-wave form / translate / evaluate kernels (K6, K7, K8).
//
// Per box, one CTA keeps the whole spreading sub-grid in shared memory (a
// global-memory slice per CTA when it does not fit): spread (ES kernel,
// Barnett-Magland-af Klinteberg 2019) -> in-place pruned DFT passes along the
// last, middle and first dimension -> deconvolution and PW weights fused into
// the pass that writes the expansion.  Only the sub-grid the box's points can
// reach is stored: for boxes of the cut-off size the scaled coordinates lie
// in [-pi/3, pi/3], about a third of the 2*pi period.
//
// Spreading and interpolation are thread-per-point over a bank-balanced
// processing order of each box's points (see order_chunk), so the 32 lanes
// of a warp touch 32 distinct shared-memory banks at every stencil offset.
#include <math.h>

#include <algorithm>
#include <vector>

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
  const T* twf;   // [G][2K+1] fwd full
  const T* twh;   // [G][K+1]  fwd half
  const T* tif;   // [2K+1][G] inv full
  const T* tih;   // [K+1][G]  inv half (with 1/2/2/.. weights)
  const T* facf;  // [2K+1] dx*wsym/phihat
  const T* faci;  // [2K+1] dx/phihat
  const T* ts;    // [2K+1] ts(k)
  T inv_sqd0;
  T* gscratch;  // global buffer slices when the grid does not fit in smem
};

// byte offset of the grid buffer in shared memory: twiddles, then the
// ordering scratch (ORDER_CHUNK ints + 32 counters + ORDER_CHUNK u16)
template <typename T>
__host__ __device__ constexpr size_t order_offset(int G, int K) {
  return (((size_t)sizeof(T) * 2 * G * ((2 * K + 1) + (K + 1)) +
           sizeof(int) * (ORDER_CHUNK + 32) + sizeof(unsigned short) * ORDER_CHUNK) + 15) &
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
  // register tile: LG lines x KG outputs per thread; a round covers whole
  // lines (all of a line's inputs are read before any output is written)
  constexpr int LG = 2, KG = sizeof(T) == 4 ? 4 : 2;
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
          const int k = kg * KG + j;
          const bool ok = k < nout;
          tr[j] = ok ? tw[2 * (l * nout + k)] : T(0);
          ti[j] = ok ? tw[2 * (l * nout + k) + 1] : T(0);
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
        const int k = kg * KG + j;
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

// Stencil cell offsets (T units) along each dimension.  Lin: the sub-grid
// case, cells base..base+W-1 (offsets fold into address immediates); Tab:
// the periodic full grid, cells wrap modulo nf (one modulo per dimension).
// ki[i] for a run-time i without demoting ki to local memory
__device__ __forceinline__ int sel3(const int* ki, int i) {
  return i == 0 ? ki[0] : (i == 1 ? ki[1] : ki[2]);
}

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

template <typename T, int DIM, int W, class IX>
__device__ __forceinline__ T interp_cells(const T* B, const IX& ix, const T (*ph)[W]) {
  T acc = T(0);
  if constexpr (DIM == 1) {
#pragma unroll
    for (int j = 0; j < W; j++) acc += B[ix.x(j)] * ph[0][j];
  } else if constexpr (DIM == 2) {
    outer_cells<T, W, 16>(ix, ph[0], [&](int xo, T p0) {
      const T* bx = B + xo;
      T sy = T(0);
#pragma unroll
      for (int jy = 0; jy < W; jy++) sy += bx[ix.z(jy)] * ph[1][jy];
      acc += sy * p0;
    });
  } else {
    outer_cells<T, W, 8>(ix, ph[0], [&](int xo, T p0) {
      const T* bx = B + xo;
      T sx = T(0);
#pragma unroll
      for (int jy = 0; jy < W; jy++) {
        const T* bxy = bx + ix.y(jy);
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

template <typename T, int DIM, int W>
__device__ __forceinline__ T interp_point(const PWArgs<T>& a, const T* B, const double* x) {
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
template <typename T, int W>
__device__ __forceinline__ int kernel_row_d(const PWArgs<T>& a, double x, T* phi, T* dphi) {
  const double u = x * a.inv_dx_d;
  const int i0 = (int)ceil(u - a.hwdx_d);
  const T f0 = (T)((double)i0 - u);
#pragma unroll
  for (int j = 0; j < W; j++) {
    const T z = (f0 + (T)j) * a.inv_hw;
    const T q = T(1) - z * z;
    const T rq = q > T(0) ? Real<T>::rsqrt_(q) : T(0);
    const T e = Real<T>::expm(Real<T>::div12(a.beta * (z * z), T(1) + q * rq));
    phi[j] = e;
    dphi[j] = e * (a.beta * a.dscale) * z * rq;
  }
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

// Potential and gradient of one grid at one point: v[0] = pot, v[1+d] = d/dx_d.
// The sums run over B - Bref (Bref = the stencil's centre cell): the
// derivative stencils sum to the derivative of the kernel's partition of
// unity, which is at the aliasing level, so dropping Bref from them changes
// nothing, while the smaller summands keep the FP32 sums from cancelling
// when the field varies slowly over the stencil.  The potential adds Bref
// times the product of the kernel row sums back.
template <typename T, int DIM, int W, class IX>
__device__ __forceinline__ void interp_grad_cells(const T* B, const IX& ix, const T (*ph)[W],
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
      const T* bx = B + xo;
      T s0 = T(0), s1 = T(0);
#pragma unroll
      for (int jy = 0; jy < W; jy++) {
        const T b = bx[ix.z(jy)] - bref;
        s0 += b * ph[1][jy];
        s1 += b * dph[1][jy];
      }
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
      const T* bx = B + xo;
      T t0 = T(0), t1 = T(0), t2 = T(0);
#pragma unroll
      for (int jy = 0; jy < W; jy++) {
        const T* bxy = bx + ix.y(jy);
        T s0 = T(0), s1 = T(0);
#pragma unroll
        for (int jz = 0; jz < W; jz++) {
          const T b = bxy[ix.z(jz)] - bref;
          s0 += b * ph[2][jz];
          s1 += b * dph[2][jz];
        }
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

template <typename T, int DIM, int W>
__device__ __forceinline__ void interp_grad_point(const PWArgs<T>& a, const T* B, const double* x,
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

template <typename T>
__device__ __forceinline__ void load_tw(T* dst, const T* src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// ---------------------------------------------------------------- form
struct FormIO {
  int n_form, ns, nd, ncomp;  // ncomp: charge (1) and/or dipole (dim)
  int has_q, has_dip;
  const int *form_box, *s_lo, *s_hi;
};

template <typename T>
struct FormPtrs {
  const double* off;     // sorted SoA FP64 offsets
  const T *q, *ds, *rn;  // sorted SoA
  T* mp;                 // [n_form][nd][nexp] complex
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
constexpr int FCH = 8192;       // points sorted per round
constexpr int PB = 8;           // points per warp batch
constexpr int TP = 12;          // padded kernel row (TILE <= TP - 1)

template <typename T>
__host__ __device__ constexpr size_t tiled_offset(int G, int K) {
  return ((size_t)sizeof(T) * 2 * G * ((2 * K + 1) + (K + 1)) + sizeof(int) * (2 * NBLK_MAX + 32) +
          sizeof(int) * FCH + sizeof(unsigned short) * FCH +
          sizeof(float) * (PW_THREADS / 32) * PB * 3 * TP + 15) &
         ~(size_t)15;
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
  constexpr int TILE = TB + W - 1, NCOL = (TILE * TILE + 31) / 32;
  static_assert(TILE <= TP - 1, "tile row too long");
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
    T acc[NCOL][TILE];
#pragma unroll
    for (int j = 0; j < NCOL; j++)
#pragma unroll
      for (int t = 0; t < TILE; t++) acc[j][t] = T(0);
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
        const T* row = R + pq * 3 * TP;
        T rz[TP];
#pragma unroll
        for (int t = 0; t < TP; t++) rz[t] = row[2 * TP + t];
#pragma unroll
        for (int j = 0; j < NCOL; j++) {
          const T v = row[cx[j]] * row[TP + cy[j]];
#pragma unroll
          for (int t = 0; t < TILE; t++) acc[j][t] = fma(v, rz[t], acc[j][t]);
        }
      }
      __syncwarp();
    }
#pragma unroll
    for (int j = 0; j < NCOL; j++) {
      const int x = org[0] + cx[j], y = org[1] + cy[j];
      if (lane + 32 * j < TILE * TILE && x < g.G && y < g.G) {
        T* col = B + x * g.str[0] + y * g.str[1] + org[2];
#pragma unroll
        for (int t = 0; t < TILE; t++)
          if (org[2] + t < g.G && acc[j][t] != T(0)) atomicAdd(col + t, acc[j][t]);
      }
    }
  }
  __syncthreads();
}

template <typename T, int DIM, int W, bool GB, bool TILED>
__global__ void __launch_bounds__(PW_THREADS) k_form(PWArgs<T> a, FormIO io, FormPtrs<T> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Geo& g = a.g;
  const int K = g.K, NF = 2 * K + 1, NH = K + 1, G = g.G;
  T* sm = reinterpret_cast<T*>(smem_raw);
  T* twf = sm;                // G*NF complex
  T* twh = twf + 2 * G * NF;  // G*NH complex
  // atomic-spreading scratch
  int* ordtmp = reinterpret_cast<int*>(twh + 2 * G * NH);  // ORDER_CHUNK
  int* ordcnt = ordtmp + ORDER_CHUNK;                        // 32
  unsigned short* perm = reinterpret_cast<unsigned short*>(ordcnt + 32);  // ORDER_CHUNK
  // tiled-spreading scratch
  int* tcnt = reinterpret_cast<int*>(twh + 2 * G * NH);  // NBLK_MAX
  int* toff = tcnt + NBLK_MAX;                             // NBLK_MAX
  int* tmisc = toff + NBLK_MAX;                            // 32
  int* ttmp = tmisc + 32;                                  // FCH
  unsigned short* tperm = reinterpret_cast<unsigned short*>(ttmp + FCH);  // FCH
  T* trows = reinterpret_cast<T*>(tperm + FCH);  // warps * PB * 3 * TP
  T* B = GB ? a.gscratch + (size_t)blockIdx.x * g.bufsz
            : reinterpret_cast<T*>(smem_raw + (TILED ? tiled_offset<T>(G, K)
                                                     : order_offset<T>(G, K)));
  load_tw(twf, a.twf, 2 * G * NF);
  load_tw(twh, a.twh, 2 * G * NH);
  __syncthreads();
  for (int fb = blockIdx.x; fb < io.n_form; fb += gridDim.x) {
    const int box = io.form_box[fb];
    const int p0 = io.s_lo[box], p1 = io.s_hi[box];
    for (int id = 0; id < io.nd; id++) {
      T* mp = p.mp + ((size_t)fb * io.nd + id) * 2 * g.nexp;
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
          for (int c0 = p0; c0 < p1; c0 += FCH)
            spread_tiled<T, W>(a, B, p.off, io.ns, sq, sr, is_q, c0, min(FCH, p1 - c0), tcnt, toff,
                               tmisc, ttmp, tperm, trows);
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
        } else if (DIM == 2) {
          pass_inplace<T, 0>(B, G, 1, g.str[0], 0, 1, 2, G, NH, twh);
        }
        // final pass along x to the expansion, with weights and deconvolution
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
              re += gv * twh[2 * (l * NH + kxi)];
              im += gv * twh[2 * (l * NH + kxi) + 1];
            }
          } else {
            for (int l = 0; l < G; l++) {
              const T xr = B[l * g.str[0] + lb], xi = B[l * g.str[0] + lb + 1];
              const T tr = twf[2 * (l * NF + kxi)], ti = twf[2 * (l * NF + kxi) + 1];
              re += xr * tr - xi * ti;
              im += xr * ti + xi * tr;
            }
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

// ---------------------------------------------------------------- translate
template <typename T>
__global__ void k_translate(int n_eval, int nexp, int nd, const int* __restrict__ self,
                            const int* __restrict__ ptr, const int* __restrict__ src,
                            const int* __restrict__ widx, const T* __restrict__ mp,
                            const T* __restrict__ wtab, T* __restrict__ loc) {
  const int e = blockIdx.y;
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < nexp; m += gridDim.x * blockDim.x) {
    for (int id = 0; id < nd; id++) {
      T re = T(0), im = T(0);
      const int sf = self[e];
      if (sf >= 0) {
        re = mp[(((size_t)sf * nd + id) * nexp + m) * 2];
        im = mp[(((size_t)sf * nd + id) * nexp + m) * 2 + 1];
      }
      for (int j = ptr[e]; j < ptr[e + 1]; j++) {
        const size_t mi = (((size_t)src[j] * nd + id) * nexp + m) * 2;
        const size_t wi = ((size_t)widx[j] * nexp + m) * 2;
        const T ar = mp[mi], ai = mp[mi + 1], wr = wtab[wi], wi_ = wtab[wi + 1];
        re += ar * wr - ai * wi_;
        im += ar * wi_ + ai * wr;
      }
      loc[(((size_t)e * nd + id) * nexp + m) * 2] = re;
      loc[(((size_t)e * nd + id) * nexp + m) * 2 + 1] = im;
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

// ---------------------------------------------------------------- eval
template <typename T>
struct EvalPtrs {
  const T* loc;      // [n_eval][nd][nexp]
  const int* boxes;  // eval slots handled by this launch
  const int* eval_box;
  int nbox;
  // two evaluation sets (sources, targets)
  const double* off[2];
  const int* lo[2];
  const int* hi[2];
  double* out[2];
  int n[2], ncomp[2];
  int nd, ncomp_max;
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
        acc += mr * tih[2 * (k * G + l)] - mi * tih[2 * (k * G + l) + 1];
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
template <typename T, int DIM, int W, bool GB, bool DERIV>
__global__ void __launch_bounds__(PW_THREADS) k_eval_comp(PWArgs<T> a, EvalPtrs<T> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Geo& g = a.g;
  const int K = g.K, NF = 2 * K + 1, NH = K + 1, G = g.G;
  T* sm = reinterpret_cast<T*>(smem_raw);
  T* tif = sm;
  T* tih = tif + 2 * NF * G;
  int* ordtmp = reinterpret_cast<int*>(tih + 2 * NH * G);
  int* ordcnt = ordtmp + ORDER_CHUNK;
  unsigned short* perm = reinterpret_cast<unsigned short*>(ordcnt + 32);
  T* B = GB ? a.gscratch + (size_t)blockIdx.x * g.bufsz
            : reinterpret_cast<T*>(smem_raw + order_offset<T>(G, K));
  load_tw(tif, a.tif, 2 * NF * G);
  load_tw(tih, a.tih, 2 * NH * G);
  __syncthreads();
  for (int bi = blockIdx.x; bi < p.nbox; bi += gridDim.x) {
    const int e = p.boxes[bi];
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
          const int q0 = set ? p.lo[1][box] : p.lo[0][box];
          const int q1 = set ? p.hi[1][box] : p.hi[0][box];
          for (int c0 = q0; c0 < q1; c0 += ORDER_CHUNK) {
            const int n = min(ORDER_CHUNK, q1 - c0);
            order_chunk<T, DIM, W>(a, offs, ne, c0, n, perm, ordtmp, ordcnt);
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
              const int pt = c0 + perm[i];
              double x[DIM];
#pragma unroll
              for (int k = 0; k < DIM; k++) x[k] = offs[(size_t)k * ne + pt] * a.scale_d;
              if constexpr (DERIV) {
                T v[1 + DIM];
                interp_grad_point<T, DIM, W>(a, B, x, v);
                const int nc = set ? p.ncomp[1] : p.ncomp[0];
                outs[(size_t)id * ne + pt] += (double)v[0];
                if (nc > 1) {
#pragma unroll
                  for (int d = 0; d < DIM; d++)
                    outs[((size_t)(1 + d) * p.nd + id) * ne + pt] += (double)v[1 + d];
                }
              } else {
                const T v = interp_point<T, DIM, W>(a, B, x);
                outs[((size_t)c * p.nd + id) * ne + pt] += (double)v;
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

// Direct modal evaluation for boxes with few points: one CTA per box, modes
// split over threads, one block reduction per point.
template <typename T, int DIM>
__global__ void __launch_bounds__(MODAL_THREADS) k_eval_modal(PWArgs<T> a, EvalPtrs<T> p) {
  const Geo& g = a.g;
  const int K = g.K, NF = 2 * K + 1, NH = K + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* E = reinterpret_cast<T*>(smem_raw);  // [DIM][NF] complex e^{i k x_d}
  __shared__ double red[MODAL_THREADS / 32][10];
  for (int bi = blockIdx.x; bi < p.nbox; bi += gridDim.x) {
    const int e = p.boxes[bi];
    const int box = p.eval_box[e];
    for (int set = 0; set < 2; set++) {
      const int ne = set ? p.n[1] : p.n[0], nc = set ? p.ncomp[1] : p.ncomp[0];
      if (ne == 0 || nc == 0) continue;
      const double* offs = set ? p.off[1] : p.off[0];
      double* outs = set ? p.out[1] : p.out[0];
      const int q0 = set ? p.lo[1][box] : p.lo[0][box];
      const int q1 = set ? p.hi[1][box] : p.hi[0][box];
      for (int pt = q0; pt < q1; pt++) {
        __syncthreads();
        for (int i = threadIdx.x; i < DIM * NF; i += blockDim.x) {
          const int d = i / NF, k = i - d * NF - K;
          const double x = offs[(size_t)d * ne + pt] * a.scale_d;
          double sn, cs;
          sincos(x * (double)k, &sn, &cs);
          E[2 * i] = (T)cs;
          E[2 * i + 1] = (T)sn;
        }
        __syncthreads();
        for (int id = 0; id < p.nd; id++) {
          const T* L = p.loc + ((size_t)e * p.nd + id) * 2 * g.nexp;
          T acc[10];
#pragma unroll
          for (int c = 0; c < 10; c++) acc[c] = T(0);
          for (int m = threadIdx.x; m < g.nexp; m += blockDim.x) {
            int ki[3];
            if (DIM == 3) { ki[0] = m / (NF * NH); ki[1] = (m / NH) % NF; ki[2] = m % NH + K; }
            else if (DIM == 2) { ki[0] = m / NH; ki[1] = m % NH + K; }
            else { ki[0] = m + K; }
            const T f = (ki[DIM - 1] == K) ? T(1) : T(2);  // Hermitian half-space weight
            T er = T(1), ei = T(0);
#pragma unroll
            for (int d = 0; d < DIM; d++) {
              const T cr = E[2 * (d * NF + ki[d])], ci = E[2 * (d * NF + ki[d]) + 1];
              const T nr = er * cr - ei * ci;
              ei = er * ci + ei * cr;
              er = nr;
            }
            const T lr = L[2 * m] * f, li = L[2 * m + 1] * f;
            const T tr = lr * er - li * ei, ti = lr * ei + li * er;  // term = L e^{ikx}
            acc[0] += tr;
            if (nc > 1)
#pragma unroll
              for (int d = 0; d < DIM; d++) acc[1 + d] += -ti * a.ts[ki[d]] * a.inv_sqd0;
            if (nc > 1 + DIM) {
              const int nh = DIM * (DIM + 1) / 2;
#pragma unroll
              for (int hm = 0; hm < nh; hm++) {
                int pp, qq;
                if (DIM == 1) { pp = 0; qq = 0; }
                else if (DIM == 2) { pp = (hm == 2) ? 1 : 0; qq = (hm == 0) ? 0 : 1; }
                else { pp = hm < 3 ? hm : (hm < 5 ? 0 : 1); qq = hm < 3 ? hm : (hm == 3 ? 1 : 2); }
                acc[1 + DIM + hm] += -tr * a.ts[sel3(ki, pp)] * a.ts[sel3(ki, qq)] * a.inv_sqd0 * a.inv_sqd0;
              }
            }
          }
          const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
          for (int c = 0; c < nc; c++) {
            double v = (double)acc[c];
            for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) red[w][c] = v;
          }
          __syncthreads();
          if (threadIdx.x < nc) {
            double v = 0;
            for (int j = 0; j < (int)(blockDim.x >> 5); j++) v += red[j][threadIdx.x];
            outs[((size_t)threadIdx.x * p.nd + id) * ne + pt] += v;
          }
          __syncthreads();
        }
      }
    }
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
__global__ void k_count_points(int n, const int* __restrict__ box, const int* __restrict__ lo,
                               const int* __restrict__ hi, unsigned long long* __restrict__ cnt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    atomicAdd(cnt, (unsigned long long)(hi[box[i]] - lo[box[i]]));
}
__global__ void k_split_fill(int n, const int* __restrict__ f, const int* __restrict__ pos,
                             int* __restrict__ big_list, int* __restrict__ small_list) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    if (f[e]) big_list[pos[e]] = e;
    else small_list[e - pos[e]] = e;
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
  DBuf<T> twf, twh, tif, tih, facf, faci, ts;
};

// Device arguments for grid parameters P; the innermost buffer stride is
// padded to W (mod 32) words for FP32 so the warp-per-point stencils are
// bank-conflict free.
template <typename T>
void make_args(const PWParams& P, PWArgs<T>& a, DevTables<T>& tb, cudaStream_t s, bool pad) {
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
  std::vector<T> twf(2 * G * NF), twh(2 * G * NH), tif(2 * NF * G), tih(2 * NH * G);
  for (int l = 0; l < G; l++) {
    double xl = (double)(P.l0 + l) * P.dx;
    for (int k = -K; k <= K; k++) {
      double c = cos(k * xl), sn = sin(k * xl);
      twf[2 * (l * NF + k + K)] = (T)c;
      twf[2 * (l * NF + k + K) + 1] = (T)(-sn);
      tif[2 * ((k + K) * G + l)] = (T)c;
      tif[2 * ((k + K) * G + l) + 1] = (T)sn;
      if (k >= 0) {
        twh[2 * (l * NH + k)] = (T)c;
        twh[2 * (l * NH + k) + 1] = (T)(-sn);
        double f = k == 0 ? 1.0 : 2.0;
        tih[2 * (k * G + l)] = (T)(f * c);
        tih[2 * (k * G + l) + 1] = (T)(f * sn);
      }
    }
  }
  std::vector<T> facf(NF), faci(NF), ts(NF);
  for (int k = 0; k < NF; k++) {
    facf[k] = (T)(P.dx * P.wsym[k] / P.phihat[k]);
    faci[k] = (T)(P.dx / P.phihat[k]);
    ts[k] = (T)P.ts[k];
  }
  auto up = [&](DBuf<T>& b, const std::vector<T>& h) {
    b.alloc(h.size(), s);
    FGT_CUDA(cudaMemcpyAsync(b.get(), h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, s));
  };
  up(tb.twf, twf);
  up(tb.twh, twh);
  up(tb.tif, tif);
  up(tb.tih, tih);
  up(tb.facf, facf);
  up(tb.faci, faci);
  up(tb.ts, ts);
  FGT_CUDA(cudaStreamSynchronize(s));  // host vectors go out of scope
  a.twf = tb.twf;
  a.twh = tb.twh;
  a.tif = tb.tif;
  a.tih = tb.tih;
  a.facf = tb.facf;
  a.faci = tb.faci;
  a.ts = tb.ts;
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

template <typename T, int DIM, int W>
int launch_form(PWArgs<T>& a, const FormIO& io, const FormPtrs<T>& fp, DBuf<T>& gs, cudaStream_t s) {
  size_t fix = fixed_smem(a, W, 1);
  size_t need = fix + sizeof(T) * (size_t)a.g.bufsz;
  int grid = std::max(1, std::min(io.n_form, kSMs));
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
  if (need <= (size_t)MAXSMEM) {
    auto k = k_form<T, DIM, W, false, false>;
    set_smem(k, need);
    k<<<grid, PW_THREADS, need, s>>>(a, io, fp);
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

template <typename T, int DIM, int W, bool DERIV>
int launch_eval_k(PWArgs<T>& a, const EvalPtrs<T>& ep, DBuf<T>& gs, cudaStream_t s) {
  size_t fix = fixed_smem(a, W, 2);
  size_t need = fix + sizeof(T) * (size_t)a.g.bufsz;
  int grid = std::max(1, std::min(ep.nbox, kSMs));
  bool gb = need > (size_t)MAXSMEM;
  if (gb) {
    gs.alloc((size_t)grid * a.g.bufsz, s);
    a.gscratch = gs;
  }
  size_t sm = gb ? fix : need;
  if (gb) {
    auto k = k_eval_comp<T, DIM, W, true, DERIV>;
    set_smem(k, sm);
    k<<<grid, PW_THREADS, sm, s>>>(a, ep);
  } else {
    auto k = k_eval_comp<T, DIM, W, false, DERIV>;
    set_smem(k, sm);
    k<<<grid, PW_THREADS, sm, s>>>(a, ep);
  }
  FGT_LAUNCH_CHECK();
  return 1;
}

// deriv: gradients through the kernel derivative (widths 8..16 only)
template <typename T, int DIM, int W>
int launch_eval(PWArgs<T>& a, const EvalPtrs<T>& ep, bool deriv, DBuf<T>& gs, cudaStream_t s) {
  if constexpr (W >= 8) {
    if (deriv) return launch_eval_k<T, DIM, W, true>(a, ep, gs, s);
  }
  FGT_REQUIRE(!deriv, FGT_ERR_UNSUPPORTED, "derivative evaluation needs a kernel width >= 8");
  return launch_eval_k<T, DIM, W, false>(a, ep, gs, s);
}

template <typename T, int DIM>
int form_w(int w, PWArgs<T>& a, const FormIO& io, const FormPtrs<T>& fp, DBuf<T>& gs, cudaStream_t s) {
  switch (w) {
    case 6: return launch_form<T, DIM, 6>(a, io, fp, gs, s);
    case 8: return launch_form<T, DIM, 8>(a, io, fp, gs, s);
    case 10: return launch_form<T, DIM, 10>(a, io, fp, gs, s);
    case 12: return launch_form<T, DIM, 12>(a, io, fp, gs, s);
    case 14: return launch_form<T, DIM, 14>(a, io, fp, gs, s);
    default: return launch_form<T, DIM, 16>(a, io, fp, gs, s);
  }
}
template <typename T, int DIM>
int eval_w(int w, PWArgs<T>& a, const EvalPtrs<T>& ep, bool deriv, DBuf<T>& gs, cudaStream_t s) {
  switch (w) {
    case 6: return launch_eval<T, DIM, 6>(a, ep, deriv, gs, s);
    case 8: return launch_eval<T, DIM, 8>(a, ep, deriv, gs, s);
    case 10: return launch_eval<T, DIM, 10>(a, ep, deriv, gs, s);
    case 12: return launch_eval<T, DIM, 12>(a, ep, deriv, gs, s);
    case 14: return launch_eval<T, DIM, 14>(a, ep, deriv, gs, s);
    default: return launch_eval<T, DIM, 16>(a, ep, deriv, gs, s);
  }
}
template <typename T>
int eval_dim(int dim, int w, PWArgs<T>& a, const EvalPtrs<T>& ep, bool deriv, DBuf<T>& gs,
             cudaStream_t s) {
  if (dim == 1) return eval_w<T, 1>(w, a, ep, deriv, gs, s);
  if (dim == 2) return eval_w<T, 2>(w, a, ep, deriv, gs, s);
  return eval_w<T, 3>(w, a, ep, deriv, gs, s);
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
void pw_grid(PWParams& P, int w) {
  const double pi = 4.0 * atan(1.0);
  const int K = P.K, NF = 2 * K + 1;
  w = supported_w(std::max(4, std::min(16, w)));
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
  std::vector<double> xq, wq;
  legendre(200, xq, wq);
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
  make_args<T>(P, a, tb, s, false);
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
  FormPtrs<T> fp;
  fp.off = src.off;
  fp.q = src.q;
  fp.ds = src.ds;
  fp.rn = src.rn;
  fp.mp = D.mp;
  DBuf<T> gs;
  int n;
  if (P.dim == 1) n = form_w<T, 1>(P.w, a, io, fp, gs, s);
  else if (P.dim == 2) n = form_w<T, 2>(P.w, a, io, fp, gs, s);
  else n = form_w<T, 3>(P.w, a, io, fp, gs, s);
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
  FGT_CUDA(cudaMemcpyAsync(ts64.get(), P.ts.data(), sizeof(double) * P.ts.size(),
                           cudaMemcpyHostToDevice, s));
  k_wtab<T><<<grid_for((long long)nsh * P.nexp, 256), 256, 0, s>>>(P.dim, P.K, P.nexp, ts64,
                                                                   P.xmin, D.wtab);
  FGT_LAUNCH_CHECK();
  D.loc.alloc((size_t)std::max(L.n_eval, 1) * P.nd * 2 * P.nexp, s);
  if (work)
    work->bytes_translate = (double)sizeof(T) * 2 * P.nexp * P.nd *
                            ((double)L.n_trans + 2.0 * L.n_eval);
  if (L.n_eval == 0) return 1;
  int gx = std::max(1, std::min(ceil_div(P.nexp, 256), 64));
  for (int e0 = 0; e0 < L.n_eval; e0 += 65535) {
    int ne = std::min(65535, L.n_eval - e0);
    dim3 grid(gx, ne);
    k_translate<T><<<grid, 256, 0, s>>>(ne, P.nexp, P.nd, L.eval_self.get() + e0,
                                        L.trans_ptr.get() + e0, L.trans_src, L.trans_w, D.mp,
                                        D.wtab, D.loc.get() + (size_t)e0 * P.nd * 2 * P.nexp);
    FGT_LAUNCH_CHECK();
  }
  FGT_CUDA(cudaStreamSynchronize(s));  // ts64 lifetime
  return 2;
}

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
  const bool deriv = pgh_max == 2 && P.w + 2 <= 16;
  const int mode = deriv ? 1 : 2;
  PWParams Pe = P;
  if (deriv) pw_grid(Pe, P.w + 2);
  PWArgs<T> a;
  DevTables<T> tb;
  make_args<T>(Pe, a, tb, s, false);
  int launches = 0;
  const int thr = small_eval >= 0 ? small_eval : (P.dim == 3 ? 48 : (P.dim == 2 ? 8 : 4));
  DBuf<int> big(L.n_eval, s), pos(L.n_eval, s), tot(1, s);
  DBuf<unsigned long long> cnt(2, s);
  cnt.zero();
  k_eval_split<<<grid_for(L.n_eval, 256), 256, 0, s>>>(
      L.n_eval, L.eval_box, u0 ? e0.lo : nullptr, u0 ? e0.hi : nullptr, u1 ? e1.lo : nullptr,
      u1 ? e1.hi : nullptr, thr, big, cnt);
  FGT_LAUNCH_CHECK();
  exclusive_scan_i32(big, pos, L.n_eval, tot, s);
  int nbig = fetch_int(tot, s);
  DBuf<int> lbig(std::max(nbig, 1), s), lsmall(std::max(L.n_eval - nbig, 1), s);
  k_split_fill<<<grid_for(L.n_eval, 256), 256, 0, s>>>(L.n_eval, big, pos, lbig, lsmall);
  FGT_LAUNCH_CHECK();
  launches += 3;
  int nh = P.dim * (P.dim + 1) / 2;
  auto ncomp = [&](int pgh) { return pgh <= 0 ? 0 : 1 + (pgh >= 2 ? P.dim : 0) + (pgh >= 3 ? nh : 0); };
  EvalPtrs<T> ep;
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
  DBuf<T> gs;
  if (nbig > 0) {
    ep.boxes = lbig;
    ep.nbox = nbig;
    launches += eval_dim<T>(P.dim, Pe.w, a, ep, deriv, gs, s);
    if (work) work->n_nufft += nbig;
  }
  int nsmall = L.n_eval - nbig;
  if (nsmall > 0) {
    ep.boxes = lsmall;
    ep.nbox = nsmall;
    int grid = std::max(1, std::min(nsmall, kSMs * 8));
    size_t sm = sizeof(T) * 2 * P.dim * (2 * P.K + 1);
    if (P.dim == 1) k_eval_modal<T, 1><<<grid, MODAL_THREADS, sm, s>>>(a, ep);
    else if (P.dim == 2) k_eval_modal<T, 2><<<grid, MODAL_THREADS, sm, s>>>(a, ep);
    else k_eval_modal<T, 3><<<grid, MODAL_THREADS, sm, s>>>(a, ep);
    FGT_LAUNCH_CHECK();
    launches++;
  }
  if (work) {
    unsigned long long h[2] = {0, 0};
    FGT_CUDA(cudaMemcpyAsync(h, cnt.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    FGT_CUDA(cudaStreamSynchronize(s));
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
  FGT_CUDA(cudaStreamSynchronize(s));  // tables lifetime
  return launches;
}

template int pw_form<float>(const PWParams&, const Tree&, const Lists&, const SourceSet<float>&,
                            PWData<float>&, PWWork*, cudaStream_t);
template int pw_form<double>(const PWParams&, const Tree&, const Lists&, const SourceSet<double>&,
                             PWData<double>&, PWWork*, cudaStream_t);
template int pw_translate<float>(const PWParams&, const Lists&, PWData<float>&, PWWork*,
                                 cudaStream_t);
template int pw_translate<double>(const PWParams&, const Lists&, PWData<double>&, PWWork*,
                                  cudaStream_t);
template int pw_eval<float>(const PWParams&, const Tree&, const Lists&, const PWData<float>&,
                            const EvalSet<float>&, const EvalSet<float>&, int, PWWork*,
                            cudaStream_t);
template int pw_eval<double>(const PWParams&, const Tree&, const Lists&, const PWData<double>&,
                             const EvalSet<double>&, const EvalSet<double>&, int, PWWork*,
                             cudaStream_t);

}  // namespace fgt
