// Direct near-field Gaussian sums (K9): warp-tiled, one evaluation point per
// lane held in registers, list-1 sources staged through shared memory and
// read as broadcasts.  Mixed precision: FP32 offsets from FP64 box centres,
// FP32 exp (ex2.approx) and FP32 per-item accumulation, FP64 output
// accumulation.  FP64 path: same kernel in double.
#include <stdlib.h>

#include <algorithm>

#include "fgt_direct.cuh"

namespace fgt {

namespace {

constexpr int DW = 4;  // warps per block

template <typename T>
struct DArgs {
  int n_items, nd, d0, ne, ns, iperiod0;  // n_items: upper bound
  int nboxes;
  const int* n_items_dev;                  // item count on the device
  T dinv, dmax, rfac;  // 1/delta, cut-off, 2/delta
  double bs0;
  const int *item_box, *item_lo;
  const int *l1_ptr, *l1_src;
  const int *s_lo, *s_hi, *e_hi;
  const double *soff, *eoff;
  const T *q, *ds, *rn;
  const double* center;
  const int* level;
  double dmax_d;  // cut-off in FP64 for the box-pair test
  double* out;
};

// A list-1 source box lies entirely beyond the cut-off when the minimum
// distance between the two boxes (centre offset dc, half sizes summed in hh)
// exceeds sqrt(dmax): every one of its pairs fails the rr < dmax test, so the
// box is skipped.  The relative margin covers the rounding of the FP32 pair
// distances.
template <int DIM>
__device__ __forceinline__ bool box_beyond_cutoff(const double* dc, double hh, double dmax) {
  double gap2 = 0.0;
#pragma unroll
  for (int k = 0; k < DIM; k++) {
    const double gk = fabs(dc[k]) - hh;
    gap2 += gk > 0.0 ? gk * gk : 0.0;
  }
  return gap2 > dmax * (1.0 + 1e-6);
}

template <int DIM>
struct HessIdx;
template <>
struct HessIdx<1> {
  static __device__ __forceinline__ int a(int m) { return 0; }
  static __device__ __forceinline__ int b(int m) { return 0; }
};
template <>
struct HessIdx<2> {  // xx, xy, yy (src/pfgt/pfgt_direct.f:185-189)
  static __device__ __forceinline__ int a(int m) { return m == 2 ? 1 : 0; }
  static __device__ __forceinline__ int b(int m) { return m == 0 ? 0 : 1; }
};
template <>
struct HessIdx<3> {  // xx, yy, zz, xy, xz, yz
  static __device__ __forceinline__ int a(int m) { return m < 3 ? m : (m < 5 ? 0 : 1); }
  static __device__ __forceinline__ int b(int m) { return m < 3 ? m : (m == 3 ? 1 : 2); }
};

template <typename T, int DIM, int PGH, bool CHG, bool DIP, int NDC>
__global__ void __launch_bounds__(DW * 32) k_direct(DArgs<T> a) {
  constexpr int NH = DIM * (DIM + 1) / 2;
  constexpr int NC = 1 + (PGH >= 2 ? DIM : 0) + (PGH >= 3 ? NH : 0);
  constexpr bool SPLIT = sizeof(T) == 4;  // FP32: pair differences from hi/lo parts
  __shared__ T sx[DW][DIM][32];
  __shared__ T sxl[DW][SPLIT ? DIM : 1][32];
  __shared__ T sq[DW][CHG ? NDC : 1][32];
  __shared__ T sd[DW][DIP ? NDC : 1][32];
  __shared__ T sn[DW][DIP ? DIM : 1][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ndc = min(NDC, a.nd - a.d0);
  const int n_items = *a.n_items_dev;
  for (int it = blockIdx.x * DW + warp; it < n_items; it += gridDim.x * DW) {
    const int tb = a.item_box[it];
    const int p = a.item_lo[it] + lane;
    const bool act = p < a.e_hi[tb];
    T tx[DIM], txl[DIM];
#pragma unroll
    for (int k = 0; k < DIM; k++) {
      const double v = act ? a.eoff[(size_t)k * a.ne + p] : 0.0;
      tx[k] = (T)v;
      txl[k] = SPLIT ? (T)(v - (double)tx[k]) : T(0);
    }
    // T sums over one staged batch of 32 sources, FP64 sums over batches
    T acc[NDC][NC];
    double accd[NDC][NC];
#pragma unroll
    for (int i = 0; i < NDC; i++)
#pragma unroll
      for (int c = 0; c < NC; c++) {
        acc[i][c] = T(0);
        accd[i][c] = 0.0;
      }
    double cT[DIM];
#pragma unroll
    for (int k = 0; k < DIM; k++) cT[k] = a.center[(size_t)tb * DIM + k];
    const int lT = a.level[tb];
    for (int li = a.l1_ptr[tb]; li < a.l1_ptr[tb + 1]; li++) {
      const int sb = a.l1_src[li];
      if (!FGT_DCHECK(sb >= 0 && sb < a.nboxes, 401)) continue;
      double dc[DIM];
#pragma unroll
      for (int k = 0; k < DIM; k++) {
        double cs = a.center[(size_t)sb * DIM + k];
        double sh = 0;
        if (a.iperiod0 == 1) {  // pfgt_find_local_shift, src/pfgt/pfgt_direct.f:620-651
          double dx = cT[k] - cs, dxp1 = dx - a.bs0, dxm1 = dx + a.bs0;
          if (fabs(dx) > fabs(dxp1)) { dx = dxp1; sh = a.bs0; }
          if (fabs(dx) > fabs(dxm1)) sh = -a.bs0;
        }
        dc[k] = (cs + sh) - cT[k];
      }
      if (box_beyond_cutoff<DIM>(dc, 0.5 * a.bs0 * (ldexp(1.0, -lT) + ldexp(1.0, -a.level[sb])),
                                 a.dmax_d))
        continue;
      const int s0 = a.s_lo[sb], s1 = a.s_hi[sb];
      for (int base = s0; base < s1; base += 32) {
        const int j = base + lane;
        __syncwarp();
        if (j < s1) {
#pragma unroll
          for (int k = 0; k < DIM; k++) {
            const double v = a.soff[(size_t)k * a.ns + j] + dc[k];
            const T hi = (T)v;
            sx[warp][k][lane] = hi;
            if (SPLIT) sxl[warp][k][lane] = (T)(v - (double)hi);
          }
          if (CHG)
#pragma unroll
            for (int i = 0; i < NDC; i++)
              if (i < ndc) sq[warp][i][lane] = a.q[(size_t)(a.d0 + i) * a.ns + j];
          if (DIP) {
#pragma unroll
            for (int i = 0; i < NDC; i++)
              if (i < ndc) sd[warp][i][lane] = a.ds[(size_t)(a.d0 + i) * a.ns + j];
#pragma unroll
            for (int k = 0; k < DIM; k++) sn[warp][k][lane] = a.rn[(size_t)k * a.ns + j];
          }
        }
        __syncwarp();
        const int cnt = min(32, s1 - base);
#pragma unroll 1
        for (int jj = 0; jj < cnt; jj++) {
          T dr[DIM], rr = T(0);
#pragma unroll
          for (int k = 0; k < DIM; k++) {
            dr[k] = SPLIT ? (tx[k] - sx[warp][k][jj]) + (txl[k] - sxl[warp][k][jj])
                          : tx[k] - sx[warp][k][jj];
            rr += dr[k] * dr[k];
          }
          if (!(rr < a.dmax)) continue;
          const T e = Real<T>::expm(rr * a.dinv);
          if (CHG) {
            // gnd_directc{p,g,h}, src/pfgt/pfgt_direct.f:47-196
            T dg[DIM];
#pragma unroll
            for (int k = 0; k < DIM; k++) dg[k] = -a.rfac * dr[k];
#pragma unroll
            for (int i = 0; i < NDC; i++) {
              if (i >= ndc) break;
              const T r = e * sq[warp][i][jj];
              acc[i][0] += r;
              if (PGH >= 2)
#pragma unroll
                for (int k = 0; k < DIM; k++) acc[i][1 + k] += dg[k] * r;
              if (PGH >= 3)
#pragma unroll
                for (int m = 0; m < NH; m++) {
                  const int ka = HessIdx<DIM>::a(m), kb = HessIdx<DIM>::b(m);
                  const T h = dg[ka] * dg[kb] + (ka == kb ? -a.rfac : T(0));
                  acc[i][1 + DIM + m] += h * r;
                }
            }
          }
          if (DIP) {
            // gnd_directd{p,g,h}, src/pfgt/pfgt_direct.f:204-384
            T d[DIM], rn[DIM], rinc = T(0);
#pragma unroll
            for (int k = 0; k < DIM; k++) {
              d[k] = a.rfac * dr[k];
              rn[k] = sn[warp][k][jj];
              rinc += d[k] * rn[k];
            }
            T rg[DIM];
#pragma unroll
            for (int k = 0; k < DIM; k++) rg[k] = rn[k] * a.rfac - rinc * d[k];
#pragma unroll
            for (int i = 0; i < NDC; i++) {
              if (i >= ndc) break;
              const T r = e * sd[warp][i][jj];
              acc[i][0] += rinc * r;
              if (PGH >= 2)
#pragma unroll
                for (int k = 0; k < DIM; k++) acc[i][1 + k] += rg[k] * r;
              if (PGH >= 3)
#pragma unroll
                for (int m = 0; m < NH; m++) {
                  const int ka = HessIdx<DIM>::a(m), kb = HessIdx<DIM>::b(m);
                  T h = (ka == kb) ? (-a.rfac * (d[ka] * rn[ka] + rinc) - rg[ka] * d[ka])
                                   : (-a.rfac * d[ka] * rn[kb] - rg[ka] * d[kb]);
                  acc[i][1 + DIM + m] += h * r;
                }
            }
          }
        }
#pragma unroll
        for (int i = 0; i < NDC; i++)
#pragma unroll
          for (int c = 0; c < NC; c++) {
            accd[i][c] += (double)acc[i][c];
            acc[i][c] = T(0);
          }
      }
    }
    if (act) {
#pragma unroll
      for (int i = 0; i < NDC; i++) {
        if (i >= ndc) break;
#pragma unroll
        for (int c = 0; c < NC; c++) {
          double* o = &a.out[((size_t)c * a.nd + a.d0 + i) * a.ne + p];
          *o += accd[i][c] + (double)acc[i][c];
        }
      }
    }
  }
}

// FP32 variant (mixed precision): each staged source is two float4s,
// (x_hi, y_hi, z_hi, q) and (x_lo, y_lo, z_lo, dipole strength), read as
// 128-bit broadcasts, and the cut-off is a select (e = 0 beyond dmax) instead
// of a divergent branch: the lanes of a warp hold different targets, so a
// branch would run the pair arithmetic anyway with most lanes idle.
template <int DIM, int PGH, bool CHG, bool DIP, int NDC>
__global__ void __launch_bounds__(DW * 32) k_direct32(DArgs<float> a) {
  constexpr int NH = DIM * (DIM + 1) / 2;
  constexpr int NC = 1 + (PGH >= 2 ? DIM : 0) + (PGH >= 3 ? NH : 0);
  constexpr bool PACKQ = NDC == 1;  // charge / dipole strength in the w slots
  __shared__ float4 shi[DW][32], slo[DW][32];
  __shared__ float4 snr[DW][DIP ? 32 : 1];
  __shared__ float sq[DW][CHG && !PACKQ ? NDC : 1][32];
  __shared__ float sd[DW][DIP && !PACKQ ? NDC : 1][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ndc = min(NDC, a.nd - a.d0);
  const float ce = a.dinv * 1.4426950408889634f;  // exp(-rr/delta) = 2^(-rr*ce)
  const int n_items = *a.n_items_dev;
  for (int it = blockIdx.x * DW + warp; it < n_items; it += gridDim.x * DW) {
    const int tb = a.item_box[it];
    const int p = a.item_lo[it] + lane;
    const bool act = p < a.e_hi[tb];
    float tx[3] = {0, 0, 0}, txl[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < DIM; k++) {
      const double v = act ? a.eoff[(size_t)k * a.ne + p] : 0.0;
      tx[k] = (float)v;
      txl[k] = (float)(v - (double)tx[k]);
    }
    float acc[NDC][NC];
    double accd[NDC][NC];
#pragma unroll
    for (int i = 0; i < NDC; i++)
#pragma unroll
      for (int c = 0; c < NC; c++) {
        acc[i][c] = 0.f;
        accd[i][c] = 0.0;
      }
    double cT[DIM];
#pragma unroll
    for (int k = 0; k < DIM; k++) cT[k] = a.center[(size_t)tb * DIM + k];
    const int lT = a.level[tb];
    for (int li = a.l1_ptr[tb]; li < a.l1_ptr[tb + 1]; li++) {
      const int sb = a.l1_src[li];
      if (!FGT_DCHECK(sb >= 0 && sb < a.nboxes, 401)) continue;
      double dc[DIM];
#pragma unroll
      for (int k = 0; k < DIM; k++) {
        double cs = a.center[(size_t)sb * DIM + k];
        double sh = 0;
        if (a.iperiod0 == 1) {  // pfgt_find_local_shift, src/pfgt/pfgt_direct.f:620-651
          double dx = cT[k] - cs, dxp1 = dx - a.bs0, dxm1 = dx + a.bs0;
          if (fabs(dx) > fabs(dxp1)) { dx = dxp1; sh = a.bs0; }
          if (fabs(dx) > fabs(dxm1)) sh = -a.bs0;
        }
        dc[k] = (cs + sh) - cT[k];
      }
      if (box_beyond_cutoff<DIM>(dc, 0.5 * a.bs0 * (ldexp(1.0, -lT) + ldexp(1.0, -a.level[sb])),
                                 a.dmax_d))
        continue;
      const int s0 = a.s_lo[sb], s1 = a.s_hi[sb];
      for (int base = s0; base < s1; base += 32) {
        const int j = base + lane;
        __syncwarp();
        if (j < s1) {
          float h[3] = {0, 0, 0}, l[3] = {0, 0, 0};
#pragma unroll
          for (int k = 0; k < DIM; k++) {
            const double v = a.soff[(size_t)k * a.ns + j] + dc[k];
            h[k] = (float)v;
            l[k] = (float)(v - (double)h[k]);
          }
          const float qv = CHG && PACKQ ? a.q[(size_t)a.d0 * a.ns + j] : 0.f;
          const float dv = DIP && PACKQ ? a.ds[(size_t)a.d0 * a.ns + j] : 0.f;
          shi[warp][lane] = make_float4(h[0], h[1], h[2], qv);
          slo[warp][lane] = make_float4(l[0], l[1], l[2], dv);
          if (DIP) {
            float r[3] = {0, 0, 0};
#pragma unroll
            for (int k = 0; k < DIM; k++) r[k] = a.rn[(size_t)k * a.ns + j];
            snr[warp][DIP ? lane : 0] = make_float4(r[0], r[1], r[2], 0.f);
          }
          if (CHG && !PACKQ)
#pragma unroll
            for (int i = 0; i < NDC; i++)
              if (i < ndc) sq[warp][i][lane] = a.q[(size_t)(a.d0 + i) * a.ns + j];
          if (DIP && !PACKQ)
#pragma unroll
            for (int i = 0; i < NDC; i++)
              if (i < ndc) sd[warp][i][lane] = a.ds[(size_t)(a.d0 + i) * a.ns + j];
        }
        __syncwarp();
        const int cnt = min(32, s1 - base);
#pragma unroll 2
        for (int jj = 0; jj < cnt; jj++) {
          const float4 hs = shi[warp][jj], ls = slo[warp][jj];
          const float hv[3] = {hs.x, hs.y, hs.z}, lv[3] = {ls.x, ls.y, ls.z};
          float dr[DIM], rr = 0.f;
#pragma unroll
          for (int k = 0; k < DIM; k++) {
            dr[k] = (tx[k] - hv[k]) + (txl[k] - lv[k]);
            rr = fmaf(dr[k], dr[k], rr);
          }
          const float e = rr < a.dmax ? fgt_ex2(-rr * ce) : 0.f;
          if (CHG) {
            // gnd_directc{p,g,h}, src/pfgt/pfgt_direct.f:47-196
            float dg[DIM];
#pragma unroll
            for (int k = 0; k < DIM; k++) dg[k] = -a.rfac * dr[k];
#pragma unroll
            for (int i = 0; i < NDC; i++) {
              if (i >= ndc) break;
              const float r = e * (PACKQ ? hs.w : sq[warp][i][jj]);
              acc[i][0] += r;
              if (PGH >= 2)
#pragma unroll
                for (int k = 0; k < DIM; k++) acc[i][1 + k] = fmaf(dg[k], r, acc[i][1 + k]);
              if (PGH >= 3)
#pragma unroll
                for (int m = 0; m < NH; m++) {
                  const int ka = HessIdx<DIM>::a(m), kb = HessIdx<DIM>::b(m);
                  const float hh = dg[ka] * dg[kb] + (ka == kb ? -a.rfac : 0.f);
                  acc[i][1 + DIM + m] = fmaf(hh, r, acc[i][1 + DIM + m]);
                }
            }
          }
          if (DIP) {
            // gnd_directd{p,g,h}, src/pfgt/pfgt_direct.f:204-384
            const float4 ns4 = snr[warp][DIP ? jj : 0];
            const float nv[3] = {ns4.x, ns4.y, ns4.z};
            float d[DIM], rn[DIM], rinc = 0.f;
#pragma unroll
            for (int k = 0; k < DIM; k++) {
              d[k] = a.rfac * dr[k];
              rn[k] = nv[k];
              rinc = fmaf(d[k], rn[k], rinc);
            }
            float rg[DIM];
#pragma unroll
            for (int k = 0; k < DIM; k++) rg[k] = rn[k] * a.rfac - rinc * d[k];
#pragma unroll
            for (int i = 0; i < NDC; i++) {
              if (i >= ndc) break;
              const float r = e * (PACKQ ? ls.w : sd[warp][i][jj]);
              acc[i][0] = fmaf(rinc, r, acc[i][0]);
              if (PGH >= 2)
#pragma unroll
                for (int k = 0; k < DIM; k++) acc[i][1 + k] = fmaf(rg[k], r, acc[i][1 + k]);
              if (PGH >= 3)
#pragma unroll
                for (int m = 0; m < NH; m++) {
                  const int ka = HessIdx<DIM>::a(m), kb = HessIdx<DIM>::b(m);
                  const float hh = (ka == kb) ? (-a.rfac * (d[ka] * rn[ka] + rinc) - rg[ka] * d[ka])
                                              : (-a.rfac * d[ka] * rn[kb] - rg[ka] * d[kb]);
                  acc[i][1 + DIM + m] = fmaf(hh, r, acc[i][1 + DIM + m]);
                }
            }
          }
        }
#pragma unroll
        for (int i = 0; i < NDC; i++)
#pragma unroll
          for (int c = 0; c < NC; c++) {
            accd[i][c] += (double)acc[i][c];
            acc[i][c] = 0.f;
          }
      }
    }
    if (act) {
#pragma unroll
      for (int i = 0; i < NDC; i++) {
        if (i >= ndc) break;
#pragma unroll
        for (int c = 0; c < NC; c++) {
          double* o = &a.out[((size_t)c * a.nd + a.d0 + i) * a.ne + p];
          *o += accd[i][c] + (double)acc[i][c];
        }
      }
    }
  }
}

// FP32 near field with two evaluation points per lane (charges, potential
// or potential + gradient, one density): a warp item is 64 points, lane l
// holds points l and l+32 as the two halves of FP32x2 registers, and each
// staged source feeds both through packed FP32x2 instructions, so the hi/lo
// differences, r^2, exponent argument and the FMAs of both pairs cost one
// instruction each.  Sources are staged negated and duplicated,
// (-x_hi, -x_hi, -y_hi, -y_hi), (-z_hi, -z_hi, q, q), (-x_lo, -x_lo, -y_lo,
// -y_lo), (-z_lo, -z_lo, 0, 0), so every operand pair is one 128-bit
// broadcast load.  Same arithmetic per pair as k_direct32.
template <int DIM, int PGH>
__global__ void __launch_bounds__(DW * 32) k_direct32x2(DArgs<float> a) {
  constexpr int NC = 1 + (PGH >= 2 ? DIM : 0);
  __shared__ float4 sa[DW][32], sb4[DW][32], sc[DW][32], sd4[DW][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const float ce = a.dinv * 1.4426950408889634f;  // exp(-rr/delta) = 2^(-rr*ce)
  const float2 nce = make_float2(-ce, -ce), nrf = make_float2(-a.rfac, -a.rfac);
  const int n_items = *a.n_items_dev;
  for (int it = blockIdx.x * DW + warp; it < n_items; it += gridDim.x * DW) {
    const int tb = a.item_box[it];
    const int pA = a.item_lo[it] + lane, pB = pA + 32;
    const int ehi = a.e_hi[tb];
    const bool actA = pA < ehi, actB = pB < ehi;
    float2 tx[3], txl[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      tx[k] = make_float2(0.f, 0.f);
      txl[k] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int k = 0; k < DIM; k++) {
      const double vA = actA ? a.eoff[(size_t)k * a.ne + pA] : 0.0;
      const double vB = actB ? a.eoff[(size_t)k * a.ne + pB] : 0.0;
      const float hA = (float)vA, hB = (float)vB;
      tx[k] = make_float2(hA, hB);
      txl[k] = make_float2((float)(vA - (double)hA), (float)(vB - (double)hB));
    }
    float2 acc[NC];
    double accA[NC], accB[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) {
      acc[c] = make_float2(0.f, 0.f);
      accA[c] = 0.0;
      accB[c] = 0.0;
    }
    double cT[DIM];
#pragma unroll
    for (int k = 0; k < DIM; k++) cT[k] = a.center[(size_t)tb * DIM + k];
    const int lT = a.level[tb];
    for (int li = a.l1_ptr[tb]; li < a.l1_ptr[tb + 1]; li++) {
      const int sbx = a.l1_src[li];
      if (!FGT_DCHECK(sbx >= 0 && sbx < a.nboxes, 402)) continue;
      double dc[DIM];
#pragma unroll
      for (int k = 0; k < DIM; k++) {
        double cs = a.center[(size_t)sbx * DIM + k];
        double sh = 0;
        if (a.iperiod0 == 1) {  // pfgt_find_local_shift, src/pfgt/pfgt_direct.f:620-651
          double dx = cT[k] - cs, dxp1 = dx - a.bs0, dxm1 = dx + a.bs0;
          if (fabs(dx) > fabs(dxp1)) { dx = dxp1; sh = a.bs0; }
          if (fabs(dx) > fabs(dxm1)) sh = -a.bs0;
        }
        dc[k] = (cs + sh) - cT[k];
      }
      if (box_beyond_cutoff<DIM>(dc, 0.5 * a.bs0 * (ldexp(1.0, -lT) + ldexp(1.0, -a.level[sbx])),
                                 a.dmax_d))
        continue;
      const int s0 = a.s_lo[sbx], s1 = a.s_hi[sbx];
      for (int base = s0; base < s1; base += 32) {
        const int j = base + lane;
        __syncwarp();
        if (j < s1) {
          float h[3] = {0, 0, 0}, l[3] = {0, 0, 0};
#pragma unroll
          for (int k = 0; k < DIM; k++) {
            const double v = a.soff[(size_t)k * a.ns + j] + dc[k];
            h[k] = (float)v;
            l[k] = (float)(v - (double)h[k]);
          }
          const float qv = a.q[(size_t)a.d0 * a.ns + j];
          sa[warp][lane] = make_float4(-h[0], -h[0], -h[1], -h[1]);
          sb4[warp][lane] = make_float4(-h[2], -h[2], qv, qv);
          sc[warp][lane] = make_float4(-l[0], -l[0], -l[1], -l[1]);
          sd4[warp][lane] = make_float4(-l[2], -l[2], 0.f, 0.f);
        }
        __syncwarp();
        const int cnt = min(32, s1 - base);
#pragma unroll 4
        for (int jj = 0; jj < cnt; jj++) {
          const float4 A = sa[warp][jj], Bq = sb4[warp][jj], Cl = sc[warp][jj], Dl = sd4[warp][jj];
          const float2 nh[3] = {make_float2(A.x, A.y), make_float2(A.z, A.w), make_float2(Bq.x, Bq.y)};
          const float2 nl[3] = {make_float2(Cl.x, Cl.y), make_float2(Cl.z, Cl.w), make_float2(Dl.x, Dl.y)};
          float2 dr[DIM], rr = make_float2(0.f, 0.f);
#pragma unroll
          for (int k = 0; k < DIM; k++) {
            dr[k] = __fadd2_rn(__fadd2_rn(tx[k], nh[k]), __fadd2_rn(txl[k], nl[k]));
            rr = __ffma2_rn(dr[k], dr[k], rr);
          }
          const float2 arg = __fmul2_rn(rr, nce);
          const float eA = rr.x < a.dmax ? fgt_ex2(arg.x) : 0.f;
          const float eB = rr.y < a.dmax ? fgt_ex2(arg.y) : 0.f;
          const float2 r = __fmul2_rn(make_float2(eA, eB), make_float2(Bq.z, Bq.w));
          acc[0] = __fadd2_rn(acc[0], r);
          if (PGH >= 2) {
            // gnd_directcg, src/pfgt/pfgt_direct.f:98-140: grad += -2/delta (t - s) r
            const float2 rg = __fmul2_rn(r, nrf);
#pragma unroll
            for (int k = 0; k < DIM; k++) acc[1 + k] = __ffma2_rn(dr[k], rg, acc[1 + k]);
          }
        }
#pragma unroll
        for (int c = 0; c < NC; c++) {
          accA[c] += (double)acc[c].x;
          accB[c] += (double)acc[c].y;
          acc[c] = make_float2(0.f, 0.f);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < NC; c++) {
      double* o = a.out + ((size_t)c * a.nd + a.d0) * a.ne;
      if (actA) o[pA] += accA[c];
      if (actB) o[pB] += accB[c];
    }
  }
}

// Packed list-1 sources.  For every target box, the sources of its list-1
// boxes that can reach the box (minimum distance to the box below the
// cut-off; the pairs of the others all fail the cut-off test), in list
// order, each as four float4 of the staging layout of k_direct32x2: FP32
// hi/lo splits of the FP64 source offset from the target box centre, negated
// and duplicated, and the charge.  Built once per call and shared by the
// source and target evaluation sets, so the near-field kernel streams one
// contiguous array per target box instead of walking the list (dependent
// loads of box ids, centres, ranges and FP64 offsets per list entry, and
// source batches shorter than a warp).  COUNT mode writes the kept count of
// every list entry; FILL mode writes the records at the scanned positions,
// taking the same decisions.
struct NearArgs {
  int nboxes, ns, iperiod0;
  double bs0, dmax;
  const int *l1_ptr, *l1_src, *s_lo, *s_hi, *t_lo, *t_hi, *level;
  const double *center, *soff;
  const float* q;                 // FILL: charges of density 0
  int* cnt;                       // COUNT: kept sources per list entry
  unsigned long long* total;      // COUNT: sum of cnt
  const int* pos;                 // FILL: first record of every list entry
  float4* rec;                    // FILL: 4 float4 per kept source
};

template <int DIM, bool FILL>
__global__ void k_near_lists(NearArgs n) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < n.nboxes; b += nw) {
    const int e0 = n.l1_ptr[b], e1 = n.l1_ptr[b + 1];
    const bool has_pts = (n.s_hi[b] > n.s_lo[b]) || (n.t_hi[b] > n.t_lo[b]);
    double cT[DIM];
#pragma unroll
    for (int k = 0; k < DIM; k++) cT[k] = n.center[(size_t)b * DIM + k];
    const double hT = 0.5 * n.bs0 * ldexp(1.0, -n.level[b]);
    unsigned long long tot = 0;
    for (int li = e0; li < e1; li++) {
      int kept = 0;
      const int sbx = n.l1_src[li];
      if (!FGT_DCHECK(sbx >= 0 && sbx < n.nboxes, 403)) continue;
      double dc[DIM];
#pragma unroll
      for (int k = 0; k < DIM; k++) {
        const double cs = n.center[(size_t)sbx * DIM + k];
        double sh = 0;
        if (n.iperiod0 == 1) {  // pfgt_find_local_shift, src/pfgt/pfgt_direct.f:620-651
          double dx = cT[k] - cs, dxp1 = dx - n.bs0, dxm1 = dx + n.bs0;
          if (fabs(dx) > fabs(dxp1)) { dx = dxp1; sh = n.bs0; }
          if (fabs(dx) > fabs(dxm1)) sh = -n.bs0;
        }
        dc[k] = (cs + sh) - cT[k];
      }
      if (has_pts &&
          !box_beyond_cutoff<DIM>(dc, hT + 0.5 * n.bs0 * ldexp(1.0, -n.level[sbx]), n.dmax)) {
        const int s0 = n.s_lo[sbx], s1 = n.s_hi[sbx];
        const int out = FILL ? n.pos[li] : 0;
        for (int base = s0; base < s1; base += 32) {
          const int j = base + lane;
          double v[DIM];
          bool keep = false;
          if (j < s1) {
#pragma unroll
            for (int k = 0; k < DIM; k++) v[k] = n.soff[(size_t)k * n.ns + j] + dc[k];
            keep = !box_beyond_cutoff<DIM>(v, hT, n.dmax);
          }
          const unsigned m = __ballot_sync(0xffffffffu, keep);
          if (FILL && keep) {
            float h[3] = {0.f, 0.f, 0.f}, l[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int k = 0; k < DIM; k++) {
              h[k] = (float)v[k];
              l[k] = (float)(v[k] - (double)h[k]);
            }
            const float qv = n.q[j];
            float4* r = n.rec + 4 * (size_t)(out + kept + __popc(m & ((1u << lane) - 1u)));
            r[0] = make_float4(-h[0], -h[0], -h[1], -h[1]);
            r[1] = make_float4(-h[2], -h[2], qv, qv);
            r[2] = make_float4(-l[0], -l[0], -l[1], -l[1]);
            r[3] = make_float4(-l[2], -l[2], 0.f, 0.f);
          }
          kept += __popc(m);
        }
      }
      if (!FILL && lane == 0) n.cnt[li] = kept;
      tot += kept;
    }
    if (!FILL && lane == 0 && tot) atomicAdd(n.total, tot);
  }
}

// ---- bulk asynchronous copies (TMA engine, non-tensor form) with mbarriers
__device__ __forceinline__ void mbar_init(uint64_t* mb, unsigned count) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(mb);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
// Arrive on the barrier expecting `bytes` of asynchronous writes, then copy
// `bytes` (a multiple of 16, both addresses 16-byte aligned) global -> shared;
// the copy's completion counts the bytes off the barrier.
__device__ __forceinline__ void bulk_load(void* smem, const void* gmem, unsigned bytes,
                                          uint64_t* mb) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
  const unsigned m = (unsigned)__cvta_generic_to_shared(mb);
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;\n" ::"r"(m),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(d),
      "l"(gmem), "r"(bytes), "r"(m)
      : "memory");
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// Waits for phase `parity` of the barrier to complete, for at most
// kWaitLimitNs; false when the limit ran out.
constexpr uint64_t kWaitLimitNs = 200000000ull;  // 0.2 s
__device__ __forceinline__ bool mbar_wait(uint64_t* mb, unsigned parity) {
  const unsigned m = (unsigned)__cvta_generic_to_shared(mb);
  uint64_t t0 = 0;
  for (int it = 0;; it++) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(m), "r"(parity)
        : "memory");
    if (done) return true;
    if (it == 0) t0 = global_ns();
    else if (global_ns() - t0 > kWaitLimitNs) return false;
  }
}

// Set on the host thread when the packed kernel was launched, so the status
// is read back only by calls that ran it.
thread_local bool t_packed_launched = false;

// Device status of the near-field kernel's waits: FGT_ERR_TIMEOUT when a
// wait ran out (the kernel then stopped early), read and cleared by the host
// at the end of a call.
__device__ int g_near_status;

// k_direct32x2 on packed list-1 sources: a warp item is 64 points of one
// target box; the box's records are streamed in batches of 32 sources
// (2 KB, contiguous) through a double-buffered shared-memory stage: lane 0
// issues one bulk copy per batch that completes on the buffer's mbarrier,
// and the warp waits on it with a time limit (the next batch lands while the
// current one is summed).  Items are taken from a device counter, the next
// index fetched while the current item runs.  Pair arithmetic as
// k_direct32x2.  stall_test != 0 (failure-detection tests only) omits the
// first copy, so the first wait runs out and the kernel reports
// FGT_ERR_TIMEOUT.
template <int DIM, int PGH>
__global__ void __launch_bounds__(DW * 32) k_direct32x2p(DArgs<float> a, const int* __restrict__ pos,
                                                         const float4* __restrict__ rec,
                                                         int* __restrict__ next, int stall_test) {
  constexpr int NC = 1 + (PGH >= 2 ? DIM : 0);
  __shared__ __align__(128) float4 stage[DW][2][32 * 4];
  __shared__ __align__(8) uint64_t mbar[DW][2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    mbar_init(&mbar[warp][0], 1);
    mbar_init(&mbar[warp][1], 1);
    mbar_init_fence();
  }
  __syncwarp();
  unsigned phase[2] = {0u, 0u};
  bool first_copy = true;
  const float ce = a.dinv * 1.4426950408889634f;  // exp(-rr/delta) = 2^(-rr*ce)
  const float2 nce = make_float2(-ce, -ce), nrf = make_float2(-a.rfac, -a.rfac);
  const int n_items = *a.n_items_dev;
  int it = 0;
  if (lane == 0) it = atomicAdd(next, 1);
  it = __shfl_sync(0xffffffffu, it, 0);
  while (it < n_items) {
    int nxt = 0;
    if (lane == 0) nxt = atomicAdd(next, 1);
    const int tb = a.item_box[it];
    const int pA = a.item_lo[it] + lane, pB = pA + 32;
    const int ehi = a.e_hi[tb];
    const bool actA = pA < ehi, actB = pB < ehi;
    const int c0 = pos[a.l1_ptr[tb]], c1 = pos[a.l1_ptr[tb + 1]];
    // first batch in flight before the target set-up
    if (lane == 0 && c0 < c1) {
      if (!(stall_test && first_copy))
        bulk_load(stage[warp][0], rec + 4 * (size_t)c0, 64u * (unsigned)min(32, c1 - c0),
                  &mbar[warp][0]);
      first_copy = false;
    }
    float2 tx[3], txl[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      tx[k] = make_float2(0.f, 0.f);
      txl[k] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int k = 0; k < DIM; k++) {
      const double vA = actA ? a.eoff[(size_t)k * a.ne + pA] : 0.0;
      const double vB = actB ? a.eoff[(size_t)k * a.ne + pB] : 0.0;
      const float hA = (float)vA, hB = (float)vB;
      tx[k] = make_float2(hA, hB);
      txl[k] = make_float2((float)(vA - (double)hA), (float)(vB - (double)hB));
    }
    float2 acc[NC];
    double accA[NC], accB[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) {
      acc[c] = make_float2(0.f, 0.f);
      accA[c] = 0.0;
      accB[c] = 0.0;
    }
    int buf = 0;
    for (int base = c0; base < c1; base += 32, buf ^= 1) {
      // issue the next batch into the other buffer (read completely by the
      // warp two batches ago), then wait for this one
      const int nb = base + 32;
      if (lane == 0 && nb < c1)
        bulk_load(stage[warp][buf ^ 1], rec + 4 * (size_t)nb, 64u * (unsigned)min(32, c1 - nb),
                  &mbar[warp][buf ^ 1]);
      const bool ok = mbar_wait(&mbar[warp][buf], phase[buf]);
      phase[buf] ^= 1u;
      if (!__all_sync(0xffffffffu, ok)) {
        // the wait ran out: report, let the other buffer's copy land (also
        // with a limit) so no copy outlives the block, and stop
        if (lane == 0) atomicExch(&g_near_status, FGT_ERR_TIMEOUT);
        if (nb < c1) (void)mbar_wait(&mbar[warp][buf ^ 1], phase[buf ^ 1]);
        return;
      }
      const float4* S = stage[warp][buf];
      const int cnt = min(32, c1 - base);
#pragma unroll 4
      for (int jj = 0; jj < cnt; jj++) {
        const float4 A = S[4 * jj], Bq = S[4 * jj + 1], Cl = S[4 * jj + 2], Dl = S[4 * jj + 3];
        const float2 nh[3] = {make_float2(A.x, A.y), make_float2(A.z, A.w), make_float2(Bq.x, Bq.y)};
        const float2 nl[3] = {make_float2(Cl.x, Cl.y), make_float2(Cl.z, Cl.w), make_float2(Dl.x, Dl.y)};
        float2 dr[DIM], rr = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 0; k < DIM; k++) {
          dr[k] = __fadd2_rn(__fadd2_rn(tx[k], nh[k]), __fadd2_rn(txl[k], nl[k]));
          rr = __ffma2_rn(dr[k], dr[k], rr);
        }
        const float2 arg = __fmul2_rn(rr, nce);
        const float eA = rr.x < a.dmax ? fgt_ex2(arg.x) : 0.f;
        const float eB = rr.y < a.dmax ? fgt_ex2(arg.y) : 0.f;
        const float2 r = __fmul2_rn(make_float2(eA, eB), make_float2(Bq.z, Bq.w));
        acc[0] = __fadd2_rn(acc[0], r);
        if (PGH >= 2) {
          // gnd_directcg, src/pfgt/pfgt_direct.f:98-140: grad += -2/delta (t - s) r
          const float2 rg = __fmul2_rn(r, nrf);
#pragma unroll
          for (int k = 0; k < DIM; k++) acc[1 + k] = __ffma2_rn(dr[k], rg, acc[1 + k]);
        }
      }
#pragma unroll
      for (int c = 0; c < NC; c++) {
        accA[c] += (double)acc[c].x;
        accB[c] += (double)acc[c].y;
        acc[c] = make_float2(0.f, 0.f);
      }
      __syncwarp();  // this buffer is refilled two batches on
    }
#pragma unroll
    for (int c = 0; c < NC; c++) {
      double* o = a.out + ((size_t)c * a.nd + a.d0) * a.ne;
      if (actA) o[pA] += accA[c];
      if (actB) o[pB] += accB[c];
    }
    it = __shfl_sync(0xffffffffu, nxt, 0);
  }
}

__global__ void k_items_count(int nboxes, const int* __restrict__ l1_ptr, const int* __restrict__ lo,
                              const int* __restrict__ hi, const int* __restrict__ s_lo,
                              const int* __restrict__ s_hi, const int* __restrict__ l1_src,
                              int tpi, int* __restrict__ cnt, double* __restrict__ pairs) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nboxes; b += gridDim.x * blockDim.x) {
    int ne = hi[b] - lo[b], nl = l1_ptr[b + 1] - l1_ptr[b];
    cnt[b] = (ne > 0 && nl > 0) ? (ne + tpi - 1) / tpi : 0;
    if (pairs && ne > 0 && nl > 0) {
      double ns = 0;
      for (int i = l1_ptr[b]; i < l1_ptr[b + 1]; i++) ns += s_hi[l1_src[i]] - s_lo[l1_src[i]];
      atomicAdd(pairs, ns * ne);
    }
  }
}
__global__ void k_items_fill(int nboxes, int tpi, const int* __restrict__ cnt,
                             const int* __restrict__ pos, const int* __restrict__ lo,
                             int* __restrict__ ibox, int* __restrict__ ilo) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nboxes; b += gridDim.x * blockDim.x)
    for (int c = 0; c < cnt[b]; c++) {
      ibox[pos[b] + c] = b;
      ilo[pos[b] + c] = lo[b] + tpi * c;
    }
}

template <typename T, int DIM, int PGH, bool CHG, bool DIP, int NDC>
void launch_direct(const DArgs<T>& a, cudaStream_t s) {
  int grid = std::max(1, std::min(ceil_div(a.n_items, DW), kSMs * 16));
  if constexpr (sizeof(T) == 4)
    k_direct32<DIM, PGH, CHG, DIP, NDC><<<grid, DW * 32, 0, s>>>(a);
  else
    k_direct<T, DIM, PGH, CHG, DIP, NDC><<<grid, DW * 32, 0, s>>>(a);
  FGT_LAUNCH_CHECK();
}

template <typename T, int DIM, int PGH, int NDC>
void dispatch_cd(const DArgs<T>& a, bool chg, bool dip, cudaStream_t s) {
  if (chg && dip) launch_direct<T, DIM, PGH, true, true, NDC>(a, s);
  else if (chg) launch_direct<T, DIM, PGH, true, false, NDC>(a, s);
  else launch_direct<T, DIM, PGH, false, true, NDC>(a, s);
}
template <typename T, int DIM, int NDC>
void dispatch_pgh(const DArgs<T>& a, int pgh, bool chg, bool dip, cudaStream_t s) {
  if (pgh == 1) dispatch_cd<T, DIM, 1, NDC>(a, chg, dip, s);
  else if (pgh == 2) dispatch_cd<T, DIM, 2, NDC>(a, chg, dip, s);
  else dispatch_cd<T, DIM, 3, NDC>(a, chg, dip, s);
}
template <typename T, int NDC>
void dispatch_dim(const DArgs<T>& a, int dim, int pgh, bool chg, bool dip, cudaStream_t s) {
  if (dim == 1) dispatch_pgh<T, 1, NDC>(a, pgh, chg, dip, s);
  else if (dim == 2) dispatch_pgh<T, 2, NDC>(a, pgh, chg, dip, s);
  else dispatch_pgh<T, 3, NDC>(a, pgh, chg, dip, s);
}

}  // namespace

namespace {
NearArgs near_args(const DirectGeom& g, const Lists& L, const int* s_lo, const int* s_hi,
                   const int* t_lo, const int* t_hi, const double* soff, int ns) {
  NearArgs n{};
  n.nboxes = g.nboxes;
  n.ns = ns;
  n.iperiod0 = g.iperiod0;
  n.bs0 = g.bs0;
  n.dmax = g.dmax;
  n.l1_ptr = L.l1_ptr;
  n.l1_src = L.l1_src;
  n.s_lo = s_lo;
  n.s_hi = s_hi;
  n.t_lo = t_lo;
  n.t_hi = t_hi;
  n.level = g.level;
  n.center = g.center;
  n.soff = soff;
  return n;
}
template <bool FILL>
void launch_near_lists(int dim, const NearArgs& n, cudaStream_t s) {
  const int grid = grid_for((long long)n.nboxes * 32, 256);
  if (dim == 1) k_near_lists<1, FILL><<<grid, 256, 0, s>>>(n);
  else if (dim == 2) k_near_lists<2, FILL><<<grid, 256, 0, s>>>(n);
  else k_near_lists<3, FILL><<<grid, 256, 0, s>>>(n);
  FGT_LAUNCH_CHECK();
}
}  // namespace

long long near_lists_count(const DirectGeom& g, const Lists& L, const int* s_lo, const int* s_hi,
                           const int* t_lo, const int* t_hi, const double* soff, int ns,
                           long long max_records, DBuf<int>& pos, cudaStream_t s) {
  if (L.n_l1 <= 0) return -1;
  NearArgs n = near_args(g, L, s_lo, s_hi, t_lo, t_hi, soff, ns);
  DBuf<int> cnt(L.n_l1, s);
  DBuf<unsigned long long> tot(1, s);
  tot.zero();
  n.cnt = cnt;
  n.total = tot;
  launch_near_lists<false>(g.dim, n, s);
  unsigned long long h = 0;
  FGT_CUDA(cudaMemcpyAsync(&h, tot.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
  FGT_CUDA(cudaStreamSynchronize(s));
  if ((long long)h > max_records) return -1;
  pos.alloc((size_t)L.n_l1 + 1, s);
  exclusive_scan_i32(cnt, pos, L.n_l1, pos.get() + L.n_l1, s);
  return (long long)h;
}

int near_wait_status(cudaStream_t s) {
  if (!t_packed_launched) return FGT_OK;
  t_packed_launched = false;
  int v = 0, z = 0;
  FGT_CUDA(cudaMemcpyFromSymbolAsync(&v, g_near_status, sizeof(v), 0, cudaMemcpyDeviceToHost, s));
  FGT_CUDA(cudaStreamSynchronize(s));
  if (v) FGT_CUDA(cudaMemcpyToSymbolAsync(g_near_status, &z, sizeof(z), 0, cudaMemcpyHostToDevice, s));
  return v;
}

void near_lists_fill(const DirectGeom& g, const Lists& L, const SourceSet<float>& src,
                     const int* t_lo, const int* t_hi, const int* pos, float4* rec,
                     cudaStream_t s) {
  NearArgs n = near_args(g, L, src.lo, src.hi, t_lo, t_hi, src.off, src.n);
  n.q = src.q;
  n.pos = pos;
  n.rec = rec;
  launch_near_lists<true>(g.dim, n, s);
}

namespace {
// Blocks of k_direct32x2p resident on the device at once (the grid of the
// dynamically scheduled launch).
template <int DIM, int PGH>
int resident_blocks_p() {
  static int nb = 0;
  if (nb == 0) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_direct32x2p<DIM, PGH>, DW * 32, 0) !=
            cudaSuccess ||
        per_sm <= 0) {
      (void)cudaGetLastError();
      per_sm = 4;
    }
    int dev = 0, sms = kSMs;
    if (cudaGetDevice(&dev) == cudaSuccess)
      (void)cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    nb = per_sm * sms;
  }
  return nb;
}
// FGT_TEST_NEAR_STALL=1 (failure-detection tests only): the packed
// near-field kernel omits its first copy and must report FGT_ERR_TIMEOUT.
int near_stall_test() {
  const char* e = getenv("FGT_TEST_NEAR_STALL");
  return (e && e[0] == '1') ? 1 : 0;
}
template <int DIM, int PGH>
void launch_packed(const DArgs<float>& a, const NearPacked& p, int* next, cudaStream_t s) {
  t_packed_launched = true;
  const int grid = std::max(1, std::min(ceil_div(a.n_items, DW), resident_blocks_p<DIM, PGH>()));
  k_direct32x2p<DIM, PGH><<<grid, DW * 32, 0, s>>>(a, p.pos, p.rec, next, near_stall_test());
  FGT_LAUNCH_CHECK();
}
}  // namespace

template <typename T>
int direct_near_field(const DirectGeom& g, const Lists& L, const SourceSet<T>& src,
                      const EvalSet<T>& e, double* pairs, cudaStream_t s, const NearPacked* packed) {
  if (e.pgh <= 0 || e.n <= 0 || L.n_l1 <= 0) return 0;
  int nb = g.nboxes, launches = 0;
  bool chg = src.q != nullptr, dip = src.ds != nullptr;
  // two evaluation points per lane: FP32, charges only, pot or pot + grad, one density
  const bool paired = sizeof(T) == 4 && chg && !dip && e.pgh <= 2 && g.nd == 1;
  const int tpi = paired ? 64 : 32;
  DBuf<int> cnt(nb, s), pos(nb, s), tot(1, s);
  DBuf<double> dpairs(1, s);
  dpairs.zero();
  k_items_count<<<grid_for(nb, 128), 128, 0, s>>>(nb, L.l1_ptr, e.lo, e.hi, src.lo, src.hi,
                                                   L.l1_src, tpi, cnt,
                                                   pairs ? dpairs.get() : nullptr);
  FGT_LAUNCH_CHECK();
  exclusive_scan_i32(cnt, pos, nb, tot, s);
  if (pairs) {  // statistics only: the one read-back of this function
    double h = 0;
    FGT_CUDA(cudaMemcpyAsync(&h, dpairs.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
    FGT_CUDA(cudaStreamSynchronize(s));
    *pairs += h;
  }
  launches += 2;
  // the item count stays on the device: sum_b ceil(ne_b / tpi) <= ne / tpi + nboxes
  const int n_items = (int)std::min<long long>((long long)e.n / tpi + nb + 1, INT32_MAX);
  DBuf<int> ibox(n_items, s), ilo(n_items, s);
  k_items_fill<<<grid_for(nb, 128), 128, 0, s>>>(nb, tpi, cnt, pos, e.lo, ibox, ilo);
  FGT_LAUNCH_CHECK();
  launches++;
  DArgs<T> a;
  a.n_items = n_items;
  a.n_items_dev = tot;
  a.nd = g.nd;
  a.ne = e.n;
  a.ns = src.n;
  a.iperiod0 = g.iperiod0;
  a.nboxes = g.nboxes;
  a.dinv = (T)(1.0 / g.delta);
  a.dmax = (T)g.dmax;
  a.rfac = (T)(2.0 / g.delta);
  a.bs0 = g.bs0;
  a.item_box = ibox;
  a.item_lo = ilo;
  a.l1_ptr = L.l1_ptr;
  a.l1_src = L.l1_src;
  a.s_lo = src.lo;
  a.s_hi = src.hi;
  a.e_hi = e.hi;
  a.soff = src.off;  // FP64
  a.q = src.q;
  a.ds = src.ds;
  a.rn = src.rn;
  a.eoff = e.off;
  a.center = g.center;
  a.level = g.level;
  a.dmax_d = g.dmax;
  a.out = e.out;
  if constexpr (sizeof(T) == 4) {
    if (paired && packed && packed->rec) {
      a.d0 = 0;
      DBuf<int> next(1, s);
      next.zero();
      const DArgs<float>& af = a;
      if (g.dim == 1) {
        if (e.pgh == 1) launch_packed<1, 1>(af, *packed, next, s);
        else launch_packed<1, 2>(af, *packed, next, s);
      } else if (g.dim == 2) {
        if (e.pgh == 1) launch_packed<2, 1>(af, *packed, next, s);
        else launch_packed<2, 2>(af, *packed, next, s);
      } else {
        if (e.pgh == 1) launch_packed<3, 1>(af, *packed, next, s);
        else launch_packed<3, 2>(af, *packed, next, s);
      }
      return launches + 1;
    }
    if (paired) {
      a.d0 = 0;
      const int grid = std::max(1, std::min(ceil_div(n_items, DW), kSMs * 16));
      const DArgs<float>& af = a;
      if (g.dim == 1) {
        if (e.pgh == 1) k_direct32x2<1, 1><<<grid, DW * 32, 0, s>>>(af);
        else k_direct32x2<1, 2><<<grid, DW * 32, 0, s>>>(af);
      } else if (g.dim == 2) {
        if (e.pgh == 1) k_direct32x2<2, 1><<<grid, DW * 32, 0, s>>>(af);
        else k_direct32x2<2, 2><<<grid, DW * 32, 0, s>>>(af);
      } else {
        if (e.pgh == 1) k_direct32x2<3, 1><<<grid, DW * 32, 0, s>>>(af);
        else k_direct32x2<3, 2><<<grid, DW * 32, 0, s>>>(af);
      }
      FGT_LAUNCH_CHECK();
      return launches + 1;
    }
  }
  for (int d0 = 0; d0 < g.nd; d0 += (g.nd == 1 ? 1 : 4)) {
    a.d0 = d0;
    if (g.nd == 1) dispatch_dim<T, 1>(a, g.dim, e.pgh, chg, dip, s);
    else dispatch_dim<T, 4>(a, g.dim, e.pgh, chg, dip, s);
    launches++;
  }
  return launches;
}

template int direct_near_field<float>(const DirectGeom&, const Lists&, const SourceSet<float>&,
                                      const EvalSet<float>&, double*, cudaStream_t,
                                      const NearPacked*);
template int direct_near_field<double>(const DirectGeom&, const Lists&, const SourceSet<double>&,
                                       const EvalSet<double>&, double*, cudaStream_t,
                                       const NearPacked*);

}  // namespace fgt

// ---------------------------------------------------------------------------
// All-pairs FP64 direct sum with the argument list of the reference's
// pfgt_direct (src/pfgt/pfgt.f:1156-1382): used by the pfgt_direct_ export.
namespace fgt {
namespace {
__global__ void k_direct_all(int nd, int dim, double delta, double dmax, const double* __restrict__ shift,
                             int ns, const double* __restrict__ src, const double* __restrict__ q,
                             const double* __restrict__ rn, const double* __restrict__ ds, int nt,
                             const double* __restrict__ trg, int pgh, double* __restrict__ pot,
                             double* __restrict__ grad, double* __restrict__ hess) {
  const int nh = dim * (dim + 1) / 2;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nt; j += gridDim.x * blockDim.x) {
    for (int i = 0; i < ns; i++) {
      double dr[3], rr = 0;
      for (int k = 0; k < dim; k++) {
        dr[k] = trg[(size_t)j * dim + k] - (src[(size_t)i * dim + k] + (shift ? shift[k] : 0.0));
        rr += dr[k] * dr[k];
      }
      if (!(rr < dmax)) continue;
      double e = exp(-rr / delta);
      int ha[6], hb[6];
      if (dim == 1) { ha[0] = 0; hb[0] = 0; }
      else if (dim == 2) { ha[0] = 0; hb[0] = 0; ha[1] = 0; hb[1] = 1; ha[2] = 1; hb[2] = 1; }
      else {
        ha[0] = 0; hb[0] = 0; ha[1] = 1; hb[1] = 1; ha[2] = 2; hb[2] = 2;
        ha[3] = 0; hb[3] = 1; ha[4] = 0; hb[4] = 2; ha[5] = 1; hb[5] = 2;
      }
      if (q) {
        double rf = -2.0 / delta, dg[3];
        for (int k = 0; k < dim; k++) dg[k] = rf * dr[k];
        for (int id = 0; id < nd; id++) {
          double r = e * q[(size_t)i * nd + id];
          pot[(size_t)j * nd + id] += r;
          if (pgh >= 2)
            for (int k = 0; k < dim; k++) grad[((size_t)j * dim + k) * nd + id] += dg[k] * r;
          if (pgh >= 3)
            for (int m = 0; m < nh; m++)
              hess[((size_t)j * nh + m) * nd + id] +=
                  (dg[ha[m]] * dg[hb[m]] + (ha[m] == hb[m] ? rf : 0.0)) * r;
        }
      }
      if (ds) {
        double rf = 2.0 / delta, d[3], n[3], rinc = 0, rg[3];
        for (int k = 0; k < dim; k++) {
          d[k] = rf * dr[k];
          n[k] = rn[(size_t)i * dim + k];
          rinc += d[k] * n[k];
        }
        for (int k = 0; k < dim; k++) rg[k] = n[k] * rf - rinc * d[k];
        for (int id = 0; id < nd; id++) {
          double r = e * ds[(size_t)i * nd + id];
          pot[(size_t)j * nd + id] += rinc * r;
          if (pgh >= 2)
            for (int k = 0; k < dim; k++) grad[((size_t)j * dim + k) * nd + id] += rg[k] * r;
          if (pgh >= 3)
            for (int m = 0; m < nh; m++) {
              int a = ha[m], b = hb[m];
              double h = (a == b) ? (-rf * (d[a] * n[a] + rinc) - rg[a] * d[a])
                                  : (-rf * d[a] * n[b] - rg[a] * d[b]);
              hess[((size_t)j * nh + m) * nd + id] += h * r;
            }
        }
      }
    }
  }
}
}  // namespace

void direct_all_pairs(int nd, int dim, double delta, double dmax, const double* shift, int ns,
                      const double* src, const double* q, const double* rn, const double* ds,
                      int nt, const double* trg, int pgh, double* pot, double* grad, double* hess,
                      cudaStream_t s) {
  if (nt <= 0 || ns <= 0 || pgh <= 0) return;
  k_direct_all<<<grid_for(nt, 128), 128, 0, s>>>(nd, dim, delta, dmax, shift, ns, src, q, rn, ds,
                                                 nt, trg, pgh, pot, grad, hess);
  FGT_LAUNCH_CHECK();
}

}  // namespace fgt
