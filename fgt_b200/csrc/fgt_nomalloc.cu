// fgt_direct_nomalloc: the FP64 all-pairs direct Gauss sum of pfgt_direct_
// for callers that cannot allocate device memory.
//
// Callers that cannot allocate: host codes that hand (nearly) the whole GPU
// to another allocator up front -- a PyTorch or RAPIDS memory pool, or a
// solver's own arena -- where cudaMalloc fails although the pool has room,
// and latency-bound loops that cannot take the implicit device
// synchronisation of cudaMalloc/cudaFree.  They pass device buffers they
// already own; the only other memory used is the fixed array below.
//
// Scratch: one file-scope __device__ array of FGT_NOMALLOC_SCRATCH_BYTES,
// held by every GPU that loads the library until the process exits.  It
// holds the FP64 accumulators of all outputs (pot, grad, hess of nt targets)
// so that CTAs working on different source chunks of the same targets can
// add into it; it is cleared at the start of every call and added onto the
// caller's outputs at the end.  Every call shares it: calls that overlap on
// the GPU (on any streams) race.  In host code `g_scratch` only names the
// symbol; its device address comes from cudaGetSymbolAddress, resolved once
// per device by the first call made with that device current.  CUDA loads a
// module's device memory lazily, so that first call is also when the GPU
// reserves the array: make it (a call with nt = 0 does it and computes
// nothing) before the host hands the GPU's memory to its pool and before
// any stream capture.
#include <algorithm>
#include <mutex>

#include "fgt_b200.h"
#include "fgt_common.cuh"

namespace fgt {
namespace {

constexpr size_t kScratchDoubles = (size_t)FGT_NOMALLOC_SCRATCH_BYTES / sizeof(double);
static __device__ __align__(256) double g_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
constexpr int kTargets = 128;   // targets per CTA (one per thread)
constexpr int kChunk = 1024;    // sources per CTA
constexpr int kTile = 128;      // sources staged in shared memory at a time

std::mutex g_setup_mutex;
double* g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of g_scratch on device dev (current), resolved once.
double* scratch_on(int dev) {
  FGT_REQUIRE(dev >= 0 && dev < kMaxDevices, FGT_ERR_UNSUPPORTED, "device ordinal too large");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    FGT_CUDA(cudaGetSymbolAddress(&p, g_scratch));
    FGT_REQUIRE(p != nullptr, FGT_ERR_CUDA, "cudaGetSymbolAddress returned no address");
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  return g_scratch_ptr[dev];
}

struct Shift {
  double v[3];
};

// Hessian component m -> (a, b): 3D xx,yy,zz,xy,xz,yz; 2D xx,xy,yy; 1D xx.
__device__ __forceinline__ void hess_pair(int dim, int m, int& a, int& b) {
  if (dim == 1) {
    a = 0;
    b = 0;
  } else if (dim == 2) {
    a = m == 2 ? 1 : 0;
    b = m == 0 ? 0 : 1;
  } else {
    a = m < 3 ? m : (m < 5 ? 0 : 1);
    b = m < 3 ? m : (m == 3 ? 1 : 2);
  }
}

// Variant of the all-pairs kernel behind pfgt_direct_: CTA (x, y) takes
// kTargets targets and source chunk y, stages the chunk through shared
// memory and adds its sums into the scratch accumulators acc, laid out like
// the outputs: pot [nt][nd], grad [nt][dim][nd], hess [nt][nh][nd] at
// offsets 0, nt*nd, nt*nd*(1+dim).
__global__ void __launch_bounds__(kTargets)
    k_direct_scratch(int nd, int dim, double delta, double dmax, Shift sh, int ns,
                     const double* __restrict__ src, const double* __restrict__ q,
                     const double* __restrict__ rn, const double* __restrict__ ds, int nt,
                     const double* __restrict__ trg, int pgh, double* __restrict__ acc) {
  __shared__ double sx[3][kTile], sq[kTile], sn[3][kTile], sd[kTile];
  const int nh = dim * (dim + 1) / 2;
  const int j = blockIdx.x * kTargets + threadIdx.x;
  const bool active = j < nt;
  double t[3] = {0, 0, 0};
  if (active)
    for (int k = 0; k < dim; k++) t[k] = trg[(size_t)j * dim + k];
  double* apot = acc;
  double* agrad = acc + (size_t)nt * nd;
  double* ahess = agrad + (pgh >= 2 ? (size_t)nt * nd * dim : 0);
  for (int c0 = blockIdx.y * kChunk; c0 < ns; c0 += gridDim.y * kChunk) {
    const int c1 = min(ns, c0 + kChunk);
    for (int id = 0; id < nd; id++) {
      double v[10];
#pragma unroll
      for (int c = 0; c < 10; c++) v[c] = 0;
      for (int s0 = c0; s0 < c1; s0 += kTile) {
        const int n = min(kTile, c1 - s0);
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
          const size_t si = (size_t)(s0 + i);
          for (int k = 0; k < dim; k++) {
            sx[k][i] = src[si * dim + k] + sh.v[k];
            if (ds) sn[k][i] = rn[si * dim + k];
          }
          sq[i] = q ? q[si * nd + id] : 0.0;
          sd[i] = ds ? ds[si * nd + id] : 0.0;
        }
        __syncthreads();
        if (!active) continue;
        for (int i = 0; i < n; i++) {
          double dr[3] = {0, 0, 0}, rr = 0;
          for (int k = 0; k < dim; k++) {
            dr[k] = t[k] - sx[k][i];
            rr += dr[k] * dr[k];
          }
          if (!(rr < dmax)) continue;
          const double e = exp(-rr / delta);
          if (q) {
            const double rf = -2.0 / delta, r = e * sq[i];
            v[0] += r;
            if (pgh >= 2)
              for (int k = 0; k < dim; k++) v[1 + k] += rf * dr[k] * r;
            if (pgh >= 3)
              for (int m = 0; m < nh; m++) {
                int a, b;
                hess_pair(dim, m, a, b);
                v[1 + dim + m] += (rf * dr[a] * rf * dr[b] + (a == b ? rf : 0.0)) * r;
              }
          }
          if (ds) {
            const double rf = 2.0 / delta, r = e * sd[i];
            double d[3], nn[3], rinc = 0, rg[3];
            for (int k = 0; k < dim; k++) {
              d[k] = rf * dr[k];
              nn[k] = sn[k][i];
              rinc += d[k] * nn[k];
            }
            for (int k = 0; k < dim; k++) rg[k] = nn[k] * rf - rinc * d[k];
            v[0] += rinc * r;
            if (pgh >= 2)
              for (int k = 0; k < dim; k++) v[1 + k] += rg[k] * r;
            if (pgh >= 3)
              for (int m = 0; m < nh; m++) {
                int a, b;
                hess_pair(dim, m, a, b);
                const double h = (a == b) ? (-rf * (d[a] * nn[a] + rinc) - rg[a] * d[a])
                                          : (-rf * d[a] * nn[b] - rg[a] * d[b]);
                v[1 + dim + m] += h * r;
              }
          }
        }
      }
      if (active) {
        atomicAdd(&apot[(size_t)j * nd + id], v[0]);
        if (pgh >= 2)
          for (int k = 0; k < dim; k++) atomicAdd(&agrad[((size_t)j * dim + k) * nd + id], v[1 + k]);
        if (pgh >= 3)
          for (int m = 0; m < nh; m++)
            atomicAdd(&ahess[((size_t)j * nh + m) * nd + id], v[1 + dim + m]);
      }
    }
  }
}

// out[i] += acc[i] for the three output blocks.
__global__ void k_add_scratch(const double* __restrict__ acc, size_t npot, size_t ngrad,
                              size_t nhess, double* __restrict__ pot, double* __restrict__ grad,
                              double* __restrict__ hess) {
  const size_t n = npot + ngrad + nhess;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    if (i < npot) pot[i] += acc[i];
    else if (i < npot + ngrad) grad[i - npot] += acc[i];
    else hess[i - npot - ngrad] += acc[i];
  }
}

int direct_nomalloc(int nd, int dim, double delta, double dmax, const double* shifts, int ns,
                    const double* sources, int ifcharge, const double* charge, int ifdipole,
                    const double* rnormal, const double* dipstr, int nt, const double* targ,
                    int ifpgh, double* pot, double* grad, double* hess, void* stream) {
  FGT_REQUIRE(nd >= 1 && dim >= 1 && dim <= 3 && ns >= 0 && nt >= 0, FGT_ERR_ARG,
              "bad nd/dim/ns/nt");
  FGT_REQUIRE(ifpgh >= 1 && ifpgh <= 3, FGT_ERR_ARG, "ifpgh must be 1, 2 or 3");
  FGT_REQUIRE(delta > 0, FGT_ERR_ARG, "delta must be positive");
  const int nh = dim * (dim + 1) / 2;
  const size_t npot = (size_t)nt * nd;
  const size_t ngrad = ifpgh >= 2 ? npot * dim : 0;
  const size_t nhess = ifpgh >= 3 ? npot * nh : 0;
  FGT_REQUIRE(npot + ngrad + nhess <= kScratchDoubles, FGT_ERR_UNSUPPORTED,
              "outputs exceed the static scratch of fgt_direct_nomalloc "
              "(nt*nd*(1 + dim*[ifpgh>=2] + nhess*[ifpgh>=3]) * 8 bytes must be <= "
              "FGT_NOMALLOC_SCRATCH_BYTES = 8 MiB)");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    (void)cudaGetLastError();
    FGT_REQUIRE(false, FGT_ERR_NODEVICE, "no CUDA device");
  }
  int dev = 0;
  FGT_CUDA(cudaGetDevice(&dev));
  // Resolved before the empty-call return: a call with nt = 0 or ns = 0
  // loads this module on the device (its static scratch is reserved then)
  // and looks up the address, so a host can make that warm-up call before
  // it hands the GPU's memory to its own pool or starts a stream capture.
  double* acc = scratch_on(dev);
  if (nt == 0 || ns == 0) return FGT_OK;
  FGT_REQUIRE(sources && targ && pot, FGT_ERR_ARG, "sources, targ and pot are required");
  FGT_REQUIRE(ifcharge != 1 || charge, FGT_ERR_ARG, "charge is required when ifcharge=1");
  FGT_REQUIRE(ifdipole != 1 || (rnormal && dipstr), FGT_ERR_ARG,
              "rnormal and dipstr are required when ifdipole=1");
  FGT_REQUIRE(ifpgh < 2 || grad, FGT_ERR_ARG, "grad is required when ifpgh>=2");
  FGT_REQUIRE(ifpgh < 3 || hess, FGT_ERR_ARG, "hess is required when ifpgh=3");
  if (ifcharge != 1 && ifdipole != 1) return FGT_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  FGT_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * (npot + ngrad + nhess), s));
  Shift sh = {{0, 0, 0}};
  if (shifts)
    for (int k = 0; k < dim; k++) sh.v[k] = shifts[k];
  const int gx = (nt + kTargets - 1) / kTargets;
  const int gy = std::min((ns + kChunk - 1) / kChunk, 65535);
  k_direct_scratch<<<dim3(gx, gy), kTargets, 0, s>>>(
      nd, dim, delta, dmax, sh, ns, sources, ifcharge == 1 ? charge : nullptr,
      ifdipole == 1 ? rnormal : nullptr, ifdipole == 1 ? dipstr : nullptr, nt, targ, ifpgh, acc);
  FGT_LAUNCH_CHECK();
  const size_t ntot = npot + ngrad + nhess;
  const int ga = (int)std::min<size_t>((ntot + 255) / 256, (size_t)kSMs * 8);
  k_add_scratch<<<ga, 256, 0, s>>>(acc, npot, ngrad, nhess, pot, grad, hess);
  FGT_LAUNCH_CHECK();
  return FGT_OK;
}

}  // namespace
}  // namespace fgt

extern "C" int fgt_direct_nomalloc(int nd, int dim, double delta, double dmax,
                                   const double* shifts, int ns, const double* sources,
                                   int ifcharge, const double* charge, int ifdipole,
                                   const double* rnormal, const double* dipstr, int nt,
                                   const double* targ, int ifpgh, double* pot, double* grad,
                                   double* hess, void* stream) {
  try {
    return fgt::direct_nomalloc(nd, dim, delta, dmax, shifts, ns, sources, ifcharge, charge,
                                ifdipole, rnormal, dipstr, nt, targ, ifpgh, pot, grad, hess,
                                stream);
  } catch (const fgt::Error& e) {
    return e.code;
  } catch (...) {
    fgt_set_error_message("unexpected host exception", __FILE__, __LINE__);
    return FGT_ERR_CUDA;
  }
}
