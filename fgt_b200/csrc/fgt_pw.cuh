// Plane-wave part of the point FGT on the device: form (K6, type-1 NUFFT:
// spread + pruned DFT + deconvolution), translate (K7, diagonal shifts),
// evaluate (K8, type-2: pruned inverse DFT + interpolation, or direct modal
// sums for boxes with few points).
//
// Hermitian half-space storage.  For real strengths the expansion satisfies
// M(-k) = conj(M(k)), so only modes with k_last >= 0 are stored: k_1..k_{d-1}
// in [-K, K], k_d in [0, K], K = npw/2, x fastest.  The reference's mode set
// [-K, K-1]^d (src/pfgt/pfgt.f:612-613) is symmetrised by splitting the
// k = -K term evenly between -K and +K in every dimension (real part
// unchanged up to O(w_K^2) ~ 1e-14 relative).
#pragma once
#include <vector>

#include "fgt_direct.cuh"

namespace fgt {

struct PWParams {
  int dim = 0, nd = 0, K = 0;   // modes per dim: 2K+1 (last dim: K+1 stored)
  int nexp = 0;                 // stored complex coefficients per expansion per density
  double delta0 = 1, hpw = 0;   // xj = off * hpw / sqrt(delta0)
  double sqd0 = 1;              // sqrt(delta0)
  // spreading grid: spacing dx = 2pi/nf, kernel width w cells, ES beta
  int nf = 0, w = 0, G = 0, l0 = 0;  // sub-grid cells l0 .. l0+G-1 (periodic if G == nf)
  bool wrap = false;
  double beta = 0, dx = 0, halfw = 0;  // halfw = w*dx/2
  std::vector<double> ts;   // ts(k) for k = -K..K (index k+K)
  std::vector<double> wsym; // symmetrised weights, index k+K
  std::vector<double> phihat;  // FT of the spreading kernel at k = -K..K
  double xmin = 0;          // box size at the cutoff level / sqrt(delta0)
  double boxsize_cut = 0;   // box size at the cutoff level
};

// Host set-up of the plane-wave parameters (FP64): nodes and weights of
// get_pwnodes / get_periodic_pwnodes (src/common/fgtterms.f:151-211), grid
// and kernel of the spreader, kernel Fourier transform by quadrature.
void pw_setup(PWParams& P, int dim, int nd, int npw, double pmax, int periodic_nodes,
              double bs0, double delta, double eps, double boxsize_cut, int spread_width);
// (Re)computes the width-dependent grid of P (kernel width w cells).
// exact_w: use width w as given (odd widths of the FP32 derivative
// evaluation); otherwise w is rounded up to an even supported width
void pw_grid(PWParams& P, int w, bool exact_w = false);

template <typename T>
struct PWData {
  DBuf<T> mp;    // [n_form][nd][nexp] complex (2 T each)
  DBuf<T> loc;   // [n_eval][nd][nexp] complex
  DBuf<T> wtab;  // [3^dim][nexp] complex shift tables
};

// Algorithmic work counters of one call (optional).
struct PWWork {
  double pts_form = 0, pts_nufft = 0, pts_modal = 0;
  double flops_form = 0, flops_eval = 0, bytes_translate = 0;
  int n_nufft = 0, w_eval = 0, G_eval = 0;
  int slabs_form = 1, slabs_eval = 1;  // x-slabs per sub-grid (1: whole grids)
};

// Forms the expansions of all form boxes.  Returns launches.
template <typename T>
int pw_form(const PWParams& P, const Tree& t, const Lists& L, const SourceSet<T>& src,
            PWData<T>& D, PWWork* work, cudaStream_t s);
template <typename T>
int pw_translate(const PWParams& P, const Lists& L, PWData<T>& D, PWWork* work, cudaStream_t s);
template <typename T>
int pw_eval(const PWParams& P, const Tree& t, const Lists& L, const PWData<T>& D,
            const EvalSet<T>& e0, const EvalSet<T>& e1, int small_eval, PWWork* work,
            cudaStream_t s);

}  // namespace fgt
