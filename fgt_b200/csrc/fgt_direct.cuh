// Direct near-field Gaussian sums over the modified list 1 (K9).
#pragma once
#include "fgt_lists.cuh"

namespace fgt {

// One evaluation set (the sorted sources or the sorted targets).
template <typename T>
struct EvalSet {
  int n = 0;                 // number of points
  int pgh = 0;               // 1 pot, 2 +grad, 3 +hess (0: nothing requested)
  const double* off = nullptr;  // SoA [dim][n], FP64 offsets from the reference-box centre
  const int* lo = nullptr;   // per box: first sorted index
  const int* hi = nullptr;   // per box: one past the last
  double* out = nullptr;     // SoA [(comp*nd + id)*n + i], comps pot,grad..,hess..
};

// Sources (sorted, SoA) with their strengths.
template <typename T>
struct SourceSet {
  int n = 0;
  const double* off = nullptr;  // [dim][n], FP64 offsets from the box centre
  const T* q = nullptr;    // [nd][n] or null
  const T* ds = nullptr;   // [nd][n] or null (dipole strengths)
  const T* rn = nullptr;   // [dim][n] or null (dipole directions)
  const int* lo = nullptr;
  const int* hi = nullptr;
};

struct DirectGeom {
  int dim, nd, iperiod0, nboxes;
  double delta, dmax, bs0;
  const double* center;
  const int* level;  // box levels (box size bs0 * 2^-level)
};

// Adds the list-1 interactions onto every point of `e`.  Returns the number
// of kernel launches; *pairs receives the near-field pair count if not null.
template <typename T>
int direct_near_field(const DirectGeom& g, const Lists& L, const SourceSet<T>& src,
                      const EvalSet<T>& e, double* pairs, cudaStream_t s);

}  // namespace fgt

namespace fgt {
// All-pairs FP64 direct sum (AoS layouts of the reference), outputs incremented.
void direct_all_pairs(int nd, int dim, double delta, double dmax, const double* shift, int ns,
                      const double* src, const double* q, const double* rn, const double* ds,
                      int nt, const double* trg, int pgh, double* pot, double* grad, double* hess,
                      cudaStream_t s);
}  // namespace fgt
