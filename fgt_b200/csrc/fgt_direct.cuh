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

// Packed list-1 sources of the FP32 charge path (one density, potential or
// potential + gradient): for list entry i, records pos[i] .. pos[i+1]-1 of
// rec (4 float4 each) are the sources of the entry's box that can reach the
// target box, as hi/lo FP32 offsets from the target box centre and charges.
struct NearPacked {
  const int* pos = nullptr;    // n_l1 + 1
  const float4* rec = nullptr;
};

// Counts the packed records (geometry only: boxes, offsets, cut-off) and
// scans their positions into pos (n_l1 + 1 entries).  Returns the record
// count, or -1 when there is no list 1 or the count exceeds max_records.
// Reads the count back to the host (one stream synchronisation).
long long near_lists_count(const DirectGeom& g, const Lists& L, const int* s_lo, const int* s_hi,
                           const int* t_lo, const int* t_hi, const double* soff, int ns,
                           long long max_records, DBuf<int>& pos, cudaStream_t s);
// Writes the records (charges of density 0) for positions from near_lists_count
// with the same geometry.
void near_lists_fill(const DirectGeom& g, const Lists& L, const SourceSet<float>& src,
                     const int* t_lo, const int* t_hi, const int* pos, float4* rec,
                     cudaStream_t s);

// Status of the bounded waits of the packed near-field kernel since the last
// read: FGT_OK, or FGT_ERR_TIMEOUT when a wait ran out (the kernel stopped
// early and the results are incomplete).  Clears it; synchronises the stream.
int near_wait_status(cudaStream_t s);

// Adds the list-1 interactions onto every point of `e`.  Returns the number
// of kernel launches; *pairs receives the near-field pair count if not null.
// With packed records (FP32, charges, one density, pgh <= 2) the near field
// streams them instead of walking the list.
template <typename T>
int direct_near_field(const DirectGeom& g, const Lists& L, const SourceSet<T>& src,
                      const EvalSet<T>& e, double* pairs, cudaStream_t s,
                      const NearPacked* packed = nullptr);

}  // namespace fgt

namespace fgt {
// All-pairs FP64 direct sum (AoS layouts of the reference), outputs incremented.
void direct_all_pairs(int nd, int dim, double delta, double dmax, const double* shift, int ns,
                      const double* src, const double* q, const double* rn, const double* ds,
                      int nt, const double* trg, int pgh, double* pot, double* grad, double* hess,
                      cudaStream_t s);
}  // namespace fgt
