// Adaptive 2^d-tree of the point FGT built on the device.
//
// Boxes are identified by (level l, path key P): P holds l digits of `dim`
// bits, the digit of level j being the child index inside the level-j box
// (bit k set iff the point's coordinate k is >= the box centre), most
// significant digit first.  This is the child numbering of the reference
// (get_child_box_sign / find_childbox_ind, src/common/pts_tree_nd.f:713-741,
// 1418-1464), so ordering boxes and points by key reproduces the
// hierarchical order of pts_tree_sort (src/common/pts_tree_nd.f:1226-1256).
#pragma once
#include <vector>

#include "fgt_prims.cuh"

namespace fgt {

struct Tree {
  int dim = 0, mc = 0, D = 0;  // D = key depth (levels of digits in a full key)
  int nlevels = 0, nboxes = 0, npwlevel = 0, ncutoff = 0, ndiv = 0, iperiod = 0;
  int ns = 0, nt = 0, nleaves = 0;
  double bs0 = 0, cen0[FGT_MAXDIM] = {0, 0, 0};
  std::vector<double> boxsize;  // 0..nlevels
  std::vector<int> lev_start;   // nlevels+2 entries; level l = [lev_start[l], lev_start[l+1])
  // per box (global id = level-major order, keys ascending inside a level)
  DBuf<uint64_t> key;
  DBuf<int> level, nonleaf, parent, child0;
  DBuf<double> center;  // nboxes*dim
  DBuf<int> src_lo, src_hi, trg_lo, trg_hi;  // sorted point ranges [lo, hi)
  // sorted point -> original index
  DBuf<uint32_t> isrc, itrg;
  DBuf<int> src_ref, trg_ref;  // reference box of each sorted point
};

// Scalar set-up of pts_tree_boxsize0 (src/common/pts_tree_nd.f:1330-1414):
// computes levcut, and bs0/cen0 in free space (bbox reduction on the device).
void tree_setup_scalars(int dim, double delta, double eps, int iperiod, const double* d_src,
                        int ns, const double* d_trg, int nt, int* levcut, double* bs0,
                        double* cen0, cudaStream_t s);

// Builds the level-restricted tree, sorts sources and targets into it.
void tree_build(Tree& t, int dim, int iperiod, int npwlevel, int ndiv, double bs0,
                const double* cen0, const double* d_src, int ns, const double* d_trg, int nt,
                cudaStream_t s);

// Host copy of the box tables (for tests / debugging).
struct TreeHost {
  std::vector<uint64_t> key;
  std::vector<int> level, nonleaf, parent, child0, src_lo, src_hi, trg_lo, trg_hi;
  std::vector<double> center;
  std::vector<uint32_t> isrc, itrg;
};
void tree_download(const Tree& t, TreeHost& h, cudaStream_t s);

}  // namespace fgt
