// Interaction lists of the point FGT on the device: colleagues, plane-wave
// boxes and lists, and the modified list 1 of the direct near field.
#pragma once
#include "fgt_tree.cuh"

namespace fgt {

struct Lists {
  // plane-wave part (boxes at the cutoff level)
  int n_form = 0, n_eval = 0, n_trans = 0;
  DBuf<int> form_box;    // boxes that form a PW expansion (npts > ndiv)
  DBuf<int> eval_box;    // boxes with ifpwexp = 1
  DBuf<int> eval_self;   // per eval box: its own form slot or -1
  DBuf<int> trans_ptr;   // per eval box: CSR offsets into trans_src/trans_w (n_eval+1)
  DBuf<int> trans_src;   // form slot of the source expansion
  DBuf<int> trans_w;     // shift-table index 0..3^dim-1
  // direct part: CSR over all boxes (targets), sources are box ids
  DBuf<int> l1_ptr, l1_src;
  int n_l1 = 0;
};

// nlevend / iperiod0 follow pfgtmain (src/pfgt/pfgt.f:618-650).
void build_lists(const Tree& t, int npwlevel, int iperiod0, int nlevend, bool do_pw, Lists& L,
                 cudaStream_t s);

struct ListsHost {
  std::vector<int> form_box, eval_box, eval_self, trans_ptr, trans_src, trans_w, l1_ptr, l1_src;
};
void lists_download(const Lists& L, int nboxes, ListsHost& h, cudaStream_t s);

}  // namespace fgt
