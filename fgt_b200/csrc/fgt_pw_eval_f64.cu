// Plane-wave evaluation (K8), FP64 instantiation: the kernels and the driver
// pw_eval are in fgt_pw_eval_impl.cuh.
#include "fgt_pw_eval_impl.cuh"

namespace fgt {

template int pw_eval<double>(const PWParams&, const Tree&, const Lists&, const PWData<double>&,
                          const EvalSet<double>&, const EvalSet<double>&, int, PWWork*, cudaStream_t);

}  // namespace fgt
