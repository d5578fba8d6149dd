// Plane-wave evaluation (K8), FP32 instantiation: the kernels and the driver
// pw_eval are in fgt_pw_eval_impl.cuh.
#include "fgt_pw_eval_impl.cuh"

namespace fgt {

template int pw_eval<float>(const PWParams&, const Tree&, const Lists&, const PWData<float>&,
                          const EvalSet<float>&, const EvalSet<float>&, int, PWWork*, cudaStream_t);

}  // namespace fgt
