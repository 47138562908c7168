// Instantiates the gather kernel for OP_ADJ (one op per translation unit).
#include "pstm_gather.cuh"

namespace pstm {

pstm_status launch_adjoint(Plan* p, const float* image, const float* vel, int64_t vst,
                           int64_t vsc, cudaStream_t s, std::string* why) {
  KArgs A = make_args(p, vel, vst, vsc);
  A.in_img = image;
  cudaError_t e = dispatch_shape<OP_ADJ>(p, A, needs_lowclamp(p), s);
  return e == cudaSuccess ? PSTM_OK : cuda_fail(e, "adjoint kernel", why);
}

}  // namespace pstm
