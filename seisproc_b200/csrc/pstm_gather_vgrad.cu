// Instantiates the gather kernel for OP_VGRAD (warp-specialised pipeline; one op per translation unit).
#include "pstm_gather2.cuh"

namespace pstm {

pstm_status launch_vgrad(Plan* p, const float* grad_image, const float* vel, int64_t vst,
                         int64_t vsc, float* grad_v, cudaStream_t s, std::string* why) {
  KArgs A = make_args(p, vel, vst, vsc);
  A.in_img = grad_image;
  A.out = grad_v;
  cudaError_t e = dispatch2_shape<OP_VGRAD>(p, A, s);
  return e == cudaSuccess ? PSTM_OK : cuda_fail(e, "velocity-gradient kernel", why);
}

}  // namespace pstm
