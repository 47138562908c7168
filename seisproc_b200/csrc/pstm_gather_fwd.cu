// Instantiates the gather kernel for OP_FWD (warp-specialised pipeline; one op per translation unit).
#include "pstm_gather2.cuh"

namespace pstm {

pstm_status launch_forward(Plan* p, const float* vel, int64_t vst, int64_t vsc, float* image,
                           float* fold, cudaStream_t s, std::string* why) {
  KArgs A = make_args(p, vel, vst, vsc);
  A.out = image;
  A.fold_out = fold;
  cudaError_t e = dispatch2_shape<OP_FWD>(p, A, s);
  return e == cudaSuccess ? PSTM_OK : cuda_fail(e, "forward kernel", why);
}

}  // namespace pstm
