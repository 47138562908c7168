// Instantiates the forward gather kernel over intercept-form float32 rows
// (plans built forward_only), apart from pstm_gather_fwd.cu so the two
// compile in parallel.
#include "pstm_gather2.cuh"

namespace pstm {

cudaError_t launch_forward_icpt(const Plan* p, const KArgs& A, cudaStream_t s) {
  switch (p->shape.id) {
    case 1:
    case 5:
      return dispatch2_wm<8, 2, 8, RowIcpt, OP_FWD>(p, A, s);
    case 2:
    case 8:
      return dispatch2_wm<4, 4, 4, RowIcpt, OP_FWD>(p, A, s);
    case 4:
    case 6:
      return dispatch2_wm<4, 2, 4, RowIcpt, OP_FWD>(p, A, s);
    case 7:
      return dispatch2_wm<2, 4, 2, RowIcpt, OP_FWD>(p, A, s);
    case 3:
    case 9:
      return dispatch2_wm<16, 1, 8, RowIcpt, OP_FWD>(p, A, s);
    case 10:
    case 12:
      return dispatch2_wm<16, 1, 4, RowIcpt, OP_FWD>(p, A, s);
    case 11:
      return dispatch2_wm<16, 1, 2, RowIcpt, OP_FWD>(p, A, s);
    case 13:
      return dispatch2_wm<8, 1, 8, RowIcpt, OP_FWD>(p, A, s);
  }
  return cudaErrorInvalidValue;
}

}  // namespace pstm
