// Instantiates the forward gather kernel with the aperture controller's cosine
// tapers (float32 plans built with a taper width) and with curved-ray
// traveltimes (plans built with a ray gradient), apart from pstm_gather_fwd.cu
// so they compile in parallel.
#include "pstm_gather2.cuh"

namespace pstm {

namespace {
template <int COLS, int WPC, int M>
cudaError_t taper_rows(const Plan* p, const KArgs& A, cudaStream_t s) {
  return p->row_origin != 0 ? dispatch2_wm<COLS, WPC, M, RowIcpt, OP_FWD, true>(p, A, s)
                            : dispatch2_wm<COLS, WPC, M, float2, OP_FWD, true>(p, A, s);
}
template <int COLS, int WPC, int M>
cudaError_t curved_rows(const Plan* p, const KArgs& A, cudaStream_t s) {
  return p->row_origin != 0 ? dispatch2_wm<COLS, WPC, M, RowIcpt, OP_FWD, false, true>(p, A, s)
                            : dispatch2_wm<COLS, WPC, M, float2, OP_FWD, false, true>(p, A, s);
}
}  // namespace

cudaError_t launch_forward_curved(const Plan* p, const KArgs& A, cudaStream_t s) {
  if (p->shape.id == 3 || p->shape.id == 9) return curved_rows<16, 1, 8>(p, A, s);
  return cudaErrorNotSupported;
}

// Taper plans run the 16-column shape only (3: 4 x 4 tiles, 9: 16-inline
// strips), which the plan forces for them; this keeps the instantiations few.
cudaError_t launch_forward_taper(const Plan* p, const KArgs& A, cudaStream_t s) {
  if (p->shape.id == 3 || p->shape.id == 9) return taper_rows<16, 1, 8>(p, A, s);
  return cudaErrorNotSupported;
}

}  // namespace pstm
