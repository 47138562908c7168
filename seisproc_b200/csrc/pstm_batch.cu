// Batched migration: many plans (e.g. offset/azimuth classes of one survey,
// each with its own traces and its own output image) in ONE persistent launch.
//
// pstm_batch_create gathers the per-class kernel arguments into a device
// descriptor array and builds the list of (class, tile, window) work items,
// ordered by descending trace-list length so that the longest items start
// first and the tail of the launch stays short.  pstm_batch_migrate resets
// the work counter and launches one CTA per SM of the persistent kernel; each
// CTA pulls items until the queue is empty.  The launch sequence contains no
// allocation and no host synchronisation, so it can be captured in a CUDA
// graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "pstm_gather2.cuh"

namespace {

using namespace pstm;

struct Batch {
  std::vector<Plan*> plans;
  std::vector<float*> images, folds;
  const float* vel = nullptr;
  int64_t vst = 0, vsc = 0;
  KArgs* d_descs = nullptr;
  int4* d_items = nullptr;
  int* d_counter = nullptr;
  int n_items = 0;
  int ring_stages = 0, ring_rows = 0;
  int hist16 = 0;  // 16-bit fold histogram: every class's tile lists < 65536 traces
  int sms = 0;
};

pstm_status bfail(pstm_status st, const std::string& m) {
  set_last_error(m);
  return st;
}

template <int COLS, int WPC, int M, typename ST, int WM, bool LC>
cudaError_t launch_batch_one(const Batch* b, cudaStream_t s) {
  auto kern = pstm_batch_kernel<COLS, WPC, M, ST, WM, LC, OP_FWD>;
  const Plan* p = b->plans[0];
  const int T = WPC * 64 * M;
  const Smem2 L = smem2_layout(COLS, T, p->row_stride, (int)sizeof(ST), b->ring_stages, b->ring_rows,
                               hist_entry_bytes(b->hist16 != 0));
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L.total);
  if (e != cudaSuccess) return e;
  int per_sm = 1;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, COLS * WPC * 32, L.total);
  if (e != cudaSuccess) return e;
  const int grid = std::max(1, std::min(b->n_items, b->sms * std::max(per_sm, 1)));
  kern<<<grid, COLS * WPC * 32, L.total, s>>>(b->d_descs, b->d_items, b->n_items, b->d_counter);
  count_launch();
  return cudaGetLastError();
}

template <int COLS, int WPC, int M, typename ST>
cudaError_t batch_wm(const Batch* b, cudaStream_t s) {
  const Plan* p = b->plans[0];
  const bool lc = needs_lowclamp(p);
  if constexpr (!std::is_same<ST, float2>::value && !std::is_same<ST, RowIcpt>::value) {
    if (p->params.weight != W_OBL_SPREAD) return cudaErrorNotSupported;
    return lc ? launch_batch_one<COLS, WPC, M, ST, W_OBL_SPREAD, true>(b, s)
              : launch_batch_one<COLS, WPC, M, ST, W_OBL_SPREAD, false>(b, s);
  } else {
    switch (p->params.weight) {
      case W_OBL_SPREAD:
        return lc ? launch_batch_one<COLS, WPC, M, ST, W_OBL_SPREAD, true>(b, s)
                  : launch_batch_one<COLS, WPC, M, ST, W_OBL_SPREAD, false>(b, s);
      case W_SPREAD:
        return lc ? launch_batch_one<COLS, WPC, M, ST, W_SPREAD, true>(b, s)
                  : launch_batch_one<COLS, WPC, M, ST, W_SPREAD, false>(b, s);
      case W_OBL:
        return lc ? launch_batch_one<COLS, WPC, M, ST, W_OBL, true>(b, s)
                  : launch_batch_one<COLS, WPC, M, ST, W_OBL, false>(b, s);
      case W_NONE:
        return lc ? launch_batch_one<COLS, WPC, M, ST, W_NONE, true>(b, s)
                  : launch_batch_one<COLS, WPC, M, ST, W_NONE, false>(b, s);
    }
    return cudaErrorInvalidValue;
  }
}

template <int COLS, int WPC, int M>
cudaError_t batch_st(const Batch* b, cudaStream_t s) {
  switch (b->plans[0]->params.storage) {
    case PSTM_F32:
      // forward_only class plans stage intercept-form rows, the others (x, dx)
      return b->plans[0]->row_origin != 0 ? batch_wm<COLS, WPC, M, RowIcpt>(b, s)
                                          : batch_wm<COLS, WPC, M, float2>(b, s);
    case PSTM_BF16:
      return batch_wm<COLS, WPC, M, __nv_bfloat16>(b, s);
    case PSTM_F16:
      return batch_wm<COLS, WPC, M, __half>(b, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t batch_dispatch(const Batch* b, cudaStream_t s) {
  switch (b->plans[0]->shape.id) {
    case 1:
    case 5:
      return batch_st<8, 2, 8>(b, s);
    case 2:
    case 8:
      return batch_st<4, 4, 4>(b, s);
    case 4:
    case 6:
      return batch_st<4, 2, 4>(b, s);
    case 7:
      return batch_st<2, 4, 2>(b, s);
    case 3:
    case 9:
      return batch_st<16, 1, 8>(b, s);
    case 10:
    case 12:
      return batch_st<16, 1, 4>(b, s);
    case 11:
      return batch_st<16, 1, 2>(b, s);
    case 13:
      return batch_st<8, 1, 8>(b, s);
  }
  return cudaErrorInvalidValue;
}

void free_batch(Batch* b) {
  if (!b) return;
  cudaFree(b->d_descs);
  cudaFree(b->d_items);
  cudaFree(b->d_counter);
  delete b;
}

}  // namespace

extern "C" {

pstm_status pstm_batch_create(pstm_batch** out, pstm_plan* const* plans, int32_t n_plans,
                              float* const* images, float* const* folds, const float* velocity,
                              int64_t v_stride_t, int64_t v_stride_c, void* stream) {
  if (!out || !plans || n_plans < 1 || !images || !velocity)
    return bfail(PSTM_EINVAL, "null argument or empty batch");
  *out = nullptr;
  if (v_stride_t < 0 || v_stride_c < 0) return bfail(PSTM_EINVAL, "negative velocity stride");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  Batch* b = new Batch();
  const Plan* p0 = reinterpret_cast<const Plan*>(plans[0]);
  for (int i = 0; i < n_plans; ++i) {
    Plan* p = reinterpret_cast<Plan*>(plans[i]);
    if (!p || !images[i]) {
      free_batch(b);
      return bfail(PSTM_EINVAL, "null plan or image in batch");
    }
    if (p->params.antialias) {
      free_batch(b);
      return bfail(PSTM_ENOTSUP, "the batched launch is built for the plain operator");
    }
    if (p->params.taper_width > 0 || p->params.ray_gradient != 0) {
      free_batch(b);
      return bfail(PSTM_ENOTSUP, "the batched launch applies no aperture taper or curved rays: "
                                 "build the class plans without taper_width or ray_gradient");
    }
    // the descriptors capture the staging buffers, so they must exist now
    const pstm_status st = ensure_trace_storage(p, s);
    if (st != PSTM_OK) {
      free_batch(b);
      return st;
    }
    if (p->n_traces > 0 && (!p->traces || !p->tile_list || !p->geo ||
                            (p->params.storage == PSTM_F16 && !p->scales))) {
      free_batch(b);
      return bfail(PSTM_EINVAL, "batched plan without device buffers");
    }
    if (p->shape.id != p0->shape.id || p->params.storage != p0->params.storage ||
        p->params.weight != p0->params.weight || p->row_stride != p0->row_stride ||
        p->grid.n_times != p0->grid.n_times || p->params.clamp != p0->params.clamp ||
        needs_lowclamp(p) != needs_lowclamp(p0) || p->row_origin != p0->row_origin) {
      free_batch(b);
      return bfail(PSTM_EINVAL, "batched plans must share kernel shape, storage, weight, clamp, "
                                "time axis, trace length and forward_only");
    }
    b->plans.push_back(p);
    b->images.push_back(images[i]);
    b->folds.push_back(folds ? folds[i] : nullptr);
  }
  b->vel = velocity;
  b->vst = v_stride_t;
  b->vsc = v_stride_c;
  b->hist16 = 1;
  for (const Plan* p : b->plans)
    if (p->longest_list >= 65536) b->hist16 = 0;
  if (!ring_shape(p0->shape.cols, p0->shape.t_window(), p0->row_stride, p0->elt_bytes,
                  &b->ring_stages, &b->ring_rows, smem_budget(p0->shape.threads()),
                  hist_entry_bytes(b->hist16 != 0))) {
    free_batch(b);
    return bfail(PSTM_EINVAL, "traces too long for the staged kernel");
  }
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
  // descriptors
  std::vector<KArgs> descs(n_plans);
  std::vector<std::pair<int64_t, int4>> items;
  for (int i = 0; i < n_plans; ++i) {
    Plan* p = b->plans[i];
    descs[i] = make_args(p, velocity, v_stride_t, v_stride_c);
    descs[i].out = b->images[i];
    descs[i].fold_out = b->folds[i];  // fold counted in the same launch (or nullptr)
    descs[i].ring_stages = b->ring_stages;
    descs[i].ring_rows = b->ring_rows;
    descs[i].hist16 = b->hist16;  // one shared-memory layout for every class
    std::vector<int64_t> off(p->n_tiles + 1);
    cudaError_t e = cudaMemcpyAsync(off.data(), p->tile_off, off.size() * sizeof(int64_t),
                                    cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      free_batch(b);
      return bfail(PSTM_ECUDA, cudaGetErrorString(e));
    }
    for (int64_t t = 0; t < p->n_tiles; ++t)
      for (int w = 0; w < p->n_windows; ++w)
        items.push_back({off[t + 1] - off[t], make_int4(i, (int)t, w, 0)});
  }
  std::stable_sort(items.begin(), items.end(),
                   [](const auto& a, const auto& c) { return a.first > c.first; });
  std::vector<int4> hitems(items.size());
  for (size_t k = 0; k < items.size(); ++k) hitems[k] = items[k].second;
  b->n_items = (int)hitems.size();
  cudaError_t e = cudaMalloc(&b->d_descs, descs.size() * sizeof(KArgs));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_items, std::max<size_t>(1, hitems.size()) * sizeof(int4));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_counter, sizeof(int));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_descs, descs.data(), descs.size() * sizeof(KArgs),
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && !hitems.empty())
    e = cudaMemcpyAsync(b->d_items, hitems.data(), hitems.size() * sizeof(int4),
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    free_batch(b);
    return bfail(e == cudaErrorMemoryAllocation ? PSTM_ENOMEM : PSTM_ECUDA, cudaGetErrorString(e));
  }
  *out = reinterpret_cast<pstm_batch*>(b);
  return PSTM_OK;
}

pstm_status pstm_batch_migrate(pstm_batch* batch, void* stream) {
  if (!batch) return bfail(PSTM_EINVAL, "null batch");
  Batch* b = reinterpret_cast<Batch*>(batch);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  for (Plan* p : b->plans)
    if (!p->traces_loaded) return bfail(PSTM_EINVAL, "a batched plan has no traces loaded");
  std::string why;
  pstm_status st = launch_velocity_check(b->plans[0], b->vel, b->vst, b->vsc, s, &why);
  if (st != PSTM_OK) return bfail(st, why);
  cudaError_t e = cudaMemsetAsync(b->d_counter, 0, sizeof(int), s);
  if (e == cudaSuccess && b->n_items > 0) e = batch_dispatch(b, s);
  if (e != cudaSuccess) return bfail(PSTM_ECUDA, std::string("batch kernel: ") + cudaGetErrorString(e));
  return PSTM_OK;
}

pstm_status pstm_batch_destroy(pstm_batch* batch) {
  free_batch(reinterpret_cast<Batch*>(batch));
  return PSTM_OK;
}

int32_t pstm_batch_size(const pstm_batch* batch) {
  return batch ? (int32_t)reinterpret_cast<const Batch*>(batch)->plans.size() : 0;
}

}  // extern "C"
